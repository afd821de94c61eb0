// Learned path guiding: network state, training on the GPU (own FP32 forward / backward kernels and
// Adam), the BF16 tensor-core inference of a batch, and the pilot records.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.hpp"
#include "guide_internal.hpp"
#include "guide_mma.cuh"

namespace skg {

namespace {

// ---------------------------------------------------------------------------------------------
// FP32 forward / backward of one sample (training and gradient checks)
// ---------------------------------------------------------------------------------------------

// raw outputs and the activations of the hidden layers
SKG_D void mlpForward(const float* P, const float* in, float* h /*4 x 64*/, float* out)
{
    const float* cur = in;
    int nin = GUIDE_IN;
    for (int l = 0; l < GUIDE_LAYERS; ++l)
    {
        const float* W = P + guideParamOffset(l);
        const float* b = W + guideDimOut(l) * nin;
        float* dst = l + 1 < GUIDE_LAYERS ? h + 64 * l : out;
        for (int o = 0; o < guideDimOut(l); ++o)
        {
            float acc = b[o];
            for (int i = 0; i < nin; ++i) acc = fmaf(W[o * nin + i], cur[i], acc);
            dst[o] = l + 1 < GUIDE_LAYERS ? fmaxf(acc, 0.f) : acc;
        }
        cur = dst;
        nin = guideDimOut(l);
    }
}

// log q(k) of the mixture and its gradient with respect to the 40 raw outputs
SKG_D float headLogDensityGrad(const float* o, const float* k, float* g)
{
    GuideMixture m;
    guideMixture(o, m);
    float l[GUIDE_LOBES], cs[GUIDE_LOBES];
    float lmax = -INFINITY;
    for (int j = 0; j < GUIDE_LOBES; ++j)
    {
        cs[j] = m.mu[j][0] * k[0] + m.mu[j][1] * k[1] + m.mu[j][2] * k[2];
        l[j] = m.logw[j] + logVmf(m.kappa[j], cs[j]);
        lmax = fmaxf(lmax, l[j]);
    }
    float s = 0.f;
    for (int j = 0; j < GUIDE_LOBES; ++j) s += expf(l[j] - lmax);
    float logq = lmax + logf(s);
    for (int j = 0; j < GUIDE_LOBES; ++j)
    {
        float r = expf(l[j] - logq);   // responsibility
        float w = expf(m.logw[j]);     // mixture weight
        g[5 * j] = r - w;
        // direction: mu = a / |a|, d log f / d a = kappa (k - (mu.k) mu) / |a|
        float a0 = o[5 * j + 1], a1 = o[5 * j + 2], a2 = o[5 * j + 3];
        float n = sqrtf(a0 * a0 + a1 * a1 + a2 * a2);
        if (n > 1e-12f)
        {
            float c = r * m.kappa[j] / n;
            g[5 * j + 1] = c * (k[0] - cs[j] * m.mu[j][0]);
            g[5 * j + 2] = c * (k[1] - cs[j] * m.mu[j][1]);
            g[5 * j + 3] = c * (k[2] - cs[j] * m.mu[j][2]);
        }
        else
        {
            g[5 * j + 1] = g[5 * j + 2] = g[5 * j + 3] = 0.f;
        }
        // concentration: kappa = softplus(s) + kmin, clamped at kmax
        float kap = m.kappa[j];
        float e = expf(-2.f * kap);
        float dlogf = 1.f / kap - 2.f * e / (1.f - e) + (cs[j] - 1.f);
        float sraw = o[5 * j + 4];
        float dk = (softplusf(sraw) + GUIDE_KAPPA_MIN < GUIDE_KAPPA_MAX) ? 1.f / (1.f + expf(-sraw)) : 0.f;
        g[5 * j + 4] = r * dlogf * dk;
    }
    return logq;
}

// Per-sample pass of a batch: forward, loss -w log q, and the back-propagated deltas. Writes, per
// sample b, the inputs (8), hidden activations (4 x 64) and the deltas of every layer's
// pre-activation (4 x 64 hidden, 40 output) to the scratch rows used by the weight-gradient kernel.
struct BatchScratch
{
    float* in;     // B x 8
    float* h;      // B x 256
    float* delta;  // B x 296 (hidden 4 x 64, then 40)
    float* loss;   // 1 (accumulated)
};

constexpr int DELTA_W = 4 * 64 + GUIDE_OUT;

SKG_D void samplePass(const float* P, const float* in, const float* k, float w, const BatchScratch& s, int b,
                      float& lossOut)
{
    float h[4 * 64], out[GUIDE_OUT], g[GUIDE_OUT];
    mlpForward(P, in, h, out);
    float logq = headLogDensityGrad(out, k, g);
    lossOut = -w * logq;
    float* d = s.delta + static_cast<size_t>(b) * DELTA_W;
    // loss = -w log q: delta of the outputs
    float dout[GUIDE_OUT];
    for (int o = 0; o < GUIDE_OUT; ++o)
    {
        dout[o] = -w * g[o];
        d[256 + o] = dout[o];
    }
    // back through the hidden layers: delta_l = (W_{l+1}^T delta_{l+1}) * relu'(h_l)
    float nextDelta[64];
    const float* dn = dout;
    int nOut = GUIDE_OUT;
    for (int l = GUIDE_LAYERS - 2; l >= 0; --l)
    {
        const float* W = P + guideParamOffset(l + 1);  // (nOut x 64)
        float cur[64];
        for (int i = 0; i < 64; ++i)
        {
            float acc = 0.f;
            for (int o = 0; o < nOut; ++o) acc = fmaf(W[o * 64 + i], dn[o], acc);
            cur[i] = h[64 * l + i] > 0.f ? acc : 0.f;
        }
        for (int i = 0; i < 64; ++i)
        {
            nextDelta[i] = cur[i];
            d[64 * l + i] = cur[i];
        }
        dn = nextDelta;
        nOut = 64;
    }
    float* hs = s.h + static_cast<size_t>(b) * 256;
    for (int i = 0; i < 256; ++i) hs[i] = h[i];
    float* is = s.in + static_cast<size_t>(b) * GUIDE_IN;
    for (int i = 0; i < GUIDE_IN; ++i) is[i] = in[i];
}

// explicit samples (gradient checks)
__global__ void passExplicitKernel(const float* P, int n, const float* in, const float* k, const float* w,
                                   BatchScratch s)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    float l;
    samplePass(P, in + static_cast<size_t>(b) * GUIDE_IN, k + 3 * static_cast<size_t>(b), w[b], s, b, l);
    atomicAdd(s.loss, l);
}

// position bin of a record (inputs 0..2 are the position scaled to [-1, 1])
SKG_D int positionBin(const GuideRecord& q, int nb)
{
    int idx = 0;
    for (int a = 0; a < 3; ++a)
    {
        int i = static_cast<int>((q.f[a] + 1.f) * 0.5f * static_cast<float>(nb));
        idx = idx * nb + min(nb - 1, max(0, i));
    }
    return idx;
}

// per position bin: sum of I (binSum) and number of records (binCount)
__global__ void binRecordsKernel(const GuideRecord* rec, unsigned long long n, int nb, float* binSum, unsigned* binCount)
{
    unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    int b = positionBin(rec[i], nb);
    atomicAdd(binSum + b, rec[i].I);
    atomicAdd(binCount + b, 1u);
}

__global__ void binMeanKernel(int nbins, const float* binSum, const unsigned* binCount, float* binMean)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbins) binMean[b] = binCount[b] ? binSum[b] / static_cast<float>(binCount[b]) : 0.f;
}

// a random batch of pilot records, weight I / (mean I * B), or I / (mean I of the bin * B)
__global__ void passRecordsKernel(const float* P, const GuideRecord* rec, unsigned long long nrec, int B, float invMeanI,
                                  int nb, const float* binMean, unsigned long long seed, unsigned step, BatchScratch s)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    U4 r = philox4x32_10(U4{step, static_cast<uint32_t>(b), 0x6d6c70u, 0u}, static_cast<uint32_t>(seed),
                         static_cast<uint32_t>(seed >> 32));
    unsigned long long j = ((static_cast<unsigned long long>(r.x) << 32) | r.y) % nrec;
    const GuideRecord& q = rec[j];
    float w = q.I * invMeanI;
    if (nb > 0)
    {
        float m = binMean[positionBin(q, nb)];
        w = m > 0.f ? q.I / m : 0.f;
    }
    float l;
    samplePass(P, q.f, q.k, w / static_cast<float>(B), s, b, l);
    atomicAdd(s.loss, l);
}

// gradient of one parameter: sum over the batch of delta[b][o] * input[b][i] (or delta for a bias)
__global__ void weightGradKernel(int B, BatchScratch s, float* grad)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= GUIDE_NPARAMS) return;
    int l = 0;
    while (l + 1 < GUIDE_LAYERS && p >= guideParamOffset(l + 1)) ++l;
    int local = p - guideParamOffset(l);
    int nin = guideDimIn(l), nout = guideDimOut(l);
    int dcol = l + 1 < GUIDE_LAYERS ? 64 * l : 256;
    float acc = 0.f;
    if (local < nout * nin)
    {
        int o = local / nin, i = local % nin;
        for (int b = 0; b < B; ++b)
        {
            float x = l == 0 ? s.in[static_cast<size_t>(b) * GUIDE_IN + i] : s.h[static_cast<size_t>(b) * 256 + 64 * (l - 1) + i];
            acc = fmaf(s.delta[static_cast<size_t>(b) * DELTA_W + dcol + o], x, acc);
        }
    }
    else
    {
        int o = local - nout * nin;
        for (int b = 0; b < B; ++b) acc += s.delta[static_cast<size_t>(b) * DELTA_W + dcol + o];
    }
    grad[p] = acc;
}

__global__ void adamKernel(float* P, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                           float c1, float c2, float clip)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= GUIDE_NPARAMS) return;
    float gp = fminf(clip, fmaxf(-clip, g[p]));
    if (!isfinite(gp)) gp = 0.f;
    float mp = b1 * m[p] + (1.f - b1) * gp;
    float vp = b2 * v[p] + (1.f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    P[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

// tensor-core forward pass of n explicit samples (tests): 128 samples per CTA
__global__ void __launch_bounds__(GM_TILE) inferKernel(const unsigned char* blob, int n, const float* in, float* out,
                                                       int* err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    GuideTile t;
    guideTileBegin(t, smem, blob);
    for (int tile = blockIdx.x; tile * GM_TILE < n; tile += gridDim.x)
    {
        int i = tile * GM_TILE + threadIdx.x;
        float f[GUIDE_IN], o[GUIDE_OUT];
        for (int k = 0; k < GUIDE_IN; ++k) f[k] = i < n ? in[static_cast<size_t>(i) * GUIDE_IN + k] : 0.f;
        if (!guideTileForward(t, f, o))
        {
            if (threadIdx.x == 0) atomicOr(err, 1);
            break;  // uniform across the CTA
        }
        if (i < n)
            for (int k = 0; k < GUIDE_OUT; ++k) out[static_cast<size_t>(i) * GUIDE_OUT + k] = o[k];
    }
    guideTileEnd(t);
}

// FP32 (CUDA-core) forward pass of n explicit samples (reference for the tensor-core pass)
__global__ void inferFp32Kernel(const float* P, int n, const float* in, float* out)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    float h[256];
    mlpForward(P, in + static_cast<size_t>(b) * GUIDE_IN, h, out + static_cast<size_t>(b) * GUIDE_OUT);
}

// sum of the records' downstream luminosities (set at the end of each recorded history)
__global__ void sumRecordsKernel(const GuideRecord* rec, unsigned long long n, double* sumI)
{
    unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x;
    double v = i < n ? static_cast<double>(rec[i].I) : 0.;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(sumI, v);
}

template<typename T>
cudaError_t allocN(T** p, size_t n)
{
    return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T));
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// state
// ---------------------------------------------------------------------------------------------
GuideState::~GuideState()
{
    void* ps[] = {params, blob, adamM, adamV, grad, records, recCount, scratchIn, scratchH, scratchDelta, lossAcc,
                  importance, errFlag, binMean};
    for (void* p : ps)
        if (p) cudaFree(p);
}

cudaError_t guideEnsure(skgpu_ctx* ctx)
{
    if (ctx->guide) return cudaSuccess;
    GuideState* g = new GuideState();
    cudaError_t e = allocN(&g->params, GUIDE_NPARAMS);
    if (e == cudaSuccess) e = allocN(&g->blob, GM_BLOB_BYTES);
    if (e == cudaSuccess) e = allocN(&g->adamM, GUIDE_NPARAMS);
    if (e == cudaSuccess) e = allocN(&g->adamV, GUIDE_NPARAMS);
    if (e == cudaSuccess) e = allocN(&g->grad, GUIDE_NPARAMS);
    if (e == cudaSuccess) e = allocN(&g->recCount, 1);
    if (e == cudaSuccess) e = allocN(&g->lossAcc, 1);
    if (e == cudaSuccess) e = allocN(&g->errFlag, 1);
    if (e == cudaSuccess) e = cudaMemset(g->recCount, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(g->errFlag, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(inferKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GM_SMEM_BYTES);
    if (e != cudaSuccess)
    {
        delete g;
        return e;
    }
    ctx->guide = g;
    return cudaSuccess;
}

void guideDestroy(skgpu_ctx* ctx)
{
    delete ctx->guide;
    ctx->guide = nullptr;
}

cudaError_t guideSetParams(skgpu_ctx* ctx, const float* host)
{
    GuideState* g = ctx->guide;
    cudaError_t e = cudaMemcpy(g->params, host, GUIDE_NPARAMS * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    e = cudaMemset(g->adamM, 0, GUIDE_NPARAMS * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(g->adamV, 0, GUIDE_NPARAMS * sizeof(float));
    g->adamStep = 0;
    g->hasParams = true;
    return e == cudaSuccess ? guideRepack(ctx) : e;
}

cudaError_t guideGetParams(skgpu_ctx* ctx, float* host)
{
    return cudaMemcpy(host, ctx->guide->params, GUIDE_NPARAMS * sizeof(float), cudaMemcpyDeviceToHost);
}

// BF16 blob of the inference kernel from the FP32 master parameters
cudaError_t guideRepack(skgpu_ctx* ctx)
{
    GuideState* g = ctx->guide;
    std::vector<float> p(GUIDE_NPARAMS);
    cudaError_t e = cudaMemcpy(p.data(), g->params, p.size() * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    std::vector<unsigned char> blob(GM_BLOB_BYTES);
    guidePackBlob(p.data(), blob.data());
    return cudaMemcpy(g->blob, blob.data(), blob.size(), cudaMemcpyHostToDevice);
}

static cudaError_t ensureScratch(GuideState* g, int B)
{
    if (g->scratchRows >= B) return cudaSuccess;
    cudaFree(g->scratchIn);
    cudaFree(g->scratchH);
    cudaFree(g->scratchDelta);
    g->scratchIn = g->scratchH = g->scratchDelta = nullptr;
    g->scratchRows = 0;
    cudaError_t e = allocN(&g->scratchIn, static_cast<size_t>(B) * GUIDE_IN);
    if (e == cudaSuccess) e = allocN(&g->scratchH, static_cast<size_t>(B) * 256);
    if (e == cudaSuccess) e = allocN(&g->scratchDelta, static_cast<size_t>(B) * DELTA_W);
    if (e == cudaSuccess) g->scratchRows = B;
    return e;
}

cudaError_t guideLossGrad(skgpu_ctx* ctx, int n, const float* in, const float* k, const float* w, float* loss,
                          float* grad)
{
    GuideState* g = ctx->guide;
    cudaError_t e = ensureScratch(g, n);
    if (e != cudaSuccess) return e;
    float *dIn = nullptr, *dK = nullptr, *dW = nullptr;
    e = allocN(&dIn, static_cast<size_t>(n) * GUIDE_IN);
    if (e == cudaSuccess) e = allocN(&dK, 3 * static_cast<size_t>(n));
    if (e == cudaSuccess) e = allocN(&dW, n);
    if (e == cudaSuccess) e = cudaMemcpy(dIn, in, static_cast<size_t>(n) * GUIDE_IN * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dK, k, 3 * static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dW, w, static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(g->lossAcc, 0, sizeof(float));
    BatchScratch s{g->scratchIn, g->scratchH, g->scratchDelta, g->lossAcc};
    if (e == cudaSuccess)
    {
        passExplicitKernel<<<(n + 127) / 128, 128>>>(g->params, n, dIn, dK, dW, s);
        weightGradKernel<<<(GUIDE_NPARAMS + 255) / 256, 256>>>(n, s, g->grad);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(loss, g->lossAcc, sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(grad, g->grad, GUIDE_NPARAMS * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dIn);
    cudaFree(dK);
    cudaFree(dW);
    return e;
}

cudaError_t guideInfer(skgpu_ctx* ctx, int n, const float* in, float* out, int tensorCores, int* deviceErr)
{
    GuideState* g = ctx->guide;
    float *dIn = nullptr, *dOut = nullptr;
    cudaError_t e = allocN(&dIn, static_cast<size_t>(n) * GUIDE_IN);
    if (e == cudaSuccess) e = allocN(&dOut, static_cast<size_t>(n) * GUIDE_OUT);
    if (e == cudaSuccess) e = cudaMemcpy(dIn, in, static_cast<size_t>(n) * GUIDE_IN * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(g->errFlag, 0, sizeof(int));
    if (e == cudaSuccess)
    {
        if (tensorCores)
        {
            int tiles = (n + GM_TILE - 1) / GM_TILE;
            int grid = std::max(1, std::min(tiles, 4 * ctx->numSMs));
            inferKernel<<<grid, GM_TILE, GM_SMEM_BYTES>>>(g->blob, n, dIn, dOut, g->errFlag);
        }
        else
        {
            inferFp32Kernel<<<(n + 127) / 128, 128>>>(g->params, n, dIn, dOut);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(out, dOut, static_cast<size_t>(n) * GUIDE_OUT * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(deviceErr, g->errFlag, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dIn);
    cudaFree(dOut);
    return e;
}

cudaError_t guideEnsureRecords(skgpu_ctx* ctx, unsigned long long capacity)
{
    GuideState* g = ctx->guide;
    if (g->recCapacity != capacity)
    {
        cudaFree(g->records);
        g->records = nullptr;
        g->recCapacity = 0;
        cudaError_t e = allocN(&g->records, capacity);
        if (e != cudaSuccess) return e;
        g->recCapacity = capacity;
    }
    return cudaMemset(g->recCount, 0, sizeof(unsigned long long));
}

cudaError_t guideRecordCount(skgpu_ctx* ctx, unsigned long long* n)
{
    cudaError_t e = cudaMemcpy(n, ctx->guide->recCount, sizeof *n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) *n = std::min(*n, ctx->guide->recCapacity);
    return e;
}

cudaError_t guideFetchRecords(skgpu_ctx* ctx, unsigned long long n, float* out /* n x 13: f[8], k[3], I, L */)
{
    std::vector<GuideRecord> r(n);
    cudaError_t e = cudaMemcpy(r.data(), ctx->guide->records, n * sizeof(GuideRecord), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    for (unsigned long long i = 0; i < n; ++i)
    {
        float* o = out + 13 * i;
        for (int k = 0; k < GUIDE_IN; ++k) o[k] = r[i].f[k];
        for (int k = 0; k < 3; ++k) o[8 + k] = r[i].k[k];
        o[11] = r[i].I;
        o[12] = r[i].L;
    }
    return cudaSuccess;
}

cudaError_t guideTrain(skgpu_ctx* ctx, int steps, int batch, float lr, unsigned long long seed, float* lossOut)
{
    GuideState* g = ctx->guide;
    unsigned long long nrec = 0;
    cudaError_t e = guideRecordCount(ctx, &nrec);
    if (e != cudaSuccess) return e;
    if (nrec == 0) return cudaErrorInvalidValue;
    e = ensureScratch(g, batch);
    if (e != cudaSuccess) return e;
    // mean downstream luminosity of the records (weights are I / mean I)
    double* dSum = nullptr;
    e = allocN(&dSum, 1);
    if (e == cudaSuccess) e = cudaMemset(dSum, 0, sizeof(double));
    if (e == cudaSuccess)
    {
        sumRecordsKernel<<<static_cast<unsigned>((nrec + 255) / 256), 256>>>(g->records, nrec, dSum);
        e = cudaGetLastError();
    }
    double sumI = 0.;
    if (e == cudaSuccess) e = cudaMemcpy(&sumI, dSum, sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dSum);
    if (e != cudaSuccess) return e;
    if (!(sumI > 0.)) return cudaErrorInvalidValue;  // the pilot detected nothing downstream
    float invMeanI = static_cast<float>(static_cast<double>(nrec) / sumI);
    int nb = g->positionBins;
    if (nb > 0)
    {
        int nbins = nb * nb * nb;
        float* binSum = nullptr;
        unsigned* binCount = nullptr;
        cudaFree(g->binMean);
        g->binMean = nullptr;
        e = allocN(&g->binMean, nbins);
        if (e == cudaSuccess) e = allocN(&binSum, nbins);
        if (e == cudaSuccess) e = allocN(&binCount, nbins);
        if (e == cudaSuccess) e = cudaMemset(binSum, 0, nbins * sizeof(float));
        if (e == cudaSuccess) e = cudaMemset(binCount, 0, nbins * sizeof(unsigned));
        if (e == cudaSuccess)
        {
            binRecordsKernel<<<static_cast<unsigned>((nrec + 255) / 256), 256>>>(g->records, nrec, nb, binSum, binCount);
            binMeanKernel<<<(nbins + 255) / 256, 256>>>(nbins, binSum, binCount, g->binMean);
            e = cudaGetLastError();
        }
        cudaFree(binSum);
        cudaFree(binCount);
        if (e != cudaSuccess) return e;
    }
    BatchScratch s{g->scratchIn, g->scratchH, g->scratchDelta, g->lossAcc};
    const float b1 = 0.9f, b2 = 0.999f;
    float lastLoss = 0.f;
    for (int it = 0; it < steps && e == cudaSuccess; ++it)
    {
        e = cudaMemset(g->lossAcc, 0, sizeof(float));
        passRecordsKernel<<<(batch + 127) / 128, 128>>>(g->params, g->records, nrec, batch, invMeanI, nb, g->binMean,
                                                        seed, static_cast<unsigned>(g->adamStep), s);
        weightGradKernel<<<(GUIDE_NPARAMS + 255) / 256, 256>>>(batch, s, g->grad);
        g->adamStep++;
        float c1 = 1.f - std::pow(b1, static_cast<float>(g->adamStep));
        float c2 = 1.f - std::pow(b2, static_cast<float>(g->adamStep));
        adamKernel<<<(GUIDE_NPARAMS + 255) / 256, 256>>>(g->params, g->grad, g->adamM, g->adamV, lr, b1, b2, 1e-8f, c1,
                                                         c2, 10.f);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess && (it + 1 == steps)) e = cudaMemcpy(&lastLoss, g->lossAcc, sizeof(float), cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess) e = guideRepack(ctx);
    if (lossOut) *lossOut = lastLoss;
    return e;
}

}  // namespace skg

// BF16 tensor-core forward pass of the guiding MLP on sm_100a: tcgen05.mma with both operands in
// shared memory and the FP32 accumulator in tensor memory, 128 samples (M = 128) per tile.
//
// Shared-memory operands use the K-major layout without swizzle: 8 x 16-byte core matrices, an
// element (r, k) of an R x K bf16 matrix at byte ((r/8) * SBO + (k/8) * LBO + (r%8) * 16 + (k%8) * 2)
// with LBO = 128 and SBO = K/8 * 128. One MMA consumes K = 16 (two core-matrix columns); the
// descriptor of step s starts 256 * s bytes into the matrix.
//
// Per tile: every thread writes its sample's row of the layer input, one thread issues the K/16
// MMAs of the layer and commits them to an mbarrier, and after the barrier every warp reads its 32
// accumulator rows from tensor memory (tcgen05.ld 32x32b), adds the bias, applies ReLU and writes
// the bf16 row back as the next layer's input. All waits are bounded: a wait that gives up makes
// the forward pass return false in every thread of the CTA.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

#include "guide.cuh"

namespace skg {

constexpr int GM_TILE = 128;       // samples per tile (MMA M)
constexpr int GM_K0 = 16;          // padded input width
constexpr int GM_N_OUT = 48;       // padded output width (multiple of 16)
constexpr int GM_TMEM_COLS = 64;   // accumulator columns (power of two >= 32)
// packed parameter blob: bf16 weight matrices (core-matrix layout), then FP32 biases
SKG_HD constexpr int gmWOff(int l) { return l == 0 ? 0 : 2048 + (l - 1) * 8192; }
constexpr int GM_B_OFF = 2048 + 3 * 8192 + GM_N_OUT * 64 * 2;   // 32768
constexpr int GM_B_FLOATS = 4 * 64 + GM_N_OUT;                   // 304
constexpr int GM_BLOB_BYTES = GM_B_OFF + GM_B_FLOATS * 4;        // 33984
constexpr int GM_X_BYTES = GM_TILE * 64 * 2;                     // 16384
// dynamic shared memory of a tile kernel: blob, activations, mbarrier + tensor-memory address
constexpr int GM_SMEM_BYTES = GM_BLOB_BYTES + GM_X_BYTES + 64;
SKG_HD constexpr int gmLayerK(int l) { return l == 0 ? GM_K0 : 64; }
SKG_HD constexpr int gmLayerN(int l) { return l == GUIDE_LAYERS - 1 ? GM_N_OUT : 64; }

// byte offset of element (r, k) in a K-major core-matrix layout of width K
SKG_HD constexpr int gmOffset(int r, int k, int K) { return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2; }

// ---------------------------------------------------------------------------------------------
// PTX wrappers (sm_100a)
// ---------------------------------------------------------------------------------------------
SKG_D uint32_t smemAddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

SKG_D uint64_t gmSmemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16)
           | (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major, M x N
SKG_HD constexpr uint32_t gmInstrDesc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

SKG_D void gmFenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
SKG_D void gmFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
SKG_D void gmFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

SKG_D void gmMma(uint32_t tmemD, uint64_t descA, uint64_t descB, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n"
        :
        : "r"(tmemD), "l"(descA), "l"(descB), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

SKG_D void gmCommit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

SKG_D void gmMbarInit(uint32_t mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// waits for the completion of the given phase; false when the bounded wait gave up
SKG_D bool gmMbarWait(uint32_t mbar, uint32_t phase)
{
    for (int it = 0; it < (1 << 24); ++it)
    {
        uint32_t ok;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

SKG_D void gmTmemAlloc(uint32_t slotAddr, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slotAddr), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

SKG_D void gmTmemFree(uint32_t taddr, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's row
SKG_D void gmLoad16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------------------------
// tile state and forward pass
// ---------------------------------------------------------------------------------------------
struct GuideTile
{
    unsigned char* blob;  // packed parameters in shared memory
    unsigned char* x;     // layer input, 128 rows, K-major core-matrix layout
    uint32_t mbar;        // shared address of the mbarrier
    uint32_t taddr;       // tensor-memory accumulator (64 columns)
    uint32_t phase;
};

// Sets up a 128-thread CTA: copies the packed parameters into shared memory, allocates the
// accumulator columns and initialises the mbarrier. Every thread of the CTA must call it.
SKG_D void guideTileBegin(GuideTile& t, unsigned char* smem, const unsigned char* blobGlobal)
{
    t.blob = smem;
    t.x = smem + GM_BLOB_BYTES;
    uint32_t* misc = reinterpret_cast<uint32_t*>(smem + GM_BLOB_BYTES + GM_X_BYTES);  // [0..1] mbarrier, [2] tmem
    const uint4* src = reinterpret_cast<const uint4*>(blobGlobal);
    uint4* dst = reinterpret_cast<uint4*>(smem);
    for (int i = threadIdx.x; i < GM_BLOB_BYTES / 16; i += blockDim.x) dst[i] = src[i];
    t.mbar = smemAddr(misc);
    if (threadIdx.x == 0)
    {
        gmMbarInit(t.mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 32) gmTmemAlloc(smemAddr(misc + 2), GM_TMEM_COLS);
    gmFenceBefore();
    __syncthreads();
    gmFenceAfter();
    t.taddr = misc[2];
    t.phase = 0;
}

SKG_D void guideTileEnd(GuideTile& t)
{
    gmFenceBefore();
    __syncthreads();
    if (threadIdx.x < 32) gmTmemFree(t.taddr, GM_TMEM_COLS);
}

// Forward pass of the 128 samples of a tile; thread i owns row i: in[8] are its inputs (ignored
// rows may hold anything finite), out[40] receives its raw outputs. Returns false, in every thread
// of the CTA alike, when a wait gave up (the tile's outputs are then undefined).
SKG_D bool guideTileForward(GuideTile& t, const float* in, float* out)
{
    const int row = threadIdx.x;
    const int warp = threadIdx.x >> 5;
    // layer input 0: the 8 inputs padded with zeros to K = 16
#pragma unroll
    for (int k = 0; k < GM_K0; ++k)
        *reinterpret_cast<__nv_bfloat16*>(t.x + gmOffset(row, k, GM_K0)) = __float2bfloat16_rn(k < GUIDE_IN ? in[k] : 0.f);
    const float* bias = reinterpret_cast<const float*>(t.blob + GM_B_OFF);
    for (int l = 0; l < GUIDE_LAYERS; ++l)
    {
        const int K = gmLayerK(l), N = gmLayerN(l);
        gmFenceProxyAsync();  // the generic-proxy writes of the layer input, before the MMA reads them
        gmFenceBefore();
        __syncthreads();
        if (threadIdx.x == 0)
        {
            gmFenceAfter();
            uint32_t idesc = gmInstrDesc(GM_TILE, N);
            uint32_t xa = smemAddr(t.x), wb = smemAddr(t.blob + gmWOff(l));
            for (int s = 0; s < K / 16; ++s)
            {
                uint64_t da = gmSmemDesc(xa + 256 * s, 128, K * 16);
                uint64_t db = gmSmemDesc(wb + 256 * s, 128, K * 16);
                gmMma(t.taddr, da, db, idesc, s > 0 ? 1u : 0u);
            }
            gmCommit(t.mbar);
        }
        bool ok = gmMbarWait(t.mbar, t.phase);
        if (__syncthreads_or(!ok))
        {
            // give the MMAs in flight one more bounded wait before the caller releases the tensor memory
            if (!ok) gmMbarWait(t.mbar, t.phase);
            __syncthreads();
            return false;
        }
        t.phase ^= 1u;
        gmFenceAfter();
        // this warp's 32 accumulator rows: lanes 32 * warp ... 32 * warp + 31
        uint32_t rowAddr = t.taddr + (static_cast<uint32_t>(32 * warp) << 16);
        const float* b = bias + 64 * l;
        if (l + 1 < GUIDE_LAYERS)
        {
            for (int c0 = 0; c0 < N; c0 += 16)
            {
                float v[16];
                gmLoad16(rowAddr + c0, v);
#pragma unroll
                for (int i = 0; i < 16; ++i)
                {
                    float h = fmaxf(v[i] + b[c0 + i], 0.f);
                    *reinterpret_cast<__nv_bfloat16*>(t.x + gmOffset(row, c0 + i, 64)) = __float2bfloat16_rn(h);
                }
            }
        }
        else
        {
            for (int c0 = 0; c0 < N; c0 += 16)
            {
                float v[16];
                gmLoad16(rowAddr + c0, v);
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (c0 + i < GUIDE_OUT) out[c0 + i] = v[i] + b[c0 + i];
            }
        }
    }
    // the accumulator is rewritten by the next tile's first MMA: every read must be complete
    gmFenceBefore();
    __syncthreads();
    return true;
}

// ---------------------------------------------------------------------------------------------
// host-side packing of the FP32 master parameters into the blob
// ---------------------------------------------------------------------------------------------
inline uint16_t gmBf16Bits(float f)
{
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return static_cast<uint16_t>(u >> 16);  // inf / nan
    u += 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even
    return static_cast<uint16_t>(u >> 16);
}

inline void guidePackBlob(const float* params, unsigned char* blob)
{
    for (int i = 0; i < GM_BLOB_BYTES; ++i) blob[i] = 0;
    float* bias = reinterpret_cast<float*>(blob + GM_B_OFF);
    for (int l = 0; l < GUIDE_LAYERS; ++l)
    {
        const float* W = params + guideParamOffset(l);
        const float* b = W + guideDimOut(l) * guideDimIn(l);
        int K = gmLayerK(l);
        for (int n = 0; n < guideDimOut(l); ++n)
        {
            for (int k = 0; k < guideDimIn(l); ++k)
            {
                uint16_t v = gmBf16Bits(W[n * guideDimIn(l) + k]);
                __builtin_memcpy(blob + gmWOff(l) + gmOffset(n, k, K), &v, 2);
            }
            bias[64 * l + n] = b[n];
        }
    }
}

}  // namespace skg

// The C ABI of include/skgpu.h: context, uploads into HBM, the life-cycle launch, tallies.
//
// Host data layouts follow what SKIRT's objects already hold (border arrays, CSR neighbour lists,
// MediumState densities, DustMix tables), so the SKIRT-side bridge only copies flat arrays. The
// library builds two search structures of its own at upload time: a uniform site grid for the
// Voronoi nearest-site search and a uniform grid of tetrahedron bounding boxes for the tetra
// cell search.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <type_traits>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>

#include "../../include/skgpu.h"
#include "internal.hpp"
#include "ctx.hpp"
#include "guide_internal.hpp"

using namespace skg;

namespace {

struct DevArray
{
    void* ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace


namespace {

int fail(skgpu_ctx* c, int code, const std::string& msg)
{
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                   \
    do                                                                                             \
    {                                                                                              \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(ctx, SKGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void freeBufs(std::vector<void*>& v)
{
    for (void* p : v) cudaFree(p);
    v.clear();
}

template<typename T>
cudaError_t devAlloc(T** p, size_t n)
{
    *p = nullptr;
    if (n == 0) n = 1;
    return cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
}

template<typename T>
cudaError_t devUpload(T** p, const T* host, size_t n)
{
    cudaError_t e = devAlloc(p, n);
    if (e != cudaSuccess) return e;
    if (n && host) e = cudaMemcpy(*p, host, n * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

template<typename T>
void devFree(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

// warp aggregation of the radiation-field atomics (off unless SKGPU_RF_WARP_AGG=1; a switch for
// comparing the two forms)
int rfWarpAggregation()
{
    static const int on = [] {
        const char* v = std::getenv("SKGPU_RF_WARP_AGG");
        return v && v[0] == '1' ? 1 : 0;
    }();
    return on;
}

void freeGrid(skgpu_ctx* ctx)
{
    for (void* p : ctx->gridBufs) cudaFree(p);
    ctx->gridBufs.clear();
    ctx->g = GridDev{};
    ctx->hasGrid = false;
}

template<typename T>
int gridUpload(skgpu_ctx* ctx, const T** dst, const T* host, size_t n)
{
    T* d = nullptr;
    CK(devUpload(&d, host, n));
    ctx->gridBufs.push_back(d);
    *dst = d;
    return SKGPU_OK;
}

void freeInstruments(skgpu_ctx* ctx)
{
    for (void* p : ctx->instrBufs) cudaFree(p);
    for (void* p : ctx->instrAux) cudaFree(p);
    ctx->instrAux.clear();
    ctx->instrBufs.clear();
    ctx->instrBufLens.clear();
    ctx->instrHost.clear();
    devFree(ctx->instr);
    devFree(ctx->wlgB);
    devFree(ctx->wlgEll);
}

bool finiteAll(const double* v, size_t n)
{
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

// copies the number densities into the FP32 leaf records of an octree grid (4 float4 per leaf)
__global__ void fillLeafDensityKernel(int4* rec, const double* dens, int n)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) rec[4 * static_cast<size_t>(c)].w = __float_as_int(static_cast<float>(dens[c]));
}

int syncLeafDensity(skgpu_ctx* ctx)
{
    if (!ctx->hasGrid || ctx->g.kind != SKGPU_GRID_OCTREE || !ctx->g.tRec || !ctx->dens) return SKGPU_OK;
    if (ctx->numCells != ctx->g.numCells) return SKGPU_OK;  // checked again at run time
    int n = ctx->numCells;
    fillLeafDensityKernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(const_cast<int4*>(ctx->g.tRec), ctx->dens, n);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return SKGPU_OK;
}

// histories in flight at most; a larger range streams through the pool
constexpr uint64_t POOL_DEFAULT = 1u << 22;  // packet slots in flight unless a launch shape sets them
constexpr uint64_t POOL_MAX = 1u << 22;
// wavefront passes per run at most (each history needs about two passes per scattering event)
constexpr long long MAX_PASSES = 2LL * MAX_SCATT_EVENTS + 64;

template<typename T>
int secAlloc(skgpu_ctx* ctx, std::vector<void*>& bufs, T** p, size_t n)
{
    CK(devAlloc(p, n));
    bufs.push_back(*p);
    return SKGPU_OK;
}

template<typename T>
int secUpload(skgpu_ctx* ctx, std::vector<void*>& bufs, const T** p, const T* host, size_t n)
{
    T* d = nullptr;
    CK(devUpload(&d, host, n));
    bufs.push_back(d);
    *p = d;
    return SKGPU_OK;
}

void freeWave(skgpu_ctx* ctx)
{
    ctx->graphCache.reset();  // its kernel nodes point into the buffers freed here
    for (void* p : ctx->waveBufs) cudaFree(p);
    ctx->waveBufs.clear();
    ctx->wave = Wave{};
    ctx->waveP = ctx->waveGroups = ctx->waveStats = 0;
}

template<typename T>
int waveAlloc(skgpu_ctx* ctx, T** p, size_t n)
{
    CK(devAlloc(p, n));
    ctx->waveBufs.push_back(*p);
    return SKGPU_OK;
}

// packet pool of P slots (128-byte records), task buffers (peel: P per observer group; propagation: P per
// kind), two parities each, and the control block
int ensureWaveBuffers(skgpu_ctx* ctx, int P, int groups, int stats)
{
    if (ctx->waveP >= P && ctx->waveGroups >= groups && ctx->waveStats >= stats) return SKGPU_OK;
    P = std::max(P, ctx->waveP);
    groups = std::max(groups, ctx->waveGroups);
    stats = std::max(stats, ctx->waveStats);
    freeWave(ctx);
    Wave& w = ctx->wave;
    PacketPool& k = w.pk;
    int rc = 0;
    if ((rc = waveAlloc(ctx, &k.rec, P))) return rc;
    if ((rc = waveAlloc(ctx, &k.nstat, P))) return rc;
    if ((rc = waveAlloc(ctx, &k.freeSlots, P))) return rc;
    size_t ns = stats ? static_cast<size_t>(P) * STATS_CAP : 1;
    if ((rc = waveAlloc(ctx, &k.skey, ns))) return rc;
    if ((rc = waveAlloc(ctx, &k.sw, ns))) return rc;
    // spill log of the per-history statistics: histories with more than STATS_CAP distinct keys
    k.spillCap = stats ? std::max<size_t>(size_t(1) << 20, 2 * static_cast<size_t>(P)) : 1;
    if ((rc = waveAlloc(ctx, &k.spill, k.spillCap))) return rc;
    if ((rc = waveAlloc(ctx, &k.gD, P))) return rc;
    if ((rc = waveAlloc(ctx, &k.gLast, P))) return rc;
    if ((rc = waveAlloc(ctx, &k.gPend, P))) return rc;
    if ((rc = waveAlloc(ctx, &k.gRatio, P))) return rc;
    for (int b = 0; b < 2; ++b)
        for (int kind = 0; kind < NUM_KINDS; ++kind)
        {
            TaskBuf& t = w.q[b][kind];
            size_t cap = kind == K_PEEL ? static_cast<size_t>(P) * groups : static_cast<size_t>(P);
            if ((rc = waveAlloc(ctx, &t.slot, cap))) return rc;
            if (kind == K_GUIDE) continue;  // the guided-scattering queue holds packet slots only
            if ((rc = waveAlloc(ctx, &t.par, cap))) return rc;
            if (kind == K_PEEL)
            {
                if ((rc = waveAlloc(ctx, &t.info, cap))) return rc;
                if ((rc = waveAlloc(ctx, &t.x, cap))) return rc;
                if ((rc = waveAlloc(ctx, &t.y, cap))) return rc;
                if ((rc = waveAlloc(ctx, &t.z, cap))) return rc;
            }
            if (kind == K_PEEL || kind == K_PROP1)
            {
                if ((rc = waveAlloc(ctx, &t.tau, cap))) return rc;
            }
            else
            {
                if ((rc = waveAlloc(ctx, &t.m, cap))) return rc;
                if ((rc = waveAlloc(ctx, &t.s, cap))) return rc;
                if ((rc = waveAlloc(ctx, &t.found, cap))) return rc;
            }
        }
    if ((rc = waveAlloc(ctx, &w.ctl, 1))) return rc;
    ctx->waveP = P;
    ctx->waveGroups = groups;
    ctx->waveStats = stats;
    return SKGPU_OK;
}

}  // namespace

extern "C" {

int skgpu_abi_version(void) { return SKGPU_ABI_VERSION; }

int skgpu_device_count(int32_t* count)
{
    if (!count) return SKGPU_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
    *count = n;
    return SKGPU_OK;
}

int skgpu_create(int device, skgpu_ctx** out)
{
    if (!out) return SKGPU_ERR_ARG;
    *out = nullptr;
    skgpu_ctx* ctx = new skgpu_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->numSMs, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
    if (e == cudaSuccess) e = devAlloc(&ctx->errFlag, 1);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&ctx->doneHost), sizeof(unsigned long long));
    if (e != cudaSuccess)
    {
        // keep the context so the caller can read the message; the handle must still be destroyed
        ctx->err = std::string("skgpu_create: ") + cudaGetErrorString(e);
        *out = ctx;
        return SKGPU_ERR_CUDA;
    }
    ctx->opt.force_scattering = 1;
    ctx->opt.min_weight_reduction = 1e4;
    ctx->opt.path_length_bias = 0.5;
    ctx->opt.peel_off = 1;
    *out = ctx;
    return SKGPU_OK;
}

void skgpu_destroy(skgpu_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    freeGrid(ctx);
    freeInstruments(ctx);
    devFree(ctx->dens);
    devFree(ctx->mixLb);
    devFree(ctx->mixExt);
    devFree(ctx->mixSca);
    devFree(ctx->mixG);
    devFree(ctx->rfB);
    devFree(ctx->rfEll);
    devFree(ctx->rf);
    devFree(ctx->src);
    devFree(ctx->tabL);
    devFree(ctx->tabA);
    devFree(ctx->tabB);
    devFree(ctx->radR);
    devFree(ctx->radP);
    freeWave(ctx);
    ctx->graphCache.release();
    for (void* p : ctx->batchBufs) cudaFree(p);
    cudaFree(ctx->rfT);
    cudaFree(ctx->orderKeys);
    cudaFree(ctx->orderIdx);
    cudaFree(ctx->orderCounts);
    guideDestroy(ctx);
    freeBufs(ctx->deBufs);
    freeBufs(ctx->secBufs);
    devFree(ctx->errFlag);
    if (ctx->doneHost) cudaFreeHost(ctx->doneHost);
    for (int i = 0; i < 2; ++i)
    {
        if (ctx->pin[i]) cudaFreeHost(ctx->pin[i]);
        if (ctx->pinEv[i]) cudaEventDestroy(ctx->pinEv[i]);
    }
    if (ctx->timerEvents)
        for (auto& row : ctx->timer.ev)
            for (cudaEvent_t ev : row)
                if (ev) cudaEventDestroy(ev);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* skgpu_last_error(const skgpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// ------------------------------------------------------------------------------------------------
// grids
// ------------------------------------------------------------------------------------------------

int skgpu_upload_grid_cartesian(skgpu_ctx* ctx, const double* xb, int32_t nxb, const double* yb, int32_t nyb,
                                const double* zb, int32_t nzb)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!xb || !yb || !zb || nxb < 2 || nyb < 2 || nzb < 2)
        return fail(ctx, SKGPU_ERR_ARG, "cartesian grid needs at least 2 borders per axis");
    auto ascending = [](const double* v, int n) {
        for (int i = 1; i < n; ++i)
            if (!(v[i] > v[i - 1])) return false;
        return true;
    };
    if (!ascending(xb, nxb) || !ascending(yb, nyb) || !ascending(zb, nzb))
        return fail(ctx, SKGPU_ERR_ARG, "cartesian borders must be strictly ascending");
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_CARTESIAN;
    g.nx = nxb - 1;
    g.ny = nyb - 1;
    g.nz = nzb - 1;
    g.ext[0] = xb[0]; g.ext[1] = yb[0]; g.ext[2] = zb[0];
    g.ext[3] = xb[nxb - 1]; g.ext[4] = yb[nyb - 1]; g.ext[5] = zb[nzb - 1];
    long long nc = 1LL * g.nx * g.ny * g.nz;
    if (nc > 2147483647LL) return fail(ctx, SKGPU_ERR_ARG, "too many cells");
    g.numCells = static_cast<int>(nc);
    int rc;
    if ((rc = gridUpload(ctx, &g.xb, xb, nxb))) return rc;
    if ((rc = gridUpload(ctx, &g.yb, yb, nyb))) return rc;
    if ((rc = gridUpload(ctx, &g.zb, zb, nzb))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

namespace {
// AdaptiveMeshSnapshot::Node::leaf / child on the host (AdaptiveMeshSnapshot.cpp:103-145), over the
// traversal arrays and the derived subdivisions: -1 outside the root, -2 where the reference stops
// with "Can't locate the appropriate child node"
int adaptiveLeafHost(const double* bounds, const int* div, const int* childBegin, const int* child, double x, double y,
                     double z)
{
    auto contains = [&](int l) {
        const double* b = bounds + 6 * static_cast<size_t>(l);
        return x >= b[0] && x <= b[3] && y >= b[1] && y <= b[4] && z >= b[2] && z <= b[5];
    };
    if (!contains(0)) return -1;
    int node = 0;
    for (int guard = 0; guard < 256; ++guard)
    {
        int nx = div[3 * node], ny = div[3 * node + 1], nz = div[3 * node + 2];
        if (nx == 0) return node;
        const double* b = bounds + 6 * static_cast<size_t>(node);
        int i = std::max(0, std::min(nx - 1, static_cast<int>(nx * (x - b[0]) / (b[3] - b[0]))));
        int j = std::max(0, std::min(ny - 1, static_cast<int>(ny * (y - b[1]) / (b[4] - b[1]))));
        int k = std::max(0, std::min(nz - 1, static_cast<int>(nz * (z - b[2]) / (b[5] - b[2]))));
        const int* kids = child + childBegin[node];
        int c = kids[(k * ny + j) * nx + i];
        if (!contains(c))
        {
            const double* cb = bounds + 6 * static_cast<size_t>(c);
            if (x < cb[0]) i--;
            else if (x > cb[3]) i++;
            if (y < cb[1]) j--;
            else if (y > cb[4]) j++;
            if (z < cb[2]) k--;
            else if (z > cb[5]) k++;
            if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) return -2;
            c = kids[(k * ny + j) * nx + i];
            if (!contains(c)) return -2;
        }
        node = c;
    }
    return -2;
}
}  // namespace

int skgpu_upload_grid_adaptive_mesh(skgpu_ctx* ctx, int32_t num_nodes, const double* bounds, const int32_t* cell_index,
                                    const int32_t* child_begin, const int32_t* child_count, const int32_t* child_index,
                                    int32_t num_child_index, double eps)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_nodes < 1 || !bounds || !cell_index || !child_begin || !child_count || (num_child_index > 0 && !child_index))
        return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: missing arrays");
    if (num_child_index < 0) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: negative sizes");
    if (!finiteAll(bounds, 6 * static_cast<size_t>(num_nodes))) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: non-finite bounds");
    if (!(eps > 0) || !std::isfinite(eps)) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: bad eps");
    // the subdivision of every nonleaf node from its children's bounds: the children form an
    // nx x ny x nz lattice in local Morton order (x fastest), each the parent's Box::fracPos cell
    std::vector<int> div(3 * static_cast<size_t>(num_nodes), 0);
    std::vector<int> parents(num_nodes, 0);
    int numCells = 0, numLeaves = 0;
    for (int l = 0; l < num_nodes; ++l)
    {
        int cnt = child_count[l];
        const double* b = bounds + 6 * static_cast<size_t>(l);
        if (cnt == 0)
        {
            if (cell_index[l] < 0 || cell_index[l] >= num_nodes) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: leaf without cell index");
            numCells = std::max(numCells, cell_index[l] + 1);
            numLeaves++;
            continue;
        }
        int cb = child_begin[l];
        if (cnt < 0 || cb < 0 || cb + cnt > num_child_index) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: child index out of range");
        const int* kids = child_index + cb;
        for (int q = 0; q < cnt; ++q)
        {
            if (kids[q] <= 0 || kids[q] >= num_nodes) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: child id out of range");
            if (++parents[kids[q]] > 1) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: a node is the child of two nodes");
        }
        const double* c0 = bounds + 6 * static_cast<size_t>(kids[0]);
        int nx = 0, ny = 0, nz = 0;
        for (int q = 0; q < cnt; ++q)
        {
            const double* c = bounds + 6 * static_cast<size_t>(kids[q]);
            if (c[1] == c0[1] && c[2] == c0[2]) nx++;
            if (c[0] == c0[0] && c[2] == c0[2]) ny++;
            if (c[0] == c0[0] && c[1] == c0[1]) nz++;
        }
        if (nx * ny * nz != cnt) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: children are not a lattice");
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                {
                    // Box::fracPos(i, j, k, nx, ny, nz) and (i+1, j+1, k+1) (SKIRT/utils/Box.hpp:154-158)
                    const double* c = bounds + 6 * static_cast<size_t>(kids[(k * ny + j) * nx + i]);
                    double e[6] = {b[0] + i * (b[3] - b[0]) / nx, b[1] + j * (b[4] - b[1]) / ny, b[2] + k * (b[5] - b[2]) / nz,
                                   b[0] + (i + 1) * (b[3] - b[0]) / nx, b[1] + (j + 1) * (b[4] - b[1]) / ny,
                                   b[2] + (k + 1) * (b[5] - b[2]) / nz};
                    for (int a = 0; a < 6; ++a)
                        if (c[a] != e[a]) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: children not in local Morton order");
                }
        div[3 * static_cast<size_t>(l)] = nx;
        div[3 * static_cast<size_t>(l) + 1] = ny;
        div[3 * static_cast<size_t>(l) + 2] = nz;
    }
    if (numCells != numLeaves) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: cell indices are not 0..leaves-1");
    for (int l = 1; l < num_nodes; ++l)
        if (parents[l] != 1) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: node unreachable from the root");
    // Node::addNeighbors (AdaptiveMeshSnapshot.cpp:67-83): per leaf wall the leaf holding the point
    // eps beyond the centre of the wall, in CSR form (no entry at domain walls)
    std::vector<int32_t> nbBegin(6 * static_cast<size_t>(num_nodes) + 1, 0), nb;
    for (int l = 0; l < num_nodes; ++l)
    {
        for (int w = 0; w < 6; ++w)
        {
            nbBegin[6 * static_cast<size_t>(l) + w] = static_cast<int32_t>(nb.size());
            if (child_count[l] != 0) continue;
            const double* b = bounds + 6 * static_cast<size_t>(l);
            double cx = 0.5 * (b[0] + b[3]), cy = 0.5 * (b[1] + b[4]), cz = 0.5 * (b[2] + b[5]);
            double x = cx + (w == 0 ? -eps : w == 1 ? eps : 0.);
            double y = cy + (w == 2 ? -eps : w == 3 ? eps : 0.);
            double z = cz + (w == 4 ? -eps : w == 5 ? eps : 0.);
            int n = adaptiveLeafHost(bounds, div.data(), child_begin, child_index, x, y, z);
            if (n == -2) return fail(ctx, SKGPU_ERR_ARG, "adaptive mesh: cannot locate a child node");
            if (n >= 0) nb.push_back(n);
        }
    }
    nbBegin[6 * static_cast<size_t>(num_nodes)] = static_cast<int32_t>(nb.size());
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_ADAPTIVE_MESH;
    for (int q = 0; q < 6; ++q) g.ext[q] = bounds[q];
    g.eps = eps;
    g.tNodes = num_nodes;
    g.numCells = numCells;
    int rc;
    if ((rc = gridUpload(ctx, &g.tBounds, bounds, 6 * static_cast<size_t>(num_nodes)))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.tCell, cell_index, num_nodes))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.tNbBegin, nbBegin.data(), nbBegin.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.tNb, nb.data(), nb.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.amDiv, div.data(), div.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.amChildBegin, child_begin, num_nodes))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.amChild, child_index, static_cast<size_t>(num_child_index)))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

int skgpu_upload_grid_octree(skgpu_ctx* ctx, int32_t num_nodes, const double* bounds, const int32_t* cell_index,
                             const int32_t* child_begin, const int32_t* child_count, const int32_t* child_index,
                             int32_t num_child_index, const int32_t* nb_begin, const int32_t* nb_index,
                             int32_t num_nb_index, double eps)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_nodes < 1 || !bounds || !cell_index || !child_begin || !child_count || !nb_begin)
        return fail(ctx, SKGPU_ERR_ARG, "octree: missing arrays");
    if (num_child_index < 0 || num_nb_index < 0) return fail(ctx, SKGPU_ERR_ARG, "octree: negative sizes");
    // first-child table; OctTreeNode children are created with consecutive ids (OctTreeNode.cpp:15-25)
    std::vector<int> firstChild(num_nodes, -1);
    int numCells = 0;
    for (int l = 0; l < num_nodes; ++l)
    {
        int cnt = child_count[l];
        if (cnt == 0)
        {
            if (cell_index[l] < 0) return fail(ctx, SKGPU_ERR_ARG, "octree: leaf without cell index");
            numCells = std::max(numCells, cell_index[l] + 1);
            continue;
        }
        if (cnt != 8) return fail(ctx, SKGPU_ERR_UNSUPPORTED, "octree: only 8-way subdivision is supported");
        int b = child_begin[l];
        if (b < 0 || b + 8 > num_child_index) return fail(ctx, SKGPU_ERR_ARG, "octree: child index out of range");
        int c0 = child_index[b];
        for (int q = 0; q < 8; ++q)
            if (child_index[b + q] != c0 + q || c0 + q >= num_nodes)
                return fail(ctx, SKGPU_ERR_ARG, "octree: children must have consecutive node ids");
        firstChild[l] = c0;
    }
    if (nb_begin[0] != 0 || nb_begin[6 * static_cast<size_t>(num_nodes)] != num_nb_index)
        return fail(ctx, SKGPU_ERR_ARG, "octree: neighbour CSR inconsistent");
    for (int e = 0; e < num_nb_index; ++e)
        if (nb_index[e] < 0 || nb_index[e] >= num_nodes) return fail(ctx, SKGPU_ERR_ARG, "octree: neighbour id out of range");
    if (!finiteAll(bounds, 6 * static_cast<size_t>(num_nodes))) return fail(ctx, SKGPU_ERR_ARG, "octree: non-finite bounds");
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_OCTREE;
    for (int q = 0; q < 6; ++q) g.ext[q] = bounds[q];
    g.eps = eps;
    g.tNodes = num_nodes;
    g.numCells = numCells;
    int rc;
    if ((rc = gridUpload(ctx, &g.tBounds, bounds, 6 * static_cast<size_t>(num_nodes)))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.tCell, cell_index, num_nodes))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.tChild, firstChild.data(), num_nodes))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.tNbBegin, nb_begin, 6 * static_cast<size_t>(num_nodes) + 1))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.tNb, nb_index, num_nb_index))) return rc;
    // The octree's lattice. OctTreeNode::createChildren (OctTreeNode.cpp:15-25) gives each child a
    // copy of its parent's bounds and centre, so in a tree of depth L every wall coordinate is one of
    // 2^L + 1 FP64 values per axis, indexed by its position at the finest level (root [0, 2^L]).
    // The production walker's records hold these 16-bit indices (L <= 15) and the walker reads the
    // exact FP64 walls from three small tables. A tree that is not such a lattice (or deeper) gets
    // no production records; its FP32-precision runs use the FP64 node walker.
    std::vector<int> depth(num_nodes, -1), ilo(3 * static_cast<size_t>(num_nodes)), ihi(3 * static_cast<size_t>(num_nodes));
    std::vector<int> queue{0};
    depth[0] = 0;
    int L = 0;
    for (size_t qi = 0; qi < queue.size(); ++qi)
    {
        int l = queue[qi];
        L = std::max(L, depth[l]);
        if (firstChild[l] < 0) continue;
        for (int q = 0; q < 8; ++q)
        {
            int c = firstChild[l] + q;
            if (depth[c] >= 0) return fail(ctx, SKGPU_ERR_ARG, "octree: a node is the child of two nodes");
            depth[c] = depth[l] + 1;
            queue.push_back(c);
        }
    }
    if (static_cast<int>(queue.size()) != num_nodes) return fail(ctx, SKGPU_ERR_ARG, "octree: nodes unreachable from the root");
    bool lattice = L <= 15;
    const int N = lattice ? (1 << L) : 0;
    std::vector<double> wall(lattice ? 3 * static_cast<size_t>(N + 1) : 0, std::numeric_limits<double>::quiet_NaN());
    if (lattice)
    {
        for (int a = 0; a < 3; ++a)
        {
            ilo[a] = 0;
            ihi[a] = N;
        }
        for (size_t qi = 0; qi < queue.size() && lattice; ++qi)
        {
            int l = queue[qi];
            const double* b = bounds + 6 * static_cast<size_t>(l);
            for (int a = 0; a < 3 && lattice; ++a)
            {
                int lo = ilo[3 * static_cast<size_t>(l) + a], hi = ihi[3 * static_cast<size_t>(l) + a];
                double* wl = &wall[static_cast<size_t>(a) * (N + 1) + lo];
                double* wh = &wall[static_cast<size_t>(a) * (N + 1) + hi];
                if (std::isnan(*wl)) *wl = b[a];
                if (std::isnan(*wh)) *wh = b[3 + a];
                lattice = *wl == b[a] && *wh == b[3 + a] && hi > lo;
            }
            if (!lattice || firstChild[l] < 0) continue;
            for (int q = 0; q < 8; ++q)
            {
                int c = firstChild[l] + q;
                for (int a = 0; a < 3; ++a)
                {
                    int lo = ilo[3 * static_cast<size_t>(l) + a], hi = ihi[3 * static_cast<size_t>(l) + a], mid = (lo + hi) / 2;
                    bool upper = (q >> a) & 1;
                    ilo[3 * static_cast<size_t>(c) + a] = upper ? mid : lo;
                    ihi[3 * static_cast<size_t>(c) + a] = upper ? hi : mid;
                }
            }
        }
    }
    g.tWallN = 0;
    if (!lattice)
    {
        ctx->hasGrid = true;
        return syncLeafDensity(ctx);
    }
    // Leaf-indexed 64-byte records of the production walker (cell c <-> its leaf node), four int4:
    //   [0] wall indices x lo | hi << 16, y, z; FP32 density (filled when the medium is uploaded)
    //   [1] neighbour-list base, the 9-bit cumulative offsets of the 6 walls in the list (64 bits, all
    //       ones: no list), the leaf's node id (for the full neighbour lists of the exact fallback)
    //   [2] [3] per wall the one neighbour across it when there is exactly one (-1: no neighbour, the
    //       domain wall; -2: several, scan the list), two spare words
    // The lists hold per wall the positive-overlap neighbours in the reference's overlap order;
    // zero-overlap entries, which only touch an edge, come last in the reference's lists (TreeNode
    // sortNeighbors, TreeNode.cpp:200-207) and are left to the walker's exact fallback.
    std::vector<int> leafNode(numCells, -1);
    for (int l = 0; l < num_nodes; ++l)
        if (cell_index[l] >= 0) leafNode[cell_index[l]] = l;
    std::vector<int4> rec(4 * static_cast<size_t>(numCells));
    std::vector<int> leafNb;
    leafNb.reserve(static_cast<size_t>(numCells) * 8);
    for (int c = 0; c < numCells; ++c)
    {
        int l = leafNode[c];
        if (l < 0) return fail(ctx, SKGPU_ERR_ARG, "octree: cell index without leaf");
        const double* b = bounds + 6 * static_cast<size_t>(l);
        int base = static_cast<int>(leafNb.size());
        // per wall the positive-overlap neighbours; 9-bit cumulative offsets of the 6 walls + end
        // (a leaf with more than 511 such neighbours gets no list: its exits use the exact fallback)
        std::vector<int> lists[6];
        size_t total = 0;
        for (int w = 0; w < 6; ++w)
        {
            int a = w / 2, u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;
            for (int e = nb_begin[6 * static_cast<size_t>(l) + w]; e < nb_begin[6 * static_cast<size_t>(l) + w + 1]; ++e)
            {
                int nn = nb_index[e];
                const double* q = bounds + 6 * static_cast<size_t>(nn);
                double ou = std::min(b[3 + u], q[3 + u]) - std::max(b[u], q[u]);
                double ov = std::min(b[3 + v], q[3 + v]) - std::max(b[v], q[v]);
                if (!(ou > 0 && ov > 0) || cell_index[nn] < 0) continue;
                lists[w].push_back(cell_index[nn]);
            }
            total += lists[w].size();
        }
        unsigned long long cnt = 0;
        if (total > 511)
        {
            cnt = ~0ULL;
        }
        else
        {
            unsigned long long off = 0;
            for (int w = 0; w < 6; ++w)
            {
                cnt |= off << (9 * w);
                leafNb.insert(leafNb.end(), lists[w].begin(), lists[w].end());
                off += lists[w].size();
            }
            cnt |= off << 54;
        }
        int one[6];
        for (int w = 0; w < 6; ++w)
            one[w] = lists[w].size() == 1 ? lists[w][0] : (lists[w].empty() && total <= 511 ? -1 : -2);
        auto idx = [&](int a) {
            return static_cast<int>(static_cast<unsigned>(ilo[3 * static_cast<size_t>(l) + a])
                                    | (static_cast<unsigned>(ihi[3 * static_cast<size_t>(l) + a]) << 16));
        };
        int4* r = &rec[4 * static_cast<size_t>(c)];
        r[0] = make_int4(idx(0), idx(1), idx(2), 0);
        r[1] = make_int4(base, static_cast<int>(static_cast<unsigned>(cnt)), static_cast<int>(static_cast<unsigned>(cnt >> 32)), l);
        r[2] = make_int4(one[0], one[1], one[2], one[3]);
        r[3] = make_int4(one[4], one[5], 0, 0);
        if (leafNb.size() > 2147483647ULL) return fail(ctx, SKGPU_ERR_ARG, "octree: neighbour lists too long");
    }
    if (leafNb.empty()) leafNb.push_back(0);
    if ((rc = gridUpload<int4>(ctx, &g.tRec, rec.data(), rec.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.tLeafNb, leafNb.data(), leafNb.size()))) return rc;
    if ((rc = gridUpload<double>(ctx, &g.tWall, wall.data(), wall.size()))) return rc;
    g.tWallN = N + 1;
    ctx->hasGrid = true;
    return syncLeafDensity(ctx);
}

int skgpu_upload_grid_voronoi(skgpu_ctx* ctx, int32_t num_sites, const double* sites, const int32_t* nb_begin,
                              const int32_t* nb_index, int32_t num_nb_index, const double* extent, double eps)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_sites < 1 || !sites || !nb_begin || !extent) return fail(ctx, SKGPU_ERR_ARG, "voronoi: missing arrays");
    if (nb_begin[0] != 0 || nb_begin[num_sites] != num_nb_index) return fail(ctx, SKGPU_ERR_ARG, "voronoi: neighbour CSR inconsistent");
    for (int e = 0; e < num_nb_index; ++e)
        if (nb_index[e] >= num_sites || nb_index[e] < -6) return fail(ctx, SKGPU_ERR_ARG, "voronoi: neighbour id out of range");
    if (!finiteAll(sites, 3 * static_cast<size_t>(num_sites))) return fail(ctx, SKGPU_ERR_ARG, "voronoi: non-finite sites");
    // uniform site-search grid, about two sites per block
    int n = static_cast<int>(std::cbrt(num_sites / 2.0));
    n = std::max(1, std::min(256, n));
    std::vector<int> cnt(static_cast<size_t>(n) * n * n + 1, 0), blk(num_sites);
    for (int s = 0; s < num_sites; ++s)
    {
        auto idx = [&](double x, double lo, double hi) {
            return std::min(n - 1, std::max(0, static_cast<int>((x - lo) / ((hi - lo) / n))));
        };
        int i = idx(sites[3 * s], extent[0], extent[3]);
        int j = idx(sites[3 * s + 1], extent[1], extent[4]);
        int k = idx(sites[3 * s + 2], extent[2], extent[5]);
        blk[s] = (i * n + j) * n + k;
        cnt[blk[s] + 1]++;
    }
    for (size_t b = 1; b < cnt.size(); ++b) cnt[b] += cnt[b - 1];
    std::vector<int> fill(cnt.begin(), cnt.end() - 1), list(num_sites);
    for (int s = 0; s < num_sites; ++s) list[fill[blk[s]]++] = s;
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_VORONOI;
    for (int q = 0; q < 6; ++q) g.ext[q] = extent[q];
    g.eps = eps;
    g.vN = num_sites;
    g.numCells = num_sites;
    g.vGridN = n;
    int rc;
    if ((rc = gridUpload(ctx, &g.vSites, sites, 3 * static_cast<size_t>(num_sites)))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.vNbBegin, nb_begin, num_sites + 1))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.vNb, nb_index, num_nb_index))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.vBlkBegin, cnt.data(), cnt.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.vBlkSites, list.data(), list.size()))) return rc;
    // a representative site per block: its first site, or for an empty block that of the nearest
    // filled block found by growing the filled region one block at a time
    {
        size_t nb3 = static_cast<size_t>(n) * n * n;
        std::vector<int> rep(nb3, -1);
        for (size_t b = 0; b < nb3; ++b)
            if (cnt[b + 1] > cnt[b]) rep[b] = list[cnt[b]];
        for (int pass = 0; pass < 3 * n; ++pass)
        {
            bool open = false;
            std::vector<int> nxt = rep;
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                    for (int k = 0; k < n; ++k)
                    {
                        size_t b = (static_cast<size_t>(i) * n + j) * n + k;
                        if (rep[b] >= 0) continue;
                        open = true;
                        const int di[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
                        for (const auto& d : di)
                        {
                            int a = i + d[0], bb = j + d[1], c = k + d[2];
                            if (a < 0 || bb < 0 || c < 0 || a >= n || bb >= n || c >= n) continue;
                            int r = rep[(static_cast<size_t>(a) * n + bb) * n + c];
                            if (r >= 0)
                            {
                                nxt[b] = r;
                                break;
                            }
                        }
                    }
            rep.swap(nxt);
            if (!open) break;
        }
        for (int& r : rep)
            if (r < 0) r = 0;
        if ((rc = gridUpload<int>(ctx, &g.vBlkRep, rep.data(), rep.size()))) return rc;
    }
    // records of the FP32 walker, one per cell in 16-byte units: the FP64 site and the cell's face
    // count, then per face the outward unit normal and the distance of the face's plane from the site
    // (half the site distance for a neighbour, the distance to the domain wall for a wall), so that
    // s = (d - n . l) / (n . k) needs no squares of metre-scale coordinates, then per face the
    // neighbour's record offset (or the wall id); the faces are padded to a multiple of 4
    // The records are laid out in the Morton order of their sites (21 bits per axis over the
    // domain), not in cell order: a record spans several cache lines, and cells that are close in
    // space (and so visited together) then share lines and DRAM pages. Only the layout changes;
    // every record keeps its cell index.
    std::vector<int> layout(num_sites);
    {
        auto spread = [](uint64_t v) {
            v &= 0x1FFFFF;
            v = (v | v << 32) & 0x1F00000000FFFFULL;
            v = (v | v << 16) & 0x1F0000FF0000FFULL;
            v = (v | v << 8) & 0x100F00F00F00F00FULL;
            v = (v | v << 4) & 0x10C30C30C30C30C3ULL;
            v = (v | v << 2) & 0x1249249249249249ULL;
            return v;
        };
        std::vector<uint64_t> key(num_sites);
        for (int c = 0; c < num_sites; ++c)
        {
            uint64_t q[3];
            for (int a = 0; a < 3; ++a)
            {
                double f = (sites[3 * static_cast<size_t>(c) + a] - extent[a]) / (extent[a + 3] - extent[a]);
                f = std::min(std::max(f, 0.), 1.);
                q[a] = static_cast<uint64_t>(f * 2097151.);
            }
            key[c] = spread(q[0]) | spread(q[1]) << 1 | spread(q[2]) << 2;
        }
        for (int c = 0; c < num_sites; ++c) layout[c] = c;
        std::stable_sort(layout.begin(), layout.end(), [&](int a, int b) { return key[a] < key[b]; });
    }
    std::vector<int> recOff(num_sites);
    size_t units = 0;
    for (int q = 0; q < num_sites; ++q)
    {
        int c = layout[q];
        size_t n4 = (static_cast<size_t>(nb_begin[c + 1] - nb_begin[c]) + 3) & ~static_cast<size_t>(3);
        recOff[c] = static_cast<int>(units);
        units += 2 + n4 + n4 / 4;
        if (units > 2147483647ULL) return fail(ctx, SKGPU_ERR_ARG, "voronoi: mesh too large for 32-bit record offsets");
    }
    std::vector<float4> rec(units);
    for (int c = 0; c < num_sites; ++c)
    {
        const double* pc = sites + 3 * static_cast<size_t>(c);
        float4* R = rec.data() + recOff[c];
        int nf = nb_begin[c + 1] - nb_begin[c];
        int n4 = (nf + 3) & ~3;
        double* hd = reinterpret_cast<double*>(R);
        hd[0] = pc[0];
        hd[1] = pc[1];
        hd[2] = pc[2];
        int* hi = reinterpret_cast<int*>(R + 1);
        hi[2] = c;
        hi[3] = nf;
        int* ids = reinterpret_cast<int*>(R + 2 + n4);
        for (int j = 0; j < n4; ++j)
        {
            if (j >= nf)
            {
                R[2 + j] = make_float4(0.f, 0.f, 0.f, 0.f);
                ids[j] = -100;  // padding face: never ahead
                continue;
            }
            int mi = nb_index[nb_begin[c] + j];
            double n[3] = {0, 0, 0}, d = 0;
            if (mi >= 0)
            {
                const double* pi = sites + 3 * static_cast<size_t>(mi);
                for (int a = 0; a < 3; ++a) n[a] = pi[a] - pc[a];
                double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                if (len > 0)
                    for (int a = 0; a < 3; ++a) n[a] /= len;
                d = 0.5 * len;
                ids[j] = recOff[mi];
            }
            else
            {
                int a = (-mi - 1) >> 1;
                bool upper = ((-mi - 1) & 1) != 0;
                n[a] = upper ? 1.0 : -1.0;
                d = upper ? extent[3 + a] - pc[a] : pc[a] - extent[a];
                ids[j] = mi;
            }
            R[2 + j] = make_float4(static_cast<float>(n[0]), static_cast<float>(n[1]), static_cast<float>(n[2]),
                                   static_cast<float>(d));
        }
    }
    if ((rc = gridUpload<float4>(ctx, &g.vRec, rec.data(), rec.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.vRecOff, recOff.data(), recOff.size()))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

int skgpu_upload_voronoi_cell_boxes(skgpu_ctx* ctx, int32_t num_cells, const double* boxes)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!ctx->hasGrid || ctx->g.kind != SKGPU_GRID_VORONOI) return fail(ctx, SKGPU_ERR_STATE, "voronoi boxes: no Voronoi grid");
    if (num_cells != ctx->g.vN || !boxes) return fail(ctx, SKGPU_ERR_ARG, "voronoi boxes: one box per cell expected");
    if (!finiteAll(boxes, 6 * static_cast<size_t>(num_cells))) return fail(ctx, SKGPU_ERR_ARG, "voronoi boxes: non-finite value");
    CK(cudaSetDevice(ctx->device));
    return gridUpload(ctx, &ctx->g.vBox, boxes, 6 * static_cast<size_t>(num_cells));
}

int skgpu_upload_grid_sphere1d(skgpu_ctx* ctx, int32_t num_borders, const double* rv)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_borders < 2 || !rv || !(rv[0] >= 0.)) return fail(ctx, SKGPU_ERR_ARG, "sphere1d: need >= 2 borders from r >= 0");
    if (!finiteAll(rv, num_borders)) return fail(ctx, SKGPU_ERR_ARG, "sphere1d: non-finite border");
    for (int i = 1; i < num_borders; ++i)
        if (!(rv[i] > rv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "sphere1d: borders must ascend");
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_SPHERE1D;
    double r = rv[num_borders - 1];
    double e[6] = {-r, -r, -r, r, r, r};
    for (int q = 0; q < 6; ++q) g.ext[q] = e[q];
    g.eps = 1e-12 * std::sqrt(3.) * 2. * r;
    g.sNr = num_borders - 1;
    g.numCells = g.sNr;
    int rc;
    if ((rc = gridUpload(ctx, &g.sRv, rv, static_cast<size_t>(num_borders)))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

int skgpu_upload_grid_cylinder2d(skgpu_ctx* ctx, int32_t nrb, const double* rv, int32_t nzb, const double* zv)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (nrb < 2 || nzb < 2 || !rv || !zv || !(rv[0] >= 0.)) return fail(ctx, SKGPU_ERR_ARG, "cylinder2d: need >= 2 radial borders from R >= 0 and >= 2 z borders");
    if (!finiteAll(rv, nrb) || !finiteAll(zv, nzb)) return fail(ctx, SKGPU_ERR_ARG, "cylinder2d: non-finite border");
    for (int i = 1; i < nrb; ++i)
        if (!(rv[i] > rv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "cylinder2d: radial borders must ascend");
    for (int i = 1; i < nzb; ++i)
        if (!(zv[i] > zv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "cylinder2d: z borders must ascend");
    if (static_cast<int64_t>(nrb - 1) * (nzb - 1) > 2147483647LL) return fail(ctx, SKGPU_ERR_ARG, "cylinder2d: too many cells");
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_CYLINDER2D;
    double r = rv[nrb - 1];
    double e[6] = {-r, -r, zv[0], r, r, zv[nzb - 1]};
    for (int q = 0; q < 6; ++q) g.ext[q] = e[q];
    g.eps = 1e-12 * std::sqrt(2. * (2. * r) * (2. * r) + (zv[nzb - 1] - zv[0]) * (zv[nzb - 1] - zv[0]));
    g.cNR = nrb - 1;
    g.cNz = nzb - 1;
    g.numCells = g.cNR * g.cNz;
    int rc;
    if ((rc = gridUpload(ctx, &g.cRv, rv, static_cast<size_t>(nrb)))) return rc;
    if ((rc = gridUpload(ctx, &g.czv, zv, static_cast<size_t>(nzb)))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

int skgpu_upload_grid_sphere2d(skgpu_ctx* ctx, int32_t nrb, const double* rv, int32_t ntb, const double* tv,
                               const double* cv)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (nrb < 2 || ntb < 2 || !rv || !tv || !cv || !(rv[0] >= 0.)) return fail(ctx, SKGPU_ERR_ARG, "sphere2d: need >= 2 radial borders from r >= 0 and >= 2 polar borders");
    if (!finiteAll(rv, nrb) || !finiteAll(tv, ntb) || !finiteAll(cv, ntb)) return fail(ctx, SKGPU_ERR_ARG, "sphere2d: non-finite border");
    for (int i = 1; i < nrb; ++i)
        if (!(rv[i] > rv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "sphere2d: radial borders must ascend");
    for (int i = 1; i < ntb; ++i)
        if (!(tv[i] > tv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "sphere2d: polar borders must ascend");
    if (static_cast<int64_t>(nrb - 1) * (ntb - 1) > 2147483647LL) return fail(ctx, SKGPU_ERR_ARG, "sphere2d: too many cells");
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_SPHERE2D;
    double r = rv[nrb - 1];
    double e[6] = {-r, -r, -r, r, r, r};
    for (int q = 0; q < 6; ++q) g.ext[q] = e[q];
    g.eps = 1e-11 * r;
    g.s2Nr = nrb - 1;
    g.s2Nt = ntb - 1;
    g.numCells = g.s2Nr * g.s2Nt;
    int rc;
    if ((rc = gridUpload(ctx, &g.s2r, rv, static_cast<size_t>(nrb)))) return rc;
    if ((rc = gridUpload(ctx, &g.s2t, tv, static_cast<size_t>(ntb)))) return rc;
    if ((rc = gridUpload(ctx, &g.s2c, cv, static_cast<size_t>(ntb)))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

int skgpu_upload_grid_sphere3d(skgpu_ctx* ctx, int32_t nrb, const double* rv, int32_t ntb, const double* tv,
                               const double* cv, int32_t npb, const double* pv, const double* sv, const double* kv,
                               double eps)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (nrb < 2 || ntb < 2 || npb < 2 || !rv || !tv || !cv || !pv || !sv || !kv || !(rv[0] >= 0.) || !(eps > 0.))
        return fail(ctx, SKGPU_ERR_ARG, "sphere3d: need >= 2 radial, polar and azimuthal borders, r >= 0 and eps > 0");
    if (!finiteAll(rv, nrb) || !finiteAll(tv, ntb) || !finiteAll(cv, ntb) || !finiteAll(pv, npb) || !finiteAll(sv, npb)
        || !finiteAll(kv, npb))
        return fail(ctx, SKGPU_ERR_ARG, "sphere3d: non-finite border");
    for (int i = 1; i < nrb; ++i)
        if (!(rv[i] > rv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "sphere3d: radial borders must ascend");
    for (int i = 1; i < ntb; ++i)
        if (!(tv[i] > tv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "sphere3d: polar borders must ascend");
    for (int i = 1; i < npb; ++i)
        if (!(pv[i] > pv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "sphere3d: azimuthal borders must ascend");
    if (static_cast<int64_t>(nrb - 1) * (ntb - 1) * (npb - 1) > 2147483647LL) return fail(ctx, SKGPU_ERR_ARG, "sphere3d: too many cells");
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_SPHERE3D;
    double r = rv[nrb - 1];
    double e[6] = {-r, -r, -r, r, r, r};
    for (int q = 0; q < 6; ++q) g.ext[q] = e[q];
    g.eps = eps;
    g.s3eps = eps;
    g.s3Nr = nrb - 1;
    g.s3Nt = ntb - 1;
    g.s3Np = npb - 1;
    g.numCells = g.s3Nr * g.s3Nt * g.s3Np;
    int rc;
    if ((rc = gridUpload(ctx, &g.s3r, rv, static_cast<size_t>(nrb)))) return rc;
    if ((rc = gridUpload(ctx, &g.s3t, tv, static_cast<size_t>(ntb)))) return rc;
    if ((rc = gridUpload(ctx, &g.s3c, cv, static_cast<size_t>(ntb)))) return rc;
    if ((rc = gridUpload(ctx, &g.s3p, pv, static_cast<size_t>(npb)))) return rc;
    if ((rc = gridUpload(ctx, &g.s3s, sv, static_cast<size_t>(npb)))) return rc;
    if ((rc = gridUpload(ctx, &g.s3k, kv, static_cast<size_t>(npb)))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

int skgpu_upload_grid_cylinder3d(skgpu_ctx* ctx, int32_t nrb, const double* rv, int32_t npb, const double* pv,
                                 const double* sv, const double* kv, int32_t nzb, const double* zv, double eps,
                                 int32_t has_hole)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (nrb < 2 || npb < 2 || nzb < 2 || !rv || !pv || !sv || !kv || !zv || !(rv[0] >= 0.) || !(eps > 0.))
        return fail(ctx, SKGPU_ERR_ARG, "cylinder3d: need >= 2 radial, azimuthal and vertical borders, R >= 0 and eps > 0");
    if (!finiteAll(rv, nrb) || !finiteAll(pv, npb) || !finiteAll(sv, npb) || !finiteAll(kv, npb) || !finiteAll(zv, nzb))
        return fail(ctx, SKGPU_ERR_ARG, "cylinder3d: non-finite border");
    for (int i = 1; i < nrb; ++i)
        if (!(rv[i] > rv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "cylinder3d: radial borders must ascend");
    for (int i = 1; i < npb; ++i)
        if (!(pv[i] > pv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "cylinder3d: azimuthal borders must ascend");
    for (int i = 1; i < nzb; ++i)
        if (!(zv[i] > zv[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "cylinder3d: vertical borders must ascend");
    if (static_cast<int64_t>(nrb - 1) * (npb - 1) * (nzb - 1) > 2147483647LL) return fail(ctx, SKGPU_ERR_ARG, "cylinder3d: too many cells");
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_CYLINDER3D;
    double r = rv[nrb - 1];
    double e[6] = {-r, -r, zv[0], r, r, zv[nzb - 1]};
    for (int q = 0; q < 6; ++q) g.ext[q] = e[q];
    g.eps = eps;
    g.c3eps = eps;
    g.c3Hole = has_hole ? 1 : 0;
    g.c3Nr = nrb - 1;
    g.c3Np = npb - 1;
    g.c3Nz = nzb - 1;
    g.numCells = g.c3Nr * g.c3Np * g.c3Nz;
    int rc;
    if ((rc = gridUpload(ctx, &g.c3r, rv, static_cast<size_t>(nrb)))) return rc;
    if ((rc = gridUpload(ctx, &g.c3p, pv, static_cast<size_t>(npb)))) return rc;
    if ((rc = gridUpload(ctx, &g.c3s, sv, static_cast<size_t>(npb)))) return rc;
    if ((rc = gridUpload(ctx, &g.c3k, kv, static_cast<size_t>(npb)))) return rc;
    if ((rc = gridUpload(ctx, &g.c3z, zv, static_cast<size_t>(nzb)))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

int skgpu_upload_grid_tetra(skgpu_ctx* ctx, int32_t num_vertices, const double* vertices, int32_t num_tetra,
                            const int32_t* tetra_vertices, const double* face_normals, const int32_t* face_ntetra,
                            const int32_t* face_nface, const double* extent, double eps)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_vertices < 4 || num_tetra < 1 || !vertices || !tetra_vertices || !face_normals || !face_ntetra
        || !face_nface || !extent)
        return fail(ctx, SKGPU_ERR_ARG, "tetra: missing arrays");
    size_t nt = static_cast<size_t>(num_tetra);
    for (size_t q = 0; q < 4 * nt; ++q)
    {
        if (tetra_vertices[q] < 0 || tetra_vertices[q] >= num_vertices) return fail(ctx, SKGPU_ERR_ARG, "tetra: vertex index out of range");
        if (face_ntetra[q] >= num_tetra || face_ntetra[q] < -1) return fail(ctx, SKGPU_ERR_ARG, "tetra: neighbour out of range");
        if (face_nface[q] < -1 || face_nface[q] > 3) return fail(ctx, SKGPU_ERR_ARG, "tetra: face index out of range");
    }
    // bounding boxes (Tetra constructor, TetraMeshSpatialGrid.cpp:54-81) and a uniform box grid
    std::vector<double> box(6 * nt);
    for (size_t t = 0; t < nt; ++t)
    {
        double b[6] = {DBL_MAX, DBL_MAX, DBL_MAX, -DBL_MAX, -DBL_MAX, -DBL_MAX};
        for (int v = 0; v < 4; ++v)
        {
            const double* p = vertices + 3 * static_cast<size_t>(tetra_vertices[4 * t + v]);
            for (int a = 0; a < 3; ++a)
            {
                b[a] = std::min(b[a], p[a]);
                b[3 + a] = std::max(b[3 + a], p[a]);
            }
        }
        std::memcpy(&box[6 * t], b, sizeof b);
    }
    int n = static_cast<int>(std::cbrt(num_tetra / 2.0));
    n = std::max(1, std::min(192, n));
    auto bidx = [&](double x, int a) {
        return std::min(n - 1, std::max(0, static_cast<int>(n * (x - extent[a]) / (extent[3 + a] - extent[a]))));
    };
    std::vector<long long> cnt(static_cast<size_t>(n) * n * n + 1, 0);
    for (size_t t = 0; t < nt; ++t)
    {
        int i0 = bidx(box[6 * t], 0), i1 = bidx(box[6 * t + 3], 0);
        int j0 = bidx(box[6 * t + 1], 1), j1 = bidx(box[6 * t + 4], 1);
        int k0 = bidx(box[6 * t + 2], 2), k1 = bidx(box[6 * t + 5], 2);
        for (int i = i0; i <= i1; ++i)
            for (int j = j0; j <= j1; ++j)
                for (int k = k0; k <= k1; ++k) cnt[(static_cast<size_t>(i) * n + j) * n + k + 1]++;
    }
    for (size_t b = 1; b < cnt.size(); ++b) cnt[b] += cnt[b - 1];
    if (cnt.back() > 2147483647LL) return fail(ctx, SKGPU_ERR_ARG, "tetra: search grid too large");
    std::vector<int> begin(cnt.size()), list(static_cast<size_t>(cnt.back()));
    std::vector<long long> fill(cnt.begin(), cnt.end() - 1);
    for (size_t b = 0; b < cnt.size(); ++b) begin[b] = static_cast<int>(cnt[b]);
    for (size_t t = 0; t < nt; ++t)
    {
        int i0 = bidx(box[6 * t], 0), i1 = bidx(box[6 * t + 3], 0);
        int j0 = bidx(box[6 * t + 1], 1), j1 = bidx(box[6 * t + 4], 1);
        int k0 = bidx(box[6 * t + 2], 2), k1 = bidx(box[6 * t + 5], 2);
        for (int i = i0; i <= i1; ++i)
            for (int j = j0; j <= j1; ++j)
                for (int k = k0; k <= k1; ++k) list[fill[(static_cast<size_t>(i) * n + j) * n + k]++] = static_cast<int>(t);
    }
    // production walker records: each shared face becomes one plane, taken from the side of the
    // lower-numbered tetrahedron (its outward normal rounded to FP32, the offset through the face
    // vertex with the lowest index, in FP64) and exactly negated for the other side
    std::vector<TetRec> rec(nt);
    for (size_t t = 0; t < nt; ++t)
    {
        TetRec& r = rec[t];
        std::memset(&r, 0, sizeof r);
        r.nface = 0;
        for (int f = 0; f < 4; ++f)
        {
            int nb = face_ntetra[4 * t + f];
            int nf = face_nface[4 * t + f];
            r.nb[f] = nb;
            r.nface |= (nb >= 0 ? (nf & 0xff) : 0) << (8 * f);
            size_t owner = t;
            int of = f;
            double sign = 1.0;
            if (nb >= 0 && static_cast<size_t>(nb) < t)
            {
                owner = static_cast<size_t>(nb);
                of = nf;
                sign = -1.0;
            }
            float n32[3];
            for (int a = 0; a < 3; ++a) n32[a] = static_cast<float>(face_normals[12 * owner + 3 * of + a]);
            int vmin = INT32_MAX;
            for (int v = 0; v < 4; ++v)
                if (v != of) vmin = std::min(vmin, tetra_vertices[4 * owner + v]);
            const double* p = vertices + 3 * static_cast<size_t>(vmin);
            double c = static_cast<double>(n32[0]) * p[0] + static_cast<double>(n32[1]) * p[1] + static_cast<double>(n32[2]) * p[2];
            for (int a = 0; a < 3; ++a) r.n[3 * f + a] = static_cast<float>(sign) * n32[a];
            r.c[f] = sign * c;
        }
    }
    std::vector<int> rep(static_cast<size_t>(n) * n * n);
    for (size_t b = 0; b < rep.size(); ++b) rep[b] = begin[b] < begin[b + 1] ? list[begin[b]] : 0;
    CK(cudaSetDevice(ctx->device));
    freeGrid(ctx);
    GridDev& g = ctx->g;
    g.kind = SKGPU_GRID_TETRA;
    for (int q = 0; q < 6; ++q) g.ext[q] = extent[q];
    g.eps = eps;
    g.teN = num_tetra;
    g.numCells = num_tetra;
    g.teGridN = n;
    int rc;
    if ((rc = gridUpload(ctx, &g.teVerts, vertices, 3 * static_cast<size_t>(num_vertices)))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.teTet, tetra_vertices, 4 * nt))) return rc;
    if ((rc = gridUpload(ctx, &g.teNormals, face_normals, 12 * nt))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.teNTet, face_ntetra, 4 * nt))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.teNFace, face_nface, 4 * nt))) return rc;
    if ((rc = gridUpload(ctx, &g.teBox, box.data(), box.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.teBlkBegin, begin.data(), begin.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.teBlkTets, list.data(), list.size()))) return rc;
    if ((rc = gridUpload<TetRec>(ctx, &g.teRec, rec.data(), rec.size()))) return rc;
    if ((rc = gridUpload<int>(ctx, &g.teBlkRep, rep.data(), rep.size()))) return rc;
    ctx->hasGrid = true;
    return SKGPU_OK;
}

// ------------------------------------------------------------------------------------------------
// medium
// ------------------------------------------------------------------------------------------------

int skgpu_upload_medium(skgpu_ctx* ctx, int32_t num_cells, const double* number_density)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_cells < 1 || !number_density) return fail(ctx, SKGPU_ERR_ARG, "medium: missing densities");
    if (!finiteAll(number_density, num_cells)) return fail(ctx, SKGPU_ERR_ARG, "medium: non-finite density");
    CK(cudaSetDevice(ctx->device));
    if (ctx->numCells != num_cells)
    {
        devFree(ctx->dens);
        CK(devAlloc(&ctx->dens, num_cells));
        ctx->numCells = num_cells;
    }
    CK(cudaMemcpy(ctx->dens, number_density, num_cells * sizeof(double), cudaMemcpyHostToDevice));
    return syncLeafDensity(ctx);
}

int skgpu_upload_dust_mix(skgpu_ctx* ctx, int32_t num_lambda, const double* lambda_borders, const double* sigma_ext,
                          const double* sigma_sca, const double* asymmpar)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_lambda < 1 || !lambda_borders || !sigma_ext || !sigma_sca || !asymmpar)
        return fail(ctx, SKGPU_ERR_ARG, "dust mix: missing tables");
    CK(cudaSetDevice(ctx->device));
    devFree(ctx->mixLb);
    devFree(ctx->mixExt);
    devFree(ctx->mixSca);
    devFree(ctx->mixG);
    CK(devUpload(&ctx->mixLb, lambda_borders, num_lambda));
    CK(devUpload(&ctx->mixExt, sigma_ext, num_lambda));
    CK(devUpload(&ctx->mixSca, sigma_sca, num_lambda));
    CK(devUpload(&ctx->mixG, asymmpar, num_lambda));
    ctx->nmix = num_lambda;
    return SKGPU_OK;
}

int skgpu_upload_rf_grid(skgpu_ctx* ctx, int32_t num_bins, int32_t num_borders, const double* borders, const int32_t* ellv)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_bins < 1 || num_borders < 1 || !borders || !ellv) return fail(ctx, SKGPU_ERR_ARG, "rf grid: missing arrays");
    for (int q = 0; q <= num_borders; ++q)
        if (ellv[q] < -1 || ellv[q] >= num_bins) return fail(ctx, SKGPU_ERR_ARG, "rf grid: bin map out of range");
    CK(cudaSetDevice(ctx->device));
    devFree(ctx->rfB);
    devFree(ctx->rfEll);
    CK(devUpload(&ctx->rfB, borders, num_borders));
    CK(devUpload<int>(&ctx->rfEll, ellv, num_borders + 1));
    ctx->nrf = num_bins;
    ctx->rfNb = num_borders;
    return SKGPU_OK;
}

// ------------------------------------------------------------------------------------------------
// sources and instruments
// ------------------------------------------------------------------------------------------------

int skgpu_upload_sources(skgpu_ctx* ctx, int32_t num_sources, const skgpu_source* sources, int32_t table_len,
                         const double* table_lambda, const double* table_a, const double* table_b, int32_t radial_len,
                         const double* radial_r, const double* radial_P)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_sources < 1 || !sources) return fail(ctx, SKGPU_ERR_ARG, "sources: none given");
    std::vector<SourceDev> v(num_sources);
    for (int h = 0; h < num_sources; ++h)
    {
        const skgpu_source& s = sources[h];
        SourceDev& d = v[h];
        if (s.position_model < 0 || s.position_model > 3) return fail(ctx, SKGPU_ERR_ARG, "sources: bad position model");
        if (s.spectral_model < 0 || s.spectral_model > 1) return fail(ctx, SKGPU_ERR_ARG, "sources: bad spectral model");
        if (s.table_size < 1 || s.table_offset < 0 || s.table_offset + s.table_size > table_len)
            return fail(ctx, SKGPU_ERR_ARG, "sources: spectral table out of range");
        if (s.spectral_model == 1 && s.table_size < 2) return fail(ctx, SKGPU_ERR_ARG, "sources: SED table needs 2 points");
        if ((s.position_model == 2 || s.position_model == 3)
            && (s.radial_size < 2 || s.radial_offset < 0 || s.radial_offset + s.radial_size > radial_len))
            return fail(ctx, SKGPU_ERR_ARG, "sources: radial table out of range");
        if (s.position_model == 3)
        {
            for (int i = 0; i < s.radial_size; ++i)
            {
                double sv = radial_r[s.radial_offset + i], mv = radial_P[s.radial_offset + i];
                if (!(sv > 0.) || !(mv >= 0.) || (i > 0 && !(mv >= radial_P[s.radial_offset + i - 1])))
                    return fail(ctx, SKGPU_ERR_ARG, "sources: log-log radial table needs positive radii and ascending masses");
            }
            if (!(s.geometry[0] > 0.)) return fail(ctx, SKGPU_ERR_ARG, "sources: log-log radial table needs a positive scale");
        }
        if (h > 0 && s.first_history < sources[h - 1].first_history)
            return fail(ctx, SKGPU_ERR_ARG, "sources: first_history must be ascending");
        d.posModel = s.position_model;
        d.specModel = s.spectral_model;
        for (int a = 0; a < 3; ++a) d.pos[a] = s.position[a];
        for (int a = 0; a < 6; ++a) d.geom[a] = s.geometry[a];
        d.first = s.first_history;
        d.num = s.num_histories;
        d.Lpk = s.packet_luminosity;
        d.xi = s.wavelength_bias;
        d.bmin = s.bias_lambda_min;
        d.bmax = s.bias_lambda_max;
        d.toff = s.table_offset;
        d.tsize = s.table_size;
        d.roff = s.radial_offset;
        d.rsize = s.radial_size;
    }
    CK(cudaSetDevice(ctx->device));
    devFree(ctx->src);
    devFree(ctx->tabL);
    devFree(ctx->tabA);
    devFree(ctx->tabB);
    devFree(ctx->radR);
    devFree(ctx->radP);
    CK(devUpload(&ctx->src, v.data(), v.size()));
    CK(devUpload(&ctx->tabL, table_lambda, table_len));
    CK(devUpload(&ctx->tabA, table_a, table_len));
    CK(devUpload(&ctx->tabB, table_b, table_b ? table_len : 0));
    CK(devUpload(&ctx->radR, radial_r, radial_r ? radial_len : 0));
    CK(devUpload(&ctx->radP, radial_P, radial_P ? radial_len : 0));
    ctx->srcHost = v;
    return SKGPU_OK;
}

int skgpu_upload_instruments(skgpu_ctx* ctx, int32_t num_instruments, const skgpu_instrument* instruments,
                             int32_t wlg_len, const double* wlg_borders, const int32_t* wlg_ellv)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_instruments < 0 || num_instruments > MAX_INSTR) return fail(ctx, SKGPU_ERR_ARG, "instruments: count out of range");
    if (num_instruments > 0 && instruments[0].same_observer) return fail(ctx, SKGPU_ERR_ARG, "instruments: first cannot share an observer");
    CK(cudaSetDevice(ctx->device));
    freeInstruments(ctx);
    std::vector<InstrDev> v(num_instruments);
    for (int i = 0; i < num_instruments; ++i)
    {
        const skgpu_instrument& s = instruments[i];
        InstrDev& d = v[i];
        if (s.kind != SKGPU_INSTR_FRAME && s.kind != SKGPU_INSTR_SED) return fail(ctx, SKGPU_ERR_ARG, "instruments: bad kind");
        if (s.num_wavelength_bins < 1 || s.wlg_num_borders < 1 || s.wlg_offset < 0
            || s.wlg_offset + s.wlg_num_borders + 1 > wlg_len)
            return fail(ctx, SKGPU_ERR_ARG, "instruments: wavelength grid out of range");
        if (s.kind == SKGPU_INSTR_FRAME && (s.num_pixels_x < 1 || s.num_pixels_y < 1 || !(s.xp_size > 0) || !(s.yp_size > 0)))
            return fail(ctx, SKGPU_ERR_ARG, "instruments: bad frame geometry");
        for (int q = 0; q <= s.wlg_num_borders; ++q)
            if (wlg_ellv[s.wlg_offset + q] < -1 || wlg_ellv[s.wlg_offset + q] >= s.num_wavelength_bins)
                return fail(ctx, SKGPU_ERR_ARG, "instruments: bin map out of range");
        d.kind = s.kind;
        d.same = s.same_observer;
        d.stats = s.record_statistics;
        d.comps = s.record_components;
        d.npx = s.kind == SKGPU_INSTR_FRAME ? s.num_pixels_x : 1;
        d.npy = s.kind == SKGPU_INSTR_FRAME ? s.num_pixels_y : 1;
        d.nbins = s.num_wavelength_bins;
        d.woff = s.wlg_offset;
        d.wnb = s.wlg_num_borders;
        for (int a = 0; a < 3; ++a) d.kobs[a] = s.kobs[a];
        d.ct = s.cos_theta; d.st = s.sin_theta; d.cp = s.cos_phi; d.sp = s.sin_phi; d.co = s.cos_omega; d.so = s.sin_omega;
        d.xpmin = s.xp_min; d.xpsiz = s.xp_size; d.ypmin = s.yp_min; d.ypsiz = s.yp_size;
        d.ifu = d.sed = d.ifuComp = d.sedComp = d.ifuStats = d.sedStats = nullptr;
        d.levels = 0;
        d.zfac = 1.;
        d.apR2 = 0.;
        d.nband = 0;
        d.bandBeg = nullptr;
        d.bandLam = d.bandTr = d.bandW = nullptr;
        size_t n = static_cast<size_t>(d.nbins) * (d.kind == SKGPU_INSTR_FRAME ? static_cast<size_t>(d.npx) * d.npy : 1);
        auto alloc = [&](double** p, size_t cnt) -> int {
            CK(devAlloc(p, cnt));
            CK(cudaMemset(*p, 0, cnt * sizeof(double)));
            ctx->instrBufs.push_back(*p);
            ctx->instrBufLens.push_back(cnt);
            return SKGPU_OK;
        };
        int rc;
        double** total = d.kind == SKGPU_INSTR_FRAME ? &d.ifu : &d.sed;
        double** comp = d.kind == SKGPU_INSTR_FRAME ? &d.ifuComp : &d.sedComp;
        double** stats = d.kind == SKGPU_INSTR_FRAME ? &d.ifuStats : &d.sedStats;
        if ((rc = alloc(total, n))) return rc;
        if (d.comps && (rc = alloc(comp, 3 * n))) return rc;
        if (d.stats && (rc = alloc(stats, 5 * n))) return rc;
    }
    CK(devUpload(&ctx->instr, v.data(), v.size()));
    CK(devUpload(&ctx->wlgB, wlg_borders, wlg_len));
    CK(devUpload<int>(&ctx->wlgEll, wlg_ellv, wlg_len));
    ctx->instrHost = v;
    return SKGPU_OK;
}

int skgpu_set_instrument_scattering_levels(skgpu_ctx* ctx, int32_t instrument, int32_t levels)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (instrument < 0 || instrument >= static_cast<int>(ctx->instrHost.size())) return fail(ctx, SKGPU_ERR_ARG, "levels: bad instrument index");
    InstrDev& d = ctx->instrHost[instrument];
    if (!d.comps) return fail(ctx, SKGPU_ERR_STATE, "levels: instrument does not record components");
    if (levels < 0 || levels > 1000) return fail(ctx, SKGPU_ERR_ARG, "levels: out of range [0, 1000]");
    CK(cudaSetDevice(ctx->device));
    double*& comp = d.kind == SKGPU_INSTR_FRAME ? d.ifuComp : d.sedComp;
    size_t n = static_cast<size_t>(d.nbins) * d.npx * d.npy;
    size_t cnt = static_cast<size_t>(3 + levels) * n;
    double* p = nullptr;
    CK(devAlloc(&p, cnt));
    CK(cudaMemset(p, 0, cnt * sizeof(double)));
    for (size_t b = 0; b < ctx->instrBufs.size(); ++b)
        if (ctx->instrBufs[b] == comp)
        {
            cudaFree(comp);
            ctx->instrBufs[b] = p;
            ctx->instrBufLens[b] = cnt;
        }
    comp = p;
    d.levels = levels;
    CK(cudaMemcpy(ctx->instr + instrument, &d, sizeof(InstrDev), cudaMemcpyHostToDevice));
    return SKGPU_OK;
}

int skgpu_set_instrument_observer(skgpu_ctx* ctx, int32_t instrument, double redshift, double aperture_radius)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (instrument < 0 || instrument >= static_cast<int>(ctx->instrHost.size())) return fail(ctx, SKGPU_ERR_ARG, "observer: bad instrument index");
    if (!(redshift >= 0.) || !std::isfinite(redshift)) return fail(ctx, SKGPU_ERR_ARG, "observer: redshift must be finite and >= 0");
    if (!(aperture_radius >= 0.) || !std::isfinite(aperture_radius)) return fail(ctx, SKGPU_ERR_ARG, "observer: bad aperture radius");
    InstrDev& d = ctx->instrHost[instrument];
    if (aperture_radius > 0. && d.kind != SKGPU_INSTR_SED) return fail(ctx, SKGPU_ERR_ARG, "observer: apertures belong to SED instruments");
    CK(cudaSetDevice(ctx->device));
    d.zfac = 1. + redshift;
    d.apR2 = aperture_radius * aperture_radius;
    CK(cudaMemcpy(ctx->instr + instrument, &d, sizeof(InstrDev), cudaMemcpyHostToDevice));
    return SKGPU_OK;
}

int skgpu_set_instrument_bands(skgpu_ctx* ctx, int32_t instrument, int32_t num_bands, const int32_t* band_sizes,
                               const double* lambda, const double* transmission, const double* width)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (instrument < 0 || instrument >= static_cast<int>(ctx->instrHost.size())) return fail(ctx, SKGPU_ERR_ARG, "bands: bad instrument index");
    InstrDev& d = ctx->instrHost[instrument];
    if (num_bands != d.nbins) return fail(ctx, SKGPU_ERR_ARG, "bands: count differs from the instrument's wavelength bins");
    if (!band_sizes || !lambda || !transmission || !width) return fail(ctx, SKGPU_ERR_ARG, "bands: missing tables");
    std::vector<int> beg(static_cast<size_t>(num_bands) + 1, 0);
    for (int b = 0; b < num_bands; ++b)
    {
        if (band_sizes[b] < 2) return fail(ctx, SKGPU_ERR_ARG, "bands: fewer than 2 table points");
        if (!(std::isfinite(width[b]) && width[b] > 0)) return fail(ctx, SKGPU_ERR_ARG, "bands: bad effective width");
        beg[b + 1] = beg[b] + band_sizes[b];
        const double* lv = lambda + beg[b];
        for (int k = 0; k < band_sizes[b]; ++k)
        {
            if (!std::isfinite(lv[k]) || !std::isfinite(transmission[beg[b] + k]))
                return fail(ctx, SKGPU_ERR_ARG, "bands: non-finite table value");
            if (k > 0 && lv[k] < lv[k - 1]) return fail(ctx, SKGPU_ERR_ARG, "bands: wavelengths not increasing");
        }
        if (!(lv[0] < lv[band_sizes[b] - 1])) return fail(ctx, SKGPU_ERR_ARG, "bands: empty wavelength range");
    }
    CK(cudaSetDevice(ctx->device));
    size_t tot = static_cast<size_t>(beg[num_bands]);
    int* dBeg = nullptr;
    double *dLam = nullptr, *dTr = nullptr, *dW = nullptr;
    CK(devUpload<int>(&dBeg, beg.data(), beg.size()));
    ctx->instrAux.push_back(dBeg);
    CK(devUpload(&dLam, lambda, tot));
    ctx->instrAux.push_back(dLam);
    CK(devUpload(&dTr, transmission, tot));
    ctx->instrAux.push_back(dTr);
    CK(devUpload(&dW, width, static_cast<size_t>(num_bands)));
    ctx->instrAux.push_back(dW);
    d.nband = num_bands;
    d.bandBeg = dBeg;
    d.bandLam = dLam;
    d.bandTr = dTr;
    d.bandW = dW;
    CK(cudaMemcpy(ctx->instr + instrument, &d, sizeof(InstrDev), cudaMemcpyHostToDevice));
    return SKGPU_OK;
}

int skgpu_set_options(skgpu_ctx* ctx, const skgpu_options* options)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!options) return fail(ctx, SKGPU_ERR_ARG, "options: null");
    if (!(options->min_weight_reduction > 0)) return fail(ctx, SKGPU_ERR_ARG, "options: min_weight_reduction must be > 0");
    if (options->path_length_bias < 0 || options->path_length_bias >= 1) return fail(ctx, SKGPU_ERR_ARG, "options: path_length_bias must be in [0,1)");
    if (options->precision != SKGPU_PREC_FP64_EXACT && options->precision != SKGPU_PREC_FP32)
        return fail(ctx, SKGPU_ERR_ARG, "options: bad precision");
    ctx->opt = *options;
    ctx->hasOptions = true;
    return SKGPU_OK;
}

// ------------------------------------------------------------------------------------------------
// run and tallies
// ------------------------------------------------------------------------------------------------

// scene record of the kernels from the context's uploads
static Scene sceneOf(const skgpu_ctx* ctx)
{
    Scene p{};
    p.g = ctx->g;
    p.dens = ctx->dens;
    p.mixLb = ctx->mixLb; p.mixExt = ctx->mixExt; p.mixSca = ctx->mixSca; p.mixG = ctx->mixG; p.nmix = ctx->nmix;
    p.nsrc = static_cast<int>(ctx->srcHost.size());
    p.src = ctx->src;
    p.tabL = ctx->tabL; p.tabA = ctx->tabA; p.tabB = ctx->tabB; p.radR = ctx->radR; p.radP = ctx->radP;
    p.ninstr = static_cast<int>(ctx->instrHost.size());
    p.instr = ctx->instr;
    p.wlgB = ctx->wlgB; p.wlgEll = ctx->wlgEll;
    p.rfOn = ctx->opt.store_radiation_field ? 1 : 0;
    p.nrf = ctx->nrf; p.rfNb = ctx->rfNb; p.rfB = ctx->rfB; p.rfEll = ctx->rfEll; p.rf = ctx->rf;
    p.forced = ctx->opt.force_scattering ? 1 : 0;
    p.minScatt = ctx->opt.min_scatt_events;
    p.peel = ctx->opt.peel_off ? 1 : 0;
    p.explicitAbs = ctx->opt.explicit_absorption ? 1 : 0;
    p.minWeightRed = ctx->opt.min_weight_reduction;
    p.pathLengthBias = ctx->opt.path_length_bias;
    p.seed = ctx->opt.seed;
    p.guideMode = 0;
    if (const GuideState* gs = ctx->guide)
    {
        p.guideMode = gs->mode;
        p.guideTarget = gs->target;
        p.guideAlpha = gs->alpha;
        p.guideRecFrac = gs->recordFraction;
        p.guideRec = gs->records;
        p.guideRecCount = gs->recCount;
        p.guideRecCap = gs->recCapacity;
        p.guideImportance = gs->importance;
        p.guideBlob = gs->blob;
        p.guideErr = gs->errFlag;
    }
    return p;
}

static int checkRunnable(skgpu_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets)
{
    if (!ctx->hasGrid) return fail(ctx, SKGPU_ERR_STATE, "run: no grid uploaded");
    if (!ctx->dens || ctx->numCells != ctx->g.numCells) return fail(ctx, SKGPU_ERR_STATE, "run: medium does not match the grid");
    if (!ctx->nmix) return fail(ctx, SKGPU_ERR_STATE, "run: no dust mix uploaded");
    if (ctx->srcHost.empty()) return fail(ctx, SKGPU_ERR_STATE, "run: no sources uploaded");
    if (ctx->opt.store_radiation_field && !ctx->nrf) return fail(ctx, SKGPU_ERR_STATE, "run: radiation field requested without RF grid");
    if (total_packets == 0 || first + count > total_packets) return fail(ctx, SKGPU_ERR_ARG, "run: history range outside the segment");
    return SKGPU_OK;
}

static void waveShape(const skgpu_ctx* ctx, int& groups, int& anyStats)
{
    anyStats = 0;
    groups = 0;
    for (const InstrDev& d : ctx->instrHost)
    {
        anyStats |= d.stats;
        groups += d.same ? 0 : 1;
    }
    groups = std::max(groups, 1);
}

// Chooses the launch order of a run: wavelength order when it is on and the range is larger than
// the pool (otherwise every history is in flight at once), index order otherwise.
static int prepareOrder(skgpu_ctx* ctx, Wave& w)
{
    w.order = nullptr;
    if (!ctx->historyOrder || w.count <= static_cast<unsigned long long>(w.P) || w.count >= (1ULL << 32)) return SKGPU_OK;
    if (ctx->orderCap < w.count)
    {
        cudaFree(ctx->orderKeys);
        cudaFree(ctx->orderIdx);
        ctx->orderKeys = nullptr;
        ctx->orderIdx = nullptr;
        ctx->orderCap = 0;
        CK(devAlloc(&ctx->orderKeys, w.count));
        CK(devAlloc(&ctx->orderIdx, w.count));
        ctx->orderCap = w.count;
    }
    if (!ctx->orderCounts) CK(devAlloc(&ctx->orderCounts, 2 * static_cast<size_t>(ORDER_BUCKETS)));
    w.order = ctx->orderIdx;
    return SKGPU_OK;
}

// FluxRecorder::recordContributions for the histories that spilled: their contributions (all in the
// spill log once they ended) are summed per (history, key) on the host, written back over the log,
// and a kernel adds w^0..w^4 of each sum into the statistics tallies. Allocates no device memory.
static int groupSpilledStats(skgpu_ctx* ctx, const Wave& w, unsigned long long n)
{
    std::vector<StatSpill> log(n);
    CK(cudaMemcpy(log.data(), w.pk.spill, n * sizeof(StatSpill), cudaMemcpyDeviceToHost));
    std::stable_sort(log.begin(), log.end(), [](const StatSpill& a, const StatSpill& b) {
        if (a.scene != b.scene) return a.scene < b.scene;
        if (a.hist != b.hist) return a.hist < b.hist;
        return a.key < b.key;
    });
    std::vector<StatSpill> groups;
    for (size_t i = 0; i < log.size();)
    {
        StatSpill g = log[i];
        size_t j = i + 1;
        for (; j < log.size() && log[j].scene == g.scene && log[j].hist == g.hist && log[j].key == g.key; ++j) g.w += log[j].w;
        groups.push_back(g);
        i = j;
    }
    CK(cudaMemcpy(w.pk.spill, groups.data(), groups.size() * sizeof(StatSpill), cudaMemcpyHostToDevice));
    CK(groupStats(w, w.pk.spill, groups.size(), ctx->numSMs, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SKGPU_OK;
}

// runs the wavefront on prepared buffers and collects the counters and status of the run
static int runAndCollect(skgpu_ctx* ctx, const Wave& w, bool useGraph, bool timed)
{
    int prec = ctx->opt.precision;
    long long passes = 0;
    StageTimer* timer = timed && ctx->timer.level ? &ctx->timer : nullptr;
    for (int i = 0; i < StageTimer::kStages; ++i)
    {
        ctx->timer.ms[i] = 0.;
        ctx->timer.launches[i] = 0;
    }
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (w.order)
    {
        cudaError_t eo = orderHistories(w, ctx->orderKeys, ctx->orderCounts, ctx->orderCounts + ORDER_BUCKETS,
                                        ctx->orderIdx, ctx->numSMs, ctx->stream);
        if (eo != cudaSuccess) return fail(ctx, SKGPU_ERR_CUDA, std::string("run: ordering: ") + cudaGetErrorString(eo));
    }
    cudaError_t e = prec == SKGPU_PREC_FP64_EXACT
                        ? runWaveFP64(ctx->g.kind, w, ctx->numSMs, ctx->stream, ctx->doneHost, &passes, MAX_PASSES, useGraph, timer,
                                      &ctx->graphCache)
                        : runWaveFP32(ctx->g.kind, w, ctx->numSMs, ctx->stream, ctx->doneHost, &passes, MAX_PASSES, useGraph, timer,
                                      &ctx->graphCache);
    if (e == cudaErrorNotSupported) return fail(ctx, SKGPU_ERR_UNSUPPORTED, "run: no FP32 walker for this grid kind");
    if (e == cudaErrorLaunchTimeout) return fail(ctx, SKGPU_ERR_TIMEOUT, "run: pass limit reached before all histories finished");
    if (e != cudaSuccess) return fail(ctx, SKGPU_ERR_CUDA, std::string("run: ") + cudaGetErrorString(e));
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->lastMs = ms;
    Control ctl;
    CK(cudaMemcpy(&ctl, w.ctl, sizeof ctl, cudaMemcpyDeviceToHost));
    int errFlag = ctl.err;
    ctx->lastCounters.histories = ctl.counters[0];
    ctx->lastCounters.crossings = ctl.counters[1];
    ctx->lastCounters.scatterings = ctl.counters[2];
    ctx->lastCounters.peel_detections = ctl.counters[3];
    ctx->lastCounters.rf_stores = ctl.counters[4];
    ctx->lastCounters.stats_overflows = ctl.counters[5];
    ctx->lastCounters.stats_spilled = ctl.counters[6];
    const int perPass = (w.sc.guideMode == 2 ? 8 : 7) + (useGraph && ctx->graphCache.lastSplit ? 1 : 0);
    ctx->lastCounters.kernel_launches = static_cast<uint64_t>(passes) * perPass + 1 + (w.order ? 3 : 0);
    ctx->lastPasses = passes;
    ctx->lastGuideWeightSum = ctl.guideWeightSum;
    ctx->lastGuideEvents = ctl.guideEvents;
    if (w.count > 0 && ctl.done != w.count) return fail(ctx, SKGPU_ERR_DEVICE, "run: not every history finished");
    if (errFlag & 64)
        return fail(ctx, SKGPU_ERR_DEVICE, "run: the per-history statistics spill log is full ("
                                               + std::to_string(ctl.counters[5]) + " contributions lost)");
    if (ctl.spillN > 0)
    {
        int rc = groupSpilledStats(ctx, w, ctl.spillN);
        if (rc) return rc;
    }
    if (errFlag & 4) return fail(ctx, SKGPU_ERR_TIMEOUT, "run: a traversal exceeded its segment guard");
    if (errFlag & 8) return fail(ctx, SKGPU_ERR_TIMEOUT, "run: a history exceeded the scattering-event guard");
    if (errFlag & 16) return fail(ctx, SKGPU_ERR_TIMEOUT, "run: a tensor-core wait of the guided-scattering stage gave up");
    if (errFlag & 32) return fail(ctx, SKGPU_ERR_DEVICE, "run: non-finite guided-scattering weight");
    if (errFlag) return fail(ctx, SKGPU_ERR_DEVICE, "run: interaction point outside the grid (device check)");
    return SKGPU_OK;
}

// allocates the radiation-field tally for the current medium and RF grid if it does not exist yet
static int ensureRadiationField(skgpu_ctx* ctx)
{
    if (!ctx->opt.store_radiation_field || !ctx->nrf || !ctx->numCells) return SKGPU_OK;
    size_t len = static_cast<size_t>(ctx->numCells) * ctx->nrf;
    if (ctx->rfLen == len) return SKGPU_OK;
    devFree(ctx->rf);
    devFree(ctx->rfT);
    CK(devAlloc(&ctx->rf, len));
    CK(cudaMemset(ctx->rf, 0, len * sizeof(double)));
    ctx->rfLen = len;
    return SKGPU_OK;
}

int skgpu_run_primary(skgpu_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets)
{
    if (!ctx) return SKGPU_ERR_ARG;
    int rc = checkRunnable(ctx, first, count, total_packets);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    if ((rc = ensureRadiationField(ctx))) return rc;
    // packet pool and task queues, sized for up to POOL_DEFAULT histories in flight (or the launch shape's pool)
    int groups, anyStats;
    waveShape(ctx, groups, anyStats);
    uint64_t poolMax = ctx->shapePool > 0 ? static_cast<uint64_t>(ctx->shapePool) : POOL_DEFAULT;
    int P = static_cast<int>(std::min<uint64_t>(std::max<uint64_t>(count, 1), poolMax));
    if ((rc = ensureWaveBuffers(ctx, P, groups, anyStats))) return rc;
    Wave w = ctx->wave;
    w.sc = sceneOf(ctx);
    w.traceBlocksPerSM = ctx->shapeTraceBlocks;
    w.refillMin = ctx->shapeRefill;
    w.rfAgg = rfWarpAggregation();
    w.shadeBlocksPerSM = ctx->shapeShadeBlocks;
    w.P = P;
    w.first = first;
    w.count = count;
    w.anyStats = anyStats;
    w.statCap = STATS_CAP;
    if ((rc = prepareOrder(ctx, w))) return rc;
    return runAndCollect(ctx, w, true, true);
}

// ------------------------------------------------------------------------------------------------
// secondary (dust) emission
// ------------------------------------------------------------------------------------------------

int skgpu_upload_dust_emission(skgpu_ctx* ctx, int32_t num_rf, const double* rf_sigma_abs, const double* rf_width,
                               const double* rf_cmb, const double* rf_sigma_abs_lum, int32_t num_T, const double* T,
                               const double* planck_abs, int32_t num_em, const double* em_lambda,
                               const double* em_sigma_abs, const double* em_range, int32_t num_cells,
                               const double* cell_volume)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (num_rf < 1 || num_T < 2 || num_em < 2 || num_cells < 1 || !rf_sigma_abs || !rf_width || !rf_cmb
        || !rf_sigma_abs_lum || !T || !planck_abs || !em_lambda || !em_sigma_abs || !em_range || !cell_volume)
        return fail(ctx, SKGPU_ERR_ARG, "dust emission: missing tables");
    if (!(em_range[0] > 0. && em_range[1] > em_range[0]))
        return fail(ctx, SKGPU_ERR_ARG, "dust emission: empty wavelength range");
    for (int i = 1; i < num_em; ++i)
        if (!(em_lambda[i] > em_lambda[i - 1])) return fail(ctx, SKGPU_ERR_ARG, "dust emission: wavelengths not ascending");
    if (!finiteAll(cell_volume, num_cells)) return fail(ctx, SKGPU_ERR_ARG, "dust emission: non-finite cell volume");
    CK(cudaSetDevice(ctx->device));
    freeBufs(ctx->deBufs);
    ctx->de = DustEmissionDev{};
    int rc = 0;
    DustEmissionDev& d = ctx->de;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.rfSig, rf_sigma_abs, num_rf))) return rc;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.rfW, rf_width, num_rf))) return rc;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.rfCmb, rf_cmb, num_rf))) return rc;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.rfSigL, rf_sigma_abs_lum, num_rf))) return rc;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.T, T, num_T))) return rc;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.planck, planck_abs, num_T))) return rc;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.emL, em_lambda, num_em))) return rc;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.emSig, em_sigma_abs, num_em))) return rc;
    if ((rc = secUpload(ctx, ctx->deBufs, &d.vol, cell_volume, num_cells))) return rc;
    d.nrf = num_rf;
    d.nT = num_T;
    d.nem = num_em;
    ctx->deEmLHost.assign(em_lambda, em_lambda + num_em);
    ctx->deEmRange[0] = em_range[0];
    ctx->deEmRange[1] = em_range[1];
    ctx->deCells = num_cells;
    ctx->secPackets = 0;
    return SKGPU_OK;
}

int skgpu_upload_radiation_field(skgpu_ctx* ctx, const double* rf)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!rf) return fail(ctx, SKGPU_ERR_ARG, "radiation field: missing array");
    if (!ctx->nrf || !ctx->numCells) return fail(ctx, SKGPU_ERR_STATE, "radiation field: no medium or RF grid uploaded");
    if (!finiteAll(rf, static_cast<size_t>(ctx->numCells) * ctx->nrf))
        return fail(ctx, SKGPU_ERR_ARG, "radiation field: non-finite value");
    CK(cudaSetDevice(ctx->device));
    size_t len = static_cast<size_t>(ctx->numCells) * ctx->nrf;
    if (ctx->rfLen != len)
    {
        devFree(ctx->rf);
        devFree(ctx->rfT);
        CK(devAlloc(&ctx->rf, len));
        ctx->rfLen = len;
    }
    // the caller's layout is cell-major (m * nbins + ell), the device tally wavelength-major
    std::vector<double> t(len);
    const size_t cells = ctx->numCells, nb = ctx->nrf;
    for (size_t m = 0; m < cells; ++m)
        for (size_t e = 0; e < nb; ++e) t[e * cells + m] = rf[m * nb + e];
    CK(cudaMemcpy(ctx->rf, t.data(), len * sizeof(double), cudaMemcpyHostToDevice));
    return SKGPU_OK;
}

int skgpu_prepare_secondary(skgpu_ctx* ctx, const skgpu_secondary_options* opt, uint64_t total_packets,
                            double* luminosity)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!opt || total_packets == 0) return fail(ctx, SKGPU_ERR_ARG, "secondary: missing options or packets");
    if (!ctx->hasGrid || (ctx->g.kind != SKGPU_GRID_CARTESIAN && ctx->g.kind != SKGPU_GRID_OCTREE
                          && ctx->g.kind != SKGPU_GRID_ADAPTIVE_MESH && ctx->g.kind != SKGPU_GRID_TETRA
                          && (ctx->g.kind < SKGPU_GRID_SPHERE1D || ctx->g.kind > SKGPU_GRID_CYLINDER3D)
                          && !(ctx->g.kind == SKGPU_GRID_VORONOI && ctx->g.vBox)))
        return fail(ctx, SKGPU_ERR_UNSUPPORTED, "secondary: a Voronoi grid needs its cell boxes (skgpu_upload_voronoi_cell_boxes)");
    if (!ctx->dens || ctx->numCells != ctx->g.numCells) return fail(ctx, SKGPU_ERR_STATE, "secondary: medium does not match the grid");
    if (!ctx->de.nrf || ctx->deCells != ctx->numCells || ctx->de.nrf != ctx->nrf)
        return fail(ctx, SKGPU_ERR_STATE, "secondary: dust emission tables do not match the medium and RF grid");
    if (!ctx->rf || ctx->rfLen != static_cast<size_t>(ctx->numCells) * ctx->nrf)
        return fail(ctx, SKGPU_ERR_STATE, "secondary: no radiation field on the device");
    if (!(opt->spatial_bias >= 0. && opt->spatial_bias <= 1. && opt->source_bias >= 0. && opt->source_bias <= 1.
          && opt->wavelength_bias >= 0. && opt->wavelength_bias <= 1.))
        return fail(ctx, SKGPU_ERR_ARG, "secondary: bias fractions outside [0, 1]");
    if (opt->wavelength_bias > 0. && !(opt->bias_lambda_min > 0. && opt->bias_lambda_max > opt->bias_lambda_min))
        return fail(ctx, SKGPU_ERR_ARG, "secondary: empty wavelength-bias range");
    CK(cudaSetDevice(ctx->device));
    const int cells = ctx->numCells;

    // the spectrum axis of NR::cdf: the range ends with the emission-grid wavelengths between them
    const std::vector<double>& inx = ctx->deEmLHost;
    const double rmin = ctx->deEmRange[0], rmax = ctx->deEmRange[1];
    int minRight = static_cast<int>(std::upper_bound(inx.begin(), inx.end(), rmin) - inx.begin());
    int maxRight = static_cast<int>(std::lower_bound(inx.begin(), inx.end(), rmax) - inx.begin());
    int nb = 1 + maxRight - minRight;
    if (nb < 1) return fail(ctx, SKGPU_ERR_ARG, "secondary: emission range outside the emission grid");
    std::vector<double> xv(nb + 1);
    xv[0] = rmin;
    for (int j = minRight, i = 1; j < maxRight; ++j, ++i) xv[i] = inx[j];
    xv[nb] = rmax;
    const int npts = nb + 1;

    if (ctx->secCells != cells || ctx->secNpts != npts)
    {
        freeBufs(ctx->secBufs);
        ctx->secCells = ctx->secNpts = 0;
        int rc = 0;
        size_t rows = static_cast<size_t>(cells) * npts;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secL, cells))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secT, cells))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secPv, rows))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secCv, rows))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secXv, npts))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secLv, cells))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secWv, cells))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secIv, static_cast<size_t>(cells) + 1))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secCellNode, cells))) return rc;
        if ((rc = secAlloc(ctx, ctx->secBufs, &ctx->secDev, 1))) return rc;
        ctx->secCells = cells;
        ctx->secNpts = npts;
    }
    ctx->secPackets = 0;
    CK(cudaMemcpy(ctx->secXv, xv.data(), npts * sizeof(double), cudaMemcpyHostToDevice));
    CK(launchDustCells(ctx->de, ctx->dens, ctx->rf, cells, ctx->secXv, npts, minRight, maxRight, ctx->secL, ctx->secT,
                       ctx->secPv, ctx->secCv, ctx->stream));
    if (ctx->g.kind == SKGPU_GRID_OCTREE || ctx->g.kind == SKGPU_GRID_ADAPTIVE_MESH)
        CK(launchCellNodes(ctx->g.tCell, ctx->g.tNodes, ctx->secCellNode, ctx->stream));
    std::vector<double> Lv(cells);
    CK(cudaMemcpyAsync(Lv.data(), ctx->secL, cells * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));

    // DustSecondarySource::prepareLuminosities (DustSecondarySource.cpp:27-120) with the
    // AllCellsLibrary (every cell its own entry, launch order = cell order): the cell luminosities
    // normalised by their sum (valarray::sum, first to last)
    double L = Lv[0];
    for (int m = 1; m < cells; ++m) L += Lv[m];
    if (luminosity) *luminosity = L;
    ctx->secLuminosity = L;
    if (!(L > 0.)) return SKGPU_OK;  // nothing to launch (SecondarySourceSystem::prepareForLaunch fails)
    for (int m = 0; m < cells; ++m) Lv[m] /= L;
    // DustSecondarySource::preparePacketMap (DustSecondarySource.cpp:124-152): composite-biased
    // weights (1 - xi) Lv + xi / (number of emitting cells), and the first history index of every cell
    // from the cumulative weight rounded to the nearest index
    const double xi = opt->spatial_bias;
    std::vector<double> wv(cells), Wv(cells);
    for (int m = 0; m < cells; ++m) wv[m] = Lv[m] > 0 ? 1. : 0.;
    double ws = wv[0];
    for (int m = 1; m < cells; ++m) ws += wv[m];
    for (int m = 0; m < cells; ++m) wv[m] /= ws;
    for (int m = 0; m < cells; ++m) Wv[m] = (1 - xi) * Lv[m] + xi * wv[m];
    const uint64_t N = total_packets;
    std::vector<unsigned long long> Iv(static_cast<size_t>(cells) + 1);
    Iv[0] = 0;
    double W = 0.;
    for (int p = 1; p != cells; ++p)
    {
        W += Wv[p - 1];
        Iv[p] = std::min<uint64_t>(N, static_cast<uint64_t>(std::round(W * N)));
    }
    Iv[cells] = N;
    CK(cudaMemcpy(ctx->secLv, Lv.data(), cells * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->secWv, Wv.data(), cells * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->secIv, Iv.data(), Iv.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice));

    // SecondarySourceSystem::prepareForLaunch / launch (SecondarySourceSystem.cpp:62-118) with the
    // dust source alone (source weight 1): the source's launch weight Lv_s / Wv_s and the average
    // packet luminosity L / N
    const double xs = opt->source_bias;
    const double Lpp = L / static_cast<double>(N);
    const double Ws = (1 - xs) * 1. / 1. + xs * 1. / 1.;
    SecondaryDev sd{};
    sd.Iv = ctx->secIv;
    sd.Lv = ctx->secLv;
    sd.Wv = ctx->secWv;
    sd.xv = ctx->secXv;
    sd.pv = ctx->secPv;
    sd.Pv = ctx->secCv;
    sd.cellNode = ctx->secCellNode;
    sd.npts = npts;
    sd.numCells = cells;
    sd.Lpk = Lpp * (1. / Ws);
    sd.xi = opt->wavelength_bias;
    sd.bmin = opt->bias_lambda_min;
    sd.bmax = opt->bias_lambda_max;
    sd.logMin = opt->wavelength_bias > 0. ? std::log(sd.bmin) : 0.;
    sd.logWidth = opt->wavelength_bias > 0. ? std::log(sd.bmax) - std::log(sd.bmin) : 0.;
    CK(cudaMemcpy(ctx->secDev, &sd, sizeof sd, cudaMemcpyHostToDevice));
    ctx->secPackets = N;
    // the uploaded radiation field has served the cells' emission: the tally starts empty for a
    // segment that stores its own (MediumSystem::clearRadiationField(false) before it)
    if (ctx->rf) CK(cudaMemset(ctx->rf, 0, ctx->rfLen * sizeof(double)));
    return SKGPU_OK;
}

int skgpu_fetch_dust_emission(skgpu_ctx* ctx, double* luminosity, double* temperature, int32_t* num_points,
                              double* lambda, double* pdf, double* cdf)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!ctx->secCells || ctx->secCells != ctx->numCells) return fail(ctx, SKGPU_ERR_STATE, "fetch: no prepared dust emission");
    CK(cudaSetDevice(ctx->device));
    size_t cells = ctx->secCells, rows = cells * ctx->secNpts;
    if (num_points) *num_points = ctx->secNpts;
    if (luminosity) CK(cudaMemcpy(luminosity, ctx->secL, cells * sizeof(double), cudaMemcpyDeviceToHost));
    if (temperature) CK(cudaMemcpy(temperature, ctx->secT, cells * sizeof(double), cudaMemcpyDeviceToHost));
    if (lambda) CK(cudaMemcpy(lambda, ctx->secXv, ctx->secNpts * sizeof(double), cudaMemcpyDeviceToHost));
    if (pdf) CK(cudaMemcpy(pdf, ctx->secPv, rows * sizeof(double), cudaMemcpyDeviceToHost));
    if (cdf) CK(cudaMemcpy(cdf, ctx->secCv, rows * sizeof(double), cudaMemcpyDeviceToHost));
    return SKGPU_OK;
}

int skgpu_run_secondary(skgpu_ctx* ctx, uint64_t first, uint64_t count)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!ctx->secPackets || ctx->secCells != ctx->numCells)
        return fail(ctx, SKGPU_ERR_STATE, "secondary: no prepared segment (skgpu_prepare_secondary)");
    if (!ctx->hasOptions) return fail(ctx, SKGPU_ERR_STATE, "secondary: no options set");
    if (!ctx->nmix) return fail(ctx, SKGPU_ERR_STATE, "secondary: no dust mix uploaded");
    if (first + count > ctx->secPackets) return fail(ctx, SKGPU_ERR_ARG, "secondary: history range outside the segment");
    CK(cudaSetDevice(ctx->device));
    int groups, anyStats;
    waveShape(ctx, groups, anyStats);
    uint64_t poolMax = ctx->shapePool > 0 ? static_cast<uint64_t>(ctx->shapePool) : POOL_DEFAULT;
    int P = static_cast<int>(std::min<uint64_t>(std::max<uint64_t>(count, 1), poolMax));
    int rc = 0;
    if ((rc = ensureWaveBuffers(ctx, P, groups, anyStats))) return rc;
    Wave w = ctx->wave;
    w.sc = sceneOf(ctx);
    // the secondary source replaces the primary ones; with store_radiation_field the segment tallies
    // its own radiation field (SecondaryEmissionOptions::storeEmissionRadiationField, the secondary
    // iterations: MediumSystem::storeRadiationField(false, ...) into _rf2c); the histories draw from
    // streams of their own (a Philox key distinct from the primary segment's)
    if ((rc = ensureRadiationField(ctx))) return rc;
    w.sc.sec = ctx->secDev;
    w.sc.seed = ctx->opt.seed ^ SKGPU_SECONDARY_KEY;
    w.traceBlocksPerSM = ctx->shapeTraceBlocks;
    w.refillMin = ctx->shapeRefill;
    w.rfAgg = rfWarpAggregation();
    w.shadeBlocksPerSM = ctx->shapeShadeBlocks;
    w.P = P;
    w.first = first;
    w.count = count;
    w.anyStats = anyStats;
    w.statCap = STATS_CAP;
    w.order = nullptr;
    return runAndCollect(ctx, w, true, true);
}

// ------------------------------------------------------------------------------------------------
// launch probe: the source launch of the life cycle without the traversal
// ------------------------------------------------------------------------------------------------
static __global__ void __launch_bounds__(256) probeLaunchKernel(const __grid_constant__ Scene sc, unsigned long long first,
                                                                unsigned long long count, double total, double* out)
{
    for (unsigned long long t = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; t < count;
         t += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
    {
        unsigned long long hist = first + t;
        Rng rng;
        rng.start(sc.seed, hist);
        Launched o = launchPacket(sc, hist, rng);
        double* r = out + 8 * t;
        r[0] = o.lambda;
        r[1] = o.L * total;
        r[2] = o.x; r[3] = o.y; r[4] = o.z;
        r[5] = o.kx; r[6] = o.ky; r[7] = o.kz;
    }
}

int skgpu_probe_launch(skgpu_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets, double* out)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (ctx->srcHost.empty()) return fail(ctx, SKGPU_ERR_STATE, "probe_launch: no sources uploaded");
    if (total_packets == 0 || first + count > total_packets || (count && !out))
        return fail(ctx, SKGPU_ERR_ARG, "probe_launch: history range outside the segment");
    if (count == 0) return SKGPU_OK;
    CK(cudaSetDevice(ctx->device));
    double* dev = nullptr;
    CK(devAlloc(&dev, 8 * count));
    Scene sc = sceneOf(ctx);
    unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((count + 255) / 256, 8ull * ctx->numSMs));
    probeLaunchKernel<<<blocks, 256, 0, ctx->stream>>>(sc, first, count, static_cast<double>(total_packets), dev);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dev, 8 * count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dev);
    if (e != cudaSuccess) return fail(ctx, SKGPU_ERR_CUDA, std::string("probe_launch: ") + cudaGetErrorString(e));
    return SKGPU_OK;
}

// ------------------------------------------------------------------------------------------------
// run without allocations: the wavefront scratch comes from a file-scope device array
// ------------------------------------------------------------------------------------------------

// Scratch of skgpu_run_primary_noalloc: packet pool, task queues and control block of at most
// NOALLOC_SLOTS histories in flight, NOALLOC_GROUPS observer groups, with statistics buffers. Every
// GPU that loads this library holds it until the process exits.
static __device__ __align__(256) unsigned char g_noallocScratch[SKGPU_NOALLOC_SCRATCH_BYTES];

// entries of the statistics spill log within the static scratch
constexpr size_t NOALLOC_SPILL = size_t(1) << 16;

// lays the wavefront buffers for P slots out in a scratch area (base may be null: size only)
static size_t carveWave(Wave& w, unsigned char* base, int P, int groups, int stats)
{
    size_t off = 0;
    auto take = [&](auto** p, size_t count) {
        using T = std::remove_pointer_t<std::remove_reference_t<decltype(*p)>>;
        off = (off + 255) & ~static_cast<size_t>(255);
        *p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += std::max<size_t>(count, 1) * sizeof(T);
    };
    PacketPool& k = w.pk;
    take(&k.rec, P);
    take(&k.nstat, P);
    take(&k.freeSlots, P);
    size_t ns = stats ? static_cast<size_t>(P) * STATS_CAP_NOALLOC : 1;
    take(&k.skey, ns);
    take(&k.sw, ns);
    k.spillCap = stats ? NOALLOC_SPILL : 1;
    take(&k.spill, k.spillCap);
    for (int b = 0; b < 2; ++b)
        for (int kind = 0; kind < NUM_KINDS; ++kind)
        {
            TaskBuf& t = w.q[b][kind];
            t = TaskBuf{};
            if (kind == K_GUIDE) continue;  // guiding is not available without allocation
            size_t cap = kind == K_PEEL ? static_cast<size_t>(P) * groups : static_cast<size_t>(P);
            take(&t.slot, cap);
            take(&t.par, cap);
            if (kind == K_PEEL)
            {
                take(&t.info, cap);
                take(&t.x, cap);
                take(&t.y, cap);
                take(&t.z, cap);
            }
            if (kind == K_PEEL || kind == K_PROP1)
                take(&t.tau, cap);
            else
            {
                take(&t.m, cap);
                take(&t.s, cap);
                take(&t.found, cap);
            }
        }
    take(&w.ctl, 1);
    return off;
}

int skgpu_run_primary_noalloc(skgpu_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets)
{
    if (!ctx) return SKGPU_ERR_ARG;
    int rc = checkRunnable(ctx, first, count, total_packets);
    if (rc) return rc;
    int groups, anyStats;
    waveShape(ctx, groups, anyStats);
    if (ctx->guide && ctx->guide->mode != 0)
        return fail(ctx, SKGPU_ERR_STATE, "run_noalloc: learned path guiding is not available without allocation");
    if (groups > SKGPU_NOALLOC_MAX_GROUPS)
        return fail(ctx, SKGPU_ERR_ARG, "run_noalloc: more than " + std::to_string(SKGPU_NOALLOC_MAX_GROUPS)
                                            + " observer groups exceed the static scratch");
    if (ctx->opt.store_radiation_field && ctx->rfLen != static_cast<size_t>(ctx->numCells) * ctx->nrf)
        return fail(ctx, SKGPU_ERR_STATE, "run_noalloc: the radiation-field tally is not allocated yet "
                                          "(call skgpu_clear_tallies after skgpu_set_options)");
    Wave probe{};
    if (carveWave(probe, nullptr, SKGPU_NOALLOC_MAX_SLOTS, groups, anyStats) > sizeof(g_noallocScratch))
        return fail(ctx, SKGPU_ERR_ARG, "run_noalloc: scene needs more scratch than the static array holds");
    CK(cudaSetDevice(ctx->device));
    // the host-side name of the array is not a device address: ask the runtime, with this device
    // current, on every call (the lookup allocates nothing, and a cached address would go stale after
    // a device reset or under another context on the same device)
    void* addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noallocScratch);
    if (e != cudaSuccess || !addr)
        return fail(ctx, SKGPU_ERR_CUDA, std::string("run_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    Wave w{};
    carveWave(w, static_cast<unsigned char*>(addr), SKGPU_NOALLOC_MAX_SLOTS, groups, anyStats);
    w.sc = sceneOf(ctx);
    w.traceBlocksPerSM = ctx->shapeTraceBlocks;
    w.refillMin = ctx->shapeRefill;
    w.rfAgg = rfWarpAggregation();
    w.shadeBlocksPerSM = ctx->shapeShadeBlocks;
    w.P = static_cast<int>(std::min<uint64_t>(std::max<uint64_t>(count, 1), SKGPU_NOALLOC_MAX_SLOTS));
    w.first = first;
    w.count = count;
    w.anyStats = anyStats;
    w.statCap = STATS_CAP_NOALLOC;
    return runAndCollect(ctx, w, false, false);
}

// host[i] += src[i] for i < n, split over the host cores for large n
static void parallelAdd(double* host, const double* src, size_t n)
{
    const size_t perThread = size_t(1) << 18;
    size_t hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
    size_t T = std::min(hw, (n + perThread - 1) / perThread);
    if (T <= 1)
    {
        for (size_t i = 0; i < n; ++i) host[i] += src[i];
        return;
    }
    std::vector<std::thread> pool;
    size_t per = (n + T - 1) / T;
    for (size_t t = 0; t < T; ++t)
        pool.emplace_back([=] {
            size_t a = t * per, b = std::min(n, a + per);
            for (size_t i = a; i < b; ++i) host[i] += src[i];
        });
    for (std::thread& th : pool) th.join();
}

// Adds n doubles of device memory into a host array: chunked copies into two pinned buffers, the
// copy of chunk c+1 in flight while the host cores add chunk c.
static int addInto(skgpu_ctx* ctx, const double* dev, size_t n, double* host)
{
    if (!host || !dev || n == 0) return SKGPU_OK;
    const size_t chunk = size_t(8) << 20;  // doubles per staging buffer (64 MB)
    for (int i = 0; i < 2; ++i)
    {
        if (!ctx->pin[i]) CK(cudaMallocHost(reinterpret_cast<void**>(&ctx->pin[i]), chunk * sizeof(double)));
        if (!ctx->pinEv[i]) CK(cudaEventCreateWithFlags(&ctx->pinEv[i], cudaEventDisableTiming));
    }
    size_t chunks = (n + chunk - 1) / chunk;
    auto issue = [&](size_t c) {
        size_t a = c * chunk, len = std::min(chunk, n - a);
        cudaError_t e = cudaMemcpyAsync(ctx->pin[c & 1], dev + a, len * sizeof(double), cudaMemcpyDeviceToHost,
                                        ctx->stream);
        return e == cudaSuccess ? cudaEventRecord(ctx->pinEv[c & 1], ctx->stream) : e;
    };
    CK(issue(0));
    for (size_t c = 0; c < chunks; ++c)
    {
        // buffer (c+1)&1 held chunk c-1, whose add finished in the previous iteration
        if (c + 1 < chunks) CK(issue(c + 1));
        CK(cudaEventSynchronize(ctx->pinEv[c & 1]));
        size_t a = c * chunk;
        parallelAdd(host + a, ctx->pin[c & 1], std::min(chunk, n - a));
    }
    return SKGPU_OK;
}

int skgpu_fetch_instrument(skgpu_ctx* ctx, int32_t instrument, double* ifu, double* sed, double* ifu_stats,
                           double* sed_stats)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (instrument < 0 || instrument >= static_cast<int>(ctx->instrHost.size())) return fail(ctx, SKGPU_ERR_ARG, "fetch: bad instrument index");
    CK(cudaSetDevice(ctx->device));
    const InstrDev& d = ctx->instrHost[instrument];
    size_t n = static_cast<size_t>(d.nbins) * d.npx * d.npy;
    int rc;
    if (d.kind == SKGPU_INSTR_FRAME)
    {
        if ((rc = addInto(ctx, d.ifu, n, ifu))) return rc;
        if (d.stats && (rc = addInto(ctx, d.ifuStats, 5 * n, ifu_stats))) return rc;
    }
    else
    {
        if ((rc = addInto(ctx, d.sed, n, sed))) return rc;
        if (d.stats && (rc = addInto(ctx, d.sedStats, 5 * n, sed_stats))) return rc;
    }
    return SKGPU_OK;
}

int skgpu_fetch_instrument_components(skgpu_ctx* ctx, int32_t instrument, double* ifu3, double* sed3)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (instrument < 0 || instrument >= static_cast<int>(ctx->instrHost.size())) return fail(ctx, SKGPU_ERR_ARG, "fetch: bad instrument index");
    const InstrDev& d = ctx->instrHost[instrument];
    if (!d.comps) return fail(ctx, SKGPU_ERR_STATE, "fetch: instrument does not record components");
    CK(cudaSetDevice(ctx->device));
    size_t n = static_cast<size_t>(d.nbins) * d.npx * d.npy;
    return d.kind == SKGPU_INSTR_FRAME ? addInto(ctx, d.ifuComp, 3 * n, ifu3) : addInto(ctx, d.sedComp, 3 * n, sed3);
}

// values[i] *= factors[(i % n) / npix] over `planes` planes of n = nbins * npix entries
static __global__ void calibrateKernel(double* __restrict__ values, size_t total, size_t n, size_t npix,
                                       const double* __restrict__ factors)
{
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        values[i] *= factors[(i % n) / npix];
}

int skgpu_calibrate_instrument(skgpu_ctx* ctx, int32_t instrument, const double* factors)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (instrument < 0 || instrument >= static_cast<int>(ctx->instrHost.size())) return fail(ctx, SKGPU_ERR_ARG, "calibrate: bad instrument index");
    if (!factors) return fail(ctx, SKGPU_ERR_ARG, "calibrate: missing factors");
    const InstrDev& d = ctx->instrHost[instrument];
    if (!finiteAll(factors, static_cast<size_t>(d.nbins))) return fail(ctx, SKGPU_ERR_ARG, "calibrate: non-finite factor");
    CK(cudaSetDevice(ctx->device));
    size_t npix = static_cast<size_t>(d.npx) * d.npy, n = npix * d.nbins;
    double* f = nullptr;
    CK(devUpload(&f, factors, static_cast<size_t>(d.nbins)));
    int blocks = 0;
    cudaError_t e = cudaDeviceGetAttribute(&blocks, cudaDevAttrMultiProcessorCount, ctx->device);
    if (e == cudaSuccess)
    {
        blocks *= 4;
        double* total = d.kind == SKGPU_INSTR_FRAME ? d.ifu : d.sed;
        double* comp = d.kind == SKGPU_INSTR_FRAME ? d.ifuComp : d.sedComp;
        calibrateKernel<<<blocks, 256, 0, ctx->stream>>>(total, n, n, npix, f);
        if (comp) calibrateKernel<<<blocks, 256, 0, ctx->stream>>>(comp, (3 + d.levels) * n, n, npix, f);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    cudaFree(f);
    CK(e);
    return SKGPU_OK;
}

int skgpu_fetch_instrument_levels(skgpu_ctx* ctx, int32_t instrument, double* ifu_levels, double* sed_levels)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (instrument < 0 || instrument >= static_cast<int>(ctx->instrHost.size())) return fail(ctx, SKGPU_ERR_ARG, "fetch: bad instrument index");
    const InstrDev& d = ctx->instrHost[instrument];
    if (!d.comps || d.levels < 1) return fail(ctx, SKGPU_ERR_STATE, "fetch: instrument records no scattering levels");
    CK(cudaSetDevice(ctx->device));
    size_t n = static_cast<size_t>(d.nbins) * d.npx * d.npy;
    size_t lv = static_cast<size_t>(d.levels) * n;
    return d.kind == SKGPU_INSTR_FRAME ? addInto(ctx, d.ifuComp + 3 * n, lv, ifu_levels)
                                       : addInto(ctx, d.sedComp + 3 * n, lv, sed_levels);
}

// out[m * nbins + ell] = in[ell * cells + m], through 32 x 32 shared-memory tiles (both sides coalesced)
static __global__ void rfTransposeKernel(const double* __restrict__ in, double* __restrict__ out, int cells, int nbins)
{
    __shared__ double tile[32][33];
    int m0 = blockIdx.x * 32, e0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y)
    {
        int e = e0 + j, m = m0 + threadIdx.x;
        if (e < nbins && m < cells) tile[j][threadIdx.x] = in[static_cast<size_t>(e) * cells + m];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y)
    {
        int m = m0 + j, e = e0 + threadIdx.x;
        if (e < nbins && m < cells) out[static_cast<size_t>(m) * nbins + e] = tile[threadIdx.x][j];
    }
}

int skgpu_fetch_radiation_field(skgpu_ctx* ctx, double* rf)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!ctx->rf) return fail(ctx, SKGPU_ERR_STATE, "fetch: no radiation field recorded");
    CK(cudaSetDevice(ctx->device));
    if (!rf) return SKGPU_OK;
    // the device tally is wavelength-major (ell * cells + m); the caller's layout is cell-major
    int cells = static_cast<int>(ctx->rfLen / ctx->nrf), nbins = ctx->nrf;
    if (!ctx->rfT) CK(devAlloc(&ctx->rfT, ctx->rfLen));
    dim3 grid((cells + 31) / 32, (nbins + 31) / 32);
    rfTransposeKernel<<<grid, dim3(32, 8), 0, ctx->stream>>>(ctx->rf, ctx->rfT, cells, nbins);
    CK(cudaGetLastError());
    return addInto(ctx, ctx->rfT, ctx->rfLen, rf);
}

int skgpu_tally_buffers(skgpu_ctx* ctx, int32_t max_buffers, void** ptrs, uint64_t* lengths, int32_t* num_buffers)
{
    if (!ctx || !num_buffers) return SKGPU_ERR_ARG;
    int n = static_cast<int>(ctx->instrBufs.size()) + (ctx->rf ? 1 : 0);
    *num_buffers = n;
    if (max_buffers < n) return ptrs ? fail(ctx, SKGPU_ERR_ARG, "tally_buffers: array too small") : SKGPU_OK;
    if (!ptrs || !lengths) return fail(ctx, SKGPU_ERR_ARG, "tally_buffers: null output arrays");
    size_t i = 0;
    for (; i < ctx->instrBufs.size(); ++i)
    {
        ptrs[i] = ctx->instrBufs[i];
        lengths[i] = ctx->instrBufLens[i];
    }
    if (ctx->rf)
    {
        ptrs[i] = ctx->rf;
        lengths[i] = ctx->rfLen;
    }
    return SKGPU_OK;
}

int skgpu_clear_tallies(skgpu_ctx* ctx)
{
    if (!ctx) return SKGPU_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    int rc = ensureRadiationField(ctx);
    if (rc) return rc;
    for (const InstrDev& d : ctx->instrHost)
    {
        size_t n = static_cast<size_t>(d.nbins) * d.npx * d.npy;
        double* t = d.kind == SKGPU_INSTR_FRAME ? d.ifu : d.sed;
        double* c = d.kind == SKGPU_INSTR_FRAME ? d.ifuComp : d.sedComp;
        double* s = d.kind == SKGPU_INSTR_FRAME ? d.ifuStats : d.sedStats;
        CK(cudaMemsetAsync(t, 0, n * sizeof(double), ctx->stream));
        if (c) CK(cudaMemsetAsync(c, 0, (3 + d.levels) * n * sizeof(double), ctx->stream));
        if (s) CK(cudaMemsetAsync(s, 0, 5 * n * sizeof(double), ctx->stream));
    }
    if (ctx->rf) CK(cudaMemsetAsync(ctx->rf, 0, ctx->rfLen * sizeof(double), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SKGPU_OK;
}

int skgpu_get_counters(skgpu_ctx* ctx, skgpu_counters* out)
{
    if (!ctx || !out) return SKGPU_ERR_ARG;
    *out = ctx->lastCounters;
    return SKGPU_OK;
}

int skgpu_set_stage_timing(skgpu_ctx* ctx, int32_t level)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (level < 0 || level > 2) return fail(ctx, SKGPU_ERR_ARG, "stage timing: level must be 0, 1 or 2");
    if (level && !ctx->timerEvents)
    {
        CK(cudaSetDevice(ctx->device));
        for (auto& row : ctx->timer.ev)
            for (cudaEvent_t& ev : row) CK(cudaEventCreate(&ev));
        ctx->timerEvents = true;
    }
    ctx->timer.level = level;
    return SKGPU_OK;
}

int skgpu_last_stage_times(skgpu_ctx* ctx, double* ms, uint64_t* launches)
{
    if (!ctx) return SKGPU_ERR_ARG;
    for (int i = 0; i < SKGPU_NUM_STAGES; ++i)
    {
        if (ms) ms[i] = ctx->timer.ms[i];
        if (launches) launches[i] = ctx->timer.launches[i];
    }
    return SKGPU_OK;
}

int skgpu_last_run_ms(skgpu_ctx* ctx, double* ms)
{
    if (!ctx || !ms) return SKGPU_ERR_ARG;
    *ms = ctx->lastMs;
    return SKGPU_OK;
}

// ------------------------------------------------------------------------------------------------
// path segments
// ------------------------------------------------------------------------------------------------

int skgpu_trace_paths(skgpu_ctx* ctx, int32_t num_rays, const double* rays, int32_t max_segments, int32_t precision,
                      int32_t* count, int32_t* m, double* ds)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!ctx->hasGrid) return fail(ctx, SKGPU_ERR_STATE, "trace: no grid uploaded");
    if (num_rays < 0 || max_segments < 1 || (num_rays > 0 && (!rays || !count || !m || !ds)))
        return fail(ctx, SKGPU_ERR_ARG, "trace: bad arguments");
    if (precision != SKGPU_PREC_FP64_EXACT && precision != SKGPU_PREC_FP32) return fail(ctx, SKGPU_ERR_ARG, "trace: bad precision");
    if (num_rays == 0) return SKGPU_OK;
    CK(cudaSetDevice(ctx->device));
    size_t n = num_rays, ns = n * static_cast<size_t>(max_segments);
    double *dRays = nullptr, *dDs = nullptr;
    int *dCount = nullptr, *dM = nullptr;
    auto cleanup = [&]() { devFree(dRays); devFree(dDs); devFree(dCount); devFree(dM); };
    cudaError_t e = devUpload(&dRays, rays, 6 * n);
    if (e == cudaSuccess) e = devAlloc(&dDs, ns);
    if (e == cudaSuccess) e = devAlloc(&dCount, n);
    if (e == cudaSuccess) e = devAlloc(&dM, ns);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->errFlag, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess)
        e = (precision == SKGPU_PREC_FP32 ? launchTracePathsFP32 : launchTracePathsFP64)(
            precision, ctx->g, num_rays, dRays, max_segments, dCount, dM, dDs, ctx->errFlag, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    int errFlag = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&errFlag, ctx->errFlag, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(count, dCount, n * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(m, dM, ns * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(ds, dDs, ns * sizeof(double), cudaMemcpyDeviceToHost);
    cleanup();
    if (e == cudaErrorNotSupported) return fail(ctx, SKGPU_ERR_UNSUPPORTED, "trace: no walker of this precision for the grid kind");
    if (e != cudaSuccess) return fail(ctx, SKGPU_ERR_CUDA, std::string("trace: ") + cudaGetErrorString(e));
    if (errFlag) return fail(ctx, SKGPU_ERR_TIMEOUT, "trace: a path exceeded its segment guard");
    return SKGPU_OK;
}

int skgpu_optical_depths(skgpu_ctx* ctx, int32_t num_rays, const double* rays, double lambda, int32_t precision,
                         double* tau)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!ctx->hasGrid || !ctx->dens || !ctx->nmix) return fail(ctx, SKGPU_ERR_STATE, "optical depths: grid, medium and mix required");
    if (ctx->numCells != ctx->g.numCells) return fail(ctx, SKGPU_ERR_STATE, "optical depths: medium does not match the grid");
    if (num_rays < 0 || (num_rays > 0 && (!rays || !tau))) return fail(ctx, SKGPU_ERR_ARG, "optical depths: bad arguments");
    if (precision != SKGPU_PREC_FP64_EXACT && precision != SKGPU_PREC_FP32) return fail(ctx, SKGPU_ERR_ARG, "optical depths: bad precision");
    if (num_rays == 0) return SKGPU_OK;
    // DustMix::sectionExt(lambda) = sigma_ext[locateClip(lambda borders, lambda)]
    std::vector<double> lb(ctx->nmix), se(ctx->nmix);
    CK(cudaMemcpy(lb.data(), ctx->mixLb, ctx->nmix * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(se.data(), ctx->mixExt, ctx->nmix * sizeof(double), cudaMemcpyDeviceToHost));
    double section = se[std::max(0, skg::locateClip(lb.data(), ctx->nmix, lambda))];
    size_t n = num_rays;
    double *dRays = nullptr, *dTau = nullptr;
    cudaError_t e = devUpload(&dRays, rays, 6 * n);
    if (e == cudaSuccess) e = devAlloc(&dTau, n);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->errFlag, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess)
        e = (precision == SKGPU_PREC_FP32 ? launchOpticalDepthsFP32 : launchOpticalDepthsFP64)(
            precision, ctx->g, ctx->dens, section, num_rays, dRays, dTau, ctx->errFlag, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpy(tau, dTau, n * sizeof(double), cudaMemcpyDeviceToHost);
    devFree(dRays);
    devFree(dTau);
    if (e != cudaSuccess) return fail(ctx, SKGPU_ERR_CUDA, std::string("optical depths: ") + cudaGetErrorString(e));
    return SKGPU_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// learned path guiding
// ------------------------------------------------------------------------------------------------
namespace {

// He-uniform hidden layers, small output layer with broad initial lobes (softplus(1.85) ~ 2)
void guideRandomParams(std::vector<float>& p, uint64_t seed)
{
    uint64_t st = seed ^ 0x9E3779B97F4A7C15ULL;
    auto next = [&]() {
        st += 0x9E3779B97F4A7C15ULL;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
    };
    p.assign(GUIDE_NPARAMS, 0.f);
    for (int l = 0; l < GUIDE_LAYERS; ++l)
    {
        int nin = guideDimIn(l), nout = guideDimOut(l);
        float* W = p.data() + guideParamOffset(l);
        float* b = W + nin * nout;
        double lim = std::sqrt(6.0 / nin) * (l + 1 == GUIDE_LAYERS ? 0.1 : 1.0);
        for (int i = 0; i < nin * nout; ++i) W[i] = static_cast<float>((2.0 * next() - 1.0) * lim);
        for (int o = 0; o < nout; ++o) b[o] = 0.f;
        if (l + 1 == GUIDE_LAYERS)
            for (int j = 0; j < GUIDE_LOBES; ++j)
            {
                // lobe directions spread over the sphere, concentration ~2
                double u = 2.0 * next() - 1.0, ph = 2.0 * M_PI * next(), sn = std::sqrt(1.0 - u * u);
                b[5 * j + 1] = static_cast<float>(sn * std::cos(ph));
                b[5 * j + 2] = static_cast<float>(sn * std::sin(ph));
                b[5 * j + 3] = static_cast<float>(u);
                b[5 * j + 4] = 1.85f;
            }
    }
}

int guideReady(skgpu_ctx* ctx)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (!ctx->guide) return fail(ctx, SKGPU_ERR_STATE, "guide: call skgpu_guide_init first");
    return SKGPU_OK;
}

#define GCK(call)                                                                                  \
    do                                                                                             \
    {                                                                                              \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(ctx, SKGPU_ERR_CUDA, std::string("guide: ") + cudaGetErrorString(e_));     \
    } while (0)

}  // namespace

extern "C" {

int skgpu_guide_num_params(void) { return GUIDE_NPARAMS; }

int skgpu_guide_init(skgpu_ctx* ctx, const float* params, uint64_t seed)
{
    if (!ctx) return SKGPU_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    GCK(guideEnsure(ctx));
    std::vector<float> p;
    if (params)
        p.assign(params, params + GUIDE_NPARAMS);
    else
        guideRandomParams(p, seed);
    for (float v : p)
        if (!std::isfinite(v)) return fail(ctx, SKGPU_ERR_ARG, "guide: non-finite parameter");
    GCK(guideSetParams(ctx, p.data()));
    return SKGPU_OK;
}

int skgpu_guide_get_params(skgpu_ctx* ctx, float* params)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    if (!params) return fail(ctx, SKGPU_ERR_ARG, "guide: null output");
    CK(cudaSetDevice(ctx->device));
    GCK(guideGetParams(ctx, params));
    return SKGPU_OK;
}

int skgpu_guide_set_mode(skgpu_ctx* ctx, int32_t mode, int32_t target_instrument, float alpha, float record_fraction,
                         uint64_t record_capacity)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    GuideState* g = ctx->guide;
    if (mode < 0 || mode > 2) return fail(ctx, SKGPU_ERR_ARG, "guide: mode must be 0, 1 or 2");
    if (mode != 0 && (target_instrument < 0 || target_instrument >= static_cast<int>(ctx->instrHost.size())))
        return fail(ctx, SKGPU_ERR_ARG, "guide: target instrument out of range (upload the instruments first)");
    if (mode == 2 && !(alpha >= 0.f && alpha < 1.f))
        return fail(ctx, SKGPU_ERR_ARG, "guide: alpha must lie in [0, 1): plain sampling must keep a share");
    if (mode == 1 && (!(record_fraction > 0.f && record_fraction <= 1.f) || record_capacity == 0
                      || record_capacity > 0x7FFFFFFFULL))
        return fail(ctx, SKGPU_ERR_ARG, "guide: record fraction in (0, 1] and capacity in [1, 2^31) required");
    CK(cudaSetDevice(ctx->device));
    if (mode == 1) GCK(guideEnsureRecords(ctx, record_capacity));
    g->mode = mode;
    g->target = target_instrument;
    g->alpha = alpha;
    g->recordFraction = record_fraction;
    return SKGPU_OK;
}

int skgpu_guide_set_importance(skgpu_ctx* ctx, int32_t n, const float* weights)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    GuideState* g = ctx->guide;
    CK(cudaSetDevice(ctx->device));
    if (g->importance) cudaFree(g->importance);
    g->importance = nullptr;
    g->importanceLen = 0;
    if (!weights || n <= 0) return SKGPU_OK;
    if (ctx->instrHost.empty() || g->target < 0 || g->target >= static_cast<int>(ctx->instrHost.size()))
        return fail(ctx, SKGPU_ERR_STATE, "guide: set a mode with a target instrument first");
    const InstrDev& t = ctx->instrHost[g->target];
    if (t.kind != SKGPU_INSTR_FRAME || n != t.npx * t.npy)
        return fail(ctx, SKGPU_ERR_ARG, "guide: importance needs one weight per pixel of the target frame");
    for (int i = 0; i < n; ++i)
        if (!(weights[i] >= 0.f) || !std::isfinite(weights[i]))
            return fail(ctx, SKGPU_ERR_ARG, "guide: importance weights must be finite and >= 0");
    CK(cudaMalloc(reinterpret_cast<void**>(&g->importance), static_cast<size_t>(n) * sizeof(float)));
    CK(cudaMemcpy(g->importance, weights, static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice));
    g->importanceLen = n;
    return SKGPU_OK;
}

int skgpu_guide_set_training(skgpu_ctx* ctx, int32_t position_bins)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    if (position_bins < 0 || position_bins > 64) return fail(ctx, SKGPU_ERR_ARG, "guide: position bins in [0, 64]");
    ctx->guide->positionBins = position_bins;
    return SKGPU_OK;
}

int skgpu_guide_last_weights(skgpu_ctx* ctx, uint64_t* events, double* mean_weight)
{
    if (!ctx || !events || !mean_weight) return SKGPU_ERR_ARG;
    *events = ctx->lastGuideEvents;
    *mean_weight = ctx->lastGuideEvents ? ctx->lastGuideWeightSum / static_cast<double>(ctx->lastGuideEvents) : 0.;
    return SKGPU_OK;
}

int skgpu_guide_record_count(skgpu_ctx* ctx, uint64_t* n)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    if (!n) return SKGPU_ERR_ARG;
    unsigned long long v = 0;
    if (ctx->guide->records)
    {
        CK(cudaSetDevice(ctx->device));
        GCK(guideRecordCount(ctx, &v));
    }
    *n = v;
    return SKGPU_OK;
}

int skgpu_guide_fetch_records(skgpu_ctx* ctx, uint64_t n, float* out)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    unsigned long long have = 0;
    if (ctx->guide->records) GCK(guideRecordCount(ctx, &have));
    if (!out || n > have) return fail(ctx, SKGPU_ERR_ARG, "guide: more records requested than recorded");
    GCK(guideFetchRecords(ctx, n, out));
    return SKGPU_OK;
}

int skgpu_guide_train(skgpu_ctx* ctx, int32_t steps, int32_t batch, float learning_rate, uint64_t seed, float* final_loss)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    if (steps < 0 || batch < 1 || batch > (1 << 20) || !(learning_rate > 0.f))
        return fail(ctx, SKGPU_ERR_ARG, "guide: steps >= 0, batch in [1, 2^20] and a positive learning rate required");
    if (!ctx->guide->records) return fail(ctx, SKGPU_ERR_STATE, "guide: no pilot records (run in mode 1 first)");
    CK(cudaSetDevice(ctx->device));
    cudaError_t e = guideTrain(ctx, steps, batch, learning_rate, seed, final_loss);
    if (e == cudaErrorInvalidValue) return fail(ctx, SKGPU_ERR_STATE, "guide: the pilot recorded no downstream detections");
    GCK(e);
    return SKGPU_OK;
}

int skgpu_guide_loss_grad(skgpu_ctx* ctx, int32_t n, const float* inputs, const float* directions, const float* weights,
                          float* loss, float* grad)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    if (n < 1 || n > (1 << 20) || !inputs || !directions || !weights || !loss || !grad)
        return fail(ctx, SKGPU_ERR_ARG, "guide: loss_grad arguments");
    CK(cudaSetDevice(ctx->device));
    GCK(guideLossGrad(ctx, n, inputs, directions, weights, loss, grad));
    return SKGPU_OK;
}

int skgpu_guide_infer(skgpu_ctx* ctx, int32_t n, const float* inputs, float* outputs, int32_t tensor_cores)
{
    int rc = guideReady(ctx);
    if (rc) return rc;
    if (n < 1 || n > (1 << 24) || !inputs || !outputs) return fail(ctx, SKGPU_ERR_ARG, "guide: infer arguments");
    CK(cudaSetDevice(ctx->device));
    int devErr = 0;
    GCK(guideInfer(ctx, n, inputs, outputs, tensor_cores, &devErr));
    if (devErr) return fail(ctx, SKGPU_ERR_TIMEOUT, "guide: a tensor-core wait gave up");
    return SKGPU_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// launch shape and batched runs
// ------------------------------------------------------------------------------------------------
extern "C" {

int skgpu_set_launch_shape(skgpu_ctx* ctx, int32_t pool_slots, int32_t trace_blocks_per_sm, int32_t shade_blocks_per_sm)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (pool_slots < 0 || pool_slots > static_cast<int32_t>(POOL_MAX) || trace_blocks_per_sm < 0 || trace_blocks_per_sm > 32
        || shade_blocks_per_sm < 0 || shade_blocks_per_sm > 64)
        return fail(ctx, SKGPU_ERR_ARG, "launch shape: pool in [0, 2^22], trace blocks per SM in [0, 32], shade blocks per SM in [0, 64]");
    ctx->shapePool = pool_slots;
    ctx->shapeTraceBlocks = trace_blocks_per_sm;
    ctx->shapeShadeBlocks = shade_blocks_per_sm;
    return SKGPU_OK;
}

int skgpu_set_trace_refill(skgpu_ctx* ctx, int32_t lanes)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (lanes < 0 || lanes > 32) return fail(ctx, SKGPU_ERR_ARG, "trace refill: lanes in [0, 32]");
    ctx->shapeRefill = lanes;
    return SKGPU_OK;
}

int skgpu_run_batch(skgpu_ctx* const* ctxs, int32_t n, const uint64_t* first, const uint64_t* count,
                    const uint64_t* total_packets)
{
    if (!ctxs || n < 1 || !first || !count || !total_packets) return SKGPU_ERR_ARG;
    skgpu_ctx* ctx = ctxs[0];
    if (!ctx) return SKGPU_ERR_ARG;
    if (n > MAX_BATCH) return fail(ctx, SKGPU_ERR_ARG, "batch: at most " + std::to_string(MAX_BATCH) + " contexts");
    int groups = 1, anyStats = 0;
    uint64_t sum = 0;
    for (int i = 0; i < n; ++i)
    {
        skgpu_ctx* c = ctxs[i];
        if (!c) return fail(ctx, SKGPU_ERR_ARG, "batch: null context");
        int rc = checkRunnable(c, first[i], count[i], total_packets[i]);
        if (rc) return fail(ctx, rc, "batch: context " + std::to_string(i) + ": " + c->err);
        if (c->device != ctx->device || c->g.kind != ctx->g.kind || c->opt.precision != ctx->opt.precision)
            return fail(ctx, SKGPU_ERR_ARG, "batch: contexts must share the device, grid kind and precision");
        if (c->guide && c->guide->mode != 0) return fail(ctx, SKGPU_ERR_STATE, "batch: learned path guiding is not offered in batches");
        CK(cudaSetDevice(c->device));
        if ((rc = ensureRadiationField(c))) return fail(ctx, rc, "batch: context " + std::to_string(i) + ": " + c->err);
        CK(cudaStreamSynchronize(c->stream));  // the batch runs on the first context's stream
        int g, st;
        waveShape(c, g, st);
        groups = std::max(groups, g);
        anyStats |= st;
        sum += count[i];
    }
    CK(cudaSetDevice(ctx->device));
    uint64_t poolMax = ctx->shapePool > 0 ? static_cast<uint64_t>(ctx->shapePool) : POOL_DEFAULT;
    int P = static_cast<int>(std::min<uint64_t>(std::max<uint64_t>(sum, 1), poolMax));
    int rc = ensureWaveBuffers(ctx, P, groups, anyStats);
    if (rc) return rc;
    std::vector<Scene> scenes(n);
    std::vector<unsigned long long> prefix(n + 1, 0), sfirst(n);
    for (int i = 0; i < n; ++i)
    {
        scenes[i] = sceneOf(ctxs[i]);
        prefix[i + 1] = prefix[i] + count[i];
        sfirst[i] = first[i];
    }
    for (void* p : ctx->batchBufs) cudaFree(p);
    ctx->batchBufs.clear();
    Scene* dScenes = nullptr;
    unsigned long long *dPrefix = nullptr, *dFirst = nullptr;
    CK(devAlloc(&dScenes, n));
    ctx->batchBufs.push_back(dScenes);
    CK(devAlloc(&dPrefix, n + 1));
    ctx->batchBufs.push_back(dPrefix);
    CK(devAlloc(&dFirst, n));
    ctx->batchBufs.push_back(dFirst);
    CK(cudaMemcpy(dScenes, scenes.data(), n * sizeof(Scene), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dPrefix, prefix.data(), (n + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dFirst, sfirst.data(), n * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    Wave w = ctx->wave;
    w.sc = scenes[0];
    w.scenes = dScenes;
    w.nScenes = n;
    w.prefix = dPrefix;
    w.sfirst = dFirst;
    w.P = P;
    w.first = 0;
    w.count = sum;
    w.anyStats = anyStats;
    w.statCap = STATS_CAP;
    w.traceBlocksPerSM = ctx->shapeTraceBlocks;
    w.refillMin = ctx->shapeRefill;
    w.rfAgg = rfWarpAggregation();
    w.shadeBlocksPerSM = ctx->shapeShadeBlocks;
    if ((rc = prepareOrder(ctx, w))) return rc;
    return runAndCollect(ctx, w, true, true);
}

int skgpu_set_history_order(skgpu_ctx* ctx, int32_t mode)
{
    if (!ctx) return SKGPU_ERR_ARG;
    if (mode != SKGPU_ORDER_INDEX && mode != SKGPU_ORDER_WAVELENGTH) return fail(ctx, SKGPU_ERR_ARG, "history order: 0 or 1");
    ctx->historyOrder = mode;
    return SKGPU_OK;
}

}  // extern "C"

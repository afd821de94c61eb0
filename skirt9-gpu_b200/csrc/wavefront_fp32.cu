// Wavefront life cycle with the FP32-distance walkers (production path). Grid kinds without such a
// walker are reported as unsupported; there is no silent substitution of the FP64 walkers.
#include "internal.hpp"
#include "grids_fast.cuh"
#include "wavefront_driver.cuh"

namespace skg {

cudaError_t runWaveFP32(int gridKind, const Wave& w, int numSMs, cudaStream_t s, unsigned long long* doneHost,
                        long long* passes, long long maxPasses, bool useGraph,
                        StageTimer* timer, GraphCache* cache)
{
    switch (gridKind)
    {
        case 0: return runWave<CartesianFast<float>>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 1: return runWave<OctreeLeaf32>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 2: return runWave<VoronoiRec32>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 3: return runWave<TetraPlane32>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 4: return runWave<Sphere1DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 5: return runWave<Cylinder2DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 6: return runWave<Sphere2DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 7: return runWave<Sphere3DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 8: return runWave<Cylinder3DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
    }
    return cudaErrorNotSupported;
}

cudaError_t orderHistories(const Wave& w, unsigned short* keys, unsigned* counts, unsigned* cursor, unsigned* order,
                           int numSMs, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(counts, 0, ORDER_BUCKETS * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    int sceneBits = 0;
    while ((1 << sceneBits) < w.nScenes) ++sceneBits;  // at most 6 (48 scenes)
    orderKeyKernel<<<numSMs * 8, 256, 0, s>>>(w, sceneBits, keys, counts);
    orderScanKernel<<<1, 1024, 0, s>>>(counts, cursor);
    orderScatterKernel<<<numSMs * 8, 256, 0, s>>>(w.count, keys, cursor, order);
    return cudaGetLastError();
}

}  // namespace skg

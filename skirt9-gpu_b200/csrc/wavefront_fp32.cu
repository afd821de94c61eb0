// Wavefront life cycle with the production walkers (FP32 accumulators; the Cartesian and octree
// walkers keep the reference's FP64 geometry, the Voronoi and tetrahedral ones FP32 face distances
// with FP64 re-decisions).
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
        case 0: return runWave<CartesianFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 1:
            return w.sc.g.tWallN ? runWave<OctreeRec>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache)
                                 : runWave<OctreeNodeFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 2: return runWave<VoronoiRec32>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 3: return runWave<TetraPlane32>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 4: return runWave<Sphere1DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 5: return runWave<Cylinder2DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 6: return runWave<Sphere2DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 7: return runWave<Sphere3DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 8: return runWave<Cylinder3DFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 9: return runWave<AdaptiveMeshFast>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
    }
    return cudaErrorNotSupported;
}

cudaError_t groupStats(const Wave& w, const StatSpill* groups, unsigned long long n, int numSMs, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    unsigned blocks = static_cast<unsigned>(std::min<unsigned long long>((n + 255) / 256, 4ull * numSMs));
    statGroupKernel<<<blocks, 256, 0, s>>>(w, groups, n);
    return cudaGetLastError();
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

// Wavefront life cycle with the FP64 walkers that keep the reference generators' operation order.
// Compiled with --fmad=false so that the FP64 physics outside the walkers (weights, directions,
// positions) is rounded like the reference CPU build (x86-64 SSE2, no FMA).
#include "internal.hpp"
#include "wavefront_driver.cuh"

namespace skg {

cudaError_t runWaveFP64(int gridKind, const Wave& w, int numSMs, cudaStream_t s, unsigned long long* doneHost,
                        long long* passes, long long maxPasses, bool useGraph,
                        StageTimer* timer, GraphCache* cache)
{
    switch (gridKind)
    {
        case 0: return runWave<CartesianExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 1: return runWave<OctreeExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 2: return runWave<VoronoiExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 3: return runWave<TetraExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 4: return runWave<Sphere1DExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 5: return runWave<Cylinder2DExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 6: return runWave<Sphere2DExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 7: return runWave<Sphere3DExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 8: return runWave<Cylinder3DExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
        case 9: return runWave<AdaptiveMeshExact>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer, cache);
    }
    return cudaErrorInvalidValue;
}

}  // namespace skg

// Wavefront life cycle with the FP32-distance walkers (production path). Grid kinds without such a
// walker are reported as unsupported; there is no silent substitution of the FP64 walkers.
#include "internal.hpp"
#include "grids_fast.cuh"
#include "wavefront_driver.cuh"

namespace skg {

cudaError_t runWaveFP32(int gridKind, const Wave& w, int numSMs, cudaStream_t s, unsigned long long* doneHost,
                        long long* passes, long long maxPasses, bool useGraph,
                        StageTimer* timer)
{
    switch (gridKind)
    {
        case 0: return runWave<CartesianFast<float>>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer);
        case 1: return runWave<OctreeLeaf32>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer);
        case 2: return runWave<VoronoiLocal32>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer);
        case 3: return runWave<TetraPlane32>(w, numSMs, s, doneHost, passes, maxPasses, useGraph, timer);
    }
    return cudaErrorNotSupported;
}

}  // namespace skg

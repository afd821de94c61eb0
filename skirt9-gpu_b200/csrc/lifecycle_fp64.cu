// FP64 life-cycle kernels with the reference generators' operation order. This translation unit is
// compiled with --fmad=false so that the FP64 physics (weights, directions, positions) is rounded
// like the reference CPU build (x86-64 SSE2, no FMA); the traversal itself uses explicit
// __dmul_rn/__dadd_rn and would be exact in either case.
#include "internal.hpp"

namespace skg {

template<class W>
static int blocksPerSM(int threads)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, lifecycleKernel<W>, threads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

int lifecycleBlocksPerSMFP64(int gridKind, int threads)
{
    switch (gridKind)
    {
        case 0: return blocksPerSM<CartesianExact>(threads);
        case 1: return blocksPerSM<OctreeExact>(threads);
        case 2: return blocksPerSM<VoronoiExact>(threads);
        case 3: return blocksPerSM<TetraExact>(threads);
    }
    return 1;
}

cudaError_t launchLifecycleFP64(int gridKind, const LCParams& p, int blocks, int threads, cudaStream_t s)
{
    switch (gridKind)
    {
        case 0: lifecycleKernel<CartesianExact><<<blocks, threads, 0, s>>>(p); break;
        case 1: lifecycleKernel<OctreeExact><<<blocks, threads, 0, s>>>(p); break;
        case 2: lifecycleKernel<VoronoiExact><<<blocks, threads, 0, s>>>(p); break;
        case 3: lifecycleKernel<TetraExact><<<blocks, threads, 0, s>>>(p); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace skg

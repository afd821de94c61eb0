// Path-segment and optical-depth kernels with the production walkers. They back skgpu_trace_paths /
// skgpu_optical_depths, the replacements of the reference's per-path GPU wrappers (GpuAcceleration::set*SpatialGridPath and the optical-depth
// sums, GpuAcceleration.hpp), and they are what the cell-sequence parity tests call.
#include "internal.hpp"
#include "paths.cuh"
#include "grids_fast.cuh"

namespace skg {

cudaError_t launchTracePathsFP32(int precision, const GridDev& g, int n, const double* rays, int maxSeg, int* count,
                             int* m, double* ds, int* err, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    int threads = 128, blocks = (n + threads - 1) / threads;
    (void)precision;
    switch (g.kind)
    {
        case 0: tracePathsKernel<CartesianFast><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 1:
            if (g.tWallN)
                tracePathsKernel<OctreeRec><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err);
            else
                tracePathsKernel<OctreeNodeFast><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err);
            break;
        case 2: tracePathsKernel<VoronoiRec32><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 3: tracePathsKernel<TetraPlane32><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 4: tracePathsKernel<Sphere1DFast><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 5: tracePathsKernel<Cylinder2DFast><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 6: tracePathsKernel<Sphere2DFast><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 7: tracePathsKernel<Sphere3DFast><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 8: tracePathsKernel<Cylinder3DFast><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 9: tracePathsKernel<AdaptiveMeshFast><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        default: return cudaErrorNotSupported;
    }
    return cudaGetLastError();
}

cudaError_t launchOpticalDepthsFP32(int precision, const GridDev& g, const double* dens, double section, int n,
                                const double* rays, double* tau, int* err, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    int threads = 128, blocks = (n + threads - 1) / threads;
    (void)precision;
    switch (g.kind)
    {
        case 0: opticalDepthKernel<CartesianFast><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 1:
            if (g.tWallN)
                opticalDepthKernel<OctreeRec><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err);
            else
                opticalDepthKernel<OctreeNodeFast><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err);
            break;
        case 2: opticalDepthKernel<VoronoiRec32><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 3: opticalDepthKernel<TetraPlane32><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 4: opticalDepthKernel<Sphere1DFast><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 5: opticalDepthKernel<Cylinder2DFast><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 6: opticalDepthKernel<Sphere2DFast><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 7: opticalDepthKernel<Sphere3DFast><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 8: opticalDepthKernel<Cylinder3DFast><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 9: opticalDepthKernel<AdaptiveMeshFast><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        default: return cudaErrorNotSupported;
    }
    return cudaGetLastError();
}

}  // namespace skg

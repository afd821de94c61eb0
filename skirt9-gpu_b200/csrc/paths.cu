// Path-segment and optical-depth kernels with the FP64 walkers that keep the reference generators'
// operation order. They back skgpu_trace_paths / skgpu_optical_depths, the replacements of the
// reference's per-path GPU wrappers (GpuAcceleration::set*SpatialGridPath and the optical-depth
// sums, GpuAcceleration.hpp), and they are what the cell-sequence parity tests call.
#include "internal.hpp"
#include "paths.cuh"

namespace skg {

cudaError_t launchTracePathsFP64(int precision, const GridDev& g, int n, const double* rays, int maxSeg, int* count,
                             int* m, double* ds, int* err, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    int threads = 128, blocks = (n + threads - 1) / threads;
    (void)precision;
    switch (g.kind)
    {
        case 0: tracePathsKernel<CartesianExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 1: tracePathsKernel<OctreeExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 2: tracePathsKernel<VoronoiExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 3: tracePathsKernel<TetraExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 4: tracePathsKernel<Sphere1DExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 5: tracePathsKernel<Cylinder2DExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 6: tracePathsKernel<Sphere2DExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 7: tracePathsKernel<Sphere3DExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 8: tracePathsKernel<Cylinder3DExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        case 9: tracePathsKernel<AdaptiveMeshExact><<<blocks, threads, 0, s>>>(g, n, rays, maxSeg, count, m, ds, err); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launchOpticalDepthsFP64(int precision, const GridDev& g, const double* dens, double section, int n,
                                const double* rays, double* tau, int* err, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    int threads = 128, blocks = (n + threads - 1) / threads;
    (void)precision;
    switch (g.kind)
    {
        case 0: opticalDepthKernel<CartesianExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 1: opticalDepthKernel<OctreeExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 2: opticalDepthKernel<VoronoiExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 3: opticalDepthKernel<TetraExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 4: opticalDepthKernel<Sphere1DExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 5: opticalDepthKernel<Cylinder2DExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 6: opticalDepthKernel<Sphere2DExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 7: opticalDepthKernel<Sphere3DExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 8: opticalDepthKernel<Cylinder3DExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        case 9: opticalDepthKernel<AdaptiveMeshExact><<<blocks, threads, 0, s>>>(g, dens, section, n, rays, tau, err); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace skg

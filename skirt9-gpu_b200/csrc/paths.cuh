// Path-segment and optical-depth kernels: one thread per ray, the grid's walker run to the end
// of the path (skgpu_trace_paths / skgpu_optical_depths).
#pragma once

#include "grids.cuh"

namespace skg {

constexpr int PATH_GUARD = 1 << 22;

template<class W>
__global__ void tracePathsKernel(const __grid_constant__ GridDev g, int n, const double* rays, int maxSeg, int* count, int* mo, double* dso,
                                 int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* q = rays + 6 * static_cast<size_t>(i);
    W w;
    w.start(g, q[0], q[1], q[2], q[3], q[4], q[5]);
    int c = 0;
    bool overflow = false;
    while (w.next(g))
    {
        if (c < maxSeg)
        {
            mo[static_cast<size_t>(i) * maxSeg + c] = w.m;
            dso[static_cast<size_t>(i) * maxSeg + c] = w.ds;
        }
        else
            overflow = true;
        if (++c > PATH_GUARD)
        {
            atomicOr(err, 4);
            break;
        }
    }
    count[i] = overflow ? -c : c;
}

// MediumSystem::getExtinctionOpticalDepth for a single medium with spatially constant cross
// section (MediumSystem.cpp:2328-2443), L = 1 so taumax = log(1) + 745
template<class W>
__global__ void opticalDepthKernel(const __grid_constant__ GridDev g, const double* dens, double section, int n, const double* rays,
                                   double* tau, int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* q = rays + 6 * static_cast<size_t>(i);
    W w;
    w.start(g, q[0], q[1], q[2], q[3], q[4], q[5]);
    double t = 0.;
    const double taumax = 745.;
    int c = 0;
    while (w.next(g))
    {
        if (w.m >= 0)
        {
            t = xadd(t, xmul(xmul(section, w.density(dens)), w.ds));
            if (t >= taumax)
            {
                t = INFINITY;
                break;
            }
        }
        if (++c > PATH_GUARD)
        {
            atomicOr(err, 4);
            break;
        }
    }
    tau[i] = t;
}

}  // namespace skg

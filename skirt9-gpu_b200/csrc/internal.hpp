// Declarations shared between the C-ABI translation unit and the kernel translation units.
#pragma once

#include <cuda_runtime.h>
#include "wave_types.cuh"

#include <vector>

namespace skg { struct StageTimer; }

namespace skg {

// An instantiated graph of passes kept across runs of one context: replayed while the wave
// parameters, launch shape, walker and timing it was captured with stay the same (repeated
// segments), re-captured otherwise.
struct GraphCache
{
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;
    // the second stream and the events of the split traversal (peel-off rays and propagation rays
    // walked by two kernels side by side), created with the first captured graph
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, peelDone = nullptr, join = nullptr;
    bool lastSplit = false;  // the last run split its traversal (one more kernel per pass)
    void reset()
    {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
    }
    cudaError_t ensureSplit()
    {
        cudaError_t e = cudaSuccess;
        if (!side) e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking);
        if (e == cudaSuccess && !fork) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        if (e == cudaSuccess && !peelDone) e = cudaEventCreateWithFlags(&peelDone, cudaEventDisableTiming);
        if (e == cudaSuccess && !join) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
        return e;
    }
    void release()
    {
        reset();
        if (fork) cudaEventDestroy(fork);
        if (peelDone) cudaEventDestroy(peelDone);
        if (join) cudaEventDestroy(join);
        if (side) cudaStreamDestroy(side);
        fork = peelDone = join = nullptr;
        side = nullptr;
    }
};

// wavefront life cycle, one entry per traversal precision (separate translation units, so that
// the FP64 one can be compiled without FMA contraction)
cudaError_t runWaveFP64(int gridKind, const Wave& w, int numSMs, cudaStream_t s, unsigned long long* doneHost,
                        long long* passes, long long maxPasses, bool useGraph, StageTimer* timer, GraphCache* cache);
cudaError_t runWaveFP32(int gridKind, const Wave& w, int numSMs, cudaStream_t s, unsigned long long* doneHost,
                        long long* passes, long long maxPasses, bool useGraph, StageTimer* timer, GraphCache* cache);

// moments of the grouped per-history statistics of the spill log (n records)
cudaError_t groupStats(const Wave& w, const StatSpill* groups, unsigned long long n, int numSMs, cudaStream_t s);

// wavelength order of the histories of w's range into order[] (keys: count entries, counts and
// cursor: ORDER_BUCKETS entries each, zeroed here)
cudaError_t orderHistories(const Wave& w, unsigned short* keys, unsigned* counts, unsigned* cursor, unsigned* order,
                           int numSMs, cudaStream_t s);

// tables of the equilibrium dust emission of the single dust mix (device pointers)
struct DustEmissionDev
{
    const double* rfSig;   // nrf: sigma_abs on the radiation-field wavelengths (_rfsigmaabsvv[0])
    const double* rfW;     // nrf: radiation-field bin widths (_rfdlambdav)
    const double* rfCmb;   // nrf: CMB source term (_Bcmbv)
    const double* rfSigL;  // nrf: the mix's sigma_abs at the bins' wavelengths (dust luminosity)
    const double* T;       // nT: temperature grid (_Tv)
    const double* planck;  // nT: Planck-integrated absorption cross sections (_planckabsvv[0])
    const double* emL;     // nem: dust-emission grid wavelengths (extlambdav)
    const double* emSig;   // nem: sigma_abs on the dust-emission grid (_emsigmaabsvv[0])
    const double* vol;     // cells: cell volumes
    int nrf, nT, nem;
};

// per-cell dust luminosity, equilibrium temperature and normalised emission pdf / cdf on the axis xv
// (npts points; emission-grid entries [minRight, maxRight) between the range ends)
cudaError_t launchDustCells(const DustEmissionDev& t, const double* dens, const double* rf, int numCells,
                            const double* xv, int npts, int minRight, int maxRight, double* L, double* T, double* pv,
                            double* Pv, cudaStream_t s);
// the leaf node of every octree cell
cudaError_t launchCellNodes(const int* tCell, int nodes, int* cellNode, cudaStream_t s);

// path-segment and optical-depth kernels, FP64 (reference operation order) and FP32-distance walkers
cudaError_t launchTracePathsFP64(int precision, const GridDev& g, int n, const double* rays, int maxSeg, int* count,
                                 int* m, double* ds, int* err, cudaStream_t s);
cudaError_t launchOpticalDepthsFP64(int precision, const GridDev& g, const double* dens, double section, int n,
                                    const double* rays, double* tau, int* err, cudaStream_t s);
cudaError_t launchTracePathsFP32(int precision, const GridDev& g, int n, const double* rays, int maxSeg, int* count,
                                 int* m, double* ds, int* err, cudaStream_t s);
cudaError_t launchOpticalDepthsFP32(int precision, const GridDev& g, const double* dens, double section, int n,
                                    const double* rays, double* tau, int* err, cudaStream_t s);

}  // namespace skg

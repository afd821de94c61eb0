// Device timing of the wavefront's stage kernels with CUDA events (host side only).
#pragma once

#include <cuda_runtime.h>

namespace skg {

// Optional device timing of the stage kernels with CUDA events on the launch stream. Level 1 times
// the trace kernel only (two events per pass), level 2 every stage (eight events per pass: before
// the trace kernel and after each stage; launch preparation and launch count as one stage). In a
// captured graph the events become event-record nodes; they are read after every batch, once the
// stream has synchronised, and summed into ms / launches in the order of SKGPU_STAGE_*. Stages
// that a run does not launch (the guided-scattering stage without guiding) are not counted.
struct StageTimer
{
    static constexpr int kBatch = 4;
    static constexpr int kStages = 7;
    int level = 0;
    bool active[kStages] = {true, true, true, true, true, true, true};
    cudaEvent_t ev[kBatch][kStages + 1] = {};
    double ms[kStages] = {};
    unsigned long long launches[kStages] = {};
};

inline cudaError_t stageMark(StageTimer* t, int pass, int i, cudaStream_t s, bool capturing)
{
    if (!t || t->level == 0 || (t->level == 1 && i > 1)) return cudaSuccess;
    return capturing ? cudaEventRecordWithFlags(t->ev[pass][i], s, cudaEventRecordExternal)
                     : cudaEventRecord(t->ev[pass][i], s);
}

// adds the stage durations of one completed batch
inline cudaError_t stageCollect(StageTimer* t)
{
    if (!t || t->level == 0) return cudaSuccess;
    int stages = t->level == 1 ? 1 : StageTimer::kStages;
    for (int k = 0; k < StageTimer::kBatch; ++k)
        for (int i = 0; i < stages; ++i)
        {
            if (!t->active[i]) continue;
            float ms = 0.f;
            cudaError_t e = cudaEventElapsedTime(&ms, t->ev[k][i], t->ev[k][i + 1]);
            if (e != cudaSuccess) return e;
            t->ms[i] += ms;
            t->launches[i] += 1;
        }
    return cudaSuccess;
}

}  // namespace skg

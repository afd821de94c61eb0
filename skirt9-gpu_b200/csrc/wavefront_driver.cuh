// Host driver of the wavefront: pool initialisation, then two passes (buffer parities 0 and 1)
// captured once into a CUDA graph and replayed until every history of the range is done.
#pragma once

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "internal.hpp"
#include "stage_timer.hpp"
#include "wavefront.cuh"

namespace skg {

struct WaveLaunch
{
    int traceBlocks, shadeBlocks, guideBlocks, threads;
    bool guided, multi;
    // split traversal: the peel-off kernel on the side stream, the propagation kernel on the main one
    bool split;
    int peelBlocks, propBlocks;
    cudaStream_t side;
    cudaEvent_t fork, peelDone, join;
};

// shared memory of the traversal kernel: the scene table of a batch
inline size_t traceSmemBytes(const Wave& w) { return w.nScenes > 1 ? w.nScenes * sizeof(Scene) : 0; }

template<class Walker, int Mode = TRACE_ALL>
int traceBlocksPerSM(bool multi, size_t smem)
{
    int n = 0;
    cudaError_t e = multi ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, traceKernel<Walker, true, Mode>, 256, smem)
                          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, traceKernel<Walker, false, Mode>, 256, 0);
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

template<class Walker, int Mode>
void launchTrace(const Wave& w, int cur, int blocks, const WaveLaunch& L, cudaStream_t s)
{
    if (L.multi)
        traceKernel<Walker, true, Mode><<<blocks, L.threads, traceSmemBytes(w), s>>>(w, cur);
    else
        traceKernel<Walker, false, Mode><<<blocks, L.threads, 0, s>>>(w, cur);
}

// `pass` is the index of the pass within its batch (selects the timer's events)
template<class Walker>
cudaError_t enqueuePass(const Wave& w, int pass, const WaveLaunch& L, cudaStream_t s, StageTimer* t, bool capturing)
{
    int cur = pass & 1, nxt = 1 - cur;
    cudaError_t e;
    if ((e = stageMark(t, pass, 0, s, capturing)) != cudaSuccess) return e;
    if (L.split)
    {
        // peel-off rays and their detection on the side stream, propagation rays on this one; the
        // stage kernels that end histories (and flush their statistics) wait for the detection
        if ((e = cudaEventRecord(L.fork, s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(L.side, L.fork, 0)) != cudaSuccess) return e;
        launchTrace<Walker, TRACE_PEEL>(w, cur, L.peelBlocks, L, L.side);
        if ((e = cudaEventRecord(L.peelDone, L.side)) != cudaSuccess) return e;
        shadePeelKernel<<<L.shadeBlocks, L.threads, 0, L.side>>>(w, cur);
        if ((e = cudaEventRecord(L.join, L.side)) != cudaSuccess) return e;
        launchTrace<Walker, TRACE_PROP>(w, cur, L.propBlocks, L, s);
        if ((e = cudaStreamWaitEvent(s, L.peelDone, 0)) != cudaSuccess) return e;
        if ((e = stageMark(t, pass, 1, s, capturing)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, L.join, 0)) != cudaSuccess) return e;
    }
    else
    {
        launchTrace<Walker, TRACE_ALL>(w, cur, L.traceBlocks, L, s);
        if ((e = stageMark(t, pass, 1, s, capturing)) != cudaSuccess) return e;
        shadePeelKernel<<<L.shadeBlocks, L.threads, 0, s>>>(w, cur);
    }
    if ((e = stageMark(t, pass, 2, s, capturing)) != cudaSuccess) return e;
    shadeProp1Kernel<<<L.shadeBlocks, L.threads, 0, s>>>(w, cur, nxt);
    if ((e = stageMark(t, pass, 3, s, capturing)) != cudaSuccess) return e;
    shadeProp2Kernel<<<L.shadeBlocks, L.threads, 0, s>>>(w, cur, nxt);
    if ((e = stageMark(t, pass, 4, s, capturing)) != cudaSuccess) return e;
    shadeFreeKernel<<<L.shadeBlocks, L.threads, 0, s>>>(w, cur, nxt);
    if ((e = stageMark(t, pass, 5, s, capturing)) != cudaSuccess) return e;
    if (L.guided) guideScatterKernel<<<L.guideBlocks, GM_TILE, GM_SMEM_BYTES, s>>>(w, cur, nxt);
    if ((e = stageMark(t, pass, 6, s, capturing)) != cudaSuccess) return e;
    launchPrepKernel<<<1, 1, 0, s>>>(w, nxt);
    launchKernel<<<L.shadeBlocks, L.threads, 0, s>>>(w, nxt);
    if ((e = stageMark(t, pass, 7, s, capturing)) != cudaSuccess) return e;
    return cudaGetLastError();
}

// Runs histories [w.first, w.first + w.count). `doneHost` receives the progress word (pinned host
// memory for the graph path). With `useGraph` the passes are captured once into a CUDA graph of
// four passes and replayed; without it the same kernels are launched directly (no graph objects are
// created). Returns a CUDA error, or cudaErrorLaunchTimeout (mapped to SKGPU_ERR_TIMEOUT) when the
// pass limit is reached without finishing. `passes` receives the number of passes run.
// the inputs a captured pass graph depends on: the wave parameters (by value in every kernel
// node), the launch shape, the walker and the timing events recorded into it
// the split traversal is on unless SKGPU_SPLIT_TRAVERSAL=0 (a switch for comparing the two forms)
inline bool splitTraversal()
{
    static const bool on = [] {
        const char* v = std::getenv("SKGPU_SPLIT_TRAVERSAL");
        return !(v && v[0] == '0');
    }();
    return on;
}

// the shared-memory carveout of the traversal kernels in percent (SKGPU_TRACE_CARVEOUT, unset: the
// driver's choice): the split of each SM's on-chip memory between L1 (which caches the grid records)
// and shared memory, for measuring what on-chip capacity for grid records is worth
inline int traceCarveout()
{
    static const int pct = [] {
        const char* v = std::getenv("SKGPU_TRACE_CARVEOUT");
        if (!v || !v[0]) return -1;
        int p = std::atoi(v);
        return p < 0 ? 0 : (p > 100 ? 100 : p);
    }();
    return pct;
}

template<class Walker>
void applyTraceCarveout()
{
    int pct = traceCarveout();
    if (pct < 0) return;
    auto set = [pct](const void* f) { cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, pct); };
    set(reinterpret_cast<const void*>(&traceKernel<Walker, false, TRACE_ALL>));
    set(reinterpret_cast<const void*>(&traceKernel<Walker, false, TRACE_PEEL>));
    set(reinterpret_cast<const void*>(&traceKernel<Walker, false, TRACE_PROP>));
    set(reinterpret_cast<const void*>(&traceKernel<Walker, true, TRACE_ALL>));
    set(reinterpret_cast<const void*>(&traceKernel<Walker, true, TRACE_PEEL>));
    set(reinterpret_cast<const void*>(&traceKernel<Walker, true, TRACE_PROP>));
}

template<class Walker>
std::vector<unsigned char> graphKey(const Wave& w, const WaveLaunch& L, const StageTimer* timer)
{
    std::vector<unsigned char> k(sizeof(Wave) + sizeof(WaveLaunch) + 2 * sizeof(void*) + StageTimer::kStages);
    unsigned char* p = k.data();
    std::memcpy(p, &w, sizeof(Wave));
    p += sizeof(Wave);
    std::memcpy(p, &L, sizeof(WaveLaunch));
    p += sizeof(WaveLaunch);
    const void* id = reinterpret_cast<const void*>(&traceKernel<Walker, false>);
    std::memcpy(p, &id, sizeof(void*));
    p += sizeof(void*);
    std::memcpy(p, &timer, sizeof(void*));
    p += sizeof(void*);
    for (int i = 0; i < StageTimer::kStages; ++i) p[i] = timer && timer->active[i] ? 1 : 0;
    return k;
}

template<class Walker>
cudaError_t runWave(const Wave& w, int numSMs, cudaStream_t s, unsigned long long* doneHost, long long* passes,
                    long long maxPasses, bool useGraph, StageTimer* timer, GraphCache* cache = nullptr)
{
    WaveLaunch L{};
    L.threads = 256;
    applyTraceCarveout<Walker>();
    L.multi = w.nScenes > 1;
    int resident = traceBlocksPerSM<Walker>(L.multi, traceSmemBytes(w));
    // a tuned shape may ask for fewer resident trace blocks, never for more than fit
    L.traceBlocks = numSMs * (w.traceBlocksPerSM > 0 ? std::min(w.traceBlocksPerSM, resident) : resident);
    L.shadeBlocks = numSMs * (w.shadeBlocksPerSM > 0 ? w.shadeBlocksPerSM : 4);
    L.guideBlocks = numSMs * 2;
    L.guided = w.sc.guideMode == 2;
    // the split traversal runs in captured graphs without per-stage timing, for walkers that gain
    // from it
    L.split = false;
    if (Walker::kSplit && useGraph && cache && (!timer || timer->level <= 1) && splitTraversal())
    {
        if (cache->ensureSplit() == cudaSuccess)
        {
            L.split = true;
            int cap = w.traceBlocksPerSM > 0 ? w.traceBlocksPerSM : 1 << 30;
            L.peelBlocks = numSMs * std::min(cap, traceBlocksPerSM<Walker, TRACE_PEEL>(L.multi, traceSmemBytes(w)));
            L.propBlocks = numSMs * std::min(cap, traceBlocksPerSM<Walker, TRACE_PROP>(L.multi, traceSmemBytes(w)));
            L.side = cache->side;
            L.fork = cache->fork;
            L.peelDone = cache->peelDone;
            L.join = cache->join;
        }
    }
    *passes = 0;
    if (timer)
        for (int i = 0; i < StageTimer::kStages; ++i) timer->active[i] = i != 5 || L.guided;
    if (L.guided)
    {
        cudaError_t ea = cudaFuncSetAttribute(guideScatterKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GM_SMEM_BYTES);
        if (ea != cudaSuccess) return ea;
    }
    if (cache) cache->lastSplit = L.split;
    initPoolKernel<<<L.shadeBlocks, L.threads, 0, s>>>(w);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (w.count == 0) return cudaStreamSynchronize(s);

    const int passesPerBatch = StageTimer::kBatch;  // even: the buffer parity returns to 0 after every batch
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;
    if (useGraph && cache)
    {
        // a repeated segment replays the graph captured for the previous one
        key = graphKey<Walker>(w, L, timer);
        if (cache->exec && cache->key == key)
            exec = cache->exec;
        else
            cache->reset();
    }
    if (useGraph && !exec)
    {
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        for (int k = 0; k < passesPerBatch && e == cudaSuccess; ++k) e = enqueuePass<Walker>(w, k, L, s, timer, true);
        cudaError_t e2 = cudaStreamEndCapture(s, &graph);
        if (e == cudaSuccess) e = e2;
        if (e != cudaSuccess)
        {
            if (graph) cudaGraphDestroy(graph);
            return e;
        }
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);  // the executable graph does not need it
        graph = nullptr;
        if (e != cudaSuccess) return e;
        if (cache)
        {
            cache->exec = exec;
            cache->key = key;
        }
    }
    const size_t doneOffset = offsetof(Control, done);
    unsigned long long lastDone = 0;
    long long lastProgress = 0;
    while (e == cudaSuccess)
    {
        if (useGraph)
            e = cudaGraphLaunch(exec, s);
        else
            for (int k = 0; k < passesPerBatch && e == cudaSuccess; ++k) e = enqueuePass<Walker>(w, k, L, s, timer, false);
        if (e != cudaSuccess) break;
        *passes += passesPerBatch;
        e = cudaMemcpyAsync(doneHost, reinterpret_cast<char*>(w.ctl) + doneOffset, sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) break;
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) break;
        e = stageCollect(timer);
        if (e != cudaSuccess) break;
        if (*doneHost >= w.count) break;
        if (*doneHost != lastDone)
        {
            lastDone = *doneHost;
            lastProgress = *passes;
        }
        // no history finished for 65536 passes (more than 32768 scattering events of one history),
        // or the overall pass limit: stop with a timeout status instead of looping on
        if (*passes >= maxPasses || *passes - lastProgress > 65536)
        {
            e = cudaErrorLaunchTimeout;
            break;
        }
    }
    if (exec && !(cache && cache->exec == exec)) cudaGraphExecDestroy(exec);
    if (cache && e != cudaSuccess) cache->reset();  // after an error the next run captures afresh
    return e;
}

}  // namespace skg

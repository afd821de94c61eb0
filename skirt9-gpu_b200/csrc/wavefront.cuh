// Wavefront form of the photon-packet life cycle (MonteCarloSimulation::performLifeCycle,
// SKIRT/core/MonteCarloSimulation.cpp:614-694).
//
// Packet state lives in a pool of P slots, one 128-byte record per slot. Every traversal of the
// life cycle is a task in one of four queues (a fifth holds the events of guided scattering):
//   PEEL   optical depth from a packet position to the domain edge towards one observer
//          (FluxRecorder::detect -> MediumSystem::getExtinctionOpticalDepth, MediumSystem.cpp:2328-2443)
//   PROP1  forced scattering, complete path: cumulative optical depth + radiation-field storage
//          (MediumSystem::setExtinctionOpticalDepths :1785-1846, MonteCarloSimulation::storeRadiationField :888-957)
//   PROP2  forced scattering, interaction point of the sampled optical depth
//          (MonteCarloSimulation::simulateForcedPropagation :1492-1546, SpatialGridPath::findInteractionPoint :161-203)
//   FREE   non-forced propagation (simulateNonForcedPropagation :1996-2030,
//          MediumSystem::setInteractionPointUsingExtinction :2005-2150)
// One pass of the wavefront runs:
//   trace    a persistent kernel: each lane takes a task, walks its ray to the end (one cell
//            crossing per loop iteration, so the warp's lanes stay converged on the crossing code);
//            a warp takes new task indices with one atomic once enough of its lanes wait;
//   shade    one coherent kernel per task kind: detection (peel-off tallies), forced sampling,
//            interaction + scattering peel-off emission + HG scattering, free-path interaction;
//            each emits the packet's next tasks into the other queue buffer;
//   launch   refills free slots with new histories (SourceSystem::launch; in wavelength order
//            when the range exceeds the pool) and emits their emission peel-offs and first
//            propagation.
// Random numbers: each history draws from its own Philox stream in the reference's order
// (launch, forced sampling, scattering), whatever pass the draws happen in.
#pragma once

#include <cstdio>
#include "wave_types.cuh"
#include "guide_mma.cuh"

namespace skg {

// the scene of a packet slot (batched runs keep one per slot)
SKG_D const Scene& slotScene(const Wave& w, int slot) { return w.nScenes > 1 ? w.scenes[w.pk.rec[slot].scene] : w.sc; }


// ---------------------------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------------------------

// warp-aggregated append: one atomic per group of converged lanes
SKG_D unsigned warpAppend(unsigned* counter)
{
    unsigned active = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(active) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<unsigned>(__popc(active)));
    base = __shfl_sync(active, base, leader);
    return base + __popc(active & ((1u << lane) - 1));
}

SKG_D void loadRng(const Wave& w, int slot, Rng& r)
{
    r.start(slotScene(w, slot).seed, w.pk.rec[slot].hist);
    r.ctr = w.pk.rec[slot].rngCtr;
    r.hasSpare = w.pk.rec[slot].rngHas;
    r.spare = w.pk.rec[slot].rngSpare;
}

SKG_D void storeRng(const Wave& w, int slot, const Rng& r)
{
    w.pk.rec[slot].rngCtr = r.ctr;
    w.pk.rec[slot].rngHas = r.hasSpare;
    w.pk.rec[slot].rngSpare = r.spare;
}

SKG_D void addMoments(double* base, size_t plane, size_t idx, double wsum)
{
    double wn = 1.;
    for (int k = 0; k <= 4; ++k)
    {
        atomicAdd(base + k * plane + idx, wn);
        wn *= wsum;
    }
}

SKG_D void statMoments(const Scene& sc, unsigned long long key, double wsum)
{
    int i = static_cast<int>(key >> 48);
    int ell = static_cast<int>((key >> 24) & 0xFFFFFF);
    int l = static_cast<int>(key & 0xFFFFFF) - 1;
    const InstrDev& in = sc.instr[i];
    if (l < 0)
        addMoments(in.sedStats, in.nbins, ell, wsum);
    else
    {
        size_t npix = static_cast<size_t>(in.npx) * in.npy;
        addMoments(in.ifuStats, npix * in.nbins, static_cast<size_t>(l) + static_cast<size_t>(ell) * npix, wsum);
    }
}

// appends one contribution of the slot's history to the spill log (grouped after the run)
SKG_D void spillStat(const Wave& w, int slot, unsigned long long key, double v)
{
    unsigned long long i = atomicAdd(&w.ctl->spillN, 1ULL);
    if (i < w.pk.spillCap)
    {
        StatSpill& e = w.pk.spill[i];
        e.hist = w.pk.rec[slot].hist;
        e.key = key;
        e.w = v;
        e.scene = w.nScenes > 1 ? w.pk.rec[slot].scene : 0;
        atomicAdd(&w.ctl->counters[6], 1ULL);
    }
    else
    {
        atomicAdd(&w.ctl->counters[5], 1ULL);  // lost: the run fails
        atomicOr(&w.ctl->err, 64);
    }
}

// FluxRecorder::recordContributions (FluxRecorder.cpp:1355-1409) groups a history's contributions
// per (instrument, wavelength bin, pixel). Here a contribution is added to its key's entry in the
// slot's buffer, or takes a new entry. The threads that record one slot at the same time (one
// shadePeelKernel thread per observer group of the slot's event) hold keys of different
// instruments, so a key found in the buffer comes from an earlier pass and nobody else updates it;
// an entry being written concurrently still holds the empty key ~0 or a key of another instrument.
// A contribution that finds the buffer full goes to the spill log.
SKG_D void recordStat(const Wave& w, int slot, unsigned long long key, double v)
{
    const int cap = w.statCap;
    unsigned long long* keys = w.pk.skey + static_cast<size_t>(slot) * cap;
    double* sw = w.pk.sw + static_cast<size_t>(slot) * cap;
    int n = min(*static_cast<volatile int*>(w.pk.nstat + slot), cap);
    for (int a = 0; a < n; ++a)
    {
        if (keys[a] == key)
        {
            sw[a] += v;
            return;
        }
    }
    int k = atomicAdd(&w.pk.nstat[slot], 1);
    if (k < cap)
    {
        sw[k] = v;
        keys[k] = key;
    }
    else
    {
        spillStat(w, slot, key, v);
    }
}

// end of a history: w^0..w^4 of every grouped contribution, or, when the history spilled, its
// buffered contributions join the spill log for the grouping after the run; the entries are reset
SKG_D void flushStats(const Wave& w, int slot)
{
    const int cap = w.statCap;
    int taken = w.pk.nstat[slot];
    int n = min(taken, cap);
    unsigned long long* key = w.pk.skey + static_cast<size_t>(slot) * cap;
    double* sw = w.pk.sw + static_cast<size_t>(slot) * cap;
    for (int a = 0; a < n; ++a)
    {
        unsigned long long ka = key[a];
        if (ka == ~0ULL) continue;
        if (taken > cap)
            spillStat(w, slot, ka, sw[a]);
        else
            statMoments(slotScene(w, slot), ka, sw[a]);
        key[a] = ~0ULL;
    }
    w.pk.nstat[slot] = 0;
}

// moments of the grouped spill-log sums (one record per history and key, computed after the run)
static __global__ void __launch_bounds__(256) statGroupKernel(const __grid_constant__ Wave w, const StatSpill* groups,
                                                              unsigned long long n)
{
    for (unsigned long long t = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; t < n;
         t += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
    {
        const StatSpill& g = groups[t];
        statMoments(w.nScenes > 1 ? w.scenes[g.scene] : w.sc, g.key, g.w);
    }
}

// end of a recorded pilot history: the downstream luminosity per unit packet luminosity of every
// recorded event, from the history's final detected luminosity
SKG_D void guideCloseHistory(const Wave& w, int slot)
{
    const Scene& sc = slotScene(w, slot);
    double D = w.pk.gD[slot];
    int pend = w.pk.gPend[slot];
    if (pend >= 0) sc.guideRec[pend].dStart = D;
    int r = w.pk.gLast[slot];
    for (int guard = 0; r >= 0 && guard < (1 << 20); ++guard)
    {
        GuideRecord& q = sc.guideRec[r];
        q.I = q.L > 0.f ? static_cast<float>((D - q.dStart) / static_cast<double>(q.L)) : 0.f;
        r = q.prev;
    }
}

SKG_D void endHistory(const Wave& w, int slot)
{
    if (w.anyStats && w.pk.nstat[slot]) flushStats(w, slot);
    if (slotScene(w, slot).guideMode == 1) guideCloseHistory(w, slot);
    int i = atomicAdd(&w.ctl->freeTop, 1);
    w.pk.freeSlots[i] = slot;
    atomicAdd(&w.ctl->done, 1ULL);
}

SKG_D void emitPeel(const Wave& w, int nxt, int slot, int group, int numScatt, double Lp, double x, double y,
                    double z)
{
    const TaskBuf& b = w.q[nxt][K_PEEL];
    unsigned i = warpAppend(&w.ctl->qn[nxt][K_PEEL]);
    b.slot[i] = slot;
    b.info[i] = group | (min(numScatt, (1 << 22)) << 8);
    b.par[i] = Lp;
    b.x[i] = x;
    b.y[i] = y;
    b.z[i] = z;
}

SKG_D void emitProp(const Wave& w, int nxt, int kind, int slot, double par)
{
    const TaskBuf& b = w.q[nxt][kind];
    unsigned i = warpAppend(&w.ctl->qn[nxt][kind]);
    b.slot[i] = slot;
    b.par[i] = par;
}

// peel-off tasks for every observer group that records the packet at (x,y,z);
// scattering peel-offs carry L * phase function (DustMix::peeloffScattering, DustMix.cpp:430-488)
SKG_D void emitPeels(const Wave& w, int nxt, int slot, bool scattering, int numScatt, double L, double g, double x,
                     double y, double z, double kx, double ky, double kz)
{
    const Scene& sc = slotScene(w, slot);
    for (int i = 0; i < sc.ninstr; i = nextGroup(sc, i))
    {
        if (!groupNeedsTau(sc, i, x, y, z)) continue;
        const InstrDev& in = sc.instr[i];
        double Lp = L;
        if (scattering) Lp = L * phaseHG(g, kx * in.kobs[0] + ky * in.kobs[1] + kz * in.kobs[2]);
        emitPeel(w, nxt, slot, i, numScatt, Lp, x, y, z);
    }
}

// emits the first traversal of a propagation (forced: PROP1; free: FREE with its sampled tau)
SKG_D void beginPropagation(const Wave& w, int nxt, int slot, Rng& rng)
{
    if (slotScene(w, slot).forced)
        emitProp(w, nxt, K_PROP1, slot, 0.);
    else
        emitProp(w, nxt, K_FREE, slot, -log(rng.uniform()));  // Random::expon
}

// ---------------------------------------------------------------------------------------------
// trace: walk every queued ray; one crossing per iteration, lanes refill from the queues
// ---------------------------------------------------------------------------------------------
// arithmetic of the walk accumulators: FP64 with separate roundings (reference order), or FP32
SKG_D double aadd(double a, double b) { return xadd(a, b); }
SKG_D double amul(double a, double b) { return xmul(a, b); }
SKG_D double aexp(double x) { return exp(x); }
SKG_D float aadd(float a, float b) { return a + b; }
SKG_D float amul(float a, float b) { return a * b; }
SKG_D float aexp(float x) { return __expf(x); }

// Mode selects the task kinds a launch walks: TRACE_ALL every kind; TRACE_PEEL the peel-off rays
// and TRACE_PROP the propagation rays (PROP1, PROP2, FREE), two kernels that the captured pass graph
// runs side by side on two streams, each with its own task cursor. The peel-off kernel, which walks
// two thirds of the crossings of the galaxy, then carries none of the propagation tasks' state.
enum TraceMode { TRACE_ALL = 0, TRACE_PEEL = 1, TRACE_PROP = 2 };

template<class Walker, bool Multi = false, int Mode = TRACE_ALL>
__global__ void __launch_bounds__(256, Walker::kMinBlocks) traceKernel(const __grid_constant__ Wave w, int cur)
{
    // the scene of the lane's task: the kernel parameter's for one scene; for a batch, the scene
    // table staged in shared memory (the walker reads its grid pointers there at every crossing)
    int sid = 0;
    extern __shared__ __align__(16) unsigned char traceSmem[];
    const Scene* table = reinterpret_cast<const Scene*>(traceSmem);
    if constexpr (Multi)
    {
        const int4* src = reinterpret_cast<const int4*>(w.scenes);
        int4* dst = reinterpret_cast<int4*>(traceSmem);
        const int words = w.nScenes * static_cast<int>(sizeof(Scene) / sizeof(int4));
        for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
        __syncthreads();
    }
    auto scn = [&]() -> const Scene& {
        if constexpr (Multi)
            return table[sid];
        else
            return w.sc;
    };
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int refillMin = w.refillMin > 0 ? w.refillMin : Walker::kRefillMin;
    unsigned n0 = w.ctl->qn[cur][0], n1 = w.ctl->qn[cur][1], n2 = w.ctl->qn[cur][2], n3 = w.ctl->qn[cur][3];
    const unsigned total = Mode == TRACE_PEEL ? n0 : (Mode == TRACE_PROP ? n1 + n2 + n3 : n0 + n1 + n2 + n3);
    if (total == 0) return;
    unsigned* const cursor = Mode == TRACE_PROP ? &w.ctl->traceCursor2 : &w.ctl->traceCursor;

    using Acc = typename Walker::Acc;  // FP64 (reference rounding) or FP32 optical depth and path length
    Walker wk;
    int kind = -1;  // -1: needs a task, -2: finished
    // the task kind of a lane's current task, known at compile time where the mode fixes it
    auto isPeel = [&]() { return Mode == TRACE_PEEL || (Mode == TRACE_ALL && kind == K_PEEL); };
    auto isProp1 = [&]() { return Mode != TRACE_PEEL && kind == K_PROP1; };
    unsigned idx = 0;
    int slot = 0;
    // Per-task accumulators. The task kinds never share a lane at the same time, so their
    // variables share registers (named per kind below):
    //   PEEL:       fA = optical-depth cutoff log(L) + 745
    //   PROP1:      fA = L, fB = ln(extinction) at the segment start, fC = extinction there, iA = RF bin
    //   PROP2/FREE: fA = target optical depth, fB = path length, fC = path length at the last segment, iA = last cell
    Acc tau = 0, fA = 0, fB = 0, fC = 0, sext = 0;
    int iA = -1, nseg = 0;
    unsigned cross = 0, rfStores = 0;  // flushed to the counters before they can overflow
    int guard = 0;

    while (true)
    {
        unsigned need = __ballot_sync(FULL, kind == -1);
        // A warp takes new tasks once refillMin lanes wait (or none is busy), not for every
        // lane that finishes: the refill (task-buffer and packet-state loads, walker start) then runs
        // once for several lanes instead of stalling the busy lanes at almost every crossing. The
        // best count depends on the cost of a crossing (measured: 16 for the Cartesian grid and the
        // octree, 8 for tetrahedra and Voronoi cells): Walker::kRefillMin, unless the launch shape
        // sets it (skgpu_set_trace_refill).
        if (need && (__popc(need) >= refillMin || __ballot_sync(FULL, kind >= 0) == 0))
        {
            int leader = __ffs(need) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(cursor, static_cast<unsigned>(__popc(need)));
            base = __shfl_sync(FULL, base, leader);
            if (kind == -1)
            {
                unsigned t = base + __popc(need & ((1u << lane) - 1));
                if (t >= total)
                {
                    kind = -2;
                }
                else
                {
                    if (Mode == TRACE_PROP) t += n0;
                    if (Mode == TRACE_PEEL || t < n0) { kind = K_PEEL; idx = t; }
                    else if (t < n0 + n1) { kind = K_PROP1; idx = t - n0; }
                    else if (t < n0 + n1 + n2) { kind = K_PROP2; idx = t - n0 - n1; }
                    else { kind = K_FREE; idx = t - n0 - n1 - n2; }
                    const TaskBuf& b = w.q[cur][kind];
                    slot = b.slot[idx];
                    if constexpr (Multi) sid = w.pk.rec[slot].scene;
                    // peel-off rays and complete forced paths (PROP1: radiation field) accumulate
                    // extinction; under explicit absorption the interaction searches (PROP2, FREE)
                    // walk on the scattering optical depth (setScatteringAndAbsorptionOpticalDepths)
                    {
                        int ell = w.pk.rec[slot].ellMix;
                        sext = static_cast<Acc>(scn().explicitAbs && !isPeel() && kind >= K_PROP2 ? scn().mixSca[ell]
                                                                                                   : scn().mixExt[ell]);
                    }
                    tau = 0.;
                    nseg = 0;
                    guard = 0;
                    if (isPeel())
                    {
                        const InstrDev& in = scn().instr[b.info[idx] & 0xFF];
                        fA = static_cast<Acc>(log(b.par[idx]) + 745.);  // taumax = log(L) + 745
                        wk.start(scn().g, b.x[idx], b.y[idx], b.z[idx], in.kobs[0], in.kobs[1], in.kobs[2],
                                 w.pk.rec[slot].cell);
                    }
                    else
                    {
                        wk.start(scn().g, w.pk.rec[slot].x, w.pk.rec[slot].y, w.pk.rec[slot].z, w.pk.rec[slot].kx, w.pk.rec[slot].ky,
                                 w.pk.rec[slot].kz, w.pk.rec[slot].cell);
                        if (isProp1())
                        {
                            fA = static_cast<Acc>(w.pk.rec[slot].L);
                            iA = scn().rfOn ? w.pk.rec[slot].ellRF : -1;
                            fB = 0.;
                            fC = 1.;
                        }
                        else
                        {
                            fA = static_cast<Acc>(b.par[idx]);
                            fB = 0.;
                            fC = 0.;
                            iA = -1;
                        }
                    }
                }
            }
        }
        if (__all_sync(FULL, kind == -2)) break;
        if (kind < 0) continue;

        bool got = wk.next(scn().g);
        bool done = !got;
        if (got)
        {
            cross++;
            int m = wk.m;
            Acc ds = static_cast<Acc>(wk.ds);
            if (isPeel())
            {
                if (m >= 0)
                {
                    tau = aadd(tau, amul(amul(sext, static_cast<Acc>(wk.density(scn().dens))), ds));
                    if (tau >= fA)
                    {
                        tau = static_cast<Acc>(INFINITY);
                        done = true;
                    }
                }
            }
            else if (isProp1())
            {
                if (ds > 0.)
                {
                    if (m >= 0) tau = aadd(tau, amul(amul(sext, static_cast<Acc>(wk.density(scn().dens))), ds));
                    nseg++;
                    if (iA >= 0)
                    {
                        Acc lnExtEnd = -tau;
                        Acc extEnd = aexp(lnExtEnd);
                        if (m >= 0)
                        {
                            // L * ds exceeds the FP32 range (watts times metres): the product is FP64
                            double Lds = static_cast<double>(fA) * static_cast<double>(lnmean4(extEnd, fC, lnExtEnd, fB))
                                         * static_cast<double>(ds);
                            // device layout ell * cells + m: the packets in flight (taken up in
                            // wavelength order) update one contiguous slice; the fetch transposes
                            double* at = scn().rf + static_cast<size_t>(iA) * scn().g.numCells + m;
                            if (w.rfAgg)
                                atomicAddAgg(at, Lds);
                            else
                                atomicAdd(at, Lds);
                            rfStores++;
                        }
                        fB = lnExtEnd;
                        fC = extEnd;
                    }
                }
            }
            else
            {
                // PROP2 keeps segments with ds > 0 (SpatialGridPath::addSegment); FREE uses every segment
                if (kind == K_FREE || ds > 0.)
                {
                    Acc tau0 = tau, s0 = fB;
                    if (m >= 0) tau = aadd(tau, amul(amul(sext, static_cast<Acc>(wk.density(scn().dens))), ds));
                    fB = aadd(fB, ds);
                    iA = m;
                    fC = fB;
                    if (fA < tau)
                    {
                        // NR::interpolateLinLin (SKIRT/utils/NR.hpp:328-331)
                        const TaskBuf& b = w.q[cur][kind];
                        b.m[idx] = m;
                        b.s[idx] = static_cast<double>(s0 + ((fA - tau0) / (tau - tau0)) * (fB - s0));
                        b.found[idx] = 1;
                        kind = -1;
                        continue;
                    }
                }
            }
            if (++guard > (1 << 20))
            {
                // a traversal that does not end: report the first few (task kind, start point and
                // direction, last cell) and stop it; the run returns SKGPU_ERR_TIMEOUT
                if (atomicAdd(&w.ctl->counters[7], 1ULL) < 4ULL)
                {
                    const TaskBuf& b = w.q[cur][kind];
                    bool peel = isPeel();
                    const double* ko = peel ? scn().instr[b.info[idx] & 0xFF].kobs : nullptr;
                    printf("skgpu: traversal guard: kind %d hist %llu start (%.17g %.17g %.17g) dir (%.17g %.17g %.17g) cell %d\n",
                           kind, static_cast<unsigned long long>(w.pk.rec[slot].hist), peel ? b.x[idx] : w.pk.rec[slot].x,
                           peel ? b.y[idx] : w.pk.rec[slot].y, peel ? b.z[idx] : w.pk.rec[slot].z, peel ? ko[0] : w.pk.rec[slot].kx,
                           peel ? ko[1] : w.pk.rec[slot].ky, peel ? ko[2] : w.pk.rec[slot].kz, m);
                }
                atomicOr(&w.ctl->err, 4);
                done = true;
            }
        }
        if (done)
        {
            const TaskBuf& b = w.q[cur][kind];
            if (isPeel())
                b.tau[idx] = static_cast<double>(tau);
            else if (isProp1())
                b.tau[idx] = nseg ? static_cast<double>(tau) : 0.;
            else
            {
                // beyond the last segment: PROP2 uses the last segment, FREE escapes
                b.m[idx] = iA;
                b.s[idx] = static_cast<double>(fC);
                b.found[idx] = 0;
            }
            kind = -1;
            if ((cross | rfStores) & 0x80000000u)
            {
                atomicAdd(&w.ctl->counters[1], static_cast<unsigned long long>(cross));
                atomicAdd(&w.ctl->counters[4], static_cast<unsigned long long>(rfStores));
                cross = rfStores = 0;
            }
        }
    }

    unsigned long long crossAll = cross, rfAll = rfStores;
    for (int off = 16; off > 0; off >>= 1)
    {
        crossAll += __shfl_down_sync(FULL, crossAll, off);
        rfAll += __shfl_down_sync(FULL, rfAll, off);
    }
    if (lane == 0)
    {
        if (crossAll) atomicAdd(&w.ctl->counters[1], crossAll);
        if (rfAll) atomicAdd(&w.ctl->counters[4], rfAll);
    }
}

// ---------------------------------------------------------------------------------------------
// shade kernels (one thread per completed task of one kind)
// ---------------------------------------------------------------------------------------------

// The record lambda of FluxRecorder::detect for one wavelength bin ell of instrument i
// (FluxRecorder.cpp:412-440 and the statistics at :522-536): total, components, scattering levels
// of primary packets, per-history statistics, and the guiding pilot's record.
SKG_D void detectBin(const Wave& w, const Scene& sc, const InstrDev& in, int i, int slot, int l, int ell, int numScatt,
                     double L, double Lext)
{
    if (sc.guideMode == 1 && i == sc.guideTarget)
    {
        // pilot records: the history's detected luminosity in the target instrument
        double wp = (sc.guideImportance && l >= 0) ? static_cast<double>(sc.guideImportance[l]) : 1.0;
        atomicAdd(w.pk.gD + slot, Lext * wp);
    }
    size_t plane = static_cast<size_t>(in.npx) * in.npy * in.nbins;
    size_t at = in.kind == 0 ? static_cast<size_t>(l) + static_cast<size_t>(ell) * in.npx * in.npy
                             : static_cast<size_t>(ell);
    atomicAddAgg((in.kind == 0 ? in.ifu : in.sed) + at, Lext);
    if (in.comps)
    {
        double* c = in.kind == 0 ? in.ifuComp : in.sedComp;
        if (numScatt == 0)
        {
            atomicAddAgg(c + at, L);
            atomicAddAgg(c + plane + at, Lext);
        }
        else
        {
            atomicAddAgg(c + 2 * plane + at, Lext);
            if (numScatt <= in.levels && !sc.sec) atomicAddAgg(c + (2 + numScatt) * plane + at, Lext);
        }
    }
    if (in.stats)
    {
        unsigned long long key = (static_cast<unsigned long long>(i) << 48) | (static_cast<unsigned long long>(ell) << 24)
                                 | static_cast<unsigned long long>(l + 1);
        recordStat(w, slot, key, Lext);
    }
}

// FluxRecorder::detect for the instruments of one observer group (FluxRecorder.cpp:372-538)
static __global__ void __launch_bounds__(256) shadePeelKernel(const __grid_constant__ Wave w, int cur)
{
    unsigned n = w.ctl->qn[cur][K_PEEL];
    const TaskBuf& b = w.q[cur][K_PEEL];
    unsigned long long det = 0;
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    {
        int slot = b.slot[t];
        const Scene& sc = slotScene(w, slot);
        int group = b.info[t] & 0xFF;
        int numScatt = b.info[t] >> 8;
        double Lp = b.par[t];
        double ext = exp(-b.tau[t]);
        double x = b.x[t], y = b.y[t], z = b.z[t];
        double lambda0 = w.pk.rec[slot].lam;
        for (int i = group; i < sc.ninstr && (i == group || sc.instr[i].same); ++i)
        {
            const InstrDev& in = sc.instr[i];
            int l = in.kind == 0 ? framePixel(in, x, y, z) : -1;
            if (in.kind == 0 && l < 0) continue;
            if (in.kind == 1 && !insideAperture(in, x, y, z)) continue;
            // the observer-frame wavelength (FluxRecorder.cpp:377-378)
            const double lambda = lambda0 * in.zfac;
            if (in.nband == 0)
            {
                // DisjointWavelengthGrid::bins: at most one bin, transmission 1
                int ell = wlgBin(sc.wlgB + in.woff, in.wnb, sc.wlgEll + in.woff, lambda);
                if (ell < 0) continue;
                det++;
                detectBin(w, sc, in, i, slot, l, ell, numScatt, Lp, Lp * ext);
            }
            else
            {
                // BandWavelengthGrid::bins: every band whose range holds the wavelength
                for (int ell = 0; ell < in.nband; ++ell)
                {
                    int b0 = in.bandBeg[ell], size = in.bandBeg[ell + 1] - b0;
                    const double* lv = in.bandLam + b0;
                    if (!(lambda >= lv[0] && lambda <= lv[size - 1])) continue;
                    double L = Lp * bandTransmission(lv, in.bandTr + b0, size, in.bandW[ell], lambda);
                    det++;
                    detectBin(w, sc, in, i, slot, l, ell, numScatt, L, L * ext);
                }
            }
        }
    }
    if (det) atomicAdd(&w.ctl->counters[3], det);
}

// forced scattering: sample the interaction optical depth (simulateForcedPropagation)
static __global__ void __launch_bounds__(256) shadeProp1Kernel(const __grid_constant__ Wave w, int cur, int nxt)
{
    unsigned n = w.ctl->qn[cur][K_PROP1];
    const TaskBuf& b = w.q[cur][K_PROP1];
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    {
        int slot = b.slot[t];
        double taupath = b.tau[t];
        const Scene& sc = slotScene(w, slot);
        if (sc.explicitAbs)
        {
            // explicit absorption samples on the scattering optical depth of the path: for one medium
            // with constant cross sections tau_sca = tau_ext * sca / ext (the trace accumulated
            // extinction for the radiation field)
            int ell = w.pk.rec[slot].ellMix;
            double ext = sc.mixExt[ell];
            taupath = ext > 0. ? taupath * (sc.mixSca[ell] / ext) : 0.;
        }
        if (taupath <= 0.)
        {
            w.pk.rec[slot].L *= 0.;
            endHistory(w, slot);
            continue;
        }
        Rng rng;
        loadRng(w, slot, rng);
        double xi = sc.pathLengthBias;
        double tau;
        if (xi == 0.)
            tau = exponCutoff(rng, taupath);
        else
        {
            tau = rng.uniform() < xi ? rng.uniform() * taupath : exponCutoff(rng, taupath);
            double p = -exp(-tau) / expm1(-taupath);
            double q = (1.0 - xi) * p + xi / taupath;
            w.pk.rec[slot].L *= p / q;
        }
        storeRng(w, slot, rng);
        w.pk.rec[slot].tauPath = taupath;
        emitProp(w, nxt, K_PROP2, slot, tau);
    }
}

// interaction point reached: weight, position, termination test, scattering peel-off and HG
// scattering, next propagation (MonteCarloSimulation.cpp:645-665, 670-683)
// pilot record of a scattering event (guiding mode 1): the open record of the previous event gets
// its start value (its own peel-off has been detected by now), and this event is recorded with
// probability guideRecFrac, decided by a hash of history and event index so that the packet's
// random stream is untouched
SKG_D void guideRecord(const Wave& w, int slot, int nscatt, double x, double y, double z, double kx0, double ky0,
                       double kz0, double kx, double ky, double kz, double L)
{
    const Scene& sc = slotScene(w, slot);
    int pend = w.pk.gPend[slot];
    if (pend >= 0)
    {
        sc.guideRec[pend].dStart = w.pk.gD[slot];
        w.pk.gPend[slot] = -1;
    }
    unsigned long long h = w.pk.rec[slot].hist;
    U4 r = philox4x32_10(U4{static_cast<uint32_t>(nscatt), 0x67756964u, static_cast<uint32_t>(h), static_cast<uint32_t>(h >> 32)},
                         static_cast<uint32_t>(sc.seed), static_cast<uint32_t>(sc.seed >> 32) ^ 0x5bd1e995u);
    if (static_cast<float>(r.x) * 2.3283064e-10f >= sc.guideRecFrac) return;
    unsigned long long idx = atomicAdd(sc.guideRecCount, 1ULL);
    if (idx >= sc.guideRecCap) return;
    GuideRecord& q = sc.guideRec[idx];
    guideFeatures(q.f, x, y, z, kx0, ky0, kz0, w.pk.rec[slot].lam, w.pk.rec[slot].tauPath, sc.g.ext);
    q.k[0] = static_cast<float>(kx);
    q.k[1] = static_cast<float>(ky);
    q.k[2] = static_cast<float>(kz);
    q.I = 0.f;
    q.dStart = 0.;
    q.L = static_cast<float>(L);
    q.prev = w.pk.gLast[slot];
    w.pk.gLast[slot] = static_cast<int>(idx);
    w.pk.gPend[slot] = static_cast<int>(idx);
}

// tauInt: the interaction optical depth (PROP2: the sampled one within the path; FREE: the drawn
// one), which under explicit absorption is a scattering optical depth
SKG_D void interact(const Wave& w, int cur, int nxt, int slot, int m, double sInt, bool forced, double tauInt)
{
    const Scene& sc = slotScene(w, slot);
    if (m < 0)
    {
        atomicOr(&w.ctl->err, 2);  // MediumSystem::albedoForScattering: cannot locate the interaction point
        endHistory(w, slot);
        return;
    }
    int ell = w.pk.rec[slot].ellMix;
    double L = w.pk.rec[slot].L;
    if (sc.explicitAbs)
    {
        // absorption optical depth at the interaction point: tau_int * abs / sca for one medium with
        // constant cross sections (MediumSystem.cpp:2216-2220); applied as exp(-tau_abs)
        // (MonteCarloSimulation.cpp:1531-1535, 2001-2010)
        double sca = sc.mixSca[ell];
        double tauAbs = tauInt * (sc.mixExt[ell] - sca) / sca;
        if (forced)
            L *= -expm1(-w.pk.rec[slot].tauPath) * exp(-tauAbs);
        else
            L *= exp(-tauAbs);
    }
    else
    {
        double albedo = albedoAt(sc, m, sc.mixSca[ell], sc.mixExt[ell]);
        if (forced)
            L *= -expm1(-w.pk.rec[slot].tauPath) * albedo;
        else
            L *= albedo;
    }
    w.pk.rec[slot].L = L;
    double kx = w.pk.rec[slot].kx, ky = w.pk.rec[slot].ky, kz = w.pk.rec[slot].kz;
    double x = w.pk.rec[slot].x + sInt * kx;
    double y = w.pk.rec[slot].y + sInt * ky;
    double z = w.pk.rec[slot].z + sInt * kz;
    w.pk.rec[slot].x = x;
    w.pk.rec[slot].y = y;
    w.pk.rec[slot].z = z;
    w.pk.rec[slot].cell = m;
    int nscatt = w.pk.rec[slot].nscatt;
    // termination (performLifeCycle, MonteCarloSimulation.cpp:643-660). Under guided scattering the
    // test applies to the weight without the guiding factors, so that termination depends on the
    // path alone and the guided runs estimate the same quantity as plain ones (in optically thick
    // media the threshold L0/minWeightReduction is not small against the emergent flux)
    double Lterm = L;
    if (sc.guideMode == 2 && w.pk.gRatio[slot] > 0.f) Lterm = L / static_cast<double>(w.pk.gRatio[slot]);
    if (L <= 0 || (forced && Lterm <= w.pk.rec[slot].Lth && nscatt >= sc.minScatt))
    {
        endHistory(w, slot);
        return;
    }
    double g = sc.mixG[ell];
    if (sc.peel && sc.ninstr > 0) emitPeels(w, nxt, slot, true, nscatt + 1, L, g, x, y, z, kx, ky, kz);
    Rng rng;
    loadRng(w, slot, rng);
    if (nscatt >= MAX_SCATT_EVENTS)
    {
        atomicOr(&w.ctl->err, 8);  // a history that never meets its termination criterion
        endHistory(w, slot);
        return;
    }
    if (sc.guideMode == 2)
    {
        // the guided-scattering stage of this pass samples the new direction (no draw made here)
        const TaskBuf& gb = w.q[cur][K_GUIDE];
        unsigned i = warpAppend(&w.ctl->qn[cur][K_GUIDE]);
        gb.slot[i] = slot;
        return;
    }
    double kx0 = kx, ky0 = ky, kz0 = kz;
    scatterHG(rng, g, kx, ky, kz);
    w.pk.rec[slot].kx = kx;
    w.pk.rec[slot].ky = ky;
    w.pk.rec[slot].kz = kz;
    w.pk.rec[slot].nscatt = nscatt + 1;
    atomicAdd(&w.ctl->counters[2], 1ULL);
    if (sc.guideMode == 1) guideRecord(w, slot, nscatt, x, y, z, kx0, ky0, kz0, kx, ky, kz, L);
    beginPropagation(w, nxt, slot, rng);
    storeRng(w, slot, rng);
}

// Guided scattering of one packet from the network's raw outputs: the composite density
// alpha * q_mix + (1 - alpha) * p_HG is sampled and the weight multiplied by p_HG / composite,
// which is returned.
SKG_D double guidedScatter(const Wave& w, int nxt, int slot, const float* o)
{
    const Scene& sc = slotScene(w, slot);
    GuideMixture mix;
    guideMixture(o, mix);
    Rng rng;
    loadRng(w, slot, rng);
    double g = sc.mixG[w.pk.rec[slot].ellMix];
    double kx0 = w.pk.rec[slot].kx, ky0 = w.pk.rec[slot].ky, kz0 = w.pk.rec[slot].kz;
    double kx = kx0, ky = ky0, kz = kz0;
    float ratio = w.pk.gRatio[slot];
    double alpha = ratio <= GUIDE_RATIO_MAX ? static_cast<double>(sc.guideAlpha) : 0.0;
    if (alpha > 0.0 && rng.uniform() < alpha)
    {
        double u0 = rng.uniform(), u1 = rng.uniform(), u2 = rng.uniform();
        guideSample(mix, u0, u1, u2, kx, ky, kz);
    }
    else
    {
        scatterHG(rng, g, kx, ky, kz);
    }
    double p = pdfHG(g, kx * kx0 + ky * ky0 + kz * kz0);
    double q = exp(static_cast<double>(guideLogDensity(mix, kx, ky, kz)));
    double den = alpha * q + (1.0 - alpha) * p;
    double wgt = p / den;
    if (!(den > 0.) || !isfinite(den) || !(wgt >= 0.) || !isfinite(wgt))
    {
        atomicOr(&w.ctl->err, 32);  // non-finite guiding density or weight: the packet is dropped and flagged
        wgt = 0.;
    }
    w.pk.rec[slot].L *= wgt;
    w.pk.gRatio[slot] = static_cast<float>(ratio * wgt);
    w.pk.rec[slot].kx = kx;
    w.pk.rec[slot].ky = ky;
    w.pk.rec[slot].kz = kz;
    w.pk.rec[slot].nscatt += 1;
    atomicAdd(&w.ctl->counters[2], 1ULL);
    beginPropagation(w, nxt, slot, rng);
    storeRng(w, slot, rng);
    return wgt;
}

// guided-scattering stage: the network runs on the tensor cores for 128 queued events per tile
static __global__ void __launch_bounds__(GM_TILE) guideScatterKernel(const __grid_constant__ Wave w, int cur, int nxt)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const Scene& sc = w.sc;  // the network (guiding is not offered in batched runs)
    unsigned n = w.ctl->qn[cur][K_GUIDE];
    if (blockIdx.x * GM_TILE >= n) return;  // uniform per CTA, before any tensor memory is taken
    const TaskBuf& b = w.q[cur][K_GUIDE];
    GuideTile t;
    guideTileBegin(t, smem, sc.guideBlob);
    bool failed = false;  // uniform across the CTA
    double wsum = 0.;
    unsigned wcount = 0;
    for (unsigned tile = blockIdx.x; tile * GM_TILE < n; tile += gridDim.x)
    {
        unsigned i = tile * GM_TILE + threadIdx.x;
        bool valid = i < n;
        int slot = valid ? b.slot[i] : 0;
        float f[GUIDE_IN], o[GUIDE_OUT];
        if (valid)
            guideFeatures(f, w.pk.rec[slot].x, w.pk.rec[slot].y, w.pk.rec[slot].z, w.pk.rec[slot].kx, w.pk.rec[slot].ky, w.pk.rec[slot].kz,
                          w.pk.rec[slot].lam, w.pk.rec[slot].tauPath, slotScene(w, slot).g.ext);
        else
            for (int k = 0; k < GUIDE_IN; ++k) f[k] = 0.f;
        if (!failed && !guideTileForward(t, f, o))
        {
            failed = true;
            if (threadIdx.x == 0) atomicOr(&w.ctl->err, 16);
        }
        if (!valid) continue;
        if (failed)
        {
            endHistory(w, slot);  // the run reports the error; the history is not continued
        }
        else
        {
            wsum += guidedScatter(w, nxt, slot, o);
            wcount++;
        }
    }
    guideTileEnd(t);
    // mean weight factor diagnostics: one atomic per warp
    for (int off = 16; off > 0; off >>= 1)
    {
        wsum += __shfl_down_sync(0xffffffffu, wsum, off);
        wcount += __shfl_down_sync(0xffffffffu, wcount, off);
    }
    if ((threadIdx.x & 31) == 0 && wcount)
    {
        atomicAdd(&w.ctl->guideWeightSum, wsum);
        atomicAdd(&w.ctl->guideEvents, static_cast<unsigned long long>(wcount));
    }
}

static __global__ void __launch_bounds__(256) shadeProp2Kernel(const __grid_constant__ Wave w, int cur, int nxt)
{
    unsigned n = w.ctl->qn[cur][K_PROP2];
    const TaskBuf& b = w.q[cur][K_PROP2];
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        interact(w, cur, nxt, b.slot[t], b.m[t], b.s[t], true, b.par[t]);
}

static __global__ void __launch_bounds__(256) shadeFreeKernel(const __grid_constant__ Wave w, int cur, int nxt)
{
    unsigned n = w.ctl->qn[cur][K_FREE];
    const TaskBuf& b = w.q[cur][K_FREE];
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    {
        if (!b.found[t])
            endHistory(w, b.slot[t]);  // the interaction point is outside the path: the packet escapes
        else
            interact(w, cur, nxt, b.slot[t], b.m[t], b.s[t], false, b.par[t]);
    }
}

// ---------------------------------------------------------------------------------------------
// launch
// ---------------------------------------------------------------------------------------------
static __global__ void launchPrepKernel(const __grid_constant__ Wave w, int nxt)
{
    Control* c = w.ctl;
    unsigned long long remaining = w.count - c->launched;
    int n = static_cast<int>(min(static_cast<unsigned long long>(c->freeTop), remaining));
    c->nLaunch = n;
    c->launchBase = c->freeTop - n;
    c->freeTop -= n;
    c->launchHist0 = w.first + c->launched;
    c->launched += n;
    c->traceCursor = 0;
    c->traceCursor2 = 0;
    for (int k = 0; k < NUM_KINDS; ++k) c->qn[1 - nxt][k] = 0;  // the buffer consumed by this pass
}

static __global__ void __launch_bounds__(256) launchKernel(const __grid_constant__ Wave w, int nxt)
{
    int n = w.ctl->nLaunch;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    {
        int slot = w.pk.freeSlots[w.ctl->launchBase + t];
        unsigned long long hist = w.ctl->launchHist0 + t;
        if (w.order) hist = w.first + w.order[hist - w.first];  // wavelength-ordered launch
        if (w.nScenes > 1)
        {
            // batch history -> (scene, segment history of that scene)
            int sid = 0;
            while (sid + 1 < w.nScenes && hist >= w.prefix[sid + 1]) ++sid;
            w.pk.rec[slot].scene = sid;
            hist = w.sfirst[sid] + (hist - w.prefix[sid]);
        }
        const Scene& sc = slotScene(w, slot);
        Rng rng;
        rng.start(sc.seed, hist);
        Launched o = launchPacket(sc, hist, rng);
        w.pk.rec[slot].hist = hist;
        w.pk.rec[slot].x = o.x; w.pk.rec[slot].y = o.y; w.pk.rec[slot].z = o.z;
        w.pk.rec[slot].kx = o.kx; w.pk.rec[slot].ky = o.ky; w.pk.rec[slot].kz = o.kz;
        w.pk.rec[slot].L = o.L;
        w.pk.rec[slot].Lth = o.L / sc.minWeightRed;
        w.pk.rec[slot].lam = o.lambda;
        w.pk.rec[slot].nscatt = 0;
        int ell = sc.nmix > 0 ? max(0, locateClip(sc.mixLb, sc.nmix, o.lambda)) : 0;  // DustMix::indexForLambda
        w.pk.rec[slot].ellMix = ell;
        w.pk.rec[slot].ellRF = sc.rfOn ? wlgBin(sc.rfB, sc.rfNb, sc.rfEll, o.lambda) : -1;
        if (w.anyStats) w.pk.nstat[slot] = 0;
        w.pk.rec[slot].cell = -1;
        if (sc.guideMode == 2) w.pk.gRatio[slot] = 1.f;
        if (sc.guideMode == 1)
        {
            w.pk.gD[slot] = 0.;
            w.pk.gLast[slot] = -1;
            w.pk.gPend[slot] = -1;
        }
        atomicAdd(&w.ctl->counters[0], 1ULL);
        if (!(o.L > 0))
        {
            storeRng(w, slot, rng);
            endHistory(w, slot);
            continue;
        }
        if (sc.peel && sc.ninstr > 0) emitPeels(w, nxt, slot, false, 0, o.L, 0., o.x, o.y, o.z, 0., 0., 0.);
        beginPropagation(w, nxt, slot, rng);
        storeRng(w, slot, rng);
    }
}

static __global__ void initPoolKernel(const __grid_constant__ Wave w)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < w.P; t += gridDim.x * blockDim.x)
    {
        w.pk.freeSlots[t] = t;
        if (w.anyStats)
        {
            w.pk.nstat[t] = 0;
            for (int a = 0; a < w.statCap; ++a) w.pk.skey[static_cast<size_t>(t) * w.statCap + a] = ~0ULL;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        Control* c = w.ctl;
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < NUM_KINDS; ++k) c->qn[b][k] = 0;
        c->traceCursor = 0;
        c->traceCursor2 = 0;
        c->freeTop = w.P;
        c->nLaunch = 0;
        c->launchBase = 0;
        c->launched = 0;
        c->done = 0;
        c->launchHist0 = 0;
        for (int k = 0; k < 8; ++k) c->counters[k] = 0;
        c->spillN = 0;
        c->guideWeightSum = 0.;
        c->guideEvents = 0;
        c->err = 0;
    }
}

// ---------------------------------------------------------------------------------------------
// Wavelength-ordered launch. Each history draws its own Philox stream, so the order in which the
// pool takes up histories changes no history, only which histories are in flight together. Taking
// them up in order of wavelength keeps the packets in flight on a few wavelength bins at a time, so
// that the tallies they update (radiation field m*nbins + ell, frames l + ell*npix) and the dust
// tables they read stay within a few L2-resident slices instead of spreading over the full arrays.
// The order is a counting sort of the segment's histories by the top bits of their launch
// wavelength as an FP32 number: 14 bits for one scene (32 buckets per octave). A batch keeps its
// histories grouped by scene (its meshes are separate working sets) and sorts by wavelength within
// each scene: the scene id takes the top sceneBits of the 14-bit key.
// ---------------------------------------------------------------------------------------------
SKG_D unsigned orderBucket(double lambda, int lambdaBits)
{
    // positive FP32: sign bit 0, the top lambdaBits of the remaining 31 bits
    return __float_as_uint(static_cast<float>(lambda)) >> (31 - lambdaBits);
}

// the launch wavelength of every history of the range (the launch draws of launchKernel), its
// bucket in keys[] and the bucket counts
static __global__ void __launch_bounds__(256) orderKeyKernel(const __grid_constant__ Wave w, int sceneBits,
                                                             unsigned short* keys, unsigned* counts)
{
    for (unsigned long long off = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; off < w.count;
         off += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
    {
        unsigned long long hist = w.first + off;
        const Scene* sc = &w.sc;
        int sid = 0;
        if (w.nScenes > 1)
        {
            while (sid + 1 < w.nScenes && hist >= w.prefix[sid + 1]) ++sid;
            sc = w.scenes + sid;
            hist = w.sfirst[sid] + (hist - w.prefix[sid]);
        }
        Rng rng;
        rng.start(sc->seed, hist);
        Launched o = launchPacket(*sc, hist, rng);
        const int lambdaBits = 14 - sceneBits;
        unsigned key = (static_cast<unsigned>(sid) << lambdaBits) | orderBucket(o.lambda, lambdaBits);
        key = min(key, static_cast<unsigned>(ORDER_BUCKETS - 1));
        keys[off] = static_cast<unsigned short>(key);
        // one atomic per distinct key of the warp
        unsigned active = __activemask();
        unsigned peers = __match_any_sync(active, key);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(counts + key, static_cast<unsigned>(__popc(peers)));
    }
}

// exclusive scan of the bucket counts into bucket cursors (one block of 1024 threads)
static __global__ void __launch_bounds__(1024) orderScanKernel(const unsigned* counts, unsigned* cursor)
{
    constexpr int PER = ORDER_BUCKETS / 1024;
    __shared__ unsigned part[1024];
    unsigned local[PER];
    unsigned sum = 0;
    for (int i = 0; i < PER; ++i)
    {
        local[i] = sum;
        sum += counts[threadIdx.x * PER + i];
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1)
    {
        unsigned v = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned base = part[threadIdx.x] - sum;
    for (int i = 0; i < PER; ++i) cursor[threadIdx.x * PER + i] = base + local[i];
}

// scatter: order[position] = history offset, positions taken per bucket
static __global__ void __launch_bounds__(256) orderScatterKernel(unsigned long long count, const unsigned short* keys,
                                                                 unsigned* cursor, unsigned* order)
{
    for (unsigned long long off = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; off < count;
         off += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
    {
        unsigned key = keys[off];
        unsigned active = __activemask();
        unsigned peers = __match_any_sync(active, key);
        int lane = threadIdx.x & 31;
        int leader = __ffs(peers) - 1;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(cursor + key, static_cast<unsigned>(__popc(peers)));
        base = __shfl_sync(peers, base, leader);
        order[base + __popc(peers & ((1u << lane) - 1))] = static_cast<unsigned>(off);
    }
}

}  // namespace skg

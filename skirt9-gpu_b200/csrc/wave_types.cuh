// Data layout of the wavefront life cycle: the packet pool (structure of arrays), the task
// buffers of the four traversal kinds (plus the guided-scattering queue), and the control block.
#pragma once

#include "physics.cuh"

namespace skg {

// K_GUIDE is not traversed: it queues the scattering events whose new direction the guiding
// network samples (filled and consumed within one pass)
enum TaskKind { K_PEEL = 0, K_PROP1 = 1, K_PROP2 = 2, K_FREE = 3, K_GUIDE = 4, NUM_KINDS = 5 };

// The state of one packet slot that the stage kernels and the traversal kernel's task start read:
// one 128-byte line, so that a packet taken from a task queue (slots in no particular order) costs
// one line instead of a sector from each of eighteen arrays.
struct alignas(128) PacketRec
{
    double x, y, z, kx, ky, kz;
    double L, Lth, lam, tauPath;
    unsigned long long hist;
    double rngSpare;
    unsigned rngCtr;
    int rngHas;
    int nscatt, ellMix, ellRF;
    int cell;   // cell of the last interaction (-1 after launch): start-cell hint of the next rays
    int scene;  // batched runs: the scene (simulation) of the slot's history
    int pad;
};
static_assert(sizeof(PacketRec) == 128, "one line per packet");

// A per-history statistics contribution that did not fit its slot's buffer; the history's buffered
// contributions join it when the history ends, and all are grouped per history after the run. The
// same record carries the grouped sums to the kernel that adds their moments.
struct StatSpill
{
    unsigned long long hist;
    unsigned long long key;  // instrument << 48 | wavelength bin << 24 | pixel + 1
    double w;
    int scene;
    int pad;
};

struct PacketPool
{
    PacketRec* rec;  // P
    // per-history statistics buffer (only when an instrument records statistics): statCap distinct
    // (instrument, bin, pixel) keys per slot with their summed contributions; unused keys are ~0
    unsigned long long* skey;  // P * statCap
    double* sw;
    int* nstat;                // entries taken; above statCap the history has spilled
    StatSpill* spill;          // spill log of the run
    unsigned long long spillCap;
    int* freeSlots;            // P
    // pilot records of the guiding network: luminosity of the history detected by the target
    // instrument so far, last recorded event, event whose start value is still open
    double* gD;
    int *gLast, *gPend;
    // guided scattering: product of the packet's guiding weight factors so far
    float* gRatio;
};

// one buffer of one task kind
struct TaskBuf
{
    int* slot;
    int* info;      // PEEL: first instrument of the observer group | numScatt << 8
    double* par;    // PEEL: peel-off luminosity; PROP2/FREE: interaction optical depth
    double *x, *y, *z;  // PEEL: origin (the packet position at the event)
    // results written by the trace kernel
    double* tau;    // PEEL / PROP1: optical depth (PROP1: of the complete path)
    int* m;         // PROP2 / FREE: interaction cell (-1: none)
    double* s;      // PROP2 / FREE: interaction distance
    int* found;     // FREE: interaction point inside the path
};

struct Control
{
    unsigned qn[2][NUM_KINDS];  // task counts per buffer and kind
    unsigned traceCursor;   // next task of the pass (all kinds, or the peel-off kernel's)
    unsigned traceCursor2;  // next propagation task of the pass (propagation kernel)
    int freeTop;
    int nLaunch;
    int launchBase;
    unsigned long long launched;
    unsigned long long done;
    unsigned long long launchHist0;
    // histories, crossings, scatterings, detections, rfStores, statistics contributions lost (spill
    // log full), contributions spilled, traversal-guard reports
    unsigned long long counters[8];
    unsigned long long spillN;       // entries written to the statistics spill log
    double guideWeightSum;           // guided scattering: sum of the weight factors (mean 1 in expectation)
    unsigned long long guideEvents;  // guided scattering events
    int err;
};

// Batched runs trace the histories of several independent scenes (simulations) through one
// wavefront: scene s owns the batch histories [prefix[s], prefix[s+1]), which are its segment
// histories first[s], first[s] + 1, ... With one scene, sc is that scene and scenes is null.
constexpr int MAX_BATCH = 48;
// buckets of the wavelength-ordered launch (top 14 bits of the FP32 wavelength)
constexpr int ORDER_BUCKETS = 1 << 14;
// a batch's scene table is staged in the traversal kernel's shared memory as int4 words, within the
// 48 KB available without an opt-in
static_assert(sizeof(Scene) % 16 == 0 && MAX_BATCH * sizeof(Scene) <= 48 * 1024, "scene table in shared memory");

struct Wave
{
    Scene sc;
    const Scene* scenes;               // device table of nScenes scenes (batched runs)
    int nScenes;
    const unsigned long long* prefix;  // nScenes + 1
    const unsigned long long* sfirst;  // nScenes: first segment history of each scene
    // launch shape (0: defaults): resident trace blocks per SM, shade blocks per SM, and the number
    // of waiting lanes at which a warp of the traversal kernel takes new tasks
    int traceBlocksPerSM, shadeBlocksPerSM, refillMin;
    // radiation-field updates of a warp summed per address before the atomic (SKGPU_RF_WARP_AGG=1)
    int rfAgg;
    // launch order: histories first + order[i] for i = 0, 1, ... (null: index order)
    const unsigned* order;
    PacketPool pk;
    TaskBuf q[2][NUM_KINDS];
    Control* ctl;
    int P;
    unsigned long long first, count;
    int anyStats;
    int statCap;  // per-slot statistics buffer entries
};

}  // namespace skg

// The state behind the opaque skgpu_ctx handle of include/skgpu.h (shared by the ABI translation
// units).
#pragma once

#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/skgpu.h"
#include "internal.hpp"
#include "stage_timer.hpp"

namespace skg { struct GuideState; }

using skg::GridDev;
using skg::InstrDev;
using skg::SourceDev;
using skg::StageTimer;
using skg::Wave;

struct skgpu_ctx
{
    int device = 0;
    int numSMs = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    double lastMs = 0.;

    GridDev g{};
    bool hasGrid = false;
    std::vector<void*> gridBufs;

    double* dens = nullptr;
    int numCells = 0;

    double *mixLb = nullptr, *mixExt = nullptr, *mixSca = nullptr, *mixG = nullptr;
    int nmix = 0;

    int nrf = 0, rfNb = 0;
    double* rfB = nullptr;
    int* rfEll = nullptr;
    double* rf = nullptr;
    size_t rfLen = 0;

    std::vector<SourceDev> srcHost;
    SourceDev* src = nullptr;
    double *tabL = nullptr, *tabA = nullptr, *tabB = nullptr, *radR = nullptr, *radP = nullptr;

    std::vector<InstrDev> instrHost;
    InstrDev* instr = nullptr;
    std::vector<void*> instrBufs;
    std::vector<size_t> instrBufLens;  // doubles per instrument buffer
    std::vector<void*> instrAux;       // band tables of the instruments
    double* wlgB = nullptr;
    int* wlgEll = nullptr;

    skgpu_options opt{};
    bool hasOptions = false;

    int* errFlag = nullptr;
    skgpu_counters lastCounters{};
    long long lastPasses = 0;
    double lastGuideWeightSum = 0.;
    unsigned long long lastGuideEvents = 0;

    // wavefront buffers (packet pool, task queues, control block), grown on demand
    Wave wave{};
    int waveP = 0, waveGroups = 0, waveStats = 0;
    std::vector<void*> waveBufs;
    unsigned long long* doneHost = nullptr;  // pinned progress word

    // device timing of the stage kernels (skgpu_set_stage_timing)
    StageTimer timer;
    bool timerEvents = false;

    // pinned staging of the tally read-back: the copy of one chunk overlaps the host add of the previous
    double* pin[2] = {nullptr, nullptr};
    cudaEvent_t pinEv[2] = {nullptr, nullptr};

    // launch shape set by skgpu_set_launch_shape (0: defaults)
    int shapePool = 0, shapeTraceBlocks = 0, shapeShadeBlocks = 0, shapeRefill = 0;
    // device tables of the last batched run (scene table, history prefix, first histories)
    std::vector<void*> batchBufs;
    // pass graph of the last run, replayed by the next run with the same parameters
    skg::GraphCache graphCache;
    // radiation field in the caller's layout (m * nbins + ell), transposed from the device tally at fetch
    double* rfT = nullptr;
    // wavelength-ordered launch (skgpu_set_history_order): mode, keys, order, bucket counts + cursors
    int historyOrder = 1;
    unsigned short* orderKeys = nullptr;
    unsigned* orderIdx = nullptr;
    unsigned* orderCounts = nullptr;
    size_t orderCap = 0;

    // learned path guiding (network, pilot records, optimizer state); null until first used
    skg::GuideState* guide = nullptr;

    // secondary (dust) emission: the equilibrium-emission tables (skgpu_upload_dust_emission), the
    // per-cell results and launch tables of the last skgpu_prepare_secondary, and the prepared source
    skg::DustEmissionDev de{};
    std::vector<void*> deBufs;        // the tables
    std::vector<double> deEmLHost;    // the dust-emission grid wavelengths (host copy)
    double deEmRange[2] = {0., 0.};
    int deCells = 0;
    std::vector<void*> secBufs;       // per-cell results and launch tables
    int secCells = 0, secNpts = 0;
    double *secL = nullptr, *secT = nullptr, *secPv = nullptr, *secCv = nullptr, *secXv = nullptr;
    double *secLv = nullptr, *secWv = nullptr;
    unsigned long long* secIv = nullptr;
    int* secCellNode = nullptr;
    skg::SecondaryDev* secDev = nullptr;
    uint64_t secPackets = 0;          // packets of the prepared segment (0: not prepared)
    double secLuminosity = 0.;
};

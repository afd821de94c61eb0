// Host-side state and entry points of the learned path guiding (implemented in guide.cu).
#pragma once

#include <cuda_runtime.h>

#include "guide.cuh"

struct skgpu_ctx;

namespace skg {

struct GuideState
{
    float* params = nullptr;          // FP32 master parameters (GUIDE_NPARAMS)
    unsigned char* blob = nullptr;    // packed BF16 network of the tensor-core inference
    float *adamM = nullptr, *adamV = nullptr, *grad = nullptr;
    long long adamStep = 0;
    bool hasParams = false;

    GuideRecord* records = nullptr;   // pilot records
    unsigned long long* recCount = nullptr;
    unsigned long long recCapacity = 0;

    float *scratchIn = nullptr, *scratchH = nullptr, *scratchDelta = nullptr, *lossAcc = nullptr;
    int scratchRows = 0;

    float* importance = nullptr;      // per-pixel weights of the target frame
    int importanceLen = 0;
    int* errFlag = nullptr;

    // training target: records weighted by I / (mean I of their position bin) when positionBins > 0
    // (every region of the domain gets the same total weight), by I / (mean I) otherwise
    int positionBins = 0;
    float* binMean = nullptr;         // positionBins^3

    int mode = 0;                     // 0 off, 1 pilot records, 2 guided scattering
    int target = 0;
    float alpha = 0.5f;
    float recordFraction = 1.f;

    ~GuideState();
};

cudaError_t guideEnsure(skgpu_ctx* ctx);
void guideDestroy(skgpu_ctx* ctx);
cudaError_t guideSetParams(skgpu_ctx* ctx, const float* host);
cudaError_t guideGetParams(skgpu_ctx* ctx, float* host);
cudaError_t guideRepack(skgpu_ctx* ctx);
cudaError_t guideLossGrad(skgpu_ctx* ctx, int n, const float* in, const float* k, const float* w, float* loss, float* grad);
cudaError_t guideInfer(skgpu_ctx* ctx, int n, const float* in, float* out, int tensorCores, int* deviceErr);
cudaError_t guideEnsureRecords(skgpu_ctx* ctx, unsigned long long capacity);
cudaError_t guideRecordCount(skgpu_ctx* ctx, unsigned long long* n);
cudaError_t guideFetchRecords(skgpu_ctx* ctx, unsigned long long n, float* out);
cudaError_t guideTrain(skgpu_ctx* ctx, int steps, int batch, float lr, unsigned long long seed, float* lossOut);

}  // namespace skg

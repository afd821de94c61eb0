// FP32-traversal life-cycle kernels. Walkers with FP32 traversal state are added per grid kind;
// a grid kind without one is reported as unsupported (there is no silent FP64 substitution).
#include "internal.hpp"

namespace skg {

int lifecycleBlocksPerSMFP32(int, int) { return 1; }

cudaError_t launchLifecycleFP32(int, const LCParams&, int, int, cudaStream_t) { return cudaErrorNotSupported; }

}  // namespace skg

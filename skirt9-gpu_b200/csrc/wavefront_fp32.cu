// Wavefront life cycle with FP32 traversal walkers. A grid kind without an FP32 walker is
// reported as unsupported; there is no silent substitution of the FP64 walkers.
#include "internal.hpp"


namespace skg {

cudaError_t runWaveFP32(int, const Wave&, int, cudaStream_t, unsigned long long*, long long*, long long)
{
    return cudaErrorNotSupported;
}

}  // namespace skg

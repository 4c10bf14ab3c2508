// Fused elastic step kernels for __half storage, float arithmetic (templates in fused_step.cuh).
#include "fused_step.cuh"

namespace tw {
template cudaError_t prepare_fused<__half, float>();
template void launch_fused<__half, float>(const FusedArgs<__half, float> &, int, bool, bool, cudaStream_t);
}  // namespace tw

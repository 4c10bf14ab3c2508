// Fused elastic step kernels for float storage, float arithmetic (templates in fused_step.cuh).
#include "fused_step.cuh"

namespace tw {
template cudaError_t prepare_fused<float, float>();
template void launch_fused<float, float>(const FusedArgs<float, float> &, int, bool, bool, cudaStream_t);
}  // namespace tw

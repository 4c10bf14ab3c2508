// Fused elastic step kernels for __nv_bfloat16 storage, float arithmetic (templates in fused_step.cuh).
#include "fused_step.cuh"

namespace tw {
template cudaError_t prepare_fused<__nv_bfloat16, float>();
template void launch_fused<__nv_bfloat16, float>(const FusedArgs<__nv_bfloat16, float> &, int, bool, bool, cudaStream_t);
}  // namespace tw

// Fused elastic step kernels for double storage, double arithmetic (templates in fused_step.cuh).
#include "fused_step.cuh"

namespace tw {
template cudaError_t prepare_fused<double, double>();
template void launch_fused<double, double>(const FusedArgs<double, double> &, int, bool, bool, cudaStream_t);
}  // namespace tw

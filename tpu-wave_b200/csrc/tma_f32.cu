// The TMA-staged fused elastic step (tma_step.cuh) for FP32 fields and coefficients.
#include "tma_step.cuh"

namespace tw {

int tma_strips(long My)
{
    // strip k covers core columns [TMA_Y0 + k TMA_CORE, + TMA_CORE) and loads 4 more on each side;
    // the last loaded column must stay below My (never the seam column, never a wrapped one)
    const long need = TMA_Y0 + TMA_CORE + 4;
    return My >= need ? (int)((My - need) / TMA_CORE) + 1 : 0;
}

template <bool ENERGY>
static size_t tma_smem()
{
    return (size_t)TmaLayout<ENERGY>::bytes;
}

template <>
cudaError_t prepare_tma<float, float>()
{
    cudaError_t e = cudaFuncSetAttribute(k_elastic_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_smem<false>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_elastic_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_smem<true>());
}

template <>
void launch_tma<float, float>(const FusedArgs<float, float> &a, const TmaMaps &maps, bool energy, cudaStream_t st)
{
    const dim3 grid(a.n_zone * a.n_bstrip + a.n_octa + a.n_tcta), block(FS_THREADS_MAX);
    if (energy) k_elastic_tma<true><<<grid, block, tma_smem<true>(), st>>>(a, maps);
    else k_elastic_tma<false><<<grid, block, tma_smem<false>(), st>>>(a, maps);
}

}  // namespace tw

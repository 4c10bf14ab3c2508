// The TMA-staged fused elastic step (tma_step.cuh) for FP32 fields and coefficients.
#include <algorithm>

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

// dynamic shared memory of the side launch: the boundary CTAs' velocity tile or four warp rings
template <bool ENERGY>
static size_t side_smem(int tile_rows)
{
    return fused_smem_bytes<float, float, 0, ENERGY, float>(tile_rows);
}

template <>
cudaError_t prepare_tma<float, float>()
{
    cudaError_t e = cudaFuncSetAttribute(k_elastic_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_smem<false>());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_elastic_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_smem<true>());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_elastic_side<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)side_smem<false>(FS_SMALL_MX + 1));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_elastic_side<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)side_smem<true>(FS_SMALL_MX + 1));
}

// the side launch on a second stream forked from the handle's stream, the TMA strips on the
// handle's stream, joined back (in a captured graph: two parallel branches)
template <>
void launch_tma<float, float>(FusedArgs<float, float> a, const TmaMaps &maps, bool energy, cudaStream_t st,
                              cudaStream_t side_st, cudaEvent_t fork, cudaEvent_t join)
{
    // the TMA strips' persistent grid: as many CTAs as fit on the device at once, at most one per item
    static int resident[2] = {0, 0}, n_sm = 0;
    if (!n_sm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident[0], k_elastic_tma<false>, FS_THREADS_MAX, tma_smem<false>());
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident[1], k_elastic_tma<true>, FS_THREADS_MAX, tma_smem<true>());
    }
    const int per_sm = std::max(1, resident[energy ? 1 : 0]);
    const int n_side = a.n_zone * a.n_bstrip + a.n_octa, n_strips = std::min(a.n_tcta, per_sm * n_sm);
    a.n_all_ctas = n_side + n_strips;
    const dim3 block(FS_THREADS_MAX);
    cudaEventRecord(fork, st);
    cudaStreamWaitEvent(side_st, fork, 0);
    if (energy) {
        k_elastic_side<true><<<n_side, block, side_smem<true>(a.tile_rows), side_st>>>(a);
        k_elastic_tma<true><<<n_strips, block, tma_smem<true>(), st>>>(a, maps);
    } else {
        k_elastic_side<false><<<n_side, block, side_smem<false>(a.tile_rows), side_st>>>(a);
        k_elastic_tma<false><<<n_strips, block, tma_smem<false>(), st>>>(a, maps);
    }
    cudaEventRecord(join, side_st);
    cudaStreamWaitEvent(st, join, 0);
}

}  // namespace tw

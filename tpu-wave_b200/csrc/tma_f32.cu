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

template <bool ENERGY, bool Q16 = false>
static size_t tma_smem()
{
    return (size_t)TmaLayout<ENERGY, Q16>::bytes;
}

// dynamic shared memory of the side launch: the boundary CTAs' velocity tile or four warp rings
template <bool ENERGY>
static size_t side_smem(int tile_rows)
{
    return fused_smem_bytes<float, float, 0, ENERGY, float>(tile_rows);
}

template <bool ENERGY, bool Q16, bool WITEMS>
static cudaError_t tma_attr()
{
    return cudaFuncSetAttribute(k_elastic_tma<ENERGY, Q16, WITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)tma_smem<ENERGY, Q16>());
}

template <bool ENERGY>
static cudaError_t side_attr()
{
    return cudaFuncSetAttribute(k_elastic_side<ENERGY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)side_smem<ENERGY>(FS_SMALL_MX + 1));
}

template <>
cudaError_t prepare_tma<float, float>()
{
    cudaError_t e;
    if ((e = tma_attr<false, false, false>()) != cudaSuccess || (e = tma_attr<true, false, false>()) != cudaSuccess ||
        (e = tma_attr<false, true, false>()) != cudaSuccess || (e = tma_attr<true, true, false>()) != cudaSuccess ||
        (e = tma_attr<false, false, true>()) != cudaSuccess || (e = tma_attr<true, false, true>()) != cudaSuccess ||
        (e = tma_attr<false, true, true>()) != cudaSuccess || (e = tma_attr<true, true, true>()) != cudaSuccess)
        return e;
    if ((e = side_attr<false>()) != cudaSuccess) return e;
    return side_attr<true>();
}

// the TMA strips of one variant: a persistent grid of as many CTAs as fit on the device at once
template <bool ENERGY, bool Q16, bool WITEMS>
static void launch_strips(FusedArgs<float, float> &a, const TmaMaps &maps, int n_side, cudaStream_t st, bool go)
{
    static int resident = 0, n_sm = 0;
    if (!n_sm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_elastic_tma<ENERGY, Q16, WITEMS>, FS_THREADS_MAX,
                                                      tma_smem<ENERGY, Q16>());
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    }
    const int n_items = (WITEMS ? a.n_zone * a.n_bstrip + a.n_octa : 0) + a.n_tcta;
    const int n_strips = std::min(n_items, std::max(1, resident) * n_sm);
    a.n_all_ctas = n_side + n_strips;
    if (go) k_elastic_tma<ENERGY, Q16, WITEMS><<<n_strips, FS_THREADS_MAX, tma_smem<ENERGY, Q16>(), st>>>(a, maps);
}

template <bool WITEMS>
static void launch_strips_of(FusedArgs<float, float> &a, const TmaMaps &maps, bool energy, int n_side, cudaStream_t st,
                             bool go)
{
    switch ((energy ? 1 : 0) + (a.q16 ? 2 : 0)) {
    case 0: launch_strips<false, false, WITEMS>(a, maps, n_side, st, go); break;
    case 1: launch_strips<true, false, WITEMS>(a, maps, n_side, st, go); break;
    case 2: launch_strips<false, true, WITEMS>(a, maps, n_side, st, go); break;
    default: launch_strips<true, true, WITEMS>(a, maps, n_side, st, go); break;
    }
}

// the TMA strips on the handle's stream; the side launch, when there is one, on a second stream
// forked from it and joined back (in a captured graph: two parallel branches)
template <>
void launch_tma<float, float>(FusedArgs<float, float> a, const TmaMaps &maps, bool energy, cudaStream_t st,
                              cudaStream_t side_st, cudaEvent_t fork, cudaEvent_t join)
{
    if (a.witems) {   // one launch: boundary, warp-strip and TMA items
        launch_strips_of<true>(a, maps, energy, 0, st, false);   // (sets the CTA count the last CTA waits for)
        launch_strips_of<true>(a, maps, energy, 0, st, true);
        return;
    }
    const int n_side = a.n_zone * a.n_bstrip + a.n_octa;   // the boundary CTAs and the warp strips
    launch_strips_of<false>(a, maps, energy, n_side, st, false);
    cudaEventRecord(fork, st);
    cudaStreamWaitEvent(side_st, fork, 0);
    if (energy) k_elastic_side<true><<<n_side, FS_THREADS_MAX, side_smem<true>(a.tile_rows), side_st>>>(a);
    else k_elastic_side<false><<<n_side, FS_THREADS_MAX, side_smem<false>(a.tile_rows), side_st>>>(a);
    launch_strips_of<false>(a, maps, energy, n_side, st, true);
    cudaEventRecord(join, side_st);
    cudaStreamWaitEvent(st, join, 0);
}

}  // namespace tw

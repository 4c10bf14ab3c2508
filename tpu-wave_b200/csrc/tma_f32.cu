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

template <bool ENERGY, bool WITEMS>
static cudaError_t side_attr()
{
    return cudaFuncSetAttribute(k_elastic_side<ENERGY, WITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
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
    if ((e = side_attr<false, false>()) != cudaSuccess || (e = side_attr<true, false>()) != cudaSuccess ||
        (e = side_attr<false, true>()) != cudaSuccess)
        return e;
    return side_attr<true, true>();
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
    const int n_strips = std::min((WITEMS ? a.n_octa : 0) + a.n_tcta, std::max(1, resident) * n_sm);
    a.n_all_ctas = n_side + n_strips;
    if (go) k_elastic_tma<ENERGY, Q16, WITEMS><<<n_strips, FS_THREADS_MAX, tma_smem<ENERGY, Q16>(), st>>>(a, maps);
}

template <bool ENERGY, bool WITEMS>
static void launch_side(const FusedArgs<float, float> &a, int n_side, cudaStream_t side_st)
{
    k_elastic_side<ENERGY, WITEMS><<<n_side, FS_THREADS_MAX, side_smem<ENERGY>(a.tile_rows), side_st>>>(a);
}

template <bool WITEMS>
static void launch_pair(FusedArgs<float, float> &a, const TmaMaps &maps, bool energy, int n_side, cudaStream_t st,
                        cudaStream_t side_st, bool go)
{
    if (go) {
        if (energy) launch_side<true, WITEMS>(a, n_side, side_st);
        else launch_side<false, WITEMS>(a, n_side, side_st);
    }
    switch ((energy ? 1 : 0) + (a.q16 ? 2 : 0)) {
    case 0: launch_strips<false, false, WITEMS>(a, maps, n_side, st, go); break;
    case 1: launch_strips<true, false, WITEMS>(a, maps, n_side, st, go); break;
    case 2: launch_strips<false, true, WITEMS>(a, maps, n_side, st, go); break;
    default: launch_strips<true, true, WITEMS>(a, maps, n_side, st, go); break;
    }
}

// the side launch on a second stream forked from the handle's stream, the TMA strips on the
// handle's stream, joined back (in a captured graph: two parallel branches)
template <>
void launch_tma<float, float>(FusedArgs<float, float> a, const TmaMaps &maps, bool energy, cudaStream_t st,
                              cudaStream_t side_st, cudaEvent_t fork, cudaEvent_t join)
{
    // the boundary CTAs, and the warp strips unless they are items of the strips' launch
    const int n_side = a.n_zone * a.n_bstrip + (a.witems ? 0 : a.n_octa);
    // first the strips' grid size (it sets the CTA count the last CTA waits for), then the launches
    for (int pass = 0; pass < 2; pass++) {
        const bool go = pass == 1;
        if (go) {
            cudaEventRecord(fork, st);
            cudaStreamWaitEvent(side_st, fork, 0);
        }
        if (a.witems) launch_pair<true>(a, maps, energy, n_side, st, side_st, go);
        else launch_pair<false>(a, maps, energy, n_side, st, side_st, go);
    }
    cudaEventRecord(join, side_st);
    cudaStreamWaitEvent(st, join, 0);
}

}  // namespace tw

// Batched acoustic stepping: many independent shots (grids of any size) advanced by one launch
// per half-step instead of one per shot.
//
// The tiles of all shots form one list; tile t belongs to shot tile_shot[t], whose tiles are
// numbered row-major from tile_off. Each CTA walks the list with a stride of the grid size, so a
// grid smaller than the list is a persistent launch. Per point the update is the single-shot
// kernel's (acoustic.cuh), so a batched shot equals the same shot stepped alone bit for bit.
#include <algorithm>

#include "acoustic.cuh"

namespace tw {

template <class S, class C, int CPST, bool PERIODIC, int HALF>
__global__ void __launch_bounds__(256) k_batch_half(const BatchShot<S, C> *__restrict__ shots,
                                                    const int *__restrict__ tile_shot, int n_tiles, int rpt)
{
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const BatchShot<S, C> &sh = shots[tile_shot[t]];
        const int lt = t - sh.tile_off;
        const int tr = lt / sh.tiles_x, tc = lt - tr * sh.tiles_x;
        const int iy = tc * blockDim.x + threadIdx.x;
        const int ix0 = tr * blockDim.y * rpt + threadIdx.y;
        for (int q = 0; q < rpt; q++) {
            const int ix = ix0 + q * blockDim.y;
            if constexpr (HALF == 0) acoustic_velocity_point<S, C, CPST, PERIODIC>(sh.a, ix, iy);
            else acoustic_pressure_point<S, C, CPST, PERIODIC>(sh.a, ix, iy);
        }
    }
}

namespace {
template <class S, class C, int CPST, bool PERIODIC>
void launch_p(int half, const BatchShot<S, C> *shots, const int *tile_shot, int n_tiles, const BatchShape &b,
              cudaStream_t st)
{
    const dim3 block(b.tx, b.ty), grid(std::min(b.ctas, n_tiles));
    if (half == 0) k_batch_half<S, C, CPST, PERIODIC, 0><<<grid, block, 0, st>>>(shots, tile_shot, n_tiles, b.rpt);
    else k_batch_half<S, C, CPST, PERIODIC, 1><<<grid, block, 0, st>>>(shots, tile_shot, n_tiles, b.rpt);
}

template <class S, class C, int CPST>
void launch_c(int periodic, int half, const BatchShot<S, C> *shots, const int *tile_shot, int n_tiles,
              const BatchShape &b, cudaStream_t st)
{
    if (periodic) launch_p<S, C, CPST, true>(half, shots, tile_shot, n_tiles, b, st);
    else launch_p<S, C, CPST, false>(half, shots, tile_shot, n_tiles, b, st);
}
}  // namespace

// the batch accepts the single-core tree's compensation codes: '0', '3' (3R), '6' (6R)
template <class S, class C>
void launch_batch_half(int periodic, int cpst, int half, const BatchShot<S, C> *shots, const int *tile_shot,
                       int n_tiles, const BatchShape &b, cudaStream_t st)
{
    switch (cpst) {
    case 0: launch_c<S, C, 0>(periodic, half, shots, tile_shot, n_tiles, b, st); break;
    case 4: launch_c<S, C, 4>(periodic, half, shots, tile_shot, n_tiles, b, st); break;
    default: launch_c<S, C, 6>(periodic, half, shots, tile_shot, n_tiles, b, st); break;
    }
}

template void launch_batch_half<double, double>(int, int, int, const BatchShot<double, double> *, const int *, int,
                                                const BatchShape &, cudaStream_t);
template void launch_batch_half<float, float>(int, int, int, const BatchShot<float, float> *, const int *, int,
                                              const BatchShape &, cudaStream_t);

}  // namespace tw

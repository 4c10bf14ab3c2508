// Free surfaces on the two y ends with the fused elastic step. The fused kernel applies the
// periodic y rule at every column; a point whose y stencil, closure or penalty meets an end is
// then recomputed here from the step's input buffers with the SBP-SAT rules along y
// (stepper.cuh: dy_any, satN_y, satM_y), exactly as the per-point two-launch kernels compute it,
// and written over the fused kernel's value:
//   velocities: MN columns 0..3, My-3..My (DM closures, penalty at 0, My); NM columns 0..2,
//               My-3..My-1 (DN closures, penalties);
//   stresses:   NN columns 0..4, My-4..My and MM columns 0..5, My-5..My-1 (their closures and every
//               point whose x/y stencils read a recomputed velocity).
// Every other point reads no value of these columns (its y taps stay 3 or more columns from an
// end), so the fused kernel's values stand. The step's E_k and E_p1 records get, per recomputed
// point, the difference of its energy term (E_p0 reads the unchanged input state), and the
// receivers on recomputed points are recorded again.
#include "stepper.cuh"
#include "kernels.h"

namespace tw {

namespace {

constexpr int YF_THREADS = 256;

__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double red[YF_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.;
    if (threadIdx.x == 0)
        for (int w = 0; w < YF_THREADS / 32; w++) s += red[w];
    return s;
}

// the k-th recomputed column of a grid with n0 columns at its start and n1 at its end (length L)
__device__ __forceinline__ int fix_col(int k, int n0, int L, int n1) { return k < n0 ? k : L - n1 + (k - n0); }

template <class S, class C>
__device__ __forceinline__ void record(const YFixArgs<S, C> &a, int it, int slot, int row, int col, double v)
{
    for (int q = 0; q < a.n_rcv; q++) {
        const int *e = a.rcv + 4 * q;
        if (e[2] != row || e[3] != col) continue;
        if (e[0] == slot) a.traces[(2L * q) * a.max_steps + it] = v;
        if (e[1] == slot) a.traces[(2L * q + 1) * a.max_steps + it] = v;
    }
}

template <class S, class C, int CPST>
__device__ __forceinline__ C finish(const YFixArgs<S, C> &a, int f, long i, C s, C r, C c, bool src, int it)
{
    if (src) s = to_s<C>(add((double)s, a.src_inc[it]));
    if (!finite(s)) atomicOr(a.flags, FLAG_NONFINITE);
    a.out[f][i] = to_s<S>(s);
    if constexpr (Cpst<CPST>::keep_r) a.rout[f][i] = to_s<S>(r);
    if constexpr (Cpst<CPST>::keep_c) a.rout[f][i] = to_s<S>(c);
    return s;
}

template <class S, class C, int CPST>
__device__ __forceinline__ void load_rc2(const S *res, long i, C &r, C &c)
{
    r = C(0);
    c = C(0);
    if constexpr (Cpst<CPST>::keep_r) r = to_c<C>(res[i]);
    if constexpr (Cpst<CPST>::keep_c) c = to_c<C>(res[i]);
}

// velocities: blockIdx.y selects MN (0) or NM (1); threads walk (row, recomputed column)
template <class S, class C, int CPST>
__global__ void __launch_bounds__(YF_THREADS) k_ysat_vel(YFixArgs<S, C> a)
{
    const int it = *a.step - 1;
    const int Mx = a.Mx, My = a.My;
    const long pitch = a.pitch;
    const bool mn = blockIdx.y == 0;
    const int ncol = mn ? 8 : 6, rows = mn ? Mx : Mx + 1;
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double de = 0.;
    if (k < (long)rows * ncol) {
        const int ix = (int)(k / ncol), iy = mn ? fix_col((int)(k % ncol), 4, My + 1, 4) : fix_col((int)(k % ncol), 3, My, 3);
        const long i = (long)ix * pitch + iy;
        const int f = mn ? F_MN : F_NM;
        C r, c;
        load_rc2<S, C, CPST>(a.rin[f], i, r, c);
        const C P = __ldg(a.coef[f] + i);
        C v;
        if (mn) {   // x from NN (+ SAT), y from syy (closures, penalty)
            v = dx_from_N<C>(a.op, a.in[F_NN], pitch, Mx, ix, iy);
            r = add(r, mul(v, P));
            const bool sx = a.xif ? satM_if<C>(a.op, Mx, ix, [&](int q) { return ld<C>(a.in[F_NN], (long)q * pitch + iy); }, v)
                                  : sat_MN<C>(a.op, a.in[F_NN], pitch, Mx, ix, iy, v);
            if (sx) r = add(r, mul(v, P));
            const S *m1 = a.in[F_MM1] + (long)ix * pitch;
            v = dy_sbp<false, C>(a.op, m1, My, iy);
            r = add(r, mul(v, P));
            if (satN_y<C>(a.op, m1, My, iy, v)) r = add(r, mul(v, P));
        } else {    // x from sxx (+ SAT), y from NN (closures, penalties)
            v = dx_from_M<C>(a.op, a.in[F_MM0], pitch, Mx, ix, iy);
            r = add(r, mul(v, P));
            const bool sx = a.xif ? satN_if<C>(a.op, Mx, ix, [&](int q) { return ld<C>(a.in[F_MM0], (long)q * pitch + iy); }, v)
                                  : sat_NM<C>(a.op, a.in[F_MM0], pitch, Mx, ix, iy, v);
            if (sx) r = add(r, mul(v, P));
            const S *nn = a.in[F_NN] + (long)ix * pitch;
            v = dy_sbp<true, C>(a.op, nn, My, iy);
            r = add(r, mul(v, P));
            if (satM_y<C>(a.op, nn, My, iy, v)) r = add(r, mul(v, P));
        }
        const C wrong = to_c<C>(a.out[f][i]);
        C s = to_c<C>(a.in[f][i]);
        time_update<CPST>(s, r, c);
        const int g = mn ? G_MN : G_NM;
        s = finish<S, C, CPST>(a, f, i, s, r, c, a.src_grid == g && ix == a.src_ix && iy == a.src_iy, it);
        if (a.energy) de = mul(mul((double)s, a.w[f][i]), (double)s) - mul(mul((double)wrong, a.w[f][i]), (double)wrong);
        if (a.n_rcv > 0) record(a, it, f, ix, iy, (double)s);
    }
    if (a.energy) {
        const double t = block_sum(de);
        if (threadIdx.x == 0 && t != 0. && it < a.max_steps) atomicAdd(a.energy + (long)a.max_steps + it, 0.5 * t);
    }
}

// stresses: blockIdx.y selects NN (0) or MM (1)
template <class S, class C, int CPST>
__global__ void __launch_bounds__(YF_THREADS) k_ysat_str(YFixArgs<S, C> a)
{
    const int it = *a.step - 1;
    const int Mx = a.Mx, My = a.My;
    const long pitch = a.pitch;
    const bool nn = blockIdx.y == 0;
    const int ncol = nn ? 10 : 12, rows = nn ? Mx + 1 : Mx;
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double de = 0.;
    if (k < (long)rows * ncol) {
        const int ix = (int)(k / ncol), iy = nn ? fix_col((int)(k % ncol), 5, My + 1, 5) : fix_col((int)(k % ncol), 6, My, 6);
        const long i = (long)ix * pitch + iy;
        const bool src_here = ix == a.src_ix && iy == a.src_iy;
        if (nn) {   // x from the new MN (+ the interface), y from the new NM
            C r, c;
            load_rc2<S, C, CPST>(a.rin[F_NN], i, r, c);
            const C P = __ldg(a.coef[F_NN] + i);
            C v = dx_from_M<C>(a.op, (const S *)a.out[F_MN], pitch, Mx, ix, iy);
            r = add(r, mul(v, P));
            if (a.xif && satN_if<C>(a.op, Mx, ix, [&](int q) { return ld<C>((const S *)a.out[F_MN], (long)q * pitch + iy); }, v))
                r = add(r, mul(v, P));
            v = dy_sbp<false, C>(a.op, (const S *)a.out[F_NM] + (long)ix * pitch, My, iy);
            r = add(r, mul(v, P));
            const C wrong = to_c<C>(a.out[F_NN][i]);
            C s = to_c<C>(a.in[F_NN][i]);
            time_update<CPST>(s, r, c);
            s = finish<S, C, CPST>(a, F_NN, i, s, r, c, a.src_grid == G_NN && src_here, it);
            if (a.energy) de = mul(mul((double)s, a.w[F_NN][i]), (double)s) - mul(mul((double)wrong, a.w[F_NN][i]), (double)wrong);
            if (a.n_rcv > 0) record(a, it, F_NN, ix, iy, (double)s);
        } else {    // x from the new NM (+ the interface), y from the new MN; lambda on both, 2mu on its own
            C r0, c0, r1, c1;
            load_rc2<S, C, CPST>(a.rin[F_MM0], i, r0, c0);
            load_rc2<S, C, CPST>(a.rin[F_MM1], i, r1, c1);
            const C L = __ldg(a.coef[F_MM0] + i), M2 = __ldg(a.coef[F_MM1] + i);
            C v = dx_from_N<C>(a.op, (const S *)a.out[F_NM], pitch, Mx, ix, iy);
            r0 = add(r0, mul(v, L));
            r1 = add(r1, mul(v, L));
            r0 = add(r0, mul(v, M2));
            if (a.xif && satM_if<C>(a.op, Mx, ix, [&](int q) { return ld<C>((const S *)a.out[F_NM], (long)q * pitch + iy); }, v)) {
                r0 = add(r0, mul(v, L));
                r1 = add(r1, mul(v, L));
                r0 = add(r0, mul(v, M2));
            }
            v = dy_sbp<true, C>(a.op, (const S *)a.out[F_MN] + (long)ix * pitch, My, iy);
            r0 = add(r0, mul(v, L));
            r1 = add(r1, mul(v, L));
            r1 = add(r1, mul(v, M2));
            const C w0 = to_c<C>(a.out[F_MM0][i]), w1 = to_c<C>(a.out[F_MM1][i]);
            C s0 = to_c<C>(a.in[F_MM0][i]), s1 = to_c<C>(a.in[F_MM1][i]);
            time_update<CPST>(s0, r0, c0);
            time_update<CPST>(s1, r1, c1);
            const bool src = a.src_grid == G_MM && src_here;
            s0 = finish<S, C, CPST>(a, F_MM0, i, s0, r0, c0, src, it);
            s1 = finish<S, C, CPST>(a, F_MM1, i, s1, r1, c1, src, it);
            if (a.energy) {
                auto q = [&](C x_, C y_) {
                    const double x = (double)x_, y = (double)y_, p1 = a.w[F_MM0][i], p2 = a.w[F_MM1][i];
                    return mul(mul(x, p1), x) + mul(mul(y, p1), y) + mul(mul(x, p2), y);
                };
                de = q(s0, s1) - q(w0, w1);
            }
            if (a.n_rcv > 0) {
                record(a, it, F_MM0, ix, iy, (double)s0);
                record(a, it, F_MM1, ix, iy, (double)s1);
            }
        }
    }
    if (a.energy) {
        const double t = block_sum(de);
        if (threadIdx.x == 0 && t != 0. && it < a.max_steps) atomicAdd(a.energy + 2L * a.max_steps + it, 0.5 * t);
    }
}

template <class S, class C, int CPST>
void launch_t(const YFixArgs<S, C> &a, cudaStream_t st)
{
    const long nv = (long)(a.Mx + 1) * 8, ns = (long)(a.Mx + 1) * 12;
    k_ysat_vel<S, C, CPST><<<dim3((unsigned)((nv + YF_THREADS - 1) / YF_THREADS), 2), YF_THREADS, 0, st>>>(a);
    k_ysat_str<S, C, CPST><<<dim3((unsigned)((ns + YF_THREADS - 1) / YF_THREADS), 2), YF_THREADS, 0, st>>>(a);
}

}  // namespace

template <class S, class C>
void launch_ysat_fix(const YFixArgs<S, C> &a, int cpst, cudaStream_t st)
{
    switch (cpst) {
    case 0: launch_t<S, C, 0>(a, st); break;
    case 1: launch_t<S, C, 1>(a, st); break;
    case 2: launch_t<S, C, 2>(a, st); break;
    case 3: launch_t<S, C, 3>(a, st); break;
    case 4: launch_t<S, C, 4>(a, st); break;
    case 5: launch_t<S, C, 5>(a, st); break;
    default: launch_t<S, C, 6>(a, st); break;
    }
}

template void launch_ysat_fix<double, double>(const YFixArgs<double, double> &, int, cudaStream_t);
template void launch_ysat_fix<float, float>(const YFixArgs<float, float> &, int, cudaStream_t);

}  // namespace tw

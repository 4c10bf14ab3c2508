// Per-half-step stepping kernels (one thread per grid point, all fields of that point).
//
// A time step is: velocity kernel (MN, NM: x derivative with SBP closures, SAT penalty,
// y derivative, time update, velocity source), stress kernel (NN, MM: x and y derivatives,
// time update, stress source), optional energy reductions and the receiver gather, in the order
// of forward_simulation.cpp:30-163. Per point, each right-hand side accumulates its terms in the
// reference's order (x derivative, SAT, y derivative; on MM the lambda terms before 2mu), so the
// result equals the reference's sequence of whole-grid passes. Fields are updated in place: the
// velocity kernel writes only velocities and reads only stresses (and the reverse).
#include "acoustic.cuh"

namespace tw {

// ---------------------------------------------------------------- elastic, SAT x / periodic y
template <class S, class C, int CPST>
__global__ void __launch_bounds__(256) k_elastic_velocity(StepArgs<S, C> a)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    if (iy > a.My || ix > a.Mx) return;
    const int it = *a.step;
    const long pitch = a.pitch;
    const long i = (long)ix * pitch + iy;
    constexpr bool kr = Cpst<CPST>::keep_r, kc = Cpst<CPST>::keep_c;

    const bool xif = a.bnd & BND_X_IF, ysat = a.bnd & BND_Y_SAT;
    if (ix < a.Mx) {   // MN (Mx x My+1): velocity along y; x from NN, y from MM syy
        C r, c;
        load_rc<S, C, CPST>(a.res[F_MN], i, r, c);
        const C P = __ldg(a.coef[F_MN] + i);
        C v = dx_from_N<C>(a.op, a.f[F_NN], pitch, a.Mx, ix, iy);
        r = add(r, mul(v, P));
        const bool sx = xif ? satM_if<C>(a.op, a.Mx, ix, [&](int q) { return ld<C>(a.f[F_NN], (long)q * pitch + iy); }, v)
                            : sat_MN<C>(a.op, a.f[F_NN], pitch, a.Mx, ix, iy, v);
        if (sx) r = add(r, mul(v, P));
        const S *m1 = a.f[F_MM1] + (long)ix * pitch;
        v = dy_any<false, C>(a.op, m1, a.My, iy, ysat);
        r = add(r, mul(v, P));
        if (ysat && satN_y<C>(a.op, m1, a.My, iy, v)) r = add(r, mul(v, P));
        C s = to_c<C>(a.f[F_MN][i]);
        time_update<CPST>(s, r, c);
        finish_point(a.f[F_MN], a.res[F_MN], i, s, r, c, kr, kc,
                     a.src_grid == G_MN && ix == a.src_ix && iy == a.src_iy, a.src_inc, it, a.flags);
    }
    if (iy < a.My) {   // NM (Mx+1 x My): velocity along x; x from MM sxx, y from NN
        C r, c;
        load_rc<S, C, CPST>(a.res[F_NM], i, r, c);
        const C P = __ldg(a.coef[F_NM] + i);
        C v = dx_from_M<C>(a.op, a.f[F_MM0], pitch, a.Mx, ix, iy);
        r = add(r, mul(v, P));
        const bool sx = xif ? satN_if<C>(a.op, a.Mx, ix, [&](int q) { return ld<C>(a.f[F_MM0], (long)q * pitch + iy); }, v)
                            : sat_NM<C>(a.op, a.f[F_MM0], pitch, a.Mx, ix, iy, v);
        if (sx) r = add(r, mul(v, P));
        const S *nn = a.f[F_NN] + (long)ix * pitch;
        v = dy_any<true, C>(a.op, nn, a.My, iy, ysat);
        r = add(r, mul(v, P));
        if (ysat && satM_y<C>(a.op, nn, a.My, iy, v)) r = add(r, mul(v, P));
        C s = to_c<C>(a.f[F_NM][i]);
        time_update<CPST>(s, r, c);
        finish_point(a.f[F_NM], a.res[F_NM], i, s, r, c, kr, kc,
                     a.src_grid == G_NM && ix == a.src_ix && iy == a.src_iy, a.src_inc, it, a.flags);
    }
}

template <class S, class C, int CPST>
__global__ void __launch_bounds__(256) k_elastic_stress(StepArgs<S, C> a)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    if (iy > a.My || ix > a.Mx) return;
    const int it = *a.step;
    const long pitch = a.pitch;
    const long i = (long)ix * pitch + iy;
    constexpr bool kr = Cpst<CPST>::keep_r, kc = Cpst<CPST>::keep_c;
    const double *si = a.src_inc + 0;
    const bool src_here = ix == a.src_ix && iy == a.src_iy;
    const bool xif = a.bnd & BND_X_IF, ysat = a.bnd & BND_Y_SAT;

    {   // NN (Mx+1 x My+1): shear stress; x from MN (+ the x interface), y from NM
        C r, c;
        load_rc<S, C, CPST>(a.res[F_NN], i, r, c);
        const C P = __ldg(a.coef[F_NN] + i);
        C v = dx_from_M<C>(a.op, a.f[F_MN], pitch, a.Mx, ix, iy);
        r = add(r, mul(v, P));
        if (xif && satN_if<C>(a.op, a.Mx, ix, [&](int q) { return ld<C>(a.f[F_MN], (long)q * pitch + iy); }, v))
            r = add(r, mul(v, P));
        v = dy_any<false, C>(a.op, a.f[F_NM] + (long)ix * pitch, a.My, iy, ysat);
        r = add(r, mul(v, P));
        C s = to_c<C>(a.f[F_NN][i]);
        time_update<CPST>(s, r, c);
        finish_point(a.f[F_NN], a.res[F_NN], i, s, r, c, kr, kc, a.src_grid == G_NN && src_here, si, it, a.flags);
    }
    if (ix < a.Mx && iy < a.My) {   // MM (Mx x My): normal stresses; x from NM, y from MN
        C r0, c0, r1, c1;
        load_rc<S, C, CPST>(a.res[F_MM0], i, r0, c0);
        load_rc<S, C, CPST>(a.res[F_MM1], i, r1, c1);
        const C L = __ldg(a.coef[F_MM0] + i);
        const C M2 = __ldg(a.coef[F_MM1] + i);
        C v = dx_from_N<C>(a.op, a.f[F_NM], pitch, a.Mx, ix, iy);
        r0 = add(r0, mul(v, L));
        r1 = add(r1, mul(v, L));
        r0 = add(r0, mul(v, M2));
        if (xif && satM_if<C>(a.op, a.Mx, ix, [&](int q) { return ld<C>(a.f[F_NM], (long)q * pitch + iy); }, v)) {
            r0 = add(r0, mul(v, L));
            r1 = add(r1, mul(v, L));
            r0 = add(r0, mul(v, M2));
        }
        v = dy_any<true, C>(a.op, a.f[F_MN] + (long)ix * pitch, a.My, iy, ysat);
        r0 = add(r0, mul(v, L));
        r1 = add(r1, mul(v, L));
        r1 = add(r1, mul(v, M2));
        C s0 = to_c<C>(a.f[F_MM0][i]);
        C s1 = to_c<C>(a.f[F_MM1][i]);
        time_update<CPST>(s0, r0, c0);
        time_update<CPST>(s1, r1, c1);
        const bool src = a.src_grid == G_MM && src_here;
        finish_point(a.f[F_MM0], a.res[F_MM0], i, s0, r0, c0, kr, kc, src, si, it, a.flags);
        finish_point(a.f[F_MM1], a.res[F_MM1], i, s1, r1, c1, kr, kc, src, si, it, a.flags);
    }
}

// ---------------------------------------------------------------- acoustic (p, vx, vy)
// SAT x: the elastic stepper with mu = 0, where sxx = syy = p and sxy = 0 bit for bit
// (NN terms vanish); PERIODIC x: the single-core tree (namespaces.hpp:593-668).
template <class S, class C, int CPST, bool PERIODIC>
__global__ void __launch_bounds__(256) k_acoustic_velocity(StepArgs<S, C> a)
{
    pdl_enter();
    acoustic_velocity_point<S, C, CPST, PERIODIC>(a, blockIdx.y * blockDim.y + threadIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

template <class S, class C, int CPST, bool PERIODIC>
__global__ void __launch_bounds__(256) k_acoustic_pressure(StepArgs<S, C> a)
{
    pdl_enter();
    acoustic_pressure_point<S, C, CPST, PERIODIC>(a, blockIdx.y * blockDim.y + threadIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------- launchers
namespace {
dim3 grid_for(int rows, int cols, dim3 b) { return dim3((cols + b.x - 1) / b.x, (rows + b.y - 1) / b.y); }

template <class S, class C, int CPST>
void launch_cpst(int physics, int periodic, int half, const StepArgs<S, C> &a, cudaStream_t st)
{
    const dim3 b(32, 8);
    const dim3 gN = grid_for(a.Mx + 1, a.My + 1, b), gM = grid_for(a.Mx, a.My, b);
    if (physics == 0) {
        if (half == 0) k_elastic_velocity<S, C, CPST><<<gN, b, 0, st>>>(a);
        else k_elastic_stress<S, C, CPST><<<gN, b, 0, st>>>(a);
    } else if (periodic) {
        if (half == 0) launch_pdl(k_acoustic_velocity<S, C, CPST, true>, gN, b, 0, st, a);
        else launch_pdl(k_acoustic_pressure<S, C, CPST, true>, gM, b, 0, st, a);
    } else {
        if (half == 0) launch_pdl(k_acoustic_velocity<S, C, CPST, false>, gN, b, 0, st, a);
        else launch_pdl(k_acoustic_pressure<S, C, CPST, false>, gM, b, 0, st, a);
    }
}
}  // namespace

template <class S, class C>
void launch_half(int physics, int periodic, int cpst, int half, const StepArgs<S, C> &a, cudaStream_t st)
{
    switch (cpst) {
    case 0: launch_cpst<S, C, 0>(physics, periodic, half, a, st); break;
    case 1: launch_cpst<S, C, 1>(physics, periodic, half, a, st); break;
    case 2: launch_cpst<S, C, 2>(physics, periodic, half, a, st); break;
    case 3: launch_cpst<S, C, 3>(physics, periodic, half, a, st); break;
    case 4: launch_cpst<S, C, 4>(physics, periodic, half, a, st); break;
    case 5: launch_cpst<S, C, 5>(physics, periodic, half, a, st); break;
    default: launch_cpst<S, C, 6>(physics, periodic, half, a, st); break;
    }
}

template void launch_half<double, double>(int, int, int, int, const StepArgs<double, double> &, cudaStream_t);
template void launch_half<float, float>(int, int, int, int, const StepArgs<float, float> &, cudaStream_t);

}  // namespace tw

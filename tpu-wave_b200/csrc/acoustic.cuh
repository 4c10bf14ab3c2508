// Per-point updates shared by the stepping kernels (step_kernels.cu) and the batched kernels
// (batch.cu): the time update's final store with the source and the non-finite check, the
// compensation loads, and the acoustic velocity / pressure updates of one grid point.
#pragma once
#include "stepper.cuh"
#include "kernels.h"

namespace tw {

template <class S, class C>
__device__ __forceinline__ void finish_point(S *f, S *res, long i, C s, C r, C c, bool keep_r, bool keep_c,
                                             bool is_src, const double *src_inc, int it, int *flags)
{
    if (is_src) s = to_s<C>(add((double)s, src_inc[it]));   // (double)S + A dt / dx^2, rounded once
    if (!finite(s)) atomicOr(flags, FLAG_NONFINITE);
    f[i] = to_s<S>(s);
    if (keep_r) res[i] = to_s<S>(r);
    if (keep_c) res[i] = to_s<S>(c);
}

template <class S, class C, int CPST>
__device__ __forceinline__ void load_rc(const S *res, long i, C &r, C &c)
{
    r = C(0);
    c = C(0);
    if constexpr (Cpst<CPST>::keep_r) r = to_c<C>(res[i]);
    if constexpr (Cpst<CPST>::keep_c) c = to_c<C>(res[i]);
}

// ---------------------------------------------------------------- acoustic, one point
// velocity point (ix, iy) of the N-sized region: MN velocity (y derivative of p) if ix < Mx, NM
// velocity (x derivative of p, SAT on the free surfaces) if iy < My
template <class S, class C, int CPST, bool PERIODIC>
__device__ __forceinline__ void acoustic_velocity_point(const StepArgs<S, C> &a, int ix, int iy)
{
    if (iy > a.My || ix > a.Mx) return;
    const int it = *a.step;
    const long pitch = a.pitch;
    const long i = (long)ix * pitch + iy;
    constexpr bool kr = Cpst<CPST>::keep_r, kc = Cpst<CPST>::keep_c;
    const S *p = a.f[F_MM0];
    const bool xif = !PERIODIC && (a.bnd & BND_X_IF), ysat = !PERIODIC && (a.bnd & BND_Y_SAT);

    if (ix < a.Mx) {   // MN (Mx x My+1): velocity along y, y derivative of p only (+ the y free surfaces)
        C r, c;
        load_rc<S, C, CPST>(a.res[F_MN], i, r, c);
        const C P = __ldg(a.coef[F_MN] + i);
        C v = dy_any<false, C>(a.op, p + (long)ix * pitch, a.My, iy, ysat);
        r = add(r, mul(v, P));
        if (ysat && satN_y<C>(a.op, p + (long)ix * pitch, a.My, iy, v)) r = add(r, mul(v, P));
        C s = to_c<C>(a.f[F_MN][i]);
        time_update<CPST>(s, r, c);
        finish_point(a.f[F_MN], a.res[F_MN], i, s, r, c, kr, kc,
                     a.src_grid == G_MN && ix == a.src_ix && iy == a.src_iy, a.src_inc, it, a.flags);
    }
    if (iy < a.My) {   // NM (Mx+1 x My): velocity along x, x derivative of p (+ SAT on the free surfaces)
        C r, c;
        load_rc<S, C, CPST>(a.res[F_NM], i, r, c);
        const C P = __ldg(a.coef[F_NM] + i);
        C v;
        if constexpr (PERIODIC) {
            v = dx_periodic<false, C>(a.op, p, pitch, a.Mx, ix, iy);
            r = add(r, mul(v, P));
        } else {
            v = dx_from_M<C>(a.op, p, pitch, a.Mx, ix, iy);
            r = add(r, mul(v, P));
            const bool sx = xif ? satN_if<C>(a.op, a.Mx, ix, [&](int q) { return ld<C>(p, (long)q * pitch + iy); }, v)
                                : sat_NM<C>(a.op, p, pitch, a.Mx, ix, iy, v);
            if (sx) r = add(r, mul(v, P));
        }
        C s = to_c<C>(a.f[F_NM][i]);
        time_update<CPST>(s, r, c);
        finish_point(a.f[F_NM], a.res[F_NM], i, s, r, c, kr, kc,
                     a.src_grid == G_NM && ix == a.src_ix && iy == a.src_iy, a.src_inc, it, a.flags);
    }
}

// pressure point (ix, iy): x derivative of the NM velocity, y derivative of the MN velocity
template <class S, class C, int CPST, bool PERIODIC>
__device__ __forceinline__ void acoustic_pressure_point(const StepArgs<S, C> &a, int ix, int iy)
{
    if (iy >= a.My || ix >= a.Mx) return;
    const int it = *a.step;
    const long pitch = a.pitch;
    const long i = (long)ix * pitch + iy;
    constexpr bool kr = Cpst<CPST>::keep_r, kc = Cpst<CPST>::keep_c;
    C r, c;
    load_rc<S, C, CPST>(a.res[F_MM0], i, r, c);
    const C K = __ldg(a.coef[F_MM0] + i);
    C v = PERIODIC ? dx_periodic<true, C>(a.op, a.f[F_NM], pitch, a.Mx, ix, iy)
                   : dx_from_N<C>(a.op, a.f[F_NM], pitch, a.Mx, ix, iy);
    r = add(r, mul(v, K));
    if (!PERIODIC && (a.bnd & BND_X_IF) &&
        satM_if<C>(a.op, a.Mx, ix, [&](int q) { return ld<C>(a.f[F_NM], (long)q * pitch + iy); }, v))
        r = add(r, mul(v, K));
    v = PERIODIC ? dy_periodic<true, C>(a.op, a.f[F_MN] + (long)ix * pitch, a.My, iy)
                 : dy_any<true, C>(a.op, a.f[F_MN] + (long)ix * pitch, a.My, iy, a.bnd & BND_Y_SAT);
    r = add(r, mul(v, K));
    C s = to_c<C>(a.f[F_MM0][i]);
    time_update<CPST>(s, r, c);
    finish_point(a.f[F_MM0], a.res[F_MM0], i, s, r, c, kr, kc,
                 a.src_grid == G_MM && ix == a.src_ix && iy == a.src_iy, a.src_inc, it, a.flags);
}

}  // namespace tw

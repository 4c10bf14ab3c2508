// Kernel arguments and per-point operators of the staggered SBP-SAT stepper.
//
// Device layout: every grid keeps the reference's sizes (grid.hpp:168-169), row-major with
// `pitch` elements per row (x = row): N-type directions have M+1 points, M-type ones M. Along a
// periodic direction the last N point is the reference's "duplicate" of point 0: it has its own
// material and is updated like any other point, its y derivative reads the M neighbour with the
// wrap modulo M, and the M-type grids read it directly at their last point; only beyond it do
// their reads wrap (grid_drvt.tpp:45-167 with N_modulo = M; singlecore copy_to_halo,
// namespaces.hpp:566-590). With a medium that repeats at the seam the two columns stay equal.
#pragma once
#include "device_math.cuh"
#include "sbp.hpp"

namespace tw {

enum { G_NN = 0, G_MN = 1, G_NM = 2, G_MM = 3 };
enum { F_NN = 0, F_MN = 1, F_NM = 2, F_MM0 = 3, F_MM1 = 4 };
enum { FLAG_NONFINITE = 1, FLAG_RECORD_FULL = 2, FLAG_TIMEOUT = 4 };

template <class S, class C>
struct StepArgs {
    S *f[5];              // fields NN, MN, NM, MM0 (sxx / p), MM1 (syy)
    S *res[5];            // compensation arrays (R or C), null without compensation
    const C *coef[5];     // NN mu, MN 1/rho, NM 1/rho, MM lambda (kappa), MM 2mu
    long pitch;
    int Mx, My;
    Ops<C> op;
    const double *src_inc;    // per-step source increment A(t) dt / dx^2 / scaling
    int src_grid, src_ix, src_iy;
    int max_steps;
    const int *step;          // device step counter (read by every kernel of a step)
    int *flags;               // sticky error flags
    int bnd;                  // BND_X_IF | BND_Y_SAT: the boundary variants below (0: the reference's)
};

// boundary variants beyond the reference's runs: BND_X_IF joins the two x ends by the SAT
// interface penalty (the reference's secure_bdry branch for a boundary type other than 'F',
// grid_drvt.tpp:575-693, on every grid); BND_Y_SAT puts free surfaces on the y ends too (SBP
// closures and the velocity grids' penalties along y, with the x tables)
enum { BND_X_IF = 1, BND_Y_SAT = 2 };

// read index of an M-type periodic neighbour (n points): wrap modulo n
__device__ __forceinline__ int wrap(int j, int n) { return j < 0 ? j + n : (j >= n ? j - n : j); }
// read index of an N-type periodic neighbour (n + 1 points, the last one the seam duplicate):
// read directly up to n, wrap beyond
__device__ __forceinline__ int nread(int j, int n) { return j < 0 ? j + n : (j > n ? j - n : j); }

template <class C, class S>
__device__ __forceinline__ C ld(const S *p, long i) { return to_c<C>(__ldg(p + i)); }
template <class C>
__device__ __forceinline__ C ld(const __nv_bfloat16 *p, long i) { return to_c<C>(p[i]); }
template <class C>
__device__ __forceinline__ C ld(const __half *p, long i) { return to_c<C>(p[i]); }

// a field stored as a pair hi + lo (split compensation): reads return the sum
template <class S>
struct HiLo {
    const S *hi, *lo;
    __device__ __forceinline__ HiLo operator+(long o) const { return {hi + o, lo + o}; }
};
template <class C, class S>
__device__ __forceinline__ C ld(HiLo<S> p, long i) { return add(ld<C>(p.hi, i), ld<C>(p.lo, i)); }

// derivative along x of an M-type-x row ix (rows 0..Mx-1) from its N-type neighbour with rows
// 0..Mx: DN closures on 3 rows at each end, interior shifts {-1,0,1,2} (grid_drvt.tpp:312-466,
// grid.hpp:361-362). get(r) returns the neighbour's value at row r of this column.
template <class C, class G>
__device__ __forceinline__ C dxN(const Ops<C> &o, int Mx, int ix, G get)
{
    C v = C(0);
    if (ix < 3) {
#pragma unroll
        for (int w = 0; w < 5; w++) v = add(v, mul(get(w), o.dnL[ix][w]));
    } else if (ix >= Mx - 3) {
        const int r = ix - (Mx - 3);
#pragma unroll
        for (int w = 0; w < 5; w++) v = add(v, mul(get(Mx - 4 + w), o.dnR[r][w]));
    } else {
#pragma unroll
        for (int w = 0; w < 4; w++) v = add(v, mul(get(ix - 1 + w), o.st[w]));
    }
    return v;
}

// derivative along x of an N-type-x row ix (rows 0..Mx) from its M-type neighbour with rows
// 0..Mx-1: DM closures on 4 rows at each end, interior shifts {-2,-1,0,1}.
template <class C, class G>
__device__ __forceinline__ C dxM(const Ops<C> &o, int Mx, int ix, G get)
{
    C v = C(0);
    if (ix < 4) {
#pragma unroll
        for (int w = 0; w < 5; w++) v = add(v, mul(get(w), o.dmL[ix][w]));
    } else if (ix >= Mx - 3) {
        const int r = ix - (Mx - 3);
#pragma unroll
        for (int w = 0; w < 5; w++) v = add(v, mul(get(Mx - 5 + w), o.dmR[r][w]));
    } else {
#pragma unroll
        for (int w = 0; w < 4; w++) v = add(v, mul(get(ix - 2 + w), o.st[w]));
    }
    return v;
}

template <class C, class A>
__device__ __forceinline__ C dx_from_N(const Ops<C> &o, A nb, long pitch, int Mx, int ix, int iy)
{
    return dxN<C>(o, Mx, ix, [&](int r) { return ld<C>(nb, (long)r * pitch + iy); });
}

template <class C, class A>
__device__ __forceinline__ C dx_from_M(const Ops<C> &o, A nb, long pitch, int Mx, int ix, int iy)
{
    return dxM<C>(o, Mx, ix, [&](int r) { return ld<C>(nb, (long)r * pitch + iy); });
}

// periodic x derivative (single-core acoustic tree): an N-type row reads M-type rows ix-2..ix+1
// (wrapped), an M-type row reads N-type rows ix-1..ix+2 (seam row read directly)
template <bool FROM_N, class C, class S>
__device__ __forceinline__ C dx_periodic(const Ops<C> &o, const S *nb, long pitch, int Mx, int ix, int iy)
{
    C v = C(0);
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const int r = FROM_N ? nread(ix - 1 + w, Mx) : wrap(ix - 2 + w, Mx);
        v = add(v, mul(ld<C>(nb, (long)r * pitch + iy), o.st[w]));
    }
    return v;
}

// periodic y derivative (grid.hpp:361-362, grid_drvt.tpp:45-167): an N-type-y point reads
// M-type columns iy-2..iy+1 (wrapped), an M-type-y point reads N-type columns iy-1..iy+2
template <bool FROM_N, class C, class A>
__device__ __forceinline__ C dy_periodic(const Ops<C> &o, A row, int My, int iy)
{
    C v = C(0);
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const int c = FROM_N ? nread(iy - 1 + w, My) : wrap(iy - 2 + w, My);
        v = add(v, mul(ld<C>(row, (long)c), o.st[w]));
    }
    return v;
}

// SAT penalty of the M-type-x velocity grid MN (rows 0..2 and Mx-3..Mx-1): the boundary value
// of the NN neighbour (projection {1}) times eta*A_inv_projection (grid_drvt.tpp:563-693)
template <class C, class A>
__device__ __forceinline__ bool sat_MN(const Ops<C> &o, A nn, long pitch, int Mx, int ix, int iy, C &v)
{
    if (ix < 3) {
        const C send = add(C(0), mul(o.pN, ld<C>(nn, iy)));
        v = mul(o.satML[ix], sub(send, C(0)));
        return true;
    }
    if (ix >= Mx - 3) {
        const C send = add(C(0), mul(o.pN, ld<C>(nn, (long)Mx * pitch + iy)));
        v = mul(o.satMR[ix - (Mx - 3)], sub(send, C(0)));
        return true;
    }
    return false;
}

// SAT penalty of the N-type-x velocity grid NM (rows 0 and Mx): sxx extrapolated to the
// boundary with {15/8, -5/4, 3/8} over three MM rows
template <class C, class A>
__device__ __forceinline__ bool sat_NM(const Ops<C> &o, A mm, long pitch, int Mx, int ix, int iy, C &v)
{
    if (ix == 0) {
        C send = C(0);
#pragma unroll
        for (int w = 0; w < 3; w++) send = add(send, mul(o.pML[w], ld<C>(mm, (long)w * pitch + iy)));
        v = mul(o.satNL, sub(send, C(0)));
        return true;
    }
    if (ix == Mx) {
        C send = C(0);
#pragma unroll
        for (int w = 0; w < 3; w++) send = add(send, mul(o.pMR[w], ld<C>(mm, (long)(Mx - 3 + w) * pitch + iy)));
        v = mul(o.satNR, sub(send, C(0)));
        return true;
    }
    return false;
}

// ---------------------------------------------------------------- boundary variants
// the SAT interface penalty of an M-type-x point i (rows 0..M-1) whose x neighbour is N-type
// (rows 0..M): the neighbour's end rows projected with {1}; rows 0..2 are penalised with eta = +1/2
// toward the right end's projection (RECV_L = SEND_R), rows M-3..M-1 with eta = -1/2 toward the
// left's. eta * A_inv_projection is half the free-surface product, exactly.
template <class C, class G>
__device__ __forceinline__ bool satM_if(const Ops<C> &o, int M, int i, G get, C &v)
{
    if (i >= 3 && i < M - 3) return false;
    const C sL = add(C(0), mul(o.pN, get(0))), sR = add(C(0), mul(o.pN, get(M)));
    v = i < 3 ? mul(mul(C(0.5), o.satML[i]), sub(sL, sR)) : mul(mul(C(0.5), o.satMR[i - (M - 3)]), sub(sR, sL));
    return true;
}

// the SAT interface penalty of an N-type-x point i (rows 0..M) whose neighbour is M-type (rows
// 0..M-1): the neighbour extrapolated to each end with {15/8, -5/4, 3/8}, penalties on rows 0 and M
template <class C, class G>
__device__ __forceinline__ bool satN_if(const Ops<C> &o, int M, int i, G get, C &v)
{
    if (i != 0 && i != M) return false;
    C sL = C(0), sR = C(0);
#pragma unroll
    for (int w = 0; w < 3; w++) sL = add(sL, mul(o.pML[w], get(w)));
#pragma unroll
    for (int w = 0; w < 3; w++) sR = add(sR, mul(o.pMR[w], get(M - 3 + w)));
    v = i == 0 ? mul(mul(C(0.5), o.satNL), sub(sL, sR)) : mul(mul(C(0.5), o.satNR), sub(sR, sL));
    return true;
}

// y derivative with SBP closures at both y ends (free surfaces on all four sides): the x
// operators dxN / dxM applied along the row
template <bool FROM_N, class C, class A>
__device__ __forceinline__ C dy_sbp(const Ops<C> &o, A row, int My, int iy)
{
    auto get = [&](int c) { return ld<C>(row, (long)c); };
    if constexpr (FROM_N) return dxN<C>(o, My, iy, get);
    else return dxM<C>(o, My, iy, get);
}

template <bool FROM_N, class C, class A>
__device__ __forceinline__ C dy_any(const Ops<C> &o, A row, int My, int iy, bool sat_y)
{
    return sat_y ? dy_sbp<FROM_N, C>(o, row, My, iy) : dy_periodic<FROM_N, C>(o, row, My, iy);
}

// free-surface penalty on the y ends of an N-type-y velocity point (MN, neighbour syy of M type):
// syy extrapolated to column 0 / My, eta = +1 / -1
template <class C, class A>
__device__ __forceinline__ bool satN_y(const Ops<C> &o, A row, int My, int iy, C &v)
{
    if (iy != 0 && iy != My) return false;
    C send = C(0);
    if (iy == 0) {
#pragma unroll
        for (int w = 0; w < 3; w++) send = add(send, mul(o.pML[w], ld<C>(row, (long)w)));
        v = mul(o.satNL, sub(send, C(0)));
    } else {
#pragma unroll
        for (int w = 0; w < 3; w++) send = add(send, mul(o.pMR[w], ld<C>(row, (long)(My - 3 + w))));
        v = mul(o.satNR, sub(send, C(0)));
    }
    return true;
}

// the same for an M-type-y velocity point (NM, neighbour sxy of N type): sxy at column 0 / My,
// penalties on columns 0..2 / My-3..My-1
template <class C, class A>
__device__ __forceinline__ bool satM_y(const Ops<C> &o, A row, int My, int iy, C &v)
{
    if (iy < 3) {
        const C send = add(C(0), mul(o.pN, ld<C>(row, 0L)));
        v = mul(o.satML[iy], sub(send, C(0)));
        return true;
    }
    if (iy >= My - 3) {
        const C send = add(C(0), mul(o.pN, ld<C>(row, (long)My)));
        v = mul(o.satMR[iy - (My - 3)], sub(send, C(0)));
        return true;
    }
    return false;
}

}  // namespace tw

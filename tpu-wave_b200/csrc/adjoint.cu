// Discrete adjoint of the elastic SBP-SAT step (no counterpart in the reference).
//
// One forward step n is linear in the state u = (sigma, v) = (NN, MM0, MM1; MN, NM):
//   v'     = v     + P (Dx sigma + SAT sigma + Dy sigma)            (P = 1/rho per velocity point)
//   sigma' = sigma + C (Dx v' + Dy v')                              (C = mu on NN; lambda, 2mu on MM)
// with the SBP closures, the free-surface SAT penalties and the periodic y wrap of stepper.cuh.
// Its transpose, applied to an adjoint state lam = dJ/du_{n+1}, is
//   A: lam_v     += (Dx + Dy)^T (C lam_sigma)                       (the stress update, transposed)
//   B: lam_sigma += (Dx + SAT + Dy)^T (P lam_v)                     (the velocity update, transposed)
// and the gradients with respect to the coefficients collect, per point,
//   g_C += lam_sigma_{n+1} * (Dx + Dy) v_{n+1}      g_P += lam_v(after A) * (Dx + SAT + Dy) sigma_n.
// Every transposed operator below is written as the exact transpose of the forward one: output
// point r sums, over the forward points that read r, the forward weight of r times their input.
// Gradients accumulate in FP64.
#include "kernels.h"

namespace tw {

namespace {

// forward weight of N-type-x row r in the x derivative of M-type-x row ix (dxN)
template <class C>
__device__ __forceinline__ C cN(const Ops<C> &o, int Mx, int ix, int r)
{
    if (ix < 3) return r <= 4 ? o.dnL[ix][r] : C(0);
    if (ix >= Mx - 3) {
        const int k = r - (Mx - 4);
        return (k >= 0 && k <= 4) ? o.dnR[ix - (Mx - 3)][k] : C(0);
    }
    const int w = r - (ix - 1);
    return (w >= 0 && w <= 3) ? o.st[w] : C(0);
}

// forward weight of M-type-x row r in the x derivative of N-type-x row ix (dxM)
template <class C>
__device__ __forceinline__ C cM(const Ops<C> &o, int Mx, int ix, int r)
{
    if (ix < 4) return r <= 4 ? o.dmL[ix][r] : C(0);
    if (ix >= Mx - 3) {
        const int k = r - (Mx - 5);
        return (k >= 0 && k <= 4) ? o.dmR[ix - (Mx - 3)][k] : C(0);
    }
    const int w = r - (ix - 2);
    return (w >= 0 && w <= 3) ? o.st[w] : C(0);
}

// (dxN)^T: value at N row r from the M-row inputs w(ix), ix in [0, Mx)
template <class C, class G>
__device__ __forceinline__ C dxN_T(const Ops<C> &o, int Mx, int r, G w)
{
    C v = C(0);
    if (r >= 5 && r <= Mx - 5) {   // read only by interior rows r-2..r+1 (same order as below)
#pragma unroll
        for (int t = 3; t >= 0; t--) v = add(v, mul(o.st[t], w(r + 1 - t)));
        return v;
    }
    for (int ix = max(0, r - 4); ix <= min(Mx - 1, r + 4); ix++) {
        const C c = cN(o, Mx, ix, r);
        if (c != C(0)) v = add(v, mul(c, w(ix)));
    }
    return v;
}

// (dxM)^T: value at M row r from the N-row inputs w(ix), ix in [0, Mx]
template <class C, class G>
__device__ __forceinline__ C dxM_T(const Ops<C> &o, int Mx, int r, G w)
{
    C v = C(0);
    if (r >= 5 && r <= Mx - 6) {   // read only by interior rows r-1..r+2
#pragma unroll
        for (int t = 3; t >= 0; t--) v = add(v, mul(o.st[t], w(r + 2 - t)));
        return v;
    }
    for (int ix = max(0, r - 5); ix <= min(Mx, r + 5); ix++) {
        const C c = cM(o, Mx, ix, r);
        if (c != C(0)) v = add(v, mul(c, w(ix)));
    }
    return v;
}

// transpose of the y derivative of an N-type-y point c in [0, My] from M columns wrap(c-2+w):
// value at M column k from the N-column inputs w(c)
template <class C, class G>
__device__ __forceinline__ C dyNfromM_T(const Ops<C> &o, int My, int k, G w)
{
    C v = C(0);
    if (k >= 2 && k <= My - 3) {   // no wrap: read by N columns k-1..k+2
#pragma unroll
        for (int t = 0; t < 4; t++) v = add(v, mul(o.st[t], w(k + 2 - t)));
        return v;
    }
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const int js[3] = {k, k - My, k + My};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int j = js[q];
            if (j < -2 || j > My + 1) continue;
            if (q == 1 && j >= 0) continue;    // k - My is a wrap only below 0
            if (q == 2 && j < My) continue;    // k + My is a wrap only at My and above
            const int c = j + 2 - t;
            if (c >= 0 && c <= My) v = add(v, mul(o.st[t], w(c)));
        }
    }
    return v;
}

// transpose of the y derivative of an M-type-y point c in [0, My) from N columns nread(c-1+w):
// value at N column k in [0, My] from the M-column inputs w(c)
template <class C, class G>
__device__ __forceinline__ C dyMfromN_T(const Ops<C> &o, int My, int k, G w)
{
    C v = C(0);
    if (k >= 2 && k <= My - 2) {   // no wrap: read by M columns k-2..k+1
#pragma unroll
        for (int t = 0; t < 4; t++) v = add(v, mul(o.st[t], w(k + 1 - t)));
        return v;
    }
#pragma unroll
    for (int t = 0; t < 4; t++) {
        // j = c - 1 + t reads N column nread(j): j = k directly, j = -1 -> My - 1, j = My + 1 -> 1
        int js[3] = {k, -100, -100};
        if (k == My - 1) js[1] = -1;
        if (k == 1) js[2] = My + 1;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int j = js[q];
            if (j == -100) continue;
            const int c = j + 1 - t;
            if (c >= 0 && c < My) v = add(v, mul(o.st[t], w(c)));
        }
    }
    return v;
}

}  // namespace

// ---------------------------------------------------------------- phase A
// W_nn = mu lam_xy, W_xx = lambda (lam_xx + lam_yy) + 2mu lam_xx, W_yy likewise with lam_yy;
// coefficient gradients from the stress rates of v_{n+1}
template <class C>
__global__ void k_adj_a1(AdjArgs<C> a)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    const int Mx = a.Mx, My = a.My;
    if (ix > Mx || iy > My) return;
    const long p = a.pitch, o = (long)ix * p + iy;
    const C *const *v1 = a.u1;
    {   // NN
        const C lam = a.lam[F_NN][o];
        a.w[F_NN][o] = mul(a.coef[F_NN][o], lam);
        const C h = add(dx_from_M<C>(a.op, v1[F_MN], p, Mx, ix, iy), dy_periodic<false, C>(a.op, v1[F_NM] + (long)ix * p, My, iy));
        a.g[F_NN][o] += (double)lam * (double)h;
    }
    if (ix < Mx && iy < My) {   // MM
        const C lx = a.lam[F_MM0][o], ly = a.lam[F_MM1][o];
        const C L = a.coef[F_MM0][o], M2 = a.coef[F_MM1][o];
        const C s = add(lx, ly);
        a.w[F_MM0][o] = add(mul(L, s), mul(M2, lx));
        a.w[F_MM1][o] = add(mul(L, s), mul(M2, ly));
        const C hx = dx_from_N<C>(a.op, v1[F_NM], p, Mx, ix, iy);
        const C hy = dy_periodic<true, C>(a.op, v1[F_MN] + (long)ix * p, My, iy);
        a.g[F_MM0][o] += (double)s * ((double)hx + (double)hy);
        a.g[F_MM1][o] += (double)lx * (double)hx + (double)ly * (double)hy;
    }
}

// lam_MN += (dxM)^T W_nn + (dy of MM from MN)^T W_yy;  lam_NM += (dy of NN from NM)^T W_nn + (dxN)^T W_xx
template <class C>
__global__ void k_adj_a2(AdjArgs<C> a)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    const int Mx = a.Mx, My = a.My;
    if (ix > Mx || iy > My) return;
    const long p = a.pitch, o = (long)ix * p + iy;
    if (ix < Mx) {   // MN (Mx x My+1)
        C v = dxM_T<C>(a.op, Mx, ix, [&](int r) { return a.w[F_NN][(long)r * p + iy]; });
        v = add(v, dyMfromN_T<C>(a.op, My, iy, [&](int c) { return a.w[F_MM1][(long)ix * p + c]; }));
        a.lam[F_MN][o] = add(a.lam[F_MN][o], v);
    }
    if (iy < My) {   // NM (Mx+1 x My)
        C v = dyNfromM_T<C>(a.op, My, iy, [&](int c) { return a.w[F_NN][(long)ix * p + c]; });
        v = add(v, dxN_T<C>(a.op, Mx, ix, [&](int r) { return a.w[F_MM0][(long)r * p + iy]; }));
        a.lam[F_NM][o] = add(a.lam[F_NM][o], v);
    }
}

// ---------------------------------------------------------------- phase B
// Z = P lam_v; gradients of 1/rho from the velocity rates of sigma_n
template <class C>
__global__ void k_adj_b1(AdjArgs<C> a)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    const int Mx = a.Mx, My = a.My;
    if (ix > Mx || iy > My) return;
    const long p = a.pitch, o = (long)ix * p + iy;
    const C *const *s0 = a.u0;
    if (ix < Mx) {   // MN
        const C lam = a.lam[F_MN][o];
        a.w[F_MN][o] = mul(a.coef[F_MN][o], lam);
        C g = dx_from_N<C>(a.op, s0[F_NN], p, Mx, ix, iy);
        C sat;
        if (sat_MN<C>(a.op, s0[F_NN], p, Mx, ix, iy, sat)) g = add(g, sat);
        g = add(g, dy_periodic<false, C>(a.op, s0[F_MM1] + (long)ix * p, My, iy));
        a.g[F_MN][o] += (double)lam * (double)g;
    }
    if (iy < My) {   // NM
        const C lam = a.lam[F_NM][o];
        a.w[F_NM][o] = mul(a.coef[F_NM][o], lam);
        C g = dx_from_M<C>(a.op, s0[F_MM0], p, Mx, ix, iy);
        C sat;
        if (sat_NM<C>(a.op, s0[F_MM0], p, Mx, ix, iy, sat)) g = add(g, sat);
        g = add(g, dy_periodic<true, C>(a.op, s0[F_NN] + (long)ix * p, My, iy));
        a.g[F_NM][o] += (double)lam * (double)g;
    }
}

// lam_NN += (dxN)^T Z_mn + SAT_MN^T Z_mn + (dy of NM from NN)^T Z_nm
// lam_MM0 += (dxM)^T Z_nm + SAT_NM^T Z_nm;  lam_MM1 += (dy of MN from MM)^T Z_mn
template <class C>
__global__ void k_adj_b2(AdjArgs<C> a)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    const int Mx = a.Mx, My = a.My;
    if (ix > Mx || iy > My) return;
    const long p = a.pitch, o = (long)ix * p + iy;
    const C *zmn = a.w[F_MN], *znm = a.w[F_NM];
    {   // NN (Mx+1 x My+1)
        C v = dxN_T<C>(a.op, Mx, ix, [&](int r) { return zmn[(long)r * p + iy]; });
        if (ix == 0) {   // SAT of MN rows 0..2 reads NN row 0 with weight satML[r] * pN
            for (int r = 0; r < 3; r++) v = add(v, mul(mul(a.op.satML[r], a.op.pN), zmn[(long)r * p + iy]));
        } else if (ix == Mx) {
            for (int r = 0; r < 3; r++) v = add(v, mul(mul(a.op.satMR[r], a.op.pN), zmn[(long)(Mx - 3 + r) * p + iy]));
        }
        v = add(v, dyMfromN_T<C>(a.op, My, iy, [&](int c) { return znm[(long)ix * p + c]; }));
        a.lam[F_NN][o] = add(a.lam[F_NN][o], v);
    }
    if (ix < Mx && iy < My) {   // MM
        C v = dxM_T<C>(a.op, Mx, ix, [&](int r) { return znm[(long)r * p + iy]; });
        if (ix < 3) v = add(v, mul(mul(a.op.pML[ix], a.op.satNL), znm[iy]));   // SAT of NM row 0
        if (ix >= Mx - 3) v = add(v, mul(mul(a.op.pMR[ix - (Mx - 3)], a.op.satNR), znm[(long)Mx * p + iy]));
        a.lam[F_MM0][o] = add(a.lam[F_MM0][o], v);
        const C u = dyNfromM_T<C>(a.op, My, iy, [&](int c) { return zmn[(long)ix * p + c]; });
        a.lam[F_MM1][o] = add(a.lam[F_MM1][o], u);
    }
}

// ---------------------------------------------------------------- receivers
// lam += R^T r_it: every receiver adds its residual at step `it` to the adjoint of its field(s)
template <class C>
__global__ void k_adj_inject(AdjArgs<C> a, int it)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.n_rcv) return;
    const int *e = a.rcv + 4 * q;
    const long o = (long)e[2] * a.pitch + e[3];
    for (int f = 0; f < 2; f++)
        if (e[f] >= 0) {
            const double r = a.resid[(2L * q + f) * a.nt + it];
            atomicAdd(&a.lam[e[f]][o], (C)r);   // receivers may share a point
        }
}

template <class C>
void launch_adjoint_step(const AdjArgs<C> &a, cudaStream_t st)
{
    const dim3 b(32, 8), g((a.My + 1 + 31) / 32, (a.Mx + 1 + 7) / 8);
    k_adj_a1<C><<<g, b, 0, st>>>(a);
    k_adj_a2<C><<<g, b, 0, st>>>(a);
    k_adj_b1<C><<<g, b, 0, st>>>(a);
    k_adj_b2<C><<<g, b, 0, st>>>(a);
}

template <class C>
void launch_adjoint_inject(const AdjArgs<C> &a, int it, cudaStream_t st)
{
    if (a.n_rcv > 0) k_adj_inject<C><<<(a.n_rcv + 127) / 128, 128, 0, st>>>(a, it);
}

template void launch_adjoint_step<double>(const AdjArgs<double> &, cudaStream_t);
template void launch_adjoint_step<float>(const AdjArgs<float> &, cudaStream_t);
template void launch_adjoint_inject<double>(const AdjArgs<double> &, int, cudaStream_t);
template void launch_adjoint_inject<float>(const AdjArgs<float> &, int, cudaStream_t);

// ---------------------------------------------------------------- model chain rule
// transpose of k_interp: scatter the gradient of one grid's interpolated quantity onto the four
// model nodes it was interpolated from (FP64 atomics)
__global__ void k_interp_T(int rows, int cols, int txN, int tyN, int num_dx, int den_dx, int num_dxM, int den_dxM,
                           long Nxp, long Nyp, const double *gin, double *gnode)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    if (iy >= cols || ix >= rows) return;
    long nx, dxl, ny, dyl;
    if (txN) { nx = (long)ix * num_dx; dxl = den_dx; } else { nx = (2L * ix + 1) * num_dx; dxl = 2L * den_dx; }
    if (tyN) { ny = (long)iy * num_dx; dyl = den_dx; } else { ny = (2L * iy + 1) * num_dx; dyl = 2L * den_dx; }
    const long ixM = (nx * den_dxM) / (dxl * num_dxM);
    const long iyM = (ny * den_dxM) / (dyl * num_dxM);
    if (ixM < 0 || ixM + 1 > Nxp || iyM < 0 || iyM + 1 > Nyp) return;   // the forward map rejected these
    const double xi = sub(__ddiv_rn((double)(nx * den_dxM), (double)(dxl * num_dxM)), (double)ixM);
    const double eta = sub(__ddiv_rn((double)(ny * den_dxM), (double)(dyl * num_dxM)), (double)iyM);
    const long PS = Nyp + 1;
    const double a = sub(1.0, xi), b = sub(1.0, eta), gv = gin[(long)ix * cols + iy];
    atomicAdd(gnode + ixM * PS + iyM, a * b * gv);
    atomicAdd(gnode + ixM * PS + iyM + 1, a * eta * gv);
    atomicAdd(gnode + (ixM + 1) * PS + iyM, xi * b * gv);
    atomicAdd(gnode + (ixM + 1) * PS + iyM + 1, xi * eta * gv);
}

void launch_interp_T(int rows, int cols, int txN, int tyN, int num_dx, int den_dx, int num_dxM, int den_dxM,
                     long Nx_prmt, long Ny_prmt, const double *gin, double *gnode, cudaStream_t st)
{
    const dim3 b(32, 8), g((cols + 31) / 32, (rows + 7) / 8);
    k_interp_T<<<g, b, 0, st>>>(rows, cols, txN, tyN, num_dx, den_dx, num_dxM, den_dxM, Nx_prmt, Ny_prmt, gin, gnode);
}

// transpose of k_model_derive: node gradients of mu, lambda, 2mu and rho (direct) -> rho, vp, vs
__global__ void k_model_derive_T(const double *rho, const double *vp, const double *vs, long n, const double *g_mu,
                                 const double *g_lam, const double *g_m2, const double *g_rho_direct, double *g_rho,
                                 double *g_vp, double *g_vs)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double r = rho[i], p = vp[i], s = vs[i];
        // mu = r s^2, 2mu = 2 r s^2, lambda = r p^2 - 2 r s^2
        g_rho[i] = g_rho_direct[i] + g_mu[i] * s * s + g_m2[i] * 2. * s * s + g_lam[i] * (p * p - 2. * s * s);
        g_vp[i] = g_lam[i] * 2. * r * p;
        g_vs[i] = g_mu[i] * 2. * r * s + g_m2[i] * 4. * r * s - g_lam[i] * 4. * r * s;
    }
}

void launch_model_derive_T(const double *rho, const double *vp, const double *vs, long n, const double *g_mu,
                           const double *g_lam, const double *g_m2, const double *g_rho_direct, double *g_rho,
                           double *g_vp, double *g_vs, cudaStream_t st)
{
    const int blocks = (int)((n + 255) / 256 < 65535 ? (n + 255) / 256 : 65535);
    k_model_derive_T<<<blocks, 256, 0, st>>>(rho, vp, vs, n, g_mu, g_lam, g_m2, g_rho_direct, g_rho, g_vp, g_vs);
}

}  // namespace tw

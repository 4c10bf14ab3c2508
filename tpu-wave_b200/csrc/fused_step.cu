// Fused elastic time step: one launch per step, every field read once and written once.
//
// The two half-steps of forward_simulation.cpp:38-113 (velocities from stresses, then stresses
// from the new velocities) are done by one kernel that sweeps rows. A CTA owns a strip of
// FS_TY columns and a segment of rows. Each thread owns one column ("logical" column c =
// y0 - FS_HALO + t) and walks down the rows:
//   iteration k: stage old stress row k-1 (loaded at iteration k-1) into a shared ring;
//                issue the global loads of iteration k+1;
//                compute the velocities of row j = k - LAG_V;
//                compute the stresses of row i = k - LAG_S;
//                one __syncthreads.
// x derivatives read the thread's own column from the rings; y derivatives read neighbouring
// columns of a row staged at least one iteration earlier. The lags keep every SBP closure row
// (rows 0..4 and the last five) in the rings when it is needed: a velocity row j reads old
// stress rows up to j+2 (interior) or 4 (left closure); a stress row i reads new velocity rows
// up to i+2 or 4. The FS_HALO columns on each side give the y derivatives of the stresses the
// new velocities of the neighbouring strips, computed again here; rows outside the segment are
// computed again in the same way. The state is double buffered (in -> out) because neighbouring
// CTAs read old values that this CTA overwrites.
//
// Per point the arithmetic and the order of the right-hand-side terms are those of
// step_kernels.cu (hence of the reference), so results are bit-identical to the two-kernel path.
#include "kernels.h"
#include "stepper.cuh"

namespace tw {

namespace {

constexpr int NT = FS_THREADS;
constexpr int HALO = FS_HALO;
constexpr int TY = FS_TY;
constexpr int RS = 9;     // old stress rows kept
constexpr int RV = 8;     // new velocity rows kept
constexpr int LAG_V = 5;
constexpr int LAG_S = 9;

__device__ __forceinline__ int pmod(int c, int n)
{
    const int r = c % n;
    return r < 0 ? r + n : r;
}

// thread-local energy accumulators (FP64)
struct EAcc {
    double p0 = 0., k = 0., p1 = 0.;
};

template <class C>
struct Ring {
    C *p;
    int rows;
    __device__ __forceinline__ C &at(int row, int t) const { return p[(row % rows) * NT + t]; }
};

template <class S, class C, int CPST>
struct Inputs {   // global values consumed by one iteration
    C nn, mm0, mm1;                 // old stress row (to be staged)
    C vmn, vnm, pmn, pnm;           // old velocities and 1/rho of the velocity row
    C rmn, cmn, rnm, cnm;           // compensation values of the velocity row
    C mu, lam, m2;                  // coefficients of the stress row
    C rnn, cnn, rm0, cm0, rm1, cm1; // compensation values of the stress row
    double wmn, wnm, wnn, wm3, wm4; // energy weights
};

}  // namespace

template <class S, class C, int CPST, bool ENERGY>
__global__ void __launch_bounds__(NT) k_elastic_fused(FusedArgs<S, C> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sm = reinterpret_cast<C *>(smem_raw);
    const Ring<C> rNN{sm + 0 * RS * NT, RS}, rM0{sm + 1 * RS * NT, RS}, rM1{sm + 2 * RS * NT, RS};
    const Ring<C> rMN{sm + 3 * RS * NT, RV}, rNM{sm + 3 * RS * NT + RV * NT, RV};
    constexpr bool KR = Cpst<CPST>::keep_r, KC = Cpst<CPST>::keep_c;

    const int t = threadIdx.x;
    const int Mx = a.Mx, My = a.My;
    const long pitch = a.pitch;
    const int y0 = blockIdx.x * TY;
    const int c = y0 - HALO + t;                          // logical column
    const int pM = pmod(c, My);                           // M-type-y physical column
    const int pN = (c >= 0 && c <= My) ? c : pM;          // N-type-y physical column (seam kept)
    const bool core = t >= HALO && t < HALO + TY;
    const bool ownN = core && c <= My, ownM = core && c < My;
    const bool velT = t >= 2 && t < NT - 2;               // computes velocities (y taps t-2..t+2)

    const int seg = blockIdx.y;
    const int x0 = seg * a.seg_rows;
    const int x1e = seg == a.n_seg - 1 ? Mx : x0 + a.seg_rows - 1;   // last owned row (N-type grids)
    const int lb = max(x0 - 4, 0), le = min(x1e + 4, Mx);            // stress rows loaded
    const int vb = max(x0 - 2, 0), ve = min(x1e + 2, Mx);            // velocity rows computed
    const int it = *a.step;
    const int cta = blockIdx.y * gridDim.x + blockIdx.x;
    const int rcv_b = a.rcv_off[cta], rcv_e = a.rcv_off[cta + 1];

    auto ldS = [&](int f, int row, int col) -> C { return to_c<C>(a.in[f][(long)row * pitch + col]); };
    auto ldR = [&](int f, int row, int col) -> C { return to_c<C>(a.rin[f][(long)row * pitch + col]); };
    auto ldK = [&](int f, int row, int col) -> C { return __ldg(a.coef[f] + (long)row * pitch + col); };
    auto ldW = [&](int f, int row, int col) -> double { return __ldg(a.w[f] + (long)row * pitch + col); };

    // global loads of iteration kk (stress row kk-1, velocity row kk-LAG_V, stress row kk-LAG_S)
    auto fetch = [&](int kk, Inputs<S, C, CPST> &in) {
        const int sr = kk - 1, j = kk - LAG_V, i = kk - LAG_S;
        if (sr >= lb && sr <= le) {
            in.nn = ldS(F_NN, sr, pN);
            if (sr < Mx) { in.mm0 = ldS(F_MM0, sr, pM); in.mm1 = ldS(F_MM1, sr, pM); }
        }
        if (velT && j >= vb && j <= ve) {
            if (j < Mx) {
                in.vmn = ldS(F_MN, j, pN);
                in.pmn = ldK(F_MN, j, pN);
                if (KR) in.rmn = ldR(F_MN, j, pN);
                if (KC) in.cmn = ldR(F_MN, j, pN);
            }
            in.vnm = ldS(F_NM, j, pM);
            in.pnm = ldK(F_NM, j, pM);
            if (KR) in.rnm = ldR(F_NM, j, pM);
            if (KC) in.cnm = ldR(F_NM, j, pM);
            if (ENERGY && core && j >= x0 && j <= x1e) {
                if (j < Mx && ownN) in.wmn = ldW(F_MN, j, c);
                if (ownM) in.wnm = ldW(F_NM, j, c);
            }
        }
        if (core && i >= x0 && i <= x1e) {
            if (ownN) {
                in.mu = ldK(F_NN, i, c);
                if (KR) in.rnn = ldR(F_NN, i, c);
                if (KC) in.cnn = ldR(F_NN, i, c);
                if (ENERGY) in.wnn = ldW(F_NN, i, c);
            }
            if (ownM && i < Mx) {
                in.lam = ldK(F_MM0, i, c);
                in.m2 = ldK(F_MM1, i, c);
                if (KR) { in.rm0 = ldR(F_MM0, i, c); in.rm1 = ldR(F_MM1, i, c); }
                if (KC) { in.cm0 = ldR(F_MM0, i, c); in.cm1 = ldR(F_MM1, i, c); }
                if (ENERGY) { in.wm3 = ldW(F_MM0, i, c); in.wm4 = ldW(F_MM1, i, c); }
            }
        }
    };

    auto record = [&](int slot, int row, double v) {
        for (int q = rcv_b; q < rcv_e; q++) {
            const int *e = a.rcv + 4 * q;
            if (e[0] == slot && e[1] == row && e[2] == c) a.traces[(long)e[3] * a.max_steps + it] = v;
        }
    };

    auto store = [&](int f, int row, C s, C r, C cc, bool src) {
        if (src) s = to_s<C>(add((double)s, a.src_inc[it]));
        if (!finite(s)) atomicOr(a.flags, FLAG_NONFINITE);
        const long o = (long)row * pitch + c;
        a.out[f][o] = to_s<S>(s);
        if (KR) a.rout[f][o] = to_s<S>(r);
        if (KC) a.rout[f][o] = to_s<S>(cc);
        return s;
    };

    EAcc E;
    Inputs<S, C, CPST> cur{}, nxt{};
    fetch(lb + 1, nxt);
    const int ke = x1e + LAG_S;
    for (int k = lb + 1; k <= ke; k++) {
        cur = nxt;
        if (k + 1 <= ke) fetch(k + 1, nxt);
        const int sr = k - 1;
        if (sr >= lb && sr <= le) {
            rNN.at(sr, t) = cur.nn;
            if (sr < Mx) { rM0.at(sr, t) = cur.mm0; rM1.at(sr, t) = cur.mm1; }
        }
        // old stress rows up to k-1 are staged; rows up to k-2 are visible to other threads
        const int j = k - LAG_V;
        if (velT && j >= vb && j <= ve) {
            const bool ownRow = j >= x0 && j <= x1e;
            if (j < Mx) {   // MN: x from NN (DN closures), SAT from NN rows 0 / Mx, y from MM syy
                C v = C(0);
                if (j < 3) {
#pragma unroll
                    for (int w = 0; w < 5; w++) v = add(v, mul(rNN.at(w, t), a.op.dnL[j][w]));
                } else if (j >= Mx - 3) {
#pragma unroll
                    for (int w = 0; w < 5; w++) v = add(v, mul(rNN.at(Mx - 4 + w, t), a.op.dnR[j - (Mx - 3)][w]));
                } else {
#pragma unroll
                    for (int w = 0; w < 4; w++) v = add(v, mul(rNN.at(j - 1 + w, t), a.op.st[w]));
                }
                C r = KR ? cur.rmn : C(0), cc = KC ? cur.cmn : C(0);
                const C P = cur.pmn;
                r = add(r, mul(v, P));
                if (j < 3) {
                    const C send = add(C(0), mul(a.op.pN, rNN.at(0, t)));
                    r = add(r, mul(mul(a.op.satML[j], sub(send, C(0))), P));
                } else if (j >= Mx - 3) {
                    const C send = add(C(0), mul(a.op.pN, rNN.at(Mx, t)));
                    r = add(r, mul(mul(a.op.satMR[j - (Mx - 3)], sub(send, C(0))), P));
                }
                v = C(0);
#pragma unroll
                for (int w = 0; w < 4; w++) v = add(v, mul(rM1.at(j, t - 2 + w), a.op.st[w]));
                r = add(r, mul(v, P));
                C s = cur.vmn;
                time_update<CPST>(s, r, cc);
                const bool src = a.src_grid == G_MN && j == a.src_ix && pN == a.src_iy;
                if (src) s = to_s<C>(add((double)s, a.src_inc[it]));
                rMN.at(j, t) = s;
                if (ownRow && ownN) {
                    store(F_MN, j, s, r, cc, false);
                    if (ENERGY) E.k = add(E.k, mul(mul((double)s, cur.wmn), (double)s));
                    if (rcv_b < rcv_e) record(F_MN, j, (double)s);
                }
            }
            {   // NM: x from MM sxx (DM closures), SAT from MM rows 0..2 / Mx-3..Mx-1, y from NN
                C v = C(0);
                if (j < 4) {
#pragma unroll
                    for (int w = 0; w < 5; w++) v = add(v, mul(rM0.at(w, t), a.op.dmL[j][w]));
                } else if (j >= Mx - 3) {
#pragma unroll
                    for (int w = 0; w < 5; w++) v = add(v, mul(rM0.at(Mx - 5 + w, t), a.op.dmR[j - (Mx - 3)][w]));
                } else {
#pragma unroll
                    for (int w = 0; w < 4; w++) v = add(v, mul(rM0.at(j - 2 + w, t), a.op.st[w]));
                }
                C r = KR ? cur.rnm : C(0), cc = KC ? cur.cnm : C(0);
                const C P = cur.pnm;
                r = add(r, mul(v, P));
                if (j == 0 || j == Mx) {
                    C send = C(0);
                    if (j == 0) {
#pragma unroll
                        for (int w = 0; w < 3; w++) send = add(send, mul(a.op.pML[w], rM0.at(w, t)));
                        r = add(r, mul(mul(a.op.satNL, sub(send, C(0))), P));
                    } else {
#pragma unroll
                        for (int w = 0; w < 3; w++) send = add(send, mul(a.op.pMR[w], rM0.at(Mx - 3 + w, t)));
                        r = add(r, mul(mul(a.op.satNR, sub(send, C(0))), P));
                    }
                }
                v = C(0);
                if (!(c == -2 || c == -1 || c == My || c == My + 1)) {
                    // taps c-1..c+2 of NN held in the strip's logical columns are the physical
                    // taps of this column (the only NM columns whose values are used lie in
                    // [-2, My+1]; of those, the four next to the seam differ)
#pragma unroll
                    for (int w = 0; w < 4; w++) v = add(v, mul(rNN.at(j, t - 1 + w), a.op.st[w]));
                } else {
                    // a column next to the periodic seam: NN column My and column 0 are distinct
                    // points, so read NN by the physical rule
                    const S *row = a.in[F_NN] + (long)j * pitch;
#pragma unroll
                    for (int w = 0; w < 4; w++) v = add(v, mul(to_c<C>(row[nread(pM - 1 + w, My)]), a.op.st[w]));
                }
                r = add(r, mul(v, P));
                C s = cur.vnm;
                time_update<CPST>(s, r, cc);
                const bool src = a.src_grid == G_NM && j == a.src_ix && pM == a.src_iy;
                if (src) s = to_s<C>(add((double)s, a.src_inc[it]));
                rNM.at(j, t) = s;
                if (ownRow && ownM) {
                    store(F_NM, j, s, r, cc, false);
                    if (ENERGY) E.k = add(E.k, mul(mul((double)s, cur.wnm), (double)s));
                    if (rcv_b < rcv_e) record(F_NM, j, (double)s);
                }
            }
        }
        const int i = k - LAG_S;
        if (core && i >= x0 && i <= x1e) {
            if (ownN) {   // NN: x from MN (DM closures), y from NM
                C v = C(0);
                if (i < 4) {
#pragma unroll
                    for (int w = 0; w < 5; w++) v = add(v, mul(rMN.at(w, t), a.op.dmL[i][w]));
                } else if (i >= Mx - 3) {
#pragma unroll
                    for (int w = 0; w < 5; w++) v = add(v, mul(rMN.at(Mx - 5 + w, t), a.op.dmR[i - (Mx - 3)][w]));
                } else {
#pragma unroll
                    for (int w = 0; w < 4; w++) v = add(v, mul(rMN.at(i - 2 + w, t), a.op.st[w]));
                }
                C r = KR ? cur.rnn : C(0), cc = KC ? cur.cnn : C(0);
                const C P = cur.mu;
                r = add(r, mul(v, P));
                v = C(0);
#pragma unroll
                for (int w = 0; w < 4; w++) v = add(v, mul(rNM.at(i, t - 2 + w), a.op.st[w]));
                r = add(r, mul(v, P));
                const C old = rNN.at(i, t);
                if (ENERGY) E.p0 = add(E.p0, mul(mul((double)old, cur.wnn), (double)old));
                C s = old;
                time_update<CPST>(s, r, cc);
                s = store(F_NN, i, s, r, cc, a.src_grid == G_NN && i == a.src_ix && c == a.src_iy);
                if (ENERGY) E.p1 = add(E.p1, mul(mul((double)s, cur.wnn), (double)s));
                if (rcv_b < rcv_e) record(F_NN, i, (double)s);
            }
            if (ownM && i < Mx) {   // MM: x from NM (DN closures), y from MN
                C v = C(0);
                if (i < 3) {
#pragma unroll
                    for (int w = 0; w < 5; w++) v = add(v, mul(rNM.at(w, t), a.op.dnL[i][w]));
                } else if (i >= Mx - 3) {
#pragma unroll
                    for (int w = 0; w < 5; w++) v = add(v, mul(rNM.at(Mx - 4 + w, t), a.op.dnR[i - (Mx - 3)][w]));
                } else {
#pragma unroll
                    for (int w = 0; w < 4; w++) v = add(v, mul(rNM.at(i - 1 + w, t), a.op.st[w]));
                }
                C r0 = KR ? cur.rm0 : C(0), c0 = KC ? cur.cm0 : C(0);
                C r1 = KR ? cur.rm1 : C(0), c1 = KC ? cur.cm1 : C(0);
                const C L = cur.lam, M2 = cur.m2;
                r0 = add(r0, mul(v, L));
                r1 = add(r1, mul(v, L));
                r0 = add(r0, mul(v, M2));
                v = C(0);
#pragma unroll
                for (int w = 0; w < 4; w++) v = add(v, mul(rMN.at(i, t - 1 + w), a.op.st[w]));
                r0 = add(r0, mul(v, L));
                r1 = add(r1, mul(v, L));
                r1 = add(r1, mul(v, M2));
                const C o0 = rM0.at(i, t), o1 = rM1.at(i, t);
                if (ENERGY) {
                    E.p0 = add(E.p0, mul(mul((double)o0, cur.wm3), (double)o0));
                    E.p0 = add(E.p0, mul(mul((double)o1, cur.wm3), (double)o1));
                    E.p0 = add(E.p0, mul(mul((double)o0, cur.wm4), (double)o1));
                }
                C s0 = o0, s1 = o1;
                time_update<CPST>(s0, r0, c0);
                time_update<CPST>(s1, r1, c1);
                const bool src = a.src_grid == G_MM && i == a.src_ix && c == a.src_iy;
                s0 = store(F_MM0, i, s0, r0, c0, src);
                s1 = store(F_MM1, i, s1, r1, c1, src);
                if (ENERGY) {
                    E.p1 = add(E.p1, mul(mul((double)s0, cur.wm3), (double)s0));
                    E.p1 = add(E.p1, mul(mul((double)s1, cur.wm3), (double)s1));
                    E.p1 = add(E.p1, mul(mul((double)s0, cur.wm4), (double)s1));
                }
                if (rcv_b < rcv_e) { record(F_MM0, i, (double)s0); record(F_MM1, i, (double)s1); }
            }
        }
        __syncthreads();
    }

    if (ENERGY) {
        __shared__ double red[3][NT / 32];
        double e3[3] = {E.p0, E.k, E.p1};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            double v = e3[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if ((t & 31) == 0) red[q][t >> 5] = v;
        }
        __syncthreads();
        if (t < 3) {
            double v = 0.;
            for (int w = 0; w < NT / 32; w++) v += red[t][w];
            if (it < a.max_steps) atomicAdd(a.energy + (long)t * a.max_steps + it, 0.5 * v);
        }
    }
    // the last CTA to finish advances the step counter
    __syncthreads();
    if (t == 0) {
        __threadfence();
        const int ticket = atomicAdd(a.done, 1);
        if (ticket == gridDim.x * gridDim.y - 1) {
            *a.done = 0;
            *a.step = it + 1;
            __threadfence();
        }
    }
}

// ---------------------------------------------------------------- launcher
namespace {
template <class C>
constexpr size_t fused_smem() { return sizeof(C) * (size_t)(3 * RS + 2 * RV) * NT; }

template <class S, class C, int N>
cudaError_t set_attr()
{
    cudaError_t e = cudaFuncSetAttribute(k_elastic_fused<S, C, N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fused_smem<C>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_elastic_fused<S, C, N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fused_smem<C>());
}
}  // namespace

// shared-memory opt-in for every variant; called at handle creation, outside any stream capture
template <class S, class C>
cudaError_t prepare_fused()
{
    cudaError_t e;
    if ((e = set_attr<S, C, 0>()) != cudaSuccess) return e;
    if ((e = set_attr<S, C, 1>()) != cudaSuccess) return e;
    if ((e = set_attr<S, C, 2>()) != cudaSuccess) return e;
    if ((e = set_attr<S, C, 3>()) != cudaSuccess) return e;
    if ((e = set_attr<S, C, 4>()) != cudaSuccess) return e;
    if ((e = set_attr<S, C, 5>()) != cudaSuccess) return e;
    return set_attr<S, C, 6>();
}

template <class S, class C>
void launch_fused(const FusedArgs<S, C> &a, int cpst, bool energy, cudaStream_t st)
{
    const dim3 grid(a.n_strip, a.n_seg), block(NT);
    const size_t smem = fused_smem<C>();
#define TW_FUSED_CASE(N)                                                              \
    case N:                                                                           \
        if (energy) k_elastic_fused<S, C, N, true><<<grid, block, smem, st>>>(a);    \
        else k_elastic_fused<S, C, N, false><<<grid, block, smem, st>>>(a);          \
        break;
    switch (cpst) {
        TW_FUSED_CASE(0)
        TW_FUSED_CASE(1)
        TW_FUSED_CASE(2)
        TW_FUSED_CASE(3)
        TW_FUSED_CASE(4)
        TW_FUSED_CASE(5)
        TW_FUSED_CASE(6)
    }
#undef TW_FUSED_CASE
}

template cudaError_t prepare_fused<double, double>();
template cudaError_t prepare_fused<float, float>();
template void launch_fused<double, double>(const FusedArgs<double, double> &, int, bool, cudaStream_t);
template void launch_fused<float, float>(const FusedArgs<float, float> &, int, bool, cudaStream_t);

}  // namespace tw

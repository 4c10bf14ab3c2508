// Fused acoustic time step for the periodic (single-core tree) mode: one launch per step, every
// array read once and written once, for one shot or for a whole batch of shots.
//
// A step (cpu_acoustic.cpp:231-345) updates the velocities Vx (NM grid) and Vy (MN grid) from the
// pressure, then the pressure (MM grid) from the new velocities. Each warp streams down a strip of
// FS_WARP_CORE columns over a segment of pressure rows (two columns per lane, two halo lanes on
// each side, y taps by shuffles, x taps from register windows), computing Vx row j, Vy row j and
// the pressure row j - 2 in one iteration. State ping-pongs between two buffers. Both directions
// are periodic: rows are read through the same wrap rules as the single-shot kernels (an N-type
// row beyond the seam row Mx wraps, an M-type row wraps modulo Mx), so the halo rows of a segment
// at the ends of the grid are the rows at the other end. Per point the arithmetic and the order of
// the terms are those of acoustic.cuh: results are bit-identical to the two-launch kernels.
#include "fused_step.cuh"

namespace tw {

namespace {

template <class C>
struct ARow {   // global values one iteration consumes
    P2<C> p1;                 // old pressure row j + 1
    P2<C> vx, vy;             // old Vx row j, old Vy row j
    P2<C> cx, cy, kap;        // 1/rho of Vx and Vy row j, kappa of pressure row j - 2
    P2<C> rx, ry, rp;         // residuals (R codes) of Vx, Vy row j and pressure row j - 2
};

__device__ __forceinline__ int prow(int r, int Mx) { return r < 0 ? r + Mx : (r >= Mx ? r - Mx : r); }

// per-lane row staging (as in the elastic step): slots of the storage type p1, vx, vy and the
// residuals rx, ry, rp (R codes); slots of the compute type cx, cy, kap
template <class S, class C, int CPST>
struct ARing {
    static constexpr bool KR = Cpst<CPST>::keep_r;
    static constexpr int NS = 3 + (KR ? 3 : 0), NC = 3;
    static constexpr int s_bytes = 32 * 2 * (int)sizeof(S), c_bytes = 32 * 2 * (int)sizeof(C);
    static constexpr int stage = NS * s_bytes + NC * c_bytes;
    static constexpr int depth = sizeof(C) == 8 ? 2 : TW_FS_RING;
    static constexpr int warp = stage * depth;
};

}  // namespace

template <class S, class C, int CPST, bool EDGE>
__device__ void acoustic_warp(const AcShot<S, C> &a, int wstrip, int seg, unsigned char *ring)
{
    constexpr bool KR = Cpst<CPST>::keep_r;
    const int lane = threadIdx.x & 31;
    const int Mx = a.Mx, My = a.My, pitch = (int)a.pitch;
    const int it = *a.step;
    const int y0 = wstrip * FS_WARP_CORE;
    const int c0 = y0 - 4 + 2 * lane, c1 = c0 + 1;
    const int pM0 = pmod(c0, My), pM1 = pmod(c1, My);
    const int pN0 = (c0 >= 0 && c0 <= My) ? c0 : pM0, pN1 = (c1 >= 0 && c1 <= My) ? c1 : pM1;
    const bool core = lane >= 2 && lane < 30;
    const bool oN0 = core && (!EDGE || c0 <= My), oN1 = core && (!EDGE || c1 <= My);
    const bool oM0 = core && (!EDGE || c0 < My), oM1 = core && (!EDGE || c1 < My);
    const int x0 = (int)((long)seg * Mx / a.n_seg), x1 = (int)((long)(seg + 1) * Mx / a.n_seg);   // pressure rows [x0, x1)

    auto ld2 = [&](const auto *row, int pa, int pb) {
        using T = typename std::remove_cv<typename std::remove_pointer<decltype(row)>::type>::type;
        if (!EDGE) {
            const typename Vec2<T>::T v = *reinterpret_cast<const typename Vec2<T>::T *>(row + c0);
            return P2<C>{to_c<C>(v.x), to_c<C>(v.y)};
        }
        return ld2_any<C>(row, pa, pb);
    };
    auto rowp = [&](const auto *base, int r) { return base + (long)r * pitch; };
    using RG = ARing<S, C, CPST>;
    constexpr int D = RG::depth;
    auto sslot = [&](int st, int k) { return ring + st * RG::stage + k * RG::s_bytes + lane * 2 * (int)sizeof(S); };
    auto cslot = [&](int st, int k) { return ring + st * RG::stage + RG::NS * RG::s_bytes + k * RG::c_bytes + lane * 2 * (int)sizeof(C); };
    auto put2 = [&](unsigned char *dst, const auto *row, int pa, int pb, bool pred) {
        using T = typename std::remove_cv<typename std::remove_pointer<decltype(row)>::type>::type;
        if (!EDGE) {
            cp_async<2 * (int)sizeof(T)>(dst, row + c0, pred);
        } else {
            cp_async<(int)sizeof(T)>(dst, row + pa, pred);
            cp_async<(int)sizeof(T)>(dst + sizeof(T), row + pb, pred);
        }
    };
    // row j's values into ring stage st (rows outside the segment's use are zero-filled, their
    // addresses clamped into the grid)
    auto issue = [&](int j, int st) {
        const int jn = nread(j, Mx);
        const bool vrow = j >= x0 && j < x1;
        const int jv = vrow ? j : x0, i = j - 2;
        const bool prw = i >= x0 && i < x1;
        const int ip = prw ? i : x0;
        put2(sslot(st, 0), rowp(a.in[F_MM0], prow(j + 1, Mx)), pM0, pM1, true);
        put2(sslot(st, 1), rowp(a.in[F_NM], jn), pM0, pM1, true);
        put2(sslot(st, 2), rowp(a.in[F_MN], jv), pN0, pN1, vrow);
        if constexpr (KR) {
            put2(sslot(st, 3), rowp(a.rin[F_NM], jn), pM0, pM1, true);
            put2(sslot(st, 4), rowp(a.rin[F_MN], jv), pN0, pN1, vrow);
            put2(sslot(st, 5), rowp(a.rin[F_MM0], ip), pM0, pM1, prw);
        }
        put2(cslot(st, 0), rowp(a.coef[F_NM], jn), pM0, pM1, true);
        put2(cslot(st, 1), rowp(a.coef[F_MN], jv), pN0, pN1, vrow);
        put2(cslot(st, 2), rowp(a.coef[F_MM0], ip), pM0, pM1, prw);
    };
    auto read = [&](int st, ARow<C> &in) {
        auto rS = [&](int k) {
            const typename Vec2<S>::T v = *reinterpret_cast<const typename Vec2<S>::T *>(sslot(st, k));
            return P2<C>{to_c<C>(v.x), to_c<C>(v.y)};
        };
        auto rC = [&](int k) {
            const typename Vec2<C>::T v = *reinterpret_cast<const typename Vec2<C>::T *>(cslot(st, k));
            return P2<C>{v.x, v.y};
        };
        in.p1 = rS(0);
        in.vx = rS(1);
        in.vy = rS(2);
        if constexpr (KR) {
            in.rx = rS(3);
            in.ry = rS(4);
            in.rp = rS(5);
        }
        in.cx = rC(0);
        in.cy = rC(1);
        in.kap = rC(2);
    };

    // receivers of this lane's columns (at most RC kept in registers; more: scan the shot's list).
    // The warp reads the list 32 entries at a time, one per lane, and keeps those in its strip and
    // rows, so a long list costs no chain of dependent loads.
    constexpr int RC = 2;
    int rq[RC], nr = 0;
    bool rmany = false;
    for (int base = 0; base < a.n_rcv; base += 32) {
        const int q = base + lane;
        int col = -1, row = -1;
        if (q < a.n_rcv) {
            row = a.rcv[4 * q + 1];
            col = a.rcv[4 * q + 2];
        }
        unsigned m = __ballot_sync(FULL, col >= y0 && col < y0 + FS_WARP_CORE + 2 && row >= x0 && row <= x1);
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            const int cc = __shfl_sync(FULL, col, b);
            if (core && (cc == c0 || cc == c1)) {
                if (nr < RC) rq[nr++] = base + b;
                else rmany = true;
            }
        }
    }
    auto record = [&](int slot, int row, int col, double v) {
        auto hit = [&](int q) {
            const int *e = a.rcv + 4 * q;
            if (e[0] == slot && e[1] == row && e[2] == col) a.traces[(long)e[3] * a.max_steps + it] = v;
        };
        if (rmany) {
            for (int q = 0; q < a.n_rcv; q++) hit(q);
        } else {
#pragma unroll
            for (int k = 0; k < RC; k++)
                if (k < nr) hit(rq[k]);
        }
    };
    auto put = [&](int f, int row, const P2<C> &s, const P2<C> &r, bool o0, bool o1) {
        S *o = a.out[f] + (long)row * pitch;
        S *ro = KR ? a.rout[f] + (long)row * pitch : nullptr;
        if ((o0 && !finite(s.a)) || (o1 && !finite(s.b))) atomicOr(a.flags, FLAG_NONFINITE);
        if (!EDGE) {
            if (o0) {
                *reinterpret_cast<typename Vec2<S>::T *>(o + c0) = {to_s<S>(s.a), to_s<S>(s.b)};
                if (KR) *reinterpret_cast<typename Vec2<S>::T *>(ro + c0) = {to_s<S>(r.a), to_s<S>(r.b)};
            }
        } else {
            if (o0) { o[c0] = to_s<S>(s.a); if (KR) ro[c0] = to_s<S>(r.a); }
            if (o1) { o[c1] = to_s<S>(s.b); if (KR) ro[c1] = to_s<S>(r.b); }
        }
        if (nr > 0 || rmany) {
            if (o0) record(f, row, c0, (double)s.a);
            if (o1) record(f, row, c1, (double)s.b);
        }
    };
    auto src_add = [&](int grid, int row, P2<C> &s, int pa, int pb) {
        if (a.src_grid == grid && row == a.src_ix) {
            if (pa == a.src_iy) s.a = to_s<C>(add((double)s.a, a.src_inc[it]));
            if (pb == a.src_iy) s.b = to_s<C>(add((double)s.b, a.src_inc[it]));
        }
    };
    C unused = C(0);

    // windows: pressure rows j-2..j+1 (old), Vx rows j-3..j (new), Vy rows j-2..j (new)
    P2<C> Pw[4], Xw[4], Yw[3];
    const int jb = x0 - 1, je = x1 + 1;
#pragma unroll
    for (int q = 0; q < 3; q++) Pw[q] = ld2(rowp(a.in[F_MM0], prow(jb - 2 + q, Mx)), pM0, pM1);
    ARow<C> cur;
#pragma unroll
    for (int q = 0; q < D - 1; q++) {   // the first D - 1 rows in flight
        if (jb + q <= je) issue(jb + q, q);
        cp_async_commit();
    }
    int sr = 0;   // ring stage of row j
    for (int j = jb; j <= je; j++) {
        // row j + D - 1 into the stage row j - 1 used (read in the previous iteration)
        if (j + D - 1 <= je) issue(j + D - 1, sr == 0 ? D - 1 : sr - 1);
        cp_async_commit();
        cp_async_wait<D - 1>();
        read(sr, cur);
        sr = sr + 1 == D ? 0 : sr + 1;
        Pw[3] = cur.p1;
        {   // Vx (NM) row j: x derivative of the pressure rows j-2..j+1 (dx_periodic<false>)
            P2<C> v{C(0), C(0)};
#pragma unroll
            for (int w = 0; w < 4; w++) {
                v.a = add(v.a, mul(Pw[w].a, a.op.st[w]));
                v.b = add(v.b, mul(Pw[w].b, a.op.st[w]));
            }
            P2<C> r{KR ? cur.rx.a : C(0), KR ? cur.rx.b : C(0)};
            r.a = add(r.a, mul(v.a, cur.cx.a));
            r.b = add(r.b, mul(v.b, cur.cx.b));
            P2<C> s = cur.vx;
            time_update<CPST>(s.a, r.a, unused);
            time_update<CPST>(s.b, r.b, unused);
            const int jn = nread(j, Mx);
            src_add(G_NM, jn, s, pM0, pM1);
            Xw[3] = s;
            if ((j >= x0 && j < x1) || (j == Mx && x1 == Mx)) put(F_NM, jn, s, r, oM0, oM1);   // the seam row: last segment
        }
        if (j >= x0 && j < x1) {   // Vy (MN) row j: y derivative of pressure row j (dy_periodic<false>)
            P2<C> p, n;
            lanes(Pw[2], p, n);
            const P2<C> v = dyNfromM(a.op, Pw[2], p, n);
            P2<C> r{KR ? cur.ry.a : C(0), KR ? cur.ry.b : C(0)};
            r.a = add(r.a, mul(v.a, cur.cy.a));
            r.b = add(r.b, mul(v.b, cur.cy.b));
            P2<C> s = cur.vy;
            time_update<CPST>(s.a, r.a, unused);
            time_update<CPST>(s.b, r.b, unused);
            src_add(G_MN, j, s, pN0, pN1);
            Yw[2] = s;
            put(F_MN, j, s, r, oN0, oN1);
        }
        const int i = j - 2;
        if (i >= x0) {   // pressure row i: x from Vx rows i-1..i+2, then y from Vy row i
            P2<C> p, n;
            lanes(Yw[0], p, n);
            const P2<C> vy = dyMfromN(a.op, Yw[0], p, n);
            P2<C> vx{C(0), C(0)};
#pragma unroll
            for (int w = 0; w < 4; w++) {
                vx.a = add(vx.a, mul(Xw[w].a, a.op.st[w]));
                vx.b = add(vx.b, mul(Xw[w].b, a.op.st[w]));
            }
            P2<C> r{KR ? cur.rp.a : C(0), KR ? cur.rp.b : C(0)};
            r.a = add(r.a, mul(vx.a, cur.kap.a));
            r.b = add(r.b, mul(vx.b, cur.kap.b));
            r.a = add(r.a, mul(vy.a, cur.kap.a));
            r.b = add(r.b, mul(vy.b, cur.kap.b));
            P2<C> s = Pw[0];
            time_update<CPST>(s.a, r.a, unused);
            time_update<CPST>(s.b, r.b, unused);
            src_add(G_MM, i, s, c0, c1);
            put(F_MM0, i, s, r, oM0, oM1);
        }
        // slide the windows
#pragma unroll
        for (int q = 0; q < 3; q++) Pw[q] = Pw[q + 1];
#pragma unroll
        for (int q = 0; q < 3; q++) Xw[q] = Xw[q + 1];
#pragma unroll
        for (int q = 0; q < 2; q++) Yw[q] = Yw[q + 1];
    }
    cp_async_wait_all();
}

// warp gw of the launch -> (shot, segment, strip); the last CTA advances every shot's step
template <class S, class C, int CPST>
__device__ __forceinline__ void acoustic_fused_body(const AcShot<S, C> *shots, int n_shots, int n_warps, int *done)
{
    extern __shared__ __align__(16) unsigned char smem_ac[];
    unsigned char *ring = smem_ac + (threadIdx.x >> 5) * ARing<S, C, CPST>::warp;
    const int gw = blockIdx.x * FS_WARPS + (threadIdx.x >> 5);
    if (gw < n_warps) {
        int lo = 0, hi = n_shots - 1;   // the shot whose warp range holds gw
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (shots[mid].warp_off <= gw) lo = mid;
            else hi = mid - 1;
        }
        const AcShot<S, C> &a = shots[lo];
        const int local = gw - a.warp_off, seg = local / a.n_wstrip, wstrip = local - seg * a.n_wstrip;
        const int y0 = wstrip * FS_WARP_CORE;
        if (y0 >= 4 && y0 + 60 <= a.My) acoustic_warp<S, C, CPST, false>(a, wstrip, seg, ring);
        else acoustic_warp<S, C, CPST, true>(a, wstrip, seg, ring);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const int ticket = atomicAdd(done, 1);
        if (ticket == gridDim.x - 1) {
            *done = 0;
            for (int k = 0; k < n_shots; k++) *shots[k].step += 1;
            __threadfence();
        }
    }
}

template <class S, class C, int CPST>
__global__ void __launch_bounds__(FS_THREADS_MAX) k_acoustic_fused_one(AcShot<S, C> a, int *done)
{
    acoustic_fused_body<S, C, CPST>(&a, 1, a.n_seg * a.n_wstrip, done);
}

template <class S, class C, int CPST>
__global__ void __launch_bounds__(FS_THREADS_MAX) k_acoustic_fused_batch(const AcShot<S, C> *shots, int n_shots,
                                                                         int n_warps, int *done)
{
    acoustic_fused_body<S, C, CPST>(shots, n_shots, n_warps, done);
}

template <class S, class C, int CPST>
constexpr size_t ac_smem() { return (size_t)FS_WARPS * ARing<S, C, CPST>::warp; }

template <class S, class C>
void launch_acoustic_fused(const AcShot<S, C> &a, int cpst, int *done, cudaStream_t st)
{
    const int warps = a.n_seg * a.n_wstrip;
    const dim3 grid((warps + FS_WARPS - 1) / FS_WARPS), block(FS_THREADS_MAX);
    if (cpst == 0) k_acoustic_fused_one<S, C, 0><<<grid, block, ac_smem<S, C, 0>(), st>>>(a, done);
    else if (cpst == 4) k_acoustic_fused_one<S, C, 4><<<grid, block, ac_smem<S, C, 4>(), st>>>(a, done);
    else k_acoustic_fused_one<S, C, 6><<<grid, block, ac_smem<S, C, 6>(), st>>>(a, done);
}

template <class S, class C>
void launch_acoustic_fused_batch(const AcShot<S, C> *shots, int n_shots, int n_warps, int cpst, int *done,
                                 cudaStream_t st)
{
    const dim3 grid((n_warps + FS_WARPS - 1) / FS_WARPS), block(FS_THREADS_MAX);
    if (cpst == 0) k_acoustic_fused_batch<S, C, 0><<<grid, block, ac_smem<S, C, 0>(), st>>>(shots, n_shots, n_warps, done);
    else if (cpst == 4) k_acoustic_fused_batch<S, C, 4><<<grid, block, ac_smem<S, C, 4>(), st>>>(shots, n_shots, n_warps, done);
    else k_acoustic_fused_batch<S, C, 6><<<grid, block, ac_smem<S, C, 6>(), st>>>(shots, n_shots, n_warps, done);
}

template void launch_acoustic_fused<double, double>(const AcShot<double, double> &, int, int *, cudaStream_t);
template void launch_acoustic_fused<float, float>(const AcShot<float, float> &, int, int *, cudaStream_t);
template void launch_acoustic_fused_batch<double, double>(const AcShot<double, double> *, int, int, int, int *, cudaStream_t);
template void launch_acoustic_fused_batch<float, float>(const AcShot<float, float> *, int, int, int, int *, cudaStream_t);

}  // namespace tw

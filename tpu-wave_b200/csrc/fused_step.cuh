// Fused elastic time step: one launch per step, every field read once and written once.
//
// A step (forward_simulation.cpp:38-113) updates the velocities from the stresses, then the
// stresses from the new velocities. This kernel does both in one pass over the grid, reading
// the state from one buffer and writing it to the other (neighbouring CTAs read old values that
// this CTA overwrites). Two kinds of CTA share the launch:
//
// * interior CTAs (rows [FS_ZONE, Mx - FS_ZONE)): FS_WARPS independent warps, each streaming
//   down a strip of FS_WARP_CORE columns over one row segment, two columns per lane. The x
//   stencil windows live in registers, the y taps come from the neighbouring lanes by warp
//   shuffles, two lanes on each side are halo (their velocities feed the stress y taps of the
//   core lanes). A warp computes velocity row j and then stress row j - 2; each lane stages its
//   own rows a few ahead through a private cp.async ring in shared memory, so no block barrier
//   is used. Of the halo rows around a segment only the velocity rows that feed a stress row of
//   the segment are computed. These rows never touch an SBP closure or an SAT penalty.
// * boundary CTAs (the FS_ZONE rows at each free surface, or the whole grid when it is small):
//   a strip of FS_BND_TY columns, its threads split into row groups; phase 1 computes the
//   velocities of the zone (and two rows beyond) from global memory with the closure and SAT
//   operators into a shared tile, phase 2 the stresses from that tile. They take the lowest
//   block indices: their strips are the longest work items, and started first they end before
//   the last wave of interior CTAs instead of after it.
//
// Per point the arithmetic and the order of the right-hand-side terms are those of
// step_kernels.cu (hence of the reference): results are bit-identical.
//
// The templates are instantiated per storage type in fused_f64.cu, fused_f32.cu, fused_bf16.cu
// and fused_f16.cu (separate translation units, compiled in parallel).
#pragma once
#include <type_traits>

#include "kernels.h"
#include "stepper.cuh"

namespace tw {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int pmod(int c, int n)
{
    const int r = c % n;
    return r < 0 ? r + n : r;
}

template <class C>
struct P2 {
    C a, b;
};

template <class S> struct Vec2;
template <> struct Vec2<float> { using T = float2; };
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<__nv_bfloat16> { using T = __nv_bfloat162; };
template <> struct Vec2<__half> { using T = __half2; };

// a pair of values at physical columns pa, pb of one row (one vector load when they are
// adjacent and aligned)
template <class C, class S>
__device__ __forceinline__ P2<C> ld2_any(const S *row, int pa, int pb)
{
    if (pb == pa + 1 && !(pa & 1)) {
        const typename Vec2<S>::T v = *reinterpret_cast<const typename Vec2<S>::T *>(row + pa);
        return {to_c<C>(v.x), to_c<C>(v.y)};
    }
    return {to_c<C>(row[pa]), to_c<C>(row[pb])};
}

template <class C>
__device__ __forceinline__ P2<C> ldg2_any(const C *row, int pa, int pb)
{
    if (pb == pa + 1 && !(pa & 1)) {
        const typename Vec2<C>::T v = __ldg(reinterpret_cast<const typename Vec2<C>::T *>(row + pa));
        return {v.x, v.y};
    }
    return {__ldg(row + pa), __ldg(row + pb)};
}

struct EAcc {
    double p0 = 0., k = 0., p1 = 0.;
};

// neighbouring lanes' pairs: p = lane - 1 (columns c0-2, c0-1), n = lane + 1 (c0+2, c0+3)
template <class C>
__device__ __forceinline__ void lanes(const P2<C> &v, P2<C> &p, P2<C> &n)
{
    p.a = __shfl_up_sync(FULL, v.a, 1);
    p.b = __shfl_up_sync(FULL, v.b, 1);
    n.a = __shfl_down_sync(FULL, v.a, 1);
    n.b = __shfl_down_sync(FULL, v.b, 1);
}

// y derivative of an N-type-y point from M-type taps c-2..c+1 (a: column c0, b: column c1)
template <class C>
__device__ __forceinline__ P2<C> dyNfromM(const Ops<C> &o, const P2<C> &v, const P2<C> &p, const P2<C> &n)
{
    const C ta[4] = {p.a, p.b, v.a, v.b}, tb[4] = {p.b, v.a, v.b, n.a};
    P2<C> r{C(0), C(0)};
#pragma unroll
    for (int w = 0; w < 4; w++) {
        r.a = add(r.a, mul(ta[w], o.st[w]));
        r.b = add(r.b, mul(tb[w], o.st[w]));
    }
    return r;
}

// y derivative of an M-type-y point from N-type taps c-1..c+2
template <class C>
__device__ __forceinline__ P2<C> dyMfromN(const Ops<C> &o, const P2<C> &v, const P2<C> &p, const P2<C> &n)
{
    const C ta[4] = {p.b, v.a, v.b, n.a}, tb[4] = {v.a, v.b, n.a, n.b};
    P2<C> r{C(0), C(0)};
#pragma unroll
    for (int w = 0; w < 4; w++) {
        r.a = add(r.a, mul(ta[w], o.st[w]));
        r.b = add(r.b, mul(tb[w], o.st[w]));
    }
    return r;
}

template <class C>
struct Row {   // global values one interior iteration consumes
    P2<C> nn, mm0, mm1;           // old stress rows j+2, j+1, j
    P2<C> vmn, vnm, pmn, pnm;     // old velocities and 1/rho of velocity row j
    P2<C> rmn, rnm;               // compensation of velocity row j
    P2<C> mu, lam, m2;            // coefficients of stress row j-2
    P2<C> rnn, rm0, rm1;          // compensation of stress row j-2
    P2<double> wmn, wnm, wnn, wm3, wm4;
};

// ---- per-lane row staging through shared memory
// Each interior warp owns a ring of RING_DEPTH row stages in shared memory. A lane copies the
// values it will need for a row asynchronously (cp.async) into its own slots a few rows ahead and
// reads them back when the row comes up: the copies need no registers while in flight, and as a
// lane only ever reads what it copied itself, no warp or block barrier is involved.
// resident CTAs per SM the register allocation is sized for (an FP64 value takes two registers:
// at the FP32 counts the FP64 kernels spilled 400-640 bytes a thread)
template <class C, bool ENERGY>
constexpr int fs_min_blocks()
{
    return sizeof(C) == 8 ? (ENERGY ? TW_FS_MIN_BLOCKS_E64 : TW_FS_MIN_BLOCKS_64) : (ENERGY ? TW_FS_MIN_BLOCKS_E : TW_FS_MIN_BLOCKS);
}

template <class C, bool ENERGY>
constexpr int ring_depth() { return (sizeof(C) == 8 || ENERGY) ? 2 : TW_FS_RING; }

template <class S, class C, int CPST, bool ENERGY, class K = C>
struct RingLayout {
    static constexpr bool KR = Cpst<CPST>::keep_r, KC = Cpst<CPST>::keep_c, SPLIT = Cpst<CPST>::split;
    // slots of the storage type: nn, mm0, mm1, vmn, vnm; their lo parts (split); the residuals
    // rmn, rnm, rnn, rm0, rm1 (R and C codes)
    static constexpr int NS = 5 + (SPLIT ? 5 : 0) + ((KR || KC) ? 5 : 0);
    static constexpr int NC = 5;                      // pmn, pnm, mu, lam, m2 (coefficient type K)
    static constexpr int NE = ENERGY ? 5 : 0;         // wmn, wnm, wnn, wm3, wm4 (double)
    static constexpr int s_bytes = 32 * 2 * (int)sizeof(S), c_bytes = 32 * 2 * (int)sizeof(K), e_bytes = 32 * 16;
    static constexpr int stage = NS * s_bytes + NC * c_bytes + NE * e_bytes;
    static constexpr int warp = stage * ring_depth<C, ENERGY>();
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// copy `bytes` (4, 8 or 16) from global to shared memory asynchronously; pred false: zero fill
template <int BYTES>
__device__ __forceinline__ void cp_async(void *dst, const void *src, bool pred)
{
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(pred ? 16 : 0) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES), "r"(pred ? BYTES : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

}  // namespace

// the owned values of a lane's column pair (and their residual or low parts) into row pointers o, ro
template <class S, bool EDGE, bool TWO>
__device__ __forceinline__ void store_pair(S *o, S *ro, int c0, int c1, S h0, S h1, S l0, S l1, bool o0, bool o1)
{
    using V2 = typename Vec2<S>::T;
    if (!EDGE) {
        if (o0) {
            *reinterpret_cast<V2 *>(o + c0) = V2{h0, h1};
            if (TWO) *reinterpret_cast<V2 *>(ro + c0) = V2{l0, l1};
        }
    } else if (o0 && o1 && !(c0 & 1)) {
        *reinterpret_cast<V2 *>(o + c0) = V2{h0, h1};
        if (TWO) *reinterpret_cast<V2 *>(ro + c0) = V2{l0, l1};
    } else {
        if (o0) { o[c0] = h0; if (TWO) ro[c0] = l0; }
        if (o1) { o[c1] = h1; if (TWO) ro[c1] = l1; }
    }
}

// ------------------------------------------------------------------------------- interior warp
// EDGE: the strip touches the periodic wrap or the end of a row, so lanes may have non-adjacent
// physical columns, unowned columns or the seam; otherwise every pair is adjacent, aligned and
// owned by the core lanes, and loads and stores are single vector accesses
// PUSH: the slab is linked to its neighbours (tw_slab_run) and stores its rows next to a cut into
// their halo rows as well
template <class S, class C, int CPST, bool ENERGY, bool EDGE, class K, bool PUSH>
__device__ void interior_warp(const FusedArgs<S, C> &a, int y0, int seg, int it, int rcv_b, int rcv_e, EAcc &E,
                              unsigned char *ring)
{
    constexpr bool KR = Cpst<CPST>::keep_r, KC = Cpst<CPST>::keep_c, SPLIT = Cpst<CPST>::split;
    const int lane = threadIdx.x & 31;
    const int Mx = a.Mx, My = a.My, pitch = (int)a.pitch;
    // y0: the first of the strip's FS_WARP_CORE columns (even)
    const int c0 = y0 - 4 + 2 * lane, c1 = c0 + 1;
    const int pM0 = pmod(c0, My), pM1 = pmod(c1, My);
    const int pN0 = (c0 >= 0 && c0 <= My) ? c0 : pM0, pN1 = (c1 >= 0 && c1 <= My) ? c1 : pM1;
    const bool core = lane >= 2 && lane < 30;
    const bool oN0 = core && (!EDGE || c0 <= My), oN1 = core && (!EDGE || c1 <= My);
    const bool oM0 = core && (!EDGE || c0 < My), oM1 = core && (!EDGE || c1 < My);
    // balanced segments of the interior rows [ir0, ir0 + int_rows)
    const int x0 = a.ir0 + (int)((long)seg * a.int_rows / a.n_int_seg);
    const int x1 = a.ir0 + (int)((long)(seg + 1) * a.int_rows / a.n_int_seg);   // rows [x0, x1)
    // NM columns next to the periodic seam read NN by the physical rule (column My and column 0
    // of an N-type-y grid are distinct points)
    const bool seam0 = EDGE && (c0 == -2 || c0 == -1 || c0 == My || c0 == My + 1);
    const bool seam1 = EDGE && (c1 == -2 || c1 == -1 || c1 == My || c1 == My + 1);

    auto rowp = [&](const S *base, int r) { return base + r * pitch; };
    auto ld2 = [&](const S *row, int pa, int pb) -> P2<C> {
        if (!EDGE) {
            const typename Vec2<S>::T v = *reinterpret_cast<const typename Vec2<S>::T *>(row + c0);
            return {to_c<C>(v.x), to_c<C>(v.y)};
        }
        return ld2_any<C>(row, pa, pb);
    };
    auto ldg2 = [&](const auto *row, int pa, int pb) {
        using T = typename std::remove_cv<typename std::remove_pointer<decltype(row)>::type>::type;
        if (!EDGE) {
            const typename Vec2<T>::T v = __ldg(reinterpret_cast<const typename Vec2<T>::T *>(row + c0));
            return P2<T>{v.x, v.y};
        }
        return ldg2_any<T>(row, pa, pb);
    };
    // a field value pair as the stencil reads it (hi + lo under the split code)
    auto ld2f = [&](int f, int r, int pa, int pb) -> P2<C> {
        P2<C> v = ld2(rowp(a.in[f], r), pa, pb);
        if constexpr (SPLIT) {
            const P2<C> l = ld2(rowp(a.rin[f], r), pa, pb);
            v.a = add(v.a, l.a);
            v.b = add(v.b, l.b);
        }
        return v;
    };
    // ---- row staging: issue(j, st) copies row j's values into ring stage st, read(st, in)
    // converts them into `in`
    using RL = RingLayout<S, C, CPST, ENERGY, K>;
    constexpr int D = ring_depth<C, ENERGY>();
    const int l = lane;
    auto sslot = [&](int st, int k) { return ring + st * RL::stage + k * RL::s_bytes + l * 2 * (int)sizeof(S); };
    auto cslot = [&](int st, int k) { return ring + st * RL::stage + RL::NS * RL::s_bytes + k * RL::c_bytes + l * 2 * (int)sizeof(K); };
    auto coef = [&](int f) { return reinterpret_cast<const K *>(a.coef[f]); };
    auto eslot = [&](int st, int k) {
        return ring + st * RL::stage + RL::NS * RL::s_bytes + RL::NC * RL::c_bytes + k * RL::e_bytes + l * 16;
    };
    // one pair of T at columns (pa, pb) of `row` into dst
    auto put2 = [&](unsigned char *dst, const auto *row, int pa, int pb, bool pred) {
        using T = typename std::remove_cv<typename std::remove_pointer<decltype(row)>::type>::type;
        if (!EDGE) {
            cp_async<2 * (int)sizeof(T)>(dst, row + c0, pred);
        } else if constexpr (sizeof(T) >= 4) {
            cp_async<(int)sizeof(T)>(dst, row + pa, pred);
            cp_async<(int)sizeof(T)>(dst + sizeof(T), row + pb, pred);
        } else {   // 16-bit elements: too small for cp.async, staged through registers
            T *d = reinterpret_cast<T *>(dst);
            d[0] = pred ? row[pa] : T(0.f);
            d[1] = pred ? row[pb] : T(0.f);
        }
    };
    auto issue = [&](int j, int st) {
        put2(sslot(st, 0), rowp(a.in[F_NN], j + 2), pN0, pN1, true);
        put2(sslot(st, 1), rowp(a.in[F_MM0], j + 1), pM0, pM1, true);
        put2(sslot(st, 2), rowp(a.in[F_MM1], j), pM0, pM1, true);
        put2(sslot(st, 3), rowp(a.in[F_MN], j), pN0, pN1, true);
        put2(sslot(st, 4), rowp(a.in[F_NM], j), pM0, pM1, true);
        int k = 5;
        if constexpr (SPLIT) {
            put2(sslot(st, 5), rowp(a.rin[F_NN], j + 2), pN0, pN1, true);
            put2(sslot(st, 6), rowp(a.rin[F_MM0], j + 1), pM0, pM1, true);
            put2(sslot(st, 7), rowp(a.rin[F_MM1], j), pM0, pM1, true);
            put2(sslot(st, 8), rowp(a.rin[F_MN], j), pN0, pN1, true);
            put2(sslot(st, 9), rowp(a.rin[F_NM], j), pM0, pM1, true);
            k = 10;
        }
        const int i = j - 2;
        const bool srow = core && i >= x0 && i < x1;
        if constexpr (KR || KC) {
            put2(sslot(st, k + 0), rowp(a.rin[F_MN], j), pN0, pN1, true);
            put2(sslot(st, k + 1), rowp(a.rin[F_NM], j), pM0, pM1, true);
            put2(sslot(st, k + 2), rowp(a.rin[F_NN], i), pN0, pN1, srow);
            put2(sslot(st, k + 3), rowp(a.rin[F_MM0], i), pM0, pM1, srow);
            put2(sslot(st, k + 4), rowp(a.rin[F_MM1], i), pM0, pM1, srow);
        }
        put2(cslot(st, 0), coef(F_MN) + j * pitch, pN0, pN1, true);
        put2(cslot(st, 1), coef(F_NM) + j * pitch, pM0, pM1, true);
        put2(cslot(st, 2), coef(F_NN) + i * pitch, pN0, pN1, srow);
        put2(cslot(st, 3), coef(F_MM0) + i * pitch, pM0, pM1, srow);
        put2(cslot(st, 4), coef(F_MM1) + i * pitch, pM0, pM1, srow);
        if constexpr (ENERGY) {
            const bool vrow = core && j >= x0 && j < x1;
            put2(eslot(st, 0), a.w[F_MN] + j * pitch, pN0, pN1, vrow);
            put2(eslot(st, 1), a.w[F_NM] + j * pitch, pM0, pM1, vrow);
            put2(eslot(st, 2), a.w[F_NN] + i * pitch, pN0, pN1, srow);
            put2(eslot(st, 3), a.w[F_MM0] + i * pitch, pM0, pM1, srow);
            put2(eslot(st, 4), a.w[F_MM1] + i * pitch, pM0, pM1, srow);
        }
    };
    auto rdS = [&](int st, int k) {
        const typename Vec2<S>::T v = *reinterpret_cast<const typename Vec2<S>::T *>(sslot(st, k));
        return P2<C>{to_c<C>(v.x), to_c<C>(v.y)};
    };
    auto rdC = [&](int st, int k) {
        const typename Vec2<K>::T v = *reinterpret_cast<const typename Vec2<K>::T *>(cslot(st, k));
        return P2<C>{to_c<C>(v.x), to_c<C>(v.y)};
    };
    auto rdF = [&](int st, int k) {   // a field pair as the stencil reads it
        P2<C> v = rdS(st, k);
        if constexpr (SPLIT) {
            const P2<C> lo = rdS(st, k + 5);
            v.a = add(v.a, lo.a);
            v.b = add(v.b, lo.b);
        }
        return v;
    };
    auto read = [&](int st, int j, Row<C> &in) {
        in.nn = rdF(st, 0);
        in.mm0 = rdF(st, 1);
        in.mm1 = rdF(st, 2);
        in.vmn = rdF(st, 3);
        in.vnm = rdF(st, 4);
        if constexpr (KR || KC) {
            constexpr int k = SPLIT ? 10 : 5;
            in.rmn = rdS(st, k + 0);
            in.rnm = rdS(st, k + 1);
            in.rnn = rdS(st, k + 2);
            in.rm0 = rdS(st, k + 3);
            in.rm1 = rdS(st, k + 4);
        }
        in.pmn = rdC(st, 0);
        in.pnm = rdC(st, 1);
        in.mu = rdC(st, 2);
        in.lam = rdC(st, 3);
        in.m2 = rdC(st, 4);
        if constexpr (ENERGY) {
            auto rdE = [&](int k) {
                const double2 v = *reinterpret_cast<const double2 *>(eslot(st, k));
                return P2<double>{v.x, v.y};
            };
            in.wmn = rdE(0);
            in.wnm = rdE(1);
            in.wnn = rdE(2);
            in.wm3 = rdE(3);
            in.wm4 = rdE(4);
        }
        (void)j;
    };

    // this lane's receivers (at most RC of them in registers; more fall back to the CTA list)
    constexpr int RC = 2;
    int rq[RC], nr = 0;
    bool rmany = false;
    for (int q = rcv_b; q < rcv_e; q++) {
        const int col = a.rcv[4 * q + 2];
        if (core && (col == c0 || col == c1)) {
            if (nr < RC) rq[nr++] = q;
            else rmany = true;
        }
    }
    auto record = [&](int slot, int row, int col, double v) {
        auto hit = [&](int q) {
            const int *e = a.rcv + 4 * q;
            if (e[0] == slot && e[1] == row && e[2] == col) a.traces[(long)e[3] * a.max_steps + it] = v;
        };
        if (rmany) {
            for (int q = rcv_b; q < rcv_e; q++) hit(q);
        } else {
#pragma unroll
            for (int k = 0; k < RC; k++)
                if (k < nr) hit(rq[k]);
        }
    };
    // store the owned values of a pair (owned columns are physical: c0 >= 0 for core lanes)
    // the second array holds the residual (R, C codes) or the low part lo = s - hi (split)
    constexpr bool TWO = Cpst<CPST>::any;
    auto put = [&](int f, int row, const P2<C> &s, const P2<C> &r, const P2<C> &cc, bool o0, bool o1) {
        S *o = a.out[f] + row * pitch;
        S *ro = TWO ? a.rout[f] + row * pitch : nullptr;
        if ((o0 && !finite(s.a)) || (o1 && !finite(s.b))) atomicOr(a.flags, FLAG_NONFINITE);
        const S h0 = to_s<S>(s.a), h1 = to_s<S>(s.b);
        S l0{}, l1{};
        if constexpr (SPLIT) { l0 = to_s<S>(sub(s.a, to_c<C>(h0))); l1 = to_s<S>(sub(s.b, to_c<C>(h1))); }
        if constexpr (KR) { l0 = to_s<S>(r.a); l1 = to_s<S>(r.b); }
        if constexpr (KC) { l0 = to_s<S>(cc.a); l1 = to_s<S>(cc.b); }
        store_pair<S, EDGE, TWO>(o, ro, c0, c1, h0, h1, l0, l1, o0, o1);
        // a slab linked to its neighbours also stores its rows next to a cut into their halo rows
        // (the same column layout; peer memory on another GPU is written over NVLink)
        if constexpr (PUSH) {
#pragma unroll
            for (int side = 0; side < 2; side++)
                if ((unsigned)(row - a.push_row[side]) < (unsigned)FS_HALO) {
                    const long pr = (long)(row + a.peer_shift[side]) * pitch;
                    store_pair<S, EDGE, TWO>(a.peer_out[side][f] + pr, TWO ? a.peer_rout[side][f] + pr : nullptr, c0, c1,
                                             h0, h1, l0, l1, o0, o1);
                }
        }
        if (nr > 0 || rmany) {
            if (o0) record(f, row, c0, (double)s.a);
            if (o1) record(f, row, c1, (double)s.b);
        }
    };
    // source increment (double)S + A dt / dx^2, rounded once; only the source row takes the branch
    auto src_add = [&](int grid, int row, P2<C> &s, int pa, int pb) {
        if (a.src_grid == grid && row == a.src_ix) {
            if (pa == a.src_iy) s.a = to_s<C>(add((double)s.a, a.src_inc[it]));
            if (pb == a.src_iy) s.b = to_s<C>(add((double)s.b, a.src_inc[it]));
        }
    };
    auto pair0 = [&](bool keep, const P2<C> &v) { return P2<C>{keep ? v.a : C(0), keep ? v.b : C(0)}; };
    // a new value as storage keeps it (16-bit storage rounds here, before any later use)
    auto q2 = [&](P2<C> &v) {
        v.a = quant<S, C, CPST>(v.a);
        v.b = quant<S, C, CPST>(v.b);
    };

    // windows: NN rows j-2..j+2, MM0 rows j-2..j+1, MM1 rows j-2..j, MN rows j-4..j, NM rows j-3..j
    P2<C> NNw[5], M0w[4], M1w[3], MNw[5]{}, NMw[4]{};   // (the skipped halo rows stay zero)
    const int jb = x0 - 2, je = x1 + 1;
#pragma unroll
    for (int q = 0; q < 4; q++) NNw[q] = ld2f(F_NN, jb - 2 + q, pN0, pN1);
#pragma unroll
    for (int q = 0; q < 3; q++) M0w[q] = ld2f(F_MM0, jb - 2 + q, pM0, pM1);
#pragma unroll
    for (int q = 0; q < 2; q++) M1w[q] = ld2f(F_MM1, jb - 2 + q, pM0, pM1);
    Row<C> cur;
#pragma unroll
    for (int q = 0; q < D - 1; q++) {   // the first D - 1 rows in flight
        if (jb + q <= je) issue(jb + q, q);
        cp_async_commit();
    }
    int sr = 0;   // ring stage of row j
    for (int j = jb; j <= je; j++) {
        // row j + D - 1 goes into the stage row j - 1 used (read in the previous iteration)
        if (j + D - 1 <= je) issue(j + D - 1, sr == 0 ? D - 1 : sr - 1);
        cp_async_commit();
        cp_async_wait<D - 1>();   // row j has landed
        read(sr, j, cur);
        sr = sr + 1 == D ? 0 : sr + 1;
        NNw[4] = cur.nn;
        M0w[3] = cur.mm0;
        M1w[2] = cur.mm1;
        const bool ownV = j >= x0 && j < x1;
        // ---- velocities of row j
        if (j <= x1) {   // MN: x from NN rows j-1..j+2, y from MM syy row j (row x1 + 1 feeds no stress)
            P2<C> p, n;
            lanes(M1w[2], p, n);
            const P2<C> vy = dyNfromM(a.op, M1w[2], p, n);
            P2<C> vx{C(0), C(0)};
#pragma unroll
            for (int w = 0; w < 4; w++) {
                vx.a = add(vx.a, mul(NNw[1 + w].a, a.op.st[w]));
                vx.b = add(vx.b, mul(NNw[1 + w].b, a.op.st[w]));
            }
            P2<C> r = pair0(KR, cur.rmn), cc = pair0(KC, cur.rmn);
            r.a = add(r.a, mul(vx.a, cur.pmn.a));
            r.b = add(r.b, mul(vx.b, cur.pmn.b));
            r.a = add(r.a, mul(vy.a, cur.pmn.a));
            r.b = add(r.b, mul(vy.b, cur.pmn.b));
            P2<C> s = cur.vmn;
            time_update<CPST>(s.a, r.a, cc.a);
            time_update<CPST>(s.b, r.b, cc.b);
            src_add(G_MN, j, s, pN0, pN1);
            q2(s);
            MNw[4] = s;
            if (ownV) {
                put(F_MN, j, s, r, cc, oN0, oN1);
                if (ENERGY) {
                    if (oN0) E.k = add(E.k, mul(mul((double)s.a, cur.wmn.a), (double)s.a));
                    if (oN1) E.k = add(E.k, mul(mul((double)s.b, cur.wmn.b), (double)s.b));
                }
            }
        }
        if (j >= x0 - 1) {   // NM: x from MM sxx rows j-2..j+1, y from NN row j (row x0 - 2 feeds no stress)
            P2<C> p, n;
            lanes(NNw[2], p, n);
            P2<C> vy = dyMfromN(a.op, NNw[2], p, n);
            if (seam0 || seam1) {
                const S *row = rowp(a.in[F_NN], j), *lrow = SPLIT ? rowp(a.rin[F_NN], j) : nullptr;
                auto nnv = [&](int col) {
                    C v = to_c<C>(row[col]);
                    if constexpr (SPLIT) v = add(v, to_c<C>(lrow[col]));
                    return v;
                };
                if (seam0) {
                    vy.a = C(0);
#pragma unroll
                    for (int w = 0; w < 4; w++) vy.a = add(vy.a, mul(nnv(nread(pM0 - 1 + w, My)), a.op.st[w]));
                }
                if (seam1) {
                    vy.b = C(0);
#pragma unroll
                    for (int w = 0; w < 4; w++) vy.b = add(vy.b, mul(nnv(nread(pM1 - 1 + w, My)), a.op.st[w]));
                }
            }
            P2<C> vx{C(0), C(0)};
#pragma unroll
            for (int w = 0; w < 4; w++) {
                vx.a = add(vx.a, mul(M0w[w].a, a.op.st[w]));
                vx.b = add(vx.b, mul(M0w[w].b, a.op.st[w]));
            }
            P2<C> r = pair0(KR, cur.rnm), cc = pair0(KC, cur.rnm);
            r.a = add(r.a, mul(vx.a, cur.pnm.a));
            r.b = add(r.b, mul(vx.b, cur.pnm.b));
            r.a = add(r.a, mul(vy.a, cur.pnm.a));
            r.b = add(r.b, mul(vy.b, cur.pnm.b));
            P2<C> s = cur.vnm;
            time_update<CPST>(s.a, r.a, cc.a);
            time_update<CPST>(s.b, r.b, cc.b);
            src_add(G_NM, j, s, pM0, pM1);
            q2(s);
            NMw[3] = s;
            if (ownV) {
                put(F_NM, j, s, r, cc, oM0, oM1);
                if (ENERGY) {
                    if (oM0) E.k = add(E.k, mul(mul((double)s.a, cur.wnm.a), (double)s.a));
                    if (oM1) E.k = add(E.k, mul(mul((double)s.b, cur.wnm.b), (double)s.b));
                }
            }
        }
        // ---- stresses of row i = j - 2
        const int i = j - 2;
        if (i >= x0) {
            P2<C> p, n;
            lanes(NMw[1], p, n);
            const P2<C> vyN = dyNfromM(a.op, NMw[1], p, n);   // NN y from NM row i
            lanes(MNw[2], p, n);
            const P2<C> vyM = dyMfromN(a.op, MNw[2], p, n);   // MM y from MN row i
            if (core) {
                {   // NN: x from MN rows i-2..i+1
                    P2<C> vx{C(0), C(0)};
#pragma unroll
                    for (int w = 0; w < 4; w++) {
                        vx.a = add(vx.a, mul(MNw[w].a, a.op.st[w]));
                        vx.b = add(vx.b, mul(MNw[w].b, a.op.st[w]));
                    }
                    P2<C> r = pair0(KR, cur.rnn), cc = pair0(KC, cur.rnn);
                    r.a = add(r.a, mul(vx.a, cur.mu.a));
                    r.b = add(r.b, mul(vx.b, cur.mu.b));
                    r.a = add(r.a, mul(vyN.a, cur.mu.a));
                    r.b = add(r.b, mul(vyN.b, cur.mu.b));
                    const P2<C> old = NNw[0];
                    P2<C> s = old;
                    time_update<CPST>(s.a, r.a, cc.a);
                    time_update<CPST>(s.b, r.b, cc.b);
                    src_add(G_NN, i, s, c0, c1);
                    q2(s);
                    put(F_NN, i, s, r, cc, oN0, oN1);
                    if (ENERGY) {
                        if (oN0) {
                            E.p0 = add(E.p0, mul(mul((double)old.a, cur.wnn.a), (double)old.a));
                            E.p1 = add(E.p1, mul(mul((double)s.a, cur.wnn.a), (double)s.a));
                        }
                        if (oN1) {
                            E.p0 = add(E.p0, mul(mul((double)old.b, cur.wnn.b), (double)old.b));
                            E.p1 = add(E.p1, mul(mul((double)s.b, cur.wnn.b), (double)s.b));
                        }
                    }
                }
                {   // MM: x from NM rows i-1..i+2
                    P2<C> vx{C(0), C(0)};
#pragma unroll
                    for (int w = 0; w < 4; w++) {
                        vx.a = add(vx.a, mul(NMw[w].a, a.op.st[w]));
                        vx.b = add(vx.b, mul(NMw[w].b, a.op.st[w]));
                    }
                    P2<C> r0 = pair0(KR, cur.rm0), k0 = pair0(KC, cur.rm0);
                    P2<C> r1 = pair0(KR, cur.rm1), k1 = pair0(KC, cur.rm1);
                    const P2<C> L = cur.lam, M2 = cur.m2;
                    r0.a = add(r0.a, mul(vx.a, L.a));   r0.b = add(r0.b, mul(vx.b, L.b));
                    r1.a = add(r1.a, mul(vx.a, L.a));   r1.b = add(r1.b, mul(vx.b, L.b));
                    r0.a = add(r0.a, mul(vx.a, M2.a));  r0.b = add(r0.b, mul(vx.b, M2.b));
                    r0.a = add(r0.a, mul(vyM.a, L.a));  r0.b = add(r0.b, mul(vyM.b, L.b));
                    r1.a = add(r1.a, mul(vyM.a, L.a));  r1.b = add(r1.b, mul(vyM.b, L.b));
                    r1.a = add(r1.a, mul(vyM.a, M2.a)); r1.b = add(r1.b, mul(vyM.b, M2.b));
                    const P2<C> o0 = M0w[0], o1 = M1w[0];
                    P2<C> s0 = o0, s1 = o1;
                    time_update<CPST>(s0.a, r0.a, k0.a);
                    time_update<CPST>(s0.b, r0.b, k0.b);
                    time_update<CPST>(s1.a, r1.a, k1.a);
                    time_update<CPST>(s1.b, r1.b, k1.b);
                    src_add(G_MM, i, s0, c0, c1);
                    src_add(G_MM, i, s1, c0, c1);
                    q2(s0);
                    q2(s1);
                    put(F_MM0, i, s0, r0, k0, oM0, oM1);
                    put(F_MM1, i, s1, r1, k1, oM0, oM1);
                    if (ENERGY) {
                        if (oM0) {
                            E.p0 = add(E.p0, mul(mul((double)o0.a, cur.wm3.a), (double)o0.a));
                            E.p0 = add(E.p0, mul(mul((double)o1.a, cur.wm3.a), (double)o1.a));
                            E.p0 = add(E.p0, mul(mul((double)o0.a, cur.wm4.a), (double)o1.a));
                            E.p1 = add(E.p1, mul(mul((double)s0.a, cur.wm3.a), (double)s0.a));
                            E.p1 = add(E.p1, mul(mul((double)s1.a, cur.wm3.a), (double)s1.a));
                            E.p1 = add(E.p1, mul(mul((double)s0.a, cur.wm4.a), (double)s1.a));
                        }
                        if (oM1) {
                            E.p0 = add(E.p0, mul(mul((double)o0.b, cur.wm3.b), (double)o0.b));
                            E.p0 = add(E.p0, mul(mul((double)o1.b, cur.wm3.b), (double)o1.b));
                            E.p0 = add(E.p0, mul(mul((double)o0.b, cur.wm4.b), (double)o1.b));
                            E.p1 = add(E.p1, mul(mul((double)s0.b, cur.wm3.b), (double)s0.b));
                            E.p1 = add(E.p1, mul(mul((double)s1.b, cur.wm3.b), (double)s1.b));
                            E.p1 = add(E.p1, mul(mul((double)s0.b, cur.wm4.b), (double)s1.b));
                        }
                    }
                }
            }
        }
        // ---- slide the windows
#pragma unroll
        for (int q = 0; q < 4; q++) NNw[q] = NNw[q + 1];
#pragma unroll
        for (int q = 0; q < 3; q++) M0w[q] = M0w[q + 1];
#pragma unroll
        for (int q = 0; q < 2; q++) M1w[q] = M1w[q + 1];
#pragma unroll
        for (int q = 0; q < 4; q++) MNw[q] = MNw[q + 1];
#pragma unroll
        for (int q = 0; q < 3; q++) NMw[q] = NMw[q + 1];
    }
    cp_async_wait_all();
}

// ------------------------------------------------------------------------------- boundary CTA
// XIF: the x ends joined by the SAT interface (zone kind 3, or 2 on a small grid)
template <class S, class C, int CPST, bool ENERGY, class K, bool XIF>
__device__ void boundary_cta(const FusedArgs<S, C> &a, int bstrip, int zone, int it, int rcv_b, int rcv_e, C *tile,
                             EAcc &E)
{
    constexpr bool KR = Cpst<CPST>::keep_r, KC = Cpst<CPST>::keep_c, SPLIT = Cpst<CPST>::split;
    constexpr int NT = FS_BND_W;                 // tile row length: the strip's logical columns
    constexpr int RG = FS_BND_THREADS / FS_BND_W;   // row groups: thread rows t / NT walk rows g, g + RG, ...
    const int t = threadIdx.x % NT, g = threadIdx.x / NT;
    const int Mx = a.Mx, My = a.My;
    const long pitch = a.pitch;
    const int c = bstrip * FS_BND_TY - 4 + t;
    const int pM = pmod(c, My), pN = (c >= 0 && c <= My) ? c : pM;
    const bool core = t >= 4 && t < 4 + FS_BND_TY;
    const bool ownN = core && c <= My, ownM = core && c < My;
    const bool velT = t >= 2 && t < NT - 2;
    // zone rows zr0[p]..zr1[p] (N-type grids up to zr1, M-type up to min(zr1, Mx - 1)) of one part,
    // or of two (kind 3: the top and the bottom zone in one CTA, when the SAT interface couples
    // the two x ends); velocity rows vr0[p]..vr1[p], stored in the tile from row toff[p]
    int np = 1, zr0[2] = {0, 0}, zr1[2] = {0, 0};
    const int kind = a.zone_kind[zone];
    if (kind == 2) { zr0[0] = 0; zr1[0] = Mx; }
    else if (kind == 0) { zr0[0] = 0; zr1[0] = FS_ZONE - 1; }
    else if (kind == 1 || !XIF) { zr0[0] = Mx - FS_ZONE; zr1[0] = Mx; }
    else { np = 2; zr0[0] = 0; zr1[0] = FS_ZONE - 1; zr0[1] = Mx - FS_ZONE; zr1[1] = Mx; }
    if constexpr (!XIF) np = 1;
    int vr0[2], vr1[2], toff[2] = {0, 0};
    for (int p = 0; p < np; p++) {
        vr0[p] = max(zr0[p] - 2, 0);
        vr1[p] = min(zr1[p] + 2, Mx);
    }
    if (np == 2) toff[1] = vr1[0] - vr0[0] + 1;
    auto tr = [&](int j) { return (XIF && np == 2 && j >= vr0[1]) ? toff[1] + j - vr0[1] : j - vr0[0]; };
    C *tMN = tile, *tNM = tile + a.tile_rows * NT;

    bool mine = false;   // does any receiver of the CTA sit in this thread's column
    for (int q = rcv_b; q < rcv_e; q++) mine |= core && a.rcv[4 * q + 2] == c;
    auto record = [&](int slot, int row, double v) {
        for (int q = rcv_b; q < rcv_e; q++) {
            const int *e = a.rcv + 4 * q;
            if (e[0] == slot && e[1] == row && e[2] == c) a.traces[(long)e[3] * a.max_steps + it] = v;
        }
    };
    auto put = [&](int f, int row, C s, C r, C cc) {
        if (!finite(s)) atomicOr(a.flags, FLAG_NONFINITE);
        const long o = (long)row * pitch + c;
        const S h = to_s<S>(s);
        a.out[f][o] = h;
        if (KR) a.rout[f][o] = to_s<S>(r);
        if (KC) a.rout[f][o] = to_s<S>(cc);
        if (SPLIT) a.rout[f][o] = to_s<S>(sub(s, to_c<C>(h)));
        if (mine) record(f, row, (double)s);
    };
    // a field as the stencil reads it: the stored array, or the pair hi + lo under the split code
    auto FA = [&](int f) {
        if constexpr (SPLIT) return HiLo<S>{a.in[f], a.rin[f]};
        else return a.in[f];
    };
    auto ldr = [&](int f, int row, int col, C &r, C &cc) {
        r = C(0);
        cc = C(0);
        if (KR) r = to_c<C>(a.rin[f][(long)row * pitch + col]);
        if (KC) cc = to_c<C>(a.rin[f][(long)row * pitch + col]);
    };

    // phase 1: velocities of rows vr0..vr1 at every velocity column (physical reads)
    if (velT) {
        for (int p = 0; p < np; p++)
        for (int j = vr0[p] + g; j <= vr1[p]; j += RG) {
            const bool ownRow = j >= zr0[p] && j <= zr1[p];
            if (j < Mx) {   // MN
                C r, cc;
                ldr(F_MN, j, pN, r, cc);
                const C P = ld<C>(reinterpret_cast<const K *>(a.coef[F_MN]), (long)j * pitch + pN);
                C v = dx_from_N<C>(a.op, FA(F_NN), pitch, Mx, j, pN);
                r = add(r, mul(v, P));
                const bool sx = XIF ? satM_if<C>(a.op, Mx, j, [&](int q) { return ld<C>(FA(F_NN), (long)q * pitch + pN); }, v)
                                      : sat_MN<C>(a.op, FA(F_NN), pitch, Mx, j, pN, v);
                if (sx) r = add(r, mul(v, P));
                v = dy_periodic<false, C>(a.op, FA(F_MM1) + (long)j * pitch, My, pN);
                r = add(r, mul(v, P));
                C s = ld<C>(FA(F_MN), (long)j * pitch + pN);
                time_update<CPST>(s, r, cc);
                if (a.src_grid == G_MN && j == a.src_ix)
                    if (pN == a.src_iy) s = to_s<C>(add((double)s, a.src_inc[it]));
                s = quant<S, C, CPST>(s);
                tMN[tr(j) * NT + t] = s;
                if (ownRow && ownN) {
                    put(F_MN, j, s, r, cc);
                    if (ENERGY) E.k = add(E.k, mul(mul((double)s, __ldg(a.w[F_MN] + (long)j * pitch + c)), (double)s));
                }
            }
            {   // NM
                C r, cc;
                ldr(F_NM, j, pM, r, cc);
                const C P = ld<C>(reinterpret_cast<const K *>(a.coef[F_NM]), (long)j * pitch + pM);
                C v = dx_from_M<C>(a.op, FA(F_MM0), pitch, Mx, j, pM);
                r = add(r, mul(v, P));
                const bool sx = XIF ? satN_if<C>(a.op, Mx, j, [&](int q) { return ld<C>(FA(F_MM0), (long)q * pitch + pM); }, v)
                                      : sat_NM<C>(a.op, FA(F_MM0), pitch, Mx, j, pM, v);
                if (sx) r = add(r, mul(v, P));
                v = dy_periodic<true, C>(a.op, FA(F_NN) + (long)j * pitch, My, pM);
                r = add(r, mul(v, P));
                C s = ld<C>(FA(F_NM), (long)j * pitch + pM);
                time_update<CPST>(s, r, cc);
                if (a.src_grid == G_NM && j == a.src_ix)
                    if (pM == a.src_iy) s = to_s<C>(add((double)s, a.src_inc[it]));
                s = quant<S, C, CPST>(s);
                tNM[tr(j) * NT + t] = s;
                if (ownRow && ownM) {
                    put(F_NM, j, s, r, cc);
                    if (ENERGY) E.k = add(E.k, mul(mul((double)s, __ldg(a.w[F_NM] + (long)j * pitch + c)), (double)s));
                }
            }
        }
    }
    __syncthreads();
    // phase 2: stresses of the zone rows from the velocity tile
    if (core) {
        for (int p = 0; p < np; p++)
        for (int i = zr0[p] + g; i <= zr1[p]; i += RG) {
            const long o = (long)i * pitch + c;
            if (ownN) {   // NN
                C r, cc;
                ldr(F_NN, i, c, r, cc);
                const C P = ld<C>(reinterpret_cast<const K *>(a.coef[F_NN]), o);
                C v = dxM<C>(a.op, Mx, i, [&](int rr) { return tMN[tr(rr) * NT + t]; });
                r = add(r, mul(v, P));
                if (XIF && satN_if<C>(a.op, Mx, i, [&](int q) { return tMN[tr(q) * NT + t]; }, v)) r = add(r, mul(v, P));
                v = C(0);
#pragma unroll
                for (int w = 0; w < 4; w++) v = add(v, mul(tNM[tr(i) * NT + t - 2 + w], a.op.st[w]));
                r = add(r, mul(v, P));
                const C old = ld<C>(FA(F_NN), o);
                C s = old;
                time_update<CPST>(s, r, cc);
                if (a.src_grid == G_NN && i == a.src_ix)
                    if (c == a.src_iy) s = to_s<C>(add((double)s, a.src_inc[it]));
                s = quant<S, C, CPST>(s);
                put(F_NN, i, s, r, cc);
                if (ENERGY) {
                    const double w = __ldg(a.w[F_NN] + o);
                    E.p0 = add(E.p0, mul(mul((double)old, w), (double)old));
                    E.p1 = add(E.p1, mul(mul((double)s, w), (double)s));
                }
            }
            if (ownM && i < Mx) {   // MM
                C r0, k0, r1, k1;
                ldr(F_MM0, i, c, r0, k0);
                ldr(F_MM1, i, c, r1, k1);
                const C L = ld<C>(reinterpret_cast<const K *>(a.coef[F_MM0]), o),
                        M2 = ld<C>(reinterpret_cast<const K *>(a.coef[F_MM1]), o);
                C v = dxN<C>(a.op, Mx, i, [&](int rr) { return tNM[tr(rr) * NT + t]; });
                r0 = add(r0, mul(v, L));
                r1 = add(r1, mul(v, L));
                r0 = add(r0, mul(v, M2));
                if (XIF && satM_if<C>(a.op, Mx, i, [&](int q) { return tNM[tr(q) * NT + t]; }, v)) {
                    r0 = add(r0, mul(v, L));
                    r1 = add(r1, mul(v, L));
                    r0 = add(r0, mul(v, M2));
                }
                v = C(0);
#pragma unroll
                for (int w = 0; w < 4; w++) v = add(v, mul(tMN[tr(i) * NT + t - 1 + w], a.op.st[w]));
                r0 = add(r0, mul(v, L));
                r1 = add(r1, mul(v, L));
                r1 = add(r1, mul(v, M2));
                const C o0 = ld<C>(FA(F_MM0), o), o1 = ld<C>(FA(F_MM1), o);
                C s0 = o0, s1 = o1;
                time_update<CPST>(s0, r0, k0);
                time_update<CPST>(s1, r1, k1);
                if (a.src_grid == G_MM && i == a.src_ix && c == a.src_iy) {   // (branch taken by one thread)
                    s0 = to_s<C>(add((double)s0, a.src_inc[it]));
                    s1 = to_s<C>(add((double)s1, a.src_inc[it]));
                }
                s0 = quant<S, C, CPST>(s0);
                s1 = quant<S, C, CPST>(s1);
                put(F_MM0, i, s0, r0, k0);
                put(F_MM1, i, s1, r1, k1);
                if (ENERGY) {
                    const double w3 = __ldg(a.w[F_MM0] + o), w4 = __ldg(a.w[F_MM1] + o);
                    E.p0 = add(E.p0, mul(mul((double)o0, w3), (double)o0));
                    E.p0 = add(E.p0, mul(mul((double)o1, w3), (double)o1));
                    E.p0 = add(E.p0, mul(mul((double)o0, w4), (double)o1));
                    E.p1 = add(E.p1, mul(mul((double)s0, w3), (double)s0));
                    E.p1 = add(E.p1, mul(mul((double)s1, w3), (double)s1));
                    E.p1 = add(E.p1, mul(mul((double)s0, w4), (double)s1));
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------- the launch
// MODE 0: a handle of its own; 1: a slab linked to its neighbours (tw_slab_run); 2: the x ends
// joined by the SAT interface
template <class S, class C, int CPST, bool ENERGY, class K, int MODE = 0>
__global__ void __launch_bounds__(FS_THREADS_MAX, fs_min_blocks<C, ENERGY>()) k_elastic_fused(FusedArgs<S, C> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int it = *a.step;
    const int cta = blockIdx.x;
    const int rcv_b = a.rcv_off[cta], rcv_e = a.rcv_off[cta + 1];
    EAcc E;
    const int n_bnd = a.n_zone * a.n_bstrip;
    if (cta >= n_bnd) {   // interior CTA: FS_WARPS consecutive (segment, strip) warps, segment-major
        const int gw = (cta - n_bnd) * FS_WARPS + (threadIdx.x >> 5);
        if (gw < a.n_int_seg * a.n_wstrip) {
            const int seg = gw / a.n_wstrip, wstrip = gw - seg * a.n_wstrip;
            const int y0 = wstrip * FS_WARP_CORE;
            unsigned char *ring = smem_raw + (threadIdx.x >> 5) * RingLayout<S, C, CPST, ENERGY, K>::warp;
            if (y0 >= 4 && y0 + 60 <= a.My) interior_warp<S, C, CPST, ENERGY, false, K, MODE == 1>(a, y0, seg, it, rcv_b, rcv_e, E, ring);
            else interior_warp<S, C, CPST, ENERGY, true, K, MODE == 1>(a, y0, seg, it, rcv_b, rcv_e, E, ring);
        }
    } else {             // boundary CTA (zone, strip)
        const int b = cta;
        boundary_cta<S, C, CPST, ENERGY, K, MODE == 2>(a, b % a.n_bstrip, b / a.n_bstrip, it, rcv_b, rcv_e,
                                         reinterpret_cast<C *>(smem_raw), E);
    }
    if (ENERGY) {
        __shared__ double red[3][FS_THREADS_MAX / 32];
        double e3[3] = {E.p0, E.k, E.p1};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            double v = e3[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
            if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double v = 0.;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
            if (it < a.max_steps && v != 0.) atomicAdd(a.energy + (long)threadIdx.x * a.max_steps + it, 0.5 * v);
        }
    }
    // the last CTA to finish advances the step counter
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const int ticket = atomicAdd(a.done, 1);
        if (ticket == gridDim.x - 1) {
            *a.done = 0;
            *a.step = it + 1;
            __threadfence();
        }
    }
}

// ------------------------------------------------------------------------------- launcher
// dynamic shared memory: the boundary CTAs' velocity tile or the interior warps' rings
template <class S, class C, int CPST, bool ENERGY, class K = C>
size_t fused_smem_bytes(int tile_rows)
{
    const size_t tile = sizeof(C) * 2 * (size_t)tile_rows * FS_BND_W;
    const size_t rings = (size_t)FS_WARPS * RingLayout<S, C, CPST, ENERGY, K>::warp;
    return tile > rings ? tile : rings;
}

namespace {
template <class S, class C, int N, class K = C>
cudaError_t set_attr(int)
{
    cudaError_t e = cudaFuncSetAttribute(k_elastic_fused<S, C, N, true, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fused_smem_bytes<S, C, N, true, K>(FS_SMALL_MX + 1));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_elastic_fused<S, C, N, false, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fused_smem_bytes<S, C, N, false, K>(FS_SMALL_MX + 1));
    if (e != cudaSuccess || sizeof(S) != sizeof(C) || sizeof(K) != sizeof(C)) return e;
    // the linked-slab and SAT-interface variants (FP32 / FP64 storage)
    const int big = (int)fused_smem_bytes<S, C, N, true, K>(FS_SMALL_MX + 1), small = (int)fused_smem_bytes<S, C, N, false, K>(FS_SMALL_MX + 1);
    if ((e = cudaFuncSetAttribute(k_elastic_fused<S, C, N, true, K, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_elastic_fused<S, C, N, false, K, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, small)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_elastic_fused<S, C, N, true, K, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big)) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_elastic_fused<S, C, N, false, K, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, small);
}
}  // namespace


// shared-memory opt-in for every variant at the largest tile; called at handle creation,
// outside any stream capture
template <class S, class C>
cudaError_t prepare_fused()
{
    const int smem = 0;
    cudaError_t e;
    if constexpr (sizeof(S) < sizeof(C)) {   // 16-bit storage: plain or split; FP32 or FP16 coefficients
        if ((e = set_attr<S, C, 0>(smem)) != cudaSuccess) return e;
        if ((e = set_attr<S, C, 0, __half>(smem)) != cudaSuccess) return e;
        if ((e = set_attr<S, C, 7, __half>(smem)) != cudaSuccess) return e;
        return set_attr<S, C, 7>(smem);
    } else {
        if constexpr (sizeof(C) == 4)        // FP32: FP16 coefficients with the plain update
            if ((e = set_attr<S, C, 0, __half>(smem)) != cudaSuccess) return e;
        if ((e = set_attr<S, C, 0>(smem)) != cudaSuccess) return e;
        if ((e = set_attr<S, C, 1>(smem)) != cudaSuccess) return e;
        if ((e = set_attr<S, C, 2>(smem)) != cudaSuccess) return e;
        if ((e = set_attr<S, C, 3>(smem)) != cudaSuccess) return e;
        if ((e = set_attr<S, C, 4>(smem)) != cudaSuccess) return e;
        if ((e = set_attr<S, C, 5>(smem)) != cudaSuccess) return e;
        return set_attr<S, C, 6>(smem);
    }
}

template <class S, class C>
void launch_fused(const FusedArgs<S, C> &a, int cpst, bool energy, bool coef16, cudaStream_t st)
{
    const dim3 grid(a.n_int_cta + a.n_zone * a.n_bstrip), block(FS_THREADS_MAX);
    if constexpr (sizeof(C) == 4) {
        if (coef16) {   // FP16 coefficients: plain update (and the split pair for 16-bit fields)
#define TW_FUSED_CASE16(N)                                                                                                   \
    case N:                                                                                                                  \
        if (energy) k_elastic_fused<S, C, N, true, __half><<<grid, block, fused_smem_bytes<S, C, N, true, __half>(a.tile_rows), st>>>(a); \
        else k_elastic_fused<S, C, N, false, __half><<<grid, block, fused_smem_bytes<S, C, N, false, __half>(a.tile_rows), st>>>(a);     \
        break;
            if constexpr (sizeof(S) < sizeof(C)) {
                switch (cpst) {
                    TW_FUSED_CASE16(0)
                    TW_FUSED_CASE16(7)
                }
            } else {
                switch (cpst) { TW_FUSED_CASE16(0) }
            }
#undef TW_FUSED_CASE16
            return;
        }
    }
    if constexpr (sizeof(S) == sizeof(C)) {
        // a slab linked to its neighbours (mode 1), or the x ends joined by the SAT interface (2)
        const int mode = a.xif ? 2 : ((a.peer_out[0][0] || a.peer_out[1][0]) ? 1 : 0);
        if (mode) {
#define TW_FUSED_MODE(N)                                                                                  \
    case N:                                                                                               \
        if (mode == 1) {                                                                                  \
            if (energy) k_elastic_fused<S, C, N, true, C, 1><<<grid, block, fused_smem_bytes<S, C, N, true>(a.tile_rows), st>>>(a); \
            else k_elastic_fused<S, C, N, false, C, 1><<<grid, block, fused_smem_bytes<S, C, N, false>(a.tile_rows), st>>>(a);     \
        } else {                                                                                          \
            if (energy) k_elastic_fused<S, C, N, true, C, 2><<<grid, block, fused_smem_bytes<S, C, N, true>(a.tile_rows), st>>>(a); \
            else k_elastic_fused<S, C, N, false, C, 2><<<grid, block, fused_smem_bytes<S, C, N, false>(a.tile_rows), st>>>(a);     \
        }                                                                                                 \
        break;
            switch (cpst) {
                TW_FUSED_MODE(0)
                TW_FUSED_MODE(1)
                TW_FUSED_MODE(2)
                TW_FUSED_MODE(3)
                TW_FUSED_MODE(4)
                TW_FUSED_MODE(5)
                TW_FUSED_MODE(6)
            }
#undef TW_FUSED_MODE
            return;
        }
    }
#define TW_FUSED_CASE(N)                                                                                  \
    case N:                                                                                               \
        if (energy) k_elastic_fused<S, C, N, true, C><<<grid, block, fused_smem_bytes<S, C, N, true>(a.tile_rows), st>>>(a); \
        else k_elastic_fused<S, C, N, false, C><<<grid, block, fused_smem_bytes<S, C, N, false>(a.tile_rows), st>>>(a);     \
        break;
    if constexpr (sizeof(S) < sizeof(C)) {
        switch (cpst) {
            TW_FUSED_CASE(0)
            TW_FUSED_CASE(7)
        }
    } else {
        switch (cpst) {
            TW_FUSED_CASE(0)
            TW_FUSED_CASE(1)
            TW_FUSED_CASE(2)
            TW_FUSED_CASE(3)
            TW_FUSED_CASE(4)
            TW_FUSED_CASE(5)
            TW_FUSED_CASE(6)
        }
    }
#undef TW_FUSED_CASE
}

}  // namespace tw

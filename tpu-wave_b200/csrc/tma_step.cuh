// Fused elastic time step with TMA-staged interior strips (FP32 fields and coefficients, plain
// update): one launch per step, every field read once and written once, bit-identical to the
// per-point kernels (hence to the reference's CPU solver, forward_simulation.cpp:38-113).
//
// Three kinds of work (4 warps each) make the step, in two launches (see k_elastic_side):
// * boundary CTAs (the FS_ZONE rows at each free surface): boundary_cta of fused_step.cuh, in
//   the side launch;
// * warp-strip items: interior_warp of fused_step.cuh over the interior columns that the TMA
//   strips leave, among them the periodic seam (its reads follow the seam rule column by column),
//   the first work items of the TMA strips' persistent CTAs;
// * TMA strip CTAs: one CTA per (row segment, strip of TMA_CORE = 120 columns). Rows arrive in
//   blocks of TMA_ROWS = 4 (one per warp): one thread issues, for every array, a 2-D tensor copy
//   (cp.async.bulk.tensor, 128 columns x 4 rows, no multicast, this GPU's memory only) into a ring
//   in shared memory, completing on an mbarrier. Each warp then computes one row: thread lane
//   owns 4 adjacent columns (lanes 1..30 the strip's core, lanes 0 and 31 its y halo), reads its
//   x stencil rows straight from the rings (no register windows to slide) and its y taps with
//   one 128-bit and two narrow shared loads, writes its new velocities into a ring of their own,
//   and after a CTA barrier the same warp computes the stresses two rows behind from it. One
//   more barrier per block of rows frees the slots the next copies overwrite.
//
// Row bookkeeping of a segment [x0, x1) (stress rows): velocity rows j = x0 - 2 + 4q + warp and
// stress rows i = j - 2 in step q = 0 .. Q-1, Q = ceil((x1 - x0 + 4) / 4). Arrays whose x
// stencils reach around the row (NN, MM0, MM1) sit in 3-block rings based at row x0 - 4; the
// velocity fields and coefficients in 2-block rings based at x0 - 2, the stress coefficients (and
// energy weights) in 2-block rings based at x0 - 4. Copy group G = 0 carries the first block of
// NN, MM0, MM1; group G >= 1 their block G and block G - 1 of every other array. Step q consumes
// groups q and q + 1; group q + 2 is issued when step q starts, into the slots step q - 1 freed.
// (Issuing two steps ahead needs 4- and 3-block rings: 3 CTAs fit on an SM instead of 4, and the
// step is about 12 % slower. Carrying the pipeline on from one item into the next gains nothing
// with these rings: an item consumes one group more than it has steps, so the next item's group 1
// cannot be issued before that item starts.)
// Every wait on an mbarrier gives up after about a second and raises FLAG_TIMEOUT.
#pragma once
#include "fused_step.cuh"

namespace tw {

namespace {

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// wait for the phase of parity `parity` of an mbarrier; false after about `limit` SM cycles
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, long long limit)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
__device__ __forceinline__ void mbar_inval(unsigned long long *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// one 2-D tile (box of the tensor map) at column x, row y into shared memory; completes on bar
__device__ __forceinline__ void tma_load_2d(void *dst, const void *map, int x, int y, unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

constexpr long long TMA_WAIT_LIMIT = 2000000000LL;   // SM cycles: about one second

// shared memory of a TMA strip CTA (byte offsets from a 128-byte aligned base). Q16: the
// coefficients arrive as 16-bit codes in rows of TMA_QW columns (from 8 columns before the strip's
// core), each block padded to a multiple of 128 bytes (TMA destinations are 128-byte aligned)
template <bool ENERGY, bool Q16 = false>
struct TmaLayout {
    // ring lengths in blocks: the arrays whose x stencils reach around the row, the other loaded
    // arrays; NB mbarriers track the copy groups in flight
    static constexpr int R3 = 3, R2 = 2, NB = 3;
    static constexpr int ROW = TMA_W * 4;              // one FP32 row of the strip
    static constexpr int BLK = TMA_ROWS * ROW;         // one block of rows
    static constexpr int CROW = Q16 ? TMA_QW * 2 : ROW;                       // one coefficient row
    static constexpr int CBOX = TMA_ROWS * CROW;                              // bytes a coefficient copy lands
    static constexpr int CBLK = (CBOX + 127) / 128 * 128;                     // one coefficient block
    static constexpr int WROW = TMA_ROWS * TMA_W * 8;  // one block of one FP64 energy-weight array
    static constexpr int PAD = 128;                    // lanes 0 / 31 read up to 8 bytes beyond a row
    static constexpr int o_nn = PAD, o_mm0 = o_nn + R3 * BLK, o_mm1 = o_mm0 + R3 * BLK;
    static constexpr int o_mn = o_mm1 + R3 * BLK, o_nm = o_mn + R2 * BLK, o_pmn = o_nm + R2 * BLK,
                         o_pnm = o_pmn + R2 * CBLK, o_mu = o_pnm + R2 * CBLK, o_lam = o_mu + R2 * CBLK,
                         o_m2 = o_lam + R2 * CBLK;
    static constexpr int o_vmn = o_m2 + R2 * CBLK, o_vnm = o_vmn + 2 * BLK;  // new velocities (2 blocks)
    // the energy weights, one slot per block and set: the velocity rows' (MN, NM) at o_vw, the
    // stress rows' (NN, MM P1, P2) at o_sw, each loaded half a step before its use (see below)
    static constexpr int o_w = o_vnm + 2 * BLK, o_vw = o_w, o_sw = o_w + 2 * WROW;
    // NB mbarriers at o_bar, the item index at o_item, the energy reduction's 3 x FS_WARPS doubles
    // at o_red
    static constexpr int o_bar = o_w + (ENERGY ? 5 * WROW : 0) + PAD;
    static constexpr int NBW = NB + (ENERGY ? 2 : 0);   // barriers: the groups', then the two weight sets'
    static constexpr int o_item = o_bar + 64, o_red = o_bar + 72;
    static constexpr int bytes = o_red + 8 * 3 * FS_WARPS + 128;              // + alignment slack
    static constexpr unsigned tx0 = 3 * BLK;                                // group 0
    static constexpr unsigned tx = 5 * BLK + 5 * CBOX;                      // groups >= 1
};

__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float2 lds2(const float *p) { return *reinterpret_cast<const float2 *>(p); }

// 7 values of a row around this thread's 4 columns: columns c-2 .. c+4 (N-type point from
// M-type taps c-2..c+1) or c-1 .. c+5 (M-type point from N-type taps c-1..c+2)
__device__ __forceinline__ void taps_left2(const float *row, int c, float (&t)[7], float4 mid)
{
    const float2 l = lds2(row + c - 2);
    t[0] = l.x; t[1] = l.y; t[2] = mid.x; t[3] = mid.y; t[4] = mid.z; t[5] = mid.w;
    t[6] = row[c + 4];
}
__device__ __forceinline__ void taps_left1(const float *row, int c, float (&t)[7], float4 mid)
{
    const float2 r = lds2(row + c + 4);
    t[0] = row[c - 1]; t[1] = mid.x; t[2] = mid.y; t[3] = mid.z; t[4] = mid.w; t[5] = r.x; t[6] = r.y;
}
__device__ __forceinline__ float f4(const float4 &v, int e) { return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w)); }

}  // namespace

// one TMA strip CTA: strip `tstrip`, row segment `tseg`; returns false if a copy timed out
template <bool ENERGY, bool Q16>
__device__ bool tma_strip_cta(const FusedArgs<float, float> &a, const TmaMaps &maps, int tstrip, int tseg, int it,
                              int rcv_b, int rcv_e, EAcc &E, unsigned char *base)
{
    using L = TmaLayout<ENERGY, Q16>;
    constexpr int R3 = L::R3, R2 = L::R2, NB = L::NB;
    using C = float;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y0 = TMA_Y0 + tstrip * TMA_CORE;   // the strip's first core column
    const int xs = y0 - 4;                        // its first loaded column (a multiple of 4)
    const int cl = 4 * lane;                      // this thread's first column within the strip
    const int c0 = xs + cl;                       // ... in the grid
    const bool core = lane >= 1 && lane <= 30;
    const int x0 = a.ir0 + (int)((long)tseg * a.int_rows / a.n_tseg);
    const int x1 = a.ir0 + (int)((long)(tseg + 1) * a.int_rows / a.n_tseg);
    const int Q = (x1 - x0 + 7) / 4;
    const long pitch = a.pitch;
    const Ops<C> &op = a.op;
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(base + L::o_bar);

    // this thread's receivers (at most 2 in registers; more fall back to the CTA's list)
    constexpr int RC = 2;
    int rq[RC], nr = 0;
    bool rmany = false;
    if (core)
        for (int q = rcv_b; q < rcv_e; q++) {
            const int col = a.rcv[4 * q + 2];
            if (col >= c0 && col < c0 + 4) {
                if (nr < RC) rq[nr++] = q;
                else rmany = true;
            }
        }
    auto record = [&](int slot, int row, const float (&v)[4]) {
        auto hit = [&](int q) {
            const int *e = a.rcv + 4 * q;
            if (e[0] == slot && e[1] == row && e[2] >= c0 && e[2] < c0 + 4) {
                const int k = e[2] - c0;   // (selected, not indexed: v stays in registers)
                const float x = k == 0 ? v[0] : (k == 1 ? v[1] : (k == 2 ? v[2] : v[3]));
                a.traces[(long)e[3] * a.max_steps + it] = (double)x;
            }
        };
        if (rmany) {
            for (int q = rcv_b; q < rcv_e; q++) hit(q);
        } else {
#pragma unroll
            for (int k = 0; k < RC; k++)
                if (k < nr) hit(rq[k]);
        }
    };

    const unsigned char *mp = maps.m[0];
    auto map = [&](int k) { return static_cast<const void *>(mp + 128 * k); };
    // copy group G (see the head of the file): lane 0 of every warp issues its share of the copies
    // (so that no warp arrives at the CTA's barriers much later than the others), warp 0 also the
    // group's expected bytes on its mbarrier (a copy may complete before them: the phase waits for
    // that one arrival)
    auto issue = [&](int G) {
        unsigned long long *b = bar + G % NB;
        const int s3 = G % R3;
        const int rs = x0 - 4 + 4 * G;
        const int g = G - 1, s2 = (G + 1) % R2;   // (g mod 2, for g >= 0)
        const int rv = x0 - 2 + 4 * g, rt = x0 - 4 + 4 * g;
        const int xc = Q16 ? y0 - 8 : xs;   // (16-bit codes: x on a 16-byte boundary)
        switch (warp) {
        case 0:
            mbar_expect_tx(b, G == 0 ? L::tx0 : L::tx);
            tma_load_2d(base + L::o_nn + s3 * L::BLK, map(TM_NN), xs, rs, b);
            if (G == 0) break;
            tma_load_2d(base + L::o_pmn + s2 * L::CBLK, map(TM_PMN), xc, rv, b);
            tma_load_2d(base + L::o_pnm + s2 * L::CBLK, map(TM_PNM), xc, rv, b);
            break;
        case 1:
            tma_load_2d(base + L::o_mm0 + s3 * L::BLK, map(TM_MM0), xs, rs, b);
            if (G == 0) break;
            tma_load_2d(base + L::o_mu + s2 * L::CBLK, map(TM_MU), xc, rt, b);
            tma_load_2d(base + L::o_lam + s2 * L::CBLK, map(TM_LAM), xc, rt, b);
            break;
        case 2:
            tma_load_2d(base + L::o_mm1 + s3 * L::BLK, map(TM_MM1), xs, rs, b);
            if (G == 0) break;
            tma_load_2d(base + L::o_m2 + s2 * L::CBLK, map(TM_M2), xc, rt, b);
            break;
        default:
            if (G == 0) break;
            tma_load_2d(base + L::o_mn + s2 * L::BLK, map(TM_MN), xs, rv, b);
            tma_load_2d(base + L::o_nm + s2 * L::BLK, map(TM_NM), xs, rv, b);
            break;
        }
    };

    // the energy weights of block qq (thread 0): the velocity rows' set is needed in step qq's
    // first half and loaded during step qq - 1's second half, the stress rows' set is needed in
    // step qq's second half and loaded during its first half; one slot each suffices, and the
    // CTA keeps the shared memory of 3 CTAs per SM (a ring of two blocks per array allowed 2)
    int vw_last = -1, sw_last = -1;   // (thread 0) the last block of each set issued
    auto issue_vw = [&](int qq) {
        unsigned long long *b = bar + NB;
        mbar_expect_tx(b, 2 * L::WROW);
        const int rv = x0 - 2 + 4 * qq;
        tma_load_2d(base + L::o_vw, map(TM_WMN), xs, rv, b);
        tma_load_2d(base + L::o_vw + L::WROW, map(TM_WNM), xs, rv, b);
        vw_last = qq;
    };
    auto issue_sw = [&](int qq) {
        unsigned long long *b = bar + NB + 1;
        mbar_expect_tx(b, 3 * L::WROW);
        const int rt = x0 - 4 + 4 * qq;
        tma_load_2d(base + L::o_sw, map(TM_WNN), xs, rt, b);
        tma_load_2d(base + L::o_sw + L::WROW, map(TM_WM3), xs, rt, b);
        tma_load_2d(base + L::o_sw + 2 * L::WROW, map(TM_WM4), xs, rt, b);
        sw_last = qq;
    };

    if (threadIdx.x == 0) {
        for (int k = 0; k < L::NBW; k++) mbar_init(bar + k, 1);
        mbar_init_fence();
    }
    __syncthreads();
    int issued = -1;   // (lane 0 of each warp) the last group issued
    if (lane == 0) {
        fence_proxy_async();   // the previous item's accesses to this shared memory come first
        for (int G = 0; G <= 2 && G <= Q; G++) issue(G);
        issued = Q < 2 ? Q : 2;
        if constexpr (ENERGY)
            if (warp == 0) {
                issue_vw(0);
                issue_sw(0);
            }
    }
    int waited = -1;   // the last group this thread has seen complete
    float nf = 0.f;    // stays 0 unless a stored value is not finite (v * 0 is NaN for Inf / NaN)
    bool bad = false;
    const float st0 = op.st[0], st1 = op.st[1], st2 = op.st[2], st3 = op.st[3];
    auto rowp = [&](int off, int slot) { return reinterpret_cast<const float *>(base + off) + slot * TMA_W; };
    // this thread's 4 coefficients of ring row `row` (0..7: block row) of the ring at `off`, of
    // field slot f: FP32 values, or 16-bit codes decoded as qlo + qstep * code
    auto coef4 = [&](int off, int row, int f) -> float4 {
        if constexpr (Q16) {
            const unsigned char *r = base + off + (row >> 2) * L::CBLK + (row & 3) * L::CROW;
            const uint2 u = *reinterpret_cast<const uint2 *>(r + 2 * (cl + 4));
            const float lo = a.qlo[f], st = a.qstep[f];
            return make_float4(add(lo, mul(st, (float)(u.x & 0xffffu))), add(lo, mul(st, (float)(u.x >> 16))),
                               add(lo, mul(st, (float)(u.y & 0xffffu))), add(lo, mul(st, (float)(u.y >> 16))));
        } else {
            return lds4(rowp(off, row) + cl);
        }
    };
    // this thread's weights in the set at `off` (array k of it), row `warp` of the block
    auto wrow = [&](int off, int k) { return reinterpret_cast<const double *>(base + off + k * L::WROW) + warp * TMA_W + cl; };
    auto st4 = [&](int f, int row, const float (&v)[4]) {
        *reinterpret_cast<float4 *>(a.out[f] + row * pitch + c0) = make_float4(v[0], v[1], v[2], v[3]);
    };
    auto src = [&](int grid, int row, float (&v)[4]) {
        if (a.src_grid == grid && row == a.src_ix) {
#pragma unroll
            for (int e = 0; e < 4; e++)
                if (c0 + e == a.src_iy) v[e] = to_s<C>(add((double)v[e], a.src_inc[it]));
        }
    };

    for (int q = 0; q < Q; q++) {
        if (lane == 0 && q >= 1 && q + 2 <= Q) {   // into the slots step q - 1 freed
            fence_proxy_async();
            issue(q + 2);
            issued = q + 2;
        }
        if constexpr (ENERGY)
            if (threadIdx.x == 0 && q >= 1) {   // the stress rows' weights: step q - 1 has read their slot
                fence_proxy_async();
                issue_sw(q);
            }
        for (int G = waited + 1; G <= q + 1 && !bad; G++) {
            bad = !mbar_wait(bar + G % NB, (unsigned)((G / NB) & 1), TMA_WAIT_LIMIT);
            if (!bad) waited = G;
        }
        if constexpr (ENERGY)
            if (!bad) bad = !mbar_wait(bar + NB, (unsigned)(q & 1), TMA_WAIT_LIMIT);   // velocity rows' weights
        // 3-block rings: blocks q, q + 1; other loaded rings: block q (slot sl); new-velocity
        // rings: block q (slot s2) and q - 1 (s2p)
        const int s3a = q % R3, s3b = (q + 1) % R3, sl = q % R2, s2 = q & 1, s2p = s2 ^ 1;
        // window row k (0..7) of a 3-block ring: rows x0 - 4 + 4q + k
        auto w3 = [&](int off, int k) { return rowp(off, (k < 4 ? s3a : s3b) * 4 + (k & 3)); };
        // row k (-4..3) of a new-velocity ring relative to row x0 - 2 + 4q
        auto vr = [&](int off, int k) { return rowp(off, (k < 0 ? s2p * 4 + k + 4 : s2 * 4 + k)); };
        const int j = x0 - 2 + 4 * q + warp;   // velocity row of this warp
        const int i = j - 2;                   // stress row of this warp
        if (!bad) {
            const bool ownV = core && j >= x0 && j < x1;
            // ---- MN (row j): x from NN rows j-1..j+2 (window w+1..w+4), y from syy row j
            if (j <= x1) {
                const float4 n1 = lds4(w3(L::o_nn, warp + 1) + cl), n2 = lds4(w3(L::o_nn, warp + 2) + cl),
                             n3 = lds4(w3(L::o_nn, warp + 3) + cl), n4 = lds4(w3(L::o_nn, warp + 4) + cl);
                const float *m1row = w3(L::o_mm1, warp + 2);
                float t[7];
                taps_left2(m1row, cl, t, lds4(m1row + cl));
                const float4 old = lds4(rowp(L::o_mn, sl * 4 + warp) + cl);
                const float4 p = coef4(L::o_pmn, sl * 4 + warp, F_MN);
                float v[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    // the reference sums from 0: 0 + x differs from x only for x = -0, and a
                    // difference in the sign of a zero sum vanishes in r = 0 + vx * p below (and
                    // in any later sum that has a non-zero term): bit-identical results
                    float vx = mul(f4(n1, e), st0);
                    vx = add(vx, mul(f4(n2, e), st1));
                    vx = add(vx, mul(f4(n3, e), st2));
                    vx = add(vx, mul(f4(n4, e), st3));
                    float vy = mul(t[e], st0);
                    vy = add(vy, mul(t[e + 1], st1));
                    vy = add(vy, mul(t[e + 2], st2));
                    vy = add(vy, mul(t[e + 3], st3));
                    float r = 0.f;
                    r = add(r, mul(vx, f4(p, e)));
                    r = add(r, mul(vy, f4(p, e)));
                    v[e] = add(f4(old, e), r);
                }
                src(G_MN, j, v);
                *reinterpret_cast<float4 *>(const_cast<float *>(rowp(L::o_vmn, s2 * 4 + warp)) + cl) = make_float4(v[0], v[1], v[2], v[3]);
                if (ownV) {
                    st4(F_MN, j, v);
#pragma unroll
                    for (int e = 0; e < 4; e++) nf = __fmaf_rn(v[e], 0.f, nf);
                    if (nr > 0 || rmany) record(F_MN, j, v);
                    if constexpr (ENERGY) {
                        const double *wr = wrow(L::o_vw, 0);
#pragma unroll
                        for (int e = 0; e < 4; e++) E.k = add(E.k, mul(mul((double)v[e], wr[e]), (double)v[e]));
                    }
                }
            }
            // ---- NM (row j): x from sxx rows j-2..j+1 (window w..w+3), y from NN row j
            if (j >= x0 - 1) {
                const float4 a0 = lds4(w3(L::o_mm0, warp) + cl), a1 = lds4(w3(L::o_mm0, warp + 1) + cl),
                             a2 = lds4(w3(L::o_mm0, warp + 2) + cl), a3 = lds4(w3(L::o_mm0, warp + 3) + cl);
                const float *nrow = w3(L::o_nn, warp + 2);
                float t[7];
                taps_left1(nrow, cl, t, lds4(nrow + cl));
                const float4 old = lds4(rowp(L::o_nm, sl * 4 + warp) + cl);
                const float4 p = coef4(L::o_pnm, sl * 4 + warp, F_NM);
                float v[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    float vy = mul(t[e], st0);
                    vy = add(vy, mul(t[e + 1], st1));
                    vy = add(vy, mul(t[e + 2], st2));
                    vy = add(vy, mul(t[e + 3], st3));
                    float vx = mul(f4(a0, e), st0);
                    vx = add(vx, mul(f4(a1, e), st1));
                    vx = add(vx, mul(f4(a2, e), st2));
                    vx = add(vx, mul(f4(a3, e), st3));
                    float r = 0.f;
                    r = add(r, mul(vx, f4(p, e)));
                    r = add(r, mul(vy, f4(p, e)));
                    v[e] = add(f4(old, e), r);
                }
                src(G_NM, j, v);
                *reinterpret_cast<float4 *>(const_cast<float *>(rowp(L::o_vnm, s2 * 4 + warp)) + cl) = make_float4(v[0], v[1], v[2], v[3]);
                if (ownV) {
                    st4(F_NM, j, v);
#pragma unroll
                    for (int e = 0; e < 4; e++) nf = __fmaf_rn(v[e], 0.f, nf);
                    if (nr > 0 || rmany) record(F_NM, j, v);
                    if constexpr (ENERGY) {
                        const double *wr = wrow(L::o_vw, 1);
#pragma unroll
                        for (int e = 0; e < 4; e++) E.k = add(E.k, mul(mul((double)v[e], wr[e]), (double)v[e]));
                    }
                }
            }
        }
        if (__syncthreads_or(bad)) {
            bad = true;
            break;
        }
        if constexpr (ENERGY) {
            if (threadIdx.x == 0 && q + 1 < Q) {   // the next block's velocity-row weights: this step has read their slot
                fence_proxy_async();
                issue_vw(q + 1);
            }
            bad = !mbar_wait(bar + NB + 1, (unsigned)(q & 1), TMA_WAIT_LIMIT);   // stress rows' weights
        }
        // ---- stresses of row i = j - 2 (window row warp of the 3-block rings; new-velocity rows
        // relative to x0 - 2 + 4q: i is warp - 2)
        if (!bad && core && i >= x0 && i < x1) {
            const int ir = warp - 2;
            {   // NN: x from new MN rows i-2..i+1, y from new NM row i (taps c-2..c+1)
                const float4 m0 = lds4(vr(L::o_vmn, ir - 2) + cl), m1 = lds4(vr(L::o_vmn, ir - 1) + cl),
                             m2 = lds4(vr(L::o_vmn, ir) + cl), m3 = lds4(vr(L::o_vmn, ir + 1) + cl);
                const float *nmrow = vr(L::o_vnm, ir);
                float t[7];
                taps_left2(nmrow, cl, t, lds4(nmrow + cl));
                const float4 old = lds4(w3(L::o_nn, warp) + cl);
                const float4 mu = coef4(L::o_mu, sl * 4 + warp, F_NN);
                float v[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    float vx = mul(f4(m0, e), st0);
                    vx = add(vx, mul(f4(m1, e), st1));
                    vx = add(vx, mul(f4(m2, e), st2));
                    vx = add(vx, mul(f4(m3, e), st3));
                    float vy = mul(t[e], st0);
                    vy = add(vy, mul(t[e + 1], st1));
                    vy = add(vy, mul(t[e + 2], st2));
                    vy = add(vy, mul(t[e + 3], st3));
                    float r = 0.f;
                    r = add(r, mul(vx, f4(mu, e)));
                    r = add(r, mul(vy, f4(mu, e)));
                    v[e] = add(f4(old, e), r);
                }
                src(G_NN, i, v);
                st4(F_NN, i, v);
#pragma unroll
                for (int e = 0; e < 4; e++) nf = __fmaf_rn(v[e], 0.f, nf);
                if (nr > 0 || rmany) record(F_NN, i, v);
                if constexpr (ENERGY) {
                    const double *wr = wrow(L::o_sw, 0);
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        E.p0 = add(E.p0, mul(mul((double)f4(old, e), wr[e]), (double)f4(old, e)));
                        E.p1 = add(E.p1, mul(mul((double)v[e], wr[e]), (double)v[e]));
                    }
                }
            }
            {   // MM: x from new NM rows i-1..i+2, y from new MN row i (taps c-1..c+2)
                const float4 n0 = lds4(vr(L::o_vnm, ir - 1) + cl), n1 = lds4(vr(L::o_vnm, ir) + cl),
                             n2 = lds4(vr(L::o_vnm, ir + 1) + cl), n3 = lds4(vr(L::o_vnm, ir + 2) + cl);
                const float *mnrow = vr(L::o_vmn, ir);
                float t[7];
                taps_left1(mnrow, cl, t, lds4(mnrow + cl));
                const float4 o0 = lds4(w3(L::o_mm0, warp) + cl), o1 = lds4(w3(L::o_mm1, warp) + cl);
                const float4 lam = coef4(L::o_lam, sl * 4 + warp, F_MM0), m2c = coef4(L::o_m2, sl * 4 + warp, F_MM1);
                float s0[4], s1[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    float vx = mul(f4(n0, e), st0);
                    vx = add(vx, mul(f4(n1, e), st1));
                    vx = add(vx, mul(f4(n2, e), st2));
                    vx = add(vx, mul(f4(n3, e), st3));
                    float vy = mul(t[e], st0);
                    vy = add(vy, mul(t[e + 1], st1));
                    vy = add(vy, mul(t[e + 2], st2));
                    vy = add(vy, mul(t[e + 3], st3));
                    const float L_ = f4(lam, e), M2 = f4(m2c, e);
                    float r0 = 0.f, r1 = 0.f;
                    r0 = add(r0, mul(vx, L_));
                    r1 = add(r1, mul(vx, L_));
                    r0 = add(r0, mul(vx, M2));
                    r0 = add(r0, mul(vy, L_));
                    r1 = add(r1, mul(vy, L_));
                    r1 = add(r1, mul(vy, M2));
                    s0[e] = add(f4(o0, e), r0);
                    s1[e] = add(f4(o1, e), r1);
                }
                src(G_MM, i, s0);
                src(G_MM, i, s1);
                st4(F_MM0, i, s0);
                st4(F_MM1, i, s1);
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    nf = __fmaf_rn(s0[e], 0.f, nf);
                    nf = __fmaf_rn(s1[e], 0.f, nf);
                }
                if (nr > 0 || rmany) {
                    record(F_MM0, i, s0);
                    record(F_MM1, i, s1);
                }
                if constexpr (ENERGY) {
                    const double *w3r = wrow(L::o_sw, 1), *w4r = wrow(L::o_sw, 2);
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const double a0 = f4(o0, e), a1 = f4(o1, e), b0 = s0[e], b1 = s1[e];
                        E.p0 = add(E.p0, mul(mul(a0, w3r[e]), a0));
                        E.p0 = add(E.p0, mul(mul(a1, w3r[e]), a1));
                        E.p0 = add(E.p0, mul(mul(a0, w4r[e]), a1));
                        E.p1 = add(E.p1, mul(mul(b0, w3r[e]), b0));
                        E.p1 = add(E.p1, mul(mul(b1, w3r[e]), b1));
                        E.p1 = add(E.p1, mul(mul(b0, w4r[e]), b1));
                    }
                }
            }
        }
        if constexpr (ENERGY) {
            if (__syncthreads_or(bad)) {   // (a weight copy that timed out ends the item in every thread)
                bad = true;
                break;
            }
        } else {
            __syncthreads();
        }
    }
    if (nf != 0.f) atomicOr(a.flags, FLAG_NONFINITE);
    if (!bad) {   // every copy has landed and every thread is past the last barrier
        if (threadIdx.x == 0)
            for (int k = 0; k < L::NBW; k++) mbar_inval(bar + k);
        return true;
    }
    {
        // a copy did not arrive in time: record it, let every copy still in flight land (bounded)
        // before the CTA's shared memory is released, and leave this step's results incomplete
        if (threadIdx.x == 0) {
            atomicOr(a.flags, FLAG_TIMEOUT);
            // the last group issued on each barrier (the earlier ones on it completed before it
            // was issued)
            for (int G = issued - NB + 1 > 0 ? issued - NB + 1 : 0; G <= issued; G++)
                mbar_wait(bar + G % NB, (unsigned)((G / NB) & 1), TMA_WAIT_LIMIT);
            if constexpr (ENERGY) {   // and the last block of each weight set
                if (vw_last >= 0) mbar_wait(bar + NB, (unsigned)(vw_last & 1), TMA_WAIT_LIMIT);
                if (sw_last >= 0) mbar_wait(bar + NB + 1, (unsigned)(sw_last & 1), TMA_WAIT_LIMIT);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 0; k < L::NBW; k++) mbar_inval(bar + k);
        return false;
    }
}

// the CTA's energy sums into the step's records (red: 3 x FS_WARPS doubles of shared memory)
template <bool ENERGY>
__device__ __forceinline__ void cta_energy(const FusedArgs<float, float> &a, const EAcc &E, double *red, int it)
{
    if constexpr (ENERGY) {
        __syncthreads();   // every thread is past its use of the shared rings and tiles
        double e3[3] = {E.p0, E.k, E.p1};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            double v = e3[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
            if ((threadIdx.x & 31) == 0) red[q * FS_WARPS + (threadIdx.x >> 5)] = v;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double v = 0.;
            for (int w = 0; w < FS_WARPS; w++) v += red[threadIdx.x * FS_WARPS + w];
            if (it < a.max_steps && v != 0.) atomicAdd(a.energy + (long)threadIdx.x * a.max_steps + it, 0.5 * v);
        }
    }
}

// The step is two launches that run side by side, on two streams forked from and joined into the
// handle's stream (two parallel branches in a captured graph): k_elastic_side holds the boundary
// CTAs and the warp strips (latency-bound, few), k_elastic_tma the TMA strips. Neither reads
// what the other writes: both read only the step's input buffers and write disjoint parts of its
// output buffers. Every CTA of either counts itself done at its end; the last of all of them
// advances the step counter (and clears the TMA strips' item counter), after every CTA of the
// step has read it. Kept apart, each SM runs one hot loop most of the time, and the TMA strips
// fill whatever slots the side CTAs leave.
__device__ __forceinline__ void step_done(const FusedArgs<float, float> &a, int it)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const int ticket = atomicAdd(a.done, 1);
        if (ticket == a.n_all_ctas - 1) {
            *a.done = 0;
            *a.work = 0;
            *a.step = it + 1;
            __threadfence();
        }
    }
}

template <bool ENERGY>
__global__ void __launch_bounds__(FS_THREADS_MAX, fs_min_blocks<float, ENERGY>())
    k_elastic_side(FusedArgs<float, float> a)
{
    extern __shared__ __align__(16) unsigned char side_smem_raw[];
    __shared__ double red[3 * FS_WARPS];
    const int it = *a.step;
    const int cta = blockIdx.x;
    const int rcv_b = a.rcv_off[cta], rcv_e = a.rcv_off[cta + 1];
    EAcc E;
    const int n_bnd = a.n_zone * a.n_bstrip;
    if (cta < n_bnd) {
        boundary_cta<float, float, 0, ENERGY, float, false>(a, cta % a.n_bstrip, cta / a.n_bstrip, it, rcv_b, rcv_e,
                                                           reinterpret_cast<float *>(side_smem_raw), E);
    } else {
        // warp strips: segments of the interior rows (a.n_int_seg of them) x a.n_ostrip strips
        const int gw = (cta - n_bnd) * FS_WARPS + (threadIdx.x >> 5);
        if (gw < a.n_int_seg * a.n_ostrip) {
            const int seg = gw / a.n_ostrip, os = gw - seg * a.n_ostrip;
            const int y0 = os == 0 ? 0 : a.y_tma_end + (os - 1) * FS_WARP_CORE;
            unsigned char *ring = side_smem_raw + (threadIdx.x >> 5) * RingLayout<float, float, 0, ENERGY, float>::warp;
            // (the seam-aware variant for every strip, as in the strips' launch: 1 % faster at 8192^2)
            interior_warp<float, float, 0, ENERGY, true, float, false>(a, y0, seg, it, rcv_b, rcv_e, E, ring);
        }
    }
    cta_energy<ENERGY>(a, E, red, it);
    step_done(a, it);
}

template <bool ENERGY, bool Q16 = false, bool WITEMS = false>
__global__ void __launch_bounds__(FS_THREADS_MAX, ENERGY ? 3 : 4)
    k_elastic_tma(FusedArgs<float, float> a, const __grid_constant__ TmaMaps maps)
{
    extern __shared__ __align__(128) unsigned char tma_smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<unsigned long>(tma_smem_raw) + 127) & ~127ul);
    const int it = *a.step;
    const int n_side = a.n_zone * a.n_bstrip + a.n_octa;   // receiver lists: the side CTAs' come first
    int *item_s = reinterpret_cast<int *>(base + TmaLayout<ENERGY, Q16>::o_item);
    EAcc E;
    // a persistent grid: each CTA takes items until none is left, so CTAs that find their SM busy
    // with side CTAs at first simply take fewer. With WITEMS the whole step is this launch: the
    // first n_bnd items are the boundary CTAs' work, the next n_octa groups of 4 warp strips
    // (both latency-bound: taken first, so that none trails at the end; spread among the TMA
    // items instead, two loops on one SM were far slower), the rest (segment, strip) items of the
    // TMA strips; without, the side launch runs the boundary CTAs and the warp strips
    static_assert(FS_WARPS * RingLayout<float, float, 0, ENERGY, float>::warp <= TmaLayout<ENERGY, Q16>::o_bar,
                  "the warp strips' rings lie below the TMA strips' barriers");
    static_assert(sizeof(float) * 2 * TMA_TILE_ROWS * FS_BND_W <= (size_t)TmaLayout<ENERGY, Q16>::o_bar,
                  "the boundary CTAs' tile lies below the TMA strips' barriers");
    const int n_bnd = a.n_zone * a.n_bstrip;
    for (;;) {
        if (threadIdx.x == 0) *item_s = atomicAdd(a.work, 1);
        __syncthreads();
        const int t = *item_s;
        __syncthreads();
        const int B = WITEMS ? n_bnd : 0, W = WITEMS ? a.n_octa : 0;
        if (t >= B + W + a.n_tcta) break;
        if constexpr (WITEMS) {
          if (t < B) {   // a boundary CTA's zone rows (its velocities through a shared tile)
            boundary_cta<float, float, 0, ENERGY, float, false>(a, t % a.n_bstrip, t / a.n_bstrip, it, a.rcv_off[t],
                                                               a.rcv_off[t + 1], reinterpret_cast<float *>(base), E);
            __syncthreads();   // the tile is free before the shared memory is reused
            continue;
          }
          if (t < B + W) {   // warp strips: segments of the interior rows x a.n_ostrip strips
            const int w = t - B;
            const int rcv_b = a.rcv_off[n_bnd + w], rcv_e = a.rcv_off[n_bnd + w + 1];
            const int gw = w * FS_WARPS + (threadIdx.x >> 5);
            if (gw < a.n_int_seg * a.n_ostrip) {
                const int seg = gw / a.n_ostrip, os = gw - seg * a.n_ostrip;
                const int y0 = os == 0 ? 0 : a.y_tma_end + (os - 1) * FS_WARP_CORE;
                unsigned char *ring = base + (threadIdx.x >> 5) * RingLayout<float, float, 0, ENERGY, float>::warp;
                // (the seam-aware variant for every strip: a second, faster variant for the strips
                // away from the seam made the launch's code larger and the step 4 % slower)
                interior_warp<float, float, 0, ENERGY, true, float, false>(a, y0, seg, it, rcv_b, rcv_e, E, ring);
            }
            __syncthreads();   // every warp is done with its ring before the shared memory is reused
            continue;
          }
        }
        const int tt = t - B - W;
        const int rcv_b = a.rcv_off[n_side + tt], rcv_e = a.rcv_off[n_side + tt + 1];
        if (!tma_strip_cta<ENERGY, Q16>(a, maps, tt % a.n_tstrip, tt / a.n_tstrip, it, rcv_b, rcv_e, E, base)) break;
    }
    cta_energy<ENERGY>(a, E, reinterpret_cast<double *>(base + TmaLayout<ENERGY, Q16>::o_red), it);
    step_done(a, it);
}

}  // namespace tw

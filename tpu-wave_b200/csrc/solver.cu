// C ABI of the stepper (include/twave.h): the solver handle, set-up, stepping and readback.
//
// The handle plays the role of the reference's four Class_Grid objects plus
// Class_Forward_Specs (grid.hpp, forward.hpp): it owns the device fields, coefficients, energy
// weights, source table and receiver records of one simulation and one CUDA stream. Steps are
// enqueued asynchronously and replayed from a CUDA graph; every kernel of a step reads the step
// index from a device counter, so one captured graph serves every replay.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <array>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/twave.h"
#include "kernels.h"

using namespace tw;

namespace {

thread_local std::string g_cuda_error;

int cuda_fail(cudaError_t e, const char *where)
{
    g_cuda_error = std::string(where) + ": " + cudaGetErrorString(e);
    return TW_ERR_CUDA;
}

#define TW_CUDA(call)                                             \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);       \
    } while (0)

// Ricker wavelet as the reference evaluates it (forward_simulation.cpp:63-64)
double ricker(double t, double f)
{
    return (1 - 2 * M_PI * M_PI * f * f * t * t) * exp(-M_PI * M_PI * f * f * t * t);
}

// rational location -> grid index (forward.cpp:31-51); false if it is not a grid point
bool location_to_index(char type, long num, long den, int num_dx, int den_dx, long *out)
{
    long n, d;
    if (type == 'N') { n = num * den_dx; d = den * num_dx; }
    else if (type == 'M') { n = 2 * num * den_dx - den * num_dx; d = 2 * den * num_dx; }
    else return false;
    if (d == 0 || n % d != 0) return false;
    *out = n / d;
    return true;
}

// One memory pool per device for the handles' buffers. A destroyed handle returns its buffers
// to the pool, which keeps them (release threshold: everything), so that the next handle of a
// similar size - the next shot of an inversion, the next call of a caller that creates a handle
// per simulation - maps no new device memory. tw_release_cached_memory gives it back.
constexpr int MAX_DEVICES = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[MAX_DEVICES] = {};

cudaMemPool_t handle_pool(int device, cudaError_t *err)
{
    *err = cudaSuccess;
    if (device < 0 || device >= MAX_DEVICES) { *err = cudaErrorInvalidDevice; return nullptr; }
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        if ((*err = cudaMemPoolCreate(&p, &props)) != cudaSuccess) return nullptr;
        unsigned long long keep = ~0ull;   // cuuint64_t
        if ((*err = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return nullptr;
        }
        g_pool[device] = p;
    }
    return g_pool[device];
}

// let device `peer` read and write the handle buffers of device `owner` (peer stores of the
// linked slab step, peer copies of the slab exchange)
cudaError_t pool_peer_access(int owner, int peer)
{
    cudaError_t e;
    cudaMemPool_t p = handle_pool(owner, &e);
    if (e != cudaSuccess) return e;
    cudaMemAccessDesc a{};
    a.location.type = cudaMemLocationTypeDevice;
    a.location.id = peer;
    a.flags = cudaMemAccessFlagsProtReadWrite;
    return cudaMemPoolSetAccess(p, &a, 1);
}

}  // namespace

struct tw_solver {
    tw_grid_desc d{};
    int elastic = 1, periodic = 0;
    int esz = 4;                      // bytes per stored field value
    long pitch = 0;
    int rows[5] = {0, 0, 0, 0, 0};    // rows per field slot (0: slot unused)
    int cols[5] = {0, 0, 0, 0, 0};    // columns per field slot
    long ref_rows[4], ref_cols[4];    // reference sizes per grid
    cudaStream_t st = nullptr;
    void *f[5] = {}, *res[5] = {}, *coef[5] = {};
    // fused elastic path: double-buffered state, strip x segment geometry, per-CTA receivers
    bool fused = false;
    // fused periodic acoustic path (energy off): double-buffered state, n_int_seg x n_wstrip
    // warps, receivers as one flat list in d_rcv_list
    bool afused = false;
    bool pfuse = false;               // double-buffered periodic acoustic: may join a fused batch
    int bnd = 0;                      // BND_X_IF | BND_Y_SAT (stepper.cuh): two-launch kernels
    tw_solver *link[2] = {};          // during tw_slab_run: the slabs above / below
    int n_rcv_list = 0;
    void *f2[5] = {}, *res2[5] = {};
    int parity = 0;                   // which buffer holds the current state (0: f/res, 1: f2/res2)
    int n_int_seg = 0, int_rows = 0, n_zone = 1, n_wstrip = 0, n_bstrip = 1, n_int_cta = 0, tile_rows = 1;
    // the TMA-staged fused step (tma_step.cuh): strips, segments and CTAs, and one set of tensor
    // maps per buffer parity (the input fields alternate between f and f2)
    bool tma = false;
    int n_tseg = 0, n_tstrip = 0, n_tcta = 0, n_ostrip = 0, y_tma_end = 0;
    // the per-warp kernel's own layout on a TMA handle (n_int_seg / n_int_cta above describe the
    // side launch there), with its per-CTA receiver lists: steps between buffers other than the
    // handle's two (the adjoint's recomputation and revolve sweeps) run that kernel
    int w_int_seg = 0, w_int_cta = 0;
    // the boundary CTAs and the warp strips as the first work items of the TMA strips' launch, one
    // launch a step (grids below 2^25 points: there the side launch's latency-bound CTAs cost more
    // SM time than they overlap; B200, us a step one launch / two: 1024^2 31.3 / 34.6, 3072^2
    // 112.1 / 127.5, 4096^2 194.1 / 199.1, 6144^2 399.8 / 400.1, 8192^2 691.2 / 688.9, where the
    // latency-bound items at the head of the queue hold the strips' DRAM stream back), else in the
    // side launch; TW_TMA_WITEMS=1 / 0 selects either for comparisons
    bool tma_witems = false;
    int *d_rcv_off_w = nullptr, *d_rcv_list_w = nullptr;
    int rcv_list_cap_w = 0;
    TmaMaps *tmaps = nullptr;
    cudaStream_t st_side = nullptr;   // the side launch's stream, forked from st and joined back
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // 16-bit fixed-point coefficients (coef_fp16 = 2): the codes the TMA strips read, each array's
    // map (coef holds the decoded FP32 values for every other reader), two words of scratch
    bool q16 = false;
    unsigned short *coefq[5] = {};
    float qlo[5] = {}, qstep[5] = {};
    unsigned *d_mm = nullptr;
    int ir0 = FS_ZONE, zone_kind[2] = {0, 1};
    // a slab of a larger grid (slab decomposition along x): local row r is global row r + row_off
    // of a grid of Mx_glob cells; it owns global rows [own0, own1) of every grid (plus the last
    // N-type row when it reaches the bottom); the rows beyond are halo, refreshed by tw_slab_exchange
    bool slab = false;
    long row_off = 0, Mx_glob = 0, own0 = 0, own1 = 0;
    int *d_done = nullptr, *d_rcv_off = nullptr, *d_rcv_list = nullptr;
    int rcv_list_cap = 0;
    double *w[5] = {}, *mat[5] = {};
    // the padded node model of the last tw_set_material_model (rho, vp, vs), for the model gradient
    double *model = nullptr;
    long model_Mxp = 0, model_Myp = 0;
    int model_ndM = 0, model_ddM = 0;
    bool model_set = false;
    bool mat_set[5] = {};
    bool mat_dirty = true, mat_ready = false;
    double *src_inc = nullptr;
    int *d_step = nullptr, *d_flags = nullptr, *d_rcv = nullptr, *d_err = nullptr;
    double *d_traces = nullptr, *d_energy = nullptr;
    int rcv_cap = 0;
    std::vector<int> rcv_tab;         // n x 4 (slot0, slot1, row, col)
    int src_grid = -1;
    long src_ix = 0, src_iy = 0;
    int steps_done = 0;
    int sticky = TW_OK;
    cudaGraphExec_t gexec = nullptr;
    int graph_steps = 0;
    int graph_parity = 0;             // the buffer the captured graph starts from
    double dev_bytes = 0;

    ~tw_solver();
    // device buffers come from the device's handle pool, ordered on the handle's stream
    int alloc(void **p, size_t bytes)
    {
        cudaError_t e = cudaSuccess;
        cudaMemPool_t pool = handle_pool(d.device, &e);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes, pool, st);
        if (e != cudaSuccess) { *p = nullptr; cuda_fail(e, "cudaMallocFromPoolAsync"); return TW_ERR_NOMEM; }
        dev_bytes += (double)bytes;
        return TW_OK;
    }
    void release(void *p)
    {
        if (p) cudaFreeAsync(p, st);
    }
    bool has_slot(int slot) const { return rows[slot] > 0; }
    void drop_graph()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
        graph_steps = 0;
    }
};

tw_solver::~tw_solver()
{
    drop_graph();
    delete[] tmaps;
    if (!st) return;   // nothing was allocated before the stream
    for (int k = 0; k < 5; k++) {
        release(f[k]); release(res[k]); release(coef[k]); release(w[k]); release(mat[k]);
    }
    for (int k = 0; k < 5; k++) { release(f2[k]); release(res2[k]); }
    release(d_done); release(d_rcv_off); release(d_rcv_list); release(model);
    release(d_rcv_off_w); release(d_rcv_list_w);
    release(src_inc); release(d_step); release(d_flags); release(d_rcv); release(d_err);
    release(d_traces); release(d_energy);
    for (int k = 0; k < 5; k++) release(coefq[k]);
    release(d_mm);
    cudaStreamSynchronize(st);   // the buffers are back in the pool before the next handle asks
    cudaStreamDestroy(st);
    if (st_side) cudaStreamDestroy(st_side);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
}

namespace {

// map a reference (grid, field) to the device slot
int slot_of(const tw_solver *s, int grid, int field)
{
    switch (grid) {
    case TW_NN: return field == 0 && s->elastic ? F_NN : -1;
    case TW_MN: return field == 0 ? F_MN : -1;
    case TW_NM: return field == 0 ? F_NM : -1;
    case TW_MM: return field == 0 ? F_MM0 : (field == 1 && s->elastic ? F_MM1 : -1);
    }
    return -1;
}

// the buffers holding the current state (the second copy after an odd number of fused steps)
void *cur_f(const tw_solver *s, int k) { return s->parity ? s->f2[k] : s->f[k]; }
void *cur_res(const tw_solver *s, int k) { return s->parity ? s->res2[k] : s->res[k]; }

// arguments of the in-place per-point kernels, on the current buffers
// a slab's local row of global row gx of grid `grid`, or -1 when another slab owns it
long owned_row(const tw_solver *s, int grid, long gx)
{
    if (!s->slab) return gx;
    const bool Nx = grid == TW_NN || grid == TW_NM;
    const bool own = (gx >= s->own0 && gx < s->own1) || (Nx && gx == s->Mx_glob && s->own1 == s->Mx_glob);
    return own ? gx - s->row_off : -1;
}

template <class S, class C>
StepArgs<S, C> step_args(const tw_solver *s)
{
    StepArgs<S, C> a{};
    for (int k = 0; k < 5; k++) {
        a.f[k] = (S *)cur_f(s, k);
        a.res[k] = (S *)cur_res(s, k);
        a.coef[k] = (const C *)s->coef[k];
    }
    a.pitch = s->pitch;
    a.Mx = (int)s->d.Mx;
    a.My = (int)s->d.My;
    a.op = make_ops<C>((double)s->d.num_dx / (double)s->d.den_dx, s->d.dt, s->periodic && !s->elastic);
    a.src_inc = s->src_inc;
    a.src_grid = s->src_grid;
    a.src_ix = (int)s->src_ix;
    a.src_iy = (int)s->src_iy;
    a.max_steps = s->d.max_steps;
    a.step = s->d_step;
    a.flags = s->d_flags;
    a.bnd = s->bnd;
    return a;
}

template <class S, class C>
void energy_phase(const tw_solver *s, int phase, cudaStream_t st)
{
    // phase 0: E_p0 (stresses before the step), 1: E_k (velocities), 2: E_p1 (stresses after)
    EnergyArgs<S, C> e{};
    e.pitch = s->pitch;
    e.max_steps = s->d.max_steps;
    e.step = s->d_step;
    e.out = s->d_energy + (long)phase * s->d.max_steps;
    e.single_core = s->periodic;
    e.scale = s->periodic ? 1.0 : 0.5;
    auto term = [&](int a, int b, int wslot, int pslot) {
        const int t = e.nterms++;
        e.a[t] = (const S *)cur_f(s, a);
        e.b[t] = (const S *)cur_f(s, b);
        e.w[t] = s->w[wslot];
        e.p[t] = (const C *)s->coef[pslot];
        e.rows[t] = s->rows[a];
        e.cols[t] = s->cols[a];
    };
    if (phase == 1) {
        term(F_MN, F_MN, F_MN, F_MN);
        term(F_NM, F_NM, F_NM, F_NM);
    } else if (s->elastic) {
        term(F_MM0, F_MM0, F_MM0, F_MM0);
        term(F_MM1, F_MM1, F_MM0, F_MM0);
        term(F_MM0, F_MM1, F_MM1, F_MM0);
        term(F_NN, F_NN, F_NN, F_NN);
    } else {
        term(F_MM0, F_MM0, F_MM0, F_MM0);
    }
    launch_energy<S, C>(e, st);
}

template <class S, class C>
void enqueue_steps(tw_solver *s, int n, cudaStream_t st)
{
    const StepArgs<S, C> a = step_args<S, C>(s);
    GatherArgs<S> g{};
    for (int k = 0; k < 5; k++) g.f[k] = (const S *)cur_f(s, k);
    g.rcv = s->d_rcv;
    g.n_rcv = (int)(s->rcv_tab.size() / 4);
    g.pitch = s->pitch;
    g.traces = s->d_traces;
    g.max_steps = s->d.max_steps;
    g.step = s->d_step;
    g.flags = s->d_flags;
    const bool en = s->d.energy != 0;
    for (int k = 0; k < n; k++) {
        if (en && !s->periodic) energy_phase<S, C>(s, 0, st);
        launch_half<S, C>(s->elastic ? 0 : 1, s->periodic, s->d.cpst, 0, a, st);
        if (en) energy_phase<S, C>(s, 1, st);
        launch_half<S, C>(s->elastic ? 0 : 1, s->periodic, s->d.cpst, 1, a, st);
        if (en) energy_phase<S, C>(s, 2, st);
        launch_gather<S>(g, st);
    }
}

// arguments of one fused acoustic step of shot s whose state is in buffer `parity`
template <class S, class C>
AcShot<S, C> acoustic_shot(const tw_solver *s, int parity)
{
    AcShot<S, C> a{};
    void *const *fin = parity ? s->f2 : s->f, *const *fout = parity ? s->f : s->f2;
    void *const *rin = parity ? s->res2 : s->res, *const *rout = parity ? s->res : s->res2;
    for (int k = 0; k < 5; k++) {
        a.in[k] = (const S *)fin[k];
        a.out[k] = (S *)fout[k];
        a.rin[k] = (const S *)rin[k];
        a.rout[k] = (S *)rout[k];
        a.coef[k] = (const C *)s->coef[k];
    }
    a.pitch = s->pitch;
    a.Mx = (int)s->d.Mx;
    a.My = (int)s->d.My;
    a.op = make_ops<C>((double)s->d.num_dx / (double)s->d.den_dx, s->d.dt, true);
    a.n_seg = s->n_int_seg;
    a.n_wstrip = s->n_wstrip;
    a.warp_off = 0;
    a.src_inc = s->src_inc;
    a.src_grid = s->src_grid;
    a.src_ix = (int)s->src_ix;
    a.src_iy = (int)s->src_iy;
    a.step = s->d_step;
    a.flags = s->d_flags;
    a.max_steps = s->d.max_steps;
    a.rcv = s->d_rcv_list;
    a.n_rcv = s->n_rcv_list;
    a.traces = s->d_traces;
    return a;
}

// one fused elastic step from the buffers fin (rin) into fout (rout); with_energy false: the step
// adds nothing to the energy records (a recomputed step of the adjoint's checkpointing)
template <class S, class C>
void enqueue_fused_io(tw_solver *s, void *const *fin, void *const *fout, void *const *rin, void *const *rout,
                      cudaStream_t st, bool with_energy = true)
{
    const bool energy = with_energy && s->d.energy != 0;
    FusedArgs<S, C> a{};
    for (int k = 0; k < 5; k++) {
        a.in[k] = (const S *)fin[k];
        a.out[k] = (S *)fout[k];
        a.rin[k] = (const S *)rin[k];
        a.rout[k] = (S *)rout[k];
        a.coef[k] = s->coef[k];
        a.w[k] = s->w[k];
    }
    a.pitch = s->pitch;
    a.Mx = (int)s->d.Mx;
    a.My = (int)s->d.My;
    a.op = make_ops<C>((double)s->d.num_dx / (double)s->d.den_dx, s->d.dt, false);
    a.n_int_seg = s->n_int_seg;
    a.int_rows = s->int_rows;
    a.ir0 = s->ir0;
    a.n_zone = s->n_zone;
    a.zone_kind[0] = s->zone_kind[0];
    a.zone_kind[1] = s->zone_kind[1];
    a.xif = (s->bnd & BND_X_IF) ? 1 : 0;
    a.n_wstrip = s->n_wstrip;
    a.n_bstrip = s->n_bstrip;
    a.n_int_cta = s->n_int_cta;
    a.tile_rows = s->tile_rows;
    a.src_inc = s->src_inc;
    a.src_grid = s->src_grid;
    a.src_ix = (int)s->src_ix;
    a.src_iy = (int)s->src_iy;
    a.step = s->d_step;
    a.done = s->d_done;
    a.flags = s->d_flags;
    a.max_steps = s->d.max_steps;
    a.energy = s->d_energy;
    a.rcv_off = s->d_rcv_off;
    a.rcv = s->d_rcv_list;
    a.traces = s->d_traces;
    a.push_row[0] = a.push_row[1] = -(1 << 30);
    for (int side = 0; side < 2; side++) {
        const tw_solver *p = s->link[side];
        if (!p) continue;
        // the neighbour steps in lockstep: its output buffer of this step has our parity
        for (int k = 0; k < 5; k++) {
            a.peer_out[side][k] = (S *)(s->parity ? p->f[k] : p->f2[k]);
            a.peer_rout[side][k] = (S *)(s->parity ? p->res[k] : p->res2[k]);
        }
        a.push_row[side] = (int)(side == 0 ? s->own0 - s->row_off : s->own1 - s->row_off - FS_HALO);
        a.peer_shift[side] = (int)(s->row_off - p->row_off);
    }
    if constexpr (sizeof(S) == 4 && sizeof(C) == 4) {
        // the TMA-staged step reads through tensor maps of the handle's own two buffers; a step
        // between other buffers (the adjoint's segment recomputation) takes the per-warp kernel
        if (s->tma && (fin == s->f || fin == s->f2) && fout == (fin == s->f ? s->f2 : s->f)) {
            a.n_tseg = s->n_tseg;
            a.n_tstrip = s->n_tstrip;
            a.n_tcta = s->n_tcta;
            a.n_oseg = s->n_int_seg;
            a.n_ostrip = s->n_ostrip;
            a.n_octa = s->n_int_cta;
            a.y_tma_end = s->y_tma_end;
            a.work = s->d_done + 1;
            a.q16 = s->q16 ? 1 : 0;
            a.witems = s->tma_witems ? 1 : 0;
            for (int k = 0; k < 5; k++) { a.qlo[k] = s->qlo[k]; a.qstep[k] = s->qstep[k]; }
            launch_tma<S, C>(a, s->tmaps[fin == s->f ? 0 : 1], energy, st, s->st_side, s->ev_fork, s->ev_join);
            return;
        }
    }
    if (s->tma) {   // the per-warp kernel on a TMA handle: its own segmentation and receiver lists
        a.n_int_seg = s->w_int_seg;
        a.n_int_cta = s->w_int_cta;
        a.rcv_off = s->d_rcv_off_w;
        a.rcv = s->d_rcv_list_w;
    }
    launch_fused<S, C>(a, s->d.cpst, energy, s->d.coef_fp16 == 1, st);
}

// one fused elastic step from the current buffers into the other ones
template <class S, class C>
void enqueue_fused_step(tw_solver *s, cudaStream_t st)
{
    void **fin = s->parity ? s->f2 : s->f, **fout = s->parity ? s->f : s->f2;
    void **rin = s->parity ? s->res2 : s->res, **rout = s->parity ? s->res : s->res2;
    enqueue_fused_io<S, C>(s, fin, fout, rin, rout, st);
    if constexpr (sizeof(S) == sizeof(C)) {
        if (s->bnd & BND_Y_SAT) {   // free y ends: recompute the points next to them (ysat_fix.cu)
            YFixArgs<S, C> y{};
            for (int k = 0; k < 5; k++) {
                y.in[k] = (const S *)fin[k];
                y.out[k] = (S *)fout[k];
                y.rin[k] = (const S *)rin[k];
                y.rout[k] = (S *)rout[k];
                y.coef[k] = (const C *)s->coef[k];
                y.w[k] = s->w[k];
            }
            y.pitch = s->pitch;
            y.Mx = (int)s->d.Mx;
            y.My = (int)s->d.My;
            y.op = make_ops<C>((double)s->d.num_dx / (double)s->d.den_dx, s->d.dt, false);
            y.xif = (s->bnd & BND_X_IF) ? 1 : 0;
            y.src_inc = s->src_inc;
            y.src_grid = s->src_grid;
            y.src_ix = (int)s->src_ix;
            y.src_iy = (int)s->src_iy;
            y.step = s->d_step;
            y.flags = s->d_flags;
            y.max_steps = s->d.max_steps;
            y.energy = s->d.energy ? s->d_energy : nullptr;
            y.rcv = s->d_rcv;
            y.n_rcv = (int)(s->rcv_tab.size() / 4);
            y.traces = s->d_traces;
            launch_ysat_fix<S, C>(y, s->d.cpst, st);
        }
    }
    s->parity ^= 1;
}

// launch phase `ph` (0 velocity, 1 stress, 2 energy of the step, 3 gather) of one step
template <class S, class C>
void enqueue_phase(tw_solver *s, int ph, cudaStream_t st)
{
    const StepArgs<S, C> a = step_args<S, C>(s);
    if (ph == 0 || ph == 1) {
        launch_half<S, C>(s->elastic ? 0 : 1, s->periodic, s->d.cpst, ph, a, st);
    } else if (ph == 2) {
        if (!s->periodic) energy_phase<S, C>(s, 0, st);
        energy_phase<S, C>(s, 1, st);
        energy_phase<S, C>(s, 2, st);
    } else {
        GatherArgs<S> g{};
        for (int k = 0; k < 5; k++) g.f[k] = (const S *)cur_f(s, k);
        g.rcv = s->d_rcv;
        g.n_rcv = (int)(s->rcv_tab.size() / 4);
        g.pitch = s->pitch;
        g.traces = s->d_traces;
        g.max_steps = s->d.max_steps;
        g.step = s->d_step;
        g.flags = s->d_flags;
        launch_gather<S>(g, st);
    }
}

void enqueue(tw_solver *s, int n, cudaStream_t st)
{
    if (s->afused) {
        for (int k = 0; k < n; k++) {
            if (s->d.precision == TW_FP64) launch_acoustic_fused<double, double>(acoustic_shot<double, double>(s, s->parity), s->d.cpst, s->d_done, st);
            else launch_acoustic_fused<float, float>(acoustic_shot<float, float>(s, s->parity), s->d.cpst, s->d_done, st);
            s->parity ^= 1;
        }
        return;
    }
    if (s->fused) {
        for (int k = 0; k < n; k++) {
            switch (s->d.precision) {
            case TW_FP64: enqueue_fused_step<double, double>(s, st); break;
            case TW_FP32: enqueue_fused_step<float, float>(s, st); break;
            case TW_BF16: enqueue_fused_step<__nv_bfloat16, float>(s, st); break;
            default: enqueue_fused_step<__half, float>(s, st); break;
            }
        }
        return;
    }
    if (s->d.precision == TW_FP64) enqueue_steps<double, double>(s, n, st);
    else enqueue_steps<float, float>(s, n, st);
}

// stepping coefficients and energy weights from the FP64 material arrays
int finalize_material(tw_solver *s)
{
    for (int k = 0; k < 5; k++)
        if (s->has_slot(k) && !s->mat_set[k]) return TW_ERR_STATE;
    MaterialArgs m{};
    for (int k = 0; k < 5; k++) {
        m.mat[k] = s->mat[k];
        m.coef[k] = s->coef[k];
        m.w[k] = s->w[k];
        m.rows[k] = s->rows[k];
        m.cols[k] = s->cols[k];
    }
    m.Mx = (int)s->d.Mx;
    m.My = (int)s->d.My;
    m.pitch = s->pitch;
    m.dx = (double)s->d.num_dx / (double)s->d.den_dx;
    m.physics = s->elastic ? 0 : 1;
    m.periodic = s->periodic;
    m.row_off = (int)s->row_off;
    m.Mx_glob = (int)s->Mx_glob;
    m.sat_y = s->d.sat_y;
    const bool f64 = s->d.precision == TW_FP64;
    for (int i = 0; i < 4; i++) {
        const double l = SbpTables::A_N_L[i] * m.dx, r = SbpTables::A_N_R[i] * m.dx;
        m.nxN[i] = f64 ? l : (double)(float)l;
        m.nxN[4 + i] = f64 ? r : (double)(float)r;
    }
    for (int i = 0; i < 3; i++) {
        const double l = SbpTables::A_M_L[i] * m.dx, r = SbpTables::A_M_R[i] * m.dx;
        m.nxM[i] = f64 ? l : (double)(float)l;
        m.nxM[3 + i] = f64 ? r : (double)(float)r;
    }
    m.err = s->d_err;
    TW_CUDA(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->st));
    if (f64) launch_material_finalize<double, double>(m, s->st);
    else if (s->d.coef_fp16 == 1) launch_material_finalize<float, __half>(m, s->st);
    else launch_material_finalize<float, float>(m, s->st);
    TW_CUDA(cudaGetLastError());
    int herr = 0;
    TW_CUDA(cudaMemcpyAsync(&herr, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    if (herr & 2) return TW_ERR_UNSUPPORTED;   // a coefficient outside the normal FP16 range
    if (s->q16)   // the codes, each array's map, and the decoded values in place of the FP32 ones
        for (int k = 0; k < 5; k++)
            if (quantize_coefficients16((float *)s->coef[k], s->coefq[k], s->rows[k], s->cols[k], s->pitch, s->d_mm,
                                        &s->qlo[k], &s->qstep[k], s->st) != 0)
                return cuda_fail(cudaGetLastError(), "coefficient codes");
    s->mat_dirty = false;
    s->mat_ready = true;
    return TW_OK;
}

int rebuild_source_table(tw_solver *s)
{
    std::vector<double> inc(s->d.max_steps, 0.0);
    if (s->src_grid >= 0) {
        const double dt = s->d.dt, dx = (double)s->d.num_dx / (double)s->d.den_dx;
        const bool stress = s->src_grid == TW_NN || s->src_grid == TW_MM;
        for (int it = 0; it < s->d.max_steps; it++) {
            // V grids: t = it dt - delay; S grids: t = (it + 1/2) dt - delay (forward_simulation.cpp:63,105);
            // the single-core tree's P source uses (it + 1 - 1/2) dt, the same value (cpu_acoustic.cpp:309)
            const double t = stress ? (it + 1. / 2.) * dt - s->d.time_delay : it * dt - s->d.time_delay;
            double v = ricker(t, s->d.central_f) * dt / (dx * dx);
            if (s->d.source_scaling != 1.0) v = v / s->d.source_scaling;
            inc[it] = v;
        }
    }
    TW_CUDA(cudaMemcpyAsync(s->src_inc, inc.data(), sizeof(double) * inc.size(), cudaMemcpyHostToDevice, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    s->drop_graph();
    return TW_OK;
}

int upload_receivers(tw_solver *s)
{
    const int n = (int)(s->rcv_tab.size() / 4);
    if (n > s->rcv_cap) {
        s->release(s->d_rcv);
        s->release(s->d_traces);
        s->d_rcv = nullptr;
        s->d_traces = nullptr;
        int cap = s->rcv_cap ? s->rcv_cap : 16;
        while (cap < n) cap *= 2;
        if (s->alloc((void **)&s->d_rcv, sizeof(int) * 4 * cap) != TW_OK) return TW_ERR_NOMEM;
        if (s->alloc((void **)&s->d_traces, sizeof(double) * 2 * (size_t)cap * s->d.max_steps) != TW_OK) return TW_ERR_NOMEM;
        TW_CUDA(cudaMemsetAsync(s->d_traces, 0, sizeof(double) * 2 * (size_t)cap * s->d.max_steps, s->st));
        s->rcv_cap = cap;
    }
    if (n > 0)
        TW_CUDA(cudaMemcpyAsync(s->d_rcv, s->rcv_tab.data(), sizeof(int) * s->rcv_tab.size(), cudaMemcpyHostToDevice, s->st));
    if (s->fused) {
        // per-CTA receiver lists: a receiver belongs to the CTA whose segment owns its row and
        // whose strip owns its column (fused_step.cu); `warp_layout` numbers the CTAs of the
        // per-warp kernel on a TMA handle (its fallback for steps between other buffers)
        auto build = [&](bool warp_layout, int *d_off, int **d_list, int *cap_list) -> int {
            const bool tma = s->tma && !warp_layout;
            const int n_int_seg = warp_layout ? s->w_int_seg : s->n_int_seg;
            const int n_int_cta = warp_layout ? s->w_int_cta : s->n_int_cta;
            const int nctas = n_int_cta + s->n_zone * s->n_bstrip + (tma ? s->n_tcta : 0);
            std::vector<std::vector<int>> per(nctas);
            const int Mx = (int)s->d.Mx;
            for (int r = 0; r < n; r++) {
                const int *q = &s->rcv_tab[4 * r];
                if (q[0] < 0) continue;   // a receiver of another slab
                const int row = q[2], col = q[3];
                int zone = -1;            // the boundary zone holding the row, if any
                for (int z = 0; z < s->n_zone; z++) {
                    const int k = s->zone_kind[z];
                    if (k == 2 || ((k == 0 || k == 3) && row < FS_ZONE) || ((k == 1 || k == 3) && row >= Mx - FS_ZONE)) zone = z;
                }
                // the balanced segment of n segments of the interior rows holding the row (fused_step.cuh)
                auto seg_of = [&](int ns) {
                    int seg = 0;
                    while (s->ir0 + (int)((long)(seg + 1) * s->int_rows / ns) <= row) seg++;
                    return seg;
                };
                int cta;
                const int n_bnd = s->n_zone * s->n_bstrip;
                if (zone >= 0) {
                    cta = zone * s->n_bstrip + col / FS_BND_TY;
                } else if (tma && col >= TMA_Y0 && col < s->y_tma_end) {   // a TMA strip CTA
                    cta = n_bnd + n_int_cta + seg_of(s->n_tseg) * s->n_tstrip + (col - TMA_Y0) / TMA_CORE;
                } else if (tma) {                                         // a warp strip
                    const int os = col < TMA_Y0 ? 0 : 1 + (col - s->y_tma_end) / FS_WARP_CORE;
                    cta = n_bnd + (seg_of(n_int_seg) * s->n_ostrip + os) / FS_WARPS;
                } else {
                    cta = n_bnd + (seg_of(n_int_seg) * s->n_wstrip + col / FS_WARP_CORE) / FS_WARPS;
                }
                for (int f = 0; f < 2; f++)
                    if (q[f] >= 0) per[cta].insert(per[cta].end(), {q[f], row, col, 2 * r + f});
            }
            std::vector<int> off(nctas + 1, 0), list;
            for (int c = 0; c < nctas; c++) {
                off[c + 1] = off[c] + (int)per[c].size() / 4;
                list.insert(list.end(), per[c].begin(), per[c].end());
            }
            if ((int)list.size() > *cap_list) {
                s->release(*d_list);
                *d_list = nullptr;
                int cap = 64;
                while (cap < (int)list.size()) cap *= 2;
                if (s->alloc((void **)d_list, sizeof(int) * cap) != TW_OK) return TW_ERR_NOMEM;
                *cap_list = cap;
            }
            TW_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, s->st));
            if (!list.empty())
                TW_CUDA(cudaMemcpyAsync(*d_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, s->st));
            return TW_OK;
        };
        int rc = build(false, s->d_rcv_off, &s->d_rcv_list, &s->rcv_list_cap);
        if (rc == TW_OK && s->tma) rc = build(true, s->d_rcv_off_w, &s->d_rcv_list_w, &s->rcv_list_cap_w);
        if (rc != TW_OK) return rc;
    }
    if (s->pfuse) {   // (field slot, row, column, trace row) per recorded field, for the fused steps
        std::vector<int> list;
        for (int r = 0; r < n; r++) {
            const int *q = &s->rcv_tab[4 * r];
            for (int f = 0; f < 2; f++)
                if (q[f] >= 0) list.insert(list.end(), {q[f], q[2], q[3], 2 * r + f});
        }
        if ((int)list.size() > s->rcv_list_cap) {
            s->release(s->d_rcv_list);
            s->d_rcv_list = nullptr;
            int cap = 64;
            while (cap < (int)list.size()) cap *= 2;
            if (s->alloc((void **)&s->d_rcv_list, sizeof(int) * cap) != TW_OK) return TW_ERR_NOMEM;
            s->rcv_list_cap = cap;
        }
        if (!list.empty())
            TW_CUDA(cudaMemcpyAsync(s->d_rcv_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, s->st));
        s->n_rcv_list = (int)list.size() / 4;
    }
    TW_CUDA(cudaStreamSynchronize(s->st));
    s->drop_graph();
    return TW_OK;
}

// host conversion double -> storage bits
void to_storage(int prec, const double *src, void *dst, long n)
{
    if (prec == TW_FP64) memcpy(dst, src, sizeof(double) * n);
    else if (prec == TW_FP32) for (long i = 0; i < n; i++) ((float *)dst)[i] = (float)src[i];
    else if (prec == TW_BF16) for (long i = 0; i < n; i++) ((__nv_bfloat16 *)dst)[i] = __float2bfloat16_rn((float)src[i]);
    else for (long i = 0; i < n; i++) ((__half *)dst)[i] = __float2half_rn((float)src[i]);
}

double from_storage(int prec, const void *src, long i)
{
    if (prec == TW_FP64) return ((const double *)src)[i];
    if (prec == TW_FP32) return ((const float *)src)[i];
    if (prec == TW_BF16) return (double)__bfloat162float(((const __nv_bfloat16 *)src)[i]);
    return (double)__half2float(((const __half *)src)[i]);
}

// copy a device array (rows x pitch) of `esz`-byte values to the host in the reference layout;
// with `lo` (split storage) the value is the FP32 sum hi + lo, as the stepper reads it
int read_device_array(tw_solver *s, const void *dev, int prec, int esz, int slot, double *host, long ld,
                      const void *lo = nullptr)
{
    const long R = s->rows[slot], Cn = s->cols[slot];
    std::vector<char> buf((size_t)R * Cn * esz), lbuf(lo ? buf.size() : 0);
    TW_CUDA(cudaMemcpy2DAsync(buf.data(), Cn * esz, dev, s->pitch * esz, Cn * esz, R, cudaMemcpyDeviceToHost, s->st));
    if (lo) TW_CUDA(cudaMemcpy2DAsync(lbuf.data(), Cn * esz, lo, s->pitch * esz, Cn * esz, R, cudaMemcpyDeviceToHost, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    for (long ix = 0; ix < R; ix++)
        for (long iy = 0; iy < Cn; iy++) {
            const long i = ix * Cn + iy;
            host[ix * ld + iy] = lo ? (double)((float)from_storage(prec, buf.data(), i) + (float)from_storage(prec, lbuf.data(), i))
                                    : from_storage(prec, buf.data(), i);
        }
    return TW_OK;
}

// the inverse; with `lo` (split storage) hi = the value rounded to storage, lo = the rounded rest
int write_device_array(tw_solver *s, void *dev, int prec, int esz, int slot, const double *host, long ld,
                       void *lo = nullptr)
{
    const long R = s->rows[slot], Cn = s->cols[slot];
    std::vector<double> tmp((size_t)R * Cn), rest(lo ? tmp.size() : 0);
    for (long ix = 0; ix < R; ix++)
        for (long iy = 0; iy < Cn; iy++) tmp[ix * Cn + iy] = host[ix * ld + iy];
    std::vector<char> buf((size_t)R * Cn * esz), lbuf(lo ? buf.size() : 0);
    to_storage(prec, tmp.data(), buf.data(), R * Cn);
    if (lo) {
        for (long i = 0; i < R * Cn; i++) rest[i] = (double)((float)tmp[i] - (float)from_storage(prec, buf.data(), i));
        to_storage(prec, rest.data(), lbuf.data(), R * Cn);
        TW_CUDA(cudaMemcpy2DAsync(lo, s->pitch * esz, lbuf.data(), Cn * esz, Cn * esz, R, cudaMemcpyHostToDevice, s->st));
    }
    TW_CUDA(cudaMemcpy2DAsync(dev, s->pitch * esz, buf.data(), Cn * esz, Cn * esz, R, cudaMemcpyHostToDevice, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    s->drop_graph();
    return TW_OK;
}

// cuTensorMapEncodeTiled from the driver, found at run time (the library links the runtime only)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// a tensor map over `rows` rows of `pitch` elements (FP32 or FP64) with boxes of TMA_W x TMA_ROWS
int encode_rows(unsigned char *out, const void *ptr, int esize, long rows, long pitch, int box_w = TMA_W)
{
    const auto enc = tensor_map_encoder();
    if (!enc) return TW_ERR_UNSUPPORTED;
    const cuuint64_t dims[2] = {(cuuint64_t)pitch, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch * esize};
    const cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)TMA_ROWS};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = enc(reinterpret_cast<CUtensorMap *>(out),
                           esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                      : (esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16), 2,
                           const_cast<void *>(ptr), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        g_cuda_error = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return TW_ERR_CUDA;
    }
    return TW_OK;
}

// an integer tuning knob from the environment (absent or malformed: the default)
int env_int(const char *name, int dflt)
{
    const char *v = std::getenv(name);
    if (!v || !*v) return dflt;
    char *end = nullptr;
    const long x = std::strtol(v, &end, 10);
    return (end && *end == 0) ? (int)x : dflt;
}

int check(tw_solver *s)
{
    return s ? TW_OK : TW_ERR_INVALID;
}

// peer access between two devices in both directions, for contexts and for the handle pools
int link_devices(int d0, int d1)
{
    if (d0 == d1) return TW_OK;
    int ok01 = 0, ok10 = 0;
    TW_CUDA(cudaDeviceCanAccessPeer(&ok01, d0, d1));
    TW_CUDA(cudaDeviceCanAccessPeer(&ok10, d1, d0));
    if (!ok01 || !ok10) return TW_ERR_UNSUPPORTED;
    for (int q = 0; q < 2; q++) {
        TW_CUDA(cudaSetDevice(q ? d1 : d0));
        const cudaError_t e = cudaDeviceEnablePeerAccess(q ? d0 : d1, 0);
        if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
        else if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceEnablePeerAccess");
    }
    TW_CUDA(pool_peer_access(d0, d1));
    TW_CUDA(pool_peer_access(d1, d0));
    return TW_OK;
}

}  // namespace

// ======================================================================== C ABI
extern "C" {

const char *tw_strerror(int status)
{
    switch (status) {
    case TW_OK: return "ok";
    case TW_ERR_INVALID: return "invalid argument";
    case TW_ERR_CUDA: return "CUDA runtime error";
    case TW_ERR_NOMEM: return "out of memory";
    case TW_ERR_STATE: return "call out of order (material or set-up missing)";
    case TW_ERR_LOCATION: return "location is not a grid point";
    case TW_ERR_OUTSIDE: return "location outside the grid";
    case TW_ERR_WEAK_BOUNDARY: return "source on a weak boundary or on the periodic seam";
    case TW_ERR_RECORD_FULL: return "more steps than the records hold";
    case TW_ERR_NONFINITE: return "non-finite value in a field";
    case TW_ERR_UNSUPPORTED: return "unsupported configuration";
    case TW_ERR_MODEL_BOUNDS: return "material interpolation outside the model";
    case TW_ERR_TOO_LARGE: return "model larger than the no-allocation scratch (TW_NOALLOC_MAX_MODEL_POINTS)";
    case TW_ERR_IO: return "file missing, unreadable, unwritable or malformed";
    case TW_ERR_TIMEOUT: return "a wait inside a step kernel gave up (a staged copy did not arrive)";
    }
    return "unknown status";
}

const char *tw_last_cuda_error(void) { return g_cuda_error.c_str(); }

namespace {
struct SlabSpec {
    bool on = false;
    long row_off = 0, Mx_glob = 0, own0 = 0, own1 = 0;
};
int create_impl(tw_solver **out, const tw_grid_desc *desc, const SlabSpec &sl);
}  // namespace

int tw_create(tw_solver **out, const tw_grid_desc *desc)
{
    return create_impl(out, desc, SlabSpec{});
}

int tw_create_slab(tw_solver **out, const tw_grid_desc *desc, long row0, long row1)
{
    if (!out || !desc) return TW_ERR_INVALID;
    *out = nullptr;
    const tw_grid_desc &g = *desc;
    if (g.physics != TW_ELASTIC || g.bc_x != TW_BC_SAT_FREE || g.sat_y) return TW_ERR_UNSUPPORTED;
    constexpr long H = 4;   // halo rows: the step's x stencils reach four rows of the old state
    if (row0 < 0 || row1 > g.Mx || row1 - row0 < 2 * FS_ZONE || (row0 > 0 && row0 < 2 * FS_ZONE) ||
        (row1 < g.Mx && g.Mx - row1 < 2 * FS_ZONE))
        return TW_ERR_INVALID;
    SlabSpec sl;
    sl.on = true;
    sl.Mx_glob = g.Mx;
    sl.row_off = row0 > 0 ? row0 - H : 0;
    sl.own0 = row0;
    sl.own1 = row1;
    tw_grid_desc d = g;
    d.Mx = (row1 < g.Mx ? row1 + H : g.Mx) - sl.row_off;   // local cells
    return create_impl(out, &d, sl);
}

namespace {
int create_impl(tw_solver **out, const tw_grid_desc *desc, const SlabSpec &sl)
{
    if (!out || !desc) return TW_ERR_INVALID;
    *out = nullptr;
    const tw_grid_desc &d = *desc;
    if (d.physics != TW_ELASTIC && d.physics != TW_ACOUSTIC) return TW_ERR_INVALID;
    if (d.bc_x != TW_BC_SAT_FREE && d.bc_x != TW_BC_PERIODIC && d.bc_x != TW_BC_SAT_INTERFACE) return TW_ERR_INVALID;
    if (d.physics == TW_ELASTIC && d.bc_x == TW_BC_PERIODIC) return TW_ERR_UNSUPPORTED;
    if (d.sat_y != 0 && d.sat_y != 1) return TW_ERR_INVALID;
    // the interface and the y free surfaces: the two-launch kernels, FP64 / FP32 storage, SAT x
    if ((d.bc_x == TW_BC_SAT_INTERFACE || d.sat_y) &&
        (d.bc_x == TW_BC_PERIODIC || d.precision == TW_BF16 || d.precision == TW_FP16 || d.coef_fp16))
        return TW_ERR_UNSUPPORTED;
    // 16-bit fixed-point coefficients: read by the TMA-staged step (FP32 fields, plain update, the
    // reference's boundaries, a handle of its own, at least one TMA strip)
    if (d.coef_fp16 == 2 && (d.physics != TW_ELASTIC || d.precision != TW_FP32 || d.cpst != TW_CPST_00 ||
                             d.bc_x != TW_BC_SAT_FREE || d.sat_y || sl.on || d.Mx < FS_SMALL_MX ||
                             tma_strips(d.My) < 1))
        return TW_ERR_UNSUPPORTED;
    if (d.sat_y && d.My < 8) return TW_ERR_INVALID;
    if (d.precision < TW_FP64 || d.precision > TW_FP16) return TW_ERR_INVALID;
    if (d.cpst < TW_CPST_00 || d.cpst > TW_CPST_SPLIT) return TW_ERR_INVALID;
    const bool narrow = d.precision == TW_BF16 || d.precision == TW_FP16;
    // 16-bit storage (elastic only): plain, or the split pair hi + lo; the split pair needs a
    // storage type narrower than the FP32 compute type
    if (narrow && (d.physics != TW_ELASTIC || (d.cpst != TW_CPST_00 && d.cpst != TW_CPST_SPLIT))) return TW_ERR_UNSUPPORTED;
    if (!narrow && d.cpst == TW_CPST_SPLIT) return TW_ERR_UNSUPPORTED;
    if (d.coef_fp16 < 0 || d.coef_fp16 > 2) return TW_ERR_INVALID;
    // FP16 coefficients: elastic with FP32 arithmetic, plain update (or the split pair)
    if (d.coef_fp16 && (d.physics != TW_ELASTIC || d.precision == TW_FP64 ||
                        (d.cpst != TW_CPST_00 && d.cpst != TW_CPST_SPLIT)))
        return TW_ERR_UNSUPPORTED;
    if (d.bc_x == TW_BC_PERIODIC && d.cpst != TW_CPST_00 && d.cpst != TW_CPST_3R && d.cpst != TW_CPST_6R)
        return TW_ERR_UNSUPPORTED;   // the single-core tree offers '0', '3', '6' (namespaces.hpp:665-667)
    if (d.Mx < 8 || d.My < 4 || d.Mx > (1L << 30) / 2 || d.My > (1L << 30) / 2) return TW_ERR_INVALID;
    if (d.num_dx <= 0 || d.den_dx <= 0 || !(d.dt > 0) || d.max_steps < 1) return TW_ERR_INVALID;
    if (!(d.source_scaling != 0.0)) return TW_ERR_INVALID;

    tw_solver *s = new (std::nothrow) tw_solver();
    if (!s) return TW_ERR_NOMEM;
    s->d = d;
    s->slab = sl.on;
    s->row_off = sl.row_off;
    s->Mx_glob = sl.on ? sl.Mx_glob : d.Mx;
    s->own0 = sl.on ? sl.own0 : 0;
    s->own1 = sl.on ? sl.own1 : d.Mx;
    s->elastic = d.physics == TW_ELASTIC;
    s->periodic = d.bc_x == TW_BC_PERIODIC;
    s->bnd = (d.bc_x == TW_BC_SAT_INTERFACE ? BND_X_IF : 0) | (d.sat_y ? BND_Y_SAT : 0);
    s->esz = d.precision == TW_FP64 ? 8 : (d.precision == TW_FP32 ? 4 : 2);
    const int Mx_ = (int)d.Mx, My_ = (int)d.My;
    const int rws[5] = {Mx_ + 1, Mx_, Mx_ + 1, Mx_, Mx_}, cls[5] = {My_ + 1, My_ + 1, My_, My_, My_};
    for (int k = 0; k < 5; k++) {
        const bool used = s->elastic || (k != F_NN && k != F_MM1);
        s->rows[k] = used ? rws[k] : 0;
        s->cols[k] = used ? cls[k] : 0;
    }
    const long Mx = d.Mx, My = d.My;
    const long rr[4] = {Mx + 1, Mx, Mx + 1, Mx}, rc[4] = {My + 1, My + 1, My, My};
    for (int g = 0; g < 4; g++) { s->ref_rows[g] = rr[g]; s->ref_cols[g] = rc[g]; }
    // rows padded to a multiple of 128 bytes so that every row starts aligned
    const long align = 128 / s->esz;
    s->pitch = (My + 1 + align - 1) / align * align;

    int rc_ = TW_OK;
    auto fail = [&](int code) { delete s; return code; };
    cudaError_t e = cudaSetDevice(d.device);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaSetDevice"));
    e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamCreate"));
    const size_t csz = d.precision == TW_FP64 ? 8 : (d.coef_fp16 == 1 ? 2 : 4);   // (16-bit codes: beside)
    const bool cp = d.cpst != TW_CPST_00;
    for (int k = 0; k < 5; k++) {
        if (!s->has_slot(k)) continue;
        const size_t n = (size_t)s->rows[k] * s->pitch;
        if ((rc_ = s->alloc(&s->f[k], n * s->esz)) != TW_OK) return fail(rc_);
        if (cp && (rc_ = s->alloc(&s->res[k], n * s->esz)) != TW_OK) return fail(rc_);
        if ((rc_ = s->alloc(&s->coef[k], n * csz)) != TW_OK) return fail(rc_);
        if ((rc_ = s->alloc((void **)&s->w[k], n * sizeof(double))) != TW_OK) return fail(rc_);
        if ((rc_ = s->alloc((void **)&s->mat[k], (size_t)s->rows[k] * s->cols[k] * sizeof(double))) != TW_OK) return fail(rc_);
        cudaMemsetAsync(s->f[k], 0, n * s->esz, s->st);
        if (cp) cudaMemsetAsync(s->res[k], 0, n * s->esz, s->st);
        cudaMemsetAsync(s->coef[k], 0, n * csz, s->st);
        cudaMemsetAsync(s->w[k], 0, n * sizeof(double), s->st);
    }
    if (s->elastic && (!(s->bnd & BND_Y_SAT) || My >= 16)) {
        // fused elastic path: a second copy of the state and the strip x segment geometry (free
        // y ends: the fused step plus the recomputation of the columns next to them, which stay
        // apart from 16 columns on)
        s->fused = true;
        switch (d.precision) {
        case TW_FP64: e = prepare_fused<double, double>(); break;
        case TW_FP32: e = prepare_fused<float, float>(); break;
        case TW_BF16: e = prepare_fused<__nv_bfloat16, float>(); break;
        default: e = prepare_fused<__half, float>(); break;
        }
        if (e != cudaSuccess) return fail(cuda_fail(e, "cudaFuncSetAttribute"));
        for (int k = 0; k < 5; k++) {
            const size_t n = (size_t)s->rows[k] * s->pitch;
            if ((rc_ = s->alloc(&s->f2[k], n * s->esz)) != TW_OK) return fail(rc_);
            cudaMemsetAsync(s->f2[k], 0, n * s->esz, s->st);
            if (cp) {
                if ((rc_ = s->alloc(&s->res2[k], n * s->esz)) != TW_OK) return fail(rc_);
                cudaMemsetAsync(s->res2[k], 0, n * s->esz, s->st);
            }
        }
        s->n_bstrip = (int)((My + 1 + FS_BND_TY - 1) / FS_BND_TY);
        s->n_wstrip = (int)((My + 1 + FS_WARP_CORE - 1) / FS_WARP_CORE);
        if (!s->slab && Mx < FS_SMALL_MX) {
            s->n_int_seg = 0;
            s->n_zone = 1;
            s->zone_kind[0] = 2;
            s->tile_rows = (int)Mx + 1;
        } else {
            // balanced interior segments: TW_FS_CTAS_PER_SM CTAs of work for each of the 148 SMs,
            // the boundary CTAs included, segments of 8 rows or more; the segment x strip warps are
            // packed FS_WARPS to a CTA. A slab has a free-surface zone only at a global boundary;
            // at an open edge its interior reaches the four halo rows.
            const bool top = s->row_off == 0, bot = s->row_off + Mx == s->Mx_glob;
            s->n_zone = 0;
            if (s->bnd & BND_X_IF) {   // the interface couples the ends: both zones in one CTA
                s->zone_kind[s->n_zone++] = 3;
                s->tile_rows = 2 * (FS_ZONE + 2) + 1;
            } else {
                if (top) s->zone_kind[s->n_zone++] = 0;
                if (bot) s->zone_kind[s->n_zone++] = 1;
                s->tile_rows = 12;
            }
            s->ir0 = top ? FS_ZONE : 4;
            s->int_rows = (int)Mx - (bot ? FS_ZONE : 4) - s->ir0;
            if (s->int_rows < 8) return fail(TW_ERR_INVALID);
            const int target = std::max(1, (148 * TW_FS_CTAS_PER_SM - s->n_zone * s->n_bstrip) * FS_WARPS / s->n_wstrip);
            s->n_int_seg = std::max(1, std::min(target, s->int_rows / 8));
            s->n_int_cta = (s->n_int_seg * s->n_wstrip + FS_WARPS - 1) / FS_WARPS;
        }
        // the TMA-staged step (tma_step.cuh): FP32 fields and coefficients, plain update, the
        // reference's x ends, a handle of its own (not a linked slab), at least one TMA strip.
        // With the energy every step it stages 40 bytes of FP64 weights per point and fits 3 CTAs
        // per SM: faster than the per-warp kernel on grids below 2^25 points (98.4 against 107.5
        // us at 2048^2, 322.7 against 353.3 at 4096^2), slower above (1181 against 1161 at
        // 8192^2), so energy-on handles take it below that size. TW_TMA=1 / 0 in the environment
        // selects it / the per-warp kernel for every handle (for comparisons); its work items and
        // side segments have TW_TMA_SEG_ROWS / TW_TMA_SIDE_ROWS rows (below).
        const int nts = tma_strips(My);
        const bool want_q16 = d.coef_fp16 == 2;   // (the codes exist only where the TMA step reads them)
        if (d.precision == TW_FP32 && d.cpst == TW_CPST_00 && d.coef_fp16 != 1 && !s->slab && !(s->bnd & BND_X_IF) &&
            s->n_int_seg > 0 && nts > 0 && s->tile_rows == TMA_TILE_ROWS &&   // (the strips' launch holds this tile)
            (want_q16 || env_int("TW_TMA", (!d.energy || (long)Mx * My < (1L << 25)) ? 1 : 0) != 0)) {
            int n_sm = 148;
            cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, d.device);
            s->tma = true;
            s->q16 = want_q16;
            s->w_int_seg = s->n_int_seg;
            s->w_int_cta = s->n_int_cta;
            s->n_tstrip = nts;
            s->y_tma_end = TMA_Y0 + TMA_CORE * nts;
            // warp strips: the first at column 0, the others from y_tma_end to the seam column My
            s->n_ostrip = 1 + (int)((My + 1 - s->y_tma_end + FS_WARP_CORE - 1) / FS_WARP_CORE);
            // the boundary and warp-strip work in the strips' launch (one launch a step) or beside it
            s->tma_witems = env_int("TW_TMA_WITEMS", (long)Mx * My < (1L << 25) ? 1 : 0) != 0;
            // work items of about TW_TMA_SEG_ROWS rows for the persistent TMA CTAs. Measured, us a
            // step at 16 / 20 / 24 / 32 / 40 rows: 2048^2 61.65 / 61.3 / 63.3 / 63.4 / -, 4096^2
            // 195.6 / 188.5 / 184.8 / 186.9 / -, 8192^2 (side launch) - / - / 664.0 / 679.7 / 690.1,
            // 8192^2 with 16-bit coefficient codes - / - / 671.4 / 646.3 / 634.0; with the energy
            // on, 2048^2 99.9 / 97.7 / 97.7 / 95.8 / 102.3
            const bool small = (long)Mx * My <= (1L << 22);
            const int seg_def = s->tma_witems ? (small ? (d.energy ? 32 : 20) : 24) : (s->q16 ? 40 : 24);
            const int seg_rows = std::max(8, env_int("TW_TMA_SEG_ROWS", seg_def));
            const int max_seg = std::max(1, s->int_rows / 8);
            s->n_tseg = std::max(1, std::min(max_seg, (s->int_rows + seg_rows / 2) / seg_rows));
            (void)n_sm;
            // the warp strips run beside the TMA strips, latency-bound at about two microseconds a
            // row: short segments (TW_TMA_SIDE_ROWS rows, default 8) keep them shorter than a TMA CTA
            const int side_rows = std::max(8, env_int("TW_TMA_SIDE_ROWS", 8));
            s->n_int_seg = std::max(1, std::min(max_seg, s->int_rows / side_rows));
            s->n_int_cta = (s->n_int_seg * s->n_ostrip + FS_WARPS - 1) / FS_WARPS;
            s->n_tcta = s->n_tseg * s->n_tstrip;
            e = prepare_tma<float, float>();
            if (e != cudaSuccess) return fail(cuda_fail(e, "cudaFuncSetAttribute"));
            if ((e = cudaStreamCreateWithFlags(&s->st_side, cudaStreamNonBlocking)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming)) != cudaSuccess)
                return fail(cuda_fail(e, "side stream"));
            s->tmaps = new (std::nothrow) TmaMaps[2];
            if (!s->tmaps) return fail(TW_ERR_NOMEM);
            if (s->q16) {
                for (int k = 0; k < 5; k++) {
                    const size_t n = (size_t)s->rows[k] * s->pitch;
                    if ((rc_ = s->alloc((void **)&s->coefq[k], n * 2)) != TW_OK) return fail(rc_);
                    cudaMemsetAsync(s->coefq[k], 0, n * 2, s->st);
                }
                if ((rc_ = s->alloc((void **)&s->d_mm, 2 * sizeof(unsigned))) != TW_OK) return fail(rc_);
            }
            // maps by field slot: the fields of buffer `par`, the coefficients, the energy weights
            const int fmap[5] = {TM_NN, TM_MN, TM_NM, TM_MM0, TM_MM1};
            const int cmap[5] = {TM_MU, TM_PMN, TM_PNM, TM_LAM, TM_M2};
            const int wmap[5] = {TM_WNN, TM_WMN, TM_WNM, TM_WM3, TM_WM4};
            for (int par = 0; par < 2; par++)
                for (int k = 0; k < 5; k++) {
                    TmaMaps &m = s->tmaps[par];
                    if ((rc_ = encode_rows(m.m[fmap[k]], par ? s->f2[k] : s->f[k], 4, s->rows[k], s->pitch)) != TW_OK ||
                        (rc_ = s->q16 ? encode_rows(m.m[cmap[k]], s->coefq[k], 2, s->rows[k], s->pitch, TMA_QW)
                                      : encode_rows(m.m[cmap[k]], s->coef[k], 4, s->rows[k], s->pitch)) != TW_OK ||
                        (rc_ = encode_rows(m.m[wmap[k]], s->w[k], 8, s->rows[k], s->pitch)) != TW_OK)
                        return fail(rc_);
                }
        }
        const int nctas = s->n_int_cta + s->n_zone * s->n_bstrip + s->n_tcta;
        // d_done[0]: CTAs finished in this step; d_done[1]: the TMA strips' next work item
        if ((rc_ = s->alloc((void **)&s->d_done, 2 * sizeof(int))) != TW_OK) return fail(rc_);
        cudaMemsetAsync(s->d_done, 0, 2 * sizeof(int), s->st);
        if ((rc_ = s->alloc((void **)&s->d_rcv_off, sizeof(int) * (nctas + 1))) != TW_OK) return fail(rc_);
        cudaMemsetAsync(s->d_rcv_off, 0, sizeof(int) * (nctas + 1), s->st);
        if (s->tma) {
            const int nw = s->w_int_cta + s->n_zone * s->n_bstrip;
            if ((rc_ = s->alloc((void **)&s->d_rcv_off_w, sizeof(int) * (nw + 1))) != TW_OK) return fail(rc_);
            cudaMemsetAsync(s->d_rcv_off_w, 0, sizeof(int) * (nw + 1), s->st);
        }
    }
    if (!s->elastic && s->periodic && !d.energy) {
        // periodic acoustic with energy off: a second copy of the state, for the fused step of a
        // batch and, on grids of 2^20 points or more, of the handle alone (below that the
        // two-launch kernels are faster: a warp's short row segment is latency-bound); segments
        // of 8 rows or more, TW_AC_CTAS_PER_SM CTAs of work per SM of a 148-SM B200
        s->pfuse = true;
        s->afused = Mx * My >= (1L << 20);
        for (int k = 0; k < 5; k++) {
            if (!s->has_slot(k)) continue;
            const size_t n = (size_t)s->rows[k] * s->pitch;
            if ((rc_ = s->alloc(&s->f2[k], n * s->esz)) != TW_OK) return fail(rc_);
            cudaMemsetAsync(s->f2[k], 0, n * s->esz, s->st);
            if (cp) {
                if ((rc_ = s->alloc(&s->res2[k], n * s->esz)) != TW_OK) return fail(rc_);
                cudaMemsetAsync(s->res2[k], 0, n * s->esz, s->st);
            }
        }
        s->n_wstrip = (int)((My + 1 + FS_WARP_CORE - 1) / FS_WARP_CORE);
        const int target = std::max(1, 148 * TW_AC_CTAS_PER_SM * FS_WARPS / s->n_wstrip);
        s->n_int_seg = std::max(1, std::min(target, (int)Mx / 8));
        if ((rc_ = s->alloc((void **)&s->d_done, sizeof(int))) != TW_OK) return fail(rc_);
        cudaMemsetAsync(s->d_done, 0, sizeof(int), s->st);
    }
    if ((rc_ = s->alloc((void **)&s->src_inc, sizeof(double) * d.max_steps)) != TW_OK) return fail(rc_);
    if ((rc_ = s->alloc((void **)&s->d_energy, sizeof(double) * 3 * d.max_steps)) != TW_OK) return fail(rc_);
    if ((rc_ = s->alloc((void **)&s->d_step, sizeof(int))) != TW_OK) return fail(rc_);
    if ((rc_ = s->alloc((void **)&s->d_flags, sizeof(int))) != TW_OK) return fail(rc_);
    if ((rc_ = s->alloc((void **)&s->d_err, sizeof(int))) != TW_OK) return fail(rc_);
    cudaMemsetAsync(s->src_inc, 0, sizeof(double) * d.max_steps, s->st);
    cudaMemsetAsync(s->d_energy, 0, sizeof(double) * 3 * d.max_steps, s->st);
    cudaMemsetAsync(s->d_step, 0, sizeof(int), s->st);
    cudaMemsetAsync(s->d_flags, 0, sizeof(int), s->st);
    e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) return fail(cuda_fail(e, "tw_create"));
    if ((rc_ = upload_receivers(s)) != TW_OK) return fail(rc_);
    *out = s;
    return TW_OK;
}
}  // namespace

void tw_destroy(tw_solver *s)
{
    if (!s) return;
    cudaSetDevice(s->d.device);
    if (s->st) cudaStreamSynchronize(s->st);
    delete s;
}

int tw_release_cached_memory(int device)
{
    if (device < 0 || device >= MAX_DEVICES) return TW_ERR_INVALID;
    cudaMemPool_t p;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        p = g_pool[device];
    }
    if (!p) return TW_OK;
    TW_CUDA(cudaSetDevice(device));
    TW_CUDA(cudaDeviceSynchronize());   // frees still queued on a stream complete first
    TW_CUDA(cudaMemPoolTrimTo(p, 0));
    return TW_OK;
}

int tw_set_material_model(tw_solver *s, const double *rho, const double *vp, const double *vs, long Mx_prmt,
                          long My_prmt, int num_dxM, int den_dxM)
{
    if (check(s) || !rho || !vp || (s->elastic && !vs)) return TW_ERR_INVALID;
    if (Mx_prmt < 1 || My_prmt < 1 || num_dxM <= 0 || den_dxM <= 0) return TW_ERR_INVALID;
    // the model must span the simulation region (input_processing.cpp:203-211)
    for (int dir = 0; dir < 2; dir++) {
        const long pm = dir == 0 ? Mx_prmt : My_prmt, sm = dir == 0 ? s->Mx_glob : s->d.My;
        if (pm * num_dxM * (long)s->d.den_dx != sm * (long)s->d.num_dx * den_dxM) return TW_ERR_INVALID;
    }
    TW_CUDA(cudaSetDevice(s->d.device));
    const long Nxp = Mx_prmt + 1, Nyp = My_prmt + 1, P = (Nxp + 1) * (Nyp + 1);
    // rho, vp, vs land in the handle's model copy (kept for the model gradient of
    // tw_adjoint_gradient); lambda, 2mu, mu on the padded model in a temporary from the pool
    if (s->model && (s->model_Mxp != Mx_prmt || s->model_Myp != My_prmt)) {
        s->release(s->model);
        s->model = nullptr;
    }
    s->model_set = false;
    int rc = TW_OK;
    if (!s->model && (rc = s->alloc((void **)&s->model, sizeof(double) * 3 * P)) != TW_OK) {
        s->model = nullptr;
        return rc;
    }
    s->model_Mxp = Mx_prmt;
    s->model_Myp = My_prmt;
    double *der = nullptr;
    if ((rc = s->alloc((void **)&der, sizeof(double) * 3 * P)) != TW_OK) return rc;
    double *drho = s->model, *dvp = s->model + P, *dvs = s->model + 2 * P;
    double *lam = der, *m2 = der + P, *mu = der + 2 * P;
    auto done = [&](int code) { s->release(der); cudaStreamSynchronize(s->st); return code; };
    cudaError_t e;
    if ((e = cudaMemcpyAsync(drho, rho, sizeof(double) * P, cudaMemcpyHostToDevice, s->st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dvp, vp, sizeof(double) * P, cudaMemcpyHostToDevice, s->st)) != cudaSuccess)
        return done(cuda_fail(e, "model upload"));
    if (s->elastic) e = cudaMemcpyAsync(dvs, vs, sizeof(double) * P, cudaMemcpyHostToDevice, s->st);
    else e = cudaMemsetAsync(dvs, 0, sizeof(double) * P, s->st);   // acoustic: vs = 0, lambda = rho vp^2
    if (e != cudaSuccess) return done(cuda_fail(e, "model upload"));
    cudaMemsetAsync(s->d_err, 0, sizeof(int), s->st);
    launch_model_derive(drho, dvp, dvs, P, lam, m2, mu, s->st);
    struct { int slot, txN, tyN; const double *src; } jobs[5] = {
        {F_NN, 1, 1, mu}, {F_MN, 0, 1, drho}, {F_NM, 1, 0, drho}, {F_MM0, 0, 0, lam}, {F_MM1, 0, 0, m2}};
    for (auto &j : jobs) {
        if (!s->has_slot(j.slot)) continue;
        launch_interp(s->rows[j.slot], s->cols[j.slot], j.txN, j.tyN, s->d.num_dx, s->d.den_dx, num_dxM, den_dxM, Nxp, Nyp, j.src,
                      s->mat[j.slot], s->d_err, s->st, (int)s->row_off);
        s->mat_set[j.slot] = true;
    }
    int herr = 0;
    if ((e = cudaMemcpyAsync(&herr, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->st)) != cudaSuccess)
        return done(cuda_fail(e, "model"));
    if ((e = cudaStreamSynchronize(s->st)) != cudaSuccess) return done(cuda_fail(e, "model"));
    if (herr) return done(TW_ERR_MODEL_BOUNDS);
    rc = finalize_material(s);
    if (rc == TW_OK) {   // the node model now describes the material (tw_adjoint_gradient)
        s->model_ndM = num_dxM;
        s->model_ddM = den_dxM;
        s->model_set = true;
    }
    return done(rc);
}

int tw_set_material_grid(tw_solver *s, int grid, int idx, const double *coef, long ld)
{
    if (check(s) || !coef) return TW_ERR_INVALID;
    const int slot = slot_of(s, grid, idx);
    if (slot < 0) return TW_ERR_INVALID;
    if (ld < s->ref_cols[grid]) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    const long R = s->rows[slot], Cn = s->cols[slot];
    std::vector<double> tmp((size_t)R * Cn);
    for (long ix = 0; ix < R; ix++)   // a slab: its rows of the global grid's array
        for (long iy = 0; iy < Cn; iy++) tmp[ix * Cn + iy] = coef[(ix + s->row_off) * ld + iy];
    TW_CUDA(cudaMemcpyAsync(s->mat[slot], tmp.data(), sizeof(double) * tmp.size(), cudaMemcpyHostToDevice, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    s->mat_set[slot] = true;
    s->mat_dirty = true;
    s->model_set = false;   // the node model no longer describes the material
    bool all = true;
    for (int k = 0; k < 5; k++) all = all && (!s->has_slot(k) || s->mat_set[k]);
    if (all) {
        int rc = finalize_material(s);
        if (rc != TW_OK) return rc;
        TW_CUDA(cudaStreamSynchronize(s->st));
    }
    return TW_OK;
}

int tw_set_source(tw_solver *s, int grid, long ix, long iy)
{
    if (check(s) || grid < 0 || grid > 3) return TW_ERR_INVALID;
    if (!s->elastic && grid == TW_NN) return TW_ERR_INVALID;
    const long rows_g = s->ref_rows[grid] + (s->Mx_glob - s->d.Mx);   // global rows of the grid
    if (ix < 0 || iy < 0 || ix >= rows_g || iy >= s->ref_cols[grid]) return TW_ERR_OUTSIDE;
    const bool Nx = grid == TW_NN || grid == TW_NM;
    // the reference stops on a source on the free-surface node rows (forward.cpp:95-96); on the
    // periodic seam it only warns (:97-98) and so does nothing here
    if (!s->periodic && Nx && (ix == 0 || ix == s->Mx_glob)) return TW_ERR_WEAK_BOUNDARY;
    // free y ends: the same rule on the end columns of an N-type-y grid
    const bool Ny = grid == TW_NN || grid == TW_MN;
    if (s->d.sat_y && Ny && (iy == 0 || iy == s->d.My)) return TW_ERR_WEAK_BOUNDARY;
    const long lx = owned_row(s, grid, ix);   // a slab injects only a source in its own rows
    s->src_grid = lx >= 0 ? grid : -1;
    s->src_ix = lx;
    s->src_iy = iy;
    TW_CUDA(cudaSetDevice(s->d.device));
    return rebuild_source_table(s);
}

int tw_set_source_location(tw_solver *s, char tx, char ty, long nx, long dx_, long ny, long dy_)
{
    if (check(s)) return TW_ERR_INVALID;
    long ix, iy;
    if ((tx != 'N' && tx != 'M') || (ty != 'N' && ty != 'M')) return TW_ERR_INVALID;
    if (!location_to_index(tx, nx, dx_, s->d.num_dx, s->d.den_dx, &ix)) return TW_ERR_LOCATION;
    if (!location_to_index(ty, ny, dy_, s->d.num_dx, s->d.den_dx, &iy)) return TW_ERR_LOCATION;
    const int grid = tx == 'N' ? (ty == 'N' ? TW_NN : TW_NM) : (ty == 'N' ? TW_MN : TW_MM);
    return tw_set_source(s, grid, ix, iy);
}

int tw_clear_source(tw_solver *s)
{
    if (check(s)) return TW_ERR_INVALID;
    s->src_grid = -1;
    TW_CUDA(cudaSetDevice(s->d.device));
    return rebuild_source_table(s);
}

int tw_add_receivers(tw_solver *s, int grid, const long *ix, const long *iy, int n)
{
    if (check(s) || grid < 0 || grid > 3 || n < 0 || (n > 0 && (!ix || !iy))) return TW_ERR_INVALID;
    if (!s->elastic && grid == TW_NN) return TW_ERR_INVALID;
    const int s0 = slot_of(s, grid, 0), s1 = slot_of(s, grid, 1);
    std::vector<int> add;
    for (int k = 0; k < n; k++) {
        // the reference accepts indices up to and including the grid size (forward.cpp:154-155);
        // only points of the grid are accepted here
        const long rows_g = s->ref_rows[grid] + (s->Mx_glob - s->d.Mx);
        if (ix[k] < 0 || iy[k] < 0 || ix[k] >= rows_g || iy[k] >= s->ref_cols[grid]) return TW_ERR_OUTSIDE;
        // a slab records only the receivers in its own rows; the others keep zero traces, so the
        // traces of all slabs add up to the whole grid's
        const long lx = owned_row(s, grid, ix[k]);
        if (lx >= 0) add.insert(add.end(), {s0, s1, (int)lx, (int)iy[k]});
        else add.insert(add.end(), {-1, -1, (int)ix[k], (int)iy[k]});
    }
    s->rcv_tab.insert(s->rcv_tab.end(), add.begin(), add.end());
    TW_CUDA(cudaSetDevice(s->d.device));
    return upload_receivers(s);
}

int tw_add_receiver_location(tw_solver *s, char tx, char ty, long nx, long dx_, long ny, long dy_)
{
    if (check(s)) return TW_ERR_INVALID;
    long ix, iy;
    if ((tx != 'N' && tx != 'M') || (ty != 'N' && ty != 'M')) return TW_ERR_INVALID;
    if (!location_to_index(tx, nx, dx_, s->d.num_dx, s->d.den_dx, &ix)) return TW_ERR_LOCATION;
    if (!location_to_index(ty, ny, dy_, s->d.num_dx, s->d.den_dx, &iy)) return TW_ERR_LOCATION;
    const int grid = tx == 'N' ? (ty == 'N' ? TW_NN : TW_NM) : (ty == 'N' ? TW_MN : TW_MM);
    return tw_add_receivers(s, grid, &ix, &iy, 1);
}

int tw_reset(tw_solver *s)
{
    if (check(s)) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    for (int k = 0; k < 5; k++) {
        if (!s->has_slot(k)) continue;
        const size_t n = (size_t)s->rows[k] * s->pitch * s->esz;
        TW_CUDA(cudaMemsetAsync(s->f[k], 0, n, s->st));
        if (s->res[k]) TW_CUDA(cudaMemsetAsync(s->res[k], 0, n, s->st));
        if (s->f2[k]) TW_CUDA(cudaMemsetAsync(s->f2[k], 0, n, s->st));
        if (s->res2[k]) TW_CUDA(cudaMemsetAsync(s->res2[k], 0, n, s->st));
    }
    if (s->d_done) TW_CUDA(cudaMemsetAsync(s->d_done, 0, (s->fused ? 2 : 1) * sizeof(int), s->st));
    s->parity = 0;
    TW_CUDA(cudaMemsetAsync(s->d_energy, 0, sizeof(double) * 3 * s->d.max_steps, s->st));
    if (s->d_traces) TW_CUDA(cudaMemsetAsync(s->d_traces, 0, sizeof(double) * 2 * (size_t)s->rcv_cap * s->d.max_steps, s->st));
    TW_CUDA(cudaMemsetAsync(s->d_step, 0, sizeof(int), s->st));
    TW_CUDA(cudaMemsetAsync(s->d_flags, 0, sizeof(int), s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    s->steps_done = 0;
    s->sticky = TW_OK;
    return TW_OK;
}

int tw_step(tw_solver *s, int n)
{
    if (check(s) || n < 0) return TW_ERR_INVALID;
    if (!s->mat_ready) return TW_ERR_STATE;
    if (s->steps_done + (long)n > s->d.max_steps) return TW_ERR_RECORD_FULL;
    if (n == 0) return TW_OK;
    TW_CUDA(cudaSetDevice(s->d.device));
    // a graph of G steps captured once and replayed; leftover steps are launched directly. The
    // graph is captured on the first call of any length when the records hold G steps, so that
    // a short first call (a warm-up) leaves the next long call only replays and direct launches.
    const int G = 16;
    // the one-launch steps alternate buffers, and their graph starts from the first one; the
    // two-launch kernels update the current buffer in place, and their graph is bound to it
    // (a batch step may have moved the state of a double-buffered shot to the other buffer)
    const int gpar = (s->fused || s->afused) ? 0 : s->parity;
    if ((!s->gexec || s->graph_steps != G || s->graph_parity != gpar) && s->d.max_steps >= G) {
        s->drop_graph();
        cudaGraph_t graph;
        TW_CUDA(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
        const int parity0 = s->parity;
        s->parity = gpar;
        enqueue(s, G, s->st);
        s->parity = parity0;   // capture only records; replays advance the parity below
        TW_CUDA(cudaStreamEndCapture(s->st, &graph));
        cudaError_t e = cudaGraphInstantiate(&s->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        s->graph_steps = G;
        s->graph_parity = gpar;
    }
    int left = n;
    if ((s->fused || s->afused) && s->parity && left > 0 && n >= G) {
        enqueue(s, 1, s->st);   // captured graphs start from the first buffer
        left--;
    }
    if (left >= G && s->gexec) {
        while (left >= G) {
            TW_CUDA(cudaGraphLaunch(s->gexec, s->st));
            left -= G;   // G is even: the parity is unchanged
        }
    }
    if (left > 0) enqueue(s, left, s->st);
    TW_CUDA(cudaGetLastError());
    s->steps_done += n;
    return TW_OK;
}

int tw_sync(tw_solver *s)
{
    if (check(s)) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    int flags = 0;
    TW_CUDA(cudaMemcpyAsync(&flags, s->d_flags, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    if (flags & FLAG_TIMEOUT) s->sticky = TW_ERR_TIMEOUT;
    else if (flags & FLAG_NONFINITE) s->sticky = TW_ERR_NONFINITE;
    else if (flags & FLAG_RECORD_FULL) s->sticky = TW_ERR_RECORD_FULL;
    return s->sticky;
}

int tw_read_field(tw_solver *s, int grid, int field, double *host, long ld)
{
    if (check(s) || !host || grid < 0 || grid > 3) return TW_ERR_INVALID;
    const int slot = slot_of(s, grid, field);
    if (slot < 0 || ld < s->ref_cols[grid]) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    return read_device_array(s, cur_f(s, slot), s->d.precision, s->esz, slot, host, ld,
                             s->d.cpst == TW_CPST_SPLIT ? cur_res(s, slot) : nullptr);
}

int tw_read_coefficients(tw_solver *s, int grid, int idx, double *host, long ld)
{
    if (check(s) || !host || grid < 0 || grid > 3) return TW_ERR_INVALID;
    const int slot = slot_of(s, grid, idx);
    if (slot < 0 || ld < s->ref_cols[grid]) return TW_ERR_INVALID;
    if (!s->mat_ready) return TW_ERR_STATE;
    TW_CUDA(cudaSetDevice(s->d.device));
    const int prec = s->d.precision == TW_FP64 ? TW_FP64 : (s->d.coef_fp16 == 1 ? TW_FP16 : TW_FP32);
    const int esz = prec == TW_FP64 ? 8 : (prec == TW_FP16 ? 2 : 4);
    return read_device_array(s, s->coef[slot], prec, esz, slot, host, ld);
}

int tw_write_field(tw_solver *s, int grid, int field, const double *host, long ld)
{
    if (check(s) || !host || grid < 0 || grid > 3) return TW_ERR_INVALID;
    const int slot = slot_of(s, grid, field);
    if (slot < 0 || ld < s->ref_cols[grid]) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    return write_device_array(s, cur_f(s, slot), s->d.precision, s->esz, slot, host, ld,
                              s->d.cpst == TW_CPST_SPLIT ? cur_res(s, slot) : nullptr);
}

int tw_read_resid(tw_solver *s, int grid, int field, double *host, long ld)
{
    if (check(s) || !host || grid < 0 || grid > 3) return TW_ERR_INVALID;
    const int slot = slot_of(s, grid, field);
    if (slot < 0 || ld < s->ref_cols[grid] || !s->res[slot]) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    return read_device_array(s, cur_res(s, slot), s->d.precision, s->esz, slot, host, ld);
}

int tw_write_resid(tw_solver *s, int grid, int field, const double *host, long ld)
{
    if (check(s) || !host || grid < 0 || grid > 3) return TW_ERR_INVALID;
    const int slot = slot_of(s, grid, field);
    if (slot < 0 || ld < s->ref_cols[grid] || !s->res[slot]) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    return write_device_array(s, cur_res(s, slot), s->d.precision, s->esz, slot, host, ld);
}

int tw_read_receivers(tw_solver *s, double *host)
{
    if (check(s) || !host) return TW_ERR_INVALID;
    const int n = (int)(s->rcv_tab.size() / 4);
    if (n == 0 || s->steps_done == 0) return TW_OK;
    TW_CUDA(cudaSetDevice(s->d.device));
    TW_CUDA(cudaMemcpy2DAsync(host, sizeof(double) * s->steps_done, s->d_traces, sizeof(double) * s->d.max_steps,
                              sizeof(double) * s->steps_done, 2 * (size_t)n, cudaMemcpyDeviceToHost, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    return TW_OK;
}

int tw_read_energy(tw_solver *s, double *E_k, double *E_p0, double *E_p1)
{
    if (check(s)) return TW_ERR_INVALID;
    if (!s->d.energy) return TW_ERR_STATE;
    const int n = s->steps_done;
    if (n == 0) return TW_OK;
    TW_CUDA(cudaSetDevice(s->d.device));
    std::vector<double> e(3 * (size_t)s->d.max_steps);
    TW_CUDA(cudaMemcpyAsync(e.data(), s->d_energy, sizeof(double) * e.size(), cudaMemcpyDeviceToHost, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));
    const double *p0 = e.data(), *k = e.data() + s->d.max_steps, *p1 = e.data() + 2 * s->d.max_steps;
    for (int it = 0; it < n; it++) {
        if (E_k) E_k[it] = k[it];
        if (E_p1) E_p1[it] = p1[it];
        if (E_p0) E_p0[it] = s->periodic ? (it > 0 ? p1[it - 1] : 0.) : p0[it];
    }
    return TW_OK;
}

// halo geometry of slot f (5..9: compensation arrays) at one edge of a slab
int slab_rows(tw_solver *s, int side, int recv, int f, void **ptr, long *rows)
{
    if (!s->slab || side < 0 || side > 1 || f < 0 || f > 9) return TW_ERR_INVALID;
    const int k = f % 5;
    if (!s->has_slot(k) || (f >= 5 && !s->res[k])) return TW_ERR_INVALID;
    const bool open_top = s->row_off > 0, open_bot = s->row_off + s->d.Mx < s->Mx_glob;
    if ((side == 0 && !open_top) || (side == 1 && !open_bot)) return TW_ERR_INVALID;
    constexpr long H = 4;
    const long own0 = s->own0 - s->row_off, own1 = s->own1 - s->row_off;   // local owned rows
    long r0;
    if (side == 0) r0 = recv ? own0 - H : own0;   // top: halo above, or the first owned rows
    else r0 = recv ? own1 : own1 - H;              // bottom: halo below, or the last owned rows
    char *base = (char *)(f < 5 ? cur_f(s, k) : cur_res(s, k));
    *ptr = base + (size_t)r0 * s->pitch * s->esz;
    *rows = H;
    return TW_OK;
}

int tw_slab_halo(tw_solver *s, int side, int recv, int f, void **ptr, long *rows, long *row_bytes, long *pitch_bytes)
{
    if (check(s) || !ptr || !rows || !row_bytes || !pitch_bytes) return TW_ERR_INVALID;
    const int rc = slab_rows(s, side, recv, f, ptr, rows);
    if (rc != TW_OK) return rc;
    *row_bytes = (long)s->cols[f % 5] * s->esz;
    *pitch_bytes = s->pitch * s->esz;
    return TW_OK;
}

int tw_slab_pack(tw_solver *s, int side, void *dst, long *bytes)
{
    if (check(s) || !bytes || !s->slab) return TW_ERR_INVALID;
    const int nf = s->d.cpst != TW_CPST_00 ? 10 : 5;
    long total = 0;
    for (int f = 0; f < nf; f++) {
        void *src;
        long rows, rb, pb;
        const int rc = tw_slab_halo(s, side, 0, f, &src, &rows, &rb, &pb);
        if (rc != TW_OK) return rc;
        if (dst) TW_CUDA(cudaMemcpy2DAsync((char *)dst + total, rb, src, pb, rb, rows, cudaMemcpyDefault, s->st));
        total += rb * rows;
    }
    *bytes = total;
    return TW_OK;
}

int tw_slab_unpack(tw_solver *s, int side, const void *src)
{
    if (check(s) || !src || !s->slab) return TW_ERR_INVALID;
    const int nf = s->d.cpst != TW_CPST_00 ? 10 : 5;
    long off = 0;
    for (int f = 0; f < nf; f++) {
        void *dst;
        long rows, rb, pb;
        const int rc = tw_slab_halo(s, side, 1, f, &dst, &rows, &rb, &pb);
        if (rc != TW_OK) return rc;
        TW_CUDA(cudaMemcpy2DAsync(dst, pb, (const char *)src + off, rb, rb, rows, cudaMemcpyDefault, s->st));
        off += rb * rows;
    }
    return TW_OK;
}

int tw_slab_exchange(tw_solver *up, tw_solver *lo)
{
    if (check(up) || check(lo) || !up->slab || !lo->slab) return TW_ERR_INVALID;
    if (up->Mx_glob != lo->Mx_glob || up->own1 != lo->own0 || up->d.My != lo->d.My || up->esz != lo->esz ||
        up->d.cpst != lo->d.cpst || up->steps_done != lo->steps_done)
        return TW_ERR_INVALID;
    if (up->d.device != lo->d.device) {
        const int rc = link_devices(up->d.device, lo->d.device);
        if (rc != TW_OK) return rc;
    }
    TW_CUDA(cudaSetDevice(lo->d.device));
    TW_CUDA(cudaStreamSynchronize(lo->st));
    TW_CUDA(cudaSetDevice(up->d.device));
    TW_CUDA(cudaStreamSynchronize(up->st));
    const int nf = up->d.cpst != TW_CPST_00 ? 10 : 5;
    for (int f = 0; f < nf; f++) {
        void *src, *dst;
        long rows, rb, pb;
        // the upper slab's last owned rows -> the lower's top halo; the lower's first owned rows ->
        // the upper's bottom halo
        int rc = tw_slab_halo(up, 1, 0, f, &src, &rows, &rb, &pb);
        if (rc == TW_OK) rc = tw_slab_halo(lo, 0, 1, f, &dst, &rows, &rb, &pb);
        if (rc != TW_OK) return rc;
        TW_CUDA(cudaMemcpy2DAsync(dst, pb, src, pb, rb, rows, cudaMemcpyDefault, up->st));
        rc = tw_slab_halo(lo, 0, 0, f, &src, &rows, &rb, &pb);
        if (rc == TW_OK) rc = tw_slab_halo(up, 1, 1, f, &dst, &rows, &rb, &pb);
        if (rc != TW_OK) return rc;
        TW_CUDA(cudaMemcpy2DAsync(dst, pb, src, pb, rb, rows, cudaMemcpyDefault, up->st));
    }
    TW_CUDA(cudaStreamSynchronize(up->st));
    return TW_OK;
}

int tw_slab_run(tw_solver *const *slabs, int n, int steps)
{
    if (!slabs || n < 1 || steps < 0) return TW_ERR_INVALID;
    for (int i = 0; i < n; i++) {
        tw_solver *s = slabs[i];
        if (check(s) || !s->slab || !s->fused || !s->mat_ready) return check(s) ? TW_ERR_INVALID : TW_ERR_STATE;
        // the linked step kernels exist for FP32 / FP64 storage and coefficients
        if (s->d.precision == TW_BF16 || s->d.precision == TW_FP16 || s->d.coef_fp16) return TW_ERR_UNSUPPORTED;
        if (s->steps_done + (long)steps > s->d.max_steps) return TW_ERR_RECORD_FULL;
        const tw_solver *t = slabs[0];
        if (s->Mx_glob != t->Mx_glob || s->d.My != t->d.My || s->d.precision != t->d.precision ||
            s->d.cpst != t->d.cpst || s->steps_done != t->steps_done || s->parity != t->parity)
            return TW_ERR_INVALID;
        if (i > 0 && slabs[i - 1]->own1 != s->own0) return TW_ERR_INVALID;   // consecutive slabs, top to bottom
    }
    if (slabs[0]->own0 != 0 || slabs[n - 1]->own1 != slabs[0]->Mx_glob) return TW_ERR_INVALID;   // the whole grid
    // neighbours on other GPUs are written through peer access (NVLink)
    for (int i = 0; i + 1 < n; i++) {
        const int rc = link_devices(slabs[i]->d.device, slabs[i + 1]->d.device);
        if (rc != TW_OK) return rc;
    }
    std::vector<cudaEvent_t> ev(n, nullptr);
    int rc = TW_OK;
    for (int i = 0; i < n && rc == TW_OK; i++) {
        cudaSetDevice(slabs[i]->d.device);
        if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) rc = TW_ERR_CUDA;
    }
    for (int i = 0; i < n; i++) {
        slabs[i]->link[0] = i > 0 ? slabs[i - 1] : nullptr;
        slabs[i]->link[1] = i + 1 < n ? slabs[i + 1] : nullptr;
    }
    // step k of a slab writes its cut rows into the neighbours' output buffers of step k, which
    // their step k - 1 read as input: it starts after the neighbours' step k - 1 (and its own)
    for (int k = 0; k < steps && rc == TW_OK; k++) {
        for (int i = 0; i < n && rc == TW_OK; i++) {
            tw_solver *s = slabs[i];
            cudaSetDevice(s->d.device);
            if (k > 0) {
                if (i > 0 && cudaStreamWaitEvent(s->st, ev[i - 1], 0) != cudaSuccess) rc = TW_ERR_CUDA;
                if (i + 1 < n && cudaStreamWaitEvent(s->st, ev[i + 1], 0) != cudaSuccess) rc = TW_ERR_CUDA;
            } else {   // the first step waits for whatever the neighbours had queued before
                for (int q : {i - 1, i + 1})
                    if (q >= 0 && q < n && (cudaEventRecord(ev[q], slabs[q]->st) != cudaSuccess ||
                                            cudaStreamWaitEvent(s->st, ev[q], 0) != cudaSuccess))
                        rc = TW_ERR_CUDA;
            }
        }
        for (int i = 0; i < n && rc == TW_OK; i++) {
            tw_solver *s = slabs[i];
            cudaSetDevice(s->d.device);
            enqueue(s, 1, s->st);
            if (cudaEventRecord(ev[i], s->st) != cudaSuccess) rc = TW_ERR_CUDA;
        }
        if (rc == TW_OK)
            for (int i = 0; i < n; i++) slabs[i]->steps_done += 1;
    }
    // the last step of a slab still stores into its neighbours' rows: each slab's stream waits
    // for its neighbours' last step, so that synchronising, stepping, reading or destroying one
    // handle alone afterwards is ordered after every write into its buffers
    for (int i = 0; i < n && rc == TW_OK && steps > 0; i++) {
        cudaSetDevice(slabs[i]->d.device);
        for (int q : {i - 1, i + 1})
            if (q >= 0 && q < n && cudaStreamWaitEvent(slabs[i]->st, ev[q], 0) != cudaSuccess) rc = TW_ERR_CUDA;
    }
    for (int i = 0; i < n; i++) {
        slabs[i]->link[0] = slabs[i]->link[1] = nullptr;
        cudaSetDevice(slabs[i]->d.device);
        if (ev[i]) cudaEventDestroy(ev[i]);
    }
    if (rc == TW_OK) {
        for (int i = 0; i < n; i++) {
            cudaSetDevice(slabs[i]->d.device);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_fail(e, "tw_slab_run");
        }
    }
    return rc;
}

int tw_data_misfit(tw_solver *s, const double *obs, double *total, double *per_rcv)
{
    if (check(s) || !obs) return TW_ERR_INVALID;
    const int n = (int)(s->rcv_tab.size() / 4), nt = s->steps_done;
    std::vector<double> tr(2 * (size_t)n * std::max(nt, 1));
    if (n > 0 && nt > 0) {
        const int rc = tw_read_receivers(s, tr.data());
        if (rc != TW_OK) return rc;
    }
    // the reference keeps records and observations in its storage precision and squares their
    // difference in double: pow((double)(RESULT - record), 2) (forward.cpp:436-437)
    const bool f32 = s->d.precision == TW_FP32;
    double J = 0.;
    for (int r = 0; r < n; r++) {
        double Jr = 0.;   // sum over steps and the grid's fields, in the reference's order
        const int nf = s->rcv_tab[4 * r + 1] >= 0 ? 2 : 1;
        for (int it = 0; it < nt; it++)
            for (int f = 0; f < nf; f++) {
                const size_t i = (2 * (size_t)r + f) * nt + it;
                const double d = f32 ? (double)((float)tr[i] - (float)obs[i]) : tr[i] - obs[i];
                Jr += std::pow(d, 2);
            }
        if (per_rcv) per_rcv[r] = Jr;
        J += Jr;
    }
    if (total) *total = J;
    return TW_OK;
}

int tw_io_write_records(tw_solver *s, const char *folder, int src_index, const int *rcv_index, int snapshots)
{
    if (check(s) || !folder) return TW_ERR_INVALID;
    const int n = (int)(s->rcv_tab.size() / 4), nt = s->steps_done;
    const double sc = s->d.source_scaling;
    static const char *gname[4] = {"Sxy", "Vx", "Vy", "SMM"};       // grid.hpp:155-159
    auto gstr = [](int grid) {   // data-y type first (forward.cpp:251)
        const char tx = (grid == TW_NN || grid == TW_NM) ? 'N' : 'M', ty = (grid == TW_NN || grid == TW_MN) ? 'N' : 'M';
        return std::string(1, ty) + std::string(1, tx);
    };
    auto grid_of_slot = [](int slot) { return slot == F_NN ? TW_NN : slot == F_MN ? TW_MN : slot == F_NM ? TW_NM : TW_MM; };
    const std::string src = s->src_grid >= 0
        ? "src_" + std::to_string(src_index) + "_" + gstr(s->src_grid) + "_" + std::to_string(s->src_iy) + "_" + std::to_string(s->src_ix)
        : "src_" + std::to_string(src_index) + "_none";
    if (n > 0 && nt > 0) {
        std::vector<double> tr(2 * (size_t)n * nt);
        const int rc = tw_read_receivers(s, tr.data());
        if (rc != TW_OK) return rc;
        for (int r = 0; r < n; r++) {
            const int *q = &s->rcv_tab[4 * r];
            const int g = grid_of_slot(q[0]), nf = q[1] >= 0 ? 2 : 1;
            const std::string name = std::string(folder) + "/Signal_" + src + "_rcv_" + std::to_string(rcv_index ? rcv_index[r] : r) +
                                     "_" + gstr(g) + "_" + std::to_string(q[3]) + "_" + std::to_string(q[2]) + ".txt";
            FILE *fp = fopen(name.c_str(), "w");
            if (!fp) return TW_ERR_IO;
            for (int it = 0; it < nt; it++) {
                fprintf(fp, "% 6d  ", it);
                for (int f = 0; f < nf; f++) fprintf(fp, "% 16.15e  ", sc * tr[(2 * (size_t)r + f) * nt + it]);
                fprintf(fp, "\n");
            }
            if (fclose(fp) != 0) return TW_ERR_IO;
        }
    }
    if (s->d.energy && nt > 0) {
        std::vector<double> k(nt), p0(nt), p1(nt);
        const int rc = tw_read_energy(s, k.data(), p0.data(), p1.data());
        if (rc != TW_OK) return rc;
        FILE *fp = fopen((std::string(folder) + "/Energy_" + src + ".txt").c_str(), "w");
        if (!fp) return TW_ERR_IO;
        for (int it = 0; it < nt; it++) fprintf(fp, "%16.15e\n", sc * sc * (k[it] + (p0[it] + p1[it]) / 2.));
        if (fclose(fp) != 0) return TW_ERR_IO;
    }
    if (snapshots) {
        for (int g = 0; g < 4; g++)
            for (int f = 0; f < 2; f++) {
                const int slot = slot_of(s, g, f);
                if (slot < 0) continue;
                const long R = s->ref_rows[g], Cn = s->ref_cols[g];
                std::vector<double> v((size_t)R * Cn);
                const int rc = tw_read_field(s, g, f, v.data(), Cn);
                if (rc != TW_OK) return rc;
                const std::string name = std::string(folder) + "/Snapshot_" + gstr(g) + "_" + gname[g] + "_" + std::to_string(f) + ".txt";
                FILE *fp = fopen(name.c_str(), "w");
                if (!fp) return TW_ERR_IO;
                for (double x : v) fprintf(fp, "% 16.15e\n", sc * x);
                if (fclose(fp) != 0) return TW_ERR_IO;
            }
    }
    return TW_OK;
}

int tw_get_info(tw_solver *s, tw_info *info)
{
    if (check(s) || !info) return TW_ERR_INVALID;
    for (int g = 0; g < 4; g++) { info->rows[g] = s->ref_rows[g]; info->cols[g] = s->ref_cols[g]; }
    info->pitch = s->pitch;
    info->steps_done = s->steps_done;
    info->n_rcv = (int)(s->rcv_tab.size() / 4);
    const int nf = s->elastic ? 5 : 3;
    const double csz = s->d.precision == TW_FP64 ? 8 : (s->d.coef_fp16 ? 2 : 4);
    info->bytes_per_update = nf * (2.0 * s->esz + (s->d.cpst != TW_CPST_00 ? 2.0 * s->esz : 0.0)) + nf * csz;
    info->device_bytes = s->dev_bytes;
    info->row_off = s->row_off;
    info->own_rows[0] = s->own0;
    info->own_rows[1] = s->own1;
    info->Mx_glob = s->Mx_glob;
    info->step_kind = s->tma ? 2 : (s->fused ? 1 : (s->afused ? 3 : 0));
    info->launches_per_step = s->tma ? (s->tma_witems ? 1 : 2) : ((s->fused || s->afused) ? 1 : 3);
    if (s->fused && (s->bnd & BND_Y_SAT)) info->launches_per_step += 2;   // the y-end recomputation
    return TW_OK;
}

int tw_profile(tw_solver *s, int n, double *ms)
{
    if (check(s) || n < 1 || !ms) return TW_ERR_INVALID;
    if (!s->mat_ready) return TW_ERR_STATE;
    if (s->steps_done + (long)n > s->d.max_steps) return TW_ERR_RECORD_FULL;
    TW_CUDA(cudaSetDevice(s->d.device));
    std::vector<cudaEvent_t> ev((size_t)8 * n);
    for (auto &e : ev) TW_CUDA(cudaEventCreate(&e));
    const bool f64 = s->d.precision == TW_FP64;
    for (int k = 0; k < n; k++)
        for (int ph = 0; ph < 4; ph++) {
            cudaEventRecord(ev[(size_t)8 * k + 2 * ph], s->st);
            if (s->fused || s->afused) {
                if (ph == 0) enqueue(s, 1, s->st);   // the whole step is one launch
            } else if (ph != 2 || s->d.energy) {
                if (f64) enqueue_phase<double, double>(s, ph, s->st);
                else enqueue_phase<float, float>(s, ph, s->st);
            }
            cudaEventRecord(ev[(size_t)8 * k + 2 * ph + 1], s->st);
        }
    cudaError_t e = cudaStreamSynchronize(s->st);
    double acc[4] = {0, 0, 0, 0};
    for (int k = 0; k < n && e == cudaSuccess; k++)
        for (int ph = 0; ph < 4; ph++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[(size_t)8 * k + 2 * ph], ev[(size_t)8 * k + 2 * ph + 1]);
            acc[ph] += t;
        }
    for (auto &x : ev) cudaEventDestroy(x);
    if (e != cudaSuccess) return cuda_fail(e, "tw_profile");
    for (int ph = 0; ph < 4; ph++) ms[ph] = acc[ph] / n;
    if (s->fused || s->afused) ms[1] = ms[2] = ms[3] = 0.;   // the fused step launches nothing else
    s->steps_done += n;
    return TW_OK;
}

int tw_location_to_index(char type, long num, long den, int num_dx, int den_dx, long *index)
{
    if (!index || num_dx <= 0 || den_dx <= 0) return TW_ERR_INVALID;
    if (type != 'N' && type != 'M') return TW_ERR_INVALID;
    return location_to_index(type, num, den, num_dx, den_dx, index) ? TW_OK : TW_ERR_LOCATION;
}

int tw_get_stream(tw_solver *s, void **stream)
{
    if (check(s) || !stream) return TW_ERR_INVALID;
    *stream = (void *)s->st;
    return TW_OK;
}

}  // extern "C"

// ======================================================================== adjoint gradient
namespace {

// device copy of a whole state (five field slots, rows x pitch) between the solver and a buffer
int copy_state(tw_solver *s, void *const *dst, void *const *src)
{
    for (int k = 0; k < 5; k++)
        if (s->has_slot(k))
            TW_CUDA(cudaMemcpyAsync(dst[k], src[k], (size_t)s->rows[k] * s->pitch * s->esz, cudaMemcpyDeviceToDevice, s->st));
    return TW_OK;
}

// device memory of one gradient call: one allocation carved into 256-byte aligned pieces
// (sizes are summed on a first pass, then the same calls hand out the pieces), freed on exit
struct DevBuf {
    cudaStream_t st;
    char *base = nullptr;
    size_t used = 0, size = 0;
    bool sizing = true;
    explicit DevBuf(cudaStream_t s) : st(s) {}
    ~DevBuf()
    {
        cudaStreamSynchronize(st);
        cudaFree(base);
    }
    int get(void **out, size_t bytes)
    {
        const size_t b = (bytes + 255) / 256 * 256;
        if (sizing) {
            size += b;
            *out = nullptr;
            return TW_OK;
        }
        if (used + b > size) return TW_ERR_INVALID;
        *out = base + used;
        used += b;
        return TW_OK;
    }
    int commit()   // allocate and zero the arena, then hand out pieces in the same order
    {
        cudaError_t e = cudaMalloc((void **)&base, size);
        if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? TW_ERR_NOMEM : cuda_fail(e, "tw_adjoint_gradient");
        e = cudaMemsetAsync(base, 0, size, st);
        if (e != cudaSuccess) return cuda_fail(e, "tw_adjoint_gradient");
        sizing = false;
        return TW_OK;
    }
};

// ---- binomial checkpointing (revolve-style) with a fixed number of state slots
//
// Reversing n steps l..r-1 with the state at l in a slot and c free slots: advance a steps into a
// free slot, reverse the upper part with c - 1 free slots, then the lower part with c (binomial
// checkpointing, Griewank's revolve schedule family). Each adjoint step n needs the forward
// states n and n + 1: the end state is made by one more forward step, unless a lower part of one
// step finds it still in the slot the upper part started from. With no free slot every step's
// states are recomputed from the slot. The first advance a minimises the forward steps
// F(n, c) = min_a a + F(n - a, c - 1) + (a == 1 ? 0 : F(a, c)), F(1, c) = 1, F(n, 0) = n (n + 1) / 2,
// by dynamic programming when the table is small (n^2 c <= 4e8); otherwise it is taken from the
// binomial bound with s = c + 1 snapshots (the start state's included): t the smallest number with
// C(s + t, s) >= n, a = max(C(s + t - 2, s), n - C(s - 1 + t, s - 1)), within a fraction of the
// optimum.
struct RvAction {
    int kind;        // RV_FWD: advance state t0 by n steps from buffer a into buffer b;
                     // RV_FIN: buffer a holds the final state (residuals, first injection);
                     // RV_ADJ: adjoint step t0 with state t0 in a and t0 + 1 in b
    int a, b, t0, n;
};
enum { RV_FWD = 0, RV_FIN = 1, RV_ADJ = 2 };

long binom_capped(int c, int t, long cap)   // C(c + t, c), saturated above cap
{
    double v = 1.0;
    for (int k = 1; k <= c; k++) {
        v = v * (double)(t + k) / (double)k;
        if (v > (double)cap) return cap + 1;
    }
    return (long)(v + 0.5);
}

// optimal first advances by dynamic programming (rows c = 0..cmax, columns n = 0..nmax)
struct RvTable {
    int nmax = 0, cmax = -1;
    std::vector<long> F;
    std::vector<int> A;
    long &f(int n, int c) { return F[(size_t)c * (nmax + 1) + n]; }
    int &a(int n, int c) { return A[(size_t)c * (nmax + 1) + n]; }
    void build(int n_, int c_)
    {
        nmax = n_;
        cmax = c_;
        F.assign((size_t)(cmax + 1) * (nmax + 1), 0);
        A.assign(F.size(), 1);
        for (int c = 0; c <= cmax; c++)
            for (int n = 1; n <= nmax; n++) {
                if (n == 1) { f(n, c) = 1; continue; }
                if (c == 0) { f(n, c) = (long)n * (n + 1) / 2; continue; }
                long best = -1;
                int arg = 1;
                for (int a_ = 1; a_ < n; a_++) {
                    const long v = a_ + f(n - a_, c - 1) + (a_ == 1 ? 0 : f(a_, c));
                    if (best < 0 || v < best) { best = v; arg = a_; }
                }
                f(n, c) = best;
                a(n, c) = arg;
            }
    }
};

struct RvPlan {
    int nt, TA, TB;
    bool fin_done = false;
    std::vector<RvAction> acts;
    RvTable *tab = nullptr;   // optimal advances, when computed
    long first_advance(int n, int c)
    {
        if (tab && n <= tab->nmax && c <= tab->cmax) return tab->a(n, c);
        const int s = c + 1;
        int t = 1;
        while (binom_capped(s, t, n) < n) t++;
        const long lo = t >= 2 ? binom_capped(s, t - 2, n) : 0;
        const long hi = binom_capped(s - 1, t, n);
        return std::max(1L, std::min((long)n - 1, std::max(lo, (long)n - hi)));
    }
    void reverse(int l, int r, int p, std::vector<int> &free_slots)
    {
        const int n = r - l;
        if (n == 1) {
            acts.push_back({RV_FWD, p, TB, l, 1});
            if (!fin_done && r == nt) { acts.push_back({RV_FIN, TB, 0, nt, 0}); fin_done = true; }
            acts.push_back({RV_ADJ, p, TB, l, 0});
            return;
        }
        const int c = (int)free_slots.size();
        if (c == 0) {
            for (int k = r - 1; k >= l; k--) {
                int src = p;
                if (k > l) { acts.push_back({RV_FWD, p, TA, l, k - l}); src = TA; }
                acts.push_back({RV_FWD, src, TB, k, 1});
                if (!fin_done && k + 1 == nt) { acts.push_back({RV_FIN, TB, 0, nt, 0}); fin_done = true; }
                acts.push_back({RV_ADJ, src, TB, k, 0});
            }
            return;
        }
        const long a = first_advance(n, c);
        const int m = l + (int)a, q = free_slots.back();
        free_slots.pop_back();
        acts.push_back({RV_FWD, p, q, l, (int)a});
        reverse(m, r, q, free_slots);
        if (a == 1) {   // the lower part is one step whose end state is still in slot q
            acts.push_back({RV_ADJ, p, q, l, 0});
            free_slots.push_back(q);
            return;
        }
        free_slots.push_back(q);
        reverse(l, m, p, free_slots);
    }
};

// the action list for nt steps with `slots` state slots (slot 0 holds the initial state); buffers
// 0..slots-1 are the slots, slots and slots + 1 two more states
std::vector<RvAction> revolve_plan(int nt, int slots)
{
    RvPlan pl;
    pl.nt = nt;
    pl.TA = slots;
    pl.TB = slots + 1;
    std::vector<int> free_slots;
    for (int k = slots - 1; k >= 1; k--) free_slots.push_back(k);
    RvTable tab;
    const int c = slots - 1;
    if (c >= 1 && c < nt - 1 && (double)nt * nt * c <= 4e8) {
        tab.build(nt, c);
        pl.tab = &tab;
    }
    pl.reverse(0, nt, 0, free_slots);
    return pl.acts;
}

// replay a plan on labels: every buffer read holds the state the action expects, the final state
// is announced once before the first adjoint step, adjoint steps run nt - 1 down to 0 once each;
// returns the forward steps taken, or -1
long revolve_check(const std::vector<RvAction> &acts, int nt, int slots)
{
    std::vector<int> lab(slots + 2, -1);
    lab[0] = 0;
    long fwd = 0;
    int next_adj = nt - 1;
    bool fin = false;
    for (const RvAction &x : acts) {
        if (x.a < 0 || x.a >= slots + 2) return -1;
        if (x.kind == RV_FWD) {
            if (x.b < 0 || x.b >= slots + 2 || x.b == x.a || lab[x.a] != x.t0 || x.n < 1) return -1;
            lab[x.b] = x.t0 + x.n;
            fwd += x.n;
        } else if (x.kind == RV_FIN) {
            if (fin || lab[x.a] != nt || next_adj != nt - 1) return -1;
            fin = true;
        } else {
            if (!fin || x.t0 != next_adj || lab[x.a] != x.t0 || lab[x.b] != x.t0 + 1) return -1;
            next_adj--;
        }
    }
    return (fin && next_adj == -1) ? fwd : -1;
}

// the gradient call. K > 0: checkpoints every K steps, each segment recomputed into a buffer of
// K + 1 states; K == 0: binomial checkpointing in `slots` state slots
template <class C>
int adjoint_t(tw_solver *s, int nt, const double *obs, int K, int slots, double *misfit, double *const *g_grid,
              double *g_rho, double *g_vp, double *g_vs, double *const *g_state)
{
    const size_t fsz[5] = {(size_t)s->rows[0] * s->pitch, (size_t)s->rows[1] * s->pitch, (size_t)s->rows[2] * s->pitch,
                           (size_t)s->rows[3] * s->pitch, (size_t)s->rows[4] * s->pitch};
    const bool periodic = K > 0;
    const int n_ck = periodic ? (nt + K - 1) / K : 0;
    const int n_rcv = (int)(s->rcv_tab.size() / 4);
    DevBuf mem(s->st);
    int rc;
    // periodic: checkpoints every K steps and the states of one segment; revolve: the slots, two
    // states of the plan and two scratch states for multi-step advances; both: the final state
    std::vector<std::array<void *, 5>> ck(periodic ? n_ck : slots + 2), seg(periodic ? K + 1 : 2);
    std::array<void *, 5> fin{};
    AdjArgs<C> a{};
    double *d_res = nullptr, *gq[5] = {}, *nd = nullptr;
    const bool want_model = g_rho || g_vp || g_vs;
    const long Pm = want_model ? (s->model_Mxp + 2) * (s->model_Myp + 2) : 0;
    for (int pass = 0; pass < 2; pass++) {
        for (auto *set : {&ck, &seg})
            for (auto &st_ : *set)
                for (int k = 0; k < 5; k++)
                    if ((rc = mem.get(&st_[k], fsz[k] * sizeof(C))) != TW_OK) return rc;
        for (int k = 0; k < 5; k++) {
            if ((rc = mem.get(&fin[k], fsz[k] * sizeof(C))) != TW_OK) return rc;
            if ((rc = mem.get((void **)&a.lam[k], fsz[k] * sizeof(C))) != TW_OK) return rc;
            if ((rc = mem.get((void **)&a.w[k], fsz[k] * sizeof(C))) != TW_OK) return rc;
            if ((rc = mem.get((void **)&a.g[k], fsz[k] * sizeof(double))) != TW_OK) return rc;
            if ((rc = mem.get((void **)&gq[k], sizeof(double) * s->rows[k] * s->cols[k])) != TW_OK) return rc;
        }
        if (n_rcv > 0 && (rc = mem.get((void **)&d_res, sizeof(double) * 2 * (size_t)n_rcv * nt)) != TW_OK) return rc;
        if (want_model && (rc = mem.get((void **)&nd, sizeof(double) * 7 * Pm)) != TW_OK) return rc;
        if (pass == 0 && (rc = mem.commit()) != TW_OK) return rc;
    }
    for (int k = 0; k < 5; k++) a.coef[k] = (const C *)s->coef[k];
    auto cur = [&]() {
        std::array<void *, 5> c{};
        for (int k = 0; k < 5; k++) c[k] = cur_f(s, k);
        return c;
    };
    a.pitch = s->pitch;
    a.Mx = (int)s->d.Mx;
    a.My = (int)s->d.My;
    a.op = make_ops<C>((double)s->d.num_dx / (double)s->d.den_dx, s->d.dt, false);
    a.rcv = s->d_rcv;
    a.n_rcv = n_rcv;
    a.resid = d_res;
    a.nt = nt;
    // residuals and misfit on the host (FP64) from the recorded traces, and the first injection
    // lam_nt = R^T r_{nt-1}
    double J = 0.;
    auto residuals = [&]() -> int {
        std::vector<double> tr(2 * (size_t)n_rcv * nt), res(tr.size());
        if (n_rcv > 0) {
            TW_CUDA(cudaMemcpy2DAsync(tr.data(), sizeof(double) * nt, s->d_traces, sizeof(double) * s->d.max_steps,
                                      sizeof(double) * nt, 2 * (size_t)n_rcv, cudaMemcpyDeviceToHost, s->st));
            TW_CUDA(cudaStreamSynchronize(s->st));
            for (int q = 0; q < n_rcv; q++)
                for (int f = 0; f < 2; f++) {
                    const bool has = s->rcv_tab[4 * q + f] >= 0;
                    for (int it = 0; it < nt; it++) {
                        const size_t i = (2 * (size_t)q + f) * nt + it;
                        res[i] = has ? tr[i] - obs[i] : 0.;
                        J += 0.5 * res[i] * res[i];
                    }
                }
            TW_CUDA(cudaMemcpyAsync(d_res, res.data(), sizeof(double) * res.size(), cudaMemcpyHostToDevice, s->st));
            TW_CUDA(cudaStreamSynchronize(s->st));   // the host vector leaves scope
        }
        launch_adjoint_inject<C>(a, nt - 1, s->st);
        return TW_OK;
    };
    // one adjoint step n with the forward states n (u0) and n + 1 (u1), then the injection of n - 1
    auto adjoint_step = [&](int n, void *const *u0, void *const *u1) {
        for (int k = 0; k < 5; k++) {
            a.u0[k] = (const C *)u0[k];
            a.u1[k] = (const C *)u1[k];
        }
        launch_adjoint_step<C>(a, s->st);
        if (n >= 1) launch_adjoint_inject<C>(a, n - 1, s->st);
    };
    void *const none[5] = {};

    if (periodic) {
        // forward sweep, keeping a checkpoint every K steps
        for (int c = 0; c < n_ck; c++) {
            if ((rc = copy_state(s, ck[c].data(), cur().data())) != TW_OK) return rc;
            const int n = std::min(K, nt - c * K);
            enqueue(s, n, s->st);
            s->steps_done += n;
        }
        if ((rc = copy_state(s, fin.data(), cur().data())) != TW_OK) return rc;
        TW_CUDA(cudaGetLastError());
        if ((rc = residuals()) != TW_OK) return rc;
        // backward sweep: per segment, recompute its states from the checkpoint, then step the
        // adjoint back through it
        for (int c = n_ck - 1; c >= 0; c--) {
            const int k0 = c * K, k1 = std::min(nt, k0 + K);
            TW_CUDA(cudaMemcpyAsync(s->d_step, &k0, sizeof(int), cudaMemcpyHostToDevice, s->st));
            if ((rc = copy_state(s, seg[0].data(), ck[c].data())) != TW_OK) return rc;
            for (int k = k0; k < k1; k++)   // step k: segment state k - k0 -> k - k0 + 1 (recomputed: no energy)
                enqueue_fused_io<C, C>(s, seg[k - k0].data(), seg[k - k0 + 1].data(), none, none, s->st, false);
            for (int n = k1 - 1; n >= k0; n--) adjoint_step(n, seg[n - k0].data(), seg[n + 1 - k0].data());
            TW_CUDA(cudaGetLastError());
        }
    } else {
        // slot 0 holds the initial state; the plan's first forward steps are the forward sweep
        // (traces and energies recorded once, at the steps not computed before), the rest
        // recompute states from the slots
        if ((rc = copy_state(s, ck[0].data(), cur().data())) != TW_OK) return rc;
        const std::vector<RvAction> plan = revolve_plan(nt, slots);
        if (revolve_check(plan, nt, slots) < 0) return TW_ERR_INVALID;   // (the plan is checked on labels)
        auto buf = [&](int b) { return ck[b].data(); };
        int hw = 0;   // steps [0, hw) have been computed once
        for (const RvAction &x : plan) {
            if (x.kind == RV_FWD) {
                const bool first = x.t0 >= hw;   // (a forward advance is new or wholly recomputed)
                TW_CUDA(cudaMemcpyAsync(s->d_step, &x.t0, sizeof(int), cudaMemcpyHostToDevice, s->st));
                for (int k = 0; k < x.n; k++) {
                    void *const *in = k == 0 ? buf(x.a) : seg[(k - 1) & 1].data();
                    void *const *out = k == x.n - 1 ? buf(x.b) : seg[k & 1].data();
                    enqueue_fused_io<C, C>(s, in, out, none, none, s->st, first);
                }
                if (first) hw = x.t0 + x.n;
            } else if (x.kind == RV_FIN) {
                if ((rc = copy_state(s, fin.data(), buf(x.a))) != TW_OK) return rc;
                TW_CUDA(cudaGetLastError());
                if ((rc = residuals()) != TW_OK) return rc;
            } else {
                adjoint_step(x.t0, buf(x.a), buf(x.b));
            }
            TW_CUDA(cudaGetLastError());
        }
        s->steps_done += nt;
    }
    if (misfit) *misfit = J;
    // leave the handle as tw_step(nt) would: the final state, the step counter at nt
    if ((rc = copy_state(s, cur().data(), fin.data())) != TW_OK) return rc;
    TW_CUDA(cudaMemcpyAsync(s->d_step, &nt, sizeof(int), cudaMemcpyHostToDevice, s->st));
    TW_CUDA(cudaStreamSynchronize(s->st));

    // gradients with respect to the material on each grid: mu, rho (through 1/rho), lambda, 2mu
    for (int k = 0; k < 5; k++) {
        TW_CUDA(cudaMemcpy2DAsync(gq[k], sizeof(double) * s->cols[k], a.g[k], sizeof(double) * s->pitch,
                                  sizeof(double) * s->cols[k], s->rows[k], cudaMemcpyDeviceToDevice, s->st));
    }
    std::vector<double> h, m;
    for (int k = 0; k < 5; k++) {
        const size_t n = (size_t)s->rows[k] * s->cols[k];
        h.resize(n);
        TW_CUDA(cudaMemcpyAsync(h.data(), gq[k], sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
        TW_CUDA(cudaStreamSynchronize(s->st));
        if (k == F_MN || k == F_NM) {   // d(1/rho)/d rho = -1/rho^2 at the interpolated FP64 density
            m.resize(n);
            TW_CUDA(cudaMemcpyAsync(m.data(), s->mat[k], sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
            TW_CUDA(cudaStreamSynchronize(s->st));
            for (size_t i = 0; i < n; i++) h[i] = -h[i] / (m[i] * m[i]);
            if (want_model) TW_CUDA(cudaMemcpyAsync(gq[k], h.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->st));
        }
        if (g_grid && g_grid[k]) memcpy(g_grid[k], h.data(), sizeof(double) * n);
        TW_CUDA(cudaStreamSynchronize(s->st));
    }
    if (g_state)
        for (int k = 0; k < 5; k++) {
            if (!g_state[k]) continue;
            std::vector<C> t((size_t)s->rows[k] * s->cols[k]);
            TW_CUDA(cudaMemcpy2DAsync(t.data(), sizeof(C) * s->cols[k], a.lam[k], sizeof(C) * s->pitch,
                                      sizeof(C) * s->cols[k], s->rows[k], cudaMemcpyDeviceToHost, s->st));
            TW_CUDA(cudaStreamSynchronize(s->st));
            for (size_t i = 0; i < t.size(); i++) g_state[k][i] = (double)t[i];
        }
    if (want_model) {
        if (!s->model_set) return TW_ERR_STATE;
        const long Nxp = s->model_Mxp + 1, Nyp = s->model_Myp + 1, P = (Nxp + 1) * (Nyp + 1);
        // node gradients nd: mu, lambda, 2mu, rho (direct); then the outputs rho, vp, vs
        double *g_mu = nd, *g_lam = nd + P, *g_m2 = nd + 2 * P, *g_r = nd + 3 * P;
        struct { int slot, txN, tyN; double *node; } jobs[5] = {
            {F_NN, 1, 1, g_mu}, {F_MN, 0, 1, g_r}, {F_NM, 1, 0, g_r}, {F_MM0, 0, 0, g_lam}, {F_MM1, 0, 0, g_m2}};
        for (auto &j : jobs)
            launch_interp_T(s->rows[j.slot], s->cols[j.slot], j.txN, j.tyN, s->d.num_dx, s->d.den_dx, s->model_ndM,
                            s->model_ddM, Nxp, Nyp, gq[j.slot], j.node, s->st);
        launch_model_derive_T(s->model, s->model + P, s->model + 2 * P, P, g_mu, g_lam, g_m2, g_r, nd + 4 * P,
                              nd + 5 * P, nd + 6 * P, s->st);
        TW_CUDA(cudaGetLastError());
        double *outs[3] = {g_rho, g_vp, g_vs};
        for (int q = 0; q < 3; q++)
            if (outs[q]) TW_CUDA(cudaMemcpyAsync(outs[q], nd + (4 + q) * P, sizeof(double) * P, cudaMemcpyDeviceToHost, s->st));
        TW_CUDA(cudaStreamSynchronize(s->st));
    }
    return TW_OK;
}

// the checks both gradient entry points share
int adjoint_args(tw_solver *s, int nt, const double *obs, double *g_rho, double *g_vp, double *g_vs)
{
    if (check(s) || nt < 1 || (!obs && !s->rcv_tab.empty())) return TW_ERR_INVALID;
    if (!s->elastic || s->d.cpst != TW_CPST_00 || (s->d.precision != TW_FP64 && s->d.precision != TW_FP32) ||
        s->d.coef_fp16 || s->bnd)
        return TW_ERR_UNSUPPORTED;
    if (!s->mat_ready) return TW_ERR_STATE;
    if (s->steps_done != 0) return TW_ERR_STATE;   // the forward sweep starts at step 0
    if (nt > s->d.max_steps) return TW_ERR_RECORD_FULL;
    if ((g_rho || g_vp || g_vs) && !s->model_set) return TW_ERR_STATE;
    return TW_OK;
}

}  // namespace

extern "C" int tw_adjoint_gradient(tw_solver *s, int nt, const double *obs, int ckpt_every, double *misfit,
                                   double *const *g_grid, double *g_rho, double *g_vp, double *g_vs,
                                   double *const *g_state)
{
    int rc = adjoint_args(s, nt, obs, g_rho, g_vp, g_vs);
    if (rc != TW_OK) return rc;
    if (ckpt_every < 1) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    TW_CUDA(cudaStreamSynchronize(s->st));
    const int K = std::min(ckpt_every, nt);
    return s->d.precision == TW_FP64 ? adjoint_t<double>(s, nt, obs, K, 0, misfit, g_grid, g_rho, g_vp, g_vs, g_state)
                                     : adjoint_t<float>(s, nt, obs, K, 0, misfit, g_grid, g_rho, g_vp, g_vs, g_state);
}

extern "C" int tw_adjoint_gradient_revolve(tw_solver *s, int nt, const double *obs, int slots, double *misfit,
                                           double *const *g_grid, double *g_rho, double *g_vp, double *g_vs,
                                           double *const *g_state)
{
    int rc = adjoint_args(s, nt, obs, g_rho, g_vp, g_vs);
    if (rc != TW_OK) return rc;
    if (slots < 1) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(s->d.device));
    TW_CUDA(cudaStreamSynchronize(s->st));
    const int S = std::min(slots, nt);
    return s->d.precision == TW_FP64 ? adjoint_t<double>(s, nt, obs, 0, S, misfit, g_grid, g_rho, g_vp, g_vs, g_state)
                                     : adjoint_t<float>(s, nt, obs, 0, S, misfit, g_grid, g_rho, g_vp, g_vs, g_state);
}

extern "C" int tw_revolve_plan(int nt, int slots, long *forward_steps, int *n_actions)
{
    if (nt < 1 || slots < 1 || !forward_steps) return TW_ERR_INVALID;
    const int S = std::min(slots, nt);
    const std::vector<RvAction> plan = revolve_plan(nt, S);
    const long f = revolve_check(plan, nt, S);
    if (f < 0) return TW_ERR_INVALID;
    *forward_steps = f;
    if (n_actions) *n_actions = (int)plan.size();
    return TW_OK;
}

// ======================================================================== batched shots
// Many acoustic handles advanced together: one launch per half-step covers the tiles of every
// shot (batch.cu), one launch gathers every shot's receivers and advances every step counter.
struct tw_batch {
    std::vector<tw_solver *> shots;
    int precision = TW_FP32, cpst = 0, periodic = 0, device = 0;
    // periodic shots step with the fused acoustic kernel: per-shot arguments for both relative
    // parities (d_ac: 2 x n), the launch's warps, its CTA counter, and the CTAs-per-SM target
    bool fused = false;
    void *d_ac = nullptr;
    int *d_done = nullptr;
    int n_warps = 0, per_sm = TW_AC_CTAS_PER_SM;
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    void *d_shots = nullptr, *d_gather = nullptr;
    int *d_tile_shot = nullptr;
    int tile_cap = 0, n_tiles = 0;
    BatchShape shape{32, 8, 1, 0};
    cudaGraphExec_t gexec = nullptr;
    int graph_steps = 0;

    void drop_graph()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
        graph_steps = 0;
    }
    ~tw_batch()
    {
        drop_graph();
        cudaFree(d_shots); cudaFree(d_gather); cudaFree(d_tile_shot); cudaFree(d_ac); cudaFree(d_done);
        if (done) cudaEventDestroy(done);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

bool shape_ok(const BatchShape &b)
{
    return b.tx >= 1 && b.ty >= 1 && b.tx * b.ty <= 256 && (b.tx * b.ty) % 32 == 0 && b.rpt >= 1 && b.rpt <= 64 &&
           b.ctas >= 0;
}

// tile list and per-shot arguments for a launch shape
template <class S, class C>
int batch_layout_t(tw_batch *b, const BatchShape &shape)
{
    const int n = (int)b->shots.size();
    std::vector<BatchShot<S, C>> sh(n);
    std::vector<GatherArgs<S>> ga(n);
    std::vector<int> tile_shot;
    for (int k = 0; k < n; k++) {
        tw_solver *s = b->shots[k];
        const long rows = s->d.Mx + 1, cols = s->d.My + 1;   // the N-sized region covers every grid
        const long tx = (cols + shape.tx - 1) / shape.tx, ty = (rows + (long)shape.ty * shape.rpt - 1) / ((long)shape.ty * shape.rpt);
        if ((long)tile_shot.size() + tx * ty > (1L << 30)) return TW_ERR_INVALID;
        sh[k].a = step_args<S, C>(s);
        sh[k].tiles_x = (int)tx;
        sh[k].tile_off = (int)tile_shot.size();
        tile_shot.insert(tile_shot.end(), (size_t)(tx * ty), k);
        GatherArgs<S> &g = ga[k];
        for (int q = 0; q < 5; q++) g.f[q] = (const S *)cur_f(s, q);
        g.rcv = s->d_rcv;
        g.n_rcv = (int)(s->rcv_tab.size() / 4);
        g.pitch = s->pitch;
        g.traces = s->d_traces;
        g.max_steps = s->d.max_steps;
        g.step = s->d_step;
        g.flags = s->d_flags;
    }
    if ((int)tile_shot.size() > b->tile_cap) {
        cudaFree(b->d_tile_shot);
        b->d_tile_shot = nullptr;
        TW_CUDA(cudaMalloc((void **)&b->d_tile_shot, sizeof(int) * tile_shot.size()));
        b->tile_cap = (int)tile_shot.size();
    }
    if (!b->d_shots) {
        TW_CUDA(cudaMalloc(&b->d_shots, sizeof(BatchShot<S, C>) * n));
        TW_CUDA(cudaMalloc(&b->d_gather, sizeof(GatherArgs<S>) * n));
    }
    TW_CUDA(cudaMemcpyAsync(b->d_shots, sh.data(), sizeof(BatchShot<S, C>) * n, cudaMemcpyHostToDevice, b->st));
    TW_CUDA(cudaMemcpyAsync(b->d_gather, ga.data(), sizeof(GatherArgs<S>) * n, cudaMemcpyHostToDevice, b->st));
    TW_CUDA(cudaMemcpyAsync(b->d_tile_shot, tile_shot.data(), sizeof(int) * tile_shot.size(), cudaMemcpyHostToDevice, b->st));
    TW_CUDA(cudaStreamSynchronize(b->st));
    b->n_tiles = (int)tile_shot.size();
    b->shape = shape;
    if (b->shape.ctas == 0) b->shape.ctas = b->n_tiles;
    b->drop_graph();
    return TW_OK;
}

// fused batches: segments of about the same height in every shot, sized for per_sm CTAs of work
// on each of 148 SMs (8 rows or more); arguments for both relative parities from each shot's
// current buffer
template <class S, class C>
int batch_fused_layout_t(tw_batch *b, int per_sm)
{
    const int n = (int)b->shots.size();
    double work = 0.;   // strip x row units of all shots
    for (tw_solver *s : b->shots) work += (double)((s->d.My + 1 + FS_WARP_CORE - 1) / FS_WARP_CORE) * s->d.Mx;
    const double rows = std::max(8.0, work / (148.0 * per_sm * FS_WARPS));
    std::vector<AcShot<S, C>> ac(2 * (size_t)n);
    int off = 0;
    for (int k = 0; k < n; k++) {
        tw_solver *s = b->shots[k];
        for (int p = 0; p < 2; p++) {
            AcShot<S, C> a = acoustic_shot<S, C>(s, s->parity ^ p);
            a.n_seg = std::max(1, std::min((int)s->d.Mx / 8, (int)std::lround(s->d.Mx / rows)));
            a.warp_off = off;
            ac[(size_t)p * n + k] = a;
        }
        off += ac[k].n_seg * ac[k].n_wstrip;
    }
    if (!b->d_ac) TW_CUDA(cudaMalloc(&b->d_ac, sizeof(AcShot<S, C>) * 2 * n));
    if (!b->d_done) {
        TW_CUDA(cudaMalloc((void **)&b->d_done, sizeof(int)));
        TW_CUDA(cudaMemsetAsync(b->d_done, 0, sizeof(int), b->st));
    }
    TW_CUDA(cudaMemcpyAsync(b->d_ac, ac.data(), sizeof(AcShot<S, C>) * ac.size(), cudaMemcpyHostToDevice, b->st));
    TW_CUDA(cudaStreamSynchronize(b->st));
    if (off != b->n_warps || per_sm != b->per_sm) b->drop_graph();
    b->n_warps = off;
    b->per_sm = per_sm;
    return TW_OK;
}

int batch_fused_layout(tw_batch *b, int per_sm)
{
    return b->precision == TW_FP64 ? batch_fused_layout_t<double, double>(b, per_sm)
                                   : batch_fused_layout_t<float, float>(b, per_sm);
}

int batch_layout(tw_batch *b, const BatchShape &shape)
{
    return b->precision == TW_FP64 ? batch_layout_t<double, double>(b, shape) : batch_layout_t<float, float>(b, shape);
}

template <class S, class C>
void enqueue_batch_t(tw_batch *b, int n, cudaStream_t st)
{
    const auto *sh = (const BatchShot<S, C> *)b->d_shots;
    for (int k = 0; k < n; k++) {
        launch_batch_half<S, C>(b->periodic, b->cpst, 0, sh, b->d_tile_shot, b->n_tiles, b->shape, st);
        launch_batch_half<S, C>(b->periodic, b->cpst, 1, sh, b->d_tile_shot, b->n_tiles, b->shape, st);
        launch_batch_gather<S>((const GatherArgs<S> *)b->d_gather, (int)b->shots.size(), st);
    }
}

void enqueue_batch(tw_batch *b, int n, cudaStream_t st)
{
    if (b->fused) {   // step k uses the arguments of relative parity k & 1
        const int ns = (int)b->shots.size();
        for (int k = 0; k < n; k++) {
            if (b->precision == TW_FP64)
                launch_acoustic_fused_batch<double, double>((const AcShot<double, double> *)b->d_ac + (size_t)(k & 1) * ns, ns,
                                                            b->n_warps, b->cpst, b->d_done, st);
            else
                launch_acoustic_fused_batch<float, float>((const AcShot<float, float> *)b->d_ac + (size_t)(k & 1) * ns, ns,
                                                          b->n_warps, b->cpst, b->d_done, st);
        }
        return;
    }
    if (b->precision == TW_FP64) enqueue_batch_t<double, double>(b, n, st);
    else enqueue_batch_t<float, float>(b, n, st);
}

}  // namespace

extern "C" {

int tw_batch_create(tw_batch **out, tw_solver *const *shots, int n)
{
    if (!out || !shots || n < 1) return TW_ERR_INVALID;
    *out = nullptr;
    const tw_solver *s0 = shots[0];
    if (!s0) return TW_ERR_INVALID;
    for (int k = 0; k < n; k++) {
        const tw_solver *s = shots[k];
        if (!s) return TW_ERR_INVALID;
        for (int q = 0; q < k; q++)
            if (shots[q] == s) return TW_ERR_INVALID;
        if (s->elastic || s->d.energy) return TW_ERR_UNSUPPORTED;
        if (s->d.cpst != TW_CPST_00 && s->d.cpst != TW_CPST_3R && s->d.cpst != TW_CPST_6R) return TW_ERR_UNSUPPORTED;
        // one kernel family per batch: periodic or SAT x (each shot's own boundary variant rides in
        // its arguments)
        if (s->d.device != s0->d.device || s->d.precision != s0->d.precision || s->d.cpst != s0->d.cpst ||
            s->periodic != s0->periodic)
            return TW_ERR_UNSUPPORTED;
        if (!s->mat_ready) return TW_ERR_STATE;
    }
    tw_batch *b = new (std::nothrow) tw_batch();
    if (!b) return TW_ERR_NOMEM;
    b->shots.assign(shots, shots + n);
    b->precision = s0->d.precision;
    b->cpst = s0->d.cpst;
    b->periodic = s0->periodic;
    b->device = s0->d.device;
    auto fail = [&](int code) { delete b; return code; };
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(cuda_fail(e, "tw_batch_create"));
    b->fused = true;
    for (tw_solver *s : b->shots) b->fused = b->fused && s->pfuse;
    const int rc = b->fused ? batch_fused_layout(b, TW_AC_CTAS_PER_SM) : batch_layout(b, BatchShape{32, 8, 1, 0});
    if (rc != TW_OK) return fail(rc);
    *out = b;
    return TW_OK;
}

void tw_batch_destroy(tw_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    delete b;
}

int tw_batch_set_shape(tw_batch *b, int tx, int ty, int rows_per_thread, int ctas)
{
    if (!b) return TW_ERR_INVALID;
    const BatchShape sh{tx, ty, rows_per_thread, ctas};
    TW_CUDA(cudaSetDevice(b->device));
    if (b->fused) {   // fused batches: `ctas` is the CTAs-per-SM target of the segmentation
        if (ctas < 1) return TW_ERR_INVALID;
        return batch_fused_layout(b, ctas);
    }
    if (!shape_ok(sh)) return TW_ERR_INVALID;
    return batch_layout(b, sh);
}

int tw_batch_get_shape(tw_batch *b, int *shape4)
{
    if (!b || !shape4) return TW_ERR_INVALID;
    if (b->fused) {   // warps of FS_WARP_CORE columns, FS_WARPS per CTA, the per-SM target, the warps
        shape4[0] = FS_WARP_CORE;
        shape4[1] = FS_WARPS;
        shape4[2] = b->per_sm;
        shape4[3] = b->n_warps;
        return TW_OK;
    }
    shape4[0] = b->shape.tx;
    shape4[1] = b->shape.ty;
    shape4[2] = b->shape.rpt;
    shape4[3] = b->shape.ctas;
    return TW_OK;
}

int tw_batch_tune(tw_batch *b, int steps, double *best_ms)
{
    if (!b || steps < 1) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(b->device));
    for (tw_solver *s : b->shots) {
        TW_CUDA(cudaStreamSynchronize(s->st));
        if (steps + 3 > s->d.max_steps) steps = s->d.max_steps - 3;
    }
    if (steps < 1) return TW_ERR_RECORD_FULL;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    std::vector<BatchShape> cand;
    if (b->fused) {   // fused batches: the CTAs-per-SM target of the segmentation
        for (int per_sm : {2, 4, 8, 15, 24, 32, 48, 64}) cand.push_back(BatchShape{0, 0, 0, per_sm});
    } else {
        for (int tx : {32, 64, 128, 256})
            for (int rpt : {1, 2, 4})
                for (int per_sm : {0, 4, 8, 16}) cand.push_back(BatchShape{tx, 256 / tx, rpt, per_sm * sms});
    }
    cudaEvent_t e0, e1;
    TW_CUDA(cudaEventCreate(&e0));
    TW_CUDA(cudaEventCreate(&e1));
    double best = 1e300;
    BatchShape pick = b->shape;
    int rc = TW_OK;
    for (const BatchShape &c : cand) {
        if ((rc = b->fused ? batch_fused_layout(b, c.ctas) : batch_layout(b, c)) != TW_OK) break;
        for (tw_solver *s : b->shots) cudaMemsetAsync(s->d_step, 0, sizeof(int), b->st);
        enqueue_batch(b, 2, b->st);   // (an even count: the relative parity returns to 0)
        cudaEventRecord(e0, b->st);
        enqueue_batch(b, steps + (steps & 1), b->st);
        cudaEventRecord(e1, b->st);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) { rc = cuda_fail(e, "tw_batch_tune"); break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms / steps < best) { best = ms / steps; pick = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != TW_OK) return rc;
    for (tw_solver *s : b->shots)
        if ((rc = tw_reset(s)) != TW_OK) return rc;
    if ((rc = b->fused ? batch_fused_layout(b, pick.ctas) : batch_layout(b, pick)) != TW_OK) return rc;
    if (best_ms) *best_ms = best;
    return TW_OK;
}

int tw_batch_step(tw_batch *b, int n)
{
    if (!b || n < 0) return TW_ERR_INVALID;
    for (tw_solver *s : b->shots)
        if (s->steps_done + (long)n > s->d.max_steps) return TW_ERR_RECORD_FULL;
    if (n == 0) return TW_OK;
    TW_CUDA(cudaSetDevice(b->device));
    for (tw_solver *s : b->shots) TW_CUDA(cudaStreamSynchronize(s->st));   // queued single-shot work first
    if (b->fused) {   // each shot's current buffer may have changed since the last call
        const int rc = batch_fused_layout(b, b->per_sm);
        if (rc != TW_OK) return rc;
    }
    const int G = 16;
    int left = n;
    if (left >= G) {
        if (!b->gexec || b->graph_steps != G) {
            b->drop_graph();
            cudaGraph_t graph;
            TW_CUDA(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
            enqueue_batch(b, G, b->st);
            TW_CUDA(cudaStreamEndCapture(b->st, &graph));
            cudaError_t e = cudaGraphInstantiate(&b->gexec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
            b->graph_steps = G;
        }
        while (left >= G) {
            TW_CUDA(cudaGraphLaunch(b->gexec, b->st));
            left -= G;
        }
    }
    if (left > 0) enqueue_batch(b, left, b->st);
    TW_CUDA(cudaGetLastError());
    // later work on each shot's own stream (readback, single-shot steps) waits for the batch
    TW_CUDA(cudaEventRecord(b->done, b->st));
    for (tw_solver *s : b->shots) {
        TW_CUDA(cudaStreamWaitEvent(s->st, b->done, 0));
        s->steps_done += n;
        if (b->fused) s->parity ^= n & 1;
    }
    return TW_OK;
}

int tw_batch_sync(tw_batch *b)
{
    if (!b) return TW_ERR_INVALID;
    TW_CUDA(cudaSetDevice(b->device));
    TW_CUDA(cudaStreamSynchronize(b->st));
    int first = TW_OK;
    for (tw_solver *s : b->shots) {
        const int rc = tw_sync(s);
        if (rc != TW_OK && first == TW_OK) first = rc;
    }
    return first;
}

}  // extern "C"

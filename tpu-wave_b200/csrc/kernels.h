// Host-side declarations of the kernel launchers (implemented in the .cu files).
#pragma once
#include <cuda_runtime.h>

#include "stepper.cuh"

namespace tw {

// Programmatic dependent launch, for the short kernels of the launch-bound small-grid steps: a
// kernel launched by launch_pdl may be scheduled while the previous kernel in the stream is still
// running; it first waits (griddepcontrol.wait) until that kernel has finished and its writes are
// visible, so it reads exactly what an ordinary launch would, and then lets the next kernel be
// scheduled as its own blocks retire. What is saved is the gap between launches. (On the
// one-launch fused elastic step it did not pay, so that launch stays ordinary.)
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
template <class... P, class... A>
inline cudaError_t launch_pdl(void (*k)(P...), dim3 g, dim3 b, size_t smem, cudaStream_t st, A... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = g;
    cfg.blockDim = b;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

// one half of a time step: half 0 = velocities (+ V source), half 1 = stresses (+ S source)
template <class S, class C>
void launch_half(int physics, int periodic, int cpst, int half, const StepArgs<S, C> &a, cudaStream_t st);

// FP64 model quantities on the padded node model (grid_parameter.cpp:97-124)
void launch_model_derive(const double *rho, const double *vp, const double *vs, long n, double *lam,
                         double *m2, double *mu, cudaStream_t st);

// bilinear interpolation onto one grid (grid_parameter.cpp:7-60); out: rows x cols, compact.
// err: set to 1 on an out-of-bounds model access.
void launch_interp(int rows, int cols, int txN, int tyN, int num_dx, int den_dx, int num_dxM, int den_dxM,
                   long Nx_prmt, long Ny_prmt, const double *in, double *out, int *err, cudaStream_t st,
                   int row_off = 0);

struct MaterialArgs {
    const double *mat[5];     // FP64 NN mu, MN rho, NM rho, MM lambda (kappa), MM 2mu; rows x cols
    void *coef[5];            // stored stepping coefficients (compute type), rows x pitch
    double *w[5];             // energy weights, rows x pitch (w[4] = P2 on MM)
    int rows[5], cols[5];
    int Mx, My;
    long pitch;
    double dx;
    double nxN[8], nxM[6];    // A_diag * dx rounded to the storage type: N-type L[4] R[4], M-type L[3] R[3]
    int physics, periodic;
    int row_off, Mx_glob;     // a slab: its local row 0 is global row row_off of a grid of Mx_glob cells
    int sat_y;                // free y ends: the y factor of the energy norm follows the x rule
    int *err;                 // bit 2 set: a coefficient outside the normal range of the FP16 storage
};
// define the stepping coefficients (stored as K) and energy weights (make_density_reciprocal,
// define_parameters_energy, adjust_parameters_energy_periodic)
template <class C, class K = C>
void launch_material_finalize(const MaterialArgs &m, cudaStream_t st);

// 16-bit fixed-point coefficients (coef_fp16 = 2): codes of the FP32 array `coef` (rows x cols of
// a pitched array) on the map c = lo + step * code, lo the smallest value, step the range / 65535;
// `coef` is overwritten with the decoded values. d_mm: two unsigned of device scratch. 0 on success.
int quantize_coefficients16(float *coef, unsigned short *codes, int rows, int cols, long pitch, unsigned *d_mm,
                            float *lo, float *step, cudaStream_t st);

template <class S, class C>
struct EnergyArgs {
    const S *a[4];            // up to four terms sum_i a_i w_i b_i over rows x My
    const S *b[4];
    const double *w[4];
    const C *p[4];            // single-core form ((s p) s) w uses the stepping coefficient
    int rows[4], cols[4];
    int nterms;
    long pitch;
    double scale;             // 1/2 for the SBP energy (grid_energy.cpp:215), 1 for the single-core sums
    int single_core;
    double *out;              // energy record row of this phase, indexed by the step counter
    int max_steps;
    const int *step;
};
template <class S, class C>
void launch_energy(const EnergyArgs<S, C> &e, cudaStream_t st);

// fused elastic step (fused_step.cu): interior CTAs of FS_WARPS independent warps, each warp a
// strip of FS_WARP_CORE columns over a segment of interior rows; boundary CTAs of
// FS_BND_THREADS threads for the FS_ZONE rows at each free surface (or the whole grid when
// Mx < FS_SMALL_MX)
// tuning constants (a build may override them with -D)
#ifndef TW_FS_WARPS
#define TW_FS_WARPS 4                 // warps per interior CTA
#endif
#ifndef TW_FS_MIN_BLOCKS
#define TW_FS_MIN_BLOCKS 5            // CTAs per SM the register allocation is sized for
#endif
#ifndef TW_FS_MIN_BLOCKS_E
#define TW_FS_MIN_BLOCKS_E 4          // the same for the energy-every-step variant
#endif
#ifndef TW_FS_MIN_BLOCKS_64
#define TW_FS_MIN_BLOCKS_64 3         // FP64 fields
#endif
#ifndef TW_FS_MIN_BLOCKS_E64
#define TW_FS_MIN_BLOCKS_E64 2        // FP64 fields, energy every step
#endif
#ifndef TW_FS_CTAS_PER_SM
#define TW_FS_CTAS_PER_SM 60          // CTAs per SM the elastic row segmentation aims at (12 waves)
#endif
#ifndef TW_AC_CTAS_PER_SM
#define TW_AC_CTAS_PER_SM 32          // the same for the fused acoustic step and batches
#endif
#ifndef TW_FS_RING
#define TW_FS_RING 3                  // rows staged ahead per interior warp (FP64: 2)
#endif
constexpr int FS_WARP_CORE = 56;      // 28 core lanes x 2 columns; 2 halo lanes on each side
constexpr int FS_WARPS = TW_FS_WARPS;
constexpr int FS_ZONE = 8;
constexpr int FS_HALO = 4;              // a slab's halo rows at an open edge (the step's x reach)
// both CTA kinds share the launch and its block size
constexpr int FS_THREADS_MAX = FS_WARPS * 32;
constexpr int FS_BND_THREADS = FS_THREADS_MAX;   // row groups of FS_BND_W threads
constexpr int FS_BND_W = 64;                 // logical columns of a boundary strip (4 halo on each side)
constexpr int FS_BND_TY = FS_BND_W - 8;      // core columns of a boundary strip
constexpr int FS_SMALL_MX = 24;

template <class S, class C>
struct FusedArgs {
    const S *in[5];           // state before the step
    S *out[5];                // state after the step
    const S *rin[5];          // compensation arrays before / after
    S *rout[5];
    const void *coef[5];     // stepping coefficients: the compute type, or FP16
    long pitch;
    int Mx, My;
    Ops<C> op;
    int n_int_seg, int_rows;  // interior rows [ir0, ir0 + int_rows), in n_int_seg balanced segments
    int ir0;                  // FS_ZONE below a free surface; the halo depth below an open slab edge
    int n_zone;               // boundary zones: 0, 1 or 2, of the kinds zone_kind[]
    int zone_kind[2];         // 0: the FS_ZONE rows at the top free surface, 1: at the bottom, 2: the whole grid,
                              // 3: both ends in one CTA (the x ends joined by the SAT interface)
    int xif;                  // the x ends joined by the SAT interface (boundary CTAs only)
    int n_wstrip, n_bstrip;   // interior warp strips, boundary strips
    int n_int_cta;            // interior CTAs: the n_int_seg x n_wstrip warps, FS_WARPS per CTA
    int tile_rows;
    const double *src_inc;
    int src_grid, src_ix, src_iy;
    int *step;                // read by every CTA; the last CTA to finish advances it
    int *done;                // CTA completion counter (zero between steps)
    int *flags;
    int max_steps;
    const double *w[5];       // energy weights (ENERGY only)
    double *energy;           // [3][max_steps]: E_p0, E_k, E_p1
    // slabs linked in one process (tw_slab_run): the neighbour above (0) / below (1) receives this
    // slab's local rows [push_row[side], push_row[side] + FS_HALO) of every field (and residual)
    // at its own local row + peer_shift[side]; null pointers: no neighbour
    S *peer_out[2][5];
    S *peer_rout[2][5];
    int push_row[2], peer_shift[2];
    const int *rcv_off;       // receivers owned by each CTA (CSR over blockIdx.x: boundary CTAs
                              // zone-major, then interior CTAs segment-major)
    const int *rcv;           // [n][4]: field slot, row, column, trace row (2 * receiver + field)
    double *traces;
    // the TMA-staged step (k_elastic_tma, tma_step.cuh): the interior rows of columns
    // [TMA_Y0, y_tma_end) in n_tseg balanced segments x n_tstrip strips of TMA_CORE columns, one
    // CTA each; the other interior columns (the periodic seam among them) in n_ostrip warp strips
    // of FS_WARP_CORE columns (the first at column 0, the others from y_tma_end on) over n_oseg
    // segments, FS_WARPS warps to a CTA. Block order: boundary CTAs, warp-strip CTAs, TMA CTAs.
    int n_tseg, n_tstrip, n_tcta;
    int n_oseg, n_ostrip, n_octa;
    int y_tma_end;
    int *work;                // the TMA strips' next work item (a persistent CTA takes items until
                              // n_tcta are taken; zero between steps)
    int n_all_ctas;           // CTAs of both launches of the TMA-staged step
    // 16-bit fixed-point coefficients (coef_fp16 = 2): the TMA strips read codes (maps of the codes)
    // and decode c = qlo + qstep * code by field slot; everything else reads `coef` (decoded FP32)
    int q16;
    float qlo[5], qstep[5];
    int witems;               // the warp strips run as the first items of the TMA strips' launch
};
template <class S, class C>
void launch_fused(const FusedArgs<S, C> &a, int cpst, bool energy, bool coef16, cudaStream_t st);

// the TMA-staged fused step: FP32 fields and coefficients, plain update. The host encodes one
// tensor map per array and buffer parity (tw_tma_maps) when the handle is created.
constexpr int TMA_CORE = 120;        // core columns of a TMA strip (thread lanes 1..30, 4 columns each)
constexpr int TMA_Y0 = FS_WARP_CORE; // the first TMA strip starts after the first warp strip
constexpr int TMA_W = 128;           // columns a TMA strip loads: 4 halo on each side
constexpr int TMA_ROWS = 4;          // rows per TMA block: one per warp
constexpr int TMA_NMAP = 15;         // tensor maps: 5 fields, 5 coefficients, 5 energy weights
constexpr int TMA_TILE_ROWS = 12;    // the boundary CTAs' tile rows on a TMA handle (free-surface x ends)
struct TmaMaps {
    alignas(64) unsigned char m[TMA_NMAP][128];   // CUtensorMap objects (opaque, 128 bytes each)
};
enum { TM_NN = 0, TM_MN, TM_NM, TM_MM0, TM_MM1, TM_PMN, TM_PNM, TM_MU, TM_LAM, TM_M2,
       TM_WMN, TM_WNM, TM_WNN, TM_WM3, TM_WM4 };
// how many strips and segments the TMA-staged step uses for a grid (0 strips: not applicable)
int tma_strips(long My);
template <class S, class C>
cudaError_t prepare_tma();
// st: the handle's stream; side: a second stream of the handle; fork, join: two events of it
template <class S, class C>
void launch_tma(FusedArgs<S, C> a, const TmaMaps &maps, bool energy, cudaStream_t st, cudaStream_t side,
                cudaEvent_t fork, cudaEvent_t join);
constexpr int TMA_QW = TMA_W + 8;    // columns of a 16-bit coefficient box: from 8 before the strip's core
                                     // (a 16-byte boundary) to 4 beyond the 128 loaded field columns

// free y ends on the fused step (ysat_fix.cu): the fused kernel steps every column with the
// periodic y rule; these two launches then recompute, from the step's input buffers, the points
// whose y stencils meet an end (velocities, then the stresses that read them), with the SBP
// closures and penalties along y, overwriting the output buffers, and correct the step's energy
// records and the traces of receivers there
template <class S, class C>
struct YFixArgs {
    const S *in[5];
    S *out[5];
    const S *rin[5];
    S *rout[5];
    const C *coef[5];
    long pitch;
    int Mx, My;
    Ops<C> op;
    int xif;                  // the x ends joined by the SAT interface
    const double *src_inc;
    int src_grid, src_ix, src_iy;
    const int *step;          // advanced by the fused kernel: this step is *step - 1
    int *flags;
    int max_steps;
    const double *w[5];       // energy weights (energy on), else null
    double *energy;
    const int *rcv;           // the flat receiver table (field slots, row, column)
    int n_rcv;
    double *traces;
};
template <class S, class C>
void launch_ysat_fix(const YFixArgs<S, C> &a, int cpst, cudaStream_t st);

// fused periodic acoustic step (acoustic_fused.cu): one shot, or a batch of shots in one launch
template <class S, class C>
struct AcShot {
    const S *in[5];           // state before the step (slots F_MN Vy, F_NM Vx, F_MM0 pressure)
    S *out[5];                // state after the step
    const S *rin[5];          // residual arrays ('3' / '6' codes)
    S *rout[5];
    const C *coef[5];         // 1/rho of Vy and Vx, kappa
    long pitch;
    int Mx, My;
    Ops<C> op;
    int n_seg, n_wstrip;      // the shot's warps: n_seg row segments x n_wstrip column strips,
    int warp_off;             // numbered from warp_off within the launch
    const double *src_inc;
    int src_grid, src_ix, src_iy;
    int *step;
    int *flags;
    int max_steps;
    const int *rcv;           // [n_rcv][4]: field slot, row, column, trace row
    int n_rcv;
    double *traces;
};
template <class S, class C>
void launch_acoustic_fused(const AcShot<S, C> &a, int cpst, int *done, cudaStream_t st);
template <class S, class C>
void launch_acoustic_fused_batch(const AcShot<S, C> *shots, int n_shots, int n_warps, int cpst, int *done,
                                 cudaStream_t st);
template <class S, class C>
cudaError_t prepare_fused();

// discrete adjoint of the elastic step (adjoint.cu)
template <class C>
struct AdjArgs {
    C *lam[5];                // adjoint state (field slots), rows x pitch
    C *w[5];                  // temporaries by slot: W_nn, Z_mn, Z_nm, W_xx, W_yy
    const C *coef[5];         // stepping coefficients: mu, 1/rho, 1/rho, lambda, 2mu
    const C *u0[5];           // forward state u_n (its stresses feed the 1/rho gradients)
    const C *u1[5];           // forward state u_{n+1} (its velocities feed the mu, lambda, 2mu gradients)
    double *g[5];             // gradients with respect to the stepping coefficients
    long pitch;
    int Mx, My;
    Ops<C> op;
    const int *rcv;           // receiver table (slot0, slot1, row, column)
    int n_rcv;
    const double *resid;      // residuals [n_rcv][2][nt]
    int nt;
};
template <class C>
void launch_adjoint_step(const AdjArgs<C> &a, cudaStream_t st);
template <class C>
void launch_adjoint_inject(const AdjArgs<C> &a, int it, cudaStream_t st);
void launch_interp_T(int rows, int cols, int txN, int tyN, int num_dx, int den_dx, int num_dxM, int den_dxM,
                     long Nx_prmt, long Ny_prmt, const double *gin, double *gnode, cudaStream_t st);
void launch_model_derive_T(const double *rho, const double *vp, const double *vs, long n, const double *g_mu,
                           const double *g_lam, const double *g_m2, const double *g_rho_direct, double *g_rho,
                           double *g_vp, double *g_vs, cudaStream_t st);

template <class S>
struct GatherArgs {
    const S *f[5];
    const int *rcv;           // n_rcv x 4: field slot of field 0, of field 1 (-1: none), row, column
    int n_rcv;
    long pitch;
    double *traces;           // [n_rcv][2][max_steps]
    int max_steps;
    int *step;                // incremented by this kernel: it ends every step
    int *flags;
};
template <class S>
void launch_gather(const GatherArgs<S> &g, cudaStream_t st);
// receiver gather of every shot of a batch (one block per shot; g in device memory)
template <class S>
void launch_batch_gather(const GatherArgs<S> *g, int n_shots, cudaStream_t st);

// batched acoustic stepping (batch.cu): the shots of a batch are independent grids; one launch
// per half-step covers the tiles of all of them. A tile is tx columns x ty * rpt rows of a shot's
// N-sized region, handled by a tx x ty block (rpt rows per thread); `ctas` persistent CTAs walk
// the tile list (ctas >= the tile count: one CTA per tile).
template <class S, class C>
struct BatchShot {
    StepArgs<S, C> a;
    int tiles_x;              // tiles along y
    int tile_off;             // index of the shot's first tile
};
struct BatchShape {
    int tx, ty, rpt, ctas;
};
template <class S, class C>
void launch_batch_half(int periodic, int cpst, int half, const BatchShot<S, C> *shots, const int *tile_shot,
                       int n_tiles, const BatchShape &b, cudaStream_t st);

}  // namespace tw

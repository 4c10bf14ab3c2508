// Host-side declarations of the kernel launchers (implemented in the .cu files).
#pragma once
#include <cuda_runtime.h>

#include "stepper.cuh"

namespace tw {

// one half of a time step: half 0 = velocities (+ V source), half 1 = stresses (+ S source)
template <class S, class C>
void launch_half(int physics, int periodic, int cpst, int half, const StepArgs<S, C> &a, cudaStream_t st);

// FP64 model quantities on the padded node model (grid_parameter.cpp:97-124)
void launch_model_derive(const double *rho, const double *vp, const double *vs, long n, double *lam,
                         double *m2, double *mu, cudaStream_t st);

// bilinear interpolation onto one grid (grid_parameter.cpp:7-60); out: rows x cols, compact.
// err: set to 1 on an out-of-bounds model access.
void launch_interp(int rows, int cols, int txN, int tyN, int num_dx, int den_dx, int num_dxM, int den_dxM,
                   long Nx_prmt, long Ny_prmt, const double *in, double *out, int *err, cudaStream_t st);

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
};
// define the stepping coefficients and energy weights (make_density_reciprocal,
// define_parameters_energy, adjust_parameters_energy_periodic)
template <class C>
void launch_material_finalize(const MaterialArgs &m, cudaStream_t st);

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

// fused elastic step (fused_step.cu): one CTA per strip of FS_TY columns x segment of rows
constexpr int FS_THREADS = 256;
constexpr int FS_HALO = 4;
constexpr int FS_TY = FS_THREADS - 2 * FS_HALO;

template <class S, class C>
struct FusedArgs {
    const S *in[5];           // state before the step
    S *out[5];                // state after the step
    const S *rin[5];          // compensation arrays before / after
    S *rout[5];
    const C *coef[5];
    long pitch;
    int Mx, My;
    Ops<C> op;
    int seg_rows, n_seg, n_strip;
    const double *src_inc;
    int src_grid, src_ix, src_iy;
    int *step;                // read by every CTA; the last CTA to finish advances it
    int *done;                // CTA completion counter (zero between steps)
    int *flags;
    int max_steps;
    const double *w[5];       // energy weights (ENERGY only)
    double *energy;           // [3][max_steps]: E_p0, E_k, E_p1
    const int *rcv_off;       // receivers owned by each CTA (CSR over blockIdx.y * n_strip + blockIdx.x)
    const int *rcv;           // [n][4]: field slot, row, column, trace row (2 * receiver + field)
    double *traces;
};
template <class S, class C>
void launch_fused(const FusedArgs<S, C> &a, int cpst, bool energy, cudaStream_t st);
template <class S, class C>
cudaError_t prepare_fused();

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

}  // namespace tw

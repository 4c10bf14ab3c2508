/* ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference's 2D staggered-grid SBP-SAT stepper, used by the tests
 * (and by bench.py's CPU-baseline leg) as the checker for the CUDA product. Nothing in the
 * product links against it. Every routine follows the reference's operation order so that,
 * compiled with -ffp-contract=off, FP64 and FP32 results equal the reference's bit for bit;
 * tests/test_oracle_vs_reference.py pins that against the reference's own solver (oracle/_ref)
 * and tests/golden/.
 *
 * Conventions (the reference's): x = data slow index (rows), y = data fast index.
 * Grid codes 0 NN, 1 MN, 2 NM, 3 MM (cuda/src/cpp/namespace_forward.hpp:159-167).
 * Elastic reference sizes: NN (Mx+1)x(My+1), MN Mx x(My+1), NM (Mx+1)x My, MM Mx x My (two fields).
 * Compensation codes (grid.hpp:550-566): 0 "00", 1 "-3C", 2 "-3R", 3 "3C", 4 "3R", 5 "6C", 6 "6R".
 */
#ifndef TWAVE_ORACLE_H
#define TWAVE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int Mx, My;                 /* cells along x (slow) and y (fast) */
    double dx, dt;
    double central_f, time_delay;
    int cpst;                   /* compensation code above */
    int Nt;
    int src_grid;               /* grid code, or -1 for no source */
    long src_ix, src_iy;
    int n_rcv;
    const int *rcv_grid;
    const long *rcv_ix, *rcv_iy;
    int bc_x;                   /* x ends: 0 free surface ('F'), 2 joined by the SAT interface
                                   penalty (a boundary type other than 'F', grid_drvt.tpp:575-693) */
    int sat_y;                  /* 1: free surfaces on the y ends too (no reference run; My >= 8) */
} two_elastic_cfg;

/* grid_parameter.cpp:7-160: bilinear interpolation of the padded node model onto the four
 * staggered grids. Outputs are the FP64 values the reference rounds to its storage type:
 * NN mu, MN rho, NM rho, MM lambda, MM 2mu (reference sizes). Returns 0, or -1 on an
 * out-of-bounds model access (the reference exits there, grid_parameter.cpp:54-56). */
int two_material_map(int Mx, int My, int num_dx, int den_dx, int Mx_prmt, int My_prmt,
                     int num_dxM, int den_dxM, const double *rho, const double *vp, const double *vs,
                     double *NN_mu, double *MN_rho, double *NM_rho, double *MM_lambda, double *MM_2mu);

/* grid_energy.cpp:8-177 for storage type double / float: energy weights (norm matrices
 * included) from the stored coefficients. rho_* are the stored densities (before the
 * reciprocal, grid_parameter.cpp:131-160). Outputs FP64 at reference sizes. */
void two_energy_weights_f64(int Mx, int My, double dx, const double *NN_mu, const double *MN_rho,
                            const double *NM_rho, const double *MM_lambda, const double *MM_2mu,
                            double *w_NN, double *w_MN, double *w_NM, double *w_MM1, double *w_MM2);
void two_energy_weights_f32(int Mx, int My, double dx, const float *NN_mu, const float *MN_rho,
                            const float *NM_rho, const float *MM_lambda, const float *MM_2mu,
                            double *w_NN, double *w_MN, double *w_NM, double *w_MM1, double *w_MM2);
/* The same with sat_y = 1: the y factor of the norm is then A_diag * dx (storage-rounded) on the
 * end columns by the grid's y type and dx inside, as along x, instead of the periodic rule. */
void two_energy_weights_ext_f64(int Mx, int My, double dx, int sat_y, const double *NN_mu, const double *MN_rho,
                                const double *NM_rho, const double *MM_lambda, const double *MM_2mu,
                                double *w_NN, double *w_MN, double *w_NM, double *w_MM1, double *w_MM2);
void two_energy_weights_ext_f32(int Mx, int My, double dx, int sat_y, const float *NN_mu, const float *MN_rho,
                                const float *NM_rho, const float *MM_lambda, const float *MM_2mu,
                                double *w_NN, double *w_MN, double *w_NM, double *w_MM1, double *w_MM2);

/* forward_simulation.cpp:21-182 (+ grid_drvt.tpp, grid_update.tpp, grid_energy.cpp:180-216).
 * fields[5] = NN, MN, NM, MM0, MM1 (in: initial state, out: state after Nt steps);
 * resid[5] = the compensation arrays (the R arrays for the 'R' codes, the C arrays for the
 * 'C' codes; in/out, ignored for code 0). traces: [n_rcv][2][Nt]; energies: [Nt] each
 * (any may be NULL). Returns 0 or a negative error. */
int two_elastic_run_f64(const two_elastic_cfg *cfg, const double *NN_mu, const double *MN_irho,
                        const double *NM_irho, const double *MM_lambda, const double *MM_2mu,
                        const double *w_NN, const double *w_MN, const double *w_NM,
                        const double *w_MM1, const double *w_MM2, double *const fields[5],
                        double *const resid[5], double *traces, double *E_k, double *E_p0, double *E_p1);
int two_elastic_run_f32(const two_elastic_cfg *cfg, const float *NN_mu, const float *MN_irho,
                        const float *NM_irho, const float *MM_lambda, const float *MM_2mu,
                        const double *w_NN, const double *w_MN, const double *w_NM,
                        const double *w_MM1, const double *w_MM2, float *const fields[5],
                        float *const resid[5], double *traces, double *E_k, double *E_p0, double *E_p1);

/* Mixed precision (no counterpart in the reference): the FP32 stepper above with every new
 * field value rounded to storage: store16 2 = BF16, 3 = FP16; cfg->cpst 0 (plain) or 7 (split:
 * each value kept as hi + lo, lo = the rounded rest, reads take their FP32 sum). fields hold the
 * values the stepper reads (hi, or hi + lo); under code 7 resid receives lo. */
int two_elastic_run_mixed(const two_elastic_cfg *cfg, int store16, const float *NN_mu, const float *MN_irho,
                          const float *NM_irho, const float *MM_lambda, const float *MM_2mu, const double *w_NN,
                          const double *w_MN, const double *w_NM, const double *w_MM1, const double *w_MM2,
                          float *const fields[5], float *const resid[5], double *traces, double *E_k,
                          double *E_p0, double *E_p1);

/* singlecore/ acoustic stepper, periodic on all sides (namespaces.hpp:566-778,
 * cpu_acoustic.cpp:231-345). Grids: Vx (Nx+1)xNy, Vy Nx x(Ny+1), P Nx x Ny.
 * coef: 1/rho on Vx and Vy, kappa on P. cpst: 0 ('0'), 3 ('3'), 6 ('6').
 * rcv_mesh: 0 Vx, 1 Vy, 2 P. fields/resid [3] in/out. energy: [3][Nt] per-mesh sums. */
typedef struct {
    int Nx, Ny;
    double dx, dt, central_f, time_delay;
    int cpst, Nt;
    long src_ix, src_iy;        /* P cell, or src_ix < 0 for none */
    int n_rcv;
    const int *rcv_mesh;
    const long *rcv_ix, *rcv_iy;
} two_acoustic_cfg;

int two_acoustic_periodic_run_f64(const two_acoustic_cfg *cfg, const double *coef_vx, const double *coef_vy,
                                  const double *coef_p, double *const fields[3], double *const resid[3],
                                  double *traces, double *energy);
int two_acoustic_periodic_run_f32(const two_acoustic_cfg *cfg, const float *coef_vx, const float *coef_vy,
                                  const float *coef_p, float *const fields[3], float *const resid[3],
                                  double *traces, double *energy);

/* Ricker amplitude exactly as the reference evaluates it (forward_simulation.cpp:63-64). */
double two_ricker(double t, double central_f);

#ifdef __cplusplus
}
#endif
#endif

/* ORACLE / TEST INFRASTRUCTURE ONLY: plain-C restatement of the reference stepper.
 * See twave_oracle.h. Build with -ffp-contract=off (oracle/Makefile). */
#define _DEFAULT_SOURCE /* M_PI, as the reference takes it from <math.h> */
#include "twave_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_CAT_(a, b) a##b
#define ORACLE_CAT(a, b) ORACLE_CAT_(a, b)

/* cuda/src/cpp/namespace_forward.hpp:65 */
static const double ORACLE_STENCIL[4] = {1. / 24, -9. / 8, 9. / 8, -1. / 24};

/* namespace_forward.hpp:112-128: closures for N-type rows (DM, 4x5) and M-type rows (DN, 3x5) */
static const double ORACLE_DM_L[4][5] = {
    {-2., 3., -1., 0., 0.},
    {-1., 1., 0., 0., 0.},
    {1. / 24., -9. / 8., 9. / 8., -1. / 24., 0.},
    {-1. / 71., 6. / 71., -83. / 71., 81. / 71., -3. / 71.}};
static const double ORACLE_DM_R[4][5] = {
    {3. / 71., -81. / 71., 83. / 71., -6. / 71., 1. / 71.},
    {0., 1. / 24., -9. / 8., 9. / 8., -1. / 24.},
    {0., 0., 0., -1., 1.},
    {0., 0., 1., -3., 2.}};
static const double ORACLE_DN_L[3][5] = {
    {-79. / 78., 27. / 26., -1. / 26., 1. / 78., 0.},
    {2. / 21., -9. / 7., 9. / 7., -2. / 21., 0.},
    {1. / 75., 0., -27. / 25., 83. / 75., -1. / 25.}};
static const double ORACLE_DN_R[3][5] = {
    {1. / 25., -83. / 75., 27. / 25., 0., -1. / 75.},
    {0., 2. / 21., -9. / 7., 9. / 7., -2. / 21.},
    {0., -1. / 78., 1. / 26., -27. / 26., 79. / 78.}};

/* namespace_forward.hpp:139-154: norm diagonals and boundary projections */
static const double ORACLE_A_N_L[4] = {7. / 18., 9. / 8., 1., 71. / 72.};
static const double ORACLE_A_N_R[4] = {71. / 72., 1., 9. / 8., 7. / 18.};
static const double ORACLE_A_M_L[3] = {13. / 12., 7. / 8., 25. / 24.};
static const double ORACLE_A_M_R[3] = {25. / 24., 7. / 8., 13. / 12.};
static const double ORACLE_PROJ_N_L[1] = {1.};
static const double ORACLE_PROJ_N_R[1] = {1.};
static const double ORACLE_PROJ_M_L[3] = {15. / 8., -5. / 4., 3. / 8.};
static const double ORACLE_PROJ_M_R[3] = {3. / 8., -5. / 4., 15. / 8.};

double two_ricker(double t, double central_f)
{
    return (1 - 2 * M_PI * M_PI * central_f * central_f * t * t) *
           exp(-M_PI * M_PI * central_f * central_f * t * t);
}

/* grid_parameter.cpp:7-60 for one grid with x/y types (1 = N, 0 = M) */
static int oracle_interp(int sx, int sy, int txN, int tyN, int num_dx, int den_dx, int num_dxM, int den_dxM,
                         long Nx_prmt, long Ny_prmt, const double *Pin, double *out)
{
    const long PS = Ny_prmt + 1;
    for (long ix = 0; ix < sx; ix++)
        for (long iy = 0; iy < sy; iy++) {
            long nx, dxl, ny, dyl;
            if (txN) { nx = ix * num_dx; dxl = den_dx; } else { nx = (2 * ix + 1) * num_dx; dxl = 2L * den_dx; }
            if (tyN) { ny = iy * num_dx; dyl = den_dx; } else { ny = (2 * iy + 1) * num_dx; dyl = 2L * den_dx; }
            const long ixM = (nx * den_dxM) / (dxl * num_dxM);
            const long iyM = (ny * den_dxM) / (dyl * num_dxM);
            const double xi = (double)(nx * den_dxM) / (double)(dxl * num_dxM) - ixM;
            const double eta = (double)(ny * den_dxM) / (double)(dyl * num_dxM) - iyM;
            if (ixM < 0 || ixM + 1 > Nx_prmt || iyM < 0 || iyM + 1 > Ny_prmt) return -1;
            out[ix * sy + iy] = (1 - xi) * (1 - eta) * Pin[ixM * PS + iyM] + (1 - xi) * (eta)*Pin[ixM * PS + iyM + 1] +
                                (xi) * (1 - eta) * Pin[(ixM + 1) * PS + iyM] + (xi) * (eta)*Pin[(ixM + 1) * PS + iyM + 1];
        }
    return 0;
}

int two_material_map(int Mx, int My, int num_dx, int den_dx, int Mx_prmt, int My_prmt, int num_dxM, int den_dxM,
                     const double *rho, const double *vp, const double *vs, double *NN_mu, double *MN_rho,
                     double *NM_rho, double *MM_lambda, double *MM_2mu)
{
    const long Nxp = Mx_prmt + 1, Nyp = My_prmt + 1;
    const long P = (Nxp + 1) * (Nyp + 1);
    double *lam = (double *)malloc(sizeof(double) * P), *m2 = (double *)malloc(sizeof(double) * P),
           *mu = (double *)malloc(sizeof(double) * P);
    if (!lam || !m2 || !mu) return -2;
    /* retrieve_forward_parameter, grid_parameter.cpp:97-124 */
    for (long i = 0; i < P; i++) {
        m2[i] = 2 * rho[i] * vs[i] * vs[i];
        lam[i] = rho[i] * vp[i] * vp[i] - m2[i];
        mu[i] = rho[i] * vs[i] * vs[i];
    }
    int rc = 0;
    rc |= oracle_interp(Mx + 1, My + 1, 1, 1, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, mu, NN_mu);
    rc |= oracle_interp(Mx, My + 1, 0, 1, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, rho, MN_rho);
    rc |= oracle_interp(Mx + 1, My, 1, 0, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, rho, NM_rho);
    rc |= oracle_interp(Mx, My, 0, 0, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, lam, MM_lambda);
    rc |= oracle_interp(Mx, My, 0, 0, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, m2, MM_2mu);
    free(lam); free(m2); free(mu);
    return rc ? -1 : 0;
}

/* Storage rounding of the mixed-precision mode (no counterpart in the reference, whose 16-bit
 * build computes in 16 bits): 0 none, 2 BF16, 3 FP16, each round-to-nearest-even from FP32,
 * as cuda_bf16.h's __float2bfloat16_rn and cuda_fp16.h's __float2half_rn round. Set only for
 * the duration of two_elastic_run_mixed. */
static int oracle_store16 = 0;

static float oracle_round16(float x)
{
    if (oracle_store16 == 3) return (float)(_Float16)x;
    if (oracle_store16 == 2) {
        unsigned u;
        memcpy(&u, &x, 4);
        if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x7fffu + ((u >> 16) & 1u)) & 0xffff0000u;
        memcpy(&x, &u, 4);
    }
    return x;
}

#define T double
#define SFX _f64
#include "twave_oracle_body.inc"
#undef T
#undef SFX

#define T float
#define SFX _f32
#include "twave_oracle_body.inc"
#undef T
#undef SFX

int two_elastic_run_mixed(const two_elastic_cfg *cfg, int store16, const float *NN_mu, const float *MN_irho,
                          const float *NM_irho, const float *MM_lambda, const float *MM_2mu, const double *w_NN,
                          const double *w_MN, const double *w_NM, const double *w_MM1, const double *w_MM2,
                          float *const fields[5], float *const resid[5], double *traces, double *E_k,
                          double *E_p0, double *E_p1)
{
    if (store16 != 2 && store16 != 3) return -1;
    if (cfg->cpst != 0 && cfg->cpst != 7) return -1;
    oracle_store16 = store16;
    const int rc = two_elastic_run_f32(cfg, NN_mu, MN_irho, NM_irho, MM_lambda, MM_2mu, w_NN, w_MN, w_NM, w_MM1,
                                       w_MM2, fields, resid, traces, E_k, E_p0, E_p1);
    oracle_store16 = 0;
    return rc;
}

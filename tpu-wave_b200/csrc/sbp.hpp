// SBP operator tables and their dt/dx scaling.
//
// Values: cuda/src/cpp/namespace_forward.hpp:65 (interior stencil), :110-128 (boundary closures
// DM for N-type rows, DN for M-type rows), :137-145 (norm diagonals A), :148-156 (boundary
// projections). Scaling and rounding to the storage type follow Class_Grid::set_forward_operators
// (grid.hpp:274-481): every scaled entry is computed in double and rounded once, except
// A_inv_projection, which is rounded, then multiplied by dt rounded to the storage type
// (run_time_vector::operator*= takes a T, container_run_time.hpp:124), then rounded again.
// The periodic acoustic (single-core) tree scales its stencil as (c * dt) / dx instead
// (singlecore/src/cpp/namespaces.hpp:608-610).
#pragma once

namespace tw {

struct SbpTables {
    static constexpr double stencil[4] = {1. / 24, -9. / 8, 9. / 8, -1. / 24};
    static constexpr double DM_L[4][5] = {{-2., 3., -1., 0., 0.},
                                          {-1., 1., 0., 0., 0.},
                                          {1. / 24., -9. / 8., 9. / 8., -1. / 24., 0.},
                                          {-1. / 71., 6. / 71., -83. / 71., 81. / 71., -3. / 71.}};
    static constexpr double DM_R[4][5] = {{3. / 71., -81. / 71., 83. / 71., -6. / 71., 1. / 71.},
                                          {0., 1. / 24., -9. / 8., 9. / 8., -1. / 24.},
                                          {0., 0., 0., -1., 1.},
                                          {0., 0., 1., -3., 2.}};
    static constexpr double DN_L[3][5] = {{-79. / 78., 27. / 26., -1. / 26., 1. / 78., 0.},
                                          {2. / 21., -9. / 7., 9. / 7., -2. / 21., 0.},
                                          {1. / 75., 0., -27. / 25., 83. / 75., -1. / 25.}};
    static constexpr double DN_R[3][5] = {{1. / 25., -83. / 75., 27. / 25., 0., -1. / 75.},
                                          {0., 2. / 21., -9. / 7., 9. / 7., -2. / 21.},
                                          {0., -1. / 78., 1. / 26., -27. / 26., 79. / 78.}};
    static constexpr double A_N_L[4] = {7. / 18., 9. / 8., 1., 71. / 72.};
    static constexpr double A_N_R[4] = {71. / 72., 1., 9. / 8., 7. / 18.};
    static constexpr double A_M_L[3] = {13. / 12., 7. / 8., 25. / 24.};
    static constexpr double A_M_R[3] = {25. / 24., 7. / 8., 13. / 12.};
    static constexpr double P_N = 1.;                      // projection of an N-type neighbour
    static constexpr double P_M_L[3] = {15. / 8., -5. / 4., 3. / 8.};
    static constexpr double P_M_R[3] = {3. / 8., -5. / 4., 15. / 8.};
};

// Scaled operators in the compute type C. Shared by all four grids: a grid's operators depend
// only on its x type (N: DM closures, M: DN closures) and on dt/dx.
template <class C>
struct Ops {
    C st[4];            // interior stencil scaled
    C dmL[4][5], dmR[4][5];
    C dnL[3][5], dnR[3][5];
    C satNL, satNR;     // eta * A_inv_projection of the N-type-x velocity grid (NM), rows 0 / Mx
    C satML[3], satMR[3];   // the same for the M-type-x velocity grid (MN), rows 0..2 / Mx-3..Mx-1
    C pN;               // projection of NN onto the boundary (MN's SAT)
    C pML[3], pMR[3];   // projection of MM sxx onto the boundary (NM's SAT)
};

template <class C>
inline C scale_by_dt(C v, double dt) { return (C)((double)v * (double)(C)dt); }

// single_core: the periodic acoustic tree's stencil rounding
template <class C>
inline Ops<C> make_ops(double dx, double dt, bool single_core)
{
    using S = SbpTables;
    Ops<C> o{};
    for (int k = 0; k < 4; k++)
        o.st[k] = single_core ? (C)(S::stencil[k] * dt / dx) : (C)(S::stencil[k] * (dt / dx));
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 5; j++) {
            o.dmL[i][j] = (C)(S::DM_L[i][j] * (dt / dx));
            o.dmR[i][j] = (C)(S::DM_R[i][j] * (dt / dx));
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 5; j++) {
            o.dnL[i][j] = (C)(S::DN_L[i][j] * (dt / dx));
            o.dnR[i][j] = (C)(S::DN_R[i][j] * (dt / dx));
        }
    // eta = +1 on the left end, -1 on the right (grid_drvt.tpp:633,638); the product eta * A
    // is exact in any type, so it is folded here
    o.satNL = scale_by_dt<C>((C)(S::P_N / (dx * S::A_N_L[0])), dt);
    o.satNR = -scale_by_dt<C>((C)(S::P_N / (dx * S::A_N_R[3])), dt);
    for (int i = 0; i < 3; i++) {
        o.satML[i] = scale_by_dt<C>((C)(S::P_M_L[i] / (dx * S::A_M_L[i])), dt);
        o.satMR[i] = -scale_by_dt<C>((C)(S::P_M_R[i] / (dx * S::A_M_R[i])), dt);
    }
    o.pN = (C)S::P_N;
    for (int i = 0; i < 3; i++) {
        o.pML[i] = (C)S::P_M_L[i];
        o.pMR[i] = (C)S::P_M_R[i];
    }
    return o;
}

}  // namespace tw

// Set-up and bookkeeping kernels: FP64 material interpolation, stepping coefficients and energy
// weights, the discrete energy reductions and the receiver gather.
#include <cstring>
#include "kernels.h"

namespace tw {

// ---------------------------------------------------------------- material (FP64, exact order)
__global__ void k_model_derive(const double *rho, const double *vp, const double *vs, long n, double *lam,
                               double *m2, double *mu)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double r = rho[i], p = vp[i], s = vs[i];
        const double two_mu = mul(mul(mul(2.0, r), s), s);           // 2 * rho * vs * vs
        m2[i] = two_mu;
        lam[i] = sub(mul(mul(r, p), p), two_mu);                      // rho * vp * vp - 2mu
        mu[i] = mul(mul(r, s), s);                                    // rho * vs * vs
    }
}

void launch_model_derive(const double *rho, const double *vp, const double *vs, long n, double *lam,
                         double *m2, double *mu, cudaStream_t st)
{
    const int blocks = (int)((n + 255) / 256 < 65535 ? (n + 255) / 256 : 65535);
    k_model_derive<<<blocks, 256, 0, st>>>(rho, vp, vs, n, lam, m2, mu);
}

// interpolate_forward_parameter (grid_parameter.cpp:13-57): the location of grid point (ix, iy)
// in units of the model spacing is num/den; its integer part indexes the padded model, the
// remainder (computed in double) weights the four corners.
__global__ void k_interp(int rows, int cols, int txN, int tyN, int num_dx, int den_dx, int num_dxM, int den_dxM,
                         long Nxp, long Nyp, const double *in, double *out, int *err, int row_off)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int il = blockIdx.y * blockDim.y + threadIdx.y;
    if (iy >= cols || il >= rows) return;
    const int ix = il + row_off;   // global row (a slab's local row il)
    long nx, dxl, ny, dyl;
    if (txN) { nx = (long)ix * num_dx; dxl = den_dx; } else { nx = (2L * ix + 1) * num_dx; dxl = 2L * den_dx; }
    if (tyN) { ny = (long)iy * num_dx; dyl = den_dx; } else { ny = (2L * iy + 1) * num_dx; dyl = 2L * den_dx; }
    const long ixM = (nx * den_dxM) / (dxl * num_dxM);
    const long iyM = (ny * den_dxM) / (dyl * num_dxM);
    if (ixM < 0 || ixM + 1 > Nxp || iyM < 0 || iyM + 1 > Nyp) { atomicOr(err, 1); return; }
    const double xi = sub(__ddiv_rn((double)(nx * den_dxM), (double)(dxl * num_dxM)), (double)ixM);
    const double eta = sub(__ddiv_rn((double)(ny * den_dxM), (double)(dyl * num_dxM)), (double)iyM);
    const long PS = Nyp + 1;
    const double a = sub(1.0, xi), b = sub(1.0, eta);
    double v = mul(mul(a, b), in[ixM * PS + iyM]);
    v = add(v, mul(mul(a, eta), in[ixM * PS + iyM + 1]));
    v = add(v, mul(mul(xi, b), in[(ixM + 1) * PS + iyM]));
    v = add(v, mul(mul(xi, eta), in[(ixM + 1) * PS + iyM + 1]));
    out[(long)il * cols + iy] = v;
}

void launch_interp(int rows, int cols, int txN, int tyN, int num_dx, int den_dx, int num_dxM, int den_dxM,
                   long Nx_prmt, long Ny_prmt, const double *in, double *out, int *err, cudaStream_t st, int row_off)
{
    const dim3 b(32, 8), g((cols + 31) / 32, (rows + 7) / 8);
    k_interp<<<g, b, 0, st>>>(rows, cols, txN, tyN, num_dx, den_dx, num_dxM, den_dxM, Nx_prmt, Ny_prmt, in, out, err,
                              row_off);
}

// x factor of the energy norm for row ix of a grid with `rows` rows (adjust_parameters_energy_periodic,
// grid_energy.cpp:69-119): A_diag * dx rounded to the storage type on the SAT boundary rows (the
// host precomputes them into nxN / nxM), dx inside
__device__ __forceinline__ double norm_x(const MaterialArgs &m, int txN, int rows_local, int il)
{
    // a slab's rows are global rows il + row_off of a grid of Mx_glob cells
    (void)rows_local;
    const int ix = il + m.row_off, rows = m.Mx_glob + (txN ? 1 : 0);
    if (txN) {
        if (ix < 4) return m.nxN[ix];
        if (ix >= rows - 4) return m.nxN[4 + ix - (rows - 4)];
    } else {
        if (ix < 3) return m.nxM[ix];
        if (ix >= rows - 3) return m.nxM[3 + ix - (rows - 3)];
    }
    return m.dx;
}

// a stepping coefficient as stored: the compute type, or FP16 (range checked: the medium must
// lie in the normal FP16 range, else bit 2 of *err)
template <class C, class K>
__device__ __forceinline__ K store_coef(C v, int *err)
{
    if constexpr (sizeof(K) == 2) {
        const float a = fabsf((float)v);
        if (a > 65504.f || (a != 0.f && a < 6.103515625e-05f)) atomicOr(err, 2);
        return __float2half_rn((float)v);
    } else {
        return v;
    }
}
template <class K>
__device__ __forceinline__ double kval(K v) { return (double)to_c<float>(v); }
template <>
__device__ __forceinline__ double kval<double>(double v) { return v; }

template <class C, class K>
__global__ void k_material_finalize(MaterialArgs m)
{
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    const double dx = m.dx;
    const bool elastic = m.physics == 0;
    K **coef = (K **)m.coef;
    // y factor of the norm (grid_energy.cpp:123-152): dx everywhere, then 1 on the first and 0 on
    // the last (duplicate) point of an N-type-y grid; with free y ends the x rule along y
    // (A_diag * dx, storage-rounded, on the end columns by the grid's y type)
    auto y_factor = [&](int g, double w) {
        if (m.sat_y) {
            const int n = m.cols[g];
            double f = dx;
            if (n == m.My + 1) {
                if (iy < 4) f = m.nxN[iy];
                else if (iy >= n - 4) f = m.nxN[4 + iy - (n - 4)];
            } else {
                if (iy < 3) f = m.nxM[iy];
                else if (iy >= n - 3) f = m.nxM[3 + iy - (n - 3)];
            }
            return mul(w, f);
        }
        w = mul(w, dx);
        if (m.cols[g] == m.My + 1 && iy == m.My) w = mul(w, 0.);
        return w;
    };
    // single-core weights (namespaces.hpp:734-776): dx*dx/2, halved on the end points of an N direction
    auto sc_weight = [&](int g) {
        double w = mul(dx, dx) / 2.;
        if (m.cols[g] == m.My + 1 && (iy == 0 || iy == m.My)) w = w / 2.;
        if (m.rows[g] == m.Mx + 1 && (ix == 0 || ix == m.Mx)) w = w / 2.;
        return w;
    };
    // NN (elastic only): mu, weight 1/mu
    if (elastic && ix < m.rows[F_NN] && iy < m.cols[F_NN]) {
        const long i = (long)ix * m.cols[F_NN] + iy, o = (long)ix * m.pitch + iy;
        const K mu = store_coef<C, K>((C)m.mat[F_NN][i], m.err);
        coef[F_NN][o] = mu;
        double w = __ddiv_rn(1., kval(mu));
        w = mul(w, norm_x(m, 1, m.rows[F_NN], ix));
        m.w[F_NN][o] = y_factor(F_NN, w);
    }
    // velocity grids: 1/rho from the FP64 density (make_density_reciprocal), weight rho
    for (int g = F_MN; g <= F_NM; g++) {
        if (ix >= m.rows[g] || iy >= m.cols[g]) continue;
        const long i = (long)ix * m.cols[g] + iy, o = (long)ix * m.pitch + iy;
        const double rho = m.mat[g][i];
        coef[g][o] = store_coef<C, K>((C)__ddiv_rn(1., rho), m.err);
        if (m.periodic) {
            m.w[g][o] = sc_weight(g);
        } else {
            double w = sizeof(K) == 2 ? kval(store_coef<C, K>((C)rho, m.err)) : (double)(C)rho;
            w = mul(w, norm_x(m, g == F_NM, m.rows[g], ix));
            m.w[g][o] = y_factor(g, w);
        }
    }
    if (ix < m.rows[F_MM0] && iy < m.cols[F_MM0]) {
        const long i = (long)ix * m.cols[F_MM0] + iy, o = (long)ix * m.pitch + iy;
        const K lam = store_coef<C, K>((C)m.mat[F_MM0][i], m.err);
        coef[F_MM0][o] = lam;
        const double fx = m.periodic ? 0. : norm_x(m, 0, m.rows[F_MM0], ix);
        if (elastic) {
            const K m2 = store_coef<C, K>((C)m.mat[F_MM1][i], m.err);
            coef[F_MM1][o] = m2;
            const double l = kval(lam), t = kval(m2);
            const double den = mul(t, add(mul(2., l), t));
            const double w1 = __ddiv_rn(add(l, t), den);
            const double w2 = -__ddiv_rn(mul(l, 2.), den);
            m.w[F_MM0][o] = y_factor(F_MM0, mul(w1, fx));
            m.w[F_MM1][o] = y_factor(F_MM1, mul(w2, fx));
        } else if (m.periodic) {
            m.w[F_MM0][o] = sc_weight(F_MM0);
        } else {
            // acoustic free surface: the mu -> 0 limit of the elastic weights, (2 P1 + P2) -> 1/kappa
            m.w[F_MM0][o] = y_factor(F_MM0, mul(__ddiv_rn(1., kval(lam)), fx));
        }
    }
}

template <class C, class K>
void launch_material_finalize(const MaterialArgs &m, cudaStream_t st)
{
    const dim3 b(32, 8), g((m.My + 1 + 31) / 32, (m.Mx + 1 + 7) / 8);
    k_material_finalize<C, K><<<g, b, 0, st>>>(m);
}
template void launch_material_finalize<double, double>(const MaterialArgs &, cudaStream_t);
template void launch_material_finalize<float, float>(const MaterialArgs &, cudaStream_t);
template void launch_material_finalize<float, __half>(const MaterialArgs &, cudaStream_t);

// ---------------------------------------------------------------- 16-bit fixed-point coefficients
// (coef_fp16 = 2) Each coefficient array is stored as codes k in [0, 65535] on an affine map
// c = lo + step * k, lo its smallest value, step its range / 65535; every part of the step uses the
// decoded FP32 value fl(lo + fl(step * k)), which replaces the array's FP32 coefficient.

// an order-preserving unsigned image of a float (and back), for min / max by integer atomics
__device__ __forceinline__ unsigned f2ord(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
static float ord2f(unsigned u)
{
    u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

__global__ void k_minmax(const float *a, int rows, int cols, long pitch, unsigned *mm)
{
    unsigned lo = 0xffffffffu, hi = 0u;
    const long n = (long)rows * cols;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const unsigned o = f2ord(a[(i / cols) * pitch + i % cols]);
        lo = o < lo ? o : lo;
        hi = o > hi ? o : hi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned l2 = __shfl_down_sync(0xffffffffu, lo, o), h2 = __shfl_down_sync(0xffffffffu, hi, o);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, lo);
        atomicMax(mm + 1, hi);
    }
}

__global__ void k_quantize16(float *a, unsigned short *codes, int rows, int cols, long pitch, float lo, float step)
{
    const long n = (long)rows * cols;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long o = (i / cols) * pitch + i % cols;
        float k = step > 0.f ? rintf(__fdiv_rn(__fsub_rn(a[o], lo), step)) : 0.f;
        k = fminf(fmaxf(k, 0.f), 65535.f);
        codes[o] = (unsigned short)k;
        a[o] = __fadd_rn(lo, __fmul_rn(step, k));
    }
}

int quantize_coefficients16(float *coef, unsigned short *codes, int rows, int cols, long pitch, unsigned *d_mm,
                            float *lo, float *step, cudaStream_t st)
{
    const unsigned init[2] = {0xffffffffu, 0u};
    unsigned mm[2];
    if (cudaMemcpyAsync(d_mm, init, sizeof(init), cudaMemcpyHostToDevice, st) != cudaSuccess) return -1;
    k_minmax<<<592, 256, 0, st>>>(coef, rows, cols, pitch, d_mm);
    if (cudaMemcpyAsync(mm, d_mm, sizeof(mm), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return -1;
    const float l = ord2f(mm[0]), h = ord2f(mm[1]);
    if (!(l <= h)) return -1;   // no value, or not a number
    *lo = l;
    *step = (float)(((double)h - (double)l) / 65535.0);
    k_quantize16<<<592, 256, 0, st>>>(coef, codes, rows, cols, pitch, l, *step);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ---------------------------------------------------------------- discrete energy (FP64)
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <class S, class C>
__global__ void __launch_bounds__(256) k_energy(EnergyArgs<S, C> e)
{
    const int it = *e.step;
    if (it >= e.max_steps) return;
    int rmax = 0, cmax = 0;
    for (int t = 0; t < e.nterms; t++) {
        rmax = e.rows[t] > rmax ? e.rows[t] : rmax;
        cmax = e.cols[t] > cmax ? e.cols[t] : cmax;
    }
    const long n = (long)rmax * cmax;
    double acc = 0.;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int ix = (int)(k / cmax), iy = (int)(k - (long)ix * cmax);
        const long o = (long)ix * e.pitch + iy;
        for (int t = 0; t < e.nterms; t++) {
            if (ix >= e.rows[t] || iy >= e.cols[t]) continue;
            if (e.single_core) {   // soln * prmt * soln * weight (cpu_acoustic.cpp:341)
                const C s = to_c<C>(e.a[t][o]);
                acc = add(acc, mul((double)mul(mul(s, e.p[t][o]), s), e.w[t][o]));
            } else {               // (double)S * W * (double)S (grid_energy.cpp:196-210)
                acc = add(acc, mul(mul((double)to_c<C>(e.a[t][o]), e.w[t][o]), (double)to_c<C>(e.b[t][o])));
            }
        }
    }
    __shared__ double part[8];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.;
        acc = warp_sum(acc);
        if (threadIdx.x == 0) atomicAdd(e.out + it, acc * e.scale);
    }
}

template <class S, class C>
void launch_energy(const EnergyArgs<S, C> &e, cudaStream_t st)
{
    // 148 SMs x 4 resident blocks of 256 threads: one wave of a grid-stride reduction
    k_energy<S, C><<<148 * 4, 256, 0, st>>>(e);
}
template void launch_energy<double, double>(const EnergyArgs<double, double> &, cudaStream_t);
template void launch_energy<float, float>(const EnergyArgs<float, float> &, cudaStream_t);

// ---------------------------------------------------------------- receivers + step counter
template <class S>
__device__ __forceinline__ void gather_block(const GatherArgs<S> &g)
{
    const int it = *g.step;
    if (it < g.max_steps) {
        for (int r = threadIdx.x; r < g.n_rcv; r += blockDim.x) {
            const int *q = g.rcv + 4 * r;
            const long o = (long)q[2] * g.pitch + q[3];
            g.traces[(2L * r) * g.max_steps + it] = (double)to_c<double>(g.f[q[0]][o]);
            g.traces[(2L * r + 1) * g.max_steps + it] = q[1] >= 0 ? (double)to_c<double>(g.f[q[1]][o]) : 0.;
        }
    } else if (threadIdx.x == 0) {
        atomicOr(g.flags, FLAG_RECORD_FULL);
    }
    __syncthreads();
    if (threadIdx.x == 0) *g.step = it + 1;
}

template <class S>
__global__ void k_gather(GatherArgs<S> g)
{
    pdl_enter();
    gather_block(g);
}

// one block per shot of a batch
template <class S>
__global__ void k_batch_gather(const GatherArgs<S> *g)
{
    gather_block(g[blockIdx.x]);
}

template <class S>
void launch_gather(const GatherArgs<S> &g, cudaStream_t st)
{
    launch_pdl(k_gather<S>, dim3(1), dim3(256), 0, st, g);
}
template void launch_gather<double>(const GatherArgs<double> &, cudaStream_t);
template void launch_gather<float>(const GatherArgs<float> &, cudaStream_t);

template <class S>
void launch_batch_gather(const GatherArgs<S> *g, int n_shots, cudaStream_t st)
{
    k_batch_gather<S><<<n_shots, 128, 0, st>>>(g);
}
template void launch_batch_gather<double>(const GatherArgs<double> *, int, cudaStream_t);
template void launch_batch_gather<float>(const GatherArgs<float> *, int, cudaStream_t);

}  // namespace tw

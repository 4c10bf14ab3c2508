// tw_material_map_noalloc: the material interpolation of tw_set_material_model for callers that
// must not allocate device memory.
//
// Who needs it: a host application whose device memory is reserved up front by another
// allocator (for example a PyTorch process whose caching allocator already holds the GPU, or a
// serving process that fixes its memory budget at start-up) and that re-maps the medium
// repeatedly, as a full-waveform inversion loop does every iteration. tw_set_material_model
// allocates a temporary buffer for the derived model quantities on every call; this variant keeps
// that scratch in one file-scope device array instead and allocates nothing.
//
// The scratch (lambda, 2mu and mu on the padded model, TW_NOALLOC_MAX_MODEL_POINTS doubles each,
// 12 MiB) is part of the library image: every GPU that loads the library holds it until the
// process exits. Every call shares it and it keeps the last call's contents, so calls that
// overlap on the GPU (from two streams or two host threads at once) race; calls from one thread
// are ordered because each call waits for its own stream before returning.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/twave.h"
#include "kernels.h"

namespace {

constexpr long kMaxPoints = TW_NOALLOC_MAX_MODEL_POINTS;
constexpr int kMaxDevices = 64;

// lambda | 2mu | mu of the padded model, each kMaxPoints long
static __device__ __align__(256) double g_model_scratch[3 * kMaxPoints];
// out-of-bounds flag of the interpolation; cleared by every call
static __device__ __align__(256) int g_model_flag[1];

struct DeviceScratch {
    double *model = nullptr;
    int *flag = nullptr;
};

std::mutex g_mutex;
DeviceScratch g_scratch[kMaxDevices];

// Device addresses of the static scratch for the current device. In host code the symbols are
// host-side stand-ins, not device addresses; cudaGetSymbolAddress, called once per device with
// that device current, gives the addresses the kernels are passed.
int scratch_for_current_device(DeviceScratch *out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TW_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceScratch &d = g_scratch[dev];
    if (!d.model) {
        double *model = nullptr;
        int *flag = nullptr;
        if (cudaGetSymbolAddress((void **)&model, g_model_scratch) != cudaSuccess) return TW_ERR_CUDA;
        if (cudaGetSymbolAddress((void **)&flag, g_model_flag) != cudaSuccess) return TW_ERR_CUDA;
        d.model = model;
        d.flag = flag;
    }
    *out = d;
    return TW_OK;
}

}  // namespace

extern "C" int tw_material_map_noalloc(const double *d_rho, const double *d_vp, const double *d_vs, long Mx_prmt,
                                       long My_prmt, int num_dxM, int den_dxM, long Mx, long My, int num_dx,
                                       int den_dx, double *d_NN_mu, double *d_MN_rho, double *d_NM_rho,
                                       double *d_MM_lambda, double *d_MM_2mu, void *stream)
{
    if (!d_rho || !d_vp || !d_vs || !d_NN_mu || !d_MN_rho || !d_NM_rho || !d_MM_lambda || !d_MM_2mu)
        return TW_ERR_INVALID;
    if (Mx < 1 || My < 1 || Mx_prmt < 1 || My_prmt < 1 || num_dx <= 0 || den_dx <= 0 || num_dxM <= 0 || den_dxM <= 0)
        return TW_ERR_INVALID;
    if (Mx > (1L << 30) || My > (1L << 30) || Mx_prmt > (1L << 30) || My_prmt > (1L << 30)) return TW_ERR_INVALID;
    // the model must span the simulation region (input_processing.cpp:203-211)
    if (Mx_prmt * num_dxM * (long)den_dx != Mx * (long)num_dx * den_dxM ||
        My_prmt * num_dxM * (long)den_dx != My * (long)num_dx * den_dxM)
        return TW_ERR_INVALID;
    const long Nxp = Mx_prmt + 1, Nyp = My_prmt + 1, P = (Nxp + 1) * (Nyp + 1);
    if (P > kMaxPoints) return TW_ERR_TOO_LARGE;

    DeviceScratch sc;
    const int rc = scratch_for_current_device(&sc);
    if (rc != TW_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    double *lam = sc.model, *m2 = sc.model + kMaxPoints, *mu = sc.model + 2 * kMaxPoints;
    if (cudaMemsetAsync(sc.flag, 0, sizeof(int), st) != cudaSuccess) return TW_ERR_CUDA;
    tw::launch_model_derive(d_rho, d_vp, d_vs, P, lam, m2, mu, st);
    const int mx = (int)Mx, my = (int)My;
    tw::launch_interp(mx + 1, my + 1, 1, 1, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, mu, d_NN_mu, sc.flag, st);
    tw::launch_interp(mx, my + 1, 0, 1, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, d_rho, d_MN_rho, sc.flag, st);
    tw::launch_interp(mx + 1, my, 1, 0, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, d_rho, d_NM_rho, sc.flag, st);
    tw::launch_interp(mx, my, 0, 0, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, lam, d_MM_lambda, sc.flag, st);
    tw::launch_interp(mx, my, 0, 0, num_dx, den_dx, num_dxM, den_dxM, Nxp, Nyp, m2, d_MM_2mu, sc.flag, st);
    if (cudaGetLastError() != cudaSuccess) return TW_ERR_CUDA;
    int flag = 0;
    if (cudaMemcpyAsync(&flag, sc.flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return TW_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return TW_ERR_CUDA;
    return flag ? TW_ERR_MODEL_BOUNDS : TW_OK;
}

// Device arithmetic that rounds every operation on its own (no FMA contraction), so that the
// FP64 and FP32 steppers reproduce the reference CPU solver's results bit for bit; the stepper
// is bound by HBM bandwidth, so the extra instructions are free.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace tw {

__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }

// storage <-> compute conversions
template <class C, class S> __device__ __forceinline__ C to_c(S v) { return (C)v; }
template <> __device__ __forceinline__ float to_c<float, __nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_c<float, __half>(__half v) { return __half2float(v); }

template <class S, class C> __device__ __forceinline__ S to_s(C v) { return (S)v; }
template <> __device__ __forceinline__ float to_s<float, double>(double v) { return __double2float_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_s<__nv_bfloat16, float>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half to_s<__half, float>(float v) { return __float2half_rn(v); }

__device__ __forceinline__ bool finite(float v) { return isfinite(v); }
__device__ __forceinline__ bool finite(double v) { return isfinite(v); }

// one time update of a field value s with right-hand side r and compensation c, following
// grid_update.tpp:1-127 (codes of enum tw_cpst). keep_r: the code keeps its residual in R;
// keep_c: in the separate C array. split (code 7, 16-bit storage only): every value is stored
// as a pair hi + lo of the storage type, lo = the rounding error of hi, and every read takes
// their sum in the compute type; the update itself is a plain s + r.
template <int CPST> struct Cpst {
    static constexpr bool keep_r = (CPST == 2 || CPST == 4 || CPST == 6);
    static constexpr bool keep_c = (CPST == 1 || CPST == 3 || CPST == 5);
    static constexpr bool split = (CPST == 7);
    static constexpr bool any = keep_r || keep_c || split;
};

template <int CPST, class C>
__device__ __forceinline__ void time_update(C &s, C &r, C &c)
{
    if constexpr (CPST == 0 || CPST == 7) {
        s = add(s, r);
    } else if constexpr (CPST == 1 || CPST == 3) {   // update_3C / update_3C_fast2sum
        const C y = add(r, c);
        const C t = add(s, y);
        const C z = sub(t, s);
        c = sub(y, z);
        s = t;
    } else if constexpr (CPST == 2 || CPST == 4) {   // update_3R / update_3R_fast2sum
        const C t = add(s, r);
        const C z = sub(t, s);
        r = sub(r, z);
        s = t;
    } else {                                         // update_6C_slow2sum / update_6R_slow2sum
        const C b = (CPST == 5) ? add(r, c) : r;
        const C t = add(s, b);
        const C pa = sub(t, b);
        const C pb = sub(t, pa);
        const C da = sub(s, pa);
        const C db = sub(b, pb);
        s = t;
        if constexpr (CPST == 5) c = add(da, db); else r = add(da, db);
    }
}

// a new value as the storage keeps it: rounded to S (a pair hi + lo under the split code);
// identity when storage and compute types agree
template <class S, class C, int CPST>
__device__ __forceinline__ C quant(C v)
{
    if constexpr (sizeof(S) == sizeof(C)) {
        return v;
    } else {
        const C hi = to_c<C>(to_s<S>(v));
        if constexpr (Cpst<CPST>::split) return add(hi, to_c<C>(to_s<S>(sub(v, hi))));
        return hi;
    }
}

}  // namespace tw

// Complex helpers for the FP64 (double2) and FP32 (float2) paths.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace csipm {

template <typename T> struct cpx;
template <> struct cpx<double> { using t = double2; };
template <> struct cpx<float> { using t = float2; };
template <typename T> using cplx_t = typename cpx<T>::t;

__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
// multiply by +i / -i
template <typename C> __host__ __device__ __forceinline__ C cmul_i(C a) { return mk(-a.y, a.x); }
template <typename C> __host__ __device__ __forceinline__ C cmul_mi(C a) { return mk(a.y, -a.x); }
template <typename C, typename T> __host__ __device__ __forceinline__ C cscale(C a, T s) { return mk(a.x * s, a.y * s); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// twiddle multiply: forward uses w, inverse uses conj(w)
template <bool INV, typename C> __device__ __forceinline__ C twmul(C a, C w) {
    return INV ? cmulc(a, w) : cmul(a, w);
}

}  // namespace csipm

// Small device helpers shared by the kernels: complex arithmetic on
// double2/float2, precision traits, error macros.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace chfsi {

template <typename R> struct CplxOf;
template <> struct CplxOf<double> { using type = double2; };
template <> struct CplxOf<float> { using type = float2; };

__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }

template <typename C> struct RealOf;
template <> struct RealOf<double2> { using type = double; };
template <> struct RealOf<float2> { using type = float; };

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) {
    return mk(a.x * s, a.y * s);
}
// multiply by +i (sign > 0) or -i (sign < 0)
template <int SIGN, typename C> __host__ __device__ __forceinline__ C cmul_i(C a) {
    return SIGN > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}

__device__ __forceinline__ double2 to_c(double2 a, double2) { return a; }
__device__ __forceinline__ float2 to_c(double2 a, float2) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_c(float2 a, double2) { return make_double2(a.x, a.y); }
__device__ __forceinline__ float2 to_c(float2 a, float2) { return a; }

}  // namespace chfsi

#define CHFSI_CUDA_TRY(expr)                                                         \
    do {                                                                             \
        cudaError_t _e = (expr);                                                     \
        if (_e != cudaSuccess) return ::chfsi::cuda_fail(_e, #expr, __FILE__, __LINE__); \
    } while (0)

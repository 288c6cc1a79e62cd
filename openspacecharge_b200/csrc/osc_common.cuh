// osc_common.cuh -- shared types and helpers of the B200 space-charge library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace osc {

// Complex vector types: float2 / double2 keep 8- and 16-byte aligned loads.
template <typename T> struct VecT;
template <> struct VecT<float> { typedef float2 type; typedef float4 type4; };
template <> struct VecT<double> { typedef double2 type; typedef double4 type4; };
template <typename T> using cplx = typename VecT<T>::type;
template <typename T> using vec4 = typename VecT<T>::type4;

template <typename T> __host__ __device__ __forceinline__ cplx<T> mk(T re, T im) {
    cplx<T> r;
    r.x = re;
    r.y = im;
    return r;
}
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) {
    a.x += b.x;
    a.y += b.y;
    return a;
}
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) {
    a.x -= b.x;
    a.y -= b.y;
    return a;
}
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
// a * conj(b)
template <typename V> __host__ __device__ __forceinline__ V cmulc(V a, V b) {
    V r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.y * b.x - a.x * b.y;
    return r;
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) {
    a.y = -a.y;
    return a;
}
template <typename V, typename S> __host__ __device__ __forceinline__ V cscale(V a, S s) {
    a.x *= s;
    a.y *= s;
    return a;
}
// multiply by s*i (s = +1 or -1)
template <typename V> __host__ __device__ __forceinline__ V cmul_si(V a, int s) {
    V r;
    if (s > 0) {
        r.x = -a.y;
        r.y = a.x;
    } else {
        r.x = a.y;
        r.y = -a.x;
    }
    return r;
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace osc

// Status codes mirror include/opensc_gpu.h.
#define OSC_OK 0
#define OSC_E_INVALID 1
#define OSC_E_BOUNDS 2
#define OSC_E_FFT_SIZE 3
#define OSC_E_ALLOC 4
#define OSC_E_CUDA 5
#define OSC_E_TIMEOUT 6
#define OSC_E_NAN 7
#define OSC_E_NOCHARGE 8
#define OSC_E_UNSUPPORTED 9
#define OSC_E_STATE 10

// Common device/host helpers for libcpstep (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include "../../include/cpstep.h"

#define CPSTEP_CUDA_TRY(expr)                                                   \
  do {                                                                          \
    cudaError_t _e = (expr);                                                    \
    if (_e != cudaSuccess) {                                                    \
      cpstep_set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,              \
                       cudaGetErrorString(_e));                                 \
      return CPSTEP_ERR_CUDA;                                                   \
    }                                                                           \
  } while (0)

extern unsigned long long g_cpstep_launches;  // kernels launched by the library

#define CPSTEP_LAUNCH_CHECK()                                                   \
  do {                                                                          \
    __atomic_add_fetch(&g_cpstep_launches, 1ull, __ATOMIC_RELAXED);             \
    cudaError_t _e = cudaGetLastError();                                        \
    if (_e != cudaSuccess) {                                                    \
      cpstep_set_error("%s:%d: launch: %s", __FILE__, __LINE__,                 \
                       cudaGetErrorString(_e));                                 \
      return CPSTEP_ERR_CUDA;                                                   \
    }                                                                           \
  } while (0)

void cpstep_set_error(const char* fmt, ...);

template <typename T>
struct cplx {
  T x, y;
};

template <typename T>
__host__ __device__ __forceinline__ cplx<T> mk(T a, T b) {
  cplx<T> c;
  c.x = a;
  c.y = b;
  return c;
}
// FP32 complex arithmetic on sm_100 runs on the packed two-lane FP32 units
// (__fadd2_rn, __fmul2_rn, __ffma2_rn: per component the same IEEE operation
// as the scalar one), half the instructions of the scalar form.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
#define CPLX_F32X2 1
__device__ __forceinline__ float2 f2(cplx<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ cplx<float> c2(float2 a) { return mk<float>(a.x, a.y); }
#endif

template <typename T>
__host__ __device__ __forceinline__ cplx<T> operator+(cplx<T> a, cplx<T> b) {
#ifdef CPLX_F32X2
  if constexpr (sizeof(T) == 4) return c2(__fadd2_rn(f2(a), f2(b)));
#endif
  return mk<T>(a.x + b.x, a.y + b.y);
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> operator-(cplx<T> a, cplx<T> b) {
#ifdef CPLX_F32X2
  if constexpr (sizeof(T) == 4) return c2(__fadd2_rn(f2(a), make_float2(-b.x, -b.y)));
#endif
  return mk<T>(a.x - b.x, a.y - b.y);
}
// (a.x b.x - a.y b.y, a.x b.y + a.y b.x): packed, the second product of each
// component first and the first fused into it
template <typename T>
__host__ __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
#ifdef CPLX_F32X2_MUL
  if constexpr (sizeof(T) == 4)
    return c2(__ffma2_rn(make_float2(a.x, a.x), make_float2(b.x, b.y),
                         __fmul2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x))));
#endif
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b) = (a.x b.x + a.y b.y, a.y b.x - a.x b.y)
template <typename T>
__host__ __device__ __forceinline__ cplx<T> cmulc(cplx<T> a, cplx<T> b) {
#ifdef CPLX_F32X2_MUL
  if constexpr (sizeof(T) == 4)
    return c2(__ffma2_rn(make_float2(a.y, a.y), make_float2(b.y, b.x),
                         __fmul2_rn(make_float2(a.x, a.x), make_float2(b.x, -b.y))));
#endif
  return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> cscale(cplx<T> a, T s) {
#ifdef CPLX_F32X2_MUL
  if constexpr (sizeof(T) == 4) return c2(__fmul2_rn(f2(a), make_float2(s, s)));
#endif
  return mk<T>(a.x * s, a.y * s);
}
template <typename T>
__host__ __device__ __forceinline__ cplx<T> conjc(cplx<T> a) {
  return mk<T>(a.x, -a.y);
}
// multiply by -i (sign<0) or +i (sign>0)
template <typename T>
__host__ __device__ __forceinline__ cplx<T> mul_i(cplx<T> a, bool plus) {
  return plus ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

__host__ __device__ __forceinline__ int cdiv(int a, int b) { return (a + b - 1) / b; }

// Deterministic block reduction of a double (blockDim.x a multiple of 32, <= 1024).
__device__ __forceinline__ double block_sum(double v, double* sbuf) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sbuf[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    int nw = blockDim.x >> 5;
    r = (l < nw) ? sbuf[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

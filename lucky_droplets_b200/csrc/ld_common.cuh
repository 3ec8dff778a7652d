// Common device helpers for the lucky-droplets B200 kernels: complex arithmetic on float2 /
// double2, status codes, launch checks.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/ld.h"

namespace ld {

template <typename T> struct CT;
template <> struct CT<float>  { using type = float2; };
template <> struct CT<double> { using type = double2; };
template <typename T> using cplx = typename CT<T>::type;

__device__ __forceinline__ float2 cmk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 cmk(double a, double b) { return make_double2(a, b); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { a.x *= s; a.y *= s; return a; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}
// i * a
template <typename C> __device__ __forceinline__ C cmuli(C a) { C r; r.x = -a.y; r.y = a.x; return r; }
template <typename C> __device__ __forceinline__ C czero() { C r; r.x = 0; r.y = 0; return r; }

template <typename T> __device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

}  // namespace ld

#define LD_CUDA_CHECK(expr)                                   \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) { ld_set_last_error(_e); return LD_ERR_CUDA; } \
  } while (0)

#define LD_LAUNCH_CHECK() LD_CUDA_CHECK(cudaGetLastError())

extern "C++" void ld_set_last_error(cudaError_t e);

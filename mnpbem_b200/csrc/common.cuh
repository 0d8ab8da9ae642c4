// Shared helpers for the bem200 CUDA library: status handling, complex
// arithmetic on double2 / float2, launch checks.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/bem200.h"

namespace bem200 {

// Thread-local last-error message, read through bem200_last_error().
void set_error(const char* fmt, ...);
const char* get_error();

#define BEM_CUDA_CHECK(expr)                                                      \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      ::bem200::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr,              \
                          cudaGetErrorString(_e));                                \
      return BEM200_ERR_CUDA;                                                     \
    }                                                                             \
  } while (0)

// Kernel launches are counted (bem200_launch_count) so that callers can report
// how many device kernels a call enqueued.  Launches recorded into a CUDA
// graph by this thread are not counted (count_suspend); a replay counts the
// graph's kernels (count_launches).
void count_launch();
void count_launches(unsigned long long n);
void count_suspend(bool on);
#define BEM_LAUNCH_CHECK()          \
  do {                              \
    ::bem200::count_launch();       \
    BEM_CUDA_CHECK(cudaGetLastError()); \
  } while (0)

#define BEM_REQUIRE(cond, code, ...)                                              \
  do {                                                                            \
    if (!(cond)) {                                                                \
      ::bem200::set_error(__VA_ARGS__);                                           \
      return (code);                                                              \
    }                                                                             \
  } while (0)

// ---------------------------------------------------------------- complex
template <typename T> struct cplx_traits;
template <> struct cplx_traits<double2> { using real = double; };
template <> struct cplx_traits<float2> { using real = float; };

__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) {
  return make_float2(a.x * s, a.y * s);
}
__host__ __device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
// a / b (Smith's algorithm keeps the intermediate range safe)
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, den = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  } else {
    double r = b.x / b.y, den = b.y + b.x * r;
    return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
  }
}
__host__ __device__ __forceinline__ float2 cdiv(float2 a, float2 b) {
  if (fabsf(b.x) >= fabsf(b.y)) {
    float r = b.y / b.x, den = b.x + b.y * r;
    return make_float2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  } else {
    float r = b.x / b.y, den = b.y + b.x * r;
    return make_float2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
  }
}

template <typename C> __host__ __device__ __forceinline__ C czero();
template <> __host__ __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __host__ __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }

template <typename C> __host__ __device__ __forceinline__ C cmake(double re, double im);
template <> __host__ __device__ __forceinline__ double2 cmake<double2>(double re, double im) {
  return make_double2(re, im);
}
template <> __host__ __device__ __forceinline__ float2 cmake<float2>(double re, double im) {
  return make_float2((float)re, (float)im);
}

__host__ __device__ inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Kernel attributes are set once per kernel (the call is a host-side round
// trip that should not sit in front of every launch).  Entries are keyed by
// the kernel's address; a larger shared-memory request raises the limit again.
cudaError_t set_kernel_attrs(const void* kern, int smem_bytes, bool nonportable_cluster);

template <typename K>
inline cudaError_t set_kernel_attrs_once(K kern, int smem_bytes, bool nonportable_cluster) {
  return set_kernel_attrs(reinterpret_cast<const void*>(kern), smem_bytes, nonportable_cluster);
}

}  // namespace bem200

// Krylov-subspace kernels of the iterative BEM solver (restarted GMRES on the
// 8 n p packed BEM system, complex128): classical Gram-Schmidt with one
// re-orthogonalisation pass (CGS2) of a new Arnoldi vector against the basis,
// the combination of basis vectors at the end of a cycle, and an axpy.  The
// basis is stored as m vectors of length len, one after the other.
//
// Reference behaviour replaced: scipy.sparse.linalg.gmres driven by
// BEMIter._iter_solve (mnpbem/bem/bem_iter.py:45-101) for BEMRetIter
// (mnpbem/bem/bem_ret_iter.py:1636-1744).
#include "common.cuh"

namespace bem200 {

constexpr int kKryThreads = 256;
constexpr int kDotChunk = 8192;  // vector elements per CTA of the dot kernel

__device__ __forceinline__ double2 cconj_mul(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  T r = 0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (kKryThreads / 32) ? sh[threadIdx.x] : T(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

// h[i] += <V_i, w> for i < nv   (grid: chunks x nv)
__global__ void __launch_bounds__(kKryThreads) dots_kernel(long long len, int nv, const double2* __restrict__ V,
                                                           const double2* __restrict__ w, double* __restrict__ h) {
  __shared__ double shr[kKryThreads / 32], shi[kKryThreads / 32];
  const int i = blockIdx.y;
  const long long c0 = (long long)blockIdx.x * kDotChunk;
  const long long c1 = min(len, c0 + kDotChunk);
  const double2* vi = V + (long long)i * len;
  double re = 0, im = 0;
  for (long long e = c0 + threadIdx.x; e < c1; e += kKryThreads) {
    const double2 p = cconj_mul(vi[e], w[e]);
    re += p.x;
    im += p.y;
  }
  re = block_sum(re, shr);
  im = block_sum(im, shi);
  if (threadIdx.x == 0) {
    atomicAdd(&h[2 * i], re);
    atomicAdd(&h[2 * i + 1], im);
  }
}

// w -= sum_i hpass[i] V_i;  htot[i] += hpass[i]
__global__ void __launch_bounds__(kKryThreads) subtract_kernel(long long len, int nv, const double2* __restrict__ V,
                                                               const double* __restrict__ hpass,
                                                               double2* __restrict__ w) {
  for (long long e = (long long)blockIdx.x * kKryThreads + threadIdx.x; e < len;
       e += (long long)gridDim.x * kKryThreads) {
    double2 acc = w[e];
    for (int i = 0; i < nv; ++i) {
      const double2 h = make_double2(hpass[2 * i], hpass[2 * i + 1]);
      acc = csub(acc, cmul(h, V[(long long)i * len + e]));
    }
    w[e] = acc;
  }
}

// ssq += |w|^2
__global__ void __launch_bounds__(kKryThreads) norm2_kernel(long long len, const double2* __restrict__ w,
                                                            double* __restrict__ ssq) {
  __shared__ double sh[kKryThreads / 32];
  double s = 0;
  for (long long e = (long long)blockIdx.x * kKryThreads + threadIdx.x; e < len;
       e += (long long)gridDim.x * kKryThreads)
    s += cabs2(w[e]);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) atomicAdd(ssq, s);
}

// w *= 1 / sqrt(*ssq)  (left unchanged when the norm is zero)
__global__ void __launch_bounds__(kKryThreads) scale_kernel(long long len, const double* __restrict__ ssq,
                                                            double2* __restrict__ w) {
  const double nrm = sqrt(*ssq);
  if (!(nrm > 0)) return;
  const double s = 1.0 / nrm;
  for (long long e = (long long)blockIdx.x * kKryThreads + threadIdx.x; e < len;
       e += (long long)gridDim.x * kKryThreads)
    w[e] = cscale(w[e], s);
}

// z = sum_i y[i] V_i   (y: device copy of the host coefficients)
__global__ void __launch_bounds__(kKryThreads) combine_kernel(long long len, int nv, const double2* __restrict__ V,
                                                              const double* __restrict__ y, double2* __restrict__ z) {
  for (long long e = (long long)blockIdx.x * kKryThreads + threadIdx.x; e < len;
       e += (long long)gridDim.x * kKryThreads) {
    double2 acc = make_double2(0, 0);
    for (int i = 0; i < nv; ++i) acc = cadd(acc, cmul(make_double2(y[2 * i], y[2 * i + 1]), V[(long long)i * len + e]));
    z[e] = acc;
  }
}

__global__ void __launch_bounds__(kKryThreads) zaxpy_kernel(long long len, double2 a, const double2* __restrict__ x,
                                                            double2* __restrict__ y) {
  for (long long e = (long long)blockIdx.x * kKryThreads + threadIdx.x; e < len;
       e += (long long)gridDim.x * kKryThreads)
    y[e] = cadd(y[e], cmul(a, x[e]));
}

static int stream_grid(long long len) {
  long long g = (len + kKryThreads - 1) / kKryThreads;
  return (int)(g < 148 * 8 ? g : 148 * 8);
}

}  // namespace bem200

using namespace bem200;

extern "C" {

size_t bem200_gmres_orth_workspace_size(int j) { return sizeof(double) * (size_t)(4 * (j + 1) + 2) + 256; }

// Orthogonalise w = V + (j + 1) len (the vector after V_0 .. V_j) against
// V_0 .. V_j by CGS2 (j = -1: no basis yet), normalise it in place, and
// return on the host
// h_host[2 i], h_host[2 i + 1] = <V_i, w> (i <= j) and h_host[2 (j + 1)] = ||w||
// before normalisation.  scratch: bem200_gmres_orth_workspace_size(j) bytes.
// Synchronises the stream once.
int bem200_gmres_orth(int64_t len, int j, void* V, double* h_host, void* scratch, void* stream) {
  BEM_REQUIRE(len > 0 && j >= -1 && V && h_host && scratch, BEM200_ERR_ARG, "gmres_orth: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int nv = j + 1;
  double2* Vb = (double2*)V;
  double2* w = Vb + (long long)nv * len;
  double* hpass = (double*)scratch;     // 2 nv: one pass
  double* htot = hpass + 2 * nv;        // 2 nv: both passes
  double* ssq = htot + 2 * nv;          // 1
  BEM_CUDA_CHECK(cudaMemsetAsync(htot, 0, sizeof(double) * (2 * nv + 1), s));
  const dim3 dgrid((unsigned)((len + kDotChunk - 1) / kDotChunk), (unsigned)(nv > 0 ? nv : 1));
  BEM_REQUIRE(nv <= 65535, BEM200_ERR_ARG, "gmres_orth: basis too large");
  for (int pass = 0; pass < 2 && nv > 0; ++pass) {
    BEM_CUDA_CHECK(cudaMemsetAsync(hpass, 0, sizeof(double) * 2 * nv, s));
    dots_kernel<<<dgrid, kKryThreads, 0, s>>>(len, nv, Vb, w, hpass);
    BEM_LAUNCH_CHECK();
    subtract_kernel<<<stream_grid(len), kKryThreads, 0, s>>>(len, nv, Vb, hpass, w);
    BEM_LAUNCH_CHECK();
    zaxpy_kernel<<<1, kKryThreads, 0, s>>>(nv, make_double2(1.0, 0.0), (const double2*)hpass, (double2*)htot);
    BEM_LAUNCH_CHECK();
  }
  norm2_kernel<<<stream_grid(len), kKryThreads, 0, s>>>(len, w, ssq);
  BEM_LAUNCH_CHECK();
  scale_kernel<<<stream_grid(len), kKryThreads, 0, s>>>(len, ssq, w);
  BEM_LAUNCH_CHECK();
  BEM_CUDA_CHECK(cudaMemcpyAsync(h_host, htot, sizeof(double) * (2 * nv + 1), cudaMemcpyDeviceToHost, s));
  BEM_CUDA_CHECK(cudaStreamSynchronize(s));
  h_host[2 * nv] = sqrt(h_host[2 * nv] > 0 ? h_host[2 * nv] : 0.0);
  return BEM200_OK;
}

// z = sum_{i < m} y_i V_i  with y (complex, 2 m doubles) given on the HOST.
// scratch: 16 m bytes (device copy of y).
int bem200_gmres_combine(int64_t len, int m, const void* V, const double* y_host, void* z, void* scratch,
                         void* stream) {
  BEM_REQUIRE(len > 0 && m > 0 && V && y_host && z && scratch, BEM200_ERR_ARG, "gmres_combine: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  BEM_CUDA_CHECK(cudaMemcpyAsync(scratch, y_host, sizeof(double) * 2 * m, cudaMemcpyHostToDevice, s));
  combine_kernel<<<stream_grid(len), kKryThreads, 0, s>>>(len, m, (const double2*)V, (const double*)scratch,
                                                         (double2*)z);
  BEM_LAUNCH_CHECK();
  // the host array may be reused as soon as this returns
  BEM_CUDA_CHECK(cudaStreamSynchronize(s));
  return BEM200_OK;
}

// y += a x  (complex128; a given on the host as (re, im))
int bem200_zaxpy(int64_t len, const double* a, const void* x, void* y, void* stream) {
  BEM_REQUIRE(len >= 0 && a && (len == 0 || (x && y)), BEM200_ERR_ARG, "zaxpy: bad arguments");
  if (len == 0) return BEM200_OK;
  zaxpy_kernel<<<stream_grid(len), kKryThreads, 0, (cudaStream_t)stream>>>(len, make_double2(a[0], a[1]),
                                                                          (const double2*)x, (double2*)y);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

}  // extern "C"

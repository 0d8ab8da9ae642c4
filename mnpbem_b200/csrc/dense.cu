// Dense complex LU with partial pivoting, triangular solves and GEMM.
//
// Structure (all host-driven, kernels enqueued on one stream):
//   * recursive LU: the leaf panel (width <= kPanelNB) is factored by ONE
//     thread-block cluster that keeps the whole tall panel in distributed
//     shared memory; per column, the pivot search and the row exchange use
//     DSMEM and two cluster barriers.  The rest of the work is TRSM + GEMM.
//   * recursive TRSM with small substitution kernels at the leaves.
//   * GEMM: CUDA-core kernel for complex128 (FP64 FMA) / complex64 (FP32),
//     and the tcgen05 tensor-core path for complex64 (gemm_tc.cu).
// Pivot choice follows LAPACK izamax: largest |re| + |im|, first index on ties.
#include <cooperative_groups.h>

#include <climits>
#include <vector>

#include "dense.cuh"

namespace cg = cooperative_groups;

namespace bem200 {

template <typename C> using R_t = typename cplx_traits<C>::real;

__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ float cabs1(float2 a) { return fabsf(a.x) + fabsf(a.y); }

// ===================================================================== GEMM
// C = alpha A B + beta C; block tile 64 x 64, each thread a 4 x 4 register tile
// (rows ty + 16 i, cols tx + 16 j).
template <typename C, int BK>
__global__ void __launch_bounds__(256) gemm_simt_kernel(int m, int n, int k, C alpha, const C* __restrict__ A,
                                                        long long lda, const C* __restrict__ B, long long ldb,
                                                        C beta, C* __restrict__ Cm, long long ldc) {
  constexpr int BM = 64, BN = 64;
  __shared__ C As[BK][BM + 1];
  __shared__ C Bs[BK][BN];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  C acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = czero<C>();
  for (int k0 = 0; k0 < k; k0 += BK) {
    for (int idx = threadIdx.x; idx < BM * BK; idx += 256) {
      int r = idx / BK, c = idx % BK;
      int gr = m0 + r, gc = k0 + c;
      As[c][r] = (gr < m && gc < k) ? A[(long long)gr * lda + gc] : czero<C>();
    }
    for (int idx = threadIdx.x; idx < BK * BN; idx += 256) {
      int r = idx / BN, c = idx % BN;
      int gr = k0 + r, gc = n0 + c;
      Bs[r][c] = (gr < k && gc < n) ? B[(long long)gr * ldb + gc] : czero<C>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      C a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(a[i].x, b[j].x, acc[i][j].x);
          acc[i][j].x = fma(-a[i].y, b[j].y, acc[i][j].x);
          acc[i][j].y = fma(a[i].x, b[j].y, acc[i][j].y);
          acc[i][j].y = fma(a[i].y, b[j].x, acc[i][j].y);
        }
    }
    __syncthreads();
  }
  const bool use_beta = (beta.x != 0 || beta.y != 0);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int gr = m0 + ty + 16 * i;
    if (gr >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gc = n0 + tx + 16 * j;
      if (gc >= n) continue;
      C v = cmul(alpha, acc[i][j]);
      long long o = (long long)gr * ldc + gc;
      if (use_beta) v = cadd(v, cmul(beta, Cm[o]));
      Cm[o] = v;
    }
  }
}

template <typename C>
int gemm(const LaContext& ctx, int m, int n, int k, C alpha, const C* A, long long lda, const C* B, long long ldb,
         C beta, C* Cm, long long ldc) {
  if (m <= 0 || n <= 0) return BEM200_OK;
  if (k <= 0) {
    // C = beta C: run the kernel with k = 0 (acc = 0)
  }
  dim3 grid(ceil_div(n, 64), ceil_div(m, 64));
  BEM_REQUIRE(grid.y <= 65535, BEM200_ERR_ARG, "gemm: m too large");
  constexpr int BK = sizeof(C) == 16 ? 8 : 16;
  gemm_simt_kernel<C, BK><<<grid, 256, 0, ctx.stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

template <>
int gemm<float2>(const LaContext& ctx, int m, int n, int k, float2 alpha, const float2* A, long long lda,
                 const float2* B, long long ldb, float2 beta, float2* Cm, long long ldc) {
  if (m <= 0 || n <= 0) return BEM200_OK;
  if (ctx.engine != GemmEngine::kSimt && k >= 64 && m >= 128 && n >= 64)
    return gemm_tc_c64(ctx, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc);
  dim3 grid(ceil_div(n, 64), ceil_div(m, 64));
  BEM_REQUIRE(grid.y <= 65535, BEM200_ERR_ARG, "gemm: m too large");
  gemm_simt_kernel<float2, 16><<<grid, 256, 0, ctx.stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// ===================================================================== row swaps
// for kk in [k0, k1) (forward) swap rows kk and ipiv[kk] over columns [c0, c1)
template <typename C>
__global__ void laswp_kernel(C* A, long long ld, int c0, int c1, const int32_t* __restrict__ ipiv, int k0, int k1) {
  int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  for (int kk = k0; kk < k1; ++kk) {
    int p = ipiv[kk];
    if (p != kk) {
      C t = A[(long long)kk * ld + c];
      A[(long long)kk * ld + c] = A[(long long)p * ld + c];
      A[(long long)p * ld + c] = t;
    }
  }
}

template <typename C>
static int laswp(const LaContext& ctx, C* A, long long ld, int c0, int c1, const int32_t* ipiv, int k0, int k1) {
  if (c1 <= c0 || k1 <= k0) return BEM200_OK;
  laswp_kernel<C><<<ceil_div(c1 - c0, 128), 128, 0, ctx.stream>>>(A, ld, c0, c1, ipiv, k0, k1);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// permutation of the swaps: perm[i] = original row now at position i
__global__ void ipiv_to_perm_kernel(int n, const int32_t* __restrict__ ipiv, int32_t* __restrict__ perm) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int kk = 0; kk < n; ++kk) {
    int p = ipiv[kk];
    int t = perm[kk];
    perm[kk] = perm[p];
    perm[p] = t;
  }
}

// Y[r, perm[i]] = X[r, i]   (X P for the row-permutation matrix P of the swaps)
template <typename C>
__global__ void colperm_kernel(int m, int n, const C* __restrict__ X, long long ldx, const int32_t* __restrict__ perm,
                               C* __restrict__ Y, long long ldy) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m * n) return;
  int r = (int)(idx / n), i = (int)(idx % n);
  Y[(long long)r * ldy + perm[i]] = X[(long long)r * ldx + i];
}

// ===================================================================== panel LU
// Factor rows [col0, n) x columns [col0, col0 + w) with partial pivoting.
// One cluster of `cs` CTAs; CTA `rank` keeps panel rows [rank*R, rank*R + R)
// in shared memory.  ipiv[col0 + t] = global pivot row of step t.
constexpr int kPanelNB = 32;
constexpr int kPanelThreads = 256;

template <typename C>
struct PanelShared {
  R_t<C> red_val[kPanelThreads / 32];
  int red_row[kPanelThreads / 32];
  R_t<C> cand_val;
  int cand_row;
  int piv_row;
  int singular;
  C prow[kPanelNB];
  C trow[kPanelNB];
};

template <typename C>
__global__ void __launch_bounds__(kPanelThreads) panel_lu_kernel(int n, int col0, int w, C* __restrict__ A,
                                                                 long long ld, int32_t* __restrict__ ipiv,
                                                                 int* __restrict__ info, int R) {
  using Real = R_t<C>;
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* rows = reinterpret_cast<C*>(smem_raw);  // R x kPanelNB
  __shared__ PanelShared<C> sh;
  const int m = n - col0;
  const int r0 = rank * R;
  const int rcount = max(0, min(R, m - r0));
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

  for (int idx = tid; idx < rcount * kPanelNB; idx += kPanelThreads) {
    int r = idx / kPanelNB, c = idx % kPanelNB;
    rows[idx] = (c < w) ? A[(long long)(col0 + r0 + r) * ld + col0 + c] : czero<C>();
  }
  if (tid == 0) sh.singular = 0;
  __syncthreads();

  for (int t = 0; t < w; ++t) {
    // ---- local candidate: max |re|+|im| in column t over panel rows >= t
    Real best = -1;
    int brow = INT_MAX;
    for (int r = tid; r < rcount; r += kPanelThreads) {
      int pr = r0 + r;
      if (pr < t) continue;
      Real a = cabs1(rows[r * kPanelNB + t]);
      if (a > best || (a == best && pr < brow)) {
        best = a;
        brow = pr;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      Real ov = __shfl_xor_sync(0xffffffffu, best, o);
      int orw = __shfl_xor_sync(0xffffffffu, brow, o);
      if (ov > best || (ov == best && orw < brow)) {
        best = ov;
        brow = orw;
      }
    }
    if (lane == 0) {
      sh.red_val[wid] = best;
      sh.red_row[wid] = brow;
    }
    __syncthreads();
    if (tid == 0) {
      Real b = sh.red_val[0];
      int br = sh.red_row[0];
      for (int q = 1; q < kPanelThreads / 32; ++q) {
        if (sh.red_val[q] > b || (sh.red_val[q] == b && sh.red_row[q] < br)) {
          b = sh.red_val[q];
          br = sh.red_row[q];
        }
      }
      sh.cand_val = b;
      sh.cand_row = br;
    }
    cluster.sync();  // candidates of all CTAs visible
    if (wid == 0) {
      Real b = -1;
      int br = INT_MAX;
      if (lane < cs) {
        PanelShared<C>* rs = cluster.map_shared_rank(&sh, lane);
        b = rs->cand_val;
        br = rs->cand_row;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        Real ov = __shfl_xor_sync(0xffffffffu, b, o);
        int orw = __shfl_xor_sync(0xffffffffu, br, o);
        if (ov > b || (ov == b && orw < br)) {
          b = ov;
          br = orw;
        }
      }
      if (lane == 0) {
        if (!(b > 0) || br >= m) {  // exactly singular column (or NaN): keep the diagonal
          br = t;
          if (!sh.singular) sh.singular = col0 + t + 1;
        }
        sh.piv_row = br;
      }
    }
    __syncthreads();
    const int p = sh.piv_row;
    const int own_p = p / R, own_t = t / R;
    // read the pivot row (all CTAs) and the target row (pivot owner)
    if (tid < kPanelNB) {
      const C* src = cluster.map_shared_rank(rows, own_p) + (long long)(p - own_p * R) * kPanelNB;
      sh.prow[tid] = src[tid];
      if (rank == own_p) {
        const C* tsrc = cluster.map_shared_rank(rows, own_t) + (long long)(t - own_t * R) * kPanelNB;
        sh.trow[tid] = tsrc[tid];
      }
    }
    cluster.sync();  // every remote read of this step is done before rows change
    if (tid < kPanelNB) {
      if (rank == own_t) rows[(t - own_t * R) * kPanelNB + tid] = sh.prow[tid];
      if (rank == own_p && p != t) rows[(p - own_p * R) * kPanelNB + tid] = sh.trow[tid];
    }
    if (rank == 0 && tid == 0) ipiv[col0 + t] = col0 + p;
    __syncthreads();
    // ---- multipliers and rank-1 update of the remaining panel columns
    const C piv = sh.prow[t];
    const bool ok = (cabs1(piv) > 0);
    for (int r = tid; r < rcount; r += kPanelThreads) {
      if (r0 + r > t) {
        C l = ok ? cdiv(rows[r * kPanelNB + t], piv) : czero<C>();
        rows[r * kPanelNB + t] = l;
      }
    }
    __syncthreads();
    const int ncol = w - t - 1;
    if (ncol > 0) {
      for (int idx = tid; idx < rcount * ncol; idx += kPanelThreads) {
        int r = idx / ncol, c = t + 1 + idx % ncol;
        if (r0 + r > t) {
          C l = rows[r * kPanelNB + t];
          rows[r * kPanelNB + c] = csub(rows[r * kPanelNB + c], cmul(l, sh.prow[c]));
        }
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < rcount * kPanelNB; idx += kPanelThreads) {
    int r = idx / kPanelNB, c = idx % kPanelNB;
    if (c < w) A[(long long)(col0 + r0 + r) * ld + col0 + c] = rows[idx];
  }
  if (rank == 0 && tid == 0 && sh.singular && info) atomicCAS(info, 0, sh.singular);
  cluster.sync();  // no CTA leaves while others may still read its shared memory
}

template <typename C>
static int panel_lu(const LaContext& ctx, int n, C* A, long long ld, int32_t* ipiv, int col0, int w) {
  const int m = n - col0;
  const size_t row_bytes = sizeof(C) * kPanelNB;
  const size_t max_smem = 200 * 1024;
  int cs = 1;
  while ((size_t)ceil_div(m, cs) * row_bytes > max_smem && cs < 16) cs *= 2;
  int R = ceil_div(m, cs);
  size_t smem = (size_t)R * row_bytes;
  BEM_REQUIRE(smem <= max_smem, BEM200_ERR_UNSUPPORTED,
              "panel_lu: panel of %d rows does not fit a 16-CTA cluster", m);
  auto kern = panel_lu_kernel<C>;
  BEM_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (cs > 8) BEM_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs, 1, 1);
  cfg.blockDim = dim3(kPanelThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BEM_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, n, col0, w, A, ld, ipiv, ctx.dinfo, R));
  return BEM200_OK;
}

// ===================================================================== TRSM leaves
// Blocks of 128 threads; each thread owns one right-hand side (a column of B for
// left solves, a row of X for right solves).  The triangle (m <= 32) and the
// right-hand sides live in shared memory.
constexpr int kTrsmNB = 32;
constexpr int kTrsmThreads = 128;

// B[0:m, c] <- T^-1 B[0:m, c]; lower = unit lower (L), else upper non-unit (U)
template <typename C, bool kLower>
__global__ void __launch_bounds__(kTrsmThreads) trsm_left_leaf(int m, int ncols, const C* __restrict__ T, long long ldt,
                                                               C* __restrict__ B, long long ldb) {
  extern __shared__ __align__(16) unsigned char trsm_smem[];
  auto Ts = reinterpret_cast<C(*)[kTrsmNB + 1]>(trsm_smem);
  auto Bs = reinterpret_cast<C(*)[kTrsmThreads]>(trsm_smem + sizeof(C) * kTrsmNB * (kTrsmNB + 1));
  const int c0 = blockIdx.x * kTrsmThreads;
  for (int idx = threadIdx.x; idx < m * m; idx += kTrsmThreads) {
    int r = idx / m, c = idx % m;
    Ts[r][c] = T[(long long)r * ldt + c];
  }
  for (int idx = threadIdx.x; idx < m * kTrsmThreads; idx += kTrsmThreads) {
    int r = idx / kTrsmThreads, c = idx % kTrsmThreads;
    Bs[r][c] = (c0 + c < ncols) ? B[(long long)r * ldb + c0 + c] : czero<C>();
  }
  __syncthreads();
  const int c = threadIdx.x;
  if (kLower) {
    for (int r = 1; r < m; ++r) {
      C s = Bs[r][c];
      for (int q = 0; q < r; ++q) s = csub(s, cmul(Ts[r][q], Bs[q][c]));
      Bs[r][c] = s;
    }
  } else {
    for (int r = m - 1; r >= 0; --r) {
      C s = Bs[r][c];
      for (int q = r + 1; q < m; ++q) s = csub(s, cmul(Ts[r][q], Bs[q][c]));
      Bs[r][c] = cdiv(s, Ts[r][r]);
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < m * kTrsmThreads; idx += kTrsmThreads) {
    int r = idx / kTrsmThreads, cc = idx % kTrsmThreads;
    if (c0 + cc < ncols) B[(long long)r * ldb + c0 + cc] = Bs[r][cc];
  }
}

// X[r, 0:m] <- X[r, 0:m] T^-1 ; upper = non-unit upper (U), else unit lower (L)
template <typename C, bool kUpper>
__global__ void __launch_bounds__(kTrsmThreads) trsm_right_leaf(int m, int nrows, const C* __restrict__ T,
                                                                long long ldt, C* __restrict__ X, long long ldx) {
  extern __shared__ __align__(16) unsigned char trsm_smem[];
  auto Ts = reinterpret_cast<C(*)[kTrsmNB + 1]>(trsm_smem);
  auto Xs = reinterpret_cast<C(*)[kTrsmNB + 1]>(trsm_smem + sizeof(C) * kTrsmNB * (kTrsmNB + 1));
  const int r0 = blockIdx.x * kTrsmThreads;
  for (int idx = threadIdx.x; idx < m * m; idx += kTrsmThreads) {
    int r = idx / m, c = idx % m;
    Ts[r][c] = T[(long long)r * ldt + c];
  }
  for (int idx = threadIdx.x; idx < m * kTrsmThreads; idx += kTrsmThreads) {
    int r = idx / m, c = idx % m;
    Xs[r][c] = (r0 + r < nrows) ? X[(long long)(r0 + r) * ldx + c] : czero<C>();
  }
  __syncthreads();
  const int r = threadIdx.x;
  if (kUpper) {
    // x U = y: x_c = (y_c - sum_{q<c} x_q U_qc) / U_cc
    for (int c = 0; c < m; ++c) {
      C s = Xs[r][c];
      for (int q = 0; q < c; ++q) s = csub(s, cmul(Xs[r][q], Ts[q][c]));
      Xs[r][c] = cdiv(s, Ts[c][c]);
    }
  } else {
    // x L = y, L unit lower: x_c = y_c - sum_{q>c} x_q L_qc
    for (int c = m - 1; c >= 0; --c) {
      C s = Xs[r][c];
      for (int q = c + 1; q < m; ++q) s = csub(s, cmul(Xs[r][q], Ts[q][c]));
      Xs[r][c] = s;
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < m * kTrsmThreads; idx += kTrsmThreads) {
    int rr = idx / m, c = idx % m;
    if (r0 + rr < nrows) X[(long long)(r0 + rr) * ldx + c] = Xs[rr][c];
  }
}

template <typename C>
static size_t trsm_smem_bytes() {
  return sizeof(C) * (kTrsmNB * (kTrsmNB + 1) + kTrsmThreads * (kTrsmNB + 1));
}

template <typename K>
static int prep_smem(K kern, size_t bytes) {
  BEM_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return BEM200_OK;
}

template <typename C> static C neg_one() { return cmake<C>(-1.0, 0.0); }
template <typename C> static C one() { return cmake<C>(1.0, 0.0); }

static int split_point(int m) {
  int h = m / 2;
  h = ((h + kTrsmNB - 1) / kTrsmNB) * kTrsmNB;
  return h < m ? h : m - kTrsmNB;
}

// B <- L^-1 B, L unit lower m x m (strict lower part of T)
template <typename C>
static int trsm_llu(const LaContext& ctx, int m, int ncols, const C* T, long long ldt, C* B, long long ldb) {
  if (m <= 0 || ncols <= 0) return BEM200_OK;
  if (m <= kTrsmNB) {
    { int _st = prep_smem(trsm_left_leaf<C, true>, trsm_smem_bytes<C>()); if (_st) return _st; }
    trsm_left_leaf<C, true><<<ceil_div(ncols, kTrsmThreads), kTrsmThreads, trsm_smem_bytes<C>(), ctx.stream>>>(m, ncols, T, ldt, B, ldb);
    BEM_LAUNCH_CHECK();
    return BEM200_OK;
  }
  int m1 = split_point(m);
  int st = trsm_llu(ctx, m1, ncols, T, ldt, B, ldb);
  if (st) return st;
  st = gemm<C>(ctx, m - m1, ncols, m1, neg_one<C>(), T + (long long)m1 * ldt, ldt, B, ldb, one<C>(),
               B + (long long)m1 * ldb, ldb);
  if (st) return st;
  return trsm_llu(ctx, m - m1, ncols, T + (long long)m1 * ldt + m1, ldt, B + (long long)m1 * ldb, ldb);
}

// B <- U^-1 B, U upper non-unit
template <typename C>
static int trsm_lun(const LaContext& ctx, int m, int ncols, const C* T, long long ldt, C* B, long long ldb) {
  if (m <= 0 || ncols <= 0) return BEM200_OK;
  if (m <= kTrsmNB) {
    { int _st = prep_smem(trsm_left_leaf<C, false>, trsm_smem_bytes<C>()); if (_st) return _st; }
    trsm_left_leaf<C, false><<<ceil_div(ncols, kTrsmThreads), kTrsmThreads, trsm_smem_bytes<C>(), ctx.stream>>>(m, ncols, T, ldt, B,
                                                                                              ldb);
    BEM_LAUNCH_CHECK();
    return BEM200_OK;
  }
  int m1 = split_point(m);
  int st = trsm_lun(ctx, m - m1, ncols, T + (long long)m1 * ldt + m1, ldt, B + (long long)m1 * ldb, ldb);
  if (st) return st;
  st = gemm<C>(ctx, m1, ncols, m - m1, neg_one<C>(), T + m1, ldt, B + (long long)m1 * ldb, ldb, one<C>(), B, ldb);
  if (st) return st;
  return trsm_lun(ctx, m1, ncols, T, ldt, B, ldb);
}

// X <- X U^-1, X nrows x m
template <typename C>
static int trsm_run(const LaContext& ctx, int m, int nrows, const C* T, long long ldt, C* X, long long ldx) {
  if (m <= 0 || nrows <= 0) return BEM200_OK;
  if (m <= kTrsmNB) {
    { int _st = prep_smem(trsm_right_leaf<C, true>, trsm_smem_bytes<C>()); if (_st) return _st; }
    trsm_right_leaf<C, true><<<ceil_div(nrows, kTrsmThreads), kTrsmThreads, trsm_smem_bytes<C>(), ctx.stream>>>(m, nrows, T, ldt, X,
                                                                                             ldx);
    BEM_LAUNCH_CHECK();
    return BEM200_OK;
  }
  int m1 = split_point(m);
  int st = trsm_run(ctx, m1, nrows, T, ldt, X, ldx);
  if (st) return st;
  // X2 -= X1 U12
  st = gemm<C>(ctx, nrows, m - m1, m1, neg_one<C>(), X, ldx, T + m1, ldt, one<C>(), X + m1, ldx);
  if (st) return st;
  return trsm_run(ctx, m - m1, nrows, T + (long long)m1 * ldt + m1, ldt, X + m1, ldx);
}

// X <- X L^-1, L unit lower
template <typename C>
static int trsm_rlu(const LaContext& ctx, int m, int nrows, const C* T, long long ldt, C* X, long long ldx) {
  if (m <= 0 || nrows <= 0) return BEM200_OK;
  if (m <= kTrsmNB) {
    { int _st = prep_smem(trsm_right_leaf<C, false>, trsm_smem_bytes<C>()); if (_st) return _st; }
    trsm_right_leaf<C, false><<<ceil_div(nrows, kTrsmThreads), kTrsmThreads, trsm_smem_bytes<C>(), ctx.stream>>>(m, nrows, T, ldt, X,
                                                                                              ldx);
    BEM_LAUNCH_CHECK();
    return BEM200_OK;
  }
  int m1 = split_point(m);
  int st = trsm_rlu(ctx, m - m1, nrows, T + (long long)m1 * ldt + m1, ldt, X + m1, ldx);
  if (st) return st;
  // X1 -= X2 L21
  st = gemm<C>(ctx, nrows, m1, m - m1, neg_one<C>(), X + m1, ldx, T + (long long)m1 * ldt, ldt, one<C>(), X, ldx);
  if (st) return st;
  return trsm_rlu(ctx, m1, nrows, T, ldt, X, ldx);
}

// ===================================================================== LU
template <typename C>
static int getrf_rec(const LaContext& ctx, int n, C* A, long long ld, int32_t* ipiv, int col0, int w) {
  if (w <= kPanelNB) return panel_lu<C>(ctx, n, A, ld, ipiv, col0, w);
  int w1 = split_point(w);
  int st = getrf_rec(ctx, n, A, ld, ipiv, col0, w1);
  if (st) return st;
  // right half of this column range: apply the left half's swaps
  st = laswp(ctx, A, ld, col0 + w1, col0 + w, ipiv, col0, col0 + w1);
  if (st) return st;
  C* A11 = A + (long long)col0 * ld + col0;
  // U12 = L11^-1 A12
  st = trsm_llu(ctx, w1, w - w1, A11, ld, A11 + w1, ld);
  if (st) return st;
  // A22 -= L21 U12
  st = gemm<C>(ctx, n - col0 - w1, w - w1, w1, neg_one<C>(), A11 + (long long)w1 * ld, ld, A11 + w1, ld, one<C>(),
               A11 + (long long)w1 * ld + w1, ld);
  if (st) return st;
  st = getrf_rec(ctx, n, A, ld, ipiv, col0 + w1, w - w1);
  if (st) return st;
  // left half: apply the right half's swaps
  return laswp(ctx, A, ld, col0, col0 + w1, ipiv, col0 + w1, col0 + w);
}

template <typename C>
int getrf(const LaContext& ctx, int n, C* A, long long ld, int32_t* ipiv) {
  BEM_REQUIRE(n > 0 && A && ipiv && ld >= n, BEM200_ERR_ARG, "getrf: bad arguments");
  return getrf_rec(ctx, n, A, ld, ipiv, 0, n);
}

template <typename C>
int solve_left(const LaContext& ctx, int n, int nrhs, const C* LU, long long ld, const int32_t* ipiv, C* B,
               long long ldb) {
  if (nrhs <= 0) return BEM200_OK;
  int st = laswp(ctx, B, ldb, 0, nrhs, ipiv, 0, n);
  if (st) return st;
  st = trsm_llu(ctx, n, nrhs, LU, ld, B, ldb);
  if (st) return st;
  return trsm_lun(ctx, n, nrhs, LU, ld, B, ldb);
}

template <typename C>
int solve_right(const LaContext& ctx, int n, int m, const C* LU, long long ld, const int32_t* ipiv, C* X,
                long long ldx, C* tmp) {
  // X A = Y with P A = L U  =>  X = Y U^-1 L^-1 P
  if (m <= 0) return BEM200_OK;
  int st = trsm_run(ctx, n, m, LU, ld, X, ldx);
  if (st) return st;
  st = trsm_rlu(ctx, n, m, LU, ld, X, ldx);
  if (st) return st;
  int32_t* perm = reinterpret_cast<int32_t*>(tmp + (long long)m * n);
  ipiv_to_perm_kernel<<<1, 1, 0, ctx.stream>>>(n, ipiv, perm);
  BEM_LAUNCH_CHECK();
  long long tot = (long long)m * n;
  colperm_kernel<C><<<ceil_div(tot, 256), 256, 0, ctx.stream>>>(m, n, X, ldx, perm, tmp, n);
  BEM_LAUNCH_CHECK();
  BEM_CUDA_CHECK(cudaMemcpy2DAsync(X, ldx * sizeof(C), tmp, n * sizeof(C), n * sizeof(C), m,
                                   cudaMemcpyDeviceToDevice, ctx.stream));
  return BEM200_OK;
}

template <typename C>
__global__ void set_identity_kernel(int n, C* A, long long ld) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * n) return;
  int r = (int)(idx / n), c = (int)(idx % n);
  A[(long long)r * ld + c] = (r == c) ? cmake<C>(1.0, 0.0) : czero<C>();
}

template <typename C>
int inverse(const LaContext& ctx, int n, const C* LU, long long ld, const int32_t* ipiv, C* Inv, long long ldi) {
  set_identity_kernel<C><<<ceil_div((long long)n * n, 256), 256, 0, ctx.stream>>>(n, Inv, ldi);
  BEM_LAUNCH_CHECK();
  return solve_left(ctx, n, n, LU, ld, ipiv, Inv, ldi);
}

// explicit instantiations
template int gemm<double2>(const LaContext&, int, int, int, double2, const double2*, long long, const double2*,
                           long long, double2, double2*, long long);
template int getrf<double2>(const LaContext&, int, double2*, long long, int32_t*);
template int getrf<float2>(const LaContext&, int, float2*, long long, int32_t*);
template int solve_left<double2>(const LaContext&, int, int, const double2*, long long, const int32_t*, double2*,
                                 long long);
template int solve_left<float2>(const LaContext&, int, int, const float2*, long long, const int32_t*, float2*,
                                long long);
template int solve_right<double2>(const LaContext&, int, int, const double2*, long long, const int32_t*, double2*,
                                  long long, double2*);
template int solve_right<float2>(const LaContext&, int, int, const float2*, long long, const int32_t*, float2*,
                                 long long, float2*);
template int inverse<double2>(const LaContext&, int, const double2*, long long, const int32_t*, double2*, long long);
template int inverse<float2>(const LaContext&, int, const float2*, long long, const int32_t*, float2*, long long);

}  // namespace bem200

// ===================================================================== C ABI
using namespace bem200;

static GemmEngine engine_of(int e) {
  return e == 1 ? GemmEngine::kTcBf16x3 : (e == 2 ? GemmEngine::kTcTf32 : GemmEngine::kSimt);
}

extern "C" {

int bem200_gemm(int dtype, int engine, int m, int n, int k, const double* alpha, const void* A, int64_t lda,
                const void* B, int64_t ldb, const double* beta, void* C, int64_t ldc, void* ws, size_t ws_bytes,
                void* stream) {
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_of(engine);
  ctx.ws = ws;
  ctx.ws_bytes = ws_bytes;
  BEM_REQUIRE(alpha && beta, BEM200_ERR_ARG, "gemm: alpha/beta must be host pointers to (re, im)");
  if (dtype == BEM200_C128)
    return gemm<double2>(ctx, m, n, k, make_double2(alpha[0], alpha[1]), (const double2*)A, lda, (const double2*)B,
                         ldb, make_double2(beta[0], beta[1]), (double2*)C, ldc);
  if (dtype == BEM200_C64)
    return gemm<float2>(ctx, m, n, k, make_float2((float)alpha[0], (float)alpha[1]), (const float2*)A, lda,
                        (const float2*)B, ldb, make_float2((float)beta[0], (float)beta[1]), (float2*)C, ldc);
  set_error("gemm: bad dtype %d", dtype);
  return BEM200_ERR_ARG;
}

size_t bem200_gemm_workspace_size(int engine, int m, int n, int k) {
  return gemm_tc_workspace(m, n, k, engine_of(engine));
}

int bem200_getrf(int dtype, int engine, int n, void* A, int64_t ld, int32_t* ipiv, int32_t* info, void* ws,
                 size_t ws_bytes, void* stream) {
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_of(engine);
  ctx.ws = ws;
  ctx.ws_bytes = ws_bytes;
  ctx.dinfo = info;
  if (dtype == BEM200_C128) return getrf<double2>(ctx, n, (double2*)A, ld, ipiv);
  if (dtype == BEM200_C64) return getrf<float2>(ctx, n, (float2*)A, ld, ipiv);
  set_error("getrf: bad dtype %d", dtype);
  return BEM200_ERR_ARG;
}

int bem200_getrs(int dtype, int engine, int n, int nrhs, const void* LU, int64_t ld, const int32_t* ipiv, void* B,
                 int64_t ldb, void* ws, size_t ws_bytes, void* stream) {
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_of(engine);
  ctx.ws = ws;
  ctx.ws_bytes = ws_bytes;
  if (dtype == BEM200_C128) return solve_left<double2>(ctx, n, nrhs, (const double2*)LU, ld, ipiv, (double2*)B, ldb);
  if (dtype == BEM200_C64) return solve_left<float2>(ctx, n, nrhs, (const float2*)LU, ld, ipiv, (float2*)B, ldb);
  set_error("getrs: bad dtype %d", dtype);
  return BEM200_ERR_ARG;
}

}  // extern "C"

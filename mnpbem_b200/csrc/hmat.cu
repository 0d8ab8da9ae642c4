// H-matrix kernels: cluster-order permutation of a dense BEM matrix, packing
// of the dense (leaf x leaf) blocks, batched partially pivoted adaptive cross
// approximation of the admissible blocks (one CTA per block), and the
// two-phase H-matrix product.  complex128 throughout.
//
// Reference behaviour followed (MNPBEM Python port v1.6.2):
//   HMatrix._aca_block   mnpbem/greenfun/hmatrix.py:195-336
//   HMatrix.mtimes_vec   mnpbem/greenfun/hmatrix.py:450-541
//
// Block descriptors are (r0, m, c0, nb): rows [r0, r0 + m) and columns
// [c0, c0 + nb) in cluster order.  A low-rank block stores U (m x kcap) and
// V (nb x kcap) row-major with A_block ~ U[:, :rank] V[:, :rank]^T.
#include <cfloat>

#include "common.cuh"
#include "green_entry.cuh"

namespace bem200 {

constexpr int kHThreads = 256;

// Entry (ci, cj) of a dense n x n matrix already in cluster order.
struct DenseSource {
  const double2* Mc;
  int n;
  __device__ __forceinline__ double2 operator()(int ci, int cj) const { return Mc[(long long)ci * n + cj]; }
};

__device__ __forceinline__ double cmod(double2 a) { return hypot(a.x, a.y); }

// dst[i, :] = src[idx[i], :]  (n rows of w complex)
__global__ void gather_rows_c128_kernel(int n, int w, const double2* __restrict__ src, const int32_t* __restrict__ idx,
                                        double2* __restrict__ dst) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * w) return;
  const int i = (int)(e / w), q = (int)(e % w);
  dst[e] = src[(long long)idx[i] * w + q];
}

// dst[i][j] = src[c2p[i]][c2p[j]]: one CTA per row
__global__ void permute_kernel(int n, const double2* __restrict__ src, const int32_t* __restrict__ c2p,
                               double2* __restrict__ dst) {
  const int i = blockIdx.x;
  const double2* srow = src + (long long)c2p[i] * n;
  double2* drow = dst + (long long)i * n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) drow[j] = srow[c2p[j]];
}

template <typename Src>
__global__ void pack_dense_kernel(const int32_t* __restrict__ blk, const int64_t* __restrict__ off, Src src,
                                  double2* __restrict__ D) {
  const int b = blockIdx.x;
  const int r0 = blk[4 * b], m = blk[4 * b + 1], c0 = blk[4 * b + 2], nb = blk[4 * b + 3];
  double2* out = D + off[b];
  for (long long e = threadIdx.x; e < (long long)m * nb; e += blockDim.x) {
    const int i = (int)(e / nb), j = (int)(e % nb);
    out[e] = src(r0 + i, c0 + j);
  }
}

// block-wide argmax over (value, index): larger value wins, ties -> smaller index
__device__ void block_argmax(double& v, int& ix, double* sv, int* si) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, ix, o);
    if (ov > v || (ov == v && oi < ix)) {
      v = ov;
      ix = oi;
    }
  }
  if (lane == 0) {
    sv[wid] = v;
    si[wid] = ix;
  }
  __syncthreads();
  if (wid == 0) {
    v = lane < kHThreads / 32 ? sv[lane] : -1.0;
    ix = lane < kHThreads / 32 ? si[lane] : INT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, v, o);
      const int oi = __shfl_xor_sync(0xffffffffu, ix, o);
      if (ov > v || (ov == v && oi < ix)) {
        v = ov;
        ix = oi;
      }
    }
    if (lane == 0) {
      sv[0] = v;
      si[0] = ix;
    }
  }
  __syncthreads();
  v = sv[0];
  ix = si[0];
  __syncthreads();
}

__device__ double block_sum_d(double v, double* sv) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) sv[wid] = v;
  __syncthreads();
  double r = 0;
  for (int k = 0; k < kHThreads / 32; ++k) r += sv[k];
  __syncthreads();
  return r;
}

// Partially pivoted ACA of one admissible block per CTA.  Shared memory:
// used-row / used-column flags (m + nb bytes), U[p, :k] and V[pc, :k]
// (kcap complex each), the per-l partial cross dots (2 x kcap complex).
// The block's entries come from `src`: a stored matrix or the Green function.
template <typename Src>
__global__ void __launch_bounds__(kHThreads) aca_kernel(const int32_t* __restrict__ blk, const int64_t* __restrict__ uoff,
                                                       const int64_t* __restrict__ voff, const int32_t* __restrict__ kcap_arr,
                                                       Src src, double htol,
                                                       double2* __restrict__ Ug, double2* __restrict__ Vg,
                                                       int32_t* __restrict__ rank_out) {
  extern __shared__ __align__(16) unsigned char aca_smem[];
  __shared__ double sv[kHThreads / 32];
  __shared__ int si[kHThreads / 32];
  const int b = blockIdx.x;
  const int r0 = blk[4 * b], m = blk[4 * b + 1], c0 = blk[4 * b + 2], nb = blk[4 * b + 3];
  const int kc = kcap_arr[b];
  double2* U = Ug + uoff[b];
  double2* V = Vg + voff[b];
  double2* Up = reinterpret_cast<double2*>(aca_smem);  // kc
  double2* Vp = Up + kc;                               // kc
  double2* du = Vp + kc;                               // kc
  double2* dv = du + kc;                               // kc
  unsigned char* used_r = reinterpret_cast<unsigned char*>(dv + kc);
  unsigned char* used_c = used_r + m;
  const int tid = threadIdx.x;
  for (int i = tid; i < m; i += kHThreads) used_r[i] = 0;
  for (int j = tid; j < nb; j += kHThreads) used_c[j] = 0;
  __syncthreads();
  int p = 0;
  int rank = 0;
  double frob = 0.0;
  for (int k = 0; k < kc; ++k) {
    // residual row p -> V[:, k]
    for (int l = tid; l < k; l += kHThreads) Up[l] = U[(long long)p * kc + l];
    __syncthreads();
    double best = -1.0;
    int bj = INT_MAX;
    double vsq = 0.0;
    for (int j = tid; j < nb; j += kHThreads) {
      double2 val = src(r0 + p, c0 + j);
      const double2* vj = V + (long long)j * kc;
      for (int l = 0; l < k; ++l) val = csub(val, cmul(Up[l], vj[l]));
      V[(long long)j * kc + k] = val;
      vsq += cabs2(val);
      const double a = used_c[j] ? 0.0 : cmod(val);
      if (a > best) {
        best = a;
        bj = j;
      }
    }
    block_argmax(best, bj, sv, si);
    vsq = block_sum_d(vsq, sv);
    const int pc = bj;
    const double2 pv = V[(long long)pc * kc + k];
    if (!(cmod(pv) >= 1e-15)) break;  // (also stops on NaN)
    // residual column pc -> U[:, k] = col / pivot
    for (int l = tid; l < k; l += kHThreads) Vp[l] = V[(long long)pc * kc + l];
    if (tid == 0) {
      used_r[p] = 1;
      used_c[pc] = 1;
    }
    __syncthreads();
    double usq = 0.0;
    best = -1.0;
    int bi = INT_MAX;
    for (int i = tid; i < m; i += kHThreads) {
      double2 val = src(r0 + i, c0 + pc);
      const double2* ui = U + (long long)i * kc;
      for (int l = 0; l < k; ++l) val = csub(val, cmul(ui[l], Vp[l]));
      const double2 u = cdiv(val, pv);
      U[(long long)i * kc + k] = u;
      usq += cabs2(u);
      const double a = used_r[i] ? 0.0 : cmod(u);
      if (a > best) {
        best = a;
        bi = i;
      }
    }
    block_argmax(best, bi, sv, si);  // also orders the U[:, k] stores before the cross dots
    usq = block_sum_d(usq, sv);
    rank = k + 1;
    const double new_sq = usq * vsq;
    // cross terms 2 Re sum_l (U_l^H u)(V_l^H v), l < k
    double cross = 0.0;
    if (k > 0) {
      for (int l = tid; l < k; l += kHThreads) {
        double2 a = make_double2(0, 0), c = make_double2(0, 0);
        for (int i = 0; i < m; ++i) {
          const double2 ul = U[(long long)i * kc + l], un = U[(long long)i * kc + k];
          a = cadd(a, make_double2(ul.x * un.x + ul.y * un.y, ul.x * un.y - ul.y * un.x));
        }
        for (int j = 0; j < nb; ++j) {
          const double2 vl = V[(long long)j * kc + l], vn = V[(long long)j * kc + k];
          c = cadd(c, make_double2(vl.x * vn.x + vl.y * vn.y, vl.x * vn.y - vl.y * vn.x));
        }
        du[l] = a;
        dv[l] = c;
      }
      __syncthreads();
      double part = 0.0;
      for (int l = tid; l < k; l += kHThreads) part += du[l].x * dv[l].x - du[l].y * dv[l].y;
      cross = 2.0 * block_sum_d(part, sv);
    }
    frob += new_sq + cross;
    if (frob > 0 && sqrt(new_sq) < htol * sqrt(fabs(frob))) break;
    p = bi;  // next pivot row: largest |u| among unused rows
    __syncthreads();
  }
  if (tid == 0) rank_out[b] = rank;
}

// Phase A: T_b (rank x w) = V_b^T x[c0 : c0 + nb, :]
__global__ void __launch_bounds__(kHThreads) hmat_vt_kernel(const int32_t* __restrict__ blk,
                                                           const int64_t* __restrict__ voff,
                                                           const int64_t* __restrict__ toff,
                                                           const int32_t* __restrict__ kcap_arr,
                                                           const int32_t* __restrict__ rank_arr, int w,
                                                           const double2* __restrict__ x,
                                                           const double2* __restrict__ Vg, double2* __restrict__ T) {
  const int b = blockIdx.x;
  const int c0 = blk[4 * b + 2], nb = blk[4 * b + 3];
  const int kc = kcap_arr[b], r = rank_arr[b];
  const double2* V = Vg + voff[b];
  double2* Tb = T + toff[b] * w;
  for (int o = threadIdx.x; o < r * w; o += kHThreads) {
    const int l = o / w, q = o % w;
    double2 acc = make_double2(0, 0);
    for (int j = 0; j < nb; ++j) acc = cadd(acc, cmul(V[(long long)j * kc + l], x[(long long)(c0 + j) * w + q]));
    Tb[o] = acc;
  }
}

// Phase B: one CTA per block (dense blocks first, then low-rank ones):
// y[rows] += M_b S_b, with M_b the packed dense block (S_b = the x rows of its
// columns) or the U factor (S_b = T_b).  S_b is staged in shared memory in
// chunks of kSChunk rows with an odd pitch; 8 lanes share a matrix row (so a
// warp covers 4 rows, each read coalesced 128 B at a time), reduce over
// their 8 partial sums with 3 shuffle levels, and add the row into y with
// FP64 atomics (y is zeroed first).
constexpr int kSChunk = 128;

template <int W>
__global__ void __launch_bounds__(kHThreads) hmat_block_kernel(
    int nd, int w, const double2* __restrict__ x, const int32_t* __restrict__ lblk, const int64_t* __restrict__ uoff,
    const int64_t* __restrict__ toff, const int32_t* __restrict__ kcap_arr, const int32_t* __restrict__ rank_arr,
    const double2* __restrict__ Ug, const double2* __restrict__ T, const int32_t* __restrict__ dblk,
    const int64_t* __restrict__ doff, const double2* __restrict__ D, double2* __restrict__ y) {
  __shared__ double2 Ss[kSChunk][W + 1];
  const int b = blockIdx.x;
  int r0, m, K, ldm;
  const double2* M;
  const double2* S;
  if (b < nd) {
    r0 = dblk[4 * b];
    m = dblk[4 * b + 1];
    K = dblk[4 * b + 3];
    ldm = K;
    M = D + doff[b];
    S = x + (long long)dblk[4 * b + 2] * w;
  } else {
    const int l = b - nd;
    r0 = lblk[4 * l];
    m = lblk[4 * l + 1];
    K = rank_arr[l];
    ldm = kcap_arr[l];
    M = Ug + uoff[l];
    S = T + toff[l] * w;
  }
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int js = lane & 7, rs = lane >> 3;  // 8 lanes per row, 4 rows per warp
  for (int rbase = 0; rbase < m; rbase += 4 * (kHThreads / 32)) {
    const int rl = rbase + 4 * wid + rs;
    const bool rok = rl < m;
    double2 acc[W];
#pragma unroll
    for (int q = 0; q < W; ++q) acc[q] = make_double2(0, 0);
    for (int k0 = 0; k0 < K; k0 += kSChunk) {
      const int kn = min(kSChunk, K - k0);
      __syncthreads();
      for (int e = tid; e < kn * w; e += kHThreads) {
        const int j = e / w, q = e % w;
        Ss[j][q] = S[(long long)(k0 + j) * w + q];
      }
      __syncthreads();
      if (rok) {
        const double2* mrow = M + (long long)rl * ldm + k0;
#pragma unroll 4
        for (int j = js; j < kn; j += 8) {
          const double2 a = mrow[j];
#pragma unroll
          for (int q = 0; q < W; ++q)
            if (q < w) acc[q] = cadd(acc[q], cmul(a, Ss[j][q]));
        }
      }
    }
#pragma unroll
    for (int q = 0; q < W; ++q) {
      double2 v = acc[q];
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
      }
      acc[q] = v;
    }
    if (rok) {
#pragma unroll
      for (int q = 0; q < W; ++q)
        if (q < w && q % 8 == js) {
          double* out = reinterpret_cast<double*>(y + (long long)(r0 + rl) * w + q);
          atomicAdd(out, acc[q].x);
          atomicAdd(out + 1, acc[q].y);
        }
    }
  }
}

// ------------------------------------------------------- work-item product
// The per-block kernels above give each block one CTA, so the few largest
// admissible blocks (thousands of rows) set the kernel time.  Here large
// blocks are split over several CTAs by host-built work items:
//   phase A item (l, j0): rows [j0, j0 + kVtRows) of V_l; the partial
//     V_l^T x over those rows is added into T_l with FP64 atomics (T zeroed).
//     x rows are staged in shared memory; lanes own 32 outputs (l, q) of T_l,
//     warps split the rows, and the 8 warp partials are summed in shared memory.
//   phase B item (b, i0): rows [i0, i0 + 32) of block b (b < nd dense, else
//     low-rank b - nd), with the row kernel of hmat_block_kernel.
constexpr int kVtRows = 128;
constexpr int kItemRows = 4 * (kHThreads / 32);  // 32 rows: one pass of 8 warps x 4 rows

template <int W>
__global__ void __launch_bounds__(kHThreads) hmat_vt_items_kernel(
    const int32_t* __restrict__ items, int w, const int32_t* __restrict__ blk, const int64_t* __restrict__ voff,
    const int64_t* __restrict__ toff, const int32_t* __restrict__ kcap_arr, const int32_t* __restrict__ rank_arr,
    const double2* __restrict__ x, const double2* __restrict__ Vg, double2* __restrict__ T) {
  __shared__ double2 xs[kVtRows][W + 1];
  __shared__ double2 red[kHThreads / 32][32];
  const int l = items[2 * blockIdx.x], j0 = items[2 * blockIdx.x + 1];
  const int c0 = blk[4 * l + 2], nb = blk[4 * l + 3];
  const int kc = kcap_arr[l], r = rank_arr[l];
  const int jn = min(kVtRows, nb - j0);
  const double2* V = Vg + voff[l] + (long long)j0 * kc;
  double2* Tb = T + toff[l] * w;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int e = tid; e < jn * w; e += kHThreads) {
    const int jj = e / w, q = e % w;
    xs[jj][q] = x[(long long)(c0 + j0 + jj) * w + q];
  }
  __syncthreads();
  const int rw = r * w;
  for (int ot = 0; ot < rw; ot += 32) {
    const int o = ot + lane;
    const bool ok = o < rw;
    const int lo = ok ? o / w : 0, q = ok ? o % w : 0;
    double2 acc = make_double2(0, 0);
    if (ok) {
#pragma unroll 4
      for (int jj = wid; jj < jn; jj += kHThreads / 32) acc = cadd(acc, cmul(V[(long long)jj * kc + lo], xs[jj][q]));
    }
    red[wid][lane] = acc;
    __syncthreads();
    if (wid == 0 && ok) {
      double2 sum = red[0][lane];
#pragma unroll
      for (int k = 1; k < kHThreads / 32; ++k) sum = cadd(sum, red[k][lane]);
      double* out = reinterpret_cast<double*>(Tb + o);
      atomicAdd(out, sum.x);
      atomicAdd(out + 1, sum.y);
    }
    __syncthreads();
  }
}

template <int W>
__global__ void __launch_bounds__(kHThreads) hmat_block_items_kernel(
    const int32_t* __restrict__ items, int nd, int w, const double2* __restrict__ x,
    const int32_t* __restrict__ lblk, const int64_t* __restrict__ uoff, const int64_t* __restrict__ toff,
    const int32_t* __restrict__ kcap_arr, const int32_t* __restrict__ rank_arr, const double2* __restrict__ Ug,
    const double2* __restrict__ T, const int32_t* __restrict__ dblk, const int64_t* __restrict__ doff,
    const double2* __restrict__ D, double2* __restrict__ y) {
  __shared__ double2 Ss[kSChunk][W + 1];
  const int b = items[2 * blockIdx.x], i0 = items[2 * blockIdx.x + 1];
  int r0, m, K, ldm;
  const double2* M;
  const double2* S;
  if (b < nd) {
    r0 = dblk[4 * b];
    m = dblk[4 * b + 1];
    K = dblk[4 * b + 3];
    ldm = K;
    M = D + doff[b];
    S = x + (long long)dblk[4 * b + 2] * w;
  } else {
    const int l = b - nd;
    r0 = lblk[4 * l];
    m = lblk[4 * l + 1];
    K = rank_arr[l];
    ldm = kcap_arr[l];
    M = Ug + uoff[l];
    S = T + toff[l] * w;
  }
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int js = lane & 7, rs = lane >> 3;  // 8 lanes per row, 4 rows per warp
  const int rl = i0 + 4 * wid + rs;
  const bool rok = rl < m;
  double2 acc[W];
#pragma unroll
  for (int q = 0; q < W; ++q) acc[q] = make_double2(0, 0);
  for (int k0 = 0; k0 < K; k0 += kSChunk) {
    const int kn = min(kSChunk, K - k0);
    __syncthreads();
    for (int e = tid; e < kn * w; e += kHThreads) {
      const int j = e / w, q = e % w;
      Ss[j][q] = S[(long long)(k0 + j) * w + q];
    }
    __syncthreads();
    if (rok) {
      const double2* mrow = M + (long long)rl * ldm + k0;
#pragma unroll 4
      for (int j = js; j < kn; j += 8) {
        const double2 a = mrow[j];
#pragma unroll
        for (int q = 0; q < W; ++q)
          if (q < w) acc[q] = cadd(acc[q], cmul(a, Ss[j][q]));
      }
    }
  }
#pragma unroll
  for (int q = 0; q < W; ++q) {
    double2 v = acc[q];
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    acc[q] = v;
  }
  if (rok) {
#pragma unroll
    for (int q = 0; q < W; ++q)
      if (q < w && q % 8 == js) {
        double* out = reinterpret_cast<double*>(y + (long long)(r0 + rl) * w + q);
        atomicAdd(out, acc[q].x);
        atomicAdd(out + 1, acc[q].y);
      }
  }
}

}  // namespace bem200

using namespace bem200;

extern "C" {

int bem200_hmat_gather_rows(int n, int w, const void* src, const int32_t* idx, void* dst, void* stream) {
  BEM_REQUIRE(n > 0 && w > 0 && src && idx && dst && src != dst, BEM200_ERR_ARG, "hmat_gather_rows: bad arguments");
  gather_rows_c128_kernel<<<ceil_div((long long)n * w, 256), 256, 0, (cudaStream_t)stream>>>(
      n, w, (const double2*)src, idx, (double2*)dst);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_hmat_permute(int n, const void* src, const int32_t* c2p, void* dst, void* stream) {
  BEM_REQUIRE(n > 0 && src && c2p && dst && src != dst, BEM200_ERR_ARG, "hmat_permute: bad arguments");
  permute_kernel<<<n, 256, 0, (cudaStream_t)stream>>>(n, (const double2*)src, c2p, (double2*)dst);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_hmat_pack_dense(int nd, const int32_t* dblk, const int64_t* doff, int n, const void* Mc, void* D,
                           void* stream) {
  BEM_REQUIRE(nd >= 0 && n > 0, BEM200_ERR_ARG, "hmat_pack_dense: bad sizes");
  if (nd == 0) return BEM200_OK;
  BEM_REQUIRE(dblk && doff && Mc && D, BEM200_ERR_ARG, "hmat_pack_dense: null pointer");
  pack_dense_kernel<DenseSource><<<nd, 256, 0, (cudaStream_t)stream>>>(dblk, doff, DenseSource{(const double2*)Mc, n},
                                                                        (double2*)D);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_hmat_aca(int nl, const int32_t* lblk, const int64_t* uoff, const int64_t* voff, const int32_t* kcap,
                    int n, const void* Mc, double htol, void* U, void* V, int32_t* rank, int max_rows,
                    int max_kcap, void* stream) {
  BEM_REQUIRE(nl >= 0 && n > 0 && htol >= 0, BEM200_ERR_ARG, "hmat_aca: bad sizes");
  if (nl == 0) return BEM200_OK;
  BEM_REQUIRE(lblk && uoff && voff && kcap && Mc && U && V && rank, BEM200_ERR_ARG, "hmat_aca: null pointer");
  // flags for rows and columns (<= 2 max_rows bytes) + 4 kcap complex
  const size_t smem = (size_t)4 * max_kcap * sizeof(double2) + 2 * (size_t)max_rows + 16;
  BEM_REQUIRE(smem <= 200 * 1024, BEM200_ERR_UNSUPPORTED, "hmat_aca: block of %d rows / rank %d too large", max_rows,
              max_kcap);
  BEM_CUDA_CHECK(set_kernel_attrs_once(aca_kernel<DenseSource>, (int)smem, false));
  aca_kernel<DenseSource><<<nl, kHThreads, smem, (cudaStream_t)stream>>>(
      lblk, uoff, voff, kcap, DenseSource{(const double2*)Mc, n}, htol, (double2*)U, (double2*)V, rank);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_hmat_compress_green(int which, int n, int npart, const int32_t* pid, const int32_t* blk_mat, int nmat,
                               const double* kmat_host, const double* pos, const double* nvec, const double* area,
                               const int64_t* ref_row_ptr, const int32_t* ref_col, int order, const double* g,
                               const double* fn, const int32_t* c2p, int nd, const int32_t* dblk,
                               const int64_t* doff, void* D, int nl, const int32_t* lblk, const int64_t* uoff,
                               const int64_t* voff, const int32_t* kcap, double htol, void* U, void* V,
                               int32_t* rank, int max_rows, int max_kcap, void* stream) {
  BEM_REQUIRE(which >= 0 && which <= 3 && n > 0 && npart > 0 && nmat > 0 && nmat <= ge::kMaxMat && kmat_host &&
                  pid && blk_mat && pos && nvec && area && c2p && order >= 0 && order <= ge::kMaxOrder &&
                  nd >= 0 && nl >= 0 && htol >= 0,
              BEM200_ERR_ARG, "hmat_compress_green: bad arguments");
  BEM_REQUIRE(ref_row_ptr ? (ref_col && g && fn) : true, BEM200_ERR_ARG,
              "hmat_compress_green: refinement tables incomplete");
  ge::GreenSource src;
  src.n = n;
  src.npart = npart;
  src.which = which;
  src.order = order;
  src.pid = pid;
  src.blk_mat = blk_mat;
  src.pos = pos;
  src.nvec = nvec;
  src.area = area;
  src.row_ptr = ref_row_ptr;
  src.ref_col = ref_col;
  src.g = g;
  src.fn = fn;
  src.c2p = c2p;
  for (int m = 0; m < ge::kMaxMat; ++m) {
    src.kre[m] = m < nmat ? kmat_host[2 * m] : 0.0;
    src.kim[m] = m < nmat ? kmat_host[2 * m + 1] : 0.0;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (nd > 0) {
    BEM_REQUIRE(dblk && doff && D, BEM200_ERR_ARG, "hmat_compress_green: null dense-leaf pointer");
    pack_dense_kernel<ge::GreenSource><<<nd, 256, 0, s>>>(dblk, doff, src, (double2*)D);
    BEM_LAUNCH_CHECK();
  }
  if (nl > 0) {
    BEM_REQUIRE(lblk && uoff && voff && kcap && U && V && rank, BEM200_ERR_ARG,
                "hmat_compress_green: null low-rank pointer");
    const size_t smem = (size_t)4 * max_kcap * sizeof(double2) + 2 * (size_t)max_rows + 16;
    BEM_REQUIRE(smem <= 200 * 1024, BEM200_ERR_UNSUPPORTED, "hmat_compress_green: block of %d rows / rank %d too large",
                max_rows, max_kcap);
    BEM_CUDA_CHECK(set_kernel_attrs_once(aca_kernel<ge::GreenSource>, (int)smem, false));
    aca_kernel<ge::GreenSource><<<nl, kHThreads, smem, s>>>(lblk, uoff, voff, kcap, src, htol, (double2*)U,
                                                             (double2*)V, rank);
    BEM_LAUNCH_CHECK();
  }
  return BEM200_OK;
}

int bem200_hmat_matvec(int n, int w, const void* x, int nl, const int32_t* lblk, const int64_t* voff,
                       const int64_t* uoff, const int64_t* toff, const int32_t* kcap, const int32_t* rank,
                       const void* U, const void* V, void* T, int nd, const int32_t* dblk, const int64_t* doff,
                       const void* D, void* y, void* stream) {
  BEM_REQUIRE(n > 0 && w > 0 && w <= 16 && x && y && nl >= 0 && nd >= 0, BEM200_ERR_ARG,
              "hmat_matvec: bad arguments (w <= 16 columns)");
  cudaStream_t s = (cudaStream_t)stream;
  BEM_CUDA_CHECK(cudaMemsetAsync(y, 0, sizeof(double2) * (size_t)n * w, s));
  if (nl > 0) {
    hmat_vt_kernel<<<nl, kHThreads, 0, s>>>(lblk, voff, toff, kcap, rank, w, (const double2*)x, (const double2*)V,
                                           (double2*)T);
    BEM_LAUNCH_CHECK();
  }
  if (nd + nl == 0) return BEM200_OK;
  if (w <= 8)
    hmat_block_kernel<8><<<nd + nl, kHThreads, 0, s>>>(nd, w, (const double2*)x, lblk, uoff, toff, kcap, rank,
                                                       (const double2*)U, (const double2*)T, dblk, doff,
                                                       (const double2*)D, (double2*)y);
  else
    hmat_block_kernel<16><<<nd + nl, kHThreads, 0, s>>>(nd, w, (const double2*)x, lblk, uoff, toff, kcap, rank,
                                                        (const double2*)U, (const double2*)T, dblk, doff,
                                                        (const double2*)D, (double2*)y);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_hmat_matvec_items(int n, int w, const void* x, int nl, const int32_t* lblk, const int64_t* voff,
                             const int64_t* uoff, const int64_t* toff, const int32_t* kcap, const int32_t* rank,
                             const void* U, const void* V, void* T, int64_t t_len, int nd, const int32_t* dblk,
                             const int64_t* doff, const void* D, int nvitems, const int32_t* vitems, int nbitems,
                             const int32_t* bitems, void* y, void* stream) {
  BEM_REQUIRE(n > 0 && w > 0 && w <= 16 && x && y && nl >= 0 && nd >= 0 && nvitems >= 0 && nbitems >= 0 &&
                  t_len >= 0,
              BEM200_ERR_ARG, "hmat_matvec_items: bad arguments (w <= 16 columns)");
  BEM_REQUIRE((nvitems == 0 || (vitems && T && V && lblk)) && (nbitems == 0 || bitems), BEM200_ERR_ARG,
              "hmat_matvec_items: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  BEM_CUDA_CHECK(cudaMemsetAsync(y, 0, sizeof(double2) * (size_t)n * w, s));
  if (nvitems > 0) {
    BEM_CUDA_CHECK(cudaMemsetAsync(T, 0, sizeof(double2) * (size_t)t_len, s));
    if (w <= 8)
      hmat_vt_items_kernel<8><<<nvitems, kHThreads, 0, s>>>(vitems, w, lblk, voff, toff, kcap, rank,
                                                            (const double2*)x, (const double2*)V, (double2*)T);
    else
      hmat_vt_items_kernel<16><<<nvitems, kHThreads, 0, s>>>(vitems, w, lblk, voff, toff, kcap, rank,
                                                             (const double2*)x, (const double2*)V, (double2*)T);
    BEM_LAUNCH_CHECK();
  }
  if (nbitems == 0) return BEM200_OK;
  if (w <= 8)
    hmat_block_items_kernel<8><<<nbitems, kHThreads, 0, s>>>(bitems, nd, w, (const double2*)x, lblk, uoff, toff,
                                                             kcap, rank, (const double2*)U, (const double2*)T, dblk,
                                                             doff, (const double2*)D, (double2*)y);
  else
    hmat_block_items_kernel<16><<<nbitems, kHThreads, 0, s>>>(bitems, nd, w, (const double2*)x, lblk, uoff, toff,
                                                              kcap, rank, (const double2*)U, (const double2*)T, dblk,
                                                              doff, (const double2*)D, (double2*)y);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

}  // extern "C"

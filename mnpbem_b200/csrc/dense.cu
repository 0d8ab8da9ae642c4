// Dense complex LU with partial pivoting, triangular solves and GEMM.
//
// Structure (host-driven recursion, kernels enqueued on one stream):
//   * recursive LU; the leaf panel (width <= 32) is factored by ONE
//     thread-block cluster that keeps the tall panel in distributed shared
//     memory.  Pivoting is lazy: rows stay where they are and a rowmap
//     (logical -> storage row) is updated, so there are no row-swap passes;
//     each column costs one cluster barrier (candidates are double buffered).
//   * recursive TRSM with small substitution kernels at the leaves, and a
//     blocked triangular solve for few right-hand sides in which row blocks
//     wait on flags of the blocks they depend on (bounded waits).
//   * GEMM on row views: CUDA-core kernel for complex128 (FP64 FMA) /
//     complex64, and the tcgen05 tensor-core path for complex64 (gemm_tc.cu).
// Pivot choice follows LAPACK izamax: largest |re| + |im|.
#include <cooperative_groups.h>

#include <climits>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "dense.cuh"

namespace cg = cooperative_groups;

namespace bem200 {

template <typename C> using R_t = typename cplx_traits<C>::real;

__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ float cabs1(float2 a) { return fabsf(a.x) + fabsf(a.y); }

template <typename C>
__device__ __forceinline__ C shfl_c(C v, int src) {
  v.x = __shfl_sync(0xffffffffu, v.x, src);
  v.y = __shfl_sync(0xffffffffu, v.y, src);
  return v;
}

// ===================================================================== GEMM
// C = alpha A B + beta C on row views; block tile (16 TM) x (16 TM), each
// thread a TM x TM register tile (rows ty + 16 i, cols tx + 16 j).  TM = 4
// for most shapes, TM = 2 when 64 x 64 tiles would leave most SMs idle, TM = 1
// for the small products whose 32 x 32 tiles would fill fewer than half.
template <typename C, int BK, int TM = 4>
__global__ void __launch_bounds__(256) gemm_simt_kernel(int m, int n, int k, C alpha, RowView<C> A, RowView<C> B,
                                                        C beta, RowView<C> Cv) {
  constexpr int BM = 16 * TM, BN = 16 * TM;
  constexpr int A_LOADS = BM * BK / 256;  // rows of A loaded per thread (fixed over k)
  constexpr int B_LOADS = BK * BN / 256;
  __shared__ C As[BK][BM + 1];
  __shared__ C Bs[BK][BN];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  // this thread loads A rows ar0 + i * (256 / BK), column ac of each k-slab
  const int ac = tid % BK, ar0 = tid / BK;
  long long aoff[A_LOADS];
#pragma unroll
  for (int i = 0; i < A_LOADS; ++i) {
    int gr = m0 + ar0 + i * (256 / BK);
    aoff[i] = gr < m ? A.off(gr, 0) : -1;
  }
  const int bc = tid % BN, br0 = tid / BN;
  const bool bcol_ok = (n0 + bc) < n;
  C acc[TM][TM];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TM; ++j) acc[i][j] = czero<C>();
  // the next k-slab's operands are loaded into registers while this one is
  // multiplied, so the global-load latency overlaps the products
  C ra[A_LOADS], rb[B_LOADS];
  auto fetch = [&](int k0) {
    const int gc = k0 + ac;
#pragma unroll
    for (int i = 0; i < A_LOADS; ++i) ra[i] = (aoff[i] >= 0 && gc < k) ? A.base[aoff[i] + gc] : czero<C>();
#pragma unroll
    for (int i = 0; i < B_LOADS; ++i) {
      const int gr = k0 + br0 + i * (256 / BN);
      rb[i] = (gr < k && bcol_ok) ? B.at(gr, n0 + bc) : czero<C>();
    }
  };
  fetch(0);
  for (int k0 = 0; k0 < k; k0 += BK) {
#pragma unroll
    for (int i = 0; i < A_LOADS; ++i) As[ac][ar0 + i * (256 / BK)] = ra[i];
#pragma unroll
    for (int i = 0; i < B_LOADS; ++i) Bs[br0 + i * (256 / BN)][bc] = rb[i];
    __syncthreads();
    if (k0 + BK < k) fetch(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      C a[TM], b[TM];
#pragma unroll
      for (int i = 0; i < TM; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < TM; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TM; ++j) {
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
  for (int i = 0; i < TM; ++i) {
    int gr = m0 + ty + 16 * i;
    if (gr >= m) continue;
    const long long roff = Cv.off(gr, 0);
#pragma unroll
    for (int j = 0; j < TM; ++j) {
      int gc = n0 + tx + 16 * j;
      if (gc >= n) continue;
      C v = cmul(alpha, acc[i][j]);
      C& out = Cv.base[roff + gc];
      if (use_beta) v = cadd(v, cmul(beta, out));
      out = v;
    }
  }
}

// Skinny GEMM: C (m x w) = alpha A (m x k) B (k x w) + beta C for w <= W
// right-hand columns, a matrix-times-few-vectors product bound by streaming A
// once from HBM.  Warp g of a CTA owns RW rows; lane l handles k = l (mod 32)
// of every 128-wide k chunk, whose B rows sit in shared memory (odd pitch),
// and keeps RW x W complex partial sums that are reduced across the warp at
// the end.
template <typename C, int W, int RW>
__global__ void __launch_bounds__(256) gemm_skinny_kernel(int m, int w, int k, C alpha, RowView<C> A, RowView<C> B,
                                                          C beta, RowView<C> Cv) {
  // 256-wide k chunks where their B rows fit the static shared memory
  constexpr int KC = sizeof(C) * (W + 1) * 256 <= 48 * 1024 ? 256 : 128;
  __shared__ C bs[KC][W + 1];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int row0 = (blockIdx.x * 8 + wid) * RW;
  long long aoff[RW];
#pragma unroll
  for (int r = 0; r < RW; ++r) aoff[r] = (row0 + r < m) ? A.off(row0 + r, 0) : -1;
  C acc[RW][W];
#pragma unroll
  for (int r = 0; r < RW; ++r)
#pragma unroll
    for (int q = 0; q < W; ++q) acc[r][q] = czero<C>();
  for (int k0 = 0; k0 < k; k0 += KC) {
    // all of the chunk's loads of A issue first, before the B rows are staged
    // and before any product: KC / 32 x RW requests in flight per lane, whose
    // HBM latency overlaps the staging of B from L2
    C a[KC / 32][RW];
#pragma unroll
    for (int j = 0; j < KC / 32; ++j) {
      const int kg = k0 + lane + 32 * j;
#pragma unroll
      for (int r = 0; r < RW; ++r) a[j][r] = (aoff[r] >= 0 && kg < k) ? __ldcs(A.base + aoff[r] + kg) : czero<C>();
    }
    __syncthreads();
    for (int idx = tid; idx < KC * W; idx += 256) {
      const int kk = idx / W, q = idx % W;
      bs[kk][q] = (k0 + kk < k && q < w) ? B.at(k0 + kk, q) : czero<C>();
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < KC / 32; ++j) {
      const int kk = lane + 32 * j;
#pragma unroll
      for (int q = 0; q < W; ++q) {
        const C b = bs[kk][q];
#pragma unroll
        for (int r = 0; r < RW; ++r) {
          acc[r][q].x = fma(a[j][r].x, b.x, acc[r][q].x);
          acc[r][q].x = fma(-a[j][r].y, b.y, acc[r][q].x);
          acc[r][q].y = fma(a[j][r].x, b.y, acc[r][q].y);
          acc[r][q].y = fma(a[j][r].y, b.x, acc[r][q].y);
        }
      }
    }
  }
  const bool use_beta = (beta.x != 0 || beta.y != 0);
#pragma unroll
  for (int r = 0; r < RW; ++r) {
    C mine = czero<C>();
#pragma unroll
    for (int q = 0; q < W; ++q) {
      C v = acc[r][q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
      }
      if (lane == q) mine = v;
    }
    if (aoff[r] >= 0 && lane < w) {
      C& out = Cv.at(row0 + r, lane);
      C v = cmul(alpha, mine);
      if (use_beta) v = cadd(v, cmul(beta, out));
      out = v;
    }
  }
}

template <typename C, int W, int RW>
static int gemm_skinny(const LaContext& ctx, int m, int n, int k, C alpha, RowView<C> A, RowView<C> B, C beta,
                       RowView<C> Cv) {
  const int grid = ceil_div(m, 8 * RW);
  gemm_skinny_kernel<C, W, RW><<<grid, 256, 0, ctx.stream>>>(m, n, k, alpha, A, B, beta, Cv);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

constexpr double kTcMinMacs = 67108864.0;  // 2^26

// Whether gemm_v runs an m x n x k product on the tensor cores (the only path
// that uses the operand workspace ctx.ws).  The tensor-core path pays ~25 us of
// operand preparation, pipeline fill and launches per call: below ~2^26
// multiply-adds (about 400^3) the CUDA-core tiles finish first.
template <typename C>
static bool gemm_takes_tc(const LaContext& ctx, int m, int n, int k) {
  if (m <= 0 || n <= 0 || (n <= 16 && k >= 256)) return false;  // empty, or the skinny path
  if constexpr (sizeof(C) == 8)
    return ctx.engine != GemmEngine::kSimt && k >= 64 && m >= 128 && n >= 64 && (double)m * n * k >= kTcMinMacs;
  return false;
}

template <typename C>
int gemm_v(const LaContext& ctx, int m, int n, int k, C alpha, RowView<C> A, RowView<C> B, C beta, RowView<C> Cv) {
  if (m <= 0 || n <= 0) return BEM200_OK;
  if (n <= 16 && k >= 256) {
    // W: columns rounded up to 4, 8 or 16; rows per warp: few enough that
    // many CTAs (and their loads) are resident, and the sums stay in registers
    constexpr bool z = sizeof(C) == 16;
    if (n <= 4) return gemm_skinny<C, 4, z ? 2 : 2>(ctx, m, n, k, alpha, A, B, beta, Cv);
    if (n <= 8) return gemm_skinny<C, 8, z ? 1 : 2>(ctx, m, n, k, alpha, A, B, beta, Cv);
    return gemm_skinny<C, 16, 1>(ctx, m, n, k, alpha, A, B, beta, Cv);
  }
  if constexpr (sizeof(C) == 8) {
    if (gemm_takes_tc<C>(ctx, m, n, k)) return gemm_tc_c64(ctx, m, n, k, alpha, A, B, beta, Cv);
  }
  constexpr int BK = sizeof(C) == 16 ? 8 : 16;
  if ((long long)ceil_div(n, 32) * ceil_div(m, 32) < 74) {  // 32 x 32 tiles would fill fewer than half the SMs
    dim3 grid(ceil_div(n, 16), ceil_div(m, 16));
    gemm_simt_kernel<C, 32, 1><<<grid, 256, 0, ctx.stream>>>(m, n, k, alpha, A, B, beta, Cv);
    BEM_LAUNCH_CHECK();
    return BEM200_OK;
  }
  if ((long long)ceil_div(n, 64) * ceil_div(m, 64) < 296) {  // fewer than two 64 x 64 tiles per SM
    dim3 grid(ceil_div(n, 32), ceil_div(m, 32));
    BEM_REQUIRE(grid.y <= 65535, BEM200_ERR_ARG, "gemm: m too large");
    gemm_simt_kernel<C, 2 * BK, 2><<<grid, 256, 0, ctx.stream>>>(m, n, k, alpha, A, B, beta, Cv);
    BEM_LAUNCH_CHECK();
    return BEM200_OK;
  }
  dim3 grid(ceil_div(n, 64), ceil_div(m, 64));
  BEM_REQUIRE(grid.y <= 65535, BEM200_ERR_ARG, "gemm: m too large");
  gemm_simt_kernel<C, BK><<<grid, 256, 0, ctx.stream>>>(m, n, k, alpha, A, B, beta, Cv);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// ===================================================================== panel LU
// Factor logical rows [0, m) x columns [0, w) of view (map, col) with partial
// pivoting and no row movement.  The cluster's CTA `rank` keeps panel rows
// [rank R, rank R + R) in shared memory; warp w owns rows r = w (mod 8) and
// lane c owns panel column c.
constexpr int kPanelNB = 32;
constexpr int kPanelWarps = 16;
constexpr int kPanelThreads = 32 * kPanelWarps;
constexpr int kPanelUnroll = 4;

template <typename C>
struct PanelShared {
  R_t<C> wval[kPanelWarps];        // per-warp candidates of the current column
  int wrow[kPanelWarps];
  R_t<C> cval[2];                  // this CTA's published candidate (double buffered)
  int crow[2];
  C crowdata[2][kPanelNB];         // ... and its row
  int p;                           // pivot (panel row) of the current column
  C prow[kPanelNB];                // pivot row of the current column
  int perm[kPanelNB];
  int singular;
  int mk[2 * kPanelNB];
  int mv[2 * kPanelNB];
  int mo[2 * kPanelNB];
};

// pivot magnitude; NaN counts as 0 so that every unused row stays selectable
__device__ __forceinline__ double pmag(double2 a) {
  double v = fabs(a.x) + fabs(a.y);
  return v >= 0 ? v : 0.0;
}
__device__ __forceinline__ float pmag(float2 a) {
  float v = fabsf(a.x) + fabsf(a.y);
  return v >= 0 ? v : 0.f;
}

template <typename C>
__device__ __forceinline__ void cand_merge(R_t<C>& b, int& br, R_t<C> v, int rw) {
  if (v > b || (v == b && rw < br)) {
    b = v;
    br = rw;
  }
}


// Replay the panel's pivot sequence perm[0..w) (panel rows) as LAPACK row
// swaps on a position map with <= 2w entries held in the registers of one
// warp (two slots per lane), write ipiv, and move the rowmap entries of the
// swapped positions.  Called by a full warp.
__device__ void replay_pivots(int w, const int* __restrict__ perm, int32_t* __restrict__ ipiv, int ipiv_base,
                              int32_t* __restrict__ rowmap) {
  const int lane = threadIdx.x & 31;
  int key[2] = {-1, -1}, val[2] = {-1, -1};
  int nmap = 0;
  auto find = [&](const int (&arr)[2], int x, int& slot) -> bool {
    unsigned m0 = __ballot_sync(0xffffffffu, arr[0] == x);
    unsigned m1 = __ballot_sync(0xffffffffu, arr[1] == x);
    if (m0) { slot = __ffs(m0) - 1; return true; }
    if (m1) { slot = 32 + __ffs(m1) - 1; return true; }
    return false;
  };
  auto get = [&](const int (&arr)[2], int slot) -> int {
    return __shfl_sync(0xffffffffu, slot < 32 ? arr[0] : arr[1], slot & 31);
  };
  auto put = [&](int pos, int prow) {
    int slot;
    if (!find(key, pos, slot)) {
      slot = nmap++;
      if (lane == (slot & 31)) key[slot >> 5] = pos;
    }
    if (lane == (slot & 31)) val[slot >> 5] = prow;
  };
  for (int t = 0; t < w; ++t) {
    const int q = perm[t];
    int slot;
    const int pp = find(val, q, slot) ? get(key, slot) : q;     // current position of panel row q
    const int at_t = find(key, t, slot) ? get(val, slot) : t;   // panel row at position t
    put(t, q);
    put(pp, at_t);
    if (lane == 0) ipiv[t] = ipiv_base + pp;
  }
  // new rowmap[pos] = old rowmap[panel row now at pos]
  int mo[2];
  for (int k = 0; k < 2; ++k) mo[k] = (key[k] >= 0) ? rowmap[val[k]] : 0;
  __syncwarp();
  for (int k = 0; k < 2; ++k)
    if (key[k] >= 0) rowmap[key[k]] = mo[k];
}

template <typename C>
__device__ __forceinline__ void warp_argmax(R_t<C>& b, int& br) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    cand_merge<C>(b, br, __shfl_xor_sync(0xffffffffu, b, o), __shfl_xor_sync(0xffffffffu, br, o));
}

// Per column: warps publish candidates in shared memory; warp 0 reduces them,
// publishes the CTA's best row, and after ONE cluster barrier gathers the
// cs candidates (one remote load per lane) and the winning row (one more
// remote load per lane); everyone else reads the result from local shared
// memory.  Published slots are double buffered: a slot is rewritten two
// columns later, after every CTA has passed the next barrier.
template <typename C>
__global__ void __launch_bounds__(kPanelThreads) panel_lu_kernel(int m, int w, C* __restrict__ A, long long ld,
                                                                 int col, int32_t* __restrict__ rowmap,
                                                                 int32_t* __restrict__ ipiv, int ipiv_base,
                                                                 int* __restrict__ info, int R) {
  using Real = R_t<C>;
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* rows = reinterpret_cast<C*>(smem_raw);                                   // R x 32
  int32_t* phys = reinterpret_cast<int32_t*>(rows + (size_t)R * kPanelNB);    // R
  uint8_t* used = reinterpret_cast<uint8_t*>(phys + R);                       // R
  __shared__ PanelShared<C> sh;
  const int r0 = rank * R;
  const int rcount = max(0, min(R, m - r0));
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

  for (int r = tid; r < rcount; r += kPanelThreads) {
    phys[r] = rowmap[r0 + r];
    used[r] = 0;
  }
  __syncthreads();
  for (int idx = tid; idx < rcount * kPanelNB; idx += kPanelThreads) {
    int r = idx >> 5, c = idx & 31;
    rows[idx] = (c < w) ? A[(long long)phys[r] * ld + col + c] : czero<C>();
  }
  if (tid == 0) sh.singular = 0;
  __syncthreads();

  // candidates for column 0
  Real best = -1;
  int brow = INT_MAX;
  for (int r = wid + kPanelWarps * lane; r < rcount; r += 32 * kPanelWarps)
    cand_merge<C>(best, brow, pmag(rows[r * kPanelNB]), r);
  warp_argmax<C>(best, brow);

  for (int t = 0; t < w; ++t) {
    const int buf = t & 1;
    if (lane == 0) {
      sh.wval[wid] = best;
      sh.wrow[wid] = brow;  // local row index
    }
    __syncthreads();
    if (wid == 0) {
      Real b = lane < kPanelWarps ? sh.wval[lane] : (Real)-1;
      int br = lane < kPanelWarps ? sh.wrow[lane] : INT_MAX;
      warp_argmax<C>(b, br);
      sh.crowdata[buf][lane] = (br < rcount) ? rows[br * kPanelNB + lane] : czero<C>();
      if (lane == 0) {
        sh.cval[buf] = (br < rcount) ? b : (Real)-1;
        sh.crow[buf] = (br < rcount) ? r0 + br : INT_MAX;
      }
    }
    if (cs > 1) cluster.sync(); else __syncthreads();
    if (wid == 0) {
      Real b = -1;
      int br = INT_MAX;
      if (lane < cs) {
        const PanelShared<C>* rs = (cs > 1) ? cluster.map_shared_rank(&sh, lane) : &sh;
        b = rs->cval[buf];
        br = rs->crow[buf];
      }
      warp_argmax<C>(b, br);
      // every step has an unused row, each with magnitude >= 0 > -1: br < m
      const int p = min(br, m - 1);
      const int owner = p / R;
      const PanelShared<C>* os = (cs > 1) ? cluster.map_shared_rank(&sh, owner) : &sh;
      sh.prow[lane] = os->crowdata[buf][lane];
      if (lane == 0) {
        sh.p = p;
        sh.perm[t] = p;
        if (!(b > 0) && !sh.singular) sh.singular = t + 1;
      }
    }
    __syncthreads();
    const int p = sh.p;
    const int owner = p / R, lr = p - owner * R;
    const C pc = sh.prow[lane];
    const C piv = shfl_c(pc, t);
    const bool ok = cabs1(piv) > 0;
    // multipliers use the reciprocal of the pivot, as LAPACK's scaling does
    const C inv = ok ? cdiv(cmake<C>(1.0, 0.0), piv) : czero<C>();
    // update the unused rows owned by this warp (kPanelUnroll rows in flight,
    // straight-line selects); track candidates for column t + 1
    best = -1;
    brow = INT_MAX;
    const bool at_t = lane == t, after_t = lane > t, next_t = lane == t + 1;
    for (int rb = wid; rb < rcount; rb += kPanelWarps * kPanelUnroll) {
      C v[kPanelUnroll];
      bool act[kPanelUnroll];
      int rr[kPanelUnroll];
#pragma unroll
      for (int u = 0; u < kPanelUnroll; ++u) {
        const int r = rb + u * kPanelWarps;
        const bool in = r < rcount;
        rr[u] = in ? r : rb;
        const bool is_piv = in && rank == owner && r == lr;
        if (is_piv && lane == 0) used[r] = 1;
        act[u] = in && !is_piv && (used[rr[u]] == 0);
        v[u] = rows[rr[u] * kPanelNB + lane];
      }
#pragma unroll
      for (int u = 0; u < kPanelUnroll; ++u) {
        const C l = cmul(shfl_c(v[u], t), inv);
        const C upd = csub(v[u], cmul(l, pc));
        C r = v[u];
        r.x = after_t ? upd.x : r.x;
        r.y = after_t ? upd.y : r.y;
        r.x = at_t ? l.x : r.x;
        r.y = at_t ? l.y : r.y;
        v[u] = r;
        const Real a = (act[u] && next_t) ? pmag(r) : (Real)-1;
        const bool take = a > best || (a == best && a >= 0 && rr[u] < brow);
        best = take ? a : best;
        brow = take ? rr[u] : brow;
      }
#pragma unroll
      for (int u = 0; u < kPanelUnroll; ++u)
        if (act[u]) rows[rr[u] * kPanelNB + lane] = v[u];
    }
    if (t + 1 < w) {
      best = __shfl_sync(0xffffffffu, best, t + 1);
      brow = __shfl_sync(0xffffffffu, brow, t + 1);
    }
  }
  // no CTA may leave while others can still read its published slots
  if (cs > 1) cluster.sync(); else __syncthreads();
  for (int idx = tid; idx < rcount * kPanelNB; idx += kPanelThreads) {
    int r = idx >> 5, c = idx & 31;
    if (c < w) A[(long long)phys[r] * ld + col + c] = rows[idx];
  }
  if (rank == 0 && wid == 0) {
    replay_pivots(w, sh.perm, ipiv, ipiv_base, rowmap);
    if (lane == 0 && sh.singular && info) atomicCAS(info, 0, ipiv_base + sh.singular);
  }
}

// ----------------------------------------------------------------------------
// Register-resident panel: warp w of CTA `rank` holds panel rows
// r = w + 8 j (j < kRegRows) of the CTA's R rows, lane c holding column c, so a
// column step is shuffles and FMAs only.  Candidate exchange as above: each
// warp publishes its best row, warp 0 reduces, one cluster barrier, warp 0
// gathers the cs candidates and the winning row.
constexpr int kRegWarps = 8;
constexpr int kRegThreads = 32 * kRegWarps;
// rows per warp: 48 for complex64, 32 for complex128 (register budget)
template <typename C> struct RegRows { static constexpr int value = 48; };
template <> struct RegRows<double2> { static constexpr int value = 32; };
constexpr int kRegRowsMax = 48;

template <typename C>
struct RegPanelShared {
  R_t<C> wval[kRegWarps];
  int wrow[kRegWarps];
  C wrowdata[2][kRegWarps][kPanelNB];  // each warp's best row (double buffered)
  R_t<C> cval[2];
  int crow[2];
  int cwarp[2];
  int p;
  C prow[kPanelNB];
  int perm[kPanelNB];
  int singular;
  int mk[2 * kPanelNB];
  int mv[2 * kPanelNB];
  int mo[2 * kPanelNB];
  int32_t phys[kRegWarps * kRegRowsMax];  // storage rows of this CTA's panel rows
};

template <typename C>
__global__ void __launch_bounds__(kRegThreads, 1) panel_lu_reg_kernel(int m, int w, C* __restrict__ A, long long ld,
                                                                      int col, int32_t* __restrict__ rowmap,
                                                                      int32_t* __restrict__ ipiv, int ipiv_base,
                                                                      int* __restrict__ info, int R) {
  using Real = R_t<C>;
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  __shared__ RegPanelShared<C> sh;
  const int r0 = rank * R;
  const int rcount = max(0, min(R, m - r0));
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nmine = rcount > wid ? (rcount - wid + kRegWarps - 1) / kRegWarps : 0;  // rows of this warp

  constexpr int kRegRows = RegRows<C>::value;
  for (int r = tid; r < rcount; r += kRegThreads) sh.phys[r] = rowmap[r0 + r];
  if (tid == 0) sh.singular = 0;
  __syncthreads();
  C v[kRegRows];
  uint64_t active = 0;
#pragma unroll
  for (int j = 0; j < kRegRows; ++j) {
    v[j] = czero<C>();
    if (j < nmine) {
      const int r = wid + kRegWarps * j;
      if (lane < w) v[j] = A[(long long)sh.phys[r] * ld + col + lane];
      active |= 1ull << j;
    }
  }

  // straight-line code (selects, no branches) so the unrolled rows interleave
  auto warp_cand = [&](int c, Real& b, int& bj) {
    b = -1;
    bj = INT_MAX;
#pragma unroll
    for (int j = 0; j < kRegRows; ++j) {
      const Real a = ((active >> j) & 1ull) ? pmag(v[j]) : (Real)-1;
      const bool take = a > b;  // rows are visited in increasing j: first max wins
      b = take ? a : b;
      bj = take ? j : bj;
    }
    b = __shfl_sync(0xffffffffu, b, c);
    bj = __shfl_sync(0xffffffffu, bj, c);
  };
  Real best;
  int bj;
  warp_cand(0, best, bj);

  for (int t = 0; t < w; ++t) {
    const int buf = t & 1;
    // publish this warp's candidate (value, local row, row data)
    C sel = czero<C>();
#pragma unroll
    for (int j = 0; j < kRegRows; ++j) {
      sel.x = (j == bj) ? v[j].x : sel.x;
      sel.y = (j == bj) ? v[j].y : sel.y;
    }
    sh.wrowdata[buf][wid][lane] = sel;
    if (lane == 0) {
      sh.wval[wid] = best;
      sh.wrow[wid] = bj < nmine ? wid + kRegWarps * bj : INT_MAX;
    }
    __syncthreads();
    if (wid == 0) {
      Real b = lane < kRegWarps ? sh.wval[lane] : (Real)-1;
      int br = lane < kRegWarps ? sh.wrow[lane] : INT_MAX;
      warp_argmax<C>(b, br);
      if (lane == 0) {
        sh.cval[buf] = br < rcount ? b : (Real)-1;
        sh.crow[buf] = br < rcount ? r0 + br : INT_MAX;
        sh.cwarp[buf] = br < rcount ? br % kRegWarps : 0;
      }
    }
    if (cs > 1) cluster.sync(); else __syncthreads();
    if (wid == 0) {
      Real b = -1;
      int br = INT_MAX;
      if (lane < cs) {
        const RegPanelShared<C>* rs = (cs > 1) ? cluster.map_shared_rank(&sh, lane) : &sh;
        b = rs->cval[buf];
        br = rs->crow[buf];
      }
      warp_argmax<C>(b, br);
      const int p = min(br, m - 1);  // an unused row always exists: br < m
      const int owner = p / R;
      const RegPanelShared<C>* os = (cs > 1) ? cluster.map_shared_rank(&sh, owner) : &sh;
      sh.prow[lane] = os->wrowdata[buf][os->cwarp[buf]][lane];
      if (lane == 0) {
        sh.p = p;
        sh.perm[t] = p;
        if (!(b > 0) && !sh.singular) sh.singular = t + 1;
      }
    }
    __syncthreads();
    const int p = sh.p;
    const int owner = p / R, lr = p - owner * R;
    if (rank == owner && (lr % kRegWarps) == wid) active &= ~(1ull << (lr / kRegWarps));
    const C pc = sh.prow[lane];
    const C piv = shfl_c(pc, t);
    const bool ok = cabs1(piv) > 0;
    const C inv = ok ? cdiv(cmake<C>(1.0, 0.0), piv) : czero<C>();
    const bool at_t = lane == t, after_t = lane > t;
#pragma unroll
    for (int j = 0; j < kRegRows; ++j) {
      const C l = cmul(shfl_c(v[j], t), inv);
      const C u = csub(v[j], cmul(l, pc));
      const bool act = (active >> j) & 1ull;
      C r = v[j];
      r.x = after_t ? u.x : r.x;
      r.y = after_t ? u.y : r.y;
      r.x = at_t ? l.x : r.x;
      r.y = at_t ? l.y : r.y;
      v[j].x = act ? r.x : v[j].x;
      v[j].y = act ? r.y : v[j].y;
    }
    if (t + 1 < w) warp_cand(t + 1, best, bj);
  }
  if (cs > 1) cluster.sync(); else __syncthreads();
#pragma unroll
  for (int j = 0; j < kRegRows; ++j)
    if (j < nmine && lane < w) A[(long long)sh.phys[wid + kRegWarps * j] * ld + col + lane] = v[j];
  if (rank == 0 && wid == 0) {
    replay_pivots(w, sh.perm, ipiv, ipiv_base, rowmap);
    if (lane == 0 && sh.singular && info) atomicCAS(info, 0, ipiv_base + sh.singular);
  }
}

// ----------------------------------------------------------------------------
// Push panel: one panel row per thread, held in registers (32 complex), with
// the column loop fully unrolled so every register index is static.  Per
// column: warp argmax -> the winning lane parks its row in shared memory ->
// warp 0 picks the CTA's best row and PUSHES it (value, index, 32 elements)
// into the candidate slot of every CTA of the cluster with DSMEM stores ->
// one cluster barrier -> every warp reduces the cs candidates from its own
// shared memory and applies the update with the winning row.  Nothing is read
// remotely, so the barrier is the only cluster-wide latency per column.
// Candidate slots are double buffered: slot t & 1 is rewritten at column t + 2,
// after every CTA has passed barrier t + 1 and thus finished reading it.
constexpr int kPushThreads = 384;
constexpr int kPushWarps = kPushThreads / 32;
constexpr int kPushMaxCluster = 16;

template <typename C>
struct PushShared {
  C cand[2][kPushMaxCluster][kPanelNB];
  R_t<C> cval[2][kPushMaxCluster];
  int crow[2][kPushMaxCluster];
  C wrow[kPushWarps][kPanelNB];
  R_t<C> wval[kPushWarps];
  int widx[kPushWarps];
  int perm[kPanelNB];
  int singular;
};

template <typename C>
__global__ void __launch_bounds__(kPushThreads, 1) panel_lu_push_kernel(int m, int w, C* __restrict__ A, long long ld,
                                                                        int col, int32_t* __restrict__ rowmap,
                                                                        int32_t* __restrict__ ipiv, int ipiv_base,
                                                                        int* __restrict__ info, int R) {
  using Real = R_t<C>;
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  __shared__ PushShared<C> sh;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int r0 = rank * R;
  const int rcount = max(0, min(R, m - r0));
  const int prow_id = r0 + tid;  // panel row of this thread
  bool act = tid < rcount;
  const long long phys = act ? (long long)rowmap[prow_id] : 0;
  C v[kPanelNB];
#pragma unroll
  for (int c = 0; c < kPanelNB; ++c) v[c] = (act && c < w) ? A[phys * ld + col + c] : czero<C>();
  if (tid == 0) sh.singular = 0;
  const unsigned kFull = 0xffffffffu;

  // The column loop stays rolled (a fully unrolled one overflows the
  // instruction cache); column t of the register row is read with a select
  // chain and updated with predicated FMAs, so every register index is static.
#pragma unroll 1
  for (int t = 0; t < w; ++t) {
    const int buf = t & 1;
    C vt = v[0];
#pragma unroll
    for (int c = 1; c < kPanelNB; ++c)
      if (c == t) vt = v[c];
    // warp candidate; the winning lane parks its row in shared memory
    Real wb = act ? pmag(vt) : (Real)-1;
    int wi = act ? prow_id : INT_MAX;
    warp_argmax<C>(wb, wi);
    if (act && wi == prow_id) {
#pragma unroll
      for (int c = 0; c < kPanelNB; ++c) sh.wrow[wid][c] = v[c];
    }
    if (lane == 0) {
      sh.wval[wid] = wb;
      sh.widx[wid] = wi;
    }
    __syncthreads();
    {  // CTA candidate (every warp), pushed to the cluster: warp w serves CTAs w, w + nwarps, ...
      Real b = lane < nwarps ? sh.wval[lane] : (Real)-1;
      int bi = lane < nwarps ? sh.widx[lane] : INT_MAX;
      const Real b0 = b;
      const int i0 = bi;
      warp_argmax<C>(b, bi);
      const unsigned msk = __ballot_sync(kFull, lane < nwarps && i0 == bi && b0 == b);
      const int ww = msk ? __ffs(msk) - 1 : 0;
      const C e = sh.wrow[ww][lane];
      const Real bv = (bi != INT_MAX) ? b : (Real)-1;
      for (int d = wid; d < cs; d += nwarps) {
        PushShared<C>* dst = (cs > 1) ? cluster.map_shared_rank(&sh, d) : &sh;
        dst->cand[buf][rank][lane] = e;
        if (lane == 0) {
          dst->cval[buf][rank] = bv;
          dst->crow[buf][rank] = bi;
        }
      }
    }
    if (cs > 1) cluster.sync(); else __syncthreads();
    // cluster winner (every warp reduces the cs candidates itself)
    Real b = lane < cs ? sh.cval[buf][lane] : (Real)-1;
    int bi = lane < cs ? sh.crow[buf][lane] : INT_MAX;
    const Real b0 = b;
    const int i0 = bi;
    warp_argmax<C>(b, bi);
    const unsigned msk = __ballot_sync(kFull, lane < cs && i0 == bi && b0 == b);
    const int wc = msk ? __ffs(msk) - 1 : 0;
    const int p = min(bi, m - 1);  // an unused row always exists: bi < m
    if (tid == 0) {
      sh.perm[t] = p;
      if (!(b > 0) && !sh.singular) sh.singular = t + 1;
    }
    const C* prow = sh.cand[buf][wc];
    const C piv = prow[t];
    // multipliers use the reciprocal of the pivot, as LAPACK's scaling does
    const C inv = cabs1(piv) > 0 ? cdiv(cmake<C>(1.0, 0.0), piv) : czero<C>();
    if (prow_id == p) act = false;  // the pivot row becomes a row of U
    if (act) {
      const C l = cmul(vt, inv);
#pragma unroll
      for (int g = 0; g < kPanelNB; g += 8) {
        if (g + 7 >= t) {  // uniform: skip groups left of the pivot column
#pragma unroll
          for (int c = g; c < g + 8; ++c) {
            const C u = csub(v[c], cmul(l, prow[c]));
            v[c] = (c > t) ? u : ((c == t) ? l : v[c]);
          }
        }
      }
    }
  }
  // every remote store happened before the last barrier: no CTA touches
  // another's shared memory from here on
  if (tid < rcount) {
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c)
      if (c < w) A[phys * ld + col + c] = v[c];
  }
  __syncthreads();
  if (rank == 0 && wid == 0) {
    replay_pivots(w, sh.perm, ipiv, ipiv_base, rowmap);
    if (lane == 0 && sh.singular && info) atomicCAS(info, 0, ipiv_base + sh.singular);
  }
}

// ----------------------------------------------------------------------------
// Asynchronous push panel (complex64): the push panel's layout (one panel row
// per thread, in registers) with the cluster barrier of every column replaced
// by one-way DSMEM messages, and the rank-1 update of the remaining columns
// moved off the pivot search's critical path.
//  * Exchange: the warp holding the CTA's best row sends it (32 elements and
//    a 16-byte header: key, row, multiplier) to slot t % 3 of every CTA with
//    st.async, which signals the receiver's mbarrier (complete_tx).  Each CTA
//    arms its own barrier for cs * 272 bytes and waits for it; nobody waits
//    for an acknowledgement.  A CTA sends column t + 1 only after it received
//    all of column t, so a slot is rewritten only after every CTA has read it.
//  * Deferred update: after sending column t's candidate, a thread applies
//    pivot t - 1 to its columns > t while the candidates travel.  The column
//    that decides the next pivot (t + 1) is updated right after the pivot is
//    known.  Sent rows therefore lack pivot t - 1 in their columns > t; the
//    header carries their multiplier l, and every CTA rebuilds the pivot row
//    F = P - l F_prev (warp 0, one element per lane) for the next update.
//  * Keys: 1 + the bit pattern of |re| + |im| (monotonic for non-negative
//    floats; 0 = no candidate), reduced with redux.sync; equal keys go to the
//    lowest row, as LAPACK's first maximum.
//  * Multipliers use an approximate reciprocal of |pivot|^2 (rcp.approx);
//    the factors are preconditioners of the refinement, so they differ from
//    the exact-division ones in the last bits only.
// Every mbarrier wait is bounded; on timeout the CTA records it, finishes
// its loop without waiting and the status (or *info = -BEM200_ERR_TIMEOUT)
// reports it.  A final cluster barrier keeps every CTA alive until all have
// sent their last messages.
constexpr int kAsyncThreads = 384;
constexpr int kAsyncWarps = kAsyncThreads / 32;
constexpr int kAsyncMaxCluster = 16;
constexpr int kAsyncSpin = 1 << 22;

struct __align__(16) AsyncHdr {
  unsigned key;
  int row;
  float lx, ly;
};

struct AsyncShared {
  float2 cand[3][kAsyncMaxCluster][kPanelNB];  // received candidate rows, by slot and sender
  AsyncHdr hdr[3][kAsyncMaxCluster];
  uint64_t bar[3];
  float2 F[2][kPanelNB];  // pivot rows with the previous pivot applied
  float2 Q[2][kPanelNB];  // (-F.y, F.x), for the packed update
  float2 park[kPanelNB];  // the CTA winner's row, staged for its warp
  unsigned wkey[2][kAsyncWarps];
  int wrow[2][kAsyncWarps];
  float2 wl[2][kAsyncWarps];
  int perm[kPanelNB];
  int singular;
  int timeout;
};

__device__ __forceinline__ uint32_t as_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t dsmem_map(uint32_t a, int rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_async_f2(uint32_t ra, float2 v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];" ::"r"(ra),
               "f"(v.x), "f"(v.y), "r"(rbar)
               : "memory");
}
__device__ __forceinline__ void st_async_v4(uint32_t ra, uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                            uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                   ra),
               "r"(a), "r"(b), "r"(c), "r"(d), "r"(rbar)
               : "memory");
}
__device__ __forceinline__ void async_bar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(as_smem(b)));
}
__device__ __forceinline__ void async_bar_arm(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(as_smem(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool async_bar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(as_smem(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned redux_max_u32(unsigned v) {
  unsigned r;
  asm volatile("redux.sync.max.u32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
  return r;
}
__device__ __forceinline__ unsigned long long f2_bits(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 bits_f2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
// c - a * b as two packed FMAs (fma.rn.f32x2); q = (-b.y, b.x)
__device__ __forceinline__ float2 cfms_packed(float2 c, float2 a, float2 b, float2 q) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(make_float2(-a.x, -a.x))), "l"(f2_bits(b)),
      "l"(f2_bits(c)));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(make_float2(-a.y, -a.y))), "l"(f2_bits(q)), "l"(d));
  return bits_f2(d);
}
__device__ __forceinline__ float2 crecip_approx(float2 p) {
  const float d = p.x * p.x + p.y * p.y;
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  return d > 0.f ? make_float2(p.x * r, -p.y * r) : make_float2(0.f, 0.f);
}
__device__ __forceinline__ unsigned async_key(bool act, float2 a) { return act ? 1u + __float_as_uint(pmag(a)) : 0u; }

__global__ void __launch_bounds__(kAsyncThreads, 1)
    panel_lu_async_kernel(int m, int w, float2* __restrict__ A, long long ld, int col, int32_t* __restrict__ rowmap,
                          int32_t* __restrict__ ipiv, int ipiv_base, int* __restrict__ info,
                          int* __restrict__ status, int R) {
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  __shared__ AsyncShared sh;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nwarps = (int)(blockDim.x >> 5);
  const int r0 = rank * R;
  const int rcount = max(0, min(R, m - r0));
  const int prow_id = r0 + tid;
  bool act = tid < rcount;
  float2* arow = A + (act ? (long long)rowmap[prow_id] * ld : 0) + col;
  float2 v[kPanelNB];
#pragma unroll
  for (int c = 0; c < kPanelNB; ++c) v[c] = (act && c < w) ? arow[c] : czero<float2>();
  if (tid == 0) {
    sh.singular = 0;
    sh.timeout = 0;
    for (int i = 0; i < 3; ++i) async_bar_init(&sh.bar[i]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < kPanelNB) sh.F[1][tid] = sh.Q[1][tid] = czero<float2>();
  float2 cur = v[0], lprev = czero<float2>(), ucur = czero<float2>();
  int td = -1;
  bool timed_out = false;
  const uint32_t bytes = (uint32_t)cs * (uint32_t)(kPanelNB * sizeof(float2) + sizeof(AsyncHdr));
  cluster.sync();  // barriers initialised in every CTA before the first message

#pragma unroll 1
  for (int t = 0; t < w; ++t) {
    const int s = t % 3, b = t & 1;
    if (tid == 0) async_bar_arm(&sh.bar[s], bytes);
    // warp candidate
    const unsigned key = async_key(act, cur);
    const unsigned wk = redux_max_u32(key);
    const int wl = __ffs(__ballot_sync(0xffffffffu, key == wk)) - 1;
    if (lane == wl) sh.wl[b][wid] = lprev;
    if (lane == 0) {
      sh.wkey[b][wid] = wk;
      sh.wrow[b][wid] = wk ? r0 + wid * 32 + wl : INT_MAX;
    }
    __syncthreads();
    // CTA candidate: its warp stages the row and sends it to every CTA
    const unsigned k2 = lane < nwarps ? sh.wkey[b][lane] : 0u;
    const unsigned ck = redux_max_u32(k2);
    const int ww = __ffs(__ballot_sync(0xffffffffu, lane < nwarps && k2 == ck)) - 1;
    if (wid == ww) {
      if (lane == wl && key != 0) {
#pragma unroll
        for (int c = 0; c < kPanelNB; ++c) sh.park[c] = v[c];
        sh.park[t] = cur;
      }
      __syncwarp();
      const float2 e = sh.park[lane];
      const float2 lw = sh.wl[b][ww];
      const uint32_t la = as_smem(&sh.cand[s][rank][lane]), lh = as_smem(&sh.hdr[s][rank]),
                     lb = as_smem(&sh.bar[s]);
      for (int d = 0; d < cs; ++d) {
        const uint32_t rb = dsmem_map(lb, d);
        st_async_f2(dsmem_map(la, d), e, rb);
        if (lane == 0)
          st_async_v4(dsmem_map(lh, d), ck, (uint32_t)sh.wrow[b][ww], __float_as_uint(lw.x), __float_as_uint(lw.y),
                      rb);
      }
    }
    // while the candidates travel: pivot t - 1 on this row's columns > t
    if (act && t > 0) {
      const float2* F = sh.F[b ^ 1];
      const float2* Q = sh.Q[b ^ 1];
#pragma unroll
      for (int g = 0; g < kPanelNB; g += 8) {
        if (g + 7 > t) {
#pragma unroll
          for (int c = g; c < g + 8; ++c)
            if (c > t) v[c] = cfms_packed(v[c], lprev, F[c], Q[c]);
        }
      }
    }
    float2 nxt = v[0];
#pragma unroll
    for (int c = 1; c < kPanelNB; ++c)
      if (c == t + 1) nxt = v[c];
    // every CTA's candidate for column t has arrived
    if (!timed_out) {
      bool ok = false;
      for (int it = 0; it < kAsyncSpin; ++it) {
        if (async_bar_try(&sh.bar[s], (uint32_t)(t / 3) & 1u)) {
          ok = true;
          break;
        }
        if (it > 64) __nanosleep(32);
      }
      if (!ok) {
        timed_out = true;
        sh.timeout = 1;
      }
    }
    const unsigned k3 = lane < cs ? sh.hdr[s][lane].key : 0u;
    const unsigned gk = redux_max_u32(k3);
    const int wc = __ffs(__ballot_sync(0xffffffffu, lane < cs && k3 == gk)) - 1;
    const AsyncHdr h = sh.hdr[s][wc];
    const int p = min(max(h.row, 0), m - 1);
    const float2* P = sh.cand[s][wc];
    const float2* Fp = sh.F[b ^ 1];
    const float2 lw = t > 0 ? make_float2(h.lx, h.ly) : czero<float2>();
    if (tid == 0) {
      sh.perm[t] = p;
      if (gk <= 1u && !sh.singular) sh.singular = t + 1;
    }
    if (wid == 0) {  // the pivot row with pivot t - 1 applied, for the next column's update
      float2 f = P[lane];
      if (lane > t) f = csub(f, cmul(lw, Fp[lane]));
      sh.F[b][lane] = f;
      sh.Q[b][lane] = make_float2(-f.y, f.x);
    }
    const float2 inv = crecip_approx(P[t]);
    if (act) {
      if (prow_id == p) {  // the pivot row becomes a row of U
        act = false;
        td = t;
        ucur = cur;
      } else {
        const float2 l = cmul(cur, inv);
        arow[t] = l;
        if (t + 1 < w) cur = csub(nxt, cmul(l, csub(P[t + 1], cmul(lw, Fp[t + 1]))));
        lprev = l;
      }
    }
  }
  if (td >= 0) {
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c)
      if (c > td && c < w) arow[c] = v[c];
    arow[td] = ucur;
  }
  cluster.sync();
  if (rank == 0 && wid == 0) {
    replay_pivots(w, sh.perm, ipiv, ipiv_base, rowmap);
    if (lane == 0 && sh.singular && info) atomicCAS(info, 0, ipiv_base + sh.singular);
  }
  if (tid == 0 && sh.timeout) {
    if (status) atomicExch(status, BEM200_ERR_TIMEOUT);
    else if (info) atomicExch(info, -BEM200_ERR_TIMEOUT);
  }
}

// ----------------------------------------------------------------------------
// Grid-wide panel for tall panels (more rows than a 16-CTA cluster holds):
// one row per thread as in the push panel, CTAs spread over the whole GPU and
// launched cooperatively (all resident), one grid barrier per column.  Each
// CTA writes its best candidate (value, panel row, 32 elements) to a double
// buffered global slot before the barrier; after it, warp 0 of every CTA
// reduces the gridDim.x candidates (L2 reads, bypassing L1 so that a slot
// rewritten two columns later is never read stale) and stages the pivot row
// in shared memory.
constexpr int kGridMaxCta = 160;

template <typename C>
struct GridCand {
  C row[kPanelNB];
  R_t<C> val;
  int idx;
};

template <typename C>
__global__ void __launch_bounds__(kPushThreads, 1) panel_lu_grid_kernel(int m, int w, C* __restrict__ A, long long ld,
                                                                        int col, int32_t* __restrict__ rowmap,
                                                                        int32_t* __restrict__ ipiv, int ipiv_base,
                                                                        int* __restrict__ info, int R,
                                                                        GridCand<C>* __restrict__ cand) {
  using Real = R_t<C>;
  cg::grid_group grid = cg::this_grid();
  const int G = (int)gridDim.x, rank = (int)blockIdx.x;
  __shared__ C wrow[kPushWarps][kPanelNB];
  __shared__ Real wval[kPushWarps];
  __shared__ int widx[kPushWarps];
  __shared__ C prow[kPanelNB];
  __shared__ int perm[kPanelNB];
  __shared__ int sp, singular;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int r0 = rank * R;
  const int rcount = max(0, min(R, m - r0));
  const int prow_id = r0 + tid;
  bool act = tid < rcount;
  const long long phys = act ? (long long)rowmap[prow_id] : 0;
  C v[kPanelNB];
#pragma unroll
  for (int c = 0; c < kPanelNB; ++c) v[c] = (act && c < w) ? A[phys * ld + col + c] : czero<C>();
  if (tid == 0) singular = 0;
  const unsigned kFull = 0xffffffffu;
#pragma unroll 1
  for (int t = 0; t < w; ++t) {
    GridCand<C>* slots = cand + (size_t)(t & 1) * G;
    C vt = v[0];
#pragma unroll
    for (int c = 1; c < kPanelNB; ++c)
      if (c == t) vt = v[c];
    Real wb = act ? pmag(vt) : (Real)-1;
    int wi = act ? prow_id : INT_MAX;
    warp_argmax<C>(wb, wi);
    if (act && wi == prow_id) {
#pragma unroll
      for (int c = 0; c < kPanelNB; ++c) wrow[wid][c] = v[c];
    }
    if (lane == 0) {
      wval[wid] = wb;
      widx[wid] = wi;
    }
    __syncthreads();
    if (wid == 0) {
      Real b = lane < nwarps ? wval[lane] : (Real)-1;
      int bi = lane < nwarps ? widx[lane] : INT_MAX;
      const Real b0 = b;
      const int i0 = bi;
      warp_argmax<C>(b, bi);
      const unsigned msk = __ballot_sync(kFull, lane < nwarps && i0 == bi && b0 == b);
      const int ww = msk ? __ffs(msk) - 1 : 0;
      slots[rank].row[lane] = wrow[ww][lane];
      if (lane == 0) {
        slots[rank].val = (bi != INT_MAX) ? b : (Real)-1;
        slots[rank].idx = bi;
      }
      __threadfence();
    }
    grid.sync();
    if (wid == 0) {
      Real b = -1;
      int bi = INT_MAX;
      for (int g = lane; g < G; g += 32) {
        const Real gv = __ldcg(&slots[g].val);
        const int gi = __ldcg(&slots[g].idx);
        if (gv > b || (gv == b && gi < bi)) {
          b = gv;
          bi = gi;
        }
      }
      warp_argmax<C>(b, bi);
      // the CTA that published the winning row
      int own = INT_MAX;
      for (int g = lane; g < G; g += 32)
        if (__ldcg(&slots[g].idx) == bi) own = min(own, g);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) own = min(own, __shfl_xor_sync(kFull, own, o));
      const int wc = own < G ? own : 0;
      const C* src = &slots[wc].row[0];
      C e;
      e.x = __ldcg(&src[lane].x);
      e.y = __ldcg(&src[lane].y);
      prow[lane] = e;
      if (lane == 0) {
        const int p = min(bi, m - 1);  // an unused row always exists: bi < m
        sp = p;
        perm[t] = p;
        if (!(b > 0) && !singular) singular = t + 1;
      }
    }
    __syncthreads();
    const int p = sp;
    const C piv = prow[t];
    const C inv = cabs1(piv) > 0 ? cdiv(cmake<C>(1.0, 0.0), piv) : czero<C>();
    if (prow_id == p) act = false;
    if (act) {
      const C l = cmul(vt, inv);
#pragma unroll
      for (int g8 = 0; g8 < kPanelNB; g8 += 8) {
        if (g8 + 7 >= t) {
#pragma unroll
          for (int c = g8; c < g8 + 8; ++c) {
            const C u = csub(v[c], cmul(l, prow[c]));
            v[c] = (c > t) ? u : ((c == t) ? l : v[c]);
          }
        }
      }
    }
    __syncthreads();  // prow / sp are rewritten by warp 0 in the next column
  }
  if (tid < rcount) {
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c)
      if (c < w) A[phys * ld + col + c] = v[c];
  }
  if (rank == 0 && wid == 0) {
    replay_pivots(w, perm, ipiv, ipiv_base, rowmap);
    if (lane == 0 && singular && info) atomicCAS(info, 0, ipiv_base + singular);
  }
}

// ----------------------------------------------------------------------------
// Tournament-pivoting panel (communication-avoiding LU, Grigori, Demmel & Xiang,
// SIAM J. Matrix Anal. Appl. 32 (2011)) for the complex64 factors, whose
// accuracy is restored by iterative refinement: the pivot rows of a panel are
// chosen with one cluster-wide exchange per panel instead of one per column.
//   1. every CTA of the cluster factors its own rows with partial pivoting
//      (block barriers only) and nominates its (up to) 32 pivot rows;
//   2. CTA 0 gathers the nominated rows' ORIGINAL values and factors them with
//      partial pivoting: its pivot sequence is the panel's, and the pivot rows
//      after elimination are [L11 \ U11];
//   3. every CTA rewrites its rows: pivot rows get their [L11 \ U11] row, the
//      others L21 = A21 U11^-1 from their original values.
// One row per thread (registers); three cluster barriers per panel.
constexpr int kCaluThreads = 512;
constexpr int kCaluWarps = kCaluThreads / 32;
constexpr int kCaluMaxCluster = 16;
constexpr int kCaluMinRows = 512;  // shorter panels fit one CTA: exact partial pivoting (push panel)

template <typename C>
struct CaluShared {
  C wrow[2][kCaluWarps][kPanelNB];  // each warp's best row, double buffered
  R_t<C> wval[2][kCaluWarps];
  int widx[2][kCaluWarps];
  int lperm[kPanelNB];                          // this CTA's local pivot rows (panel row ids)
  int cand[kCaluMaxCluster * kPanelNB];         // CTA 0: nominated rows of every CTA
  int ncand[kCaluMaxCluster];                   // CTA 0: how many each CTA nominated
  int perm[kPanelNB];                           // the panel's pivot rows
  C lu11[kPanelNB][kPanelNB];                   // [L11 \ U11], row t = pivot row t after elimination
  C uinv[kPanelNB];
  int singular;
  int nsteps;
};

// Partial-pivoting LU of the rows held by this CTA's threads (row `rid` in v,
// `act` = thread holds a row), w columns.  Records the pivot row ids in
// piv_out and, when lu_out is set, the pivot rows after elimination.  Returns
// the number of pivot steps taken (fewer than w when the CTA runs out of
// rows).  All threads of the CTA call it.
template <typename C>
__device__ __forceinline__ int calu_local(CaluShared<C>& sh, C (&v)[kPanelNB], bool act, int rid, int w, int* piv_out,
                          C (*lu_out)[kPanelNB], int* singular) {
  using Real = R_t<C>;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned kFull = 0xffffffffu;
  int steps = w;
#pragma unroll 1
  for (int t = 0; t < w; ++t) {
    const int buf = t & 1;
    C vt = v[0];
#pragma unroll
    for (int c = 1; c < kPanelNB; ++c)
      if (c == t) vt = v[c];
    Real wb = act ? pmag(vt) : (Real)-1;
    int wi = act ? rid : INT_MAX;
    warp_argmax<C>(wb, wi);
    if (act && wi == rid) {
#pragma unroll
      for (int c = 0; c < kPanelNB; ++c) sh.wrow[buf][wid][c] = v[c];
    }
    if (lane == 0) {
      sh.wval[buf][wid] = wb;
      sh.widx[buf][wid] = wi;
    }
    __syncthreads();
    Real b = lane < kCaluWarps ? sh.wval[buf][lane] : (Real)-1;
    int bi = lane < kCaluWarps ? sh.widx[buf][lane] : INT_MAX;
    const Real b0 = b;
    const int i0 = bi;
    warp_argmax<C>(b, bi);
    if (bi == INT_MAX) {  // no row left in this CTA (uniform)
      steps = t;
      break;
    }
    const unsigned msk = __ballot_sync(kFull, lane < kCaluWarps && i0 == bi && b0 == b);
    const int ww = msk ? __ffs(msk) - 1 : 0;
    const C* prow = sh.wrow[buf][ww];
    if (threadIdx.x == 0) {
      piv_out[t] = bi;
      if (singular && !(b > 0) && !*singular) *singular = t + 1;
    }
    if (lu_out && wid == 0) lu_out[t][lane] = prow[lane];
    const C piv = prow[t];
    const C inv = cabs1(piv) > 0 ? cdiv(cmake<C>(1.0, 0.0), piv) : czero<C>();
    if (rid == bi) act = false;
    if (act) {
      const C l = cmul(vt, inv);
#pragma unroll
      for (int g = 0; g < kPanelNB; g += 8) {
        if (g + 7 >= t) {
#pragma unroll
          for (int c = g; c < g + 8; ++c) {
            const C u = csub(v[c], cmul(l, prow[c]));
            v[c] = (c > t) ? u : ((c == t) ? l : v[c]);
          }
        }
      }
    }
  }
  return steps;
}

template <typename C>
__global__ void __launch_bounds__(kCaluThreads, 1) panel_calu_kernel(int m, int w, C* __restrict__ A, long long ld,
                                                                    int col, int32_t* __restrict__ rowmap,
                                                                    int32_t* __restrict__ ipiv, int ipiv_base,
                                                                    int* __restrict__ info, int R) {
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  __shared__ CaluShared<C> sh;
  const int tid = threadIdx.x;
  const int r0 = rank * R;
  const int rcount = max(0, min(R, m - r0));
  const int rid = r0 + tid;  // panel row of this thread
  const bool mine = tid < rcount;
  const long long phys = mine ? (long long)rowmap[rid] : 0;
  C v[kPanelNB];
#pragma unroll
  for (int c = 0; c < kPanelNB; ++c) v[c] = (mine && c < w) ? A[phys * ld + col + c] : czero<C>();
  if (tid == 0) sh.singular = 0;
  __syncthreads();
  // 1. local partial pivoting; nominate the pivot rows to CTA 0
  const int nloc = calu_local<C>(sh, v, mine, rid, w, sh.lperm, nullptr, nullptr);
  __syncthreads();  // thread 0 wrote the last pivot after the last barrier of the sweep
  {
    CaluShared<C>* dst = cluster.map_shared_rank(&sh, 0);
    if (tid < nloc) dst->cand[rank * kPanelNB + tid] = sh.lperm[tid];
    if (tid == 0) dst->ncand[rank] = nloc;
  }
  cluster.sync();
  // 2. CTA 0: the tournament over the nominated rows' original values
  if (rank == 0) {
    int k = tid, src = -1;
    for (int r = 0; r < cs && src < 0; ++r) {
      if (k < sh.ncand[r]) src = sh.cand[r * kPanelNB + k];
      else k -= sh.ncand[r];
    }
    const bool have = src >= 0;
    const long long sp = have ? (long long)rowmap[src] : 0;
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c) v[c] = (have && c < w) ? A[sp * ld + col + c] : czero<C>();
    const int steps = calu_local<C>(sh, v, have, have ? src : INT_MAX - 1 - tid, w, sh.perm, sh.lu11, &sh.singular);
    if (tid == 0) sh.nsteps = steps;
  }
  cluster.sync();
  // 3. every CTA: pivot rows take [L11 \ U11], the others L21 = A21 U11^-1
  if (rank != 0) {
    const CaluShared<C>* src = cluster.map_shared_rank(&sh, 0);
    for (int idx = tid; idx < kPanelNB * kPanelNB; idx += kCaluThreads) {
      const int r = idx / kPanelNB, c = idx % kPanelNB;
      sh.lu11[r][c] = src->lu11[r][c];
    }
    if (tid < kPanelNB) sh.perm[tid] = src->perm[tid];
    if (tid == 0) sh.nsteps = src->nsteps;
  }
  cluster.sync();  // CTA 0's shared memory is no longer read remotely after this point
  if (tid < kPanelNB) {
    const C d = sh.lu11[tid][tid];
    sh.uinv[tid] = (tid < w && cabs1(d) > 0) ? cdiv(cmake<C>(1.0, 0.0), d) : czero<C>();
  }
  __syncthreads();
  if (mine) {
    int t_own = -1;
    for (int t = 0; t < w; ++t)
      if (sh.perm[t] == rid) t_own = t;
    if (t_own >= 0) {
      for (int c = 0; c < w; ++c) A[phys * ld + col + c] = sh.lu11[t_own][c];
    } else {
      // x U11 = a for the original row a: x_k = a_k / U_kk, then a_c -= x_k U_kc
      // (c > k); columns >= w hold zeros and stay zero
#pragma unroll
      for (int c = 0; c < kPanelNB; ++c) v[c] = (c < w) ? A[phys * ld + col + c] : czero<C>();
#pragma unroll
      for (int k = 0; k < kPanelNB; ++k) {
        v[k] = cmul(v[k], sh.uinv[k]);
#pragma unroll
        for (int c = k + 1; c < kPanelNB; ++c) v[c] = csub(v[c], cmul(v[k], sh.lu11[k][c]));
      }
#pragma unroll
      for (int c = 0; c < kPanelNB; ++c)
        if (c < w) A[phys * ld + col + c] = v[c];
    }
  }
  if (rank == 0 && (tid >> 5) == 0) {
    replay_pivots(w, sh.perm, ipiv, ipiv_base, rowmap);
    if ((tid & 31) == 0 && sh.singular && info) atomicCAS(info, 0, ipiv_base + sh.singular);
  }
}

// ----------------------------------------------------------------------------
// Panel without row exchanges, checked against partial pivoting (getrf with
// ctx.diag_pivots).  Partial pivoting exchanges no rows when at every step j
// the diagonal element is the first largest |re| + |im| of its column; the
// factor matrices of the retarded BEM (G1, G2, Delta, mostly Sigma) have
// that property, so their panels can skip the column-wide pivot search that
// bounds the pivoted panels.  Every CTA factors the w x w diagonal block in
// registers (warp 0, a lane per row), then each thread takes one row
// below it through x U11 = a (forward substitution in registers, the
// triangle fully unrolled).  Column j fails the check when some row has
// |a_ij^(j)|_1 > tau |a_jj^(j)|_1; a failing panel raises ctx.vflag and the
// caller factors the matrix again with partial pivoting.  With tau = 1 a
// passing matrix gets LAPACK's partial-pivoting factors (no exchanges).
constexpr int kNopivPanelThreads = 64;

// 1 / p for p != 0 (0 for p = 0), scaled by max(|re|, |im|) so that |p|^2
// neither overflows nor underflows: two real divisions, no branches
template <typename C>
__device__ __forceinline__ C crecip_scaled(C p) {
  using R = R_t<C>;
  const R sc = fmax(fabs(p.x), fabs(p.y));
  if (!(sc > R(0))) return czero<C>();
  const R rs = R(1) / sc;
  const R px = p.x * rs, py = p.y * rs;
  const R f = rs / (px * px + py * py);
  return cmake<C>(px * f, -py * f);
}

template <typename C>
__global__ void __launch_bounds__(kNopivPanelThreads) panel_nopiv_kernel(int m, int w, C* __restrict__ A, long long ld,
                                                                         int col, const int32_t* __restrict__ rowmap,
                                                                         int32_t* __restrict__ ipiv, int ipiv_base,
                                                                         int* __restrict__ info,
                                                                         int* __restrict__ vflag, R_t<C> tau) {
  // D is one row taller than the block: the rotated reads D[j][j + c] stay inside
  __shared__ C D[kPanelNB + 1][kPanelNB + 1];
  __shared__ C rinv[kPanelNB], prow[kPanelNB];
  __shared__ int zfirst, viol;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) {
    zfirst = INT_MAX;
    viol = 0;
  }
  for (int idx = tid; idx < w * w; idx += kNopivPanelThreads) {
    const int i = idx / w, c = idx % w;
    D[i][c] = A[(long long)rowmap[i] * ld + col + c];
  }
  // this thread's row below the diagonal block (complex64: loaded while warp
  // 0 factors the block; complex128 registers hold one row at a time)
  const int r = w + blockIdx.x * kNopivPanelThreads + tid;
  C* row = r < m ? A + (long long)rowmap[r] * ld + col : nullptr;
  C x[kPanelNB];
  if constexpr (sizeof(C) == 8) {
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c) x[c] = (row && c < w) ? row[c] : czero<C>();
  }
  __syncthreads();
  // Both parts keep the current column in register 0: every step shifts the
  // row left by one (updating the columns still open) and appends the new
  // multiplier, so register indices stay static in a rolled loop; after the
  // 32 steps of a full cycle the row is back in column order.
  if (wid == 0) {  // the diagonal block, lane i owning row i (padded with the identity)
    C v[kPanelNB];
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c)
      v[c] = (lane < w && c < w) ? D[lane][c] : (lane == c ? cmake<C>(1.0, 0.0) : czero<C>());
    bool bad = false;
#pragma unroll 1
    for (int j = 0; j < kPanelNB; ++j) {
      if (lane == j) {
#pragma unroll
        for (int c = 0; c < kPanelNB; ++c) prow[c] = v[c];
      }
      __syncwarp();
      const C piv = prow[0];
      const R_t<C> pm = pmag(piv);
      const C inv = crecip_scaled(piv);
      const bool act = lane > j;
      if (act && pmag(v[0]) > tau * pm) bad = true;
      const C l = cmul(v[0], inv);
      const C first = v[0];
      const int lim = kPanelNB - 1 - j;
#pragma unroll
      for (int c = 1; c < kPanelNB; ++c) {
        const C u = csub(v[c], cmul(l, prow[c]));
        v[c - 1] = (act && c <= lim) ? u : v[c];
      }
      v[kPanelNB - 1] = act ? l : first;
      if (lane == 0 && j < w && !(pm > 0) && zfirst == INT_MAX) zfirst = j;
      __syncwarp();
    }
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c) D[lane][c] = v[c];
    C d = v[0];
#pragma unroll
    for (int c = 1; c < kPanelNB; ++c)
      if (c == lane) d = v[c];
    rinv[lane] = crecip_scaled(d);
    if (__any_sync(0xffffffffu, bad) && lane == 0) viol = 1;
  }
  __syncthreads();
  if constexpr (sizeof(C) == 16) {
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c) x[c] = (row && c < w) ? row[c] : czero<C>();
  }
  if (row) {  // x U11 = a; padded steps j >= w see an identity pivot and leave x alone
    bool bad = false;
#pragma unroll 1
    for (int j = 0; j < kPanelNB; ++j) {
      const C* Dj = &D[j][j];
      if (pmag(x[0]) > tau * pmag(Dj[0])) bad = true;  // x[0] = a_rj^(j) here
      const C l = cmul(x[0], rinv[j]);
      const int lim = kPanelNB - 1 - j;
#pragma unroll
      for (int c = 1; c < kPanelNB; ++c) {
        const C u = csub(x[c], cmul(l, Dj[c]));
        x[c - 1] = c <= lim ? u : x[c];
      }
      x[kPanelNB - 1] = l;
    }
#pragma unroll
    for (int c = 0; c < kPanelNB; ++c)
      if (c < w) row[c] = x[c];
    if (bad) viol = 1;
  }
  if (blockIdx.x == 0) {
    for (int idx = tid; idx < w * w; idx += kNopivPanelThreads) {
      const int i = idx / w, c = idx % w;
      A[(long long)rowmap[i] * ld + col + c] = D[i][c];
    }
    if (tid < w) ipiv[tid] = ipiv_base + tid;
  }
  __syncthreads();
  if (tid == 0) {
    if (viol && vflag) atomicExch(vflag, 1);
    if (blockIdx.x == 0 && zfirst != INT_MAX && info) atomicCAS(info, 0, ipiv_base + zfirst + 1);
  }
}

template <typename C>
static int panel_lu(const LaContext& ctx, int m, int w, C* A, long long ld, int col, int32_t* rowmap, int32_t* ipiv,
                    int ipiv_base) {
  if (ctx.diag_pivots) {
    const int grid = max(1, ceil_div(m - w, kNopivPanelThreads));
    panel_nopiv_kernel<C><<<grid, kNopivPanelThreads, 0, ctx.stream>>>(m, w, A, ld, col, rowmap, ipiv, ipiv_base,
                                                                        ctx.dinfo, ctx.vflag,
                                                                        (R_t<C>)ctx.pivot_tau);
    BEM_LAUNCH_CHECK();
    count_launch();
    return BEM200_OK;
  }
  if constexpr (sizeof(C) == 8) {
    if (ctx.tournament && m > kCaluMinRows && m <= kCaluMaxCluster * kCaluThreads) {
      // complex64: tournament pivoting, 128 - 512 rows per CTA
      const int cs = min(kCaluMaxCluster, ceil_div(m, 128));
      const int R = ceil_div(m, cs);
      auto kern = panel_calu_kernel<C>;
      BEM_CUDA_CHECK(set_kernel_attrs_once(kern, 0, true));
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(cs, 1, 1);
      cfg.blockDim = dim3(kCaluThreads, 1, 1);
      cfg.dynamicSmemBytes = 0;
      cfg.stream = ctx.stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = cs;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      BEM_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, m, w, A, ld, col, rowmap, ipiv, ipiv_base, ctx.dinfo, R));
      count_launch();
      return BEM200_OK;
    }
  }
  if constexpr (sizeof(C) == 8) {
    if (m <= kAsyncMaxCluster * kAsyncThreads) {
      // complex64: asynchronous push panel, 128 - 384 rows per CTA
      const int cs = min(kAsyncMaxCluster, max(1, ceil_div(m, 128)));
      const int R = ceil_div(m, cs);
      const int threads = ceil_div(R, 32) * 32;
      auto kern = panel_lu_async_kernel;
      BEM_CUDA_CHECK(set_kernel_attrs_once(kern, 0, true));
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(cs, 1, 1);
      cfg.blockDim = dim3(threads, 1, 1);
      cfg.dynamicSmemBytes = 0;
      cfg.stream = ctx.stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = cs;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      BEM_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, m, w, reinterpret_cast<float2*>(A), ld, col, rowmap, ipiv,
                                        ipiv_base, ctx.dinfo, ctx.dstatus, R));
      count_launch();
      return BEM200_OK;
    }
  }
  if (m <= kPushMaxCluster * kPushThreads) {
    // 128 - 384 rows per CTA, as many CTAs (<= 16) as that takes
    const int cs = min(kPushMaxCluster, max(1, ceil_div(m, 128)));
    const int R = ceil_div(m, cs);
    const int threads = ceil_div(R, 32) * 32;
    auto kern = panel_lu_push_kernel<C>;
    BEM_CUDA_CHECK(set_kernel_attrs_once(kern, 0, true));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BEM_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, m, w, A, ld, col, rowmap, ipiv, ipiv_base, ctx.dinfo, R));
    count_launch();
    return BEM200_OK;
  }
  if (ctx.panel_ws) {
    // taller than one cluster holds: one row per thread over the whole GPU
    static_assert(2 * kGridMaxCta * sizeof(GridCand<double2>) <= kPanelGridScratch, "panel scratch too small");
    const int G = ceil_div(m, kPushThreads);
    const int R = ceil_div(m, G);
    const int threads = ceil_div(R, 32) * 32;
    auto kern = panel_lu_grid_kernel<C>;
    int dev = 0, nsm = 0, per_sm = 0;
    BEM_CUDA_CHECK(cudaGetDevice(&dev));
    BEM_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    BEM_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0));
    BEM_REQUIRE(G <= kGridMaxCta && G <= per_sm * nsm, BEM200_ERR_UNSUPPORTED,
                "panel_lu: panel of %d rows needs %d co-resident CTAs (device holds %d)", m, G, per_sm * nsm);
    GridCand<C>* cand = reinterpret_cast<GridCand<C>*>(ctx.panel_ws);
    int ipb = ipiv_base;
    int* info = ctx.dinfo;
    void* args[] = {(void*)&m, (void*)&w, (void*)&A, (void*)&ld, (void*)&col, (void*)&rowmap, (void*)&ipiv,
                    (void*)&ipb, (void*)&info, (void*)&R, (void*)&cand};
    BEM_CUDA_CHECK(cudaLaunchCooperativeKernel((const void*)kern, dim3(G), dim3(threads), args, 0, ctx.stream));
    count_launch();
    return BEM200_OK;
  }
  constexpr int kRegCap = kRegWarps * RegRows<C>::value;  // rows per CTA
  if (m <= 16 * kRegCap) {
    int cs = ceil_div(m, kRegCap);
    int R = ceil_div(m, cs);
    auto kern = panel_lu_reg_kernel<C>;
    BEM_CUDA_CHECK(set_kernel_attrs_once(kern, 0, true));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs, 1, 1);
    cfg.blockDim = dim3(kRegThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BEM_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, m, w, A, ld, col, rowmap, ipiv, ipiv_base, ctx.dinfo, R));
    count_launch();
    return BEM200_OK;
  }
  const size_t row_bytes = sizeof(C) * kPanelNB + sizeof(int32_t) + 1;
  const size_t max_smem = 200 * 1024;
  int cs = 1;
  while ((size_t)ceil_div(m, cs) * row_bytes > max_smem && cs < 16) cs *= 2;
  int R = ceil_div(m, cs);
  size_t smem = (size_t)R * row_bytes + 16;
  BEM_REQUIRE(smem <= max_smem, BEM200_ERR_UNSUPPORTED,
              "panel_lu: panel of %d rows does not fit a 16-CTA cluster", m);
  auto kern = panel_lu_kernel<C>;
  BEM_CUDA_CHECK(set_kernel_attrs_once(kern, (int)(max_smem + 1024), true));
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
  BEM_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, m, w, A, ld, col, rowmap, ipiv, ipiv_base, ctx.dinfo, R));
  count_launch();
  return BEM200_OK;
}

// ===================================================================== TRSM leaves
// A leaf solves with a triangle of m <= NB = 64 rows held in shared memory
// (odd pitch); larger triangles recurse, so the work above the leaves runs as
// GEMMs with k >= 64 (tensor cores for complex64).  Each warp sweeps one
// right-hand vector at a time -- a column of B for left solves, a row of X for
// right solves.  Lane l holds elements l + 32 t of the vector in registers;
// each step of the sweep finishes one element, broadcasts it with a shuffle and
// updates the elements still open (NB / 32 complex FMAs per lane at most).
// Divisions by the diagonal use reciprocals computed before the sweep.  A CTA
// owns kLeafVecs vectors, two per warp.
template <typename C> struct LeafNB { static constexpr int value = 64; };
constexpr int kLeafThreads = 256;
constexpr int kLeafVecs = 16;

enum LeafKind : int {
  kLeftLowerUnit = 0,   // B <- L^-1 B
  kLeftUpper = 1,       // B <- U^-1 B
  kRightUpper = 2,      // X <- X U^-1
  kRightLowerUnit = 3,  // X <- X L^-1
};

template <typename C, int K>
__global__ void __launch_bounds__(kLeafThreads) trsm_leaf_kernel(int m, int nvec, RowView<C> T, RowView<C> B) {
  constexpr int NB = LeafNB<C>::value, NT = NB / 32, P = NB + 1;
  constexpr bool kLeft = (K == kLeftLowerUnit || K == kLeftUpper);
  constexpr bool kForward = (K == kLeftLowerUnit || K == kRightUpper);
  constexpr bool kUnit = (K == kLeftLowerUnit || K == kRightLowerUnit);
  extern __shared__ __align__(16) unsigned char leaf_smem[];
  C* Ts = reinterpret_cast<C*>(leaf_smem);  // NB x P triangle block
  C* Vs = Ts + NB * P;                       // kLeafVecs x P: vector v, element e at Vs[v * P + e]
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int v0 = blockIdx.x * kLeafVecs;
  const int nv = min(kLeafVecs, nvec - v0);
  for (int idx = tid; idx < NB * NB; idx += kLeafThreads) {
    const int r = idx / NB, c = idx % NB;
    Ts[r * P + c] = (r < m && c < m) ? T.at(r, c) : czero<C>();
  }
  if (kLeft) {
    for (int idx = tid; idx < NB * kLeafVecs; idx += kLeafThreads) {
      const int e = idx / kLeafVecs, v = idx % kLeafVecs;
      if (v < nv) Vs[v * P + e] = (e < m) ? B.at(e, v0 + v) : czero<C>();
    }
  } else {
    for (int idx = tid; idx < NB * kLeafVecs; idx += kLeafThreads) {
      const int v = idx / NB, e = idx % NB;
      if (v < nv) Vs[v * P + e] = (e < m) ? B.at(v0 + v, e) : czero<C>();
    }
  }
  __syncthreads();
  for (int v = wid; v < nv; v += kLeafThreads / 32) {
    C x[NT], inv[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int e = lane + 32 * t;
      x[t] = Vs[v * P + e];
      inv[t] = (!kUnit && e < m) ? cdiv(cmake<C>(1.0, 0.0), Ts[e * P + e]) : czero<C>();
    }
    if (kForward) {
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        for (int rr = 0; rr < 32; ++rr) {
          const int r = 32 * t + rr;
          if (r >= m) break;
          if (!kUnit && lane == rr) x[t] = cmul(x[t], inv[t]);
          const C xr = shfl_c(x[t], rr);
#pragma unroll
          for (int u = t; u < NT; ++u) {
            const int e = lane + 32 * u;
            const C coef = kLeft ? Ts[e * P + r] : Ts[r * P + e];
            const C nx = csub(x[u], cmul(coef, xr));
            if (e > r) x[u] = nx;
          }
        }
      }
    } else {
#pragma unroll
      for (int t = NT - 1; t >= 0; --t) {
        for (int rr = 31; rr >= 0; --rr) {
          const int r = 32 * t + rr;
          if (r >= m) continue;
          if (!kUnit && lane == rr) x[t] = cmul(x[t], inv[t]);
          const C xr = shfl_c(x[t], rr);
#pragma unroll
          for (int u = 0; u <= t; ++u) {
            const int e = lane + 32 * u;
            const C coef = kLeft ? Ts[e * P + r] : Ts[r * P + e];
            const C nx = csub(x[u], cmul(coef, xr));
            if (e < r) x[u] = nx;
          }
        }
      }
    }
#pragma unroll
    for (int t = 0; t < NT; ++t) Vs[v * P + lane + 32 * t] = x[t];
  }
  __syncthreads();
  if (kLeft) {
    for (int idx = tid; idx < NB * kLeafVecs; idx += kLeafThreads) {
      const int e = idx / kLeafVecs, v = idx % kLeafVecs;
      if (v < nv && e < m) B.at(e, v0 + v) = Vs[v * P + e];
    }
  } else {
    for (int idx = tid; idx < NB * kLeafVecs; idx += kLeafThreads) {
      const int v = idx / NB, e = idx % NB;
      if (v < nv && e < m) B.at(v0 + v, e) = Vs[v * P + e];
    }
  }
}

template <typename C>
static size_t leaf_smem_bytes() {
  constexpr int NB = LeafNB<C>::value;
  return sizeof(C) * (size_t)(NB + kLeafVecs) * (NB + 1);
}

template <typename K>
static int prep_smem(K kern, size_t bytes) {
  BEM_CUDA_CHECK(set_kernel_attrs_once(kern, (int)bytes, false));
  return BEM200_OK;
}

template <typename C, int K>
static int trsm_leaf(const LaContext& ctx, int m, int nvec, RowView<C> T, RowView<C> B) {
  auto kern = trsm_leaf_kernel<C, K>;
  int st = prep_smem(kern, leaf_smem_bytes<C>());
  if (st) return st;
  kern<<<ceil_div(nvec, kLeafVecs), kLeafThreads, leaf_smem_bytes<C>(), ctx.stream>>>(m, nvec, T, B);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

template <typename C> static C neg_one() { return cmake<C>(-1.0, 0.0); }
template <typename C> static C one() { return cmake<C>(1.0, 0.0); }

// split of m rows for a recursion on multiples of q (both parts non-empty)
static int split_point(int m, int q) {
  int h = m / 2;
  h = ((h + q - 1) / q) * q;
  return h < m ? h : m - q;
}

// B <- L^-1 B, L unit lower m x m (strict lower part of T)
template <typename C>
static int trsm_llu(const LaContext& ctx, int m, int ncols, RowView<C> T, RowView<C> B) {
  constexpr int NB = LeafNB<C>::value;
  if (m <= 0 || ncols <= 0) return BEM200_OK;
  if (m <= NB) return trsm_leaf<C, kLeftLowerUnit>(ctx, m, ncols, T, B);
  int m1 = split_point(m, NB);
  int st = trsm_llu(ctx, m1, ncols, T, B);
  if (st) return st;
  st = gemm_v<C>(ctx, m - m1, ncols, m1, neg_one<C>(), T.sub(m1, 0), B, one<C>(), B.sub(m1, 0));
  if (st) return st;
  return trsm_llu(ctx, m - m1, ncols, T.sub(m1, m1), B.sub(m1, 0));
}

// B <- U^-1 B, U upper non-unit
template <typename C>
static int trsm_lun(const LaContext& ctx, int m, int ncols, RowView<C> T, RowView<C> B) {
  constexpr int NB = LeafNB<C>::value;
  if (m <= 0 || ncols <= 0) return BEM200_OK;
  if (m <= NB) return trsm_leaf<C, kLeftUpper>(ctx, m, ncols, T, B);
  int m1 = split_point(m, NB);
  int st = trsm_lun(ctx, m - m1, ncols, T.sub(m1, m1), B.sub(m1, 0));
  if (st) return st;
  st = gemm_v<C>(ctx, m1, ncols, m - m1, neg_one<C>(), T.sub(0, m1), B.sub(m1, 0), one<C>(), B);
  if (st) return st;
  return trsm_lun(ctx, m1, ncols, T, B);
}

// X <- X U^-1, X nrows x m
template <typename C>
static int trsm_run(const LaContext& ctx, int m, int nrows, RowView<C> T, RowView<C> X) {
  constexpr int NB = LeafNB<C>::value;
  if (m <= 0 || nrows <= 0) return BEM200_OK;
  if (m <= NB) return trsm_leaf<C, kRightUpper>(ctx, m, nrows, T, X);
  int m1 = split_point(m, NB);
  int st = trsm_run(ctx, m1, nrows, T, X);
  if (st) return st;
  st = gemm_v<C>(ctx, nrows, m - m1, m1, neg_one<C>(), X, T.sub(0, m1), one<C>(), X.sub(0, m1));
  if (st) return st;
  return trsm_run(ctx, m - m1, nrows, T.sub(m1, m1), X.sub(0, m1));
}

// X <- X L^-1, L unit lower
template <typename C>
static int trsm_rlu(const LaContext& ctx, int m, int nrows, RowView<C> T, RowView<C> X) {
  constexpr int NB = LeafNB<C>::value;
  if (m <= 0 || nrows <= 0) return BEM200_OK;
  if (m <= NB) return trsm_leaf<C, kRightLowerUnit>(ctx, m, nrows, T, X);
  int m1 = split_point(m, NB);
  int st = trsm_rlu(ctx, m - m1, nrows, T.sub(m1, m1), X.sub(0, m1));
  if (st) return st;
  st = gemm_v<C>(ctx, nrows, m1, m - m1, neg_one<C>(), X.sub(0, m1), T.sub(m1, 0), one<C>(), X);
  if (st) return st;
  return trsm_rlu(ctx, m1, nrows, T, X);
}

// ===================================================================== blocked TRSV
// Solves T x = b in place for nrhs <= 16 right-hand sides (X is n x nrhs, ld
// nrhs).  Row block I (64 rows) is processed by the CTA that drew ticket I from
// an atomic counter; it consumes the solution blocks it depends on as their
// flags are set, then solves its diagonal block and publishes its flag.  A CTA
// only waits on blocks whose tickets were drawn earlier, so every wait ends;
// each wait is nonetheless bounded and reports BEM200_ERR_TIMEOUT in *status
// (the block then still publishes its flag so that no other block waits long).
//
// The triangle tiles do not depend on the flags: each CTA streams its tiles
// with cp.async into a double buffer, one tile ahead of the flag it waits for.
// The diagonal block is solved by a column sweep: warp w handles right-hand
// side q = w (mod 8), lane l keeps rows l and l + 32 in registers, and each
// step broadcasts the finished x_r and updates the remaining rows (one
// shuffle and one complex FMA per lane).  The upper solve multiplies by
// reciprocals of the diagonal, computed in parallel before the sweep.
constexpr int kTrsvBS = 64;
constexpr int kTrsvMaxRhs = 16;
constexpr int kTrsvPitch = kTrsvBS + 1;  // odd pitch: the sweep's column reads are bank-conflict free
constexpr long long kSpinLimit = 1LL << 22;

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <int B>
__device__ __forceinline__ void cp_async_elem(void* s, const void* g);
template <>
__device__ __forceinline__ void cp_async_elem<8>(void* s, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(su32(s)), "l"(g) : "memory");
}
template <>
__device__ __forceinline__ void cp_async_elem<16>(void* s, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(su32(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// tile rows [r0, r0 + rb) x columns [c0, c0 + cb) of the operator -> dst (64 x
// kTrsvPitch), zero padded.  kTrans: the operator is T^T, so dst[r][c] =
// T(c0 + c, r0 + r); consecutive threads then read consecutive columns of one
// storage row of T.
template <typename C, bool kTrans>
__device__ __forceinline__ void trsv_load_tile(C* dst, const RowView<C>& T, int r0, int rb, int c0, int cb) {
  for (int idx = threadIdx.x; idx < kTrsvBS * kTrsvBS; idx += blockDim.x) {
    const int r = kTrans ? (idx & 63) : (idx >> 6), c = kTrans ? (idx >> 6) : (idx & 63);
    C* d = dst + r * kTrsvPitch + c;
    if (r < rb && c < cb)
      cp_async_elem<sizeof(C)>(d, T.base + (kTrans ? T.off(c0 + c, r0 + r) : T.off(r0 + r, c0 + c)));
    else
      *d = czero<C>();
  }
}

// kLower: forward substitution (blocks depend on earlier blocks), else
// backward.  kUnit: unit diagonal.  kTrans: the operator is T^T.  The LU
// factors give (kLower, kUnit) = (true, true) for L and (false, false) for U;
// their transposes U^T and L^T give (true, false) and (false, true).
// a 64 x 64 row-major block -> dst (64 x kTrsvPitch)
template <typename C>
__device__ __forceinline__ void trsv_load_plain(C* dst, const C* __restrict__ src) {
  for (int idx = threadIdx.x; idx < kTrsvBS * kTrsvBS; idx += blockDim.x)
    cp_async_elem<sizeof(C)>(dst + (idx >> 6) * kTrsvPitch + (idx & 63), src + idx);
}

// Dinv (optional): the inverses of the 64 x 64 diagonal blocks of the operator
// (trsv_diag_inverse); the diagonal step is then a parallel 64 x 64 product
// instead of a 64-step sweep.
template <typename C, bool kLower, bool kUnit, bool kTrans>
__global__ void __launch_bounds__(256) trsv_blocked_kernel(int n, int nrhs, RowView<C> T, C* __restrict__ X,
                                                          int* __restrict__ flags, int* __restrict__ ticket,
                                                          int* __restrict__ status, const C* __restrict__ Dinv) {
  extern __shared__ __align__(16) unsigned char trsv_smem[];
  C* tiles = reinterpret_cast<C*>(trsv_smem);        // 2 x 64 x kTrsvPitch
  C* xs = tiles + 2 * kTrsvBS * kTrsvPitch;           // 64 x 16: this block's x
  C* xj = xs + kTrsvBS * kTrsvMaxRhs;                 // 64 x 16: a finished block's x
  __shared__ int sI, sabort;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nblk = ceil_div(n, kTrsvBS);
  if (tid == 0) {
    sI = atomicAdd(ticket, 1);
    sabort = 0;
  }
  __syncthreads();
  const int tk = sI;
  if (tk >= nblk) return;
  const int I = kLower ? tk : nblk - 1 - tk;
  const int r0 = I * kTrsvBS, rb = min(kTrsvBS, n - r0);
  const int nsrc = tk;  // blocks this one depends on: I of them (lower) or nblk - 1 - I (upper)
  auto src_block = [&](int s) { return kLower ? s : nblk - 1 - s; };
  auto load_block = [&](C* dst, int J) {  // dependency tile J, or the diagonal block (J == I)
    if (J == I && Dinv)
      trsv_load_plain<C>(dst, Dinv + (long long)I * kTrsvBS * kTrsvBS);
    else
      trsv_load_tile<C, kTrans>(dst, T, r0, rb, J * kTrsvBS, min(kTrsvBS, n - J * kTrsvBS));
  };
  {  // tile 0: the first dependency, or the diagonal block
    load_block(tiles, nsrc > 0 ? src_block(0) : I);
    cp_async_commit();
  }
  for (int idx = tid; idx < kTrsvBS * nrhs; idx += 256) {
    const int r = idx / nrhs, q = idx % nrhs;
    xs[r * kTrsvMaxRhs + q] = (r < rb) ? X[(long long)(r0 + r) * nrhs + q] : czero<C>();
  }
  // split of the 64-long dot products over S lanes so that all 256 threads work
  const int S = nrhs == 1 ? 4 : (nrhs == 2 ? 2 : 1);
  const int nout = kTrsvBS * nrhs;
  int s = 0;
  for (; s < nsrc; ++s) {
    const int J = src_block(s);
    const int c0 = J * kTrsvBS, cb = min(kTrsvBS, n - c0);
    {  // prefetch tile s + 1 (the next dependency or the diagonal block)
      load_block(tiles + ((s + 1) & 1) * kTrsvBS * kTrsvPitch, (s + 1 < nsrc) ? src_block(s + 1) : I);
      cp_async_commit();
    }
    if (tid == 0) {
      // plain acquire loads: every block waiting on the same flag reads it from
      // L2 without the serialising read-modify-write of an atomic
      long long spins = 0;
      while (ld_acquire_gpu(&flags[J]) == 0) {
        if (++spins > kSpinLimit) {
          atomicExch(status, BEM200_ERR_TIMEOUT);
          sabort = 1;
          break;
        }
        if (spins > 16) __nanosleep(32);
      }
      __threadfence();
    }
    __syncthreads();
    if (sabort) break;
    for (int idx = tid; idx < kTrsvBS * nrhs; idx += 256) {
      const int c = idx / nrhs, q = idx % nrhs;
      xj[c * kTrsvMaxRhs + q] =
          (c < cb) ? __ldcg(reinterpret_cast<const C*>(X) + (long long)(c0 + c) * nrhs + q) : czero<C>();
    }
    cp_async_wait<1>();  // tile s has landed; tile s + 1 may still be in flight
    __syncthreads();
    const C* tile = tiles + (s & 1) * kTrsvBS * kTrsvPitch;
    for (int base = 0; base < nout * S; base += 256) {
      const int idx = base + tid;
      const int o = idx / S, part = idx % S;
      C acc = czero<C>();
      if (o < nout) {
        const int r = o / nrhs, q = o % nrhs;
        const C* trow = tile + r * kTrsvPitch;
#pragma unroll 8
        for (int c = part; c < kTrsvBS; c += S) acc = cadd(acc, cmul(trow[c], xj[c * kTrsvMaxRhs + q]));
      }
      for (int off = 1; off < S; off <<= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
      }
      if (o < nout && part == 0) {
        const int r = o / nrhs, q = o % nrhs;
        xs[r * kTrsvMaxRhs + q] = csub(xs[r * kTrsvMaxRhs + q], acc);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  __syncthreads();
  if (!sabort && Dinv) {
    // x_I = Dinv_I x_I: the same split dot products as the dependency updates
    const C* D = tiles + (nsrc & 1) * kTrsvBS * kTrsvPitch;
    for (int idx = tid; idx < kTrsvBS * nrhs; idx += 256) {
      const int r = idx / nrhs, q = idx % nrhs;
      xj[r * kTrsvMaxRhs + q] = xs[r * kTrsvMaxRhs + q];
    }
    __syncthreads();
    for (int base = 0; base < nout * S; base += 256) {
      const int idx = base + tid;
      const int o = idx / S, part = idx % S;
      C acc = czero<C>();
      if (o < nout) {
        const int r = o / nrhs, q = o % nrhs;
        const C* drow = D + r * kTrsvPitch;
#pragma unroll 8
        for (int c = part; c < kTrsvBS; c += S) acc = cadd(acc, cmul(drow[c], xj[c * kTrsvMaxRhs + q]));
      }
      for (int off = 1; off < S; off <<= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
      }
      if (o < nout && part == 0) {
        const int r = o / nrhs, q = o % nrhs;
        xs[r * kTrsvMaxRhs + q] = acc;
      }
    }
    __syncthreads();
    for (int idx = tid; idx < rb * nrhs; idx += 256) {
      const int r = idx / nrhs, q = idx % nrhs;
      X[(long long)(r0 + r) * nrhs + q] = xs[r * kTrsvMaxRhs + q];
    }
  } else if (!sabort) {
    const C* D = tiles + (nsrc & 1) * kTrsvBS * kTrsvPitch;  // the diagonal block
    for (int q = wid; q < nrhs; q += 8) {
      C x0 = xs[lane * kTrsvMaxRhs + q], x1 = xs[(lane + 32) * kTrsvMaxRhs + q];
      const C* d0 = D + lane * kTrsvPitch;
      const C* d1 = D + (lane + 32) * kTrsvPitch;
      const C one = cmake<C>(1.0, 0.0);
      const C inv0 = (!kUnit && lane < rb) ? cdiv(one, d0[lane]) : czero<C>();
      const C inv1 = (!kUnit && lane + 32 < rb) ? cdiv(one, d1[lane + 32]) : czero<C>();
      if (kLower) {
        for (int r = 0; r < rb; ++r) {
          if (!kUnit) {
            if (r < 32) {
              if (lane == r) x0 = cmul(x0, inv0);
            } else if (lane == r - 32) {
              x1 = cmul(x1, inv1);
            }
          }
          const C xr = shfl_c(r < 32 ? x0 : x1, r & 31);
          const C u0 = csub(x0, cmul(d0[r], xr)), u1 = csub(x1, cmul(d1[r], xr));
          if (lane > r) x0 = u0;
          if (lane + 32 > r) x1 = u1;
        }
      } else {
        for (int r = rb - 1; r >= 0; --r) {
          if (!kUnit) {
            if (r < 32) {
              if (lane == r) x0 = cmul(x0, inv0);
            } else if (lane == r - 32) {
              x1 = cmul(x1, inv1);
            }
          }
          const C xr = shfl_c(r < 32 ? x0 : x1, r & 31);
          const C u0 = csub(x0, cmul(d0[r], xr)), u1 = csub(x1, cmul(d1[r], xr));
          if (lane < r) x0 = u0;
          if (lane + 32 < r) x1 = u1;
        }
      }
      xs[lane * kTrsvMaxRhs + q] = x0;
      xs[(lane + 32) * kTrsvMaxRhs + q] = x1;
    }
    __syncthreads();
    for (int idx = tid; idx < rb * nrhs; idx += 256) {
      const int r = idx / nrhs, q = idx % nrhs;
      X[(long long)(r0 + r) * nrhs + q] = xs[r * kTrsvMaxRhs + q];
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) atomicExch(&flags[I], 1);
}

// Inverses of the 64 x 64 diagonal blocks of the factor (LU, rowmap): DL[I] =
// L_II^-1 (unit lower), DU[I] = U_II^-1 (upper), each 64 x 64 row-major, rows
// beyond n padded with the identity.  One CTA of 64 threads per block; thread
// c computes column c of each inverse by substitution.  Used by the blocked
// triangular solve so that the diagonal step of every block is a parallel
// product (the factors are reused for several solves per factorisation).
template <typename C>
__global__ void __launch_bounds__(64) trsv_diag_inverse_kernel(int n, RowView<C> T, C* __restrict__ DL,
                                                              C* __restrict__ DU) {
  extern __shared__ __align__(16) unsigned char dinv_smem[];
  C(*blk)[kTrsvBS + 1] = reinterpret_cast<C(*)[kTrsvBS + 1]>(dinv_smem);
  C(*X)[kTrsvBS + 1] = blk + kTrsvBS;
  const int I = blockIdx.x, r0 = I * kTrsvBS, rb = min(kTrsvBS, n - r0);
  const int c = threadIdx.x;
  const C one = cmake<C>(1.0, 0.0), zero = czero<C>();
  for (int r = 0; r < kTrsvBS; ++r)
    blk[r][c] = (r < rb && c < rb) ? T.at(r0 + r, r0 + c) : (r == c ? one : zero);
  __syncthreads();
  // L^-1: x_r = 0 (r < c), x_c = 1, x_r = -sum_{c <= k < r} L_rk x_k (r > c)
  for (int r = 0; r < kTrsvBS; ++r) {
    C x = (r == c) ? one : zero;
    if (r > c)
      for (int k = c; k < r; ++k) x = csub(x, cmul(blk[r][k], X[k][c]));
    X[r][c] = x;
  }
  C* dl = DL + (long long)I * kTrsvBS * kTrsvBS;
  for (int r = 0; r < kTrsvBS; ++r) dl[r * kTrsvBS + c] = X[r][c];
  // U^-1: x_r = 0 (r > c), x_c = 1 / U_cc, x_r = -(sum_{r < k <= c} U_rk x_k) / U_rr (r < c, descending)
  for (int r = kTrsvBS - 1; r >= 0; --r) {
    C x = zero;
    if (r <= c) {
      C acc = (r == c) ? one : zero;
      for (int k = r + 1; k <= c; ++k) acc = csub(acc, cmul(blk[r][k], X[k][c]));
      const C d = blk[r][r];
      x = cabs1(d) > 0 ? cdiv(acc, d) : zero;
    }
    X[r][c] = x;
  }
  C* du = DU + (long long)I * kTrsvBS * kTrsvBS;
  for (int r = 0; r < kTrsvBS; ++r) du[r * kTrsvBS + c] = X[r][c];
}

template <typename C>
size_t trsv_diag_inverse_bytes(int n) {
  return sizeof(C) * (size_t)ceil_div(n, kTrsvBS) * kTrsvBS * kTrsvBS;
}

template <typename C>
int trsv_diag_inverse(const LaContext& ctx, int n, const C* LU, long long ld, const int32_t* rowmap, C* DL, C* DU) {
  RowView<C> T{const_cast<C*>(LU), ld, rowmap, 0};
  const size_t smem = sizeof(C) * 2 * kTrsvBS * (kTrsvBS + 1);
  int st = prep_smem(trsv_diag_inverse_kernel<C>, smem);
  if (st) return st;
  trsv_diag_inverse_kernel<C><<<ceil_div(n, kTrsvBS), kTrsvBS, smem, ctx.stream>>>(n, T, DL, DU);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

template <typename C>
static size_t trsv_smem_bytes() {
  return sizeof(C) * (2 * kTrsvBS * kTrsvPitch + 2 * kTrsvBS * kTrsvMaxRhs);
}

template <typename C, bool kLower, bool kUnit = kLower, bool kTrans = false>
static int trsv_blocked(const LaContext& ctx, int n, int nrhs, RowView<C> T, C* X, int* iscratch,
                        const C* Dinv = nullptr) {
  const int nblk = ceil_div(n, kTrsvBS);
  // iscratch: flags [0, nblk), ticket [nblk], local status [nblk + 1]
  BEM_CUDA_CHECK(cudaMemsetAsync(iscratch, 0, sizeof(int) * (nblk + 2), ctx.stream));
  auto kern = trsv_blocked_kernel<C, kLower, kUnit, kTrans>;
  int st = prep_smem(kern, trsv_smem_bytes<C>());
  if (st) return st;
  kern<<<nblk, 256, trsv_smem_bytes<C>(), ctx.stream>>>(n, nrhs, T, X, iscratch, iscratch + nblk,
                                                        ctx.dstatus ? ctx.dstatus : iscratch + nblk + 1, Dinv);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// ===================================================================== LU driver
__global__ void iota_kernel(int n, int32_t* __restrict__ a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

template <typename C>
static int getrf_rec(const LaContext& ctx, int n, C* A, long long ld, int32_t* rowmap, int32_t* ipiv, int col0,
                     int w) {
  if (w <= kPanelNB) return panel_lu<C>(ctx, n - col0, w, A, ld, col0, rowmap + col0, ipiv + col0, col0);
  int w1 = split_point(w, kPanelNB);
  int st = getrf_rec(ctx, n, A, ld, rowmap, ipiv, col0, w1);
  if (st) return st;
  RowView<C> V{A, ld, rowmap + col0, col0};  // logical rows from col0, columns from col0
  // U12 = L11^-1 A12
  st = trsm_llu<C>(ctx, w1, w - w1, V, V.sub(0, w1));
  if (st) return st;
  // A22 -= L21 U12
  st = gemm_v<C>(ctx, n - col0 - w1, w - w1, w1, neg_one<C>(), V.sub(w1, 0), V.sub(0, w1), one<C>(), V.sub(w1, w1));
  if (st) return st;
  return getrf_rec(ctx, n, A, ld, rowmap, ipiv, col0 + w1, w - w1);
}

// Blocked right-looking LU with look-ahead (block columns of ctx.la_nb, a
// multiple of 32; 128 by default, tunable per size).  Step j:
//   panel(j)   : getrf_rec on block column j                [high-priority stream]
//   narrow(j)  : U(j, j+1) = L(j,j)^-1 A(j, j+1) and the update of block
//                column j+1 -- all the next panel needs     [high-priority stream]
//   wide(j)    : the same for block columns j+2..           [low-priority stream]
// so the wide TRSM + tensor-core GEMM of step j runs while panel(j+1) is
// factored.  narrow(j) waits for wide(j-1), wide(j) waits for panel(j).
// panel(j+1) permutes logical rows >= (j+1) nb while wide(j) updates them,
// so wide(j) addresses those rows through a snapshot of the row map taken
// right after panel(j) (two snapshots alternate).  The rows themselves never
// move, so both orders give the same matrix.
static int la_width(const LaContext& ctx) {
  const int w = ctx.la_nb > 0 ? ctx.la_nb : 128;
  return max(64, min(1024, (w / kPanelNB) * kPanelNB));
}

struct LaStreams {
  cudaStream_t hi = nullptr, lo = nullptr;
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // fork, panel, wide, done_hi, done_lo
  ~LaStreams() {
    for (cudaEvent_t& e : ev)
      if (e) cudaEventDestroy(e);
    if (hi) cudaStreamDestroy(hi);  // released once their queued work has finished
    if (lo) cudaStreamDestroy(lo);
  }
};

template <typename C>
static int getrf_lookahead(const LaContext& ctx, int n, C* A, long long ld, int32_t* rowmap, int32_t* ipiv,
                           int32_t* snap) {
  LaStreams ls;
  int lo_pri = 0, hi_pri = 0;
  BEM_CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri));
  BEM_CUDA_CHECK(cudaStreamCreateWithPriority(&ls.hi, cudaStreamNonBlocking, hi_pri));
  BEM_CUDA_CHECK(cudaStreamCreateWithPriority(&ls.lo, cudaStreamNonBlocking, lo_pri));
  for (cudaEvent_t& e : ls.ev) BEM_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEvent_t ev_fork = ls.ev[0], ev_panel = ls.ev[1], ev_wide = ls.ev[2];
  BEM_CUDA_CHECK(cudaEventRecord(ev_fork, ctx.stream));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(ls.hi, ev_fork, 0));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(ls.lo, ev_fork, 0));
  LaContext cm = ctx, cw = ctx;
  cm.stream = ls.hi;
  cw.stream = ls.lo;
  cm.panel_ws = reinterpret_cast<char*>(snap) + (((size_t)2 * n * sizeof(int32_t) + 255) & ~size_t(255));
  if (ctx.engine != GemmEngine::kSimt) {
    const size_t h = (ctx.ws_bytes / 2) & ~size_t(255);
    cm.ws_bytes = h;
    cw.ws = reinterpret_cast<char*>(ctx.ws) + h;
    cw.ws_bytes = h;
  }
  iota_kernel<<<ceil_div(n, 256), 256, 0, ls.hi>>>(n, rowmap);
  BEM_LAUNCH_CHECK();
  bool wide_pending = false;
  int st;
  const int nb = la_width(ctx);
  for (int c0 = 0, j = 0; c0 < n; c0 += nb, ++j) {
    const int w = min(nb, n - c0);
    if ((st = getrf_rec(cm, n, A, ld, rowmap, ipiv, c0, w))) return st;
    const int c1 = c0 + w;
    if (c1 >= n) break;
    const int w1 = min(nb, n - c1), c2 = c1 + w1;
    int32_t* sn = snap + (size_t)(j & 1) * n;  // sn[i] = rowmap[c1 + i] as of the end of panel(j)
    if (c2 < n) {
      BEM_CUDA_CHECK(cudaMemcpyAsync(sn, rowmap + c1, sizeof(int32_t) * (n - c1), cudaMemcpyDeviceToDevice, ls.hi));
      BEM_CUDA_CHECK(cudaEventRecord(ev_panel, ls.hi));
    }
    // narrow(j): block column j + 1
    if (wide_pending) BEM_CUDA_CHECK(cudaStreamWaitEvent(ls.hi, ev_wide, 0));
    RowView<C> V{A, ld, rowmap + c0, c0};  // logical rows from c0, columns from c0
    if ((st = trsm_llu<C>(cm, w, w1, V, V.sub(0, w)))) return st;
    if ((st = gemm_v<C>(cm, n - c1, w1, w, neg_one<C>(), V.sub(w, 0), V.sub(0, w), one<C>(), V.sub(w, w)))) return st;
    // wide(j): block columns j + 2 ..
    wide_pending = false;
    if (c2 < n) {
      BEM_CUDA_CHECK(cudaStreamWaitEvent(ls.lo, ev_panel, 0));
      if ((st = trsm_llu<C>(cw, w, n - c2, V, V.sub(0, c2 - c0)))) return st;
      const RowView<C> L21{A, ld, sn, c0}, A22{A, ld, sn, c2};
      if ((st = gemm_v<C>(cw, n - c1, n - c2, w, neg_one<C>(), L21, V.sub(0, c2 - c0), one<C>(), A22))) return st;
      BEM_CUDA_CHECK(cudaEventRecord(ev_wide, ls.lo));
      wide_pending = true;
    }
  }
  BEM_CUDA_CHECK(cudaEventRecord(ls.ev[3], ls.hi));
  BEM_CUDA_CHECK(cudaEventRecord(ls.ev[4], ls.lo));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(ctx.stream, ls.ev[3], 0));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(ctx.stream, ls.ev[4], 0));
  return BEM200_OK;
}

__global__ void nopiv_finish_kernel(const int* __restrict__ vflag, int* __restrict__ info) {
  if (*vflag) atomicExch(info, -BEM200_ERR_PIVOTING);
}

template <typename C>
static int getrf_dispatch(const LaContext& ctx, int n, C* A, long long ld, int32_t* rowmap, int32_t* ipiv,
                          int32_t* scratch);

// Checked diagonal pivots (ctx.diag_pivots): the same blocked look-ahead LU
// with panel_nopiv panels; the panels' verdicts collect in a flag in the LU
// scratch, turned into *info = -BEM200_ERR_PIVOTING at the end.
template <typename C>
int getrf(const LaContext& ctx, int n, C* A, long long ld, int32_t* rowmap, int32_t* ipiv, int32_t* scratch) {
  BEM_REQUIRE(n > 0 && A && rowmap && ipiv && ld >= n, BEM200_ERR_ARG, "getrf: bad arguments");
  if (!ctx.diag_pivots) return getrf_dispatch<C>(ctx, n, A, ld, rowmap, ipiv, scratch);
  BEM_REQUIRE(scratch && ctx.dinfo, BEM200_ERR_ARG, "getrf: checked diagonal pivots need the LU workspace and info");
  LaContext c = ctx;
  c.vflag = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) +
                                   (((size_t)2 * n * sizeof(int32_t) + 255) & ~size_t(255)));
  BEM_CUDA_CHECK(cudaMemsetAsync(c.vflag, 0, sizeof(int), ctx.stream));
  int st = getrf_dispatch<C>(c, n, A, ld, rowmap, ipiv, scratch);
  if (st) return st;
  nopiv_finish_kernel<<<1, 1, 0, ctx.stream>>>(c.vflag, ctx.dinfo);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

template <typename C>
static int getrf_dispatch(const LaContext& ctx, int n, C* A, long long ld, int32_t* rowmap, int32_t* ipiv,
                          int32_t* scratch) {
  // look-ahead needs the row-map snapshots (scratch) and, on the tensor-core
  // engines, room for two concurrent GEMMs in the operand workspace
  const bool ws_ok = ctx.engine == GemmEngine::kSimt ||
                     gemm_tc_workspace(n, n, la_width(ctx), ctx.engine) <= ((ctx.ws_bytes / 2) & ~size_t(255));
  if (scratch && n > 2 * la_width(ctx) && ws_ok) return getrf_lookahead<C>(ctx, n, A, ld, rowmap, ipiv, scratch);
  iota_kernel<<<ceil_div(n, 256), 256, 0, ctx.stream>>>(n, rowmap);
  BEM_LAUNCH_CHECK();
  return getrf_rec(ctx, n, A, ld, rowmap, ipiv, 0, n);
}

// ===================================================================== solves
// out[i, :] = in[map[i], :]
template <typename C>
__global__ void gather_rows_kernel(int n, int ncols, const C* __restrict__ in, long long ldi,
                                   const int32_t* __restrict__ map, C* __restrict__ out, long long ldo) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * ncols) return;
  int i = (int)(idx / ncols), c = (int)(idx % ncols);
  out[(long long)i * ldo + c] = in[(long long)map[i] * ldi + c];
}

// Y[r, map[i]] = X[r, i]
template <typename C>
__global__ void scatter_cols_kernel(int m, int n, const C* __restrict__ X, long long ldx,
                                    const int32_t* __restrict__ map, C* __restrict__ Y, long long ldy) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m * n) return;
  int r = (int)(idx / n), i = (int)(idx % n);
  Y[(long long)r * ldy + map[i]] = X[(long long)r * ldx + i];
}

static size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

template <typename C>
size_t solve_left_scratch_bytes(int n, int nrhs) {
  return round256(sizeof(C) * (size_t)n * nrhs) + round256(sizeof(int) * (ceil_div(n, kTrsvBS) + 2));
}

template <typename C>
int solve_left(const LaContext& ctx, int n, int nrhs, const C* LU, long long ld, const int32_t* rowmap, C* B,
               long long ldb, void* scratch, const C* dinv_l, const C* dinv_u) {
  if (nrhs <= 0) return BEM200_OK;
  BEM_REQUIRE(scratch, BEM200_ERR_ARG, "solve_left: scratch required");
  C* Y = reinterpret_cast<C*>(scratch);
  int* iscr = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) + round256(sizeof(C) * (size_t)n * nrhs));
  long long tot = (long long)n * nrhs;
  gather_rows_kernel<C><<<ceil_div(tot, 256), 256, 0, ctx.stream>>>(n, nrhs, B, ldb, rowmap, Y, nrhs);
  BEM_LAUNCH_CHECK();
  RowView<C> T{const_cast<C*>(LU), ld, rowmap, 0};
  int st;
  if (nrhs <= kTrsvMaxRhs) {
    if ((st = trsv_blocked<C, true>(ctx, n, nrhs, T, Y, iscr, dinv_l))) return st;
    if ((st = trsv_blocked<C, false>(ctx, n, nrhs, T, Y, iscr, dinv_u))) return st;
  } else {
    if ((st = trsm_llu<C>(ctx, n, nrhs, T, plain(Y, nrhs)))) return st;
    if ((st = trsm_lun<C>(ctx, n, nrhs, T, plain(Y, nrhs)))) return st;
  }
  BEM_CUDA_CHECK(cudaMemcpy2DAsync(B, ldb * sizeof(C), Y, nrhs * sizeof(C), nrhs * sizeof(C), n,
                                   cudaMemcpyDeviceToDevice, ctx.stream));
  return BEM200_OK;
}

// out[map[i], :] = in[i, :]
template <typename C>
__global__ void scatter_rows_kernel(int n, int ncols, const C* __restrict__ in, long long ldi,
                                    const int32_t* __restrict__ map, C* __restrict__ out, long long ldo) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * ncols) return;
  int i = (int)(idx / ncols), c = (int)(idx % ncols);
  out[(long long)map[i] * ldo + c] = in[(long long)i * ldi + c];
}

// B <- A^-T B: with P A = L U, A^T = U^T L^T P, so U^T y = B (lower, non-unit),
// L^T u = y (upper, unit), then B[rowmap[i], :] = u[i, :].  nrhs <= 16.
template <typename C>
int solve_left_T(const LaContext& ctx, int n, int nrhs, const C* LU, long long ld, const int32_t* rowmap, C* B,
                 long long ldb, void* scratch) {
  if (nrhs <= 0) return BEM200_OK;
  BEM_REQUIRE(scratch, BEM200_ERR_ARG, "solve_left_T: scratch required");
  BEM_REQUIRE(nrhs <= kTrsvMaxRhs, BEM200_ERR_UNSUPPORTED, "solve_left_T: at most %d right-hand sides", kTrsvMaxRhs);
  C* Y = reinterpret_cast<C*>(scratch);
  int* iscr = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) + round256(sizeof(C) * (size_t)n * nrhs));
  BEM_CUDA_CHECK(cudaMemcpy2DAsync(Y, nrhs * sizeof(C), B, ldb * sizeof(C), nrhs * sizeof(C), n,
                                   cudaMemcpyDeviceToDevice, ctx.stream));
  RowView<C> T{const_cast<C*>(LU), ld, rowmap, 0};
  int st;
  if ((st = trsv_blocked<C, true, false, true>(ctx, n, nrhs, T, Y, iscr))) return st;
  if ((st = trsv_blocked<C, false, true, true>(ctx, n, nrhs, T, Y, iscr))) return st;
  const long long tot = (long long)n * nrhs;
  scatter_rows_kernel<C><<<ceil_div(tot, 256), 256, 0, ctx.stream>>>(n, nrhs, Y, nrhs, rowmap, B, ldb);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// Transposed skinny GEMM: Cm (m x w) = alpha A^T B + beta Cm with A (k x m) and
// B (k x w), w <= W.  Thread t of CTA (x, s) owns column i = 128 x + t of A and
// the k rows of split s (coalesced row reads of A; the B rows of a 32-row
// chunk are staged in shared memory); partial sums go to P[s] and a second
// kernel adds the splits in a fixed order (deterministic).
constexpr int kSkinnyTCols = 128;
constexpr int kSkinnyTMaxSplit = 16;

template <typename C, int W>
__global__ void __launch_bounds__(kSkinnyTCols) gemm_skinny_t_kernel(int m, int w, int k, int kchunk,
                                                                    RowView<C> A, RowView<C> B,
                                                                    C* __restrict__ P) {
  __shared__ C bs[32][W];
  const int i = blockIdx.x * kSkinnyTCols + threadIdx.x;
  const int s = blockIdx.y;
  const int k0 = s * kchunk, k1 = min(k, k0 + kchunk);
  C acc[W];
#pragma unroll
  for (int q = 0; q < W; ++q) acc[q] = czero<C>();
  for (int kb = k0; kb < k1; kb += 32) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < 32 * W; idx += kSkinnyTCols) {
      const int r = idx / W, q = idx % W;
      bs[r][q] = (kb + r < k1 && q < w) ? B.at(kb + r, q) : czero<C>();
    }
    __syncthreads();
    const int nr = min(32, k1 - kb);
    if (i < m) {
      for (int r = 0; r < nr; ++r) {
        const C a = A.at(kb + r, i);
#pragma unroll
        for (int q = 0; q < W; ++q) {
          const C b = bs[r][q];
          acc[q].x = fma(a.x, b.x, acc[q].x);
          acc[q].x = fma(-a.y, b.y, acc[q].x);
          acc[q].y = fma(a.x, b.y, acc[q].y);
          acc[q].y = fma(a.y, b.x, acc[q].y);
        }
      }
    }
  }
  if (i < m) {
#pragma unroll
    for (int q = 0; q < W; ++q)
      if (q < w) P[((long long)s * m + i) * w + q] = acc[q];
  }
}

template <typename C>
__global__ void skinny_t_reduce_kernel(int m, int w, int nsplit, const C* __restrict__ P, C alpha, C beta,
                                       RowView<C> Cv) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m * w) return;
  const int i = (int)(idx / w), q = (int)(idx % w);
  C acc = czero<C>();
  for (int s = 0; s < nsplit; ++s) acc = cadd(acc, P[(long long)s * m * w + idx]);
  C v = cmul(alpha, acc);
  C& out = Cv.at(i, q);
  if (beta.x != 0 || beta.y != 0) v = cadd(v, cmul(beta, out));
  out = v;
}

template <typename C>
size_t gemm_t_scratch_bytes(int m, int w) {
  return round256(sizeof(C) * (size_t)kSkinnyTMaxSplit * m * w);
}

template <typename C>
int gemm_t(const LaContext& ctx, int m, int w, int k, C alpha, RowView<C> A, RowView<C> B, C beta, RowView<C> Cv,
           void* scratch) {
  if (m <= 0 || w <= 0) return BEM200_OK;
  BEM_REQUIRE(w <= 16 && scratch, BEM200_ERR_UNSUPPORTED, "gemm_t: at most 16 columns and a scratch buffer");
  const int ncol = ceil_div(m, kSkinnyTCols);
  const int nsplit = max(1, min(kSkinnyTMaxSplit, ceil_div(4 * 148, ncol)));
  const int kchunk = ceil_div(k, nsplit);
  C* P = reinterpret_cast<C*>(scratch);
  dim3 grid(ncol, nsplit);
  if (w <= 8)
    gemm_skinny_t_kernel<C, 8><<<grid, kSkinnyTCols, 0, ctx.stream>>>(m, w, k, kchunk, A, B, P);
  else
    gemm_skinny_t_kernel<C, 16><<<grid, kSkinnyTCols, 0, ctx.stream>>>(m, w, k, kchunk, A, B, P);
  BEM_LAUNCH_CHECK();
  skinny_t_reduce_kernel<C><<<ceil_div((long long)m * w, 256), 256, 0, ctx.stream>>>(m, w, nsplit, P, alpha, beta,
                                                                                       Cv);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

template <typename C>
static int solve_right_rows(const LaContext& ctx, int n, int m, const C* LU, long long ld, const int32_t* rowmap,
                            C* X, long long ldx, C* tmp);

// rows of X are independent: with enough workspace, the second half of the
// rows runs on a forked stream (the narrow deep-recursion GEMMs of the two
// halves then share the GPU)
template <typename C>
int solve_right(const LaContext& ctx, int n, int m, const C* LU, long long ld, const int32_t* rowmap, C* X,
                long long ldx, C* tmp) {
  const int h = m / 2;
  const bool split = m >= 1024 && (ctx.engine == GemmEngine::kSimt ||
                                   gemm_tc_workspace(m - h, n / 2 + 64, n / 2 + 64, ctx.engine) <= ctx.ws_bytes / 2);
  if (!split) return solve_right_rows<C>(ctx, n, m, LU, ld, rowmap, X, ldx, tmp);
  LaContext c1 = ctx, c2;
  SideStream ss;
  BEM_REQUIRE(ss.fork(c1, c2), BEM200_ERR_CUDA, "solve_right: could not fork a stream");
  int st = solve_right_rows<C>(c1, n, h, LU, ld, rowmap, X, ldx, tmp);
  if (st) return st;
  st = solve_right_rows<C>(c2, n, m - h, LU, ld, rowmap, X + (long long)h * ldx, ldx, tmp + (long long)h * n);
  if (st) return st;
  BEM_CUDA_CHECK(ss.join(ctx.stream));
  return BEM200_OK;
}

template <typename C>
static int solve_right_rows(const LaContext& ctx, int n, int m, const C* LU, long long ld, const int32_t* rowmap,
                            C* X, long long ldx, C* tmp) {
  // X A = Y with P A = L U  =>  X = Y U^-1 L^-1 P
  if (m <= 0) return BEM200_OK;
  RowView<C> T{const_cast<C*>(LU), ld, rowmap, 0};
  int st = trsm_run<C>(ctx, n, m, T, plain(X, ldx));
  if (st) return st;
  st = trsm_rlu<C>(ctx, n, m, T, plain(X, ldx));
  if (st) return st;
  long long tot = (long long)m * n;
  scatter_cols_kernel<C><<<ceil_div(tot, 256), 256, 0, ctx.stream>>>(m, n, X, ldx, rowmap, tmp, n);
  BEM_LAUNCH_CHECK();
  BEM_CUDA_CHECK(cudaMemcpy2DAsync(X, ldx * sizeof(C), tmp, n * sizeof(C), n * sizeof(C), m,
                                   cudaMemcpyDeviceToDevice, ctx.stream));
  return BEM200_OK;
}

// B[i, j] = (j == map[i])  (the permutation matrix P of P A = L U)
template <typename C>
__global__ void perm_matrix_kernel(int n, const int32_t* __restrict__ map, C* A, long long ld) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * n) return;
  int r = (int)(idx / n), c = (int)(idx % n);
  A[(long long)r * ld + c] = (c == map[r]) ? cmake<C>(1.0, 0.0) : czero<C>();
}

template <typename C>
int inverse(const LaContext& ctx, int n, const C* LU, long long ld, const int32_t* rowmap, C* Inv, long long ldi) {
  perm_matrix_kernel<C><<<ceil_div((long long)n * n, 256), 256, 0, ctx.stream>>>(n, rowmap, Inv, ldi);
  BEM_LAUNCH_CHECK();
  RowView<C> T{const_cast<C*>(LU), ld, rowmap, 0};
  // the columns of the inverse are independent: with enough workspace the
  // second half of them is solved on a forked stream
  const int h = n / 2;
  const bool split = n >= 1024 && (ctx.engine == GemmEngine::kSimt ||
                                   gemm_tc_workspace(n, n - h + 64, n, ctx.engine) <= ctx.ws_bytes / 2);
  if (!split) {
    int st = trsm_llu<C>(ctx, n, n, T, plain(Inv, ldi));
    if (st) return st;
    return trsm_lun<C>(ctx, n, n, T, plain(Inv, ldi));
  }
  LaContext c1 = ctx, c2;
  SideStream ss;
  BEM_REQUIRE(ss.fork(c1, c2), BEM200_ERR_CUDA, "inverse: could not fork a stream");
  int st;
  if ((st = trsm_llu<C>(c1, n, h, T, plain(Inv, ldi)))) return st;
  if ((st = trsm_llu<C>(c2, n, n - h, T, plain(Inv + h, ldi)))) return st;
  if ((st = trsm_lun<C>(c1, n, h, T, plain(Inv, ldi)))) return st;
  if ((st = trsm_lun<C>(c2, n, n - h, T, plain(Inv + h, ldi)))) return st;
  BEM_CUDA_CHECK(ss.join(ctx.stream));
  return BEM200_OK;
}

// ===================================================================== inverse without pivoting
// M <- M^-1 in place by the block Schur complement, for matrices whose
// partial-pivoting LU exchanges no rows (the retarded BEM's Delta):
//   A^-1 (recursive), T1 = A^-1 B, T2 = C A^-1, S = D - C T1, S^-1 (recursive),
//   B <- -T1 S^-1, C <- -S^-1 T2, A <- A^-1 - B T2.
// Nearly all of the 8 n^3 flops land in the large GEMMs of the top levels
// (tensor cores for complex64); the leaves (<= 128 x 128 complex64, 64 x 64
// complex128) are inverted by
// Gauss-Jordan elimination in registers.  No row exchanges means no check
// of the leaves' pivots can cover the rows outside them, so the caller
// verifies the result with inverse_probe (M^-1 (M v) = v for a fixed
// pseudo-random v) and falls back to the pivoted LU when it fails.
template <typename C> struct InvLeaf { static constexpr int value = 64; };
template <> struct InvLeaf<double2> { static constexpr int value = 64; };
constexpr int kInvLeafThreads = 128;

// Gauss-Jordan inversion of the nb x nb (nb <= LN = InvLeaf) block at M, in
// place.  Thread (ty, tx) of the 8 x 16 grid owns the 8 x 4 block of rows
// ty + 8 p and columns tx + 16 q of an LN x LN tile padded with the identity;
// the 16 owners of a row are lanes of one warp.  Step k: the owners of row k
// take a_kk from its lane by a shuffle, scale the row by 1 / a_kk (that is
// the row's final value) and publish it, each entry beside its product with
// i so that the update is two packed FMAs; the owners of column k publish it
// (complex64: negated, each part duplicated for the packed operands).  With
// 1 + 1 / a_kk published in place of the pivot, every other row takes
// a_ij -= a_ik r_j, which also turns column k into -a_ik / a_kk.  The
// buffers are double buffered, so one barrier per step suffices.  A pivot
// that is zero or not the first largest |re| + |im| among the rows still to
// be eliminated raises *vflag.
template <typename C> struct LeafRow { using type = C; };            // complex128: the entry
template <> struct LeafRow<float2> { using type = float4; };         // complex64: (r_j, i r_j)
template <typename C> struct LeafCol { using type = C; };            // complex128: a_ik
template <> struct LeafCol<float2> { using type = float4; };         // complex64: -(x, x, y, y)
__device__ __forceinline__ void leaf_pub(float4& d, float2 r) { d = make_float4(r.x, r.y, -r.y, r.x); }
__device__ __forceinline__ void leaf_pub(double2& d, double2 r) { d = r; }
__device__ __forceinline__ void leaf_pubcol(float4& d, float2 a) { d = make_float4(-a.x, -a.x, -a.y, -a.y); }
__device__ __forceinline__ void leaf_pubcol(double2& d, double2 a) { d = a; }
__device__ __forceinline__ float leaf_cmag(float4 c) { return fabsf(c.x) + fabsf(c.z); }
__device__ __forceinline__ double leaf_cmag(double2 c) { return pmag(c); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return bits_f2(d);
}
// a_ij - a_ik r_j over the thread's entries of one row
template <int NQ>
__device__ __forceinline__ void leaf_row_update(float2 (&a)[NQ], float4 c, const float4 (&rr)[NQ]) {
  const float2 nx = make_float2(c.x, c.y), ny = make_float2(c.z, c.w);
#pragma unroll
  for (int q = 0; q < NQ; ++q)
    a[q] = ffma2(ny, make_float2(rr[q].z, rr[q].w), ffma2(nx, make_float2(rr[q].x, rr[q].y), a[q]));
}
template <int NQ>
__device__ __forceinline__ void leaf_row_update(double2 (&a)[NQ], double2 c, const double2 (&rr)[NQ]) {
#pragma unroll
  for (int q = 0; q < NQ; ++q) a[q] = csub(a[q], cmul(c, rr[q]));
}
// 1 / p: approximate reciprocals (two MUFU operations, scaled) for complex64
__device__ __forceinline__ float2 leaf_recip(float2 p) {
  const float sc = fmaxf(fabsf(p.x), fabsf(p.y));
  if (!(sc > 0.f)) return make_float2(0.f, 0.f);
  float rs, f;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rs) : "f"(sc));
  const float px = p.x * rs, py = p.y * rs;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(f) : "f"(px * px + py * py));
  f *= rs;
  return make_float2(px * f, -py * f);
}
__device__ __forceinline__ double2 leaf_recip(double2 p) { return crecip_scaled(p); }

template <typename C>
__global__ void __launch_bounds__(kInvLeafThreads, 1) inv_leaf_kernel(int nb, C* __restrict__ M, long long ld,
                                                                      R_t<C> tau, int* __restrict__ vflag) {
  constexpr int LN = InvLeaf<C>::value;
  constexpr int TY = 8, TX = 16;             // thread grid
  constexpr int PR = LN / TY, QC = LN / TX;  // rows and columns per thread: 8 x 4
  using RowE = typename LeafRow<C>::type;
  using ColE = typename LeafCol<C>::type;
  using R = R_t<C>;
  static_assert(TY * TX == kInvLeafThreads && PR * TY == LN && QC * TX == LN && TX % TY == 0 && 32 % TX == 0,
                "leaf layout");
  __shared__ RowE rowb[2][LN];
  __shared__ ColE colb[2][LN];
  __shared__ R pmb[2];
  const int tid = threadIdx.x, ty = tid / TX, tx = tid % TX;
  const int row_lane = (tid & 31) & ~(TX - 1);  // lane of (ty, 0)
  C a[PR][QC];
#pragma unroll
  for (int p = 0; p < PR; ++p)
#pragma unroll
    for (int q = 0; q < QC; ++q) {
      const int i = ty + TY * p, c = tx + TX * q;
      a[p][q] = (i < nb && c < nb) ? M[(long long)i * ld + c] : (i == c ? cmake<C>(1.0, 0.0) : czero<C>());
    }
  bool bad = false;
#pragma unroll
  for (int kp = 0; kp < PR; ++kp) {   // k = TY kp + kr: row k is row kp of thread row kr
    const int qk = (TY * kp) / TX;   // column k is column qk of thread column k % TX
    if (TY * kp >= nb) break;        // the identity padding needs no elimination steps
#pragma unroll 1
    for (int kr = 0; kr < TY; ++kr) {
      const int k = TY * kp + kr, b = k & 1, kx = k % TX;
      if (k >= nb) break;
      if (tx == kx) {
#pragma unroll
        for (int p = 0; p < PR; ++p) leaf_pubcol(colb[b][ty + TY * p], a[p][qk]);
      }
      const C akk = shfl_c(a[kp][qk], row_lane | kx);  // a_{ty + TY kp, k}: a_kk in the lanes of row k
      if (ty == kr) {
        const C pinv = leaf_recip(akk);
#pragma unroll
        for (int q = 0; q < QC; ++q) {
          const bool diag = q == qk && tx == kx;
          const C r = diag ? cadd(cmake<C>(1.0, 0.0), pinv) : cmul(a[kp][q], pinv);
          leaf_pub(rowb[b][tx + TX * q], r);
          a[kp][q] = diag ? pinv : r;  // row k is final
        }
        if (tx == kx) pmb[b] = pmag(akk);
      }
      __syncthreads();
      const R pm = pmb[b];
      if (!(pm > 0)) bad = true;
      RowE rr[QC];
#pragma unroll
      for (int q = 0; q < QC; ++q) rr[q] = rowb[b][tx + TX * q];
      R lower = 0;  // largest |a_ik|_1 among this thread's rows below k
#pragma unroll
      for (int p = 0; p < PR; ++p) {
        const ColE cik = colb[b][ty + TY * p];
        if (p > kp || (p == kp && ty > kr)) lower = fmax(lower, leaf_cmag(cik));
        if (!(p == kp && ty == kr)) leaf_row_update(a[p], cik, rr);
      }
      if (lower > tau * pm) bad = true;
    }
  }
#pragma unroll
  for (int p = 0; p < PR; ++p)
#pragma unroll
    for (int q = 0; q < QC; ++q) {
      const int i = ty + TY * p, c = tx + TX * q;
      if (i < nb && c < nb) M[(long long)i * ld + c] = a[p][q];
    }
  if (__any_sync(0xffffffffu, bad) && (tid & 31) == 0 && vflag) atomicExch(vflag, 1);
}

// scratch elements inverse_nopiv needs for an n x n matrix
template <typename C>
static size_t inverse_nopiv_scratch(int n) {
  // the inverse of A runs first, from the start of the scratch; then T1, T2
  // stay live while the inverse of S uses what follows them
  constexpr int kInvLeaf = InvLeaf<C>::value;
  if (n <= kInvLeaf) return 0;
  const int n1 = min(n - 1, ceil_div(n / 2, kInvLeaf) * kInvLeaf), n2 = n - n1;
  return max(inverse_nopiv_scratch<C>(n1), 2 * (size_t)n1 * n2 + inverse_nopiv_scratch<C>(n2));
}

// A side stream and two events of the recording thread: in a recorded graph
// the recursion puts the second of two independent products on a parallel
// branch (fork: the side stream waits for the main one; join: the reverse).
struct RecFork {
  cudaStream_t side;
  cudaEvent_t fork, join;
};

// g1 on ctx.stream and g2 (given the context to launch on) either on the
// same stream or, with fk and when neither uses the tensor-core workspace,
// on the side stream in parallel
template <typename C, typename F1, typename F2>
static int gemm_pair(const LaContext& ctx, const RecFork* fk, bool tc, F1 g1, F2 g2) {
  int st;
  if (!fk || tc) {
    if ((st = g1(ctx))) return st;
    return g2(ctx);
  }
  LaContext side = ctx;
  side.stream = fk->side;
  BEM_CUDA_CHECK(cudaEventRecord(fk->fork, ctx.stream));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(fk->side, fk->fork, 0));
  if ((st = g1(ctx))) return st;
  if ((st = g2(side))) return st;
  BEM_CUDA_CHECK(cudaEventRecord(fk->join, fk->side));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(ctx.stream, fk->join, 0));
  return BEM200_OK;
}

template <typename C>
static int inverse_nopiv_rec(const LaContext& ctx, int n, C* M, long long ld, C* ws, int* vflag,
                             const RecFork* fk = nullptr) {
  constexpr int kInvLeaf = InvLeaf<C>::value;
  if (n <= kInvLeaf) {
    inv_leaf_kernel<C><<<1, kInvLeafThreads, 0, ctx.stream>>>(n, M, ld, (R_t<C>)ctx.pivot_tau, vflag);
    BEM_LAUNCH_CHECK();
    count_launch();
    return BEM200_OK;
  }
  const int n1 = min(n - 1, ceil_div(n / 2, kInvLeaf) * kInvLeaf), n2 = n - n1;
  C* A = M;
  C* B = M + n1;
  C* Cm = M + (long long)n1 * ld;
  C* D = Cm + n1;
  int st;
  if ((st = inverse_nopiv_rec<C>(ctx, n1, A, ld, ws, vflag, fk))) return st;
  C* T1 = ws;                            // n1 x n2
  C* T2 = ws + (size_t)n1 * n2;          // n2 x n1
  C* rest = T2 + (size_t)n2 * n1;
  const C one = cmake<C>(1.0, 0.0), mone = cmake<C>(-1.0, 0.0), zero = czero<C>();
  // T1 = A^-1 B and T2 = C A^-1 are independent
  const bool tc1 = gemm_takes_tc<C>(ctx, n1, n2, n1) || gemm_takes_tc<C>(ctx, n2, n1, n1);
  if ((st = gemm_pair<C>(
           ctx, fk, tc1, [&](const LaContext& c) { return gemm<C>(c, n1, n2, n1, one, A, ld, B, ld, zero, T1, n2); },
           [&](const LaContext& c) { return gemm<C>(c, n2, n1, n1, one, Cm, ld, A, ld, zero, T2, n1); })))
    return st;
  if ((st = gemm<C>(ctx, n2, n2, n1, mone, Cm, ld, T1, n2, one, D, ld))) return st;
  if ((st = inverse_nopiv_rec<C>(ctx, n2, D, ld, rest, vflag, fk))) return st;
  // and so are B <- -T1 S^-1 and C <- -S^-1 T2
  const bool tc2 = gemm_takes_tc<C>(ctx, n1, n2, n2) || gemm_takes_tc<C>(ctx, n2, n1, n2);
  if ((st = gemm_pair<C>(
           ctx, fk, tc2, [&](const LaContext& c) { return gemm<C>(c, n1, n2, n2, mone, T1, n2, D, ld, zero, B, ld); },
           [&](const LaContext& c) { return gemm<C>(c, n2, n1, n2, mone, D, ld, T2, n1, zero, Cm, ld); })))
    return st;
  return gemm<C>(ctx, n1, n1, n2, mone, B, ld, T2, n1, one, A, ld);
}

// v: n fixed pseudo-random complex values in [-1, 1) (a hash of the index)
template <typename C>
__global__ void probe_fill_kernel(int n, C* __restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t h = (uint32_t)i * 2654435761u + 0x9e3779b9u;
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  const uint32_t g = h * 0xc2b2ae35u;
  v[i] = cmake<C>((double)(h & 0xffffu) / 32768.0 - 1.0, (double)(g >> 16) / 32768.0 - 1.0);
}

// *vflag = 1 unless max|z - v| <= tol max|v|
template <typename C>
__global__ void __launch_bounds__(1024) probe_check_kernel(int n, const C* __restrict__ v, const C* __restrict__ z,
                                                           double tol, int* __restrict__ vflag) {
  __shared__ double se[32], sv[32];
  double e = 0, m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const C d = csub(z[i], v[i]);
    const double de = fabs((double)d.x) + fabs((double)d.y);
    e = fmax(e, de == de ? de : INFINITY);
    m = fmax(m, fabs((double)v[i].x) + fabs((double)v[i].y));
  }
  for (int o = 16; o > 0; o >>= 1) {
    e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  if ((threadIdx.x & 31) == 0) {
    se[threadIdx.x >> 5] = e;
    sv[threadIdx.x >> 5] = m;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    e = threadIdx.x < (blockDim.x >> 5) ? se[threadIdx.x] : 0.0;
    m = threadIdx.x < (blockDim.x >> 5) ? sv[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if (threadIdx.x == 0 && !(e <= tol * m)) atomicExch(vflag, 1);
  }
}

template <typename C>
size_t inverse_nopiv_scratch_elems(int n) {
  return inverse_nopiv_scratch<C>(n) + 3 * (size_t)n + 64;
}

template <typename C>
static int inverse_nopiv_launch(const LaContext& ctx, int n, C* M, long long ld, C* ws, int* vflag, double tol,
                                const RecFork* fk = nullptr) {
  C* v = ws + inverse_nopiv_scratch<C>(n) + 32;
  C* y = v + n;
  C* z = y + n;
  const C one = cmake<C>(1.0, 0.0), zero = czero<C>();
  probe_fill_kernel<C><<<ceil_div(n, 256), 256, 0, ctx.stream>>>(n, v);
  BEM_LAUNCH_CHECK();
  int st;
  if ((st = gemm<C>(ctx, n, 1, n, one, M, ld, v, 1, zero, y, 1))) return st;  // y = M v
  if ((st = inverse_nopiv_rec<C>(ctx, n, M, ld, ws, vflag, fk))) return st;
  if ((st = gemm<C>(ctx, n, 1, n, one, M, ld, y, 1, zero, z, 1))) return st;  // z = M^-1 y
  probe_check_kernel<C><<<1, 1024, 0, ctx.stream>>>(n, v, z, tol, vflag);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// ---------------------------------------------------------------- graph replay of the inverse
// An inverse's launch sequence is a function of its arguments alone (sizes,
// pointers, engine, workspace, tolerances): it is recorded once per argument
// set into a CUDA graph and replayed afterwards, so that the ~600 launches of
// an n = 5768 inverse cost one graph launch on the host and run on the device
// without per-launch gaps.  The recording runs on a private stream of the
// calling thread (so the caller's stream may be the legacy default stream);
// the replay goes to the caller's stream.  Inside a caller's own stream
// capture, or with BEM200_NO_GRAPHS set, the launches are issued directly.
// The cache keeps the most recently used graphs; an evicted executable graph
// that is still in flight is freed by CUDA on completion.
namespace {
struct InvGraph {
  int csize, n, engine;
  long long ld;
  const void *M, *ws, *tcws;
  size_t tcws_bytes;
  const int *vflag, *dstatus;
  double tol;
  float tau;
  cudaGraphExec_t exec;
  unsigned long long kernels, used;
  bool same(const InvGraph& o) const {
    return csize == o.csize && n == o.n && engine == o.engine && ld == o.ld && M == o.M && ws == o.ws &&
           tcws == o.tcws && tcws_bytes == o.tcws_bytes && vflag == o.vflag && dstatus == o.dstatus && tol == o.tol &&
           tau == o.tau;
  }
};
std::mutex g_inv_mu;
std::vector<InvGraph> g_inv_graphs;
unsigned long long g_inv_tick = 0;
constexpr size_t kInvGraphCap = 256;
struct CaptureStream {
  cudaStream_t s = nullptr;
  RecFork fk{nullptr, nullptr, nullptr};
  ~CaptureStream() {
    if (fk.fork) cudaEventDestroy(fk.fork);
    if (fk.join) cudaEventDestroy(fk.join);
    if (fk.side) cudaStreamDestroy(fk.side);
    if (s) cudaStreamDestroy(s);
  }
};
thread_local CaptureStream t_capture;
bool inv_graphs_enabled() {
  static const bool on = [] {
    const char* e = getenv("BEM200_NO_GRAPHS");
    return !(e && *e && strcmp(e, "0") != 0);
  }();
  return on;
}
}  // namespace

template <typename C>
int inverse_nopiv(const LaContext& ctx, int n, C* M, long long ld, C* ws, int* vflag, double tol) {
  BEM_REQUIRE(n > 0 && M && ws && vflag, BEM200_ERR_ARG, "inverse_nopiv: bad arguments");
  if (!inv_graphs_enabled()) return inverse_nopiv_launch<C>(ctx, n, M, ld, ws, vflag, tol);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  BEM_CUDA_CHECK(cudaStreamIsCapturing(ctx.stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) return inverse_nopiv_launch<C>(ctx, n, M, ld, ws, vflag, tol);
  InvGraph key{(int)sizeof(C), n, (int)ctx.engine, ld, M, ws, ctx.ws, ctx.ws_bytes, vflag, ctx.dstatus, tol,
               ctx.pivot_tau, nullptr, 0, 0};
  {
    std::lock_guard<std::mutex> lock(g_inv_mu);
    for (InvGraph& g : g_inv_graphs)
      if (g.same(key)) {
        g.used = ++g_inv_tick;
        BEM_CUDA_CHECK(cudaGraphLaunch(g.exec, ctx.stream));
        count_launches(g.kernels);
        return BEM200_OK;
      }
  }
  // record (launches of this thread only, on its private stream; nothing runs yet)
  if (!t_capture.s) BEM_CUDA_CHECK(cudaStreamCreateWithFlags(&t_capture.s, cudaStreamNonBlocking));
  if (!t_capture.fk.side) {
    BEM_CUDA_CHECK(cudaStreamCreateWithFlags(&t_capture.fk.side, cudaStreamNonBlocking));
    BEM_CUDA_CHECK(cudaEventCreateWithFlags(&t_capture.fk.fork, cudaEventDisableTiming));
    BEM_CUDA_CHECK(cudaEventCreateWithFlags(&t_capture.fk.join, cudaEventDisableTiming));
  }
  LaContext rc = ctx;
  rc.stream = t_capture.s;
  if (cudaStreamBeginCapture(rc.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    (void)cudaGetLastError();
    return inverse_nopiv_launch<C>(ctx, n, M, ld, ws, vflag, tol);  // not recordable here: direct launches
  }
  count_suspend(true);
  const int st = inverse_nopiv_launch<C>(rc, n, M, ld, ws, vflag, tol, &t_capture.fk);
  count_suspend(false);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(rc.stream, &graph);
  cudaGraphExec_t exec = nullptr;
  size_t nodes = 0;
  unsigned long long kernels = 0;
  bool ok = st == BEM200_OK && ce == cudaSuccess && graph;
  if (ok) ok = cudaGraphGetNodes(graph, nullptr, &nodes) == cudaSuccess;
  if (ok && nodes) {
    std::vector<cudaGraphNode_t> nv(nodes);
    ok = cudaGraphGetNodes(graph, nv.data(), &nodes) == cudaSuccess;
    for (size_t i = 0; ok && i < nodes; ++i) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nv[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
    }
  }
  if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (!ok) {
    (void)cudaGetLastError();
    if (st) return st;
    return inverse_nopiv_launch<C>(ctx, n, M, ld, ws, vflag, tol);  // not recordable: direct launches
  }
  std::lock_guard<std::mutex> lock(g_inv_mu);
  if (g_inv_graphs.size() >= kInvGraphCap) {
    size_t lru = 0;
    for (size_t i = 1; i < g_inv_graphs.size(); ++i)
      if (g_inv_graphs[i].used < g_inv_graphs[lru].used) lru = i;
    cudaGraphExecDestroy(g_inv_graphs[lru].exec);
    g_inv_graphs.erase(g_inv_graphs.begin() + lru);
  }
  key.exec = exec;
  key.kernels = kernels;
  key.used = ++g_inv_tick;
  g_inv_graphs.push_back(key);
  BEM_CUDA_CHECK(cudaGraphLaunch(exec, ctx.stream));
  count_launches(kernels);
  return BEM200_OK;
}

// explicit instantiations
#define BEM_INST(C)                                                                                              \
  template int gemm_v<C>(const LaContext&, int, int, int, C, RowView<C>, RowView<C>, C, RowView<C>);             \
  template int getrf<C>(const LaContext&, int, C*, long long, int32_t*, int32_t*, int32_t*);                     \
  template size_t solve_left_scratch_bytes<C>(int, int);                                                         \
  template int solve_left<C>(const LaContext&, int, int, const C*, long long, const int32_t*, C*, long long,     \
                             void*, const C*, const C*);                                                         \
  template size_t trsv_diag_inverse_bytes<C>(int);                                                               \
  template int trsv_diag_inverse<C>(const LaContext&, int, const C*, long long, const int32_t*, C*, C*);         \
  template int solve_right<C>(const LaContext&, int, int, const C*, long long, const int32_t*, C*, long long, C*); \
  template int inverse<C>(const LaContext&, int, const C*, long long, const int32_t*, C*, long long);         \
  template size_t inverse_nopiv_scratch_elems<C>(int);                                                          \
  template int inverse_nopiv<C>(const LaContext&, int, C*, long long, C*, int*, double);                       \
  template int solve_left_T<C>(const LaContext&, int, int, const C*, long long, const int32_t*, C*, long long,   \
                               void*);                                                                           \
  template size_t gemm_t_scratch_bytes<C>(int, int);                                                             \
  template int gemm_t<C>(const LaContext&, int, int, int, C, RowView<C>, RowView<C>, C, RowView<C>, void*);
BEM_INST(double2)
BEM_INST(float2)

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

// ws layout for getrf: [tensor-core operand space | 2 n int32 row-map snapshots]
static size_t getrf_snap_bytes(int n) {
  return (((size_t)2 * n * sizeof(int32_t) + 255) & ~size_t(255)) + kPanelGridScratch;
}

size_t bem200_getrf_workspace_size(int dtype, int engine, int n) {
  (void)dtype;
  if (n <= 0) return 0;
  return ((gemm_tc_workspace(n, n, n, engine_of(engine)) + 255) & ~size_t(255)) + getrf_snap_bytes(n);
}

int bem200_getrf_ex(int dtype, int engine, int n, void* A, int64_t ld, int32_t* rowmap, int32_t* ipiv, int32_t* info,
                    void* ws, size_t ws_bytes, int flags, int lookahead_nb, void* stream) {
  BEM_REQUIRE((flags & ~(BEM200_GETRF_PARTIAL_PIVOTING | BEM200_GETRF_TOURNAMENT_PIVOTING |
                          BEM200_GETRF_DIAGONAL_PIVOTS)) == 0,
              BEM200_ERR_ARG, "getrf: unknown flags 0x%x", flags);
  BEM_REQUIRE(!((flags & BEM200_GETRF_DIAGONAL_PIVOTS) && (flags & BEM200_GETRF_TOURNAMENT_PIVOTING)),
              BEM200_ERR_ARG, "getrf: diagonal and tournament pivoting exclude each other");
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_of(engine);
  ctx.ws = ws;
  ctx.ws_bytes = ws_bytes;
  ctx.dinfo = info;
  ctx.tournament = (flags & BEM200_GETRF_TOURNAMENT_PIVOTING) && !(flags & BEM200_GETRF_PARTIAL_PIVOTING);
  ctx.diag_pivots = (flags & BEM200_GETRF_DIAGONAL_PIVOTS) != 0;
  ctx.la_nb = lookahead_nb;
  int32_t* snap = nullptr;
  if (ws && n > 0 && ws_bytes >= bem200_getrf_workspace_size(dtype, engine, n)) {
    const size_t sb = getrf_snap_bytes(n);
    ctx.ws_bytes = (ws_bytes - sb) & ~size_t(255);
    snap = reinterpret_cast<int32_t*>(reinterpret_cast<char*>(ws) + ctx.ws_bytes);
  }
  if (dtype == BEM200_C128) return getrf<double2>(ctx, n, (double2*)A, ld, rowmap, ipiv, snap);
  if (dtype == BEM200_C64) return getrf<float2>(ctx, n, (float2*)A, ld, rowmap, ipiv, snap);
  set_error("getrf: bad dtype %d", dtype);
  return BEM200_ERR_ARG;
}

int bem200_getrf(int dtype, int engine, int n, void* A, int64_t ld, int32_t* rowmap, int32_t* ipiv, int32_t* info,
                 void* ws, size_t ws_bytes, void* stream) {
  return bem200_getrf_ex(dtype, engine, n, A, ld, rowmap, ipiv, info, ws, ws_bytes, 0, 0, stream);
}

size_t bem200_getrs_workspace_size(int dtype, int n, int nrhs) {
  return dtype == BEM200_C128 ? solve_left_scratch_bytes<double2>(n, nrhs) : solve_left_scratch_bytes<float2>(n, nrhs);
}

int bem200_getrs(int dtype, int engine, int n, int nrhs, const void* LU, int64_t ld, const int32_t* rowmap, void* B,
                 int64_t ldb, void* ws, size_t ws_bytes, void* scratch, int32_t* status, void* stream) {
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_of(engine);
  ctx.ws = ws;
  ctx.ws_bytes = ws_bytes;
  ctx.dstatus = status;
  if (dtype == BEM200_C128)
    return solve_left<double2>(ctx, n, nrhs, (const double2*)LU, ld, rowmap, (double2*)B, ldb, scratch);
  if (dtype == BEM200_C64)
    return solve_left<float2>(ctx, n, nrhs, (const float2*)LU, ld, rowmap, (float2*)B, ldb, scratch);
  set_error("getrs: bad dtype %d", dtype);
  return BEM200_ERR_ARG;
}

size_t bem200_inverse_nopiv_workspace_size(int dtype, int n) {
  if (n <= 0 || (dtype != BEM200_C128 && dtype != BEM200_C64)) return 0;
  const size_t e = dtype == BEM200_C128 ? inverse_nopiv_scratch_elems<double2>(n) : inverse_nopiv_scratch_elems<float2>(n);
  return e * (dtype == BEM200_C128 ? sizeof(double2) : sizeof(float2)) + 256;
}

int bem200_inverse_nopiv(int dtype, int engine, int n, void* A, int64_t ld, void* ws, size_t ws_bytes, void* scratch,
                         double tol, int32_t* info, void* stream) {
  BEM_REQUIRE(n > 0 && A && scratch && info && ld >= n, BEM200_ERR_ARG, "inverse_nopiv: bad arguments");
  BEM_REQUIRE(ld == n, BEM200_ERR_UNSUPPORTED, "inverse_nopiv: ld must equal n");
  BEM_REQUIRE(dtype == BEM200_C128 || dtype == BEM200_C64, BEM200_ERR_ARG, "inverse_nopiv: bad dtype %d", dtype);
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_of(engine);
  ctx.ws = ws;
  ctx.ws_bytes = ws_bytes;
  BEM_CUDA_CHECK(cudaMemsetAsync(info, 0, sizeof(int32_t), ctx.stream));
  if (dtype == BEM200_C128) return inverse_nopiv<double2>(ctx, n, (double2*)A, ld, (double2*)scratch, info, tol);
  return inverse_nopiv<float2>(ctx, n, (float2*)A, ld, (float2*)scratch, info, tol);
}

}  // extern "C"

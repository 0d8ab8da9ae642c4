// Dense retarded BEM on one GPU: Sigma/Delta build, the solve of
// Garcia de Abajo & Howie Eqs. (19, 20), the full FP64 BEM operator and the
// mixed-precision (complex64 factors, FP64 residual) iterative refinement.
//
// Reference behaviour followed (MNPBEM Python port v1.6.2):
//   BEMRet.init   mnpbem/bem/bem_ret.py:357-525 (MATLAB initmat.m:5-72)
//   BEMRet.solve  mnpbem/bem/bem_ret.py:1569-1831 (MATLAB mldivide.m:29-49)
//   _afun         mnpbem/bem/bem_ret_iter.py:1362-1501 (full operator)
//
// Workspace layout (element type C = complex128 for FP64, complex64 for the
// mixed path), n x n matrices, ld = n:
//   M0 G1 -> LU(G1)       M1 G2 -> LU(G2)      M2 H1 -> Sigma1
//   M3 H2 -> Sigma2 -> (scratch)               M4 Delta -> LU(Delta)
//   M5 Delta^-1           M6 Sigma -> LU(Sigma)
//   pivots: 4 x n int32, then one device int (info)
#include <vector>

#include "dense.cuh"

namespace bem200 {

constexpr int kSlots = 7;

template <typename C>
struct BemState {
  int n;
  C* M[kSlots];
  int32_t* map[4];   // rowmaps of LU(G1), LU(G2), LU(Delta), LU(Sigma)
  int32_t* ipiv[4];  // LAPACK swap sequences of the same factors
  int32_t* snap[2];  // look-ahead LU scratch (2 n row-map snapshots + grid-panel slots), one per chain
  C* dinv[6];        // diagonal-block inverses (L, U) of LU(G1), LU(G2), LU(Sigma) for the blocked solves
  int* info;
  int* status;
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

template <typename C>
static size_t state_bytes(int n) {
  size_t mat = align256(sizeof(C) * (size_t)n * n);
  return kSlots * mat + 8 * align256(sizeof(int32_t) * n) +
         2 * (align256(sizeof(int32_t) * 2 * (size_t)n) + kPanelGridScratch) + 6 * align256(trsv_diag_inverse_bytes<C>(n)) +
         256;
}

template <typename C>
static BemState<C> state_view(int n, void* ws) {
  BemState<C> s;
  s.n = n;
  char* p = reinterpret_cast<char*>(ws);
  size_t mat = align256(sizeof(C) * (size_t)n * n);
  for (int i = 0; i < kSlots; ++i) s.M[i] = reinterpret_cast<C*>(p + i * mat);
  p += kSlots * mat;
  for (int i = 0; i < 4; ++i) {
    s.map[i] = reinterpret_cast<int32_t*>(p);
    p += align256(sizeof(int32_t) * n);
    s.ipiv[i] = reinterpret_cast<int32_t*>(p);
    p += align256(sizeof(int32_t) * n);
  }
  for (int i = 0; i < 2; ++i) {  // snapshots, then the grid-panel candidate slots
    s.snap[i] = reinterpret_cast<int32_t*>(p);
    p += align256(sizeof(int32_t) * 2 * (size_t)n) + kPanelGridScratch;
  }
  for (int i = 0; i < 6; ++i) {
    s.dinv[i] = reinterpret_cast<C*>(p);
    p += align256(trsv_diag_inverse_bytes<C>(n));
  }
  s.info = reinterpret_cast<int*>(p);
  s.status = s.info + 1;
  return s;
}

// per-face or scalar eps (complex128 on the host side, converted per kernel)
struct EpsArg {
  int per_face;        // 0: scalar (e1, e2), 1: arrays d1, d2 (n complex128)
  double2 e1, e2;
  const double2* d1;
  const double2* d2;
};

__device__ __forceinline__ double2 eps_at(const EpsArg& e, int i, bool second) {
  if (!e.per_face) return second ? e.e2 : e.e1;
  return second ? e.d2[i] : e.d1[i];
}

template <typename C>
__device__ __forceinline__ C to_c(double2 v) {
  return cmake<C>(v.x, v.y);
}

// ------------------------------------------------------------ init kernels
template <typename C>
__global__ void delta_kernel(long long nn, const C* __restrict__ S1, const C* __restrict__ S2, C* __restrict__ D) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) D[i] = csub(S1[i], S2[i]);
}

// Sigma_ij = Sigma1_ij e1_j - Sigma2_ij e2_j + k^2 L_i Dinv_ij (n_i . n_j) L_j,  L = e1 - e2
template <typename C>
__global__ void sigma_kernel(int n, const C* __restrict__ S1, const C* __restrict__ S2, const C* __restrict__ Dinv,
                             const double* __restrict__ nvec, EpsArg eps, double k2, C* __restrict__ S) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * n) return;
  int i = (int)(idx / n), j = (int)(idx % n);
  double2 e1j = eps_at(eps, j, false), e2j = eps_at(eps, j, true);
  double2 Li = csub(eps_at(eps, i, false), eps_at(eps, i, true));
  double2 Lj = csub(e1j, e2j);
  double nn = nvec[3 * i] * nvec[3 * j] + nvec[3 * i + 1] * nvec[3 * j + 1] + nvec[3 * i + 2] * nvec[3 * j + 2];
  double2 s1 = make_double2(S1[idx].x, S1[idx].y), s2 = make_double2(S2[idx].x, S2[idx].y);
  double2 di = make_double2(Dinv[idx].x, Dinv[idx].y);
  double2 v = csub(cmul(s1, e1j), cmul(s2, e2j));
  v = cadd(v, cscale(cmul(cmul(Li, di), Lj), k2 * nn));
  S[idx] = to_c<C>(v);
}

// *info = -BEM200_ERR_PIVOTING if a check of a factorisation without row
// exchanges raised *vflag
__global__ void flag_to_info_kernel(const int* __restrict__ vflag, int* __restrict__ info) {
  if (*vflag) atomicExch(info, -BEM200_ERR_PIVOTING);
}

// probe tolerances of the complex64 inverses (relative to max|v|): the
// factors only precondition the FP64 refinement
constexpr double kDeltaProbeTol = 1e-2;
constexpr double kInverseProbeTol = 1e-2;

// the verdict flag of a checked factorisation: the first int of the LU
// scratch after its row-map snapshots (as getrf places it)
static int* lu_flag_of(int32_t* snap, int n) {
  return reinterpret_cast<int*>(reinterpret_cast<char*>(snap) + align256(sizeof(int32_t) * 2 * (size_t)n));
}

// Out = A B (m x k times k x n, dense row-major), split along k into slices
// whose tensor-core operand planes fit ctx's workspace
template <typename C>
static int gemm_fit(const LaContext& ctx, int m, int n, int k, const C* A, const C* B, C* Out) {
  int kc = k;
  if (ctx.engine != GemmEngine::kSimt)
    while (kc > 64 && gemm_tc_workspace(m, n, kc, ctx.engine) > ctx.ws_bytes) kc = ((kc / 2 + 63) / 64) * 64;
  const C one = cmake<C>(1.0, 0.0), zero = czero<C>();
  for (int k0 = 0; k0 < k; k0 += kc) {
    const int kk = min(kc, k - k0);
    const int st = gemm<C>(ctx, m, n, kk, one, A + k0, k, B + (long long)k0 * n, n, k0 ? one : zero, Out, n);
    if (st) return st;
  }
  return BEM200_OK;
}

// The factor chains of G1 and G2 are independent: LU(G2) and Sigma2 run on a
// second (non-blocking) stream forked from the caller's stream with events, so
// the latency-bound panel factorisations of the two chains overlap.  Each
// chain gets its own half of the tensor-core operand workspace; Sigma2 uses
// the Delta slot (free until the join) as its scratch matrix.
struct ForkJoin {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  ~ForkJoin() {
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (side) cudaStreamDestroy(side);  // released once its queued work has finished
  }
};

// Optional CUDA-event stage timer of the init: events at the start and after
// each phase, recorded on the caller's stream.
struct StageTimer {
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  ~StageTimer() {
    for (cudaEvent_t& e : ev)
      if (e) cudaEventDestroy(e);
  }
};

template <typename C>
static int bem_init_t(const LaContext& ctx, int n, void* ws, const EpsArg& eps, const double* nvec, double k0,
                      StageTimer* tm = nullptr, bool inv = false) {
  BemState<C> s = state_view<C>(n, ws);
  auto mark = [&](int i) -> int {
    if (tm) BEM_CUDA_CHECK(cudaEventRecord(tm->ev[i], ctx.stream));
    return BEM200_OK;
  };
  const long long nn = (long long)n * n;
  LaContext c = ctx;
  c.dinfo = s.info;
  c.dstatus = s.status;
  BEM_CUDA_CHECK(cudaMemsetAsync(s.info, 0, 2 * sizeof(int), ctx.stream));
  int* vf[2] = {lu_flag_of(s.snap[0], n), lu_flag_of(s.snap[1], n)};  // verdicts of the checked factorisations
  BEM_CUDA_CHECK(cudaMemsetAsync(vf[0], 0, sizeof(int), ctx.stream));
  BEM_CUDA_CHECK(cudaMemsetAsync(vf[1], 0, sizeof(int), ctx.stream));
  int st;
  if ((st = mark(0))) return st;
  // a second chain needs half of the operand workspace for the largest GEMM of
  // an LU / right solve (n x n/2 x n/2, rounded up)
  const int half = n / 2 + 64;
  const bool split_ws = ctx.engine != GemmEngine::kSimt;
  const bool fork = !split_ws || gemm_tc_workspace(n, half, half, ctx.engine) <= ctx.ws_bytes / 2;
  ForkJoin fj;
  LaContext c2 = c;
  if (fork) {
    BEM_CUDA_CHECK(cudaStreamCreateWithFlags(&fj.side, cudaStreamNonBlocking));
    BEM_CUDA_CHECK(cudaEventCreateWithFlags(&fj.fork, cudaEventDisableTiming));
    BEM_CUDA_CHECK(cudaEventCreateWithFlags(&fj.join, cudaEventDisableTiming));
    BEM_CUDA_CHECK(cudaEventRecord(fj.fork, ctx.stream));
    BEM_CUDA_CHECK(cudaStreamWaitEvent(fj.side, fj.fork, 0));
    c2.stream = fj.side;
    if (split_ws) {
      const size_t h = (ctx.ws_bytes / 2) & ~size_t(255);
      c.ws_bytes = h;
      c2.ws = reinterpret_cast<char*>(ctx.ws) + h;
      c2.ws_bytes = h;
    }
  }
  if constexpr (sizeof(C) == 8) {
    if (inv) {
      // explicit inverses (complex64): G1^-1 || G2^-1 by the block Schur
      // complement, Sigma_i = H_i G_i^-1 as products, then Delta^-1 and
      // Sigma^-1 the same way; every inverse is probe-checked
      BEM_REQUIRE(inverse_nopiv_scratch_elems<C>(n) <= (size_t)n * n, BEM200_ERR_UNSUPPORTED,
                  "bem_init: the inverse's scratch does not fit a slot");
      if ((st = inverse_nopiv<C>(c, n, s.M[0], n, s.M[4], vf[0], kInverseProbeTol))) return st;
      if ((st = gemm_fit<C>(c, n, n, n, s.M[2], s.M[0], s.M[4]))) return st;
      BEM_CUDA_CHECK(cudaMemcpyAsync(s.M[2], s.M[4], sizeof(C) * nn, cudaMemcpyDeviceToDevice, c.stream));
      if ((st = inverse_nopiv<C>(c2, n, s.M[1], n, s.M[5], vf[1], kInverseProbeTol))) return st;
      if ((st = gemm_fit<C>(c2, n, n, n, s.M[3], s.M[1], s.M[5]))) return st;
      BEM_CUDA_CHECK(cudaMemcpyAsync(s.M[3], s.M[5], sizeof(C) * nn, cudaMemcpyDeviceToDevice, c2.stream));
      if (fork) {  // (without a second chain, c2 is c: same stream, whole workspace)
        BEM_CUDA_CHECK(cudaEventRecord(fj.join, fj.side));
        BEM_CUDA_CHECK(cudaStreamWaitEvent(ctx.stream, fj.join, 0));
        c.ws_bytes = ctx.ws_bytes;
      }
      flag_to_info_kernel<<<1, 1, 0, ctx.stream>>>(vf[0], s.info);
      flag_to_info_kernel<<<1, 1, 0, ctx.stream>>>(vf[1], s.info);
      BEM_LAUNCH_CHECK();
      if ((st = mark(1))) return st;
      BEM_CUDA_CHECK(cudaMemsetAsync(vf[0], 0, sizeof(int), ctx.stream));
      delta_kernel<C><<<ceil_div(nn, 256), 256, 0, ctx.stream>>>(nn, s.M[2], s.M[3], s.M[5]);
      BEM_LAUNCH_CHECK();
      if ((st = mark(2))) return st;
      if ((st = inverse_nopiv<C>(c, n, s.M[5], n, s.M[4], vf[0], kDeltaProbeTol))) return st;
      if ((st = mark(3))) return st;
      sigma_kernel<C><<<ceil_div(nn, 256), 256, 0, ctx.stream>>>(n, s.M[2], s.M[3], s.M[5], nvec, eps, k0 * k0,
                                                                  s.M[6]);
      BEM_LAUNCH_CHECK();
      if ((st = inverse_nopiv<C>(c, n, s.M[6], n, s.M[4], vf[0], kInverseProbeTol))) return st;
      flag_to_info_kernel<<<1, 1, 0, ctx.stream>>>(vf[0], s.info);
      BEM_LAUNCH_CHECK();
      return mark(4);
    }
  }
  // chain 1: LU(G1), Sigma1 = H1 G1^-1 (M5 is scratch)
  if ((st = getrf<C>(c, n, s.M[0], n, s.map[0], s.ipiv[0], s.snap[0]))) return st;
  // chain 2: LU(G2), Sigma2 = H2 G2^-1 (M4 is scratch)
  if ((st = getrf<C>(c2, n, s.M[1], n, s.map[1], s.ipiv[1], s.snap[1]))) return st;
  if ((st = solve_right<C>(c, n, n, s.M[0], n, s.map[0], s.M[2], n, s.M[5]))) return st;
  if ((st = solve_right<C>(c2, n, n, s.M[1], n, s.map[1], s.M[3], n, fork ? s.M[4] : s.M[5]))) return st;
  if constexpr (sizeof(C) == 8) {  // complex64: diagonal-block inverses for the refinement sweeps' solves
    if ((st = trsv_diag_inverse<C>(c, n, s.M[0], n, s.map[0], s.dinv[0], s.dinv[1]))) return st;
    if ((st = trsv_diag_inverse<C>(c2, n, s.M[1], n, s.map[1], s.dinv[2], s.dinv[3]))) return st;
  }
  if (fork) {
    BEM_CUDA_CHECK(cudaEventRecord(fj.join, fj.side));
    BEM_CUDA_CHECK(cudaStreamWaitEvent(ctx.stream, fj.join, 0));
    c.ws_bytes = ctx.ws_bytes;
  }
  if ((st = mark(1))) return st;
  // Delta = Sigma1 - Sigma2, Delta^-1
  bool inverted = false;
  if constexpr (sizeof(C) == 8) {
    if (ctx.diag_pivots && inverse_nopiv_scratch_elems<C>(n) <= (size_t)n * n) {
      // complex64 with checked diagonal pivots: Delta^-1 by the block Schur
      // complement (GEMMs) instead of LU(Delta) + two n-column triangular
      // solves; a failed probe raises the pivoting flag (-> partial pivoting)
      int* vflag = vf[0];
      BEM_CUDA_CHECK(cudaMemsetAsync(vflag, 0, sizeof(int), ctx.stream));
      delta_kernel<C><<<ceil_div(nn, 256), 256, 0, ctx.stream>>>(nn, s.M[2], s.M[3], s.M[5]);
      BEM_LAUNCH_CHECK();
      if ((st = mark(2))) return st;
      if ((st = inverse_nopiv<C>(c, n, s.M[5], n, s.M[4], vflag, kDeltaProbeTol))) return st;
      flag_to_info_kernel<<<1, 1, 0, ctx.stream>>>(vflag, s.info);
      BEM_LAUNCH_CHECK();
      inverted = true;
    }
  }
  if (!inverted) {
    delta_kernel<C><<<ceil_div(nn, 256), 256, 0, ctx.stream>>>(nn, s.M[2], s.M[3], s.M[4]);
    BEM_LAUNCH_CHECK();
    if ((st = getrf<C>(c, n, s.M[4], n, s.map[2], s.ipiv[2], s.snap[0]))) return st;
    if ((st = mark(2))) return st;
    if ((st = inverse<C>(c, n, s.M[4], n, s.map[2], s.M[5], n))) return st;
  }
  if ((st = mark(3))) return st;
  // Sigma, LU(Sigma)
  sigma_kernel<C><<<ceil_div(nn, 256), 256, 0, ctx.stream>>>(n, s.M[2], s.M[3], s.M[5], nvec, eps, k0 * k0, s.M[6]);
  BEM_LAUNCH_CHECK();
  if ((st = getrf<C>(c, n, s.M[6], n, s.map[3], s.ipiv[3], s.snap[0]))) return st;
  if constexpr (sizeof(C) == 8) {
    if ((st = trsv_diag_inverse<C>(c, n, s.M[6], n, s.map[3], s.dinv[4], s.dinv[5]))) return st;
  }
  return mark(4);
}

// ------------------------------------------------------------ solve kernels
// RHS layout: phi (n, p), a (n, 3, p), alpha (n, 3, p), De (n, p), row-major.
// Work arrays use W = [sigma-like (p) | h-like (3p)] rows of width 4p.

// T = [L1 phi | a]  (n x 4p) for the Sigma1 product
template <typename C>
__global__ void solve_prep_kernel(int n, int p, const C* __restrict__ phi, const C* __restrict__ a, EpsArg eps,
                                  C* __restrict__ T) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * 4 * p) return;
  int i = (int)(idx / (4 * p)), c = (int)(idx % (4 * p));
  if (c < p) {
    double2 e1 = eps_at(eps, i, false);
    C v = phi[(long long)i * p + c];
    T[idx] = to_c<C>(cmul(e1, make_double2(v.x, v.y)));
  } else {
    T[idx] = a[(long long)i * 3 * p + (c - p)];
  }
}

// alpha_m = alpha - (Sigma1 a) + ik n (L1 phi);  De_m = De - Sigma1 (L1 phi) + ik n.(L1 a)
// S = Sigma1 T (n x 4p).  Output Am (n, 3p) and Dm (n, p).
template <typename C>
__global__ void solve_mod_kernel(int n, int p, const C* __restrict__ phi, const C* __restrict__ a,
                                 const C* __restrict__ alpha, const C* __restrict__ De, const C* __restrict__ S,
                                 const double* __restrict__ nvec, EpsArg eps, double k0, C* __restrict__ Am,
                                 C* __restrict__ Dm) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * p) return;
  int i = (int)(idx / p), q = (int)(idx % p);
  double2 e1 = eps_at(eps, i, false);
  const double2 ik = make_double2(0.0, k0);
  double nv[3] = {nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]};
  C ph = phi[(long long)i * p + q];
  double2 L1phi = cmul(e1, make_double2(ph.x, ph.y));
  const C* Si = S + (long long)i * 4 * p;
  double2 dot = make_double2(0, 0);
  for (int c = 0; c < 3; ++c) {
    long long ai = ((long long)i * 3 + c) * p + q;
    C al = alpha[ai];
    C s = Si[p + c * p + q];
    double2 v = csub(make_double2(al.x, al.y), make_double2(s.x, s.y));
    v = cadd(v, cscale(cmul(ik, L1phi), nv[c]));
    Am[ai] = to_c<C>(v);
    C av = a[ai];
    dot = cadd(dot, cscale(cmul(e1, make_double2(av.x, av.y)), nv[c]));
  }
  C de = De[idx];
  C s0 = Si[q];
  double2 v = csub(make_double2(de.x, de.y), make_double2(s0.x, s0.y));
  v = cadd(v, cmul(ik, dot));
  Dm[idx] = to_c<C>(v);
}

// rhs_sig = Dm + ik n.(L X),  X = Delta^-1 Am (n, 3p)
template <typename C>
__global__ void solve_rhs_sig_kernel(int n, int p, const C* __restrict__ Dm, const C* __restrict__ X,
                                     const double* __restrict__ nvec, EpsArg eps, double k0, C* __restrict__ out) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * p) return;
  int i = (int)(idx / p), q = (int)(idx % p);
  double2 L = csub(eps_at(eps, i, false), eps_at(eps, i, true));
  double2 dot = make_double2(0, 0);
  for (int c = 0; c < 3; ++c) {
    C x = X[((long long)i * 3 + c) * p + q];
    dot = cadd(dot, cscale(make_double2(x.x, x.y), nvec[3 * i + c]));
  }
  C d = Dm[idx];
  double2 v = cadd(make_double2(d.x, d.y), cmul(make_double2(0.0, k0), cmul(L, dot)));
  out[idx] = to_c<C>(v);
}

// rhs_h = ik n (L sig2) + Am
template <typename C>
__global__ void solve_rhs_h_kernel(int n, int p, const C* __restrict__ sig2, const C* __restrict__ Am,
                                   const double* __restrict__ nvec, EpsArg eps, double k0, C* __restrict__ out) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * 3 * p) return;
  int i = (int)(idx / (3 * p)), c = (int)((idx / p) % 3), q = (int)(idx % p);
  double2 L = csub(eps_at(eps, i, false), eps_at(eps, i, true));
  C s = sig2[(long long)i * p + q];
  C am = Am[idx];
  double2 v = cadd(make_double2(am.x, am.y),
                   cscale(cmul(make_double2(0.0, k0), cmul(L, make_double2(s.x, s.y))), nvec[3 * i + c]));
  out[idx] = to_c<C>(v);
}

// W1 = [sig2 + phi | h2 + a],  W2 = [sig2 | h2]   (n x 4p)
template <typename C>
__global__ void solve_pack_kernel(int n, int p, const C* __restrict__ sig2, const C* __restrict__ h2,
                                  const C* __restrict__ phi, const C* __restrict__ a, C* __restrict__ W1,
                                  C* __restrict__ W2) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * 4 * p) return;
  int i = (int)(idx / (4 * p)), c = (int)(idx % (4 * p));
  C s, x;
  if (c < p) {
    s = sig2[(long long)i * p + c];
    x = phi[(long long)i * p + c];
  } else {
    s = h2[(long long)i * 3 * p + (c - p)];
    x = a[(long long)i * 3 * p + (c - p)];
  }
  W1[idx] = cadd(s, x);
  W2[idx] = s;
}

template <typename C>
static size_t solve_scratch_bytes(int n, int p) {
  return align256(sizeof(C) * (size_t)n * p * 20) + 2 * align256(solve_left_scratch_bytes<C>(n, 4 * p));
}

// Solve for (W1 = [sig1 | h1], W2 = [sig2 | h2]) given RHS (phi, a, alpha, De)
// in element type C.  scratch: solve_scratch_bytes.
template <typename C>
static int bem_solve_core(const LaContext& ctx0, int n, int p, void* ws, const C* phi, const C* a, const C* alpha,
                          const C* De, const EpsArg& eps, const double* nvec, double k0, C* W1, C* W2, C* scratch,
                          bool inv = false) {
  BemState<C> s = state_view<C>(n, ws);
  LaContext ctx = ctx0;
  ctx.dstatus = s.status;
  void* lscr = reinterpret_cast<char*>(scratch) + align256(sizeof(C) * (size_t)n * p * 20);
  cudaStream_t st_ = ctx.stream;
  const long long np = (long long)n * p;
  C* T = scratch;             // n x 4p
  C* S = T + 4 * np;          // n x 4p
  C* Am = S + 4 * np;         // n x 3p
  C* Dm = Am + 3 * np;        // n x p
  C* X = Dm + np;             // n x 3p
  C* rs = X + 3 * np;         // n x p
  C* h2 = rs + np;            // n x 3p   (total 20 np)
  const C one = cmake<C>(1.0, 0.0), zero = czero<C>();
  int st;
  solve_prep_kernel<C><<<ceil_div(4 * np, 256), 256, 0, st_>>>(n, p, phi, a, eps, T);
  BEM_LAUNCH_CHECK();
  if ((st = gemm<C>(ctx, n, 4 * p, n, one, s.M[2], n, T, 4 * p, zero, S, 4 * p))) return st;
  solve_mod_kernel<C><<<ceil_div(np, 256), 256, 0, st_>>>(n, p, phi, a, alpha, De, S, nvec, eps, k0, Am, Dm);
  BEM_LAUNCH_CHECK();
  // X = Delta^-1 Am
  if ((st = gemm<C>(ctx, n, 3 * p, n, one, s.M[5], n, Am, 3 * p, zero, X, 3 * p))) return st;
  solve_rhs_sig_kernel<C><<<ceil_div(np, 256), 256, 0, st_>>>(n, p, Dm, X, nvec, eps, k0, rs);
  BEM_LAUNCH_CHECK();
  // sig2 = Sigma^-1 rs   (explicit inverse: a product into T; else in place in rs)
  const bool di = sizeof(C) == 8;  // complex64 LU factors carry diagonal-block inverses
  C* sig2 = rs;
  if (inv) {
    if ((st = gemm<C>(ctx, n, p, n, one, s.M[6], n, rs, p, zero, T, p))) return st;
    sig2 = T;
  } else if ((st = solve_left<C>(ctx, n, p, s.M[6], n, s.map[3], rs, p, lscr, di ? s.dinv[4] : nullptr,
                                 di ? s.dinv[5] : nullptr))) {
    return st;
  }
  // h2 = Delta^-1 (ik n L sig2 + Am)
  solve_rhs_h_kernel<C><<<ceil_div(3 * np, 256), 256, 0, st_>>>(n, p, sig2, Am, nvec, eps, k0, X);
  BEM_LAUNCH_CHECK();
  if ((st = gemm<C>(ctx, n, 3 * p, n, one, s.M[5], n, X, 3 * p, zero, h2, 3 * p))) return st;
  // explicit inverses: [sig2 + phi | h2 + a] and [sig2 | h2] go to S and Am..Dm
  // (free by now) and the G products write W1, W2
  C* P1 = inv ? S : W1;
  C* P2 = inv ? Am : W2;
  solve_pack_kernel<C><<<ceil_div(4 * np, 256), 256, 0, st_>>>(n, p, sig2, h2, phi, a, P1, P2);
  BEM_LAUNCH_CHECK();
  // sig1/h1 = G1^-1 W1 and sig2/h2 = G2^-1 W2 are independent: the second runs
  // on a stream forked from the caller's, with its own triangular-solve scratch
  ForkJoin fj;
  BEM_CUDA_CHECK(cudaStreamCreateWithFlags(&fj.side, cudaStreamNonBlocking));
  BEM_CUDA_CHECK(cudaEventCreateWithFlags(&fj.fork, cudaEventDisableTiming));
  BEM_CUDA_CHECK(cudaEventCreateWithFlags(&fj.join, cudaEventDisableTiming));
  BEM_CUDA_CHECK(cudaEventRecord(fj.fork, st_));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(fj.side, fj.fork, 0));
  LaContext c2 = ctx;
  c2.stream = fj.side;
  void* lscr2 = reinterpret_cast<char*>(lscr) + align256(solve_left_scratch_bytes<C>(n, 4 * p));
  if (inv) {
    if ((st = gemm<C>(ctx, n, 4 * p, n, one, s.M[0], n, P1, 4 * p, zero, W1, 4 * p))) return st;
    if ((st = gemm<C>(c2, n, 4 * p, n, one, s.M[1], n, P2, 4 * p, zero, W2, 4 * p))) return st;
  } else {
    if ((st = solve_left<C>(ctx, n, 4 * p, s.M[0], n, s.map[0], W1, 4 * p, lscr, di ? s.dinv[0] : nullptr,
                            di ? s.dinv[1] : nullptr)))
      return st;
    if ((st = solve_left<C>(c2, n, 4 * p, s.M[1], n, s.map[1], W2, 4 * p, lscr2, di ? s.dinv[2] : nullptr,
                            di ? s.dinv[3] : nullptr)))
      return st;
  }
  BEM_CUDA_CHECK(cudaEventRecord(fj.join, fj.side));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(st_, fj.join, 0));
  return BEM200_OK;
}

// ------------------------------------------------------------ transposed solve
// S^T of the solve above (S = A^-1 as computed by bem_solve_core), for the
// reverse-mode derivatives: unknown-space cotangents (W1c = [s1 | h1], W2c =
// [s2 | h2], n x 4p) -> equation-space cotangents (phi, a, alpha, De, the
// right-hand-side layout).  Every step of bem_solve_core transposed, in reverse
// order: G^-T and Sigma^-T are transposed LU solves, (Delta^-1)^T and Sigma1^T
// transposed products, the eps and normal products their own transposes.

// Bs = us1 + u2s, Bh = uh1 + u2h; phi_o = us1, a_o = uh1
template <typename C>
__global__ void tsolve_start_kernel(int n, int p, const C* __restrict__ U1, const C* __restrict__ U2, C* __restrict__ Bs,
                                    C* __restrict__ Bh, C* __restrict__ phi_o, C* __restrict__ a_o) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * 4 * p) return;
  const int i = (int)(idx / (4 * p)), c = (int)(idx % (4 * p));
  const C s = cadd(U1[idx], U2[idx]);
  if (c < p) {
    Bs[(long long)i * p + c] = s;
    phi_o[(long long)i * p + c] = U1[idx];
  } else {
    Bh[(long long)i * 3 * p + (c - p)] = s;
    a_o[(long long)i * 3 * p + (c - p)] = U1[idx];
  }
}

// Bs += ik L (n . w)
template <typename C>
__global__ void tsolve_addnw_kernel(int n, int p, const C* __restrict__ w, const double* __restrict__ nvec, EpsArg eps,
                                    double k0, C* __restrict__ Bs) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * p) return;
  const int i = (int)(idx / p), q = (int)(idx % p);
  const double2 L = csub(eps_at(eps, i, false), eps_at(eps, i, true));
  double2 dot = make_double2(0, 0);
  for (int c = 0; c < 3; ++c) {
    const C x = w[((long long)i * 3 + c) * p + q];
    dot = cadd(dot, cscale(make_double2(x.x, x.y), nvec[3 * i + c]));
  }
  const C b = Bs[idx];
  Bs[idx] = to_c<C>(cadd(make_double2(b.x, b.y), cmul(make_double2(0.0, k0), cmul(L, dot))));
}

// T = L n (x) (ik v)   (n x 3p)
template <typename C>
__global__ void tsolve_lift_kernel(int n, int p, const C* __restrict__ v, const double* __restrict__ nvec, EpsArg eps,
                                   double k0, C* __restrict__ T) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * 3 * p) return;
  const int i = (int)(idx / (3 * p)), c = (int)((idx / p) % 3), q = (int)(idx % p);
  const double2 L = csub(eps_at(eps, i, false), eps_at(eps, i, true));
  const C x = v[(long long)i * p + q];
  T[idx] = to_c<C>(cscale(cmul(make_double2(0.0, k0), cmul(L, make_double2(x.x, x.y))), nvec[3 * i + c]));
}

// VA = [v | w + t2]  (n x 4p);  De_o = v
template <typename C>
__global__ void tsolve_va_kernel(int n, int p, const C* __restrict__ v, const C* __restrict__ w,
                                 const C* __restrict__ t2, C* __restrict__ VA, C* __restrict__ De_o) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * 4 * p) return;
  const int i = (int)(idx / (4 * p)), c = (int)(idx % (4 * p));
  if (c < p) {
    const C x = v[(long long)i * p + c];
    VA[idx] = x;
    De_o[(long long)i * p + c] = x;
  } else {
    const long long o = (long long)i * 3 * p + (c - p);
    VA[idx] = cadd(w[o], t2[o]);
  }
}

// phi_o += -L1 SDT + ik L1 (n . alpham);  a_o += ik L1 (n (x) v) - SAT;  alpha_o = alpham
// with VA = [v | alpham] and SD = Sigma1^T VA = [SDT | SAT]
template <typename C>
__global__ void tsolve_finish_kernel(int n, int p, const C* __restrict__ VA, const C* __restrict__ SD,
                                     const double* __restrict__ nvec, EpsArg eps, double k0, C* __restrict__ phi_o,
                                     C* __restrict__ a_o, C* __restrict__ alpha_o) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * p) return;
  const int i = (int)(idx / p), q = (int)(idx % p);
  const double2 e1 = eps_at(eps, i, false);
  const double2 ik = make_double2(0.0, k0);
  const C* va = VA + (long long)i * 4 * p;
  const C* sd = SD + (long long)i * 4 * p;
  const double nv[3] = {nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]};
  double2 nal = make_double2(0, 0);
  const C vq = va[q];
  const double2 ikL1v = cmul(ik, cmul(e1, make_double2(vq.x, vq.y)));
  for (int c = 0; c < 3; ++c) {
    const C al = va[p + c * p + q];
    nal = cadd(nal, cscale(make_double2(al.x, al.y), nv[c]));
    const long long ai = ((long long)i * 3 + c) * p + q;
    const C sa = sd[p + c * p + q];
    const C ao = a_o[ai];
    a_o[ai] = to_c<C>(csub(cadd(make_double2(ao.x, ao.y), cscale(ikL1v, nv[c])), make_double2(sa.x, sa.y)));
    alpha_o[ai] = al;
  }
  const C sdt = sd[q];
  const C po = phi_o[idx];
  double2 ph = make_double2(po.x, po.y);
  ph = csub(ph, cmul(e1, make_double2(sdt.x, sdt.y)));
  ph = cadd(ph, cmul(ik, cmul(e1, nal)));
  phi_o[idx] = to_c<C>(ph);
}

template <typename C>
static size_t solve_T_scratch_bytes(int n, int p) {
  return align256(sizeof(C) * (size_t)n * p * 29) + align256(solve_left_scratch_bytes<C>(n, 4 * p)) +
         align256(gemm_t_scratch_bytes<C>(n, 4 * p));
}

// cot = [W1c | W2c] (8np, solution layout) -> b (8np, right-hand-side layout)
template <typename C>
static int bem_solve_T_core(const LaContext& ctx0, int n, int p, void* ws, const C* cot, const EpsArg& eps,
                            const double* nvec, double k0, C* b, void* scratch, bool inv = false) {
  BemState<C> s = state_view<C>(n, ws);
  LaContext ctx = ctx0;
  ctx.dstatus = s.status;
  cudaStream_t st_ = ctx.stream;
  const long long np = (long long)n * p;
  char* base = reinterpret_cast<char*>(scratch);
  C* U1 = reinterpret_cast<C*>(base);  // n x 4p
  C* U2 = U1 + 4 * np;                 // n x 4p
  C* Bs = U2 + 4 * np;                 // n x p
  C* Bh = Bs + np;                     // n x 3p
  C* w = Bh + 3 * np;                  // n x 3p
  C* T = w + 3 * np;                   // n x 3p
  C* t2 = T + 3 * np;                  // n x 3p
  C* VA = t2 + 3 * np;                 // n x 4p
  C* SD = VA + 4 * np;                 // n x 4p   (29 np)
  void* lscr = base + align256(sizeof(C) * (size_t)np * 29);
  void* tscr = reinterpret_cast<char*>(lscr) + align256(solve_left_scratch_bytes<C>(n, 4 * p));
  C* phi_o = b;
  C* a_o = b + np;
  C* alpha_o = b + 4 * np;
  C* De_o = b + 7 * np;
  const C one = cmake<C>(1.0, 0.0), zero = czero<C>();
  int st;
  if (inv) {  // explicit inverses: G^-T as transposed products
    if ((st = gemm_t<C>(ctx, n, 4 * p, n, one, plain(s.M[0], n), plain(const_cast<C*>(cot), 4 * p), zero,
                        plain(U1, 4 * p), tscr)))
      return st;
    if ((st = gemm_t<C>(ctx, n, 4 * p, n, one, plain(s.M[1], n), plain(const_cast<C*>(cot) + 4 * np, 4 * p), zero,
                        plain(U2, 4 * p), tscr)))
      return st;
  } else {
    BEM_CUDA_CHECK(cudaMemcpyAsync(U1, cot, sizeof(C) * 8 * np, cudaMemcpyDeviceToDevice, st_));
    if ((st = solve_left_T<C>(ctx, n, 4 * p, s.M[0], n, s.map[0], U1, 4 * p, lscr))) return st;
    if ((st = solve_left_T<C>(ctx, n, 4 * p, s.M[1], n, s.map[1], U2, 4 * p, lscr))) return st;
  }
  tsolve_start_kernel<C><<<ceil_div(4 * np, 256), 256, 0, st_>>>(n, p, U1, U2, Bs, Bh, phi_o, a_o);
  BEM_LAUNCH_CHECK();
  // w = Delta^-T Bh
  if ((st = gemm_t<C>(ctx, n, 3 * p, n, one, plain(s.M[5], n), plain(Bh, 3 * p), zero, plain(w, 3 * p), tscr)))
    return st;
  tsolve_addnw_kernel<C><<<ceil_div(np, 256), 256, 0, st_>>>(n, p, w, nvec, eps, k0, Bs);
  BEM_LAUNCH_CHECK();
  // v = Sigma^-T Bs (in place; with the explicit inverse through VA, free until tsolve_va)
  if (inv) {
    BEM_CUDA_CHECK(cudaMemcpyAsync(VA, Bs, sizeof(C) * np, cudaMemcpyDeviceToDevice, st_));
    if ((st = gemm_t<C>(ctx, n, p, n, one, plain(s.M[6], n), plain(VA, p), zero, plain(Bs, p), tscr))) return st;
  } else if ((st = solve_left_T<C>(ctx, n, p, s.M[6], n, s.map[3], Bs, p, lscr))) {
    return st;
  }
  tsolve_lift_kernel<C><<<ceil_div(3 * np, 256), 256, 0, st_>>>(n, p, Bs, nvec, eps, k0, T);
  BEM_LAUNCH_CHECK();
  if ((st = gemm_t<C>(ctx, n, 3 * p, n, one, plain(s.M[5], n), plain(T, 3 * p), zero, plain(t2, 3 * p), tscr)))
    return st;
  tsolve_va_kernel<C><<<ceil_div(4 * np, 256), 256, 0, st_>>>(n, p, Bs, w, t2, VA, De_o);
  BEM_LAUNCH_CHECK();
  // Sigma1^T [v | alpham]
  if ((st = gemm_t<C>(ctx, n, 4 * p, n, one, plain(s.M[2], n), plain(VA, 4 * p), zero, plain(SD, 4 * p), tscr)))
    return st;
  tsolve_finish_kernel<C><<<ceil_div(np, 256), 256, 0, st_>>>(n, p, VA, SD, nvec, eps, k0, phi_o, a_o, alpha_o);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// ------------------------------------------------------------ transposed FP64 operator
// A^T of the operator below, for equation-space cotangents l = (lphi, la,
// lalpha, lDe) -> unknown-space (s1, h1 | s2, h2), solution layout:
//   s1 =  G1^T lphi - ik e1 G1^T (n.lalpha) + e1 H1^T lDe
//   s2 = -G2^T lphi + ik e2 G2^T (n.lalpha) - e2 H2^T lDe
//   h1 =  G1^T la + H1^T lalpha - ik e1 G1^T (n lDe)
//   h2 = -G2^T la - H2^T lalpha + ik e2 G2^T (n lDe)
// U = [lphi | n.lalpha | la | n lDe] (n x 8p), V = [lDe | lalpha] (n x 4p).
__global__ void opT_prep_kernel(int n, int p, const double2* __restrict__ l, const double* __restrict__ nvec,
                                double2* __restrict__ U, double2* __restrict__ V) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = (long long)n * p;
  if (idx >= np) return;
  const int i = (int)(idx / p), q = (int)(idx % p);
  const double2* lphi = l;
  const double2* la = l + np;
  const double2* lal = l + 4 * np;
  const double2* lDe = l + 7 * np;
  double2* u = U + (long long)i * 8 * p;
  double2* v = V + (long long)i * 4 * p;
  const double nv[3] = {nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]};
  double2 na = make_double2(0, 0);
  const double2 de = lDe[idx];
  for (int c = 0; c < 3; ++c) {
    const long long ai = ((long long)i * 3 + c) * p + q;
    na = cadd(na, cscale(lal[ai], nv[c]));
    u[2 * p + c * p + q] = la[ai];
    u[5 * p + c * p + q] = cscale(de, nv[c]);
    v[p + c * p + q] = lal[ai];
  }
  u[q] = lphi[idx];
  u[p + q] = na;
  v[q] = de;
}

__global__ void opT_combine_kernel(int n, int p, const double2* __restrict__ GU1, const double2* __restrict__ GU2,
                                   const double2* __restrict__ HV1, const double2* __restrict__ HV2, EpsArg eps,
                                   double k0, const double2* __restrict__ wv, double2* __restrict__ r) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = (long long)n * p;
  if (idx >= 4 * np) return;
  const int i = (int)(idx / (4 * p)), c = (int)(idx % (4 * p));
  const double2 e1 = eps_at(eps, i, false), e2 = eps_at(eps, i, true);
  const double2 ik = make_double2(0.0, k0);
  const double2* g1 = GU1 + (long long)i * 8 * p;
  const double2* g2 = GU2 + (long long)i * 8 * p;
  const double2* h1 = HV1 + (long long)i * 4 * p;
  const double2* h2 = HV2 + (long long)i * 4 * p;
  double2 o1, o2;
  if (c < p) {  // s
    o1 = cadd(csub(g1[c], cmul(ik, cmul(e1, g1[p + c]))), cmul(e1, h1[c]));
    o2 = csub(cadd(cscale(g2[c], -1.0), cmul(ik, cmul(e2, g2[p + c]))), cmul(e2, h2[c]));
  } else {      // h, component (c - p)
    const int hc = c - p;
    o1 = csub(cadd(g1[2 * p + hc], h1[p + hc]), cmul(ik, cmul(e1, g1[5 * p + hc])));
    o2 = cadd(csub(cscale(g2[2 * p + hc], -1.0), h2[p + hc]), cmul(ik, cmul(e2, g2[5 * p + hc])));
  }
  if (wv) {
    o1 = csub(wv[idx], o1);
    o2 = csub(wv[4 * np + idx], o2);
  }
  r[idx] = o1;
  r[4 * np + idx] = o2;
}

static size_t apply_T_scratch_bytes(int n, int p) {
  return align256(sizeof(double2) * (size_t)n * p * 32) + align256(gemm_t_scratch_bytes<double2>(n, 16));
}

static int bem_apply_T(const LaContext& ctx, int n, int p, const double2* G1, const double2* G2, const double2* H1,
                       const double2* H2, const EpsArg& eps, const double* nvec, double k0, const double2* l,
                       const double2* wv, double2* r, void* scratch) {
  const long long np = (long long)n * p;
  double2* U = reinterpret_cast<double2*>(scratch);  // n x 8p
  double2* V = U + 8 * np;                           // n x 4p
  double2* GU1 = V + 4 * np;                         // n x 8p
  double2* GU2 = GU1 + 8 * np;                       // n x 8p
  double2* HV1 = GU2 + 8 * np;                       // n x 4p
  double2* HV2 = HV1 + 4 * np;                       // n x 4p   (32 np)
  void* tscr = reinterpret_cast<char*>(scratch) + align256(sizeof(double2) * (size_t)np * 32);
  opT_prep_kernel<<<ceil_div(np, 256), 256, 0, ctx.stream>>>(n, p, l, nvec, U, V);
  BEM_LAUNCH_CHECK();
  const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
  int st;
  // column blocks of at most 16 (8p columns for the G products, 4p for the H products)
  for (int c0 = 0; c0 < 8 * p; c0 += 16) {
    const int wc = min(16, 8 * p - c0);
    RowView<double2> Ub{U, 8 * p, nullptr, c0};
    if ((st = gemm_t<double2>(ctx, n, wc, n, one, plain(const_cast<double2*>(G1), n), Ub, zero,
                              RowView<double2>{GU1, 8 * p, nullptr, c0}, tscr)))
      return st;
    if ((st = gemm_t<double2>(ctx, n, wc, n, one, plain(const_cast<double2*>(G2), n), Ub, zero,
                              RowView<double2>{GU2, 8 * p, nullptr, c0}, tscr)))
      return st;
  }
  for (int c0 = 0; c0 < 4 * p; c0 += 16) {
    const int wc = min(16, 4 * p - c0);
    RowView<double2> Vb{V, 4 * p, nullptr, c0};
    if ((st = gemm_t<double2>(ctx, n, wc, n, one, plain(const_cast<double2*>(H1), n), Vb, zero,
                              RowView<double2>{HV1, 4 * p, nullptr, c0}, tscr)))
      return st;
    if ((st = gemm_t<double2>(ctx, n, wc, n, one, plain(const_cast<double2*>(H2), n), Vb, zero,
                              RowView<double2>{HV2, 4 * p, nullptr, c0}, tscr)))
      return st;
  }
  opT_combine_kernel<<<ceil_div(4 * np, 256), 256, 0, ctx.stream>>>(n, p, GU1, GU2, HV1, HV2, eps, k0, wv, r);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// ------------------------------------------------------------ FP64 operator
// U = [s | h | e s | e h] (n x 8p) from W = [s | h] (n x 4p)
__global__ void op_prep_kernel(int n, int p, const double2* __restrict__ W, EpsArg eps, bool second,
                               double2* __restrict__ U) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * 8 * p) return;
  int i = (int)(idx / (8 * p)), c = (int)(idx % (8 * p));
  double2 w = W[(long long)i * 4 * p + (c % (4 * p))];
  U[idx] = (c < 4 * p) ? w : cmul(eps_at(eps, i, second), w);
}

// r = b - A x with GU1 = G1 U1, GU2 = G2 U2, HU1 = H1 U1, HU2 = H2 U2 (n x 8p):
//   phi   = G1 s1 - G2 s2                          a  = G1 h1 - G2 h2
//   alpha = H1 h1 - H2 h2 - ik n (G1 e1 s1 - G2 e2 s2)
//   De    = H1 e1 s1 - H2 e2 s2 - ik n.(G1 e1 h1 - G2 e2 h2)
// b and r use the RHS layout (phi, a, alpha, De); when b is null, r = A x.
__global__ void op_combine_kernel(int n, int p, const double2* __restrict__ GU1, const double2* __restrict__ GU2,
                                  const double2* __restrict__ HU1, const double2* __restrict__ HU2,
                                  const double* __restrict__ nvec, double k0, const double2* __restrict__ bphi,
                                  const double2* __restrict__ ba, const double2* __restrict__ balpha,
                                  const double2* __restrict__ bDe, double2* __restrict__ rphi,
                                  double2* __restrict__ ra, double2* __restrict__ ralpha, double2* __restrict__ rDe) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * p) return;
  int i = (int)(idx / p), q = (int)(idx % p);
  const int w8 = 8 * p;
  const double2* g1 = GU1 + (long long)i * w8;
  const double2* g2 = GU2 + (long long)i * w8;
  const double2* h1 = HU1 + (long long)i * w8;
  const double2* h2 = HU2 + (long long)i * w8;
  const double2 ik = make_double2(0.0, k0);
  const double nv[3] = {nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]};
  const double sgn = bphi ? -1.0 : 1.0;
  // columns: s -> q, h_c -> p + c p + q, e s -> 4p + q, e h_c -> 5p + c p + q
  double2 phi = csub(g1[q], g2[q]);
  double2 Ges = csub(g1[4 * p + q], g2[4 * p + q]);
  double2 De = csub(h1[4 * p + q], h2[4 * p + q]);
  double2 dotGeh = make_double2(0, 0);
  for (int c = 0; c < 3; ++c) {
    int hc = p + c * p + q;
    double2 av = csub(g1[hc], g2[hc]);
    double2 al = csub(csub(h1[hc], h2[hc]), cscale(cmul(ik, Ges), nv[c]));
    dotGeh = cadd(dotGeh, cscale(csub(g1[4 * p + hc], g2[4 * p + hc]), nv[c]));
    long long ai = ((long long)i * 3 + c) * p + q;
    ra[ai] = bphi ? csub(ba[ai], av) : av;
    ralpha[ai] = bphi ? csub(balpha[ai], al) : al;
  }
  De = csub(De, cmul(ik, dotGeh));
  rphi[idx] = bphi ? csub(bphi[idx], phi) : phi;
  rDe[idx] = bphi ? csub(bDe[idx], De) : De;
  (void)sgn;
}

// A x (or b - A x) for x = (W1 = [s1|h1], W2 = [s2|h2]); scratch: 40 n p complex128
static int bem_apply(const LaContext& ctx, int n, int p, const double2* G1, const double2* G2, const double2* H1,
                     const double2* H2, const EpsArg& eps, const double* nvec, double k0, const double2* W1,
                     const double2* W2, const double2* b /* 8np or null */, double2* r /* 8np */,
                     double2* scratch) {
  const long long np = (long long)n * p;
  double2* U1 = scratch;
  double2* U2 = U1 + 8 * np;
  double2* GU1 = U2 + 8 * np;
  double2* GU2 = GU1 + 8 * np;
  double2* HU1 = GU2 + 8 * np;
  op_prep_kernel<<<ceil_div(8 * np, 256), 256, 0, ctx.stream>>>(n, p, W1, eps, false, U1);
  BEM_LAUNCH_CHECK();
  op_prep_kernel<<<ceil_div(8 * np, 256), 256, 0, ctx.stream>>>(n, p, W2, eps, true, U2);
  BEM_LAUNCH_CHECK();
  const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
  int st;
  if ((st = gemm<double2>(ctx, n, 8 * p, n, one, G1, n, U1, 8 * p, zero, GU1, 8 * p))) return st;
  if ((st = gemm<double2>(ctx, n, 8 * p, n, one, G2, n, U2, 8 * p, zero, GU2, 8 * p))) return st;
  if ((st = gemm<double2>(ctx, n, 8 * p, n, one, H1, n, U1, 8 * p, zero, HU1, 8 * p))) return st;
  // U1 is free now: reuse it for H2 U2
  if ((st = gemm<double2>(ctx, n, 8 * p, n, one, H2, n, U2, 8 * p, zero, U1, 8 * p))) return st;
  const double2* bp = b;
  op_combine_kernel<<<ceil_div(np, 256), 256, 0, ctx.stream>>>(
      n, p, GU1, GU2, HU1, U1, nvec, k0, bp, bp ? bp + np : nullptr, bp ? bp + 4 * np : nullptr,
      bp ? bp + 7 * np : nullptr, r, r + np, r + 4 * np, r + 7 * np);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// ------------------------------------------------------------ mixed IR
__global__ void c128_to_c64_kernel(long long n, const double2* __restrict__ x, float2* __restrict__ y, double scale) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = make_float2((float)(x[i].x * scale), (float)(x[i].y * scale));
}
__global__ void axpy_c64_to_c128_kernel(long long n, const float2* __restrict__ x, double scale,
                                        double2* __restrict__ y, bool accumulate) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 v = make_double2((double)x[i].x * scale, (double)x[i].y * scale);
  y[i] = accumulate ? cadd(y[i], v) : v;
}
// max |re|, |im| over a vector (non-negative doubles compare as integers)
__global__ void absmax_kernel(long long n, const double2* __restrict__ x, unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fmax(fabs(x[i].x), fabs(x[i].y)));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

static int absmax_host(cudaStream_t s, long long n, const double2* x, unsigned long long* dscratch, double* out) {
  BEM_CUDA_CHECK(cudaMemsetAsync(dscratch, 0, sizeof(unsigned long long), s));
  absmax_kernel<<<296, 256, 0, s>>>(n, x, dscratch);
  BEM_LAUNCH_CHECK();
  unsigned long long h = 0;
  BEM_CUDA_CHECK(cudaMemcpyAsync(&h, dscratch, sizeof(h), cudaMemcpyDeviceToHost, s));
  BEM_CUDA_CHECK(cudaStreamSynchronize(s));
  double d;
  memcpy(&d, &h, sizeof(d));
  *out = d;
  return BEM200_OK;
}

}  // namespace bem200

using namespace bem200;

static EpsArg make_eps(int per_face, const double* e1, const double* e2) {
  EpsArg e;
  e.per_face = per_face;
  e.d1 = nullptr;
  e.d2 = nullptr;
  if (per_face) {
    e.d1 = reinterpret_cast<const double2*>(e1);
    e.d2 = reinterpret_cast<const double2*>(e2);
    e.e1 = e.e2 = make_double2(0, 0);
  } else {
    e.e1 = make_double2(e1[0], e1[1]);
    e.e2 = make_double2(e2[0], e2[1]);
  }
  return e;
}

static GemmEngine engine_from(int e) {
  return e == 1 ? GemmEngine::kTcBf16x3 : (e == 2 ? GemmEngine::kTcTf32 : GemmEngine::kSimt);
}

extern "C" {

size_t bem200_bem_workspace_size(int precision, int n) {
  return precision == 0 ? state_bytes<double2>(n) : state_bytes<float2>(n);
}

int bem200_bem_slots(int precision, int n, void* ws, void** G1, void** G2, void** H1, void** H2) {
  BEM_REQUIRE(ws && n > 0, BEM200_ERR_ARG, "bem_slots: bad arguments");
  if (precision == 0) {
    BemState<double2> s = state_view<double2>(n, ws);
    *G1 = s.M[0]; *G2 = s.M[1]; *H1 = s.M[2]; *H2 = s.M[3];
  } else {
    BemState<float2> s = state_view<float2>(n, ws);
    *G1 = s.M[0]; *G2 = s.M[1]; *H1 = s.M[2]; *H2 = s.M[3];
  }
  return BEM200_OK;
}

int bem200_bem_init_ex(int precision, int engine, int n, void* ws, int eps_per_face, const double* eps1,
                       const double* eps2, const double* nvec, double k0, void* gemm_ws, size_t gemm_ws_bytes,
                       int lu_flags, int lookahead_nb, float* phase_ms, int32_t* info_host, void* stream) {
  BEM_REQUIRE(n > 0 && ws && eps1 && eps2 && nvec, BEM200_ERR_ARG, "bem_init: bad arguments");
  BEM_REQUIRE((lu_flags & ~(BEM200_GETRF_PARTIAL_PIVOTING | BEM200_GETRF_TOURNAMENT_PIVOTING |
                             BEM200_GETRF_DIAGONAL_PIVOTS)) == 0,
              BEM200_ERR_ARG, "bem_init: unknown LU flags 0x%x", lu_flags);
  BEM_REQUIRE(!((lu_flags & BEM200_GETRF_DIAGONAL_PIVOTS) && (lu_flags & BEM200_GETRF_TOURNAMENT_PIVOTING)),
              BEM200_ERR_ARG, "bem_init: diagonal and tournament pivoting exclude each other");
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_from(engine);
  ctx.ws = gemm_ws;
  ctx.ws_bytes = gemm_ws_bytes;
  ctx.tournament = (lu_flags & BEM200_GETRF_TOURNAMENT_PIVOTING) && !(lu_flags & BEM200_GETRF_PARTIAL_PIVOTING);
  ctx.diag_pivots = (lu_flags & BEM200_GETRF_DIAGONAL_PIVOTS) != 0;
  ctx.la_nb = lookahead_nb;
  EpsArg eps = make_eps(eps_per_face, eps1, eps2);
  StageTimer tm;
  if (phase_ms)
    for (cudaEvent_t& e : tm.ev) BEM_CUDA_CHECK(cudaEventCreate(&e));
  StageTimer* tp = phase_ms ? &tm : nullptr;
  BEM_REQUIRE(precision >= 0 && precision <= 2, BEM200_ERR_ARG, "bem_init: unknown precision %d", precision);
  int st = precision == 0 ? bem_init_t<double2>(ctx, n, ws, eps, nvec, k0, tp)
                          : bem_init_t<float2>(ctx, n, ws, eps, nvec, k0, tp, precision == 2);
  if (st) return st;
  if (phase_ms) {
    BEM_CUDA_CHECK(cudaEventSynchronize(tm.ev[4]));
    for (int i = 0; i < 4; ++i) BEM_CUDA_CHECK(cudaEventElapsedTime(&phase_ms[i], tm.ev[i], tm.ev[i + 1]));
  }
  if (info_host) {
    int* dinfo = precision == 0 ? state_view<double2>(n, ws).info : state_view<float2>(n, ws).info;
    BEM_CUDA_CHECK(cudaMemcpyAsync(info_host, dinfo, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    BEM_CUDA_CHECK(cudaStreamSynchronize(ctx.stream));
    BEM_REQUIRE(*info_host != -BEM200_ERR_PIVOTING, BEM200_ERR_PIVOTING,
                "bem_init: a factor matrix needs row exchanges (factor it with partial pivoting)");
    BEM_REQUIRE(*info_host != -BEM200_ERR_TIMEOUT, BEM200_ERR_TIMEOUT, "bem_init: a bounded device wait gave up");
    BEM_REQUIRE(*info_host == 0, BEM200_ERR_SINGULAR, "bem_init: exactly singular pivot at column %d", *info_host);
  }
  return BEM200_OK;
}

int bem200_bem_init(int precision, int engine, int n, void* ws, int eps_per_face, const double* eps1,
                    const double* eps2, const double* nvec, double k0, void* gemm_ws, size_t gemm_ws_bytes,
                    int32_t* info_host, void* stream) {
  return bem200_bem_init_ex(precision, engine, n, ws, eps_per_face, eps1, eps2, nvec, k0, gemm_ws, gemm_ws_bytes, 0, 0,
                            nullptr, info_host, stream);
}

size_t bem200_bem_solve_workspace_size(int precision, int n, int npol) {
  size_t np = (size_t)n * npol;
  if (precision == 0) return solve_scratch_bytes<double2>(n, npol);
  // mixed: c64 core scratch + c64 rhs/solution + c128 IR vectors + operator scratch
  return align256(solve_scratch_bytes<float2>(n, npol)) + 2 * align256(sizeof(float2) * 8 * np) +
         2 * align256(sizeof(double2) * 8 * np) + align256(sizeof(double2) * 40 * np) + 256;
}

int bem200_bem_solve(int precision, int engine, int n, int npol, void* ws, const void* phi, const void* a,
                     const void* alpha, const void* De, int eps_per_face, const double* eps1, const double* eps2,
                     const double* nvec, double k0, void* W1, void* W2, void* scratch, void* gemm_ws,
                     size_t gemm_ws_bytes, void* stream) {
  BEM_REQUIRE(precision == 0, BEM200_ERR_ARG, "bem_solve: use bem200_bem_solve_ir for the mixed path");
  BEM_REQUIRE(n > 0 && npol > 0 && ws && phi && a && alpha && De && W1 && W2 && scratch, BEM200_ERR_ARG,
              "bem_solve: bad arguments");
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_from(engine);
  ctx.ws = gemm_ws;
  ctx.ws_bytes = gemm_ws_bytes;
  EpsArg eps = make_eps(eps_per_face, eps1, eps2);
  return bem_solve_core<double2>(ctx, n, npol, ws, (const double2*)phi, (const double2*)a, (const double2*)alpha,
                                 (const double2*)De, eps, nvec, k0, (double2*)W1, (double2*)W2, (double2*)scratch);
}

int bem200_bem_status(int precision, int n, void* ws, int32_t* host_status, void* stream) {
  BEM_REQUIRE(ws && host_status && n > 0, BEM200_ERR_ARG, "bem_status: bad arguments");
  int* info = precision == 0 ? state_view<double2>(n, ws).info : state_view<float2>(n, ws).info;
  int h[2] = {0, 0};
  BEM_CUDA_CHECK(cudaMemcpyAsync(h, info, 2 * sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  BEM_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
  *host_status = h[1] ? h[1] : (h[0] ? BEM200_ERR_SINGULAR : 0);
  return BEM200_OK;
}

int bem200_bem_apply(int n, int npol, const void* G1, const void* G2, const void* H1, const void* H2,
                     int eps_per_face, const double* eps1, const double* eps2, const double* nvec, double k0,
                     const void* W1, const void* W2, const void* b, void* r, void* scratch, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && G1 && G2 && H1 && H2 && W1 && W2 && r && scratch, BEM200_ERR_ARG,
              "bem_apply: bad arguments");
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  EpsArg eps = make_eps(eps_per_face, eps1, eps2);
  return bem_apply(ctx, n, npol, (const double2*)G1, (const double2*)G2, (const double2*)H1, (const double2*)H2, eps,
                   nvec, k0, (const double2*)W1, (const double2*)W2, (const double2*)b, (double2*)r,
                   (double2*)scratch);
}

// The two ends of the FP64 operator, for operators whose four products come
// from elsewhere (the H-matrix path): U = [s | h | e s | e h] (n x 8p) from
// W = [s | h] (n x 4p) with eps of side `second`, and the combination of
// GU1 = G1 U1, GU2 = G2 U2, HU1 = H1 U1, HU2 = H2 U2 into r = A x (b NULL) or
// r = b - A x (reference BEMRetIter._afun, mnpbem/bem/bem_ret_iter.py:1362-1501).
int bem200_op_prep(int n, int npol, const void* W, int eps_per_face, const double* eps1, const double* eps2,
                   int second, void* U, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && W && U && eps1 && eps2, BEM200_ERR_ARG, "op_prep: bad arguments");
  EpsArg eps = make_eps(eps_per_face, eps1, eps2);
  const long long np = (long long)n * npol;
  op_prep_kernel<<<ceil_div(8 * np, 256), 256, 0, (cudaStream_t)stream>>>(n, npol, (const double2*)W, eps,
                                                                         second != 0, (double2*)U);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_op_combine(int n, int npol, const void* GU1, const void* GU2, const void* HU1, const void* HU2,
                      const double* nvec, double k0, const void* b, void* r, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && GU1 && GU2 && HU1 && HU2 && nvec && r, BEM200_ERR_ARG,
              "op_combine: bad arguments");
  const long long np = (long long)n * npol;
  const double2* bp = (const double2*)b;
  double2* rr = (double2*)r;
  op_combine_kernel<<<ceil_div(np, 256), 256, 0, (cudaStream_t)stream>>>(
      n, npol, (const double2*)GU1, (const double2*)GU2, (const double2*)HU1, (const double2*)HU2, nvec, k0, bp,
      bp ? bp + np : nullptr, bp ? bp + 4 * np : nullptr, bp ? bp + 7 * np : nullptr, rr, rr + np, rr + 4 * np,
      rr + 7 * np);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_convert_c128_c64(int64_t count, const void* src, void* dst, void* stream) {
  BEM_REQUIRE(count >= 0 && (count == 0 || (src && dst)), BEM200_ERR_ARG, "convert: bad arguments");
  if (count == 0) return BEM200_OK;
  c128_to_c64_kernel<<<ceil_div(count, 256), 256, 0, (cudaStream_t)stream>>>(count, (const double2*)src,
                                                                             (float2*)dst, 1.0);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// The identification of the right-hand-side space with the solution space
// used by the unpreconditioned iteration (M = I): phi -> sig1, a -> h1,
// De -> sig2, alpha -> h2, the pairing of the reference's packed vectors
// (pack(sig1, h1, sig2, h2) against pack(phi, a, De, alpha),
// mnpbem/bem/bem_ret_iter.py:1196-1233, 1499).
__global__ void relabel_kernel(int n, int p, const double2* __restrict__ b, double2* __restrict__ x) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = (long long)n * p;
  if (idx >= 4 * np) return;
  const int i = (int)(idx / (4 * p)), c = (int)(idx % (4 * p));
  const double2* phi = b;
  const double2* a = b + np;
  const double2* alpha = b + 4 * np;
  const double2* De = b + 7 * np;
  if (c < p) {
    x[idx] = phi[(long long)i * p + c];
    x[4 * np + idx] = De[(long long)i * p + c];
  } else {
    x[idx] = a[(long long)i * 3 * p + (c - p)];
    x[4 * np + idx] = alpha[(long long)i * 3 * p + (c - p)];
  }
}

int bem200_bem_relabel(int n, int npol, const void* b, void* x, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && b && x && b != x, BEM200_ERR_ARG, "bem_relabel: bad arguments");
  const long long np = (long long)n * npol;
  relabel_kernel<<<ceil_div(4 * np, 256), 256, 0, (cudaStream_t)stream>>>(n, npol, (const double2*)b, (double2*)x);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// y = M b: one application of the factored BEM solve (the preconditioner of
// the iterative solver).  b uses the right-hand-side layout, y the solution
// layout [W1 | W2]; both complex128.  precision 1 runs the complex64 factors
// (the input is scaled to unit max-norm before the cast and back after it).
int bem200_bem_precond(int precision, int engine, int n, int npol, void* ws, const void* b, int eps_per_face,
                       const double* eps1, const double* eps2, const double* nvec, double k0, void* y, void* scratch,
                       void* gemm_ws, size_t gemm_ws_bytes, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && ws && b && y && scratch, BEM200_ERR_ARG, "bem_precond: bad arguments");
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_from(engine);
  ctx.ws = gemm_ws;
  ctx.ws_bytes = gemm_ws_bytes;
  EpsArg eps = make_eps(eps_per_face, eps1, eps2);
  const long long np = (long long)n * npol;
  const double2* bb = (const double2*)b;
  double2* yy = (double2*)y;
  if (precision == 0)
    return bem_solve_core<double2>(ctx, n, npol, ws, bb, bb + np, bb + 4 * np, bb + 7 * np, eps, nvec, k0, yy,
                                   yy + 4 * np, (double2*)scratch);
  char* p = reinterpret_cast<char*>(scratch);
  float2* core = reinterpret_cast<float2*>(p);  p += align256(solve_scratch_bytes<float2>(n, npol));
  float2* rhs32 = reinterpret_cast<float2*>(p); p += align256(sizeof(float2) * 8 * np);
  float2* sol32 = reinterpret_cast<float2*>(p); p += align256(sizeof(float2) * 8 * np);
  p += 2 * align256(sizeof(double2) * 8 * np) + align256(sizeof(double2) * 40 * np);
  unsigned long long* red = reinterpret_cast<unsigned long long*>(p);
  double bn = 0;
  int st = absmax_host(ctx.stream, 8 * np, bb, red, &bn);
  if (st) return st;
  if (!(bn > 0 && bn < 1e300)) {
    BEM_CUDA_CHECK(cudaMemsetAsync(yy, 0, sizeof(double2) * 8 * np, ctx.stream));
    return BEM200_OK;
  }
  c128_to_c64_kernel<<<ceil_div(8 * np, 256), 256, 0, ctx.stream>>>(8 * np, bb, rhs32, 1.0 / bn);
  BEM_LAUNCH_CHECK();
  if ((st = bem_solve_core<float2>(ctx, n, npol, ws, rhs32, rhs32 + np, rhs32 + 4 * np, rhs32 + 7 * np, eps, nvec,
                                   k0, sol32, sol32 + 4 * np, core, precision == 2)))
    return st;
  axpy_c64_to_c128_kernel<<<ceil_div(8 * np, 256), 256, 0, ctx.stream>>>(8 * np, sol32, bn, yy, false);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

size_t bem200_bem_apply_workspace_size(int n, int npol) { return sizeof(double2) * 40 * (size_t)n * npol; }

size_t bem200_bem_solve_T_workspace_size(int precision, int n, int npol) {
  const size_t np = (size_t)n * npol;
  if (precision == 0) return solve_T_scratch_bytes<double2>(n, npol);
  return align256(solve_T_scratch_bytes<float2>(n, npol)) + 2 * align256(sizeof(float2) * 8 * np) + 256;
}

int bem200_bem_solve_T(int precision, int engine, int n, int npol, void* ws, const void* cot, int eps_per_face,
                       const double* eps1, const double* eps2, const double* nvec, double k0, void* b, void* scratch,
                       void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && ws && cot && b && scratch && eps1 && eps2 && nvec, BEM200_ERR_ARG,
              "bem_solve_T: bad arguments");
  BEM_REQUIRE(npol <= 4, BEM200_ERR_UNSUPPORTED, "bem_solve_T: at most 4 polarisations");
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_from(engine);
  EpsArg eps = make_eps(eps_per_face, eps1, eps2);
  const long long np = (long long)n * npol;
  if (precision == 0)
    return bem_solve_T_core<double2>(ctx, n, npol, ws, (const double2*)cot, eps, nvec, k0, (double2*)b, scratch);
  char* p = reinterpret_cast<char*>(scratch);
  void* core = p;                                   p += align256(solve_T_scratch_bytes<float2>(n, npol));
  float2* cot32 = reinterpret_cast<float2*>(p);     p += align256(sizeof(float2) * 8 * np);
  float2* b32 = reinterpret_cast<float2*>(p);       p += align256(sizeof(float2) * 8 * np);
  unsigned long long* red = reinterpret_cast<unsigned long long*>(p);
  double cn = 0;
  int st = absmax_host(ctx.stream, 8 * np, (const double2*)cot, red, &cn);
  if (st) return st;
  if (!(cn > 0 && cn < 1e300)) {
    BEM_CUDA_CHECK(cudaMemsetAsync(b, 0, sizeof(double2) * 8 * np, ctx.stream));
    return BEM200_OK;
  }
  c128_to_c64_kernel<<<ceil_div(8 * np, 256), 256, 0, ctx.stream>>>(8 * np, (const double2*)cot, cot32, 1.0 / cn);
  BEM_LAUNCH_CHECK();
  if ((st = bem_solve_T_core<float2>(ctx, n, npol, ws, cot32, eps, nvec, k0, b32, core, precision == 2))) return st;
  axpy_c64_to_c128_kernel<<<ceil_div(8 * np, 256), 256, 0, ctx.stream>>>(8 * np, b32, cn, (double2*)b, false);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

size_t bem200_bem_apply_T_workspace_size(int n, int npol) { return apply_T_scratch_bytes(n, npol); }

int bem200_bem_apply_T(int n, int npol, const void* G1, const void* G2, const void* H1, const void* H2,
                       int eps_per_face, const double* eps1, const double* eps2, const double* nvec, double k0,
                       const void* l, const void* w, void* r, void* scratch, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && G1 && G2 && H1 && H2 && l && r && scratch && eps1 && eps2 && nvec,
              BEM200_ERR_ARG, "bem_apply_T: bad arguments");
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  EpsArg eps = make_eps(eps_per_face, eps1, eps2);
  return bem_apply_T(ctx, n, npol, (const double2*)G1, (const double2*)G2, (const double2*)H1, (const double2*)H2,
                     eps, nvec, k0, (const double2*)l, (const double2*)w, (double2*)r, scratch);
}

int bem200_bem_solve_ir(int engine, int n, int npol, void* ws, const void* G1, const void* G2, const void* H1,
                        const void* H2, const void* b, int eps_per_face, const double* eps1, const double* eps2,
                        const double* nvec, double k0, double tol, int maxit, void* W1, void* W2, void* scratch,
                        void* gemm_ws, size_t gemm_ws_bytes, int32_t* iters, double* relres, void* stream) {
  return bem200_bem_solve_ir_ex(1, engine, n, npol, ws, G1, G2, H1, H2, b, eps_per_face, eps1, eps2, nvec, k0, tol,
                                maxit, W1, W2, scratch, gemm_ws, gemm_ws_bytes, iters, relres, stream);
}

int bem200_bem_solve_ir_ex(int precision, int engine, int n, int npol, void* ws, const void* G1, const void* G2,
                           const void* H1, const void* H2, const void* b, int eps_per_face, const double* eps1,
                           const double* eps2, const double* nvec, double k0, double tol, int maxit, void* W1,
                           void* W2, void* scratch, void* gemm_ws, size_t gemm_ws_bytes, int32_t* iters,
                           double* relres, void* stream) {
  BEM_REQUIRE(precision == 1 || precision == 2, BEM200_ERR_ARG, "bem_solve_ir: precision %d is not mixed",
              precision);
  const bool inv = precision == 2;
  BEM_REQUIRE(n > 0 && npol > 0 && ws && G1 && G2 && H1 && H2 && b && W1 && W2 && scratch && iters && relres,
              BEM200_ERR_ARG, "bem_solve_ir: bad arguments");
  LaContext ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.engine = engine_from(engine);
  ctx.ws = gemm_ws;
  ctx.ws_bytes = gemm_ws_bytes;
  EpsArg eps = make_eps(eps_per_face, eps1, eps2);
  const long long np = (long long)n * npol;
  // every sub-buffer starts on a 256-byte boundary
  char* p = reinterpret_cast<char*>(scratch);
  float2* core = reinterpret_cast<float2*>(p);        p += align256(solve_scratch_bytes<float2>(n, npol));
  float2* rhs32 = reinterpret_cast<float2*>(p);       p += align256(sizeof(float2) * 8 * np);
  float2* sol32 = reinterpret_cast<float2*>(p);       p += align256(sizeof(float2) * 8 * np);
  double2* r = reinterpret_cast<double2*>(p);         p += align256(sizeof(double2) * 8 * np);
  double2* x = reinterpret_cast<double2*>(p);         p += align256(sizeof(double2) * 8 * np);
  double2* opws = reinterpret_cast<double2*>(p);      p += align256(sizeof(double2) * 40 * np);
  unsigned long long* red = reinterpret_cast<unsigned long long*>(p);
  cudaStream_t s = ctx.stream;
  const double2* bb = (const double2*)b;
  double bnorm = 0;
  int st = absmax_host(s, 8 * np, bb, red, &bnorm);
  if (st) return st;
  BEM_REQUIRE(bnorm > 0 && bnorm < 1e300, BEM200_ERR_ARG, "bem_solve_ir: right-hand side is zero or not finite");
  // x = M b  (mixed solve, scaled to unit magnitude)
  const double2* res = bb;
  double rnorm = bnorm, prev = bnorm;
  int it = 0;
  bool first = true;
  int outcome = BEM200_OK;
  const BemState<float2> sv = state_view<float2>(n, ws);
  while (true) {
    double scale = 1.0 / rnorm;
    c128_to_c64_kernel<<<ceil_div(8 * np, 256), 256, 0, s>>>(8 * np, res, rhs32, scale);
    BEM_LAUNCH_CHECK();
    // rhs32 = [phi (np) | a (3np) | alpha (3np) | De (np)];  sol32 = [W1 (4np) | W2 (4np)]
    if ((st = bem_solve_core<float2>(ctx, n, npol, ws, rhs32, rhs32 + np, rhs32 + 4 * np, rhs32 + 7 * np, eps, nvec,
                                     k0, sol32, sol32 + 4 * np, core, inv)))
      return st;
    axpy_c64_to_c128_kernel<<<ceil_div(8 * np, 256), 256, 0, s>>>(8 * np, sol32, rnorm, x, !first);
    BEM_LAUNCH_CHECK();
    first = false;
    // r = b - A x
    if ((st = bem_apply(ctx, n, npol, (const double2*)G1, (const double2*)G2, (const double2*)H1, (const double2*)H2,
                        eps, nvec, k0, x, x + 4 * np, bb, r, opws)))
      return st;
    if ((st = absmax_host(s, 8 * np, r, red, &rnorm))) return st;
    ++it;
    {
      int hs[2] = {0, 0};  // info (first zero pivot of the factors), status (bounded waits)
      BEM_CUDA_CHECK(cudaMemcpyAsync(hs, sv.info, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      BEM_CUDA_CHECK(cudaStreamSynchronize(s));
      BEM_REQUIRE(hs[0] == 0, BEM200_ERR_SINGULAR, "bem_solve_ir: the complex64 factors hold a zero pivot (%d)",
                  hs[0]);
      BEM_REQUIRE(hs[1] == 0, BEM200_ERR_TIMEOUT, "bem_solve_ir: a bounded device wait gave up (status %d)", hs[1]);
    }
    if (rnorm <= tol * bnorm) break;
    if (!(rnorm < 1e300)) {  // NaN or overflow
      outcome = BEM200_ERR_NOCONV;
      set_error("bem_solve_ir: residual not finite after %d sweeps", it);
      break;
    }
    if (it >= maxit) {
      outcome = BEM200_ERR_NOCONV;
      set_error("bem_solve_ir: %d sweeps left the residual at %.3e of the right-hand side (tol %.3e)", it,
                rnorm / bnorm, tol);
      break;
    }
    if (it > 1 && rnorm >= prev) {  // a sweep that does not contract: refinement diverges
      outcome = BEM200_ERR_NOCONV;
      set_error("bem_solve_ir: refinement stagnates at %.3e of the right-hand side after %d sweeps", rnorm / bnorm,
                it);
      break;
    }
    prev = rnorm;
    res = r;
  }
  *iters = it;
  *relres = rnorm / bnorm;
  BEM_CUDA_CHECK(cudaMemcpyAsync(W1, x, sizeof(double2) * 4 * np, cudaMemcpyDeviceToDevice, s));
  BEM_CUDA_CHECK(cudaMemcpyAsync(W2, x + 4 * np, sizeof(double2) * 4 * np, cudaMemcpyDeviceToDevice, s));
  return outcome;
}

}  // extern "C"

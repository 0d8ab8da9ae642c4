// Dense complex linear algebra on one GPU (row-major, interleaved complex).
//
// Factorisations use "lazy" row pivoting: rows are never moved while a
// matrix is factored.  A factor is (storage, rowmap) where rowmap[i] is the
// storage row holding logical row i of P A = L U.  All kernels address rows
// through a RowView, so row exchanges cost nothing; LAPACK's ipiv (swap
// sequence) is produced as well.
//   getrf        : P A = L U with partial pivoting
//   solve_left   : B <- A^-1 B     (blocked TRSV kernel for few right-hand sides)
//   solve_right  : X <- X A^-1     (X A = Y)
//   inverse      : A^-1
//   gemm         : C <- alpha A B + beta C on row views
// Element types: double2 (complex128, FP64 arithmetic) and float2 (complex64).
// The complex64 GEMM runs on tcgen05 tensor cores when a tensor-core engine
// is selected (gemm_tc.cu), otherwise on CUDA cores.
#pragma once
#include "common.cuh"

namespace bem200 {

enum class GemmEngine : int {
  kSimt = 0,      // CUDA-core FMA (FP64 for complex128, FP32 for complex64)
  kTcBf16x3 = 1,  // complex64 on tcgen05: bf16 hi/lo split, 3 products, FP32 accumulate
  kTcTf32 = 2,    // reserved (complex64 on tcgen05 with TF32 inputs): not built, rejected by gemm_tc_c64
};

// Row-addressed matrix view: element (i, j) lives at
//   base[(map ? map[i] : i) * ld + col + j]
// `map` already points at the first logical row of the view.
template <typename C>
struct RowView {
  C* base;
  long long ld;
  const int32_t* map;
  int col;
  __host__ __device__ __forceinline__ long long off(int i, int j) const {
    return (long long)(map ? map[i] : i) * ld + col + j;
  }
  __host__ __device__ __forceinline__ C& at(int i, int j) const { return base[off(i, j)]; }
  // sub-view starting at logical row r, column c
  __host__ __device__ __forceinline__ RowView sub(int r, int c) const {
    RowView v = *this;
    if (map) v.map = map + r; else v.base = base + (long long)r * ld;
    v.col = col + c;
    return v;
  }
};

template <typename C>
inline RowView<C> plain(C* p, long long ld) {
  return RowView<C>{p, ld, nullptr, 0};
}

struct LaContext {
  cudaStream_t stream = nullptr;
  GemmEngine engine = GemmEngine::kSimt;
  void* ws = nullptr;  // scratch for the tensor-core operand preparation
  size_t ws_bytes = 0;
  int* dinfo = nullptr;     // device int: first exactly-zero pivot (1-based) or 0
  int* dstatus = nullptr;   // device int: set to a non-zero code if a bounded wait gave up
  void* panel_ws = nullptr; // candidate slots of the grid-wide panel (panels of more rows than a cluster holds)
  bool tournament = false;  // complex64 panels: tournament pivoting (false: partial pivoting, LAPACK's pivots)
  int la_nb = 0;            // look-ahead block width of getrf (multiple of 32; 0 = 128)
  bool diag_pivots = false; // getrf without the pivot search, checked against partial pivoting's choice
  float pivot_tau = 1.0f;   // ... passing when |a_ij|_1 <= tau |a_jj|_1 (1: exactly LAPACK's pivots)
  int* vflag = nullptr;     // device int raised by a panel that fails that check
};

// LU scratch beyond the row-map snapshots: the grid-wide panel's candidate
// slots (2 x up to 160 CTAs x (32 + 1) complex128); with checked diagonal
// pivots its first int is the panels' verdict flag
constexpr size_t kPanelGridScratch = 176u * 1024u;

// A non-blocking side stream forked from ctx.stream (fork()) and joined back
// into it (join()); the destructor releases the stream and events once their
// queued work has finished.  The side context gets the upper half of the
// tensor-core operand workspace, the main one keeps the lower half.
struct SideStream {
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  ~SideStream() {
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
  }
  // splits the workspace of `main`; returns false (nothing forked) on failure
  bool fork(LaContext& main, LaContext& aux) {
    if (cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) != cudaSuccess) return false;
    if (cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) != cudaSuccess) return false;
    if (cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming) != cudaSuccess) return false;
    if (cudaEventRecord(ev_fork, main.stream) != cudaSuccess) return false;
    if (cudaStreamWaitEvent(side, ev_fork, 0) != cudaSuccess) return false;
    aux = main;
    aux.stream = side;
    if (main.engine != GemmEngine::kSimt) {
      const size_t h = (main.ws_bytes / 2) & ~size_t(255);
      main.ws_bytes = h;
      aux.ws = reinterpret_cast<char*>(main.ws) + h;
      aux.ws_bytes = h;
    }
    return true;
  }
  cudaError_t join(cudaStream_t main_stream) {
    cudaError_t e = cudaEventRecord(ev_join, side);
    if (e != cudaSuccess) return e;
    return cudaStreamWaitEvent(main_stream, ev_join, 0);
  }
};

template <typename C>
int gemm_v(const LaContext& ctx, int m, int n, int k, C alpha, RowView<C> A, RowView<C> B, C beta, RowView<C> Cv);

template <typename C>
inline int gemm(const LaContext& ctx, int m, int n, int k, C alpha, const C* A, long long lda, const C* B,
                long long ldb, C beta, C* Cm, long long ldc) {
  return gemm_v<C>(ctx, m, n, k, alpha, plain(const_cast<C*>(A), lda), plain(const_cast<C*>(B), ldb), beta,
                   plain(Cm, ldc));
}

// P A = L U in place (storage rows stay put).  rowmap: n int32 (output),
// ipiv: n int32 (output, LAPACK swap sequence, 0-based).  scratch: 2 n ints
// (row-map snapshots) followed by kPanelGridScratch bytes, 256-aligned,
// selects the look-ahead schedule; NULL selects the single-stream recursive
// one.  Both give the same pivots.  Panels of more rows than one 16-CTA
// cluster holds (6144) need the scratch (grid-wide panel).
template <typename C>
int getrf(const LaContext& ctx, int n, C* A, long long ld, int32_t* rowmap, int32_t* ipiv, int32_t* scratch);

// B <- A^-1 B for the factor (LU, rowmap); B is n x nrhs (ldb).  scratch:
// solve_left_scratch_bytes.
template <typename C>
size_t solve_left_scratch_bytes(int n, int nrhs);
// dinv_l / dinv_u (optional): the diagonal-block inverses of trsv_diag_inverse.
template <typename C>
int solve_left(const LaContext& ctx, int n, int nrhs, const C* LU, long long ld, const int32_t* rowmap, C* B,
               long long ldb, void* scratch, const C* dinv_l = nullptr, const C* dinv_u = nullptr);

// Inverses of the 64 x 64 diagonal blocks of L and U of a factor, for the
// blocked triangular solves of solve_left: DL, DU trsv_diag_inverse_bytes(n)
// each.
template <typename C>
size_t trsv_diag_inverse_bytes(int n);
template <typename C>
int trsv_diag_inverse(const LaContext& ctx, int n, const C* LU, long long ld, const int32_t* rowmap, C* DL, C* DU);

// B <- A^-T B for the factor (LU, rowmap) (transposed solve, nrhs <= 16);
// scratch: solve_left_scratch_bytes.
template <typename C>
int solve_left_T(const LaContext& ctx, int n, int nrhs, const C* LU, long long ld, const int32_t* rowmap, C* B,
                 long long ldb, void* scratch);

// Cm (m x w) = alpha A^T B + beta Cm, A (k x m), B (k x w), w <= 16;
// scratch: gemm_t_scratch_bytes(m, w).  Deterministic (fixed summation order).
template <typename C>
size_t gemm_t_scratch_bytes(int m, int w);
template <typename C>
int gemm_t(const LaContext& ctx, int m, int w, int k, C alpha, RowView<C> A, RowView<C> B, C beta, RowView<C> Cv,
           void* scratch);

// X <- X A^-1 (X is m x n); tmp: m x n elements.
template <typename C>
int solve_right(const LaContext& ctx, int n, int m, const C* LU, long long ld, const int32_t* rowmap, C* X,
                long long ldx, C* tmp);

// Inv <- A^-1 (n x n, ld ldi)
template <typename C>
int inverse(const LaContext& ctx, int n, const C* LU, long long ld, const int32_t* rowmap, C* Inv, long long ldi);

// M <- M^-1 in place without pivoting (block Schur complement, Gauss-Jordan
// leaves), verified by a probe: *vflag (device int) is raised when
// M^-1 (M v) differs from v by more than tol max|v| for a fixed pseudo-random
// v, or a leaf pivot is zero or not partial pivoting's choice; M is then
// unusable.  ws: inverse_nopiv_scratch_elems(n) elements.
template <typename C>
size_t inverse_nopiv_scratch_elems(int n);
template <typename C>
int inverse_nopiv(const LaContext& ctx, int n, C* M, long long ld, C* ws, int* vflag, double tol);

// bytes of scratch the tensor-core GEMM needs for an m x n x k product
size_t gemm_tc_workspace(int m, int n, int k, GemmEngine e);
int gemm_tc_c64(const LaContext& ctx, int m, int n, int k, float2 alpha, RowView<float2> A, RowView<float2> B,
                float2 beta, RowView<float2> Cv);

}  // namespace bem200

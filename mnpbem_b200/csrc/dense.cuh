// Dense complex linear algebra on one GPU (row-major, interleaved complex).
//
// Routines are host functions that enqueue kernels on a stream; recursion is
// done on the host so that nearly all flops land in large GEMMs.
//   getrf        : P A = L U with partial pivoting (LAPACK ipiv convention,
//                  0-based global row indices)
//   solve_left   : B <- A^-1 B   using the factors
//   solve_right  : X <- X A^-1   using the factors (X A = Y)
//   gemm         : C <- alpha A B + beta C
// Element types: double2 (complex128, FP64 arithmetic) and float2 (complex64).
// The complex64 GEMM runs on tcgen05 tensor cores when the tensor-core engine
// is selected (see gemm_tc.cu), otherwise on CUDA cores.
#pragma once
#include "common.cuh"

namespace bem200 {

enum class GemmEngine : int {
  kSimt = 0,       // CUDA-core FMA (FP64 for complex128, FP32 for complex64)
  kTcBf16x3 = 1,   // complex64 on tcgen05: bf16 hi/lo split, 3 products, FP32 accumulate
  kTcTf32 = 2,     // complex64 on tcgen05: TF32 inputs, FP32 accumulate
};

struct LaContext {
  cudaStream_t stream = nullptr;
  GemmEngine engine = GemmEngine::kSimt;
  // scratch for the tensor-core operand preparation (bytes); may be null for kSimt
  void* ws = nullptr;
  size_t ws_bytes = 0;
  int* dinfo = nullptr;  // device int: first singular pivot (1-based) or 0
};

template <typename C>
int gemm(const LaContext& ctx, int m, int n, int k, C alpha, const C* A, long long lda, const C* B,
         long long ldb, C beta, C* Cm, long long ldc);

template <typename C>
int getrf(const LaContext& ctx, int n, C* A, long long ld, int32_t* ipiv);

template <typename C>
int solve_left(const LaContext& ctx, int n, int nrhs, const C* LU, long long ld, const int32_t* ipiv, C* B,
               long long ldb);

template <typename C>
int solve_right(const LaContext& ctx, int n, int m, const C* LU, long long ld, const int32_t* ipiv, C* X,
                long long ldx, C* tmp /* m x n scratch, ld = n */);

// inverse of a factored matrix into Inv (n x n, ld ldi)
template <typename C>
int inverse(const LaContext& ctx, int n, const C* LU, long long ld, const int32_t* ipiv, C* Inv, long long ldi);

// bytes of scratch the tensor-core GEMM needs for an m x n x k product
size_t gemm_tc_workspace(int m, int n, int k, GemmEngine e);
int gemm_tc_c64(const LaContext& ctx, int m, int n, int k, float2 alpha, const float2* A, long long lda,
                const float2* B, long long ldb, float2 beta, float2* Cm, long long ldc);

}  // namespace bem200

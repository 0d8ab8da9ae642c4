// Complex64 GEMM on the B200 tensor cores (tcgen05 + TMA + TMEM).
//
//   C (m x n) = alpha A (m x k) B (k x n) + beta C      (complex64, row views)
//
// Real embedding: A is used as its natural interleaved real matrix
// A' (m x 2k); B becomes B'^T (2n x 2k, K contiguous) with 2x2 blocks
//   row 2q   : [ Re B(p,q), -Im B(p,q) ]      row 2q+1 : [ Im B(p,q), Re B(p,q) ]
// so that A' B' is C in interleaved layout.  Precision: every fp32 operand x
// is split into bf16 hi = bf16(x) and lo = bf16(x - hi); the accumulator
// (FP32, in TMEM) receives hi.hi + hi.lo + lo.hi  ("bf16x3", ~2^-16 relative
// per product, FP32 accumulation).
//
// Kernel layout (one 128 x 256 real output tile per CTA):
//   warp 0      : TMA producer (A_hi, A_lo, B_hi, B_lo tiles per 32-wide K slab, 4 stages)
//   warp 1      : MMA issuer (one elected thread, tcgen05.mma kind::f16, M=128 N=256 K=16)
//   warp 2      : TMEM allocator (256 columns)
//   warps 4..7  : epilogue (tcgen05.ld, alpha/beta, complex64 stores via the row map)
// Every mbarrier wait is bounded; on timeout the kernel records an error in
// the status word, stops issuing work, waits (bounded) for its in-flight
// copies and MMAs, frees TMEM and returns.
#include <algorithm>
#include <cuda.h>
#include <cuda_bf16.h>

#include "dense.cuh"

namespace bem200 {

namespace tc {

constexpr int BM = 128;         // rows of the real output tile
constexpr int BN = 256;         // real columns of the output tile (128 complex)
constexpr int BK = 32;          // bf16 per K slab (64 bytes: one 64-byte swizzle row)
constexpr int STAGES = 4;        // 48 KB stages: three slabs in flight behind the one multiplied
constexpr int kGroupM = 16;       // tile rows per band of the grouped CTA order
constexpr int UMMA_K = 16;
constexpr int A_TILE = BM * BK * 2;   // bytes (8 KB)
constexpr int B_TILE = BN * BK * 2;   // bytes (16 KB)
constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE;  // 48 KB
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr int THREADS = 256;
constexpr long long kMaxSpin = 1LL << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; false (and *err set) on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  for (long long i = 0; i < kMaxSpin; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 32) __nanosleep(20);
  }
  atomicExch(err, BEM200_ERR_TIMEOUT);
  return false;
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// K-major, 64-byte swizzled operand tile: rows of 64 B, 8-row groups 512 B apart
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;            // leading-dimension offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;   // stride-dimension offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;            // descriptor version for tcgen05
  d |= (uint64_t)4 << 61;            // 64-byte swizzle
  return d;
}

// instruction descriptor: D f32, A/B bf16, both K-major, M = BM, N = BN
__host__ __device__ constexpr uint32_t idesc_bf16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct GemmArgs {
  int m, n, kslabs;     // kslabs: K slabs per split (the last split may have fewer)
  int kslabs_total;
  float2 alpha, beta;
  RowView<float2> C;
  float* part;          // split K: raw FP32 partial tiles [split][m][2n] (nullptr: write C)
  int* status;
};

__global__ void __launch_bounds__(THREADS, 1) gemm_bf16x3_kernel(const __grid_constant__ CUtensorMap mAh,
                                                                  const __grid_constant__ CUtensorMap mAl,
                                                                  const __grid_constant__ CUtensorMap mBh,
                                                                  const __grid_constant__ CUtensorMap mBl,
                                                                  GemmArgs args) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned tile region
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], acc_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh, issued_sh, consumed_sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Grouped tile order: consecutive CTAs sweep a band of kGroupM tile rows, so
  // the CTAs resident at one time share fewer A and B panels in L2 (bijective:
  // the last band has min(kGroupM, rows left) rows).
  const int nN = gridDim.x, nM = gridDim.y;
  const int lin = blockIdx.y * nN + blockIdx.x;
  const int per_group = kGroupM * nN;
  const int grp = lin / per_group;
  const int first_m = grp * kGroupM;
  const int rows = min(kGroupM, nM - first_m);
  const int local = lin - grp * per_group;
  const int tile_m = first_m + local % rows, tile_n = local / rows;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&acc_bar, 1);
    abort_sh = 0;
    issued_sh = 0;
    consumed_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_sh;
  const int kb0 = blockIdx.z * args.kslabs;  // first K slab of this split
  const int nk = max(0, min(args.kslabs, args.kslabs_total - kb0));

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      const uint32_t ph = (kb / STAGES) & 1;
      if (kb >= STAGES && !mbar_wait(&empty_bar[s], ph ^ 1, args.status)) {
        abort_sh = 1;
        break;
      }
      if (abort_sh) break;
      unsigned char* st = base + s * STAGE_BYTES;
      mbar_expect_tx(&full_bar[s], STAGE_BYTES);
      const int kx = (kb0 + kb) * BK;
      tma_load_2d(&mAh, &full_bar[s], st, kx, tile_m * BM);
      tma_load_2d(&mAl, &full_bar[s], st + A_TILE, kx, tile_m * BM);
      tma_load_2d(&mBh, &full_bar[s], st + 2 * A_TILE, kx, tile_n * BN);
      tma_load_2d(&mBl, &full_bar[s], st + 2 * A_TILE + B_TILE, kx, tile_n * BN);
      issued_sh = kb + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    constexpr uint32_t idesc = idesc_bf16();
    bool ok = true;
    for (int kb = 0; kb < nk && ok; ++kb) {
      const int s = kb % STAGES;
      const uint32_t ph = (kb / STAGES) & 1;
      if (!mbar_wait(&full_bar[s], ph, args.status)) {
        abort_sh = 1;
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* st = base + s * STAGE_BYTES;
      const uint32_t aH = smem_u32(st), aL = smem_u32(st + A_TILE);
      const uint32_t bH = smem_u32(st + 2 * A_TILE), bL = smem_u32(st + 2 * A_TILE + B_TILE);
#pragma unroll
      for (int kk = 0; kk < BK / UMMA_K; ++kk) {
        const uint32_t off = kk * UMMA_K * 2;  // bytes along the swizzled 64-byte row
        const uint32_t first = (kb == 0 && kk == 0) ? 0u : 1u;
        umma(tmem, sdesc(aH + off), sdesc(bH + off), idesc, first);
        umma(tmem, sdesc(aH + off), sdesc(bL + off), idesc, 1u);
        umma(tmem, sdesc(aL + off), sdesc(bH + off), idesc, 1u);
      }
      umma_commit(&empty_bar[s]);  // stage free once these MMAs retire
      consumed_sh = kb + 1;
    }
    umma_commit(&acc_bar);  // accumulator complete (or abandoned)
  } else if (warp >= 4) {
    // ---------------- epilogue: TMEM -> alpha/beta -> complex64 stores
    // Each thread of an epilogue warp owns one TMEM lane (one output row).  A
    // 16-column chunk is staged through shared memory (the pipeline stages are
    // idle once the accumulator is complete) and written back transposed, so
    // that 16 lanes store 128 contiguous bytes of one row.
    const int ew = warp - 4;  // TMEM lanes 32 ew .. 32 ew + 31
    bool ok = mbar_wait(&acc_bar, 0, args.status);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool tile_ok = ok && !abort_sh;
    float2(*stage)[17] = reinterpret_cast<float2(*)[17]>(base + ew * 32 * 17 * sizeof(float2));
    const bool use_beta = (args.beta.x != 0.f || args.beta.y != 0.f);
    const int q0 = tile_n * (BN / 2);
    const int row_base = tile_m * BM + ew * 32;
    const int half = lane >> 4, j = lane & 15;
    // element offset of this lane's row (row maps are read once per row)
    const long long my_off = (row_base + lane < args.m) ? args.C.off(row_base + lane, 0) : 0;
    const int nrows = min(32, args.m - row_base);
    if (args.part) {
      // split K: this split's raw FP32 tile, one 128-byte run of a row per
      // thread and column block, into its slice of the partial buffer
      const int row = row_base + lane;
      const int n2 = 2 * args.n;
      float* prow = args.part + ((long long)blockIdx.z * args.m + row) * n2;
      const bool vec = (n2 & 3) == 0;
#pragma unroll 1
      for (int cb = 0; cb < BN / 32; ++cb) {
        uint32_t r[32];
        tmem_ld32(tmem + ((uint32_t)(ew * 32) << 16) + cb * 32, r);  // all lanes take part
        const int c0 = tile_n * BN + cb * 32;
        if (!tile_ok || row >= args.m || c0 >= n2) continue;
        if (vec && c0 + 32 <= n2) {
#pragma unroll
          for (int j = 0; j < 32; j += 4)
            *reinterpret_cast<float4*>(prow + c0 + j) = make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]),
                                                                    __uint_as_float(r[j + 2]), __uint_as_float(r[j + 3]));
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (c0 + j < n2) prow[c0 + j] = __uint_as_float(r[j]);
        }
      }
    } else {
#pragma unroll 1
    for (int cb = 0; cb < BN / 32; ++cb) {
      uint32_t r[32];
      tmem_ld32(tmem + ((uint32_t)(ew * 32) << 16) + cb * 32, r);  // all lanes take part
      if (!tile_ok || nrows <= 0) continue;
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) stage[lane][jj] = make_float2(__uint_as_float(r[2 * jj]), __uint_as_float(r[2 * jj + 1]));
      __syncwarp();
      const int q = q0 + cb * 16 + j;
      const bool qok = q < args.n;
      long long ro[16];
      float2 cv[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) ro[i] = __shfl_sync(0xffffffffu, my_off, 2 * i + half);
      if (use_beta) {  // all 16 loads of C in flight before the first store
#pragma unroll
        for (int i = 0; i < 16; ++i)
          cv[i] = (qok && 2 * i + half < nrows) ? args.C.base[ro[i] + q] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int rr = 2 * i + half;
        if (qok && rr < nrows) {
          float2 v = cmul(args.alpha, stage[rr][j]);
          if (use_beta) v = cadd(v, cmul(args.beta, cv[i]));
          args.C.base[ro[i] + q] = v;
        }
      }
      __syncwarp();
    }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (abort_sh && threadIdx.x == 0) {
    // drain (bounded): committed MMAs retire before the accumulator barrier
    // fires; TMA copies issued but never consumed must land before exit
    mbar_wait(&acc_bar, 0, args.status);
    for (int kb = consumed_sh; kb < issued_sh; ++kb) mbar_wait(&full_bar[kb % STAGES], (kb / STAGES) & 1, args.status);
  }
  __syncthreads();
  if (warp == 2) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
  }
}

// ---------------------------------------------------------------- operand prep
// A (m x k complex, row view) -> hi/lo bf16 planes [Mp][Kp] of A' = interleaved (re, im)
__global__ void prep_a_kernel(int m, int k, RowView<float2> A, int Mp, int Kp, __nv_bfloat162* __restrict__ hi,
                              __nv_bfloat162* __restrict__ lo) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int kc = Kp / 2;  // complex columns incl. padding
  if (idx >= (long long)Mp * kc) return;
  int i = (int)(idx / kc), p = (int)(idx % kc);
  float2 v = (i < m && p < k) ? A.at(i, p) : make_float2(0.f, 0.f);
  __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
  float2 hf = __bfloat1622float2(h);
  __nv_bfloat162 l = __floats2bfloat162_rn(v.x - hf.x, v.y - hf.y);
  hi[idx] = h;
  lo[idx] = l;
}

// B (k x n complex, row view) -> hi/lo planes of B'^T [Np][Kp]:
//   row 2q: (Re, -Im) at columns (2p, 2p+1); row 2q+1: (Im, Re)
__global__ void prep_b_kernel(int k, int n, RowView<float2> B, int Np, int Kp, __nv_bfloat162* __restrict__ hi,
                              __nv_bfloat162* __restrict__ lo) {
  __shared__ float2 tile[32][33];
  const int p0 = blockIdx.y * 32, q0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int r = ty; r < 32; r += 8) {
    int p = p0 + r, q = q0 + tx;
    tile[r][tx] = (p < k && q < n) ? B.at(p, q) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const int kc = Kp / 2;
  for (int r = ty; r < 32; r += 8) {
    int q = q0 + r, p = p0 + tx;
    if (2 * q + 1 >= Np || p >= kc) continue;
    float2 b = tile[tx][r];
    float re = b.x, im = b.y;
    __nv_bfloat162 h0 = __floats2bfloat162_rn(re, -im);
    __nv_bfloat162 h1 = __floats2bfloat162_rn(im, re);
    float2 f0 = __bfloat1622float2(h0), f1 = __bfloat1622float2(h1);
    __nv_bfloat162 l0 = __floats2bfloat162_rn(re - f0.x, -im - f0.y);
    __nv_bfloat162 l1 = __floats2bfloat162_rn(im - f1.x, re - f1.y);
    long long o0 = (long long)(2 * q) * kc + p, o1 = (long long)(2 * q + 1) * kc + p;
    hi[o0] = h0;
    hi[o1] = h1;
    lo[o0] = l0;
    lo[o1] = l1;
  }
}

// split K: C = alpha (sum of the splits' partial tiles, in split order) + beta C
__global__ void splitk_reduce_kernel(int m, int n, int splits, const float2* __restrict__ part, float2 alpha,
                                     float2 beta, RowView<float2> C) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m * n) return;
  const int i = (int)(idx / n), q = (int)(idx % n);
  float2 acc = part[idx];
  for (int z = 1; z < splits; ++z) {
    const float2 v = part[(long long)z * m * n + idx];
    acc.x += v.x;
    acc.y += v.y;
  }
  float2 v = cmul(alpha, acc);
  float2& out = C.at(i, q);
  if (beta.x != 0.f || beta.y != 0.f) v = cadd(v, cmul(beta, out));
  out = v;
}

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  }
  return fn;
}

static int make_map(CUtensorMap* m, void* ptr, int rows, int cols_bf16, int box_rows) {
  EncodeFn fn = encode_fn();
  BEM_REQUIRE(fn, BEM200_ERR_CUDA, "gemm_tc: cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[2] = {(cuuint64_t)cols_bf16, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols_bf16 * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  BEM_REQUIRE(r == CUDA_SUCCESS, BEM200_ERR_CUDA, "gemm_tc: tensor map encode failed (%d)", (int)r);
  return BEM200_OK;
}

struct Plan {
  int Mp, Np, Kp;
  size_t a_bytes, b_bytes;
  int splits, kslabs;     // K splits and slabs per split
  size_t part_bytes;      // FP32 partial tiles of the splits (0 without split K)
};

// Products whose output tiles would occupy fewer than half of the 148 SMs
// split K (at least 4 slabs per split, at most 8 splits), so that about one
// CTA per SM runs; the splits' partial tiles are summed in a fixed order.
static Plan plan(int m, int n, int k) {
  Plan p;
  p.Mp = ((m + BM - 1) / BM) * BM;
  p.Np = ((2 * n + BN - 1) / BN) * BN;
  p.Kp = ((2 * k + BK - 1) / BK) * BK;
  p.a_bytes = (size_t)p.Mp * p.Kp * 2;
  p.b_bytes = (size_t)p.Np * p.Kp * 2;
  const int tiles = (p.Mp / BM) * (p.Np / BN), nk = p.Kp / BK;
  int s = 1;
  if (tiles < 74) s = std::min(std::min(8, std::max(1, 148 / tiles)), std::max(1, nk / 4));
  p.kslabs = (nk + s - 1) / s;
  p.splits = (nk + p.kslabs - 1) / p.kslabs;  // every split has at least one slab
  p.part_bytes = p.splits > 1 ? ((size_t)p.splits * m * n * sizeof(float2) + 255) / 256 * 256 : 0;
  return p;
}

}  // namespace tc

size_t gemm_tc_workspace(int m, int n, int k, GemmEngine e) {
  if (e == GemmEngine::kSimt) return 0;
  tc::Plan p = tc::plan(m, n, k);
  return 2 * p.a_bytes + 2 * p.b_bytes + 4096 + p.part_bytes;
}

int gemm_tc_c64(const LaContext& ctx, int m, int n, int k, float2 alpha, RowView<float2> A, RowView<float2> B,
                float2 beta, RowView<float2> Cv) {
  using namespace tc;
  BEM_REQUIRE(ctx.engine == GemmEngine::kTcBf16x3, BEM200_ERR_UNSUPPORTED,
              "gemm_tc: only the bf16x3 tensor-core engine is available");
  Plan p = plan(m, n, k);
  const size_t need = 2 * p.a_bytes + 2 * p.b_bytes + 4096;
  BEM_REQUIRE(ctx.ws && ctx.ws_bytes >= need, BEM200_ERR_ARG,
              "gemm_tc: workspace of %zu bytes needed for %d x %d x %d (have %zu)", need, m, n, k, ctx.ws_bytes);
  if (p.splits > 1 && ctx.ws_bytes < need + p.part_bytes) {  // no room for the partial tiles: one split
    p.splits = 1;
    p.kslabs = p.Kp / BK;
  }
  char* w = reinterpret_cast<char*>(ctx.ws);
  auto* ah = reinterpret_cast<__nv_bfloat162*>(w);
  auto* al = reinterpret_cast<__nv_bfloat162*>(w + p.a_bytes);
  auto* bh = reinterpret_cast<__nv_bfloat162*>(w + 2 * p.a_bytes);
  auto* bl = reinterpret_cast<__nv_bfloat162*>(w + 2 * p.a_bytes + p.b_bytes);
  int* status = ctx.dstatus ? ctx.dstatus : reinterpret_cast<int*>(w + 2 * p.a_bytes + 2 * p.b_bytes);
  if (!ctx.dstatus) BEM_CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int), ctx.stream));
  long long na = (long long)p.Mp * (p.Kp / 2);
  prep_a_kernel<<<ceil_div(na, 256), 256, 0, ctx.stream>>>(m, k, A, p.Mp, p.Kp, ah, al);
  BEM_LAUNCH_CHECK();
  dim3 gb(ceil_div(p.Np / 2, 32), ceil_div(p.Kp / 2, 32));
  prep_b_kernel<<<gb, 256, 0, ctx.stream>>>(k, n, B, p.Np, p.Kp, bh, bl);
  BEM_LAUNCH_CHECK();
  CUtensorMap mah, mal, mbh, mbl;
  int st;
  if ((st = make_map(&mah, ah, p.Mp, p.Kp, BM))) return st;
  if ((st = make_map(&mal, al, p.Mp, p.Kp, BM))) return st;
  if ((st = make_map(&mbh, bh, p.Np, p.Kp, BN))) return st;
  if ((st = make_map(&mbl, bl, p.Np, p.Kp, BN))) return st;
  GemmArgs args;
  args.m = m;
  args.n = n;
  args.kslabs = p.kslabs;
  args.kslabs_total = p.Kp / BK;
  args.alpha = alpha;
  args.beta = beta;
  args.C = Cv;
  args.part = p.splits > 1 ? reinterpret_cast<float*>(w + need) : nullptr;
  args.status = status;
  BEM_CUDA_CHECK(set_kernel_attrs_once(gemm_bf16x3_kernel, SMEM_BYTES, false));
  dim3 grid(p.Np / BN, p.Mp / BM, p.splits);
  BEM_REQUIRE(grid.y <= 65535, BEM200_ERR_ARG, "gemm_tc: m too large");
  gemm_bf16x3_kernel<<<grid, THREADS, SMEM_BYTES, ctx.stream>>>(mah, mal, mbh, mbl, args);
  BEM_LAUNCH_CHECK();
  if (p.splits > 1) {
    splitk_reduce_kernel<<<ceil_div((long long)m * n, 256), 256, 0, ctx.stream>>>(
        m, n, p.splits, reinterpret_cast<const float2*>(args.part), alpha, beta, Cv);
    BEM_LAUNCH_CHECK();
  }
  return BEM200_OK;
}

}  // namespace bem200

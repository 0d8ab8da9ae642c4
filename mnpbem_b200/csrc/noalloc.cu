// Allocation-free triangular solve from LU factors: bem200_getrs_noalloc.
//
// bem200_getrs needs n * nrhs elements plus a few flags of device scratch,
// which its caller allocates.  Some callers cannot: a host program that links
// only this library and has no device allocator of its own, or a caller that
// runs between kernels of another runtime whose device memory is all taken
// by that runtime's pool and where cudaMalloc / cudaFree (which synchronise
// the whole device) would stall the other streams.  For them this variant
// takes its scratch from one fixed buffer that lives in this library's
// device image.
//
// The buffer:
//   * is BEM200_GETRS_NOALLOC_MAX_BYTES (4 MiB) per GPU, held by every GPU
//     that loads the library until the process exits;
//   * is shared by every call on that GPU and keeps the last call's contents.
//     The parts that must start at zero (the block flags and the ticket of
//     the blocked triangular solve) are cleared on the stream by every call,
//     the rest is written before it is read.  Two calls whose work overlaps
//     on the GPU (different streams, no ordering between them) race on the
//     buffer and give wrong results: order them on one stream or with events.
//
// In host code the buffer's name is only a host-side stand-in, not a device
// address, so the address handed to the kernels is looked up with
// cudaGetSymbolAddress, once per device, by the first call on that device
// (with that device current).  That first call therefore does a little set-up
// work on the host and should come before any stream capture.
#include <mutex>

#include "dense.cuh"

namespace bem200 {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)BEM200_GETRS_NOALLOC_MAX_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_getrs_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_getrs_scratch on the current device (looked up once).
int scratch_address(void** out) {
  int dev = -1;
  BEM_CUDA_CHECK(cudaGetDevice(&dev));
  BEM_REQUIRE(dev >= 0 && dev < kMaxDevices, BEM200_ERR_UNSUPPORTED,
              "getrs_noalloc: device ordinal %d is above the supported %d devices", dev, kMaxDevices - 1);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    BEM_CUDA_CHECK(cudaGetSymbolAddress(&p, g_getrs_scratch));
    BEM_REQUIRE(p != nullptr, BEM200_ERR_CUDA, "getrs_noalloc: cudaGetSymbolAddress returned a null address");
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return BEM200_OK;
}

template <typename C>
int getrs_noalloc(int n, int nrhs, const void* LU, int64_t ld, const int32_t* rowmap, void* B, int64_t ldb,
                  int32_t* status, cudaStream_t stream) {
  const size_t need = solve_left_scratch_bytes<C>(n, nrhs);
  BEM_REQUIRE(need <= kNoAllocScratchBytes, BEM200_ERR_ARG,
              "getrs_noalloc: n = %d with nrhs = %d needs %zu bytes of scratch, more than the fixed %zu-byte "
              "buffer; use bem200_getrs with caller-provided scratch",
              n, nrhs, need, kNoAllocScratchBytes);
  void* scratch = nullptr;
  int st = scratch_address(&scratch);
  if (st) return st;
  LaContext ctx;
  ctx.stream = stream;
  ctx.engine = GemmEngine::kSimt;
  ctx.dstatus = status;
  return solve_left<C>(ctx, n, nrhs, reinterpret_cast<const C*>(LU), ld, rowmap, reinterpret_cast<C*>(B), ldb,
                       scratch);
}

}  // namespace
}  // namespace bem200

using namespace bem200;

extern "C" int bem200_getrs_noalloc(int dtype, int n, int nrhs, const void* LU, int64_t ld, const int32_t* rowmap,
                                    void* B, int64_t ldb, int32_t* status, void* stream) {
  BEM_REQUIRE(n > 0 && nrhs >= 0 && ld >= n && ldb >= nrhs, BEM200_ERR_ARG,
              "getrs_noalloc: bad sizes (n = %d, nrhs = %d, ld = %lld, ldb = %lld)", n, nrhs, (long long)ld,
              (long long)ldb);
  BEM_REQUIRE(LU && rowmap && B, BEM200_ERR_ARG, "getrs_noalloc: null pointer");
  if (dtype == BEM200_C128)
    return getrs_noalloc<double2>(n, nrhs, LU, ld, rowmap, B, ldb, status, (cudaStream_t)stream);
  if (dtype == BEM200_C64)
    return getrs_noalloc<float2>(n, nrhs, LU, ld, rowmap, B, ldb, status, (cudaStream_t)stream);
  set_error("getrs_noalloc: bad dtype %d", dtype);
  return BEM200_ERR_ARG;
}

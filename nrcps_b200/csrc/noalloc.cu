// noalloc.cu -- nrcps_slater_dets_noalloc: the leading-minor determinants
// without any device allocation.
//
// nrcps_slater_dets needs working memory for its per-thread LU factors when
// N > 64 and takes it from the context, which grows it with cudaMalloc when a
// call needs more.  Some callers cannot let a library allocate: a host
// program that has already handed (nearly) all device memory to its own
// caching pool -- PyTorch's allocator is the usual case -- where an extra
// cudaMalloc fails or fragments that pool, and measurement code that runs
// between kernels already queued on a stream, where an allocation may
// synchronise the whole device.  For them this entry point uses no memory
// beyond its inputs and outputs for N <= 64 (one warp per minor, the factor
// in shared memory, as nrcps_slater_dets does) and, for N > 64, takes its
// working memory from one fixed array compiled into the library.
//
// The array is file-scope device memory: every GPU that loads the library
// holds it (kNoAllocScratchBytes, 16 MiB) until the process exits.  Host
// code cannot use the array's name as a device address, so the first N > 64
// call on each device looks the address up with cudaGetSymbolAddress (with
// that device current) and remembers it; make that first call before any
// stream capture.  All calls share the one array: calls whose kernels can
// overlap on the GPU (different streams, or different host threads) race on
// it and must be serialised by the caller.  Nothing in it needs to start at
// zero: each LU factor is written in full before it is read.
#include <mutex>

#include "common.cuh"

namespace nrcps {

size_t slater_dets_scratch_bytes(int N, int nconf, int mode);
nrcps_status slater_dets_warp(nrcps_context* ctx, const double* S, const double* psi1, int N, int nconf, int mode,
                              int log_det, double* out, long out_conf_stride, long out_offset);
nrcps_status slater_dets_impl(nrcps_context* ctx, const double* S, const double* psi1, int N, int nconf, int mode,
                              int log_det, double* out, long out_conf_stride, long out_offset, double* scr);

constexpr size_t kNoAllocScratchBytes = 16u << 20;  // 16 MiB
constexpr int kNoAllocWarpMaxN = 64;                  // the warp kernel's limit (no working memory)

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch_addr[kMaxDevices] = {};
}  // namespace

// Device address of g_noalloc_scratch on the current device (looked up once).
static nrcps_status noalloc_scratch(nrcps_context* ctx, double** out) {
  int dev = -1;
  NRCPS_TRY(check_cuda(ctx, cudaGetDevice(&dev), "cudaGetDevice"));
  if (dev < 0 || dev >= kMaxDevices) return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess) return check_cuda(ctx, e, "cudaGetSymbolAddress(noalloc scratch)");
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return NRCPS_OK;
}

}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_slater_dets_noalloc(nrcps_context* ctx, const double* dev_S, const double* dev_psi1,
                                                  int N, int nconf, int mode, int log_det, double* dev_out) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, N > 0 && nconf >= 0 && (mode == 0 || mode == 1), "nrcps_slater_dets_noalloc: bad arguments");
  const bool warp = N <= kNoAllocWarpMaxN;
  const size_t need = warp ? 0 : slater_dets_scratch_bytes(N, nconf, mode);
  if (need > kNoAllocScratchBytes)
    return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT,
                     "nrcps_slater_dets_noalloc: %d matrices of size %d need %zu bytes of working memory, "
                     "more than the fixed %zu; split the batch or use nrcps_slater_dets",
                     nconf, N, need, kNoAllocScratchBytes);
  if (nconf == 0) return NRCPS_OK;  // an empty batch: nothing to read or write, null buffers allowed
  NRCPS_REQUIRE(ctx, dev_S && dev_out && (mode == 0 || dev_psi1), "nrcps_slater_dets_noalloc: null pointer");
  NRCPS_REQUIRE(ctx, ctx->device >= 0, "nrcps_slater_dets_noalloc: bad context");
  int cur = -1;
  NRCPS_TRY(check_cuda(ctx, cudaGetDevice(&cur), "cudaGetDevice"));
  if (cur != ctx->device) NRCPS_TRY(check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice"));
  const int nmeas = mode ? 2 * N : N;
  nrcps_status st = NRCPS_OK;
  if (warp) {
    st = slater_dets_warp(ctx, dev_S, dev_psi1, N, nconf, mode, log_det, dev_out, 2L * nmeas, 0);
  } else {
    double* scr = nullptr;
    st = noalloc_scratch(ctx, &scr);
    if (st == NRCPS_OK) st = slater_dets_impl(ctx, dev_S, dev_psi1, N, nconf, mode, log_det, dev_out, 2L * nmeas, 0, scr);
  }
  if (cur != ctx->device) cudaSetDevice(cur);
  return st;
}

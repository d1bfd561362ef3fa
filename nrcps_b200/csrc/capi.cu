// capi.cu -- context lifecycle, error reporting and scratch memory of the C ABI.
#include <cstdarg>
#include <cstdio>

#include "common.cuh"

namespace nrcps {

nrcps_status set_error(nrcps_context* ctx, nrcps_status st, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return st;
}

nrcps_status check_cuda(nrcps_context* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return NRCPS_OK;
  nrcps_status st = (e == cudaErrorMemoryAllocation) ? NRCPS_ERR_OUT_OF_MEMORY : NRCPS_ERR_CUDA;
  return set_error(ctx, st, "%s: %s", what, cudaGetErrorString(e));
}

nrcps_status check_launch(nrcps_context* ctx, const char* what) {
  return check_cuda(ctx, cudaGetLastError(), what);
}

void* scratch(nrcps_context* ctx, size_t bytes, nrcps_status* st) {
  *st = NRCPS_OK;
  // a side-stream field draw may still be using the scratch (no scratch
  // user runs inside a graph capture, where an outside event cannot be waited)
  if (ctx->side_pending) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->stream, &cs);
    if (cs == cudaStreamCaptureStatusNone) cudaStreamWaitEvent(ctx->stream, ctx->side_done, 0);
  }
  if (bytes <= ctx->scratch_bytes) return ctx->scratch;
  if (ctx->scratch) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
  }
  size_t want = bytes + bytes / 4;
  cudaError_t e = cudaMalloc(&ctx->scratch, want);
  if (e != cudaSuccess) {
    *st = check_cuda(ctx, e, "cudaMalloc(scratch)");
    ctx->scratch = nullptr;
    return nullptr;
  }
  ctx->scratch_bytes = want;
  return ctx->scratch;
}

}  // namespace nrcps

using namespace nrcps;

extern "C" const char* nrcps_version(void) { return "nrcps_b200 0.1 sm_100a"; }

extern "C" nrcps_status nrcps_create(int device, nrcps_context** out) {
  if (!out) return NRCPS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return NRCPS_ERR_CUDA;
  if (device < 0 || device >= n) return NRCPS_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return NRCPS_ERR_CUDA;
  nrcps_context* ctx = new nrcps_context();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaMalloc((void**)&ctx->dev_err, 2 * sizeof(int)) != cudaSuccess ||
      cudaMemset(ctx->dev_err, 0, 2 * sizeof(int)) != cudaSuccess) {
    delete ctx;
    return NRCPS_ERR_CUDA;
  }
  ctx->dev_pair_flag = ctx->dev_err + 1;
  *out = ctx;
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_destroy(nrcps_context* ctx) {
  if (!ctx) return NRCPS_OK;
  cudaStreamSynchronize(ctx->stream);
  cudaDeviceSynchronize();  // side-stream draws included
  if (ctx->side_done) cudaEventDestroy(ctx->side_done);
  if (ctx->scratch) cudaFree(ctx->scratch);
  if (ctx->gen_args) cudaFree(ctx->gen_args);
  if (ctx->kin_f32) cudaFree(ctx->kin_f32);
  if (ctx->zpos) cudaFree(ctx->zpos);
  if (ctx->tc_split) cudaFree(ctx->tc_split);
  if (ctx->dev_err) cudaFree(ctx->dev_err);
  delete ctx;
  return NRCPS_OK;
}

extern "C" const char* nrcps_last_error(const nrcps_context* ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

extern "C" nrcps_status nrcps_set_stream(nrcps_context* ctx, void* stream) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  ctx->stream = (cudaStream_t)stream;
  return NRCPS_OK;
}

namespace nrcps {
nrcps_status fused_autotune(nrcps_context* ctx, nrcps_precision prec, int L, int* chosen_cluster);
nrcps_status fused_choice(nrcps_context* ctx, nrcps_precision prec, int L, int* kind, int* cluster);
}

extern "C" nrcps_status nrcps_set_option(nrcps_context* ctx, const char* name, long value) {
  if (!ctx || !name) return NRCPS_ERR_INVALID_ARGUMENT;
  std::string n(name);
  if (n == "propagate.fused") {
    ctx->fused_enabled = value != 0;
  } else if (n == "fused.cluster") {
    if (value < 0 || value > 16) return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT, "fused.cluster out of range");
    ctx->fused_cluster = (int)value;
  } else if (n == "fused.split") {
    if (value < -1 || value > 1) return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT, "fused.split out of range");
    ctx->fused_split = (int)value;
  } else if (n == "fused.kind") {
    if (value < -1 || value > 12) return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT, "fused.kind out of range");
    ctx->fused_kind = (int)value;
  } else if (n == "fused.wait_ns") {
    if (value < 1000) return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT, "fused.wait_ns below 1000 ns");
    ctx->fused_wait_ns = (unsigned long long)value;
  } else if (n == "fused.stall_test") {
    ctx->fused_stall_test = value != 0;
  } else if (n == "lu.warp") {
    ctx->lu_warp = value != 0;
  } else if (n == "overlap.tc") {
    ctx->overlap_tc = value != 0;
  } else if (n == "fused.zpos") {
    ctx->fused_zpos = value != 0;
  } else if (n == "pair.tile") {
    ctx->pair_tile = value != 0;
  } else if (n == "qr.gram_tc") {
    ctx->qr_gram_tc = value != 0;
  } else if (n == "batch.real_weights") {
    ctx->batch_real_weights = value != 0;
  } else if (n == "batch.prefetch_fields") {
    ctx->batch_prefetch_fields = value != 0;
  } else {
    return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT, "unknown option %s", name);
  }
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_autotune(nrcps_context* ctx, nrcps_precision prec, int L, int* cluster) {
  if (!ctx || L <= 0 || L >= 64) return NRCPS_ERR_INVALID_ARGUMENT;
  if (cluster) *cluster = 0;
  return fused_autotune(ctx, prec, L, cluster);
}

extern "C" nrcps_status nrcps_fused_choice(nrcps_context* ctx, nrcps_precision prec, int L, int* kind, int* cluster) {
  if (!ctx || !kind || !cluster || L <= 0) return NRCPS_ERR_INVALID_ARGUMENT;
  if (prec != NRCPS_F32 && prec != NRCPS_F64) return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT, "bad precision");
  return fused_choice(ctx, prec, L, kind, cluster);
}

// Waits for the context's stream, then reports a timed-out bounded wait in
// any kernel since the last check (NRCPS_ERR_TIMEOUT; the flag is cleared).
extern "C" nrcps_status nrcps_synchronize(nrcps_context* ctx) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_TRY(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"));
  int flag = 0;
  NRCPS_TRY(check_cuda(ctx, cudaMemcpy(&flag, ctx->dev_err, sizeof(int), cudaMemcpyDeviceToHost), "read flag"));
  if (flag) {
    cudaMemset(ctx->dev_err, 0, sizeof(int));
    return set_error(ctx, NRCPS_ERR_TIMEOUT, "a device wait timed out (bulk copy did not complete)");
  }
  return NRCPS_OK;
}

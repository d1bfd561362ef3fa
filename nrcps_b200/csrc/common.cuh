// common.cuh -- shared types and helpers of libnrcps_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/nrcps_b200.h"

namespace nrcps {

// ------------------------------------------------------------------ complex
// Aligned to its full size so that shared/global accesses are single
// 8-byte (FP32) or 16-byte (FP64) transactions.
template <typename R>
struct alignas(2 * sizeof(R)) cplx {
  R re, im;
};

// Vector type carrying one complex number, for 8/16-byte accesses.
template <typename R>
struct vec2;
template <>
struct vec2<float> {
  typedef float2 type;
};
template <>
struct vec2<double> {
  typedef double2 type;
};

template <typename R>
__device__ __forceinline__ cplx<R> ld(const void* base, long i) {
  typedef typename vec2<R>::type V;
  V v = reinterpret_cast<const V*>(base)[i];
  return cplx<R>{v.x, v.y};
}
template <typename R>
__device__ __forceinline__ void st(void* base, long i, cplx<R> c) {
  typedef typename vec2<R>::type V;
  V v;
  v.x = c.re;
  v.y = c.im;
  reinterpret_cast<V*>(base)[i] = v;
}

template <typename R>
__host__ __device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b) {
  return cplx<R>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// x * (hi + lo) for a real factor carried as two floats in FP32:
// fma(x, hi, x*lo) adds the small product before the single rounding of the
// sum.  Rounding x*lo first costs at most 2^-24 |x lo| <= 2^-48 |x hi|, so
// the result is the correctly rounded x*(hi + lo) but for sums within 2^-48
// of a rounding boundary.  A plain x*k with k rounded to one float -- or
// fma(x, lo, x*hi), which rounds x*hi first and so loses lo -- scales a mode
// by the same wrong factor every step: a deterministic drift of ~1e-8 per
// application that reaches ~5e-6 in |det|^2 after 32 steps.
template <typename R>
__host__ __device__ __forceinline__ R mul2(R x, R hi, R lo) {
  if constexpr (sizeof(R) == 4) {
    return fmaf(x, hi, x * lo);
  } else {
    return x * hi;
  }
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> scale2(cplx<R> x, R hi, R lo) {
  return cplx<R>{mul2<R>(x.re, hi, lo), mul2<R>(x.im, hi, lo)};
}

template <typename R>
__device__ __forceinline__ void split(double v, R& hi, R& lo) {
  hi = (R)v;
  lo = (sizeof(R) == 4) ? (R)(v - (double)hi) : (R)0;
}

// ---------------------------------------------------------------- context
struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  int sm_count = 148;
  // Scratch owned by the context (grown on demand, never shrunk).
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // The last field draw issued on a side stream (a batch drawing its next
  // run's fields during a run); work on the context's stream that uses the
  // shared scratch waits for it, and each side draw waits for the previous.
  cudaEvent_t side_done = nullptr;
  bool side_pending = false;
  long launches = 0;  // kernels queued through this context
  // Device copy of the ranlux generation arguments for (gen_kind, gen_seed).
  void* gen_args = nullptr;
  int gen_kind = -1;
  long gen_seed = 0;
  // Tuning options (nrcps_set_option).
  int fused_enabled = 1;  // single-pass cluster kernel where a variant exists
  int fused_cluster = 0;  // 0: autotuned / default cluster size
  int fused_split = -1;   // -1: autotuned; 0: one lane per pencil; 1: two lanes per pencil
  int fused_kind = -1;    // -1: autotuned; else the fused kernel's kind (0..10)
  int lu_warp = 1;        // 1: warp-per-minor determinant kernel for N <= 64; 0: thread-per-minor kernel
  int overlap_tc = 1;     // 1: tensor-core overlap for FP32 orbitals where the shape allows; 0: CUDA cores
  int fused_zpos = 1;     // 1: Z2 fields with a position factor read per-site weight tables in the fused step
  int pair_tile = 1;      // 1: pair matrices by the tiled cluster kernel (n <= 32); 0: one block per (s, t)
  int qr_gram_tc = 0;     // 1: QR Gram matrices of FP32 orbitals on the tensor cores (N <= 32); 0: CUDA cores
  int batch_real_weights = 1;  // 1: FP32 batches with real Gaussian fields step on one FP32 weight per site
  int batch_prefetch_fields = 1;  // 1: such batches draw the next run's fields during a run (two weight buffers)
  // TF32 hi / lo split of the sources for nrcps_overlap's tensor-core path (grown on demand)
  void* tc_split = nullptr;
  size_t tc_split_bytes = 0;
  int* dev_err = nullptr;
  int* dev_pair_flag = nullptr;  // the word after dev_err: 1 = the last checked opposite-site table is no involution  // device flag set by kernels whose bounded waits time out
  // Time limit of every mbarrier wait in the fused step (nanoseconds of the
  // GPU's global timer; the legitimate waits take microseconds).
  unsigned long long fused_wait_ns = 2000000000ull;
  // Time-out test: the first wait of one CTA of the fused step is on an
  // mbarrier nothing arrives on, so that it runs out (nrcps_synchronize then
  // reports NRCPS_ERR_TIMEOUT and the context stays usable).
  int fused_stall_test = 0;
  // FP32 copy of a kinetic table for nrcps_propagate(F32).
  float2* kin_f32 = nullptr;  // (hi, lo) split of the last table
  long kin_f32_len = 0;
  void* zpos = nullptr;       // Z2-times-position-factor weights of the last fused step that had none given
  long zpos_len = 0;          // bytes
};

}  // namespace nrcps

struct nrcps_context : public nrcps::Context {};

namespace nrcps {

nrcps_status set_error(nrcps_context* ctx, nrcps_status st, const char* fmt, ...);
nrcps_status check_cuda(nrcps_context* ctx, cudaError_t e, const char* what);
nrcps_status check_launch(nrcps_context* ctx, const char* what);
void* scratch(nrcps_context* ctx, size_t bytes, nrcps_status* st);

inline long vol_of(const int dims[3]) { return (long)dims[0] * dims[1] * dims[2]; }

// tensor-core overlap (overlap_tc.cu)
bool overlap_tc_supported(long vol, int ns, int nt, int nconf);
size_t overlap_tc_split_bytes(int ns, long vol);
nrcps_status overlap_tc_prepare(nrcps_context* ctx, const double* src, int ns, long vol, float* split);
nrcps_status overlap_tc(nrcps_context* ctx, const float* split, int ns, const void* psi, int nt, int nconf, long vol,
                        double* S);

// The pair kernels' view of a TwoBody table (host copies): bit 0 set unless
// opp is an involution of [0, vol) (TwoBody's parity mirror is), bit 1 set
// unless also w(opp(i)) = w(i) for every site (TwoBody's weights are)
inline int pair_table_props(const int* opp, const double* w, long vol) {
  int props = 0;
  for (long i = 0; i < vol; ++i) {
    if (opp[i] < 0 || opp[i] >= vol) return 3;
    if (opp[opp[i]] != i) props |= 1;
    if (w[opp[i]] != w[i]) props |= 2;
  }
  return props & 1 ? 3 : props;
}

inline unsigned grid_for(long n, int block, long cap = 148L * 64) {
  long g = (n + block - 1) / block;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

}  // namespace nrcps

#define NRCPS_TRY(expr)                       \
  do {                                        \
    nrcps_status _s = (expr);                 \
    if (_s != NRCPS_OK) return _s;            \
  } while (0)

#define NRCPS_REQUIRE(ctx, cond, ...)                                            \
  do {                                                                           \
    if (!(cond)) return nrcps::set_error((ctx), NRCPS_ERR_INVALID_ARGUMENT, __VA_ARGS__); \
  } while (0)

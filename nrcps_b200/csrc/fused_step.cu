// fused_step.cu -- one transfer-matrix step per orbital in a single HBM pass.
//
//   psi(p) <- k(p) . B[ w(x) . F[ k(p) . psi(p) ] ]
//
// (Propagator::Run over [K, (V), I, (V), K], src/alg/propagator.C:35-45.)
//
// One thread-block cluster of C CTAs owns one orbital at a time (a
// persistent loop over orbitals).  CTA c of the cluster holds the x-slab
// x in [c*S, (c+1)*S), S = L/C, in shared memory, organised as C regions:
// region r holds the (x in slab c, y in slab r) block as [xl][yl][z] with a
// padded z row (LP = L + 1) so that every pass is bank-conflict free.
//
//   1. z-pencils straight from HBM (one thread per (xl, y), 16-byte loads),
//      times k(p), forward DFT along z in registers, into shared memory;
//   2. forward DFT along y (thread per (xl, z));
//   3. cluster barrier; forward DFT along x, times w(x, y, z), backward DFT
//      along x for the pencils of y-slab c (thread per (yl, z)).  Element x
//      of such a pencil sits in region c of CTA x/S and is read and written
//      in place through distributed shared memory; w = P(x) (1 + a phi)/V
//      with phi from the packed Z2 field bits or an interleaved complex
//      phi / fld array; cluster barrier;
//   4. backward DFT along y;
//   5. backward DFT along z, times k(p), 16-byte stores to HBM.
//
// HBM traffic per orbital and step: one read and one write of the orbital
// (plus the L2-resident k table and field bits).
#include <cooperative_groups.h>

#include "common.cuh"
#include "fft.cuh"

namespace cg = cooperative_groups;

namespace nrcps {

struct FusedArgs {
  void* psi;              // [orbitals][V] complex R
  long n_orb_total;       // nconf * batch
  int batch;              // orbitals per configuration
  const float2* kin_f;    // k(p) split as (hi, lo) floats, hi + lo = k to ~1e-15 (R = float)
  const double* kin_d;    // k(p) in FP64 (R = double)
  const double* pos;      // optional P(x)
  int field_mode;         // 1 bits, 2 complex phi, 0 complex fld
  const void* field;
  uint64_t off0;          // element/bit offset of configuration 0
  uint64_t conf_stride;
  double a;
  double vol;
  double w_plus, w_minus;  // (1 + a)/V and (1 - a)/V for Z2 fields
};

// x * w for the position-space factor of site `site` (general modes).
template <typename R>
__device__ __forceinline__ cplx<R> apply_w_general(const FusedArgs& f, uint64_t kb, int site, cplx<R> x) {
  double wr, wi;
  const uint64_t k = kb + (uint64_t)site;
  if (f.field_mode == 1) {
    uint32_t word = __ldg(reinterpret_cast<const uint32_t*>(f.field) + (k >> 5));
    wr = ((word >> (k & 31)) & 1u) ? f.w_plus : f.w_minus;
    wi = 0.0;
  } else if (f.field_mode == 2) {
    double2 phi = __ldg(reinterpret_cast<const double2*>(f.field) + k);
    wr = (1.0 + f.a * phi.x) / f.vol;
    wi = (f.a * phi.y) / f.vol;
  } else {
    double2 v = __ldg(reinterpret_cast<const double2*>(f.field) + k);
    wr = v.x;
    wi = v.y;
  }
  if (f.pos) {
    double p = __ldg(f.pos + site);
    wr *= p;
    wi *= p;
  }
  R rh, rl, ih, il;
  split<R>(wr, rh, rl);
  split<R>(wi, ih, il);
  cplx<R> y = cmul(cplx<R>{rh, ih}, x);
  if constexpr (sizeof(R) == 4) {
    y.re = fmaf(x.re, rl, fmaf(-x.im, il, y.re));
    y.im = fmaf(x.im, rl, fmaf(x.re, il, y.im));
  }
  return y;
}

template <typename R>
__device__ __forceinline__ cplx<R> apply_kin(const FusedArgs& f, int site, cplx<R> x) {
  if constexpr (sizeof(R) == 4) {
    float2 k = __ldg(f.kin_f + site);
    return scale2<R>(x, k.x, k.y);
  } else {
    R k = __ldg(f.kin_d + site);
    return cplx<R>{x.re * k, x.im * k};
  }
}

template <typename R, int L, int C>
struct FusedShape {
  static constexpr int S = L / C;             // x (or y) planes per CTA
  static constexpr int LP = L + 1;            // padded z row
  // complex elements per region; the extra S elements shift consecutive
  // regions by half a bank row so the z-pass stores (lanes spanning two
  // regions) do not alias
  static constexpr int REGION = S * S * LP + S;
  static constexpr int THREADS = S * L;       // one pencil per thread per pass
  static constexpr size_t SMEM = sizeof(cplx<R>) * (size_t)C * REGION;
  // FP32: ask for <= 128 registers per thread so two 256-thread CTAs share an SM
  static constexpr int MIN_BLOCKS = (sizeof(R) == 4 && THREADS * 128 <= 32768) ? 32768 / (THREADS * 128) * 2 : 1;
  static_assert(L % C == 0, "cluster size must divide L");
};

template <typename R, int L, int C>
__global__ void __launch_bounds__(FusedShape<R, L, C>::THREADS, FusedShape<R, L, C>::MIN_BLOCKS)
    fused_step_kernel(FusedArgs f) {
  using Sh = FusedShape<R, L, C>;
  constexpr int S = Sh::S, LP = Sh::LP, REGION = Sh::REGION, NT = Sh::THREADS;
  constexpr int V = L * L * L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* sm = reinterpret_cast<cplx<R>*>(smem_raw);

  cg::cluster_group cluster = cg::this_cluster();
  const int c = (int)cluster.block_rank();
  const long cluster_id = blockIdx.x / C;
  const long n_clusters = gridDim.x / C;
  const int tid = threadIdx.x;

  // local offset of (region r, xl, yl, z); regions are REGION apart
  auto off = [](int r, int xl, int yl, int z) { return r * REGION + (xl * S + yl) * LP + z; };

  // Z2 fields without a static factor take the fast path: one 32-bit word
  // per pencil element, the bit position fixed per thread (L*L % 32 == 0).
  const bool z2_fast = (f.field_mode == 1) && (f.pos == nullptr) && ((L * L) % 32 == 0);
  R wp_hi, wp_lo, wm_hi, wm_lo;
  split<R>(f.w_plus, wp_hi, wp_lo);
  split<R>(f.w_minus, wm_hi, wm_lo);

  for (long orb = cluster_id; orb < f.n_orb_total; orb += n_clusters) {
    const long conf = orb / f.batch;
    const uint64_t kb = f.off0 + (uint64_t)conf * f.conf_stride;  // field offset of this configuration
    cplx<R>* gpsi = reinterpret_cast<cplx<R>*>(f.psi) + (size_t)orb * V;
    cplx<R> x[L];
    // ---- 1. z-pencils from HBM: thread -> (xl, y), y fastest
    {
      const int y = tid % L, xl = tid / L;
      const int base = ((c * S + xl) * L + y) * L;
      if constexpr (sizeof(R) == 4) {
        const float4* src = reinterpret_cast<const float4*>(gpsi + base);
#pragma unroll
        for (int j = 0; j < L / 2; ++j) {
          float4 v = __ldcs(src + j);
          x[2 * j] = cplx<R>{v.x, v.y};
          x[2 * j + 1] = cplx<R>{v.z, v.w};
        }
      } else {
        const double2* src = reinterpret_cast<const double2*>(gpsi + base);
#pragma unroll
        for (int j = 0; j < L; ++j) {
          double2 v = __ldcs(src + j);
          x[j] = cplx<R>{v.x, v.y};
        }
      }
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = apply_kin<R>(f, base + j, x[j]);
      fft::Dft<L, -1, R>::run(x);
      cplx<R>* row = sm + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int j = 0; j < L; ++j) row[j] = x[j];
    }
    __syncthreads();
    // ---- 2. forward DFT along y: thread -> (xl, z), z fastest
    {
      const int z = tid % L, xl = tid / L;
#pragma unroll
      for (int y = 0; y < L; ++y) x[y] = sm[off(y / S, xl, y % S, z)];
      fft::Dft<L, -1, R>::run(x);
#pragma unroll
      for (int y = 0; y < L; ++y) sm[off(y / S, xl, y % S, z)] = x[y];
    }
    // ---- 3. x: forward DFT, times w, backward DFT on the pencils of
    // y-slab c.  The pencil's element x lives in region c of CTA x/S; it is
    // read and written in place through distributed shared memory (CTA c
    // touches only region c of its peers, so the accesses are disjoint).
    if constexpr (C > 1) cluster.sync();
    else __syncthreads();
    {
      cplx<R>* base[C];
#pragma unroll
      for (int r = 0; r < C; ++r) base[r] = (C > 1 ? cluster.map_shared_rank(sm, r) : sm) + c * REGION;
      const int z = tid % L, yl = tid / L;
      const int site0 = (c * S + yl) * L + z;  // site of x = 0
#pragma unroll
      for (int xx = 0; xx < L; ++xx) x[xx] = base[xx / S][((xx % S) * S + yl) * LP + z];
      fft::Dft<L, -1, R>::run(x);
      if (z2_fast) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
#pragma unroll
        for (int xx = 0; xx < L; ++xx) {
          const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
          x[xx] = scale2<R>(x[xx], up ? wp_hi : wm_hi, up ? wp_lo : wm_lo);
        }
      } else {
#pragma unroll
        for (int xx = 0; xx < L; ++xx) x[xx] = apply_w_general<R>(f, kb, site0 + xx * L * L, x[xx]);
      }
      fft::Dft<L, +1, R>::run(x);
#pragma unroll
      for (int xx = 0; xx < L; ++xx) base[xx / S][((xx % S) * S + yl) * LP + z] = x[xx];
    }
    if constexpr (C > 1) cluster.sync();
    else __syncthreads();
    // ---- 4. backward DFT along y
    {
      const int z = tid % L, xl = tid / L;
#pragma unroll
      for (int y = 0; y < L; ++y) x[y] = sm[off(y / S, xl, y % S, z)];
      fft::Dft<L, +1, R>::run(x);
#pragma unroll
      for (int y = 0; y < L; ++y) sm[off(y / S, xl, y % S, z)] = x[y];
    }
    __syncthreads();
    // ---- 5. backward DFT along z, times k, store
    {
      const int y = tid % L, xl = tid / L;
      const int base = ((c * S + xl) * L + y) * L;
      const cplx<R>* row = sm + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = row[j];
      fft::Dft<L, +1, R>::run(x);
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = apply_kin<R>(f, base + j, x[j]);
      if constexpr (sizeof(R) == 4) {
        float4* dst = reinterpret_cast<float4*>(gpsi + base);
#pragma unroll
        for (int j = 0; j < L / 2; ++j)
          __stcs(dst + j, make_float4(x[2 * j].re, x[2 * j].im, x[2 * j + 1].re, x[2 * j + 1].im));
      } else {
        double2* dst = reinterpret_cast<double2*>(gpsi + base);
#pragma unroll
        for (int j = 0; j < L; ++j) __stcs(dst + j, make_double2(x[j].re, x[j].im));
      }
    }
    // Peers touch this CTA's shared memory only between the two cluster
    // barriers of step 3, which every CTA has passed; a CTA-local barrier
    // protects the next orbital's z-pass stores.
    __syncthreads();
  }
  // keep shared memory alive until every CTA of the cluster is done with it
  if constexpr (C > 1) cluster.sync();
}

template <typename R, int L, int C>
static nrcps_status launch_fused(nrcps_context* ctx, const FusedArgs& f, int ctas_per_sm_hint) {
  using Sh = FusedShape<R, L, C>;
  auto kern = fused_step_kernel<R, L, C>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::SMEM);
  if (e != cudaSuccess) return check_cuda(ctx, e, "fused_step: smem attribute");
  if (C > 8) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return check_cuda(ctx, e, "fused_step: cluster attribute");
  }
  // persistent grid: as many clusters as fit, capped by the work
  int max_clusters = 0;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(Sh::THREADS);
  cfg.dynamicSmemBytes = Sh::SMEM;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(C * ctx->sm_count);
  e = cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg);
  if (e != cudaSuccess || max_clusters <= 0) {
    cudaGetLastError();
    max_clusters = ctx->sm_count / C;
  }
  (void)ctas_per_sm_hint;
  long clusters = max_clusters;
  if (clusters > f.n_orb_total) clusters = f.n_orb_total;
  if (clusters < 1) clusters = 1;
  cfg.gridDim = dim3((unsigned)(clusters * C));
  e = cudaLaunchKernelEx(&cfg, kern, f);
  ctx->launches++;
  return check_cuda(ctx, e, "fused_step_kernel launch");
}

// ------------------------------------------------------------- dispatch
typedef nrcps_status (*FusedLauncher)(nrcps_context*, const FusedArgs&, int);

struct FusedVariant {
  int prec;  // nrcps_precision
  int L;
  int C;
  FusedLauncher fn;
};

// Instantiated (precision, L, cluster size) variants.  Shared memory per CTA
// is C regions of (L/C)^2 (L+1) + L/C complex values; all fit in 227 KB and
// one pencil per thread keeps L/C * L <= 1024 threads.
static const FusedVariant kVariants[] = {
    {NRCPS_F32, 8, 1, launch_fused<float, 8, 1>},     {NRCPS_F32, 16, 1, launch_fused<float, 16, 1>},
    {NRCPS_F32, 16, 2, launch_fused<float, 16, 2>},   {NRCPS_F32, 24, 2, launch_fused<float, 24, 2>},
    {NRCPS_F32, 24, 3, launch_fused<float, 24, 3>},   {NRCPS_F32, 32, 2, launch_fused<float, 32, 2>},
    {NRCPS_F32, 32, 4, launch_fused<float, 32, 4>},   {NRCPS_F32, 32, 8, launch_fused<float, 32, 8>},
    {NRCPS_F32, 48, 8, launch_fused<float, 48, 8>},   {NRCPS_F64, 8, 1, launch_fused<double, 8, 1>},
    {NRCPS_F64, 16, 1, launch_fused<double, 16, 1>},  {NRCPS_F64, 16, 2, launch_fused<double, 16, 2>},
    {NRCPS_F64, 24, 4, launch_fused<double, 24, 4>},  {NRCPS_F64, 32, 4, launch_fused<double, 32, 4>},
    {NRCPS_F64, 32, 8, launch_fused<double, 32, 8>},
};
static const int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// Autotuned choice per (device, precision, L): index into kVariants, -1 unset.
static int g_choice[16][2][64];
static bool g_choice_init = false;

static void init_choices() {
  if (g_choice_init) return;
  for (auto& a : g_choice)
    for (auto& b : a)
      for (int& c : b) c = -1;
  g_choice_init = true;
}

bool fused_supported(nrcps_precision prec, const int d[3]) {
  if (d[0] != d[1] || d[1] != d[2]) return false;
  for (int i = 0; i < kNumVariants; ++i)
    if (kVariants[i].prec == prec && kVariants[i].L == d[0]) return true;
  return false;
}

// Times every cluster size for (prec, L) on a scratch batch and records the
// fastest.  Runs outside graph capture (it allocates and synchronises).
nrcps_status fused_autotune(nrcps_context* ctx, nrcps_precision prec, int L, int* chosen_cluster) {
  init_choices();
  int dev = ctx->device & 15;
  if (L < 64 && g_choice[dev][prec][L] >= 0) {
    if (chosen_cluster) *chosen_cluster = kVariants[g_choice[dev][prec][L]].C;
    return NRCPS_OK;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cs);
  if (cs != cudaStreamCaptureStatusNone) return NRCPS_OK;  // keep the default
  const long V = (long)L * L * L;
  const size_t esz = prec == NRCPS_F64 ? 16 : 8;
  long norb = (long)(512L * 1024 * 1024 / (V * esz));  // ~512 MB: larger than L2
  if (norb > 4096) norb = 4096;
  if (norb < 8) norb = 8;
  void* psi = nullptr;
  void* kin = nullptr;
  uint32_t* bits = nullptr;
  cudaError_t e = cudaMalloc(&psi, esz * V * norb);
  if (e == cudaSuccess) e = cudaMalloc(&kin, esz * V);
  if (e == cudaSuccess) e = cudaMalloc((void**)&bits, (size_t)(V / 32 + 1) * 4);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (psi) cudaFree(psi);
    if (kin) cudaFree(kin);
    return NRCPS_OK;  // keep the default choice
  }
  cudaMemsetAsync(psi, 0, esz * V * norb, ctx->stream);
  cudaMemsetAsync(kin, 0, esz * V, ctx->stream);
  cudaMemsetAsync(bits, 0, (size_t)(V / 32 + 1) * 4, ctx->stream);
  FusedArgs f{};
  f.psi = psi;
  f.n_orb_total = norb;
  f.batch = (int)norb;
  f.kin_f = (const float2*)kin;
  f.kin_d = (const double*)kin;
  f.field_mode = 1;
  f.field = bits;
  f.a = 0.5;
  f.vol = (double)V;
  f.w_plus = 1.5 / V;
  f.w_minus = 0.5 / V;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  float best = 1e30f;
  int best_i = -1;
  long saved = ctx->launches;
  for (int i = 0; i < kNumVariants; ++i) {
    if (kVariants[i].prec != prec || kVariants[i].L != L) continue;
    if (kVariants[i].fn(ctx, f, 0) != NRCPS_OK) {
      cudaGetLastError();
      continue;
    }
    cudaEventRecord(t0, ctx->stream);
    for (int r = 0; r < 3; ++r) kVariants[i].fn(ctx, f, 0);
    cudaEventRecord(t1, ctx->stream);
    if (cudaEventSynchronize(t1) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    if (ms < best) {
      best = ms;
      best_i = i;
    }
  }
  ctx->launches = saved;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(psi);
  cudaFree(kin);
  cudaFree(bits);
  if (best_i >= 0 && L < 64) g_choice[dev][prec][L] = best_i;
  if (chosen_cluster && best_i >= 0) *chosen_cluster = kVariants[best_i].C;
  return NRCPS_OK;
}

// One fused step; `kin_table` is (hi, lo) float pairs for prec F32 and FP64 for F64.
// cluster = 0 selects the autotuned (or default) cluster size.
nrcps_status fused_step(nrcps_context* ctx, void* psi, int batch, int nconf, const int d[3], const void* kin_table,
                        nrcps_precision prec, const nrcps_position_factor* w, int cluster) {
  if (!fused_supported(prec, d)) return NRCPS_ERR_UNSUPPORTED;
  FusedArgs f;
  f.psi = psi;
  f.n_orb_total = (long)batch * nconf;
  f.batch = batch;
  f.kin_f = prec == NRCPS_F32 ? (const float2*)kin_table : nullptr;
  f.kin_d = prec == NRCPS_F64 ? (const double*)kin_table : nullptr;
  f.pos = w->dev_pos;
  f.field_mode = w->field_mode;
  f.field = w->dev_field;
  f.off0 = w->bit0;
  f.conf_stride = w->conf_stride;
  f.a = w->a;
  f.vol = (double)d[0] * d[1] * d[2];
  f.w_plus = (1.0 + f.a) / f.vol;
  f.w_minus = (1.0 - f.a) / f.vol;
  if (f.n_orb_total == 0) return NRCPS_OK;
  init_choices();
  const int L = d[0];
  int pick = -1;
  if (cluster > 0) {
    for (int i = 0; i < kNumVariants; ++i)
      if (kVariants[i].prec == prec && kVariants[i].L == L && kVariants[i].C == cluster) pick = i;
    if (pick < 0) return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "no fused variant with cluster size %d", cluster);
  } else {
    pick = g_choice[ctx->device & 15][prec][L];
    if (pick < 0)  // default: the largest instantiated cluster for this shape
      for (int i = 0; i < kNumVariants; ++i)
        if (kVariants[i].prec == prec && kVariants[i].L == L) pick = i;
  }
  return kVariants[pick].fn(ctx, f, 0);
}

}  // namespace nrcps

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
  const void* zpos;       // Z2 fields with P(x): per site the weights (1 + a) P(x)/V and (1 - a) P(x)/V,
                          // split (hi, lo, hi, lo) as float4 for R = float, (plus, minus) double2 for double
  int field_mode;         // 1 bits, 2 complex phi, 0 complex fld, 3 real FP32 weights (FP32 orbitals)
  const void* field;
  uint64_t off0;          // element/bit offset of configuration 0
  uint64_t conf_stride;
  const uint64_t* conf_base;  // optional per-configuration offsets (replace conf * conf_stride)
  double a;
  double vol;
  double inv_vol;          // 1 / vol (a product per site instead of a division)
  double w_plus, w_minus;  // (1 + a)/V and (1 - a)/V for Z2 fields
  int* err;                // device flag: 1 = a bounded wait timed out
  unsigned long long wait_ns;  // time limit of every mbarrier wait (%globaltimer nanoseconds)
  int stall_test;          // 1: the first wait of CTA 0 of cluster 0 is on an mbarrier nothing arrives on
};

// x * w for the position-space factor of site `site` (general modes).
template <typename R>
__device__ __forceinline__ cplx<R> apply_w_general(const FusedArgs& f, uint64_t kb, int site, cplx<R> x) {
  double wr, wi;
  const uint64_t k = kb + (uint64_t)site;
  if (sizeof(R) == 4 && f.field_mode == 3) {  // the site's weight, made once per run
    const float w = __ldg(reinterpret_cast<const float*>(f.field) + k);
    // rounded products (never fused into a following add): every kind gives
    // the same values
    return cplx<R>{(R)__fmul_rn((float)x.re, w), (R)__fmul_rn((float)x.im, w)};
  }
  if (f.field_mode == 1) {
    uint32_t word = __ldg(reinterpret_cast<const uint32_t*>(f.field) + (k >> 5));
    wr = ((word >> (k & 31)) & 1u) ? f.w_plus : f.w_minus;
    wi = 0.0;
  } else if (f.field_mode == 2) {
    double2 phi = __ldg(reinterpret_cast<const double2*>(f.field) + k);
    wr = (1.0 + f.a * phi.x) * f.inv_vol;
    wi = (f.a * phi.y) * f.inv_vol;
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
  if (wi == 0.0) return scale2<R>(x, rh, rl);  // real weight (Z2, Gaussian, potential): the same value, half the work
  split<R>(wi, ih, il);
  // (x.re + i x.im)(wr + i wi) with each real product taken correctly rounded
  cplx<R> y;
  y.re = mul2<R>(x.re, rh, rl) - mul2<R>(x.im, ih, il);
  y.im = mul2<R>(x.re, ih, il) + mul2<R>(x.im, rh, rl);
  return y;
}

template <typename R, bool PK = false>
__device__ __forceinline__ cplx<R> apply_kin(const FusedArgs& f, int site, cplx<R> x) {
  if constexpr (sizeof(R) == 4) {
    float2 k = __ldg(f.kin_f + site);
    if constexpr (PK) return fft::scale2_packed(x, k.x, k.y);
    else return scale2<R>(x, k.x, k.y);
  } else {
    R k = __ldg(f.kin_d + site);
    return cplx<R>{x.re * k, x.im * k};
  }
}

// x * (hi + lo), packed when PK (FP32 only)
template <typename R, bool PK>
__device__ __forceinline__ cplx<R> scale_w(cplx<R> x, R hi, R lo);

// x * w for a Z2 site with a position factor, from the table of both weights
// of every site: the value apply_w_general gives (the table holds the same
// products w_plus * P and w_minus * P, split the same way)
template <typename R, bool PK>
__device__ __forceinline__ cplx<R> scale_w_zpos(const void* tab, int site, bool up, cplx<R> x) {
  if constexpr (sizeof(R) == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(tab) + site);
    return scale_w<R, PK>(x, up ? t.x : t.z, up ? t.y : t.w);
  } else {
    const double2 t = __ldg(reinterpret_cast<const double2*>(tab) + site);
    return scale_w<R, PK>(x, up ? t.x : t.y, (R)0);
  }
}

// x * (hi + lo), packed when PK (FP32 only)
template <typename R, bool PK>
__device__ __forceinline__ cplx<R> scale_w(cplx<R> x, R hi, R lo) {
  if constexpr (PK && sizeof(R) == 4) return fft::scale2_packed(x, hi, lo);
  else return scale2<R>(x, hi, lo);
}

// x * w for a weight that one float holds exactly (lo = 0): the same value
// as scale_w(x, w, 0), in one product per component
template <typename R, bool PK>
__device__ __forceinline__ cplx<R> scale_w1(cplx<R> x, R w) {
  if constexpr (PK && sizeof(R) == 4) {
    const float2 r = __fmul2_rn(make_float2(x.re, x.im), make_float2(w, w));
    return cplx<R>{r.x, r.y};
  } else {
    return cplx<R>{x.re * w, x.im * w};
  }
}

template <typename R, int L, int C>
struct FusedShape {
  static constexpr int S = L / C;             // x (or y) planes per CTA
  static constexpr int LP = L + 1;            // padded z row
  // complex elements per region; the extra S elements shift consecutive
  // regions so that a warp's rows spread over all banks
  static constexpr int REGION = S * S * LP + S;
  static constexpr int WORK = C * REGION;     // padded working copy of the slab
  static constexpr int STAGE = S * L * L;     // unpadded slab, landing zone of the bulk copy
  static constexpr int THREADS = S * L;       // one pencil per thread per pass
  // + the slab's mbarrier, the time-out test's idle mbarrier and the cluster's abort word
  static constexpr size_t SMEM = sizeof(cplx<R>) * (size_t)(STAGE + WORK) + 32;
  static constexpr int CTAS_PER_SM = (int)(228 * 1024 / (SMEM + 1024)) > 4 ? 4 : (int)(228 * 1024 / (SMEM + 1024));
  static constexpr int MIN_BLOCKS = CTAS_PER_SM < 1 ? 1 : CTAS_PER_SM;
  static_assert(L % C == 0, "cluster size must divide L");
  static_assert((STAGE * sizeof(cplx<R>)) % 16 == 0, "bulk copy size must be a multiple of 16 bytes");
};

// ------------------------------------------------ bulk copy + mbarrier PTX
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// One poll of an mbarrier phase; ACQ_CLUSTER: acquire at cluster scope (the
// awaited bytes were written by other CTAs of the cluster).
template <bool ACQ_CLUSTER = false>
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  if constexpr (ACQ_CLUSTER)
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
  else
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for a phase: true once it completed; false when the cluster's
// abort word (this CTA's copy, written by whichever CTA gave up first) is
// raised, or when f.wait_ns of wall time passed -- then the timeout is
// recorded in *f.err.  A false return is acted on by the caller: the whole
// cluster leaves its orbital loop (see the abort paths of the kernels).
// abort_word = nullptr: the final wait of an abort path (only the time limit).
template <bool ACQ_CLUSTER = false>
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, const FusedArgs& f,
                                                  const volatile int* abort_word) {
  if (mbar_try_wait<ACQ_CLUSTER>(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait<ACQ_CLUSTER>(bar, parity)) return true;
    if (abort_word && *abort_word) return false;
    if (global_ns() - t0 > f.wait_ns) {
      if (f.err) atomicExch(f.err, 1);
      return false;
    }
  }
}

// Raises the abort word of every CTA of the cluster (C = 1: this CTA's).
template <int C>
__device__ __forceinline__ void raise_abort(cg::cluster_group& cluster, int* abort_word) {
#pragma unroll
  for (int r = 0; r < C; ++r) {
    volatile int* w = C > 1 ? cluster.map_shared_rank(abort_word, r) : abort_word;
    *w = 1;
  }
  __threadfence_block();
}

// The time-out test's stand-in for a stuck copy: the first wait of CTA 0 of
// cluster 0 is on `idle`, an initialised mbarrier nothing ever arrives on.
__device__ __forceinline__ bool stall_here(const FusedArgs& f, long cluster_id, int rank, bool first) {
  return f.stall_test && first && cluster_id == 0 && rank == 0;
}

// Prefetch of a global range into L2 by the bulk copy engine (no completion).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Launch shape of the peer-access kernel: STAGED keeps the HBM landing zone
// of the next slab in shared memory (bulk copy); unstaged, the next slab is
// prefetched into L2 and pass 1 reads it from there, which halves the shared
// memory and lets four CTAs share an SM (registers capped accordingly).
template <typename R, int L, int C, bool STAGED>
struct PullShape {
  using Base = FusedShape<R, L, C>;
  static constexpr int THREADS = Base::THREADS;
  static constexpr size_t SMEM = STAGED ? Base::SMEM : sizeof(cplx<R>) * (size_t)Base::WORK + 32;
  static constexpr int FIT = (int)(228 * 1024 / (SMEM + 1024));
  // a pencil alone takes 2 L registers: leave each thread 128 at L = 32
  // and 168 at L >= 48
  static constexpr int WARP_THREADS = (THREADS + 31) / 32 * 32;
  static constexpr int REG_FIT = L >= 48 ? 65536 / (WARP_THREADS * 168) : L >= 32 ? 65536 / (WARP_THREADS * 128) : 4;
  static constexpr int CAP = REG_FIT < 4 ? REG_FIT : 4;
  static constexpr int MIN_BLOCKS = STAGED ? Base::MIN_BLOCKS : (FIT > CAP ? CAP : (FIT < 1 ? 1 : FIT));
};

template <typename R, int L, int C, bool PK = false, bool STAGED = true>
__global__ void __launch_bounds__(PullShape<R, L, C, STAGED>::THREADS, PullShape<R, L, C, STAGED>::MIN_BLOCKS)
    fused_step_kernel(FusedArgs f) {
  using Sh = FusedShape<R, L, C>;
  constexpr int S = Sh::S, LP = Sh::LP, REGION = Sh::REGION;
  constexpr int V = L * L * L;
  constexpr uint32_t STAGE_BYTES = (uint32_t)(Sh::STAGE * sizeof(cplx<R>));
  extern __shared__ __align__(128) unsigned char smem_raw[];
  cplx<R>* stage = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* sm = stage + (STAGED ? Sh::STAGE : 0);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + Sh::WORK);
  uint64_t* idle = bar + 1;                              // the time-out test's mbarrier
  int* abort_word = reinterpret_cast<int*>(bar + 2);     // raised by the first CTA that gives up

  cg::cluster_group cluster = cg::this_cluster();
  const int c = (int)cluster.block_rank();
  const long cluster_id = blockIdx.x / C;
  const long n_clusters = gridDim.x / C;
  const int tid = threadIdx.x;

  // local offset of (region r, xl, yl, z); regions are REGION apart
  auto off = [](int r, int xl, int yl, int z) { return r * REGION + (xl * S + yl) * LP + z; };
  auto slab = [&](long orb) {  // this CTA's x-slab of orbital `orb` in HBM
    return reinterpret_cast<const cplx<R>*>(f.psi) + (size_t)orb * V + (size_t)c * S * L * L;
  };

  const bool z2_fast = (f.field_mode == 1) && (f.pos == nullptr) && ((L * L) % 32 == 0);
  const bool z2_pos = (f.field_mode == 1) && (f.zpos != nullptr) && ((L * L) % 32 == 0);
  R wp_hi, wp_lo, wm_hi, wm_lo;
  split<R>(f.w_plus, wp_hi, wp_lo);
  split<R>(f.w_minus, wm_hi, wm_lo);
  // (1 +- a)/V held exactly by one float (a = 0.5 with V a power of two):
  // one product per component instead of the hi + lo product
  const bool w_exact = wp_lo == (R)0 && wm_lo == (R)0;

  if (tid == 0) {
    *reinterpret_cast<volatile int*>(abort_word) = 0;
    if constexpr (STAGED) {
      mbar_init(bar);
      mbar_init(idle);
    }
  }
  // every CTA's abort word is set up before any peer can raise it
  if constexpr (C > 1) cluster.sync();
  else __syncthreads();
  uint32_t parity = 0;
  bool outstanding = false;  // a slab copy on `bar` (phase `parity`) that nobody has waited for
  bool aborted = false;
  long orb = cluster_id;
  if (orb < f.n_orb_total) {
    if constexpr (STAGED) {
      if (tid == 0) bulk_load(stage, slab(orb), STAGE_BYTES, bar);
      outstanding = true;
    } else if (tid == 0) {
      prefetch_l2(slab(orb), STAGE_BYTES);
    }
  }

  for (; orb < f.n_orb_total; orb += n_clusters) {
    const long conf = orb / f.batch;
    const uint64_t kb = f.off0 + (f.conf_base ? __ldg(f.conf_base + conf) : (uint64_t)conf * f.conf_stride);  // field offset of this configuration
    cplx<R>* gpsi = reinterpret_cast<cplx<R>*>(f.psi) + (size_t)orb * V;
    cplx<R> x[L];
    bool ok = true;
    if constexpr (STAGED) {
      ok = stall_here(f, cluster_id, c, orb == cluster_id) ? mbar_wait_bounded(idle, 0u, f, abort_word)
                                                           : mbar_wait_bounded(bar, parity, f, abort_word);
    } else if (tid == 0 && orb + n_clusters < f.n_orb_total) {
      prefetch_l2(slab(orb + n_clusters), STAGE_BYTES);
    }
    // ---- 1. k(p), forward DFT along y from the slab: thread -> (xl, z)
    {
      const int z = tid % L, xl = tid / L;
      const int site0 = (c * S + xl) * L * L + z;
      if constexpr (STAGED) {
#pragma unroll
        for (int y = 0; y < L; ++y) x[y] = apply_kin<R, PK>(f, site0 + y * L, stage[(xl * L + y) * L + z]);
      } else {
        const cplx<R>* src = slab(orb);
#pragma unroll
        for (int y = 0; y < L; ++y) {
          cplx<R> v;
          if constexpr (sizeof(R) == 4) {
            float2 t = __ldcg(reinterpret_cast<const float2*>(src) + (xl * L + y) * L + z);
            v = cplx<R>{t.x, t.y};
          } else {
            double2 t = __ldcg(reinterpret_cast<const double2*>(src) + (xl * L + y) * L + z);
            v = cplx<R>{t.x, t.y};
          }
          x[y] = apply_kin<R, PK>(f, site0 + y * L, v);
        }
      }
      fft::dft<L, -1, R, PK>(x);
#pragma unroll
      for (int y = 0; y < L; ++y) sm[off(y / S, xl, y % S, z)] = x[y];
    }
    if constexpr (STAGED) {
      if (__syncthreads_or(!ok)) {
        // the slab copy timed out (or a peer gave up): no further copy on
        // `bar`; the whole cluster leaves after the next cluster barrier
        if (tid == 0) raise_abort<C>(cluster, abort_word);
      } else {
        parity ^= 1u;
        outstanding = orb + n_clusters < f.n_orb_total;
        // the staging buffer is free: prefetch this cluster's next orbital
        if (tid == 0 && outstanding) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          bulk_load(stage, slab(orb + n_clusters), STAGE_BYTES, bar);
        }
      }
    } else {
      __syncthreads();
    }
    // ---- 2. forward DFT along z in place: thread -> (xl, y)
    {
      const int y = tid % L, xl = tid / L;
      cplx<R>* row = sm + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = row[j];
      fft::dft<L, -1, R, PK>(x);
#pragma unroll
      for (int j = 0; j < L; ++j) row[j] = x[j];
    }
    // ---- 3. x: forward DFT, times w, backward DFT on the pencils of
    // y-slab c.  Element x of such a pencil lives in region c of CTA x/S and
    // is read and written in place through distributed shared memory (CTA c
    // touches only region c of its peers, so the accesses are disjoint).
    if constexpr (C > 1) cluster.sync();
    else __syncthreads();
    if constexpr (STAGED) {
      // an abort word is raised only before this barrier (after the slab
      // wait) and read only between it and the next one: every CTA of the
      // cluster takes the same decision
      if (*reinterpret_cast<volatile int*>(abort_word)) {
        aborted = true;
        break;
      }
    }
    {
      cplx<R>* base[C];
#pragma unroll
      for (int r = 0; r < C; ++r) base[r] = (C > 1 ? cluster.map_shared_rank(sm, r) : sm) + c * REGION;
      const int z = tid % L, yl = tid / L;
      const int site0 = (c * S + yl) * L + z;  // site of x = 0
#pragma unroll
      for (int xx = 0; xx < L; ++xx) x[xx] = base[xx / S][((xx % S) * S + yl) * LP + z];
      fft::dft<L, -1, R, PK>(x);
      if (z2_fast) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
        if (w_exact) {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
            x[xx] = scale_w1<R, PK>(x[xx], up ? wp_hi : wm_hi);
          }
        } else {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
            x[xx] = scale_w<R, PK>(x[xx], up ? wp_hi : wm_hi, up ? wp_lo : wm_lo);
          }
        }
      } else if (z2_pos) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
#pragma unroll
        for (int xx = 0; xx < L; ++xx) {
          const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
          x[xx] = scale_w_zpos<R, PK>(f.zpos, site0 + xx * L * L, up, x[xx]);
        }
      } else {
#pragma unroll
        for (int xx = 0; xx < L; ++xx) x[xx] = apply_w_general<R>(f, kb, site0 + xx * L * L, x[xx]);
      }
      fft::dft<L, +1, R, PK>(x);
#pragma unroll
      for (int xx = 0; xx < L; ++xx) base[xx / S][((xx % S) * S + yl) * LP + z] = x[xx];
    }
    if constexpr (C > 1) cluster.sync();
    else __syncthreads();
    // ---- 4. backward DFT along z in place
    {
      const int y = tid % L, xl = tid / L;
      cplx<R>* row = sm + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = row[j];
      fft::dft<L, +1, R, PK>(x);
#pragma unroll
      for (int j = 0; j < L; ++j) row[j] = x[j];
    }
    __syncthreads();
    // ---- 5. backward DFT along y, times k(p), coalesced streaming stores
    {
      const int z = tid % L, xl = tid / L;
      const int site0 = (c * S + xl) * L * L + z;
#pragma unroll
      for (int y = 0; y < L; ++y) x[y] = sm[off(y / S, xl, y % S, z)];
      fft::dft<L, +1, R, PK>(x);
#pragma unroll
      for (int y = 0; y < L; ++y) {
        cplx<R> v = apply_kin<R, PK>(f, site0 + y * L, x[y]);
        if constexpr (sizeof(R) == 4)
          __stcs(reinterpret_cast<float2*>(gpsi) + site0 + y * L, make_float2(v.re, v.im));
        else
          __stcs(reinterpret_cast<double2*>(gpsi) + site0 + y * L, make_double2(v.re, v.im));
      }
    }
    // Thread (xl, z) of step 1 of the next orbital writes exactly the
    // working-copy elements it read in step 5, and peers touch this CTA's
    // shared memory only between the barriers of step 3: no barrier needed.
  }
  if constexpr (STAGED) {
    // leaving early: the slab copy this CTA started last lands before its
    // shared memory goes away (bounded like every other wait)
    if (aborted && outstanding && tid == 0) mbar_wait_bounded(bar, parity, f, nullptr);
  }
  // keep shared memory alive until every CTA of the cluster is done with it
  if constexpr (C > 1) cluster.sync();
}

// ------------------------------------------------ lane-split variant
// Same algorithm and shared-memory layout as fused_step_kernel, but every
// pencil is held by two lanes (lane and lane ^ 16), each with L/2 values:
// half the registers per thread and twice the resident warps.  Forward
// transforms run decimation-in-time (input split by parity, output by
// halves), inverse ones decimation-in-frequency (the reverse), so each pass
// reads and writes shared memory in the split its transform wants.
template <typename R, int L, int C>
struct SplitShape {
  using Base = FusedShape<R, L, C>;
  static constexpr int THREADS = 2 * Base::S * L;
  static constexpr int H = L / 2;
  static constexpr int MIN_BLOCKS = Base::CTAS_PER_SM < 1 ? 1 : Base::CTAS_PER_SM;
  static_assert(L % 2 == 0 && (Base::S * L) % 16 == 0, "lane-split pencils need L even and S*L % 16 == 0");
};

template <typename R, int L, int C>
__global__ void __launch_bounds__(SplitShape<R, L, C>::THREADS, SplitShape<R, L, C>::MIN_BLOCKS)
    fused_step_split_kernel(FusedArgs f) {
  using Sh = FusedShape<R, L, C>;
  constexpr int S = Sh::S, LP = Sh::LP, REGION = Sh::REGION;
  constexpr int H = L / 2;
  constexpr int V = L * L * L;
  constexpr uint32_t STAGE_BYTES = (uint32_t)(Sh::STAGE * sizeof(cplx<R>));
  extern __shared__ __align__(128) unsigned char smem_raw[];
  cplx<R>* stage = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* sm = stage + Sh::STAGE;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + Sh::WORK);
  uint64_t* idle = bar + 1;                           // the time-out test's mbarrier
  int* abort_word = reinterpret_cast<int*>(bar + 2);  // raised by the first CTA that gives up

  cg::cluster_group cluster = cg::this_cluster();
  const int c = (int)cluster.block_rank();
  const long cluster_id = blockIdx.x / C;
  const long n_clusters = gridDim.x / C;
  const int tid = threadIdx.x;
  const int h = (tid >> 4) & 1;                   // which half of the pencil
  const int p = (tid >> 5) * 16 + (tid & 15);     // pencil index within the pass

  auto off = [](int r, int xl, int yl, int z) { return r * REGION + (xl * S + yl) * LP + z; };
  auto slab = [&](long orb) {
    return reinterpret_cast<const cplx<R>*>(f.psi) + (size_t)orb * V + (size_t)c * S * L * L;
  };

  const bool z2_fast = (f.field_mode == 1) && (f.pos == nullptr) && ((L * L) % 32 == 0);
  const bool z2_pos = (f.field_mode == 1) && (f.zpos != nullptr) && ((L * L) % 32 == 0);
  R wp_hi, wp_lo, wm_hi, wm_lo;
  split<R>(f.w_plus, wp_hi, wp_lo);
  split<R>(f.w_minus, wm_hi, wm_lo);
  // (1 +- a)/V held exactly by one float (a = 0.5 with V a power of two):
  // one product per component instead of the hi + lo product
  const bool w_exact = wp_lo == (R)0 && wm_lo == (R)0;

  if (tid == 0) {
    *reinterpret_cast<volatile int*>(abort_word) = 0;
    mbar_init(bar);
    mbar_init(idle);
  }
  // every CTA's abort word is set up before any peer can raise it
  if constexpr (C > 1) cluster.sync();
  else __syncthreads();
  uint32_t parity = 0;
  bool outstanding = false;  // a slab copy on `bar` (phase `parity`) that nobody has waited for
  bool aborted = false;
  long orb = cluster_id;
  if (orb < f.n_orb_total) {
    if (tid == 0) bulk_load(stage, slab(orb), STAGE_BYTES, bar);
    outstanding = true;
  }

  for (; orb < f.n_orb_total; orb += n_clusters) {
    const long conf = orb / f.batch;
    const uint64_t kb = f.off0 + (f.conf_base ? __ldg(f.conf_base + conf) : (uint64_t)conf * f.conf_stride);
    cplx<R>* gpsi = reinterpret_cast<cplx<R>*>(f.psi) + (size_t)orb * V;
    cplx<R> v[H];
    const bool ok = stall_here(f, cluster_id, c, orb == cluster_id) ? mbar_wait_bounded(idle, 0u, f, abort_word)
                                                                    : mbar_wait_bounded(bar, parity, f, abort_word);
    // ---- 1. k(p), forward DFT along y from the staged slab: pencil (xl, z)
    {
      const int z = p % L, xl = p / L;
      const int site0 = (c * S + xl) * L * L + z;
#pragma unroll
      for (int m = 0; m < H; ++m) {
        const int y = 2 * m + h;
        v[m] = apply_kin<R>(f, site0 + y * L, stage[(xl * L + y) * L + z]);
      }
      fft::dft_split_dit<L, -1, R>(v, h);
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const int y = h * H + k;
        sm[off(y / S, xl, y % S, z)] = v[k];
      }
    }
    if (__syncthreads_or(!ok)) {
      // the slab copy timed out (or a peer gave up): no further copy on
      // `bar`; the whole cluster leaves after the next cluster barrier
      if (tid == 0) raise_abort<C>(cluster, abort_word);
    } else {
      parity ^= 1u;
      outstanding = orb + n_clusters < f.n_orb_total;
      if (tid == 0 && outstanding) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        bulk_load(stage, slab(orb + n_clusters), STAGE_BYTES, bar);
      }
    }
    // ---- 2. forward DFT along z in place: pencil (xl, y)
    {
      const int y = p % L, xl = p / L;
      cplx<R>* row = sm + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int m = 0; m < H; ++m) v[m] = row[2 * m + h];
      __syncwarp();
      fft::dft_split_dit<L, -1, R>(v, h);
#pragma unroll
      for (int k = 0; k < H; ++k) row[h * H + k] = v[k];
    }
    if constexpr (C > 1) cluster.sync();
    else __syncthreads();
    // raised only before this barrier, read only before the next: one decision per cluster
    if (*reinterpret_cast<volatile int*>(abort_word)) {
      aborted = true;
      break;
    }
    // ---- 3. x: forward DFT, times w, backward DFT through DSMEM: pencil (yl, z)
    {
      cplx<R>* base[C];
#pragma unroll
      for (int r = 0; r < C; ++r) base[r] = (C > 1 ? cluster.map_shared_rank(sm, r) : sm) + c * REGION;
      const int z = p % L, yl = p / L;
      const int site0 = (c * S + yl) * L + z;
#pragma unroll
      for (int m = 0; m < H; ++m) {
        const int xx = 2 * m + h;
        v[m] = base[xx / S][((xx % S) * S + yl) * LP + z];
      }
      fft::dft_split_dit<L, -1, R>(v, h);
      if (z2_fast) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
        if (w_exact) {
#pragma unroll
          for (int k = 0; k < H; ++k) {
            const int xx = h * H + k;
            const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
            v[k] = scale_w1<R, false>(v[k], up ? wp_hi : wm_hi);
          }
        } else {
#pragma unroll
          for (int k = 0; k < H; ++k) {
            const int xx = h * H + k;
            const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
            v[k] = scale2<R>(v[k], up ? wp_hi : wm_hi, up ? wp_lo : wm_lo);
          }
        }
      } else if (z2_pos) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
#pragma unroll
        for (int k = 0; k < H; ++k) {
          const int xx = h * H + k;
          const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
          v[k] = scale_w_zpos<R, false>(f.zpos, site0 + xx * L * L, up, v[k]);
        }
      } else {
#pragma unroll
        for (int k = 0; k < H; ++k) v[k] = apply_w_general<R>(f, kb, site0 + (h * H + k) * L * L, v[k]);
      }
      fft::dft_split_dif<L, +1, R>(v, h);
#pragma unroll
      for (int m = 0; m < H; ++m) {
        const int xx = 2 * m + h;
        base[xx / S][((xx % S) * S + yl) * LP + z] = v[m];
      }
    }
    if constexpr (C > 1) cluster.sync();
    else __syncthreads();
    // ---- 4. backward DFT along z in place
    {
      const int y = p % L, xl = p / L;
      cplx<R>* row = sm + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int k = 0; k < H; ++k) v[k] = row[h * H + k];
      __syncwarp();
      fft::dft_split_dif<L, +1, R>(v, h);
#pragma unroll
      for (int m = 0; m < H; ++m) row[2 * m + h] = v[m];
    }
    __syncthreads();
    // ---- 5. backward DFT along y, times k(p), streaming stores
    {
      const int z = p % L, xl = p / L;
      const int site0 = (c * S + xl) * L * L + z;
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const int y = h * H + k;
        v[k] = sm[off(y / S, xl, y % S, z)];
      }
      fft::dft_split_dif<L, +1, R>(v, h);
#pragma unroll
      for (int m = 0; m < H; ++m) {
        const int y = 2 * m + h;
        cplx<R> w = apply_kin<R>(f, site0 + y * L, v[m]);
        if constexpr (sizeof(R) == 4)
          __stcs(reinterpret_cast<float2*>(gpsi) + site0 + y * L, make_float2(w.re, w.im));
        else
          __stcs(reinterpret_cast<double2*>(gpsi) + site0 + y * L, make_double2(w.re, w.im));
      }
    }
    // the next orbital's step 1 writes, per pencil, the elements this pencil
    // read in step 5 -- but split differently between the two lanes, so the
    // pair must be done reading first
    __syncwarp();
  }
  // leaving early: the slab copy this CTA started last lands first (bounded)
  if (aborted && outstanding && tid == 0) mbar_wait_bounded(bar, parity, f, nullptr);
  if constexpr (C > 1) cluster.sync();
}

// ------------------------------------------------ cluster helpers
__device__ __forceinline__ uint32_t mapa_u32(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}

__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// ------------------------------------------------ bulk-copy exchange variant
// Same passes, but both exchanges move whole padded regions with the bulk
// copy engine (cp.async.bulk shared::cta -> shared::cluster), completing on
// the receiver's mbarrier: no per-element remote access and no cluster
// barrier in the loop.
//
// Shared memory per CTA: stage (HBM landing zone of the next slab), work
// (x-slab c, region r = y-slab r) and recv (y-slab c, slot s = x-slab s).
//   1. wait for the slab; k(p), DFT along y: stage -> work; prefetch the
//      next slab into stage;
//   2. DFT along z of the rows of work, in place; region r is copied to
//      slot c of the recv of CTA r;
//   3. wait for recv (C regions); DFT along x, times w, inverse DFT, in
//      place; slot s is copied back to region c of the work of CTA s;
//   4. wait for work; inverse DFT along z in place;
//   5. inverse DFT along y, times k(p), streaming stores to HBM.
// Buffer reuse needs no extra signal: slot s of recv is written only by
// CTA s and copied back only to CTA s, so when s has received its results
// (its work mbarrier) it knows that slot s of this CTA has been read out;
// the same holds for region r of work with CTA r.  Every mbarrier wait is
// bounded.
template <typename R, int L, int C, bool STAGED = true, bool KSM = false>
struct BulkShape {
  using Base = FusedShape<R, L, C>;
  static constexpr int THREADS = Base::THREADS;
  static constexpr uint32_t REGION_BYTES = (uint32_t)(Base::REGION * sizeof(cplx<R>));
  static constexpr uint32_t XBYTES = (uint32_t)(C * REGION_BYTES);       // one exchange, received
  static constexpr uint32_t STAGE_BYTES = (uint32_t)(Base::STAGE * sizeof(cplx<R>));
  static constexpr uint32_t KIN_BYTES = KSM ? (uint32_t)(Base::STAGE * sizeof(float2)) : 0u;  // slab of k(p)
  static constexpr size_t SMEM = 128 + (STAGED ? STAGE_BYTES : 0) + 2 * (size_t)XBYTES + KIN_BYTES;
  static constexpr int CTAS = (int)(228 * 1024 / (SMEM + 1024));
  static constexpr int WANT = (384 / THREADS) < 1 ? 1 : 384 / THREADS;
  static constexpr int MIN_BLOCKS = CTAS < 1 ? 1 : (CTAS > WANT ? WANT : CTAS);
  static_assert(REGION_BYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
  static_assert(XBYTES < (1u << 20), "mbarrier transaction count range");
};

// One bulk copy from this CTA's shared memory to a cluster peer's (dst and
// bar are shared::cluster addresses), completing on the peer's mbarrier.
__device__ __forceinline__ void bulk_to_peer(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst),
               "r"(smem_u32(src)), "r"(bytes), "r"(bar)
               : "memory");
}

// STAGED = false: no stage buffer; the next slab is prefetched into L2 and
// pass 1 reads it from there (two buffers instead of three per CTA).
// KSM (FP32): the CTA's slab of the kinetic table (hi, lo) stays in shared
// memory for the whole launch -- the slab index c of a CTA never changes, so
// passes 1 and 5 read k(p) there instead of from L2.
template <typename R, int L, int C, bool STAGED, bool PK = false, bool KSM = false>
__global__ void __launch_bounds__(BulkShape<R, L, C, STAGED, KSM>::THREADS,
                                  BulkShape<R, L, C, STAGED, KSM>::MIN_BLOCKS)
    fused_step_bulk_kernel(FusedArgs f) {
  using Sh = FusedShape<R, L, C>;
  using Bs = BulkShape<R, L, C, STAGED, KSM>;
  static_assert(!KSM || sizeof(R) == 4, "the resident kinetic slab is the FP32 (hi, lo) table");
  static_assert(C > 1, "the exchange is between CTAs of a cluster");
  constexpr int S = Sh::S, LP = Sh::LP, REGION = Sh::REGION;
  constexpr int V = L * L * L;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar_hbm = reinterpret_cast<uint64_t*>(smem_raw);
  uint64_t* bar_recv = bar_hbm + 1;
  uint64_t* bar_work = bar_hbm + 2;
  uint64_t* idle = bar_hbm + 3;                           // the time-out test's mbarrier
  int* abort_word = reinterpret_cast<int*>(bar_hbm + 4);  // raised by the first CTA that gives up
  cplx<R>* stage = reinterpret_cast<cplx<R>*>(smem_raw + 128);
  cplx<R>* work = stage + (STAGED ? Sh::STAGE : 0);
  cplx<R>* recv = work + Sh::WORK;
  float2* kin_s = reinterpret_cast<float2*>(recv + Sh::WORK);  // KSM: k(p) of sites c S L^2 + i
  // k(p) x for global site `site` = c S L^2 + `local`
  auto kin = [&](int site, int local, cplx<R> v) -> cplx<R> {
    if constexpr (KSM) {
      const float2 k = kin_s[local];
      return scale_w<R, PK>(v, k.x, k.y);
    } else {
      return apply_kin<R, PK>(f, site, v);
    }
  };

  cg::cluster_group cluster = cg::this_cluster();
  const int c = (int)cluster.block_rank();
  const long cluster_id = blockIdx.x / C;
  const long n_clusters = gridDim.x / C;
  const int tid = threadIdx.x;

  auto off = [](int r, int xl, int yl, int z) { return r * REGION + (xl * S + yl) * LP + z; };
  auto slab = [&](long orb) {
    return reinterpret_cast<const cplx<R>*>(f.psi) + (size_t)orb * V + (size_t)c * S * L * L;
  };

  const bool z2_fast = (f.field_mode == 1) && (f.pos == nullptr) && ((L * L) % 32 == 0);
  const bool z2_pos = (f.field_mode == 1) && (f.zpos != nullptr) && ((L * L) % 32 == 0);
  R wp_hi, wp_lo, wm_hi, wm_lo;
  split<R>(f.w_plus, wp_hi, wp_lo);
  split<R>(f.w_minus, wm_hi, wm_lo);
  // (1 +- a)/V held exactly by one float (a = 0.5 with V a power of two):
  // one product per component instead of the hi + lo product
  const bool w_exact = wp_lo == (R)0 && wm_lo == (R)0;

  if (tid == 0) {
    *reinterpret_cast<volatile int*>(abort_word) = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar_hbm)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar_recv)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar_work)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(idle)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if constexpr (KSM)
    for (int i = tid; i < Sh::STAGE; i += Bs::THREADS) kin_s[i] = __ldg(f.kin_f + (size_t)c * Sh::STAGE + i);
  cluster.sync();  // every CTA's mbarriers and abort word are set up before any copy or abort targets them
  uint32_t parity = 0;
  // phases this CTA expects bytes on and has not yet seen complete (all
  // three barriers advance one phase per orbital, so `parity` is theirs)
  bool hbm_out = false, recv_out = false, work_out = false;
  uint32_t hbm_phase = 0;  // phase of the outstanding HBM slab copy
  bool aborted = false;
  const volatile int* abort_flag = abort_word;
  long orb = cluster_id;
  if (orb < f.n_orb_total) {
    if constexpr (STAGED) {
      if (tid == 0) bulk_load(stage, slab(orb), Bs::STAGE_BYTES, bar_hbm);
      hbm_out = true;
    } else if (tid == 0) {
      prefetch_l2(slab(orb), Bs::STAGE_BYTES);
    }
  }
  // A CTA that gives up (a wait timed out, or it found the abort word
  // raised) raises every peer's abort word and leaves the loop at its next
  // block barrier, before it issues another copy; its peers' waits see the
  // word and they follow.  Every wait is bounded, so every CTA reaches the
  // exit.

  for (; orb < f.n_orb_total; orb += n_clusters) {
    const long conf = orb / f.batch;
    const uint64_t kb = f.off0 + (f.conf_base ? __ldg(f.conf_base + conf) : (uint64_t)conf * f.conf_stride);
    cplx<R>* gpsi = reinterpret_cast<cplx<R>*>(f.psi) + (size_t)orb * V;
    cplx<R> x[L];
    const bool first = orb == cluster_id;
    bool ok = true;
    if constexpr (STAGED) {
      ok = stall_here(f, cluster_id, c, first) ? mbar_wait_bounded(idle, 0u, f, abort_word)
                                               : mbar_wait_bounded(bar_hbm, parity, f, abort_word);
    } else if (tid == 0 && orb + n_clusters < f.n_orb_total) {
      prefetch_l2(slab(orb + n_clusters), Bs::STAGE_BYTES);
    }
    // ---- 1. k(p), forward DFT along y from the slab: thread -> (xl, z)
    {
      const int z = tid % L, xl = tid / L;
      const int site0 = (c * S + xl) * L * L + z;
      if constexpr (STAGED) {
#pragma unroll
        for (int y = 0; y < L; ++y) x[y] = kin(site0 + y * L, (xl * L + y) * L + z, stage[(xl * L + y) * L + z]);
      } else {
        const cplx<R>* src = slab(orb);
#pragma unroll
        for (int y = 0; y < L; ++y) {
          cplx<R> v;
          if constexpr (sizeof(R) == 4) {
            float2 t = __ldcg(reinterpret_cast<const float2*>(src) + (xl * L + y) * L + z);
            v = cplx<R>{t.x, t.y};
          } else {
            double2 t = __ldcg(reinterpret_cast<const double2*>(src) + (xl * L + y) * L + z);
            v = cplx<R>{t.x, t.y};
          }
          x[y] = kin(site0 + y * L, (xl * L + y) * L + z, v);
        }
      }
      fft::dft<L, -1, R, PK>(x);
#pragma unroll
      for (int y = 0; y < L; ++y) work[off(y / S, xl, y % S, z)] = x[y];
    }
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    if constexpr (STAGED) {
      hbm_out = orb + n_clusters < f.n_orb_total;  // the next slab, on the barrier's next phase
      hbm_phase = parity ^ 1u;
      if (tid == 0 && hbm_out) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        bulk_load(stage, slab(orb + n_clusters), Bs::STAGE_BYTES, bar_hbm);
      }
    }
    // ---- 2. forward DFT along z in place: thread -> (xl, y); then region r -> CTA r
    {
      const int y = tid % L, xl = tid / L;
      cplx<R>* row = work + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = row[j];
      fft::dft<L, -1, R, PK>(x);
#pragma unroll
      for (int j = 0; j < L; ++j) row[j] = x[j];
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> bulk copy reads
    if (__syncthreads_or(*abort_flag != 0)) {  // a peer gave up: send nothing more
      aborted = true;
      break;
    }
    if (tid < C) {
      const uint32_t dst = mapa_u32(smem_u32(recv + c * REGION), (uint32_t)tid);
      const uint32_t bar = mapa_u32(smem_u32(bar_recv), (uint32_t)tid);
      bulk_to_peer(dst, work + tid * REGION, Bs::REGION_BYTES, bar);
    }
    if (tid == 0) expect_tx(bar_recv, Bs::XBYTES);
    recv_out = true;
    ok = (!STAGED && stall_here(f, cluster_id, c, first)) ? mbar_wait_bounded(idle, 0u, f, abort_word)
                                                          : mbar_wait_bounded<true>(bar_recv, parity, f, abort_word);
    // ---- 3. x: forward DFT, times w, backward DFT on the pencils of y-slab c, in recv
    {
      const int z = tid % L, yl = tid / L;
      const int site0 = (c * S + yl) * L + z;
#pragma unroll
      for (int xx = 0; xx < L; ++xx) x[xx] = recv[off(xx / S, xx % S, yl, z)];
      fft::dft<L, -1, R, PK>(x);
      if (z2_fast) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
        if (w_exact) {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
            x[xx] = scale_w1<R, PK>(x[xx], up ? wp_hi : wm_hi);
          }
        } else {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
            x[xx] = scale_w<R, PK>(x[xx], up ? wp_hi : wm_hi, up ? wp_lo : wm_lo);
          }
        }
      } else if (z2_pos) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
#pragma unroll
        for (int xx = 0; xx < L; ++xx) {
          const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
          x[xx] = scale_w_zpos<R, PK>(f.zpos, site0 + xx * L * L, up, x[xx]);
        }
      } else {
#pragma unroll
        for (int xx = 0; xx < L; ++xx) x[xx] = apply_w_general<R>(f, kb, site0 + xx * L * L, x[xx]);
      }
      fft::dft<L, +1, R, PK>(x);
#pragma unroll
      for (int xx = 0; xx < L; ++xx) recv[off(xx / S, xx % S, yl, z)] = x[xx];
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (__syncthreads_or(!ok || *abort_flag != 0)) {
      aborted = true;
      break;
    }
    recv_out = false;
    if (tid < C) {
      const uint32_t dst = mapa_u32(smem_u32(work + c * REGION), (uint32_t)tid);
      const uint32_t bar = mapa_u32(smem_u32(bar_work), (uint32_t)tid);
      bulk_to_peer(dst, recv + tid * REGION, Bs::REGION_BYTES, bar);
    }
    if (tid == 0) expect_tx(bar_work, Bs::XBYTES);
    work_out = true;
    ok = mbar_wait_bounded<true>(bar_work, parity, f, abort_word);
    // ---- 4. backward DFT along z in place
    {
      const int y = tid % L, xl = tid / L;
      cplx<R>* row = work + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = row[j];
      fft::dft<L, +1, R, PK>(x);
#pragma unroll
      for (int j = 0; j < L; ++j) row[j] = x[j];
    }
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    work_out = false;
    parity ^= 1u;
    // ---- 5. backward DFT along y, times k(p), streaming stores
    {
      const int z = tid % L, xl = tid / L;
      const int site0 = (c * S + xl) * L * L + z;
#pragma unroll
      for (int y = 0; y < L; ++y) x[y] = work[off(y / S, xl, y % S, z)];
      fft::dft<L, +1, R, PK>(x);
#pragma unroll
      for (int y = 0; y < L; ++y) {
        cplx<R> v = kin(site0 + y * L, (xl * L + y) * L + z, x[y]);
        if constexpr (sizeof(R) == 4)
          __stcs(reinterpret_cast<float2*>(gpsi) + site0 + y * L, make_float2(v.re, v.im));
        else
          __stcs(reinterpret_cast<double2*>(gpsi) + site0 + y * L, make_double2(v.re, v.im));
      }
    }
    // Pass 1 of the next orbital writes, per thread, the work elements this
    // thread read in pass 5; no copy reads work between pass 4 and the next
    // pass 2 (all copies out of work completed before this CTA's recv filled).
  }
  if (aborted) {
    if (tid == 0) {
      raise_abort<C>(cluster, abort_word);
      // Copies into this CTA whose bytes it announced either land or time
      // out here; then a short grace period for the copies its peers issued
      // just before they saw the abort word (each lands within microseconds).
      if (hbm_out) mbar_wait_bounded(bar_hbm, hbm_phase, f, nullptr);
      if (recv_out) mbar_wait_bounded<true>(bar_recv, parity, f, nullptr);
      if (work_out) mbar_wait_bounded<true>(bar_work, parity, f, nullptr);
      const unsigned long long t0 = global_ns();
      while (global_ns() - t0 < 20000ull) __nanosleep(1000);
    }
    __syncthreads();
  }
  cluster.sync();  // no CTA leaves while a copy may still target it
}

// ------------------------------------------------ asynchronous write-back variant
// The x pass reads its pencils from the peers' shared memory as kind 7 does,
// but stores the results back with st.async, each store completing on the
// owner CTA's mbarrier (complete_tx).  A CTA starts its inverse z pass as
// soon as every write-back into its slab has landed, so the second cluster
// barrier of the step goes away, and with it that barrier's cluster-wide
// release, which orders every outstanding memory operation of the thread,
// the HBM stores of the previous orbital included.  The one remaining
// cluster barrier (after pass 2) orders shared memory only: since its last
// crossing the CTA has written nothing but its own shared memory (the
// write-backs are tracked by the receivers' mbarriers), so its release is
// restricted to shared::cta.  The slab is prefetched into L2 (as kind 7).
// Addresses into the peers' shared memory are 32-bit shared::cluster ones
// (mapa), which also keeps the pass-3 pointers out of 64-bit registers.
//
// Reuse without further signals: a peer reads and writes back region c of
// this CTA only between the cluster barrier and the completion of this
// CTA's mbarrier phase (it reads before it writes back, and the phase needs
// all of its write-backs); this CTA touches that region again only after
// the phase completed.
__device__ __forceinline__ void cluster_barrier_shared_release() {
  asm volatile("fence.release.sync_restrict::shared::cta.cluster;" ::: "memory");
  asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.aligned;" ::: "memory");
}

template <typename R>
__device__ __forceinline__ cplx<R> ld_cluster(uint32_t addr) {
  cplx<R> v;
  if constexpr (sizeof(R) == 4)
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.re), "=f"(v.im) : "r"(addr) : "memory");
  else
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.re), "=d"(v.im) : "r"(addr) : "memory");
  return v;
}

template <typename R>
__device__ __forceinline__ void st_async(uint32_t addr, cplx<R> v, uint32_t bar) {
  if constexpr (sizeof(R) == 4)
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];" ::"r"(addr),
                 "f"(v.re), "f"(v.im), "r"(bar)
                 : "memory");
  else
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(addr),
                 "d"(v.re), "d"(v.im), "r"(bar)
                 : "memory");
}

// Shared memory of the st.async kernel: the padded slab, the mbarriers and
// abort words, and (when the CTA's rows of an x-plane fill whole 32-bit
// words) the orbital's Z2 field words, fetched during pass 1 for pass 3.
// The general-field instance (FK = 2) instead stages the CTA's rows of a run's
// real FP32 weight table (field mode 3): S L floats of every x-plane.
template <typename R, int L, int C, int FK = 1>
struct AsyncShape {
  using Base = FusedShape<R, L, C>;
  static constexpr bool FW = (Base::S * L) % 32 == 0 && (L * L) % 32 == 0;
  static constexpr int W = FW ? Base::S * L / 32 : 0;  // words per x-plane of the CTA's rows
  // FK 2 with FP32 orbitals: room for a real weight table's rows, copied in
  // 16-byte pieces (rows of whole pieces, planes on 4 floats, an aligned start)
  static constexpr bool WT = (FK == 2 || FK == 3) && sizeof(R) == 4 && (Base::S * L) % 4 == 0 && L % 2 == 0 &&
                             (sizeof(cplx<R>) * Base::WORK + 32) % 16 == 0;
  static constexpr size_t EXTRA = WT ? (size_t)4 * Base::S * L * L : (size_t)(4 * L * W + 15) / 16 * 16;
  static constexpr size_t SMEM = PullShape<R, L, C, false>::SMEM + EXTRA;
};

// FK: 1 = compiled for Z2 fields only (with or without a position factor),
// 2 = for every other field, 3 = for a real FP32 weight table only (field
// mode 3, FP32); one instance per field class keeps the other classes' code,
// and its registers, out of the kernel.
template <typename R, int L, int C, bool PK = false, int FK = 1>
__global__ void __launch_bounds__(PullShape<R, L, C, false>::THREADS, PullShape<R, L, C, false>::MIN_BLOCKS)
    fused_step_async_kernel(FusedArgs f) {
  using Sh = FusedShape<R, L, C>;
  static_assert(C > 1, "the write-back goes to cluster peers");
  constexpr int S = Sh::S, LP = Sh::LP, REGION = Sh::REGION;
  constexpr int V = L * L * L;
  constexpr uint32_t SLAB_BYTES = (uint32_t)(Sh::STAGE * sizeof(cplx<R>));  // bytes written back into a CTA
  extern __shared__ __align__(128) unsigned char smem_raw[];
  cplx<R>* sm = reinterpret_cast<cplx<R>*>(smem_raw);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + Sh::WORK);  // write-backs into this CTA's slab
  uint64_t* idle = bar + 1;                                    // the time-out test's mbarrier
  // This CTA's abort words, by iteration parity: set (in this CTA's own
  // shared memory only) when a write-back wait of iteration i gave up, read
  // by every CTA of the cluster after the cluster barrier of iteration i + 1.
  // A word of parity p is written only between the barriers of iterations
  // with parity p and p + 1 and read only after the latter: every CTA sees
  // the same words and leaves at the same barrier.
  int* abort_words = reinterpret_cast<int*>(bar + 2);
  using AS = AsyncShape<R, L, C, FK>;
  uint32_t* fw = reinterpret_cast<uint32_t*>(bar + 4);  // [L][AS::W]: the orbital's field words (Z2)
  float* wbuf = reinterpret_cast<float*>(bar + 4);      // FK 2, [L][S L]: the CTA's rows of the weight table

  cg::cluster_group cluster = cg::this_cluster();
  const int c = (int)cluster.block_rank();
  const long cluster_id = blockIdx.x / C;
  const long n_clusters = gridDim.x / C;
  const int tid = threadIdx.x;

  auto off = [](int r, int xl, int yl, int z) { return r * REGION + (xl * S + yl) * LP + z; };
  auto slab = [&](long orb) {
    return reinterpret_cast<const cplx<R>*>(f.psi) + (size_t)orb * V + (size_t)c * S * L * L;
  };

  const bool z2_fast = FK == 1 && (f.field_mode == 1) && (f.pos == nullptr) && ((L * L) % 32 == 0);
  const bool z2_pos = FK == 1 && (f.field_mode == 1) && (f.zpos != nullptr) && ((L * L) % 32 == 0);
  R wp_hi, wp_lo, wm_hi, wm_lo;
  split<R>(f.w_plus, wp_hi, wp_lo);
  split<R>(f.w_minus, wm_hi, wm_lo);
  const bool w_exact = wp_lo == (R)0 && wm_lo == (R)0;

  if (tid == 0) {
    reinterpret_cast<volatile int*>(abort_words)[0] = 0;
    reinterpret_cast<volatile int*>(abort_words)[1] = 0;
    mbar_init(bar);
    mbar_init(idle);
  }
  cluster.sync();  // mbarriers and abort words are set up before any peer uses them
  // this CTA's region c and abort words; mapa turns them into every peer's copy
  const uint32_t my_region = smem_u32(sm + c * REGION);
  const uint32_t my_words = smem_u32(abort_words);
  uint32_t parity = 0;       // of this CTA's write-back phase and of the iteration
  bool outstanding = false;  // a write-back phase of `bar` (parity x_phase) not seen complete
  uint32_t x_phase = 0;
  bool aborted = false;
  long orb = cluster_id;
  if (tid == 0 && orb < f.n_orb_total) prefetch_l2(slab(orb), SLAB_BYTES);

  for (; orb < f.n_orb_total; orb += n_clusters) {
    const long conf = orb / f.batch;
    const uint64_t kb = f.off0 + (f.conf_base ? __ldg(f.conf_base + conf) : (uint64_t)conf * f.conf_stride);
    cplx<R>* gpsi = reinterpret_cast<cplx<R>*>(f.psi) + (size_t)orb * V;
    cplx<R> x[L];
    if (tid == 0 && orb + n_clusters < f.n_orb_total) prefetch_l2(slab(orb + n_clusters), SLAB_BYTES);
    // the field words pass 3 reads: the CTA's S rows of every x-plane (from
    // shared memory when the configuration's field starts on a word)
    const bool fw_ok = AS::FW && (z2_fast || z2_pos) && (kb & 31) == 0;
    if constexpr (AS::FW) {
      if (fw_ok) {
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (kb >> 5) + c * AS::W;
        for (int e = tid; e < L * AS::W; e += Sh::THREADS) fw[e] = __ldg(words + (e / AS::W) * (L * L / 32) + e % AS::W);
      }
    }
    // a real weight table (field mode 3): the CTA's rows of every x-plane,
    // S L floats each, copied by cp.async while pass 1 runs (16-byte pieces:
    // the table must start on 16 bytes and the configuration's part of it on
    // 4 floats; otherwise pass 3 reads the weights per site)
    const bool wt = AS::WT && f.field_mode == 3 && (kb & 3) == 0 &&
                    (reinterpret_cast<uintptr_t>(f.field) & 15) == 0;
    if constexpr (AS::WT) {
      if (wt) {
        constexpr int CH = S * L / 4;  // 16-byte pieces per x-plane
        const float* tab = reinterpret_cast<const float*>(f.field) + kb + (size_t)c * S * L;
        for (int e = tid; e < L * CH; e += Sh::THREADS) {
          const int xx = e / CH, j = e - xx * CH;
          const uint32_t d = smem_u32(wbuf + xx * S * L + 4 * j);
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(tab + (size_t)xx * L * L + 4 * j)
                       : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
      }
    }
    // ---- 1. k(p), forward DFT along y from the slab (L2): thread -> (xl, z)
    {
      const int z = tid % L, xl = tid / L;
      const int site0 = (c * S + xl) * L * L + z;
      const cplx<R>* src = slab(orb);
#pragma unroll
      for (int y = 0; y < L; ++y) {
        cplx<R> v;
        if constexpr (sizeof(R) == 4) {
          float2 t = __ldcg(reinterpret_cast<const float2*>(src) + (xl * L + y) * L + z);
          v = cplx<R>{t.x, t.y};
        } else {
          double2 t = __ldcg(reinterpret_cast<const double2*>(src) + (xl * L + y) * L + z);
          v = cplx<R>{t.x, t.y};
        }
        x[y] = apply_kin<R, PK>(f, site0 + y * L, v);
      }
      fft::dft<L, -1, R, PK>(x);
#pragma unroll
      for (int y = 0; y < L; ++y) sm[off(y / S, xl, y % S, z)] = x[y];
    }
    if constexpr (AS::WT) {
      if (wt) asm volatile("cp.async.wait_all;" ::: "memory");  // this thread's weight pieces have landed
    }
    __syncthreads();
    // ---- 2. forward DFT along z in place: thread -> (xl, y)
    {
      const int y = tid % L, xl = tid / L;
      cplx<R>* row = sm + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = row[j];
      fft::dft<L, -1, R, PK>(x);
#pragma unroll
      for (int j = 0; j < L; ++j) row[j] = x[j];
    }
    cluster_barrier_shared_release();
    if (orb != cluster_id) {  // did any CTA give up in the previous iteration?
      int any = 0;
#pragma unroll
      for (int r = 0; r < C; ++r) {
        int w;
        asm volatile("ld.shared::cluster.b32 %0, [%1];"
                     : "=r"(w)
                     : "r"(mapa_u32(my_words, (uint32_t)r) + 4u * (parity ^ 1u))
                     : "memory");
        any |= w;
      }
      if (any) {
        aborted = true;
        break;
      }
    }
    // ---- 3. x: forward DFT, times w, backward DFT on the pencils of y-slab
    // c, read from and written back to region c of CTA x/S
    if (tid == 0) expect_tx(bar, SLAB_BYTES);
    outstanding = true;
    x_phase = parity;
    {
      const int z = tid % L, yl = tid / L;
      const int site0 = (c * S + yl) * L + z;  // site of x = 0
#pragma unroll
      for (int xx = 0; xx < L; ++xx)
        x[xx] = ld_cluster<R>(mapa_u32(my_region, (uint32_t)(xx / S)) +
                              (uint32_t)((((xx % S) * S + yl) * LP + z) * sizeof(cplx<R>)));
      fft::dft<L, -1, R, PK>(x);
      if (fw_ok) {
        // words from shared memory: bit (yl L + z) of the CTA's rows of plane xx
        const uint32_t* wrow = fw + (yl * L + z) / 32;
        const int bit = (yl * L + z) % 32;
        if (z2_pos) {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (wrow[xx * AS::W] >> bit) & 1u;
            x[xx] = scale_w_zpos<R, PK>(f.zpos, site0 + xx * L * L, up, x[xx]);
          }
        } else if (w_exact) {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (wrow[xx * AS::W] >> bit) & 1u;
            x[xx] = scale_w1<R, PK>(x[xx], up ? wp_hi : wm_hi);
          }
        } else {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (wrow[xx * AS::W] >> bit) & 1u;
            x[xx] = scale_w<R, PK>(x[xx], up ? wp_hi : wm_hi, up ? wp_lo : wm_lo);
          }
        }
      } else if (z2_fast) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
        if (w_exact) {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
            x[xx] = scale_w1<R, PK>(x[xx], up ? wp_hi : wm_hi);
          }
        } else {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
            x[xx] = scale_w<R, PK>(x[xx], up ? wp_hi : wm_hi, up ? wp_lo : wm_lo);
          }
        }
      } else if (z2_pos) {
        const uint64_t k0 = kb + (uint64_t)site0;
        const uint32_t* words = reinterpret_cast<const uint32_t*>(f.field) + (k0 >> 5);
        const int bit = (int)(k0 & 31);
#pragma unroll
        for (int xx = 0; xx < L; ++xx) {
          const bool up = (__ldg(words + xx * (L * L / 32)) >> bit) & 1u;
          x[xx] = scale_w_zpos<R, PK>(f.zpos, site0 + xx * L * L, up, x[xx]);
        }
      } else if constexpr (FK == 2 || FK == 3) {
        if (AS::WT && wt) {
          // the weights of this thread's pencil, from the staged rows (rounded
          // products, as apply_w_general forms them)
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const float w = wbuf[xx * S * L + yl * L + z];
            x[xx] = cplx<R>{(R)__fmul_rn((float)x[xx].re, w), (R)__fmul_rn((float)x[xx].im, w)};
          }
        } else if constexpr (FK == 3) {
          // a table that cannot be staged: the same weights per site
          const float* tab = reinterpret_cast<const float*>(f.field) + kb + site0;
#pragma unroll
          for (int xx = 0; xx < L; ++xx) {
            const float w = __ldg(tab + xx * L * L);
            x[xx] = cplx<R>{(R)__fmul_rn((float)x[xx].re, w), (R)__fmul_rn((float)x[xx].im, w)};
          }
        } else {
#pragma unroll
          for (int xx = 0; xx < L; ++xx) x[xx] = apply_w_general<R>(f, kb, site0 + xx * L * L, x[xx]);
        }
      }
      fft::dft<L, +1, R, PK>(x);
      const uint32_t my_bar = smem_u32(bar);
#pragma unroll
      for (int xx = 0; xx < L; ++xx) {
        const uint32_t rank = (uint32_t)(xx / S);
        st_async<R>(mapa_u32(my_region, rank) + (uint32_t)((((xx % S) * S + yl) * LP + z) * sizeof(cplx<R>)), x[xx],
                    mapa_u32(my_bar, rank));
      }
    }
    // every peer's write-back into this CTA's slab
    const bool ok = stall_here(f, cluster_id, c, orb == cluster_id) ? mbar_wait_bounded(idle, 0u, f, nullptr)
                                                                    : mbar_wait_bounded<true>(bar, parity, f, nullptr);
    // ---- 4. backward DFT along z in place
    {
      const int y = tid % L, xl = tid / L;
      cplx<R>* row = sm + off(y / S, xl, y % S, 0);
#pragma unroll
      for (int j = 0; j < L; ++j) x[j] = row[j];
      fft::dft<L, +1, R, PK>(x);
#pragma unroll
      for (int j = 0; j < L; ++j) row[j] = x[j];
    }
    if (__syncthreads_or(!ok)) {
      // the write-backs did not all land: the cluster leaves at the next
      // cluster barrier (no further expect_tx on the stuck phase)
      if (tid == 0) reinterpret_cast<volatile int*>(abort_words)[parity] = 1;
    } else {
      outstanding = false;
    }
    parity ^= 1u;
    // ---- 5. backward DFT along y, times k(p), streaming stores
    {
      const int z = tid % L, xl = tid / L;
      const int site0 = (c * S + xl) * L * L + z;
#pragma unroll
      for (int y = 0; y < L; ++y) x[y] = sm[off(y / S, xl, y % S, z)];
      fft::dft<L, +1, R, PK>(x);
#pragma unroll
      for (int y = 0; y < L; ++y) {
        cplx<R> v = apply_kin<R, PK>(f, site0 + y * L, x[y]);
        if constexpr (sizeof(R) == 4)
          __stcs(reinterpret_cast<float2*>(gpsi) + site0 + y * L, make_float2(v.re, v.im));
        else
          __stcs(reinterpret_cast<double2*>(gpsi) + site0 + y * L, make_double2(v.re, v.im));
      }
    }
    // pass 1 of the next orbital writes, per thread, the elements this thread
    // read in pass 5; no peer touches this CTA's shared memory before the
    // next cluster barrier
  }
  // leaving early: write-backs this CTA expected land (or time out) first
  if (aborted && outstanding && tid == 0) mbar_wait_bounded<true>(bar, x_phase, f, nullptr);
  cluster.sync();
}

// KIND 0: one lane per pencil, exchange through peers' shared memory;
// 1: two lanes per pencil; 2: bulk-copy exchange, staged slab; 3: bulk-copy
// exchange, slab prefetched into L2; 4, 5, 6: kinds 0, 2, 3 with the packed
// FP32x2 transforms (FP32 only); 7, 8: kinds 0, 4 with the slab prefetched
// into L2 instead of staged (four CTAs per SM); 9, 10: kinds 6, 3 with the
// CTA's slab of the kinetic table resident in shared memory (FP32 only);
// 11, 12: kinds 7, 8 with the x pass written back by st.async onto the
// owners' mbarriers (one cluster barrier per orbital).
template <typename R, int L, int C, int KIND = 0>
static nrcps_status launch_fused(nrcps_context* ctx, const FusedArgs& f, int ctas_per_sm_hint) {
  using Sh = FusedShape<R, L, C>;
  static_assert(KIND < 4 || KIND == 7 || KIND == 11 || sizeof(R) == 4,
                "packed transforms and the resident k(p) slab are FP32");
  constexpr int THREADS = KIND == 1 ? SplitShape<R, L, C>::THREADS : Sh::THREADS;
  size_t SMEM = (KIND == 2 || KIND == 5)   ? BulkShape<R, L, C, true>::SMEM
                          : (KIND == 3 || KIND == 6) ? BulkShape<R, L, C, false>::SMEM
                          : (KIND == 9 || KIND == 10) ? BulkShape<R, L, C, false, true>::SMEM
                          : (KIND >= 11) ? AsyncShape<R, L, C, 1>::SMEM
                          : (KIND == 7 || KIND == 8) ? PullShape<R, L, C, false>::SMEM
                                                     : Sh::SMEM;
  void (*kern)(FusedArgs);
  if constexpr (KIND == 1) kern = fused_step_split_kernel<R, L, C>;
  else if constexpr (KIND == 2) kern = fused_step_bulk_kernel<R, L, C, true>;
  else if constexpr (KIND == 3) kern = fused_step_bulk_kernel<R, L, C, false>;
  else if constexpr (KIND == 4) kern = fused_step_kernel<R, L, C, true>;
  else if constexpr (KIND == 5) kern = fused_step_bulk_kernel<R, L, C, true, true>;
  else if constexpr (KIND == 6) kern = fused_step_bulk_kernel<R, L, C, false, true>;
  else if constexpr (KIND == 9) kern = fused_step_bulk_kernel<R, L, C, false, true, true>;
  else if constexpr (KIND == 10) kern = fused_step_bulk_kernel<R, L, C, false, false, true>;
  else if constexpr (KIND == 7) kern = fused_step_kernel<R, L, C, false, false>;
  else if constexpr (KIND == 8) kern = fused_step_kernel<R, L, C, true, false>;
  else if constexpr (KIND == 11 || KIND == 12) {
    // the instance of the field's class: Z2 (bits, with or without a
    // position factor) or any other field
    const bool z2 = f.field_mode == 1 && (L * L) % 32 == 0 && (f.pos == nullptr || f.zpos != nullptr);
    kern = z2 ? fused_step_async_kernel<R, L, C, KIND == 12, 1> : fused_step_async_kernel<R, L, C, KIND == 12, 2>;
    if (!z2) SMEM = AsyncShape<R, L, C, 2>::SMEM;
    if constexpr (sizeof(R) == 4) {
      if (f.field_mode == 3) {  // (FP32 only: the host sends mode 3 with FP32 orbitals alone)
        kern = fused_step_async_kernel<R, L, C, KIND == 12, 3>;
        SMEM = AsyncShape<R, L, C, 3>::SMEM;
      }
    }
  }
  else kern = fused_step_kernel<R, L, C>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
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
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = SMEM;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(C * ctx->sm_count);
  e = cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg);
  if (e != cudaSuccess || max_clusters <= 0) {
    cudaGetLastError();
    max_clusters = ctx->sm_count / C;
    if (max_clusters < 1) return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "fused_step: cluster of %d does not fit", C);
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
  int kind;  // 0: exchange through peers' shared memory; 1: lane split; 2/3: bulk-copy exchange; 4-6: packed;
             // 7/8: peer access with the slab prefetched into L2; 9/10: kinds 6/3 with k(p) resident
  FusedLauncher fn;
};

// Instantiated (precision, L, cluster size, kind) variants.  Shared memory
// per CTA is one or two buffers of C padded regions of (L/C)^2 (L+1) + L/C
// complex values, plus the staged slab (L/C) L^2 for kinds 0-2; cluster
// sizes are chosen so that 2-4 CTAs share an SM.  Sizes above 8 are
// non-portable cluster shapes (allowed on B200).
// Listed best-first per (precision, L) as measured on B200 (the first entry
// is the default before autotuning).
static const FusedVariant kVariants[] = {
    {NRCPS_F32, 8, 1, 4, launch_fused<float, 8, 1, 4>},
    {NRCPS_F32, 8, 1, 0, launch_fused<float, 8, 1>},
    {NRCPS_F32, 16, 1, 4, launch_fused<float, 16, 1, 4>},
    {NRCPS_F32, 16, 1, 0, launch_fused<float, 16, 1>},
    {NRCPS_F32, 16, 2, 2, launch_fused<float, 16, 2, 2>},
    {NRCPS_F32, 16, 2, 9, launch_fused<float, 16, 2, 9>},
    {NRCPS_F32, 16, 2, 10, launch_fused<float, 16, 2, 10>},
    {NRCPS_F32, 16, 2, 0, launch_fused<float, 16, 2>},
    {NRCPS_F32, 16, 2, 11, launch_fused<float, 16, 2, 11>},
    {NRCPS_F32, 16, 1, 1, launch_fused<float, 16, 1, 1>},
    {NRCPS_F32, 24, 3, 5, launch_fused<float, 24, 3, 5>},
    {NRCPS_F32, 24, 4, 4, launch_fused<float, 24, 4, 4>},
    {NRCPS_F32, 24, 3, 2, launch_fused<float, 24, 3, 2>},
    {NRCPS_F32, 24, 4, 2, launch_fused<float, 24, 4, 2>},
    {NRCPS_F32, 24, 4, 9, launch_fused<float, 24, 4, 9>},
    {NRCPS_F32, 24, 4, 10, launch_fused<float, 24, 4, 10>},
    {NRCPS_F32, 24, 3, 0, launch_fused<float, 24, 3>},
    {NRCPS_F32, 24, 4, 0, launch_fused<float, 24, 4>},
    {NRCPS_F32, 24, 4, 11, launch_fused<float, 24, 4, 11>},
    {NRCPS_F32, 32, 8, 4, launch_fused<float, 32, 8, 4>},
    {NRCPS_F32, 32, 8, 7, launch_fused<float, 32, 8, 7>},
    {NRCPS_F32, 32, 8, 11, launch_fused<float, 32, 8, 11>},
    {NRCPS_F32, 32, 8, 12, launch_fused<float, 32, 8, 12>},
    {NRCPS_F32, 32, 4, 11, launch_fused<float, 32, 4, 11>},
    {NRCPS_F32, 32, 2, 11, launch_fused<float, 32, 2, 11>},
    {NRCPS_F32, 32, 16, 11, launch_fused<float, 32, 16, 11>},
    {NRCPS_F32, 32, 8, 8, launch_fused<float, 32, 8, 8>},
    {NRCPS_F32, 32, 8, 6, launch_fused<float, 32, 8, 6>},
    {NRCPS_F32, 32, 8, 5, launch_fused<float, 32, 8, 5>},
    {NRCPS_F32, 32, 8, 3, launch_fused<float, 32, 8, 3>},
    {NRCPS_F32, 32, 8, 9, launch_fused<float, 32, 8, 9>},
    {NRCPS_F32, 32, 8, 10, launch_fused<float, 32, 8, 10>},
    {NRCPS_F32, 32, 16, 3, launch_fused<float, 32, 16, 3>},
    {NRCPS_F32, 32, 8, 0, launch_fused<float, 32, 8>},
    {NRCPS_F32, 32, 8, 2, launch_fused<float, 32, 8, 2>},
    {NRCPS_F32, 32, 8, 1, launch_fused<float, 32, 8, 1>},
    {NRCPS_F32, 48, 12, 11, launch_fused<float, 48, 12, 11>},
    {NRCPS_F32, 48, 12, 7, launch_fused<float, 48, 12, 7>},
    {NRCPS_F32, 48, 12, 3, launch_fused<float, 48, 12, 3>},
    {NRCPS_F32, 48, 16, 4, launch_fused<float, 48, 16, 4>},
    {NRCPS_F32, 48, 16, 0, launch_fused<float, 48, 16>},
    {NRCPS_F32, 48, 16, 3, launch_fused<float, 48, 16, 3>},
    {NRCPS_F32, 48, 16, 1, launch_fused<float, 48, 16, 1>},
    {NRCPS_F64, 8, 1, 0, launch_fused<double, 8, 1>},
    {NRCPS_F64, 16, 2, 2, launch_fused<double, 16, 2, 2>},
    {NRCPS_F64, 16, 2, 0, launch_fused<double, 16, 2>},
    {NRCPS_F64, 16, 2, 1, launch_fused<double, 16, 2, 1>},
    {NRCPS_F64, 24, 4, 2, launch_fused<double, 24, 4, 2>},
    {NRCPS_F64, 24, 4, 0, launch_fused<double, 24, 4>},
    {NRCPS_F64, 24, 4, 11, launch_fused<double, 24, 4, 11>},
    {NRCPS_F64, 32, 16, 3, launch_fused<double, 32, 16, 3>},
    {NRCPS_F64, 32, 16, 7, launch_fused<double, 32, 16, 7>},
    {NRCPS_F64, 32, 16, 11, launch_fused<double, 32, 16, 11>},
    {NRCPS_F64, 32, 16, 0, launch_fused<double, 32, 16>},
    {NRCPS_F64, 32, 8, 0, launch_fused<double, 32, 8>},
    {NRCPS_F64, 32, 16, 2, launch_fused<double, 32, 16, 2>},
    {NRCPS_F64, 32, 8, 1, launch_fused<double, 32, 8, 1>},
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
// Scratch orbitals for the autotuner: values of order one that vary from
// word to word (all-zero buffers move through the memory system differently
// from real orbitals), k(p) = 1 and a half-filled Z2 field.
__global__ void autotune_fill_kernel(uint32_t* words, long n_words, int fp64) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_words; i += (long)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 0x9E3779B1u;
    h ^= h >> 15;
    h *= 0x85EBCA77u;
    h ^= h >> 13;
    // FP32: a float in [0.5, 1) with random mantissa and sign; FP64: keep the
    // high word of each double in [0.5, 1) the same way, the low word random
    if (!fp64 || (i & 1)) words[i] = 0x3F000000u | (h & 0x807FFFFFu);
    else words[i] = h;
  }
}

__global__ void autotune_unit_kin_kernel(void* kin, long V, int fp64) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V; i += (long)gridDim.x * blockDim.x) {
    if (fp64) reinterpret_cast<double*>(kin)[i] = 1.0;
    else reinterpret_cast<float2*>(kin)[i] = make_float2(1.0f, 0.0f);
  }
}

nrcps_status fused_autotune(nrcps_context* ctx, nrcps_precision prec, int L, int* chosen_cluster) {
  init_choices();
  int dev = ctx->device & 15;
  if (L < 64 && g_choice[dev][prec][L] >= 0) {
    if (chosen_cluster)
      *chosen_cluster = kVariants[g_choice[dev][prec][L]].C * (kVariants[g_choice[dev][prec][L]].kind == 1 ? -1 : 1);
    return NRCPS_OK;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cs);
  if (cs != cudaStreamCaptureStatusNone) return NRCPS_OK;  // keep the default
  const long V = (long)L * L * L;
  const size_t esz = prec == NRCPS_F64 ? 16 : 8;
  // ~2 GB (16x L2), up to 8192 orbitals: at 2048 orbitals the ranking of the
  // L=32 variants differed from the one at production batch sizes
  long norb = (long)(2048L * 1024 * 1024 / (V * esz));
  if (norb > 8192) norb = 8192;
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
  {
    const long n_words = (long)(esz / 4) * V * norb;
    autotune_fill_kernel<<<grid_for(n_words, 256, (long)ctx->sm_count * 8), 256, 0, ctx->stream>>>(
        reinterpret_cast<uint32_t*>(psi), n_words, prec == NRCPS_F64 ? 1 : 0);
  }
  autotune_unit_kin_kernel<<<grid_for(V, 256, (long)ctx->sm_count * 8), 256, 0, ctx->stream>>>(
      kin, V, prec == NRCPS_F64 ? 1 : 0);
  cudaMemsetAsync(bits, 0x5A, (size_t)(V / 32 + 1) * 4, ctx->stream);
  FusedArgs f{};
  f.psi = psi;
  f.n_orb_total = norb;
  f.batch = (int)norb;
  f.kin_f = (const float2*)kin;
  f.kin_d = (const double*)kin;
  f.field_mode = 1;
  f.field = bits;
  // a = 0 with k = 1: the step preserves the norm, so the ~100 timing
  // launches on the same buffer keep the values of order one
  f.a = 0.0;
  f.vol = (double)V;
  f.inv_vol = 1.0 / (double)V;
  f.w_plus = 1.0 / V;
  f.w_minus = 1.0 / V;
  f.err = ctx->dev_err;
  f.wait_ns = ctx->fused_wait_ns;
  f.stall_test = 0;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  // Three rounds over the variants, each timed on 3 launches after one
  // untimed launch; a variant's time is its fastest round (single rounds
  // varied by ~15 % between neighbouring variants on B200).
  float best = 1e30f;
  int best_i = -1;
  long saved = ctx->launches;
  float round_ms[kNumVariants];
  bool ok[kNumVariants];
  for (int i = 0; i < kNumVariants; ++i) {
    round_ms[i] = 1e30f;
    ok[i] = kVariants[i].prec == prec && kVariants[i].L == L;
  }
  for (int round = 0; round < 3; ++round) {
    for (int i = 0; i < kNumVariants; ++i) {
      if (!ok[i]) continue;
      if (kVariants[i].fn(ctx, f, 0) != NRCPS_OK) {
        cudaGetLastError();
        ok[i] = false;
        continue;
      }
      cudaEventRecord(t0, ctx->stream);
      for (int r = 0; r < 3; ++r) kVariants[i].fn(ctx, f, 0);
      cudaEventRecord(t1, ctx->stream);
      if (cudaEventSynchronize(t1) != cudaSuccess) {
        cudaGetLastError();
        ok[i] = false;
        continue;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, t0, t1);
      if (ms < round_ms[i]) round_ms[i] = ms;
    }
  }
  for (int i = 0; i < kNumVariants; ++i)
    if (ok[i] && round_ms[i] < best) {
      best = round_ms[i];
      best_i = i;
    }
  ctx->launches = saved;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(psi);
  cudaFree(kin);
  cudaFree(bits);
  if (best_i >= 0 && L < 64) g_choice[dev][prec][L] = best_i;
  if (chosen_cluster && best_i >= 0) *chosen_cluster = kVariants[best_i].C * (kVariants[best_i].kind == 1 ? -1 : 1);
  return NRCPS_OK;
}

// The variant (index into kVariants) a step of (prec, L) runs under the
// context's options: the autotuned one, or the first listed, restricted to
// the forced cluster size / split / kind; -1 if none qualifies.
static int fused_pick(nrcps_context* ctx, nrcps_precision prec, int L, int cluster) {
  init_choices();
  int pick = -1;
  const int want_split = ctx->fused_split;  // -1: any
  const int want_kind = ctx->fused_kind;    // -1: any
  auto admissible = [&](const FusedVariant& v) {
    return (cluster <= 0 || v.C == cluster) && (want_split < 0 || (v.kind == 1) == (want_split == 1)) &&
           (want_kind < 0 || v.kind == want_kind);
  };
  const int tuned = L < 64 ? g_choice[ctx->device & 15][prec][L] : -1;
  if (cluster > 0 || want_split >= 0 || want_kind >= 0) {
    if (tuned >= 0 && admissible(kVariants[tuned])) pick = tuned;
    for (int i = 0; i < kNumVariants && pick < 0; ++i)
      if (kVariants[i].prec == prec && kVariants[i].L == L && admissible(kVariants[i])) pick = i;
  } else {
    pick = tuned;
    for (int i = 0; i < kNumVariants && pick < 0; ++i)  // default: the first listed variant
      if (kVariants[i].prec == prec && kVariants[i].L == L) pick = i;
  }
  return pick;
}

nrcps_status fused_choice(nrcps_context* ctx, nrcps_precision prec, int L, int* kind, int* cluster) {
  const int d[3] = {L, L, L};
  const int pick = (ctx->fused_enabled && fused_supported(prec, d)) ? fused_pick(ctx, prec, L, ctx->fused_cluster) : -1;
  *kind = pick >= 0 ? kVariants[pick].kind : -1;
  *cluster = pick >= 0 ? kVariants[pick].C : -1;
  return NRCPS_OK;
}

// One fused step; `kin_table` is (hi, lo) float pairs for prec F32 and FP64 for F64.
// cluster = 0 selects the autotuned (or default) cluster size.
nrcps_status fused_step(nrcps_context* ctx, void* psi, int batch, int nconf, const int d[3], const void* kin_table,
                        nrcps_precision prec, const nrcps_position_factor* w, int cluster, const void* zpos) {
  if (!fused_supported(prec, d)) return NRCPS_ERR_UNSUPPORTED;
  // the bulk-copy kinds move slabs of psi in 16-byte units: a psi that does
  // not start on 16 bytes (a caller's view at an odd FP32 element) takes the
  // pencil passes
  if (reinterpret_cast<uintptr_t>(psi) & 15) return NRCPS_ERR_UNSUPPORTED;
  // FP32 weight tables carry the whole factor: FP32 orbitals, no position factor
  if (w->field_mode == 3 && (prec != NRCPS_F32 || w->dev_pos)) return NRCPS_ERR_UNSUPPORTED;
  FusedArgs f;
  f.psi = psi;
  f.n_orb_total = (long)batch * nconf;
  f.batch = batch;
  f.kin_f = prec == NRCPS_F32 ? (const float2*)kin_table : nullptr;
  f.kin_d = prec == NRCPS_F64 ? (const double*)kin_table : nullptr;
  f.pos = w->dev_pos;
  f.zpos = (w->field_mode == 1 && w->dev_pos && ctx->fused_zpos) ? zpos : nullptr;
  f.field_mode = w->field_mode;
  f.field = w->dev_field;
  f.off0 = w->bit0;
  f.conf_stride = w->conf_stride;
  f.conf_base = w->dev_conf_base;
  f.a = w->a;
  f.vol = (double)d[0] * d[1] * d[2];
  f.inv_vol = 1.0 / f.vol;
  f.w_plus = (1.0 + f.a) / f.vol;
  f.w_minus = (1.0 - f.a) / f.vol;
  f.err = ctx->dev_err;
  f.wait_ns = ctx->fused_wait_ns;
  f.stall_test = ctx->fused_stall_test;
  if (f.n_orb_total == 0) return NRCPS_OK;
  const int pick = fused_pick(ctx, prec, d[0], cluster);
  if (pick < 0)
    return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "no fused variant with cluster size %d, split %d, kind %d",
                     cluster, ctx->fused_split, ctx->fused_kind);
  return kVariants[pick].fn(ctx, f, 0);
}

}  // namespace nrcps

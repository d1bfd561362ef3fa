// gram_tc.cu -- the Gram matrices G_c = Psi_c^H Psi_c of the QR
// re-orthonormalisation (qr.cu) on the tcgen05 tensor cores, for FP32
// orbitals and N <= 32.
//
// G_ij = sum_p conj(psi_i(p)) psi_j(p) over the interleaved (re, im) floats
// k = 2p + r of an orbital is two real products per entry:
//   Re G_ij = sum_k psi_i[k] psi_j[k],
//   Im G_ij = sum_k rot(psi_i)[k] psi_j[k],  rot(x)[2p] = -Im x(p), rot(x)[2p+1] = Re x(p).
// Every float is split into TF32 hi + lo (x = hi + lo to ~2^-22), and
//   psi_i . psi_j ~ hi_i.hi_j + hi_i.lo_j + lo_i.hi_j,
// where the last product is the second with i and j exchanged (and, for the
// imaginary part, rot(lo_i).hi_j = -rot(hi_j).lo_i).  So one MMA per k-step
// with A = [hi; rot(hi)] of the orbitals and B = [hi; lo] gives every term:
// the drain adds D[i][hi j] + D[i][lo j] and +-D[j][lo i] (a transpose
// within one warp).  Two configurations share a tile: A rows 0-31 hi c0,
// 32-63 rot(hi) c0, 64-95 hi c1, 96-127 rot(hi) c1; B rows 0-31 hi c0, 32-63
// lo c0, 64-95 hi c1, 96-127 lo c1 (M = N = 128, K = 8 per MMA).  The
// tensor core accumulates in FP32 over 256 floats of K only (a chunk): a
// longer FP32 accumulation in TMEM drifts (a relative bias of ~3e-4 over
// K = 65536 was measured), so every chunk is drained into FP64 registers
// while the next accumulates in the other TMEM buffer.
//
// The Gram only has to be accurate enough for R^-1 to make the orbitals
// well conditioned: the measured determinants use the identity
// det S_n(Psi) = det S_n(Psi R^-1) / prod_{i<=n} (R^-1)_ii for the R^-1 that
// is actually applied, whatever its accuracy (see qr.cu).
//
// One persistent CTA per SM over configuration pairs; 10 warps:
//   warp 0      TMA producer: each configuration's raw k-block (rows
//               c N .. c N + NR - 1, NR = N rounded up to 8, 32 floats,
//               128-byte swizzle) into the B hi rows of the stage, STAGES deep;
//   warp 1      TMEM owner (2 x 128 columns) and MMA issuer (one thread);
//   warps 2-5   build B lo, A hi and A rot(hi) from the raw rows (the swizzle
//               permutes 16-byte chunks within a row by the row's index mod
//               8, which the copies keep, so every copy is chunk for chunk);
//   warps 6-9   drain an accumulator buffer per configuration pair (warp q of
//               the TMEM lane quarters owns one 32-row block of A) and write
//               Re or Im of G.
// Every mbarrier wait is bounded; a timeout sets the context's error flag and
// every role leaves its loop, waits (bounded) for its own copies and MMAs in
// flight, frees the TMEM and returns.
#include <cuda.h>

#include "common.cuh"

namespace nrcps {

bool make_fp32_map_sw128(CUtensorMap* m, const void* ptr, long rows, long K, int box_rows);

namespace gtc {

constexpr int BK = 32;                             // floats of K per k-block: one 128-byte swizzle row
constexpr int ROWS = 32;                           // operand rows per configuration block
constexpr int STAGES = 6;
constexpr int CHUNK = 8;                           // k-blocks (256 floats of K) per FP32 accumulation
constexpr uint32_t BLOCK_BYTES = ROWS * BK * 4;    // 4 KB: 32 rows of one k-block
constexpr uint32_t OP_BYTES = 4 * BLOCK_BYTES;     // 16 KB: 128 operand rows
constexpr uint32_t STAGE_BYTES = 2 * OP_BYTES;     // A then B
constexpr int THREADS = 320;
constexpr uint32_t TMEM_COLS = 256;                // two 128-column accumulators
constexpr int XLD = 33;                            // padded row of a drain warp's transpose buffer
constexpr uint32_t X_BYTES = 4 * 32 * XLD * 4;
constexpr size_t SMEM = (size_t)STAGES * STAGE_BYTES + X_BYTES + 1024 /* alignment */ + 256 /* barriers */;
// instruction descriptor: D F32, A/B TF32, both K-major, N = 128, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

struct Args {
  int nconf;
  int N;
  int nr;        // rows per configuration load: N rounded up to 8
  int nkb;       // k-blocks per configuration: 2 V / BK
  int nch;       // chunks per configuration: ceil(nkb / CHUNK)
  int ntiles;    // configuration pairs
  double* G;     // [nconf][N][N] complex
  int* err;
};

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long gns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait (two seconds of the global timer) that also gives up once
// another role has aborted; a timeout raises the abort flag and the
// context's error flag.
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag, int* err) {
  if (bar_try(b, parity)) return true;
  const unsigned long long t0 = gns();
  for (int i = 0;; ++i) {
    if (bar_try(b, parity)) return true;
    if ((i & 63) == 63) {
      if (*abort_flag) return false;
      if (gns() - t0 > 2000000000ull) break;
    }
  }
  *abort_flag = 1;
  if (err) atomicExch(err, 1);
  return false;
}
// Bounded wait on the way out (ignores the abort flag).
__device__ __forceinline__ void bar_drain(uint64_t* b, uint32_t parity, int* err) {
  const unsigned long long t0 = gns();
  while (!bar_try(b, parity))
    if (gns() - t0 > 2000000000ull) {
      if (err) atomicExch(err, 1);
      return;
    }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          su32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(su32(bar))
      : "memory");
}

// K-major operand tile with the 128-byte swizzle: 8-row atoms of 1024 bytes.
__device__ __forceinline__ uint64_t smem_desc(const void* p) {
  const uint64_t a = (uint64_t)((su32(p) >> 4) & 0x3FFFu);
  return a | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}

// TF32 rounding of a float's bit pattern (nearest, ties away from zero).
__device__ __forceinline__ uint32_t tf32_round_bits(uint32_t b) { return (b + 0x1000u) & 0xFFFFE000u; }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(THREADS, 1) gram_tc_kernel(const __grid_constant__ CUtensorMap map_psi, Args g) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  float* xbuf = reinterpret_cast<float*>(base + (size_t)STAGES * STAGE_BYTES);  // [4][32][XLD]
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + (size_t)STAGES * STAGE_BYTES + X_BYTES);
  uint64_t* full = bars;               // raw rows landed
  uint64_t* conv = bars + STAGES;      // operands built (4 converter warps)
  uint64_t* empty = bars + 2 * STAGES; // MMAs of the stage completed
  uint64_t* tfull = bars + 3 * STAGES; // [2] a pair's MMAs completed in TMEM buffer b
  uint64_t* tempty = tfull + 2;        // [2] TMEM buffer b read out (4 drain warps)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  volatile int* last_commit = abort_flag + 1;  // last chunk (of this CTA) whose TMEM-full commit was issued

  auto stage_a = [&](int s) { return base + (size_t)s * STAGE_BYTES; };
  auto stage_b = [&](int s) { return base + (size_t)s * STAGE_BYTES + OP_BYTES; };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_local = (int)blockIdx.x < g.ntiles ? (g.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int total = n_local * g.nkb;  // k-blocks this CTA streams

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      bar_init(full + s, 1);
      bar_init(conv + s, 4);
      bar_init(empty + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      bar_init(tfull + b, 1);
      bar_init(tempty + b, 4);
    }
    *abort_flag = 0;
    *last_commit = -1;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t load_bytes = (uint32_t)g.nr * BK * 4;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int issued = 0;
      for (int i = 0; i < total; ++i) {
        const int s = i % STAGES;
        if (i >= STAGES && !bar_wait(empty + s, (uint32_t)((i / STAGES) - 1) & 1u, abort_flag, g.err)) break;
        const int t = (int)blockIdx.x + (i / g.nkb) * (int)gridDim.x;  // configuration pair
        const int x = (i % g.nkb) * BK;
        bar_expect_tx(full + s, 2 * load_bytes);
        // rows beyond the last configuration read the fill value (zero)
        tma_load_2d(stage_b(s), &map_psi, x, (2 * t) * g.N, full + s);
        tma_load_2d(stage_b(s) + 2 * BLOCK_BYTES, &map_psi, x, (2 * t + 1) * g.N, full + s);
        ++issued;
      }
      for (int i = issued - STAGES < 0 ? 0 : issued - STAGES; i < issued; ++i)
        bar_drain(full + (i % STAGES), (uint32_t)(i / STAGES) & 1u, g.err);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      int i = 0, gc = 0;  // k-block and chunk counters of this CTA
      bool stop = false;
      for (int j = 0; j < n_local && !stop; ++j) {
        for (int ch = 0; ch < g.nch && !stop; ++ch, ++gc) {
          const int b = gc & 1;
          if (gc >= 2 && !bar_wait(tempty + b, (uint32_t)((gc >> 1) - 1) & 1u, abort_flag, g.err)) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t d = tmem + (uint32_t)(b * 128);
          const int kb1 = (ch + 1) * CHUNK < g.nkb ? (ch + 1) * CHUNK : g.nkb;
          for (int kb = ch * CHUNK; kb < kb1; ++kb, ++i) {
            const int s = i % STAGES;
            if (!bar_wait(conv + s, (uint32_t)(i / STAGES) & 1u, abort_flag, g.err)) {
              stop = true;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint64_t ad = smem_desc(stage_a(s)), bd = smem_desc(stage_b(s));
#pragma unroll
            for (int k = 0; k < BK / 8; ++k)  // K = 8 TF32 = 32 bytes per MMA: advance the start address
              mma_tf32(d, ad + (uint64_t)(2 * k), bd + (uint64_t)(2 * k), (kb > ch * CHUNK || k > 0) ? 1u : 0u);
            mma_commit(empty + s);
          }
          mma_commit(tfull + b);  // completes once every MMA issued so far has
          *last_commit = gc;
        }
      }
    }
  } else if (warp < 6) {
    // ------------------------------------------------------------ converters
    // raw x (B hi rows) -> B hi = tf32(x), B lo = tf32(x - hi), A hi = hi,
    // A rot = (-hi.im, hi.re) per complex pair; chunk for chunk (16 bytes =
    // two complex values) at the same position in rows with the same index
    // mod 8, so the swizzle needs no attention.
    const int ct = threadIdx.x - 64;  // 0..127
    bool ok = true;
    for (int i = 0; i < total && ok; ++i) {
      const int s = i % STAGES;
      if (!bar_wait(full + s, (uint32_t)(i / STAGES) & 1u, abort_flag, g.err)) ok = false;
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      unsigned char* A = stage_a(s);
      unsigned char* B = stage_b(s);
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int e = ct + 128 * r;              // 0..511: (configuration, row, chunk)
        const int q = e >> 8, row = (e >> 3) & 31, ch = e & 7;
        if (row >= g.nr) continue;
        const size_t hi_off = (size_t)(64 * q + row) * 128 + 16 * ch;
        const size_t lo_off = hi_off + 32 * 128;
        const uint4 x = *reinterpret_cast<const uint4*>(B + hi_off);
        uint4 hi, lo, rot;
        hi.x = tf32_round_bits(x.x);
        hi.y = tf32_round_bits(x.y);
        hi.z = tf32_round_bits(x.z);
        hi.w = tf32_round_bits(x.w);
        lo.x = tf32_round_bits(__float_as_uint(__uint_as_float(x.x) - __uint_as_float(hi.x)));
        lo.y = tf32_round_bits(__float_as_uint(__uint_as_float(x.y) - __uint_as_float(hi.y)));
        lo.z = tf32_round_bits(__float_as_uint(__uint_as_float(x.z) - __uint_as_float(hi.z)));
        lo.w = tf32_round_bits(__float_as_uint(__uint_as_float(x.w) - __uint_as_float(hi.w)));
        rot.x = hi.y ^ 0x80000000u;  // -Im
        rot.y = hi.x;                // Re
        rot.z = hi.w ^ 0x80000000u;
        rot.w = hi.z;
        *reinterpret_cast<uint4*>(B + hi_off) = hi;
        *reinterpret_cast<uint4*>(B + lo_off) = lo;
        *reinterpret_cast<uint4*>(A + hi_off) = hi;
        *reinterpret_cast<uint4*>(A + lo_off) = rot;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor-core reads
      __syncwarp();
      if (lane == 0) bar_arrive(conv + s);
    }
  } else {
    // ------------------------------------------------------------ drains
    const int q = warp & 3;            // TMEM lane quarter = A block: hi c0, rot c0, hi c1, rot c1
    const int pair_half = q >> 1;      // configuration 0 or 1 of the pair
    const bool imag = (q & 1) != 0;    // rot(hi) rows: Im G
    const uint32_t col0 = (uint32_t)(64 * pair_half);  // B hi columns; lo at +32
    float* X = xbuf + (size_t)q * 32 * XLD;
    bool ok = true;
    int gc = 0;
    for (int j = 0; j < n_local && ok; ++j) {
      double acc_hi[32], acc_lo[32];  // D[row][hi j], D[row][lo j] summed over the chunks in FP64
#pragma unroll
      for (int k = 0; k < 32; ++k) acc_hi[k] = acc_lo[k] = 0.0;
      for (int ch = 0; ch < g.nch; ++ch, ++gc) {
        const int b = gc & 1;
        if (ok && !bar_wait(tfull + b, (uint32_t)(gc >> 1) & 1u, abort_flag, g.err)) ok = false;
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t t0 = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * 128) + col0;
        float v[32];
        tmem_ld32(t0, v);
#pragma unroll
        for (int k = 0; k < 32; ++k) acc_hi[k] += (double)v[k];
        tmem_ld32(t0 + 32, v);
#pragma unroll
        for (int k = 0; k < 32; ++k) acc_lo[k] += (double)v[k];
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) bar_arrive(tempty + b);
      }
      if (!ok) break;
#pragma unroll
      for (int k = 0; k < 32; ++k) X[lane * XLD + k] = (float)acc_lo[k];  // the exchanged term: ~2^-11 of G
      __syncwarp();
      const int t = (int)blockIdx.x + j * (int)gridDim.x;
      const int c = 2 * t + pair_half;
      if (c < g.nconf && lane < g.N) {
        // Re: hi_i.hi_j + hi_i.lo_j + hi_j.lo_i; Im: the same with rot(hi_i),
        // the exchanged term entering with a minus sign
        double* out = g.G + 2 * ((size_t)c * g.N + lane) * g.N + (imag ? 1 : 0);
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          if (k < g.N) {
            const double x = (double)X[k * XLD + lane];
            out[2 * k] = acc_hi[k] + acc_lo[k] + (imag ? -x : x);
          }
        }
      }
      __syncwarp();  // X is rewritten for the next pair
    }
  }
  // ---------------------------------------------------------------- teardown
  __syncthreads();
  if (warp == 1) {
    const int last = *last_commit;  // every MMA of this CTA is covered by its last chunk commit
    if (last >= 0) bar_drain(tfull + (last & 1), (uint32_t)(last >> 1) & 1u, g.err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace gtc

// The shapes the tensor-core Gram takes: N <= 32 orbitals, K = 2V a multiple
// of 32 floats, rows addressable by the tensor map, and at least one load
// box (N rounded up to 8 rows) of orbitals in the batch.
bool gram_tc_supported(int N, long vol, int nconf) {
  return N > 0 && N <= gtc::ROWS && vol % 16 == 0 && (long)N * (nconf + 1) < (1L << 31) && 2 * vol < (1L << 31) &&
         (long)N * nconf >= (long)((N + 7) / 8 * 8);
}

// G (nconf x N x N complex FP64, every entry) of FP32 orbitals psi.
nrcps_status gram_tc(nrcps_context* ctx, const void* psi, int N, long vol, int nconf, double* G) {
  if (nconf == 0) return NRCPS_OK;
  static bool attr_set[16] = {false};
  if (!attr_set[ctx->device & 15]) {
    NRCPS_TRY(check_cuda(ctx,
                         cudaFuncSetAttribute(gtc::gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)gtc::SMEM),
                         "gram_tc: smem attribute"));
    attr_set[ctx->device & 15] = true;
  }
  const long K = 2 * vol;
  const int nr = (N + 7) / 8 * 8;
  CUtensorMap map;
  if (!make_fp32_map_sw128(&map, psi, (long)nconf * N, K, nr))
    return set_error(ctx, NRCPS_ERR_CUDA, "gram_tc: tensor map of psi");
  gtc::Args a;
  a.nconf = nconf;
  a.N = N;
  a.nr = nr;
  a.nkb = (int)(K / gtc::BK);
  a.nch = (a.nkb + gtc::CHUNK - 1) / gtc::CHUNK;
  a.ntiles = (nconf + 1) / 2;
  a.G = G;
  a.err = ctx->dev_err;
  const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
  const int grid = a.ntiles < sms ? a.ntiles : sms;
  gtc::gram_tc_kernel<<<grid, gtc::THREADS, gtc::SMEM, ctx->stream>>>(map, a);
  ctx->launches++;
  return check_launch(ctx, "gram_tc_kernel");
}

}  // namespace nrcps

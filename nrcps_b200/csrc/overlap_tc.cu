// overlap_tc.cu -- the Slater overlap S = Psi_src^H Psi(tau) on the tcgen05
// tensor cores (FP32 orbitals; the FP64 mode keeps the CUDA-core kernel of
// measure.cu).
//
// S[c][s][t] = sum_p conj(src_s(p)) psi_{c,t}(p)   (OneBody::Project,
// src/one_body/noarch/one_body_project.C:14-27, into SlaterDet's S[t + N s],
// src/slater_det/slater_det.C:33-37) is one real GEMM D = A B^T with
//   k = 2p + j over the interleaved (re, im) floats of an orbital (K = 2V),
//   n = c * nt + t: B[n][k] is psi exactly as it lies in HBM (K-major),
//   m < ns:       A[m][2p] = Re src_m, A[m][2p+1] = Im src_m     -> Re S,
//   ns <= m < 2ns: A[m][2p] = -Im src_s, A[m][2p+1] = Re src_s   -> Im S.
// Precision: every operand is split into TF32 hi + lo (x = hi + lo to ~2^-22)
// and the four products are formed by ONE M=128, N=256, K=8 MMA per k-step:
// the A tile stacks [A_hi; A_lo] (rows 0-63, 64-127) and the B tile stacks
// [B_hi; B_lo] (rows 0-127, 128-255), so the FP32 accumulator holds A_x B_y^T
// in its four quadrants (the drain adds hi hi + hi lo in FP32 and lo hi;
// lo lo, 2^-44 of a product, is dropped).  The tensor core accumulates in
// FP32 for 256 floats of K only (a chunk); each chunk's accumulator is
// drained into FP64 sums in shared memory while the next chunk accumulates
// in the second TMEM buffer, so the result carries FP64 accumulation across K.
//
// One CTA per (128 orbitals, K range); 10 warps:
//   warp 0      TMA producer: the raw FP32 psi tile (128 x 32 floats, into the
//               B_hi half of the operand tile) and the A hi / lo tiles
//               (64 x 32 each), 128-byte swizzle, 3 stages;
//   warp 1      TMEM owner (2 x 256 columns) and MMA issuer (one thread);
//   warps 2-5   split the raw psi tile in place into its hi / lo halves
//               (the swizzle is position-preserving, so the split is
//               elementwise);
//   warps 6-9   drain every chunk (tcgen05.ld of the accumulator, quadrant
//               sums in FP64 shared memory) and write the results
//               (atomically added when K is split over CTAs).
// Every mbarrier wait is bounded; a timeout sets the context's error flag
// and all roles leave their loops, wait for their own copies and MMAs in
// flight (bounded), free the TMEM and return.
#include <cuda.h>

#include "common.cuh"

namespace nrcps {
namespace tc {

constexpr int BN = 128;                        // orbitals (n) per tile
constexpr int BN2 = 2 * BN;                    // MMA N: [B_hi; B_lo] rows = accumulator columns per buffer
constexpr int BK = 32;                         // floats of K per stage: one 128-byte swizzle row
constexpr int CHUNK = 8;                       // k-blocks (256 floats of K) per FP32 accumulation in TMEM
constexpr uint32_t RAW_BYTES = BN * BK * 4;    // 16 KB: raw psi tile
constexpr uint32_t BP_BYTES = 2 * RAW_BYTES;   // 32 KB: [B_hi; B_lo], 256 rows
constexpr uint32_t AH_BYTES = 64 * BK * 4;     // 8 KB: one A half (64 rows)
constexpr uint32_t A_BYTES = 2 * AH_BYTES;     // 16 KB: [A_hi; A_lo], 128 rows
constexpr uint32_t STAGE_BYTES = A_BYTES + BP_BYTES;  // 48 KB, 1024-aligned pieces
constexpr uint32_t TX_BYTES = RAW_BYTES + A_BYTES;
constexpr int ACC_LD = BN + 1;                 // padded row: lane i's row starts 2 banks after lane i-1's
// FP64 running sums of `rows` result rows (2 ns of them are used)
constexpr uint32_t acc_bytes(int rows) { return ((rows * ACC_LD * 8 + 1023) / 1024) * 1024; }
constexpr int THREADS = 320;
constexpr uint32_t TMEM_COLS = 2 * BN2;        // two accumulator buffers
// STG stages and ACCR FP64 result rows: 3 and 64 in general; 4 and 32 when
// 2 ns <= 32 (the smaller sum buffer leaves room for one more stage in flight)
constexpr size_t smem_bytes(int stg, int accr) {
  return (size_t)stg * STAGE_BYTES + acc_bytes(accr) + 1024 /* alignment */ + 256 /* barriers */;
}
constexpr int MAX_NS_BLOCK = 32;               // 2 ns <= 64 accumulator rows per half

// instruction descriptor: D F32, A/B TF32, both K-major, N = 256, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (((uint32_t)BN2 >> 3) << 17) | ((128u >> 4) << 24);

struct Args {
  int n_rows;        // nconf * nt
  int nt;
  int ns_total;      // sources of the whole S (row stride of S is ns_total)
  int s_base;        // first source of this launch
  int ns;            // sources of this launch (<= 32)
  int kb_total;      // K / BK
  int kb_per_split;
  int atomic_out;    // 1: atomicAdd into S (K split over CTAs)
  double* S;
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

// Bounded wait that also gives up once another role has aborted.
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag, int* err) {
  for (int i = 0; i < (1 << 22); ++i) {
    if (bar_try(b, parity)) return true;
    if ((i & 255) == 255 && *abort_flag) return false;
  }
  *abort_flag = 1;
  if (err) atomicExch(err, 1);
  return false;
}
// Bounded wait used on the way out (ignores the abort flag).
__device__ __forceinline__ void bar_drain(uint64_t* b, uint32_t parity, int* err) {
  for (int i = 0; i < (1 << 22); ++i)
    if (bar_try(b, parity)) return;
  if (err) atomicExch(err, 1);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          su32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(su32(bar))
      : "memory");
}

// K-major operand tile with the 128-byte swizzle: 8-row atoms of 1024 bytes
// (stride byte offset 1024), leading byte offset unused (1), version 1.
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

// TF32 rounding of a finite float's bit pattern, to nearest with ties away
// from zero (as cvt.rna.tf32.f32): two integer operations.
__device__ __forceinline__ uint32_t tf32_round_bits(uint32_t b) { return (b + 0x1000u) & 0xFFFFE000u; }

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
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

template <int STAGES, int ACCR>
__global__ void __launch_bounds__(THREADS, 1)
    overlap_tc_kernel(const __grid_constant__ CUtensorMap map_psi, const __grid_constant__ CUtensorMap map_ahi,
                      const __grid_constant__ CUtensorMap map_alo, Args g) {
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte aligned stage area (the swizzle atoms repeat every 1024 bytes)
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t ACC_BYTES = acc_bytes(ACCR);
  double* acc = reinterpret_cast<double*>(base + (size_t)STAGES * STAGE_BYTES);  // [ACCR][ACC_LD] FP64 sums
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + (size_t)STAGES * STAGE_BYTES + ACC_BYTES);
  uint64_t* full = bars;                  // TMA landed (raw psi + A)
  uint64_t* conv = bars + STAGES;         // operand tile split (4 converter warps)
  uint64_t* empty = bars + 2 * STAGES;    // MMAs of the stage completed
  uint64_t* tfull = bars + 3 * STAGES;    // [2] MMAs of a chunk completed in TMEM buffer b
  uint64_t* tempty = tfull + 2;           // [2] TMEM buffer b drained (4 warps)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  volatile int* last_commit = abort_flag + 1;  // last chunk whose TMEM-full commit was issued

  auto stage_a = [&](int s) { return base + (size_t)s * STAGE_BYTES; };
  auto stage_b = [&](int s) { return base + (size_t)s * STAGE_BYTES + A_BYTES; };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x, split = blockIdx.y;
  const int n0 = tile * BN;
  const int kb0 = split * g.kb_per_split;
  int kb1 = kb0 + g.kb_per_split;
  if (kb1 > g.kb_total) kb1 = g.kb_total;
  const int nk = kb1 > kb0 ? kb1 - kb0 : 0;
  const int nchunks = (nk + CHUNK - 1) / CHUNK;

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
  for (int i = threadIdx.x; i < ACCR * ACC_LD; i += THREADS) acc[i] = 0.0;
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

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int issued = 0;
      for (int i = 0; i < nk; ++i) {
        const int s = i % STAGES;
        if (i >= STAGES && !bar_wait(empty + s, (uint32_t)((i / STAGES) - 1) & 1u, abort_flag, g.err)) break;
        bar_expect_tx(full + s, TX_BYTES);
        const int kx = (kb0 + i) * BK;
        tma_load_2d(stage_a(s), &map_ahi, kx, 0, full + s);
        tma_load_2d(stage_a(s) + AH_BYTES, &map_alo, kx, 0, full + s);
        tma_load_2d(stage_b(s), &map_psi, kx, n0, full + s);  // raw psi lands in the B_hi half
        ++issued;
      }
      // copies still in flight land before the CTA may leave
      for (int i = issued - STAGES < 0 ? 0 : issued - STAGES; i < issued; ++i)
        bar_drain(full + (i % STAGES), (uint32_t)(i / STAGES) & 1u, g.err);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      for (int j = 0; j < nchunks; ++j) {
        const int b = j & 1;
        if (j >= 2 && !bar_wait(tempty + b, (uint32_t)((j >> 1) - 1) & 1u, abort_flag, g.err)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(b * BN2);
        bool stop = false;
        const int i1 = (j + 1) * CHUNK < nk ? (j + 1) * CHUNK : nk;
        for (int i = j * CHUNK; i < i1; ++i) {
          const int s = i % STAGES;
          if (!bar_wait(conv + s, (uint32_t)(i / STAGES) & 1u, abort_flag, g.err)) {
            stop = true;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint64_t ad = smem_desc(stage_a(s)), bd = smem_desc(stage_b(s));
#pragma unroll
          for (int k = 0; k < BK / 8; ++k)  // K = 8 TF32 = 32 bytes per MMA: advance the start address
            mma_tf32(d, ad + (uint64_t)(2 * k), bd + (uint64_t)(2 * k), (i > j * CHUNK || k > 0) ? 1u : 0u);
          mma_commit(empty + s);
        }
        mma_commit(tfull + b);  // completes once every MMA issued so far has
        *last_commit = j;
        if (stop) break;
      }
    }
  } else if (warp < 6) {
    // ------------------------------------------------------------ converters
    // In place: the raw tile becomes B_hi = x rounded to TF32 (nearest, ties
    // away: add half a TF32 ulp to the magnitude bits, clear the 13 low
    // mantissa bits) and B_lo = x - B_hi (exact in FP32), itself rounded to
    // TF32 the same way, so the tensor core reads exactly hi and lo and
    // hi + lo carries x to ~2^-22.
    const int ct = threadIdx.x - 64;  // 0..127
    bool ok = true;
    for (int i = 0; i < nk && ok; ++i) {
      const int s = i % STAGES;
      if (!bar_wait(full + s, (uint32_t)(i / STAGES) & 1u, abort_flag, g.err)) ok = false;
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      uint4* bp = reinterpret_cast<uint4*>(stage_b(s));
#pragma unroll
      for (int r = 0; r < (int)(RAW_BYTES / 16 / 128); ++r) {
        const int e = ct + 128 * r;
        const uint4 x = bp[e];
        uint4 hi, lo;
        hi.x = tf32_round_bits(x.x);
        hi.y = tf32_round_bits(x.y);
        hi.z = tf32_round_bits(x.z);
        hi.w = tf32_round_bits(x.w);
        lo.x = tf32_round_bits(__float_as_uint(__uint_as_float(x.x) - __uint_as_float(hi.x)));
        lo.y = tf32_round_bits(__float_as_uint(__uint_as_float(x.y) - __uint_as_float(hi.y)));
        lo.z = tf32_round_bits(__float_as_uint(__uint_as_float(x.z) - __uint_as_float(hi.z)));
        lo.w = tf32_round_bits(__float_as_uint(__uint_as_float(x.w) - __uint_as_float(hi.w)));
        bp[e] = hi;
        bp[e + RAW_BYTES / 16] = lo;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor-core reads
      __syncwarp();
      if (lane == 0) bar_arrive(conv + s);
    }
  } else {
    // ------------------------------------------------------ drains + output
    const int et = threadIdx.x - 192;  // 0..127
    const int q = warp & 3;            // TMEM lane quarter this warp may access
    const int row = 32 * q + lane;     // accumulator row (M)
    // tcgen05.ld is warp-collective: `live` is warp-uniform; rows >= 2 ns of
    // a live quarter load and discard
    const bool live = 32 * (q & 1) < 2 * g.ns;
    bool ok = true;
    // Every drain warp runs the same sequence of named barriers on every
    // path; after a failed wait (ok false, warp-uniform) it only skips work.
    for (int j = 0; j < nchunks; ++j) {
      const int b = j & 1;
      if (ok && !bar_wait(tfull + b, (uint32_t)(j >> 1) & 1u, abort_flag, g.err)) ok = false;
      ok = __all_sync(0xffffffffu, ok);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // rows 64..127 (A_lo) add first, rows 0..63 (A_hi) after the barrier
      for (int phase = 0; phase < 2; ++phase) {
        if (ok && live && (q >= 2) == (phase == 0)) {
          const uint32_t t0 = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * BN2);
          double* arow = acc + (size_t)(row & 63) * ACC_LD;
#pragma unroll 1
          for (int c0 = 0; c0 < BN; c0 += 32) {
            float u[32];
            tmem_ld32(t0 + (uint32_t)c0, u);
            if (q < 2) {
              // A_hi rows: hi*hi + hi*lo, added in FP32 (one rounding, below
              // the error of the chunk's own FP32 accumulation), one conversion
              float v[32];
              tmem_ld32(t0 + (uint32_t)(c0 + BN), v);
#pragma unroll
              for (int k = 0; k < 32; ++k) arow[c0 + k] += (double)(u[k] + v[k]);
            } else {
              // A_lo rows: lo*hi; lo*lo (2^-44 of the product) is dropped
#pragma unroll
              for (int k = 0; k < 32; ++k) arow[c0 + k] += (double)u[k];
            }
          }
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) bar_arrive(tempty + b);
    }
    // ------------------------------------------------------------ output
    if (ok) {
      for (int e = et; e < 2 * g.ns * BN; e += 128) {
        const int m = e / BN, col = e - m * BN;
        const int n = n0 + col;
        if (n >= g.n_rows) continue;
        const bool im = m >= g.ns;
        const int s = g.s_base + (im ? m - g.ns : m);
        const int c = n / g.nt, t = n - c * g.nt;
        double* o = g.S + (((long)c * g.ns_total + s) * g.nt + t) * 2 + (im ? 1 : 0);
        const double val = acc[(size_t)m * ACC_LD + col];
        if (g.atomic_out) atomicAdd(o, val);
        else *o = val;
      }
    }
  }
  // ---------------------------------------------------------------- teardown
  __syncthreads();
  if (warp == 1) {
    // every MMA this CTA issued is covered by the last TMEM-full commit; wait
    // for it before the TMEM goes back (the drains may have given up early)
    const int last = *last_commit;
    if (last >= 0) bar_drain(tfull + (last & 1), (uint32_t)(last >> 1) & 1u, g.err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// A operand rows for sources [s_base, s_base + ns): hi and lo TF32 halves,
// each 2 ns rows of K = 2V floats (row m < ns: Re part, m >= ns: Im part).
__global__ void split_sources_kernel(const double* __restrict__ src, int s_base, int ns, long vol, float* __restrict__ ahi,
                                     float* __restrict__ alo) {
  const long K = 2 * vol;
  const long total = 2L * ns * K;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int m = (int)(e / K);
    const long k = e - (long)m * K;
    const long p = k >> 1;
    const int j = (int)(k & 1);
    const int s = s_base + (m < ns ? m : m - ns);
    const double2 a = reinterpret_cast<const double2*>(src)[(long)s * vol + p];
    double v;
    if (m < ns) v = j ? a.y : a.x;   // Re S: re*re + im*im
    else v = j ? a.x : -a.y;         // Im S: re*im - im*re
    const float hi = __uint_as_float(tf32_rna((float)v));
    const float lo = __uint_as_float(tf32_rna((float)(v - (double)hi)));
    ahi[e] = hi;
    alo[e] = lo;
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

// 2-D FP32 map over rows x K floats (row stride K * 4 bytes), box 32 x box_rows.
static bool make_map(CUtensorMap* m, const void* ptr, long rows, long K, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)K * 4};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace tc

// 2-D FP32 tensor map (rows x K floats, 128-byte swizzle, box 32 floats x
// box_rows) for the other tcgen05 kernels of the library; false when the
// driver's encoder is unavailable or rejects the shape.
bool make_fp32_map_sw128(CUtensorMap* m, const void* ptr, long rows, long K, int box_rows) {
  return tc::make_map(m, ptr, rows, K, box_rows);
}

// Shapes the tensor-core path takes: FP32 orbitals, K = 2V a multiple of 32
// floats, rows addressable as int.
bool overlap_tc_supported(long vol, int ns, int nt, int nconf) {
  return vol % 16 == 0 && ns > 0 && nt > 0 && (long)nt * nconf < (1L << 30) && 2 * vol < (1L << 31) &&
         tc::encode_fn() != nullptr;
}

size_t overlap_tc_split_bytes(int ns, long vol) { return sizeof(float) * 2 * (size_t)(2 * ns) * (size_t)(2 * vol); }

// Builds the hi / lo A operands of every source block into `split`
// (overlap_tc_split_bytes(ns, vol) bytes): block b (sources 32 b ...) at
// float offset 2 * 2 * 32 b * 2V.
nrcps_status overlap_tc_prepare(nrcps_context* ctx, const double* src, int ns, long vol, float* split) {
  const long K = 2 * vol;
  for (int sb = 0; sb < ns; sb += tc::MAX_NS_BLOCK) {
    const int nsb = ns - sb < tc::MAX_NS_BLOCK ? ns - sb : tc::MAX_NS_BLOCK;
    float* hi = split + 2L * (2L * sb) * K;
    float* lo = hi + (2L * nsb) * K;
    tc::split_sources_kernel<<<grid_for(2L * nsb * K, 256, (long)ctx->sm_count * 16), 256, 0, ctx->stream>>>(
        src, sb, nsb, vol, hi, lo);
    ctx->launches++;
    NRCPS_TRY(check_launch(ctx, "split_sources_kernel"));
  }
  return NRCPS_OK;
}

// S (nconf x ns x nt complex FP64) from FP32 psi and the prepared split sources.
nrcps_status overlap_tc(nrcps_context* ctx, const float* split, int ns, const void* psi, int nt, int nconf, long vol,
                        double* S) {
  const long K = 2 * vol;
  const int n_rows = nt * nconf;
  if (n_rows == 0 || ns == 0) return NRCPS_OK;
  static bool attr_set[16] = {false};
  if (!attr_set[ctx->device & 15]) {
    NRCPS_TRY(check_cuda(ctx,
                         cudaFuncSetAttribute(tc::overlap_tc_kernel<3, 64>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::smem_bytes(3, 64)),
                         "overlap_tc: smem attribute"));
    NRCPS_TRY(check_cuda(ctx,
                         cudaFuncSetAttribute(tc::overlap_tc_kernel<4, 32>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::smem_bytes(4, 32)),
                         "overlap_tc: smem attribute"));
    attr_set[ctx->device & 15] = true;
  }
  const int tiles = (n_rows + tc::BN - 1) / tc::BN;
  const int kb_total = (int)(K / tc::BK);
  // Split K over CTAs so that the grid fills its last wave (one CTA per SM):
  // the smallest split count whose waves are at least 90 % full, else the
  // fullest of 1..8; at least two waves when the tiles alone are fewer.
  int splits = 1;
  {
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    const int min_s = tiles < 2 * sms ? (2 * sms + tiles - 1) / tiles : 1;
    double best = -1.0;
    for (int sp = min_s; sp <= min_s + 7; ++sp) {
      const long ctas = (long)tiles * sp;
      const long waves = (ctas + sms - 1) / sms;
      const double eff = (double)ctas / (double)(waves * sms);
      if (eff >= 0.9) {
        splits = sp;
        break;
      }
      if (eff > best) {
        best = eff;
        splits = sp;
      }
    }
  }
  if (splits > kb_total / 8) splits = kb_total / 8 > 0 ? kb_total / 8 : 1;
  if (splits < 1) splits = 1;
  const int per = (kb_total + splits - 1) / splits;
  splits = (kb_total + per - 1) / per;
  CUtensorMap mpsi;
  if (!tc::make_map(&mpsi, psi, n_rows, K, tc::BN))
    return set_error(ctx, NRCPS_ERR_CUDA, "overlap_tc: tensor map of psi");
  if (splits > 1)
    NRCPS_TRY(check_cuda(ctx, cudaMemsetAsync(S, 0, sizeof(double) * 2 * (size_t)nconf * ns * nt, ctx->stream),
                         "overlap_tc: memset"));
  for (int sb = 0; sb < ns; sb += tc::MAX_NS_BLOCK) {
    const int nsb = ns - sb < tc::MAX_NS_BLOCK ? ns - sb : tc::MAX_NS_BLOCK;
    const float* hi = split + 2L * (2L * sb) * K;
    const float* lo = hi + (2L * nsb) * K;
    CUtensorMap mhi, mlo;
    if (!tc::make_map(&mhi, hi, 2 * nsb, K, 64) || !tc::make_map(&mlo, lo, 2 * nsb, K, 64))
      return set_error(ctx, NRCPS_ERR_CUDA, "overlap_tc: tensor map of the sources");
    tc::Args a;
    a.n_rows = n_rows;
    a.nt = nt;
    a.ns_total = ns;
    a.s_base = sb;
    a.ns = nsb;
    a.kb_total = kb_total;
    a.kb_per_split = per;
    a.atomic_out = splits > 1;
    a.S = S;
    a.err = ctx->dev_err;
    if (2 * nsb <= 32)
      tc::overlap_tc_kernel<4, 32><<<dim3((unsigned)tiles, (unsigned)splits), tc::THREADS, tc::smem_bytes(4, 32),
                                     ctx->stream>>>(mpsi, mhi, mlo, a);
    else
      tc::overlap_tc_kernel<3, 64><<<dim3((unsigned)tiles, (unsigned)splits), tc::THREADS, tc::smem_bytes(3, 64),
                                     ctx->stream>>>(mpsi, mhi, mlo, a);
    ctx->launches++;
    NRCPS_TRY(check_launch(ctx, "overlap_tc_kernel"));
  }
  return NRCPS_OK;
}

}  // namespace nrcps

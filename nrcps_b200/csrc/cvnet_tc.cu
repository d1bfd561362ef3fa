// cvnet_tc.cu -- inference of the control-variate network on the tcgen05
// tensor cores: the three 3x3x3 periodic convolutions, the mean pool and the
// head in ONE kernel per sample, for the 8^3 coarse lattice.
//
// Each convolution is a sum over the 27 taps of shifted GEMMs,
//   Z[s][co] = b[co] + sum_tap sum_ci X[s + d_tap][ci] W_tap[ci][co],
// run as M=128 (sites), N=16 (output channels), K=16 (input channels) BF16
// MMAs with FP32 accumulators in TMEM.  The shift is free: the input lives in
// shared memory as a padded, periodically extended 10 x 10 x 10 grid of
// 16-byte entries (8 channels each, one grid per group of 8 channels), the
// no-swizzle K-major operand layout of the tensor core (a core matrix is 8
// consecutive z entries of one (x, y) row).  Output rows are the 80 padded
// rows (x', y') with x' in 1..8, y' in 0..9 (five M tiles of 16 rows); rows
// with y' = 0 or 9 are computed and discarded.  For a tap (dx, dy, dz) the
// A operand of a tile starts dx rows of 10, dy rows and dz entries away from
// the unshifted one, so every tap reads the same buffer through another
// descriptor.
//
// Per sample: layer 1 streams the input in chunks of 16 channels: the bulk
// copy engine brings each 16 KiB chunk into shared memory two chunks ahead,
// threads transpose it into one of two padded operand buffers while the
// previous chunk's MMAs run; each epilogue reads the accumulators (tcgen05.ld), adds
// the bias, applies tanh, rounds to BF16 and writes every periodic copy of
// the site into the next layer's padded input; layer 3's epilogue sums into
// the mean pool, and the head (tanh hidden layer, linear output) finishes
// the sample.  Same BF16 roundings as the CUDA-core path (weights,
// activations); FP32 accumulation in another order.
//
// One persistent CTA per SM (the weights of all three layers stay in shared
// memory), 8 warps (warp w drains TMEM lanes 32 (w % 4).. for channels
// 8 (w / 4)..); thread 0 issues the bulk copies and the MMAs.  Every mbarrier wait is
// bounded: a timeout sets the error flag, the CTA drains its MMAs (bounded),
// frees its TMEM and returns.
#include <cuda_bf16.h>

#include "common.cuh"

namespace nrcps {
namespace cvtc {

constexpr int G = 8;
constexpr int GS = G * G * G;
constexpr int C = 16;                       // conv channels
constexpr int ENT = 10;                     // padded z entries per row
constexpr int ROWS = 102;                   // 1 guard + 10 x 10 padded (x', y') rows + 1 guard
constexpr int ROW_BYTES = ENT * 16;         // 160
constexpr int GRID_BYTES = ROWS * ROW_BYTES;  // 16320: one group of 8 channels
constexpr int BUF_BYTES = 2 * GRID_BYTES;   // 16 channels: one K step of 16
constexpr int TILES = 5;                    // M tiles of 16 rows
constexpr int WK_BYTES = 512;               // weights of one (tap, K step): 2 K groups x 16 co x 16 B
constexpr int THREADS = 256;             // 8 warps: warp w reads TMEM lanes 32 (w % 4).., channels 8 (w / 4)..
constexpr int STG_BYTES = 16 * GS * 2;      // one raw chunk: 16 channels x 512 sites BF16
constexpr int MAX_CIN = 64;
constexpr int MAX_H = 64;
constexpr int MAX_T = 256;
constexpr uint32_t TMEM_COLS = 128;         // 5 accumulators of 16 columns

// instruction descriptor: D F32, A/B BF16, both K-major, N = 16, M = 128
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

struct Args {
  const __nv_bfloat16* x;  // [B][Cin][512]
  int B, Cin, H, T;
  const __nv_bfloat16* w[3];  // [16][cin][27]
  const float* b[3];          // [16]
  const float* hw;            // [H][16]
  const float* hb;            // [H]
  const float* ow;            // [T][H]
  const float* ob;            // [T]
  float* y;                   // [B][T]
  int* err;
};

__host__ __device__ constexpr size_t smem_bytes(int cin) {
  // weights (all layers) + 2 layer-1 input buffers + 1 activation buffer + pool/head scratch + barriers
  return (size_t)27 * (cin / 16 + 2) * WK_BYTES + 3 * (size_t)BUF_BYTES + 2 * (size_t)STG_BYTES + 16 * 4 +
         MAX_H * 4 + 64;
}

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, int* err) {
  for (int i = 0; i < (1 << 24); ++i)
    if (bar_try(b, parity)) return true;
  if (err) atomicExch(err, 1);
  return false;
}

// no-swizzle K-major operand: core matrices of 8 rows x 16 B; LBO = stride
// between the two core matrices along K, SBO = stride between 8-row groups.
__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// byte offset of padded entry (x', y', z') of one channel group's grid
__device__ __forceinline__ int entry_off(int xp, int yp, int zp) { return (1 + xp * 10 + yp) * ROW_BYTES + zp * 16; }

// Padded coordinates that hold a copy of lattice coordinate v (0..7):
// v + 1 always, 0 when v = 7, 9 when v = 0.
__device__ __forceinline__ int copies(int v, int* out) {
  out[0] = v + 1;
  if (v == 7) {
    out[1] = 0;
    return 2;
  }
  if (v == 0) {
    out[1] = 9;
    return 2;
  }
  return 1;
}

// Issues the 27 x 5 MMAs of one K step of 16 channels in `buf`, weights at `wk`
// (27 blocks of WK_BYTES, `wstride` apart).
__device__ __forceinline__ void issue_layer_step(uint32_t tmem, uint32_t buf, uint32_t wk, uint32_t wstride,
                                                 bool first_step) {
#pragma unroll 1
  for (int tap = 0; tap < 27; ++tap) {
    const int dx = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dz = tap % 3 - 1;
    const uint64_t bdesc = desc(wk + tap * wstride, 256, 128);
#pragma unroll
    for (int j = 0; j < TILES; ++j) {
      // output rows 10 + 16 j .. +15 (storage + 1); the tap shifts by 10 dx + dy rows and dz entries
      const uint32_t a = buf + (uint32_t)((1 + 10 + 16 * j + 10 * dx + dy) * ROW_BYTES + (1 + dz) * 16);
      mma(tmem + 16 * j, desc(a, GRID_BYTES, ROW_BYTES), bdesc, (first_step && tap == 0) ? 0u : 1u);
    }
  }
}

__global__ void __launch_bounds__(THREADS, 1) cv_forward_tc_kernel(Args g) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int nks1 = g.Cin / 16;
  unsigned char* wsm = smem;                                  // [layer][tap][kstep] blocks of WK_BYTES
  unsigned char* buf0 = wsm + (size_t)27 * (nks1 + 2) * WK_BYTES;
  unsigned char* buf1 = buf0 + BUF_BYTES;
  unsigned char* act = buf1 + BUF_BYTES;                      // layer-2 input (A1)
  unsigned char* stg0 = act + BUF_BYTES;                      // raw 16-channel chunks (bulk-copy landing zones)
  unsigned char* stg1 = stg0 + STG_BYTES;
  float* pool = reinterpret_cast<float*>(stg1 + STG_BYTES);   // [16]
  float* hid = pool + 16;                                     // [MAX_H]
  // bars[0], [1]: MMAs of the layer-1 buffers; [2]: MMAs of layers 2, 3; [3], [4]: staged chunks landed
  uint64_t* bars = reinterpret_cast<uint64_t*>(hid + MAX_H);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 5);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quad = warp & 3, half = warp >> 2;  // TMEM lanes 32 quad.., channels 8 half..

  // ---- one-time setup: weights in the operand layout, zeroed guard rows, barriers, TMEM
  const int wl_off[3] = {0, 27 * nks1 * WK_BYTES, 27 * (nks1 + 1) * WK_BYTES};
  for (int l = 0; l < 3; ++l) {
    const int cin = l == 0 ? g.Cin : C, nks = cin / 16;
    // entry (tap, ks, kg, co): 8 channels ci = 16 ks + 8 kg + 0..7 of W[co][ci][tap]
    for (int e = tid; e < 27 * nks * 2 * C; e += THREADS) {
      const int co = e % C, kg = (e / C) % 2, ks = (e / (2 * C)) % nks, tap = e / (2 * C * nks);
      uint32_t pk[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int ci = 16 * ks + 8 * kg + 2 * i;
        const unsigned short lo = __bfloat16_as_ushort(g.w[l][((size_t)co * cin + ci) * 27 + tap]);
        const unsigned short hi = __bfloat16_as_ushort(g.w[l][((size_t)co * cin + ci + 1) * 27 + tap]);
        pk[i] = (uint32_t)lo | ((uint32_t)hi << 16);
      }
      // block (tap, ks) at (tap * nks + ks) * WK_BYTES; K group kg at 256 kg; row co at 16 co
      *reinterpret_cast<uint4*>(wsm + wl_off[l] + (size_t)(tap * nks + ks) * WK_BYTES + 256 * kg + 16 * co) =
          make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  }
  for (int e = tid; e < 3 * 2 * 2 * ENT; e += THREADS) {  // guard rows 0 and 101 of every grid
    const int i = e % ENT, r = (e / ENT) % 2, gidx = e / (2 * ENT);
    unsigned char* grid = (gidx < 2 ? buf0 : gidx < 4 ? buf1 : act) + (gidx % 2) * GRID_BYTES;
    *reinterpret_cast<uint4*>(grid + (r ? 101 : 0) * ROW_BYTES + i * 16) = make_uint4(0, 0, 0, 0);
  }
  if (tid == 0) {
    for (int i = 0; i < 5; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bars + i)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t wbase = su32(wsm);
  uint32_t ph[5] = {0, 0, 0, 0, 0};   // parities of the barriers
  int pending[5] = {0, 0, 0, 0, 0};   // arrivals expected on bars[i] and not yet waited for
  bool ok = true;
  // waits for the pending phase of bars[i]; the outcome is made block-uniform
  auto wait_bar = [&](int i) {
    const bool done = bar_wait(bars + i, ph[i], g.err);
    if (done) {
      ph[i] ^= 1u;
      pending[i] = 0;
    }
    return __syncthreads_and(done) != 0;
  };

  // chunk q of this CTA: sample blockIdx.x + (q / nks1) gridDim.x, channels 16 (q % nks1) ..
  const long n_chunks = g.B > blockIdx.x ? ((g.B - 1 - blockIdx.x) / gridDim.x + 1) * nks1 : 0;
  auto chunk_src = [&](long q) {
    const long b = blockIdx.x + (q / nks1) * (long)gridDim.x;
    return reinterpret_cast<const unsigned char*>(g.x) + ((size_t)b * g.Cin + 16 * (q % nks1)) * GS * 2;
  };
  // one thread: bulk copy of chunk q (16 KiB contiguous) into stage q % 2
  auto load_chunk = [&](long q) {
    uint64_t* bar = bars + 3 + (q & 1);
    unsigned char* dst = (q & 1) ? stg1 : stg0;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"((uint32_t)STG_BYTES)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     su32(dst)),
                 "l"(chunk_src(q)), "r"((uint32_t)STG_BYTES), "r"(su32(bar))
                 : "memory");
  };
  if (tid == 0)
    for (long q = 0; q < 2 && q < n_chunks; ++q) load_chunk(q);
  for (long q = 0; q < 2 && q < n_chunks; ++q) pending[3 + q] = 1;

  // staged chunk (16 channels x 512 sites) -> padded operand grid of 2 channel groups
  auto transpose = [&](unsigned char* dst, const unsigned char* src) {
    const unsigned short* xs = reinterpret_cast<const unsigned short*>(src);
    for (int e = tid; e < 2 * 1000; e += THREADS) {
      const int kg = e / 1000, p = e % 1000;
      const int xp = p / 100, yp = (p / 10) % 10, zp = p % 10;
      const int x = (xp + 7) % 8, y = (yp + 7) % 8, z = (zp + 7) % 8;
      const int s = z + G * (y + G * x);
      uint32_t pk[4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        pk[i] = (uint32_t)xs[(8 * kg + 2 * i) * GS + s] | ((uint32_t)xs[(8 * kg + 2 * i + 1) * GS + s] << 16);
      *reinterpret_cast<uint4*>(dst + kg * GRID_BYTES + entry_off(xp, yp, zp)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  };

  // accumulators of this thread's row and channel half of tile j -> bias, tanh, BF16
  auto activations = [&](int j, const float* bias, float* a) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tmem_ld8(tmem + ((uint32_t)(32 * quad) << 16) + 16 * j + 8 * half, a);
#pragma unroll
    for (int co = 0; co < 8; ++co) a[co] = __bfloat162float(__float2bfloat16(tanhf(a[co] + bias[co])));
  };

  long q = 0;  // next chunk
  for (long b = blockIdx.x; b < g.B && ok; b += gridDim.x) {
    // ---------------- layer 1: K steps of 16 channels through two operand buffers
    for (int ks = 0; ks < nks1 && ok; ++ks, ++q) {
      const int bi = ks & 1;
      unsigned char* buf = bi ? buf1 : buf0;
      if (pending[bi]) {  // the MMAs that read this buffer two steps ago
        ok = wait_bar(bi);
        if (!ok) break;
      }
      ok = wait_bar(3 + (int)(q & 1));  // chunk q landed
      if (!ok) break;
      transpose(buf, (q & 1) ? stg1 : stg0);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        if (q + 2 < n_chunks) load_chunk(q + 2);  // the stage is free again
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        issue_layer_step(tmem, su32(buf), wbase + wl_off[0] + ks * WK_BYTES, nks1 * WK_BYTES, ks == 0);
        commit(bars + bi);
      }
      if (q + 2 < n_chunks) pending[3 + (int)(q & 1)] = 1;
      pending[bi] = 1;
    }
    if (!ok) break;
    for (int bi = 0; bi < 2 && ok; ++bi)
      if (pending[bi]) ok = wait_bar(bi);
    if (!ok) break;
    // ---------------- layers 2 and 3
    for (int layer = 1; layer < 3; ++layer) {
      // epilogue of the previous layer into the next input: A1 -> act, A2 -> buf0
      unsigned char* dst = layer == 1 ? act : buf0;
      float bias[8];
#pragma unroll
      for (int co = 0; co < 8; ++co) bias[co] = __ldg(g.b[layer - 1] + 8 * half + co);
      for (int j = 0; j < TILES; ++j) {
        float a[8];
        activations(j, bias, a);
        const int r = 10 + 16 * j + 4 * quad + lane / 8, z = lane % 8;  // row m = 32 quad + lane
        const int xp = r / 10, yp = r % 10;
        if (yp >= 1 && yp <= 8) {
          uint32_t pk[4];
#pragma unroll
          for (int i = 0; i < 4; ++i)
            pk[i] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16(a[2 * i])) |
                    ((uint32_t)__bfloat16_as_ushort(__float2bfloat16(a[2 * i + 1])) << 16);
          int cx[2], cy[2], cz[2];
          const int nx = copies(xp - 1, cx), ny = copies(yp - 1, cy), nz = copies(z, cz);
          for (int ix = 0; ix < nx; ++ix)
            for (int iy = 0; iy < ny; ++iy)
              for (int iz = 0; iz < nz; ++iz)
                *reinterpret_cast<uint4*>(dst + half * GRID_BYTES + entry_off(cx[ix], cy[iy], cz[iz])) =
                    make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        issue_layer_step(tmem, su32(dst), wbase + wl_off[layer], WK_BYTES, true);
        commit(bars + 2);
      }
      pending[2] = 1;
      ok = wait_bar(2);
      if (!ok) break;
    }
    if (!ok) break;
    // ---------------- layer 3 epilogue: mean pool, head
    if (tid < 16) pool[tid] = 0.0f;
    __syncthreads();
    {
      float bias[8], sum[8];
#pragma unroll
      for (int co = 0; co < 8; ++co) {
        bias[co] = __ldg(g.b[2] + 8 * half + co);
        sum[co] = 0.0f;
      }
      for (int j = 0; j < TILES; ++j) {
        float a[8];
        activations(j, bias, a);
        const int r = 10 + 16 * j + 4 * quad + lane / 8;
        const int yp = r % 10;
        const bool valid = yp >= 1 && yp <= 8;
#pragma unroll
        for (int co = 0; co < 8; ++co) sum[co] += valid ? a[co] : 0.0f;
      }
#pragma unroll
      for (int co = 0; co < 8; ++co) {
        float v = sum[co];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) atomicAdd(pool + 8 * half + co, v);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    for (int jh = tid; jh < g.H; jh += THREADS) {
      float s = __ldg(g.hb + jh);
      for (int c = 0; c < C; ++c) s = fmaf(__ldg(g.hw + jh * C + c), pool[c] * (1.0f / GS), s);
      hid[jh] = tanhf(s);
    }
    __syncthreads();
    for (int t = tid; t < g.T; t += THREADS) {
      float s = __ldg(g.ob + t);
      for (int jh = 0; jh < g.H; ++jh) s = fmaf(__ldg(g.ow + t * g.H + jh), hid[jh], s);
      g.y[(size_t)b * g.T + t] = s;
    }
    __syncthreads();
  }
  // ---- leave: no MMA or bulk copy may still be in flight (bounded drains), then free TMEM
  for (int i = 0; i < 5; ++i)
    if (pending[i]) bar_wait(bars + i, ph[i], g.err);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace cvtc
}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_cv_forward_tc(nrcps_context* ctx, const void* dev_x, int Cin, int G, int B,
                                            const void* const* dev_W, const float* const* dev_bias,
                                            const float* dev_hw, const float* dev_hb, int H, const float* dev_ow,
                                            const float* dev_ob, int T, float* dev_y) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, G == cvtc::G && Cin > 0 && Cin % 16 == 0 && Cin <= cvtc::MAX_CIN,
                "nrcps_cv_forward_tc: needs G = 8 and Cin a multiple of 16 up to 64");
  NRCPS_REQUIRE(ctx, H > 0 && H <= cvtc::MAX_H && T > 0 && T <= cvtc::MAX_T && B >= 0 && ((dev_x && dev_y) || B == 0) &&
                         dev_W && dev_bias && dev_hw && dev_hb && dev_ow && dev_ob,
                "nrcps_cv_forward_tc: bad arguments");
  NRCPS_REQUIRE(ctx, reinterpret_cast<uintptr_t>(dev_x) % 16 == 0,
                "nrcps_cv_forward_tc: the features must start on a 16-byte boundary (bulk copies)");
  if (B == 0) return NRCPS_OK;
  cvtc::Args a{};
  a.x = reinterpret_cast<const __nv_bfloat16*>(dev_x);
  a.B = B;
  a.Cin = Cin;
  a.H = H;
  a.T = T;
  for (int l = 0; l < 3; ++l) {
    a.w[l] = reinterpret_cast<const __nv_bfloat16*>(dev_W[l]);
    a.b[l] = dev_bias[l];
  }
  a.hw = dev_hw;
  a.hb = dev_hb;
  a.ow = dev_ow;
  a.ob = dev_ob;
  a.y = dev_y;
  a.err = ctx->dev_err;
  const size_t sh = cvtc::smem_bytes(Cin);
  NRCPS_TRY(check_cuda(ctx, cudaFuncSetAttribute(cvtc::cv_forward_tc_kernel,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh),
                       "cv_forward_tc attribute"));
  const int grid = B < ctx->sm_count ? B : ctx->sm_count;
  cvtc::cv_forward_tc_kernel<<<grid, cvtc::THREADS, sh, ctx->stream>>>(a);
  ctx->launches++;
  return check_launch(ctx, "cv_forward_tc_kernel");
}

// rng.cu -- the reference's uniform-deviate stream and auxiliary-field draws
// on the GPU (UniformDeviate/Random/Lattice::Refresh replacements).
//
// ranlxs/ranlxd: the stream is cut into blocks of 96 (ranlxs) or 48
// (ranlxd) outputs, one per generator Update (src/random/ranlxs.C:112-168,
// src/random/ranlxd.C:115-170).  Groups of four threads (one per SWB lane)
// each own a run of blocks; a group jumps straight to its first block with
// the exact LCG skip-ahead of rng_math.cuh, then runs the SWB recurrence in
// registers and emits its outputs in the reference's order (oldest word
// first; per word the low digits of lanes 0..3, then the high digits for
// ranlxs; one 48-bit word per lane for ranlxd).
//
// ran2 (src/random/ran2.C) carries a Bays-Durham shuffle table whose state
// depends on the whole history, so it cannot be split; it runs on the host.
#include <cstring>
#include <vector>

#include "common.cuh"
#include "rng_math.cuh"

namespace nrcps {
namespace rng {

// ------------------------------------------------------------ host side
struct RanluxState {  // reference layout (src/random/ranlxs.C:193-213)
  int num[96];
  int carry[4];
  int pr, ir, jr, is, is_old;
  bool dbl;
};

static int pr_of(int kind) {
  switch (kind) {
    case NRCPS_RANLXS0: return 109;
    case NRCPS_RANLXS1: return 202;
    case NRCPS_RANLXS2: return 397;
    case NRCPS_RANLXD1: return 202;
    case NRCPS_RANLXD2: return 397;
    default: return 0;
  }
}
static bool is_ranlux(int kind) { return pr_of(kind) != 0; }
static bool is_dbl(int kind) { return kind == NRCPS_RANLXD1 || kind == NRCPS_RANLXD2; }
static int block_len(int kind) { return is_dbl(kind) ? 48 : 96; }

// Ranlxs::Init / Ranlxd::Init (src/random/ranlxs.C:60-110, ranlxd.C:61-113).
static bool ranlux_seed(RanluxState& s, int kind, long seed) {
  if (seed <= 0 || seed > 2147483647L) return false;
  s.dbl = is_dbl(kind);
  s.pr = pr_of(kind);
  int xbit[31];
  long i = seed;
  for (int k = 0; k < 31; ++k) {
    xbit[k] = (int)(i % 2);
    i /= 2;
  }
  int ibit = 0, jbit = 18;
  for (int lane = 0; lane < 4; ++lane)
    for (int k = 0; k < 24; ++k) {
      int ix = 0;
      for (int l = 0; l < 24; ++l) {
        ix = 2 * ix + xbit[ibit];
        xbit[ibit] = (xbit[ibit] + xbit[jbit]) % 2;
        ibit = (ibit + 1) % 31;
        jbit = (jbit + 1) % 31;
      }
      bool flip = s.dbl ? ((k % 4) != lane) : ((k % 4) == lane);
      s.num[4 * k + lane] = flip ? 16777215 - ix : ix;
    }
  for (int l = 0; l < 4; ++l) s.carry[l] = 0;
  s.ir = 0;
  s.jr = 7;
  s.is = s.dbl ? 91 : 95;
  s.is_old = 0;
  return true;
}

static void to_lanes(const RanluxState& s, Lane lanes[4]) {
  for (int l = 0; l < 4; ++l) {
    for (int j = 0; j < 12; ++j) {
      int p = (s.ir + j) % 12;
      lanes[l].words[j] = ((uint64_t)s.num[8 * p + 4 + l] << 24) | (uint64_t)s.num[8 * p + l];
    }
    lanes[l].carry = (uint32_t)s.carry[l];
  }
}

static void from_lanes(RanluxState& s, const Lane lanes[4]) {
  for (int l = 0; l < 4; ++l) {
    for (int j = 0; j < 12; ++j) {
      int p = (s.ir + j) % 12;
      s.num[8 * p + l] = (int)(lanes[l].words[j] & 0xffffff);
      s.num[8 * p + 4 + l] = (int)(lanes[l].words[j] >> 24);
    }
    s.carry[l] = (int)lanes[l].carry;
  }
}

static U576 multiplier() {  // a = b^{-1} mod m = m - (m-1)/b = 2^576 - 2^528 - 2^240 + 2^192 + 1
  U576 a;
  uint64_t m[kLimbs], t[kLimbs];
  modulus(m);
  set_zero(t, kLimbs);
  for (int bit = 192; bit < 528; ++bit) t[bit / 64] |= 1ull << (bit % 64);  // (m-1)/b = 2^528 - 2^192
  sub_n(a.w, m, t, kLimbs);
  return a;
}

static U576 one() {
  U576 r;
  set_zero(r.w, kLimbs);
  r.w[0] = 1;
  return r;
}

// a^e mod m for a 64-bit exponent.
static U576 powmod(U576 base, uint64_t e) {
  U576 r = one();
  while (e) {
    if (e & 1) mulmod(r, r, base);
    mulmod(base, base, base);
    e >>= 1;
  }
  return r;
}

// Number of outputs already consumed from the current block, in [1, P].
static int consumed_in_block(const RanluxState& s) {
  int idx = ((s.is - s.is_old) % 96 + 96) % 96;
  if (!s.dbl) return idx + 1;
  return 4 * (idx / 8) + (idx % 8) + 1;
}

// Advance by n uniforms.
static void ranlux_skip(RanluxState& s, uint64_t n) {
  const int P = s.dbl ? 48 : 96;
  int k = consumed_in_block(s);
  uint64_t rem = (uint64_t)(P - k);
  uint64_t kk;
  if (n <= rem) {
    kk = k + n;
  } else {
    uint64_t np = n - rem;
    uint64_t u = (np + P - 1) / P;
    kk = np - (u - 1) * P;
    // jump u * pr recurrence steps on every lane
    Lane lanes[4];
    to_lanes(s, lanes);
    U576 A = powmod(multiplier(), 1);  // a
    // a^(u*pr): exponentiate in two stages to keep the exponent in 64 bits
    U576 step = powmod(A, (uint64_t)s.pr);
    U576 jump = powmod(step, u);
    for (int l = 0; l < 4; ++l) {
      U576 Y;
      encode(Y, lanes[l]);
      mulmod(Y, Y, jump);
      decode(lanes[l], Y);
    }
    int prm = s.pr % 12;
    s.ir = (int)((s.ir + (u % 12) * prm) % 12);
    s.jr = (s.ir + 7) % 12;
    from_lanes(s, lanes);
    s.is_old = 8 * s.ir;
  }
  // position of output kk (1-based) within the block starting at is_old
  int idx = (int)kk - 1;
  int off = s.dbl ? 8 * (idx / 4) + (idx % 4) : idx;
  s.is = (s.is_old + off) % 96;
}

// ran2 (src/random/ran2.C:42-81).
struct Ran2 {
  long idum, idum2, iy, iv[32];
  void seed(long sd) {
    idum = sd <= 0 ? 1 : sd;
    idum2 = idum;
    for (int j = 32 + 7; j >= 0; --j) {
      long k = idum / 53668L;
      idum = 40014L * (idum - k * 53668L) - k * 12211L;
      if (idum < 0) idum += 2147483563L;
      if (j < 32) iv[j] = idum;
    }
    iy = iv[0];
  }
  double next() {
    long k = idum / 53668L;
    idum = 40014L * (idum - k * 53668L) - k * 12211L;
    if (idum < 0) idum += 2147483563L;
    k = idum2 / 52774L;
    idum2 = 40692L * (idum2 - k * 52774L) - k * 3791L;
    if (idum2 < 0) idum2 += 2147483399L;
    int j = (int)(iy / (1 + (2147483563L - 1) / 32));
    iy = iv[j] - idum2;
    iv[j] = idum;
    if (iy < 1) iy += 2147483563L - 1;
    float temp = (float)((1.0 / 2147483563L) * iy);
    const double rnmx = 1.0 - 1.2e-7;
    if (temp > rnmx) return rnmx;
    return temp;
  }
};

// ------------------------------------------------------------ device side
enum OutKind { OUT_UNIFORM = 0, OUT_Z2_BITS = 1, OUT_FIELD_Z2 = 2, OUT_FIELD_Z3 = 3 };

struct GenArgs {
  U576 y_seed[4];
  Lane lane_seed[4];
  U576 pow_tab[48];  // a^(pr * 2^i)
};

struct OutArgs {
  uint64_t u_lo, u_hi;  // window of uniform indices written
  double* d;
  uint32_t* bits;
};

__device__ __forceinline__ void emit(const OutArgs& o, int kind, uint64_t u, uint64_t digit, int digit_bits) {
  if (u < o.u_lo || u >= o.u_hi) return;
  const uint64_t i = u - o.u_lo;
  if (kind == OUT_UNIFORM) {
    o.d[i] = (double)digit * (digit_bits == 24 ? 5.9604644775390625e-08 : 3.5527136788005009e-15);
  } else if (kind == OUT_Z2_BITS) {
    if ((digit >> (digit_bits - 1)) & 1) atomicOr(&o.bits[i >> 5], 1u << (i & 31));
  } else if (kind == OUT_FIELD_Z2) {
    o.d[2 * i] = ((digit >> (digit_bits - 1)) & 1) ? 1.0 : -1.0;
    o.d[2 * i + 1] = 0.0;
  } else {
    int z = (int)((3 * digit) >> digit_bits);
    o.d[2 * i] = z == 0 ? 1.0 : -0.5;
    o.d[2 * i + 1] = z == 0 ? 0.0 : (z == 1 ? 0.8660254037844388 : -0.8660254037844388);
  }
}

template <int PR, bool DBL>
__global__ void __launch_bounds__(128) ranlux_kernel(const GenArgs* __restrict__ ga, uint64_t b_first,
                                                     uint64_t b_count, int per_group, int out_kind, OutArgs o) {
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = (int)(gtid & 3);
  const uint64_t g = gtid >> 2;
  const uint64_t b0 = b_first + g * (uint64_t)per_group;
  if (b0 >= b_first + b_count) return;
  uint64_t nb = b_first + b_count - b0;
  if (nb > (uint64_t)per_group) nb = per_group;

  Lane s;
  if (b0 == 0) {
    s = ga->lane_seed[lane];
  } else {
    U576 y = ga->y_seed[lane];
    uint64_t e = b0;
    for (int i = 0; e; ++i, e >>= 1)
      if (e & 1) mulmod(y, y, ga->pow_tab[i]);
    decode(s, y);
  }
  uint64_t w[12];
#pragma unroll
  for (int j = 0; j < 12; ++j) w[j] = s.words[j];
  int64_t c = s.carry;
  constexpr int P = DBL ? 48 : 96;
  constexpr int PRM = PR % 12;
  for (uint64_t blk = 0; blk < nb; ++blk) {
#pragma unroll 1
    for (int cyc = 0; cyc < PR / 12; ++cyc) {
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        int64_t d = (int64_t)w[(i + 7) % 12] - (int64_t)w[i] - c;
        c = (d >> 63) & 1;
        w[i] = (uint64_t)d & kMask48;
      }
    }
#pragma unroll
    for (int i = 0; i < PRM; ++i) {
      int64_t d = (int64_t)w[(i + 7) % 12] - (int64_t)w[i] - c;
      c = (d >> 63) & 1;
      w[i] = (uint64_t)d & kMask48;
    }
    // rotate so that the oldest word is w[0] again
    uint64_t t[12];
#pragma unroll
    for (int j = 0; j < 12; ++j) t[j] = w[(j + PRM) % 12];
#pragma unroll
    for (int j = 0; j < 12; ++j) w[j] = t[j];
    const uint64_t ub = (b0 + blk) * (uint64_t)P;
#pragma unroll
    for (int j = 0; j < 12; ++j) {
      if (DBL) {
        emit(o, out_kind, ub + 4 * j + lane, w[j], 48);
      } else {
        emit(o, out_kind, ub + 8 * j + lane, w[j] & 0xffffff, 24);
        emit(o, out_kind, ub + 8 * j + 4 + lane, w[j] >> 24, 24);
      }
    }
  }
}

// Builds the per-(kind, seed) generation arguments on the host.
static void make_gen_args(GenArgs& ga, int kind, long seed) {
  RanluxState s;
  ranlux_seed(s, kind, seed);
  to_lanes(s, ga.lane_seed);
  for (int l = 0; l < 4; ++l) encode(ga.y_seed[l], ga.lane_seed[l]);
  U576 p = powmod(multiplier(), (uint64_t)s.pr);
  for (int i = 0; i < 48; ++i) {
    ga.pow_tab[i] = p;
    mulmod(p, p, p);
  }
}

}  // namespace rng

// Generates outputs [u_lo, u_hi) of the (kind, seed) ranlux stream.
nrcps_status ranlux_generate(nrcps_context* ctx, int kind, long seed, uint64_t u_lo, uint64_t u_hi, int out_kind,
                             double* d, uint32_t* bits) {
  using namespace rng;
  if (u_hi <= u_lo) return NRCPS_OK;
  if (ctx->gen_kind != kind || ctx->gen_seed != seed || ctx->gen_args == nullptr) {
    GenArgs* h = new GenArgs;
    make_gen_args(*h, kind, seed);
    if (!ctx->gen_args) {
      NRCPS_TRY(check_cuda(ctx, cudaMalloc(&ctx->gen_args, sizeof(GenArgs)), "cudaMalloc(GenArgs)"));
    }
    // every stream's draws (a batch's side stream included) are done with
    // the old arguments before they are replaced
    NRCPS_TRY(check_cuda(ctx, cudaDeviceSynchronize(), "sync before GenArgs update"));
    cudaError_t e = cudaMemcpy(ctx->gen_args, h, sizeof(GenArgs), cudaMemcpyHostToDevice);
    delete h;
    NRCPS_TRY(check_cuda(ctx, e, "cudaMemcpy(GenArgs)"));
    ctx->gen_kind = kind;
    ctx->gen_seed = seed;
  }
  const GenArgs* gargs = (const GenArgs*)ctx->gen_args;
  const int P = block_len(kind);
  uint64_t b_first = u_lo / P, b_last = (u_hi - 1) / P;
  uint64_t b_count = b_last - b_first + 1;
  // Blocks per group: enough groups to fill the GPU, at most 64 blocks each.
  uint64_t groups_wanted = (uint64_t)ctx->sm_count * 512;
  int per_group = (int)((b_count + groups_wanted - 1) / groups_wanted);
  if (per_group < 1) per_group = 1;
  if (per_group > 64) per_group = 64;
  uint64_t groups = (b_count + per_group - 1) / per_group;
  uint64_t threads = groups * 4;
  unsigned grid = (unsigned)((threads + 127) / 128);
  OutArgs o{u_lo, u_hi, d, bits};
  switch (kind) {
    case NRCPS_RANLXS0: ranlux_kernel<109, false><<<grid, 128, 0, ctx->stream>>>(gargs, b_first, b_count, per_group, out_kind, o); break;
    case NRCPS_RANLXS1: ranlux_kernel<202, false><<<grid, 128, 0, ctx->stream>>>(gargs, b_first, b_count, per_group, out_kind, o); break;
    case NRCPS_RANLXS2: ranlux_kernel<397, false><<<grid, 128, 0, ctx->stream>>>(gargs, b_first, b_count, per_group, out_kind, o); break;
    case NRCPS_RANLXD1: ranlux_kernel<202, true><<<grid, 128, 0, ctx->stream>>>(gargs, b_first, b_count, per_group, out_kind, o); break;
    case NRCPS_RANLXD2: ranlux_kernel<397, true><<<grid, 128, 0, ctx->stream>>>(gargs, b_first, b_count, per_group, out_kind, o); break;
    default: return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "generator %d has no device path", kind);
  }
  ctx->launches++;
  return check_launch(ctx, "ranlux_kernel");
}

// ------------------------------------------------------------ Gauss fields
// Polar method (src/random/random.C:105-116): pair i = (u[2i], u[2i+1]) of
// the window is accepted when 0 < r2 <= 1; accepted pairs give the field
// values in order.
__global__ void gauss_flags_kernel(const double* u, long npairs, int* flag) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < npairs; i += (long)gridDim.x * blockDim.x) {
    double x = 2 * u[2 * i] - 1, y = 2 * u[2 * i + 1] - 1;
    double r2 = x * x + y * y;
    flag[i] = (r2 > 1.0 || r2 == 0) ? 0 : 1;
  }
}

// Exclusive scan of int flags, one block of 1024 threads per tile of 1024,
// tile sums then scanned on one block (any number of tiles).
__global__ void scan_tiles_kernel(const int* in, int* out, int* tile_sums, long n) {
  __shared__ int s[1024];
  long i = (long)blockIdx.x * 1024 + threadIdx.x;
  int v = i < n ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == 1023) tile_sums[blockIdx.x] = s[1023];
}
__global__ void scan_sums_kernel(int* tile_sums, int ntiles, int* total) {
  __shared__ int s[1024];
  // thread t owns tiles [t per, (t + 1) per)
  const int per = (ntiles + 1023) / 1024, b0 = threadIdx.x * per;
  int v = 0;
  for (int k = 0; k < per; ++k)
    if (b0 + k < ntiles) v += tile_sums[b0 + k];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  int run = s[threadIdx.x] - v;  // tiles before this thread's range
  for (int k = 0; k < per; ++k)
    if (b0 + k < ntiles) {
      const int t = tile_sums[b0 + k];
      tile_sums[b0 + k] = run;
      run += t;
    }
  if (threadIdx.x == 1023) *total = s[1023];
}
// out value index k = rank of the accepted pair; last_pair[k] remembers the
// pair index so that the host learns how many uniforms were consumed.
__global__ void gauss_values_kernel(const double* u, const int* flag, const int* rank, const int* tile_off,
                                    long npairs, long need, long out_base, int complex_pairs, double* out,
                                    int* pair_of_rank) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < npairs; i += (long)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    long k = rank[i] + tile_off[i / 1024];
    if (k >= need) continue;
    double x = 2 * u[2 * i] - 1, y = 2 * u[2 * i + 1] - 1;
    double r2 = x * x + y * y;
    double g = 1.0 * y * sqrt(-2.0 * log(r2) / r2);
    long kk = out_base + k;
    if (complex_pairs) {
      out[kk] = g;  // consecutive Gaussians fill re, im alternately
    } else {
      out[2 * kk] = g;
      out[2 * kk + 1] = 0.0;
    }
    pair_of_rank[k] = (int)i;
  }
}

}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_rng_seed_state(int kind, long seed, long* state, int* state_size) {
  if (!state || !state_size) return NRCPS_ERR_INVALID_ARGUMENT;
  if (rng::is_ranlux(kind)) {
    rng::RanluxState s;
    if (!rng::ranlux_seed(s, kind, seed)) return NRCPS_ERR_INVALID_ARGUMENT;
    state[0] = 105;
    for (int k = 0; k < 96; ++k) state[k + 1] = s.num[k];
    for (int l = 0; l < 4; ++l) state[97 + l] = s.carry[l];
    state[101] = s.pr;
    state[102] = s.ir;
    state[103] = s.jr;
    state[104] = s.is;
    *state_size = 105;
    return NRCPS_OK;
  }
  if (kind == NRCPS_RAN2) {
    rng::Ran2 r;
    r.seed(seed);
    state[0] = 36;
    state[1] = r.idum;
    state[2] = r.idum2;
    state[3] = r.iy;
    for (int i = 0; i < 32; ++i) state[4 + i] = r.iv[i];
    *state_size = 36;
    return NRCPS_OK;
  }
  return NRCPS_ERR_UNSUPPORTED;
}

extern "C" nrcps_status nrcps_rng_skip(int kind, long* state, uint64_t n) {
  if (!state || !rng::is_ranlux(kind)) return NRCPS_ERR_UNSUPPORTED;
  rng::RanluxState s;
  s.dbl = rng::is_dbl(kind);
  for (int k = 0; k < 96; ++k) s.num[k] = (int)state[k + 1];
  for (int l = 0; l < 4; ++l) s.carry[l] = (int)state[97 + l];
  s.pr = (int)state[101];
  s.ir = (int)state[102];
  s.jr = (int)state[103];
  s.is = (int)state[104];
  s.is_old = 8 * s.ir;
  if (s.pr != rng::pr_of(kind) || s.ir < 0 || s.ir > 11) return NRCPS_ERR_INVALID_ARGUMENT;
  rng::ranlux_skip(s, n);
  for (int k = 0; k < 96; ++k) state[k + 1] = s.num[k];
  for (int l = 0; l < 4; ++l) state[97 + l] = s.carry[l];
  state[102] = s.ir;
  state[103] = s.jr;
  state[104] = s.is;
  return NRCPS_OK;
}

// Host generation for ran2 into a device array.
static nrcps_status ran2_upload(nrcps_context* ctx, long seed, uint64_t offset, uint64_t count, int out_kind,
                                double* d, uint32_t* bits) {
  rng::Ran2 r;
  r.seed(seed);
  for (uint64_t i = 0; i < offset; ++i) r.next();
  if (out_kind == rng::OUT_Z2_BITS) {
    std::vector<uint32_t> h((count + 31) / 32, 0u);
    for (uint64_t i = 0; i < count; ++i)
      if (std::floor(2 * r.next()) >= 1.0) h[i >> 5] |= 1u << (i & 31);
    return check_cuda(ctx, cudaMemcpyAsync(bits, h.data(), h.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
                      "ran2 upload");
  }
  int mult = out_kind == rng::OUT_UNIFORM ? 1 : 2;
  std::vector<double> h(count * mult);
  for (uint64_t i = 0; i < count; ++i) {
    double u = r.next();
    if (out_kind == rng::OUT_UNIFORM) {
      h[i] = u;
    } else if (out_kind == rng::OUT_FIELD_Z2) {
      h[2 * i] = 2.0 * (int)std::floor(2 * u) - 1.0;
      h[2 * i + 1] = 0.0;
    } else {
      int z = (int)std::floor(3 * u);
      h[2 * i] = z == 0 ? 1.0 : -0.5;
      h[2 * i + 1] = z == 0 ? 0.0 : (z == 1 ? 0.8660254037844388 : -0.8660254037844388);
    }
  }
  NRCPS_TRY(check_cuda(ctx, cudaMemcpyAsync(d, h.data(), h.size() * 8, cudaMemcpyHostToDevice, ctx->stream),
                       "ran2 upload"));
  return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "ran2 upload sync");
}

static nrcps_status generate(nrcps_context* ctx, int kind, long seed, uint64_t offset, uint64_t count, int out_kind,
                             double* d, uint32_t* bits) {
  if (rng::is_ranlux(kind)) {
    if (seed <= 0 || seed > 2147483647L)
      return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT, "ranlux seed must be in [1, 2^31-1]");
    return ranlux_generate(ctx, kind, seed, offset, offset + count, out_kind, d, bits);
  }
  if (kind == NRCPS_RAN2) return ran2_upload(ctx, seed, offset, count, out_kind, d, bits);
  return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "generator kind %d not supported", kind);
}

extern "C" nrcps_status nrcps_rng_uniforms(nrcps_context* ctx, int kind, long seed, uint64_t offset,
                                           uint64_t count, double* dev_out) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, dev_out || count == 0, "nrcps_rng_uniforms: null output");
  return generate(ctx, kind, seed, offset, count, rng::OUT_UNIFORM, dev_out, nullptr);
}

extern "C" nrcps_status nrcps_draw_z2_bits(nrcps_context* ctx, int kind, long seed, uint64_t first, uint64_t count,
                                           uint32_t* dev_bits) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, dev_bits || count == 0, "nrcps_draw_z2_bits: null output");
  if (count == 0) return NRCPS_OK;
  NRCPS_TRY(check_cuda(ctx, cudaMemsetAsync(dev_bits, 0, ((count + 31) / 32) * 4, ctx->stream), "memset bits"));
  return generate(ctx, kind, seed, first, count, rng::OUT_Z2_BITS, nullptr, dev_bits);
}

extern "C" nrcps_status nrcps_draw_fields(nrcps_context* ctx, int kind, long seed, int field_kind, long vol,
                                          long slices, uint64_t* offset, double* dev_out) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, offset && dev_out && vol > 0 && slices >= 0, "nrcps_draw_fields: bad arguments");
  const uint64_t sites = (uint64_t)vol * slices;
  if (sites == 0) return NRCPS_OK;
  if (field_kind == NRCPS_FIELD_ZTWO || field_kind == NRCPS_FIELD_ZTHREE) {
    NRCPS_TRY(generate(ctx, kind, seed, *offset, sites,
                       field_kind == NRCPS_FIELD_ZTWO ? rng::OUT_FIELD_Z2 : rng::OUT_FIELD_Z3, dev_out, nullptr));
    *offset += sites;
    return NRCPS_OK;
  }
  if (field_kind != NRCPS_FIELD_GAUSS && field_kind != NRCPS_FIELD_COMPLEXGAUSS)
    return set_error(ctx, NRCPS_ERR_INVALID_ARGUMENT, "unknown field kind %d", field_kind);
  // Gaussian: need one (GAUSS) or two (COMPLEXGAUSS) accepted pairs per site.
  const int cpx = field_kind == NRCPS_FIELD_COMPLEXGAUSS;
  const long need_total = (long)sites * (cpx ? 2 : 1);
  long done = 0;
  while (done < need_total) {
    long need = need_total - done;
    // pairs per round: acceptance pi/4 = 0.785; up to 128 M pairs (3.5 GB of
    // working memory), so a large draw takes few host round trips
    long npairs = (long)(need * 1.35) + 4096;
    if (npairs > 128L * 1024 * 1024) npairs = 128L * 1024 * 1024;
    const long ntiles_max = (npairs + 1023) / 1024;
    size_t bytes_u = sizeof(double) * 2 * npairs;
    size_t bytes_i = sizeof(int) * (3 * npairs + ntiles_max + 16);
    nrcps_status st;
    char* base = (char*)scratch(ctx, bytes_u + bytes_i, &st);
    if (!base) return st;
    double* u = (double*)base;
    int* flag = (int*)(base + bytes_u);
    int* rank = flag + npairs;
    int* pair_of_rank = rank + npairs;
    int* tiles = pair_of_rank + npairs;
    int* total = tiles + ntiles_max;
    NRCPS_TRY(generate(ctx, kind, seed, *offset, 2 * (uint64_t)npairs, rng::OUT_UNIFORM, u, nullptr));
    unsigned g = grid_for(npairs, 256, (long)ctx->sm_count * 8);
    gauss_flags_kernel<<<g, 256, 0, ctx->stream>>>(u, npairs, flag);
    int ntiles = (int)((npairs + 1023) / 1024);
    scan_tiles_kernel<<<ntiles, 1024, 0, ctx->stream>>>(flag, rank, tiles, npairs);
    scan_sums_kernel<<<1, 1024, 0, ctx->stream>>>(tiles, ntiles, total);
    long take = need;
    gauss_values_kernel<<<g, 256, 0, ctx->stream>>>(u, flag, rank, tiles, npairs, take, done, cpx,
                                                    cpx ? dev_out : dev_out, pair_of_rank);
    ctx->launches += 4;
    NRCPS_TRY(check_launch(ctx, "gauss kernels"));
    int h_total = 0;
    NRCPS_TRY(check_cuda(ctx, cudaMemcpyAsync(&h_total, total, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream),
                         "gauss total"));
    NRCPS_TRY(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "gauss sync"));
    long got = h_total < take ? h_total : take;
    int last_pair = 0;
    if (got > 0) {
      NRCPS_TRY(check_cuda(ctx, cudaMemcpy(&last_pair, pair_of_rank + (got - 1), sizeof(int),
                                           cudaMemcpyDeviceToHost), "gauss last pair"));
      *offset += 2 * (uint64_t)(last_pair + 1);
    } else {
      *offset += 2 * (uint64_t)npairs;
    }
    done += got;
  }
  return NRCPS_OK;
}

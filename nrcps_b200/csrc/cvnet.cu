// cvnet.cu -- kernels of the learned control variate (no counterpart in the
// reference): a small 3-D convolutional network reads the auxiliary-field
// time slices of a configuration and predicts log C(tau); its prediction g
// enters the estimator C - c (g - <g>) with <g> from many extra field draws.
//
// Network (per configuration):
//   x   [T][G^3]       block means of phi over (L/G)^3 sites per slice (BF16)
//   conv1  T -> 16, conv2 16 -> 16, conv3 16 -> 16: 3x3x3 periodic
//          cross-correlation out[s] = b + sum_ci sum_k W[co][ci][k] in[ci][s+k],
//          tanh, activations stored in BF16, pre-activations in FP32
//   pool   mean over the G^3 sites -> 16 features (FP32)
//   head   tanh(W1 p + b1) (32 units) -> W2 h + b2 (T outputs, FP32)
// BF16 conv weights (an FP32 master copy is updated by Adam), FP32
// accumulation everywhere.  Layouts are per sample contiguous: act[b][c][s],
// s = z + G (y + G x).
#include <cuda_bf16.h>

#include "common.cuh"

namespace nrcps {
namespace cv {

constexpr int K27 = 27;

__device__ __forceinline__ int nbr(int s, int k, int G) {
  const int x = s / (G * G), y = (s / G) % G, z = s % G;
  const int dx = k / 9 - 1, dy = (k / 3) % 3 - 1, dz = k % 3 - 1;
  const int xx = (x + dx + G) % G, yy = (y + dy + G) % G, zz = (z + dz + G) % G;
  return zz + G * (yy + G * xx);
}

// ------------------------------------------------------------ input stage
// Block means of the Z2 field: config c, slice t, cell q of G^3: mean of
// phi = +-1 over its f^3 sites (f = L/G).  Bit (bit0 + (c T + t) V + site)
// of `bits` is phi = +1 (the packed layout of nrcps_draw_z2_bits).
__global__ void coarse_z2_kernel(const uint32_t* __restrict__ bits, uint64_t bit0, int L, int T, int G, int B,
                                 __nv_bfloat16* __restrict__ x) {
  const long V = (long)L * L * L;
  const int GS = G * G * G, f = L / G;
  const long total = (long)B * T * GS;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int q = (int)(e % GS);
    const long ct = e / GS;  // c * T + t
    const int qx = q / (G * G), qy = (q / G) % G, qz = q % G;
    int sum = 0;
    for (int a = 0; a < f; ++a)
      for (int b2 = 0; b2 < f; ++b2)
        for (int d = 0; d < f; ++d) {
          const long site = (long)(qz * f + d) + L * ((long)(qy * f + b2) + L * (long)(qx * f + a));
          const uint64_t k = bit0 + (uint64_t)ct * V + (uint64_t)site;
          sum += ((bits[k >> 5] >> (k & 31)) & 1u) ? 1 : -1;
        }
    x[e] = __float2bfloat16((float)sum / (float)(f * f * f));
  }
}

// Same block means when every z-row starts on a 32-bit word (L % 32 == 0,
// bit0 % 32 == 0) and f divides 32: one thread per (configuration, slice,
// qx, qy) column of G cells reads the f^2 rows of its column one word at a
// time and counts the +1 sites of each f-bit group with popc -- one load per
// 32 sites instead of one per site.
__global__ void coarse_z2_rows_kernel(const uint32_t* __restrict__ bits, uint64_t bit0, int L, int T, int G, int B,
                                      __nv_bfloat16* __restrict__ x) {
  const long V = (long)L * L * L;
  const int GS = G * G * G, f = L / G, per_word = 32 / f, words = L / 32;
  const uint32_t mask = f >= 32 ? 0xffffffffu : ((1u << f) - 1u);
  const long total = (long)B * T * G * G;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int qy = (int)(e % G), qx = (int)((e / G) % G);
    const long ct = e / ((long)G * G);
    int cnt[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) cnt[q] = 0;
    for (int a = 0; a < f; ++a)
      for (int b2 = 0; b2 < f; ++b2) {
        const uint64_t r0 = bit0 + (uint64_t)ct * V + (uint64_t)L * ((uint64_t)(qy * f + b2) + (uint64_t)L * (qx * f + a));
        const uint32_t* row = bits + (r0 >> 5);
        for (int w = 0; w < words; ++w) {
          const uint32_t word = __ldg(row + w);
#pragma unroll
          for (int g = 0; g < 16; ++g)
            if (g < per_word) cnt[w * per_word + g] += __popc((word >> (g * f)) & mask);
        }
      }
    const float inv = 1.0f / (float)(f * f * f);
    const long o = ct * GS + (long)G * (qy + (long)G * qx);
#pragma unroll
    for (int qz = 0; qz < 16; ++qz)
      if (qz < G) x[o + qz] = __float2bfloat16((float)(2 * cnt[qz] - f * f * f) * inv);
  }
}

// ------------------------------------------------- direct feature draws
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): ten rounds of two
// 32x32 -> 64-bit products with the key bumped by the Weyl constants.
struct U4 {
  uint32_t x, y, z, w;
};
__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Block means of a uniform Z2 field drawn directly: the n = f^3 sites of a
// cell are n independent fair bits, so the mean is (2 popc - n)/n.  Cell
// g = ((first + b) T + t) G^3 + q takes word i from output i % 4 of the
// Philox call with counter (lo g, hi g, i / 4, 0x5A32), key = seed; the last
// word keeps its n mod 32 low bits.  One thread per cell.
__global__ void sample_z2_features_kernel(uint64_t seed, uint64_t first, int T, int GS, int n, long total,
                                          __nv_bfloat16* __restrict__ x) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const int words = (n + 31) / 32;
  const float inv = 1.0f / (float)n;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const uint64_t g = first * (uint64_t)T * (uint64_t)GS + (uint64_t)e;
    int cnt = 0;
    for (int grp = 0; grp * 4 < words; ++grp) {
      const U4 o = philox4x32_10(U4{(uint32_t)g, (uint32_t)(g >> 32), (uint32_t)grp, 0x5A32u}, k0, k1);
      const uint32_t w4[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = grp * 4 + j;
        if (i < words) {
          const int rem = n - 32 * i;
          cnt += __popc(rem < 32 ? (w4[j] & ((1u << rem) - 1u)) : w4[j]);
        }
      }
    }
    x[e] = __float2bfloat16((float)(2 * cnt - n) * inv);
  }
}

// ------------------------------------------------------------- conv fwd
// One block per sample; the sample's input and the layer's weights in
// shared memory (BF16); each thread computes all Cout outputs of its sites.
template <int COUT>
__global__ void __launch_bounds__(256) conv_fwd_kernel(const __nv_bfloat16* __restrict__ in, int Cin, int G,
                                                       const __nv_bfloat16* __restrict__ W,
                                                       const float* __restrict__ bias, float* __restrict__ Z,
                                                       __nv_bfloat16* __restrict__ A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int GS = G * G * G;
  __nv_bfloat16* sin = reinterpret_cast<__nv_bfloat16*>(smem);
  __nv_bfloat16* sw = sin + (size_t)Cin * GS;
  const long b = blockIdx.x;
  for (int e = threadIdx.x; e < Cin * GS; e += blockDim.x) sin[e] = in[b * Cin * GS + e];
  for (int e = threadIdx.x; e < COUT * Cin * K27; e += blockDim.x) sw[e] = W[e];
  __syncthreads();
  for (int s = threadIdx.x; s < GS; s += blockDim.x) {
    float acc[COUT];
#pragma unroll
    for (int co = 0; co < COUT; ++co) acc[co] = bias[co];
    for (int k = 0; k < K27; ++k) {
      const int nb = nbr(s, k, G);
      for (int ci = 0; ci < Cin; ++ci) {
        const float v = __bfloat162float(sin[ci * GS + nb]);
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] = fmaf(__bfloat162float(sw[(co * Cin + ci) * K27 + k]), v, acc[co]);
      }
    }
#pragma unroll
    for (int co = 0; co < COUT; ++co) {
      const long o = (b * COUT + co) * GS + s;
      Z[o] = acc[co];
      A[o] = __float2bfloat16(tanhf(acc[co]));
    }
  }
}

// ------------------------------------------------------- conv bwd (data)
// dZprev[b][ci][s] = (1 - Aprev^2) sum_co sum_k W[co][ci][k] dZ[b][co][s - k]
template <int CIN>
__global__ void __launch_bounds__(256) conv_bwd_data_kernel(const float* __restrict__ dZ, int Cout, int G,
                                                            const __nv_bfloat16* __restrict__ W,
                                                            const __nv_bfloat16* __restrict__ Aprev,
                                                            float* __restrict__ dZprev) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int GS = G * G * G;
  float* sdz = reinterpret_cast<float*>(smem);
  __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(sdz + (size_t)Cout * GS);
  const long b = blockIdx.x;
  for (int e = threadIdx.x; e < Cout * GS; e += blockDim.x) sdz[e] = dZ[b * Cout * GS + e];
  for (int e = threadIdx.x; e < Cout * CIN * K27; e += blockDim.x) sw[e] = W[e];
  __syncthreads();
  for (int s = threadIdx.x; s < GS; s += blockDim.x) {
    float acc[CIN];
#pragma unroll
    for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.0f;
    for (int k = 0; k < K27; ++k) {
      const int src = nbr(s, K27 - 1 - k, G);  // s - k: the mirrored offset
      for (int co = 0; co < Cout; ++co) {
        const float d = sdz[co * GS + src];
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) acc[ci] = fmaf(__bfloat162float(sw[(co * CIN + ci) * K27 + k]), d, acc[ci]);
      }
    }
#pragma unroll
    for (int ci = 0; ci < CIN; ++ci) {
      const long o = (b * CIN + ci) * GS + s;
      const float a = __bfloat162float(Aprev[o]);
      dZprev[o] = acc[ci] * (1.0f - a * a);
    }
  }
}

// ----------------------------------------------------- conv bwd (weight)
// dW[co][ci][k] = sum_b sum_s dZ[b][co][s] in[b][ci][s + k]; one thread per
// (ci, k) column of a column chunk, all COUT rows; blocks take chunks of
// samples and add their partial sums atomically (dW zeroed by the caller).
template <int COUT>
__global__ void __launch_bounds__(256) conv_bwd_weight_kernel(const float* __restrict__ dZ,
                                                              const __nv_bfloat16* __restrict__ in, int Cin, int G,
                                                              int B, int samples_per_block, float* __restrict__ dW) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int GS = G * G * G;
  const int ci0 = blockIdx.y * 8;                 // 8 input channels per column chunk
  const int nci = Cin - ci0 < 8 ? Cin - ci0 : 8;
  float* sdz = reinterpret_cast<float*>(smem);                                      // [COUT][GS]
  __nv_bfloat16* sin = reinterpret_cast<__nv_bfloat16*>(sdz + (size_t)COUT * GS);  // [8][GS]
  const int col = threadIdx.x;                    // (ci_local, k) = (col / 27, col % 27)
  const bool active = col < nci * K27;
  const int cil = active ? col / K27 : 0, k = active ? col % K27 : 0;
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) acc[co] = 0.0f;
  const int b0 = blockIdx.x * samples_per_block;
  const int b1 = b0 + samples_per_block < B ? b0 + samples_per_block : B;
  for (int b = b0; b < b1; ++b) {
    __syncthreads();
    for (int e = threadIdx.x; e < COUT * GS; e += blockDim.x) sdz[e] = dZ[(long)b * COUT * GS + e];
    for (int e = threadIdx.x; e < nci * GS; e += blockDim.x) sin[e] = in[((long)b * Cin + ci0) * GS + e];
    __syncthreads();
    if (active) {
      for (int s = 0; s < GS; ++s) {
        const float p = __bfloat162float(sin[cil * GS + nbr(s, k, G)]);
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] = fmaf(sdz[co * GS + s], p, acc[co]);
      }
    }
  }
  if (active)
#pragma unroll
    for (int co = 0; co < COUT; ++co) atomicAdd(&dW[(co * Cin + ci0 + cil) * K27 + k], acc[co]);
}

// db[c] = sum_b sum_s dZ[b][c][s]; one block per channel.
__global__ void bias_grad_kernel(const float* __restrict__ dZ, int C, int GS, int B, float* __restrict__ db) {
  __shared__ float red[256];
  const int c = blockIdx.x;
  float s = 0.0f;
  for (long e = threadIdx.x; e < (long)B * GS; e += blockDim.x) {
    const long b = e / GS, q = e % GS;
    s += dZ[(b * C + c) * GS + q];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] = red[0];
}

// --------------------------------------------------------- pool + head
// One thread per sample: p = mean_s A3, h = tanh(W1 p + b1), y = W2 h + b2.
__global__ void head_fwd_kernel(const __nv_bfloat16* __restrict__ A3, int C, int GS, int B, const float* __restrict__ W1,
                                const float* __restrict__ b1, int H, const float* __restrict__ W2,
                                const float* __restrict__ b2, int T, float* __restrict__ P, float* __restrict__ Hact,
                                float* __restrict__ Y) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  float p[16];
  for (int c = 0; c < C && c < 16; ++c) {
    float s = 0.0f;
    for (int q = 0; q < GS; ++q) s += __bfloat162float(A3[((long)b * C + c) * GS + q]);
    p[c] = s / (float)GS;
    P[(long)b * C + c] = p[c];
  }
  for (int j = 0; j < H; ++j) {
    float s = b1[j];
    for (int c = 0; c < C; ++c) s = fmaf(W1[j * C + c], p[c], s);
    Hact[(long)b * H + j] = tanhf(s);
  }
  for (int t = 0; t < T; ++t) {
    float s = b2[t];
    for (int j = 0; j < H; ++j) s = fmaf(W2[t * H + j], Hact[(long)b * H + j], s);
    Y[(long)b * T + t] = s;
  }
}

// Loss 0.5 mean (y - target)^2 over B x T; per sample: dY, dh, dP and the
// pool backward into dZ3 = dP / GS (1 - A3^2).  loss_parts[b] = per-sample sum.
__global__ void head_bwd_kernel(const float* __restrict__ Y, const float* __restrict__ target, int T, int B,
                                const float* __restrict__ Hact, int H, const float* __restrict__ W2,
                                const float* __restrict__ W1, int C, const __nv_bfloat16* __restrict__ A3, int GS,
                                float* __restrict__ dY, float* __restrict__ dZh, float* __restrict__ dZ3,
                                float* __restrict__ loss_parts) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const float scale = 1.0f / ((float)B * (float)T);
  float l = 0.0f;
  for (int t = 0; t < T; ++t) {
    const float d = Y[(long)b * T + t] - target[(long)b * T + t];
    l += 0.5f * d * d;
    dY[(long)b * T + t] = d * scale;
  }
  loss_parts[b] = l;
  float dp[16];
  for (int c = 0; c < C && c < 16; ++c) dp[c] = 0.0f;
  for (int j = 0; j < H; ++j) {
    float s = 0.0f;
    for (int t = 0; t < T; ++t) s = fmaf(W2[t * H + j], dY[(long)b * T + t], s);
    const float h = Hact[(long)b * H + j];
    const float dz = s * (1.0f - h * h);
    dZh[(long)b * H + j] = dz;
    for (int c = 0; c < C; ++c) dp[c] = fmaf(W1[j * C + c], dz, dp[c]);
  }
  for (int c = 0; c < C; ++c)
    for (int q = 0; q < GS; ++q) {
      const long o = ((long)b * C + c) * GS + q;
      const float a = __bfloat162float(A3[o]);
      dZ3[o] = dp[c] / (float)GS * (1.0f - a * a);
    }
}

// dM[r][c] = sum_b dR[b][r] X[b][c] (dense weight gradient), db[r] = sum_b dR[b][r]; one thread per (r, c).
__global__ void dense_grad_kernel(const float* __restrict__ dR, int R, const float* __restrict__ X, int Cc, int B,
                                  float* __restrict__ dM, float* __restrict__ db) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= R * (Cc + 1)) return;
  const int r = e / (Cc + 1), c = e % (Cc + 1);
  float s = 0.0f;
  for (int b = 0; b < B; ++b) s += dR[(long)b * R + r] * (c < Cc ? X[(long)b * Cc + c] : 1.0f);
  if (c < Cc) dM[r * Cc + c] = s;
  else db[r] = s;
}

// Adam on FP32 masters; bf16 != nullptr refreshes the BF16 copy.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long n, float lr, float b1, float b2, float eps, float c1, float c2,
                            __nv_bfloat16* __restrict__ bf16) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (bf16) bf16[i] = __float2bfloat16(wi);
  }
}

}  // namespace cv
}  // namespace nrcps

using namespace nrcps;
using namespace nrcps::cv;

static size_t conv_fwd_smem(int Cin, int GS, int Cout) { return 2 * ((size_t)Cin * GS + (size_t)Cout * Cin * 27); }

extern "C" nrcps_status nrcps_cv_coarse_z2(nrcps_context* ctx, const uint32_t* dev_bits, uint64_t bit0, int L, int T,
                                           int G, int B, void* dev_x) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, ((dev_bits && dev_x) || B == 0) && L > 0 && G > 0 && L % G == 0 && T > 0 && B >= 0,
                "nrcps_cv_coarse_z2: bad arguments (G must divide L)");
  const long total = (long)B * T * G * G * G;
  if (total == 0) return NRCPS_OK;
  const int f = L / G;
  if (L % 32 == 0 && bit0 % 32 == 0 && 32 % f == 0 && G <= 16) {
    const long cols = (long)B * T * G * G;
    coarse_z2_rows_kernel<<<grid_for(cols, 256, (long)ctx->sm_count * 32), 256, 0, ctx->stream>>>(
        dev_bits, bit0, L, T, G, B, reinterpret_cast<__nv_bfloat16*>(dev_x));
    ctx->launches++;
    return check_launch(ctx, "coarse_z2_rows_kernel");
  }
  coarse_z2_kernel<<<grid_for(total, 256, (long)ctx->sm_count * 32), 256, 0, ctx->stream>>>(
      dev_bits, bit0, L, T, G, B, reinterpret_cast<__nv_bfloat16*>(dev_x));
  ctx->launches++;
  return check_launch(ctx, "coarse_z2_kernel");
}

extern "C" nrcps_status nrcps_cv_sample_z2_features(nrcps_context* ctx, uint64_t seed, uint64_t first, int L, int T,
                                                    int G, int B, void* dev_x) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, (dev_x || B == 0) && L > 0 && G > 0 && L % G == 0 && T > 0 && B >= 0,
                "nrcps_cv_sample_z2_features: bad arguments (G must divide L)");
  const int f = L / G;
  const long total = (long)B * T * G * G * G;
  if (total == 0) return NRCPS_OK;
  sample_z2_features_kernel<<<grid_for(total, 256, (long)ctx->sm_count * 16), 256, 0, ctx->stream>>>(
      seed, first, T, G * G * G, f * f * f, total, reinterpret_cast<__nv_bfloat16*>(dev_x));
  ctx->launches++;
  return check_launch(ctx, "sample_z2_features_kernel");
}

extern "C" nrcps_status nrcps_cv_conv_forward(nrcps_context* ctx, const void* dev_in, int Cin, int Cout, int G,
                                              int B, const void* dev_W, const float* dev_bias, float* dev_Z,
                                              void* dev_A) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, Cout == 16 && Cin > 0 && G > 0 && B >= 0, "nrcps_cv_conv_forward: Cout must be 16");
  const int GS = G * G * G;
  const size_t sh = conv_fwd_smem(Cin, GS, Cout);
  NRCPS_REQUIRE(ctx, sh <= 200 * 1024, "nrcps_cv_conv_forward: input sample and weights exceed shared memory");
  if (B == 0) return NRCPS_OK;
  NRCPS_TRY(check_cuda(ctx, cudaFuncSetAttribute(conv_fwd_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 200 * 1024),
                       "conv fwd attribute"));
  conv_fwd_kernel<16><<<B, 256, sh, ctx->stream>>>(reinterpret_cast<const __nv_bfloat16*>(dev_in), Cin, G,
                                                   reinterpret_cast<const __nv_bfloat16*>(dev_W), dev_bias, dev_Z,
                                                   reinterpret_cast<__nv_bfloat16*>(dev_A));
  ctx->launches++;
  return check_launch(ctx, "conv_fwd_kernel");
}

extern "C" nrcps_status nrcps_cv_conv_backward(nrcps_context* ctx, const float* dev_dZ, const void* dev_in,
                                               const void* dev_Ain, int Cin, int Cout, int G, int B, const void* dev_W,
                                               float* dev_dW, float* dev_db, float* dev_dZin) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, Cout == 16 && Cin > 0 && G > 0 && B > 0 && dev_dW && dev_db,
                "nrcps_cv_conv_backward: bad arguments");
  const int GS = G * G * G;
  NRCPS_TRY(check_cuda(ctx, cudaMemsetAsync(dev_dW, 0, sizeof(float) * (size_t)Cout * Cin * 27, ctx->stream),
                       "memset dW"));
  {
    const int spb = 8;
    dim3 grid((unsigned)((B + spb - 1) / spb), (unsigned)((Cin + 7) / 8));
    const size_t sh = sizeof(float) * (size_t)Cout * GS + 2 * (size_t)8 * GS;
    NRCPS_TRY(check_cuda(ctx,
                         cudaFuncSetAttribute(conv_bwd_weight_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              200 * 1024),
                         "conv bwd weight attribute"));
    conv_bwd_weight_kernel<16><<<grid, 256, sh, ctx->stream>>>(dev_dZ, reinterpret_cast<const __nv_bfloat16*>(dev_in),
                                                               Cin, G, B, spb, dev_dW);
    ctx->launches++;
    NRCPS_TRY(check_launch(ctx, "conv_bwd_weight_kernel"));
  }
  bias_grad_kernel<<<Cout, 256, 0, ctx->stream>>>(dev_dZ, Cout, GS, B, dev_db);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "bias_grad_kernel"));
  if (dev_dZin) {
    NRCPS_REQUIRE(ctx, Cin == 16 && dev_Ain, "nrcps_cv_conv_backward: data gradient needs Cin = 16 and Ain");
    const size_t sh = sizeof(float) * (size_t)Cout * GS + 2 * (size_t)Cout * 16 * 27;
    NRCPS_TRY(check_cuda(ctx,
                         cudaFuncSetAttribute(conv_bwd_data_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              200 * 1024),
                         "conv bwd data attribute"));
    conv_bwd_data_kernel<16><<<B, 256, sh, ctx->stream>>>(dev_dZ, Cout, G,
                                                          reinterpret_cast<const __nv_bfloat16*>(dev_W),
                                                          reinterpret_cast<const __nv_bfloat16*>(dev_Ain), dev_dZin);
    ctx->launches++;
    NRCPS_TRY(check_launch(ctx, "conv_bwd_data_kernel"));
  }
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_cv_head_forward(nrcps_context* ctx, const void* dev_A3, int C, int G, int B,
                                              const float* W1, const float* b1, int H, const float* W2,
                                              const float* b2, int T, float* P, float* Hact, float* Y) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, C > 0 && C <= 16 && H > 0 && T > 0 && B >= 0, "nrcps_cv_head_forward: bad arguments");
  if (B == 0) return NRCPS_OK;
  head_fwd_kernel<<<(B + 127) / 128, 128, 0, ctx->stream>>>(reinterpret_cast<const __nv_bfloat16*>(dev_A3), C,
                                                            G * G * G, B, W1, b1, H, W2, b2, T, P, Hact, Y);
  ctx->launches++;
  return check_launch(ctx, "head_fwd_kernel");
}

extern "C" nrcps_status nrcps_cv_head_backward(nrcps_context* ctx, const float* Y, const float* target, int T, int B,
                                               const float* Hact, int H, const float* W2, const float* W1, int C,
                                               const void* dev_A3, int G, const float* P, float* dY, float* dZh,
                                               float* dZ3, float* loss_parts, float* dW2, float* db2, float* dW1,
                                               float* db1) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, C > 0 && C <= 16 && H > 0 && T > 0 && B > 0, "nrcps_cv_head_backward: bad arguments");
  const int GS = G * G * G;
  head_bwd_kernel<<<(B + 127) / 128, 128, 0, ctx->stream>>>(Y, target, T, B, Hact, H, W2, W1, C,
                                                            reinterpret_cast<const __nv_bfloat16*>(dev_A3), GS, dY,
                                                            dZh, dZ3, loss_parts);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "head_bwd_kernel"));
  dense_grad_kernel<<<(T * (H + 1) + 127) / 128, 128, 0, ctx->stream>>>(dY, T, Hact, H, B, dW2, db2);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "dense_grad_kernel(W2)"));
  dense_grad_kernel<<<(H * (C + 1) + 127) / 128, 128, 0, ctx->stream>>>(dZh, H, P, C, B, dW1, db1);
  ctx->launches++;
  return check_launch(ctx, "dense_grad_kernel(W1)");
}

extern "C" nrcps_status nrcps_cv_adam(nrcps_context* ctx, float* w, const float* g, float* m, float* v, long n,
                                      float lr, float beta1, float beta2, float eps, int step, void* bf16_copy) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, w && g && m && v && n > 0 && step > 0, "nrcps_cv_adam: bad arguments");
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  adam_kernel<<<grid_for(n, 256, (long)ctx->sm_count * 8), 256, 0, ctx->stream>>>(
      w, g, m, v, n, lr, beta1, beta2, eps, c1, c2, reinterpret_cast<__nv_bfloat16*>(bf16_copy));
  ctx->launches++;
  return check_launch(ctx, "adam_kernel");
}

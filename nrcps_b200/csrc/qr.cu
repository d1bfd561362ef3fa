// qr.cu -- periodic re-orthonormalisation of the orbitals (CholeskyQR in FP64).
//
// The reference propagates unstabilised (its only option is a host-side
// norm rescale, Propagator::Normalize, src/alg/propagator.C:78-135).  At
// long Euclidean times the orbitals of a configuration align and the Slater
// matrices lose precision.  Here, every qr_period slices, each
// configuration's orbital block Psi (V x N) is replaced by Q with Psi = Q R:
//   G = Psi^H Psi (FP64 accumulation), G = R^H R (Cholesky), Psi <- Psi R^-1.
// R is upper triangular in orbital order, so the first n columns of Psi are
// the first n columns of Q times the leading n x n block of R, and every
// leading-minor determinant the measurement needs is recovered as
//   det S_n(Psi) = det S_n(Q) * prod_{i <= n} R_ii.
// The running sum of log R_ii per orbital is kept per configuration and the
// measured determinants are rescaled by exp(sum_{i<=n} log R_ii).
#include "common.cuh"

namespace nrcps {

bool gram_tc_supported(int N, long vol, int nconf);
nrcps_status gram_tc(nrcps_context* ctx, const void* psi, int N, long vol, int nconf, double* G);

// G[c][i][j] for i <= j (the upper triangle the Cholesky reads), one block
// per configuration reading its orbitals once: tiles of GT sites of all N
// orbitals go through shared memory (rows padded by one element so that the
// rows a warp reads fall in different banks); each thread accumulates 2 x 2
// blocks (i, i+1) x (j, j+1) of G over a quarter of each tile's sites, in R
// within a tile and in FP64 across tiles; the four quarters are summed at
// the end.
constexpr int GT = 128;
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src, int bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if (bytes == 16) asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}

// DB: double-buffered tiles (the next tile's asynchronous copies overlap the
// current tile's products); else one tile buffer.
template <typename R, int MAXB, bool DB = false>
__global__ void __launch_bounds__(256) gram_tile_kernel(const void* __restrict__ psi, int N, long vol,
                                                        double* __restrict__ G) {
  extern __shared__ __align__(16) unsigned char gsm[];
  cplx<R>* tiles = reinterpret_cast<cplx<R>*>(gsm);  // [DB ? 2 : 1][N][GT + 1]
  const long c = blockIdx.x;
  const cplx<R>* base = reinterpret_cast<const cplx<R>*>(psi) + (size_t)c * N * vol;
  const int nb = (N + 1) / 2;                // 2-row blocks
  const int nblk = nb * (nb + 1) / 2;        // upper-triangular block pairs
  const int lane64 = threadIdx.x & 63, grp = threadIdx.x >> 6;
  // MAXB: 2-row block pairs per thread, ceil(nblk / 64): 2 for N <= 22, 3 for N <= 32, 9 for N <= 64
  double acc[MAXB][8];
#pragma unroll
  for (int b = 0; b < MAXB; ++b)
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[b][k] = 0.0;
  auto fill = [&](long p0, cplx<R>* t) {
    const int ts = (int)((vol - p0) < GT ? (vol - p0) : GT);
    for (int e = threadIdx.x; e < N * GT; e += blockDim.x) {
      const int i = e / GT, s = e - i * GT;
      if (!DB || s >= ts) t[i * (GT + 1) + s] = s < ts ? base[(size_t)i * vol + p0 + s] : cplx<R>{(R)0, (R)0};
      else cp_async_elem(t + i * (GT + 1) + s, base + (size_t)i * vol + p0 + s, (int)sizeof(cplx<R>));
    }
    if (DB) asm volatile("cp.async.commit_group;" ::: "memory");
  };
  const size_t tsz = (size_t)N * (GT + 1);
  if (DB) fill(0, tiles);
  int buf = 0;
  for (long p0 = 0; p0 < vol; p0 += GT, buf ^= 1) {
    cplx<R>* tile = tiles + (DB ? buf : 0) * tsz;
    if (DB) {
      __syncthreads();  // every thread is done with the tile the next copies overwrite
      if (p0 + GT < vol) fill(p0 + GT, tiles + (buf ^ 1) * tsz);
      else asm volatile("cp.async.commit_group;" ::: "memory");
      asm volatile("cp.async.wait_group 1;" ::: "memory");  // every group but the newest has landed
      __syncthreads();
    } else {
      __syncthreads();
      fill(p0, tile);
      __syncthreads();
    }
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
      const int blk = lane64 + 64 * b;
      if (blk >= nblk) break;
      // blk -> (bi, bj), bi <= bj, row-major over the upper triangle
      int bi = 0, rem = blk;
      while (rem >= nb - bi) {
        rem -= nb - bi;
        ++bi;
      }
      const int bj = bi + rem;
      const int i0 = 2 * bi, j0 = 2 * bj;
      const int i1 = i0 + 1 < N ? i0 + 1 : i0, j1 = j0 + 1 < N ? j0 + 1 : j0;
      R s[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) s[k] = (R)0;
      for (int q = grp; q < GT; q += 4) {
        const cplx<R> a0 = tile[i0 * (GT + 1) + q], a1 = tile[i1 * (GT + 1) + q];
        const cplx<R> b0 = tile[j0 * (GT + 1) + q], b1 = tile[j1 * (GT + 1) + q];
        // conj(a) b: two fused multiply-adds per component
        s[0] = fma(a0.re, b0.re, s[0]);
        s[0] = fma(a0.im, b0.im, s[0]);
        s[1] = fma(a0.re, b0.im, s[1]);
        s[1] = fma(-a0.im, b0.re, s[1]);
        s[2] = fma(a0.re, b1.re, s[2]);
        s[2] = fma(a0.im, b1.im, s[2]);
        s[3] = fma(a0.re, b1.im, s[3]);
        s[3] = fma(-a0.im, b1.re, s[3]);
        s[4] = fma(a1.re, b0.re, s[4]);
        s[4] = fma(a1.im, b0.im, s[4]);
        s[5] = fma(a1.re, b0.im, s[5]);
        s[5] = fma(-a1.im, b0.re, s[5]);
        s[6] = fma(a1.re, b1.re, s[6]);
        s[6] = fma(a1.im, b1.im, s[6]);
        s[7] = fma(a1.re, b1.im, s[7]);
        s[7] = fma(-a1.im, b1.re, s[7]);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[b][k] += (double)s[k];
    }
  }
  // sum the four site quarters through shared memory, write the upper triangle
  __syncthreads();
  double* red = reinterpret_cast<double*>(gsm);  // [nblk][8] (fits: tile area >= 9 KB)
  for (int g = 0; g < 4; ++g) {
    if (grp == g) {
#pragma unroll
      for (int b = 0; b < MAXB; ++b) {
        const int blk = lane64 + 64 * b;
        if (blk >= nblk) break;
#pragma unroll
        for (int k = 0; k < 8; ++k) red[blk * 8 + k] = (g == 0 ? 0.0 : red[blk * 8 + k]) + acc[b][k];
      }
    }
    __syncthreads();
  }
  for (int blk = threadIdx.x; blk < nblk; blk += blockDim.x) {
    int bi = 0, rem = blk;
    while (rem >= nb - bi) {
      rem -= nb - bi;
      ++bi;
    }
    const int bj = bi + rem;
    for (int u = 0; u < 2; ++u)
      for (int v = 0; v < 2; ++v) {
        const int i = 2 * bi + u, j = 2 * bj + v;
        if (i >= N || j >= N || i > j) continue;
        double* g = G + 2 * ((c * N + i) * (long)N + j);
        g[0] = red[blk * 8 + 4 * u + 2 * v];
        g[1] = red[blk * 8 + 4 * u + 2 * v + 1];
      }
  }
}

// Per configuration: Cholesky G = R^H R (R upper), Rinv = R^{-1}, and
// logR[c][i] += log R_ii.  One thread per configuration; G is overwritten
// with Rinv.  A non-positive pivot marks the configuration with NaN in logR.
// f32_apply: the orbitals are FP32 and Rinv will be applied rounded to FP32;
// the leading-minor identity det S_n(Psi) = det S_n(Psi Rinv) / prod_{i<n}
// Rinv_ii then holds for the ROUNDED diagonal, so logR accumulates
// -log(float(Rinv_ii)) instead of log R_ii.
__global__ void chol_inv_kernel(double* __restrict__ G, int N, int nconf, double* __restrict__ logR, int f32_apply) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nconf; c += gridDim.x * blockDim.x) {
    double* g = G + 2L * c * N * N;
    auto re = [&](int i, int j) -> double& { return g[2 * (i * N + j)]; };
    auto im = [&](int i, int j) -> double& { return g[2 * (i * N + j) + 1]; };
    // Cholesky in place, upper triangle: G = R^H R
    bool ok = true;
    for (int i = 0; i < N && ok; ++i) {
      double d = re(i, i);
      for (int k = 0; k < i; ++k) d -= re(k, i) * re(k, i) + im(k, i) * im(k, i);
      if (!(d > 0.0)) {
        ok = false;
        break;
      }
      const double rii = sqrt(d);
      re(i, i) = rii;
      im(i, i) = 0.0;
      for (int j = i + 1; j < N; ++j) {
        // R_ij = (G_ij - sum_k conj(R_ki) R_kj) / R_ii
        double sr = re(i, j), si = im(i, j);
        for (int k = 0; k < i; ++k) {
          const double ar = re(k, i), ai = -im(k, i), br = re(k, j), bi = im(k, j);
          sr -= ar * br - ai * bi;
          si -= ar * bi + ai * br;
        }
        re(i, j) = sr / rii;
        im(i, j) = si / rii;
      }
    }
    if (!ok) {
      for (int i = 0; i < N; ++i) logR[(long)c * N + i] = nan("");
      continue;
    }
    if (!f32_apply)
      for (int i = 0; i < N; ++i) logR[(long)c * N + i] += log(re(i, i));
    // Rinv (upper triangular) by back substitution, column by column, into
    // the lower-left (unused) storage is not possible for complex R; invert
    // in place row by row from the bottom: Rinv_ii = 1/R_ii,
    // Rinv_ij = -(sum_{k=i+1..j} R_ik Rinv_kj) / R_ii for j > i.
    for (int i = N - 1; i >= 0; --i) {
      const double rii = re(i, i);
      for (int j = N - 1; j > i; --j) {
        double sr = 0, si = 0;
        for (int k = i + 1; k <= j; ++k) {
          const double ar = re(i, k), ai = im(i, k), br = re(k, j), bi = im(k, j);
          sr += ar * br - ai * bi;
          si += ar * bi + ai * br;
        }
        re(i, j) = -sr / rii;
        im(i, j) = -si / rii;
      }
      re(i, i) = 1.0 / rii;
    }
    if (f32_apply)
      for (int i = 0; i < N; ++i) logR[(long)c * N + i] -= log((double)(float)re(i, i));
  }
}

// Register-blocked variant for FP32 orbitals and N <= 20: thread (pair, g)
// accumulates one 4 x 4 block (rows 4 bi.., columns 4 bj.., bi <= bj) of G
// over the sites g, g + NG, .. of every tile -- 8 shared-memory loads per 64
// FMAs instead of 4 per 16, as packed FP32x2 FMAs -- in FP32 over 32 sites
// (4 tiles), then in FP64;
// the NG = 16 site groups of a pair (16 adjacent lanes of one warp) are
// summed by shuffles in FP64 at the end.
// Tile rows N .. 19 are zero, so partial blocks need no special case.
constexpr int G4_ROWS = 20;  // 5 row blocks of 4
constexpr int G4_NG = 16;    // site groups per block pair
__global__ void __launch_bounds__(256, 2) gram4_kernel(const void* __restrict__ psi, int N, long vol,
                                                  double* __restrict__ G) {
  extern __shared__ __align__(16) unsigned char gsm[];
  float2* tiles = reinterpret_cast<float2*>(gsm);  // [2][G4_ROWS][GT + 1]
  constexpr int TS = G4_ROWS * (GT + 1);
  const long c = blockIdx.x;
  const float2* base = reinterpret_cast<const float2*>(psi) + (size_t)c * N * vol;
  const int nb = (N + 3) / 4, npairs = nb * (nb + 1) / 2;
  const int g = threadIdx.x % G4_NG, pair = threadIdx.x / G4_NG;
  const bool active = pair < npairs;
  int bi = 0, rem = active ? pair : 0;
  while (rem >= nb - bi) {
    rem -= nb - bi;
    ++bi;
  }
  const int bj = bi + rem;
  for (int e = threadIdx.x; e < 2 * (G4_ROWS - N) * (GT + 1); e += blockDim.x) {  // zero rows N..
    const int b = e / ((G4_ROWS - N) * (GT + 1)), r = e % ((G4_ROWS - N) * (GT + 1));
    tiles[b * TS + N * (GT + 1) + r] = make_float2(0.f, 0.f);
  }
  auto fill = [&](long p0, float2* t) {
    const int ts = (int)((vol - p0) < GT ? (vol - p0) : GT);
    for (int e = threadIdx.x; e < N * GT; e += blockDim.x) {
      const int i = e / GT, q = e - i * GT;
      if (q >= ts) t[i * (GT + 1) + q] = make_float2(0.f, 0.f);
      else cp_async_elem(t + i * (GT + 1) + q, base + (size_t)i * vol + p0 + q, 8);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // FP32 partial sums over 4 tiles (32 sites per thread), then FP64
  double acc[32];
  float2 s[16];  // (re, im) of the 4 x 4 block, FP32 over 4 tiles
#pragma unroll
  for (int k = 0; k < 32; ++k) acc[k] = 0.0;
#pragma unroll
  for (int k = 0; k < 16; ++k) s[k] = make_float2(0.f, 0.f);
  fill(0, tiles);
  int buf = 0, ntile = 0;
  for (long p0 = 0; p0 < vol; p0 += GT, buf ^= 1, ++ntile) {
    const float2* tile = tiles + buf * TS;
    __syncthreads();  // every thread is done with the tile the next copies overwrite
    if (p0 + GT < vol) fill(p0 + GT, tiles + (buf ^ 1) * TS);
    else asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncthreads();
    if (active) {
      const float2* ta = tile + 4 * bi * (GT + 1) + g;
      const float2* tb = tile + 4 * bj * (GT + 1) + g;
#pragma unroll
      for (int k = 0; k < GT / G4_NG; ++k) {
        float2 a[4], b[4], bn[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          a[u] = ta[u * (GT + 1) + G4_NG * k];
          b[u] = tb[u * (GT + 1) + G4_NG * k];
          bn[u] = make_float2(b[u].y, -b[u].x);
        }
        // conj(a_u) b_v = (a.x b.x + a.y b.y, a.x b.y - a.y b.x): two packed FMAs
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float2 ax = make_float2(a[u].x, a[u].x), ay = make_float2(a[u].y, a[u].y);
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            s[4 * u + v] = __ffma2_rn(ax, b[v], s[4 * u + v]);
            s[4 * u + v] = __ffma2_rn(ay, bn[v], s[4 * u + v]);
          }
        }
      }
      if ((ntile & 3) == 3 || p0 + GT >= vol) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          acc[2 * k] += (double)s[k].x;
          acc[2 * k + 1] += (double)s[k].y;
          s[k] = make_float2(0.f, 0.f);
        }
      }
    }
  }
  // sum the 16 site groups of a pair (adjacent lanes) and write the upper triangle
#pragma unroll
  for (int k = 0; k < 32; ++k)
    for (int o = G4_NG / 2; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if (active && g == 0)
    for (int u = 0; u < 4; ++u)
      for (int v = 0; v < 4; ++v) {
        const int i = 4 * bi + u, j = 4 * bj + v;
        if (i >= N || j >= N || i > j) continue;
        double* out = G + 2 * ((c * N + i) * (long)N + j);
        out[0] = acc[2 * (4 * u + v)];
        out[1] = acc[2 * (4 * u + v) + 1];
      }
}

// psi_{c,t}(p) <- sum_{i <= t} psi_{c,i}(p) Rinv[i][t]; one thread per site,
// all N orbitals of a configuration in registers (N <= 64), arithmetic in R
// (FP32 orbitals: Rinv rounded to FP32, see chol_inv_kernel).
template <typename R, int NMAX>
__global__ void __launch_bounds__(256) apply_rinv_kernel(void* __restrict__ psi, int N, long vol, int nconf,
                                                          const double* __restrict__ Rinv) {
  // R^-1 of this block's configuration: 2 N^2 values in R (FP64), or for FP32
  // N^2 float4 (re, re, im, im) entries that feed packed FMAs
  extern __shared__ __align__(16) double rs_raw[];
  R* rs = reinterpret_cast<R*>(rs_raw);
  const long sites_per_block = blockDim.x;
  const long blocks_per_conf = (vol + sites_per_block - 1) / sites_per_block;
  const long c = blockIdx.x / blocks_per_conf;
  if (c >= nconf) return;
  const long p = (blockIdx.x % blocks_per_conf) * sites_per_block + threadIdx.x;
  const bool live = p < vol;
  cplx<R>* base = reinterpret_cast<cplx<R>*>(psi) + (size_t)c * N * vol + (live ? p : 0);
  // the orbital loads go out first; their latency covers the fill of R below
  R xr[NMAX], xi[NMAX];
#pragma unroll
  for (int i = 0; i < NMAX; ++i)
    if (i < N && live) {
      cplx<R> v = base[(size_t)i * vol];
      xr[i] = v.re;
      xi[i] = v.im;
    }
  if constexpr (sizeof(R) == 4) {
    // x r = (xr ar - xi ai, xr ai + xi ar): with X = (xr, xi) the packed sums
    // s = sum X (ar, ar) and u = sum X (ai, ai) give re = s.x - u.y, im = s.y + u.x
    float4* r4 = reinterpret_cast<float4*>(rs_raw);
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
      const float ar = (float)Rinv[2L * (c * N * N + e)], ai = (float)Rinv[2L * (c * N * N + e) + 1];
      r4[e] = make_float4(ar, ar, ai, ai);
    }
    __syncthreads();
    if (!live) return;
#pragma unroll
    for (int t = NMAX - 1; t >= 0; --t) {
      if (t >= N) continue;
      float2 sa = make_float2(0.f, 0.f), ua = make_float2(0.f, 0.f);
#pragma unroll
      for (int i = 0; i <= t; ++i) {
        const float4 r = r4[i * N + t];
        const float2 x = make_float2(xr[i], xi[i]);
        sa = __ffma2_rn(x, make_float2(r.x, r.y), sa);
        ua = __ffma2_rn(x, make_float2(r.z, r.w), ua);
      }
      base[(size_t)t * vol] = cplx<R>{sa.x - ua.y, sa.y + ua.x};
    }
  } else {
    for (int e = threadIdx.x; e < 2 * N * N; e += blockDim.x) rs[e] = (R)Rinv[2L * c * N * N + e];
    __syncthreads();
    if (!live) return;
#pragma unroll
    for (int t = NMAX - 1; t >= 0; --t) {
      if (t >= N) continue;
      R sr = 0, si = 0;
#pragma unroll
      for (int i = 0; i <= t; ++i) {
        const R ar = rs[2 * (i * N + t)], ai = rs[2 * (i * N + t) + 1];
        sr = fma(xr[i], ar, sr);
        sr = fma(-xi[i], ai, sr);
        si = fma(xr[i], ai, si);
        si = fma(xi[i], ar, si);
      }
      base[(size_t)t * vol] = cplx<R>{(R)sr, (R)si};
    }
  }
}

// The determinants measured at slice t on the re-orthonormalised orbitals
// Q = Psi R^-1, turned into those of Psi, with S_n = sum_{i<=n} log R_ii:
//  mode 0 (SlaterDet::Run, S = <src|Psi> = <src|Q> R):
//    dets[c][t][n]    *= exp(S_n)                      (det S_{n+1})
//  mode 1 (SlaterDet2::Run on the pair matrix Phi(Psi) = R^T Phi(Q) R, whose
//  column n is replaced by v_s = <src_n|psi_s>, v(Psi) = R^T v(Q)):
//    dets[c][t][2n+1] *= exp(2 S_n)                    (det Phi_{n+1})
//    dets[c][t][2n]   *= exp(S_n + S_{n-1})            (det R_{n+1} det R_n)
// (slater_det2.C:78-148; R upper triangular, so the leading blocks of R^T
// Phi R involve only the leading blocks of R).
__global__ void rescale_dets_kernel(double* dets, const double* logR, int N, int nconf, long conf_stride,
                                    long offset, int mode) {
  const long total = (long)nconf * N;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long c = e / N;
    const int n = (int)(e % N);
    double s = 0;
    for (int i = 0; i < n; ++i) s += logR[c * N + i];
    const double s_prev = s;  // S_{n-1}
    s += logR[c * N + n];     // S_n
    double* base = dets + c * conf_stride + offset;
    if (mode == 0) {
      const double f = exp(s);
      base[2L * n] *= f;
      base[2L * n + 1] *= f;
    } else {
      const double f1 = exp(2.0 * s), f0 = exp(s + s_prev);
      base[2L * (2 * n + 1)] *= f1;
      base[2L * (2 * n + 1) + 1] *= f1;
      base[2L * (2 * n)] *= f0;
      base[2L * (2 * n) + 1] *= f0;
    }
  }
}

template <int NMAX>
static nrcps_status launch_apply(nrcps_context* ctx, void* psi, int N, long vol, int nconf, nrcps_precision prec,
                                 const double* Rinv) {
  const long bpc = (vol + 255) / 256;
  const size_t sh = sizeof(double) * 2 * N * N;
  if (prec == NRCPS_F64)
    apply_rinv_kernel<double, NMAX><<<(unsigned)(bpc * nconf), 256, sh, ctx->stream>>>(psi, N, vol, nconf, Rinv);
  else
    apply_rinv_kernel<float, NMAX><<<(unsigned)(bpc * nconf), 256, sh, ctx->stream>>>(psi, N, vol, nconf, Rinv);
  ctx->launches++;
  return check_launch(ctx, "apply_rinv_kernel");
}

// One re-orthonormalisation of nconf configurations of N orbitals.
// G: scratch of nconf * N * N complex doubles; logR accumulates.
nrcps_status qr_reorthonormalise(nrcps_context* ctx, void* psi, int N, long vol, int nconf, nrcps_precision prec,
                                 double* G, double* logR) {
  if (N > 64) return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "QR re-orthonormalisation supports N <= 64");
  if (prec == NRCPS_F32 && ctx->qr_gram_tc && gram_tc_supported(N, vol, nconf)) {
    NRCPS_TRY(gram_tc(ctx, psi, N, vol, nconf, G));  // tcgen05, TF32 hi/lo (gram_tc.cu)
  } else {
    const size_t esz = prec == NRCPS_F64 ? sizeof(cplx<double>) : sizeof(cplx<float>);
    const size_t tile_bytes = esz * (size_t)N * (GT + 1);
    const bool db = 2 * tile_bytes <= 200 * 1024;
    size_t sh = db ? 2 * tile_bytes : tile_bytes;
    const size_t red = sizeof(double) * 8 * 528;
    if (sh < red) sh = red;
    auto launch = [&](auto kern) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      kern<<<(unsigned)nconf, 256, sh, ctx->stream>>>(psi, N, vol, G);
    };
    if (prec == NRCPS_F64) {
      if (N <= 22) launch(gram_tile_kernel<double, 2, true>);
      else if (N <= 32) launch(gram_tile_kernel<double, 3, true>);
      else if (db) launch(gram_tile_kernel<double, 9, true>);
      else launch(gram_tile_kernel<double, 9, false>);
    } else if (N <= G4_ROWS) {
      const size_t sh4 = sizeof(float2) * 2 * G4_ROWS * (GT + 1);
      cudaFuncSetAttribute(gram4_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh4);
      gram4_kernel<<<(unsigned)nconf, 256, sh4, ctx->stream>>>(psi, N, vol, G);
    } else {
      if (N <= 22) launch(gram_tile_kernel<float, 2, true>);
      else if (N <= 32) launch(gram_tile_kernel<float, 3, true>);
      else launch(gram_tile_kernel<float, 9, true>);
    }
    ctx->launches++;
    NRCPS_TRY(check_launch(ctx, "gram_tile_kernel"));
  }
  chol_inv_kernel<<<grid_for(nconf, 64), 64, 0, ctx->stream>>>(G, N, nconf, logR, prec == NRCPS_F32);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "chol_inv_kernel"));
  if (N <= 8) return launch_apply<8>(ctx, psi, N, vol, nconf, prec, G);
  if (N <= 16) return launch_apply<16>(ctx, psi, N, vol, nconf, prec, G);
  if (N <= 24) return launch_apply<24>(ctx, psi, N, vol, nconf, prec, G);
  if (N <= 40) return launch_apply<40>(ctx, psi, N, vol, nconf, prec, G);
  return launch_apply<64>(ctx, psi, N, vol, nconf, prec, G);
}

nrcps_status rescale_dets(nrcps_context* ctx, double* dets, const double* logR, int N, int nconf, long conf_stride,
                          long offset, int mode) {
  rescale_dets_kernel<<<grid_for((long)nconf * N, 256), 256, 0, ctx->stream>>>(dets, logR, N, nconf, conf_stride,
                                                                               offset, mode);
  ctx->launches++;
  return check_launch(ctx, "rescale_dets_kernel");
}

}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_reorthonormalise(nrcps_context* ctx, void* dev_psi, int N, long vol, int nconf,
                                               nrcps_precision prec, double* dev_work, double* dev_logR) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, N > 0 && vol > 0 && nconf >= 0 && (prec == NRCPS_F32 || prec == NRCPS_F64),
                "nrcps_reorthonormalise: bad arguments");
  if (nconf == 0) return NRCPS_OK;
  NRCPS_REQUIRE(ctx, dev_psi && dev_work && dev_logR, "nrcps_reorthonormalise: null pointer");
  return qr_reorthonormalise(ctx, dev_psi, N, vol, nconf, prec, dev_work, dev_logR);
}

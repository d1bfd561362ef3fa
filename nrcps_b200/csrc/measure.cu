// measure.cu -- Slater-matrix fills and determinants (the measurement half of
// every time slice): overlaps S = <src|psi>, the pair matrix of TwoBody, and
// FP64 LU of every leading minor with the reference's pivoting rule.
#include <cooperative_groups.h>

#include "common.cuh"

namespace nrcps {
namespace cg = cooperative_groups;

// ---------------------------------------------------------------- overlap
// One block per (configuration, orbital t); sources in chunks of 8.  FP64
// accumulation for both orbital precisions.
template <typename R>
__global__ void __launch_bounds__(256) overlap_kernel(const double* __restrict__ src, int ns,
                                                      const void* __restrict__ psi, int nt, long vol,
                                                      double* __restrict__ S) {
  const long ct = blockIdx.x;  // conf * nt + t
  const long conf = ct / nt;
  const int t = (int)(ct % nt);
  const char* p = reinterpret_cast<const char*>(psi) + (size_t)ct * vol * 2 * sizeof(R);
  __shared__ double red[8][2][8];
  for (int s0 = 0; s0 < ns; s0 += 8) {
    double ar[8], ai[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) ar[k] = ai[k] = 0.0;
    for (long i = threadIdx.x; i < vol; i += blockDim.x) {
      cplx<R> q = ld<R>(p, i);
      double qr = (double)q.re, qi = (double)q.im;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (s0 + k < ns) {
          double2 a = reinterpret_cast<const double2*>(src)[(long)(s0 + k) * vol + i];
          ar[k] = fma(a.x, qr, ar[k]);  // two fused multiply-adds per component
          ar[k] = fma(a.y, qi, ar[k]);
          ai[k] = fma(a.x, qi, ai[k]);
          ai[k] = fma(-a.y, qr, ai[k]);
        }
      }
    }
    // warp reduce then block reduce
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      for (int off = 16; off > 0; off >>= 1) {
        ar[k] += __shfl_down_sync(0xffffffffu, ar[k], off);
        ai[k] += __shfl_down_sync(0xffffffffu, ai[k], off);
      }
    }
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (ln == 0) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        red[warp][0][k] = ar[k];
        red[warp][1][k] = ai[k];
      }
    }
    __syncthreads();
    if (threadIdx.x < 8 && s0 + (int)threadIdx.x < ns) {
      const int k = threadIdx.x;
      double sr = 0.0, si = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        sr += red[w][0][k];
        si += red[w][1][k];
      }
      long o = ((conf * ns + (s0 + k)) * (long)nt + t) * 2;
      S[o] = sr;
      S[o + 1] = si;
    }
    __syncthreads();
  }
}

// Plane-wave sources: S[c][s][t] = psi_{c,t}(p_s) exactly.
template <typename R>
__global__ void gather_kernel(const int* __restrict__ index, int ns, const void* __restrict__ psi, int nt,
                              int nconf, long vol, double* __restrict__ S) {
  long total = (long)nconf * ns * nt;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long conf = e / ((long)ns * nt);
    int s = (int)((e / nt) % ns), t = (int)(e % nt);
    const int p = index[s];
    // a lattice index outside [0, vol) has no overlap with the orbitals
    cplx<R> q = (p >= 0 && p < vol) ? ld<R>(psi, ((conf * nt + t) * vol) + p) : cplx<R>{(R)0, (R)0};
    S[2 * e] = (double)q.re;
    S[2 * e + 1] = (double)q.im;
  }
}

// ------------------------------------------------------------ pair matrix
// One block per (configuration, s, t): phi = sum_i w_i psi1_s(i) psi2_t(opp(i)).
template <typename R>
__global__ void __launch_bounds__(256) pair_kernel(const void* __restrict__ psi1, const void* __restrict__ psi2,
                                                   int n, long vol, const double* __restrict__ w,
                                                   const int* __restrict__ opp, double* __restrict__ phi) {
  const long e = blockIdx.x;  // (conf * n + s) * n + t
  const long conf = e / ((long)n * n);
  const int s = (int)((e / n) % n), t = (int)(e % n);
  const char* a = reinterpret_cast<const char*>(psi1) + (size_t)(conf * n + s) * vol * 2 * sizeof(R);
  const char* b = reinterpret_cast<const char*>(psi2) + (size_t)(conf * n + t) * vol * 2 * sizeof(R);
  double re = 0.0, im = 0.0;
  for (long i = threadIdx.x; i < vol; i += blockDim.x) {
    const int j = opp[i];
    if (j < 0 || j >= vol) continue;  // a partner outside the lattice contributes nothing
    cplx<R> x = ld<R>(a, i), y = ld<R>(b, j);
    double wi = w[i];
    re += ((double)x.re * y.re - (double)x.im * y.im) * wi;
    im += ((double)x.re * y.im + (double)x.im * y.re) * wi;
  }
  __shared__ double red[2][8];
  for (int off = 16; off > 0; off >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, off);
    im += __shfl_down_sync(0xffffffffu, im, off);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = re;
    red[1][threadIdx.x >> 5] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sr = 0, si = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      sr += red[0][k];
      si += red[1][k];
    }
    phi[2 * e] = sr;
    phi[2 * e + 1] = si;
  }
}

// Tiled pair matrices for n <= 32 (the path of nrcps_pair_matrix and of the
// ensemble's pair sink).  One thread-block cluster of up to eight CTAs per
// configuration; CTA r of C takes every C-th tile of ts sites.
//
// TwoBody's opposite-parity index is an involution (opp(opp(i)) = i), so the
// sites pair up: a tile stages, for every site i of the tile with i <= opp(i),
// the term of i, a_s = w_i psi1_s(i) and b_t = psi2_t(opp(i)), and (when
// i < opp(i)) the term of j = opp(i), a_s = w_j psi1_s(j) and b_t = psi2_t(i).
// Every term is summed exactly once and every orbital element is read once
// (the gathered rows are the rows the pair's other term reads directly);
// tiles whose sites all have i > opp(i) are skipped after reading opp.  When
// `bad_opp` points at a nonzero word (the table is not an involution) the
// tiles stage the term of every site instead: the plain gather.
//
// Thread (block, group) accumulates a 2 x 2 block of phi over the group's
// slots of every tile, in R within a tile and in FP64 across tiles; the
// groups are summed in shared memory and the cluster's CTAs in rank order
// through distributed shared memory: the result does not depend on timing.
//
// With psi1 = psi2 and a weight even under the pairing (w(opp(i)) = w(i),
// TwoBody's tables), the pair of terms of i and opp(i) is symmetric in
// (s, t), so phi is: only the blocks on and above the diagonal are summed
// and each is written to both triangles.
constexpr int PAIR_THREADS = 256;
constexpr int PAIR_MAXN = 32;
constexpr int PB = 2;                // register block: PB x PB complex pair-matrix entries per thread
constexpr int PAIR_E = PB * PB * 2;  // doubles per block

template <typename R>
struct PairShape {
  static int rows(int n) { return (n + PB - 1) / PB * PB; }  // staged rows, padded to whole blocks
  // sites per tile: at most about 20 KB of staged rows per array (four CTAs per SM)
  static int ts(int n) {
    const int budget = (sizeof(R) == 4 ? 1280 : 640) / rows(n);
    int t = 16;
    while (t * 2 <= budget && t < 128) t *= 2;
    return t;
  }
  static int ld(int n) { return 2 * ts(n) + 1; }  // slots per staged row, padded: rows start in different banks
  static size_t smem(int n) {
    const size_t t = 2 * (size_t)rows(n) * ld(n) * sizeof(cplx<R>);
    const size_t nb = rows(n) / PB, red = nb * nb * PAIR_E * sizeof(double);
    return t > red ? t : red;
  }
};

// Block blk of the upper triangle (row-major, bi <= bj) or of the full
// nb x nb grid
__device__ __forceinline__ void pair_block(int blk, int nb, bool sym, int& bi, int& bj) {
  if (!sym) {
    bi = blk / nb;
    bj = blk % nb;
    return;
  }
  bi = 0;
  while (blk >= nb - bi) {
    blk -= nb - bi;
    ++bi;
  }
  bj = bi + blk;
}

// The end of a tiled pair kernel: the groups of every block summed in shared
// memory (fixed order), then the cluster's CTAs in rank order through
// distributed shared memory, written by rank 0 (to both triangles for the
// symmetric form).
__device__ __forceinline__ void pair_reduce_store(const double (&acc)[PB][PB][2], unsigned char* smem, int n,
                                                  int nb, bool sym, int nblk, int groups, int g, int blk,
                                                  bool active, long conf, double* __restrict__ phi) {
  cg::cluster_group cluster = cg::this_cluster();
  const int split = (int)cluster.num_blocks(), rank = (int)cluster.block_rank();
  __syncthreads();
  double* red = reinterpret_cast<double*>(smem);  // [nblk][PAIR_E], over the staged tiles
  for (int gg = 0; gg < groups; ++gg) {
    if (active && g == gg) {
#pragma unroll
      for (int a = 0; a < PB; ++a)
#pragma unroll
        for (int b = 0; b < PB; ++b)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const int e = blk * PAIR_E + (a * PB + b) * 2 + c;
            red[e] = (gg == 0 ? 0.0 : red[e]) + acc[a][b][c];
          }
    }
    __syncthreads();
  }
  cluster.sync();  // every CTA's sums are in its shared memory
  if (rank == 0) {
    for (int e = threadIdx.x; e < nblk * PAIR_E; e += PAIR_THREADS) {
      double v = 0.0;
      for (int r2 = 0; r2 < split; ++r2) v += cluster.map_shared_rank(red, r2)[e];
      const int k = e % PAIR_E;
      int bi, bj;
      pair_block(e / PAIR_E, nb, sym, bi, bj);
      const int s = PB * bi + (k / 2) / PB, t = PB * bj + (k / 2) % PB;
      // (the symmetric form writes each entry with s <= t to both places)
      if (s < n && t < n && (!sym || s <= t)) {
        phi[2 * ((conf * n + s) * (long)n + t) + (k & 1)] = v;
        if (sym && s != t) phi[2 * ((conf * n + t) * (long)n + s) + (k & 1)] = v;
      }
    }
  }
  cluster.sync();  // peers keep their shared memory until rank 0 has read it
}

template <typename R>
__global__ void __launch_bounds__(PAIR_THREADS, 4)
    pair_tile_kernel(const void* __restrict__ psi1, const void* __restrict__ psi2, int n, long vol,
                     const double* __restrict__ w, const int* __restrict__ opp, const int* __restrict__ flags,
                     int host_flags, int ts, double* __restrict__ phi) {
  extern __shared__ __align__(16) unsigned char pair_smem[];
  const int LD = 2 * ts + 1;
  const int nb = (n + PB - 1) / PB, rows = nb * PB;
  cplx<R>* A = reinterpret_cast<cplx<R>*>(pair_smem);  // [rows][LD]: w psi1 of each slot's term
  cplx<R>* B = A + (size_t)rows * LD;                   // [rows][LD]: psi2 at the term's partner site
  cg::cluster_group cluster = cg::this_cluster();
  const int split = (int)cluster.num_blocks(), rank = (int)cluster.block_rank();
  const long conf = blockIdx.x / split;
  const cplx<R>* p1 = reinterpret_cast<const cplx<R>*>(psi1) + (size_t)conf * n * vol;
  const cplx<R>* p2 = reinterpret_cast<const cplx<R>*>(psi2) + (size_t)conf * n * vol;
  // the table's properties: bit 0 opp is no involution, bit 1 w is not even
  // under opp (from the device check when there is one)
  const int fl = flags ? *flags : host_flags;
  const bool paired = !(fl & 1);
  const bool sym = paired && !(fl & 2) && psi1 == psi2;
  // staging: thread -> (slot q of the tile, orbital lane)
  const int q = threadIdx.x % ts, olane = threadIdx.x / ts, ostride = PAIR_THREADS / ts;
  // accumulation: thread -> (PB x PB block, group), blocks fastest: the
  // lanes of a warp read one slot of at most 2 nb rows, in distinct banks
  const int nblk = sym ? nb * (nb + 1) / 2 : nb * nb;
  const int groups = PAIR_THREADS / nblk;  // >= 1 for n <= 32
  const int g = threadIdx.x / nblk, blk = threadIdx.x % nblk;
  const bool active = g < groups;
  int bi = 0, bj = 0;
  if (active) pair_block(blk, nb, sym, bi, bj);
  const int abase = bi * PB * LD, bbase = bj * PB * LD;
  for (int e = threadIdx.x; e < (rows - n) * LD; e += PAIR_THREADS) {  // the padding row stays zero
    A[n * LD + e] = cplx<R>{(R)0, (R)0};
    B[n * LD + e] = cplx<R>{(R)0, (R)0};
  }
  double acc[PB][PB][2];
#pragma unroll
  for (int a = 0; a < PB; ++a)
#pragma unroll
    for (int b = 0; b < PB; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  const long ntiles = (vol + ts - 1) / ts;
  for (long tile = rank; tile < ntiles; tile += split) {
    const long i = tile * ts + q;
    const bool valid = i < vol;
    const long j = valid ? (long)__ldg(opp + i) : 0;
    // (the plain gather skips a partner outside the lattice; a paired table
    // has none)
    const bool take = valid && (paired ? i <= j : (j >= 0 && j < vol));
    const bool second = paired && valid && i < j;
    // also the barrier after the previous tile's accumulation
    if (!__syncthreads_or(take)) continue;
    const R wi = take ? (R)__ldg(w + i) : (R)0, wj = second ? (R)__ldg(w + j) : (R)0;
#pragma unroll 4
    for (int o = olane; o < n; o += ostride) {
      const cplx<R>* r1 = p1 + (size_t)o * vol;
      const cplx<R>* r2 = p2 + (size_t)o * vol;
      cplx<R> a1{(R)0, (R)0}, b1{(R)0, (R)0}, a2{(R)0, (R)0}, b2{(R)0, (R)0};
      if (take) {
        a1 = r1[i];
        b1 = r2[j];
      }
      if (second) {
        a2 = r1[j];
        b2 = r2[i];
      }
      A[o * LD + q] = cplx<R>{a1.re * wi, a1.im * wi};
      B[o * LD + q] = b1;
      A[o * LD + ts + q] = cplx<R>{a2.re * wj, a2.im * wj};
      B[o * LD + ts + q] = b2;
    }
    __syncthreads();
    if (active) {
      // sum over the slots of a_s b_t (complex, no conjugation) in R: two
      // fused multiply-adds per real component; then into the FP64 sums
      R r[PB][PB][2];
#pragma unroll
      for (int a = 0; a < PB; ++a)
#pragma unroll
        for (int b = 0; b < PB; ++b) r[a][b][0] = r[a][b][1] = (R)0;
      for (int slot = g; slot < 2 * ts; slot += groups) {
        cplx<R> av[PB], bv[PB];
#pragma unroll
        for (int k = 0; k < PB; ++k) {
          av[k] = A[abase + k * LD + slot];
          bv[k] = B[bbase + k * LD + slot];
        }
#pragma unroll
        for (int a = 0; a < PB; ++a)
#pragma unroll
          for (int b = 0; b < PB; ++b) {
            r[a][b][0] = fma(av[a].re, bv[b].re, r[a][b][0]);
            r[a][b][0] = fma(-av[a].im, bv[b].im, r[a][b][0]);
            r[a][b][1] = fma(av[a].re, bv[b].im, r[a][b][1]);
            r[a][b][1] = fma(av[a].im, bv[b].re, r[a][b][1]);
          }
      }
#pragma unroll
      for (int a = 0; a < PB; ++a)
#pragma unroll
        for (int b = 0; b < PB; ++b) {
          acc[a][b][0] += (double)r[a][b][0];
          acc[a][b][1] += (double)r[a][b][1];
        }
    }
  }
  pair_reduce_store(acc, pair_smem, n, nb, sym, nblk, groups, g, blk, active, conf, phi);
}

// *flags |= 1 unless opp is an involution of [0, vol) (TwoBody's parity
// mirror is), |= 2 unless w(opp(i)) = w(i) for every i
__global__ void opp_involution_check_kernel(const int* __restrict__ opp, const double* __restrict__ w, long vol,
                                            int* flags) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < vol; i += (long)gridDim.x * blockDim.x) {
    const int j = opp[i];
    if (j < 0 || j >= vol) {
      atomicOr(flags, 3);
    } else {
      if (opp[j] != i) atomicOr(flags, 1);
      if (w[j] != w[i]) atomicOr(flags, 2);
    }
  }
}

// GeneralizedTwoBody::Run (src/two_body/noarch/two_body_run.C:45-75) batched:
// phi[c][s][t] = sum_l sum_i wl[l][i] psi1_{c,s}(shift[l][i]) psi2_{c,t}(opp(i))
// with wl[l][i] = weight(R, l) * half_site_wavefunc[l][i] folded by the
// caller.  One block per (conf, s, t); the term loop is outermost, as in the
// reference.
template <typename R>
__global__ void __launch_bounds__(256) shifted_pair_kernel(const void* __restrict__ psi1,
                                                           const void* __restrict__ psi2, int n, long vol, int nterms,
                                                           const int* __restrict__ shift,
                                                           const double* __restrict__ wl,
                                                           const int* __restrict__ opp, double* __restrict__ phi) {
  const long e = blockIdx.x;  // (conf * n + s) * n + t
  const long conf = e / ((long)n * n);
  const int s = (int)((e / n) % n), t = (int)(e % n);
  const char* a = reinterpret_cast<const char*>(psi1) + (size_t)(conf * n + s) * vol * 2 * sizeof(R);
  const char* b = reinterpret_cast<const char*>(psi2) + (size_t)(conf * n + t) * vol * 2 * sizeof(R);
  double re = 0.0, im = 0.0;
  for (int l = 0; l < nterms; ++l) {
    const int* sh = shift + (size_t)l * vol;
    const double* w = wl + (size_t)l * vol;
    for (long i = threadIdx.x; i < vol; i += blockDim.x) {
      const int si = sh[i], j = opp[i];
      if (si < 0 || si >= vol || j < 0 || j >= vol) continue;  // outside the lattice: no term
      cplx<R> x = ld<R>(a, si), y = ld<R>(b, j);
      const double wi = w[i];
      re += ((double)x.re * y.re - (double)x.im * y.im) * wi;
      im += ((double)x.re * y.im + (double)x.im * y.re) * wi;
    }
  }
  __shared__ double red[2][8];
  for (int off = 16; off > 0; off >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, off);
    im += __shfl_down_sync(0xffffffffu, im, off);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = re;
    red[1][threadIdx.x >> 5] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sr = 0, si = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      sr += red[0][k];
      si += red[1][k];
    }
    phi[2 * e] = sr;
    phi[2 * e + 1] = si;
  }
}

// ------------------------------------------------- pointer-array variants
// mat[t + nf*s] = <kets[s] | bras[t]> (the layout of Cuda::InnerProduct,
// src/utils/cuda/cuda_utils_kernels.cu:4-48), FP64, one block per (s, t).
__global__ void __launch_bounds__(256) inner_ptrs_kernel(const double* const* __restrict__ kets,
                                                         const double* const* __restrict__ bras, int nf, long vol,
                                                         double* __restrict__ mat) {
  const int s = blockIdx.x / nf, t = blockIdx.x % nf;
  const double2* a = reinterpret_cast<const double2*>(kets[s]);
  const double2* b = reinterpret_cast<const double2*>(bras[t]);
  double re = 0.0, im = 0.0;
  for (long i = threadIdx.x; i < vol; i += blockDim.x) {
    double2 x = a[i], y = b[i];
    re = fma(x.x, y.x, re);
    re = fma(x.y, y.y, re);
    im = fma(x.x, y.y, im);
    im = fma(-x.y, y.x, im);
  }
  __shared__ double red[2][8];
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = re;
    red[1][threadIdx.x >> 5] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sr = 0, si = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      sr += red[0][k];
      si += red[1][k];
    }
    mat[2L * (t + (long)nf * s)] = sr;
    mat[2L * (t + (long)nf * s) + 1] = si;
  }
}

// phi[t + nf*s] = sum_i w_i props1[s](i) props2[t](opp(i)), FP64.
__global__ void __launch_bounds__(256) pair_ptrs_kernel(const double* const* __restrict__ p1,
                                                        const double* const* __restrict__ p2, int nf, long vol,
                                                        const double* __restrict__ w, const int* __restrict__ opp,
                                                        double* __restrict__ phi) {
  const int s = blockIdx.x / nf, t = blockIdx.x % nf;
  const double2* a = reinterpret_cast<const double2*>(p1[s]);
  const double2* b = reinterpret_cast<const double2*>(p2[t]);
  double re = 0.0, im = 0.0;
  for (long i = threadIdx.x; i < vol; i += blockDim.x) {
    double2 x = a[i], y = b[opp[i]];
    const double wi = w[i];
    re += (x.x * y.x - x.y * y.y) * wi;
    im += (x.x * y.y + x.y * y.x) * wi;
  }
  __shared__ double red[2][8];
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = re;
    red[1][threadIdx.x >> 5] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sr = 0, si = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      sr += red[0][k];
      si += red[1][k];
    }
    phi[2L * (t + (long)nf * s)] = sr;
    phi[2L * (t + (long)nf * s) + 1] = si;
  }
}

// ------------------------------------------------------------------- LU
struct dc {
  double re, im;
};
__device__ __forceinline__ dc dmul(dc a, dc b) { return dc{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ double dabs(dc a) { return hypot(a.re, a.im); }
__device__ __forceinline__ dc drecip(dc b) {
  // 1 / b with Smith's scaling
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return dc{1.0 / d, -r / d};
  }
  double r = b.re / b.im, d = b.re * r + b.im;
  return dc{r / d, -1.0 / d};
}

// Crout LU with implicit-scaled partial pivoting (src/utils/ludcmp.C:9-65)
// on the n x n matrix a (row-major, stride n).  Returns the permutation
// parity d, or 0 when a row is all zero (the reference exits there).
__device__ double ludcmp_dev(dc* a, int n, double* vv) {
  double d = 1.0;
  for (int i = 0; i < n; ++i) {
    double big = 0.0;
    for (int j = 0; j < n; ++j) {
      double t = dabs(a[n * i + j]);
      if (t > big) big = t;
    }
    if (big == 0.0) return 0.0;
    vv[i] = 1.0 / big;
  }
  int imax = 0;
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < j; ++i) {
      dc sum = a[n * i + j];
      for (int k = 0; k < i; ++k) {
        dc p = dmul(a[n * i + k], a[n * k + j]);
        sum.re -= p.re;
        sum.im -= p.im;
      }
      a[n * i + j] = sum;
    }
    double big = 0.0;
    for (int i = j; i < n; ++i) {
      dc sum = a[n * i + j];
      for (int k = 0; k < j; ++k) {
        dc p = dmul(a[n * i + k], a[n * k + j]);
        sum.re -= p.re;
        sum.im -= p.im;
      }
      a[n * i + j] = sum;
      double dum = vv[i] * dabs(sum);
      if (dum >= big) {
        big = dum;
        imax = i;
      }
    }
    if (j != imax) {
      for (int k = 0; k < n; ++k) {
        dc t = a[n * imax + k];
        a[n * imax + k] = a[n * j + k];
        a[n * j + k] = t;
      }
      d = -d;
      vv[imax] = vv[j];
    }
    if (dabs(a[n * j + j]) == 0.0) a[n * j + j] = dc{1.0e-20, 0.0};
    dc r = drecip(a[n * j + j]);
    for (int i = j + 1; i < n; ++i) a[n * i + j] = dmul(a[n * i + j], r);
  }
  return d;
}

// One thread per (matrix, measured minor).  Scratch: per thread n*n complex
// + n doubles in global memory (L2-resident).
__global__ void slater_dets_kernel(const double* __restrict__ S, const double* __restrict__ psi1, int N, int nconf,
                                   int mode, int log_det, double* __restrict__ out, double* scratch,
                                   long out_conf_stride, long out_offset) {
  const int nmeas = mode ? 2 * N : N;
  const long total = (long)nconf * nmeas;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long c = e / nmeas;
    const int m = (int)(e % nmeas);
    const int n = mode ? m / 2 + 1 : m + 1;
    const int t0 = (mode && (m % 2 == 0)) ? n - 1 : -1;
    dc* a = reinterpret_cast<dc*>(scratch + e * (2L * N * N + N));
    double* vv = scratch + e * (2L * N * N + N) + 2L * N * N;
    const dc* Sc = reinterpret_cast<const dc*>(S) + c * (long)N * N;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) a[n * i + j] = Sc[(long)N * i + j];
    if (t0 >= 0) {
      // SlaterDet2::Run column t0 from psi1[s + t0*N] (slater_det2.C:102-106)
      const dc* P = reinterpret_cast<const dc*>(psi1) + c * (long)N * N;
      for (int i = 0; i < n; ++i) a[n * i + t0] = P[i + (long)t0 * N];
    }
    double d = ludcmp_dev(a, n, vv);
    dc r;
    if (!log_det) {
      r = dc{d, 0.0};
      for (int i = 0; i < n; ++i) r = dmul(r, a[n * i + i]);
    } else {
      // log(d) + sum log(U_ii), principal branches (slater_det.C:102-109)
      r = dc{log(fabs(d)), d < 0 ? 3.14159265358979323846 : 0.0};
      for (int i = 0; i < n; ++i) {
        r.re += log(dabs(a[n * i + i]));
        r.im += atan2(a[n * i + i].im, a[n * i + i].re);
      }
    }
    if (d == 0.0) r = dc{nan(""), nan("")};  // singular: flagged to the host
    double* o = out + c * out_conf_stride + out_offset + 2L * m;
    o[0] = r.re;
    o[1] = r.im;
  }
}

// One warp per (matrix, measured minor), the minor in shared memory.  The
// same Crout factorisation with implicit-scaled partial pivoting as
// ludcmp_dev, organised right-looking: element (i, k) receives the products
// l_ij u_jk in the same order j = 0, 1, ... as Crout's running sum, the
// pivot search sees the same updated column, ties go to the last row as
// in `if (dum >= big)`, and rows swap whole -- so the factors and the
// determinant follow the same arithmetic.  Lanes split rows (pivot search,
// multipliers) and columns (swaps, trailing update); no global scratch.
constexpr int kWarpLuMaxWarps = 4;  // warps per block (fewer for large N: shared memory)

__global__ void __launch_bounds__(32 * kWarpLuMaxWarps) slater_dets_warp_kernel(const double* __restrict__ S,
                                                                            const double* __restrict__ psi1, int N,
                                                                            int nconf, int mode, int log_det,
                                                                            double* __restrict__ out,
                                                                            long out_conf_stride, long out_offset) {
  extern __shared__ __align__(16) unsigned char lu_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  dc* a = reinterpret_cast<dc*>(lu_smem) + (size_t)warp * N * N;
  double* vv = reinterpret_cast<double*>(reinterpret_cast<dc*>(lu_smem) + (size_t)wpb * N * N) + warp * N;
  const int nmeas = mode ? 2 * N : N;
  const long total = (long)nconf * nmeas;
  for (long e = (long)blockIdx.x * wpb + warp; e < total; e += (long)gridDim.x * wpb) {
    const long c = e / nmeas;
    const int m = (int)(e % nmeas);
    const int n = mode ? m / 2 + 1 : m + 1;
    const int t0 = (mode && (m % 2 == 0)) ? n - 1 : -1;
    const dc* Sc = reinterpret_cast<const dc*>(S) + c * (long)N * N;
    const dc* P = mode ? reinterpret_cast<const dc*>(psi1) + c * (long)N * N : nullptr;
    for (int idx = lane; idx < n * n; idx += 32) {
      const int i = idx / n, k = idx - i * n;
      // SlaterDet2::Run column t0 from psi1[s + t0*N] (slater_det2.C:102-106)
      a[idx] = (k == t0) ? P[i + (long)t0 * N] : Sc[(long)N * i + k];
    }
    __syncwarp();
    bool zero_row = false;
    for (int i = lane; i < n; i += 32) {
      double big = 0.0;
      for (int k = 0; k < n; ++k) big = fmax(big, dabs(a[n * i + k]));
      if (big == 0.0) zero_row = true;
      vv[i] = 1.0 / big;
    }
    const bool singular = __any_sync(0xffffffffu, zero_row);
    __syncwarp();
    double d = 1.0;
    for (int j = 0; j < n && !singular; ++j) {
      double best = -1.0;
      int bi = -1;
      for (int i = j + lane; i < n; i += 32) {
        const double dum = vv[i] * dabs(a[n * i + j]);
        if (dum >= best) {
          best = dum;
          bi = i;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi > bi)) {
          best = ob;
          bi = oi;
        }
      }
      const int imax = bi;
      if (imax != j) {
        for (int k = lane; k < n; k += 32) {
          const dc t = a[n * imax + k];
          a[n * imax + k] = a[n * j + k];
          a[n * j + k] = t;
        }
        d = -d;
        if (lane == 0) vv[imax] = vv[j];
      }
      __syncwarp();
      if (lane == 0 && dabs(a[n * j + j]) == 0.0) a[n * j + j] = dc{1.0e-20, 0.0};
      __syncwarp();
      const dc r = drecip(a[n * j + j]);
      for (int i = j + 1 + lane; i < n; i += 32) a[n * i + j] = dmul(a[n * i + j], r);
      __syncwarp();
      for (int k = j + 1 + lane; k < n; k += 32) {
        const dc u = a[n * j + k];
        for (int i = j + 1; i < n; ++i) {
          const dc p = dmul(a[n * i + j], u);
          a[n * i + k].re -= p.re;
          a[n * i + k].im -= p.im;
        }
      }
      __syncwarp();
    }
    if (lane == 0) {
      dc r;
      if (singular) {
        r = dc{nan(""), nan("")};  // an all-zero row: flagged to the host
      } else if (!log_det) {
        r = dc{d, 0.0};
        for (int i = 0; i < n; ++i) r = dmul(r, a[n * i + i]);
      } else {
        r = dc{log(fabs(d)), d < 0 ? 3.14159265358979323846 : 0.0};
        for (int i = 0; i < n; ++i) {
          r.re += log(dabs(a[n * i + i]));
          r.im += atan2(a[n * i + i].im, a[n * i + i].re);
        }
      }
      double* o = out + c * out_conf_stride + out_offset + 2L * m;
      o[0] = r.re;
      o[1] = r.im;
    }
    __syncwarp();
  }
}

constexpr int kWarpLuMaxN = 64;
constexpr size_t kWarpLuSmemCap = 200 * 1024;

static size_t warp_lu_bytes(int N) { return (size_t)N * N * sizeof(dc) + N * sizeof(double); }
static int warp_lu_warps(int N) {
  int w = (int)(kWarpLuSmemCap / warp_lu_bytes(N));
  return w < 1 ? 1 : (w > kWarpLuMaxWarps ? kWarpLuMaxWarps : w);
}

// Leading-minor determinants through the warp kernel (N <= 64, no scratch).
nrcps_status slater_dets_warp(nrcps_context* ctx, const double* S, const double* psi1, int N, int nconf, int mode,
                              int log_det, double* out, long out_conf_stride, long out_offset) {
  const int nmeas = mode ? 2 * N : N;
  const long total = (long)nconf * nmeas;
  if (total == 0) return NRCPS_OK;
  static bool attr_set[16] = {false};
  if (!attr_set[ctx->device & 15]) {
    NRCPS_TRY(check_cuda(ctx,
                         cudaFuncSetAttribute(slater_dets_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kWarpLuSmemCap),
                         "slater_dets_warp: smem attribute"));
    attr_set[ctx->device & 15] = true;
  }
  const int wpb = warp_lu_warps(N);
  const long blocks = (total + wpb - 1) / wpb;
  const unsigned g = (unsigned)(blocks < (long)ctx->sm_count * 64 ? blocks : (long)ctx->sm_count * 64);
  slater_dets_warp_kernel<<<g, 32 * wpb, (size_t)wpb * warp_lu_bytes(N), ctx->stream>>>(S, psi1, N, nconf, mode, log_det,
                                                                                   out, out_conf_stride, out_offset);
  ctx->launches++;
  return check_launch(ctx, "slater_dets_warp_kernel");
}

size_t slater_dets_scratch_bytes(int N, int nconf, int mode) {
  const int nmeas = mode ? 2 * N : N;
  return sizeof(double) * (size_t)nconf * nmeas * (2L * N * N + N);
}

// scr: caller-owned scratch of slater_dets_scratch_bytes(), or NULL for the
// context's scratch.
nrcps_status slater_dets_impl(nrcps_context* ctx, const double* S, const double* psi1, int N, int nconf, int mode,
                              int log_det, double* out, long out_conf_stride, long out_offset, double* scr) {
  const int nmeas = mode ? 2 * N : N;
  const long total = (long)nconf * nmeas;
  if (total == 0) return NRCPS_OK;
  if (!scr) {
    nrcps_status st;
    scr = (double*)scratch(ctx, slater_dets_scratch_bytes(N, nconf, mode), &st);
    if (!scr) return st;
  }
  slater_dets_kernel<<<grid_for(total, 64, 1L << 20), 64, 0, ctx->stream>>>(S, psi1, N, nconf, mode, log_det, out,
                                                                             scr, out_conf_stride, out_offset);
  ctx->launches++;
  return check_launch(ctx, "slater_dets_kernel");
}

// The determinant path of the library: the warp kernel for N <= 64 (unless
// the "lu.warp" option is 0), else the per-thread kernel with scratch.
nrcps_status slater_dets_dispatch(nrcps_context* ctx, const double* S, const double* psi1, int N, int nconf, int mode,
                                  int log_det, double* out, long out_conf_stride, long out_offset, double* scr) {
  if (N <= kWarpLuMaxN && ctx->lu_warp)
    return slater_dets_warp(ctx, S, psi1, N, nconf, mode, log_det, out, out_conf_stride, out_offset);
  return slater_dets_impl(ctx, S, psi1, N, nconf, mode, log_det, out, out_conf_stride, out_offset, scr);
}

nrcps_status overlap_impl(nrcps_context* ctx, const double* src, int ns, const void* psi, int nt, int nconf,
                          long vol, nrcps_precision prec, double* S) {
  long blocks = (long)nconf * nt;
  if (blocks == 0) return NRCPS_OK;
  if (prec == NRCPS_F64) overlap_kernel<double><<<(unsigned)blocks, 256, 0, ctx->stream>>>(src, ns, psi, nt, vol, S);
  else overlap_kernel<float><<<(unsigned)blocks, 256, 0, ctx->stream>>>(src, ns, psi, nt, vol, S);
  ctx->launches++;
  return check_launch(ctx, "overlap_kernel");
}

nrcps_status gather_impl(nrcps_context* ctx, const int* index, int ns, const void* psi, int nt, int nconf, long vol,
                         nrcps_precision prec, double* S) {
  long total = (long)nconf * ns * nt;
  if (total == 0) return NRCPS_OK;
  unsigned g = grid_for(total, 256, (long)ctx->sm_count * 8);
  if (prec == NRCPS_F64) gather_kernel<double><<<g, 256, 0, ctx->stream>>>(index, ns, psi, nt, nconf, vol, S);
  else gather_kernel<float><<<g, 256, 0, ctx->stream>>>(index, ns, psi, nt, nconf, vol, S);
  ctx->launches++;
  return check_launch(ctx, "gather_kernel");
}

template <typename R>
static nrcps_status launch_pair_tile(nrcps_context* ctx, const void* psi1, const void* psi2, int n, int nconf,
                                     long vol, const double* w, const int* opp, const int* flags, int host_flags,
                                     double* phi) {
  using Sh = PairShape<R>;
  const int ts = Sh::ts(n);
  const size_t smem = Sh::smem(n);
  static bool attr_set[16] = {false};
  if (!attr_set[ctx->device & 15]) {
    size_t most = 0;
    for (int m = 1; m <= PAIR_MAXN; ++m) most = Sh::smem(m) > most ? Sh::smem(m) : most;
    NRCPS_TRY(check_cuda(ctx, cudaFuncSetAttribute(pair_tile_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)most),
                         "pair_tile: smem attribute"));
    attr_set[ctx->device & 15] = true;
  }
  // CTAs per configuration: enough CTAs for about four per SM, at most 8
  // (a portable cluster) and no more than the tiles
  const long ntiles = (vol + ts - 1) / ts;
  int split = (int)((4L * ctx->sm_count + nconf - 1) / nconf);
  if (split > 8) split = 8;
  if (split > ntiles) split = (int)ntiles;
  if (split < 1) split = 1;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)split;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)((long)nconf * split));
  cfg.blockDim = dim3(PAIR_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e =
      cudaLaunchKernelEx(&cfg, pair_tile_kernel<R>, psi1, psi2, n, vol, w, opp, flags, host_flags, ts, phi);
  ctx->launches++;
  return check_cuda(ctx, e, "pair_tile_kernel launch");
}

// props: the table's properties as the caller checked them on the host
// (pair_table_props), or -1: the device checks them before the tiles.
nrcps_status pair_impl(nrcps_context* ctx, const void* psi1, const void* psi2, int n, int nconf, long vol,
                       const double* w, const int* opp, nrcps_precision prec, double* phi, int props) {
  long blocks = (long)nconf * n * n;
  if (blocks == 0) return NRCPS_OK;
  if (n <= PAIR_MAXN && ctx->pair_tile && (long)nconf * 8 < (1L << 31)) {
    const int* flags = nullptr;
    if (props < 0) {
      NRCPS_TRY(check_cuda(ctx, cudaMemsetAsync(ctx->dev_pair_flag, 0, sizeof(int), ctx->stream), "pair flag"));
      opp_involution_check_kernel<<<grid_for(vol, 256), 256, 0, ctx->stream>>>(opp, w, vol, ctx->dev_pair_flag);
      ctx->launches++;
      NRCPS_TRY(check_launch(ctx, "opp_involution_check_kernel"));
      flags = ctx->dev_pair_flag;
    }
    if (prec == NRCPS_F64)
      return launch_pair_tile<double>(ctx, psi1, psi2, n, nconf, vol, w, opp, flags, props, phi);
    return launch_pair_tile<float>(ctx, psi1, psi2, n, nconf, vol, w, opp, flags, props, phi);
  }
  if (prec == NRCPS_F64) pair_kernel<double><<<(unsigned)blocks, 256, 0, ctx->stream>>>(psi1, psi2, n, vol, w, opp, phi);
  else pair_kernel<float><<<(unsigned)blocks, 256, 0, ctx->stream>>>(psi1, psi2, n, vol, w, opp, phi);
  ctx->launches++;
  return check_launch(ctx, "pair_kernel");
}

}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_overlap(nrcps_context* ctx, const double* dev_src, int ns, const void* dev_psi, int nt,
                                      int nconf, long vol, nrcps_precision prec, double* dev_S) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, ns >= 0 && nt >= 0 && nconf >= 0 && vol > 0, "nrcps_overlap: bad arguments");
  if ((long)ns * nt * nconf == 0) return NRCPS_OK;  // empty batch: nothing to read or write
  NRCPS_REQUIRE(ctx, dev_src && dev_psi && dev_S, "nrcps_overlap: null pointer");
  if (prec == NRCPS_F32 && ctx->overlap_tc && ns > 0 && nt > 0 && nconf > 0 && ((uintptr_t)dev_psi & 15) == 0 &&
      overlap_tc_supported(vol, ns, nt, nconf)) {
    const size_t need = overlap_tc_split_bytes(ns, vol);
    if (need > ctx->tc_split_bytes) {
      if (ctx->tc_split) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->tc_split);
        ctx->tc_split = nullptr;
        ctx->tc_split_bytes = 0;
      }
      NRCPS_TRY(check_cuda(ctx, cudaMalloc(&ctx->tc_split, need), "cudaMalloc(overlap split)"));
      ctx->tc_split_bytes = need;
    }
    NRCPS_TRY(overlap_tc_prepare(ctx, dev_src, ns, vol, (float*)ctx->tc_split));
    return overlap_tc(ctx, (const float*)ctx->tc_split, ns, dev_psi, nt, nconf, vol, dev_S);
  }
  return overlap_impl(ctx, dev_src, ns, dev_psi, nt, nconf, vol, prec, dev_S);
}

extern "C" nrcps_status nrcps_overlap_planewave(nrcps_context* ctx, const int* dev_index, int ns, const void* dev_psi,
                                                int nt, int nconf, long vol, nrcps_precision prec, double* dev_S) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, ns >= 0 && nt >= 0 && nconf >= 0 && vol > 0, "nrcps_overlap_planewave: bad arguments");
  if ((long)ns * nt * nconf == 0) return NRCPS_OK;
  NRCPS_REQUIRE(ctx, dev_index && dev_psi && dev_S, "nrcps_overlap_planewave: null pointer");
  return gather_impl(ctx, dev_index, ns, dev_psi, nt, nconf, vol, prec, dev_S);
}

extern "C" nrcps_status nrcps_pair_matrix(nrcps_context* ctx, const void* dev_psi1, const void* dev_psi2, int n,
                                          int nconf, long vol, const double* dev_w, const int* dev_opposite,
                                          nrcps_precision prec, double* dev_phi) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, n >= 0 && nconf >= 0 && vol > 0, "nrcps_pair_matrix: bad arguments");
  if ((long)n * nconf == 0) return NRCPS_OK;
  NRCPS_REQUIRE(ctx, dev_psi1 && dev_psi2 && dev_w && dev_opposite && dev_phi, "nrcps_pair_matrix: null pointer");
  return pair_impl(ctx, dev_psi1, dev_psi2, n, nconf, vol, dev_w, dev_opposite, prec, dev_phi, -1);
}

extern "C" nrcps_status nrcps_shifted_pair_matrix(nrcps_context* ctx, const void* dev_psi1, const void* dev_psi2,
                                                  int n, int nconf, long vol, int nterms, const int* dev_shift,
                                                  const double* dev_wl, const int* dev_opposite,
                                                  nrcps_precision prec, double* dev_phi) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, n >= 0 && nconf >= 0 && vol > 0 && nterms > 0, "nrcps_shifted_pair_matrix: bad arguments");
  const long blocks = (long)nconf * n * n;
  if (blocks == 0) return NRCPS_OK;
  NRCPS_REQUIRE(ctx, dev_psi1 && dev_psi2 && dev_shift && dev_wl && dev_opposite && dev_phi,
                "nrcps_shifted_pair_matrix: null pointer");
  if (prec == NRCPS_F64)
    shifted_pair_kernel<double><<<(unsigned)blocks, 256, 0, ctx->stream>>>(dev_psi1, dev_psi2, n, vol, nterms,
                                                                          dev_shift, dev_wl, dev_opposite, dev_phi);
  else
    shifted_pair_kernel<float><<<(unsigned)blocks, 256, 0, ctx->stream>>>(dev_psi1, dev_psi2, n, vol, nterms,
                                                                         dev_shift, dev_wl, dev_opposite, dev_phi);
  ctx->launches++;
  return check_launch(ctx, "shifted_pair_kernel");
}

extern "C" nrcps_status nrcps_inner_product_ptrs(nrcps_context* ctx, const double* const* dev_kets,
                                                 const double* const* dev_bras, int nf, long vol, double* dev_mat) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, dev_kets && dev_bras && dev_mat && nf >= 0 && vol > 0, "nrcps_inner_product_ptrs: bad arguments");
  if (nf == 0) return NRCPS_OK;
  inner_ptrs_kernel<<<(unsigned)(nf * nf), 256, 0, ctx->stream>>>(dev_kets, dev_bras, nf, vol, dev_mat);
  ctx->launches++;
  return check_launch(ctx, "inner_ptrs_kernel");
}

extern "C" nrcps_status nrcps_pair_matrix_ptrs(nrcps_context* ctx, const double* const* dev_props1,
                                               const double* const* dev_props2, int nf, long vol, const double* dev_w,
                                               const int* dev_opposite, double* dev_phi) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, dev_props1 && dev_props2 && dev_w && dev_opposite && dev_phi && nf >= 0 && vol > 0,
                "nrcps_pair_matrix_ptrs: bad arguments");
  if (nf == 0) return NRCPS_OK;
  pair_ptrs_kernel<<<(unsigned)(nf * nf), 256, 0, ctx->stream>>>(dev_props1, dev_props2, nf, vol, dev_w,
                                                                 dev_opposite, dev_phi);
  ctx->launches++;
  return check_launch(ctx, "pair_ptrs_kernel");
}

extern "C" nrcps_status nrcps_slater_dets(nrcps_context* ctx, const double* dev_S, const double* dev_psi1, int N,
                                          int nconf, int mode, int log_det, double* dev_out) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, N > 0 && nconf >= 0 && (mode == 0 || mode == 1), "nrcps_slater_dets: bad arguments");
  if (nconf == 0) return NRCPS_OK;
  NRCPS_REQUIRE(ctx, dev_S && dev_out && (mode == 0 || dev_psi1), "nrcps_slater_dets: null pointer");
  const int nmeas = mode ? 2 * N : N;
  return slater_dets_dispatch(ctx, dev_S, dev_psi1, N, nconf, mode, log_det, dev_out, 2L * nmeas, 0, nullptr);
}

/*
 * fft64.c -- double-precision mixed-radix complex DFT, FFTW conventions.
 *
 * TEST INFRASTRUCTURE ONLY (oracle).  See fft64.h for the conventions.
 *
 * Algorithm: recursive decimation-in-time Cooley-Tukey over the prime
 * factorisation of n (radix 2, 3, 5, ... and a direct DFT for any remaining
 * prime).  Twiddles come from one table per length, w[t] = exp(-2*pi*i*t/n),
 * evaluated with cos/sin of the exact angle, so the transform is accurate to
 * a few ulp * log2(n).  This is a plain textbook restatement of the DFT the
 * reference obtains from FFTW (src/fourier/noarch/fourier.C:34-35,75-101);
 * it is not FFTW's code.
 */
#include "fft64.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int n;
  double *w; /* n complex twiddles exp(-2 pi i t / n) */
} twtab;

#define MAX_TABS 64
static twtab g_tabs[MAX_TABS];
static int g_ntabs = 0;

static const double *twiddles(int n) {
  for (int i = 0; i < g_ntabs; ++i)
    if (g_tabs[i].n == n) return g_tabs[i].w;
  double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  const long double two_pi = 6.283185307179586476925286766559L;
  for (int t = 0; t < n; ++t) {
    long double ang = two_pi * (long double)t / (long double)n;
    w[2 * t] = (double)cosl(ang);
    w[2 * t + 1] = -(double)sinl(ang);
  }
  if (g_ntabs < MAX_TABS) {
    g_tabs[g_ntabs].n = n;
    g_tabs[g_ntabs].w = w;
    ++g_ntabs;
  }
  return w;
}

static int smallest_factor(int n) {
  if (n % 2 == 0) return 2;
  for (int p = 3; p * p <= n; p += 2)
    if (n % p == 0) return p;
  return n;
}

/* out[k] = sum_{j<n} in[j*stride] * W_N^{(N/n) j k * s}, where W_N = exp(-2 pi i/N)
 * and s = +1 for sign -1 (forward), conjugated for sign +1. `scale` = N/n. */
static void dft_rec(const double *in, long stride, double *out, int n, const double *w, int N,
                    int sign) {
  if (n == 1) {
    out[0] = in[0];
    out[1] = in[1];
    return;
  }
  int p = smallest_factor(n);
  int m = n / p;
  for (int q = 0; q < p; ++q) dft_rec(in + 2 * q * stride, stride * p, out + 2 * q * m, m, w, N, sign);
  /* combine: X[k + s*m] = sum_q W_n^{q(k+s m)} F_q[k] */
  const int scale = N / n;
  double tmp[2 * 64];
  double *t = tmp;
  double *heap = NULL;
  if (p > 64) {
    heap = (double *)malloc(sizeof(double) * 2 * (size_t)p);
    t = heap;
  }
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) {
      t[2 * q] = out[2 * (q * m + k)];
      t[2 * q + 1] = out[2 * (q * m + k) + 1];
    }
    for (int s = 0; s < p; ++s) {
      int kk = k + s * m;
      double re = 0.0, im = 0.0;
      for (int q = 0; q < p; ++q) {
        long idx = ((long)q * kk) % n;
        double wr = w[2 * idx * scale];
        double wi = w[2 * idx * scale + 1];
        if (sign > 0) wi = -wi;
        double xr = t[2 * q], xi = t[2 * q + 1];
        re += xr * wr - xi * wi;
        im += xr * wi + xi * wr;
      }
      out[2 * kk] = re;
      out[2 * kk + 1] = im;
    }
  }
  free(heap);
}

void o_fft1d_many(double *data, int n, int howmany, long stride, long dist, int sign) {
  if (n <= 1) return;
  const double *w = twiddles(n);
  double *a = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  double *b = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (int h = 0; h < howmany; ++h) {
    double *x = data + 2 * h * dist;
    for (int j = 0; j < n; ++j) {
      a[2 * j] = x[2 * j * stride];
      a[2 * j + 1] = x[2 * j * stride + 1];
    }
    dft_rec(a, 1, b, n, w, n, sign);
    for (int j = 0; j < n; ++j) {
      x[2 * j * stride] = b[2 * j];
      x[2 * j * stride + 1] = b[2 * j + 1];
    }
  }
  free(a);
  free(b);
}

void o_fftnd(double *data, int rank, const int *dims, int batch, long dist, int sign) {
  long vol = 1;
  for (int d = 0; d < rank; ++d) vol *= dims[d];
  for (int bb = 0; bb < batch; ++bb) {
    double *x = data + 2 * bb * dist;
    for (int d = rank - 1; d >= 0; --d) {
      long stride = 1;
      for (int e = d + 1; e < rank; ++e) stride *= dims[e];
      long outer = vol / (stride * dims[d]);
      for (long o = 0; o < outer; ++o) {
        /* all pencils along axis d inside this outer slab */
        o_fft1d_many(x + 2 * o * stride * dims[d], dims[d], (int)stride, stride, 1, sign);
      }
    }
  }
}

void o_fft3d(double *data, const int dims[3], int batch, int sign) {
  long vol = (long)dims[0] * dims[1] * dims[2];
  o_fftnd(data, 3, dims, batch, vol, sign);
}

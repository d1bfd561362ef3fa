/*
 * fft64.h -- double-precision mixed-radix complex DFT with FFTW's conventions.
 *
 * TEST INFRASTRUCTURE ONLY.  This file belongs to the oracle (the CPU checker
 * of the B200 path).  It is linked into (a) the FFTW-compatible shim that lets
 * the reference's own CPU code build without FFTW, and (b) the C restatement
 * of the reference algorithm in oracle.c.  The product library never links it.
 *
 * Conventions (FFTW 3, which the reference calls in src/fourier/noarch/fourier.C:34-35):
 *   X[k] = sum_j x[j] * exp(sign * 2*pi*i * j*k / n),   unnormalised,
 *   sign = -1 is FFTW_FORWARD, sign = +1 is FFTW_BACKWARD,
 *   multi-dimensional arrays are row-major (last index fastest).
 * Validated against numpy.fft.fftn in tests/test_oracle_fft.py.
 */
#ifndef NRCPS_ORACLE_FFT64_H
#define NRCPS_ORACLE_FFT64_H

#ifdef __cplusplus
extern "C" {
#endif

/* In-place 1-D transform of `howmany` sequences of length n.  Element j of
 * sequence b sits at data[2*(b*dist + j*stride)] (re) and [..+1] (im). */
void o_fft1d_many(double *data, int n, int howmany, long stride, long dist, int sign);

/* In-place unnormalised 3-D transform of `batch` row-major arrays
 * dims[0] x dims[1] x dims[2] stored back to back (distance = volume). */
void o_fft3d(double *data, const int dims[3], int batch, int sign);

/* Generic rank-d transform (1 <= d <= 3) used by the FFTW shim. */
void o_fftnd(double *data, int rank, const int *dims, int batch, long dist, int sign);

#ifdef __cplusplus
}
#endif
#endif

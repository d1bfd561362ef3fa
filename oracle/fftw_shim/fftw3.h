/*
 * fftw3.h -- minimal FFTW-3-compatible interface over the oracle's own FFT.
 *
 * TEST INFRASTRUCTURE ONLY.  FFTW 3 (3.2.2 / 3.3.3, named by the reference's
 * build scripts) is not installed here, so the reference's own CPU code is
 * compiled against this header instead.  Only the entry points the reference
 * calls are provided (src/fourier/noarch/fourier.C:16-23,30-40,53-69,78-99):
 * fftw_malloc/free, fftw_plan_many_dft (contiguous, in-place or out-of-place,
 * inembed/onembed NULL), fftw_execute, fftw_destroy_plan, fftw_cleanup.
 * The transform itself is oracle/fft64.c (unnormalised, FFTW sign convention).
 */
#ifndef NRCPS_FFTW_SHIM_H
#define NRCPS_FFTW_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in,
                             const int *inembed, int istride, int idist, fftw_complex *out,
                             const int *onembed, int ostride, int odist, int sign,
                             unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif
#endif

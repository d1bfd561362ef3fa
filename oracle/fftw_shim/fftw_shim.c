/*
 * fftw_shim.c -- FFTW-3-compatible plan/execute layer over oracle/fft64.c.
 *
 * TEST INFRASTRUCTURE ONLY: lets the reference's CPU path
 * (src/fourier/noarch/fourier.C) build and run here without FFTW.
 */
#include "fftw3.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../fft64.h"

struct fftw_plan_s {
  int rank;
  int dims[3];
  int howmany;
  int istride, idist, ostride, odist;
  double *in, *out;
  int sign;
};

void *fftw_malloc(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
  return p;
}

void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in,
                             const int *inembed, int istride, int idist, fftw_complex *out,
                             const int *onembed, int ostride, int odist, int sign,
                             unsigned flags) {
  (void)flags;
  if (rank < 1 || rank > 3 || inembed || onembed || istride != 1 || ostride != 1) {
    fprintf(stderr, "fftw shim: unsupported plan layout\n");
    abort();
  }
  struct fftw_plan_s *p = (struct fftw_plan_s *)calloc(1, sizeof(*p));
  p->rank = rank;
  for (int d = 0; d < rank; ++d) p->dims[d] = n[d];
  p->howmany = howmany;
  p->istride = istride;
  p->idist = idist;
  p->ostride = ostride;
  p->odist = odist;
  p->in = (double *)in;
  p->out = (double *)out;
  p->sign = sign;
  return p;
}

void fftw_execute(const fftw_plan p) {
  long vol = 1;
  for (int d = 0; d < p->rank; ++d) vol *= p->dims[d];
  if (p->in != p->out) {
    for (int b = 0; b < p->howmany; ++b)
      memcpy(p->out + 2 * (long)b * p->odist, p->in + 2 * (long)b * p->idist,
             sizeof(double) * 2 * (size_t)vol);
  }
  o_fftnd(p->out, p->rank, p->dims, p->howmany, p->odist, p->sign);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

void fftw_cleanup(void) {}

// fourier.cc -- replaces src/fourier/cuda/fourier.cu of the reference:
// the batch buffer lives on the device, the transforms are nrcps_fft3d.
#include <fourier.h>

#include <cuda_runtime.h>
#include "cuda_utils.h"
#include "error.h"
#include "global_job_parameter.h"
#include "shim_context.h"
#include "verbose.h"

Fourier::Fourier(int n) {
  batch_size = n;
  Cuda::Malloc((void**)&b, batch_size * GJP.Vol() * sizeof(fftComplex));
  plan = 0;  // no library plan: the transform is planned at compile time
}

Fourier::~Fourier() { Cuda::Free(b); }

static void transform(fftComplex* b, int batch, int sign, const char* fname) {
  int dims[3] = {GJP.Xsites(), GJP.Ysites(), GJP.Zsites()};
  nrcps_shim_check(nrcps_fft3d(nrcps_shim_context(), b, batch, dims, NRCPS_F64, sign), fname);
}

void Fourier::Forward() { transform(b, batch_size, -1, "void Fourier::Forward()"); }

void Fourier::Backward() { transform(b, batch_size, +1, "void Fourier::Backward()"); }

// two_body_run.cc -- replaces src/two_body/cuda/two_body_run.cu.
#include <complex>

#include <cuda_runtime.h>
using namespace std;
#include "cuda_utils.h"
#include "shim_context.h"
#include "two_body.h"

complex<Float> TwoBody::Run(Float* prop1, Float* prop2) {
  const char* fname = "complex<Float> TwoBody::Run(Float*, Float*)";
  nrcps_shim_check(nrcps_pair_matrix(nrcps_shim_context(), prop1, prop2, 1, 1, vol, dev_wavefunc,
                                     dev_opposite_parity_index, NRCPS_F64, dev_psum),
                   fname);
  double h[2];
  Cuda::MemCopy(h, dev_psum, sizeof h, cudaMemcpyDeviceToHost);
  return complex<Float>(h[0], h[1]);
}

// props1, props2: device arrays of nf device pointers; slater: host, [t+nf*s].
void TwoBody::Run(Float** props1, Float** props2, complex<Float>* slater, int nf) {
  const char* fname = "void TwoBody::Run(Float**, Float**, complex<Float>*, int)";
  double* dev = nullptr;
  Cuda::Malloc((void**)&dev, sizeof(double) * 2 * nf * nf);
  nrcps_shim_check(nrcps_pair_matrix_ptrs(nrcps_shim_context(), (const double* const*)props1,
                                          (const double* const*)props2, nf, vol, dev_wavefunc,
                                          dev_opposite_parity_index, dev),
                   fname);
  Cuda::MemCopy(slater, dev, sizeof(double) * 2 * nf * nf, cudaMemcpyDeviceToHost);
  Cuda::Free(dev);
}

// one_body_project.cc -- replaces src/one_body/cuda/one_body_project.cu:
// <psi|phi> for device vectors through nrcps_overlap (FP64, one reduction).
#include <complex>

#include <cuda_runtime.h>
using namespace std;
#include "cuda_utils.h"
#include "one_body.h"
#include "shim_context.h"

complex<Float> OneBody::Project(Float* phi) {
  const char* fname = "complex<Float> OneBody::Project(Float*)";
  nrcps_shim_check(nrcps_overlap(nrcps_shim_context(), dev_psi, 1, phi, 1, 1, vol, NRCPS_F64, dev_psum), fname);
  double h[2];
  Cuda::MemCopy(h, dev_psum, sizeof h, cudaMemcpyDeviceToHost);
  return complex<Float>(h[0], h[1]);
}

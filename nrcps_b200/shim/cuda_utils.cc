// cuda_utils.cc -- replaces src/utils/cuda/cuda_utils.cu of the reference.
//
// Memory plumbing keeps the reference's semantics (error-checked CUDA
// runtime calls); Cuda::InnerProduct runs through the C ABI.
#include <complex>
#include <cstdio>
#include <vector>

#include <cuda_runtime.h>
#include "cuda_utils.h"
#include "error.h"
#include "shim_context.h"
#include "sysfunc.h"
#include "verbose.h"

using namespace std;

// Name reported by Lattice::Mean/Variance in the GPU build (lattice_fname.h).
const char* nrcps_fname = "Lattice (GPU build)";

nrcps_context* nrcps_shim_context() {
  static nrcps_context* ctx = nullptr;
  if (!ctx) {
    int dev = 0;
    cudaGetDevice(&dev);
    nrcps_status st = nrcps_create(dev, &ctx);
    if (st != NRCPS_OK) ERR.General("nrcps_shim_context()", "nrcps_create failed (status %d)", (int)st);
  }
  return ctx;
}

void nrcps_shim_check(nrcps_status st, const char* fname) {
  if (st != NRCPS_OK) ERR.General(fname, "%s", nrcps_last_error(nrcps_shim_context()));
}

void Cuda::Malloc(void** devPtr, size_t size) {
  const char* fname = "void Cuda::Malloc(void**, size_t)";
  cudaError_t err = cudaMalloc(devPtr, size);
  if (cudaSuccess != err) ERR.General(fname, "Cuda error: %s\n", cudaGetErrorString(err));
}

void Cuda::HostAlloc(void** pHost, size_t size, unsigned int flags) {
  const char* fname = "void Cuda::HostMalloc(void**, size_t , unsigned int )";
  cudaError_t err = cudaHostAlloc(pHost, size, flags);
  if (cudaSuccess != err) ERR.General(fname, "Cuda error: %s\n", cudaGetErrorString(err));
}

void Cuda::Free(void* devPtr) {
  const char* fname = "void Cuda::Free(void*)";
  cudaError_t err = cudaFree(devPtr);
  if (cudaSuccess != err) ERR.General(fname, "Cuda error: %s\n", cudaGetErrorString(err));
}

void Cuda::FreeHost(void* pHost) {
  const char* fname = "void Cuda::FreeHost(void*)";
  cudaError_t err = cudaFreeHost(pHost);
  if (cudaSuccess != err) ERR.General(fname, "Cuda error: %s\n", cudaGetErrorString(err));
}

void Cuda::MemCopy(void* dst, void* src, size_t size, cudaMemcpyKind kind) {
  const char* fname = "void Cuda::MemCopy(void*, void*, size_t, cudaMemcpyKind)";
  cudaError_t err = cudaMemcpy(dst, src, size, kind);
  if (cudaSuccess != err) ERR.General(fname, "Cuda error: %s\n", cudaGetErrorString(err));
}

void Cuda::DeviceQ() {
  int count = 0;
  cudaGetDeviceCount(&count);
  for (int j = 0; j < count; ++j) {
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, j);
    VRB.Flow("void Cuda::DeviceQ()", "Device %d: %s, compute capability %d.%d, %d SMs, %ld bytes", j, p.name,
             p.major, p.minor, p.multiProcessorCount, (long)p.totalGlobalMem);
  }
}

// kets, bras: device arrays of nf device pointers; mat: host, mat[t+nf*s].
void Cuda::InnerProduct(Float** kets, Float** bras, complex<Float>* mat, int nf, int vol) {
  const char* fname = "void Cuda::InnerProduct(Float**, Float**, complex<Float>*, int, int)";
  nrcps_context* ctx = nrcps_shim_context();
  double* dev_mat = nullptr;
  Cuda::Malloc((void**)&dev_mat, sizeof(double) * 2 * nf * nf);
  nrcps_shim_check(nrcps_inner_product_ptrs(ctx, (const double* const*)kets, (const double* const*)bras, nf, vol,
                                            dev_mat),
                   fname);
  Cuda::MemCopy(mat, dev_mat, sizeof(double) * 2 * nf * nf, cudaMemcpyDeviceToHost);
  Cuda::Free(dev_mat);
}

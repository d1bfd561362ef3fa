// eigensystem_stub.cc -- link-time stand-in for src/linalg/eigensystem.C.
//
// TEST INFRASTRUCTURE ONLY.  The reference's Eigensystem wraps LAPACK from
// Apple Accelerate (src/linalg/eigensystem.C:3), which is absent here.  Only
// OhProjector (src/utils/oh_group.C) references it, and nothing on the
// propagation / Slater-determinant path calls OhProjector, so these stubs
// abort loudly if they are ever reached.
#include <cstdio>
#include <cstdlib>

void Eigensystem(char*, char*, int*, double*, int*, double*) {
  std::fprintf(stderr, "Eigensystem (LAPACK) is not available in the oracle build\n");
  std::abort();
}

void Eigensystem(char*, char*, int*, double*, double*, int*) {
  std::fprintf(stderr, "Eigensystem (LAPACK) is not available in the oracle build\n");
  std::abort();
}

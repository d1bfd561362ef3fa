// hamiltonian_gpu.cc -- replaces src/hamiltonian/cuda/hamiltonian_evolve.cu
// and hamiltonian_initialize.cu of the reference.  The device tables
// (dev_xi, dev_potential, dev_interaction) are the ones the reference's
// constructors upload (src/hamiltonian/hamiltonian.C:140-143,236-239,275-278).
#include <iostream>
#include <vector>

using namespace std;
#include "error.h"
#include "global_job_parameter.h"
#include "hamiltonian.h"
#include "shim_context.h"
#include "verbose.h"

static void dims3(int d[3]) {
  d[0] = GJP.Xsites();
  d[1] = GJP.Ysites();
  d[2] = GJP.Zsites();
}

// The CPU build's Interactions::Evolve has its body commented out (a no-op,
// src/hamiltonian/noarch/hamiltonian_evolve.C:19-31); the GPU build raises
// NotImplemented.  The CPU behaviour is kept.
void Interactions::Evolve(Fourier* b) { VRB.Func("Interactions::Evolve(Fourier*)"); }

void Interaction::Evolve(Fourier* b) {
  const char* fname = "void Interaction::Evolve(Fourier*)";
  if (GJP.APBCQuery()) ERR.NotImplemented(fname, "APBCs not permitted.");
  int d[3];
  dims3(d);
  nrcps_shim_check(nrcps_interaction_evolve(nrcps_shim_context(), b->Get(0), b->BatchSize(), d,
                                            (const double*)field->Get(0), NRCPS_F64),
                   fname);
}

void Potential::Evolve(Fourier* b) {
  const char* fname = "void Potential::Evolve(Fourier*)";
  if (GJP.APBCQuery()) ERR.NotImplemented(fname, "APBCs not permitted.");
  int d[3];
  dims3(d);
  nrcps_shim_check(nrcps_potential_evolve(nrcps_shim_context(), b->Get(0), b->BatchSize(), d, dev_potential,
                                          NRCPS_F64),
                   fname);
}

void Kinetic::Evolve(Fourier* b) {
  const char* fname = "void Kinetic::Evolve(Fourier*)";
  nrcps_shim_check(nrcps_kinetic_evolve(nrcps_shim_context(), b->Get(0), b->BatchSize(), GJP.Vol(), dev_xi,
                                        NRCPS_F64),
                   fname);
}

void Interaction::Initialize() {
  int d[3];
  dims3(d);
  nrcps_shim_check(nrcps_interaction_initialize(nrcps_shim_context(), lattice->Get(), dev_interaction, d,
                                                (double*)field->Get(0)),
                   "void Interaction::Initialize()");
}

void Potential::Initialize() {}

void Kinetic::Initialize() {}

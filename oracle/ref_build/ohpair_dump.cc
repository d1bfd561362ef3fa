// ohpair_dump.cc -- dumps the tables and results of the reference's
// GeneralizedTwoBody (src/two_body/two_body.C:209-288,
// src/two_body/noarch/two_body_run.C:45-103) for golden fixtures.
//
// TEST INFRASTRUCTURE ONLY (built by this directory's Makefile into
// oracle/_ref/).  The class keeps its tables private; this translation unit
// alone opens them for reading.
//
//   ohpair_dump L=8 vec=1,0,2 wf=TGND lambda=0.25 seed=3 out=file
//
// Output (binary, little endian): int nterms, int vol; int opp[vol];
// int shift[nterms][vol]; double hsw[nterms][vol]; double weight[nterms][10];
// double props[2][2 vol] (interleaved complex); double run[10][2];
// double run2[10][2].
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

using namespace std;

#include "arg.h"
#include "enum.h"
#include "global_job_parameter.h"
#include "vector3.h"
#define private public
#include "oh_group.h"
#include "two_body.h"
#undef private

static string arg(int argc, char** argv, const char* key, const char* def) {
  size_t n = strlen(key);
  for (int i = 1; i < argc; ++i)
    if (!strncmp(argv[i], key, n) && argv[i][n] == '=') return string(argv[i] + n + 1);
  return def;
}

int main(int argc, char** argv) {
  const int L = atoi(arg(argc, argv, "L", "8").c_str());
  int vx = 0, vy = 0, vz = 0;
  sscanf(arg(argc, argv, "vec", "1,0,0").c_str(), "%d,%d,%d", &vx, &vy, &vz);
  const string wf = arg(argc, argv, "wf", "TGND");
  const double lambda = atof(arg(argc, argv, "lambda", "0.25").c_str());
  unsigned long long state = strtoull(arg(argc, argv, "seed", "3").c_str(), nullptr, 10) * 2654435761ull + 1;
  const string out = arg(argc, argv, "out", "ohpair.bin");

  DoArg d;
  d.t_sites = 4;
  d.x_sites = d.y_sites = d.z_sites = L;
  d.x_boundary_type = d.y_boundary_type = d.z_boundary_type = BOUNDARY_TYPE_PRD;
  d.cutoff = 2.0;
  GJP.Initialize(d);

  GeneralizedTwoBodyArg ga;
  ga.wavefunc_type = wf == "UNIFORM" ? WAVEFUNC_TYPE_UNIFORM
                     : wf == "PAIR1" ? WAVEFUNC_TYPE_PAIR1
                     : wf == "PAIR2" ? WAVEFUNC_TYPE_PAIR2
                                     : WAVEFUNC_TYPE_TGND;
  ga.distinct_vec = Vector3(vx, vy, vz);
  ga.lambda = lambda;
  GeneralizedTwoBody g(ga);
  const int vol = GJP.Vol();
  const int nt = g.oh_group.GetSubshellDimension();

  double* props = new double[4 * (size_t)vol];
  for (int i = 0; i < 4 * vol; ++i) {  // xorshift64* uniform in [-1, 1)
    state ^= state >> 12;
    state ^= state << 25;
    state ^= state >> 27;
    props[i] = (double)((state * 2685821657736338717ull) >> 11) / 9007199254740992.0 * 2.0 - 1.0;
  }
  FILE* f = fopen(out.c_str(), "wb");
  if (!f) return 2;
  fwrite(&nt, sizeof(int), 1, f);
  fwrite(&vol, sizeof(int), 1, f);
  fwrite(g.opposite_parity_index, sizeof(int), vol, f);
  fwrite(g.shift_indices, sizeof(int), (size_t)nt * vol, f);
  fwrite(g.half_site_wavefunc, sizeof(double), (size_t)nt * vol, f);
  for (int l = 0; l < nt; ++l)
    for (int r = 0; r < 10; ++r) {
      double w = g.oh_group.GetWeight((OctahedralRep)r, l);
      fwrite(&w, sizeof(double), 1, f);
    }
  fwrite(props, sizeof(double), 4 * (size_t)vol, f);
  for (int r = 0; r < 10; ++r) {
    complex<double> v = g.Run(props, props + 2 * vol, (OctahedralRep)r);
    double re = v.real(), im = v.imag();
    fwrite(&re, sizeof(double), 1, f);
    fwrite(&im, sizeof(double), 1, f);
  }
  for (int r = 0; r < 10; ++r) {
    complex<double> v = g.Run2(props, props + 2 * vol, (OctahedralRep)r);
    double re = v.real(), im = v.imag();
    fwrite(&re, sizeof(double), 1, f);
    fwrite(&im, sizeof(double), 1, f);
  }
  fclose(f);
  delete[] props;
  return 0;
}

// ref_driver.cc -- command-line driver over the reference's own CPU classes.
//
// TEST INFRASTRUCTURE ONLY.  Linked against the reference's unchanged
// src/*/*.C and src/*/noarch/*.C (compiled where they lie, by the Makefile in
// this directory) plus the FFTW shim.  It reproduces the call sequence of the
// reference's production drivers and dumps raw results in binary so that the
// oracle restatement (oracle/oracle.c) and the B200 library can be checked
// against the reference itself:
//
//   ensemble  -- the loop of production/slater_det/main.C:185-220 (mode=slater)
//                or production/slater_det2_trapped/main-no_cum.C:185-210
//                (mode=slater2); writes every per-configuration determinant
//                det S_n(tau) before any accumulation, and with
//                results=<dir> also the drivers' own result files
//                <dir>/slater.<m> (and <dir>/z<k>.<m> for cumulants=<Nc>),
//                a row per block of unload=<k> configurations, accumulated
//                and printed as production/slater_det/main.C:208-247 and
//                production/slater_det2_trapped/main-cum.C:219-270 do.
//   rng       -- Random::Uniform stream (src/random/random.C:100-103).
//   gauss     -- Random::Gauss stream (src/random/random.C:105-116).
//   field     -- Lattice::Refresh slices (src/alg/lattice.C:60-109).
//   lu        -- ludcmp + det on matrices read from a file (src/utils/ludcmp.C).
//   branch    -- the multilevel branching recursion of
//                production/two_body-branched/main.C:23-80 over the current
//                classes (see run_branch).
//   bench     -- the ensemble loop timed with clock_gettime, for the CPU baseline.
//
// Built twice: against the reference's CPU units (nrcps_ref) and, as
// nrcps_dropin, against its GPU configuration with the shims of
// nrcps_b200/shim in place of its CUDA units (the drop-in check).
//
// Arguments are key=value pairs; see parse_job() for the keys.

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <string>
#include <vector>

using namespace std;

#include "arg.h"
#include "constants.h"
#include "dispersion.h"
#include "enum.h"
#include "global_job_parameter.h"
#include "hamiltonian.h"
#include "lattice.h"
#include "ludcmp.h"
#include "momenta.h"
#include "one_body.h"
#include "propagator.h"
#include "random.h"
#include "slater_det.h"
#include "slater_det2.h"
#include "sysfunc.h"
#include "sysio.h"
#include "two_body.h"
#include "uniform_deviates.h"
#include "verbose.h"

#ifdef USE_GPU
#include <cuda_runtime.h>
#endif

namespace {

// Vectors handed out by the reference's classes are device pointers in its
// GPU build (Propagator::Get, OneBody::Get, Lattice::Get); copy to the host
// before writing them.
void to_host(double* dst, const double* src, size_t n) {
#ifdef USE_GPU
  cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost);
#else
  memcpy(dst, src, n * sizeof(double));
#endif
}

void write_vec(FILE* f, const double* src, size_t n) {
  vector<double> h(n);
  to_host(&h[0], src, n);
  fwrite(&h[0], sizeof(double), n, f);
}

typedef map<string, string> KV;

KV parse_kv(int argc, char** argv, int first) {
  KV kv;
  for (int i = first; i < argc; ++i) {
    const char* eq = strchr(argv[i], '=');
    if (!eq) {
      fprintf(stderr, "bad argument %s (want key=value)\n", argv[i]);
      exit(2);
    }
    kv[string(argv[i], eq - argv[i])] = string(eq + 1);
  }
  return kv;
}

string get(const KV& kv, const string& k, const string& dflt) {
  KV::const_iterator it = kv.find(k);
  return it == kv.end() ? dflt : it->second;
}
double getd(const KV& kv, const string& k, double d) {
  KV::const_iterator it = kv.find(k);
  return it == kv.end() ? d : atof(it->second.c_str());
}
long getl(const KV& kv, const string& k, long d) {
  KV::const_iterator it = kv.find(k);
  return it == kv.end() ? d : atol(it->second.c_str());
}

RandomType random_type_of(const string& s) {
  if (s == "RAN0") return RANDOM_TYPE_RAN0;
  if (s == "RAN1") return RANDOM_TYPE_RAN1;
  if (s == "RAN2") return RANDOM_TYPE_RAN2;
  if (s == "RAN3") return RANDOM_TYPE_RAN3;
  if (s == "RANLXS0") return RANDOM_TYPE_RANLXS0;
  if (s == "RANLXS1") return RANDOM_TYPE_RANLXS1;
  if (s == "RANLXS2") return RANDOM_TYPE_RANLXS2;
  if (s == "RANLXD1") return RANDOM_TYPE_RANLXD1;
  if (s == "RANLXD2") return RANDOM_TYPE_RANLXD2;
  fprintf(stderr, "unknown rng %s\n", s.c_str());
  exit(2);
}

FieldType field_type_of(const string& s) {
  if (s == "GAUSS") return FIELD_TYPE_GAUSS;
  if (s == "COMPLEXGAUSS") return FIELD_TYPE_COMPLEXGAUSS;
  if (s == "ZTWO") return FIELD_TYPE_ZTWO;
  if (s == "ZTHREE") return FIELD_TYPE_ZTHREE;
  fprintf(stderr, "unknown field %s\n", s.c_str());
  exit(2);
}

DispersionType disp_type_of(const string& s) {
  if (s == "STANDARD") return DISPERSION_TYPE_STANDARD;
  if (s == "QUADRATIC") return DISPERSION_TYPE_QUADRATIC;
  if (s == "PERFECT") return DISPERSION_TYPE_PERFECT;
  fprintf(stderr, "unknown dispersion %s\n", s.c_str());
  exit(2);
}

WavefuncType wavefunc_type_of(const string& s) {
  if (s == "NONE") return WAVEFUNC_TYPE_NONE;
  if (s == "UNIFORM") return WAVEFUNC_TYPE_UNIFORM;
  if (s == "GND") return WAVEFUNC_TYPE_GND;
  if (s == "TGND") return WAVEFUNC_TYPE_TGND;
  if (s == "PAIR1") return WAVEFUNC_TYPE_PAIR1;
  if (s == "PAIR2") return WAVEFUNC_TYPE_PAIR2;
  fprintf(stderr, "unknown wavefunc %s\n", s.c_str());
  exit(2);
}

vector<double> parse_list(const string& s) {
  vector<double> v;
  size_t pos = 0;
  while (pos < s.size()) {
    size_t c = s.find(',', pos);
    if (c == string::npos) c = s.size();
    v.push_back(atof(s.substr(pos, c - pos).c_str()));
    pos = c + 1;
  }
  return v;
}

void quiet() {
  VerboseArg va;
  va.func_level = false;
  va.warn_level = false;
  va.result_level = false;
  va.flow_level = false;
  va.debug_level = false;
  VRB.SetLevel(va);
}

void init_geometry(const KV& kv) {
  DoArg d;
  d.t_sites = (int)getl(kv, "T", 8);
  int L = (int)getl(kv, "L", 8);
  d.x_sites = (int)getl(kv, "Lx", L);
  d.y_sites = (int)getl(kv, "Ly", L);
  d.z_sites = (int)getl(kv, "Lz", L);
  d.x_boundary_type = BOUNDARY_TYPE_PRD;
  d.y_boundary_type = BOUNDARY_TYPE_PRD;
  d.z_boundary_type = BOUNDARY_TYPE_PRD;
  d.cutoff = getd(kv, "cutoff", 2.0);
  GJP.Initialize(d);
}

void make_random_arg(const KV& kv, RandomArg* ra) {
  ra->random_type = random_type_of(get(kv, "rng", "RANLXS2"));
  ra->seed_type = SEED_TYPE_INPUT;
  ra->seed = getl(kv, "seed", 1234);
  ra->file_stem = get(kv, "rngfile", "nrcps_ref_rng_state");
}

FILE* open_out(const string& path) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path.c_str());
    exit(2);
  }
  return f;
}

double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// Determinant of the leading n x n block of the row-major N x N matrix `m`
// (with an optional struck row s0 / column t0 taken from `row_s0` / `col_t0`),
// by the reference's ludcmp and d * prod U_ii (src/slater_det/slater_det.C:59-115,
// src/slater_det/slater_det2.C:78-148).  The reference builds this minor as a
// jagged array (one `new` per row, slater_det.C:78-80) and then hands
// &mat[0][0] to ludcmp, which indexes it as one contiguous n x n block; with
// glibc's allocator that reads allocator headers between rows (det S(0) = 0
// instead of 1 for n >= 3 on this machine).  The intended semantics -- the
// commented-out contiguous `complex<Float> mat[n][n]` at slater_det.C:77 --
// are used here, with the reference's own fill and ludcmp.
complex<double> minor_det(const vector<complex<double> >& m, int N, int n, int s0, int t0,
                          const vector<complex<double> >* psi1) {
  vector<complex<double> > a((size_t)n * n);
  for (int s = 0; s < n; ++s)
    for (int t = 0; t < n; ++t) a[(size_t)s * n + t] = m[(size_t)s * N + t];
  if (t0 >= 0 && t0 < n)
    for (int s = 0; s < n; ++s) a[(size_t)s * n + t0] = (*psi1)[s + (size_t)t0 * N];
  (void)s0;
  vector<int> indx(n);
  Float d;
  ludcmp(&a[0], n, &indx[0], &d);
  complex<double> det(d, 0.0);
  for (int i = 0; i < n; ++i) det *= a[(size_t)i * n + i];
  return det;
}

// ---------------------------------------------------------------- ensemble
// Mirrors production/slater_det/main.C:98-220 (mode=slater) and
// production/slater_det2_trapped/main-no_cum.C:85-210 (mode=slater2), with
// the MPI reduce and text output replaced by a binary dump of every raw
// determinant: dets[config][t][m] (complex double), m over the measured
// minors (N for slater, 2N for slater2: [Run(n+1,-1,n), Run(n+1,-1,-1)]).
int run_ensemble(const KV& kv, bool timed_only) {
  init_geometry(kv);
  Comms::Initialize();
  RandomArg random_arg;
  make_random_arg(kv, &random_arg);
  Random rng(random_arg);

  LatticeArg lattice_arg;
  lattice_arg.field_type = field_type_of(get(kv, "field", "ZTWO"));
  Lattice lattice(lattice_arg, &rng);

  InteractionArg interaction_arg;
  interaction_arg.mass = getd(kv, "imass", 1.0);
  interaction_arg.interaction_type =
      get(kv, "itype", "ONEMINUSXIINVSQ") == "XISQMINUSONE" ? INTERACTION_TYPE_XISQMINUSONE
                                                            : INTERACTION_TYPE_ONEMINUSXIINVSQ;
  interaction_arg.couplings = parse_list(get(kv, "couplings", "0.019894367886486918"));
  interaction_arg.num_couplings = interaction_arg.couplings.size();

  KineticArg kinetic_arg;
  kinetic_arg.dispersion_type = disp_type_of(get(kv, "kdisp", "PERFECT"));
  kinetic_arg.mass = getd(kv, "kmass", 1.0);

  const string mode = get(kv, "mode", "slater");
  const bool trapped = getl(kv, "potential", 0) != 0;

  PotentialArg potential_arg;
  potential_arg.potential_form = POTENTIAL_FORM_HARMONIC;
  potential_arg.potential_type = get(kv, "ptype", "EXP") == "LIN" ? POTENTIAL_TYPE_LIN : POTENTIAL_TYPE_EXP;
  potential_arg.spring_constant1 = getd(kv, "kappa", 0.005);
  potential_arg.spring_constant2 = getd(kv, "kappa", 0.005);
  potential_arg.spring_constant3 = getd(kv, "kappa", 0.005);

  Interaction interaction(&lattice, interaction_arg, getd(kv, "idt", 1.0));
  Kinetic kinetic(kinetic_arg, getd(kv, "kdt", 0.5));
  Potential* potential = 0;
  vector<Hamiltonian*> hamiltonians;
  hamiltonians.push_back(&kinetic);
  if (trapped) {
    potential = new Potential(potential_arg, getd(kv, "pdt", 0.5));
    hamiltonians.push_back(potential);
  }
  hamiltonians.push_back(&interaction);
  if (trapped) hamiltonians.push_back(potential);
  hamiltonians.push_back(&kinetic);

  // Sources.
  const string src = get(kv, "sources", "mom");
  int N = 0;
  vector<OneBody*> one_bodies;
  OneBodyArg one_body_arg;
  if (src == "mom") {
    MomentaArg momenta_arg;
    momenta_arg.dispersion_type = kinetic_arg.dispersion_type;
    momenta_arg.fermi_energy = getd(kv, "ef", 0.1);
    momenta_arg.mass = kinetic_arg.mass;
    Momenta momenta(momenta_arg);
    N = momenta.MomentaCount();
    one_body_arg.source_type = SOURCE_TYPE_MOM;
    for (int n = 0; n < N; ++n) {
      vector<int> p = momenta.GetMomentum(n);
      OneBody* ob = new OneBody(one_body_arg);
      ob->Set(p[0], p[1], p[2]);
      one_bodies.push_back(ob);
    }
    if (kv.count("out")) {
      FILE* f = open_out(get(kv, "out", ".") + "/momenta.txt");
      for (int n = 0; n < N; ++n) {
        vector<int> p = momenta.GetMomentum(n);
        fprintf(f, "%d %d %d %d\n", p[0], p[1], p[2], momenta.OppositeParityIndex(n));
      }
      fclose(f);
    }
  } else {
    // SHO sources from coefficient files: sho_dir/source.<n>
    N = (int)getl(kv, "N", 2);
    one_body_arg.source_type = SOURCE_TYPE_SHO;
    one_body_arg.lambda1 = getd(kv, "lambda1", 4.0);
    one_body_arg.lambda2 = getd(kv, "lambda2", 4.0);
    one_body_arg.lambda3 = getd(kv, "lambda3", 4.0);
    string dir = get(kv, "sho_dir", ".");
    for (int n = 0; n < N; ++n) {
      OneBody* ob = new OneBody(one_body_arg);
      char fn[512];
      snprintf(fn, sizeof fn, "%s/source.%d", dir.c_str(), n);
      ob->Set(string(fn));
      one_bodies.push_back(ob);
    }
  }

  TwoBody* two_body = 0;
  if (mode == "slater2") {
    TwoBodyArg tb;
    tb.wavefunc_type = wavefunc_type_of(get(kv, "wavefunc", "TGND"));
    tb.dispersion_type1 = disp_type_of(get(kv, "tb_disp", "STANDARD"));
    tb.dispersion_type2 = tb.dispersion_type1;
    tb.mass1 = getd(kv, "tb_mass", 1.0);
    tb.mass2 = tb.mass1;
    tb.lambda = getd(kv, "tb_lambda", 0.176776695);
    two_body = new TwoBody(tb);
  }

  const int vol = GJP.Vol();
  const string out = get(kv, "out", ".");
  if (!timed_only && kv.count("out")) {
    FILE* f = open_out(out + "/sources.bin");
    for (int n = 0; n < N; ++n) write_vec(f, one_bodies[n]->Get(), 2 * vol);
    fclose(f);
  }

  const int configs = (int)getl(kv, "configs", 1);
  const int T = GJP.Tsites();
  const int nmeas = (mode == "slater2") ? 2 * N : N;
  const long dump_fields = getl(kv, "dump_fields", 0);  // number of slices to dump
  const long dump_props = getl(kv, "dump_props", 0);    // number of slices (config 0) to dump

  PropagatorArg prop_arg;
  prop_arg.n_fermions = N;
  Propagator propagator(prop_arg);
  vector<Float*> props(N);
  for (int n = 0; n < N; ++n) props[n] = propagator.Get(n);

  FILE* fd = timed_only ? 0 : open_out(out + "/dets.bin");
  FILE* ff = (!timed_only && dump_fields > 0) ? open_out(out + "/fields.bin") : 0;
  FILE* fp = (!timed_only && dump_props > 0) ? open_out(out + "/props.bin") : 0;
  long slices_done = 0;
  double t0 = now_s();
  const double budget = getd(kv, "budget_s", 1e30);
  const long max_slices = getl(kv, "max_slices", -1);  // bounded sample for timing
  vector<complex<double> > row(nmeas);
  vector<complex<double> > smat((size_t)N * N), psi1((size_t)N * N);

  // The drivers' block accumulators and result files (Comms::Size() is 1
  // here, so GlobalSum is the identity and block_size = unload_period).
  const string results = get(kv, "results", "");
  const int unload = (int)getl(kv, "unload", 1);
  const int Nc = (int)getl(kv, "cumulants", 0);
  vector<FILE*> rfile, zfile;
  vector<complex<Float> > corr((size_t)nmeas * T, complex<Float>(0.0, 0.0));
  vector<complex<Float> > zacc((size_t)(Nc > 0 ? Nc : 1) * nmeas * T, complex<Float>(0.0, 0.0));
  vector<complex<Float> > cum(Nc > 0 ? Nc : 1);
  if (!timed_only && !results.empty()) {
    char f_name[512];
    for (int m = 0; m < nmeas; ++m) {
      snprintf(f_name, sizeof f_name, "%s/slater.%d", results.c_str(), m + 1);
      rfile.push_back(Fopen(IO_TYPE_ROOT, f_name, "a"));
      for (int nc = 0; nc < Nc; ++nc) {
        snprintf(f_name, sizeof f_name, "%s/z%d.%d", results.c_str(), nc + 1, m + 1);
        zfile.push_back(Fopen(IO_TYPE_ROOT, f_name, "a"));  // zfile[m * Nc + nc]
      }
    }
  }

  for (int j = 0; j < configs; ++j) {
    for (int n = 0; n < N; ++n) propagator.Set(one_bodies[n]->Get(), n);
    for (int t = 0; t < T; ++t) {
      if (fp && j == 0 && t < dump_props) {
        for (int n = 0; n < N; ++n) write_vec(fp, props[n], 2 * vol);
      }
      if (mode == "slater2") {
        // production/slater_det2_trapped/main-no_cum.C:201-208: pair matrix from
        // SlaterDet2's own fill, one-body column psi1[t+N*s] = <src_s|prop_t>.
        SlaterDet2 sd(&props[0], &props[0], &one_bodies[0], NULL, two_body, N);
        for (int s = 0; s < N; ++s)
          for (int t = 0; t < N; ++t) {
            smat[(size_t)s * N + t] = sd.SlaterMat(s, t);
            psi1[t + (size_t)N * s] = one_bodies[s]->Project(props[t]);
          }
        for (int n = 0; n < N; ++n) {
          row[2 * n + 1] = minor_det(smat, N, n + 1, -1, -1, &psi1);
          row[2 * n] = minor_det(smat, N, n + 1, -1, n, &psi1);
        }
      } else {
        // production/slater_det/main.C:206-211 with SlaterDet's own fill.
        SlaterDet sd(&props[0], &one_bodies[0], N);
        for (int s = 0; s < N; ++s)
          for (int t = 0; t < N; ++t) smat[(size_t)s * N + t] = sd.SlaterMat(s, t);
        for (int n = 0; n < N; ++n) row[n] = minor_det(smat, N, n + 1, -1, -1, 0);
      }
      if (fd) fwrite(&row[0], sizeof(complex<double>), nmeas, fd);
      if (!rfile.empty()) {
        for (int m = 0; m < nmeas; ++m) {
          complex<Float> slat = row[m];
          // main.C:209-210 (|det|^2 as tmp * conj(tmp)); main-no_cum.C:205-207 (det)
          corr[(size_t)m * T + t] += (mode == "slater2") ? slat : slat * conj(slat);
          if (Nc > 0) {  // main-cum.C:220-224
            cum[0] = log(abs(slat));
            for (int nc = 1; nc < Nc; ++nc) cum[nc] = cum[0] * cum[nc - 1];
            for (int nc = 0; nc < Nc; ++nc) zacc[((size_t)nc * nmeas + m) * T + t] += cum[nc];
          }
        }
      }
      if (ff && slices_done < dump_fields) {
        write_vec(ff, lattice.Get(), 2 * vol);
      }
      for (size_t p = 0; p < hamiltonians.size(); ++p) hamiltonians[p]->Initialize();
      propagator.Run(hamiltonians);
      lattice.Refresh();
      ++slices_done;
      if (max_slices > 0 && slices_done >= max_slices) break;
    }
    if (max_slices > 0 && slices_done >= max_slices) break;
    if (timed_only && now_s() - t0 > budget) break;
    if (!rfile.empty() && (j + 1) % unload == 0) {
      // main.C:225-247 / main-cum.C:256-270 with Comms::Size() = 1
      Float block_size = Comms::Size() * unload;
      for (int m = 0; m < nmeas; ++m) {
        for (int t = 0; t < T; ++t) {
          complex<Float>& c = corr[(size_t)m * T + t];
          Fprintf(rfile[m], "%.*e %.*e ", PREC, c.real() / block_size, PREC, c.imag() / block_size);
          c = 0.0;
          for (int nc = 0; nc < Nc; ++nc) {
            complex<Float>& zz = zacc[((size_t)nc * nmeas + m) * T + t];
            Fprintf(zfile[(size_t)m * Nc + nc], "%.*e ", PREC, zz.real() / block_size);
            zz = 0.0;
          }
        }
        Fprintf(rfile[m], "\n");
        for (int nc = 0; nc < Nc; ++nc) Fprintf(zfile[(size_t)m * Nc + nc], "\n");
      }
    }
  }
  for (size_t i = 0; i < rfile.size(); ++i) Fclose(rfile[i]);
  for (size_t i = 0; i < zfile.size(); ++i) Fclose(zfile[i]);
  double el = now_s() - t0;
  if (fd) fclose(fd);
  if (ff) fclose(ff);
  if (fp) fclose(fp);
  printf("{\"slices\": %ld, \"seconds\": %.6f, \"config_slices_per_s\": %.6f, \"N\": %d, \"V\": %d}\n",
         slices_done, el, slices_done / el, N, vol);
  for (int n = 0; n < N; ++n) delete one_bodies[n];
  delete potential;
  delete two_body;
  return 0;
}

// ---------------------------------------------------------------- rng
int run_rng(const KV& kv, bool gauss) {
  Comms::Initialize();
  RandomArg ra;
  make_random_arg(kv, &ra);
  Random rng(ra);
  long skip = getl(kv, "skip", 0), count = getl(kv, "count", 16);
  for (long i = 0; i < skip; ++i) (void)(gauss ? rng.Gauss(1.0) : rng.Uniform());
  FILE* f = open_out(get(kv, "out", "rng.bin"));
  for (long i = 0; i < count; ++i) {
    double u = gauss ? rng.Gauss(1.0) : rng.Uniform();
    fwrite(&u, sizeof u, 1, f);
  }
  fclose(f);
  return 0;
}

// ---------------------------------------------------------------- field
int run_field(const KV& kv) {
  init_geometry(kv);
  Comms::Initialize();
  RandomArg ra;
  make_random_arg(kv, &ra);
  Random rng(ra);
  LatticeArg la;
  la.field_type = field_type_of(get(kv, "field", "ZTWO"));
  Lattice lattice(la, &rng);
  long slices = getl(kv, "slices", 1);
  FILE* f = open_out(get(kv, "out", "field.bin"));
  for (long s = 0; s < slices; ++s) {
    fwrite(lattice.Get(), sizeof(double), lattice.FieldSize(), f);
    lattice.Refresh();
  }
  fclose(f);
  return 0;
}

// ---------------------------------------------------------------- lu
// Input file: int32 count, int32 n, then count*n*n complex doubles (row-major).
// Output: count complex dets.
int run_lu(const KV& kv) {
  FILE* f = fopen(get(kv, "in", "mats.bin").c_str(), "rb");
  if (!f) return 2;
  int hdr[2];
  if (fread(hdr, sizeof(int), 2, f) != 2) return 2;
  int count = hdr[0], n = hdr[1];
  vector<complex<double> > m((size_t)n * n);
  vector<int> indx(n);
  FILE* g = open_out(get(kv, "out", "dets.bin"));
  for (int c = 0; c < count; ++c) {
    if (fread(&m[0], sizeof(complex<double>), (size_t)n * n, f) != (size_t)n * n) return 2;
    Float d;
    ludcmp(&m[0], n, &indx[0], &d);
    complex<double> det(d, 0.0);
    for (int i = 0; i < n; ++i) det *= m[(size_t)i * n + i];
    fwrite(&det, sizeof det, 1, g);
  }
  fclose(f);
  fclose(g);
  return 0;
}

}  // namespace

// ---------------------------------------------------------------- branch
// The multilevel branching driver of production/two_body-branched/main.C:23-80
// (MultiLevel), written against the reference's current classes: that file
// still calls Propagator::SetSource, Get() and Interaction3, which its headers
// no longer declare, so it does not compile.  The recursion is kept as is;
// Set(psi, 0) and Get(0) stand for SetSource(psi) and Get() of a
// one-orbital Propagator, and the Hamiltonians are [K, I, K] (one coupling).
struct Branch {
  int branches, steps, levels;
  Propagator *prop1, *prop2;
  TwoBody* two_body;
  Lattice* lattice;
  vector<Hamiltonian*> hamiltonians;
  vector<complex<Float> >* corr;
};

void multi_level(Branch& b, int level) {
  if (level <= 0) return;
  const int vol = GJP.Vol();
  Float* p1 = b.prop1->Get(0);
  Float* p2 = b.prop2->Get(0);
  vector<Float> source1(p1, p1 + 2 * vol), source2(p2, p2 + 2 * vol);
  const Float norm = pow((Float)b.branches, (Float)(b.levels - level + 1));
  for (int i = 0; i < b.branches; ++i) {
    b.prop1->Set(&source1[0], 0);
    b.prop2->Set(&source2[0], 0);
    for (int s = 0; s < b.steps; ++s) {
      const int t = GJP.Tsites() - (level - 1) * b.steps - (b.steps - s);
      (*b.corr)[t] += (b.two_body->Run(p1, p2) / norm);
      for (size_t p = 0; p < b.hamiltonians.size(); ++p) b.hamiltonians[p]->Initialize();
      b.prop1->Run(b.hamiltonians);
      b.prop2->Run(b.hamiltonians);
      b.lattice->Refresh();
    }
    multi_level(b, level - 1);
  }
}

// Keys: L, levels, branches, steps, trees, seed, rng, field, couplings,
// cutoff, p1 / p2 (momentum of each plane-wave source, "n1,n2,n3"),
// wavefunc, tb_disp, tb_lambda, out (corr[T] complex doubles, summed over
// the trees).
int run_branch(const KV& kv) {
  KV g = kv;
  const int levels = (int)getl(kv, "levels", 3), steps = (int)getl(kv, "steps", 2);
  char tbuf[32];
  snprintf(tbuf, sizeof tbuf, "%d", levels * steps);
  g["T"] = tbuf;
  init_geometry(g);
  Comms::Initialize();
  RandomArg random_arg;
  make_random_arg(kv, &random_arg);
  Random rng(random_arg);
  LatticeArg lattice_arg;
  lattice_arg.field_type = field_type_of(get(kv, "field", "ZTWO"));
  Lattice lattice(lattice_arg, &rng);
  InteractionArg interaction_arg;
  interaction_arg.mass = 1.0;
  interaction_arg.interaction_type = INTERACTION_TYPE_ONEMINUSXIINVSQ;
  interaction_arg.couplings = parse_list(get(kv, "couplings", "0.019894367886486918"));
  interaction_arg.num_couplings = interaction_arg.couplings.size();
  KineticArg kinetic_arg;
  kinetic_arg.dispersion_type = DISPERSION_TYPE_PERFECT;
  kinetic_arg.mass = 1.0;
  Interaction interaction(&lattice, interaction_arg, 1.0);
  Kinetic kinetic(kinetic_arg, 0.5);
  OneBodyArg one_body_arg;
  one_body_arg.source_type = SOURCE_TYPE_MOM;
  OneBody source1(one_body_arg), source2(one_body_arg);
  vector<double> m1 = parse_list(get(kv, "p1", "0,0,0")), m2 = parse_list(get(kv, "p2", "0,0,0"));
  source1.Set((int)m1[0], (int)m1[1], (int)m1[2]);
  source2.Set((int)m2[0], (int)m2[1], (int)m2[2]);
  TwoBodyArg tb;
  tb.wavefunc_type = wavefunc_type_of(get(kv, "wavefunc", "TGND"));
  tb.dispersion_type1 = disp_type_of(get(kv, "tb_disp", "STANDARD"));
  tb.dispersion_type2 = tb.dispersion_type1;
  tb.mass1 = tb.mass2 = 1.0;
  tb.lambda = getd(kv, "tb_lambda", 0.176776695);
  TwoBody two_body(tb);
  PropagatorArg prop_arg;
  prop_arg.n_fermions = 1;
  Propagator prop1(prop_arg), prop2(prop_arg);
  vector<complex<Float> > corr(GJP.Tsites(), complex<Float>(0.0, 0.0));
  Branch b;
  b.branches = (int)getl(kv, "branches", 2);
  b.steps = steps;
  b.levels = levels;
  b.prop1 = &prop1;
  b.prop2 = &prop2;
  b.two_body = &two_body;
  b.lattice = &lattice;
  b.hamiltonians.push_back(&kinetic);
  b.hamiltonians.push_back(&interaction);
  b.hamiltonians.push_back(&kinetic);
  b.corr = &corr;
  const int trees = (int)getl(kv, "trees", 1);
  for (int r = 0; r < trees; ++r) {
    prop1.Set(source1.Get(), 0);
    prop2.Set(source2.Get(), 0);
    multi_level(b, levels);
  }
  FILE* f = open_out(get(kv, "out", "branch.bin"));
  fwrite(&corr[0], sizeof(complex<Float>), corr.size(), f);
  fclose(f);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s ensemble|bench|rng|gauss|field|lu|branch key=value...\n", argv[0]);
    return 2;
  }
  quiet();
  KV kv = parse_kv(argc, argv, 2);
  string cmd = argv[1];
  if (cmd == "ensemble") return run_ensemble(kv, false);
  if (cmd == "bench") return run_ensemble(kv, true);
  if (cmd == "rng") return run_rng(kv, false);
  if (cmd == "gauss") return run_rng(kv, true);
  if (cmd == "field") return run_field(kv);
  if (cmd == "lu") return run_lu(kv);
  if (cmd == "branch") return run_branch(kv);
  fprintf(stderr, "unknown command %s\n", cmd.c_str());
  return 2;
}

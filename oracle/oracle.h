/*
 * oracle.h -- CPU restatement of nrCPS's auxiliary-field transfer-matrix path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the B200 library: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it,
 * and only to compare against.  The product path never links it.
 *
 * Every function restates one piece of the reference (file:line of
 * mgendres/nrCPS v2_7_6 cited beside it) with the same arithmetic order, so
 * that it agrees bit-for-bit with the reference compiled from its own sources
 * (oracle/ref_build), which tests/test_oracle_vs_reference.py checks.  It is
 * pinned further by the reference's known-answer tests (tests/ranlx,
 * tests/ludcmp_test) and by numpy.fft for the transform.
 *
 * Layout conventions follow the reference: a lattice site (x,y,z) has index
 * z + Z*(y + Y*x) (src/utils/vector3.C:190-215); complex arrays are
 * interleaved (re, im) doubles.
 */
#ifndef NRCPS_ORACLE_H
#define NRCPS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ RNG */
/* Generator kinds, numbered as the reference's RandomType (include/enum.h). */
enum { O_RAN0 = 0, O_RAN1, O_RAN2, O_RAN3, O_RANLXS0, O_RANLXS1, O_RANLXS2, O_RANLXD1, O_RANLXD2 };

typedef struct {
  int kind;
  /* ranlux */
  int num[96];
  int carry[4];
  int pr, prm, ir, jr, is, is_old;
  int next[96];
  int dbl; /* 1 for ranlxd */
  /* ran2 */
  long idum, idum2, iy, iv[32];
} o_rng;

void o_rng_init(o_rng *r, int kind, long seed);
double o_rng_uniform(o_rng *r);
double o_rng_gauss(o_rng *r, double sigma);
int o_rng_z(o_rng *r, int p);
/* Reference binary state layout (src/random/ranlxs.C GetState: 105 longs). */
void o_rng_get_state(const o_rng *r, long *state);
void o_rng_set_state(o_rng *r, const long *state);

/* Convenience: `count` uniforms after skipping `skip`, from a fresh generator. */
void o_uniforms(int kind, long seed, long skip, long count, double *out);
void o_gaussians(int kind, long seed, long skip, long count, double *out);

/* Field types, numbered as the reference's FieldType. */
enum { O_FIELD_GAUSS = 0, O_FIELD_COMPLEXGAUSS, O_FIELD_ZTWO, O_FIELD_ZTHREE };
/* Lattice::Refresh (src/alg/lattice.C:60-109) for `slices` consecutive slices
 * of `vol` sites; out = slices * 2*vol doubles. */
void o_field_slices(o_rng *r, int field_type, long vol, long slices, double *out);

/* --------------------------------------------------------------- tables */
enum { O_DISP_STANDARD = 0, O_DISP_QUADRATIC, O_DISP_PERFECT };
enum { O_CUTOFF_NONE = 0, O_CUTOFF_HARD };
void o_dispersion(const int dims[3], int type, double mass, int cutoff_type, double cutoff_sq,
                  double *out);
void o_kinetic_xi(const int dims[3], int type, double mass, double dt, double cutoff_sq, double *out);
enum { O_ITYPE_NONE = 0, O_ITYPE_XISQMINUSONE, O_ITYPE_ONEMINUSXIINVSQ };
int o_interaction_table(const int dims[3], double mass, int itype, const double *couplings, int ncoup,
                        double dt, double cutoff_sq, double *out);
enum { O_POT_LIN = 0, O_POT_EXP };
void o_potential_table(const int dims[3], int ptype, double k1, double k2, double k3, double dt,
                       double *out);
/* Momenta (src/alg/momenta.C:12-139): returns the count; fills idx (lattice
 * index of each momentum in sorted order), energies and parity partners. */
int o_momenta(const int dims[3], int disp_type, double mass, double fermi_energy, double cutoff_sq,
              int *idx, double *energy, int *parity, int cap);
/* SHO source (src/one_body/one_body.C:53-171); coeffs = V complex with the
 * file coefficients stored at their lattice index. */
void o_sho_source(const int dims[3], double l1, double l2, double l3, const double *coeffs,
                  double *psi);
double o_dawson(double x);
enum { O_WF_NONE = 0, O_WF_UNIFORM, O_WF_GND, O_WF_TGND, O_WF_PAIR1, O_WF_PAIR2 };
void o_two_body_tables(const int dims[3], int wf_type, int disp1, int disp2, double m1, double m2,
                       double lambda, double cutoff_sq, double *wavefunc, int *opp);

/* ---------------------------------------------------------- propagation */
void o_interaction_initialize(const int dims[3], const double *lat, const double *itab, double *fld);
void o_kinetic_evolve(long vol, int batch, double *psi, const double *xi);
void o_potential_evolve(const int dims[3], int batch, double *psi, const double *pot);
void o_interaction_evolve(const int dims[3], int batch, double *psi, const double *fld);

/* ---------------------------------------------------------- measurement */
void o_project(long vol, int ns, const double *src, int nt, const double *psi, double *S);
void o_pair_matrix(long vol, int n, const double *psi1, const double *psi2, const double *wf,
                   const int *opp, double *phi);
/* ludcmp (src/utils/ludcmp.C:9-65) on a row-major n x n complex matrix, in place. */
int o_ludcmp(double *a, int n, int *indx, double *d);
/* det (det_type 0) or log det (det_type 1) of the leading n x n block of an
 * N x N row-major complex matrix, optional struck column t0 from psi1. */
void o_minor_det(const double *S, int N, int n, int t0, const double *psi1, int det_type, double *out);

/* ------------------------------------------------------------- ensemble */
typedef struct {
  int dims[3];
  int T;
  int n_orb;            /* N */
  int configs;
  int rng_kind;
  long seed;
  int field_type;
  double kin_mass, kin_dt;
  int kin_disp;
  double cutoff_sq;
  double int_mass, int_dt;
  int int_type;
  int n_coup;
  double coup[8];
  int use_potential;
  int pot_type;
  double pot_k[3], pot_dt;
  int mode;             /* 0: slater (N minors), 1: slater2 (2N: [struck col n, full]) */
  int wf_type, wf_disp;
  double wf_mass, wf_lambda;
} o_job;

/* Runs the production-driver loop (production/slater_det/main.C:185-220 or
 * production/slater_det2_trapped/main-no_cum.C:185-210) for job->configs
 * configurations from a fresh generator.  sources = n_orb * V complex.
 * dets = configs * T * nmeas complex (nmeas = N or 2N). */
int o_run_ensemble(const o_job *job, const double *sources, double *dets);

/* Jobs run one after another by one process with ONE generator (the stream
 * semantics of nrcps_batch): job j = (L_j, T_j, n_conf_j) with plane-wave
 * sources idx_j (N_j lattice indices), local interaction fld = (1 + a phi)/V,
 * Kinetic xi from (disp PERFECT, mass 1, dt, cutoff_sq); dets_j =
 * [n_conf_j][T_j][N_j] complex.  Slice t of configuration k of job j is the
 * (k T_j + t)-th field drawn after all earlier jobs' fields. */
/* The multilevel branching driver (production/two_body-branched/main.C:23-80,
 * MultiLevel) for `trees` trees of depth `levels`, `branches` branches per
 * node and `steps` steps per level, T = levels * steps: corr[t] (complex,
 * summed over trees) accumulates TwoBody::Run(prop1, prop2) / branches^(d+1)
 * over the nodes of depth d = t / steps.  Hamiltonians [K, I, K] with the
 * local interaction (1 + a phi)/V (the reference driver's Interaction3 and
 * Propagator::SetSource no longer exist in its headers); fields from one
 * generator in the recursion's order. */
void o_run_branching(const int dims[3], int levels, int branches, int steps, int trees, int rng_kind, long seed,
                     int field_type, double a, double kin_dt, double cutoff_sq, const double *sources2,
                     const double *wf, const int *opp, double *corr);

void o_run_batch(int njobs, const int *L, const int *T, const int *nconf, const int *N, const int *const *idx,
                 int rng_kind, long seed, int field_type, double a, double kin_dt, double cutoff_sq,
                 double *const *dets);

#ifdef __cplusplus
}
#endif
#endif

/*
 * nrcps_b200.h -- C ABI of libnrcps_b200.so, the B200 (sm_100a) implementation
 * of nrCPS's auxiliary-field transfer-matrix hot path.
 *
 * The reference (mgendres/nrCPS v2_7_6) swaps its CPU and GPU backends per
 * translation unit behind fixed class headers (include/fourier.h,
 * include/hamiltonian.h, include/propagator.h, include/one_body.h,
 * include/two_body.h, include/slater_det*.h, include/lattice.h,
 * include/random.h, include/cuda_utils.h).  Every entry point below replaces
 * one of those GPU translation units' methods (cited beside it); the C++
 * shims that re-implement the class methods over this ABI live in
 * nrcps_b200/shim/.  Plain pointers and sizes only: device pointers are
 * CUDA device addresses, host pointers are ordinary host memory.
 *
 * Conventions shared with the reference:
 *   - lattice site (x,y,z) has index z + Z*(y + Y*x) (src/utils/vector3.C:190-215);
 *   - an orbital is V = X*Y*Z complex numbers in momentum space, interleaved
 *     (re, im); a batch of orbitals is contiguous, orbital n at offset n*V;
 *   - sign -1 is FFTW_FORWARD (momentum -> position), +1 FFTW_BACKWARD;
 *     transforms are unnormalised (src/fourier/noarch/fourier.C:34-35).
 *
 * Errors: every call returns nrcps_status; nothing in the library exits or
 * traps.  The reference instead prints and calls exit() (src/utils/error.C:36-46);
 * the shims translate a non-OK status into ERR.General to keep that behaviour.
 * nrcps_last_error() describes the most recent failure on a context.
 *
 * Threading: a context is used by one host thread at a time; all its work is
 * queued on the context's stream (nrcps_set_stream).
 */
#ifndef NRCPS_B200_H
#define NRCPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Every entry point below is exported even when the library is built with
 * hidden default visibility. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum {
  NRCPS_OK = 0,
  NRCPS_ERR_INVALID_ARGUMENT = 1,
  NRCPS_ERR_UNSUPPORTED = 2,
  NRCPS_ERR_CUDA = 3,
  NRCPS_ERR_OUT_OF_MEMORY = 4,
  NRCPS_ERR_SINGULAR = 5,  /* ludcmp's "singular matrix" (src/utils/ludcmp.C:31-34) */
  NRCPS_ERR_NONFINITE = 6,
  NRCPS_ERR_TIMEOUT = 7
} nrcps_status;

typedef enum { NRCPS_F64 = 0, NRCPS_F32 = 1 } nrcps_precision;

/* Generator kinds, numbered as the reference's RandomType (include/enum.h:7-18). */
typedef enum {
  NRCPS_RAN0 = 0, NRCPS_RAN1 = 1, NRCPS_RAN2 = 2, NRCPS_RAN3 = 3,
  NRCPS_RANLXS0 = 4, NRCPS_RANLXS1 = 5, NRCPS_RANLXS2 = 6,
  NRCPS_RANLXD1 = 7, NRCPS_RANLXD2 = 8
} nrcps_rng_kind;

/* Field kinds, numbered as the reference's FieldType (include/enum.h:27-33). */
typedef enum {
  NRCPS_FIELD_GAUSS = 0, NRCPS_FIELD_COMPLEXGAUSS = 1,
  NRCPS_FIELD_ZTWO = 2, NRCPS_FIELD_ZTHREE = 3
} nrcps_field_kind;

typedef struct nrcps_context nrcps_context;

/* ------------------------------------------------------------ lifecycle */
nrcps_status nrcps_create(int device, nrcps_context **ctx);
nrcps_status nrcps_destroy(nrcps_context *ctx);
const char *nrcps_last_error(const nrcps_context *ctx);
/* cudaStream_t passed as void*; NULL selects the legacy default stream. */
nrcps_status nrcps_set_stream(nrcps_context *ctx, void *stream);
/* Waits for the context's stream; returns NRCPS_ERR_TIMEOUT if a kernel's
 * bounded wait (on an asynchronous bulk copy) gave up since the last call. */
nrcps_status nrcps_synchronize(nrcps_context *ctx);
/* Library version string, e.g. "nrcps_b200 0.1 sm_100a". */
const char *nrcps_version(void);
/* Tuning options of a context (no counterpart in the reference, whose launch
 * shape is the compile-time BLOCKS/THREADS of include/config.h:30-33):
 *   "propagate.fused"  1 (default): single-pass cluster kernel where one
 *                      exists for the shape; 0: five pencil passes;
 *   "fused.cluster"    0 (default): autotuned cluster size; else force it;
 *   "fused.split"      -1 (default): autotuned; 0: one thread per pencil;
 *                      1: each pencil split over two lanes;
 *   "fused.kind"       -1 (default): autotuned; 0: one thread per pencil,
 *                      the x-pass reads and writes peers' shared memory;
 *                      1: lane split; 2: whole regions move between CTAs
 *                      by bulk copy; 3: as 2, with the slab prefetched into
 *                      L2 instead of staged in shared memory; 4, 5, 6: kinds
 *                      0, 2, 3 with packed FP32x2 transforms (two
 *                      half-length DFTs per instruction; FP32 only); 7, 8:
 *                      kinds 0, 4 with the slab prefetched into L2 instead
 *                      of staged in shared memory (four CTAs per SM);
 *                      9, 10: kinds 6, 3 with the CTA's slab of the
 *                      kinetic table resident in shared memory (FP32);
 *                      11, 12: kinds 7, 8 with the x pass written back by
 *                      st.async onto the owner CTA's mbarrier (one cluster
 *                      barrier per orbital);
 *   "overlap.tc"       1 (default): dense-source overlaps of FP32 orbitals
 *                      on the tcgen05 tensor cores (TF32 hi/lo split, FP32
 *                      accumulation) where V is a multiple of 16; 0: the
 *                      CUDA-core kernel with FP64 accumulation;
 *   "fused.zpos"       1 (default): for a Z2 field with a position factor the
 *                      fused step reads both weights of every site,
 *                      (1 +- a) P(x)/V, from a table made ahead of the step;
 *                      0: forms them per site (the same values);
 *   "pair.tile"        1 (default): TwoBody pair matrices (n <= 32) by tiles of
 *                      sites staged in shared memory, one thread-block cluster
 *                      per configuration; 0: one block per (s, t) pair;
 *   "qr.gram_tc"       1: the Gram matrices of the re-orthonormalisation of
 *                      FP32 orbitals (N <= 32) on the tcgen05 tensor cores
 *                      (TF32 hi/lo); 0 (default): the CUDA-core kernel;
 *   "batch.real_weights" 1 (default): a batch created afterwards with FP32
 *                      orbitals and a real Gaussian field turns each run's
 *                      field into one FP32 weight per site, (1 + a phi)/V
 *                      rounded once, which the fused step stages in shared
 *                      memory; 0: the step forms the weight from phi per
 *                      site and orbital (split into two FP32 parts);
 *   "batch.prefetch_fields" 1 (default): such a batch (FP32 weights) draws
 *                      the next run's fields on a side stream while a run's
 *                      graph executes, into a second weight buffer (the same
 *                      stream windows, the same results); 0: each run draws
 *                      its own fields before its graph;
 *   "lu.warp"          1 (default): leading-minor determinants with one warp
 *                      per minor in shared memory (N <= 64); 0: one thread
 *                      per minor with global scratch;
 *   "fused.wait_ns"    time limit of every mbarrier wait in the fused step,
 *                      in nanoseconds (default 2e9, minimum 1000).  A wait
 *                      that runs out sets the context's time-out flag and
 *                      its whole cluster leaves the orbital loop; the next
 *                      nrcps_synchronize returns NRCPS_ERR_TIMEOUT;
 *   "fused.stall_test" 1: the first wait of one CTA of the next fused steps
 *                      is made on an mbarrier nothing arrives on, so that it
 *                      runs out (a test of the time-out path); 0 (default). */
nrcps_status nrcps_set_option(nrcps_context *ctx, const char *name, long value);
/* Times every fused-kernel variant (cluster size, lane split) for (prec, L)
 * on this device and keeps the fastest for later calls; *cluster receives
 * its cluster size, negated for the lane-split variants (may be NULL). */
nrcps_status nrcps_autotune(nrcps_context *ctx, nrcps_precision prec, int L, int *cluster);
/* The fused-kernel variant that nrcps_propagate uses for (prec, L^3) on this
 * context's device under its current options (no counterpart in the
 * reference; it names the kernel behind a measurement): *kind (0..12, see
 * "fused.kind") and *cluster (CTAs per cluster); both -1 when no fused
 * variant serves the shape.  Tunes nothing. */
nrcps_status nrcps_fused_choice(nrcps_context *ctx, nrcps_precision prec, int L, int *kind, int *cluster);

/* ----------------------------------------------------- host-side tables
 * Replace the reference's host constructors' table builds so that callers
 * without the reference classes get identical tables.  All outputs are host
 * arrays of V doubles unless stated. cutoff_sq = (DoArg.cutoff * pi)^2. */

/* Dispersion ctor (src/alg/dispersion.C:11-75); type = DispersionType,
 * hard_cutoff = CutoffType.  Periodic boundaries. */
nrcps_status nrcps_dispersion_table(const int dims[3], int type, double mass, int hard_cutoff,
                                    double cutoff_sq, double *out);
/* Kinetic ctor (src/hamiltonian/hamiltonian.C:260-281): xi = 1 + disp(m/dt). */
nrcps_status nrcps_kinetic_table(const int dims[3], int type, double mass, double dt,
                                 double cutoff_sq, double *xi);
/* Interaction ctor (src/hamiltonian/hamiltonian.C:77-147): momentum factor
 * c(p) incl. 1/V and dt; itype = InteractionType. */
nrcps_status nrcps_interaction_table(const int dims[3], double mass, int itype,
                                     const double *couplings, int ncoup, double dt,
                                     double cutoff_sq, double *out);
/* Potential ctor (src/hamiltonian/hamiltonian.C:165-244), harmonic form;
 * ptype = PotentialType (0 LIN, 1 EXP).  Includes 1/V. */
nrcps_status nrcps_potential_table(const int dims[3], int ptype, double k1, double k2, double k3,
                                   double dt, double *out);
/* Momenta ctor (src/alg/momenta.C:12-139).  Writes up to cap entries of the
 * energy-sorted momenta (lattice index, energy, opposite-parity slot) and
 * stores the total count in *count. */
nrcps_status nrcps_momenta(const int dims[3], int disp_type, double mass, double fermi_energy,
                           double cutoff_sq, int cap, int *index, double *energy, int *parity,
                           int *count);
/* OneBody::Set() SHO branch (src/one_body/one_body.C:66-166): coeffs = V
 * complex with each file coefficient (n1,n2,n3,re,im) at its lattice index;
 * psi = V complex. */
nrcps_status nrcps_sho_source(const int dims[3], double lambda1, double lambda2, double lambda3,
                              const double *coeffs, double *psi);
/* TwoBody ctor (src/two_body/two_body.C:21-141): pair wave function w (V
 * doubles) and opposite-parity index (V ints).  wf_type = WavefuncType. */
nrcps_status nrcps_two_body_tables(const int dims[3], int wf_type, int disp1, int disp2, double m1,
                                   double m2, double lambda, double cutoff_sq, double *w,
                                   int *opposite);

/* ------------------------------------------------------------------ RNG
 * UniformDeviate/Random replacements (src/random/*.C).  The stream is the
 * reference's: generator `kind` seeded with `seed` (the reference adds
 * 491*rank first, src/random/random.C:88). */

/* Reference binary state after Init(seed) (105 longs for ranlux,
 * src/random/ranlxs.C:193-213; 36 for ran2, src/random/ran2.C:85-95). */
nrcps_status nrcps_rng_seed_state(int kind, long seed, long *state, int *state_size);
/* Advance a ranlux state by n uniforms without generating them (exact
 * skip-ahead through the generator's equivalent linear congruential form). */
nrcps_status nrcps_rng_skip(int kind, long *state, uint64_t n);
/* `count` uniforms from stream position `offset` of (kind, seed), generated
 * on the GPU into dev_out (doubles).  Bit-identical to Random::Uniform. */
nrcps_status nrcps_rng_uniforms(nrcps_context *ctx, int kind, long seed, uint64_t offset,
                                uint64_t count, double *dev_out);

/* Lattice::Refresh (src/alg/lattice.C:60-109) on the GPU: `slices`
 * consecutive field slices of `vol` sites starting at uniform position
 * *offset of (kind, seed); writes interleaved complex doubles (2*vol per
 * slice) to dev_out and advances *offset past the uniforms consumed.
 * Z2/Z3 consume one uniform per site; Gauss consumes a data-dependent number
 * (polar rejection, src/random/random.C:105-116). */
nrcps_status nrcps_draw_fields(nrcps_context *ctx, int kind, long seed, int field_kind, long vol,
                               long slices, uint64_t *offset, double *dev_out);
/* Z2 fields as packed sign bits: bit u of dev_bits (32-bit words) is set when
 * the site drawn from uniform u of the stream window has phi = +1, for
 * u in [first, first + count). */
nrcps_status nrcps_draw_z2_bits(nrcps_context *ctx, int kind, long seed, uint64_t first,
                                uint64_t count, uint32_t *dev_bits);

/* --------------------------------------------------------------- Fourier
 * Fourier::Forward/Backward (src/fourier/cuda/fourier.cu:43-79): in-place
 * unnormalised 3-D DFT of `batch` orbitals. */
nrcps_status nrcps_fft3d(nrcps_context *ctx, void *data, int batch, const int dims[3],
                         nrcps_precision prec, int sign);

/* ------------------------------------------------------------ Hamiltonian
 * Kinetic::Evolve (src/hamiltonian/cuda/hamiltonian_evolve.cu:95-104):
 * psi /= xi on `batch` orbitals; xi is a device array of V doubles. */
nrcps_status nrcps_kinetic_evolve(nrcps_context *ctx, void *psi, int batch, long vol,
                                  const double *dev_xi, nrcps_precision prec);
/* Potential::Evolve (hamiltonian_evolve.cu:73-92): FFT, psi *= v(x), IFFT. */
nrcps_status nrcps_potential_evolve(nrcps_context *ctx, void *psi, int batch, const int dims[3],
                                    const double *dev_pot, nrcps_precision prec);
/* Interaction::Initialize (src/hamiltonian/cuda/hamiltonian_initialize.cu:17-35):
 * fld = (1 + IFFT_fwd[c(p) * FFT_bwd[phi]]) / V, all FP64 device arrays. */
nrcps_status nrcps_interaction_initialize(nrcps_context *ctx, const double *dev_lat,
                                          const double *dev_itab, const int dims[3],
                                          double *dev_fld);
/* Interaction::Evolve (hamiltonian_evolve.cu:42-69): FFT, psi *= fld, IFFT. */
nrcps_status nrcps_interaction_evolve(nrcps_context *ctx, void *psi, int batch, const int dims[3],
                                      const double *dev_fld, nrcps_precision prec);

/* Fused Propagator::Run (src/alg/propagator.C:35-45) over the ordering
 * [K, (V), I, (V), K] for `nconf` independent configurations of `batch`
 * orbitals each (psi[conf][orb][V]).  One pass: psi <- k .* B[w .* F[k .* psi]]
 * with k = 1/xi (dev_kin, V doubles), w(x) = P(x) * fld_conf(x), where
 * P (dev_pos, V doubles, may be NULL) folds the potential steps and the
 * position-space factor fld_conf is chosen by field_mode (k = bit0 +
 * conf*conf_stride + site):
 *   0: complex FP64 fld (Interaction::Initialize output), element k of dev_field;
 *   1: Z2 bits: fld = (1 + a*phi)/V with phi = +1 when bit k of dev_field is set;
 *   2: interleaved complex FP64 phi (Lattice::Get layout), fld = (1 + a*phi)/V;
 *   3: one real FP32 weight per site, element k of dev_field (float), the
 *      whole factor (a and P unused: dev_pos must be NULL); for a real
 *      field made once per run, as nrcps_batch does for FP32 orbitals.
 * Mathematically identical to the reference's sequence (F*B = V). */
typedef struct {
  int field_mode;
  const void *dev_field;
  uint64_t bit0;        /* element (mode 0/2/3) or bit (mode 1) offset of configuration 0 */
  uint64_t conf_stride; /* elements (mode 0/2/3) or bits (mode 1) between configurations */
  double a;
  const double *dev_pos; /* may be NULL */
  /* may be NULL; else a device array of nconf offsets that replaces
   * conf * conf_stride (configurations whose fields are not evenly spaced,
   * as in a batch of jobs of different sizes): k = bit0 + conf_base[conf] + site */
  const uint64_t *dev_conf_base;
} nrcps_position_factor;
nrcps_status nrcps_propagate(nrcps_context *ctx, void *psi, int batch, int nconf, const int dims[3],
                             const double *dev_kin, const nrcps_position_factor *w,
                             nrcps_precision prec);

/* --------------------------------------------------------- measurement */
/* SlaterDet fill (src/slater_det/slater_det.C:33-37) via OneBody::Project
 * (src/one_body/noarch/one_body_project.C:14-27) and Cuda::InnerProduct
 * (src/utils/cuda/cuda_utils.cu:88-127): S[c][s][t] = sum_p conj(src_s(p))
 * psi_{c,t}(p), for nconf configurations; src (ns x V, FP64 complex) shared,
 * psi (nconf x nt x V, precision prec), S FP64 complex, row-major per conf. */
nrcps_status nrcps_overlap(nrcps_context *ctx, const double *dev_src, int ns, const void *dev_psi,
                           int nt, int nconf, long vol, nrcps_precision prec, double *dev_S);
/* Plane-wave sources (OneBody::Set(n1,n2,n3), src/one_body/one_body.C:215-228):
 * S[c][s][t] = psi_{c,t}(p_s), an exact gather; dev_index = ns lattice indices
 * (an index outside [0, vol) gives zeros). */
nrcps_status nrcps_overlap_planewave(nrcps_context *ctx, const int *dev_index, int ns,
                                     const void *dev_psi, int nt, int nconf, long vol,
                                     nrcps_precision prec, double *dev_S);
/* TwoBody::Run (src/two_body/noarch/two_body_run.C:16-43): phi[c][s][t] =
 * sum_i w_i psi1_{c,s}(i) psi2_{c,t}(opp(i)), no conjugation.  A site whose
 * opp(i) lies outside [0, vol) contributes nothing (the reference's tables
 * have none). */
nrcps_status nrcps_pair_matrix(nrcps_context *ctx, const void *dev_psi1, const void *dev_psi2, int n,
                               int nconf, long vol, const double *dev_w, const int *dev_opposite,
                               nrcps_precision prec, double *dev_phi);
/* GeneralizedTwoBody::Run(prop1, prop2, R) (src/two_body/noarch/two_body_run.C:45-75),
 * the Oh-projected pair contraction, for every orbital pair of nconf
 * configurations: phi[c][s][t] = sum_l sum_i wl[l][i] psi1_{c,s}(shift[l][i])
 * psi2_{c,t}(opposite(i)), l < nterms (the subshell vectors of OhGroup);
 * the caller folds wl[l][i] = OhGroup::GetWeight(R, l) * half_site_wavefunc[l][i]
 * and passes shift_indices (nterms x V) as GeneralizedTwoBody builds them
 * (src/two_body/two_body.C:226-284). */
nrcps_status nrcps_shifted_pair_matrix(nrcps_context *ctx, const void *dev_psi1, const void *dev_psi2, int n,
                                       int nconf, long vol, int nterms, const int *dev_shift, const double *dev_wl,
                                       const int *dev_opposite, nrcps_precision prec, double *dev_phi);
/* Cuda::InnerProduct (src/utils/cuda/cuda_utils.cu:88-127) as the
 * reference's GPU build calls it: kets and bras are device arrays of nf
 * device pointers to V complex FP64 vectors; dev_mat[t + nf*s] =
 * <kets[s] | bras[t]> (nf*nf complex FP64, device). */
nrcps_status nrcps_inner_product_ptrs(nrcps_context *ctx, const double *const *dev_kets,
                                      const double *const *dev_bras, int nf, long vol,
                                      double *dev_mat);
/* TwoBody::Run(Float**, Float**, complex<Float>*, int)
 * (src/two_body/cuda/two_body_run.cu:41-83) with the same pointer arrays:
 * dev_phi[t + nf*s] = sum_i w_i props1[s](i) props2[t](opposite(i)).  Every
 * element is computed (the reference's batched kernel drops rows and
 * columns when nf is not a multiple of 3, two_body_run.cu:56). */
nrcps_status nrcps_pair_matrix_ptrs(nrcps_context *ctx, const double *const *dev_props1,
                                    const double *const *dev_props2, int nf, long vol,
                                    const double *dev_w, const int *dev_opposite, double *dev_phi);
/* SlaterDet::Run / SlaterDet2::Run (src/slater_det/slater_det.C:59-115,
 * slater_det2.C:78-148) with ludcmp (src/utils/ludcmp.C:9-65) in FP64 for
 * every leading minor n = 1..N of nconf matrices S (N x N complex):
 *   mode 0: out[c][n-1] = det S_n (N values per matrix);
 *   mode 1: out[c][2(n-1)] = det with column n-1 from dev_psi1 (struck
 *           column), out[c][2(n-1)+1] = det S_n (2N values per matrix).
 * log_det != 0 returns log det instead (DET_TYPE_LOG). */
nrcps_status nrcps_slater_dets(nrcps_context *ctx, const double *dev_S, const double *dev_psi1,
                               int N, int nconf, int mode, int log_det, double *dev_out);
/* nrcps_slater_dets without any device allocation (no counterpart in the
 * reference).  For callers that cannot let a library allocate device memory
 * -- a host whose caching pool already owns the device memory, or code
 * measuring between kernels already queued, where an allocation could stall
 * the device.  N <= 64 runs the warp-per-minor kernel, which needs no memory
 * beyond the inputs and outputs.  For N > 64 the working memory comes from
 * one fixed 16 MiB array in the library, which every GPU that loads the
 * library keeps until exit; batches needing more (nconf * nmeas * (2N^2 + N)
 * doubles) are rejected with NRCPS_ERR_INVALID_ARGUMENT.  The first N > 64
 * call on a device looks up the array's address; make it before any stream
 * capture.  Calls that may run concurrently on the GPU share the array and
 * race: serialise them.  nconf = 0 is a no-op (null buffers allowed). */
nrcps_status nrcps_slater_dets_noalloc(nrcps_context *ctx, const double *dev_S, const double *dev_psi1,
                                       int N, int nconf, int mode, int log_det, double *dev_out);

/* ------------------------------------------------------------ ensemble
 * The production loop (production/slater_det/main.C:185-220, mode 0;
 * production/slater_det2_trapped/main-no_cum.C:185-210, mode 1) for many
 * independent configurations at once, the time loop captured in a CUDA
 * graph.  Tables are host arrays (see the table builders above). */
typedef struct {
  int dims[3];
  int T;
  int n_orb;             /* N: orbitals = sources */
  int n_conf;            /* configurations in one run() */
  int rng_kind;
  long seed;             /* already including 491*rank */
  int field_kind;
  int mode;              /* 0 slater (N minors), 1 slater2 (2N) */
  int precision;         /* nrcps_precision of the orbital propagation */
  int plane_wave;        /* 1: sources are plane waves given by index */
  int use_potential;
  int qr_period;         /* k > 0: CholeskyQR of every configuration's orbitals after each
                            k-th step; the measured determinants are rescaled to those of
                            the unstabilised orbitals (mode 0: det S_n by prod_{i<n} R_ii;
                            mode 1: the pair-matrix minors by prod_{i<n} R_ii^2, the
                            replaced-column minors by prod_{i<n} R_ii prod_{i<n-1} R_ii);
                            0: never (the reference's unstabilised propagation) */
  double a;              /* (1 + a*phi) coupling when the interaction is local */
  int local_interaction; /* 1: c(p) constant, use a; 0: full Interaction::Initialize */
} nrcps_job;

typedef struct nrcps_ensemble nrcps_ensemble;

/* kin_xi = xi table (V), itab = interaction c(p) table (V), pot = potential
 * table (V, or NULL), sources = n_orb x V complex (ignored when plane_wave),
 * pw_index = n_orb lattice indices (plane_wave only), w/opposite = pair tables
 * (mode 1 only). */
nrcps_status nrcps_ensemble_create(nrcps_context *ctx, const nrcps_job *job, const double *kin_xi,
                                   const double *itab, const double *pot, const double *sources,
                                   const int *pw_index, const double *w, const int *opposite,
                                   nrcps_ensemble **ens);
/* Runs configurations [first_conf, first_conf + n_conf) of the stream:
 * configuration c uses field slices c*T .. c*T+T-1 (slice 0 = the Lattice
 * constructor's draw).  dets: device array n_conf x T x nmeas complex
 * doubles, nmeas = N (mode 0) or 2N (mode 1), raw determinants before any
 * accumulation. */
nrcps_status nrcps_ensemble_run(nrcps_ensemble *ens, uint64_t first_conf, double *dev_dets);
/* Replaces the sources of later runs from host memory, the kind given at
 * creation: sources (N x V complex doubles) for dense sources, pw_index (N
 * site indices) for plane waves; the other pointer may be NULL.  The copy is
 * queued on the context's stream ahead of later runs (pinned host memory
 * keeps it asynchronous).  Every run starts from the current sources, as
 * the reference's drivers call Propagator::Set(OneBody::Get(), n) for every
 * configuration (src/alg/propagator.C:47-63, production/slater_det/main.C:196-199). */
nrcps_status nrcps_ensemble_set_sources(nrcps_ensemble *ens, const double *sources, const int *pw_index);
nrcps_status nrcps_ensemble_destroy(nrcps_ensemble *ens);
/* Kernel launches issued by the last run (for launch accounting). */
nrcps_status nrcps_ensemble_launches(const nrcps_ensemble *ens, long *launches);
/* Z2 fields: *dev_bits receives the device array of the last run's field
 * bits (slice t of configuration c at bit (c T + t) V), valid until the
 * next run or destroy; NULL for other fields.  No counterpart in the
 * reference (its Lattice keeps one slice); lets a caller reuse the run's
 * fields (the control variate's features) instead of drawing them again. */
nrcps_status nrcps_ensemble_field_bits(const nrcps_ensemble *ens, const uint32_t **dev_bits);

/* --------------------------------------------------------------- batch
 * Jobs of different lattice size, particle number and time extent advanced
 * together, the time loops of all jobs in one CUDA graph launch (no
 * counterpart in the reference, whose drivers run one system per process:
 * production/slater_det/main.C:185-220).  Every job: plane-wave sources
 * (pw_index, n_orb lattice indices), the local interaction (1 + a phi)/V,
 * Kinetic with the given xi table (L^3 entries), measurement mode 0.  Jobs
 * with equal (L, n_orb) share launches; fields come from one generator
 * stream in job order (job j, configuration k, slice t reads sites
 * base_j + (k T_j + t) L_j^3 ...), and every run continues the stream. */
typedef struct {
  int L;
  int n_orb;
  int T;
  int n_conf;
  const int *pw_index; /* host */
  const double *kin_xi; /* host */
} nrcps_batch_job;
typedef struct {
  int rng_kind;
  long seed;
  int field_kind;
  int precision; /* nrcps_precision of the orbitals */
  double a;
  int qr_period; /* 0: none */
} nrcps_batch_params;
typedef struct nrcps_batch nrcps_batch;
nrcps_status nrcps_batch_create(nrcps_context *ctx, const nrcps_batch_params *params, const nrcps_batch_job *jobs,
                                int njobs, nrcps_batch **batch);
/* Output of a run: one device buffer of *doubles doubles; job j's
 * determinants are [n_conf][T][n_orb] complex at *offset (nrcps_batch_layout).
 * *launches = kernel launches inside the graph of one run. */
nrcps_status nrcps_batch_output_size(const nrcps_batch *batch, long *doubles, long *launches);
nrcps_status nrcps_batch_layout(const nrcps_batch *batch, int job, long *offset, long *doubles);
nrcps_status nrcps_batch_run(nrcps_batch *batch, double *dev_out);
nrcps_status nrcps_batch_destroy(nrcps_batch *batch);

/* ----------------------------------------------------------- branching
 * The multilevel branching driver (production/two_body-branched/main.C:23-80,
 * MultiLevel): trees of `levels` levels, `branches` children per node and
 * `steps` slices per level (T = levels * steps); prop1 / prop2 start from
 * sources2 (2 x V complex, host), every node restarts its children from its
 * end state, and corr[t] accumulates TwoBody::Run(prop1, prop2) /
 * branches^(d+1) over the nodes of depth d = t / steps.  Hamiltonians
 * [K, (V), I, (V), K] with the local interaction (1 + a phi)/V (the driver's
 * Interaction3 is not in the reference's headers); fields are the slices the
 * reference's depth-first walk draws from one stream. */
typedef struct {
  int dims[3];
  int levels;
  int branches;
  int steps;
  int rng_kind;
  long seed;
  int field_kind;
  int precision;
  double a;
} nrcps_branch_params;
typedef struct nrcps_branch nrcps_branch;
/* kin_xi: V xi values; pot: V potential values or NULL; w / opposite: the
 * TwoBody tables (nrcps_two_body_tables). */
nrcps_status nrcps_branch_create(nrcps_context *ctx, const nrcps_branch_params *params, const double *kin_xi,
                                 const double *pot, const double *sources2, const double *w, const int *opposite,
                                 nrcps_branch **branch);
/* The next tree; dev_corr (T complex doubles, device) accumulates its sums. */
nrcps_status nrcps_branch_run(nrcps_branch *branch, double *dev_corr);
nrcps_status nrcps_branch_destroy(nrcps_branch *branch);

/* CholeskyQR of every configuration's orbital block, in place:
 * Psi = Q R (G = Psi^H Psi accumulated in FP64, Cholesky and R^-1 in FP64,
 * Psi <- Psi R^-1), dev_logR[c][i] += log R_ii (FP32 orbitals: -log of the
 * FP32-rounded (R^-1)_ii that was applied).  The reference's only
 * stabilisation is a norm rescale (Propagator::Normalize,
 * src/alg/propagator.C:78-135); the ensemble runners call this every
 * qr_period slices.  dev_psi [nconf][N][vol]; dev_work: 2 nconf N^2 doubles
 * of scratch; N <= 64. */
nrcps_status nrcps_reorthonormalise(nrcps_context *ctx, void *dev_psi, int N, long vol, int nconf,
                                    nrcps_precision prec, double *dev_work, double *dev_logR);

/* ------------------------------------------- learned control variate
 * Kernels of the control-variate network (no counterpart in the reference;
 * nrcps_b200/cv.py drives them): a 3-layer 3x3x3 periodic convolution net
 * over block means of the field slices, BF16 conv weights and activations,
 * FP32 accumulation, an MLP head predicting log C(tau).  Tensors are per
 * sample contiguous (act[b][c][s], s = z + G (y + G x)). */
/* x[b][t][q] = mean of phi = +-1 over the (L/G)^3 sites of cell q of slice t
 * of configuration b (BF16); bit bit0 + (b T + t) L^3 + site of dev_bits is
 * phi = +1. */
nrcps_status nrcps_cv_coarse_z2(nrcps_context *ctx, const uint32_t *dev_bits, uint64_t bit0, int L, int T, int G,
                                int B, void *dev_x);
/* The same features for B fresh uniform Z2 fields (numbers first ..
 * first + B - 1 of the stream `seed`), drawn directly: the block mean of
 * n = (L/G)^3 independent +-1 sites is (2 c - n)/n with c the set bits of n
 * Philox4x32-10 bits (counter (cell lo, cell hi, word / 4, 0x5A32), key
 * seed).  For the control variate's mean <g> over the field distribution. */
nrcps_status nrcps_cv_sample_z2_features(nrcps_context *ctx, uint64_t seed, uint64_t first, int L, int T, int G,
                                         int B, void *dev_x);
/* Inference of the whole network on the tcgen05 tensor cores, one kernel:
 * three conv layers (BF16 MMAs, FP32 accumulation in TMEM, BF16
 * activations), mean pool and head; y[b][t] = standardised prediction.
 * G = 8; Cin a multiple of 16 up to 64; H <= 64; T <= 256.  dev_W[l] BF16
 * [16][cin][27], dev_bias[l] FP32 [16] for l = 0..2 (device pointers held in
 * host arrays). */
nrcps_status nrcps_cv_forward_tc(nrcps_context *ctx, const void *dev_x, int Cin, int G, int B,
                                 const void *const *dev_W, const float *const *dev_bias, const float *dev_hw,
                                 const float *dev_hb, int H, const float *dev_ow, const float *dev_ob, int T,
                                 float *dev_y);
/* Z = conv(in) + bias (FP32), A = tanh(Z) (BF16); Cout = 16; W BF16 [Cout][Cin][27]. */
nrcps_status nrcps_cv_conv_forward(nrcps_context *ctx, const void *dev_in, int Cin, int Cout, int G, int B,
                                   const void *dev_W, const float *dev_bias, float *dev_Z, void *dev_A);
/* dW, db from dZ and the layer input; with dev_dZin (Cin = 16) also the data
 * gradient times tanh' of the input activations dev_Ain. */
nrcps_status nrcps_cv_conv_backward(nrcps_context *ctx, const float *dev_dZ, const void *dev_in, const void *dev_Ain,
                                    int Cin, int Cout, int G, int B, const void *dev_W, float *dev_dW, float *dev_db,
                                    float *dev_dZin);
/* pool (mean over sites) + tanh hidden layer (H) + linear output (T). */
nrcps_status nrcps_cv_head_forward(nrcps_context *ctx, const void *dev_A3, int C, int G, int B, const float *W1,
                                   const float *b1, int H, const float *W2, const float *b2, int T, float *P,
                                   float *Hact, float *Y);
/* loss 0.5 mean (Y - target)^2 (per-sample sums in loss_parts), head weight
 * gradients and dZ3 of the last conv layer. */
nrcps_status nrcps_cv_head_backward(nrcps_context *ctx, const float *Y, const float *target, int T, int B,
                                    const float *Hact, int H, const float *W2, const float *W1, int C,
                                    const void *dev_A3, int G, const float *P, float *dY, float *dZh, float *dZ3,
                                    float *loss_parts, float *dW2, float *db2, float *dW1, float *db1);
/* Adam on FP32 master weights (bias-corrected, step >= 1); bf16_copy (may be
 * NULL) receives the updated weights in BF16. */
nrcps_status nrcps_cv_adam(nrcps_context *ctx, float *w, const float *g, float *m, float *v, long n, float lr,
                           float beta1, float beta2, float eps, int step, void *bf16_copy);

/* ---------------------------------------------------------- estimators
 * Block accumulators of the production drivers in FP64, configurations added
 * in index order: dev_dets = n_conf x T x nmeas complex (nrcps_ensemble_run
 * layout); dev_corr = nmeas x T complex,
 *   mode 0: corr[m][t] = sum_c |det|^2      (production/slater_det/main.C:208-211),
 *   mode 1: corr[m][t] = sum_c det          (production/slater_det2_trapped/main-no_cum.C:205-207);
 * n_cumulants = Nc in 0..8: dev_z = Nc x nmeas x T doubles,
 *   z[k][m][t] = sum_c (log|det|)^(k+1)     (production/slater_det2_trapped/main-cum.C:219-233). */
nrcps_status nrcps_accumulate(nrcps_context *ctx, const double *dev_dets, int n_conf, int T, int nmeas,
                              int mode, int n_cumulants, double *dev_corr, double *dev_z);
/* Binned jackknife (no counterpart in the reference, whose drivers write
 * block averages for offline analysis): dev_x = n_samples x n_obs doubles;
 * mean / err of every observable over n_bins bins of consecutive samples
 * (remainder dropped).  With dev_eff_mean / dev_eff_err (n_obs - 1 each, or
 * both NULL) the observables are read as C(t) of consecutive slices and the
 * effective energies log(C(t) / C(t+1)) are estimated with jackknife errors. */
nrcps_status nrcps_jackknife(nrcps_context *ctx, const double *dev_x, long n_samples, int n_obs, int n_bins,
                             double *dev_mean, double *dev_err, double *dev_eff_mean, double *dev_eff_err);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif

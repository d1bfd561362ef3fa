// ensemble.cu -- the production driver loop for many configurations at once.
//
// Reference loop (production/slater_det/main.C:185-220): per configuration,
// sources are copied into the propagator; then for every time slice the
// Slater matrix of the current orbitals is measured (all leading-minor
// determinants), the Hamiltonians are initialised on the current field and
// applied, and the lattice draws the next field.  Here all configurations of
// a run advance together: one fused propagator step, one measurement and one
// LU launch per slice cover every configuration, and the whole time loop is
// captured once in a CUDA graph and replayed for every run.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace nrcps {
nrcps_status ranlux_generate(nrcps_context* ctx, int kind, long seed, uint64_t u_lo, uint64_t u_hi, int out_kind,
                             double* d, uint32_t* bits);
nrcps_status slater_dets_dispatch(nrcps_context* ctx, const double* S, const double* psi1, int N, int nconf, int mode,
                              int log_det, double* out, long out_conf_stride, long out_offset, double* scr);
size_t slater_dets_scratch_bytes(int N, int nconf, int mode);
nrcps_status overlap_impl(nrcps_context* ctx, const double* src, int ns, const void* psi, int nt, int nconf,
                          long vol, nrcps_precision prec, double* S);
nrcps_status gather_impl(nrcps_context* ctx, const int* index, int ns, const void* psi, int nt, int nconf, long vol,
                         nrcps_precision prec, double* S);
nrcps_status pair_impl(nrcps_context* ctx, const void* psi1, const void* psi2, int n, int nconf, long vol,
                       const double* w, const int* opp, nrcps_precision prec, double* phi, int props);
nrcps_status propagate_impl(nrcps_context* ctx, void* psi, int batch, int nconf, const int d[3], const double* kin,
                            const float2* kin_f32, const nrcps_position_factor* w, nrcps_precision prec,
                            const void* zpos);
nrcps_status fused_autotune(nrcps_context* ctx, nrcps_precision prec, int L, int* chosen_cluster);
nrcps_status qr_reorthonormalise(nrcps_context* ctx, void* psi, int N, long vol, int nconf, nrcps_precision prec,
                                 double* G, double* logR);
nrcps_status rescale_dets(nrcps_context* ctx, double* dets, const double* logR, int N, int nconf, long conf_stride,
                          long offset, int mode);
}  // namespace nrcps

struct nrcps_ensemble {
  nrcps_context* ctx = nullptr;
  nrcps_job job{};
  long vol = 0;
  int N = 0, nmeas = 0;
  size_t esize = 0;  // bytes per complex orbital entry
  void* psi = nullptr;
  double* src = nullptr;
  float* src_split = nullptr;  // TF32 hi/lo sources of the tensor-core overlap (FP32 orbitals)
  int* pw_index = nullptr;
  double* kinv = nullptr;
  float2* kinv_f = nullptr;  // (hi, lo) split of kinv
  double* pos = nullptr;
  void* zpos = nullptr;        // Z2 fields with the potential: per-site weights (zpos_table_kernel's layout)
  double* itab = nullptr;
  double* w = nullptr;
  int* opp = nullptr;
  int pair_props = 3;  // the pair table's properties, checked on the host (pair_table_props)
  uint32_t* bits = nullptr;   // Z2 fields of a run
  double* phi = nullptr;      // other fields of a run (interleaved complex)
  double* fld = nullptr;      // non-local interaction factor of one slice
  double* S = nullptr;
  double* P1 = nullptr;
  double* lu_scr = nullptr;
  double* qr_G = nullptr;     // Gram matrices / R^-1 of a re-orthonormalisation
  double* qr_logR = nullptr;  // running sum of log R_ii per configuration and orbital
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t gauss_offset = 0;    // stream position of the next configuration (Gaussian fields)
  uint64_t gauss_next_conf = 0;
  long launches_per_run = 0;
  double* dets_captured = nullptr;  // output buffer baked into the graph
};

namespace nrcps {

__global__ void scatter_sources_kernel(void* psi, int esize_is_f64, int N, int nconf, long vol, const int* pw_index,
                                       const double* src) {
  long total = (long)nconf * N * vol;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long i = e % vol;
    int n = (int)((e / vol) % N);
    double re, im;
    if (pw_index) {
      re = (i == pw_index[n]) ? 1.0 : 0.0;
      im = 0.0;
    } else {
      re = src[2 * ((long)n * vol + i)];
      im = src[2 * ((long)n * vol + i) + 1];
    }
    if (esize_is_f64) reinterpret_cast<double2*>(psi)[e] = make_double2(re, im);
    else reinterpret_cast<float2*>(psi)[e] = make_float2((float)re, (float)im);
  }
}

// phi (bits or interleaved complex) of slice t for every configuration -> fld buffer.
__global__ void expand_field_kernel(const uint32_t* bits, const double* phi, int T, int t, long vol, int nconf,
                                    double* fld) {
  long total = (long)nconf * vol;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long c = e / vol, i = e % vol;
    uint64_t k = ((uint64_t)c * T + t) * vol + i;
    if (bits) {
      fld[2 * e] = ((bits[k >> 5] >> (k & 31)) & 1u) ? 1.0 : -1.0;
      fld[2 * e + 1] = 0.0;
    } else {
      fld[2 * e] = phi[2 * k];
      fld[2 * e + 1] = phi[2 * k + 1];
    }
  }
}

__global__ void mul_itab_kernel(double* fld, long vol, long total, const double* itab) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    double k = itab[e % vol];
    fld[2 * e] *= k;
    fld[2 * e + 1] *= k;
  }
}

__global__ void plus_one_div_kernel(double* fld, long vol, long total) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    double re = fld[2 * e] + 1.0;
    fld[2 * e] = re / vol;
    fld[2 * e + 1] = fld[2 * e + 1] / vol;
  }
}

template <typename T>
static nrcps_status dalloc(nrcps_context* ctx, T** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return NRCPS_OK;
  return check_cuda(ctx, cudaMalloc((void**)p, bytes), "cudaMalloc(ensemble)");
}

static nrcps_status upload(nrcps_context* ctx, void* dst, const void* src, size_t bytes) {
  return check_cuda(ctx, cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(ensemble)");
}

// The time loop of one run (captured into a graph).
static nrcps_status record_time_loop(nrcps_ensemble* e, double* dets) {
  nrcps_context* ctx = e->ctx;
  const nrcps_job& j = e->job;
  const int N = e->N, nc = j.n_conf, T = j.T;
  const long vol = e->vol;
  const nrcps_precision prec = (nrcps_precision)j.precision;
  const int d3[3] = {j.dims[0], j.dims[1], j.dims[2]};
  long n0 = ctx->launches;
  scatter_sources_kernel<<<grid_for((long)nc * N * vol, 256, (long)ctx->sm_count * 16), 256, 0, ctx->stream>>>(
      e->psi, prec == NRCPS_F64, N, nc, vol, e->pw_index, e->src);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "scatter_sources_kernel"));
  if (e->qr_logR)
    NRCPS_TRY(check_cuda(ctx, cudaMemsetAsync(e->qr_logR, 0, sizeof(double) * nc * N, ctx->stream), "memset logR"));
  for (int t = 0; t < T; ++t) {
    // -------- measurement at slice t (before the step, main.C:204-211)
    if (j.mode == 0) {
      if (e->pw_index) NRCPS_TRY(gather_impl(ctx, e->pw_index, N, e->psi, N, nc, vol, prec, e->S));
      else if (e->src_split) NRCPS_TRY(overlap_tc(ctx, e->src_split, N, e->psi, N, nc, vol, e->S));
      else NRCPS_TRY(overlap_impl(ctx, e->src, N, e->psi, N, nc, vol, prec, e->S));
      NRCPS_TRY(slater_dets_dispatch(ctx, e->S, nullptr, N, nc, 0, 0, dets, 2L * T * e->nmeas, 2L * t * e->nmeas,
                                 e->lu_scr));
      if (e->qr_logR && t >= j.qr_period)
        NRCPS_TRY(rescale_dets(ctx, dets, e->qr_logR, N, nc, 2L * T * e->nmeas, 2L * t * e->nmeas, 0));
    } else {
      NRCPS_TRY(pair_impl(ctx, e->psi, e->psi, N, nc, vol, e->w, e->opp, prec, e->S, e->pair_props));
      if (e->pw_index) NRCPS_TRY(gather_impl(ctx, e->pw_index, N, e->psi, N, nc, vol, prec, e->P1));
      else if (e->src_split) NRCPS_TRY(overlap_tc(ctx, e->src_split, N, e->psi, N, nc, vol, e->P1));
      else NRCPS_TRY(overlap_impl(ctx, e->src, N, e->psi, N, nc, vol, prec, e->P1));
      NRCPS_TRY(slater_dets_dispatch(ctx, e->S, e->P1, N, nc, 1, 0, dets, 2L * T * e->nmeas, 2L * t * e->nmeas,
                                 e->lu_scr));
      if (e->qr_logR && t >= j.qr_period)
        NRCPS_TRY(rescale_dets(ctx, dets, e->qr_logR, N, nc, 2L * T * e->nmeas, 2L * t * e->nmeas, 1));
    }
    // -------- Hamiltonians on the field of slice t, then the step
    nrcps_position_factor pf{};
    pf.dev_pos = e->pos;
    pf.a = j.a;
    if (!j.local_interaction) {
      long total = (long)nc * vol;
      unsigned g = grid_for(total, 256, (long)ctx->sm_count * 16);
      expand_field_kernel<<<g, 256, 0, ctx->stream>>>(e->bits, e->phi, T, t, vol, nc, e->fld);
      ctx->launches++;
      NRCPS_TRY(nrcps_fft3d(ctx, e->fld, nc, d3, NRCPS_F64, +1));
      mul_itab_kernel<<<g, 256, 0, ctx->stream>>>(e->fld, vol, total, e->itab);
      ctx->launches++;
      NRCPS_TRY(nrcps_fft3d(ctx, e->fld, nc, d3, NRCPS_F64, -1));
      plus_one_div_kernel<<<g, 256, 0, ctx->stream>>>(e->fld, vol, total);
      ctx->launches++;
      NRCPS_TRY(check_launch(ctx, "interaction initialise"));
      pf.field_mode = 0;
      pf.dev_field = e->fld;
      pf.bit0 = 0;
      pf.conf_stride = (uint64_t)vol;
    } else if (e->bits) {
      pf.field_mode = 1;
      pf.dev_field = e->bits;
      pf.bit0 = (uint64_t)t * vol;
      pf.conf_stride = (uint64_t)T * vol;
    } else {
      pf.field_mode = 2;
      pf.dev_field = e->phi;
      pf.bit0 = (uint64_t)t * vol;
      pf.conf_stride = (uint64_t)T * vol;
    }
    NRCPS_TRY(propagate_impl(ctx, e->psi, N, nc, d3, e->kinv, e->kinv_f, &pf, prec, e->zpos));
    if (e->qr_logR && (t + 1) % j.qr_period == 0 && t + 1 < T)
      NRCPS_TRY(qr_reorthonormalise(ctx, e->psi, N, vol, nc, prec, e->qr_G, e->qr_logR));
  }
  e->launches_per_run = ctx->launches - n0;
  return NRCPS_OK;
}

}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_ensemble_create(nrcps_context* ctx, const nrcps_job* job, const double* kin_xi,
                                              const double* itab, const double* pot, const double* sources,
                                              const int* pw_index, const double* w, const int* opposite,
                                              nrcps_ensemble** out) {
  if (!ctx || !out) return NRCPS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  NRCPS_REQUIRE(ctx, job && kin_xi && job->T > 0 && job->n_orb > 0 && job->n_conf > 0,
                "nrcps_ensemble_create: bad job");
  NRCPS_REQUIRE(ctx, job->plane_wave ? pw_index != nullptr : sources != nullptr,
                "nrcps_ensemble_create: sources missing");
  NRCPS_REQUIRE(ctx, job->mode == 0 || (job->mode == 1 && w && opposite), "nrcps_ensemble_create: pair tables missing");
  NRCPS_REQUIRE(ctx, job->local_interaction || itab, "nrcps_ensemble_create: interaction table missing");
  NRCPS_REQUIRE(ctx, !job->use_potential || pot, "nrcps_ensemble_create: potential table missing");
  NRCPS_REQUIRE(ctx, job->qr_period >= 0, "nrcps_ensemble_create: qr_period < 0");
  if (job->qr_period > 0 && job->n_orb > 64)
    return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "nrcps_ensemble_create: re-orthonormalisation needs N <= 64");
  const int fk = job->field_kind;
  NRCPS_REQUIRE(ctx, fk >= 0 && fk <= 3, "nrcps_ensemble_create: bad field kind");
  nrcps_ensemble* e = new nrcps_ensemble();
  e->ctx = ctx;
  e->job = *job;
  e->vol = (long)job->dims[0] * job->dims[1] * job->dims[2];
  e->N = job->n_orb;
  e->nmeas = job->mode ? 2 * e->N : e->N;
  e->esize = job->precision == NRCPS_F64 ? 16 : 8;
  const long V = e->vol;
  const int N = e->N, nc = job->n_conf;
  nrcps_status st = NRCPS_OK;
  auto fail = [&](nrcps_status s) {
    nrcps_ensemble_destroy(e);
    return s;
  };
  if ((st = dalloc(ctx, (char**)&e->psi, e->esize * (size_t)nc * N * V))) return fail(st);
  if ((st = dalloc(ctx, &e->kinv, 8 * V))) return fail(st);
  std::vector<double> h(V);
  for (long i = 0; i < V; ++i) h[i] = 1.0 / kin_xi[i];
  if ((st = upload(ctx, e->kinv, h.data(), 8 * V))) return fail(st);
  {
    std::vector<float2> hf(V);
    for (long i = 0; i < V; ++i) {
      float hi = (float)h[i];
      hf[i] = make_float2(hi, (float)(h[i] - (double)hi));
    }
    if ((st = dalloc(ctx, &e->kinv_f, 8 * V)) || (st = upload(ctx, e->kinv_f, hf.data(), 8 * V))) return fail(st);
  }
  if (job->dims[0] == job->dims[1] && job->dims[1] == job->dims[2] && job->dims[0] < 64)
    fused_autotune(ctx, (nrcps_precision)job->precision, job->dims[0], nullptr);
  if (job->use_potential) {
    // [K,V,I,V,K] = K B diag(V^2 v^2 fld) F K since F B = V (unnormalised transforms)
    for (long i = 0; i < V; ++i) h[i] = ((double)V * pot[i]) * ((double)V * pot[i]);
    if ((st = dalloc(ctx, &e->pos, 8 * V)) || (st = upload(ctx, e->pos, h.data(), 8 * V))) return fail(st);
  }
  if (!job->local_interaction) {
    if ((st = dalloc(ctx, &e->itab, 8 * V)) || (st = upload(ctx, e->itab, itab, 8 * V))) return fail(st);
    if ((st = dalloc(ctx, &e->fld, 16 * (size_t)nc * V))) return fail(st);
  }
  if (job->plane_wave) {
    if ((st = dalloc(ctx, &e->pw_index, 4 * N)) || (st = upload(ctx, e->pw_index, pw_index, 4 * N))) return fail(st);
  } else {
    if ((st = dalloc(ctx, &e->src, 16 * (size_t)N * V)) || (st = upload(ctx, e->src, sources, 16 * (size_t)N * V)))
      return fail(st);
    if (job->precision == NRCPS_F32 && ctx->overlap_tc && overlap_tc_supported(V, N, N, nc)) {
      if ((st = dalloc(ctx, (char**)&e->src_split, overlap_tc_split_bytes(N, V))) ||
          (st = overlap_tc_prepare(ctx, e->src, N, V, e->src_split)))
        return fail(st);
    }
  }
  if (job->mode == 1) {
    if ((st = dalloc(ctx, &e->w, 8 * V)) || (st = upload(ctx, e->w, w, 8 * V))) return fail(st);
    if ((st = dalloc(ctx, &e->opp, 4 * V)) || (st = upload(ctx, e->opp, opposite, 4 * V))) return fail(st);
    e->pair_props = pair_table_props(opposite, w, V);
    if ((st = dalloc(ctx, &e->P1, 16 * (size_t)nc * N * N))) return fail(st);
  }
  const uint64_t sites = (uint64_t)nc * job->T * V;
  if (fk == NRCPS_FIELD_ZTWO) {
    if ((st = dalloc(ctx, &e->bits, 4 * ((sites + 31) / 32 + 1)))) return fail(st);
    if (job->use_potential && job->local_interaction) {
      // the fused step's per-site weights (1 +- a) P/V, P = h (the squared,
      // scaled potential above): the products the general path forms per site
      const double wp = (1.0 + job->a) / (double)V, wm = (1.0 - job->a) / (double)V;
      if (job->precision == NRCPS_F32) {
        std::vector<float4> t(V);
        for (long i = 0; i < V; ++i) {
          const double p = wp * h[i], m = wm * h[i];
          const float hp = (float)p, hm = (float)m;
          t[i] = make_float4(hp, (float)(p - (double)hp), hm, (float)(m - (double)hm));
        }
        if ((st = dalloc(ctx, (char**)&e->zpos, 16 * V)) || (st = upload(ctx, e->zpos, t.data(), 16 * V)))
          return fail(st);
      } else {
        std::vector<double2> t(V);
        for (long i = 0; i < V; ++i) t[i] = make_double2(wp * h[i], wm * h[i]);
        if ((st = dalloc(ctx, (char**)&e->zpos, 16 * V)) || (st = upload(ctx, e->zpos, t.data(), 16 * V)))
          return fail(st);
      }
    }
  } else {
    if ((st = dalloc(ctx, &e->phi, 16 * sites))) return fail(st);
  }
  if ((st = dalloc(ctx, &e->S, 16 * (size_t)nc * N * N))) return fail(st);
  if ((st = dalloc(ctx, &e->lu_scr, slater_dets_scratch_bytes(N, nc, job->mode)))) return fail(st);
  if (job->qr_period > 0) {
    if ((st = dalloc(ctx, &e->qr_G, 16 * (size_t)nc * N * N))) return fail(st);
    if ((st = dalloc(ctx, &e->qr_logR, 8 * (size_t)nc * N))) return fail(st);
  }
  *out = e;
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_ensemble_run(nrcps_ensemble* e, uint64_t first_conf, double* dev_dets) {
  if (!e) return NRCPS_ERR_INVALID_ARGUMENT;
  nrcps_context* ctx = e->ctx;
  NRCPS_REQUIRE(ctx, dev_dets, "nrcps_ensemble_run: null output");
  const nrcps_job& j = e->job;
  const uint64_t per_conf = (uint64_t)j.T * e->vol;
  const uint64_t sites = (uint64_t)j.n_conf * per_conf;
  long n0 = ctx->launches;
  // ---- fields of configurations [first_conf, first_conf + n_conf)
  if (j.field_kind == NRCPS_FIELD_ZTWO) {
    NRCPS_TRY(nrcps_draw_z2_bits(ctx, j.rng_kind, j.seed, first_conf * per_conf, sites, e->bits));
  } else if (j.field_kind == NRCPS_FIELD_ZTHREE) {
    uint64_t off = first_conf * per_conf;
    NRCPS_TRY(nrcps_draw_fields(ctx, j.rng_kind, j.seed, j.field_kind, e->vol, (long)j.n_conf * j.T, &off, e->phi));
  } else {
    // Gaussian fields consume a data-dependent number of uniforms: runs must
    // follow each other in stream order.
    if (first_conf != e->gauss_next_conf)
      return set_error(ctx, NRCPS_ERR_UNSUPPORTED,
                       "Gaussian fields: configurations must be run in order (next is %llu)",
                       (unsigned long long)e->gauss_next_conf);
    NRCPS_TRY(nrcps_draw_fields(ctx, j.rng_kind, j.seed, j.field_kind, e->vol, (long)j.n_conf * j.T,
                                &e->gauss_offset, e->phi));
    e->gauss_next_conf += j.n_conf;
  }
  long gen_launches = ctx->launches - n0;
  // ---- the time loop, captured once per output buffer and replayed
  if (e->exec && e->dets_captured != dev_dets) {
    cudaGraphExecDestroy(e->exec);
    cudaGraphDestroy(e->graph);
    e->exec = nullptr;
    e->graph = nullptr;
  }
  if (!e->exec) {
    e->dets_captured = dev_dets;
    NRCPS_TRY(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "sync before capture"));
    cudaStream_t cap = ctx->stream;
    bool own = false;
    if (cap == nullptr) {
      NRCPS_TRY(check_cuda(ctx, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "stream create"));
      own = true;
    }
    cudaStream_t saved = ctx->stream;
    ctx->stream = cap;
    NRCPS_TRY(check_cuda(ctx, cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture"));
    nrcps_status rs = record_time_loop(e, dev_dets);
    cudaError_t ce = cudaStreamEndCapture(cap, &e->graph);
    ctx->stream = saved;
    if (rs != NRCPS_OK) {
      if (own) cudaStreamDestroy(cap);
      return rs;
    }
    NRCPS_TRY(check_cuda(ctx, ce, "end capture"));
    NRCPS_TRY(check_cuda(ctx, cudaGraphInstantiate(&e->exec, e->graph, 0), "graph instantiate"));
    if (own) cudaStreamDestroy(cap);
  }
  NRCPS_TRY(check_cuda(ctx, cudaGraphLaunch(e->exec, ctx->stream), "graph launch"));
  ctx->launches = n0 + gen_launches + e->launches_per_run;
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_ensemble_set_sources(nrcps_ensemble* e, const double* sources, const int* pw_index) {
  if (!e) return NRCPS_ERR_INVALID_ARGUMENT;
  nrcps_context* ctx = e->ctx;
  if (e->pw_index) {
    NRCPS_REQUIRE(ctx, pw_index, "nrcps_ensemble_set_sources: plane-wave ensemble needs pw_index");
    for (int n = 0; n < e->N; ++n)
      NRCPS_REQUIRE(ctx, pw_index[n] >= 0 && pw_index[n] < e->vol, "nrcps_ensemble_set_sources: index out of range");
    return check_cuda(ctx, cudaMemcpyAsync(e->pw_index, pw_index, sizeof(int) * e->N, cudaMemcpyHostToDevice,
                                           ctx->stream), "set_sources: copy index");
  }
  NRCPS_REQUIRE(ctx, sources, "nrcps_ensemble_set_sources: dense-source ensemble needs sources");
  NRCPS_TRY(check_cuda(ctx, cudaMemcpyAsync(e->src, sources, 16 * (size_t)e->N * e->vol, cudaMemcpyHostToDevice,
                                            ctx->stream), "set_sources: copy sources"));
  if (e->src_split) NRCPS_TRY(overlap_tc_prepare(ctx, e->src, e->N, e->vol, e->src_split));
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_ensemble_launches(const nrcps_ensemble* e, long* launches) {
  if (!e || !launches) return NRCPS_ERR_INVALID_ARGUMENT;
  *launches = e->launches_per_run;
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_ensemble_field_bits(const nrcps_ensemble* e, const uint32_t** dev_bits) {
  if (!e || !dev_bits) return NRCPS_ERR_INVALID_ARGUMENT;
  *dev_bits = e->job.field_kind == NRCPS_FIELD_ZTWO ? e->bits : nullptr;
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_ensemble_destroy(nrcps_ensemble* e) {
  if (!e) return NRCPS_OK;
  if (e->ctx) cudaStreamSynchronize(e->ctx->stream);
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  void* bufs[] = {e->psi, e->src, e->src_split, e->pw_index, e->kinv, e->kinv_f, e->pos, e->zpos, e->itab, e->w, e->opp,
                  e->bits, e->phi, e->fld, e->S, e->P1, e->lu_scr, e->qr_G, e->qr_logR};
  for (void* b : bufs)
    if (b) cudaFree(b);
  delete e;
  return NRCPS_OK;
}

// batch.cu -- jobs of different lattice size L, particle number N and time
// extent T advanced together, the whole time loop of every job in ONE graph
// launch (no counterpart in the reference, whose drivers run one system per
// process: production/slater_det/main.C:185-220).
//
// Jobs of equal (L, N) form a group.  A group holds every configuration of
// its jobs, sorted by time extent (longest first), so the configurations
// still running at slice t are a prefix and each launch of slice t covers
// exactly those (the shorter jobs drop out as t grows).  Each group's time
// loop -- plane-wave measurement, leading-minor determinants, fused step,
// optional re-orthonormalisation -- is captured on its own stream, forked
// from and joined back to the context's stream, so the captured graph runs
// the groups as parallel branches; a last kernel scatters every
// configuration's determinants to its job's place in the output.
//
// Fields come from ONE generator stream in job order, as one process would
// draw them running the jobs one after another: job j, configuration k,
// slice t reads sites [base_j + (k T_j + t) V_j, ... + V_j) of the stream,
// base_j = sum_{i<j} n_conf_i T_i V_i.  Each run continues the stream.
// With FP32 orbitals a real Gaussian field reaches the fused step as one
// FP32 weight (1 + a phi)/V per site, made once per run; such a batch draws
// the next run's fields on a side stream while the current run's graph
// executes, into the second of two weight buffers (one captured graph per
// buffer), so the stream order and the results are those of drawing them
// at the start of each run.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace nrcps {
nrcps_status slater_dets_dispatch(nrcps_context* ctx, const double* S, const double* psi1, int N, int nconf, int mode,
                                  int log_det, double* out, long out_conf_stride, long out_offset, double* scr);
size_t slater_dets_scratch_bytes(int N, int nconf, int mode);
nrcps_status gather_impl(nrcps_context* ctx, const int* index, int ns, const void* psi, int nt, int nconf, long vol,
                         nrcps_precision prec, double* S);
nrcps_status propagate_impl(nrcps_context* ctx, void* psi, int batch, int nconf, const int d[3], const double* kin,
                            const float2* kin_f32, const nrcps_position_factor* w, nrcps_precision prec,
                            const void* zpos);
nrcps_status fused_autotune(nrcps_context* ctx, nrcps_precision prec, int L, int* chosen_cluster);
nrcps_status qr_reorthonormalise(nrcps_context* ctx, void* psi, int N, long vol, int nconf, nrcps_precision prec,
                                 double* G, double* logR);
nrcps_status rescale_dets(nrcps_context* ctx, double* dets, const double* logR, int N, int nconf, long conf_stride,
                          long offset, int mode);

struct Group {
  int L = 0, N = 0;
  long V = 0;
  int nconf = 0, Tmax = 0;
  std::vector<int> nact;     // per slice: configurations with T_c > t
  void* psi = nullptr;
  double* kinv = nullptr;
  float2* kinv_f = nullptr;
  int* pw_index = nullptr;
  uint64_t* conf_base = nullptr;  // device: field site offset of each configuration's slice 0
  long* out_off = nullptr;        // device: output offset (doubles) of each configuration
  int* conf_T = nullptr;          // device: T of each configuration
  double* S = nullptr;
  double* lu_scr = nullptr;
  double* dets = nullptr;         // nconf x Tmax x N complex
  double* qr_G = nullptr;
  double* qr_logR = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

namespace {

__global__ void batch_scatter_sources_kernel(void* psi, int is_f64, int N, int nconf, long vol, const int* pw_index) {
  const long total = (long)nconf * N * vol;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % vol;
    const int n = (int)((e / vol) % N);
    const float v = (i == pw_index[n]) ? 1.0f : 0.0f;
    if (is_f64) reinterpret_cast<double2*>(psi)[e] = make_double2((double)v, 0.0);
    else reinterpret_cast<float2*>(psi)[e] = make_float2(v, 0.0f);
  }
}

// dets of configuration c (slices < T_c) -> out + out_off[c], [T_c][N] complex
__global__ void batch_gather_dets_kernel(const double* __restrict__ dets, int N, int Tmax, int nconf,
                                         const int* __restrict__ conf_T, const long* __restrict__ out_off,
                                         double* __restrict__ out) {
  const long total = (long)nconf * Tmax * N;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long c = e / ((long)Tmax * N);
    const int r = (int)(e - c * Tmax * N);
    const int t = r / N;
    if (t >= conf_T[c]) continue;
    const double2 v = reinterpret_cast<const double2*>(dets)[e];
    reinterpret_cast<double2*>(out + out_off[c])[r] = v;
  }
}

// One FP32 weight per site of a real Gaussian field, (1 + a phi)/V with the
// V of the site's job (the same double expression the fused step forms per
// site), rounded to FP32 once per run.  start[j]: the first site of job j.
__global__ void real_weights_kernel(float* __restrict__ w, const double2* __restrict__ phi,
                                    const uint64_t* __restrict__ start, const double* __restrict__ inv_vol,
                                    int njobs, double a, uint64_t sites) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < sites; e += (uint64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = njobs - 1;  // the last job that starts at or before e
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(start + mid) <= e) lo = mid;
      else hi = mid - 1;
    }
    w[e] = (float)((1.0 + a * __ldg(phi + e).x) * __ldg(inv_vol + lo));
  }
}

}  // namespace
}  // namespace nrcps

struct nrcps_batch {
  nrcps_context* ctx = nullptr;
  nrcps_batch_params params{};
  std::vector<nrcps::Group> groups;
  std::vector<long> job_off, job_size;  // output offset / size (doubles) per job
  long out_doubles = 0;
  uint64_t sites = 0;              // field sites of one run
  double* phi = nullptr;           // Gaussian / Z3 fields, interleaved complex
  uint32_t* bits = nullptr;        // Z2 fields
  float* wt[2] = {nullptr, nullptr};  // FP32 orbitals, real Gaussian fields: one weight per site (two
                                      // buffers when the next run's fields are drawn during this run)
  uint64_t* job_start = nullptr;   // first field site of every job (device)
  double* job_inv_vol = nullptr;   // 1 / V of every job (device)
  int njobs = 0;
  uint64_t stream_pos = 0;         // generator position (uniforms) of the next run
  cudaGraph_t graph[2] = {nullptr, nullptr};  // one time loop per weight buffer
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  double* out_captured = nullptr;
  long launches_per_run = 0;
  // drawing the next run's fields on a side stream while a run's graph runs
  bool prefetch = false;
  cudaStream_t side = nullptr;
  cudaEvent_t ready[2] = {nullptr, nullptr};  // buffer j's fields drawn
  cudaEvent_t used[2] = {nullptr, nullptr};   // the graph that read buffer j is done
  cudaEvent_t before = nullptr;               // the work issued before a run's graph
  bool prepared[2] = {false, false};
  bool used_recorded[2] = {false, false};
  int next = 0;  // buffer of the next run
};

namespace nrcps {

static nrcps_status record_batch(nrcps_batch* b, double* out, const float* wtab) {
  nrcps_context* ctx = b->ctx;
  const nrcps_precision prec = (nrcps_precision)b->params.precision;
  const long n0 = ctx->launches;
  cudaStream_t main = ctx->stream;
  cudaEvent_t fork;
  NRCPS_TRY(check_cuda(ctx, cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event"));
  NRCPS_TRY(check_cuda(ctx, cudaEventRecord(fork, main), "fork record"));
  nrcps_status st = NRCPS_OK;
  for (Group& g : b->groups) {
    if ((st = check_cuda(ctx, cudaStreamWaitEvent(g.stream, fork, 0), "fork wait"))) break;
    ctx->stream = g.stream;
    const int d3[3] = {g.L, g.L, g.L};
    batch_scatter_sources_kernel<<<grid_for((long)g.nconf * g.N * g.V, 256, (long)ctx->sm_count * 16), 256, 0,
                                   g.stream>>>(g.psi, prec == NRCPS_F64, g.N, g.nconf, g.V, g.pw_index);
    ctx->launches++;
    if ((st = check_launch(ctx, "batch_scatter_sources_kernel"))) break;
    if (g.qr_logR &&
        (st = check_cuda(ctx, cudaMemsetAsync(g.qr_logR, 0, sizeof(double) * g.nconf * g.N, g.stream), "memset")))
      break;
    const long cstride = 2L * g.Tmax * g.N;
    for (int t = 0; t < g.Tmax && !st; ++t) {
      const int na = g.nact[t];
      if ((st = gather_impl(ctx, g.pw_index, g.N, g.psi, g.N, na, g.V, prec, g.S))) break;
      if ((st = slater_dets_dispatch(ctx, g.S, nullptr, g.N, na, 0, 0, g.dets, cstride, 2L * t * g.N, g.lu_scr)))
        break;
      if (g.qr_logR && t >= b->params.qr_period &&
          (st = rescale_dets(ctx, g.dets, g.qr_logR, g.N, na, cstride, 2L * t * g.N, 0)))
        break;
      if (t + 1 >= g.Tmax) break;
      const int nn = g.nact[t + 1];  // configurations measured again at t + 1
      nrcps_position_factor pf{};
      pf.field_mode = b->bits ? 1 : wtab ? 3 : 2;
      pf.dev_field = b->bits ? (const void*)b->bits : wtab ? (const void*)wtab : (const void*)b->phi;
      pf.bit0 = (uint64_t)t * g.V;
      pf.conf_stride = 0;
      pf.dev_conf_base = g.conf_base;
      pf.a = b->params.a;
      pf.dev_pos = nullptr;
      if ((st = propagate_impl(ctx, g.psi, g.N, nn, d3, g.kinv, g.kinv_f, &pf, prec, nullptr))) break;
      if (g.qr_logR && (t + 1) % b->params.qr_period == 0 &&
          (st = qr_reorthonormalise(ctx, g.psi, g.N, g.V, nn, prec, g.qr_G, g.qr_logR)))
        break;
    }
    if (st) break;
    batch_gather_dets_kernel<<<grid_for((long)g.nconf * g.Tmax * g.N, 256, (long)ctx->sm_count * 8), 256, 0,
                               g.stream>>>(g.dets, g.N, g.Tmax, g.nconf, g.conf_T, g.out_off, out);
    ctx->launches++;
    if ((st = check_launch(ctx, "batch_gather_dets_kernel"))) break;
    if ((st = check_cuda(ctx, cudaEventRecord(g.done, g.stream), "join record"))) break;
    ctx->stream = main;
    if ((st = check_cuda(ctx, cudaStreamWaitEvent(main, g.done, 0), "join wait"))) break;
  }
  ctx->stream = main;
  cudaEventDestroy(fork);
  b->launches_per_run = ctx->launches - n0;
  return st;
}

}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_batch_destroy(nrcps_batch* b) {
  if (!b) return NRCPS_OK;
  if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
  if (b->side) cudaStreamSynchronize(b->side);
  for (int j = 0; j < 2; ++j) {
    if (b->exec[j]) cudaGraphExecDestroy(b->exec[j]);
    if (b->graph[j]) cudaGraphDestroy(b->graph[j]);
    if (b->ready[j]) cudaEventDestroy(b->ready[j]);
    if (b->used[j]) cudaEventDestroy(b->used[j]);
  }
  if (b->before) cudaEventDestroy(b->before);
  if (b->side) cudaStreamDestroy(b->side);
  for (Group& g : b->groups) {
    if (g.stream) cudaStreamSynchronize(g.stream);
    void* bufs[] = {g.psi, g.kinv, g.kinv_f, g.pw_index, g.conf_base, g.out_off, g.conf_T,
                    g.S, g.lu_scr, g.dets, g.qr_G, g.qr_logR};
    for (void* p : bufs)
      if (p) cudaFree(p);
    if (g.done) cudaEventDestroy(g.done);
    if (g.stream) cudaStreamDestroy(g.stream);
  }
  void* fields[] = {b->phi, b->bits, b->wt[0], b->wt[1], b->job_start, b->job_inv_vol};
  for (void* p : fields)
    if (p) cudaFree(p);
  delete b;
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_batch_create(nrcps_context* ctx, const nrcps_batch_params* params,
                                           const nrcps_batch_job* jobs, int njobs, nrcps_batch** out) {
  if (!ctx || !out) return NRCPS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  NRCPS_REQUIRE(ctx, params && jobs && njobs > 0, "nrcps_batch_create: bad arguments");
  NRCPS_REQUIRE(ctx, params->field_kind >= 0 && params->field_kind <= 3 && params->qr_period >= 0,
                "nrcps_batch_create: bad field kind or qr_period");
  NRCPS_REQUIRE(ctx, params->precision == NRCPS_F32 || params->precision == NRCPS_F64,
                "nrcps_batch_create: bad precision");
  for (int j = 0; j < njobs; ++j) {
    const nrcps_batch_job& jb = jobs[j];
    NRCPS_REQUIRE(ctx, jb.L > 0 && jb.n_orb > 0 && jb.T > 0 && jb.n_conf > 0 && jb.pw_index && jb.kin_xi,
                  "nrcps_batch_create: bad job %d", j);
    NRCPS_REQUIRE(ctx, jb.n_orb <= 64 || params->qr_period == 0, "nrcps_batch_create: QR needs N <= 64 (job %d)", j);
  }
  nrcps_batch* b = new nrcps_batch();
  b->ctx = ctx;
  b->params = *params;
  auto fail = [&](nrcps_status s) {
    nrcps_batch_destroy(b);
    return s;
  };
  // ---- layout: groups by (L, N); field bases in job order
  std::vector<uint64_t> base(njobs);
  uint64_t acc = 0;
  b->job_off.resize(njobs);
  b->job_size.resize(njobs);
  long out_acc = 0;
  for (int j = 0; j < njobs; ++j) {
    const long V = (long)jobs[j].L * jobs[j].L * jobs[j].L;
    base[j] = acc;
    acc += (uint64_t)jobs[j].n_conf * jobs[j].T * V;
    b->job_off[j] = out_acc;
    b->job_size[j] = 2L * jobs[j].n_conf * jobs[j].T * jobs[j].n_orb;
    out_acc += b->job_size[j];
  }
  b->sites = acc;
  b->out_doubles = out_acc;
  std::vector<std::pair<int, int>> keys;
  for (int j = 0; j < njobs; ++j) {
    std::pair<int, int> k(jobs[j].L, jobs[j].n_orb);
    if (std::find(keys.begin(), keys.end(), k) == keys.end()) keys.push_back(k);
  }
  b->groups.resize(keys.size());
  nrcps_status st = NRCPS_OK;
  for (size_t gi = 0; gi < keys.size(); ++gi) {
    Group& g = b->groups[gi];
    g.L = keys[gi].first;
    g.N = keys[gi].second;
    g.V = (long)g.L * g.L * g.L;
    // configurations of this group: (T, field base, output offset), longest first
    struct Conf {
      int T;
      uint64_t base;
      long out;
      int job;
    };
    std::vector<Conf> confs;
    const int* idx0 = nullptr;
    const double* xi0 = nullptr;
    for (int j = 0; j < njobs; ++j) {
      if (jobs[j].L != g.L || jobs[j].n_orb != g.N) continue;
      if (!idx0) {
        idx0 = jobs[j].pw_index;
        xi0 = jobs[j].kin_xi;
      }
      for (int k = 0; k < jobs[j].n_conf; ++k)
        confs.push_back(Conf{jobs[j].T, base[j] + (uint64_t)k * jobs[j].T * g.V,
                             b->job_off[j] + 2L * k * jobs[j].T * g.N, j});
    }
    std::stable_sort(confs.begin(), confs.end(), [](const Conf& a, const Conf& c) { return a.T > c.T; });
    g.nconf = (int)confs.size();
    g.Tmax = confs.front().T;
    g.nact.assign(g.Tmax, 0);
    for (const Conf& c : confs)
      for (int t = 0; t < c.T; ++t) g.nact[t]++;
    std::vector<uint64_t> hb(g.nconf);
    std::vector<long> ho(g.nconf);
    std::vector<int> ht(g.nconf);
    for (int c = 0; c < g.nconf; ++c) {
      hb[c] = confs[c].base;
      ho[c] = confs[c].out;
      ht[c] = confs[c].T;
    }
    const size_t es = params->precision == NRCPS_F64 ? 16 : 8;
    auto alloc = [&](void** p, size_t bytes) { return check_cuda(ctx, cudaMalloc(p, bytes), "cudaMalloc(batch)"); };
    auto up = [&](void* d, const void* h, size_t bytes) {
      return check_cuda(ctx, cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(batch)");
    };
    std::vector<double> kinv(g.V);
    std::vector<float2> kf(g.V);
    for (long i = 0; i < g.V; ++i) {
      kinv[i] = 1.0 / xi0[i];
      const float hi = (float)kinv[i];
      kf[i] = make_float2(hi, (float)(kinv[i] - (double)hi));
    }
    if ((st = alloc(&g.psi, es * (size_t)g.nconf * g.N * g.V)) || (st = alloc((void**)&g.kinv, 8 * g.V)) ||
        (st = up(g.kinv, kinv.data(), 8 * g.V)) || (st = alloc((void**)&g.kinv_f, 8 * g.V)) ||
        (st = up(g.kinv_f, kf.data(), 8 * g.V)) || (st = alloc((void**)&g.pw_index, 4 * g.N)) ||
        (st = up(g.pw_index, idx0, 4 * g.N)) || (st = alloc((void**)&g.conf_base, 8 * g.nconf)) ||
        (st = up(g.conf_base, hb.data(), 8 * g.nconf)) || (st = alloc((void**)&g.out_off, 8 * g.nconf)) ||
        (st = up(g.out_off, ho.data(), 8 * g.nconf)) || (st = alloc((void**)&g.conf_T, 4 * g.nconf)) ||
        (st = up(g.conf_T, ht.data(), 4 * g.nconf)) || (st = alloc((void**)&g.S, 16 * (size_t)g.nconf * g.N * g.N)) ||
        (st = alloc((void**)&g.lu_scr, slater_dets_scratch_bytes(g.N, g.nconf, 0))) ||
        (st = alloc((void**)&g.dets, 16 * (size_t)g.nconf * g.Tmax * g.N)))
      return fail(st);
    if (params->qr_period > 0 &&
        ((st = alloc((void**)&g.qr_G, 16 * (size_t)g.nconf * g.N * g.N)) ||
         (st = alloc((void**)&g.qr_logR, 8 * (size_t)g.nconf * g.N))))
      return fail(st);
    if ((st = check_cuda(ctx, cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking), "stream")) ||
        (st = check_cuda(ctx, cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming), "event")))
      return fail(st);
    if (g.L < 64) fused_autotune(ctx, (nrcps_precision)params->precision, g.L, nullptr);
  }
  if (params->field_kind == NRCPS_FIELD_ZTWO) {
    if ((st = check_cuda(ctx, cudaMalloc((void**)&b->bits, 4 * ((b->sites + 31) / 32 + 1)), "cudaMalloc(bits)")))
      return fail(st);
  } else {
    if ((st = check_cuda(ctx, cudaMalloc((void**)&b->phi, 16 * (size_t)b->sites), "cudaMalloc(phi)")))
      return fail(st);
    if (params->field_kind == NRCPS_FIELD_GAUSS && params->precision == NRCPS_F32 && ctx->batch_real_weights) {
      std::vector<double> iv(njobs);
      for (int j = 0; j < njobs; ++j) iv[j] = 1.0 / ((double)jobs[j].L * jobs[j].L * jobs[j].L);
      b->njobs = njobs;
      if ((st = check_cuda(ctx, cudaMalloc((void**)&b->wt[0], 4 * (size_t)b->sites), "cudaMalloc(weights)")) ||
          (st = check_cuda(ctx, cudaMalloc((void**)&b->job_start, 8 * (size_t)njobs), "cudaMalloc(job starts)")) ||
          (st = check_cuda(ctx, cudaMalloc((void**)&b->job_inv_vol, 8 * (size_t)njobs), "cudaMalloc(job 1/V)")) ||
          (st = check_cuda(ctx, cudaMemcpy(b->job_start, base.data(), 8 * (size_t)njobs, cudaMemcpyHostToDevice),
                           "cudaMemcpy(job starts)")) ||
          (st = check_cuda(ctx, cudaMemcpy(b->job_inv_vol, iv.data(), 8 * (size_t)njobs, cudaMemcpyHostToDevice),
                           "cudaMemcpy(job 1/V)")))
        return fail(st);
      if (ctx->batch_prefetch_fields) {
        b->prefetch = true;
        if ((st = check_cuda(ctx, cudaMalloc((void**)&b->wt[1], 4 * (size_t)b->sites), "cudaMalloc(weights)")) ||
            (st = check_cuda(ctx, cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking), "stream")))
          return fail(st);
        for (int j = 0; j < 2; ++j)
          if ((st = check_cuda(ctx, cudaEventCreateWithFlags(&b->ready[j], cudaEventDisableTiming), "event")) ||
              (st = check_cuda(ctx, cudaEventCreateWithFlags(&b->used[j], cudaEventDisableTiming), "event")))
            return fail(st);
        if ((st = check_cuda(ctx, cudaEventCreateWithFlags(&b->before, cudaEventDisableTiming), "event")))
          return fail(st);
      }
    }
  }
  *out = b;
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_batch_layout(const nrcps_batch* b, int job, long* offset, long* doubles) {
  if (!b || job < 0 || job >= (int)b->job_off.size()) return NRCPS_ERR_INVALID_ARGUMENT;
  if (offset) *offset = b->job_off[job];
  if (doubles) *doubles = b->job_size[job];
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_batch_output_size(const nrcps_batch* b, long* doubles, long* launches) {
  if (!b) return NRCPS_ERR_INVALID_ARGUMENT;
  if (doubles) *doubles = b->out_doubles;
  if (launches) *launches = b->launches_per_run;
  return NRCPS_OK;
}

namespace nrcps {

// One run's fields, the next window of the stream, on the context's current
// stream: Z2 bits, or phi and (FP32, real Gaussian) weight buffer j.
static nrcps_status draw_run_fields(nrcps_batch* b, int j) {
  nrcps_context* ctx = b->ctx;
  if (b->params.field_kind == NRCPS_FIELD_ZTWO) {
    NRCPS_TRY(nrcps_draw_z2_bits(ctx, b->params.rng_kind, b->params.seed, b->stream_pos, b->sites, b->bits));
    b->stream_pos += b->sites;
    return NRCPS_OK;
  }
  NRCPS_TRY(nrcps_draw_fields(ctx, b->params.rng_kind, b->params.seed, b->params.field_kind, (long)b->sites, 1,
                              &b->stream_pos, b->phi));
  if (b->wt[j]) {
    real_weights_kernel<<<grid_for((long)b->sites, 256, (long)ctx->sm_count * 16), 256, 0, ctx->stream>>>(
        b->wt[j], reinterpret_cast<const double2*>(b->phi), b->job_start, b->job_inv_vol, b->njobs, b->params.a,
        b->sites);
    ctx->launches++;
    NRCPS_TRY(check_launch(ctx, "real_weights_kernel"));
  }
  return NRCPS_OK;
}

// The time loop of weight buffer j captured into graph j.
static nrcps_status capture_batch(nrcps_batch* b, double* dev_out, int j) {
  nrcps_context* ctx = b->ctx;
  NRCPS_TRY(check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "sync before capture"));
  cudaStream_t cap = ctx->stream;
  bool own = false;
  if (cap == nullptr) {
    NRCPS_TRY(check_cuda(ctx, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "stream create"));
    own = true;
  }
  cudaStream_t saved = ctx->stream;
  ctx->stream = cap;
  nrcps_status rs = check_cuda(ctx, cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
  if (rs == NRCPS_OK) {
    rs = record_batch(b, dev_out, b->wt[j]);
    cudaError_t ce = cudaStreamEndCapture(cap, &b->graph[j]);
    if (rs == NRCPS_OK) rs = check_cuda(ctx, ce, "end capture");
  }
  ctx->stream = saved;
  if (rs == NRCPS_OK) rs = check_cuda(ctx, cudaGraphInstantiate(&b->exec[j], b->graph[j], 0), "graph instantiate");
  if (own) cudaStreamDestroy(cap);
  return rs;
}

}  // namespace nrcps

extern "C" nrcps_status nrcps_batch_run(nrcps_batch* b, double* dev_out) {
  if (!b) return NRCPS_ERR_INVALID_ARGUMENT;
  nrcps_context* ctx = b->ctx;
  NRCPS_REQUIRE(ctx, dev_out, "nrcps_batch_run: null output");
  const int j = b->prefetch ? b->next : 0;  // this run's weight buffer
  // ---- this run's fields: the next window of the one stream (drawn during
  // the previous run when prefetching)
  if (b->prefetch && b->prepared[j]) {
    NRCPS_TRY(check_cuda(ctx, cudaStreamWaitEvent(ctx->stream, b->ready[j], 0), "wait fields"));
    b->prepared[j] = false;
  } else {
    NRCPS_TRY(draw_run_fields(b, j));
  }
  const int ngraphs = b->prefetch ? 2 : 1;
  if (b->out_captured != dev_out) {
    for (int i = 0; i < 2; ++i) {
      if (b->exec[i]) cudaGraphExecDestroy(b->exec[i]);
      if (b->graph[i]) cudaGraphDestroy(b->graph[i]);
      b->exec[i] = nullptr;
      b->graph[i] = nullptr;
    }
    b->out_captured = dev_out;
  }
  for (int i = 0; i < ngraphs; ++i)
    if (!b->exec[i]) NRCPS_TRY(capture_batch(b, dev_out, i));
  // the side draw below starts after everything issued before this graph
  // (it may share the context's scratch and generator arguments with it)
  if (b->prefetch) NRCPS_TRY(check_cuda(ctx, cudaEventRecord(b->before, ctx->stream), "record before"));
  NRCPS_TRY(check_cuda(ctx, cudaGraphLaunch(b->exec[j], ctx->stream), "graph launch"));
  if (!b->prefetch) return NRCPS_OK;
  // ---- the next run's fields into the other buffer, on the side stream,
  // once the graph that last read that buffer is done
  NRCPS_TRY(check_cuda(ctx, cudaEventRecord(b->used[j], ctx->stream), "record used"));
  b->used_recorded[j] = true;
  const int o = j ^ 1;
  if (b->used_recorded[o]) NRCPS_TRY(check_cuda(ctx, cudaStreamWaitEvent(b->side, b->used[o], 0), "wait used"));
  NRCPS_TRY(check_cuda(ctx, cudaStreamWaitEvent(b->side, b->before, 0), "wait before"));
  if (ctx->side_pending) NRCPS_TRY(check_cuda(ctx, cudaStreamWaitEvent(b->side, ctx->side_done, 0), "wait side"));
  cudaStream_t main = ctx->stream;
  ctx->stream = b->side;
  const nrcps_status st = draw_run_fields(b, o);
  ctx->stream = main;
  NRCPS_TRY(st);
  NRCPS_TRY(check_cuda(ctx, cudaEventRecord(b->ready[o], b->side), "record ready"));
  if (!ctx->side_done)
    NRCPS_TRY(check_cuda(ctx, cudaEventCreateWithFlags(&ctx->side_done, cudaEventDisableTiming), "event"));
  NRCPS_TRY(check_cuda(ctx, cudaEventRecord(ctx->side_done, b->side), "record side"));
  ctx->side_pending = true;
  b->prepared[o] = true;
  b->next = o;
  return NRCPS_OK;
}

// branch.cu -- the multilevel branching driver
// (production/two_body-branched/main.C:23-80, MultiLevel) on the device.
//
// The reference walks the tree depth first: a node of depth d (level
// levels - d) restarts its `branches` children from its end state, each child
// evolves prop1 and prop2 for `steps` slices -- measuring
// TwoBody::Run(prop1, prop2) / branches^(d+1) into corr[t] before every step
// and drawing a fresh field after it -- and recurses.  Here the tree is
// walked breadth first: all branches^(d+1) nodes of depth d advance together
// (one batched pair measurement, one fused propagation of 2 orbitals per node
// per slice), then every node's end state is copied to its children.  Each
// node reads the field slices the depth-first walk would have drawn for it:
// with f(l) = steps * b (b^l - 1)/(b - 1) slices consumed below a call at
// level l, the node with branch digits (i_0 .. i_d) starts at slice
//   sum_k i_k (steps + f(levels - k - 1)) + d * steps
// of its tree, and tree r starts at r f(levels) (the stream continues across
// trees; slice 0 is the Lattice constructor's draw).
//
// Hamiltonians [K, (V), I, (V), K] with the local interaction (1 + a phi)/V:
// the driver's Interaction3 and Propagator::SetSource are no longer in the
// reference's headers.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace nrcps {
nrcps_status pair_impl(nrcps_context* ctx, const void* psi1, const void* psi2, int n, int nconf, long vol,
                       const double* w, const int* opp, nrcps_precision prec, double* phi, int props);
nrcps_status propagate_impl(nrcps_context* ctx, void* psi, int batch, int nconf, const int d[3], const double* kin,
                            const float2* kin_f32, const nrcps_position_factor* w, nrcps_precision prec,
                            const void* zpos);
nrcps_status fused_autotune(nrcps_context* ctx, nrcps_precision prec, int L, int* chosen_cluster);

namespace {

__global__ void branch_seed_kernel(void* psi, int is_f64, int nstates, long vol, const double* src2) {
  const long total = (long)nstates * 2 * vol;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long r = e % (2 * vol);  // orbital * vol + site within a state
    const double re = src2[2 * r], im = src2[2 * r + 1];
    if (is_f64) reinterpret_cast<double2*>(psi)[e] = make_double2(re, im);
    else reinterpret_cast<float2*>(psi)[e] = make_float2((float)re, (float)im);
  }
}

// child c (depth d + 1) = parent c / b (depth d)
__global__ void branch_expand_kernel(const void* src, void* dst, int esize16, long state_elems, int b, long nchild) {
  const long total = nchild * state_elems;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long child = e / state_elems, r = e - child * state_elems;
    const long from = (child / b) * state_elems + r;
    if (esize16) reinterpret_cast<double2*>(dst)[e] = reinterpret_cast<const double2*>(src)[from];
    else reinterpret_cast<float2*>(dst)[e] = reinterpret_cast<const float2*>(src)[from];
  }
}

// conf_base[n] = (tree0 + start(path of node n at depth d)) * vol
__global__ void branch_bases_kernel(uint64_t* base, long nnodes, int d, int levels, int b, int steps,
                                    const long* fsub, uint64_t tree0, long vol) {
  for (long n = (long)blockIdx.x * blockDim.x + threadIdx.x; n < nnodes; n += (long)gridDim.x * blockDim.x) {
    long rem = n;
    uint64_t start = (uint64_t)d * steps;
    for (int k = d; k >= 0; --k) {  // digit i_k is the base-b digit of weight b^(d-k)
      const long ik = rem % b;
      rem /= b;
      start += (uint64_t)ik * (uint64_t)(steps + fsub[levels - k - 1]);
    }
    base[n] = (tree0 + start) * (uint64_t)vol;
  }
}

// corr[t] += sum_n phi[n][0][1] / norm  (phi: 2 x 2 complex per node; element
// (s = 0, t = 1) at offset 2 (1 + 2 * 0) is TwoBody::Run(prop1, prop2))
__global__ void branch_reduce_kernel(const double* phi, long nnodes, double inv_norm, double* corr_t) {
  __shared__ double red[2][256];
  double re = 0.0, im = 0.0;
  for (long n = threadIdx.x; n < nnodes; n += blockDim.x) {
    re += phi[8 * n + 2];
    im += phi[8 * n + 3];
  }
  red[0][threadIdx.x] = re;
  red[1][threadIdx.x] = im;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    corr_t[0] += red[0][0] * inv_norm;
    corr_t[1] += red[1][0] * inv_norm;
  }
}

}  // namespace
}  // namespace nrcps

struct nrcps_branch {
  nrcps_context* ctx = nullptr;
  nrcps_branch_params p{};
  long vol = 0;
  int T = 0;
  long nmax = 0;                 // nodes at the deepest level
  std::vector<long> fsub;        // f(l), l = 0 .. levels
  void* psi[2] = {nullptr, nullptr};
  double* kinv = nullptr;
  float2* kinv_f = nullptr;
  double* pos = nullptr;
  double* w = nullptr;
  int* opp = nullptr;
  int pair_props = 3;  // the pair table's properties, checked on the host (pair_table_props)
  double* src2 = nullptr;
  double* phi = nullptr;         // nmax x 2 x 2 complex
  uint64_t* base = nullptr;
  long* fsub_dev = nullptr;
  uint32_t* bits = nullptr;
  double* phif = nullptr;
  uint64_t tree_slices = 0;
  uint64_t next_tree = 0;
  uint64_t gauss_pos = 0;
};

using namespace nrcps;

extern "C" nrcps_status nrcps_branch_destroy(nrcps_branch* b) {
  if (!b) return NRCPS_OK;
  if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
  void* bufs[] = {b->psi[0], b->psi[1], b->kinv, b->kinv_f, b->pos, b->w, b->opp, b->src2, b->phi, b->base,
                  b->fsub_dev, b->bits, b->phif};
  for (void* q : bufs)
    if (q) cudaFree(q);
  delete b;
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_branch_create(nrcps_context* ctx, const nrcps_branch_params* p, const double* kin_xi,
                                            const double* pot, const double* sources2, const double* w,
                                            const int* opposite, nrcps_branch** out) {
  if (!ctx || !out) return NRCPS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  NRCPS_REQUIRE(ctx, p && kin_xi && sources2 && w && opposite, "nrcps_branch_create: bad arguments");
  NRCPS_REQUIRE(ctx, p->levels > 0 && p->branches > 0 && p->steps > 0,
                "nrcps_branch_create: levels, branches and steps must be positive");
  NRCPS_REQUIRE(ctx, p->field_kind >= 0 && p->field_kind <= 3, "nrcps_branch_create: bad field kind");
  double nodes = std::pow((double)p->branches, (double)p->levels);
  NRCPS_REQUIRE(ctx, nodes <= (double)(1L << 26), "nrcps_branch_create: branches^levels above 2^26");
  nrcps_branch* b = new nrcps_branch();
  b->ctx = ctx;
  b->p = *p;
  b->vol = (long)p->dims[0] * p->dims[1] * p->dims[2];
  b->T = p->levels * p->steps;
  b->nmax = (long)nodes;
  b->fsub.assign(p->levels + 1, 0);
  for (int l = 1; l <= p->levels; ++l) b->fsub[l] = (long)p->branches * (p->steps + b->fsub[l - 1]);
  b->tree_slices = (uint64_t)b->fsub[p->levels];
  auto fail = [&](nrcps_status s) {
    nrcps_branch_destroy(b);
    return s;
  };
  const long V = b->vol;
  const size_t es = p->precision == NRCPS_F64 ? 16 : 8;
  auto alloc = [&](void** q, size_t bytes) { return check_cuda(ctx, cudaMalloc(q, bytes), "cudaMalloc(branch)"); };
  auto up = [&](void* d, const void* h, size_t bytes) {
    return check_cuda(ctx, cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(branch)");
  };
  std::vector<double> kinv(V);
  std::vector<float2> kf(V);
  for (long i = 0; i < V; ++i) {
    kinv[i] = 1.0 / kin_xi[i];
    const float hi = (float)kinv[i];
    kf[i] = make_float2(hi, (float)(kinv[i] - (double)hi));
  }
  b->pair_props = pair_table_props(opposite, w, V);
  nrcps_status st;
  if ((st = alloc(&b->psi[0], es * 2 * (size_t)b->nmax * V)) || (st = alloc(&b->psi[1], es * 2 * (size_t)b->nmax * V)) ||
      (st = alloc((void**)&b->kinv, 8 * V)) || (st = up(b->kinv, kinv.data(), 8 * V)) ||
      (st = alloc((void**)&b->kinv_f, 8 * V)) || (st = up(b->kinv_f, kf.data(), 8 * V)) ||
      (st = alloc((void**)&b->w, 8 * V)) || (st = up(b->w, w, 8 * V)) || (st = alloc((void**)&b->opp, 4 * V)) ||
      (st = up(b->opp, opposite, 4 * V)) || (st = alloc((void**)&b->src2, 32 * V)) ||
      (st = up(b->src2, sources2, 32 * V)) || (st = alloc((void**)&b->phi, 64 * (size_t)b->nmax)) ||
      (st = alloc((void**)&b->base, 8 * (size_t)b->nmax)) ||
      (st = alloc((void**)&b->fsub_dev, 8 * (size_t)(p->levels + 1))) ||
      (st = up(b->fsub_dev, b->fsub.data(), 8 * (size_t)(p->levels + 1))))
    return fail(st);
  if (pot) {
    // [K,V,I,V,K] = K B diag(V^2 v^2 fld) F K (unnormalised transforms)
    std::vector<double> h(V);
    for (long i = 0; i < V; ++i) h[i] = ((double)V * pot[i]) * ((double)V * pot[i]);
    if ((st = alloc((void**)&b->pos, 8 * V)) || (st = up(b->pos, h.data(), 8 * V))) return fail(st);
  }
  const uint64_t sites = (b->tree_slices + 1) * (uint64_t)V;
  if (p->field_kind == NRCPS_FIELD_ZTWO) {
    if ((st = alloc((void**)&b->bits, 4 * ((sites + 31) / 32 + 1)))) return fail(st);
  } else {
    if ((st = alloc((void**)&b->phif, 16 * (size_t)sites))) return fail(st);
  }
  if (p->dims[0] == p->dims[1] && p->dims[1] == p->dims[2] && p->dims[0] < 64)
    fused_autotune(ctx, (nrcps_precision)p->precision, p->dims[0], nullptr);
  *out = b;
  return NRCPS_OK;
}

// One tree: dev_corr (levels * steps complex doubles, device) receives the
// tree's weighted sums (added to what it holds).
extern "C" nrcps_status nrcps_branch_run(nrcps_branch* b, double* dev_corr) {
  if (!b) return NRCPS_ERR_INVALID_ARGUMENT;
  nrcps_context* ctx = b->ctx;
  NRCPS_REQUIRE(ctx, dev_corr, "nrcps_branch_run: null output");
  const nrcps_branch_params& p = b->p;
  const long V = b->vol;
  const nrcps_precision prec = (nrcps_precision)p.precision;
  // fields of this tree: slices [r f, (r + 1) f) of the stream
  const uint64_t slices = b->tree_slices;
  if (p.field_kind == NRCPS_FIELD_ZTWO) {
    NRCPS_TRY(nrcps_draw_z2_bits(ctx, p.rng_kind, p.seed, b->next_tree * slices * V, slices * V, b->bits));
  } else if (p.field_kind == NRCPS_FIELD_ZTHREE) {
    uint64_t off = b->next_tree * slices * V;
    NRCPS_TRY(nrcps_draw_fields(ctx, p.rng_kind, p.seed, p.field_kind, V, (long)slices, &off, b->phif));
  } else {
    NRCPS_TRY(nrcps_draw_fields(ctx, p.rng_kind, p.seed, p.field_kind, V, (long)slices, &b->gauss_pos, b->phif));
  }
  b->next_tree++;
  const int B = p.branches;
  int cur = 0;
  long nn = B;
  branch_seed_kernel<<<grid_for(nn * 2 * V, 256, (long)ctx->sm_count * 16), 256, 0, ctx->stream>>>(
      b->psi[cur], prec == NRCPS_F64, (int)nn, V, b->src2);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "branch_seed_kernel"));
  for (int d = 0; d < p.levels; ++d) {
    if (d > 0) {
      const long nchild = nn * B;
      branch_expand_kernel<<<grid_for(nchild * 2 * V, 256, (long)ctx->sm_count * 16), 256, 0, ctx->stream>>>(
          b->psi[cur], b->psi[1 - cur], prec == NRCPS_F64, 2 * V, B, nchild);
      ctx->launches++;
      NRCPS_TRY(check_launch(ctx, "branch_expand_kernel"));
      cur = 1 - cur;
      nn = nchild;
    }
    branch_bases_kernel<<<grid_for(nn, 256), 256, 0, ctx->stream>>>(b->base, nn, d, p.levels, B, p.steps, b->fsub_dev,
                                                                    0, V);
    ctx->launches++;
    NRCPS_TRY(check_launch(ctx, "branch_bases_kernel"));
    const double inv_norm = 1.0 / std::pow((double)B, (double)(d + 1));
    for (int s = 0; s < p.steps; ++s) {
      const int t = d * p.steps + s;
      NRCPS_TRY(pair_impl(ctx, b->psi[cur], b->psi[cur], 2, (int)nn, V, b->w, b->opp, prec, b->phi, b->pair_props));
      branch_reduce_kernel<<<1, 256, 0, ctx->stream>>>(b->phi, nn, inv_norm, dev_corr + 2L * t);
      ctx->launches++;
      NRCPS_TRY(check_launch(ctx, "branch_reduce_kernel"));
      if (d == p.levels - 1 && s == p.steps - 1) break;  // nothing measures the leaves' last step
      nrcps_position_factor pf{};
      pf.field_mode = b->bits ? 1 : 2;
      pf.dev_field = b->bits ? (const void*)b->bits : (const void*)b->phif;
      pf.bit0 = (uint64_t)s * V;
      pf.conf_stride = 0;
      pf.dev_conf_base = b->base;
      pf.a = p.a;
      pf.dev_pos = b->pos;
      NRCPS_TRY(propagate_impl(ctx, b->psi[cur], 2, (int)nn, p.dims, b->kinv, b->kinv_f, &pf, prec, nullptr));
    }
  }
  return NRCPS_OK;
}

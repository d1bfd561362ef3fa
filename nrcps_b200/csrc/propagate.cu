// propagate.cu -- batched 3-D FFT and the Hamiltonian steps of the transfer
// matrix (Fourier, Kinetic, Potential, Interaction, Propagator::Run).
//
// Pencil kernels: one thread owns one pencil of N sites along one axis of one
// orbital, holds it in registers and transforms it with fft::Dft<N>.  A 3-D
// transform is three pencil passes (z, y, x).  The fused propagator step
//   psi <- k .* B[ w .* F[ k .* psi ] ]
// runs as five passes: z-forward with the kinetic pre-factor, y-forward,
// x-forward * w(x) * x-backward in one pass, y-backward, z-backward with the
// kinetic post-factor.
#include <cstring>

#include "common.cuh"
#include "fft.cuh"

namespace nrcps {

struct PencilGeom {
  long vol;           // sites per orbital
  long npencils;      // pencils per orbital (vol / N)
  long inner;         // pencil index r -> site base (r / inner) * outer + (r % inner)
  long outer;
  long stride;        // site stride along the pencil
};

enum PencilOp { OP_NONE = 0, OP_PRE_MUL = 1, OP_POST_MUL = 2, OP_MID_FIELD = 3 };

struct FieldArgs {
  int mode;              // 0 complex fld, 1 Z2 bits, 2 interleaved complex phi, 3 real FP32 weights
  const void* field;
  uint64_t bit0;         // element (mode 0/2) or bit (mode 1) offset of configuration 0
  uint64_t conf_stride;  // elements or bits between configurations
  const uint64_t* conf_base;  // optional per-configuration offsets (replace conf * conf_stride)
  double a;
  double vol;
  const double* pos;     // optional static real factor
  int orbs_per_conf;
};

template <typename R>
__device__ __forceinline__ cplx<R> field_factor(const FieldArgs& f, long conf, long site) {
  cplx<R> w;
  const uint64_t k = f.bit0 + (f.conf_base ? f.conf_base[conf] : (uint64_t)conf * f.conf_stride) + (uint64_t)site;
  if (f.mode == 0) {
    double2 v = reinterpret_cast<const double2*>(f.field)[k];
    w = cplx<R>{(R)v.x, (R)v.y};
  } else if (f.mode == 1) {
    uint32_t word = reinterpret_cast<const uint32_t*>(f.field)[k >> 5];
    double phi = ((word >> (k & 31)) & 1u) ? 1.0 : -1.0;
    w = cplx<R>{(R)((1.0 + f.a * phi) / f.vol), (R)0};
  } else if (f.mode == 3) {
    w = cplx<R>{(R)reinterpret_cast<const float*>(f.field)[k], (R)0};
  } else {
    double2 phi = reinterpret_cast<const double2*>(f.field)[k];
    w = cplx<R>{(R)((1.0 + f.a * phi.x) / f.vol), (R)((f.a * phi.y) / f.vol)};
  }
  if (f.pos) {
    R p = (R)f.pos[site];
    w.re *= p;
    w.im *= p;
  }
  return w;
}

template <typename R, int N, int SIGN, int OP>
__global__ void __launch_bounds__(128) pencil_kernel(void* data, long total, PencilGeom g,
                                                     const double* table, FieldArgs f) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (long)gridDim.x * blockDim.x) {
    const long b = p / g.npencils;
    const long r = p - b * g.npencils;
    const long site0 = (r / g.inner) * g.outer + (r % g.inner);
    const long base = b * g.vol + site0;
    cplx<R> x[N];
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = ld<R>(data, base + j * g.stride);
    if constexpr (OP == OP_PRE_MUL) {
#pragma unroll
      for (int j = 0; j < N; ++j) {
        R hi, lo;
        split<R>(table[site0 + j * g.stride], hi, lo);
        x[j] = scale2<R>(x[j], hi, lo);
      }
    }
    fft::Dft<N, SIGN, R>::run(x);
    if constexpr (OP == OP_MID_FIELD) {
      const long conf = b / f.orbs_per_conf;
#pragma unroll
      for (int j = 0; j < N; ++j) x[j] = cmul(field_factor<R>(f, conf, site0 + j * g.stride), x[j]);
      fft::Dft<N, -SIGN, R>::run(x);
    }
    if constexpr (OP == OP_POST_MUL) {
#pragma unroll
      for (int j = 0; j < N; ++j) {
        R hi, lo;
        split<R>(table[site0 + j * g.stride], hi, lo);
        x[j] = scale2<R>(x[j], hi, lo);
      }
    }
#pragma unroll
    for (int j = 0; j < N; ++j) st<R>(data, base + j * g.stride, x[j]);
  }
}

// Geometry of the pencils along `axis` (0 = x, 1 = y, 2 = z).
static PencilGeom geom(const int d[3], int axis) {
  PencilGeom g;
  g.vol = (long)d[0] * d[1] * d[2];
  g.npencils = g.vol / d[axis];
  if (axis == 2) {
    g.inner = 1;
    g.outer = d[2];
    g.stride = 1;
  } else if (axis == 1) {
    g.inner = d[2];
    g.outer = (long)d[1] * d[2];
    g.stride = d[2];
  } else {
    g.inner = (long)d[1] * d[2];
    g.outer = 0;
    g.stride = (long)d[1] * d[2];
  }
  return g;
}

template <typename R, int SIGN, int OP>
static nrcps_status launch_axis(nrcps_context* ctx, void* data, int batch, const int d[3], int axis,
                                const double* table, const FieldArgs& f) {
  PencilGeom g = geom(d, axis);
  long total = g.npencils * batch;
  unsigned grid = grid_for(total, 128, (long)ctx->sm_count * 16);
#define NRCPS_CASE(NN)                                                                   \
  case NN:                                                                               \
    pencil_kernel<R, NN, SIGN, OP><<<grid, 128, 0, ctx->stream>>>(data, total, g, table, f); \
    break;
  switch (d[axis]) {
    NRCPS_CASE(2)
    NRCPS_CASE(4)
    NRCPS_CASE(6)
    NRCPS_CASE(8)
    NRCPS_CASE(12)
    NRCPS_CASE(16)
    NRCPS_CASE(24)
    NRCPS_CASE(32)
    NRCPS_CASE(48)
    default:
      return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "lattice extent %d not supported (2,4,6,8,12,16,24,32,48)",
                       d[axis]);
  }
#undef NRCPS_CASE
  ctx->launches++;
  return check_launch(ctx, "pencil_kernel");
}

static bool extent_ok(int n) {
  switch (n) {
    case 2: case 4: case 6: case 8: case 12: case 16: case 24: case 32: case 48: return true;
    default: return false;
  }
}

static nrcps_status check_dims(nrcps_context* ctx, const int d[3]) {
  for (int i = 0; i < 3; ++i)
    if (!extent_ok(d[i]))
      return set_error(ctx, NRCPS_ERR_UNSUPPORTED, "lattice extent %d not supported (2,4,6,8,12,16,24,32,48)", d[i]);
  return NRCPS_OK;
}

template <typename R>
static nrcps_status fft3d_t(nrcps_context* ctx, void* data, int batch, const int d[3], int sign) {
  FieldArgs f{};
  for (int axis = 2; axis >= 0; --axis) {
    if (sign < 0) NRCPS_TRY((launch_axis<R, -1, OP_NONE>(ctx, data, batch, d, axis, nullptr, f)));
    else NRCPS_TRY((launch_axis<R, +1, OP_NONE>(ctx, data, batch, d, axis, nullptr, f)));
  }
  return NRCPS_OK;
}

static nrcps_status fft3d_any(nrcps_context* ctx, void* data, int batch, const int d[3], nrcps_precision prec,
                              int sign) {
  return prec == NRCPS_F64 ? fft3d_t<double>(ctx, data, batch, d, sign) : fft3d_t<float>(ctx, data, batch, d, sign);
}

// ------------------------------------------------------------ elementwise
template <typename R>
__global__ void div_real_kernel(void* psi, long n, long vol, const double* xi) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    cplx<R> a = ld<R>(psi, i);
    R k = (R)xi[i % vol];
    a.re /= k;
    a.im /= k;
    st<R>(psi, i, a);
  }
}

template <typename R>
__global__ void mul_real_kernel(void* psi, long n, long vol, const double* v) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    cplx<R> a = ld<R>(psi, i);
    R k = (R)v[i % vol];
    a.re *= k;
    a.im *= k;
    st<R>(psi, i, a);
  }
}

template <typename R>
__global__ void mul_complex_kernel(void* psi, long n, long vol, const double* fld) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    cplx<R> a = ld<R>(psi, i);
    double2 f = reinterpret_cast<const double2*>(fld)[i % vol];
    cplx<R> w{(R)f.x, (R)f.y};
    st<R>(psi, i, cmul(w, a));
  }
}

// fld <- lat (interleaved), then after the transforms fld = (fld + 1) / V.
__global__ void copy_kernel(double* dst, const double* src, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) dst[i] = src[i];
}
__global__ void plus_one_div_vol_kernel(double* fld, long vol) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < vol; i += (long)gridDim.x * blockDim.x) {
    double re = fld[2 * i] + 1.0;
    fld[2 * i] = re / vol;
    fld[2 * i + 1] = fld[2 * i + 1] / vol;
  }
}

}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_fft3d(nrcps_context* ctx, void* data, int batch, const int dims[3],
                                    nrcps_precision prec, int sign) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, (data || batch == 0) && dims && batch >= 0 && (sign == 1 || sign == -1),
                "nrcps_fft3d: bad arguments");
  NRCPS_TRY(check_dims(ctx, dims));
  if (batch == 0) return NRCPS_OK;
  return fft3d_any(ctx, data, batch, dims, prec, sign);
}

extern "C" nrcps_status nrcps_kinetic_evolve(nrcps_context* ctx, void* psi, int batch, long vol,
                                             const double* dev_xi, nrcps_precision prec) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, (psi || batch == 0) && dev_xi && batch >= 0 && vol > 0, "nrcps_kinetic_evolve: bad arguments");
  long n = vol * batch;
  if (n == 0) return NRCPS_OK;
  unsigned grid = grid_for(n, 256, (long)ctx->sm_count * 8);
  if (prec == NRCPS_F64) div_real_kernel<double><<<grid, 256, 0, ctx->stream>>>(psi, n, vol, dev_xi);
  else div_real_kernel<float><<<grid, 256, 0, ctx->stream>>>(psi, n, vol, dev_xi);
  ctx->launches++;
  return check_launch(ctx, "div_real_kernel");
}

extern "C" nrcps_status nrcps_potential_evolve(nrcps_context* ctx, void* psi, int batch, const int dims[3],
                                               const double* dev_pot, nrcps_precision prec) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, (psi || batch == 0) && dev_pot && dims && batch >= 0, "nrcps_potential_evolve: bad arguments");
  NRCPS_TRY(check_dims(ctx, dims));
  long vol = vol_of(dims), n = vol * batch;
  if (n == 0) return NRCPS_OK;
  NRCPS_TRY(fft3d_any(ctx, psi, batch, dims, prec, -1));
  unsigned grid = grid_for(n, 256, (long)ctx->sm_count * 8);
  if (prec == NRCPS_F64) mul_real_kernel<double><<<grid, 256, 0, ctx->stream>>>(psi, n, vol, dev_pot);
  else mul_real_kernel<float><<<grid, 256, 0, ctx->stream>>>(psi, n, vol, dev_pot);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "mul_real_kernel"));
  return fft3d_any(ctx, psi, batch, dims, prec, +1);
}

extern "C" nrcps_status nrcps_interaction_evolve(nrcps_context* ctx, void* psi, int batch, const int dims[3],
                                                 const double* dev_fld, nrcps_precision prec) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, (psi || batch == 0) && dev_fld && dims && batch >= 0, "nrcps_interaction_evolve: bad arguments");
  NRCPS_TRY(check_dims(ctx, dims));
  long vol = vol_of(dims), n = vol * batch;
  if (n == 0) return NRCPS_OK;
  NRCPS_TRY(fft3d_any(ctx, psi, batch, dims, prec, -1));
  unsigned grid = grid_for(n, 256, (long)ctx->sm_count * 8);
  if (prec == NRCPS_F64) mul_complex_kernel<double><<<grid, 256, 0, ctx->stream>>>(psi, n, vol, dev_fld);
  else mul_complex_kernel<float><<<grid, 256, 0, ctx->stream>>>(psi, n, vol, dev_fld);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "mul_complex_kernel"));
  return fft3d_any(ctx, psi, batch, dims, prec, +1);
}

extern "C" nrcps_status nrcps_interaction_initialize(nrcps_context* ctx, const double* dev_lat,
                                                     const double* dev_itab, const int dims[3],
                                                     double* dev_fld) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, dev_lat && dev_itab && dev_fld && dims, "nrcps_interaction_initialize: bad arguments");
  NRCPS_TRY(check_dims(ctx, dims));
  long vol = vol_of(dims);
  unsigned grid = grid_for(2 * vol, 256, (long)ctx->sm_count * 8);
  copy_kernel<<<grid, 256, 0, ctx->stream>>>(dev_fld, dev_lat, 2 * vol);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "copy_kernel"));
  NRCPS_TRY(fft3d_t<double>(ctx, dev_fld, 1, dims, +1));
  mul_real_kernel<double><<<grid_for(vol, 256), 256, 0, ctx->stream>>>(dev_fld, vol, vol, dev_itab);
  ctx->launches++;
  NRCPS_TRY(check_launch(ctx, "mul_real_kernel"));
  NRCPS_TRY(fft3d_t<double>(ctx, dev_fld, 1, dims, -1));
  plus_one_div_vol_kernel<<<grid_for(vol, 256), 256, 0, ctx->stream>>>(dev_fld, vol);
  ctx->launches++;
  return check_launch(ctx, "plus_one_div_vol_kernel");
}

namespace nrcps {
bool fused_supported(nrcps_precision prec, const int d[3]);
nrcps_status fused_step(nrcps_context* ctx, void* psi, int batch, int nconf, const int d[3], const void* kin_table,
                        nrcps_precision prec, const nrcps_position_factor* w, int cluster, const void* zpos);

// The per-site weights of a Z2 field times a position factor P:
// (1 + a) P/V and (1 - a) P/V, each split (hi, lo) into floats (float4 per
// site) for FP32 orbitals, plain doubles (double2 per site) for FP64.
__global__ void zpos_table_kernel(void* tab, const double* pos, double w_plus, double w_minus, long n, int f32) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double p = pos[i];
    const double wp = w_plus * p, wm = w_minus * p;
    if (f32) {
      const float hp = (float)wp, hm = (float)wm;
      reinterpret_cast<float4*>(tab)[i] = make_float4(hp, (float)(wp - (double)hp), hm, (float)(wm - (double)hm));
    } else {
      reinterpret_cast<double2*>(tab)[i] = make_double2(wp, wm);
    }
  }
}

// k -> (hi, lo) float pairs with hi + lo = k to ~1e-15.
__global__ void split_f32_kernel(float2* dst, const double* src, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float hi = (float)src[i];
    dst[i] = make_float2(hi, (float)(src[i] - (double)hi));
  }
}

template <typename R>
static nrcps_status propagate_t(nrcps_context* ctx, void* psi, int batch, int nconf, const int d[3],
                                const double* kin, const FieldArgs& f) {
  const int tot = batch * nconf;
  FieldArgs none{};
  NRCPS_TRY((launch_axis<R, -1, OP_PRE_MUL>(ctx, psi, tot, d, 2, kin, none)));
  NRCPS_TRY((launch_axis<R, -1, OP_NONE>(ctx, psi, tot, d, 1, nullptr, none)));
  NRCPS_TRY((launch_axis<R, -1, OP_MID_FIELD>(ctx, psi, tot, d, 0, nullptr, f)));
  NRCPS_TRY((launch_axis<R, +1, OP_NONE>(ctx, psi, tot, d, 1, nullptr, none)));
  NRCPS_TRY((launch_axis<R, +1, OP_POST_MUL>(ctx, psi, tot, d, 2, kin, none)));
  return NRCPS_OK;
}
}  // namespace nrcps

namespace nrcps {
// Propagator step for the ensemble and the C ABI.  kin_f32 may be NULL (then
// an FP32 copy of kin is made in the context when the FP32 fused kernel runs);
// so may zpos, the Z2-times-position-factor weights (zpos_table_kernel), which
// the fused kernel reads for a Z2 field with a position factor: then they are
// made in the context.
nrcps_status propagate_impl(nrcps_context* ctx, void* psi, int batch, int nconf, const int d[3], const double* kin,
                            const float2* kin_f32, const nrcps_position_factor* w, nrcps_precision prec,
                            const void* zpos) {
  if (ctx->fused_enabled && fused_supported(prec, d)) {
    const void* table = kin;
    if (prec == NRCPS_F32) {
      if (!kin_f32) {
        const long V = vol_of(d);
        if (ctx->kin_f32_len < V) {
          if (ctx->kin_f32) cudaFree(ctx->kin_f32);
          ctx->kin_f32 = nullptr;
          ctx->kin_f32_len = 0;
          NRCPS_TRY(check_cuda(ctx, cudaMalloc((void**)&ctx->kin_f32, sizeof(float2) * V), "cudaMalloc(kin f32)"));
          ctx->kin_f32_len = V;
        }
        split_f32_kernel<<<grid_for(V, 256), 256, 0, ctx->stream>>>(ctx->kin_f32, kin, V);
        ctx->launches++;
        NRCPS_TRY(check_launch(ctx, "split_f32_kernel"));
        kin_f32 = ctx->kin_f32;
      }
      table = kin_f32;
    }
    if (w->field_mode == 1 && w->dev_pos && !zpos && ctx->fused_zpos) {
      const long V = vol_of(d);
      if (ctx->zpos_len < 16 * V) {
        if (ctx->zpos) cudaFree(ctx->zpos);
        ctx->zpos = nullptr;
        ctx->zpos_len = 0;
        NRCPS_TRY(check_cuda(ctx, cudaMalloc(&ctx->zpos, 16 * V), "cudaMalloc(Z2 position weights)"));
        ctx->zpos_len = 16 * V;
      }
      zpos_table_kernel<<<grid_for(V, 256), 256, 0, ctx->stream>>>(ctx->zpos, w->dev_pos, (1.0 + w->a) / (double)V,
                                                                   (1.0 - w->a) / (double)V, V, prec == NRCPS_F32);
      ctx->launches++;
      NRCPS_TRY(check_launch(ctx, "zpos_table_kernel"));
      zpos = ctx->zpos;
    }
    nrcps_status st = fused_step(ctx, psi, batch, nconf, d, table, prec, w, ctx->fused_cluster, zpos);
    if (st != NRCPS_ERR_UNSUPPORTED) return st;
  }
  FieldArgs f;
  f.mode = w->field_mode;
  f.field = w->dev_field;
  f.bit0 = w->bit0;
  f.conf_stride = w->conf_stride;
  f.conf_base = w->dev_conf_base;
  f.a = w->a;
  f.vol = (double)vol_of(d);
  f.pos = w->dev_pos;
  f.orbs_per_conf = batch;
  return prec == NRCPS_F64 ? propagate_t<double>(ctx, psi, batch, nconf, d, kin, f)
                           : propagate_t<float>(ctx, psi, batch, nconf, d, kin, f);
}
}  // namespace nrcps

// Fused Propagator::Run; dev_kin holds k = 1/xi.
extern "C" nrcps_status nrcps_propagate(nrcps_context* ctx, void* psi, int batch, int nconf, const int dims[3],
                                       const double* dev_kin, const nrcps_position_factor* w,
                                       nrcps_precision prec) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, (psi || nconf == 0) && dims && dev_kin && w && w->dev_field && batch > 0 && nconf >= 0,
                "nrcps_propagate: bad arguments");
  NRCPS_REQUIRE(ctx, w->field_mode >= 0 && w->field_mode <= 3, "nrcps_propagate: bad field_mode");
  NRCPS_REQUIRE(ctx, w->field_mode != 3 || !w->dev_pos, "nrcps_propagate: field_mode 3 carries the whole factor");
  NRCPS_TRY(check_dims(ctx, dims));
  if (nconf == 0) return NRCPS_OK;
  return propagate_impl(ctx, psi, batch, nconf, dims, dev_kin, nullptr, w, prec, nullptr);
}

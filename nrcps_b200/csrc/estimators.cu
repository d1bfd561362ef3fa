// estimators.cu -- ensemble accumulators, cumulant (log-det moment) sums and
// jackknife errors in FP64 on the device.
//
// Accumulation follows the production drivers per block of configurations:
//   production/slater_det/main.C:208-211           corr[n][t] += |det S_{n+1}(t)|^2
//   production/slater_det2_trapped/main-no_cum.C:205-207  corr[m][t] += det
//   production/slater_det2_trapped/main-cum.C:219-233     z[k][m][t] += (log|det|)^(k+1), k < Nc
// with configurations added one after another in index order, as the host
// loop of the reference adds them.
#include <math.h>

#include "common.cuh"

namespace nrcps {

// One thread per (measured minor m, slice t); the configuration loop is
// sequential so the sums have the reference's order.
__global__ void accumulate_kernel(const double* __restrict__ dets, int n_conf, int T, int nmeas, int mode, int nc,
                                  double* __restrict__ corr, double* __restrict__ z) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;  // m + nmeas * t (coalesced over m)
  if (e >= T * nmeas) return;
  const int m = e % nmeas, t = e / nmeas;
  double cr = 0.0, ci = 0.0;
  double zs[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) zs[k] = 0.0;
  for (int c = 0; c < n_conf; ++c) {
    const double2 d = reinterpret_cast<const double2*>(dets)[((long)c * T + t) * nmeas + m];
    // explicitly rounded products and sums (no fused multiply-add): the
    // reference's arithmetic to the bit
    if (mode == 0) {
      // tmp * conj(tmp) (main.C:210): real part re*re + im*im
      cr = __dadd_rn(cr, __dadd_rn(__dmul_rn(d.x, d.x), __dmul_rn(d.y, d.y)));
    } else {
      cr = __dadd_rn(cr, d.x);
      ci = __dadd_rn(ci, d.y);
    }
    if (nc > 0) {
      const double l = log(hypot(d.x, d.y));  // cum[0] = log(abs(slat)) (main-cum.C:221)
      double p = l;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (k < nc) {
          zs[k] = __dadd_rn(zs[k], p);
          p = __dmul_rn(p, l);  // cum[nc] = cum[0] * cum[nc-1]
        }
      }
    }
  }
  // corr[m][t] (row per measured minor, as the result files)
  corr[2L * (m * (long)T + t)] = cr;
  corr[2L * (m * (long)T + t) + 1] = ci;
  for (int k = 0; k < nc && k < 8; ++k) z[((long)k * nmeas + m) * T + t] = zs[k];
}

// Binned jackknife of the means of n_obs observables over n samples
// (x[s][j], row-major): bins of floor(n / n_bins) consecutive samples (the
// remainder is dropped, as usual for blocked jackknife).  mean[j] over the
// binned samples; err[j] = sqrt((nb-1)/nb sum_b (mean_{-b} - mean)^2).
// When eff != 0 the observables are consecutive slices of one correlator
// and effective-energy estimates E(t) = log(C(t) / C(t+1)) are also formed,
// their errors from the same leave-one-bin-out means.
__global__ void jackknife_kernel(const double* __restrict__ x, long n, int n_obs, int n_bins, double* __restrict__ mean,
                                 double* __restrict__ err, double* __restrict__ eff_mean, double* __restrict__ eff_err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_obs) return;
  const long per = n / n_bins;
  const long used = per * n_bins;
  double tot = 0.0, tot2 = 0.0;
  const bool eff = eff_mean != nullptr && j + 1 < n_obs;
  for (long s = 0; s < used; ++s) {
    tot += x[s * n_obs + j];
    if (eff) tot2 += x[s * n_obs + j + 1];
  }
  const double mu = tot / (double)used;
  double acc = 0.0, acc_e = 0.0;
  const double e0 = eff ? log(tot / tot2) : 0.0;
  for (int b = 0; b < n_bins; ++b) {
    double bs = 0.0, bs2 = 0.0;
    for (long s = b * per; s < (b + 1) * per; ++s) {
      bs += x[s * n_obs + j];
      if (eff) bs2 += x[s * n_obs + j + 1];
    }
    const double mb = (tot - bs) / (double)(used - per);
    acc += (mb - mu) * (mb - mu);
    if (eff) {
      const double eb = log((tot - bs) / (tot2 - bs2));
      acc_e += (eb - e0) * (eb - e0);
    }
  }
  const double f = (double)(n_bins - 1) / (double)n_bins;
  mean[j] = mu;
  err[j] = sqrt(f * acc);
  if (eff_mean && j + 1 < n_obs) {
    eff_mean[j] = e0;
    eff_err[j] = sqrt(f * acc_e);
  }
}

}  // namespace nrcps

using namespace nrcps;

extern "C" nrcps_status nrcps_accumulate(nrcps_context* ctx, const double* dev_dets, int n_conf, int T, int nmeas,
                                         int mode, int n_cumulants, double* dev_corr, double* dev_z) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, (dev_dets || n_conf == 0) && dev_corr && n_conf >= 0 && T > 0 && nmeas > 0 &&
                         (mode == 0 || mode == 1),
                "nrcps_accumulate: bad arguments");
  NRCPS_REQUIRE(ctx, n_cumulants >= 0 && n_cumulants <= 8 && (n_cumulants == 0 || dev_z),
                "nrcps_accumulate: 0 <= n_cumulants <= 8 (z required when > 0)");
  const int total = T * nmeas;
  accumulate_kernel<<<(total + 127) / 128, 128, 0, ctx->stream>>>(dev_dets, n_conf, T, nmeas, mode, n_cumulants,
                                                                  dev_corr, dev_z);
  ctx->launches++;
  return check_launch(ctx, "accumulate_kernel");
}

extern "C" nrcps_status nrcps_jackknife(nrcps_context* ctx, const double* dev_x, long n_samples, int n_obs,
                                        int n_bins, double* dev_mean, double* dev_err, double* dev_eff_mean,
                                        double* dev_eff_err) {
  if (!ctx) return NRCPS_ERR_INVALID_ARGUMENT;
  NRCPS_REQUIRE(ctx, dev_x && dev_mean && dev_err && n_obs > 0 && n_bins >= 2 && n_samples >= n_bins,
                "nrcps_jackknife: bad arguments (need n_bins >= 2 and n_samples >= n_bins)");
  NRCPS_REQUIRE(ctx, (dev_eff_mean == nullptr) == (dev_eff_err == nullptr),
                "nrcps_jackknife: effective-energy outputs come in pairs");
  jackknife_kernel<<<(n_obs + 127) / 128, 128, 0, ctx->stream>>>(dev_x, n_samples, n_obs, n_bins, dev_mean, dev_err,
                                                                 dev_eff_mean, dev_eff_err);
  ctx->launches++;
  return check_launch(ctx, "jackknife_kernel");
}

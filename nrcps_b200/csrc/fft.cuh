// fft.cuh -- register-resident DFTs of compile-time length for 3-D lattice FFTs.
//
// A pencil of N complex values lives in one thread's registers; the
// transform is a fully unrolled mixed-radix (4, 2, 3) decimation-in-time
// Cooley-Tukey.  Twiddles W_N^k = exp(SIGN * 2*pi*i * k / N) are
// compile-time constants: every loop index that reaches a twiddle is a
// template parameter (static_for), and the constants come from a constexpr
// sine/cosine written here from their Taylor series after exact octant
// reduction of the rational angle k/N (no runtime math library involved).
// Conventions match FFTW's (src/fourier/noarch/fourier.C:34-35 of the
// reference): SIGN = -1 is FFTW_FORWARD, +1 FFTW_BACKWARD, unnormalised.
#pragma once

#include <utility>

#include "common.cuh"

namespace nrcps {
namespace fft {

// ------------------------------------------------------------- static_for
template <typename F, int... Is>
__host__ __device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// --------------------------------------------------- constexpr sin / cos
// sin and cos of phi in [0, pi/4] by Taylor series (terms to phi^27, below
// 1e-30 relative), evaluated in double at compile time.
constexpr double taylor_sin(double x) {
  double term = x, sum = x;
  for (int n = 1; n < 14; ++n) {
    term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double taylor_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 14; ++n) {
    term *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
    sum += term;
  }
  return sum;
}
constexpr double kHalfPi = 1.57079632679489661923132169163975144;

// cos and sin of 2*pi*k/n for integers k, n > 0, reduced exactly to the
// first octant with integer arithmetic.
struct CS {
  double c, s;
};
constexpr CS unit_root(long k, long n) {
  long kk = ((k % n) + n) % n;
  long q = (4 * kk) / n;        // quadrant
  long r = 4 * kk - q * n;      // angle within quadrant = (pi/2) * r / n
  double c = 0, s = 0;
  if (2 * r <= n) {
    double phi = kHalfPi * (double)r / (double)n;
    c = taylor_cos(phi);
    s = taylor_sin(phi);
  } else {
    double phi = kHalfPi * (double)(n - r) / (double)n;
    c = taylor_sin(phi);
    s = taylor_cos(phi);
  }
  // rotate by q quarter turns
  for (long i = 0; i < q; ++i) {
    double t = c;
    c = -s;
    s = t;
  }
  return CS{c, s};
}

// x * W_N^K with W_N = exp(SIGN 2 pi i / N); exact for multiples of N/4.
template <int N, int K, int SIGN, typename R>
__device__ __forceinline__ cplx<R> twiddle(cplx<R> x) {
  constexpr int k = ((K % N) + N) % N;
  if constexpr (k == 0) {
    return x;
  } else if constexpr ((4 * k) % N == 0) {
    constexpr int q = (4 * k) / N;  // quarter turns of exp(+2 pi i k/N)
    constexpr int qs = SIGN > 0 ? q : (4 - q) % 4;
    if constexpr (qs == 1) return cplx<R>{-x.im, x.re};
    else if constexpr (qs == 2) return cplx<R>{-x.re, -x.im};
    else return cplx<R>{x.im, -x.re};
  } else if constexpr (sizeof(R) == 4 && (8 * k) % N == 0) {
    // an odd multiple of pi/4: |cos| = |sin| = m, so
    // x w = m (cs x.re - ss x.im) + i m (ss x.re + cs x.im) with the signs
    // cs, ss of cos and sin: two adds and two products by m = hi + lo
    constexpr CS w = unit_root(k, N);
    constexpr double sd = SIGN > 0 ? w.s : -w.s;
    constexpr double m = w.c > 0 ? w.c : -w.c;
    constexpr float mh = (float)m, ml = (float)(m - (double)(float)m);
    constexpr float cs = w.c > 0 ? 1.f : -1.f, ss = sd > 0 ? 1.f : -1.f;
    const float a = cs * x.re - ss * x.im;
    const float b = ss * x.re + cs * x.im;
    return cplx<R>{fmaf(a, mh, a * ml), fmaf(b, mh, b * ml)};
  } else {
    if constexpr (sizeof(R) == 4) {
      // The root carried as an unevaluated float pair hi + lo (exact to
      // ~1e-15): a single-float root is off by up to half an ulp in phase
      // and modulus, the same error at every step, and drives a systematic
      // drift of |det|^2 (~2e-6 per step at L = 32, N = 19).  The small
      // terms are added first, the hi products last.
      constexpr CS w = unit_root(k, N);
      constexpr double sd = SIGN > 0 ? w.s : -w.s;
      constexpr float ch = (float)w.c, cl = (float)(w.c - (double)(float)w.c);
      constexpr float sh = (float)sd, sl = (float)(sd - (double)(float)sd);
      const float re = fmaf(x.re, ch, fmaf(-x.im, sh, fmaf(x.re, cl, -x.im * sl)));
      const float im = fmaf(x.re, sh, fmaf(x.im, ch, fmaf(x.re, sl, x.im * cl)));
      return cplx<R>{re, im};
    } else {
      constexpr CS w = unit_root(k, N);
      constexpr R c = (R)w.c;
      constexpr R s = (R)(SIGN > 0 ? w.s : -w.s);
      return cplx<R>{x.re * c - x.im * s, x.re * s + x.im * c};
    }
  }
}

template <int SIGN, typename R>
__device__ __forceinline__ cplx<R> mul_i(cplx<R> z) {  // SIGN * i * z
  if constexpr (SIGN > 0) return cplx<R>{-z.im, z.re};
  else return cplx<R>{z.im, -z.re};
}

template <typename R>
__device__ __forceinline__ cplx<R> add(cplx<R> a, cplx<R> b) { return cplx<R>{a.re + b.re, a.im + b.im}; }
template <typename R>
__device__ __forceinline__ cplx<R> sub(cplx<R> a, cplx<R> b) { return cplx<R>{a.re - b.re, a.im - b.im}; }

// ------------------------------------------------------------ butterflies
template <int P, int SIGN, typename R>
struct Butterfly;

template <int SIGN, typename R>
struct Butterfly<2, SIGN, R> {
  static __device__ __forceinline__ void run(cplx<R>* t) {
    cplx<R> a = t[0], b = t[1];
    t[0] = add(a, b);
    t[1] = sub(a, b);
  }
};

template <int SIGN, typename R>
struct Butterfly<4, SIGN, R> {
  static __device__ __forceinline__ void run(cplx<R>* t) {
    cplx<R> s02 = add(t[0], t[2]), d02 = sub(t[0], t[2]);
    cplx<R> s13 = add(t[1], t[3]), d13 = mul_i<SIGN>(sub(t[1], t[3]));
    t[0] = add(s02, s13);
    t[2] = sub(s02, s13);
    t[1] = add(d02, d13);
    t[3] = sub(d02, d13);
  }
};

template <int SIGN, typename R>
struct Butterfly<3, SIGN, R> {
  static __device__ __forceinline__ void run(cplx<R>* t) {
    constexpr R c = (R)-0.5;
    // sin(2 pi / 3), in FP32 as hi + lo (see twiddle())
    constexpr double sd = 0.86602540378443864676372317075293618;
    constexpr R sh = (R)sd;
    constexpr R sl = (R)(sd - (double)(R)sd);
    cplx<R> u = add(t[1], t[2]);
    cplx<R> v = sub(t[1], t[2]);
    cplx<R> m{t[0].re + c * u.re, t[0].im + c * u.im};
    cplx<R> sv;
    if constexpr (sizeof(R) == 4) sv = cplx<R>{fmaf(v.re, sh, v.re * sl), fmaf(v.im, sh, v.im * sl)};
    else sv = cplx<R>{sh * v.re, sh * v.im};
    cplx<R> iv = mul_i<SIGN>(sv);
    t[0] = add(t[0], u);
    t[1] = add(m, iv);
    t[2] = sub(m, iv);
  }
};

template <int N>
struct Radix {
  static constexpr int value = (N % 4 == 0) ? 4 : (N % 2 == 0 ? 2 : (N % 3 == 0 ? 3 : N));
};

// ------------------------------------------------------------------- DFT
// In-place DFT of x[0..N) (natural order in and out).
template <int N, int SIGN, typename R>
struct Dft {
  static_assert(N == 1 || Radix<N>::value <= 4, "only lengths 2^a 3^b are supported");
  static __device__ __forceinline__ void run(cplx<R>* x) {
    constexpr int P = Radix<N>::value;
    constexpr int M = N / P;
    if constexpr (N == 1) {
      return;
    } else if constexpr (M == 1) {
      Butterfly<P, SIGN, R>::run(x);
    } else {
      cplx<R> s[P][M];
#pragma unroll
      for (int q = 0; q < P; ++q)
#pragma unroll
        for (int j = 0; j < M; ++j) s[q][j] = x[j * P + q];
#pragma unroll
      for (int q = 0; q < P; ++q) Dft<M, SIGN, R>::run(s[q]);
      static_for<M>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        cplx<R> t[P];
        static_for<P>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          t[q] = twiddle<N, q * k, SIGN, R>(s[q][k]);
        });
        Butterfly<P, SIGN, R>::run(t);
#pragma unroll
        for (int ss = 0; ss < P; ++ss) x[k + ss * M] = t[ss];
      });
    }
  }
};

// ------------------------------------------- packed FP32x2 transforms
// Two independent complex sequences carried in the two lanes of float2
// registers (re = (re_0, re_1), im = (im_0, im_1)), so that every butterfly
// add and every twiddle product is one sm_100 packed instruction
// (FADD2 / FMUL2 / FFMA2) for both sequences.  The structure and the
// constants are those of Dft above; only the issue count changes.
struct cpk {
  float2 re, im;
};

__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b with one rounding: b * (-1) is exact inside the fused multiply-add
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ cpk padd(cpk a, cpk b) { return cpk{padd(a.re, b.re), padd(a.im, b.im)}; }
__device__ __forceinline__ cpk psub(cpk a, cpk b) { return cpk{psub(a.re, b.re), psub(a.im, b.im)}; }

// x * W_N^K (lane-uniform twiddle)
template <int N, int K, int SIGN>
__device__ __forceinline__ cpk ptwiddle(cpk x) {
  constexpr int k = ((K % N) + N) % N;
  if constexpr (k == 0) {
    return x;
  } else if constexpr ((4 * k) % N == 0) {
    constexpr int q = (4 * k) / N;
    constexpr int qs = SIGN > 0 ? q : (4 - q) % 4;
    const float2 z = make_float2(0.f, 0.f);
    if constexpr (qs == 1) return cpk{psub(z, x.im), x.re};
    else if constexpr (qs == 2) return cpk{psub(z, x.re), psub(z, x.im)};
    else return cpk{x.im, psub(z, x.re)};
  } else if constexpr ((8 * k) % N == 0) {
    // odd multiple of pi/4 as in twiddle() above, with the sign cs of the
    // cosine folded into m: re = (cs m)(x.re - cs ss x.im), im = (cs m)(x.im + cs ss x.re)
    constexpr CS w = unit_root(k, N);
    constexpr double sd = SIGN > 0 ? w.s : -w.s;
    constexpr double cm = w.c;  // cs m
    constexpr float mh = (float)cm, ml = (float)(cm - (double)(float)cm);
    constexpr float t = (w.c > 0) == (sd > 0) ? 1.f : -1.f;  // cs ss
    const float2 a = __ffma2_rn(x.im, make_float2(-t, -t), x.re);
    const float2 b = __ffma2_rn(x.re, make_float2(t, t), x.im);
    const float2 u = __ffma2_rn(a, make_float2(mh, mh), __fmul2_rn(a, make_float2(ml, ml)));
    const float2 v = __ffma2_rn(b, make_float2(mh, mh), __fmul2_rn(b, make_float2(ml, ml)));
    return cpk{u, v};
  } else {
    // hi + lo root as in twiddle() above
    constexpr CS w = unit_root(k, N);
    constexpr double sd = SIGN > 0 ? w.s : -w.s;
    constexpr float ch = (float)w.c, cl = (float)(w.c - (double)(float)w.c);
    constexpr float sh = (float)sd, sl = (float)(sd - (double)(float)sd);
    float2 u = __fmul2_rn(x.im, make_float2(-sl, -sl));
    u = __ffma2_rn(x.re, make_float2(cl, cl), u);
    u = __ffma2_rn(x.im, make_float2(-sh, -sh), u);
    u = __ffma2_rn(x.re, make_float2(ch, ch), u);
    float2 v = __fmul2_rn(x.im, make_float2(cl, cl));
    v = __ffma2_rn(x.re, make_float2(sl, sl), v);
    v = __ffma2_rn(x.im, make_float2(ch, ch), v);
    v = __ffma2_rn(x.re, make_float2(sh, sh), v);
    return cpk{u, v};
  }
}

template <int P, int SIGN>
struct PButterfly;

template <int SIGN>
struct PButterfly<2, SIGN> {
  static __device__ __forceinline__ void run(cpk* t) {
    cpk a = t[0], b = t[1];
    t[0] = padd(a, b);
    t[1] = psub(a, b);
  }
};

template <int SIGN>
struct PButterfly<4, SIGN> {
  static __device__ __forceinline__ void run(cpk* t) {
    cpk s02 = padd(t[0], t[2]), d02 = psub(t[0], t[2]);
    cpk s13 = padd(t[1], t[3]), d = psub(t[1], t[3]);
    t[0] = padd(s02, s13);
    t[2] = psub(s02, s13);
    // d02 +- SIGN i d, with the multiplication by i folded into the adds
    if constexpr (SIGN > 0) {
      t[1] = cpk{psub(d02.re, d.im), padd(d02.im, d.re)};
      t[3] = cpk{padd(d02.re, d.im), psub(d02.im, d.re)};
    } else {
      t[1] = cpk{padd(d02.re, d.im), psub(d02.im, d.re)};
      t[3] = cpk{psub(d02.re, d.im), padd(d02.im, d.re)};
    }
  }
};

template <int SIGN>
struct PButterfly<3, SIGN> {
  static __device__ __forceinline__ void run(cpk* t) {
    constexpr float c = -0.5f;
    constexpr double sd = 0.86602540378443864676372317075293618;
    constexpr float sh = (float)sd, sl = (float)(sd - (double)(float)sd);
    cpk u = padd(t[1], t[2]);
    cpk v = psub(t[1], t[2]);
    cpk m{__ffma2_rn(u.re, make_float2(c, c), t[0].re), __ffma2_rn(u.im, make_float2(c, c), t[0].im)};
    cpk sv{__ffma2_rn(v.re, make_float2(sh, sh), __fmul2_rn(v.re, make_float2(sl, sl))),
           __ffma2_rn(v.im, make_float2(sh, sh), __fmul2_rn(v.im, make_float2(sl, sl)))};
    t[0] = padd(t[0], u);
    if constexpr (SIGN > 0) {  // m +- i sv
      t[1] = cpk{psub(m.re, sv.im), padd(m.im, sv.re)};
      t[2] = cpk{padd(m.re, sv.im), psub(m.im, sv.re)};
    } else {
      t[1] = cpk{padd(m.re, sv.im), psub(m.im, sv.re)};
      t[2] = cpk{psub(m.re, sv.im), padd(m.im, sv.re)};
    }
  }
};

// In-place DFT of two sequences at once (natural order in and out).
template <int N, int SIGN>
struct PDft {
  static __device__ __forceinline__ void run(cpk* x) {
    constexpr int P = Radix<N>::value;
    constexpr int M = N / P;
    if constexpr (N == 1) {
      return;
    } else if constexpr (M == 1) {
      PButterfly<P, SIGN>::run(x);
    } else {
      cpk s[P][M];
#pragma unroll
      for (int q = 0; q < P; ++q)
#pragma unroll
        for (int j = 0; j < M; ++j) s[q][j] = x[j * P + q];
#pragma unroll
      for (int q = 0; q < P; ++q) PDft<M, SIGN>::run(s[q]);
      static_for<M>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        cpk t[P];
        static_for<P>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          t[q] = ptwiddle<N, q * k, SIGN>(s[q][k]);
        });
        PButterfly<P, SIGN>::run(t);
#pragma unroll
        for (int ss = 0; ss < P; ++ss) x[k + ss * M] = t[ss];
      });
    }
  }
};

// Length-N DFT of one FP32 pencil (N even) through the packed half-length
// transform.  Decimation in time: the even and odd subsequences ride in the
// two lanes of one length-N/2 packed DFT, then one scalar radix-2 stage
// X[k] = E[k] + W^k O[k], X[k + N/2] = E[k] - W^k O[k].
template <int N, int SIGN>
__device__ __forceinline__ void dft_packed(cplx<float>* x) {
  constexpr int H = N / 2;
  cpk e[H];
#pragma unroll
  for (int m = 0; m < H; ++m) {
    e[m].re = make_float2(x[2 * m].re, x[2 * m + 1].re);
    e[m].im = make_float2(x[2 * m].im, x[2 * m + 1].im);
  }
  PDft<H, SIGN>::run(e);
  static_for<H>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    const cplx<float> E{e[k].re.x, e[k].im.x};
    const cplx<float> t = twiddle<N, k, SIGN, float>(cplx<float>{e[k].re.y, e[k].im.y});
    x[k] = cplx<float>{E.re + t.re, E.im + t.im};
    x[k + H] = cplx<float>{E.re - t.re, E.im - t.im};
  });
}

// Dispatch: the packed transform for FP32 pencils of even length when PK.
template <int N, int SIGN, typename R, bool PK>
__device__ __forceinline__ void dft(cplx<R>* x) {
  if constexpr (PK && sizeof(R) == 4 && N % 2 == 0 && N >= 4) dft_packed<N, SIGN>(reinterpret_cast<cplx<float>*>(x));
  else Dft<N, SIGN, R>::run(x);
}

// x * (hi + lo) on both components at once, as mul2: fma(x, hi, x lo).
__device__ __forceinline__ cplx<float> scale2_packed(cplx<float> x, float hi, float lo) {
  const float2 v = make_float2(x.re, x.im);
  const float2 g = __fmul2_rn(v, make_float2(lo, lo));
  const float2 r = __ffma2_rn(v, make_float2(hi, hi), g);
  return cplx<float>{r.x, r.y};
}

// -------------------------------------------------- pencils split over lanes
// A pencil of N values held by two lanes (lane and lane ^ 16), h = 0 / 1.
//
// dft_split_dit: on entry lane h holds x[2m + h] (m < N/2) in v[m]; on exit
// it holds X[h N/2 + k] in v[k].  Decimation in time: a length-N/2 DFT per
// lane, the odd half times W_N^k, then one radix-2 stage whose partner
// values come through one warp shuffle per real.
//
// dft_split_dif: on entry lane h holds X[h N/2 + k]; on exit x[2m + h].
// Decimation in frequency: the radix-2 stage first (a = X[k] + X[k+N/2] on
// lane 0, b = (X[k] - X[k+N/2]) W_N^k on lane 1), then the half-length DFT.
//
// Both are branch-free: per-lane choices are selects, so the warp never
// diverges.
template <int N, int SIGN, typename R>
__device__ __forceinline__ void dft_split_dit(cplx<R>* v, int h) {
  constexpr int H = N / 2;
  Dft<H, SIGN, R>::run(v);
  static_for<H>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    cplx<R> t = twiddle<N, k, SIGN, R>(v[k]);
    v[k] = h ? t : v[k];
  });
  const R sg = h ? (R)-1 : (R)1;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    cplx<R> o{__shfl_xor_sync(0xffffffffu, v[k].re, 16), __shfl_xor_sync(0xffffffffu, v[k].im, 16)};
    v[k] = cplx<R>{o.re + sg * v[k].re, o.im + sg * v[k].im};
  }
}

template <int N, int SIGN, typename R>
__device__ __forceinline__ void dft_split_dif(cplx<R>* v, int h) {
  constexpr int H = N / 2;
  const R sg = h ? (R)-1 : (R)1;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    cplx<R> o{__shfl_xor_sync(0xffffffffu, v[k].re, 16), __shfl_xor_sync(0xffffffffu, v[k].im, 16)};
    v[k] = cplx<R>{o.re + sg * v[k].re, o.im + sg * v[k].im};
  }
  static_for<H>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    cplx<R> t = twiddle<N, k, SIGN, R>(v[k]);
    v[k] = h ? t : v[k];
  });
  Dft<H, SIGN, R>::run(v);
}

}  // namespace fft
}  // namespace nrcps

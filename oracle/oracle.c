/*
 * oracle.c -- CPU restatement of nrCPS's auxiliary-field transfer-matrix path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Plain C99; double precision;
 * complex arithmetic through C's double _Complex, which GCC lowers exactly as
 * it lowers std::complex<double> in the reference (inline products, __divdc3
 * division, cabs = hypot), so the restatement agrees with the reference build
 * bit for bit.
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fft64.h"

/* include/constants.h:11-16 */
static const double K_PI = 3.1415926535897932;
static const double K_TWOPI = 6.2831853071795864;
static const double K_PISQ = 9.8696044010893586;
static const double K_PIM4 = 0.7511255444649425;
static const double K_SQRTPI = 1.7724538509055159;

/* =================================================================== RNG */

/* Ranlxs/Ranlxd seeding (src/random/ranlxs.C:60-110, src/random/ranlxd.C:61-113):
 * a 31-bit shift register fed by the seed produces 4 lanes x 24 digits. */
static void ranlux_seed(o_rng *r, long seed, int dbl) {
  int xbit[31];
  long i = seed;
  for (int k = 0; k < 31; ++k) {
    xbit[k] = (int)(i % 2);
    i /= 2;
  }
  int ibit = 0, jbit = 18;
  for (int lane = 0; lane < 4; ++lane) {
    for (int k = 0; k < 24; ++k) {
      int ix = 0;
      for (int l = 0; l < 24; ++l) {
        int iy = xbit[ibit];
        ix = 2 * ix + iy;
        xbit[ibit] = (xbit[ibit] + xbit[jbit]) % 2;
        ibit = (ibit + 1) % 31;
        jbit = (jbit + 1) % 31;
      }
      int flip = dbl ? ((k % 4) != lane) : ((k % 4) == lane);
      if (flip) ix = 16777215 - ix;
      r->num[4 * k + lane] = ix;
    }
  }
  for (int l = 0; l < 4; ++l) r->carry[l] = 0;
  r->ir = 0;
  r->jr = 7;
  r->is = dbl ? 91 : 95;
  r->is_old = 0;
  r->prm = r->pr % 12;
  for (int k = 0; k < 96; ++k) {
    r->next[k] = (k + 1) % 96;
    if (dbl && (k % 4) == 3) r->next[k] = (k + 5) % 96;
  }
}

/* Subtract-with-borrow update on 4 lanes of 48-bit words stored as two
 * 24-bit digits (src/random/ranlxs.C:14-46 STEP, :143-168 Update). */
static void ranlux_update(o_rng *r) {
  int pi = r->ir, pj = r->jr;
  for (int k = 0; k < r->pr; ++k) {
    for (int l = 0; l < 4; ++l) {
      int *lo_i = &r->num[8 * pi + l], *hi_i = &r->num[8 * pi + 4 + l];
      int lo_j = r->num[8 * pj + l], hi_j = r->num[8 * pj + 4 + l];
      int d = lo_j - *lo_i - r->carry[l];
      *hi_i += (d < 0);
      d += 0x1000000;
      *lo_i = d & 0xffffff;
      d = hi_j - *hi_i;
      r->carry[l] = (d < 0);
      d += 0x1000000;
      *hi_i = d & 0xffffff;
    }
    if (++pi == 12) pi = 0;
    if (++pj == 12) pj = 0;
  }
  r->ir += r->prm;
  r->jr += r->prm;
  if (r->ir >= 12) r->ir -= 12;
  if (r->jr >= 12) r->jr -= 12;
  r->is = 8 * r->ir;
  r->is_old = r->is;
}

/* ran2 (src/random/ran2.C:42-81), L'Ecuyer with Bays-Durham shuffle. */
#define R2_IM1 2147483563L
#define R2_IM2 2147483399L
#define R2_AM (1.0 / R2_IM1)
#define R2_IMM1 (R2_IM1 - 1)
#define R2_IA1 40014L
#define R2_IA2 40692L
#define R2_IQ1 53668L
#define R2_IQ2 52774L
#define R2_IR1 12211L
#define R2_IR2 3791L
#define R2_NTAB 32
#define R2_NDIV (1 + R2_IMM1 / R2_NTAB)
#define R2_RNMX (1.0 - 1.2e-7)

static void ran2_seed(o_rng *r, long seed) {
  r->idum = seed;
  if (r->idum <= 0) r->idum = 1;
  r->idum2 = r->idum;
  for (int j = R2_NTAB + 7; j >= 0; --j) {
    long k = r->idum / R2_IQ1;
    r->idum = R2_IA1 * (r->idum - k * R2_IQ1) - k * R2_IR1;
    if (r->idum < 0) r->idum += R2_IM1;
    if (j < R2_NTAB) r->iv[j] = r->idum;
  }
  r->iy = r->iv[0];
}

static double ran2_next(o_rng *r) {
  long k = r->idum / R2_IQ1;
  r->idum = R2_IA1 * (r->idum - k * R2_IQ1) - k * R2_IR1;
  if (r->idum < 0) r->idum += R2_IM1;
  k = r->idum2 / R2_IQ2;
  r->idum2 = R2_IA2 * (r->idum2 - k * R2_IQ2) - k * R2_IR2;
  if (r->idum2 < 0) r->idum2 += R2_IM2;
  int j = (int)(r->iy / R2_NDIV);
  r->iy = r->iv[j] - r->idum2;
  r->iv[j] = r->idum;
  if (r->iy < 1) r->iy += R2_IMM1;
  float temp = (float)(R2_AM * r->iy);
  if (temp > R2_RNMX) return R2_RNMX;
  return temp;
}

void o_rng_init(o_rng *r, int kind, long seed) {
  memset(r, 0, sizeof *r);
  r->kind = kind;
  switch (kind) {
    case O_RANLXS0: r->pr = 109; break;
    case O_RANLXS1: r->pr = 202; break;
    case O_RANLXS2: r->pr = 397; break;
    case O_RANLXD1: r->pr = 202; break;
    case O_RANLXD2: r->pr = 397; break;
    default: break;
  }
  if (kind >= O_RANLXS0) {
    r->dbl = (kind >= O_RANLXD1);
    ranlux_seed(r, seed, r->dbl);
  } else {
    ran2_seed(r, seed);
  }
}

double o_rng_uniform(o_rng *r) {
  if (r->kind < O_RANLXS0) return ran2_next(r);
  r->is = r->next[r->is];
  if (r->is == r->is_old) ranlux_update(r);
  if (r->dbl) {
    /* src/random/ranlxd.C:117-129 */
    const double ob = ldexp(1.0, -24);
    return ob * ((double)r->num[r->is + 4] + ob * (double)r->num[r->is]);
  }
  /* src/random/ranlxs.C:112-126: float product, then widened */
  const float ob = (float)ldexp(1.0, -24);
  return (double)(ob * (float)r->num[r->is]);
}

/* Random::Gauss (src/random/random.C:105-116): polar method, keeps y only. */
double o_rng_gauss(o_rng *r, double sigma) {
  double x, y, r2;
  do {
    x = 2 * o_rng_uniform(r) - 1;
    y = 2 * o_rng_uniform(r) - 1;
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0);
  return sigma * y * sqrt(-2.0 * log(r2) / r2);
}

/* Random::Z (src/random/random.C:129-132). */
int o_rng_z(o_rng *r, int p) { return (int)floor(p * o_rng_uniform(r)); }

void o_rng_get_state(const o_rng *r, long *state) {
  state[0] = 105;
  for (int k = 0; k < 96; ++k) state[k + 1] = r->num[k];
  for (int l = 0; l < 4; ++l) state[97 + l] = r->carry[l];
  state[101] = r->pr;
  state[102] = r->ir;
  state[103] = r->jr;
  state[104] = r->is;
}

void o_rng_set_state(o_rng *r, const long *state) {
  for (int k = 0; k < 96; ++k) r->num[k] = (int)state[k + 1];
  for (int l = 0; l < 4; ++l) r->carry[l] = (int)state[97 + l];
  r->pr = (int)state[101];
  r->ir = (int)state[102];
  r->jr = (int)state[103];
  r->is = (int)state[104];
  r->is_old = 8 * r->ir;
  r->prm = r->pr % 12;
}

void o_uniforms(int kind, long seed, long skip, long count, double *out) {
  o_rng r;
  o_rng_init(&r, kind, seed);
  for (long i = 0; i < skip; ++i) (void)o_rng_uniform(&r);
  for (long i = 0; i < count; ++i) out[i] = o_rng_uniform(&r);
}

void o_gaussians(int kind, long seed, long skip, long count, double *out) {
  o_rng r;
  o_rng_init(&r, kind, seed);
  for (long i = 0; i < skip; ++i) (void)o_rng_gauss(&r, 1.0);
  for (long i = 0; i < count; ++i) out[i] = o_rng_gauss(&r, 1.0);
}

/* Lattice::Refresh (src/alg/lattice.C:60-109). */
void o_field_slices(o_rng *r, int field_type, long vol, long slices, double *out) {
  for (long s = 0; s < slices; ++s) {
    double *f = out + 2 * vol * s;
    for (long i = 0; i < 2 * vol; i += 2) {
      switch (field_type) {
        case O_FIELD_GAUSS:
          f[i] = o_rng_gauss(r, 1.0);
          f[i + 1] = 0.0;
          break;
        case O_FIELD_COMPLEXGAUSS:
          f[i] = o_rng_gauss(r, 1.0);
          f[i + 1] = o_rng_gauss(r, 1.0);
          break;
        case O_FIELD_ZTWO:
          f[i] = 2.0 * o_rng_z(r, 2) - 1.0;
          f[i + 1] = 0.0;
          break;
        default: {
          int z = o_rng_z(r, 3);
          if (z == 0) {
            f[i] = 1.0;
            f[i + 1] = 0.0;
          } else if (z == 1) {
            f[i] = -0.5;
            f[i + 1] = 0.8660254037844388;
          } else {
            f[i] = -0.5;
            f[i + 1] = -0.8660254037844388;
          }
        }
      }
    }
  }
}

/* ================================================================ tables */

/* Dispersion (src/alg/dispersion.C:11-75), periodic boundaries. */
void o_dispersion(const int dims[3], int type, double mass, int cutoff_type, double cutoff_sq,
                  double *out) {
  const int X = dims[0], Y = dims[1], Z = dims[2];
  const long vol = (long)X * Y * Z;
  for (long i = 0; i < vol; ++i) {
    int z = (int)(i % Z);
    int y = (int)((i / Z) % Y);
    int x = (int)(i / ((long)Y * Z));
    if (type == O_DISP_STANDARD) {
      double sx = sin((x + 0.0) * K_PI / X);
      double sy = sin((y + 0.0) * K_PI / Y);
      double sz = sin((z + 0.0) * K_PI / Z);
      out[i] = 2.0 * (sx * sx + sy * sy + sz * sz);
      out[i] /= mass;
    } else {
      if (x >= X / 2) x = X - x - 0;
      if (y >= Y / 2) y = Y - y - 0;
      if (z >= Z / 2) z = Z - z - 0;
      double sx = (x + 0.0) / (double)X;
      double sy = (y + 0.0) / (double)Y;
      double sz = (z + 0.0) / (double)Z;
      double psq = (sx * sx + sy * sy + sz * sz) * 4.0 * K_PISQ;
      if (cutoff_type == O_CUTOFF_HARD && psq > cutoff_sq) {
        out[i] = INFINITY;
      } else if (type == O_DISP_QUADRATIC) {
        out[i] = psq / (2.0 * mass);
      } else {
        out[i] = (exp(psq / (2.0 * mass)) - 1.0);
      }
    }
  }
}

/* Kinetic (src/hamiltonian/hamiltonian.C:260-281): xi = 1 + disp(m/dt). */
void o_kinetic_xi(const int dims[3], int type, double mass, double dt, double cutoff_sq, double *out) {
  const long vol = (long)dims[0] * dims[1] * dims[2];
  o_dispersion(dims, type, mass / dt, O_CUTOFF_HARD, cutoff_sq, out);
  for (long i = 0; i < vol; ++i) out[i] = 1.0 + out[i];
}

/* Interaction momentum factor (src/hamiltonian/hamiltonian.C:77-147). */
int o_interaction_table(const int dims[3], double mass, int itype, const double *couplings, int ncoup,
                        double dt, double cutoff_sq, double *out) {
  const long vol = (long)dims[0] * dims[1] * dims[2];
  double *disp = (double *)malloc(sizeof(double) * vol);
  o_dispersion(dims, O_DISP_PERFECT, mass, O_CUTOFF_NONE, cutoff_sq, disp);
  const double XI = exp(cutoff_sq / (2.0 * mass));
  int bad = 0;
  for (long i = 0; i < vol; ++i) {
    double xi = 1.0 + disp[i];
    if (xi > XI) xi = XI;
    double psq = (itype == O_ITYPE_XISQMINUSONE) ? xi * xi - 1.0 : 1.0 - 1.0 / (xi * xi);
    psq *= mass;
    out[i] = 0.0;
    for (int j = 0; j < ncoup; ++j) out[i] += couplings[j] * pow(psq, j);
    if (out[i] < 0.0) bad = 1;
    out[i] *= 2.0 * K_TWOPI / mass;
    out[i] = sqrt(out[i]);
    out[i] /= vol;
    out[i] *= dt;
  }
  free(disp);
  return bad;
}

/* Potential (src/hamiltonian/hamiltonian.C:165-244), harmonic form. */
void o_potential_table(const int dims[3], int ptype, double k1, double k2, double k3, double dt,
                       double *out) {
  const int X = dims[0], Yn = dims[1], Z = dims[2];
  const long vol = (long)X * Yn * Z;
  for (long i = 0; i < vol; ++i) {
    int z = (int)(i % Z);
    long Y = i / Z;
    int y = (int)(Y % Yn);
    int x = (int)(Y / Yn);
    if (x >= X / 2) x -= X;
    if (y >= Yn / 2) y -= Yn;
    if (z >= Z / 2) z -= Z;
    double v = k1 * x * x;
    v += k2 * y * y;
    v += k3 * z * z;
    v /= 2.0;
    if (ptype == O_POT_LIN) {
      out[i] = 1.0 - dt * v;
    } else {
      out[i] = exp(-dt * v);
    }
    out[i] /= vol;
  }
}

/* Momenta (src/alg/momenta.C:12-139). */
int o_momenta(const int dims[3], int disp_type, double mass, double fermi_energy, double cutoff_sq,
              int *idx, double *energy, int *parity, int cap) {
  const int X = dims[0], Y = dims[1], Z = dims[2];
  const long vol = (long)X * Y * Z;
  double *disp = (double *)malloc(sizeof(double) * vol);
  o_dispersion(dims, disp_type, mass, O_CUTOFF_HARD, cutoff_sq, disp);
  int count = 0;
  for (int n1 = 0; n1 < X; ++n1)
    for (int n2 = 0; n2 < Y; ++n2)
      for (int n3 = 0; n3 < Z; ++n3) {
        long i = n3 + (long)n2 * Z + (long)n1 * Y * Z;
        double e = log(1 + disp[i]);
        if (e <= fermi_energy) {
          if (count < cap) {
            energy[count] = e;
            idx[count] = (int)i;
          }
          ++count;
        }
      }
  free(disp);
  if (count > cap) return -count;
  /* insertion sort exactly as momenta.C:61-74 (j>0: slot 0 never moves) */
  for (int i = 1; i < count; ++i) {
    double e = energy[i];
    int m = idx[i];
    int j = i - 1;
    while ((j > 0) && (energy[j] > e)) {
      energy[j + 1] = energy[j];
      idx[j + 1] = idx[j];
      j--;
    }
    energy[j + 1] = e;
    idx[j + 1] = m;
  }
  for (int i = 0; i < count; ++i) {
    int x = idx[i] / (Y * Z), y = (idx[i] / Z) % Y, z = idx[i] % Z;
    int px = (X - x) % X, py = (Y - y) % Y, pz = (Z - z) % Z;
    int target = pz + Z * (py + Y * px);
    parity[i] = -1;
    for (int j = 0; j < count; ++j)
      if (idx[j] == target) parity[i] = j;
  }
  return count;
}

/* Normalised Hermite functions (src/utils/special_functions.C:26-36). */
static void hermite(double *h, int n, double x) {
  double a = 0.0, b;
  h[0] = K_PIM4;
  for (int j = 1; j < n; ++j) {
    b = a;
    a = h[j - 1];
    h[j] = x * sqrt(2.0 / j) * a - sqrt((double)(j - 1) / j) * b;
  }
}

/* OneBody::Set() SHO branch (src/one_body/one_body.C:66-166). */
void o_sho_source(const int dims[3], double l1, double l2, double l3, const double *coeffs,
                  double *psi) {
  const int X = dims[0], Y = dims[1], Z = dims[2];
  const long vol = (long)X * Y * Z;
  int n1m = X < 10 ? X : 10, n2m = Y < 10 ? Y : 10, n3m = Z < 10 ? Z : 10;
  double c[10][10][10][2];
  for (int a = 0; a < n1m; ++a)
    for (int b = 0; b < n2m; ++b)
      for (int e = 0; e < n3m; ++e) {
        long j = 2 * (e + (long)Z * (b + (long)Y * a));
        c[a][b][e][0] = coeffs[j];
        c[a][b][e][1] = coeffs[j + 1];
      }
  double h1[10], h2[10], h3[10];
  for (long i = 0; i < vol; ++i) {
    int x = (int)(i / ((long)Y * Z)), y = (int)((i / Z) % Y), z = (int)(i % Z);
    if (x >= X / 2) x -= X;
    if (y >= Y / 2) y -= Y;
    if (z >= Z / 2) z -= Z;
    double dx = K_TWOPI * x * l1 / (double)X;
    double dy = K_TWOPI * y * l2 / (double)Y;
    double dz = K_TWOPI * z * l2 / (double)Z; /* the reference uses lambda2 here (one_body.C:132) */
    hermite(h1, n1m, dx);
    hermite(h2, n2m, dy);
    hermite(h3, n3m, dz);
    double re = 0.0, im = 0.0, tmp;
    for (int a = 0; a < n1m; ++a)
      for (int b = 0; b < n2m; ++b)
        for (int e = 0; e < n3m; ++e) {
          tmp = h1[a] * h2[b] * h3[e];
          re += c[a][b][e][0] * tmp;
          im += c[a][b][e][1] * tmp;
        }
    tmp = exp(-(dx * dx + dy * dy + dz * dz) / 2.0);
    tmp *= sqrt(l1 * l2 * l3);
    tmp *= sqrt((K_TWOPI * K_TWOPI * K_TWOPI) / vol);
    psi[2 * i] = re * tmp;
    psi[2 * i + 1] = im * tmp;
  }
}

/* Dawson's integral by Rybicki's sampling method, as the reference's
 * DawsonF (src/utils/special_functions.C:48-78). */
double o_dawson(double x) {
  static double c[7];
  static int init = 0;
  const double H = 0.4, A1 = 2.0 / 3.0, A2 = 0.4, A3 = 2.0 / 7.0;
  if (!init) {
    init = 1;
    for (int i = 1; i <= 6; ++i) {
      double t = (2.0 * i - 1.0) * H;
      c[i] = exp(-(t * t));
    }
  }
  if (fabs(x) < 0.2) {
    double x2 = x * x;
    return x * (1.0 - A1 * x2 * (1.0 - A2 * x2 * (1.0 - A3 * x2)));
  }
  double xx = fabs(x);
  int n0 = 2 * (int)(0.5 * xx / H + 0.5);
  double xp = xx - n0 * H;
  double e1 = exp(2.0 * xp * H);
  double e2 = e1 * e1;
  double d1 = n0 + 1;
  double d2 = d1 - 2.0;
  double sum = 0.0;
  for (int i = 1; i <= 6; ++i, d1 += 2.0, d2 -= 2.0, e1 *= e2) sum += c[i] * (e1 / d1 + 1.0 / (d2 * e1));
  double ex = exp(-xp * xp);
  double s = (x >= 0.0) ? fabs(ex) : -fabs(ex);
  return s * sum / K_SQRTPI;
}

/* TwoBody constructor tables (src/two_body/two_body.C:21-141), periodic. */
void o_two_body_tables(const int dims[3], int wf_type, int disp1, int disp2, double m1, double m2,
                       double lambda, double cutoff_sq, double *wf, int *opp) {
  const int X = dims[0], Y = dims[1], Z = dims[2];
  const long vol = (long)X * Y * Z;
  for (long i = 0; i < vol; ++i) {
    int x = (int)(i / ((long)Y * Z)), y = (int)((i / Z) % Y), z = (int)(i % Z);
    int px = (X - x) % X, py = (Y - y) % Y, pz = (Z - z) % Z;
    opp[i] = pz + Z * (py + Y * px);
  }
  double *d1 = (double *)malloc(sizeof(double) * vol);
  double *d2 = (double *)malloc(sizeof(double) * vol);
  switch (wf_type) {
    case O_WF_NONE:
      for (long i = 0; i < vol; ++i) wf[i] = 0.0;
      break;
    case O_WF_UNIFORM:
      for (long i = 0; i < vol; ++i) wf[i] = 1.0 / vol;
      break;
    case O_WF_GND:
      o_dispersion(dims, disp1, m1, O_CUTOFF_HARD, cutoff_sq, d1);
      o_dispersion(dims, disp2, m2, O_CUTOFF_HARD, cutoff_sq, d2);
      for (long i = 0; i < vol; ++i) {
        double xi1 = 1.0 + d1[i], xi2 = 1.0 + d2[i];
        wf[i] = 1.0;
        wf[i] /= lambda - 1.0 / (xi1 * xi2);
      }
      break;
    case O_WF_TGND:
      o_dispersion(dims, O_DISP_QUADRATIC, 1.0, O_CUTOFF_HARD, cutoff_sq, d1);
      for (long i = 0; i < vol; ++i) {
        double psq = 2.0 * d1[i];
        if (psq > cutoff_sq) {
          wf[i] = 0.0;
        } else {
          double xi = sqrt(psq) / (2.0 * lambda);
          wf[i] = (xi < 1e-15) ? 1.0 : o_dawson(xi) / xi;
        }
      }
      break;
    case O_WF_PAIR1:
      o_dispersion(dims, O_DISP_QUADRATIC, 1.0, O_CUTOFF_HARD, cutoff_sq, d1);
      for (long i = 0; i < vol; ++i) wf[i] = 1.0 / (2.0 * d1[i] + lambda);
      break;
    default:
      o_dispersion(dims, O_DISP_QUADRATIC, 1.0, O_CUTOFF_HARD, cutoff_sq, d1);
      for (long i = 0; i < vol; ++i) {
        double psq = 2.0 * d1[i];
        wf[i] = (psq < 1e-15) ? 0.0 : exp(-lambda * sqrt(psq)) / psq;
      }
  }
  free(d1);
  free(d2);
}

/* =========================================================== propagation */

/* Interaction::Initialize (src/hamiltonian/noarch/hamiltonian_initialize.C:14-47). */
void o_interaction_initialize(const int dims[3], const double *lat, const double *itab, double *fld) {
  const long vol = (long)dims[0] * dims[1] * dims[2];
  memcpy(fld, lat, sizeof(double) * 2 * vol);
  o_fft3d(fld, dims, 1, +1);
  for (long i = 0; i < vol; ++i) {
    fld[2 * i] *= itab[i];
    fld[2 * i + 1] *= itab[i];
  }
  o_fft3d(fld, dims, 1, -1);
  for (long i = 0; i < vol; ++i) {
    fld[2 * i] += 1.0;
    fld[2 * i] /= vol;
    fld[2 * i + 1] /= vol;
  }
}

/* Kinetic::Evolve (src/hamiltonian/noarch/hamiltonian_evolve.C:96-116). */
void o_kinetic_evolve(long vol, int batch, double *psi, const double *xi) {
  for (int n = 0; n < batch; ++n) {
    double *a = psi + 2 * vol * n;
    for (long i = 0; i < vol; ++i) {
      a[2 * i] /= xi[i];
      a[2 * i + 1] /= xi[i];
    }
  }
}

/* Potential::Evolve (src/hamiltonian/noarch/hamiltonian_evolve.C:69-94). */
void o_potential_evolve(const int dims[3], int batch, double *psi, const double *pot) {
  const long vol = (long)dims[0] * dims[1] * dims[2];
  o_fft3d(psi, dims, batch, -1);
  for (int n = 0; n < batch; ++n) {
    double *a = psi + 2 * vol * n;
    for (long i = 0; i < vol; ++i) {
      a[2 * i] *= pot[i];
      a[2 * i + 1] *= pot[i];
    }
  }
  o_fft3d(psi, dims, batch, +1);
}

/* Interaction::Evolve (src/hamiltonian/noarch/hamiltonian_evolve.C:34-67). */
void o_interaction_evolve(const int dims[3], int batch, double *psi, const double *fld) {
  const long vol = (long)dims[0] * dims[1] * dims[2];
  o_fft3d(psi, dims, batch, -1);
  for (int n = 0; n < batch; ++n) {
    double *a = psi + 2 * vol * n;
    for (long i = 0; i < vol; ++i) {
      double re = fld[2 * i] * a[2 * i] - fld[2 * i + 1] * a[2 * i + 1];
      double im = fld[2 * i] * a[2 * i + 1] + fld[2 * i + 1] * a[2 * i];
      a[2 * i] = re;
      a[2 * i + 1] = im;
    }
  }
  o_fft3d(psi, dims, batch, +1);
}

/* =========================================================== measurement */

/* OneBody::Project (src/one_body/noarch/one_body_project.C:14-27) filling
 * S[s][t] = <src_s | psi_t> row-major (src/slater_det/slater_det.C:33-37). */
void o_project(long vol, int ns, const double *src, int nt, const double *psi, double *S) {
  for (int s = 0; s < ns; ++s) {
    const double *p = src + 2 * vol * s;
    for (int t = 0; t < nt; ++t) {
      const double *q = psi + 2 * vol * t;
      double re = 0.0, im = 0.0;
      for (long i = 0; i < 2 * vol; i += 2) {
        re += p[i] * q[i] + p[i + 1] * q[i + 1];
        im += p[i] * q[i + 1] - p[i + 1] * q[i];
      }
      S[2 * (t + (long)nt * s)] = re;
      S[2 * (t + (long)nt * s) + 1] = im;
    }
  }
}

/* TwoBody::Run (src/two_body/noarch/two_body_run.C:16-43) filling
 * phi[s][t] = sum_i w_i psi1_s(i) psi2_t(-i) (src/slater_det/slater_det2.C:52-57). */
void o_pair_matrix(long vol, int n, const double *psi1, const double *psi2, const double *wf,
                   const int *opp, double *phi) {
  for (int s = 0; s < n; ++s) {
    const double *p1 = psi1 + 2 * vol * s;
    for (int t = 0; t < n; ++t) {
      const double *p2 = psi2 + 2 * vol * t;
      double re = 0.0, im = 0.0;
      for (long i = 0; i < vol; ++i) {
        long j = 2 * i, k = 2 * (long)opp[i];
        re += (p1[j] * p2[k] - p1[j + 1] * p2[k + 1]) * wf[i];
        im += (p1[j] * p2[k + 1] + p1[j + 1] * p2[k]) * wf[i];
      }
      phi[2 * (t + (long)n * s)] = re;
      phi[2 * (t + (long)n * s) + 1] = im;
    }
  }
}

/* Crout LU with implicit-scaled partial pivoting (src/utils/ludcmp.C:9-65).
 * Returns 1 for an all-zero row (the reference prints and exits there). */
int o_ludcmp(double *araw, int n, int *indx, double *d) {
  double complex *a = (double complex *)araw;
  double *vv = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  int imax = 0;
  *d = 1.0;
  for (int i = 0; i < n; ++i) {
    double big = 0.0, temp;
    for (int j = 0; j < n; ++j)
      if ((temp = cabs(a[n * i + j])) > big) big = temp;
    if (big == 0.0) {
      free(vv);
      return 1;
    }
    vv[i] = 1.0 / big;
  }
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < j; ++i) {
      double complex sum = a[n * i + j];
      for (int k = 0; k < i; ++k) sum -= a[n * i + k] * a[n * k + j];
      a[n * i + j] = sum;
    }
    double big = 0.0;
    for (int i = j; i < n; ++i) {
      double complex sum = a[n * i + j];
      for (int k = 0; k < j; ++k) sum -= a[n * i + k] * a[n * k + j];
      a[n * i + j] = sum;
      double dum = vv[i] * cabs(sum);
      if (dum >= big) {
        big = dum;
        imax = i;
      }
    }
    if (j != imax) {
      for (int k = 0; k < n; ++k) {
        double complex t = a[n * imax + k];
        a[n * imax + k] = a[n * j + k];
        a[n * j + k] = t;
      }
      *d = -(*d);
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (cabs(a[n * j + j]) == 0.0) a[n * j + j] = 1.0e-20;
    if (j != n) {
      double complex dum = CMPLX(1.0, 0.0) / a[n * j + j];
      for (int i = j + 1; i < n; ++i) a[n * i + j] *= dum;
    }
  }
  free(vv);
  return 0;
}

/* SlaterDet::Run / SlaterDet2::Run (src/slater_det/slater_det.C:59-115,
 * slater_det2.C:78-148) on a contiguous n x n minor. */
void o_minor_det(const double *S, int N, int n, int t0, const double *psi1, int det_type, double *out) {
  double complex *a = (double complex *)malloc(sizeof(double complex) * n * n);
  const double complex *s = (const double complex *)S;
  const double complex *p1 = (const double complex *)psi1;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) a[n * i + j] = s[(long)N * i + j];
  if (t0 >= 0 && t0 < n)
    for (int i = 0; i < n; ++i) a[n * i + t0] = p1[i + (long)t0 * N];
  int *indx = (int *)malloc(sizeof(int) * n);
  double d;
  o_ludcmp((double *)a, n, indx, &d);
  double complex r;
  if (det_type == 0) {
    r = CMPLX(d, 0.0);
    for (int i = 0; i < n; ++i) r *= a[n * i + i];
  } else {
    r = clog(CMPLX(d, 0.0));
    for (int i = 0; i < n; ++i) r += clog(a[n * i + i]);
  }
  out[0] = creal(r);
  out[1] = cimag(r);
  free(indx);
  free(a);
}

/* ============================================================== ensemble */

int o_run_ensemble(const o_job *job, const double *sources, double *dets) {
  const int *dims = job->dims;
  const long vol = (long)dims[0] * dims[1] * dims[2];
  const int N = job->n_orb, T = job->T;
  const int nmeas = job->mode ? 2 * N : N;
  double *xi = (double *)malloc(sizeof(double) * vol);
  double *itab = (double *)malloc(sizeof(double) * vol);
  double *pot = (double *)malloc(sizeof(double) * vol);
  double *lat = (double *)malloc(sizeof(double) * 2 * vol);
  double *fld = (double *)malloc(sizeof(double) * 2 * vol);
  double *psi = (double *)malloc(sizeof(double) * 2 * vol * N);
  double *S = (double *)malloc(sizeof(double) * 2 * N * N);
  double *P1 = (double *)malloc(sizeof(double) * 2 * N * N);
  double *wf = (double *)malloc(sizeof(double) * vol);
  int *opp = (int *)malloc(sizeof(int) * vol);
  o_kinetic_xi(dims, job->kin_disp, job->kin_mass, job->kin_dt, job->cutoff_sq, xi);
  int bad = o_interaction_table(dims, job->int_mass, job->int_type, job->coup, job->n_coup, job->int_dt,
                                job->cutoff_sq, itab);
  if (job->use_potential)
    o_potential_table(dims, job->pot_type, job->pot_k[0], job->pot_k[1], job->pot_k[2], job->pot_dt, pot);
  if (job->mode)
    o_two_body_tables(dims, job->wf_type, job->wf_disp, job->wf_disp, job->wf_mass, job->wf_mass,
                      job->wf_lambda, job->cutoff_sq, wf, opp);
  o_rng rng;
  o_rng_init(&rng, job->rng_kind, job->seed);
  o_field_slices(&rng, job->field_type, vol, 1, lat); /* Lattice constructor draw */
  for (int c = 0; c < job->configs; ++c) {
    memcpy(psi, sources, sizeof(double) * 2 * vol * N);
    for (int t = 0; t < T; ++t) {
      double *row = dets + 2 * ((long)c * T + t) * nmeas;
      if (job->mode) {
        o_pair_matrix(vol, N, psi, psi, wf, opp, S);
        o_project(vol, N, sources, N, psi, P1);
        for (int n = 0; n < N; ++n) {
          o_minor_det(S, N, n + 1, -1, P1, 0, row + 2 * (2 * n + 1));
          o_minor_det(S, N, n + 1, n, P1, 0, row + 2 * (2 * n));
        }
      } else {
        o_project(vol, N, sources, N, psi, S);
        for (int n = 0; n < N; ++n) o_minor_det(S, N, n + 1, -1, NULL, 0, row + 2 * n);
      }
      o_interaction_initialize(dims, lat, itab, fld);
      o_kinetic_evolve(vol, N, psi, xi);
      if (job->use_potential) o_potential_evolve(dims, N, psi, pot);
      o_interaction_evolve(dims, N, psi, fld);
      if (job->use_potential) o_potential_evolve(dims, N, psi, pot);
      o_kinetic_evolve(vol, N, psi, xi);
      o_field_slices(&rng, job->field_type, vol, 1, lat);
    }
  }
  free(xi);
  free(itab);
  free(pot);
  free(lat);
  free(fld);
  free(psi);
  free(S);
  free(P1);
  free(wf);
  free(opp);
  return bad;
}

/* Jobs in sequence with one generator (see oracle.h).  Follows the driver
 * loop of production/slater_det/main.C:185-220 per configuration, with the
 * single-coupling interaction written as its position-space factor. */
void o_run_batch(int njobs, const int *L, const int *T, const int *nconf, const int *N, const int *const *idx,
                 int rng_kind, long seed, int field_type, double a, double kin_dt, double cutoff_sq,
                 double *const *dets) {
  o_rng rng;
  o_rng_init(&rng, rng_kind, seed);
  for (int j = 0; j < njobs; ++j) {
    const int dims[3] = {L[j], L[j], L[j]};
    const long vol = (long)L[j] * L[j] * L[j];
    const int n = N[j];
    double *xi = (double *)malloc(sizeof(double) * vol);
    double *lat = (double *)malloc(sizeof(double) * 2 * vol);
    double *fld = (double *)malloc(sizeof(double) * 2 * vol);
    double *psi = (double *)malloc(sizeof(double) * 2 * vol * n);
    double *src = (double *)calloc(2 * vol * n, sizeof(double));
    double *S = (double *)malloc(sizeof(double) * 2 * n * n);
    o_kinetic_xi(dims, 2 /* PERFECT */, 1.0, kin_dt, cutoff_sq, xi);
    for (int m = 0; m < n; ++m) src[2 * ((long)m * vol + idx[j][m])] = 1.0;
    for (int k = 0; k < nconf[j]; ++k) {
      memcpy(psi, src, sizeof(double) * 2 * vol * n);
      for (int t = 0; t < T[j]; ++t) {
        o_field_slices(&rng, field_type, vol, 1, lat);
        double *row = dets[j] + 2 * ((long)k * T[j] + t) * n;
        o_project(vol, n, src, n, psi, S);
        for (int m = 0; m < n; ++m) o_minor_det(S, n, m + 1, -1, NULL, 0, row + 2 * m);
        for (long x = 0; x < vol; ++x) {
          fld[2 * x] = (1.0 + a * lat[2 * x]) / (double)vol;
          fld[2 * x + 1] = (a * lat[2 * x + 1]) / (double)vol;
        }
        o_kinetic_evolve(vol, n, psi, xi);
        o_interaction_evolve(dims, n, psi, fld);
        o_kinetic_evolve(vol, n, psi, xi);
      }
    }
    free(xi);
    free(lat);
    free(fld);
    free(psi);
    free(src);
    free(S);
  }
}

/* ---------------------------------------------- multilevel branching */
typedef struct {
  const int *dims;
  long vol;
  int levels, branches, steps;
  o_rng *rng;
  int field_type;
  double a;
  const double *xi, *wf;
  const int *opp;
  double *lat, *fld, *corr;
} o_branch_ctx;

/* MultiLevel (production/two_body-branched/main.C:23-80) */
static void o_multilevel(o_branch_ctx *b, int level, double *p1, double *p2) {
  if (level <= 0) return;
  const long vol = b->vol;
  const int T = b->levels * b->steps;
  double *s1 = (double *)malloc(sizeof(double) * 2 * vol);
  double *s2 = (double *)malloc(sizeof(double) * 2 * vol);
  memcpy(s1, p1, sizeof(double) * 2 * vol);
  memcpy(s2, p2, sizeof(double) * 2 * vol);
  const double norm = pow((double)b->branches, (double)(b->levels - level + 1));
  for (int i = 0; i < b->branches; ++i) {
    memcpy(p1, s1, sizeof(double) * 2 * vol);
    memcpy(p2, s2, sizeof(double) * 2 * vol);
    for (int s = 0; s < b->steps; ++s) {
      const int t = T - (level - 1) * b->steps - (b->steps - s);
      double phi[2];
      o_pair_matrix(vol, 1, p1, p2, b->wf, b->opp, phi);
      b->corr[2 * t] += phi[0] / norm;
      b->corr[2 * t + 1] += phi[1] / norm;
      for (long x = 0; x < vol; ++x) {
        b->fld[2 * x] = (1.0 + b->a * b->lat[2 * x]) / (double)vol;
        b->fld[2 * x + 1] = (b->a * b->lat[2 * x + 1]) / (double)vol;
      }
      o_kinetic_evolve(vol, 1, p1, b->xi);
      o_interaction_evolve(b->dims, 1, p1, b->fld);
      o_kinetic_evolve(vol, 1, p1, b->xi);
      o_kinetic_evolve(vol, 1, p2, b->xi);
      o_interaction_evolve(b->dims, 1, p2, b->fld);
      o_kinetic_evolve(vol, 1, p2, b->xi);
      o_field_slices(b->rng, b->field_type, vol, 1, b->lat); /* lattice->Refresh() */
    }
    o_multilevel(b, level - 1, p1, p2);
  }
  free(s1);
  free(s2);
}

void o_run_branching(const int dims[3], int levels, int branches, int steps, int trees, int rng_kind, long seed,
                     int field_type, double a, double kin_dt, double cutoff_sq, const double *sources2,
                     const double *wf, const int *opp, double *corr) {
  const long vol = (long)dims[0] * dims[1] * dims[2];
  o_rng rng;
  o_rng_init(&rng, rng_kind, seed);
  double *xi = (double *)malloc(sizeof(double) * vol);
  double *lat = (double *)malloc(sizeof(double) * 2 * vol);
  double *fld = (double *)malloc(sizeof(double) * 2 * vol);
  double *p1 = (double *)malloc(sizeof(double) * 2 * vol);
  double *p2 = (double *)malloc(sizeof(double) * 2 * vol);
  o_kinetic_xi(dims, 2 /* PERFECT */, 1.0, kin_dt, cutoff_sq, xi);
  o_field_slices(&rng, field_type, vol, 1, lat); /* the Lattice constructor's draw */
  o_branch_ctx b = {dims, vol, levels, branches, steps, &rng, field_type, a, xi, wf, opp, lat, fld, corr};
  for (int r = 0; r < trees; ++r) {
    memcpy(p1, sources2, sizeof(double) * 2 * vol);
    memcpy(p2, sources2 + 2 * vol, sizeof(double) * 2 * vol);
    o_multilevel(&b, levels, p1, p2);
  }
  free(xi);
  free(lat);
  free(fld);
  free(p1);
  free(p2);
}

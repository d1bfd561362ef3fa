// tables.cc -- host construction of the per-lattice tables of the hot path.
//
// These replace the table-building parts of the reference's constructors so
// that a caller of the C ABI gets bit-identical tables without the
// reference's classes.  Arithmetic follows the reference operation by
// operation (same constants, same evaluation order), which tests check
// against tables produced by the reference itself.
#include <cmath>
#include <cstdlib>
#include <limits>
#include <vector>

#include "../../include/nrcps_b200.h"

namespace {

// include/constants.h:11-16
const double kPi = 3.1415926535897932;
const double kTwoPi = 6.2831853071795864;
const double kPiSq = 9.8696044010893586;
const double kPiM4 = 0.7511255444649425;
const double kSqrtPi = 1.7724538509055159;

inline long vol3(const int d[3]) { return (long)d[0] * d[1] * d[2]; }

bool dims_ok(const int d[3]) {
  if (!d) return false;
  for (int i = 0; i < 3; ++i)
    if (d[i] <= 0 || d[i] % 2 != 0) return false;  // GJP requires even extents (global_job_parameter.C:40-42)
  return true;
}

// Dispersion ctor (src/alg/dispersion.C:11-75), periodic boundaries.
void dispersion(const int d[3], int type, double mass, int hard, double cutoff_sq, double* out) {
  const int X = d[0], Y = d[1], Z = d[2];
  const long V = vol3(d);
  for (long i = 0; i < V; ++i) {
    int z = (int)(i % Z), y = (int)((i / Z) % Y), x = (int)(i / ((long)Y * Z));
    if (type == 0) {  // STANDARD: 2 sum sin^2(p/2) / m
      double sx = std::sin((x + 0.0) * kPi / X);
      double sy = std::sin((y + 0.0) * kPi / Y);
      double sz = std::sin((z + 0.0) * kPi / Z);
      out[i] = 2.0 * (sx * sx + sy * sy + sz * sz);
      out[i] /= mass;
      continue;
    }
    if (x >= X / 2) x = X - x;  // fold into the Brillouin zone (dispersion.C:54-56)
    if (y >= Y / 2) y = Y - y;
    if (z >= Z / 2) z = Z - z;
    double sx = (x + 0.0) / (double)X, sy = (y + 0.0) / (double)Y, sz = (z + 0.0) / (double)Z;
    double psq = (sx * sx + sy * sy + sz * sz) * 4.0 * kPiSq;
    if (hard && psq > cutoff_sq) {
      out[i] = std::numeric_limits<double>::infinity();
    } else if (type == 1) {
      out[i] = psq / (2.0 * mass);
    } else {
      out[i] = (std::exp(psq / (2.0 * mass)) - 1.0);
    }
  }
}

void hermite(double* h, int n, double x) {  // src/utils/special_functions.C:26-36
  double a = 0.0, b;
  h[0] = kPiM4;
  for (int j = 1; j < n; ++j) {
    b = a;
    a = h[j - 1];
    h[j] = x * std::sqrt(2.0 / j) * a - std::sqrt((double)(j - 1) / j) * b;
  }
}

// Dawson's integral by Rybicki's sampling method with six terms, h = 0.4,
// and the three-term series below 0.2 (src/utils/special_functions.C:48-78).
double dawson(double x) {
  const double H = 0.4, A1 = 2.0 / 3.0, A2 = 0.4, A3 = 2.0 / 7.0;
  double c[7];
  for (int i = 1; i <= 6; ++i) {
    double t = (2.0 * i - 1.0) * H;
    c[i] = std::exp(-(t * t));
  }
  if (std::fabs(x) < 0.2) {
    double x2 = x * x;
    return x * (1.0 - A1 * x2 * (1.0 - A2 * x2 * (1.0 - A3 * x2)));
  }
  double xx = std::fabs(x);
  int n0 = 2 * (int)(0.5 * xx / H + 0.5);
  double xp = xx - n0 * H, e1 = std::exp(2.0 * xp * H), e2 = e1 * e1;
  double d1 = n0 + 1, d2 = d1 - 2.0, sum = 0.0;
  for (int i = 1; i <= 6; ++i, d1 += 2.0, d2 -= 2.0, e1 *= e2) sum += c[i] * (e1 / d1 + 1.0 / (d2 * e1));
  double ex = std::exp(-xp * xp);
  double s = (x >= 0.0) ? std::fabs(ex) : -std::fabs(ex);
  return s * sum / kSqrtPi;
}

}  // namespace

extern "C" nrcps_status nrcps_dispersion_table(const int dims[3], int type, double mass, int hard_cutoff,
                                               double cutoff_sq, double* out) {
  if (!dims_ok(dims) || !out || type < 0 || type > 2) return NRCPS_ERR_INVALID_ARGUMENT;
  dispersion(dims, type, mass, hard_cutoff, cutoff_sq, out);
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_kinetic_table(const int dims[3], int type, double mass, double dt, double cutoff_sq,
                                            double* xi) {
  if (!dims_ok(dims) || !xi || type < 0 || type > 2) return NRCPS_ERR_INVALID_ARGUMENT;
  dispersion(dims, type, mass / dt, 1, cutoff_sq, xi);
  const long V = vol3(dims);
  for (long i = 0; i < V; ++i) xi[i] = 1.0 + xi[i];
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_interaction_table(const int dims[3], double mass, int itype, const double* couplings,
                                                int ncoup, double dt, double cutoff_sq, double* out) {
  if (!dims_ok(dims) || !out || (ncoup > 0 && !couplings) || ncoup < 0) return NRCPS_ERR_INVALID_ARGUMENT;
  if (itype != 1 && itype != 2) return NRCPS_ERR_UNSUPPORTED;  // INTERACTION_TYPE_NONE is NotImplemented
  const long V = vol3(dims);
  std::vector<double> disp(V);
  dispersion(dims, 2, mass, 0, cutoff_sq, disp.data());
  const double XI = std::exp(cutoff_sq / (2.0 * mass));
  for (long i = 0; i < V; ++i) {
    double xi = 1.0 + disp[i];
    if (xi > XI) xi = XI;
    double psq = (itype == 1) ? xi * xi - 1.0 : 1.0 - 1.0 / (xi * xi);
    psq *= mass;
    out[i] = 0.0;
    for (int j = 0; j < ncoup; ++j) out[i] += couplings[j] * std::pow(psq, j);
    if (out[i] < 0.0) return NRCPS_ERR_INVALID_ARGUMENT;  // hamiltonian.C:126-128
    out[i] *= 2.0 * kTwoPi / mass;
    out[i] = std::sqrt(out[i]);
    out[i] /= V;
    out[i] *= dt;
  }
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_potential_table(const int dims[3], int ptype, double k1, double k2, double k3,
                                              double dt, double* out) {
  if (!dims_ok(dims) || !out || (ptype != 0 && ptype != 1)) return NRCPS_ERR_INVALID_ARGUMENT;
  const int X = dims[0], Yn = dims[1], Z = dims[2];
  const long V = vol3(dims);
  for (long i = 0; i < V; ++i) {
    int z = (int)(i % Z);
    long Y = i / Z;
    int y = (int)(Y % Yn), x = (int)(Y / Yn);
    if (x >= X / 2) x -= X;
    if (y >= Yn / 2) y -= Yn;
    if (z >= Z / 2) z -= Z;
    double v = k1 * x * x;
    v += k2 * y * y;
    v += k3 * z * z;
    v /= 2.0;
    out[i] = (ptype == 0) ? 1.0 - dt * v : std::exp(-dt * v);
    out[i] /= V;
  }
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_momenta(const int dims[3], int disp_type, double mass, double fermi_energy,
                                      double cutoff_sq, int cap, int* index, double* energy, int* parity,
                                      int* count) {
  if (!dims_ok(dims) || !count || cap < 0) return NRCPS_ERR_INVALID_ARGUMENT;
  const int X = dims[0], Y = dims[1], Z = dims[2];
  const long V = vol3(dims);
  std::vector<double> disp(V);
  dispersion(dims, disp_type, mass, 1, cutoff_sq, disp.data());
  std::vector<int> idx;
  std::vector<double> en;
  for (int n1 = 0; n1 < X; ++n1)
    for (int n2 = 0; n2 < Y; ++n2)
      for (int n3 = 0; n3 < Z; ++n3) {
        long i = n3 + (long)n2 * Z + (long)n1 * Y * Z;
        double e = std::log(1 + disp[i]);
        if (e <= fermi_energy) {
          idx.push_back((int)i);
          en.push_back(e);
        }
      }
  const int n = (int)idx.size();
  *count = n;
  if (n == 0) return NRCPS_ERR_INVALID_ARGUMENT;  // "No energy levels exceed the specified fermi level."
  // Insertion sort by energy as src/alg/momenta.C:61-74 (slot 0 never moves).
  for (int i = 1; i < n; ++i) {
    double e = en[i];
    int m = idx[i];
    int j = i - 1;
    while ((j > 0) && (en[j] > e)) {
      en[j + 1] = en[j];
      idx[j + 1] = idx[j];
      j--;
    }
    en[j + 1] = e;
    idx[j + 1] = m;
  }
  for (int i = 0; i < n && i < cap; ++i) {
    if (index) index[i] = idx[i];
    if (energy) energy[i] = en[i];
    if (parity) {
      int x = idx[i] / (Y * Z), y = (idx[i] / Z) % Y, z = idx[i] % Z;
      int target = ((Z - z) % Z) + Z * (((Y - y) % Y) + Y * ((X - x) % X));
      parity[i] = -1;
      for (int j = 0; j < n; ++j)
        if (idx[j] == target) parity[i] = j;
      if (parity[i] < 0) return NRCPS_ERR_INVALID_ARGUMENT;  // momenta.C:122-125
    }
  }
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_sho_source(const int dims[3], double l1, double l2, double l3, const double* coeffs,
                                         double* psi) {
  if (!dims_ok(dims) || !coeffs || !psi) return NRCPS_ERR_INVALID_ARGUMENT;
  const int X = dims[0], Y = dims[1], Z = dims[2];
  const long V = vol3(dims);
  const int n1m = X < 10 ? X : 10, n2m = Y < 10 ? Y : 10, n3m = Z < 10 ? Z : 10;
  static thread_local double c[10][10][10][2];
  for (int a = 0; a < n1m; ++a)
    for (int b = 0; b < n2m; ++b)
      for (int e = 0; e < n3m; ++e) {
        long j = 2 * (e + (long)Z * (b + (long)Y * a));
        c[a][b][e][0] = coeffs[j];
        c[a][b][e][1] = coeffs[j + 1];
      }
  double h1[10], h2[10], h3[10];
  for (long i = 0; i < V; ++i) {
    int x = (int)(i / ((long)Y * Z)), y = (int)((i / Z) % Y), z = (int)(i % Z);
    if (x >= X / 2) x -= X;
    if (y >= Y / 2) y -= Y;
    if (z >= Z / 2) z -= Z;
    double dx = kTwoPi * x * l1 / (double)X;
    double dy = kTwoPi * y * l2 / (double)Y;
    double dz = kTwoPi * z * l2 / (double)Z;  // the reference uses lambda2 for z (one_body.C:132)
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
    tmp = std::exp(-(dx * dx + dy * dy + dz * dz) / 2.0);
    tmp *= std::sqrt(l1 * l2 * l3);
    tmp *= std::sqrt((kTwoPi * kTwoPi * kTwoPi) / V);
    psi[2 * i] = re * tmp;
    psi[2 * i + 1] = im * tmp;
  }
  return NRCPS_OK;
}

extern "C" nrcps_status nrcps_two_body_tables(const int dims[3], int wf_type, int disp1, int disp2, double m1,
                                              double m2, double lambda, double cutoff_sq, double* w,
                                              int* opposite) {
  if (!dims_ok(dims) || !w || !opposite || wf_type < 0 || wf_type > 5) return NRCPS_ERR_INVALID_ARGUMENT;
  const int X = dims[0], Y = dims[1], Z = dims[2];
  const long V = vol3(dims);
  for (long i = 0; i < V; ++i) {
    int x = (int)(i / ((long)Y * Z)), y = (int)((i / Z) % Y), z = (int)(i % Z);
    opposite[i] = ((Z - z) % Z) + Z * (((Y - y) % Y) + Y * ((X - x) % X));
  }
  std::vector<double> d1(V), d2(V);
  switch (wf_type) {
    case 0:
      for (long i = 0; i < V; ++i) w[i] = 0.0;
      break;
    case 1:
      for (long i = 0; i < V; ++i) w[i] = 1.0 / V;
      break;
    case 2:
      dispersion(dims, disp1, m1, 1, cutoff_sq, d1.data());
      dispersion(dims, disp2, m2, 1, cutoff_sq, d2.data());
      for (long i = 0; i < V; ++i) {
        double xi1 = 1.0 + d1[i], xi2 = 1.0 + d2[i];
        w[i] = 1.0;
        w[i] /= lambda - 1.0 / (xi1 * xi2);
      }
      break;
    case 3:
      dispersion(dims, 1, 1.0, 1, cutoff_sq, d1.data());
      for (long i = 0; i < V; ++i) {
        double psq = 2.0 * d1[i];
        if (psq > cutoff_sq) {
          w[i] = 0.0;
        } else {
          double xi = std::sqrt(psq) / (2.0 * lambda);
          w[i] = (xi < 1e-15) ? 1.0 : dawson(xi) / xi;
        }
      }
      break;
    case 4:
      dispersion(dims, 1, 1.0, 1, cutoff_sq, d1.data());
      for (long i = 0; i < V; ++i) w[i] = 1.0 / (2.0 * d1[i] + lambda);
      break;
    default:
      dispersion(dims, 1, 1.0, 1, cutoff_sq, d1.data());
      for (long i = 0; i < V; ++i) {
        double psq = 2.0 * d1[i];
        w[i] = (psq < 1e-15) ? 0.0 : std::exp(-lambda * std::sqrt(psq)) / psq;
      }
  }
  return NRCPS_OK;
}

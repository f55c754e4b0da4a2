// Operation count of the Z4c right-hand side, taken from the oracle itself.
//
// TEST INFRASTRUCTURE ONLY.  The oracle's C restatement (z4c_oracle.c, which
// follows the reference's arithmetic operation by operation) is compiled here
// as C++ with its floating-point type replaced by a counting type, so that
// every FP64 +, -, x, / (and every call of sqrt, cbrt, pow, fabs) the
// reference algorithm performs is tallied.  The program prints the counts per
// interior vertex of one MeshBlock for
//   rhs   Z4c::PrepareZ4cDerivatives + Z4c::Z4cRHS (adm_z4c.cpp:972-1037,
//         calculate_z4c_rhs.cpp:29-916), Kreiss-Oliger included
//   stage one low-storage RK stage update per variable: u1 += d*u, u = g1*u +
//         g2*u1, u += (b*dt)*rhs (weighted_ave.cpp:20-150 twice and
//         add_z4c_rhs.cpp:24-35), 2 + 3 + 2 = 7 operations, counted by hand
// as one JSON line.  usage: count_ops <nx>   (cells per block axis)
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace opcount {
unsigned long long add = 0, mul = 0, div = 0, fn = 0, cmp = 0;
}

struct CReal {
  double v;
  CReal() = default;
  CReal(double x) : v(x) {}
  CReal(int x) : v(x) {}
  CReal(long x) : v((double)x) {}
  CReal(long long x) : v((double)x) {}
  CReal(unsigned long x) : v((double)x) {}
  explicit operator int() const { return (int)v; }
  CReal& operator+=(CReal o) { ++opcount::add; v += o.v; return *this; }
  CReal& operator-=(CReal o) { ++opcount::add; v -= o.v; return *this; }
  CReal& operator*=(CReal o) { ++opcount::mul; v *= o.v; return *this; }
  CReal& operator/=(CReal o) { ++opcount::div; v /= o.v; return *this; }
};
inline CReal operator+(CReal a, CReal b) { ++opcount::add; return CReal(a.v + b.v); }
inline CReal operator-(CReal a, CReal b) { ++opcount::add; return CReal(a.v - b.v); }
inline CReal operator*(CReal a, CReal b) { ++opcount::mul; return CReal(a.v * b.v); }
inline CReal operator/(CReal a, CReal b) { ++opcount::div; return CReal(a.v / b.v); }
inline CReal operator-(CReal a) { return CReal(-a.v); }  // sign flip: not an operation
inline bool operator<(CReal a, CReal b) { ++opcount::cmp; return a.v < b.v; }
inline bool operator>(CReal a, CReal b) { ++opcount::cmp; return a.v > b.v; }
inline bool operator<=(CReal a, CReal b) { ++opcount::cmp; return a.v <= b.v; }
inline bool operator>=(CReal a, CReal b) { ++opcount::cmp; return a.v >= b.v; }
inline bool operator==(CReal a, CReal b) { ++opcount::cmp; return a.v == b.v; }
inline bool operator!=(CReal a, CReal b) { ++opcount::cmp; return a.v != b.v; }
inline CReal fabs(CReal a) { ++opcount::fn; return CReal(std::fabs(a.v)); }
inline CReal sqrt(CReal a) { ++opcount::fn; return CReal(std::sqrt(a.v)); }
inline CReal cbrt(CReal a) { ++opcount::fn; return CReal(std::cbrt(a.v)); }
inline CReal pow(CReal a, CReal b) { ++opcount::fn; return CReal(std::pow(a.v, b.v)); }
inline CReal pow(int a, int b) { return CReal(std::pow((double)a, (double)b)); }
inline int isfinite(CReal a) { return std::isfinite(a.v); }
inline CReal floor(CReal a) { return CReal(std::floor(a.v)); }
// trigonometry of the extraction-sphere set-up (not on the counted path)
inline CReal sin(CReal a) { ++opcount::fn; return CReal(std::sin(a.v)); }
inline CReal cos(CReal a) { ++opcount::fn; return CReal(std::cos(a.v)); }
inline CReal acos(CReal a) { ++opcount::fn; return CReal(std::acos(a.v)); }
inline CReal atan(CReal a) { ++opcount::fn; return CReal(std::atan(a.v)); }
inline CReal atan2(CReal a, CReal b) { ++opcount::fn; return CReal(std::atan2(a.v, b.v)); }
inline long lrint(CReal a) { return std::lrint(a.v); }

#define double CReal
#include "../z4c_oracle.c"
#undef double

int main(int argc, char** argv) {
  const int nx = argc > 1 ? atoi(argv[1]) : 16;
  const int nn = nx + 1 + 2 * ORC_NG;
  const int64_t nvol = (int64_t)nn * nn * nn;
  const int64_t npts = (int64_t)(nx + 1) * (nx + 1) * (nx + 1);
  // a smooth, non-trivial state: every variable varies, the shift has both signs
  CReal* x = (CReal*)malloc(sizeof(CReal) * nn);
  for (int i = 0; i < nn; ++i) x[i] = CReal(-1.0 + 2.0 * (i - ORC_NG) / nx);
  orc_block_t b;
  for (int a = 0; a < 3; ++a) {
    b.nx[a] = nx;
    b.dx[a] = CReal(2.0 / nx);
    b.x[a] = x;
    b.xc[a] = x;
  }
  CReal* u = (CReal*)malloc(sizeof(CReal) * Z4C_NVAR * nvol);
  CReal* rhs = (CReal*)calloc((size_t)Z4C_NVAR * nvol, sizeof(CReal));
  for (int n = 0; n < Z4C_NVAR; ++n)
    for (int64_t p = 0; p < nvol; ++p) {
      const double s = std::sin(0.37 * n + 0.011 * (double)p);
      const bool diag = (n == Z4C_CHI || n == Z4C_GXX || n == Z4C_GYY || n == Z4C_GZZ ||
                         n == Z4C_ALPHA);
      u[n * nvol + p] = CReal((diag ? 1.0 : 0.0) + 0.05 * s);
    }
  z4c_params_t opt;
  opt.chi_psi_power = -4; opt.chi_div_floor = 1e-5; opt.diss = 0.02; opt.eps_floor = 1e-12;
  opt.damp_kappa1 = 0.02; opt.damp_kappa2 = 0; opt.lapse_oplog = 2; opt.lapse_harmonicf = 1;
  opt.lapse_harmonic = 0; opt.lapse_advect = 1; opt.lapse_K = 0; opt.shift_Gamma = 1;
  opt.shift_alpha2Gamma = 0; opt.shift_H = 0; opt.shift_advect = 1; opt.shift_eta = 2;
  opt.r_max_con = 1e300; opt.tf_force_regularization = 1; opt.force_regularization = 0;

  orc_derivs_t d;
  orc_derivs_alloc(&b, &d);
  opcount::add = opcount::mul = opcount::div = opcount::fn = opcount::cmp = 0;
  orc_prepare_derivs(&b, u, &d);
  orc_rhs(&b, &opt, u, &d, rhs);
  const unsigned long long r_add = opcount::add, r_mul = opcount::mul, r_div = opcount::div,
                           r_fn = opcount::fn;
  // Z4cWeyl after PrepareZ4cDerivatives on the ADM image of the same state
  CReal* adm = (CReal*)calloc((size_t)Z4C_NADM * nvol, sizeof(CReal));
  CReal* weyl = (CReal*)calloc((size_t)2 * nvol, sizeof(CReal));
  orc_z4c_to_adm(&b, &opt, u, adm);
  opcount::add = opcount::mul = opcount::div = opcount::fn = opcount::cmp = 0;
  orc_prepare_derivs(&b, u, &d);
  orc_weyl(&b, &opt, adm, u, &d, weyl);
  const unsigned long long w_all = opcount::add + opcount::mul + opcount::div + opcount::fn;
  const unsigned long long w_div = opcount::div, w_fn = opcount::fn;
  const double P = (double)npts;
  printf("{\"nx\": %d, \"interior_vertices\": %lld, "
         "\"rhs\": {\"add\": %.3f, \"mul\": %.3f, \"div\": %.3f, \"fn\": %.3f, \"total\": %.3f}, "
         "\"stage\": {\"total\": %d}, "
         "\"weyl\": {\"div\": %.3f, \"fn\": %.3f, \"total\": %.3f}}\n",
         nx, (long long)npts, r_add / P, r_mul / P, r_div / P, r_fn / P,
         (r_add + r_mul + r_div + r_fn) / P, 7 * Z4C_NVAR, w_div / P, w_fn / P, w_all / P);
  free(adm); free(weyl);
  orc_derivs_free(&d);
  free(u); free(rhs); free(x);
  return 0;
}

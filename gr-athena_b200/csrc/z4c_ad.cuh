// Pointwise pieces of the differentiated Z4c path: the tangent-linear model
// (forward mode) and the hand-written adjoint (reverse mode) of
//   Z4c::Z4cRHS        z4c/calculate_z4c_rhs.cpp:29-916 (vacuum, constant eta)
//   Z4c::AlgConstr     z4c/z4c.cpp:677-799
//   Z4c::Z4cToADM      z4c/adm_z4c.cpp:200-260 and the Hamiltonian constraint
//                      of Z4c::ADMConstraints, z4c/adm_z4c.cpp:382-760
// at one vertex, as functions of the values a vertex's stencils gather.
//
// The right-hand side at an interior vertex is a function of the 158 "local
// inputs" of RhsLocal: the 22 variables there, the stored first derivatives
// of chi, g~_ab, alpha, beta^a (PrepareZ4cDerivatives, adm_z4c.cpp:972-1037),
// the centred first derivatives of Gamma~^a, Khat and Theta, the second
// derivatives of chi, g~_ab, alpha, beta^a (Dxx on the diagonal, Dx of the
// stored Dx off it), and the 22 advection sums beta^a L_a f.  Every one of
// those is linear in the state (the advection sums bilinear in the state and
// the shift); the kernels gather them and scatter their adjoints back through
// the transposed stencils.  Kreiss-Oliger dissipation is linear and handled
// by the kernels alone.
//
// The forward functions are templates on the number type: with double they
// follow the reference's evaluation order (calculate_z4c_rhs.cpp, line
// numbers in the comments), with Dual they carry one tangent direction (the
// tangent-linear model).  The *_adj functions are the reverse sweeps, written
// by hand: they recompute the forward intermediates they need and accumulate
// the adjoints of the local inputs (and of the gauge parameters eta and
// kappa1) with +=.
//
// Branch conventions (the forward is piecewise smooth):
//   max(chi, chi_div_floor)   the adjoint flows into chi where chi >= floor,
//                             and nowhere below it;
//   regularize_nth_root       below the threshold the value is a constant and
//                             its derivative 0 (AlgConstr: det g~ < 1 + eps);
//   det g~ > 0 ? det g~ : 1   derivative 0 where det g~ <= 0;
//   upwind stencil side       the side the sign of beta^a selects at the
//                             linearisation point is held fixed (beta^a = 0
//                             selects the right-biased side, as the forward).
//
// Everything here compiles for the host too (no device intrinsics), so the
// reverse sweeps are checked against the forward-mode ones on the CPU.
#pragma once

#include <cmath>

#include "../../include/z4c_b200.h"

#ifdef __CUDACC__
#define Z4C_HD __host__ __device__ __forceinline__
#define Z4C_UNROLL _Pragma("unroll")
// loops of the forward templates
#define Z4C_UNROLL_T _Pragma("unroll")
#else
#define Z4C_HD inline
#define Z4C_UNROLL
#define Z4C_UNROLL_T
#endif

namespace z4c {
namespace ad {

constexpr int NV = Z4C_NVAR;

// index of the symmetric pair (a,b) in xx,xy,xz,yy,yz,zz order
Z4C_HD constexpr int sid(int a, int b) {
  return (a == b) ? (a == 0 ? 0 : (a == 1 ? 3 : 5)) : ((a + b == 1) ? 1 : ((a + b == 2) ? 2 : 4));
}
// weight of the pair (a,b) in a sum over a <= b of a symmetric contraction
Z4C_HD constexpr double wsym(int a, int b) { return a == b ? 1.0 : 2.0; }

// ---- forward-mode number ---------------------------------------------------
struct Dual {
  double v, d;
  Z4C_HD Dual() : v(0), d(0) {}
  Z4C_HD Dual(double x) : v(x), d(0) {}
  Z4C_HD Dual(double x, double dx) : v(x), d(dx) {}
  Z4C_HD Dual& operator+=(const Dual& o) { v += o.v; d += o.d; return *this; }
  Z4C_HD Dual& operator-=(const Dual& o) { v -= o.v; d -= o.d; return *this; }
  Z4C_HD Dual& operator*=(const Dual& o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
};
Z4C_HD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
Z4C_HD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
Z4C_HD Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
Z4C_HD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
Z4C_HD Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
Z4C_HD Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
Z4C_HD Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
Z4C_HD Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
Z4C_HD Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
Z4C_HD Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
Z4C_HD Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
Z4C_HD Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
Z4C_HD Dual operator/(double a, Dual b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
Z4C_HD bool operator<(Dual a, Dual b) { return a.v < b.v; }
Z4C_HD bool operator<(Dual a, double b) { return a.v < b; }
Z4C_HD bool operator<(double a, Dual b) { return a < b.v; }
Z4C_HD bool operator>(Dual a, double b) { return a.v > b; }

Z4C_HD double val(double x) { return x; }
Z4C_HD double val(const Dual& x) { return x.v; }
Z4C_HD double ad_pow(double x, double e) { return pow(x, e); }
Z4C_HD Dual ad_pow(const Dual& x, double e) {
  const double p = pow(x.v, e);
  return Dual(p, e * pow(x.v, e - 1.0) * x.d);
}
// dmax(a, b) = (a < b) ? b : a with a constant b (the chi floor)
template <class T>
Z4C_HD T ad_max_c(const T& a, double b) {
  return (a < b) ? T(b) : a;
}

// ---- the local inputs of the right-hand side at one interior vertex -------
template <class T>
struct RhsLocal {
  T u[NV];           // the 22 variables at the vertex (Z4C_* order)
  T dchi[3];         // stored d_a chi
  T dg[3][6];        // stored d_c g~_q  [c][q]
  T dalpha[3];       // stored d_a alpha
  T dbeta[3][3];     // stored d_b beta^a  [b][a]
  T dGam[3][3];      // d_b Gamma~^c  [b][c]
  T dKhat[3];        // d_b Khat
  T dTheta[3];       // d_b Theta
  T ddchi[6];        // d_a d_b chi, pair (a,b)
  T ddg[6][6];       // d_c d_d g~_q  [q][pair(c,d)]
  T ddalpha[6];      // d_a d_b alpha
  T ddbeta[3][6];    // d_a d_b beta^c  [c][pair(a,b)]
  T lv[NV];          // advection sums sum_a beta^a L_a f_n
  static constexpr int N = NV + 3 + 18 + 3 + 9 + 9 + 3 + 3 + 6 + 36 + 6 + 18 + NV;
  Z4C_HD T* data() { return u; }
  Z4C_HD const T* data() const { return u; }
};

// Adjoints of the gauge and damping parameters the reverse sweep reports.
struct ParamBar {
  double shift_eta, damp_kappa1;
};

// ---- 3x3 symmetric helpers (linear_algebra.hpp:47-118) ---------------------
template <class T>
Z4C_HD T det3s(const T* g) {
  const T gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
  return (-(gxz * gxz) * gyy + 2. * gxy * gxz * gyz - gxx * (gyz * gyz) - (gxy * gxy) * gzz +
          gxx * gyy * gzz);
}
template <class T>
Z4C_HD void inv3s(const T& oodetg, const T* g, T* gu) {
  const T gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
  gu[0] = (-(gyz * gyz) + gyy * gzz) * oodetg;
  gu[1] = (gxz * gyz - gxy * gzz) * oodetg;
  gu[3] = (-(gxz * gxz) + gxx * gzz) * oodetg;
  gu[2] = (-gxz * gyy + gxy * gyz) * oodetg;
  gu[4] = (gxy * gxz - gxx * gyz) * oodetg;
  gu[5] = (-(gxy * gxy) + gxx * gyy) * oodetg;
}
// d det / d g_q for the six stored components
Z4C_HD void det3s_grad(const double* g, double* dd) {
  const double gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
  dd[0] = -(gyz * gyz) + gyy * gzz;
  dd[1] = 2. * (gxz * gyz - gxy * gzz);
  dd[2] = 2. * (gxy * gyz - gxz * gyy);
  dd[3] = -(gxz * gxz) + gxx * gzz;
  dd[4] = 2. * (gxy * gxz - gxx * gyz);
  dd[5] = -(gxy * gxy) + gxx * gyy;
}
// Reverse of H = g^-1 (six stored components each): gb += (dH/dg)^T Hb, with
// dH = -H dG H and dG = E_ab + E_ba for an off-diagonal stored component.
Z4C_HD void inv3s_adj(const double* H, const double* Hb, double* gb) {
#define HH(i, j) H[sid(i, j)]
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      double acc = 0.;
      Z4C_UNROLL
      for (int i = 0; i < 3; ++i)
        Z4C_UNROLL
        for (int j = i; j < 3; ++j) {
          const double t = (a == b) ? HH(i, a) * HH(a, j) : HH(i, a) * HH(b, j) + HH(i, b) * HH(a, j);
          acc -= Hb[sid(i, j)] * t;
        }
      gb[sid(a, b)] += acc;
    }
#undef HH
}

// ---- forward: Christoffel symbols, Ricci, the right-hand side --------------
// Inverse conformal metric (:295-311) and Christoffel symbols (:317-352).
template <class T>
Z4C_HD void christoffel_local(const RhsLocal<T>& v, T guu[6], T Gd[3][6], T Gudd[3][6],
                              T Gu[3]) {
  const T* g = v.u + Z4C_GXX;
  {
    const T detg = det3s(g);
    inv3s(T(1.0) / detg, g, guu);
  }
  Z4C_UNROLL_T
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL_T
    for (int a = 0; a < 3; ++a)
      Z4C_UNROLL_T
      for (int b = a; b < 3; ++b)
        Gd[c][sid(a, b)] = 0.5 * (v.dg[a][sid(b, c)] + v.dg[b][sid(a, c)] - v.dg[c][sid(a, b)]);
  Z4C_UNROLL_T
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL_T
    for (int a = 0; a < 3; ++a)
      Z4C_UNROLL_T
      for (int b = a; b < 3; ++b) {
        T s = T(0.);
        Z4C_UNROLL_T
        for (int d = 0; d < 3; ++d) s += guu[sid(c, d)] * Gd[d][sid(a, b)];
        Gudd[c][sid(a, b)] = s;
      }
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) {
    T s = T(0.);
    Z4C_UNROLL_T
    for (int b = 0; b < 3; ++b)
      Z4C_UNROLL_T
      for (int c = b; c < 3; ++c) s += wsym(b, c) * guu[sid(b, c)] * Gudd[a][sid(b, c)];
    Gu[a] = s;
  }
}

// Rsum_ab = R_ab + Rphi_ab (:357-458)
template <class T>
Z4C_HD void ricci_local(const z4c_params_t& opt, const RhsLocal<T>& v, T Rsum[6]) {
  T guu[6], Gd[3][6], Gudd[3][6], Gu[3];
  christoffel_local(v, guu, Gd, Gudd, Gu);
  const T* g = v.u + Z4C_GXX;
  T Rdd[6];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      T s = T(0.);
      Z4C_UNROLL_T
      for (int c = 0; c < 3; ++c)
        s += 0.5 * (g[sid(c, a)] * v.dGam[b][c] + g[sid(c, b)] * v.dGam[a][c] +
                    Gu[c] * (Gd[a][sid(b, c)] + Gd[b][sid(a, c)]));
      Rdd[sid(a, b)] = s;
    }
  Z4C_UNROLL_T
  for (int q = 0; q < 6; ++q) {
    T s = Rdd[q];
    Z4C_UNROLL_T
    for (int c = 0; c < 3; ++c)
      Z4C_UNROLL_T
      for (int d = c; d < 3; ++d)
        s -= ((c == d) ? 0.5 : 1.0) * guu[sid(c, d)] * v.ddg[q][sid(c, d)];
    Rdd[q] = s;
  }
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      T s = Rdd[sid(a, b)];
      Z4C_UNROLL_T
      for (int c = 0; c < 3; ++c)
        Z4C_UNROLL_T
        for (int d = 0; d < 3; ++d)
          Z4C_UNROLL_T
          for (int e = 0; e < 3; ++e)
            s += guu[sid(c, d)] * (Gudd[e][sid(c, a)] * Gd[b][sid(e, d)] +
                                   Gudd[e][sid(c, b)] * Gd[a][sid(e, d)] +
                                   Gudd[e][sid(a, d)] * Gd[e][sid(c, b)]);
      Rdd[sid(a, b)] = s;
    }
  const T chi_g = ad_max_c(v.u[Z4C_CHI], opt.chi_div_floor);
  const T oochi = T(1.0) / chi_g;
  const double ooc = 1.0 / opt.chi_psi_power;
  T dphi[3];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) dphi[a] = v.dchi[a] * oochi * ooc;
  T Ddphi[6];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      T x = v.ddchi[sid(a, b)] * oochi * ooc - opt.chi_psi_power * dphi[a] * dphi[b];
      Z4C_UNROLL_T
      for (int c = 0; c < 3; ++c) x -= Gudd[c][sid(a, b)] * dphi[c];
      Ddphi[sid(a, b)] = x;
    }
  T Stmp = T(0.);
  Z4C_UNROLL_T
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL_T
    for (int d = c; d < 3; ++d)
      Stmp += wsym(c, d) * guu[sid(c, d)] * (Ddphi[sid(c, d)] + 2. * dphi[c] * dphi[d]);
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      const T rphi = 4. * dphi[a] * dphi[b] - 2. * Ddphi[sid(a, b)] - 2. * g[sid(a, b)] * Stmp;
      Rsum[sid(a, b)] = Rdd[sid(a, b)] + rphi;
    }
}

// The 22 right-hand-side values without Kreiss-Oliger, given Rsum (:231-902)
template <class T>
Z4C_HD void main_local(const z4c_params_t& opt, const RhsLocal<T>& v, const T Rsum[6],
                       T out[NV]) {
  T guu[6], Gd[3][6], Gudd[3][6], Gu[3];
  christoffel_local(v, guu, Gd, Gudd, Gu);
  const T* g = v.u + Z4C_GXX;
  const T* A = v.u + Z4C_AXX;
  const T chi = v.u[Z4C_CHI], Khat = v.u[Z4C_KHAT], Theta = v.u[Z4C_THETA];
  const T alpha = v.u[Z4C_ALPHA];
  const double pw = opt.chi_psi_power;
  const T K = Khat + 2. * Theta;
  const T chi_g = ad_max_c(chi, opt.chi_div_floor);
  const T oochi = T(1.0) / chi_g;
  T oopsi4;
  if (pw == -4.) oopsi4 = chi_g;
  else oopsi4 = ad_pow(chi_g, -4. / pw);
  const double ooc = 1.0 / pw;
  T dphi[3];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) dphi[a] = v.dchi[a] * oochi * ooc;
  // D D alpha (:482-521)
  T Dda_s = T(0.);
  Z4C_UNROLL_T
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL_T
    for (int d = 0; d < 3; ++d) Dda_s += guu[sid(c, d)] * dphi[c] * v.dalpha[d];
  T Dda_dd[6];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      T x = v.ddalpha[sid(a, b)] - 2. * (dphi[a] * v.dalpha[b] + dphi[b] * v.dalpha[a]) +
            2. * g[sid(a, b)] * Dda_s;
      Z4C_UNROLL_T
      for (int c = 0; c < 3; ++c) x -= Gudd[c][sid(a, b)] * v.dalpha[c];
      Dda_dd[sid(a, b)] = x;
    }
  T Ddalpha = T(0.);
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) Ddalpha += wsym(a, b) * oopsi4 * guu[sid(a, b)] * Dda_dd[sid(a, b)];
  // A contractions (:525-589)
  T A_ud[3][3];
  Z4C_UNROLL_T
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL_T
    for (int b = 0; b < 3; ++b) {
      T s = T(0.);
      Z4C_UNROLL_T
      for (int d = 0; d < 3; ++d) s += guu[sid(c, d)] * A[sid(d, b)];
      A_ud[c][b] = s;
    }
  T AA[6];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      T s = T(0.);
      Z4C_UNROLL_T
      for (int c = 0; c < 3; ++c) s += A[sid(a, c)] * A_ud[c][b];
      AA[sid(a, b)] = s;
    }
  T trAA = T(0.);
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) trAA += wsym(a, b) * guu[sid(a, b)] * AA[sid(a, b)];
  T A_uu[6];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      T s = T(0.);
      Z4C_UNROLL_T
      for (int c = 0; c < 3; ++c) s += guu[sid(b, c)] * A_ud[a][c];
      A_uu[sid(a, b)] = s;
    }
  const double cpow = -6.0 / pw;
  T DA_u[3];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) {
    T s = T(0.);
    Z4C_UNROLL_T
    for (int b = 0; b < 3; ++b) {
      s -= cpow * A_uu[sid(a, b)] * v.dchi[b] * oochi;
      s -= (1. / 3.) * guu[sid(a, b)] * (2. * v.dKhat[b] + v.dTheta[b]);
    }
    Z4C_UNROLL_T
    for (int b = 0; b < 3; ++b)
      Z4C_UNROLL_T
      for (int c = b; c < 3; ++c) s += wsym(b, c) * Gudd[a][sid(b, c)] * A_uu[sid(b, c)];
    DA_u[a] = s;
  }
  // Ricci scalar and Ht (:596-613)
  T R = T(0.);
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) R += wsym(a, b) * oopsi4 * guu[sid(a, b)] * Rsum[sid(a, b)];
  const T Ht = R + (2. / 3.) * (K * K) - trAA;
  // Lie derivatives (:619-687)
  T dbtr = T(0.);
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) dbtr += v.dbeta[a][a];
  T ddbeta_d[3];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) {
    T s = T(0.);
    Z4C_UNROLL_T
    for (int b = 0; b < 3; ++b) s += (1. / 3.) * v.ddbeta[b][sid(a, b)];
    ddbeta_d[a] = s;
  }
  const T Lchi = v.lv[Z4C_CHI] + (1. / 6.) * pw * chi_g * dbtr;
  T LGam[3];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) {
    T x = v.lv[Z4C_GAMX + a];
    x += (2. / 3.) * Gu[a] * dbtr;
    Z4C_UNROLL_T
    for (int b = 0; b < 3; ++b) {
      x += guu[sid(a, b)] * ddbeta_d[b] - Gu[b] * v.dbeta[b][a];
      Z4C_UNROLL_T
      for (int c = b; c < 3; ++c) x += wsym(b, c) * guu[sid(b, c)] * v.ddbeta[a][sid(b, c)];
    }
    LGam[a] = x;
  }
  T Lg[6], LA[6];
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      T lg = v.lv[Z4C_GXX + sid(a, b)], la = v.lv[Z4C_AXX + sid(a, b)];
      lg -= (2. / 3.) * g[sid(a, b)] * dbtr;
      la -= (2. / 3.) * A[sid(a, b)] * dbtr;
      Z4C_UNROLL_T
      for (int c = 0; c < 3; ++c) {
        lg += v.dbeta[a][c] * g[sid(b, c)];
        la += v.dbeta[b][c] * A[sid(a, c)];
        lg += v.dbeta[b][c] * g[sid(a, c)];
        la += v.dbeta[a][c] * A[sid(b, c)];
      }
      Lg[sid(a, b)] = lg;
      LA[sid(a, b)] = la;
    }
  // assemble (:694-902)
  const double k1 = opt.damp_kappa1, k2 = opt.damp_kappa2;
  out[Z4C_KHAT] = -Ddalpha + alpha * (trAA + (1. / 3.) * (K * K)) + v.lv[Z4C_KHAT] +
                  k1 * (1 - k2) * alpha * Theta;
  out[Z4C_CHI] = Lchi - (1. / 6.) * pw * chi_g * alpha * K;
  out[Z4C_THETA] = v.lv[Z4C_THETA] + alpha * (0.5 * Ht - (2. + k2) * k1 * Theta);
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) {
    T x = 2. * alpha * DA_u[a] + LGam[a];
    x -= 2. * alpha * k1 * (v.u[Z4C_GAMX + a] - Gu[a]);
    Z4C_UNROLL_T
    for (int b = 0; b < 3; ++b) x -= 2. * A_uu[sid(a, b)] * v.dalpha[b];
    out[Z4C_GAMX + a] = x;
  }
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL_T
    for (int b = a; b < 3; ++b) {
      const int q = sid(a, b);
      out[Z4C_GXX + q] = -2. * alpha * A[q] + Lg[q];
      T x = oopsi4 * (-Dda_dd[q] + alpha * Rsum[q]);
      x -= (1. / 3.) * g[q] * (-Ddalpha + alpha * R);
      x += alpha * (K * A[q] - 2. * AA[q]);
      x += LA[q];
      out[Z4C_AXX + q] = x;
    }
  {
    const T fl = opt.lapse_oplog * opt.lapse_harmonicf + opt.lapse_harmonic * alpha;
    out[Z4C_ALPHA] = opt.lapse_advect * v.lv[Z4C_ALPHA] -
                     fl * alpha * (Khat + 2. * opt.lapse_K * Theta);
  }
  Z4C_UNROLL_T
  for (int a = 0; a < 3; ++a) {
    const T gam = v.u[Z4C_GAMX + a];
    T x = opt.shift_Gamma * gam + opt.shift_advect * v.lv[Z4C_BETAX + a];
    if (fabs(opt.shift_alpha2Gamma) > 0.0) x += opt.shift_alpha2Gamma * (alpha * alpha) * gam;
    if (fabs(opt.shift_H) > 0.0)
      Z4C_UNROLL_T
      for (int b = 0; b < 3; ++b)
        x += opt.shift_H * alpha * chi_g * (0.5 * alpha * v.dchi[b] - v.dalpha[b]) * guu[sid(a, b)];
    x -= opt.shift_eta * v.u[Z4C_BETAX + a];
    out[Z4C_BETAX + a] = x;
  }
}

template <class T>
Z4C_HD void rhs_local(const z4c_params_t& opt, const RhsLocal<T>& v, T out[NV]) {
  T Rsum[6];
  ricci_local(opt, v, Rsum);
  main_local(opt, v, Rsum, out);
}

// Coefficient with which the advection sum of variable n enters its
// right-hand side (1, or lapse_advect, shift_advect).
Z4C_HD double adv_coef(const z4c_params_t& opt, int n) {
  if (n == Z4C_ALPHA) return opt.lapse_advect;
  if (n >= Z4C_BETAX) return opt.shift_advect;
  return 1.0;
}


// ---- reverse sweeps of the right-hand side --------------------------------
// Christoffel symbols: bars of guu, Gd, Gudd, Gu into g~ and its stored first
// derivatives.  The bars are consumed (left modified).
Z4C_HD void christoffel_adj(const RhsLocal<double>& v, const double guu[6],
                            const double Gd[3][6], const double Gudd[3][6], double guub[6],
                            double Gdb[3][6], double Guddb[3][6], const double Gub[3],
                            RhsLocal<double>& vb) {
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b)
      Z4C_UNROLL
      for (int c = b; c < 3; ++c) {
        guub[sid(b, c)] += wsym(b, c) * Gudd[a][sid(b, c)] * Gub[a];
        Guddb[a][sid(b, c)] += wsym(b, c) * guu[sid(b, c)] * Gub[a];
      }
  Z4C_UNROLL
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL
    for (int a = 0; a < 3; ++a)
      Z4C_UNROLL
      for (int b = a; b < 3; ++b) {
        const double X = Guddb[c][sid(a, b)];
        Z4C_UNROLL
        for (int d = 0; d < 3; ++d) {
          guub[sid(c, d)] += Gd[d][sid(a, b)] * X;
          Gdb[d][sid(a, b)] += guu[sid(c, d)] * X;
        }
      }
  Z4C_UNROLL
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL
    for (int a = 0; a < 3; ++a)
      Z4C_UNROLL
      for (int b = a; b < 3; ++b) {
        const double X = 0.5 * Gdb[c][sid(a, b)];
        vb.dg[a][sid(b, c)] += X;
        vb.dg[b][sid(a, c)] += X;
        vb.dg[c][sid(a, b)] -= X;
      }
  inv3s_adj(guu, guub, vb.u + Z4C_GXX);
}

// Reverse of ricci_local: Rsb = adjoint of Rsum_ab (six stored pairs).
// chr_bar (may be null): adjoints of the Christoffel quantities from the
// main algebra's reverse (guu 6, Gamma^c_ab 18, Gamma^a 3), added before the
// Christoffel reverse runs once for both parts.
Z4C_HD void ricci_local_adj(const z4c_params_t& opt, const RhsLocal<double>& v,
                            const double Rsb[6], RhsLocal<double>& vb,
                            const double* chr_bar = nullptr) {
  double guu[6], Gd[3][6], Gudd[3][6], Gu[3];
  christoffel_local(v, guu, Gd, Gudd, Gu);
  const double* g = v.u + Z4C_GXX;
  const double chi = v.u[Z4C_CHI];
  const double chi_g = ad_max_c(chi, opt.chi_div_floor);
  const double oochi = 1.0 / chi_g;
  const double pw = opt.chi_psi_power, ooc = 1.0 / pw;
  double dphi[3];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) dphi[a] = v.dchi[a] * oochi * ooc;
  double Ddphi[6];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      double x = v.ddchi[sid(a, b)] * oochi * ooc - pw * dphi[a] * dphi[b];
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) x -= Gudd[c][sid(a, b)] * dphi[c];
      Ddphi[sid(a, b)] = x;
    }
  double Stmp = 0.;
  Z4C_UNROLL
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL
    for (int d = c; d < 3; ++d)
      Stmp += wsym(c, d) * guu[sid(c, d)] * (Ddphi[sid(c, d)] + 2. * dphi[c] * dphi[d]);

  double guub[6] = {0, 0, 0, 0, 0, 0}, Gdb[3][6] = {}, Guddb[3][6] = {}, Gub[3] = {0, 0, 0};
  double Rddb[6], dphib[3] = {0, 0, 0}, Ddphib[6] = {0, 0, 0, 0, 0, 0}, Stmpb = 0., oochib = 0.;
  // Rsum = Rdd + 4 dphi dphi - 2 Ddphi - 2 g Stmp
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const int q = sid(a, b);
      const double X = Rsb[q];
      Rddb[q] = X;
      dphib[a] += 4. * dphi[b] * X;
      dphib[b] += 4. * dphi[a] * X;
      Ddphib[q] -= 2. * X;
      vb.u[Z4C_GXX + q] -= 2. * Stmp * X;
      Stmpb -= 2. * g[q] * X;
    }
  Z4C_UNROLL
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL
    for (int d = c; d < 3; ++d) {
      const int q = sid(c, d);
      const double w = wsym(c, d);
      guub[q] += w * (Ddphi[q] + 2. * dphi[c] * dphi[d]) * Stmpb;
      Ddphib[q] += w * guu[q] * Stmpb;
      dphib[c] += w * guu[q] * 2. * dphi[d] * Stmpb;
      dphib[d] += w * guu[q] * 2. * dphi[c] * Stmpb;
    }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const int q = sid(a, b);
      const double X = Ddphib[q];
      vb.ddchi[q] += oochi * ooc * X;
      oochib += v.ddchi[q] * ooc * X;
      dphib[a] -= pw * dphi[b] * X;
      dphib[b] -= pw * dphi[a] * X;
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) {
        Guddb[c][q] -= dphi[c] * X;
        dphib[c] -= Gudd[c][q] * X;
      }
    }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) {
    vb.dchi[a] += oochi * ooc * dphib[a];
    oochib += v.dchi[a] * ooc * dphib[a];
  }
  {
    const double chigb = -oochi * oochi * oochib;
    if (!(chi < opt.chi_div_floor)) vb.u[Z4C_CHI] += chigb;
  }
  // the three groups of R_ab, each linear in Rdd
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const double X = Rddb[sid(a, b)];
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c)
        Z4C_UNROLL
        for (int d = 0; d < 3; ++d) {
          const double gcd = guu[sid(c, d)];
          double t = 0.;
          Z4C_UNROLL
          for (int e = 0; e < 3; ++e) {
            const double g1 = Gudd[e][sid(c, a)], d1 = Gd[b][sid(e, d)];
            const double g2 = Gudd[e][sid(c, b)], d2 = Gd[a][sid(e, d)];
            const double g3 = Gudd[e][sid(a, d)], d3 = Gd[e][sid(c, b)];
            t += g1 * d1 + g2 * d2 + g3 * d3;
            Guddb[e][sid(c, a)] += gcd * d1 * X;
            Gdb[b][sid(e, d)] += gcd * g1 * X;
            Guddb[e][sid(c, b)] += gcd * d2 * X;
            Gdb[a][sid(e, d)] += gcd * g2 * X;
            Guddb[e][sid(a, d)] += gcd * d3 * X;
            Gdb[e][sid(c, b)] += gcd * g3 * X;
          }
          guub[sid(c, d)] += t * X;
        }
    }
  Z4C_UNROLL
  for (int q = 0; q < 6; ++q) {
    const double X = Rddb[q];
    Z4C_UNROLL
    for (int c = 0; c < 3; ++c)
      Z4C_UNROLL
      for (int d = c; d < 3; ++d) {
        const double w = (c == d) ? 0.5 : 1.0;
        guub[sid(c, d)] -= w * v.ddg[q][sid(c, d)] * X;
        vb.ddg[q][sid(c, d)] -= w * guu[sid(c, d)] * X;
      }
  }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const double X = 0.5 * Rddb[sid(a, b)];
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) {
        vb.u[Z4C_GXX + sid(c, a)] += v.dGam[b][c] * X;
        vb.dGam[b][c] += g[sid(c, a)] * X;
        vb.u[Z4C_GXX + sid(c, b)] += v.dGam[a][c] * X;
        vb.dGam[a][c] += g[sid(c, b)] * X;
        Gub[c] += (Gd[a][sid(b, c)] + Gd[b][sid(a, c)]) * X;
        Gdb[a][sid(b, c)] += Gu[c] * X;
        Gdb[b][sid(a, c)] += Gu[c] * X;
      }
    }
  if (chr_bar) {
Z4C_UNROLL
    for (int q = 0; q < 6; ++q) guub[q] += chr_bar[q];
Z4C_UNROLL
    for (int c = 0; c < 3; ++c)
Z4C_UNROLL
      for (int q = 0; q < 6; ++q) Guddb[c][q] += chr_bar[6 + c * 6 + q];
Z4C_UNROLL
    for (int a = 0; a < 3; ++a) Gub[a] += chr_bar[24 + a];
  }
  christoffel_adj(v, guu, Gd, Gudd, guub, Gdb, Guddb, Gub, vb);
}

// Reverse of main_local: ob = adjoint of the 22 outputs; accumulates into vb,
// into Rsb (adjoint of Rsum) and into the parameter adjoints pb.  With
// chr_bar non-null the adjoints of the Christoffel quantities (guu 6,
// Gamma^c_ab 18, Gamma^a 3) are written there instead of being reversed into
// g~ and its derivatives (ricci_local_adj takes them up).
Z4C_HD void main_local_adj(const z4c_params_t& opt, const RhsLocal<double>& v,
                           const double Rsum[6], const double ob[NV], RhsLocal<double>& vb,
                           double Rsb[6], ParamBar& pb, double* chr_bar = nullptr) {
  double guu[6], Gd[3][6], Gudd[3][6], Gu[3];
  christoffel_local(v, guu, Gd, Gudd, Gu);
  const double* g = v.u + Z4C_GXX;
  const double* A = v.u + Z4C_AXX;
  const double chi = v.u[Z4C_CHI], Khat = v.u[Z4C_KHAT], Theta = v.u[Z4C_THETA];
  const double alpha = v.u[Z4C_ALPHA];
  const double pw = opt.chi_psi_power, ooc = 1.0 / pw;
  const double K = Khat + 2. * Theta;
  const double chi_g = ad_max_c(chi, opt.chi_div_floor);
  const double oochi = 1.0 / chi_g;
  const double oopsi4 = (pw == -4.) ? chi_g : pow(chi_g, -4. / pw);
  double dphi[3];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) dphi[a] = v.dchi[a] * oochi * ooc;
  double Dda_s = 0.;
  Z4C_UNROLL
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL
    for (int d = 0; d < 3; ++d) Dda_s += guu[sid(c, d)] * dphi[c] * v.dalpha[d];
  double Dda_dd[6];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      double x = v.ddalpha[sid(a, b)] - 2. * (dphi[a] * v.dalpha[b] + dphi[b] * v.dalpha[a]) +
                 2. * g[sid(a, b)] * Dda_s;
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) x -= Gudd[c][sid(a, b)] * v.dalpha[c];
      Dda_dd[sid(a, b)] = x;
    }
  double Ddalpha = 0.;
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) Ddalpha += wsym(a, b) * oopsi4 * guu[sid(a, b)] * Dda_dd[sid(a, b)];
  double A_ud[3][3];
  Z4C_UNROLL
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b) {
      double s = 0.;
      Z4C_UNROLL
      for (int d = 0; d < 3; ++d) s += guu[sid(c, d)] * A[sid(d, b)];
      A_ud[c][b] = s;
    }
  double AA[6];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      double s = 0.;
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) s += A[sid(a, c)] * A_ud[c][b];
      AA[sid(a, b)] = s;
    }
  double trAA = 0.;
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) trAA += wsym(a, b) * guu[sid(a, b)] * AA[sid(a, b)];
  double A_uu[6];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      double s = 0.;
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) s += guu[sid(b, c)] * A_ud[a][c];
      A_uu[sid(a, b)] = s;
    }
  const double cpow = -6.0 / pw;
  double DA_u[3];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) {
    double s = 0.;
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b) {
      s -= cpow * A_uu[sid(a, b)] * v.dchi[b] * oochi;
      s -= (1. / 3.) * guu[sid(a, b)] * (2. * v.dKhat[b] + v.dTheta[b]);
    }
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b)
      Z4C_UNROLL
      for (int c = b; c < 3; ++c) s += wsym(b, c) * Gudd[a][sid(b, c)] * A_uu[sid(b, c)];
    DA_u[a] = s;
  }
  double R = 0.;
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) R += wsym(a, b) * oopsi4 * guu[sid(a, b)] * Rsum[sid(a, b)];
  const double Ht = R + (2. / 3.) * (K * K) - trAA;
  double dbtr = 0.;
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) dbtr += v.dbeta[a][a];
  double ddbeta_d[3];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) {
    double s = 0.;
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b) s += (1. / 3.) * v.ddbeta[b][sid(a, b)];
    ddbeta_d[a] = s;
  }

  // adjoints of the intermediates
  double guub[6] = {0, 0, 0, 0, 0, 0}, Gdb[3][6] = {}, Guddb[3][6] = {}, Gub[3] = {0, 0, 0};
  double Kb = 0., chigb = 0., oochib = 0., oopsi4b = 0., alphab = 0.;
  double dphib[3] = {0, 0, 0}, Dda_sb = 0., Dda_ddb[6] = {0, 0, 0, 0, 0, 0}, Ddalphab = 0.;
  double A_udb[3][3] = {}, AAb[6] = {0, 0, 0, 0, 0, 0}, trAAb = 0., A_uub[6] = {0, 0, 0, 0, 0, 0};
  double DAb[3] = {0, 0, 0}, Rb = 0., Htb = 0., dbtrb = 0., ddbeta_db[3] = {0, 0, 0};
  double Lchib = 0., LGamb[3] = {0, 0, 0}, Lgb[6] = {0, 0, 0, 0, 0, 0}, LAb[6] = {0, 0, 0, 0, 0, 0};
  const double k1 = opt.damp_kappa1, k2 = opt.damp_kappa2;

  // assemble (:694-902), each output in turn
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) {
    const double X = ob[Z4C_BETAX + a];
    const double gam = v.u[Z4C_GAMX + a];
    vb.u[Z4C_GAMX + a] += opt.shift_Gamma * X;
    vb.lv[Z4C_BETAX + a] += opt.shift_advect * X;
    if (fabs(opt.shift_alpha2Gamma) > 0.0) {
      vb.u[Z4C_GAMX + a] += opt.shift_alpha2Gamma * (alpha * alpha) * X;
      alphab += opt.shift_alpha2Gamma * 2. * alpha * gam * X;
    }
    if (fabs(opt.shift_H) > 0.0)
      Z4C_UNROLL
      for (int b = 0; b < 3; ++b) {
        const double gab = guu[sid(a, b)];
        const double in = 0.5 * alpha * v.dchi[b] - v.dalpha[b];
        const double Y = opt.shift_H * X;
        alphab += Y * (chi_g * in * gab + alpha * chi_g * 0.5 * v.dchi[b] * gab);
        chigb += Y * alpha * in * gab;
        vb.dchi[b] += Y * alpha * chi_g * 0.5 * alpha * gab;
        vb.dalpha[b] -= Y * alpha * chi_g * gab;
        guub[sid(a, b)] += Y * alpha * chi_g * in;
      }
    vb.u[Z4C_BETAX + a] -= opt.shift_eta * X;
    pb.shift_eta -= v.u[Z4C_BETAX + a] * X;
  }
  {
    const double X = ob[Z4C_ALPHA];
    const double fl = opt.lapse_oplog * opt.lapse_harmonicf + opt.lapse_harmonic * alpha;
    const double Pk = Khat + 2. * opt.lapse_K * Theta;
    vb.lv[Z4C_ALPHA] += opt.lapse_advect * X;
    alphab -= (fl + opt.lapse_harmonic * alpha) * Pk * X;
    vb.u[Z4C_KHAT] -= fl * alpha * X;
    vb.u[Z4C_THETA] -= fl * alpha * 2. * opt.lapse_K * X;
  }
  Z4C_UNROLL
  for (int q = 0; q < 6; ++q) {
    const double X = ob[Z4C_AXX + q];
    oopsi4b += (-Dda_dd[q] + alpha * Rsum[q]) * X;
    Dda_ddb[q] -= oopsi4 * X;
    alphab += oopsi4 * Rsum[q] * X;
    Rsb[q] += oopsi4 * alpha * X;
    vb.u[Z4C_GXX + q] -= (1. / 3.) * (-Ddalpha + alpha * R) * X;
    Ddalphab += (1. / 3.) * g[q] * X;
    alphab -= (1. / 3.) * g[q] * R * X;
    Rb -= (1. / 3.) * g[q] * alpha * X;
    alphab += (K * A[q] - 2. * AA[q]) * X;
    Kb += alpha * A[q] * X;
    vb.u[Z4C_AXX + q] += alpha * K * X;
    AAb[q] -= 2. * alpha * X;
    LAb[q] += X;
    const double Y = ob[Z4C_GXX + q];
    alphab -= 2. * A[q] * Y;
    vb.u[Z4C_AXX + q] -= 2. * alpha * Y;
    Lgb[q] += Y;
  }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) {
    const double X = ob[Z4C_GAMX + a];
    const double gam = v.u[Z4C_GAMX + a];
    alphab += 2. * DA_u[a] * X;
    DAb[a] += 2. * alpha * X;
    LGamb[a] += X;
    alphab -= 2. * k1 * (gam - Gu[a]) * X;
    vb.u[Z4C_GAMX + a] -= 2. * alpha * k1 * X;
    Gub[a] += 2. * alpha * k1 * X;
    pb.damp_kappa1 -= 2. * alpha * (gam - Gu[a]) * X;
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b) {
      A_uub[sid(a, b)] -= 2. * v.dalpha[b] * X;
      vb.dalpha[b] -= 2. * A_uu[sid(a, b)] * X;
    }
  }
  {
    const double X = ob[Z4C_THETA];
    vb.lv[Z4C_THETA] += X;
    alphab += (0.5 * Ht - (2. + k2) * k1 * Theta) * X;
    Htb += 0.5 * alpha * X;
    vb.u[Z4C_THETA] -= alpha * (2. + k2) * k1 * X;
    pb.damp_kappa1 -= alpha * (2. + k2) * Theta * X;
  }
  {
    const double X = ob[Z4C_CHI];
    Lchib += X;
    chigb -= (1. / 6.) * pw * alpha * K * X;
    alphab -= (1. / 6.) * pw * chi_g * K * X;
    Kb -= (1. / 6.) * pw * chi_g * alpha * X;
  }
  {
    const double X = ob[Z4C_KHAT];
    Ddalphab -= X;
    alphab += (trAA + (1. / 3.) * (K * K) + k1 * (1 - k2) * Theta) * X;
    trAAb += alpha * X;
    Kb += alpha * (2. / 3.) * K * X;
    vb.lv[Z4C_KHAT] += X;
    vb.u[Z4C_THETA] += k1 * (1 - k2) * alpha * X;
    pb.damp_kappa1 += (1 - k2) * alpha * Theta * X;
  }
  // Lie derivatives (:619-687)
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const int q = sid(a, b);
      const double XG = Lgb[q], XA = LAb[q];
      vb.lv[Z4C_GXX + q] += XG;
      vb.lv[Z4C_AXX + q] += XA;
      vb.u[Z4C_GXX + q] -= (2. / 3.) * dbtr * XG;
      dbtrb -= (2. / 3.) * g[q] * XG;
      vb.u[Z4C_AXX + q] -= (2. / 3.) * dbtr * XA;
      dbtrb -= (2. / 3.) * A[q] * XA;
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) {
        vb.dbeta[a][c] += g[sid(b, c)] * XG;
        vb.u[Z4C_GXX + sid(b, c)] += v.dbeta[a][c] * XG;
        vb.dbeta[b][c] += A[sid(a, c)] * XA;
        vb.u[Z4C_AXX + sid(a, c)] += v.dbeta[b][c] * XA;
        vb.dbeta[b][c] += g[sid(a, c)] * XG;
        vb.u[Z4C_GXX + sid(a, c)] += v.dbeta[b][c] * XG;
        vb.dbeta[a][c] += A[sid(b, c)] * XA;
        vb.u[Z4C_AXX + sid(b, c)] += v.dbeta[a][c] * XA;
      }
    }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) {
    const double X = LGamb[a];
    vb.lv[Z4C_GAMX + a] += X;
    Gub[a] += (2. / 3.) * dbtr * X;
    dbtrb += (2. / 3.) * Gu[a] * X;
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b) {
      guub[sid(a, b)] += ddbeta_d[b] * X;
      ddbeta_db[b] += guu[sid(a, b)] * X;
      Gub[b] -= v.dbeta[b][a] * X;
      vb.dbeta[b][a] -= Gu[b] * X;
      Z4C_UNROLL
      for (int c = b; c < 3; ++c) {
        guub[sid(b, c)] += wsym(b, c) * v.ddbeta[a][sid(b, c)] * X;
        vb.ddbeta[a][sid(b, c)] += wsym(b, c) * guu[sid(b, c)] * X;
      }
    }
  }
  vb.lv[Z4C_CHI] += Lchib;
  chigb += (1. / 6.) * pw * dbtr * Lchib;
  dbtrb += (1. / 6.) * pw * chi_g * Lchib;
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b) vb.ddbeta[b][sid(a, b)] += (1. / 3.) * ddbeta_db[a];
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) vb.dbeta[a][a] += dbtrb;
  // Ricci scalar and Ht
  Rb += Htb;
  Kb += (4. / 3.) * K * Htb;
  trAAb -= Htb;
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const int q = sid(a, b);
      const double w = wsym(a, b);
      oopsi4b += w * guu[q] * Rsum[q] * Rb;
      guub[q] += w * oopsi4 * Rsum[q] * Rb;
      Rsb[q] += w * oopsi4 * guu[q] * Rb;
    }
  // D_i A^ij
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) {
    const double X = DAb[a];
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b) {
      A_uub[sid(a, b)] -= cpow * v.dchi[b] * oochi * X;
      vb.dchi[b] -= cpow * A_uu[sid(a, b)] * oochi * X;
      oochib -= cpow * A_uu[sid(a, b)] * v.dchi[b] * X;
      guub[sid(a, b)] -= (1. / 3.) * (2. * v.dKhat[b] + v.dTheta[b]) * X;
      vb.dKhat[b] -= (2. / 3.) * guu[sid(a, b)] * X;
      vb.dTheta[b] -= (1. / 3.) * guu[sid(a, b)] * X;
    }
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b)
      Z4C_UNROLL
      for (int c = b; c < 3; ++c) {
        Guddb[a][sid(b, c)] += wsym(b, c) * A_uu[sid(b, c)] * X;
        A_uub[sid(b, c)] += wsym(b, c) * Gudd[a][sid(b, c)] * X;
      }
  }
  // A contractions
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const double X = A_uub[sid(a, b)];
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) {
        guub[sid(b, c)] += A_ud[a][c] * X;
        A_udb[a][c] += guu[sid(b, c)] * X;
      }
    }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const int q = sid(a, b);
      guub[q] += wsym(a, b) * AA[q] * trAAb;
      AAb[q] += wsym(a, b) * guu[q] * trAAb;
    }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const double X = AAb[sid(a, b)];
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) {
        vb.u[Z4C_AXX + sid(a, c)] += A_ud[c][b] * X;
        A_udb[c][b] += A[sid(a, c)] * X;
      }
    }
  Z4C_UNROLL
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL
    for (int b = 0; b < 3; ++b) {
      const double X = A_udb[c][b];
      Z4C_UNROLL
      for (int d = 0; d < 3; ++d) {
        guub[sid(c, d)] += A[sid(d, b)] * X;
        vb.u[Z4C_AXX + sid(d, b)] += guu[sid(c, d)] * X;
      }
    }
  // D D alpha
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const int q = sid(a, b);
      const double w = wsym(a, b);
      oopsi4b += w * guu[q] * Dda_dd[q] * Ddalphab;
      guub[q] += w * oopsi4 * Dda_dd[q] * Ddalphab;
      Dda_ddb[q] += w * oopsi4 * guu[q] * Ddalphab;
    }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a)
    Z4C_UNROLL
    for (int b = a; b < 3; ++b) {
      const int q = sid(a, b);
      const double X = Dda_ddb[q];
      vb.ddalpha[q] += X;
      dphib[a] -= 2. * v.dalpha[b] * X;
      vb.dalpha[b] -= 2. * dphi[a] * X;
      dphib[b] -= 2. * v.dalpha[a] * X;
      vb.dalpha[a] -= 2. * dphi[b] * X;
      vb.u[Z4C_GXX + q] += 2. * Dda_s * X;
      Dda_sb += 2. * g[q] * X;
      Z4C_UNROLL
      for (int c = 0; c < 3; ++c) {
        Guddb[c][q] -= v.dalpha[c] * X;
        vb.dalpha[c] -= Gudd[c][q] * X;
      }
    }
  Z4C_UNROLL
  for (int c = 0; c < 3; ++c)
    Z4C_UNROLL
    for (int d = 0; d < 3; ++d) {
      const double gcd = guu[sid(c, d)];
      guub[sid(c, d)] += dphi[c] * v.dalpha[d] * Dda_sb;
      dphib[c] += gcd * v.dalpha[d] * Dda_sb;
      vb.dalpha[d] += gcd * dphi[c] * Dda_sb;
    }
  Z4C_UNROLL
  for (int a = 0; a < 3; ++a) {
    vb.dchi[a] += oochi * ooc * dphib[a];
    oochib += v.dchi[a] * ooc * dphib[a];
  }
  chigb += (pw == -4.) ? oopsi4b : (-4. / pw) * pow(chi_g, -4. / pw - 1.) * oopsi4b;
  chigb -= oochi * oochi * oochib;
  if (!(chi < opt.chi_div_floor)) vb.u[Z4C_CHI] += chigb;
  vb.u[Z4C_ALPHA] += alphab;
  vb.u[Z4C_KHAT] += Kb;
  vb.u[Z4C_THETA] += 2. * Kb;
  if (chr_bar) {
Z4C_UNROLL
    for (int q = 0; q < 6; ++q) chr_bar[q] = guub[q];
Z4C_UNROLL
    for (int c = 0; c < 3; ++c)
Z4C_UNROLL
      for (int q = 0; q < 6; ++q) chr_bar[6 + c * 6 + q] = Guddb[c][q];
Z4C_UNROLL
    for (int a = 0; a < 3; ++a) chr_bar[24 + a] = Gub[a];
    return;
  }
  christoffel_adj(v, guu, Gd, Gudd, guub, Gdb, Guddb, Gub, vb);
}

// ---- AlgConstr (z4c.cpp:677-799) --------------------------------------------
// trace_rank2 with detginv = 1: P(g, A) = adj(g) : A, the cofactor contraction
template <class T>
Z4C_HD T trace_adj(const T* g, const T* A) {
  const T gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
  const T Axx = A[0], Axy = A[1], Axz = A[2], Ayy = A[3], Ayz = A[4], Azz = A[5];
  return 1.0 * (-2. * Ayz * gxx * gyz + Axx * gyy * gzz + gxx * (Azz * gyy + Ayy * gzz) +
                2. * (gxz * (Ayz * gxy - Axz * gyy + Axy * gyz) + gxy * (Axz * gyz - Axy * gzz)) -
                Azz * (gxy * gxy) - Ayy * (gxz * gxz) - Axx * (gyz * gyz));
}
Z4C_HD void trace_adj_grad(const double* g, const double* A, double* dg, double* dA) {
  const double gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
  const double Axx = A[0], Axy = A[1], Axz = A[2], Ayy = A[3], Ayz = A[4], Azz = A[5];
  dA[0] = gyy * gzz - gyz * gyz;
  dA[1] = 2. * (gxz * gyz - gxy * gzz);
  dA[2] = 2. * (gxy * gyz - gxz * gyy);
  dA[3] = gxx * gzz - gxz * gxz;
  dA[4] = 2. * (gxz * gxy - gxx * gyz);
  dA[5] = gxx * gyy - gxy * gxy;
  dg[0] = -2. * Ayz * gyz + Azz * gyy + Ayy * gzz;
  dg[1] = 2. * gxz * Ayz + 2. * (Axz * gyz - Axy * gzz) - 2. * Azz * gxy;
  dg[2] = 2. * (Ayz * gxy - Axz * gyy + Axy * gyz) - 2. * Ayy * gxz;
  dg[3] = Axx * gzz + gxx * Azz - 2. * gxz * Axz;
  dg[4] = -2. * Ayz * gxx + 2. * gxz * Axy + 2. * gxy * Axz - 2. * Axx * gyz;
  dg[5] = Axx * gyy + gxx * Ayy - 2. * gxy * Axy;
}
// AlgConstr on the 22 values of one vertex, in place.
template <class T>
Z4C_HD void alg_constr_local(const z4c_params_t& opt, T* u) {
  T* g = u + Z4C_GXX;
  T* A = u + Z4C_AXX;
  bool apply = true;
  T detg = det3s(g);
  if (opt.tf_force_regularization) {
    if (!(detg > 0.)) detg = T(1.);
  } else {
    apply = detg > opt.eps_floor;
  }
  if (apply) {
    const T oopsi4 = ((val(detg) - 1.0) < opt.eps_floor) ? T(1.0 + opt.eps_floor / -3.0)
                                                         : ad_pow(detg, 1.0 / -3.0);
    Z4C_UNROLL_T
    for (int c = 0; c < 6; ++c) g[c] = g[c] * oopsi4;
    const T tr = trace_adj(g, A);
    Z4C_UNROLL_T
    for (int c = 0; c < 6; ++c) A[c] = A[c] - (1.0 / 3.0) * tr * g[c];
  }
  if (opt.force_regularization) {
    u[Z4C_CHI] = ad_max_c(u[Z4C_CHI], opt.eps_floor);
    const double a = val(u[Z4C_ALPHA]);
    if (a >= 0 ? a < opt.eps_floor : a > -opt.eps_floor)
      u[Z4C_ALPHA] = T(a >= 0 ? opt.eps_floor : -opt.eps_floor);
  }
}
// Reverse: u is the vertex's state BEFORE AlgConstr; ub holds the adjoint of
// the state after it and is overwritten by the adjoint of the state before.
Z4C_HD void alg_constr_adj(const z4c_params_t& opt, const double* u, double* ub) {
  if (opt.force_regularization) {
    if (u[Z4C_CHI] < opt.eps_floor) ub[Z4C_CHI] = 0.;
    const double a = u[Z4C_ALPHA];
    if (a >= 0 ? a < opt.eps_floor : a > -opt.eps_floor) ub[Z4C_ALPHA] = 0.;
  }
  const double* g0 = u + Z4C_GXX;
  const double* A0 = u + Z4C_AXX;
  const double detraw = det3s(g0);
  double detg = detraw;
  bool apply = true, det_live = true;
  if (opt.tf_force_regularization) {
    if (!(detg > 0.)) {
      detg = 1.;
      det_live = false;
    }
  } else {
    apply = detg > opt.eps_floor;
  }
  if (!apply) return;
  const bool pow_branch = !((detg - 1.0) < opt.eps_floor);
  const double oopsi4 = pow_branch ? pow(detg, 1.0 / -3.0) : 1.0 + opt.eps_floor / -3.0;
  double g[6];
  Z4C_UNROLL
  for (int c = 0; c < 6; ++c) g[c] = g0[c] * oopsi4;
  const double tr = trace_adj(g, A0);
  double* gb = ub + Z4C_GXX;
  double* Ab = ub + Z4C_AXX;
  // A' = A - tr g' / 3
  double trb = 0., gpb[6];
  Z4C_UNROLL
  for (int c = 0; c < 6; ++c) {
    trb -= (1.0 / 3.0) * g[c] * Ab[c];
    gpb[c] = gb[c] - (1.0 / 3.0) * tr * Ab[c];
  }
  double dPg[6], dPA[6];
  trace_adj_grad(g, A0, dPg, dPA);
  Z4C_UNROLL
  for (int c = 0; c < 6; ++c) {
    gpb[c] += trb * dPg[c];
    Ab[c] += trb * dPA[c];
  }
  // g' = g oopsi4
  double oopsi4b = 0.;
  Z4C_UNROLL
  for (int c = 0; c < 6; ++c) {
    oopsi4b += g0[c] * gpb[c];
    gb[c] = oopsi4 * gpb[c];
  }
  if (pow_branch && det_live) {
    const double detb = oopsi4b * (-1.0 / 3.0) * pow(detg, -1.0 / 3.0 - 1.0);
    double dd[6];
    det3s_grad(g0, dd);
    Z4C_UNROLL
    for (int c = 0; c < 6; ++c) gb[c] += detb * dd[c];
  }
  (void)detraw;
}

// ---- Z4cToADM and the Hamiltonian constraint --------------------------------
// Local inputs of H at one interior vertex.
template <class T>
struct HLocal {
  T chi, gt[6], At[6], Khat, Theta;  // Z4c variables at the vertex
  T dchi[3];       // centred d_a chi
  T dg3[3][6];     // centred d_c g~_q  [c][q]
  T ddchi[6];      // d_a d_b chi: Dxx on the diagonal, the two-dimensional Dxy off it
  T ddg[6][6];     // d_a d_b g~_q  [q][pair(a,b)]
  static constexpr int N = 1 + 6 + 6 + 1 + 1 + 3 + 18 + 6 + 36;
  Z4C_HD T* data() { return &chi; }
  Z4C_HD const T* data() const { return &chi; }
};

// H = R + K^2 - K_ij K^ij of ADMConstraints (adm_z4c.cpp:382-760) with the ADM
// metric and curvature of Z4cToADM (adm_z4c.cpp:200-260) at the vertex;
// chi_psi_power = -4.
template <class T>
Z4C_HD T ham_local(const z4c_params_t& opt, const HLocal<T>& v) {
  const T psi4 = T(1.0) / v.chi;
  T gph[6], Kd[6];
    for (int c = 0; c < 6; ++c) gph[c] = psi4 * v.gt[c];
    for (int c = 0; c < 6; ++c) Kd[c] = psi4 * v.At[c] + (1. / 3.) * (v.Khat + 2. * v.Theta) * gph[c];
  const T chi_g = ad_max_c(v.chi, opt.chi_div_floor);
  const T oochi = T(1.0) / chi_g;
  T dg[3][6];
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 6; ++q) dg[c][q] = oochi * (v.dg3[c][q] - oochi * v.gt[q] * v.dchi[c]);
  T guu[6];
  {
    const T detg = det3s(gph);
    inv3s(T(1.) / detg, gph, guu);
  }
  T Gddd[3][6], Gudd[3][6];
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b)
        Gddd[c][sid(a, b)] = 0.5 * (dg[a][sid(b, c)] + dg[b][sid(a, c)] - dg[c][sid(a, b)]);
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b) {
        T acc = T(0.);
                for (int d = 0; d < 3; ++d) acc += guu[sid(c, d)] * Gddd[d][sid(a, b)];
        Gudd[c][sid(a, b)] = acc;
      }
  T DDG[6][6];  // [pair(a,b) of the derivatives][pair(c,d) of the metric]
    for (int a = 0; a < 3; ++a)
        for (int b = a; b < 3; ++b)
            for (int q = 0; q < 6; ++q) {
        const T gtil = v.gt[q];
        const T ddchi = v.ddchi[sid(a, b)];
        const T ddgc = v.ddg[q][sid(a, b)];
        if (a == b)
          DDG[sid(a, b)][q] = oochi * (ddgc - oochi * (2.0 * v.dchi[a] * v.dg3[a][q] + ddchi * gtil) +
                                       2.0 * oochi * oochi * v.dchi[a] * v.dchi[a] * gtil);
        else
          DDG[sid(a, b)][q] =
              oochi * (ddgc - oochi * (v.dchi[a] * v.dg3[b][q] + v.dchi[b] * v.dg3[a][q] + ddchi * gtil) +
                       2.0 * oochi * oochi * v.dchi[a] * v.dchi[b] * gtil);
      }
  T R = T(0.);
    for (int a = 0; a < 3; ++a)
        for (int b = a; b < 3; ++b) {
      T acc = T(0.);
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d)
                    for (int f = 0; f < 3; ++f)
            acc += guu[sid(d, f)] * (Gudd[c][sid(a, f)] * Gddd[c][sid(b, d)] -
                                     Gudd[c][sid(a, b)] * Gddd[c][sid(f, d)]);
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d)
          acc += 0.5 * guu[sid(c, d)] *
                 (-DDG[sid(b, a)][sid(c, d)] + DDG[sid(d, a)][sid(b, c)] +
                  DDG[sid(d, b)][sid(a, c)] - DDG[sid(d, c)][sid(a, b)]);
      R += wsym(a, b) * guu[sid(a, b)] * acc;
    }
  T K = T(0.), K_ud[3][3], KK = T(0.);
    for (int a = 0; a < 3; ++a) {
        for (int b = 0; b < 3; ++b) {
      T acc = T(0.);
            for (int c = 0; c < 3; ++c) acc += guu[sid(a, c)] * Kd[sid(c, b)];
      K_ud[a][b] = acc;
    }
    K += K_ud[a][a];
  }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) KK += K_ud[a][b] * K_ud[b][a];
  return R + (K * K) - KK;
}

// Reverse of ham_local: vb += Hb dH/dv.
Z4C_HD void ham_local_adj(const z4c_params_t& opt, const HLocal<double>& v, double Hb,
                          HLocal<double>& vb) {
  const double psi4 = 1.0 / v.chi;
  double gph[6], Kd[6];
    for (int c = 0; c < 6; ++c) gph[c] = psi4 * v.gt[c];
  const double Kt = v.Khat + 2. * v.Theta;
    for (int c = 0; c < 6; ++c) Kd[c] = psi4 * v.At[c] + (1. / 3.) * Kt * gph[c];
  const double chi_g = ad_max_c(v.chi, opt.chi_div_floor);
  const double oochi = 1.0 / chi_g;
  double dg[3][6];
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 6; ++q) dg[c][q] = oochi * (v.dg3[c][q] - oochi * v.gt[q] * v.dchi[c]);
  double guu[6];
  {
    const double detg = det3s(gph);
    inv3s(1. / detg, gph, guu);
  }
  double Gddd[3][6], Gudd[3][6];
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b)
        Gddd[c][sid(a, b)] = 0.5 * (dg[a][sid(b, c)] + dg[b][sid(a, c)] - dg[c][sid(a, b)]);
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b) {
        double acc = 0.;
                for (int d = 0; d < 3; ++d) acc += guu[sid(c, d)] * Gddd[d][sid(a, b)];
        Gudd[c][sid(a, b)] = acc;
      }
  double DDG[6][6];
    for (int a = 0; a < 3; ++a)
        for (int b = a; b < 3; ++b)
            for (int q = 0; q < 6; ++q) {
        const double gtil = v.gt[q], ddchi = v.ddchi[sid(a, b)], ddgc = v.ddg[q][sid(a, b)];
        if (a == b)
          DDG[sid(a, b)][q] = oochi * (ddgc - oochi * (2.0 * v.dchi[a] * v.dg3[a][q] + ddchi * gtil) +
                                       2.0 * oochi * oochi * v.dchi[a] * v.dchi[a] * gtil);
        else
          DDG[sid(a, b)][q] =
              oochi * (ddgc - oochi * (v.dchi[a] * v.dg3[b][q] + v.dchi[b] * v.dg3[a][q] + ddchi * gtil) +
                       2.0 * oochi * oochi * v.dchi[a] * v.dchi[b] * gtil);
      }
  double K_ud[3][3], K = 0.;
    for (int a = 0; a < 3; ++a) {
        for (int b = 0; b < 3; ++b) {
      double acc = 0.;
            for (int c = 0; c < 3; ++c) acc += guu[sid(a, c)] * Kd[sid(c, b)];
      K_ud[a][b] = acc;
    }
    K += K_ud[a][a];
  }
  // reverse
  double guub[6] = {0, 0, 0, 0, 0, 0}, Gdddb[3][6] = {}, Guddb[3][6] = {}, DDGb[6][6] = {};
  double Kdb[6] = {0, 0, 0, 0, 0, 0}, dgb[3][6] = {}, gphb[6] = {0, 0, 0, 0, 0, 0};
  double oochib = 0., psi4b = 0.;
  const double Rb = Hb, Kb = 2. * K * Hb, KKb = -Hb;
  double K_udb[3][3] = {};
    for (int a = 0; a < 3; ++a) {
    K_udb[a][a] += Kb;
        for (int b = 0; b < 3; ++b) {
      K_udb[a][b] += K_ud[b][a] * KKb;
      K_udb[b][a] += K_ud[a][b] * KKb;
    }
  }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) {
        guub[sid(a, c)] += Kd[sid(c, b)] * K_udb[a][b];
        Kdb[sid(c, b)] += guu[sid(a, c)] * K_udb[a][b];
      }
    for (int a = 0; a < 3; ++a)
        for (int b = a; b < 3; ++b) {
      double acc = 0.;
      const double X = wsym(a, b) * guu[sid(a, b)] * Rb;
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d)
                    for (int f = 0; f < 3; ++f) {
            const double gdf = guu[sid(d, f)];
            const double u1 = Gudd[c][sid(a, f)], d1 = Gddd[c][sid(b, d)];
            const double u2 = Gudd[c][sid(a, b)], d2 = Gddd[c][sid(f, d)];
            acc += gdf * (u1 * d1 - u2 * d2);
            guub[sid(d, f)] += (u1 * d1 - u2 * d2) * X;
            Guddb[c][sid(a, f)] += gdf * d1 * X;
            Gdddb[c][sid(b, d)] += gdf * u1 * X;
            Guddb[c][sid(a, b)] -= gdf * d2 * X;
            Gdddb[c][sid(f, d)] -= gdf * u2 * X;
          }
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d) {
          const double s = -DDG[sid(b, a)][sid(c, d)] + DDG[sid(d, a)][sid(b, c)] +
                           DDG[sid(d, b)][sid(a, c)] - DDG[sid(d, c)][sid(a, b)];
          acc += 0.5 * guu[sid(c, d)] * s;
          guub[sid(c, d)] += 0.5 * s * X;
          const double Y = 0.5 * guu[sid(c, d)] * X;
          DDGb[sid(b, a)][sid(c, d)] -= Y;
          DDGb[sid(d, a)][sid(b, c)] += Y;
          DDGb[sid(d, b)][sid(a, c)] += Y;
          DDGb[sid(d, c)][sid(a, b)] -= Y;
        }
      guub[sid(a, b)] += wsym(a, b) * acc * Rb;
    }
    for (int a = 0; a < 3; ++a)
        for (int b = a; b < 3; ++b)
            for (int q = 0; q < 6; ++q) {
        const double X = DDGb[sid(a, b)][q];
        const double gtil = v.gt[q], ddchi = v.ddchi[sid(a, b)], ddgc = v.ddg[q][sid(a, b)];
        if (a == b) {
          const double da = v.dchi[a], d3 = v.dg3[a][q];
          const double inner = ddgc - oochi * (2.0 * da * d3 + ddchi * gtil) +
                               2.0 * oochi * oochi * da * da * gtil;
          oochib += inner * X;
          const double Y = oochi * X;
          vb.ddg[q][sid(a, b)] += Y;
          oochib -= (2.0 * da * d3 + ddchi * gtil) * Y;
          vb.dchi[a] -= oochi * 2.0 * d3 * Y;
          vb.dg3[a][q] -= oochi * 2.0 * da * Y;
          vb.ddchi[sid(a, b)] -= oochi * gtil * Y;
          vb.gt[q] -= oochi * ddchi * Y;
          oochib += 4.0 * oochi * da * da * gtil * Y;
          vb.dchi[a] += 4.0 * oochi * oochi * da * gtil * Y;
          vb.gt[q] += 2.0 * oochi * oochi * da * da * Y;
        } else {
          const double da = v.dchi[a], db = v.dchi[b];
          const double dga = v.dg3[a][q], dgb3 = v.dg3[b][q];
          const double inner = ddgc - oochi * (da * dgb3 + db * dga + ddchi * gtil) +
                               2.0 * oochi * oochi * da * db * gtil;
          oochib += inner * X;
          const double Y = oochi * X;
          vb.ddg[q][sid(a, b)] += Y;
          oochib -= (da * dgb3 + db * dga + ddchi * gtil) * Y;
          vb.dchi[a] -= oochi * dgb3 * Y;
          vb.dg3[b][q] -= oochi * da * Y;
          vb.dchi[b] -= oochi * dga * Y;
          vb.dg3[a][q] -= oochi * db * Y;
          vb.ddchi[sid(a, b)] -= oochi * gtil * Y;
          vb.gt[q] -= oochi * ddchi * Y;
          oochib += 4.0 * oochi * da * db * gtil * Y;
          vb.dchi[a] += 2.0 * oochi * oochi * db * gtil * Y;
          vb.dchi[b] += 2.0 * oochi * oochi * da * gtil * Y;
          vb.gt[q] += 2.0 * oochi * oochi * da * db * Y;
        }
      }
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b) {
        const double X = Guddb[c][sid(a, b)];
                for (int d = 0; d < 3; ++d) {
          guub[sid(c, d)] += Gddd[d][sid(a, b)] * X;
          Gdddb[d][sid(a, b)] += guu[sid(c, d)] * X;
        }
      }
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b) {
        const double X = 0.5 * Gdddb[c][sid(a, b)];
        dgb[a][sid(b, c)] += X;
        dgb[b][sid(a, c)] += X;
        dgb[c][sid(a, b)] -= X;
      }
  inv3s_adj(guu, guub, gphb);
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 6; ++q) {
      const double X = dgb[c][q];
      oochib += (v.dg3[c][q] - 2.0 * oochi * v.gt[q] * v.dchi[c]) * X;
      vb.dg3[c][q] += oochi * X;
      vb.gt[q] -= oochi * oochi * v.dchi[c] * X;
      vb.dchi[c] -= oochi * oochi * v.gt[q] * X;
    }
  const double chigb = -oochi * oochi * oochib;
  if (!(v.chi < opt.chi_div_floor)) vb.chi += chigb;
    for (int c = 0; c < 6; ++c) {
    const double X = Kdb[c];
    psi4b += v.At[c] * X;
    vb.At[c] += psi4 * X;
    vb.Khat += (1. / 3.) * gph[c] * X;
    vb.Theta += (2. / 3.) * gph[c] * X;
    gphb[c] += (1. / 3.) * Kt * X;
  }
    for (int c = 0; c < 6; ++c) {
    psi4b += v.gt[c] * gphb[c];
    vb.gt[c] += psi4 * gphb[c];
  }
  vb.chi -= psi4 * psi4 * psi4b;
}

// ---- ADMToZ4c, pointwise part (adm_z4c.cpp:56-163) ------------------------
// in: the ADM metric G and curvature K at a vertex (six stored components
// each); out: chi, g~ (6), Khat, A~ (6) and the inverse conformal metric
// guu (6) whose derivatives give Gamma~ (chi_psi_power = -4: chi =
// cbrt(1 / det G)).  The lapse and shift are copied.
template <class T>
Z4C_HD T ad_cbrt(const T& x);
template <>
Z4C_HD double ad_cbrt(const double& x) { return cbrt(x); }
template <>
Z4C_HD Dual ad_cbrt(const Dual& x) {
  const double c = cbrt(x.v);
  return Dual(c, x.d * c / (3.0 * x.v));
}
template <class T>
Z4C_HD void adm_to_z4c_local(const T G[6], const T Kd[6], T* chi, T g[6], T* Khat, T A[6],
                             T guu[6]) {
  const T detg = det3s(G);
  const T oopsi4 = ad_cbrt(T(1.0) / detg);
  *chi = oopsi4;
  T Kt[6];
  for (int c = 0; c < 6; ++c) {
    g[c] = oopsi4 * G[c];
    Kt[c] = oopsi4 * Kd[c];
  }
  const T detg2 = det3s(g);
  const T kh = (T(1.0) / detg2) * trace_adj(g, Kt);
  *Khat = kh;
  for (int c = 0; c < 6; ++c) A[c] = Kt[c] - (1. / 3.) * kh * g[c];
  const T detg3 = det3s(g);
  inv3s(T(1.0) / detg3, g, guu);
}


// ---- psi4 of Z4cWeyl from its local inputs (the Weyl-scalar objective) ---
Z4C_HD double ad_sqrt(double x) { return sqrt(x); }
Z4C_HD Dual ad_sqrt(const Dual& x) {
  const double r = sqrt(x.v);
  return Dual(r, 0.5 * x.d / r);
}

// The inputs of weyl_point at one interior vertex (chi_psi_power = -4): the
// conformal metric and chi, the ADM curvature and metric, the stored first
// derivatives of chi and g~, the second derivatives (Dxx on the diagonal,
// D_a of the stored D_b off it), and the first derivatives of the ADM
// curvature.
template <class T>
struct WeylLocal {
  T chi, gt[6];      // Z4c chi, g~_q
  T Kd[6], gph[6];   // ADM K_q, gamma_q
  T dchi[3];         // stored d_a chi
  T dg3[3][6];       // stored d_c g~_q  [c][q]
  T ddchi[6];        // d_a d_b chi, pair (a,b)
  T ddg[6][6];       // d_a d_b g~_cd  [pair(a,b)][cd]
  T dK[3][6];        // d_c K_q  [c][q]
  static constexpr int N = 1 + 6 + 6 + 6 + 3 + 18 + 6 + 36 + 18;
  Z4C_HD T* data() { return &chi; }
  Z4C_HD const T* data() const { return &chi; }
};

// Re, Im psi4 of weyl_point (z4c/calculate_weyl_scalars.cpp:44-630) from
// the local inputs, in its operation order, for T = double or Dual.
template <class T>
Z4C_HD void weyl_local(const z4c_params_t& opt, const WeylLocal<T>& v, double x1, double x2,
                       double x3, T& rpsi4, T& ipsi4) {
  const T chi_g = ad_max_c(v.chi, opt.chi_div_floor);
  const T oochi = T(1.0) / chi_g;
  T dg[3][6];
  for (int c = 0; c < 3; ++c)
    for (int q = 0; q < 6; ++q) dg[c][q] = oochi * (v.dg3[c][q] - oochi * v.gt[q] * v.dchi[c]);
  T DDG[6][6];
  for (int ab = 0; ab < 6; ++ab) {
    const int a = ab < 3 ? 0 : (ab < 5 ? 1 : 2), b = ab < 3 ? ab : (ab < 5 ? ab - 2 : 2);
    const T ddchi = v.ddchi[ab];
    const T dchi_a = v.dchi[a], dchi_b = v.dchi[b];
    for (int cd = 0; cd < 6; ++cd) {
      const T gtil = v.gt[cd];
      const T ddg_conf = v.ddg[ab][cd];
      const T da3 = v.dg3[a][cd], db3 = v.dg3[b][cd];
      T w;
      if (a == b)
        w = oochi * (ddg_conf - oochi * (2.0 * dchi_a * da3 + ddchi * gtil) +
                     2.0 * oochi * oochi * dchi_a * dchi_a * gtil);
      else
        w = oochi * (ddg_conf - oochi * (dchi_a * db3 + dchi_b * da3 + ddchi * gtil) +
                     2.0 * oochi * oochi * dchi_a * dchi_b * gtil);
      DDG[ab][cd] = w;
    }
  }
  T g_uu[6];
  {
    const T detg = det3s(v.gph);
    inv3s(T(1.) / detg, v.gph, g_uu);
  }
  T Gddd[3][6], Gudd[3][6];
  for (int c = 0; c < 3; ++c)
    for (int a = 0; a < 3; ++a)
      for (int b = a; b < 3; ++b)
        Gddd[c][sid(a, b)] = 0.5 * (dg[a][sid(b, c)] + dg[b][sid(a, c)] - dg[c][sid(a, b)]);
  for (int c = 0; c < 3; ++c)
    for (int a = 0; a < 3; ++a)
      for (int b = a; b < 3; ++b) {
        T acc = T(0.0);
        for (int d = 0; d < 3; ++d) acc += g_uu[sid(c, d)] * Gddd[d][sid(a, b)];
        Gudd[c][sid(a, b)] = acc;
      }
  T Rd[6], R = T(0.0);
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      T acc = T(0.0);
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) {
          for (int e = 0; e < 3; ++e) {
            acc += g_uu[sid(c, d)] * Gudd[e][sid(a, c)] * Gddd[e][sid(b, d)];
            acc -= g_uu[sid(c, d)] * Gudd[e][sid(a, b)] * Gddd[e][sid(c, d)];
          }
          acc += 0.5 * g_uu[sid(c, d)] *
                 (-DDG[sid(c, d)][sid(a, b)] - DDG[sid(a, b)][sid(c, d)] +
                  DDG[sid(a, c)][sid(b, d)] + DDG[sid(b, c)][sid(a, d)]);
        }
      Rd[sid(a, b)] = acc;
      R += wsym(a, b) * g_uu[sid(a, b)] * acc;
    }
  T K = T(0.0);
  for (int a = 0; a < 3; ++a) {
    T kaa = T(0.0);
    for (int c = 0; c < 3; ++c) kaa += g_uu[sid(a, c)] * v.Kd[sid(c, a)];
    K += kaa;
  }
  T DK[3][6];
  for (int a = 0; a < 3; ++a)
    for (int lo = 0; lo < 3; ++lo)
      for (int hi = lo; hi < 3; ++hi) {
        const int b = hi, c = lo;
        T w = v.dK[a][sid(b, c)];
        for (int d = 0; d < 3; ++d) {
          w -= Gudd[d][sid(a, b)] * v.Kd[sid(d, c)];
          w -= Gudd[d][sid(a, c)] * v.Kd[sid(b, d)];
        }
        DK[a][sid(lo, hi)] = w;
      }
  double xx = x1;
  if (x1 * x1 + x2 * x2 < 1e-10) xx = xx + 1e-8;
  T uv[3] = {T(xx), T(x2), T(x3)};
  T vv[3] = {T(xx * x3), T(x2 * x3), T(-(xx * xx) - (x2 * x2))};
  T wv[3] = {T(x2 * -1.0), T(xx), T(0.0)};
  auto gdot = [&](const T* l, const T* r) -> T {
    T acc = T(0.0);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) acc += v.gph[sid(a, b)] * l[a] * r[b];
    return acc;
  };
  T dot = gdot(wv, wv);
  for (int a = 0; a < 3; ++a) wv[a] = wv[a] / ad_sqrt(dot);
  dot = gdot(wv, uv);
  for (int a = 0; a < 3; ++a) uv[a] -= dot * wv[a];
  dot = gdot(uv, uv);
  for (int a = 0; a < 3; ++a) uv[a] = uv[a] / ad_sqrt(dot);
  dot = gdot(wv, vv);
  const T dot2 = gdot(uv, vv);
  for (int a = 0; a < 3; ++a) vv[a] -= dot * wv[a] + dot2 * uv[a];
  dot = gdot(vv, vv);
  for (int a = 0; a < 3; ++a) vv[a] = vv[a] / ad_sqrt(dot);
  const double FR4 = 0.25;
  T rp = T(0.0), ip = T(0.0);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      T R4 = Rd[sid(a, b)] + K * v.Kd[sid(a, b)];
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) R4 -= g_uu[sid(c, d)] * v.Kd[sid(a, c)] * v.Kd[sid(d, b)];
      const T Tr = vv[a] * vv[b] - wv[a] * wv[b];
      const T Ti = -vv[a] * wv[b] - wv[a] * vv[b];
      rp += -FR4 * R4 * Tr;
      ip += -FR4 * R4 * Ti;
    }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const T Tr = vv[a] * vv[b] - wv[a] * wv[b];
      const T Ti = -vv[a] * wv[b] - wv[a] * vv[b];
      for (int c = 0; c < 3; ++c) {
        const T R4 = -(DK[b][sid(a, c)] - DK[c][sid(a, b)]);
        rp += 0.5 * R4 * uv[c] * Tr;
        ip += 0.5 * R4 * uv[c] * Ti;
      }
    }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const T Tr = vv[a] * vv[b] - wv[a] * wv[b];
      const T Ti = -vv[a] * wv[b] - wv[a] * vv[b];
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) {
          const T R4 = v.gph[sid(d, c)] * Rd[sid(a, b)] + v.gph[sid(a, b)] * Rd[sid(d, c)] -
                       v.gph[sid(d, b)] * Rd[sid(a, c)] - v.gph[sid(a, c)] * Rd[sid(d, b)] -
                       0.5 * R * (v.gph[sid(d, c)] * v.gph[sid(a, b)] -
                                  v.gph[sid(d, b)] * v.gph[sid(a, c)]) +
                       v.Kd[sid(d, c)] * v.Kd[sid(a, b)] - v.Kd[sid(d, b)] * v.Kd[sid(a, c)];
          rp += -FR4 * R4 * uv[d] * uv[c] * Tr;
          ip += -FR4 * R4 * uv[d] * uv[c] * Ti;
        }
    }
  rpsi4 = rp;
  ipsi4 = ip;
}

}  // namespace ad
}  // namespace z4c

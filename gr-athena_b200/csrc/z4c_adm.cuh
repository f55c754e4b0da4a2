// Pointwise ADM <-> Z4c maps and the ADM constraints.
//   Z4c::Z4cToADM        z4c/adm_z4c.cpp:200-260
//   Z4c::ADMToZ4c        z4c/adm_z4c.cpp:46-192
//   Z4c::ADMConstraints  z4c/adm_z4c.cpp:382-930 (vacuum), reading the
//                        conformal first derivatives that
//                        Z4c::PrepareZ4cDerivatives (:972-1037) would store,
//                        evaluated in place.
#pragma once

#include "z4c_common.cuh"

namespace z4c {

__device__ __forceinline__ void z4c_to_adm_point(const z4c_params_t& opt, const double* u,
                                                 double* adm, int64_t nvol) {
#define U_(n) u[(int64_t)(n) * nvol]
#define A_(n) adm[(int64_t)(n) * nvol]
  A_(Z4C_ADM_ALPHA) = U_(Z4C_ALPHA);
#pragma unroll
  for (int a = 0; a < 3; ++a) A_(Z4C_ADM_BETAX + a) = U_(Z4C_BETAX + a);
  double psi4;
  if (opt.chi_psi_power == -4.) psi4 = 1.0 / U_(Z4C_CHI);
  else psi4 = pow(U_(Z4C_CHI), 4. / opt.chi_psi_power);
  A_(Z4C_ADM_PSI4) = psi4;
  double gph[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    gph[c] = psi4 * U_(Z4C_GXX + c);
    A_(Z4C_ADM_GXX + c) = gph[c];
  }
  const double khat = U_(Z4C_KHAT), theta = U_(Z4C_THETA);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    A_(Z4C_ADM_KXX + c) = psi4 * U_(Z4C_AXX + c) + (1. / 3.) * (khat + 2. * theta) * gph[c];
#undef U_
#undef A_
}

// Pointwise part of ADMToZ4c (:56-136); Gamma^i and the final AlgConstr are
// separate passes.  guu receives the inverse conformal metric (:146-163).
__device__ __forceinline__ void adm_to_z4c_point(const z4c_params_t& opt, const double* adm,
                                                 double* u, double* guu, int64_t nvol) {
#define U_(n) u[(int64_t)(n) * nvol]
#define A_(n) adm[(int64_t)(n) * nvol]
  U_(Z4C_ALPHA) = A_(Z4C_ADM_ALPHA);
#pragma unroll
  for (int a = 0; a < 3; ++a) U_(Z4C_BETAX + a) = A_(Z4C_ADM_BETAX + a);
  double G[6], Kd[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    G[c] = A_(Z4C_ADM_GXX + c);
    Kd[c] = A_(Z4C_ADM_KXX + c);
  }
  double detg = det3(G[0], G[1], G[2], G[3], G[4], G[5]);
  double oopsi4;
  if (opt.chi_psi_power == -4.) {
    oopsi4 = cbrt(1.0 / detg);
    U_(Z4C_CHI) = oopsi4;
  } else {
    oopsi4 = pow(detg, -1. / 3.);
    U_(Z4C_CHI) = pow(detg, 1. / 12. * opt.chi_psi_power);
  }
  double g[6], Kt[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    g[c] = oopsi4 * G[c];
    Kt[c] = oopsi4 * Kd[c];
    U_(Z4C_GXX + c) = g[c];
  }
  detg = det3(g[0], g[1], g[2], g[3], g[4], g[5]);
  const double Khat = trace_rank2(1.0 / detg, g, Kt);
  U_(Z4C_KHAT) = Khat;
#pragma unroll
  for (int c = 0; c < 6; ++c) U_(Z4C_AXX + c) = Kt[c] - (1. / 3.) * Khat * g[c];
  U_(Z4C_THETA) = 0.0;
  double gu[6];
  const double detg2 = det3(g[0], g[1], g[2], g[3], g[4], g[5]);
  inv3(1.0 / detg2, g, gu);
#pragma unroll
  for (int c = 0; c < 6; ++c) guu[(int64_t)c * nvol] = gu[c];
#undef U_
#undef A_
}

// ADMConstraints at one interior vertex; writes the 7 constraint values.
__device__ __forceinline__ void adm_constraints_point(const double* __restrict__ uB,
                                                      const double* __restrict__ admB,
                                                      int64_t nvol, int64_t p,
                                                      const int64_t s[3], const DevParams& P,
                                                      const FdScale& F,
                                                      double x1, double x2, double x3,
                                                      double con[7]) {
  const z4c_params_t& opt = P.p;
  const double* U = uB + p;
  const double* AD = admB + p;
#define UV(n) (U + (int64_t)(n) * nvol)
#define AV(n) (AD + (int64_t)(n) * nvol)
  const double pw = opt.chi_psi_power;
  const double chi = __ldg(UV(Z4C_CHI));
  const double chi_g = dmax(chi, opt.chi_div_floor);
  const double oochi = 1.0 / chi_g;
  const double psi4c = (pw != -4.) ? pow(chi_g, 4.0 / pw) : 0.0;
  double gt[6], Kd[6], gph[6], dchi[3];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    gt[c] = __ldg(UV(Z4C_GXX + c));
    Kd[c] = __ldg(AV(Z4C_ADM_KXX + c));
    gph[c] = __ldg(AV(Z4C_ADM_GXX + c));
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) dchi[a] = fd_dx(UV(Z4C_CHI), s[a], F.cidx1[a]);
  // conformal first derivatives d_c g~_ab (stored dg_ddd_3d)
  double dg3[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int q = 0; q < 6; ++q) dg3[c][q] = fd_dx(UV(Z4C_GXX + q), s[c], F.cidx1[c]);
  // pass 1: physical first derivatives, :446-460 / :532-546
  double dg[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      if (pw == -4.) dg[c][q] = oochi * (dg3[c][q] - oochi * gt[q] * dchi[c]);
      else dg[c][q] = psi4c * (dg3[c][q] + (4.0 / pw) * oochi * gt[q] * dchi[c]);
    }
  // inverse physical metric
  double g_uu[6];
  {
    const double detg = det3(gph[0], gph[1], gph[2], gph[3], gph[4], gph[5]);
    inv3(1. / detg, gph, g_uu);
  }
#define GUU(a, b) g_uu[sidx(a, b)]
  double Gddd[3][6], Gudd[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b)
        Gddd[c][sidx(a, b)] = 0.5 * (dg[a][sidx(b, c)] + dg[b][sidx(a, c)] - dg[c][sidx(a, b)]);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        double acc = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) acc += GUU(c, d) * Gddd[d][sidx(a, b)];
        Gudd[c][sidx(a, b)] = acc;
      }
  // physical second derivatives ddg(a,b,c,d) = d_a d_b gamma_cd, :463-596
  auto ddg = [&](int a, int b, int c, int d) -> double {
    const int ab_lo = a < b ? a : b, ab_hi = a < b ? b : a;
    const int q = sidx(c, d);
    const double* f = UV(Z4C_GXX + q);
    const double dchi_a = dchi[ab_lo], dchi_b = dchi[ab_hi];
    const double gtil = gt[q];
    double ddchi;
    if (ab_lo == ab_hi) ddchi = fd_dxx(UV(Z4C_CHI), s[ab_lo], F.cidx2[ab_lo]);
    else ddchi = fd_dxy(UV(Z4C_CHI), s[ab_lo], s[ab_hi], F.cidx1[ab_lo], F.cidx1[ab_hi]);
    if (ab_lo == ab_hi) {
      const double ddg_conf = fd_dxx(f, s[ab_lo], F.cidx2[ab_lo]);
      const double d3 = dg3[ab_lo][q];
      if (pw == -4.)
        return oochi * (ddg_conf - oochi * (2.0 * dchi_a * d3 + ddchi * gtil) +
                        2.0 * oochi * oochi * dchi_a * dchi_a * gtil);
      const double fac = 4.0 / pw, fac2 = fac - 1.0;
      return psi4c * (ddg_conf + fac * oochi * (2.0 * dchi_a * d3 + ddchi * gtil) +
                      fac * fac2 * oochi * oochi * dchi_a * dchi_a * gtil);
    }
    const double ddg_conf = fd_dxy(f, s[ab_lo], s[ab_hi], F.cidx1[ab_lo], F.cidx1[ab_hi]);
    const double dgb = dg3[ab_hi][q], dga = dg3[ab_lo][q];
    if (pw == -4.)
      return oochi * (ddg_conf - oochi * (dchi_a * dgb + dchi_b * dga + ddchi * gtil) +
                      2.0 * oochi * oochi * dchi_a * dchi_b * gtil);
    const double fac = 4.0 / pw, fac2 = fac - 1.0;
    return psi4c * (ddg_conf + fac * oochi * (dchi_a * dgb + dchi_b * dga + ddchi * gtil) +
                    fac * fac2 * oochi * oochi * dchi_a * dchi_b * gtil);
  };
  double DDG[6][6];  // [sym(a,b)][sym(c,d)], computed once as the reference stores it
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = c; d < 3; ++d) DDG[sidx(a, b)][sidx(c, d)] = ddg(a, b, c, d);
  // Ricci, :655-689
  double R = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double acc = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
          for (int f = 0; f < 3; ++f)
            acc += GUU(d, f) * (Gudd[c][sidx(a, f)] * Gddd[c][sidx(b, d)] -
                                Gudd[c][sidx(a, b)] * Gddd[c][sidx(f, d)]);
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          acc += 0.5 * GUU(c, d) *
                 (-DDG[sidx(b, a)][sidx(c, d)] + DDG[sidx(d, a)][sidx(b, c)] +
                  DDG[sidx(d, b)][sidx(a, c)] - DDG[sidx(d, c)][sidx(a, b)]);
      R += ((a == b) ? 1.0 : 2.0) * GUU(a, b) * acc;
    }
  // extrinsic curvature, :694-753
  double K = 0, K_ud[3][3], KK = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double acc = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) acc += GUU(a, c) * Kd[sidx(c, b)];
      K_ud[a][b] = acc;
    }
    K += K_ud[a][a];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) KK += K_ud[a][b] * K_ud[b][a];
  double DK[3][6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c) {
        double v = fd_dx(AV(Z4C_ADM_KXX + sidx(b, c)), s[a], F.cidx1[a]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          v -= Gudd[d][sidx(a, b)] * Kd[sidx(d, c)];
          v -= Gudd[d][sidx(a, c)] * Kd[sidx(b, d)];
        }
        DK[a][sidx(b, c)] = v;
      }
  double DKu[3][6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c) {
        double acc = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) acc += GUU(a, d) * DK[d][sidx(b, c)];
        DKu[a][sidx(b, c)] = acc;
      }
  // constraints, :760-814 (rho = S_i = 0)
  const double H = R + (K * K) - KK;
  double M_u[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        M_u[a] += GUU(a, b) * DKu[c][sidx(b, c)];
        M_u[a] -= GUU(b, c) * DKu[a][sidx(b, c)];
      }
  double M_d[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double acc = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b) acc += gph[sidx(a, b)] * M_u[b];
    M_d[a] = acc;
  }
  double M = 0.;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) M += ((a == b) ? 1.0 : 2.0) * gph[sidx(a, b)] * M_u[a] * M_u[b];
  // conformal connection functions for Z, :819-906
  double gc[6];
  {
    const double detg = det3(gt[0], gt[1], gt[2], gt[3], gt[4], gt[5]);
    inv3(1. / detg, gt, gc);
  }
  double cGd[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b)
        cGd[c][sidx(a, b)] = 0.5 * (dg3[a][sidx(b, c)] + dg3[b][sidx(a, c)] - dg3[c][sidx(a, b)]);
  double cGu[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double acc = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c) {
        double gudd = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) gudd += gc[sidx(a, d)] * cGd[d][sidx(b, c)];
        acc += ((b == c) ? 1.0 : 2.0) * gc[sidx(b, c)] * gudd;
      }
    cGu[a] = acc;
  }
  double Z = 0.;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b)
      Z += ((a == b) ? 0.25 : 0.5) * gph[sidx(a, b)] * (__ldg(UV(Z4C_GAMX + a)) - cGu[a]) *
           (__ldg(UV(Z4C_GAMX + b)) - cGu[b]);
  const double R2 = x1 * x1 + x2 * x2 + x3 * x3;
  const double r2_max = opt.r_max_con * opt.r_max_con;
#pragma unroll
  for (int q = 0; q < 7; ++q) con[q] = 0.0;
  if (!(R2 > r2_max)) {
    const double Theta = __ldg(UV(Z4C_THETA));
    con[Z4C_CON_H] = H;
    con[Z4C_CON_M] = M;
    con[Z4C_CON_Z] = Z;
#pragma unroll
    for (int a = 0; a < 3; ++a) con[Z4C_CON_MX + a] = M_d[a];
    con[Z4C_CON_C] = (H * H) + M + (Theta * Theta) + 4.0 * Z;
  }
#undef GUU
#undef UV
#undef AV
}

}  // namespace z4c

// Pointwise Z4c right-hand side: Z4c::Z4cRHS (z4c/calculate_z4c_rhs.cpp:29-916)
// with the derivative precompute of Z4c::PrepareZ4cDerivatives
// (z4c/adm_z4c.cpp:972-1037) evaluated in place from the state, constant-eta
// branch, vacuum (matter terms vanish), Kreiss-Oliger dissipation included.
//
// One call computes the 22 right-hand-side values of one interior vertex.
// The operation order follows the reference line by line; line numbers in
// the comments refer to calculate_z4c_rhs.cpp.
#pragma once

#include "z4c_common.cuh"

namespace z4c {

// u: base of one block register ([var][k][j][i]); p: vertex offset.
__device__ __forceinline__ void rhs_point(const double* __restrict__ u, int64_t nvol,
                                          int64_t p, const int64_t s[3],
                                          const DevParams& P, const FdScale& F,
                                          double out[NVAR]) {
  const z4c_params_t& opt = P.p;
  const double* U = u + p;
#define UV(n) (U + (int64_t)(n) * nvol)

  double g_dd[6], A_dd[6], beta_u[3], Gam_u[3];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    g_dd[c] = __ldg(UV(Z4C_GXX + c));
    A_dd[c] = __ldg(UV(Z4C_AXX + c));
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    beta_u[a] = __ldg(UV(Z4C_BETAX + a));
    Gam_u[a] = __ldg(UV(Z4C_GAMX + a));
  }
  const double chi = __ldg(UV(Z4C_CHI)), Khat = __ldg(UV(Z4C_KHAT));
  const double Theta = __ldg(UV(Z4C_THETA)), alpha = __ldg(UV(Z4C_ALPHA));

  // --- first derivatives, :84-114 (dA_ddd of :112 is never read) ---
  double dalpha_d[3], dchi_d[3], dKhat_d[3], dTheta_d[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    dalpha_d[a] = fd_dx(UV(Z4C_ALPHA), s[a], F.cidx1[a]);
    dchi_d[a] = fd_dx(UV(Z4C_CHI), s[a], F.cidx1[a]);
    dKhat_d[a] = fd_dx(UV(Z4C_KHAT), s[a], F.cidx1[a]);
    dTheta_d[a] = fd_dx(UV(Z4C_THETA), s[a], F.cidx1[a]);
  }
  double dbeta_du[3][3];  // [b][a] = d_b beta^a
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int a = 0; a < 3; ++a) dbeta_du[b][a] = fd_dx(UV(Z4C_BETAX + a), s[b], F.cidx1[b]);

  // --- Christoffel symbols, :317-352 (needs d g only here) ---
  double g_uu[6];
  {
    const double detg = det3(g_dd[0], g_dd[1], g_dd[2], g_dd[3], g_dd[4], g_dd[5]);
    inv3(1.0 / detg, g_dd, g_uu);
  }
#define GUU(a, b) g_uu[sidx(a, b)]
#define GDD(a, b) g_dd[sidx(a, b)]
#define ADD(a, b) A_dd[sidx(a, b)]
  double Gamma_ddd[3][6];  // [c][ab]
  {
    double dg[3][6];       // [c][ab] = d_c g_ab
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int q = 0; q < 6; ++q) dg[c][q] = fd_dx(UV(Z4C_GXX + q), s[c], F.cidx1[c]);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b)
          Gamma_ddd[c][sidx(a, b)] =
              0.5 * (dg[a][sidx(b, c)] + dg[b][sidx(a, c)] - dg[c][sidx(a, b)]);
  }
  double Gamma_udd[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        double sacc = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) sacc += GUU(c, d) * Gamma_ddd[d][sidx(a, b)];
        Gamma_udd[c][sidx(a, b)] = sacc;
      }
  double Gamma_u[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double sacc = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c)
        sacc += ((b == c) ? 1.0 : 2.0) * GUU(b, c) * Gamma_udd[a][sidx(b, c)];
    Gamma_u[a] = sacc;
  }
#define GDDD(c, a, b) Gamma_ddd[c][sidx(a, b)]
#define GUDD(c, a, b) Gamma_udd[c][sidx(a, b)]

  // --- Ricci tensor of the conformal metric, :357-396 ---
  double R_dd[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double sacc = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double dGam_bc = fd_dx(UV(Z4C_GAMX + c), s[b], F.cidx1[b]);
        const double dGam_ac = fd_dx(UV(Z4C_GAMX + c), s[a], F.cidx1[a]);
        sacc += 0.5 * (GDD(c, a) * dGam_bc + GDD(c, b) * dGam_ac +
                       Gamma_u[c] * (GDDD(a, b, c) + GDDD(b, a, c)));
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = c; d < 3; ++d) {
          // ddg_dddd(c,d,a,b): second derivative along c,d of g_ab, :158-178
          const double* f = UV(Z4C_GXX + sidx(a, b));
          const double dd = (c == d) ? fd_dxx(f, s[c], F.cidx2[c])
                                     : fd_dxy(f, s[c], s[d], F.cidx1[c], F.cidx1[d]);
          sacc -= ((c == d) ? 0.5 : 1.0) * GUU(c, d) * dd;
        }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
          for (int e = 0; e < 3; ++e)
            sacc += GUU(c, d) * (GUDD(e, c, a) * GDDD(b, e, d) + GUDD(e, c, b) * GDDD(a, e, d) +
                                 GUDD(e, a, d) * GDDD(e, c, b));
      R_dd[sidx(a, b)] = sacc;
    }

  // --- conformal factor, :231-274, :402-426 ---
  const double K = Khat + 2. * Theta;
  const double chi_guarded = dmax(chi, opt.chi_div_floor);
  const double oochi = 1.0 / chi_guarded;
  double oopsi4;
  if (opt.chi_psi_power == -4.) oopsi4 = chi_guarded;
  else oopsi4 = pow(chi_guarded, -4. / opt.chi_psi_power);
  const double oochi_psi_power = 1.0 / opt.chi_psi_power;
  double dphi_d[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) dphi_d[a] = dchi_d[a] * oochi * oochi_psi_power;
  double Ddphi_dd[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const double* f = UV(Z4C_CHI);
      const double ddchi = (a == b) ? fd_dxx(f, s[a], F.cidx2[a])
                                    : fd_dxy(f, s[a], s[b], F.cidx1[a], F.cidx1[b]);
      double v = ddchi * oochi * oochi_psi_power - opt.chi_psi_power * dphi_d[a] * dphi_d[b];
#pragma unroll
      for (int c = 0; c < 3; ++c) v -= GUDD(c, a, b) * dphi_d[c];
      Ddphi_dd[sidx(a, b)] = v;
    }
  // Rphi, :436-458
  double Stmp = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = c; d < 3; ++d)
      Stmp += ((c == d) ? 1.0 : 2.0) * GUU(c, d) *
              (Ddphi_dd[sidx(c, d)] + 2. * dphi_d[c] * dphi_d[d]);
  double Rphi_dd[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b)
      Rphi_dd[sidx(a, b)] = 4. * dphi_d[a] * dphi_d[b] - 2. * Ddphi_dd[sidx(a, b)] -
                            2. * GDD(a, b) * Stmp;

  // --- D D alpha, :482-521 ---
  double Ddalpha = 0;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d) Ddalpha += GUU(c, d) * dphi_d[c] * dalpha_d[d];
  double Ddalpha_dd[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const double* f = UV(Z4C_ALPHA);
      const double ddal = (a == b) ? fd_dxx(f, s[a], F.cidx2[a])
                                   : fd_dxy(f, s[a], s[b], F.cidx1[a], F.cidx1[b]);
      double v = ddal - 2. * (dphi_d[a] * dalpha_d[b] + dphi_d[b] * dalpha_d[a]) +
                 2. * GDD(a, b) * Ddalpha;
#pragma unroll
      for (int c = 0; c < 3; ++c) v -= GUDD(c, a, b) * dalpha_d[c];
      Ddalpha_dd[sidx(a, b)] = v;
    }
  Ddalpha = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b)
      Ddalpha += ((a == b) ? 1.0 : 2.0) * oopsi4 * GUU(a, b) * Ddalpha_dd[sidx(a, b)];

  // --- A contractions, :525-589 ---
  double A_ud[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double sacc = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) sacc += GUU(c, d) * ADD(d, b);
      A_ud[c][b] = sacc;
    }
  double AA_dd[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double sacc = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) sacc += ADD(a, c) * A_ud[c][b];
      AA_dd[sidx(a, b)] = sacc;
    }
  double trAA = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) trAA += ((a == b) ? 1.0 : 2.0) * GUU(a, b) * AA_dd[sidx(a, b)];
  double A_uu[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double sacc = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) sacc += GUU(b, c) * A_ud[a][c];
      A_uu[sidx(a, b)] = sacc;
    }
  const double chi_pow_DA_u = -6.0 / opt.chi_psi_power;
  double DA_u[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double sacc = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      sacc -= chi_pow_DA_u * A_uu[sidx(a, b)] * dchi_d[b] * oochi;
      sacc -= (1. / 3.) * GUU(a, b) * (2. * dKhat_d[b] + dTheta_d[b]);
    }
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c)
        sacc += ((b == c) ? 1.0 : 2.0) * GUDD(a, b, c) * A_uu[sidx(b, c)];
    DA_u[a] = sacc;
  }

  // --- Ricci scalar, Ht, :596-613 ---
  double R = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b)
      R += ((a == b) ? 1.0 : 2.0) * oopsi4 * GUU(a, b) * (R_dd[sidx(a, b)] + Rphi_dd[sidx(a, b)]);
  const double Ht = R + (2. / 3.) * (K * K) - trAA;

  // --- advective derivatives, :184-226 ---
  double Lsc[4] = {0, 0, 0, 0};  // alpha, chi, Khat, Theta
  double Lbeta_u[3] = {0, 0, 0}, LGam_u[3] = {0, 0, 0};
  double Lg_dd[6] = {0, 0, 0, 0, 0, 0}, LA_dd[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int64_t sa = s[a];
    const double la = F.lidx[a];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) {
      const Line9 L = load9(UV(n), sa);
      const double lx = fd_lx(L, beta_u[a], la);
      if (n == Z4C_ALPHA) Lsc[0] += lx;
      else if (n == Z4C_CHI) Lsc[1] += lx;
      else if (n == Z4C_KHAT) Lsc[2] += lx;
      else if (n == Z4C_THETA) Lsc[3] += lx;
      else if (n >= Z4C_BETAX) Lbeta_u[n - Z4C_BETAX] += lx;
      else if (n >= Z4C_GAMX && n <= Z4C_GAMZ) LGam_u[n - Z4C_GAMX] += lx;
      else if (n >= Z4C_GXX && n <= Z4C_GZZ) Lg_dd[n - Z4C_GXX] += lx;
      else if (n >= Z4C_AXX && n <= Z4C_AZZ) LA_dd[n - Z4C_AXX] += lx;
    }
  }

  // --- finalize Lie derivatives, :619-687 ---
  double dbeta = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) dbeta += dbeta_du[a][a];
  double ddbeta_d[3] = {0, 0, 0};
  // ddbeta_ddu(a,b,c): second derivative along a,b of beta^c, :138-156
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double* f = UV(Z4C_BETAX + b);
      const double v = (a == b) ? fd_dxx(f, s[a], F.cidx2[a])
                                : fd_dxy(f, s[a < b ? a : b], s[a < b ? b : a],
                                         F.cidx1[a < b ? a : b], F.cidx1[a < b ? b : a]);
      ddbeta_d[a] += (1. / 3.) * v;
    }
  double Lchi = Lsc[1] + (1. / 6.) * opt.chi_psi_power * chi_guarded * dbeta;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    LGam_u[a] += (2. / 3.) * Gamma_u[a] * dbeta;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      LGam_u[a] += GUU(a, b) * ddbeta_d[b] - Gamma_u[b] * dbeta_du[b][a];
#pragma unroll
      for (int c = b; c < 3; ++c) {
        const double* f = UV(Z4C_BETAX + a);
        const double v = (b == c) ? fd_dxx(f, s[b], F.cidx2[b])
                                  : fd_dxy(f, s[b], s[c], F.cidx1[b], F.cidx1[c]);
        LGam_u[a] += ((b == c) ? 1.0 : 2.0) * GUU(b, c) * v;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double lg = Lg_dd[sidx(a, b)], la = LA_dd[sidx(a, b)];
      lg -= (2. / 3.) * GDD(a, b) * dbeta;
      la -= (2. / 3.) * ADD(a, b) * dbeta;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lg += dbeta_du[a][c] * GDD(b, c);
        la += dbeta_du[b][c] * ADD(a, c);
        lg += dbeta_du[b][c] * GDD(a, c);
        la += dbeta_du[a][c] * ADD(b, c);
      }
      Lg_dd[sidx(a, b)] = lg;
      LA_dd[sidx(a, b)] = la;
    }

  // --- assemble, :694-902 (matter fields are zero: S = rho = S_i = S_ij = 0) ---
  const double S = 0.0;
  out[Z4C_KHAT] = -Ddalpha + alpha * (trAA + (1. / 3.) * (K * K)) + Lsc[2] +
                  opt.damp_kappa1 * (1 - opt.damp_kappa2) * alpha * Theta;
  out[Z4C_CHI] = Lchi - (1. / 6.) * opt.chi_psi_power * chi_guarded * alpha * K;
  out[Z4C_THETA] = Lsc[3] + alpha * (0.5 * Ht - (2. + opt.damp_kappa2) * opt.damp_kappa1 * Theta);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double v = 2. * alpha * DA_u[a] + LGam_u[a];
    v -= 2. * alpha * opt.damp_kappa1 * (Gam_u[a] - Gamma_u[a]);
#pragma unroll
    for (int b = 0; b < 3; ++b) v -= 2. * A_uu[sidx(a, b)] * dalpha_d[b];
    out[Z4C_GAMX + a] = v;
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const int q = sidx(a, b);
      out[Z4C_GXX + q] = -2. * alpha * A_dd[q] + Lg_dd[q];
      double v = oopsi4 * (-Ddalpha_dd[q] + alpha * (R_dd[q] + Rphi_dd[q]));
      v -= (1. / 3.) * g_dd[q] * (-Ddalpha + alpha * R);
      v += alpha * (K * A_dd[q] - 2. * AA_dd[q]);
      v += LA_dd[q];
      (void)S;
      out[Z4C_AXX + q] = v;
    }
  {
    const double fl = opt.lapse_oplog * opt.lapse_harmonicf + opt.lapse_harmonic * alpha;
    out[Z4C_ALPHA] = (opt.lapse_advect * Lsc[0] - fl * alpha * (Khat + 2 * opt.lapse_K * Theta));
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double v = opt.shift_Gamma * Gam_u[a] + opt.shift_advect * Lbeta_u[a];
    if (fabs(opt.shift_alpha2Gamma) > 0.0) v += opt.shift_alpha2Gamma * (alpha * alpha) * Gam_u[a];
    if (fabs(opt.shift_H) > 0.0) {
#pragma unroll
      for (int b = 0; b < 3; ++b)
        v += opt.shift_H * alpha * chi_guarded * (0.5 * alpha * dchi_d[b] - dalpha_d[b]) * GUU(a, b);
    }
    v -= opt.shift_eta * beta_u[a];
    out[Z4C_BETAX + a] = v;
  }
  // Kreiss-Oliger, :908-915: rhs += Diss_x; rhs += Diss_y; rhs += Diss_z
#pragma unroll
  for (int n = 0; n < NVAR; ++n)
#pragma unroll
    for (int a = 0; a < 3; ++a)
      out[n] += fd_diss(load9(UV(n), s[a]), F.cidxd[a], opt.diss);

#undef UV
#undef GUU
#undef GDD
#undef ADD
#undef GDDD
#undef GUDD
}

}  // namespace z4c

// Pointwise Z4c right-hand side: Z4c::Z4cRHS (z4c/calculate_z4c_rhs.cpp:29-916)
// with the derivative precompute of Z4c::PrepareZ4cDerivatives
// (z4c/adm_z4c.cpp:972-1037) evaluated in place from the state, constant-eta
// branch, vacuum (matter terms vanish), Kreiss-Oliger dissipation included.
//
// The first derivatives that the reference stores in PrepareZ4cDerivatives
// (chi, g~_ab, alpha, beta^a along every direction, on the interior extended
// by 3 vertices across) are computed by a separate pass into the `sd`
// scratch, exactly as the reference computes them; the passes below read
// them there, both as first derivatives and as the inputs of the mixed
// second derivatives (Dx_a of the stored Dx_b, Q1 of the reference).
//
// The work per vertex is split in two passes so that each keeps its live
// values in registers:
//   ricci_point  the Ricci tensor of the conformal metric and its
//                conformal-factor part, stored as Rsum_ab = R_ab + Rphi_ab
//                (the reference only ever uses the sum, :603, :745);
//   rhs_point    everything else, reading Rsum_ab and the advection sums;
// the advection sums (advect_point) and the Kreiss-Oliger terms (add_ko) run
// in separate light kernels, one thread per vertex and variable.
// The operation order of every quantity follows the reference line by line;
// line numbers in the comments refer to calculate_z4c_rhs.cpp.
#pragma once

#include "z4c_common.cuh"

namespace z4c {

#define UV(n) (U + (int64_t)(n) * nvol)
#define GUU(a, b) g_uu[sidx(a, b)]

// (a,b) of the symmetric pair q in xx,xy,xz,yy,yz,zz order
__device__ __forceinline__ int pair_a(int q) { return q < 3 ? 0 : (q < 5 ? 1 : 2); }
__device__ __forceinline__ int pair_b(int q) { return q < 3 ? q : (q < 5 ? q - 2 : 2); }

// Slots of the fields with stored first derivatives; component
// slot*3 + direction of the sd scratch ([block][33][vertex]).
constexpr int kSdChi = 0, kSdG = 1, kSdAlpha = 7, kSdBeta = 8, kSdFields = 11;
__host__ __device__ __forceinline__ constexpr int sd_field_var(int slot) {
  return slot == 0 ? Z4C_CHI : (slot <= 6 ? Z4C_GXX + slot - 1 : (slot == 7 ? Z4C_ALPHA
                                                                        : Z4C_BETAX + slot - 8));
}

// Second derivative of f along the pair q: Dxx on the diagonal, otherwise Dx
// along the first index of the stored Dx along the second (a < b); sdf points
// at the three stored first derivatives of f (stride nvol).
__device__ __forceinline__ double fd_d2(const double* __restrict__ f,
                                        const double* __restrict__ sdf, int64_t nvol, int q,
                                        const int64_t s[3], const FdScale& F) {
  const int a = pair_a(q), b = pair_b(q);
  if (a == b) return fd_dxx(f, s[a], F.cidx2[a]);
  return fd_dx(sdf + b * nvol, s[a], F.cidx1[a]);
}
#define SDF(slot) (SD + (int64_t)(slot) * 3 * nvol)
#define SDV(slot, dir) __ldg(SD + ((int64_t)(slot) * 3 + (dir)) * nvol)

// The heavy derivative gathers below run as rolled loops (GATHER_LOOP)
// writing small per-thread arrays; the tensor algebra that consumes them is
// fully unrolled.  Unrolled gathers let the compiler hoist hundreds of
// stencil loads at once and spill.
#ifndef Z4C_ROLLED_GATHERS
#define Z4C_ROLLED_GATHERS 0
#endif
#if Z4C_ROLLED_GATHERS
#define GATHER_LOOP _Pragma("unroll 1")
#else
#define GATHER_LOOP _Pragma("unroll")
#endif
#define GDD(a, b) g_dd[sidx(a, b)]
#define ADD(a, b) A_dd[sidx(a, b)]

// Inverse conformal metric (:295-311) and Christoffel symbols (:317-352).
// Gamma_ddd is written only when the caller passes storage for it.
__device__ __forceinline__ void christoffel(const double* __restrict__ SD, int64_t nvol,
                                            const double g_dd[6], double g_uu[6],
                                            double Gamma_ddd[3][6], double Gamma_udd[3][6],
                                            double Gamma_u[3]) {
  {
    const double detg = det3(g_dd[0], g_dd[1], g_dd[2], g_dd[3], g_dd[4], g_dd[5]);
    inv3(1.0 / detg, g_dd, g_uu);
  }
  double Gd[3][6];
  {
    double dg[3][6];  // [c][ab] = d_c g_ab (stored dg_ddd_3d)
#pragma unroll
    for (int q = 0; q < 6; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) dg[c][q] = SDV(kSdG + q, c);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b)
          Gd[c][sidx(a, b)] = 0.5 * (dg[a][sidx(b, c)] + dg[b][sidx(a, c)] - dg[c][sidx(a, b)]);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        double sacc = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) sacc += GUU(c, d) * Gd[d][sidx(a, b)];
        Gamma_udd[c][sidx(a, b)] = sacc;
      }
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
  if (Gamma_ddd) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int q = 0; q < 6; ++q) Gamma_ddd[c][q] = Gd[c][q];
  }
}

// Rsum_ab = R_ab + Rphi_ab at one interior vertex (:357-458).
__device__ __forceinline__ void ricci_point(const double* __restrict__ u,
                                            const double* __restrict__ sd, int64_t nvol,
                                            int64_t p, const int64_t s[3],
                                            const DevParams& P, const FdScale& F,
                                            double Rsum[6]) {
  const z4c_params_t& opt = P.p;
  const double* U = u + p;
  const double* SD = sd + p;
  double g_dd[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) g_dd[c] = __ldg(UV(Z4C_GXX + c));
  double g_uu[6], Gamma_ddd[3][6], Gamma_udd[3][6], Gamma_u[3];
  christoffel(SD, nvol, g_dd, g_uu, Gamma_ddd, Gamma_udd, Gamma_u);
#define GDDD(c, a, b) Gamma_ddd[c][sidx(a, b)]
#define GUDD(c, a, b) Gamma_udd[c][sidx(a, b)]

  // Ricci tensor of the conformal metric, :357-396; each R_ab accumulates
  // its three groups of terms in the reference's order
  double dGam[3][3];  // [b][c] = d_b Gamma^c
GATHER_LOOP
  for (int c = 0; c < 3; ++c) {
    const double* f = UV(Z4C_GAMX + c);
#pragma unroll
    for (int b = 0; b < 3; ++b) dGam[b][c] = fd_dx(f, s[b], F.cidx1[b]);
  }
  double R_dd[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double sacc = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        sacc += 0.5 * (GDD(c, a) * dGam[b][c] + GDD(c, b) * dGam[a][c] +
                       Gamma_u[c] * (GDDD(a, b, c) + GDDD(b, a, c)));
      R_dd[sidx(a, b)] = sacc;
    }
  // ddg_dddd(c,d,a,b): second derivative along c,d of g_ab, :158-178
GATHER_LOOP
  for (int q = 0; q < 6; ++q) {
    const double* f = UV(Z4C_GXX + q);
    const double* sdf = SDF(kSdG + q);
    double sacc = R_dd[q];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int d = c; d < 3; ++d)
        sacc -= ((c == d) ? 0.5 : 1.0) * GUU(c, d) * fd_d2(f, sdf, nvol, sidx(c, d), s, F);
    R_dd[q] = sacc;
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double sacc = R_dd[sidx(a, b)];
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

  // conformal-factor part, :241-245, :402-458
  const double chi = __ldg(UV(Z4C_CHI));
  const double chi_guarded = dmax(chi, opt.chi_div_floor);
  const double oochi = 1.0 / chi_guarded;
  const double oochi_psi_power = 1.0 / opt.chi_psi_power;
  double dphi_d[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) dphi_d[a] = SDV(kSdChi, a) * oochi * oochi_psi_power;
  double ddchi[6];  // stored ddchi_dd_3d
GATHER_LOOP
  for (int q = 0; q < 6; ++q) ddchi[q] = fd_d2(UV(Z4C_CHI), SDF(kSdChi), nvol, q, s, F);
  double Ddphi_dd[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double v = ddchi[sidx(a, b)] * oochi * oochi_psi_power -
                 opt.chi_psi_power * dphi_d[a] * dphi_d[b];
#pragma unroll
      for (int c = 0; c < 3; ++c) v -= GUDD(c, a, b) * dphi_d[c];
      Ddphi_dd[sidx(a, b)] = v;
    }
  double Stmp = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = c; d < 3; ++d)
      Stmp += ((c == d) ? 1.0 : 2.0) * GUU(c, d) *
              (Ddphi_dd[sidx(c, d)] + 2. * dphi_d[c] * dphi_d[d]);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const double rphi = 4. * dphi_d[a] * dphi_d[b] - 2. * Ddphi_dd[sidx(a, b)] -
                          2. * GDD(a, b) * Stmp;
      Rsum[sidx(a, b)] = R_dd[sidx(a, b)] + rphi;
    }
#undef GDDD
#undef GUDD
}

// The 22 right-hand-side values at one interior vertex without the
// Kreiss-Oliger terms, given Rsum_ab (rsum[q * stride]) and the advection sums
// (lv[n * stride]).  With LV = false the advection sums are left out (read
// as zero; lv is not read): the contracted path adds them, scaled, with the
// Kreiss-Oliger terms afterwards.
template <bool LV = true>
__device__ __forceinline__ void rhs_point(const double* __restrict__ u,
                                          const double* __restrict__ sd, int64_t nvol,
                                          int64_t p, const int64_t s[3],
                                          const DevParams& P, const FdScale& F,
                                          const double* __restrict__ rsum,
                                          const double* __restrict__ lv, int64_t stride,
                                          double out[NVAR]) {
  const z4c_params_t& opt = P.p;
  const double* U = u + p;
  const double* SD = sd + p;
  double g_dd[6], A_dd[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    g_dd[c] = __ldg(UV(Z4C_GXX + c));
    A_dd[c] = __ldg(UV(Z4C_AXX + c));
  }
  const double chi = __ldg(UV(Z4C_CHI)), Khat = __ldg(UV(Z4C_KHAT));
  const double Theta = __ldg(UV(Z4C_THETA)), alpha = __ldg(UV(Z4C_ALPHA));

  double g_uu[6], Gamma_udd[3][6], Gamma_u[3];
  christoffel(SD, nvol, g_dd, g_uu, nullptr, Gamma_udd, Gamma_u);
#define GUDD(c, a, b) Gamma_udd[c][sidx(a, b)]

  // :231-274
  const double K = Khat + 2. * Theta;
  const double chi_guarded = dmax(chi, opt.chi_div_floor);
  const double oochi = 1.0 / chi_guarded;
  double oopsi4;
  if (opt.chi_psi_power == -4.) oopsi4 = chi_guarded;
  else oopsi4 = pow(chi_guarded, -4. / opt.chi_psi_power);
  const double oochi_psi_power = 1.0 / opt.chi_psi_power;
  double dchi_d[3], dphi_d[3], dalpha_d[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    dchi_d[a] = SDV(kSdChi, a);
    dphi_d[a] = dchi_d[a] * oochi * oochi_psi_power;
    dalpha_d[a] = SDV(kSdAlpha, a);
  }

  // D D alpha, :482-521
  double Ddalpha = 0;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d) Ddalpha += GUU(c, d) * dphi_d[c] * dalpha_d[d];
  double ddalpha[6];
GATHER_LOOP
  for (int q = 0; q < 6; ++q) ddalpha[q] = fd_d2(UV(Z4C_ALPHA), SDF(kSdAlpha), nvol, q, s, F);
  double Ddalpha_dd[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const double ddal = ddalpha[sidx(a, b)];
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

  // A contractions, :525-589
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
      const double dKhat_b = fd_dx(UV(Z4C_KHAT), s[b], F.cidx1[b]);
      const double dTheta_b = fd_dx(UV(Z4C_THETA), s[b], F.cidx1[b]);
      sacc -= chi_pow_DA_u * A_uu[sidx(a, b)] * dchi_d[b] * oochi;
      sacc -= (1. / 3.) * GUU(a, b) * (2. * dKhat_b + dTheta_b);
    }
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c)
        sacc += ((b == c) ? 1.0 : 2.0) * GUDD(a, b, c) * A_uu[sidx(b, c)];
    DA_u[a] = sacc;
  }
#undef GUDD

  // Ricci scalar, Ht, :596-613
  double R = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b)
      R += ((a == b) ? 1.0 : 2.0) * oopsi4 * GUU(a, b) * __ldg(rsum + sidx(a, b) * stride);
  const double Ht = R + (2. / 3.) * (K * K) - trAA;

  // advective derivatives, :184-226
  double beta_u[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) beta_u[a] = __ldg(UV(Z4C_BETAX + a));
  // the advection sums, each read where it enters (lv[n * stride])
  auto Lv = [&](int n) {
    if constexpr (LV) return __ldg(lv + (int64_t)n * stride);
    else return 0.0;
  };
  double LGam_u[3], Lg_dd[6], LA_dd[6];

  // finalize Lie derivatives, :619-687
  double dbeta_du[3][3];  // [b][a] = d_b beta^a
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) dbeta_du[b][a] = SDV(kSdBeta + a, b);
  double dbeta = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) dbeta += dbeta_du[a][a];
  // ddbeta_ddu(a,b,c): second derivative along a,b of beta^c, :138-156
  double ddbeta[3][6];  // [c][pair(a,b)]
GATHER_LOOP
  for (int i = 0; i < 18; ++i) {
    const int c = i / 6, q = i % 6;
    ddbeta[c][q] = fd_d2(UV(Z4C_BETAX + c), SDF(kSdBeta + c), nvol, q, s, F);
  }
  double ddbeta_d[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) ddbeta_d[a] += (1. / 3.) * ddbeta[b][sidx(a, b)];
  const double Lchi = Lv(Z4C_CHI) + (1. / 6.) * opt.chi_psi_power * chi_guarded * dbeta;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    LGam_u[a] = Lv(Z4C_GAMX + a);
    LGam_u[a] += (2. / 3.) * Gamma_u[a] * dbeta;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      LGam_u[a] += GUU(a, b) * ddbeta_d[b] - Gamma_u[b] * dbeta_du[b][a];
#pragma unroll
      for (int c = b; c < 3; ++c)
        LGam_u[a] += ((b == c) ? 1.0 : 2.0) * GUU(b, c) * ddbeta[a][sidx(b, c)];
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double lg = Lv(Z4C_GXX + sidx(a, b)), la = Lv(Z4C_AXX + sidx(a, b));
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

  // assemble, :694-902 (matter fields are zero, so their terms vanish exactly)
  out[Z4C_KHAT] = -Ddalpha + alpha * (trAA + (1. / 3.) * (K * K)) + Lv(Z4C_KHAT) +
                  opt.damp_kappa1 * (1 - opt.damp_kappa2) * alpha * Theta;
  out[Z4C_CHI] = Lchi - (1. / 6.) * opt.chi_psi_power * chi_guarded * alpha * K;
  out[Z4C_THETA] = Lv(Z4C_THETA) + alpha * (0.5 * Ht - (2. + opt.damp_kappa2) * opt.damp_kappa1 * Theta);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double v = 2. * alpha * DA_u[a] + LGam_u[a];
    v -= 2. * alpha * opt.damp_kappa1 * (__ldg(UV(Z4C_GAMX + a)) - Gamma_u[a]);
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
      double v = oopsi4 * (-Ddalpha_dd[q] + alpha * __ldg(rsum + q * stride));
      v -= (1. / 3.) * g_dd[q] * (-Ddalpha + alpha * R);
      v += alpha * (K * A_dd[q] - 2. * AA_dd[q]);
      v += LA_dd[q];
      out[Z4C_AXX + q] = v;
    }
  {
    const double fl = opt.lapse_oplog * opt.lapse_harmonicf + opt.lapse_harmonic * alpha;
    out[Z4C_ALPHA] = (opt.lapse_advect * Lv(Z4C_ALPHA) - fl * alpha * (Khat + 2 * opt.lapse_K * Theta));
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double gam_a = __ldg(UV(Z4C_GAMX + a));
    double v = opt.shift_Gamma * gam_a + opt.shift_advect * Lv(Z4C_BETAX + a);
    if (fabs(opt.shift_alpha2Gamma) > 0.0) v += opt.shift_alpha2Gamma * (alpha * alpha) * gam_a;
    if (fabs(opt.shift_H) > 0.0) {
#pragma unroll
      for (int b = 0; b < 3; ++b)
        v += opt.shift_H * alpha * chi_guarded * (0.5 * alpha * dchi_d[b] - dalpha_d[b]) * GUU(a, b);
    }
    v -= opt.shift_eta * beta_u[a];
    out[Z4C_BETAX + a] = v;
  }
}

#undef UV
#undef SDF
#undef SDV
#undef GUU
#undef GDD
#undef ADD

}  // namespace z4c

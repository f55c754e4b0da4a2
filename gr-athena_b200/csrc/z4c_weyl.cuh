// Weyl scalar psi4 at one interior vertex: Z4c::Z4cWeyl,
// z4c/calculate_weyl_scalars.cpp:44-630 (vacuum).
//
// Inputs: the ADM variables (physical metric and extrinsic curvature), the
// Z4c state (conformal metric and chi) and the stored first derivatives of
// the Z4c state (the sd array of k_prep, the reference's
// PrepareZ4cDerivatives).  Every sum runs in the reference's order; the
// chain rule of the physical metric derivatives (:112-290), the Ricci tensor
// (:342-378), the covariant derivative of K (:383-420), the Gram-Schmidt
// tetrad (:426-524) and the three accumulation phases of psi4 (:532-630).
#pragma once

#include "z4c_common.cuh"
#include "z4c_rhs.cuh"

namespace z4c {

// First phase: with RICCI the spatial Ricci tensor Rd (symmetric, 6) and its
// trace R with the physical inverse metric, with DKPART the trace K of the
// extrinsic curvature and its covariant derivative DK[a][sym(b,c)] = D_a K_bc
// (18); each part recomputes the metric derivatives and Christoffels it
// needs, so that either runs on half the live state.
template <bool RICCI = true, bool DKPART = true>
__device__ __forceinline__ void weyl_curvature(const double* __restrict__ uB,
                                               const double* __restrict__ admB,
                                               const double* __restrict__ sdB, int64_t nvol,
                                               int64_t p, const int64_t s[3], const DevParams& P,
                                               const FdScale& F, double Rd[6], double& R,
                                               double& K, double DK[3][6]) {
  const z4c_params_t& opt = P.p;
  const double* U = uB + p;
  const double* AD = admB + p;
  const double* SD = sdB + p;
#define UV(n) (U + (int64_t)(n) * nvol)
#define AV(n) (AD + (int64_t)(n) * nvol)
#define WSDF(slot) (SD + (int64_t)(slot) * 3 * nvol)
#define WSDV(slot, dir) __ldg(SD + ((int64_t)(slot) * 3 + (dir)) * nvol)
  const double pw = opt.chi_psi_power;
  const double chi_g = dmax(__ldg(UV(Z4C_CHI)), opt.chi_div_floor);
  const double oochi = 1.0 / chi_g;
  const double fac = 4.0 / pw, fac2 = fac - 1.0;
  const double psi4c = (pw != -4.) ? pow(chi_g, fac) : 0.0;
  double gt[6], Kd[6], gph[6], dchi[3];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    gt[q] = __ldg(UV(Z4C_GXX + q));
    Kd[q] = __ldg(AV(Z4C_ADM_KXX + q));
    gph[q] = __ldg(AV(Z4C_ADM_GXX + q));
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) dchi[a] = WSDV(kSdChi, a);
  // pass 1: physical first derivatives of the metric, first derivatives of K
  double dg[3][6], dK[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const double d3 = WSDV(kSdG + q, c);
      if (pw == -4.) dg[c][q] = oochi * (d3 - oochi * gt[q] * dchi[c]);
      else dg[c][q] = psi4c * (d3 + fac * oochi * gt[q] * dchi[c]);
      if constexpr (DKPART) dK[c][q] = fd_dx(AV(Z4C_ADM_KXX + q), s[c], F.cidx1[c]);
    }
  double DDG[6][6];  // [sym(a,b)][sym(c,d)]
  if constexpr (RICCI) {
    // pass 2: physical second derivatives ddg(a,b,c,d) = d_a d_b gamma_cd; the
    // mixed a < b ones are D_a of the stored D_b g~_cd
#pragma unroll
    for (int ab = 0; ab < 6; ++ab) {
      const int a = pair_a(ab), b = pair_b(ab);
      const double ddchi = fd_d2(UV(Z4C_CHI), WSDF(kSdChi), nvol, ab, s, F);
      const double dchi_a = dchi[a], dchi_b = dchi[b];
#pragma unroll
      for (int cd = 0; cd < 6; ++cd) {
        const double gtil = gt[cd];
        const double ddg_conf = fd_d2(UV(Z4C_GXX + cd), WSDF(kSdG + cd), nvol, ab, s, F);
        const double da3 = WSDV(kSdG + cd, a), db3 = WSDV(kSdG + cd, b);
        double v;
        if (a == b) {
          if (pw == -4.)
            v = oochi * (ddg_conf - oochi * (2.0 * dchi_a * da3 + ddchi * gtil) +
                         2.0 * oochi * oochi * dchi_a * dchi_a * gtil);
          else
            v = psi4c * (ddg_conf + fac * oochi * (2.0 * dchi_a * da3 + ddchi * gtil) +
                         fac * fac2 * oochi * oochi * dchi_a * dchi_a * gtil);
        } else {
          if (pw == -4.)
            v = oochi * (ddg_conf - oochi * (dchi_a * db3 + dchi_b * da3 + ddchi * gtil) +
                         2.0 * oochi * oochi * dchi_a * dchi_b * gtil);
          else
            v = psi4c * (ddg_conf + fac * oochi * (dchi_a * db3 + dchi_b * da3 + ddchi * gtil) +
                         fac * fac2 * oochi * oochi * dchi_a * dchi_b * gtil);
        }
        DDG[ab][cd] = v;
      }
    }
  }
  // inverse physical metric
  double g_uu[6];
  {
    const double detg = det3(gph[0], gph[1], gph[2], gph[3], gph[4], gph[5]);
    inv3(1. / detg, gph, g_uu);
  }
#define GUU(a, b) g_uu[sidx(a, b)]
  // Christoffel symbols of the first and second kind
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
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) acc += GUU(c, d) * Gddd[d][sidx(a, b)];
        Gudd[c][sidx(a, b)] = acc;
      }
  if constexpr (RICCI) {
    // Ricci tensor and scalar
    R = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
#pragma unroll
            for (int e = 0; e < 3; ++e) {
              acc += GUU(c, d) * Gudd[e][sidx(a, c)] * Gddd[e][sidx(b, d)];
              acc -= GUU(c, d) * Gudd[e][sidx(a, b)] * Gddd[e][sidx(c, d)];
            }
            acc += 0.5 * GUU(c, d) *
                   (-DDG[sidx(c, d)][sidx(a, b)] - DDG[sidx(a, b)][sidx(c, d)] +
                    DDG[sidx(a, c)][sidx(b, d)] + DDG[sidx(b, c)][sidx(a, d)]);
          }
        Rd[sidx(a, b)] = acc;
        R += ((a == b) ? 1.0 : 2.0) * GUU(a, b) * acc;
      }
  }
  if constexpr (DKPART) {
    // trace of K and its covariant derivative DK(a,b,c) = D_a K_bc
    K = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double kaa = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) kaa += GUU(a, c) * Kd[sidx(c, a)];
      K += kaa;
    }
    // DK is stored symmetric in (b,c) and filled over all (b,c): the entry
    // b < c keeps the value of the later (c,b) pass, whose two subtractions run
    // in the other order
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int lo = 0; lo < 3; ++lo)
#pragma unroll
        for (int hi = lo; hi < 3; ++hi) {
          const int b = hi, c = lo;
          double v = dK[a][sidx(b, c)];
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            v -= Gudd[d][sidx(a, b)] * Kd[sidx(d, c)];
            v -= Gudd[d][sidx(a, c)] * Kd[sidx(b, d)];
          }
          DK[a][sidx(lo, hi)] = v;
        }
  }
#undef GUU
#undef UV
#undef AV
#undef WSDF
#undef WSDV
}

// Second phase at the vertex (x1, x2, x3): the Gram-Schmidt tetrad and the
// three accumulation phases of psi4 from the physical metric gph and K_ab
// (Kd) at the vertex and the first phase's Rd, R, K, DK.
__device__ __forceinline__ void weyl_contract(const double gph[6], const double Kd[6],
                                              const double Rd[6], double R, double K,
                                              const double DK[3][6], double x1, double x2,
                                              double x3, double* rpsi4, double* ipsi4) {
  double g_uu[6];
  {
    const double detg = det3(gph[0], gph[1], gph[2], gph[3], gph[4], gph[5]);
    inv3(1. / detg, gph, g_uu);
  }
#define GUU(a, b) g_uu[sidx(a, b)]
  // tetrad, orthonormalised with the physical metric
  double xx = x1;
  if (x1 * x1 + x2 * x2 < 1e-10) xx = xx + 1e-8;
  double uv[3] = {xx, x2, x3};
  double vv[3] = {xx * x3, x2 * x3, -(xx * xx) - (x2 * x2)};
  double wv[3] = {x2 * -1.0, xx, 0.0};
  auto gdot = [&](const double (&l)[3], const double (&r)[3]) -> double {
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) acc += gph[sidx(a, b)] * l[a] * r[b];
    return acc;
  };
  double dot = gdot(wv, wv);
#pragma unroll
  for (int a = 0; a < 3; ++a) wv[a] = wv[a] / sqrt(dot);
  dot = gdot(wv, uv);
#pragma unroll
  for (int a = 0; a < 3; ++a) uv[a] -= dot * wv[a];
  dot = gdot(uv, uv);
#pragma unroll
  for (int a = 0; a < 3; ++a) uv[a] = uv[a] / sqrt(dot);
  dot = gdot(wv, vv);
  const double dot2 = gdot(uv, vv);
#pragma unroll
  for (int a = 0; a < 3; ++a) vv[a] -= dot * wv[a] + dot2 * uv[a];
  dot = gdot(vv, vv);
#pragma unroll
  for (int a = 0; a < 3; ++a) vv[a] = vv[a] / sqrt(dot);
  // psi4 = -1/4 R4(l? n m* m*) assembled from the 3+1 pieces
  const double FR4 = 0.25;
  double rp = 0.0, ip = 0.0;
  // Ricci part with K K terms
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double R4 = Rd[sidx(a, b)] + K * Kd[sidx(a, b)];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) R4 -= GUU(c, d) * Kd[sidx(a, c)] * Kd[sidx(d, b)];
      const double Tr = vv[a] * vv[b] - wv[a] * wv[b];
      const double Ti = -vv[a] * wv[b] - wv[a] * vv[b];
      rp += -FR4 * R4 * Tr;
      ip += -FR4 * R4 * Ti;
    }
  // Codazzi part
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double Tr = vv[a] * vv[b] - wv[a] * wv[b];
      const double Ti = -vv[a] * wv[b] - wv[a] * vv[b];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double R4 = -(DK[b][sidx(a, c)] - DK[c][sidx(a, b)]);
        rp += 0.5 * R4 * uv[c] * Tr;
        ip += 0.5 * R4 * uv[c] * Ti;
      }
    }
  // Gauss part
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double Tr = vv[a] * vv[b] - wv[a] * wv[b];
      const double Ti = -vv[a] * wv[b] - wv[a] * vv[b];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double R4 = gph[sidx(d, c)] * Rd[sidx(a, b)] + gph[sidx(a, b)] * Rd[sidx(d, c)] -
                            gph[sidx(d, b)] * Rd[sidx(a, c)] - gph[sidx(a, c)] * Rd[sidx(d, b)] -
                            0.5 * R *
                                (gph[sidx(d, c)] * gph[sidx(a, b)] -
                                 gph[sidx(d, b)] * gph[sidx(a, c)]) +
                            Kd[sidx(d, c)] * Kd[sidx(a, b)] - Kd[sidx(d, b)] * Kd[sidx(a, c)];
          rp += -FR4 * R4 * uv[d] * uv[c] * Tr;
          ip += -FR4 * R4 * uv[d] * uv[c] * Ti;
        }
    }
  *rpsi4 = rp;
  *ipsi4 = ip;
#undef GUU
}

// Both phases at one interior vertex.
__device__ __forceinline__ void weyl_point(const double* __restrict__ uB,
                                           const double* __restrict__ admB,
                                           const double* __restrict__ sdB, int64_t nvol,
                                           int64_t p, const int64_t s[3], const DevParams& P,
                                           const FdScale& F, double x1, double x2, double x3,
                                           double* rpsi4, double* ipsi4) {
  double Rd[6], R, K, DK[3][6], gph[6], Kd[6];
  weyl_curvature(uB, admB, sdB, nvol, p, s, P, F, Rd, R, K, DK);
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    gph[q] = __ldg(admB + p + (int64_t)(Z4C_ADM_GXX + q) * nvol);
    Kd[q] = __ldg(admB + p + (int64_t)(Z4C_ADM_KXX + q) * nvol);
  }
  weyl_contract(gph, Kd, Rd, R, K, DK, x1, x2, x3, rpsi4, ipsi4);
}

}  // namespace z4c

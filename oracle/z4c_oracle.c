/* CPU restatement of the GR-Athena++ Z4c hot path: the parity oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see z4c_oracle.h).  Parity of this file with the
 * reference is pinned by tests/test_oracle_golden.py against record files
 * produced by the reference CPU build itself (oracle/ref, tests/golden).
 *
 * Floating-point expressions keep the reference's evaluation order (the
 * reference is built with -ffp-contract=off; so is this file).  Symmetric
 * tensors are held as full 3x3 arrays whose lower triangle mirrors the upper
 * one, which is how the reference's AthenaTensor SYM2 accessors read them.
 */
#define _GNU_SOURCE
#include "z4c_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NG ORC_NG
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---- finite differences, utils/finite_differencing.tpp with the
 *      DBG_SYMMETRIZE_FD stencils (defs.hpp.in:18 defines it) -------------- */

/* FDStencilCenteredDegreeOdd<1,3>, finite_differencing_stencils.tpp:266-272 */
static const double C1[3] = {-1, 9, -45};
static const double C1_LCM = 60;
/* FDStencilCenteredDegreeEven<2,3>, :316-322 */
static const double C2[4] = {2, -27, 270, -490};
static const double C2_LCM = 180;
/* FDStencilCenteredDegreeEven<8,4>, :372-378 */
static const double CD[5] = {1, -8, 28, -56, 70};
/* FDStencilBiasedLeft/Right<1,4,2>, :470-486 */
static const double CL[7] = {1, -8, 30, -80, 35, 24, -2};
static const double CR[7] = {2, -24, -35, 80, -30, 8, -1};
static const double CLR_LCM = 60;

typedef struct {
  int nn1, nn2, nn3;
  int64_t s[3];         /* strides */
  double cidx1[3], cidx2[3], cidxd[3], lidx[3];
  int il, iu, jl, ju, kl, ku; /* vertex interior range (ivs..ive) */
} fd_t;

static void fd_init(const orc_block_t *b, fd_t *f) {
  f->nn1 = b->nx[0] + 1 + 2 * NG;
  f->nn2 = b->nx[1] + 1 + 2 * NG;
  f->nn3 = b->nx[2] + 1 + 2 * NG;
  f->s[0] = 1;
  f->s[1] = f->nn1;
  f->s[2] = (int64_t)f->nn2 * f->nn1;
  /* finite_differencing.tpp:24 */
  const double diss_scaling = pow(2, -2 * NG) * (NG % 2 == 0 ? -1 : 1);
  for (int a = 0; a < 3; ++a) {
    const double dx = b->dx[a];
    f->cidx1[a] = 1.0 / (dx * C1_LCM);                 /* .tpp:36-38 */
    f->cidx2[a] = ((1.0 / dx) * (1.0 / dx)) / C2_LCM;  /* .tpp:40-42 */
    f->cidxd[a] = diss_scaling / (dx * 1.0);           /* .tpp:48-50 */
    f->lidx[a] = 1.0 / (dx * CLR_LCM);                 /* .tpp:53-55 */
  }
  f->il = NG; f->iu = NG + b->nx[0];
  f->jl = NG; f->ju = NG + b->nx[1];
  f->kl = NG; f->ku = NG + b->nx[2];
}

/* Uniform::Dx, finite_differencing.tpp:63-112 (symmetrized branch) */
static inline double Dx(const fd_t *f, int dir, const double *u) {
  const int64_t s = f->s[dir];
  const double *pu = u - 3 * s;
  double out = 0.;
  for (int n1 = 0; n1 < 3; ++n1) {
    const int n2 = 6 - n1;
    out += C1[n1] * (pu[n1 * s] - pu[n2 * s]);
  }
  return out * f->cidx1[dir];
}

/* Uniform::Dxx, finite_differencing.tpp:196-236 */
static inline double Dxx(const fd_t *f, int dir, const double *u) {
  const int64_t s = f->s[dir];
  const double *pu = u - 3 * s;
  double out = 0.;
  for (int n1 = 0; n1 < 3; ++n1) {
    const int n2 = 6 - n1;
    out += C2[n1] * (pu[n1 * s] + pu[n2 * s]);
  }
  out += C2[3] * pu[3 * s];
  return out * f->cidx2[dir];
}

/* Uniform::Diss, finite_differencing.tpp:335-352 */
static inline double Diss(const fd_t *f, int dir, const double *u, double diss) {
  const int64_t s = f->s[dir];
  const double *pu = u - 4 * s;
  double out = 0.;
  for (int n1 = 0; n1 < 4; ++n1) {
    const int n2 = 8 - n1;
    out += CD[n1] * (pu[n1 * s] + pu[n2 * s]);
  }
  out += CD[4] * pu[4 * s];
  return out * f->cidxd[dir] * diss;
}

/* Uniform::Lx, finite_differencing.tpp:152-174 */
static inline double Lx(const fd_t *f, int dir, double vx, const double *u) {
  const int64_t s = f->s[dir];
  double dl = 0.;
  for (int n = 0; n < 7; ++n) dl += CL[n] * u[(n - 4) * s];
  double dr = 0.;
  for (int n = 6; n >= 0; --n) dr += CR[n] * u[(n - 2) * s];
  return ((vx < 0) ? (vx * dl) : (vx * dr)) * f->lidx[dir];
}

/* ---- small linear algebra, utils/linear_algebra.hpp -------------------- */

static const int SI[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

/* Det3Metric, linear_algebra.hpp:47-56 */
static inline double det3(double gxx, double gxy, double gxz, double gyy,
                          double gyz, double gzz) {
  return (-(gxz * gxz) * gyy + 2 * gxy * gxz * gyz - gxx * (gyz * gyz) -
          (gxy * gxy) * gzz + gxx * gyy * gzz);
}

/* Inv3Metric, linear_algebra.hpp:98-118 */
static inline void inv3(double oodetg, double gxx, double gxy, double gxz,
                        double gyy, double gyz, double gzz, double g_uu[3][3]) {
  const double uxx = (-(gyz * gyz) + gyy * gzz) * oodetg;
  const double uxy = (gxz * gyz - gxy * gzz) * oodetg;
  const double uyy = (-(gxz * gxz) + gxx * gzz) * oodetg;
  const double uxz = (-gxz * gyy + gxy * gyz) * oodetg;
  const double uyz = (gxy * gxz - gxx * gyz) * oodetg;
  const double uzz = (-(gxy * gxy) + gxx * gyy) * oodetg;
  g_uu[0][0] = uxx; g_uu[0][1] = uxy; g_uu[0][2] = uxz;
  g_uu[1][0] = uxy; g_uu[1][1] = uyy; g_uu[1][2] = uyz;
  g_uu[2][0] = uxz; g_uu[2][1] = uyz; g_uu[2][2] = uzz;
}

/* TraceRank2, linear_algebra.hpp:271-290 */
static inline double trace_rank2(double detginv, double gxx, double gxy,
                                 double gxz, double gyy, double gyz, double gzz,
                                 double Axx, double Axy, double Axz, double Ayy,
                                 double Ayz, double Azz) {
  return detginv * (-2. * Ayz * gxx * gyz + Axx * gyy * gzz +
                    gxx * (Azz * gyy + Ayy * gzz) +
                    2. * (gxz * (Ayz * gxy - Axz * gyy + Axy * gyz) +
                          gxy * (Axz * gyz - Axy * gzz)) -
                    Azz * (gxy * gxy) - Ayy * (gxz * gxz) - Axx * (gyz * gyz));
}

/* regularize_nth_root, utils/floating_point.hpp:120-131 */
static inline double regularize_nth_root(double value, double value_reg,
                                         double eps_floor, double npow) {
  const double eps = value - value_reg;
  return ((eps < eps_floor) ? (1.0 + eps_floor / npow) : pow(value, 1.0 / npow));
}

/* regularize_near_zero, floating_point.hpp:110-115 */
static inline double regularize_near_zero(double value, double value_eps) {
  return (value >= 0) ? ((value < value_eps) ? value_eps : value)
                      : ((value > -value_eps) ? -value_eps : value);
}

static inline double dmax(double a, double b) { return (a < b) ? b : a; }

/* ---- storage ------------------------------------------------------------ */

int64_t orc_nvol(const orc_block_t *b) {
  return (int64_t)(b->nx[0] + 1 + 2 * NG) * (b->nx[1] + 1 + 2 * NG) *
         (b->nx[2] + 1 + 2 * NG);
}

int orc_derivs_alloc(const orc_block_t *b, orc_derivs_t *d) {
  const int64_t n = orc_nvol(b);
  memset(d, 0, sizeof(*d));
  double **slots[3 + 3 + 9 + 18 + 6];
  int ns = 0;
  for (int a = 0; a < 3; ++a) slots[ns++] = &d->dalpha[a];
  for (int a = 0; a < 3; ++a) slots[ns++] = &d->dchi[a];
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c) slots[ns++] = &d->dbeta[a][c];
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 6; ++c) slots[ns++] = &d->dg[a][c];
  for (int c = 0; c < 6; ++c) slots[ns++] = &d->ddchi[c];
  for (int s = 0; s < ns; ++s) {
    *slots[s] = (double *)calloc((size_t)n, sizeof(double));
    if (!*slots[s]) { orc_derivs_free(d); return -1; }
  }
  return 0;
}

void orc_derivs_free(orc_derivs_t *d) {
  for (int a = 0; a < 3; ++a) {
    free(d->dalpha[a]); free(d->dchi[a]);
    for (int c = 0; c < 3; ++c) free(d->dbeta[a][c]);
    for (int c = 0; c < 6; ++c) free(d->dg[a][c]);
  }
  for (int c = 0; c < 6; ++c) free(d->ddchi[c]);
  memset(d, 0, sizeof(*d));
}

#define V(u, n) ((u) + (int64_t)(n) * nvol)
#define P(k, j, i) (((int64_t)(k) * f.nn2 + (j)) * f.nn1 + (i))

/* ---- Z4c::PrepareZ4cDerivatives, adm_z4c.cpp:972-1037 ------------------ */
void orc_prepare_derivs(const orc_block_t *b, const double *u, orc_derivs_t *d) {
  fd_t f;
  fd_init(b, &f);
  const int64_t nvol = orc_nvol(b);
  const int ng_ext = NG - 1;
  for (int bd = 0; bd < 3; ++bd) {
    const int klo = (bd == 2) ? f.kl : f.kl - ng_ext;
    const int khi = (bd == 2) ? f.ku : f.ku + ng_ext;
    const int jlo = (bd == 1) ? f.jl : f.jl - ng_ext;
    const int jhi = (bd == 1) ? f.ju : f.ju + ng_ext;
    const int ilo = (bd == 0) ? f.il : f.il - ng_ext;
    const int ihi = (bd == 0) ? f.iu : f.iu + ng_ext;
    for (int k = klo; k <= khi; ++k)
      for (int j = jlo; j <= jhi; ++j)
        for (int i = ilo; i <= ihi; ++i) {
          const int64_t p = P(k, j, i);
          d->dalpha[bd][p] = Dx(&f, bd, V(u, Z4C_ALPHA) + p);
          d->dchi[bd][p] = Dx(&f, bd, V(u, Z4C_CHI) + p);
          for (int c = 0; c < 3; ++c)
            d->dbeta[bd][c][p] = Dx(&f, bd, V(u, Z4C_BETAX + c) + p);
          for (int c = 0; c < 6; ++c)
            d->dg[bd][c][p] = Dx(&f, bd, V(u, Z4C_GXX + c) + p);
        }
  }
  for (int a = 0; a < 3; ++a) {
    for (int k = f.kl; k <= f.ku; ++k)
      for (int j = f.jl; j <= f.ju; ++j)
        for (int i = f.il; i <= f.iu; ++i) {
          const int64_t p = P(k, j, i);
          d->ddchi[SI[a][a]][p] = Dxx(&f, a, V(u, Z4C_CHI) + p);
        }
    for (int bb = a + 1; bb < 3; ++bb)
      for (int k = f.kl; k <= f.ku; ++k)
        for (int j = f.jl; j <= f.ju; ++j)
          for (int i = f.il; i <= f.iu; ++i) {
            const int64_t p = P(k, j, i);
            d->ddchi[SI[a][bb]][p] = Dx(&f, a, d->dchi[bb] + p);
          }
  }
}

/* ---- Z4c::Z4cRHS, calculate_z4c_rhs.cpp:29-916 -------------------------- */
void orc_rhs(const orc_block_t *b, const z4c_params_t *opt, const double *u,
             const orc_derivs_t *D, double *rhs) {
  fd_t f;
  fd_init(b, &f);
  const int64_t nvol = orc_nvol(b);
  const double oochi_psi_power = 1.0 / opt->chi_psi_power;
  const double chi_pow_DA_u = -6.0 / opt->chi_psi_power;
  const double rho = 0.0, S_d[3] = {0, 0, 0};  /* vacuum matter fields */

  for (int k = f.kl; k <= f.ku; ++k)
    for (int j = f.jl; j <= f.ju; ++j)
      for (int i = f.il; i <= f.iu; ++i) {
        const int64_t p = P(k, j, i);
        double g_dd[3][3], A_dd[3][3], beta_u[3], Gam_u[3];
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) {
            g_dd[a][c] = V(u, Z4C_GXX + SI[a][c])[p];
            A_dd[a][c] = V(u, Z4C_AXX + SI[a][c])[p];
          }
        for (int a = 0; a < 3; ++a) {
          beta_u[a] = V(u, Z4C_BETAX + a)[p];
          Gam_u[a] = V(u, Z4C_GAMX + a)[p];
        }
        const double chi = V(u, Z4C_CHI)[p], Khat = V(u, Z4C_KHAT)[p];
        const double Theta = V(u, Z4C_THETA)[p], alpha = V(u, Z4C_ALPHA)[p];

        /* 1st derivatives, :84-114 */
        double dalpha_d[3], dchi_d[3], dKhat_d[3], dTheta_d[3];
        double dbeta_du[3][3], dGam_du[3][3], dg_ddd[3][3][3], dA_ddd[3][3][3];
        for (int a = 0; a < 3; ++a) {
          dalpha_d[a] = D->dalpha[a][p];
          dchi_d[a] = D->dchi[a][p];
          dKhat_d[a] = Dx(&f, a, V(u, Z4C_KHAT) + p);
          dTheta_d[a] = Dx(&f, a, V(u, Z4C_THETA) + p);
        }
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) {
            dbeta_du[bb][a] = D->dbeta[bb][a][p];
            dGam_du[bb][a] = Dx(&f, bb, V(u, Z4C_GAMX + a) + p);
          }
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            for (int c = 0; c < 3; ++c) {
              dg_ddd[c][a][bb] = dg_ddd[c][bb][a] = D->dg[c][SI[a][bb]][p];
              dA_ddd[c][a][bb] = dA_ddd[c][bb][a] =
                  Dx(&f, c, V(u, Z4C_AXX + SI[a][bb]) + p);
            }

        /* 2nd derivatives, :121-178 */
        double ddalpha_dd[3][3], ddchi_dd[3][3], ddbeta_ddu[3][3][3];
        double ddg_dddd[3][3][3][3];
        for (int a = 0; a < 3; ++a) {
          ddalpha_dd[a][a] = Dxx(&f, a, V(u, Z4C_ALPHA) + p);
          ddchi_dd[a][a] = D->ddchi[SI[a][a]][p];
          for (int bb = a + 1; bb < 3; ++bb) {
            ddalpha_dd[a][bb] = ddalpha_dd[bb][a] = Dx(&f, a, D->dalpha[bb] + p);
            ddchi_dd[a][bb] = ddchi_dd[bb][a] = D->ddchi[SI[a][bb]][p];
          }
        }
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb) {
              double v;
              if (a == bb) v = Dxx(&f, a, V(u, Z4C_BETAX + c) + p);
              else v = Dx(&f, a, D->dbeta[bb][c] + p);
              ddbeta_ddu[a][bb][c] = ddbeta_ddu[bb][a][c] = v;
            }
        for (int c = 0; c < 3; ++c)
          for (int dd = c; dd < 3; ++dd)
            for (int a = 0; a < 3; ++a)
              for (int bb = a; bb < 3; ++bb) {
                double v;
                if (a == bb) v = Dxx(&f, a, V(u, Z4C_GXX + SI[c][dd]) + p);
                else v = Dx(&f, a, D->dg[bb][SI[c][dd]] + p);
                ddg_dddd[a][bb][c][dd] = ddg_dddd[bb][a][c][dd] =
                    ddg_dddd[a][bb][dd][c] = ddg_dddd[bb][a][dd][c] = v;
              }

        /* advective derivatives, :184-226 */
        double Lalpha = 0, Lchi = 0, LKhat = 0, LTheta = 0;
        for (int a = 0; a < 3; ++a) {
          Lalpha += Lx(&f, a, beta_u[a], V(u, Z4C_ALPHA) + p);
          Lchi += Lx(&f, a, beta_u[a], V(u, Z4C_CHI) + p);
          LKhat += Lx(&f, a, beta_u[a], V(u, Z4C_KHAT) + p);
          LTheta += Lx(&f, a, beta_u[a], V(u, Z4C_THETA) + p);
        }
        double Lbeta_u[3] = {0, 0, 0}, LGam_u[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) {
            Lbeta_u[bb] += Lx(&f, a, beta_u[a], V(u, Z4C_BETAX + bb) + p);
            LGam_u[bb] += Lx(&f, a, beta_u[a], V(u, Z4C_GAMX + bb) + p);
          }
        double Lg_dd[3][3] = {{0}}, LA_dd[3][3] = {{0}};
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            for (int c = 0; c < 3; ++c) {
              Lg_dd[a][bb] += Lx(&f, c, beta_u[c], V(u, Z4C_GXX + SI[a][bb]) + p);
              LA_dd[a][bb] += Lx(&f, c, beta_u[c], V(u, Z4C_AXX + SI[a][bb]) + p);
            }

        /* :231-274 */
        const double K = Khat + 2. * Theta;
        const double chi_guarded = dmax(chi, opt->chi_div_floor);
        const double oochi = 1.0 / chi_guarded;
        double oopsi4;
        if (opt->chi_psi_power == -4.) oopsi4 = chi_guarded;
        else oopsi4 = pow(chi_guarded, -4. / opt->chi_psi_power);

        /* inverse conformal metric, :295-311 */
        double g_uu[3][3];
        {
          const double detg = det3(g_dd[0][0], g_dd[0][1], g_dd[0][2], g_dd[1][1],
                                   g_dd[1][2], g_dd[2][2]);
          inv3(1.0 / detg, g_dd[0][0], g_dd[0][1], g_dd[0][2], g_dd[1][1],
               g_dd[1][2], g_dd[2][2], g_uu);
        }

        /* Christoffels, :317-352 */
        double Gamma_ddd[3][3][3], Gamma_udd[3][3][3], Gamma_u[3];
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb)
              Gamma_ddd[c][a][bb] = Gamma_ddd[c][bb][a] =
                  0.5 * (dg_ddd[a][bb][c] + dg_ddd[bb][a][c] - dg_ddd[c][a][bb]);
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb) {
              double s = 0;
              for (int dd = 0; dd < 3; ++dd) s += g_uu[c][dd] * Gamma_ddd[dd][a][bb];
              Gamma_udd[c][a][bb] = Gamma_udd[c][bb][a] = s;
            }
        for (int a = 0; a < 3; ++a) {
          double s = 0;
          for (int bb = 0; bb < 3; ++bb)
            for (int c = bb; c < 3; ++c)
              s += ((bb == c) ? 1.0 : 2.0) * g_uu[bb][c] * Gamma_udd[a][bb][c];
          Gamma_u[a] = s;
        }

        /* Ricci of the conformal metric, :357-396 */
        double R_dd[3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            double s = 0;
            for (int c = 0; c < 3; ++c)
              s += 0.5 * (g_dd[c][a] * dGam_du[bb][c] + g_dd[c][bb] * dGam_du[a][c] +
                          Gamma_u[c] * (Gamma_ddd[a][bb][c] + Gamma_ddd[bb][a][c]));
            for (int c = 0; c < 3; ++c)
              for (int dd = c; dd < 3; ++dd)
                s -= ((c == dd) ? 0.5 : 1.0) * g_uu[c][dd] * ddg_dddd[c][dd][a][bb];
            for (int c = 0; c < 3; ++c)
              for (int dd = 0; dd < 3; ++dd)
                for (int e = 0; e < 3; ++e)
                  s += g_uu[c][dd] * (Gamma_udd[e][c][a] * Gamma_ddd[bb][e][dd] +
                                      Gamma_udd[e][c][bb] * Gamma_ddd[a][e][dd] +
                                      Gamma_udd[e][a][dd] * Gamma_ddd[e][c][bb]);
            R_dd[a][bb] = R_dd[bb][a] = s;
          }

        /* conformal factor derivatives, :402-426 */
        double dphi_d[3], Ddphi_dd[3][3];
        for (int a = 0; a < 3; ++a) dphi_d[a] = dchi_d[a] * oochi * oochi_psi_power;
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            double v = ddchi_dd[a][bb] * oochi * oochi_psi_power -
                       opt->chi_psi_power * dphi_d[a] * dphi_d[bb];
            for (int c = 0; c < 3; ++c) v -= Gamma_udd[c][a][bb] * dphi_d[c];
            Ddphi_dd[a][bb] = Ddphi_dd[bb][a] = v;
          }

        /* Rphi, :436-458 */
        double Stmp = 0.0;
        for (int c = 0; c < 3; ++c)
          for (int dd = c; dd < 3; ++dd)
            Stmp += ((c == dd) ? 1.0 : 2.0) * g_uu[c][dd] *
                    (Ddphi_dd[c][dd] + 2. * dphi_d[c] * dphi_d[dd]);
        double Rphi_dd[3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            Rphi_dd[a][bb] = Rphi_dd[bb][a] = 4. * dphi_d[a] * dphi_d[bb] -
                                              2. * Ddphi_dd[a][bb] -
                                              2. * g_dd[a][bb] * Stmp;

        /* matter trace (zero matter), :465-474 */
        double S = 0;
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            S += ((a == bb) ? 1.0 : 2.0) * oopsi4 * g_uu[a][bb] * 0.0;

        /* D D alpha, :482-521 */
        double Ddalpha = 0;
        for (int c = 0; c < 3; ++c)
          for (int dd = 0; dd < 3; ++dd) Ddalpha += g_uu[c][dd] * dphi_d[c] * dalpha_d[dd];
        double Ddalpha_dd[3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            double v = ddalpha_dd[a][bb] -
                       2. * (dphi_d[a] * dalpha_d[bb] + dphi_d[bb] * dalpha_d[a]) +
                       2. * g_dd[a][bb] * Ddalpha;
            for (int c = 0; c < 3; ++c) v -= Gamma_udd[c][a][bb] * dalpha_d[c];
            Ddalpha_dd[a][bb] = Ddalpha_dd[bb][a] = v;
          }
        Ddalpha = 0;
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            Ddalpha += ((a == bb) ? 1.0 : 2.0) * oopsi4 * g_uu[a][bb] * Ddalpha_dd[a][bb];

        /* A contractions, :525-589 */
        double A_ud[3][3], AA_dd[3][3], A_uu[3][3], DA_u[3];
        for (int c = 0; c < 3; ++c)
          for (int bb = 0; bb < 3; ++bb) {
            double s = 0;
            for (int dd = 0; dd < 3; ++dd) s += g_uu[c][dd] * A_dd[dd][bb];
            A_ud[c][bb] = s;
          }
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            double s = 0;
            for (int c = 0; c < 3; ++c) s += A_dd[a][c] * A_ud[c][bb];
            AA_dd[a][bb] = AA_dd[bb][a] = s;
          }
        double trAA = 0;
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            trAA += ((a == bb) ? 1.0 : 2.0) * g_uu[a][bb] * AA_dd[a][bb];
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            double s = 0;
            for (int c = 0; c < 3; ++c) s += g_uu[bb][c] * A_ud[a][c];
            A_uu[a][bb] = A_uu[bb][a] = s;
          }
        for (int a = 0; a < 3; ++a) {
          double s = 0;
          for (int bb = 0; bb < 3; ++bb) {
            s -= chi_pow_DA_u * A_uu[a][bb] * dchi_d[bb] * oochi;
            s -= (1. / 3.) * g_uu[a][bb] * (2. * dKhat_d[bb] + dTheta_d[bb]);
          }
          for (int bb = 0; bb < 3; ++bb)
            for (int c = bb; c < 3; ++c)
              s += ((bb == c) ? 1.0 : 2.0) * Gamma_udd[a][bb][c] * A_uu[bb][c];
          DA_u[a] = s;
        }

        /* Ricci scalar and Ht, :596-613 */
        double R = 0;
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            R += ((a == bb) ? 1.0 : 2.0) * oopsi4 * g_uu[a][bb] *
                 (R_dd[a][bb] + Rphi_dd[a][bb]);
        const double Ht = R + (2. / 3.) * (K * K) - trAA;

        /* Lie derivatives, :619-687 */
        double dbeta = 0;
        for (int a = 0; a < 3; ++a) dbeta += dbeta_du[a][a];
        double ddbeta_d[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) ddbeta_d[a] += (1. / 3.) * ddbeta_ddu[a][bb][bb];
        Lchi += (1. / 6.) * opt->chi_psi_power * chi_guarded * dbeta;
        for (int a = 0; a < 3; ++a) {
          LGam_u[a] += (2. / 3.) * Gamma_u[a] * dbeta;
          for (int bb = 0; bb < 3; ++bb) {
            LGam_u[a] += g_uu[a][bb] * ddbeta_d[bb] - Gamma_u[bb] * dbeta_du[bb][a];
            for (int c = bb; c < 3; ++c)
              LGam_u[a] += ((bb == c) ? 1.0 : 2.0) * g_uu[bb][c] * ddbeta_ddu[bb][c][a];
          }
        }
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            Lg_dd[a][bb] -= (2. / 3.) * g_dd[a][bb] * dbeta;
            LA_dd[a][bb] -= (2. / 3.) * A_dd[a][bb] * dbeta;
            for (int c = 0; c < 3; ++c) {
              Lg_dd[a][bb] += dbeta_du[a][c] * g_dd[bb][c];
              LA_dd[a][bb] += dbeta_du[bb][c] * A_dd[a][c];
              Lg_dd[a][bb] += dbeta_du[bb][c] * g_dd[a][c];
              LA_dd[a][bb] += dbeta_du[a][c] * A_dd[bb][c];
            }
          }

        /* assemble, :694-902 */
        double r_Khat = -Ddalpha + alpha * (trAA + (1. / 3.) * (K * K)) + LKhat +
                        opt->damp_kappa1 * (1 - opt->damp_kappa2) * alpha * Theta;
        r_Khat += 4 * M_PI * alpha * (S + rho);
        const double r_chi = Lchi - (1. / 6.) * opt->chi_psi_power * chi_guarded * alpha * K;
        double r_Theta = LTheta + alpha * (0.5 * Ht - (2. + opt->damp_kappa2) *
                                                          opt->damp_kappa1 * Theta);
        r_Theta -= 8. * M_PI * alpha * rho;
        V(rhs, Z4C_KHAT)[p] = r_Khat;
        V(rhs, Z4C_CHI)[p] = r_chi;
        V(rhs, Z4C_THETA)[p] = r_Theta;
        for (int a = 0; a < 3; ++a) {
          double v = 2. * alpha * DA_u[a] + LGam_u[a];
          v -= 2. * alpha * opt->damp_kappa1 * (Gam_u[a] - Gamma_u[a]);
          for (int bb = 0; bb < 3; ++bb) {
            v -= 2. * A_uu[a][bb] * dalpha_d[bb];
            v -= 16. * M_PI * alpha * g_uu[a][bb] * S_d[bb];
          }
          V(rhs, Z4C_GAMX + a)[p] = v;
        }
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            V(rhs, Z4C_GXX + SI[a][bb])[p] = -2. * alpha * A_dd[a][bb] + Lg_dd[a][bb];
            double v = oopsi4 * (-Ddalpha_dd[a][bb] + alpha * (R_dd[a][bb] + Rphi_dd[a][bb]));
            v -= (1. / 3.) * g_dd[a][bb] * (-Ddalpha + alpha * R);
            v += alpha * (K * A_dd[a][bb] - 2. * AA_dd[a][bb]);
            v += LA_dd[a][bb];
            v -= 8. * M_PI * alpha * (oopsi4 * 0.0 - (1. / 3.) * S * g_dd[a][bb]);
            V(rhs, Z4C_AXX + SI[a][bb])[p] = v;
          }
        {
          const double fl = opt->lapse_oplog * opt->lapse_harmonicf + opt->lapse_harmonic * alpha;
          V(rhs, Z4C_ALPHA)[p] = (opt->lapse_advect * Lalpha -
                                  fl * alpha * (Khat + 2 * opt->lapse_K * Theta));
        }
        for (int a = 0; a < 3; ++a) {
          double v = opt->shift_Gamma * Gam_u[a] + opt->shift_advect * Lbeta_u[a];
          if (fabs(opt->shift_alpha2Gamma) > 0.0)
            v += opt->shift_alpha2Gamma * (alpha * alpha) * Gam_u[a];
          if (fabs(opt->shift_H) > 0.0)
            for (int bb = 0; bb < 3; ++bb)
              v += opt->shift_H * alpha * chi_guarded *
                   (0.5 * alpha * dchi_d[bb] - dalpha_d[bb]) * g_uu[a][bb];
          v -= opt->shift_eta * beta_u[a];
          V(rhs, Z4C_BETAX + a)[p] = v;
        }
      }

  /* Kreiss-Oliger dissipation, :908-915 */
  for (int n = 0; n < Z4C_NVAR; ++n)
    for (int k = f.kl; k <= f.ku; ++k)
      for (int j = f.jl; j <= f.ju; ++j)
        for (int i = f.il; i <= f.iu; ++i) {
          const int64_t p = P(k, j, i);
          for (int a = 0; a < 3; ++a)
            V(rhs, n)[p] += Diss(&f, a, V(u, n) + p, opt->diss);
        }
}

/* ---- Z4c::Z4cBoundaryRHS, z4c/boundary_conditions.cpp:16-174 ------------ */

/* Uniform::Ds with DBG_SYMMETRIZE_FD (finite_differencing.tpp:132-150):
 * FDStencilCenteredDegreeOdd<1,1> = {-1} / 2. */
static inline double Ds(const fd_t *f, int dir, const double *u, double cidx1_lo) {
  const int64_t s = f->s[dir];
  double out = 0.;
  out += -1. * (u[-s] - u[s]);
  return out * cidx1_lo;
}

/* Z4c::Z4cSommerfeld_ (:66-174) at one vertex p with coordinates x, y, z. */
static void sommerfeld_point(const fd_t *f, const double cl[3], const double *u, double *rhs,
                             int64_t p, double x, double y, double z) {
  const int64_t nvol = (int64_t)f->nn1 * f->nn2 * f->nn3;
  double dKhat[3], dTheta[3], dGam[3][3], dA[3][6];
  for (int a = 0; a < 3; ++a) {
    dKhat[a] = Ds(f, a, u + Z4C_KHAT * nvol + p, cl[a]);
    dTheta[a] = Ds(f, a, u + Z4C_THETA * nvol + p, cl[a]);
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) dGam[b][a] = Ds(f, b, u + (Z4C_GAMX + a) * nvol + p, cl[b]);
  for (int q = 0; q < 6; ++q)
    for (int c = 0; c < 3; ++c) dA[c][q] = Ds(f, c, u + (Z4C_AXX + q) * nvol + p, cl[c]);
  const double r = sqrt(x * x + y * y + z * z);
  const double s_u[3] = {x / r, y / r, z / r};
  double th = -u[Z4C_THETA * nvol + p] / r;
  double kh = -sqrt(2.) * u[Z4C_KHAT * nvol + p] / r;
  for (int a = 0; a < 3; ++a) {
    th -= s_u[a] * dTheta[a];
    kh -= sqrt(2.) * s_u[a] * dKhat[a];
  }
  rhs[Z4C_THETA * nvol + p] = th;
  rhs[Z4C_KHAT * nvol + p] = kh;
  for (int a = 0; a < 3; ++a) {
    double v = -u[(Z4C_GAMX + a) * nvol + p] / r;
    for (int b = 0; b < 3; ++b) v -= s_u[b] * dGam[b][a];
    rhs[(Z4C_GAMX + a) * nvol + p] = v;
  }
  for (int q = 0; q < 6; ++q) {
    double v = -u[(Z4C_AXX + q) * nvol + p] / r;
    for (int c = 0; c < 3; ++c) v -= s_u[c] * dA[c][q];
    rhs[(Z4C_AXX + q) * nvol + p] = v;
  }
}

void orc_boundary_rhs(const orc_block_t *b, const double *u, double *rhs, const int som[6]) {
  fd_t f;
  fd_init(b, &f);
  /* cidx1_lo, finite_differencing.tpp:43-45 */
  const double cl[3] = {1.0 / (b->dx[0] * 2), 1.0 / (b->dx[1] * 2), 1.0 / (b->dx[2] * 2)};
  for (int face = 0; face < 6; ++face) {
    if (!som[face]) continue;
    const int ax = face / 2;
    int lo[3] = {f.il, f.jl, f.kl}, hi[3] = {f.iu, f.ju, f.ku};
    if (face % 2 == 0) hi[ax] = lo[ax];
    else lo[ax] = hi[ax];
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i)
          sommerfeld_point(&f, cl, u, rhs, P(k, j, i), b->x[0][i], b->x[1][j], b->x[2][k]);
  }
}

/* ---- Z4c::AlgConstr, z4c.cpp:677-799 / 801-991 --------------------------- */
static void algconstr_point(const z4c_params_t *opt, double *u, int64_t nvol,
                            int64_t p) {
  double *g[6], *A[6];
  for (int c = 0; c < 6; ++c) {
    g[c] = V(u, Z4C_GXX + c) + p;
    A[c] = V(u, Z4C_AXX + c) + p;
  }
  if (opt->tf_force_regularization) {
    double detg = det3(*g[0], *g[1], *g[2], *g[3], *g[4], *g[5]);
    detg = detg > 0. ? detg : 1.;
    const double oopsi4 = regularize_nth_root(detg, 1.0, opt->eps_floor, -3.0);
    for (int c = 0; c < 6; ++c) *g[c] *= oopsi4;
    const double tr = trace_rank2(1.0, *g[0], *g[1], *g[2], *g[3], *g[4], *g[5],
                                  *A[0], *A[1], *A[2], *A[3], *A[4], *A[5]);
    for (int c = 0; c < 6; ++c) *A[c] -= (1.0 / 3.0) * tr * *g[c];
  } else {
    const double detg = det3(*g[0], *g[1], *g[2], *g[3], *g[4], *g[5]);
    if (detg > opt->eps_floor) {
      const double oopsi4 = regularize_nth_root(detg, 1.0, opt->eps_floor, -3.0);
      for (int c = 0; c < 6; ++c) *g[c] *= oopsi4;
      const double tr = trace_rank2(1.0, *g[0], *g[1], *g[2], *g[3], *g[4], *g[5],
                                    *A[0], *A[1], *A[2], *A[3], *A[4], *A[5]);
      for (int c = 0; c < 6; ++c) *A[c] -= (1.0 / 3.0) * tr * *g[c];
    }
  }
  if (opt->force_regularization) {
    double *chi = V(u, Z4C_CHI) + p, *alpha = V(u, Z4C_ALPHA) + p;
    *chi = dmax(*chi, opt->eps_floor);
    *alpha = regularize_near_zero(*alpha, opt->eps_floor);
  }
}

void orc_algconstr(const orc_block_t *b, const z4c_params_t *opt, double *u) {
  const int64_t nvol = orc_nvol(b);
  for (int64_t p = 0; p < nvol; ++p) algconstr_point(opt, u, nvol, p);
}

void orc_algconstr_ghosts(const orc_block_t *b, const z4c_params_t *opt, double *u) {
  fd_t f;
  fd_init(b, &f);
  const int64_t nvol = orc_nvol(b);
  for (int k = 0; k < f.nn3; ++k)
    for (int j = 0; j < f.nn2; ++j)
      for (int i = 0; i < f.nn1; ++i) {
        const int interior = (k >= f.kl && k <= f.ku && j >= f.jl && j <= f.ju &&
                              i >= f.il && i <= f.iu);
        if (!interior) algconstr_point(opt, u, nvol, P(k, j, i));
      }
}

/* ---- Z4c::Z4cToADM, adm_z4c.cpp:200-260 --------------------------------- */
static void z4c_to_adm_point(const z4c_params_t *opt, const double *u, double *adm,
                             int64_t nvol, int64_t p) {
  V(adm, Z4C_ADM_ALPHA)[p] = V(u, Z4C_ALPHA)[p];
  for (int a = 0; a < 3; ++a) V(adm, Z4C_ADM_BETAX + a)[p] = V(u, Z4C_BETAX + a)[p];
  double psi4;
  if (opt->chi_psi_power == -4.) psi4 = 1.0 / V(u, Z4C_CHI)[p];
  else psi4 = pow(V(u, Z4C_CHI)[p], 4. / opt->chi_psi_power);
  V(adm, Z4C_ADM_PSI4)[p] = psi4;
  for (int c = 0; c < 6; ++c)
    V(adm, Z4C_ADM_GXX + c)[p] = psi4 * V(u, Z4C_GXX + c)[p];
  for (int c = 0; c < 6; ++c)
    V(adm, Z4C_ADM_KXX + c)[p] =
        psi4 * V(u, Z4C_AXX + c)[p] +
        (1. / 3.) * (V(u, Z4C_KHAT)[p] + 2. * V(u, Z4C_THETA)[p]) * V(adm, Z4C_ADM_GXX + c)[p];
}

void orc_z4c_to_adm(const orc_block_t *b, const z4c_params_t *opt, const double *u,
                    double *adm) {
  const int64_t nvol = orc_nvol(b);
  for (int64_t p = 0; p < nvol; ++p) z4c_to_adm_point(opt, u, adm, nvol, p);
}

void orc_z4c_to_adm_ghosts(const orc_block_t *b, const z4c_params_t *opt,
                           const double *u, double *adm) {
  fd_t f;
  fd_init(b, &f);
  const int64_t nvol = orc_nvol(b);
  for (int k = 0; k < f.nn3; ++k)
    for (int j = 0; j < f.nn2; ++j)
      for (int i = 0; i < f.nn1; ++i) {
        const int interior = (k >= f.kl && k <= f.ku && j >= f.jl && j <= f.ju &&
                              i >= f.il && i <= f.iu);
        if (!interior) z4c_to_adm_point(opt, u, adm, nvol, P(k, j, i));
      }
}

/* ---- Z4c::ADMToZ4c, adm_z4c.cpp:46-192 ---------------------------------- */
void orc_adm_to_z4c(const orc_block_t *b, const z4c_params_t *opt, const double *adm,
                    double *u) {
  fd_t f;
  fd_init(b, &f);
  const int64_t nvol = orc_nvol(b);
  for (int64_t p = 0; p < nvol; ++p) {
    V(u, Z4C_ALPHA)[p] = V(adm, Z4C_ADM_ALPHA)[p];
    for (int a = 0; a < 3; ++a) V(u, Z4C_BETAX + a)[p] = V(adm, Z4C_ADM_BETAX + a)[p];
    const double *G[6], *Kd[6];
    for (int c = 0; c < 6; ++c) {
      G[c] = V(adm, Z4C_ADM_GXX + c) + p;
      Kd[c] = V(adm, Z4C_ADM_KXX + c) + p;
    }
    double detg = det3(*G[0], *G[1], *G[2], *G[3], *G[4], *G[5]);
    double oopsi4;
    if (opt->chi_psi_power == -4.) {
      oopsi4 = cbrt(1.0 / detg);
      V(u, Z4C_CHI)[p] = oopsi4;
    } else {
      oopsi4 = pow(detg, -1. / 3.);
      V(u, Z4C_CHI)[p] = pow(detg, 1. / 12. * opt->chi_psi_power);
    }
    double Kt[6];
    for (int c = 0; c < 6; ++c) {
      V(u, Z4C_GXX + c)[p] = oopsi4 * *G[c];
      Kt[c] = oopsi4 * *Kd[c];
    }
    double g[6];
    for (int c = 0; c < 6; ++c) g[c] = V(u, Z4C_GXX + c)[p];
    detg = det3(g[0], g[1], g[2], g[3], g[4], g[5]);
    const double Khat = trace_rank2(1.0 / detg, g[0], g[1], g[2], g[3], g[4], g[5],
                                    Kt[0], Kt[1], Kt[2], Kt[3], Kt[4], Kt[5]);
    V(u, Z4C_KHAT)[p] = Khat;
    for (int c = 0; c < 6; ++c) V(u, Z4C_AXX + c)[p] = Kt[c] - (1. / 3.) * Khat * g[c];
  }
  /* inverse conformal metric on all points, :146-163 */
  double *guu = (double *)malloc(sizeof(double) * 6 * (size_t)nvol);
  for (int64_t p = 0; p < nvol; ++p) {
    double g[6], gu[3][3];
    for (int c = 0; c < 6; ++c) g[c] = V(u, Z4C_GXX + c)[p];
    const double detg = det3(g[0], g[1], g[2], g[3], g[4], g[5]);
    inv3(1.0 / detg, g[0], g[1], g[2], g[3], g[4], g[5], gu);
    for (int a = 0; a < 3; ++a)
      for (int c = a; c < 3; ++c) guu[SI[a][c] * nvol + p] = gu[a][c];
  }
  /* Gammas, interior only, :166-176 */
  for (int a = 0; a < 3; ++a) memset(V(u, Z4C_GAMX + a), 0, sizeof(double) * (size_t)nvol);
  for (int k = f.kl; k <= f.ku; ++k)
    for (int j = f.jl; j <= f.ju; ++j)
      for (int a = 0; a < 3; ++a)
        for (int bb = 0; bb < 3; ++bb)
          for (int i = f.il; i <= f.iu; ++i) {
            const int64_t p = P(k, j, i);
            V(u, Z4C_GAMX + a)[p] -= Dx(&f, bb, guu + SI[bb][a] * nvol + p);
          }
  free(guu);
  memset(V(u, Z4C_THETA), 0, sizeof(double) * (size_t)nvol);
  orc_algconstr(b, opt, u);
}

/* ---- Z4c::ADMConstraints, adm_z4c.cpp:382-930 --------------------------- */
void orc_adm_constraints(const orc_block_t *b, const z4c_params_t *opt,
                         const double *adm, const double *u, const orc_derivs_t *D,
                         double *con) {
  fd_t f;
  fd_init(b, &f);
  const int64_t nvol = orc_nvol(b);
  memset(con, 0, sizeof(double) * Z4C_NCON * (size_t)nvol);
  const double pw = opt->chi_psi_power;
  const double rho = 0.0, S_d[3] = {0, 0, 0};
  const double r2_max = opt->r_max_con * opt->r_max_con;

  for (int k = f.kl; k <= f.ku; ++k)
    for (int j = f.jl; j <= f.ju; ++j)
      for (int i = f.il; i <= f.iu; ++i) {
        const int64_t p = P(k, j, i);
        double ddchi_dd[3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            ddchi_dd[a][bb] = ddchi_dd[bb][a] = D->ddchi[SI[a][bb]][p];
        const double chi = V(u, Z4C_CHI)[p];
        const double chi_g = dmax(chi, opt->chi_div_floor);
        const double oochi = 1.0 / chi_g;
        double psi4c = 0.0;
        if (pw != -4.) psi4c = pow(chi_g, 4.0 / pw);

        double gt[3][3], Kd[3][3], gph[3][3];
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) {
            gt[a][c] = V(u, Z4C_GXX + SI[a][c])[p];
            Kd[a][c] = V(adm, Z4C_ADM_KXX + SI[a][c])[p];
            gph[a][c] = V(adm, Z4C_ADM_GXX + SI[a][c])[p];
          }
        double dg_ddd[3][3][3], dK_ddd[3][3][3], ddg_dddd[3][3][3][3];
        /* pass 1, :446-460 / :532-546 */
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb) {
              const double dg3 = D->dg[c][SI[a][bb]][p];
              double v;
              if (pw == -4.)
                v = oochi * (dg3 - oochi * gt[a][bb] * D->dchi[c][p]);
              else
                v = psi4c * (dg3 + (4.0 / pw) * oochi * gt[a][bb] * D->dchi[c][p]);
              dg_ddd[c][a][bb] = dg_ddd[c][bb][a] = v;
              dK_ddd[c][a][bb] = dK_ddd[c][bb][a] =
                  Dx(&f, c, V(adm, Z4C_ADM_KXX + SI[a][bb]) + p);
            }
        /* pass 2, :463-520 / :549-596 */
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            for (int c = 0; c < 3; ++c)
              for (int dd = c; dd < 3; ++dd) {
                const double dchi_a = D->dchi[a][p], dchi_b = D->dchi[bb][p];
                const double gtil = gt[c][dd];
                double v;
                if (a == bb) {
                  const double ddg_conf = Dxx(&f, a, V(u, Z4C_GXX + SI[c][dd]) + p);
                  const double dg3 = D->dg[a][SI[c][dd]][p];
                  if (pw == -4.)
                    v = oochi * (ddg_conf - oochi * (2.0 * dchi_a * dg3 + ddchi_dd[a][a] * gtil) +
                                 2.0 * oochi * oochi * dchi_a * dchi_a * gtil);
                  else {
                    const double fac = 4.0 / pw, fac2 = fac - 1.0;
                    v = psi4c * (ddg_conf + fac * oochi * (2.0 * dchi_a * dg3 + ddchi_dd[a][a] * gtil) +
                                 fac * fac2 * oochi * oochi * dchi_a * dchi_a * gtil);
                  }
                } else {
                  const double ddg_conf = Dx(&f, a, D->dg[bb][SI[c][dd]] + p);
                  const double dgb = D->dg[bb][SI[c][dd]][p], dga = D->dg[a][SI[c][dd]][p];
                  if (pw == -4.)
                    v = oochi * (ddg_conf -
                                 oochi * (dchi_a * dgb + dchi_b * dga + ddchi_dd[a][bb] * gtil) +
                                 2.0 * oochi * oochi * dchi_a * dchi_b * gtil);
                  else {
                    const double fac = 4.0 / pw, fac2 = fac - 1.0;
                    v = psi4c * (ddg_conf +
                                 fac * oochi * (dchi_a * dgb + dchi_b * dga + ddchi_dd[a][bb] * gtil) +
                                 fac * fac2 * oochi * oochi * dchi_a * dchi_b * gtil);
                  }
                }
                ddg_dddd[a][bb][c][dd] = ddg_dddd[bb][a][c][dd] =
                    ddg_dddd[a][bb][dd][c] = ddg_dddd[bb][a][dd][c] = v;
              }
        /* inverse physical metric, :601-618 */
        double g_uu[3][3];
        {
          const double detg = det3(gph[0][0], gph[0][1], gph[0][2], gph[1][1], gph[1][2], gph[2][2]);
          inv3(1. / detg, gph[0][0], gph[0][1], gph[0][2], gph[1][1], gph[1][2], gph[2][2], g_uu);
        }
        double Gamma_ddd[3][3][3], Gamma_udd[3][3][3];
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb)
              Gamma_ddd[c][a][bb] = Gamma_ddd[c][bb][a] =
                  0.5 * (dg_ddd[a][bb][c] + dg_ddd[bb][a][c] - dg_ddd[c][a][bb]);
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb) {
              double s = 0;
              for (int dd = 0; dd < 3; ++dd) s += g_uu[c][dd] * Gamma_ddd[dd][a][bb];
              Gamma_udd[c][a][bb] = Gamma_udd[c][bb][a] = s;
            }
        /* Ricci tensor and scalar, :655-689 */
        double R = 0, R_dd[3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            double s = 0;
            for (int c = 0; c < 3; ++c)
              for (int dd = 0; dd < 3; ++dd)
                for (int ff = 0; ff < 3; ++ff)
                  s += g_uu[dd][ff] * (Gamma_udd[c][a][ff] * Gamma_ddd[c][bb][dd] -
                                       Gamma_udd[c][a][bb] * Gamma_ddd[c][ff][dd]);
            for (int c = 0; c < 3; ++c)
              for (int dd = 0; dd < 3; ++dd)
                s += 0.5 * g_uu[c][dd] *
                     (-ddg_dddd[bb][a][c][dd] + ddg_dddd[dd][a][bb][c] +
                      ddg_dddd[dd][bb][a][c] - ddg_dddd[dd][c][a][bb]);
            R_dd[a][bb] = R_dd[bb][a] = s;
            R += ((a == bb) ? 1.0 : 2.0) * g_uu[a][bb] * R_dd[a][bb];
          }
        /* extrinsic curvature, :694-753 */
        double K = 0, K_ud[3][3] = {{0}}, KK = 0;
        for (int a = 0; a < 3; ++a) {
          for (int bb = 0; bb < 3; ++bb)
            for (int c = 0; c < 3; ++c) K_ud[a][bb] += g_uu[a][c] * Kd[c][bb];
          K += K_ud[a][a];
        }
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) KK += K_ud[a][bb] * K_ud[bb][a];
        double DK_ddd[3][3][3], DK_udd[3][3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb)
            for (int c = bb; c < 3; ++c) {
              double v = dK_ddd[a][bb][c];
              for (int dd = 0; dd < 3; ++dd) {
                v -= Gamma_udd[dd][a][bb] * Kd[dd][c];
                v -= Gamma_udd[dd][a][c] * Kd[bb][dd];
              }
              DK_ddd[a][bb][c] = DK_ddd[a][c][bb] = v;
            }
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb)
            for (int c = bb; c < 3; ++c) {
              double s = 0;
              for (int dd = 0; dd < 3; ++dd) s += g_uu[a][dd] * DK_ddd[dd][bb][c];
              DK_udd[a][bb][c] = DK_udd[a][c][bb] = s;
            }
        /* constraints, :760-814 */
        const double H = R + (K * K) - KK - 16 * M_PI * rho;
        double M_u[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) {
            M_u[a] -= 8 * M_PI * g_uu[a][bb] * S_d[bb];
            for (int c = 0; c < 3; ++c) {
              M_u[a] += g_uu[a][bb] * DK_udd[c][bb][c];
              M_u[a] -= g_uu[bb][c] * DK_udd[a][bb][c];
            }
          }
        double M_d[3];
        for (int a = 0; a < 3; ++a) {
          M_d[a] = 0;
          for (int bb = 0; bb < 3; ++bb) M_d[a] += gph[a][bb] * M_u[bb];
        }
        double M = 0.;
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            M += ((a == bb) ? 1.0 : 2.0) * gph[a][bb] * M_u[a] * M_u[bb];
        /* conformal connection functions for Z, :819-906 */
        double gc_uu[3][3];
        {
          const double detg = det3(gt[0][0], gt[0][1], gt[0][2], gt[1][1], gt[1][2], gt[2][2]);
          inv3(1. / detg, gt[0][0], gt[0][1], gt[0][2], gt[1][1], gt[1][2], gt[2][2], gc_uu);
        }
        double cG_ddd[3][3][3], cG_udd[3][3][3], cG_u[3];
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb) {
              const double d1 = D->dg[a][SI[bb][c]][p], d2 = D->dg[bb][SI[a][c]][p],
                           d3 = D->dg[c][SI[a][bb]][p];
              cG_ddd[c][a][bb] = cG_ddd[c][bb][a] = 0.5 * (d1 + d2 - d3);
            }
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb) {
              double s = 0;
              for (int dd = 0; dd < 3; ++dd) s += gc_uu[c][dd] * cG_ddd[dd][a][bb];
              cG_udd[c][a][bb] = cG_udd[c][bb][a] = s;
            }
        for (int a = 0; a < 3; ++a) {
          double s = 0;
          for (int bb = 0; bb < 3; ++bb)
            for (int c = bb; c < 3; ++c)
              s += ((bb == c) ? 1.0 : 2.0) * gc_uu[bb][c] * cG_udd[a][bb][c];
          cG_u[a] = s;
        }
        double Z = 0.;
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb)
            Z += ((a == bb) ? 0.25 : 0.5) * gph[a][bb] *
                 (V(u, Z4C_GAMX + a)[p] - cG_u[a]) * (V(u, Z4C_GAMX + bb)[p] - cG_u[bb]);
        /* radius cut + C, :908-928 */
        const double x1 = b->x[0][i], x2 = b->x[1][j], x3 = b->x[2][k];
        const double R2 = x1 * x1 + x2 * x2 + x3 * x3;
        if (R2 > r2_max) {
          /* all zero already */
        } else {
          const double Theta = V(u, Z4C_THETA)[p];
          V(con, Z4C_CON_H)[p] = H;
          V(con, Z4C_CON_M)[p] = M;
          V(con, Z4C_CON_Z)[p] = Z;
          for (int a = 0; a < 3; ++a) V(con, Z4C_CON_MX + a)[p] = M_d[a];
          V(con, Z4C_CON_C)[p] = (H * H) + M + (Theta * Theta) + 4.0 * Z;
        }
      }
}

/* ---- uniform-mesh ghost exchange and physical BCs ------------------------ */

/* Neighbour directions in the order MeshBlock::SearchAndSetNeighbors lists
 * them (mesh/mesh_topology.cpp:329-960): x1, x2, x3 faces, then x1x2, x1x3,
 * x2x3 edges, then corners, each with the first offset varying fastest.  The
 * additive unpack (comm_channel.cpp:990+, comm_registry.cpp:1006+) adds the
 * neighbours' contributions in this order. */
static int neighbour_dirs(int dirs[26][3]) {
  int n = 0;
  for (int s = -1; s <= 1; s += 2) { dirs[n][0] = s; dirs[n][1] = 0; dirs[n][2] = 0; ++n; }
  for (int s = -1; s <= 1; s += 2) { dirs[n][0] = 0; dirs[n][1] = s; dirs[n][2] = 0; ++n; }
  for (int s = -1; s <= 1; s += 2) { dirs[n][0] = 0; dirs[n][1] = 0; dirs[n][2] = s; ++n; }
  for (int m = -1; m <= 1; m += 2)
    for (int s = -1; s <= 1; s += 2) { dirs[n][0] = s; dirs[n][1] = m; dirs[n][2] = 0; ++n; }
  for (int m = -1; m <= 1; m += 2)
    for (int s = -1; s <= 1; s += 2) { dirs[n][0] = s; dirs[n][1] = 0; dirs[n][2] = m; ++n; }
  for (int m = -1; m <= 1; m += 2)
    for (int s = -1; s <= 1; s += 2) { dirs[n][0] = 0; dirs[n][1] = s; dirs[n][2] = m; ++n; }
  for (int l = -1; l <= 1; l += 2)
    for (int m = -1; m <= 1; m += 2)
      for (int s = -1; s <= 1; s += 2) { dirs[n][0] = s; dirs[n][1] = m; dirs[n][2] = l; ++n; }
  return n;
}

void orc_mesh_exchange(const orc_mesh_t *m, int nvar, double *u_all) {
  const int nn[3] = {m->nx[0] + 1 + 2 * NG, m->nx[1] + 1 + 2 * NG, m->nx[2] + 1 + 2 * NG};
  const int64_t nvol = (int64_t)nn[0] * nn[1] * nn[2];
  const int nblocks = m->nb[0] * m->nb[1] * m->nb[2];
  const int64_t bstride = nvol * nvar;
  int dirs[26][3];
  neighbour_dirs(dirs);
  /* every block unpacks from the pre-exchange state of its neighbours */
  double *out = (double *)malloc(sizeof(double) * (size_t)bstride * nblocks);
  memcpy(out, u_all, sizeof(double) * (size_t)bstride * nblocks);
  for (int bl = 0; bl < nblocks; ++bl) {
    const int loc[3] = {bl % m->nb[0], (bl / m->nb[0]) % m->nb[1], bl / (m->nb[0] * m->nb[1])};
    /* neighbour block of each direction, -1 beyond a non-periodic face */
    int nbr[26];
    for (int d = 0; d < 26; ++d) {
      int l[3], ok = 1;
      for (int a = 0; a < 3; ++a) {
        l[a] = loc[a] + dirs[d][a];
        if (l[a] < 0 || l[a] >= m->nb[a]) {
          if (m->bc[2 * a] == Z4C_BC_PERIODIC) l[a] = (l[a] + m->nb[a]) % m->nb[a];
          else ok = 0;
        }
      }
      nbr[d] = ok ? l[0] + m->nb[0] * (l[1] + m->nb[1] * l[2]) : -1;
    }
    for (int k = 0; k < nn[2]; ++k)
      for (int j = 0; j < nn[1]; ++j)
        for (int i = 0; i < nn[0]; ++i) {
          const int idx[3] = {i, j, k};
          int interior = 1, on_edge = 0;
          for (int a = 0; a < 3; ++a) {
            const int vs = NG, ve = NG + m->nx[a];
            if (idx[a] < vs || idx[a] > ve) interior = 0;
            if (idx[a] <= vs || idx[a] >= ve) on_edge = 1;
          }
          if (!on_edge) continue; /* strictly interior: untouched */
          /* SetRangeVC (index_utilities.hpp:155-163) coverage per direction */
          int cov[26], mult = interior ? 1 : 0;
          for (int d = 0; d < 26; ++d) {
            cov[d] = (nbr[d] >= 0);
            for (int a = 0; a < 3 && cov[d]; ++a) {
              const int vs = NG, ve = NG + m->nx[a], o = dirs[d][a];
              if (o > 0) cov[d] = (idx[a] >= ve);
              else if (o < 0) cov[d] = (idx[a] <= vs);
              else cov[d] = (idx[a] >= vs && idx[a] <= ve);
            }
            mult += cov[d];
          }
          const int64_t p = ((int64_t)k * nn[1] + j) * nn[0] + i;
          for (int n = 0; n < nvar; ++n) {
            double s = interior ? u_all[bl * bstride + n * nvol + p] : 0.0;
            for (int d = 0; d < 26; ++d) {
              if (!cov[d]) continue;
              const int64_t q = ((int64_t)(k - dirs[d][2] * m->nx[2]) * nn[1] +
                                 (j - dirs[d][1] * m->nx[1])) * nn[0] +
                                (i - dirs[d][0] * m->nx[0]);
              s += u_all[(int64_t)nbr[d] * bstride + n * nvol + q];
            }
            if (mult > 1) s *= 1.0 / (double)mult;
            out[bl * bstride + n * nvol + p] = s;
          }
        }
  }
  memcpy(u_all, out, sizeof(double) * (size_t)bstride * nblocks);
  free(out);
  for (int bl = 0; bl < nblocks; ++bl) {
    const int loc[3] = {bl % m->nb[0], (bl / m->nb[0]) % m->nb[1], bl / (m->nb[0] * m->nb[1])};
    orc_block_physical_bcs(m, loc, nvar, u_all + bl * bstride);
  }
}

/* ExtrapolateOutflowBC with NEXTRAPOLATE=5 (physical_bcs.cpp:187-260); the
 * index ranges follow ApplyPhysicalBCs (:506-670), which uses the
 * cell-centred interior end ie = is + nx - 1 also for vertex data. */
static const double CE[5] = {5., -10., 10., -5., 1.};

void orc_block_physical_bcs(const orc_mesh_t *m, const int loc[3], int nvar, double *u) {
  const int nn[3] = {m->nx[0] + 1 + 2 * NG, m->nx[1] + 1 + 2 * NG, m->nx[2] + 1 + 2 * NG};
  const int64_t nvol = (int64_t)nn[0] * nn[1] * nn[2];
  const int64_t st[3] = {1, nn[0], (int64_t)nn[0] * nn[1]};
  int need[6];
  for (int a = 0; a < 3; ++a) {
    need[2 * a] = (m->bc[2 * a] != Z4C_BC_PERIODIC) && loc[a] == 0;
    need[2 * a + 1] = (m->bc[2 * a + 1] != Z4C_BC_PERIODIC) && loc[a] == m->nb[a] - 1;
  }
  int is[3], ie[3];
  for (int a = 0; a < 3; ++a) { is[a] = NG; ie[a] = NG + m->nx[a] - 1; }
  /* transverse limits, :516-528 */
  int bis = is[0] - NG, bie = ie[0] + NG;
  int bjs = is[1], bje = ie[1], bks = is[2], bke = ie[2];
  if (!need[2]) bjs = is[1] - NG;
  if (!need[3]) bje = ie[1] + NG;
  if (!need[4]) bks = is[2] - NG;
  if (!need[5]) bke = ie[2] + NG;
  for (int face = 0; face < 6; ++face) {
    if (!need[face]) continue;
    const int ax = face / 2, outer = face % 2;
    int lo[3], hi[3];
    if (ax == 0) { lo[1] = bjs; hi[1] = bje; lo[2] = bks; hi[2] = bke; }
    else if (ax == 1) { lo[0] = bis; hi[0] = bie; lo[2] = bks; hi[2] = bke; }
    else { lo[0] = bis; hi[0] = bie; lo[1] = is[1] - NG; hi[1] = ie[1] + NG; }
    /* the x3 faces use the extended j range, :619-621 */
    const int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
    for (int n = 0; n < nvar; ++n)
      for (int t2 = lo[o2]; t2 <= hi[o2]; ++t2)
        for (int t1 = lo[o1]; t1 <= hi[o1]; ++t1)
          for (int g = 1; g <= NG; ++g) {
            const int ia = outer ? ie[ax] + g : is[ax] - g;
            const int dir = outer ? -1 : 1;
            int64_t p = (int64_t)ia * st[ax] + (int64_t)t1 * st[o1] + (int64_t)t2 * st[o2];
            double v = 0.0;
            for (int q = 0; q < 5; ++q) v += CE[q] * u[n * nvol + p + dir * (q + 1) * st[ax]];
            u[n * nvol + p] = v;
          }
  }
}

/* ---- vertex-centred refinement operators, mesh/mesh_refinement_vc.cpp ---- */

/* InterpolateLagrangeUniform<3>::coeff, utils/interp_univariate_stencils.tpp:99-101 */
static const double LAG3[3] = {3. / 256., -25. / 256., 75. / 128.};

void orc_vc_restrict(const int nx[3], int nvar, const double *fine, double *coarse,
                     const int box[6]) {
  const int nn[3] = {nx[0] + 1 + 2 * NG, nx[1] + 1 + 2 * NG, nx[2] + 1 + 2 * NG};
  const int cn[3] = {nx[0] / 2 + 1 + 2 * ORC_NCG, nx[1] / 2 + 1 + 2 * ORC_NCG,
                     nx[2] / 2 + 1 + 2 * ORC_NCG};
  const int64_t fvol = (int64_t)nn[0] * nn[1] * nn[2], cvol = (int64_t)cn[0] * cn[1] * cn[2];
  /* RestrictVertexCenteredIndicialHelper (:24-46): every branch maps a
   * coarse index c to the fine index 2 (c - cvs) + vs */
  for (int n = 0; n < nvar; ++n)
    for (int ck = box[4]; ck <= box[5]; ++ck) {
      const int k = 2 * (ck - ORC_NCG) + NG;
      for (int cj = box[2]; cj <= box[3]; ++cj) {
        const int j = 2 * (cj - ORC_NCG) + NG;
        for (int ci = box[0]; ci <= box[1]; ++ci) {
          const int i = 2 * (ci - ORC_NCG) + NG;
          coarse[n * cvol + ((int64_t)ck * cn[1] + cj) * cn[0] + ci] =
              fine[n * fvol + ((int64_t)k * nn[1] + j) * nn[0] + i];
        }
      }
    }
}

void orc_vc_prolongate(const int nx[3], int nvar, const double *coarse, double *fine,
                       const int box[6]) {
  const int H = 3, HNC = (2 * ORC_NCG - NG) / 2; /* H_SZ, H_NCGHOST */
  const int nn[3] = {nx[0] + 1 + 2 * NG, nx[1] + 1 + 2 * NG, nx[2] + 1 + 2 * NG};
  const int cn[3] = {nx[0] / 2 + 1 + 2 * ORC_NCG, nx[1] / 2 + 1 + 2 * ORC_NCG,
                     nx[2] / 2 + 1 + 2 * ORC_NCG};
  const int cmp[3] = {ORC_NCG + nx[0] / 4, ORC_NCG + nx[1] / 4, ORC_NCG + nx[2] / 4};
  const int64_t fvol = (int64_t)nn[0] * nn[1] * nn[2], cvol = (int64_t)cn[0] * cn[1] * cn[2];
  const int si = box[0], ei = box[1], sj = box[2], ej = box[3], sk = box[4], ek = box[5];
  /* bias offsets, :351-356 */
  const int si_p = (si > cmp[0]) ? si - 1 : si, ei_p = (ei < cmp[0]) ? ei + 1 : ei;
  const int sj_p = (sj > cmp[1]) ? sj - 1 : sj, ej_p = (ej < cmp[1]) ? ej + 1 : ej;
  const int sk_p = (sk > cmp[2]) ? sk - 1 : sk, ek_p = (ek < cmp[2]) ? ek + 1 : ek;
#define CO(k, j, i) c[((int64_t)(k) * cn[1] + (j)) * cn[0] + (i)]
#define FI(k, j, i) f[((int64_t)(k) * nn[1] + (j)) * nn[0] + (i)]
  for (int n = 0; n < nvar; ++n) {
    const double *c = coarse + n * cvol;
    double *f = fine + n * fvol;
    /* (prl, prl, prl) */
    for (int k = sk_p; k < ek_p; ++k)
      for (int j = sj_p; j < ej_p; ++j)
        for (int i = si_p; i < ei_p; ++i) {
          double *o = &FI(2 * (k - HNC) + 1, 2 * (j - HNC) + 1, 2 * (i - HNC) + 1);
          *o = 0.;
          for (int dk = 0; dk < H; ++dk) {
            const int ku = k + dk + 1, kl = k - dk;
            const double lck = LAG3[H - dk - 1];
            for (int dj = 0; dj < H; ++dj) {
              const int ju = j + dj + 1, jl = j - dj;
              const double lckj = lck * LAG3[H - dj - 1];
              for (int di = 0; di < H; ++di) {
                const int iu = i + di + 1, il = i - di;
                const double lckji = lckj * LAG3[H - di - 1];
                /* FloatingPoint::sum_corners (utils/floating_point.hpp:50-55) */
                *o += lckji * (((CO(ku, ju, iu) + CO(kl, jl, il)) +
                                (CO(ku, ju, il) + CO(kl, jl, iu))) +
                               ((CO(kl, ju, il) + CO(ku, jl, iu)) +
                                (CO(kl, ju, iu) + CO(ku, jl, il))));
              }
            }
          }
        }
    /* (inj, prl, prl) */
    for (int k = sk; k <= ek; ++k)
      for (int j = sj_p; j < ej_p; ++j)
        for (int i = si_p; i < ei_p; ++i) {
          double *o = &FI(2 * (k - HNC), 2 * (j - HNC) + 1, 2 * (i - HNC) + 1);
          *o = 0.;
          for (int dj = 0; dj < H; ++dj) {
            const int ju = j + dj + 1, jl = j - dj;
            const double lcj = LAG3[H - dj - 1];
            for (int di = 0; di < H; ++di) {
              const int iu = i + di + 1, il = i - di;
              const double lcji = lcj * LAG3[H - di - 1];
              *o += lcji * ((CO(k, ju, iu) + CO(k, jl, il)) + (CO(k, jl, iu) + CO(k, ju, il)));
            }
          }
        }
    /* (prl, inj, prl) */
    for (int k = sk_p; k < ek_p; ++k)
      for (int j = sj; j <= ej; ++j)
        for (int i = si_p; i < ei_p; ++i) {
          double *o = &FI(2 * (k - HNC) + 1, 2 * (j - HNC), 2 * (i - HNC) + 1);
          *o = 0.;
          for (int dk = 0; dk < H; ++dk) {
            const int ku = k + dk + 1, kl = k - dk;
            const double lck = LAG3[H - dk - 1];
            for (int di = 0; di < H; ++di) {
              const int iu = i + di + 1, il = i - di;
              const double lcki = lck * LAG3[H - di - 1];
              *o += lcki * ((CO(kl, j, iu) + CO(ku, j, il)) + (CO(ku, j, iu) + CO(kl, j, il)));
            }
          }
        }
    /* (prl, prl, inj) */
    for (int k = sk_p; k < ek_p; ++k)
      for (int j = sj_p; j < ej_p; ++j)
        for (int i = si; i <= ei; ++i) {
          double *o = &FI(2 * (k - HNC) + 1, 2 * (j - HNC) + 1, 2 * (i - HNC));
          *o = 0.;
          for (int dk = 0; dk < H; ++dk) {
            const int ku = k + dk + 1, kl = k - dk;
            const double lck = LAG3[H - dk - 1];
            for (int dj = 0; dj < H; ++dj) {
              const int ju = j + dj + 1, jl = j - dj;
              const double lckj = lck * LAG3[H - dj - 1];
              *o += lckj * ((CO(ku, ju, i) + CO(kl, jl, i)) + (CO(kl, ju, i) + CO(ku, jl, i)));
            }
          }
        }
    /* (inj, inj, prl) */
    for (int k = sk; k <= ek; ++k)
      for (int j = sj; j <= ej; ++j)
        for (int i = si_p; i < ei_p; ++i) {
          double *o = &FI(2 * (k - HNC), 2 * (j - HNC), 2 * (i - HNC) + 1);
          *o = 0.;
          for (int di = 0; di < H; ++di)
            *o += LAG3[H - di - 1] * (CO(k, j, i - di) + CO(k, j, i + di + 1));
        }
    /* (inj, prl, inj) */
    for (int k = sk; k <= ek; ++k)
      for (int j = sj_p; j < ej_p; ++j)
        for (int i = si; i <= ei; ++i) {
          double *o = &FI(2 * (k - HNC), 2 * (j - HNC) + 1, 2 * (i - HNC));
          *o = 0.;
          for (int dj = 0; dj < H; ++dj)
            *o += LAG3[H - dj - 1] * (CO(k, j - dj, i) + CO(k, j + dj + 1, i));
        }
    /* (prl, inj, inj) */
    for (int k = sk_p; k < ek_p; ++k)
      for (int j = sj; j <= ej; ++j)
        for (int i = si; i <= ei; ++i) {
          double *o = &FI(2 * (k - HNC) + 1, 2 * (j - HNC), 2 * (i - HNC));
          *o = 0.;
          for (int dk = 0; dk < H; ++dk)
            *o += LAG3[H - dk - 1] * (CO(k - dk, j, i) + CO(k + dk + 1, j, i));
        }
    /* (inj, inj, inj) */
    for (int k = sk; k <= ek; ++k)
      for (int j = sj; j <= ej; ++j)
        for (int i = si; i <= ei; ++i)
          FI(2 * (k - HNC), 2 * (j - HNC), 2 * (i - HNC)) = CO(k, j, i);
  }
#undef CO
#undef FI
}

/* ---- Z4c::Z4cWeyl, z4c/calculate_weyl_scalars.cpp:44-630 ----------------- */
void orc_weyl(const orc_block_t *b, const z4c_params_t *opt, const double *adm, const double *u,
              const orc_derivs_t *d, double *weyl) {
  fd_t f;
  fd_init(b, &f);
  const int64_t nvol = orc_nvol(b);
  for (int64_t q = 0; q < 2 * nvol; ++q) weyl[q] = NAN;
  const double FR4 = 0.25;
  const double pw = opt->chi_psi_power;
#define G3(a, b) V(adm, Z4C_ADM_GXX + SI[a][b])[p]
#define K3(a, b) V(adm, Z4C_ADM_KXX + SI[a][b])[p]
#define GT(a, b) V(u, Z4C_GXX + SI[a][b])[p]
  for (int k = f.kl; k <= f.ku; ++k)
    for (int j = f.jl; j <= f.ju; ++j)
      for (int i = f.il; i <= f.iu; ++i) {
        const int64_t p = P(k, j, i);
        double ddchi[3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) ddchi[a][bb] = d->ddchi[SI[a][bb]][p];
        const double chi_g = dmax(V(u, Z4C_CHI)[p], opt->chi_div_floor);
        /* pass 1: physical first derivatives and dK, :150-166 / :224-239 */
        double dg[3][3][3], dK[3][3][3];
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb) {
              double v;
              if (pw == -4.) {
                const double oochi = 1.0 / chi_g;
                v = oochi * (d->dg[c][SI[a][bb]][p] - oochi * GT(a, bb) * d->dchi[c][p]);
              } else {
                const double fac = 4.0 / pw;
                const double psi4 = pow(chi_g, fac);
                const double oochi = 1.0 / chi_g;
                v = psi4 * (d->dg[c][SI[a][bb]][p] + fac * oochi * GT(a, bb) * d->dchi[c][p]);
              }
              dg[c][a][bb] = dg[c][bb][a] = v;
              const double dk = Dx(&f, c, V(adm, Z4C_ADM_KXX + SI[a][bb]) + p);
              dK[c][a][bb] = dK[c][bb][a] = dk;
            }
        /* pass 2: physical second derivatives, :169-206 / :242-288 */
        double ddg[3][3][3][3];
        for (int c = 0; c < 3; ++c)
          for (int dd = c; dd < 3; ++dd)
            for (int a = 0; a < 3; ++a)
              for (int bb = a; bb < 3; ++bb) {
                const double dchi_a = d->dchi[a][p], dchi_b = d->dchi[bb][p];
                const double gtil = GT(c, dd);
                double v;
                if (a == bb) {
                  const double ddg_conf = Dxx(&f, a, V(u, Z4C_GXX + SI[c][dd]) + p);
                  const double d3 = d->dg[a][SI[c][dd]][p];
                  if (pw == -4.) {
                    const double oochi = 1.0 / chi_g;
                    v = oochi * (ddg_conf - oochi * (2.0 * dchi_a * d3 + ddchi[a][a] * gtil) +
                                 2.0 * oochi * oochi * dchi_a * dchi_a * gtil);
                  } else {
                    const double fac = 4.0 / pw, fac2 = fac - 1.0;
                    const double psi4 = pow(chi_g, fac);
                    const double oochi = 1.0 / chi_g;
                    v = psi4 * (ddg_conf + fac * oochi * (2.0 * dchi_a * d3 + ddchi[a][a] * gtil) +
                                fac * fac2 * oochi * oochi * dchi_a * dchi_a * gtil);
                  }
                } else {
                  const double ddg_conf = Dx(&f, a, d->dg[bb][SI[c][dd]] + p);
                  const double db3 = d->dg[bb][SI[c][dd]][p], da3 = d->dg[a][SI[c][dd]][p];
                  if (pw == -4.) {
                    const double oochi = 1.0 / chi_g;
                    v = oochi * (ddg_conf - oochi * (dchi_a * db3 + dchi_b * da3 +
                                                     ddchi[a][bb] * gtil) +
                                 2.0 * oochi * oochi * dchi_a * dchi_b * gtil);
                  } else {
                    const double fac = 4.0 / pw, fac2 = fac - 1.0;
                    const double psi4 = pow(chi_g, fac);
                    const double oochi = 1.0 / chi_g;
                    v = psi4 * (ddg_conf + fac * oochi * (dchi_a * db3 + dchi_b * da3 +
                                                          ddchi[a][bb] * gtil) +
                                fac * fac2 * oochi * oochi * dchi_a * dchi_b * gtil);
                  }
                }
                ddg[a][bb][c][dd] = ddg[bb][a][c][dd] = ddg[a][bb][dd][c] = ddg[bb][a][dd][c] = v;
              }
        /* inverse metric, :293-309 */
        double gu[3][3];
        {
          const double detg = det3(G3(0, 0), G3(0, 1), G3(0, 2), G3(1, 1), G3(1, 2), G3(2, 2));
          inv3(1. / detg, G3(0, 0), G3(0, 1), G3(0, 2), G3(1, 1), G3(1, 2), G3(2, 2), gu);
        }
        /* Christoffels, :314-337 */
        double Gd[3][3][3], Gu[3][3][3];
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb)
              Gd[c][a][bb] = Gd[c][bb][a] =
                  0.5 * (dg[a][bb][c] + dg[bb][a][c] - dg[c][a][bb]);
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int bb = a; bb < 3; ++bb) {
              double acc = 0.0;
              for (int dd = 0; dd < 3; ++dd) acc += gu[c][dd] * Gd[dd][a][bb];
              Gu[c][a][bb] = Gu[c][bb][a] = acc;
            }
        /* Ricci tensor and scalar, :342-378 */
        double R = 0.0, Rd[3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = a; bb < 3; ++bb) {
            double acc = 0.0;
            for (int c = 0; c < 3; ++c)
              for (int dd = 0; dd < 3; ++dd) {
                for (int e = 0; e < 3; ++e) {
                  acc += gu[c][dd] * Gu[e][a][c] * Gd[e][bb][dd];
                  acc -= gu[c][dd] * Gu[e][a][bb] * Gd[e][c][dd];
                }
                acc += 0.5 * gu[c][dd] *
                       (-ddg[c][dd][a][bb] - ddg[a][bb][c][dd] + ddg[a][c][bb][dd] +
                        ddg[bb][c][a][dd]);
              }
            Rd[a][bb] = Rd[bb][a] = acc;
            R += ((a == bb) ? 1.0 : 2.0) * gu[a][bb] * acc;
          }
        /* extrinsic curvature, :383-420 */
        double Kt = 0.0, Kud[3][3];
        for (int a = 0; a < 3; ++a) {
          for (int bb = 0; bb < 3; ++bb) {
            double acc = 0.0;
            for (int c = 0; c < 3; ++c) acc += gu[a][c] * K3(c, bb);
            Kud[a][bb] = acc;
          }
          Kt += Kud[a][a];
        }
        /* DK_ddd is stored symmetric in its last two indices and the loop
         * runs over all (b, c): for b < c the (c, b) pass comes later and its
         * value, with the two subtractions in the other order, is kept */
        double DK[3][3][3];
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb)
            for (int c = 0; c < 3; ++c) {
              double v = dK[a][bb][c];
              for (int dd = 0; dd < 3; ++dd) {
                v -= Gu[dd][a][bb] * K3(dd, c);
                v -= Gu[dd][a][c] * K3(bb, dd);
              }
              DK[a][bb][c] = DK[a][c][bb] = v;
            }
        /* tetrad and Gram-Schmidt, :426-524 */
        const double x1 = b->x[0][i], x2 = b->x[1][j], x3 = b->x[2][k];
        double xx = x1;
        if (x1 * x1 + x2 * x2 < 1e-10) xx = xx + 1e-8;
        double uv[3] = {xx, x2, x3};
        double vv[3] = {xx * x3, x2 * x3, -(xx * xx) - (x2 * x2)};
        double wv[3] = {x2 * -1.0, xx, 0.0};
        double dot = 0.0, dot2;
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) dot += G3(a, bb) * wv[a] * wv[bb];
        for (int a = 0; a < 3; ++a) wv[a] = wv[a] / sqrt(dot);
        dot = 0.0;
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) dot += G3(a, bb) * wv[a] * uv[bb];
        for (int a = 0; a < 3; ++a) uv[a] -= dot * wv[a];
        dot = 0.0;
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) dot += G3(a, bb) * uv[a] * uv[bb];
        for (int a = 0; a < 3; ++a) uv[a] = uv[a] / sqrt(dot);
        dot = 0.0;
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) dot += G3(a, bb) * wv[a] * vv[bb];
        dot2 = 0.0;
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) dot2 += G3(a, bb) * uv[a] * vv[bb];
        for (int a = 0; a < 3; ++a) vv[a] -= dot * wv[a] + dot2 * uv[a];
        dot = 0.0;
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) dot += G3(a, bb) * vv[a] * vv[bb];
        for (int a = 0; a < 3; ++a) vv[a] = vv[a] / sqrt(dot);
        /* psi4, :532-630 */
        double rp = 0, ip = 0;
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) {
            double R4 = Rd[a][bb] + Kt * K3(a, bb);
            for (int c = 0; c < 3; ++c)
              for (int dd = 0; dd < 3; ++dd) R4 -= gu[c][dd] * K3(a, c) * K3(dd, bb);
            const double Tr = vv[a] * vv[bb] - wv[a] * wv[bb];
            const double Ti = -vv[a] * wv[bb] - wv[a] * vv[bb];
            rp += -FR4 * R4 * Tr;
            ip += -FR4 * R4 * Ti;
          }
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb)
            for (int c = 0; c < 3; ++c) {
              const double R4 = -(DK[bb][a][c] - DK[c][a][bb]);
              const double Tr = vv[a] * vv[bb] - wv[a] * wv[bb];
              const double Ti = -vv[a] * wv[bb] - wv[a] * vv[bb];
              rp += 0.5 * R4 * uv[c] * Tr;
              ip += 0.5 * R4 * uv[c] * Ti;
            }
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb)
            for (int c = 0; c < 3; ++c)
              for (int dd = 0; dd < 3; ++dd) {
                const double R4 = G3(dd, c) * Rd[a][bb] + G3(a, bb) * Rd[dd][c] -
                                  G3(dd, bb) * Rd[a][c] - G3(a, c) * Rd[dd][bb] -
                                  0.5 * R * (G3(dd, c) * G3(a, bb) - G3(dd, bb) * G3(a, c)) +
                                  K3(dd, c) * K3(a, bb) - K3(dd, bb) * K3(a, c);
                const double Tr = vv[a] * vv[bb] - wv[a] * wv[bb];
                const double Ti = -vv[a] * wv[bb] - wv[a] * vv[bb];
                rp += -FR4 * R4 * uv[dd] * uv[c] * Tr;
                ip += -FR4 * R4 * uv[dd] * uv[c] * Ti;
              }
        weyl[p] = rp;
        weyl[nvol + p] = ip;
      }
#undef G3
#undef K3
#undef GT
}

/* ---- regrid-time transfer, comm/amr_registry.cpp:814-1233 (VC) ----------- */
void orc_regrid_refine(const int nx[3], int nvar, const double *parent, double *child,
                       const int oct[3]) {
  const int NCG = Z4C_NCG, ndg = NCG < NG ? NCG : NG;
  int nn[3], cn[3], box[6];
  for (int a = 0; a < 3; ++a) {
    nn[a] = nx[a] + 1 + 2 * NG;
    cn[a] = nx[a] / 2 + 1 + 2 * NCG;
    box[2 * a] = NCG;                 /* civs */
    box[2 * a + 1] = NCG + nx[a] / 2; /* cive */
  }
  const int64_t fvol = (int64_t)nn[0] * nn[1] * nn[2], cvol = (int64_t)cn[0] * cn[1] * cn[2];
  double *coarse = (double *)calloc((size_t)(nvar * cvol), sizeof(double));
  /* coarse [civs - ndg, cive + ndg] <- parent from oct*nx/2 + ivs - ndg */
  int c0[3], s0[3];
  for (int a = 0; a < 3; ++a) {
    c0[a] = NCG - ndg;
    s0[a] = oct[a] * (nx[a] / 2) + NG - ndg;
  }
  for (int n = 0; n < nvar; ++n)
    for (int k = c0[2]; k <= NCG + nx[2] / 2 + ndg; ++k)
      for (int j = c0[1]; j <= NCG + nx[1] / 2 + ndg; ++j)
        for (int i = c0[0]; i <= NCG + nx[0] / 2 + ndg; ++i)
          coarse[n * cvol + ((int64_t)k * cn[1] + j) * cn[0] + i] =
              parent[n * fvol + ((int64_t)(s0[2] + k - c0[2]) * nn[1] + (s0[1] + j - c0[1])) * nn[0] +
                     (s0[0] + i - c0[0])];
  orc_vc_prolongate(nx, nvar, coarse, child, box);
  free(coarse);
}

void orc_regrid_derefine(const int nx[3], int nvar, const double *child, double *parent,
                         const int oct[3]) {
  const int NCG = Z4C_NCG;
  int nn[3], cn[3], box[6];
  for (int a = 0; a < 3; ++a) {
    nn[a] = nx[a] + 1 + 2 * NG;
    cn[a] = nx[a] / 2 + 1 + 2 * NCG;
    box[2 * a] = NCG;
    box[2 * a + 1] = NCG + nx[a] / 2;
  }
  const int64_t fvol = (int64_t)nn[0] * nn[1] * nn[2], cvol = (int64_t)cn[0] * cn[1] * cn[2];
  double *coarse = (double *)calloc((size_t)(nvar * cvol), sizeof(double));
  orc_vc_restrict(nx, nvar, child, coarse, box);
  for (int n = 0; n < nvar; ++n)
    for (int k = box[4]; k <= box[5]; ++k)
      for (int j = box[2]; j <= box[3]; ++j)
        for (int i = box[0]; i <= box[1]; ++i)
          parent[n * fvol +
                 ((int64_t)(NG + oct[2] * (nx[2] / 2) + k - box[4]) * nn[1] +
                  (NG + oct[1] * (nx[1] / 2) + j - box[2])) * nn[0] +
                 (NG + oct[0] * (nx[0] / 2) + i - box[0])] =
              coarse[n * cvol + ((int64_t)k * cn[1] + j) * cn[0] + i];
  free(coarse);
}

/* ---- puncture tracker, z4c/puncture_tracker.cpp:95-129 ------------------ */

/* LagrangeInterp1D<7> (utils/lagrange_interp.hpp:33-146), odd order: first
 * stencil point and the coefficients of the 8-point stencil. */
#define TRK_ORDER (2 * NG - 1)
static int lagrange1d(double origin, double delta, int siz, double coord, double coeff[]) {
  const double delta_inv = 1.0 / delta;
  int point = (int)lrint(floor((coord - origin) * delta_inv - 0.5 * (TRK_ORDER - 1)));
  int shift = point;
  if (shift < 0) point -= shift;
  shift = point + TRK_ORDER - (siz - 1);
  if (shift > 0) point -= shift;
  double xp[TRK_ORDER + 1];
  for (int i = 0; i <= TRK_ORDER; ++i) xp[i] = (point + i) * delta + origin;
  for (int j = 0; j <= TRK_ORDER; ++j) {
    double num = 1.0, den = 1.0;
    for (int i = 0; i <= TRK_ORDER; ++i) {
      if (i == j) continue;
      num = num * (coord - xp[i]);
      den = den * (xp[j] - xp[i]);
    }
    coeff[j] = num / den;
  }
  return point;
}

void orc_tracker_interp(const orc_block_t *b, const double *u, const double pos[3],
                        double beta[3]) {
  const int nn[3] = {b->nx[0] + 1 + 2 * NG, b->nx[1] + 1 + 2 * NG, b->nx[2] + 1 + 2 * NG};
  const int64_t nvol = (int64_t)nn[0] * nn[1] * nn[2];
  double c[3][TRK_ORDER + 1];
  int pt[3];
  for (int a = 0; a < 3; ++a) pt[a] = lagrange1d(b->x[a][0], b->dx[a], nn[a], pos[a], c[a]);
  for (int v = 0; v < 3; ++v) {
    const double *f = u + (Z4C_BETAX + v) * nvol;
    /* LagrangeInterpND::m_fill_stencil: x innermost, then y, then z */
    double vz[TRK_ORDER + 1];
    for (int ez = 0; ez <= TRK_ORDER; ++ez) {
      double vy[TRK_ORDER + 1];
      for (int ey = 0; ey <= TRK_ORDER; ++ey) {
        const double *row = f + ((int64_t)(pt[2] + ez) * nn[1] + (pt[1] + ey)) * nn[0] + pt[0];
        double o = 0;
        for (int i = 0; i <= TRK_ORDER; ++i) o += c[0][i] * row[i];
        vy[ey] = o;
      }
      double o = 0;
      for (int i = 0; i <= TRK_ORDER; ++i) o += c[1][i] * vy[i];
      vz[ez] = o;
    }
    double o = 0;
    for (int i = 0; i <= TRK_ORDER; ++i) o += c[2][i] * vz[i];
    beta[v] = o;
  }
}

/* ---- psi4 extraction -------------------------------------------------------
 * GeodesicGrid (mesh/geodesic_grid.cpp:21-160, geodesic_grid.hpp:145-160):
 * five blocks of nlev x 2 nlev vertices plus the two poles, each block held
 * with one ghost row/column; vertex ic = bl 2 nlev^2 + l 2 nlev + m. */
#define GEO_PI 3.1415926535897932 /* PI of the reference's defs.hpp.in:250 */
typedef struct {
  int nlev;
  double *c[3]; /* [5][nlev+2][2 nlev+2] unit-vector components */
  int *idx;     /* [5][nlev+2][2 nlev+2] vertex indices */
  double pol[3][2];
  int poli[2];
} geo_t;

static inline int64_t geo_at(const geo_t *g, int bl, int l, int m) {
  return ((int64_t)bl * (g->nlev + 2) + l) * (2 * g->nlev + 2) + m;
}

static void geo_fill_ghosts_d(const geo_t *g, double *a, const double *pole) {
  const int n = g->nlev;
  for (int bl = 0; bl < 5; ++bl) {
    for (int k = 0; k < n; ++k) {
      a[geo_at(g, bl, 0, k + 1)] = a[geo_at(g, (bl + 4) % 5, k + 1, 1)];
      a[geo_at(g, bl, 0, k + n + 1)] = a[geo_at(g, (bl + 4) % 5, n, k + 1)];
      a[geo_at(g, bl, k + 1, 2 * n + 1)] = a[geo_at(g, (bl + 4) % 5, n, k + n + 1)];
      a[geo_at(g, bl, k + 2, 0)] = a[geo_at(g, (bl + 1) % 5, 1, k + 1)];
      a[geo_at(g, bl, n + 1, k + 1)] = a[geo_at(g, (bl + 1) % 5, 1, k + n + 1)];
      a[geo_at(g, bl, n + 1, k + n + 1)] = a[geo_at(g, (bl + 1) % 5, k + 2, 2 * n)];
    }
    a[geo_at(g, bl, 1, 0)] = pole[0];
    a[geo_at(g, bl, n + 1, 2 * n)] = pole[1];
    a[geo_at(g, bl, 0, 2 * n + 1)] = a[geo_at(g, bl, 0, 2 * n)];
  }
}

static void geo_fill_ghosts_i(const geo_t *g, int *a, const int *pole) {
  const int n = g->nlev;
  for (int bl = 0; bl < 5; ++bl) {
    for (int k = 0; k < n; ++k) {
      a[geo_at(g, bl, 0, k + 1)] = a[geo_at(g, (bl + 4) % 5, k + 1, 1)];
      a[geo_at(g, bl, 0, k + n + 1)] = a[geo_at(g, (bl + 4) % 5, n, k + 1)];
      a[geo_at(g, bl, k + 1, 2 * n + 1)] = a[geo_at(g, (bl + 4) % 5, n, k + n + 1)];
      a[geo_at(g, bl, k + 2, 0)] = a[geo_at(g, (bl + 1) % 5, 1, k + 1)];
      a[geo_at(g, bl, n + 1, k + 1)] = a[geo_at(g, (bl + 1) % 5, 1, k + n + 1)];
      a[geo_at(g, bl, n + 1, k + n + 1)] = a[geo_at(g, (bl + 1) % 5, k + 2, 2 * n)];
    }
    a[geo_at(g, bl, 1, 0)] = pole[0];
    a[geo_at(g, bl, n + 1, 2 * n)] = pole[1];
    a[geo_at(g, bl, 0, 2 * n + 1)] = a[geo_at(g, bl, 0, 2 * n)];
  }
}

/* one vertex of row l of block 0: the normalised (wa A + wb B + wc C) / nlev */
static void geo_put(geo_t *g, int row, int col, int wa, const double *A, int wb, const double *B,
                    int wc, const double *C) {
  const double n = (double)g->nlev;
  const double x = (wa * A[0] + wb * B[0] + wc * C[0]) / n;
  const double y = (wa * A[1] + wb * B[1] + wc * C[1]) / n;
  const double z = (wa * A[2] + wb * B[2] + wc * C[2]) / n;
  const double norm = sqrt(x * x + y * y + z * z);
  const int64_t q = geo_at(g, 0, row, col);
  g->c[0][q] = x / norm;
  g->c[1][q] = y / norm;
  g->c[2][q] = z / norm;
}

static int geo_init(geo_t *g, int nlev) {
  g->nlev = nlev;
  const int64_t sz = (int64_t)5 * (nlev + 2) * (2 * nlev + 2);
  for (int a = 0; a < 3; ++a) g->c[a] = (double *)calloc((size_t)sz, sizeof(double));
  g->idx = (int *)calloc((size_t)sz, sizeof(int));
  if (!g->c[0] || !g->c[1] || !g->c[2] || !g->idx) return -1;
  const double sa = 2.0 / sqrt(5.0), ca = 1.0 / sqrt(5.0);
  const double P1[3] = {0.0, 0.0, 1.0};
  const double P2[3] = {sa, 0.0, ca};
  const double P3[3] = {sa * cos(0.2 * GEO_PI), sa * sin(0.2 * GEO_PI), -ca};
  const double P4[3] = {sa * cos(-0.4 * GEO_PI), sa * sin(-0.4 * GEO_PI), ca};
  const double P5[3] = {sa * cos(-0.2 * GEO_PI), sa * sin(-0.2 * GEO_PI), -ca};
  const double P6[3] = {0.0, 0.0, -1.0};
  for (int l = 0; l < nlev; ++l) {
    int col = 1;
    for (int m = l; m < nlev; ++m) geo_put(g, l + 1, col++, m - l + 1, P2, nlev - m - 1, P1, l, P4);
    for (int m = nlev - l; m < nlev; ++m)
      geo_put(g, l + 1, col++, nlev - l, P2, m - nlev + l + 1, P5, nlev - m - 1, P4);
    for (int m = l; m < nlev; ++m) geo_put(g, l + 1, col++, m - l + 1, P3, nlev - m - 1, P2, l, P5);
    for (int m = nlev - l; m < nlev; ++m)
      geo_put(g, l + 1, col++, nlev - l, P3, m - nlev + l + 1, P6, nlev - m - 1, P5);
  }
  for (int bl = 1; bl < 5; ++bl)
    for (int l = 1; l < nlev + 1; ++l)
      for (int m = 1; m < 2 * nlev + 1; ++m) {
        const int64_t q0 = geo_at(g, 0, l, m), q = geo_at(g, bl, l, m);
        const double x0 = g->c[0][q0], y0 = g->c[1][q0];
        g->c[0][q] = x0 * cos(bl * 0.4 * GEO_PI) + y0 * sin(bl * 0.4 * GEO_PI);
        g->c[1][q] = y0 * cos(bl * 0.4 * GEO_PI) - x0 * sin(bl * 0.4 * GEO_PI);
        g->c[2][q] = g->c[2][q0];
      }
  g->pol[0][0] = 0.0; g->pol[1][0] = 0.0; g->pol[2][0] = 1.0;
  g->pol[0][1] = 0.0; g->pol[1][1] = 0.0; g->pol[2][1] = -1.0;
  for (int a = 0; a < 3; ++a) geo_fill_ghosts_d(g, g->c[a], g->pol[a]);
  for (int bl = 0; bl < 5; ++bl)
    for (int l = 0; l < nlev; ++l)
      for (int m = 0; m < 2 * nlev; ++m)
        g->idx[geo_at(g, bl, l + 1, m + 1)] = bl * 2 * nlev * nlev + l * 2 * nlev + m;
  g->poli[0] = 10 * nlev * nlev;
  g->poli[1] = 10 * nlev * nlev + 1;
  geo_fill_ghosts_i(g, g->idx, g->poli);
  return 0;
}

static void geo_free(geo_t *g) {
  for (int a = 0; a < 3; ++a) free(g->c[a]);
  free(g->idx);
}

/* GeodesicGrid::Position (:219-236) */
static void geo_position(const geo_t *g, int ic, double out[3]) {
  const int n = g->nlev;
  const int b0 = ic / (2 * n * n), b1 = (ic % (2 * n * n)) / (2 * n), b2 = (ic % (2 * n * n)) % (2 * n);
  for (int a = 0; a < 3; ++a)
    out[a] = (b0 == 5) ? g->pol[a][b2] : g->c[a][geo_at(g, b0, b1 + 1, b2 + 1)];
}

/* GeodesicGrid::NumNeighbors (:168-206) */
static int geo_neighbours(const geo_t *g, int ic, int nb[6]) {
  const int n = g->nlev;
  if (ic == 10 * n * n) {
    for (int bl = 0; bl < 5; ++bl) nb[bl] = g->idx[geo_at(g, bl, 1, 1)];
    return 5;
  }
  if (ic == 10 * n * n + 1) {
    for (int bl = 0; bl < 5; ++bl) nb[bl] = g->idx[geo_at(g, bl, n, 2 * n)];
    return 5;
  }
  const int b0 = ic / (2 * n * n), b1 = (ic % (2 * n * n)) / (2 * n), b2 = (ic % (2 * n * n)) % (2 * n);
  nb[0] = g->idx[geo_at(g, b0, b1 + 1, b2 + 2)];
  nb[1] = g->idx[geo_at(g, b0, b1 + 2, b2 + 1)];
  nb[2] = g->idx[geo_at(g, b0, b1 + 2, b2)];
  nb[3] = g->idx[geo_at(g, b0, b1 + 1, b2)];
  nb[4] = g->idx[geo_at(g, b0, b1, b2 + 1)];
  if (ic % (2 * n * n) == n - 1 || ic % (2 * n * n) == 2 * n - 1) return 5;
  nb[5] = g->idx[geo_at(g, b0, b1, b2 + 2)];
  return 6;
}

/* GeodesicGrid::CircumcenterNormalized (:463-475) */
static void geo_circumcentre(const double p1[3], const double p2[3], const double p3[3],
                             double out[3]) {
  const double x1 = p1[0], x2 = p2[0], x3 = p3[0];
  const double y1 = p1[1], y2 = p2[1], y3 = p3[1];
  const double z1 = p1[2], z2 = p2[2], z3 = p3[2];
  const double a = sqrt((x3 - x2) * (x3 - x2) + (y3 - y2) * (y3 - y2) + (z3 - z2) * (z3 - z2));
  const double b = sqrt((x1 - x3) * (x1 - x3) + (y1 - y3) * (y1 - y3) + (z1 - z3) * (z1 - z3));
  const double c = sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1) + (z2 - z1) * (z2 - z1));
  const double den = 1.0 / ((a + c + b) * (a + c - b) * (a + b - c) * (b + c - a));
  const double xc = (x1 * a * a * (b * b + c * c - a * a) + x2 * b * b * (c * c + a * a - b * b) +
                     x3 * c * c * (a * a + b * b - c * c)) * den;
  const double yc = (y1 * a * a * (b * b + c * c - a * a) + y2 * b * b * (c * c + a * a - b * b) +
                     y3 * c * c * (a * a + b * b - c * c)) * den;
  const double zc = (z1 * a * a * (b * b + c * c - a * a) + z2 * b * b * (c * c + a * a - b * b) +
                     z3 * c * c * (a * a + b * b - c * c)) * den;
  const double nc = sqrt(xc * xc + yc * yc + zc * zc);
  out[0] = xc / nc;
  out[1] = yc / nc;
  out[2] = zc / nc;
}

/* GeodesicGrid::ComputeWeightAndDualEdges (:312-360): the dual-cell area */
static double geo_weight(const geo_t *g, int ic) {
  int nv[6];
  const int nn = geo_neighbours(g, ic, nv);
  double p0[3];
  geo_position(g, ic, p0);
  double w = 0.0;
  for (int q = 0; q < nn; ++q) {
    double n1[3], n2[3], n3[3], c1[3], c2[3];
    geo_position(g, nv[(q + nn - 1) % nn], n1);
    geo_position(g, nv[q], n2);
    geo_position(g, nv[(q + 1) % nn], n3);
    geo_circumcentre(p0, n1, n2, c1);
    geo_circumcentre(p0, n2, n3, c2);
    const double s1 = p0[0] * c1[0] + p0[1] * c1[1] + p0[2] * c1[2];
    const double s2 = p0[0] * c2[0] + p0[1] * c2[1] + p0[2] * c2[2];
    const double s12 = c1[0] * c2[0] + c1[1] * c2[1] + c1[2] * c2[2];
    const double num = fabs(p0[0] * (c1[1] * c2[2] - c2[1] * c1[2]) +
                            p0[1] * (c2[0] * c1[2] - c1[0] * c2[2]) +
                            p0[2] * (c1[0] * c2[1] - c1[1] * c2[0]));
    const double den = 1.0 + s1 + s2 + s12;
    w += 2.0 * atan(num / den);
  }
  return w;
}

/* SphericalGrid (mesh/spherical_grid.cpp:17-36) over GeodesicGrid */
int orc_sphere_grid(int nlev, double rad, int bitant, double *geo) {
  geo_t g;
  if (geo_init(&g, nlev)) {
    geo_free(&g);
    return -1;
  }
  const int np = 10 * nlev * nlev + 2;
  for (int ic = 0; ic < np; ++ic) {
    double p[3];
    geo_position(&g, ic, p);
    const double th = acos(p[2]), ph = atan2(p[1], p[0]);
    double *o = geo + 6 * (int64_t)ic;
    o[0] = th;
    o[1] = ph;
    o[2] = rad * sin(th) * cos(ph);
    o[3] = rad * sin(th) * sin(ph);
    o[4] = rad * cos(th);
    if (bitant) o[4] = fabs(o[4]);
    o[5] = rad * rad * geo_weight(&g, ic);
  }
  geo_free(&g);
  return np;
}

/* gra::sph_harm::Factorial over its table (spherical_harmonics.hpp:20-60) */
static double sph_fact(int n) {
  double t = 1.0;
  for (int i = 1; i <= n; ++i) t = t * (double)i;
  return t;
}

void orc_sylm(int s, int l, int m, double theta, double phi, double *re, double *im) {
  double wd = 0;
  const int k1 = (0 > m + s) ? 0 : m + s;
  const int k2 = (l + m < l + s) ? l + m : l + s;
  for (int k = k1; k <= k2; ++k) {
    wd += ((k % 2 == 0) ? 1.0 : -1.0) *
          sqrt(sph_fact(l + m) * sph_fact(l - m) * sph_fact(l - s) * sph_fact(l + s)) *
          pow(cos(theta / 2.0), (double)(2 * l + m + s - 2 * k)) *
          pow(sin(theta / 2.0), (double)(2 * k - m - s)) /
          (sph_fact(l + m - k) * sph_fact(l + s - k) * sph_fact(k) * sph_fact(k - m - s));
  }
  const double norm = sqrt((2 * l + 1) / (4.0 * GEO_PI));
  *re = norm * wd * cos(m * phi);
  *im = norm * wd * sin(m * phi);
}

/* LagrangeInterpND<7, 3>::eval of one variable: x innermost, then y, then z */
static double lagrange_eval3(const double *f, const int nn[3], const int pt[3],
                             double c[3][TRK_ORDER + 1]) {
  double vz[TRK_ORDER + 1];
  for (int ez = 0; ez <= TRK_ORDER; ++ez) {
    double vy[TRK_ORDER + 1];
    for (int ey = 0; ey <= TRK_ORDER; ++ey) {
      const double *row = f + ((int64_t)(pt[2] + ez) * nn[1] + (pt[1] + ey)) * nn[0] + pt[0];
      double o = 0;
      for (int i = 0; i <= TRK_ORDER; ++i) o += c[0][i] * row[i];
      vy[ey] = o;
    }
    double o = 0;
    for (int i = 0; i <= TRK_ORDER; ++i) o += c[1][i] * vy[i];
    vz[ez] = o;
  }
  double o = 0;
  for (int i = 0; i <= TRK_ORDER; ++i) o += c[2][i] * vz[i];
  return o;
}

/* SphericalPatch (spherical_grid.cpp:44-116, vertex collocation) and
 * WaveExtractLocal::Decompose_multipole (wave_extract.cpp:160-234) */
int orc_wave_block(const orc_block_t *b, const double *weyl, int np, const double *geo,
                   double rad, int lmax, int bitant, int *owned, double *psi) {
  const int nn[3] = {b->nx[0] + 1 + 2 * NG, b->nx[1] + 1 + 2 * NG, b->nx[2] + 1 + 2 * NG};
  const int64_t nvol = (int64_t)nn[0] * nn[1] * nn[2];
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = b->x[a][NG];
    hi[a] = b->x[a][NG + b->nx[a]];
  }
  int n = 0;
  for (int ic = 0; ic < np; ++ic) {
    const double *o = geo + 6 * (int64_t)ic;
    if (o[2] >= lo[0] && o[2] < hi[0] && o[3] >= lo[1] && o[3] < hi[1] && o[4] >= lo[2] &&
        o[4] < hi[2])
      owned[n++] = ic;
  }
  double *dr = (double *)malloc(sizeof(double) * (n ? n : 1));
  double *di = (double *)malloc(sizeof(double) * (n ? n : 1));
  double *wt = (double *)malloc(sizeof(double) * (n ? n : 1));
  for (int q = 0; q < n; ++q) {
    const double *o = geo + 6 * (int64_t)owned[q];
    double c[3][TRK_ORDER + 1];
    int pt[3];
    for (int a = 0; a < 3; ++a) pt[a] = lagrange1d(b->x[a][0], b->dx[a], nn[a], o[2 + a], c[a]);
    dr[q] = lagrange_eval3(weyl, nn, pt, c);
    di[q] = lagrange_eval3(weyl + nvol, nn, pt, c);
    wt[q] = o[5];
    wt[q] /= rad * rad;
  }
  const int nm = 2 * lmax + 1;
  for (int q = 0; q < (lmax - 1) * nm * 2; ++q) psi[q] = 0.0;
  for (int l = 2; l < lmax + 1; ++l)
    for (int m = -l; m < l + 1; ++m) {
      double pr = 0.0, pi = 0.0;
      for (int q = 0; q < n; ++q) {
        const double *o = geo + 6 * (int64_t)owned[q];
        double yr, yi;
        orc_sylm(-2, l, m, o[0], o[1], &yr, &yi);
        const double bz = (bitant && o[0] > GEO_PI / 2) ? -1 : 1;
        pr += dr[q] * wt[q] * yr + bz * di[q] * wt[q] * yi;
        pi += bz * di[q] * wt[q] * yr - dr[q] * wt[q] * yi;
      }
      psi[((l - 2) * nm + (m + l)) * 2 + 0] = pr;
      psi[((l - 2) * nm + (m + l)) * 2 + 1] = pi;
    }
  free(dr);
  free(di);
  free(wt);
  return n;
}

/* ---- history sums, outputs/history.cpp:168-200 --------------------------- */
void orc_hst_accumulate(const orc_block_t *b, const z4c_params_t *opt,
                        const double *con, const double *u, double out[8]) {
  fd_t f;
  fd_init(b, &f);
  const int64_t nvol = orc_nvol(b);
  const double r2_max = opt->r_max_con * opt->r_max_con;
  for (int k = NG; k <= NG + b->nx[2] - 1; ++k)
    for (int j = NG; j <= NG + b->nx[1] - 1; ++j)
      for (int i = NG; i <= NG + b->nx[0] - 1; ++i) {
        const double vol = b->dx[0] * b->dx[1] * b->dx[2];
        const double x1 = b->xc[0][i], x2 = b->xc[1][j], x3 = b->xc[2][k];
        const double R2 = x1 * x1 + x2 * x2 + x3 * x3;
        if (!(R2 <= r2_max)) continue;
        const int64_t p = P(k, j, i);
        const double H = fabs(V(con, Z4C_CON_H)[p]);
        out[0] += vol * (H * H);
        out[1] += vol * fabs(V(con, Z4C_CON_M)[p]);
        for (int a = 0; a < 3; ++a) {
          const double m = fabs(V(con, Z4C_CON_MX + a)[p]);
          out[2 + a] += vol * (m * m);
        }
        out[5] += vol * fabs(V(con, Z4C_CON_Z)[p]);
        const double th = fabs(V(u, Z4C_THETA)[p]);
        out[6] += vol * (th * th);
        out[7] += vol * fabs(V(con, Z4C_CON_C)[p]);
      }
}

/* ---- multilevel (static mesh refinement) ghost exchange ------------------
 *
 * The vertex-centred exchange of a mesh whose MeshBlocks sit on several
 * refinement levels, restated step by step as the reference runs it for one
 * ghost fill of the Z4c state (task order of task_list/gr/
 * task_list_gr_z4c.cpp:52-64: SEND, RECV, SETB, PROLONG, PHY_BVAL):
 *   1. every block restricts its interior into its coarse buffer
 *      (CommRegistry::SendBoundaryBuffers, comm_registry.cpp:246-296, and
 *      RestrictInterior, refinement_ops.cpp:167-195: injection);
 *   2. every block packs one message per neighbour from that pre-exchange
 *      state (CommChannel::PackAndSend, comm_channel.cpp:733-787);
 *   3. every block zeroes its fine and coarse ghosts, unpacks the messages in
 *      neighbour order (same level: added into the fine array and, for the
 *      coarse payload, into the coarse buffer; from a coarser block: copied
 *      into the coarse buffer; from a finer block: added into the fine array;
 *      comm_channel.cpp:1278-1474) and multiplies by the inverse node
 *      multiplicity (node_multiplicity.cpp:102-430);
 *   4. coarse-level physical BCs and prolongation into the ghosts next to
 *      coarser blocks (CommRegistry::ProlongateAndApplyPhysicalBCs,
 *      comm_registry.cpp:533-570; physical_bcs.cpp:687-890;
 *      refinement_ops.cpp:24-160);
 *   5. fine-level physical BCs (physical_bcs.cpp:506-670).
 * The neighbour list follows mesh_topology.cpp:278-960, the index ranges
 * comm/index_utilities.{hpp,cpp}. */

typedef struct {
  int gid, level, ox[3], fi[2];
} ml_nb_t;

typedef struct {
  const orc_ml_mesh_t *m;
  int nn[3], cn[3];
  int64_t fvol, cvol;
} ml_geo_t;

static int ml_leaf(const orc_ml_mesh_t *m, int level, const int64_t l[3]) {
  for (int b = 0; b < m->nblocks; ++b)
    if (m->loc[4 * b] == level && m->loc[4 * b + 1] == l[0] && m->loc[4 * b + 2] == l[1] &&
        m->loc[4 * b + 3] == l[2])
      return b;
  return -1;
}

/* MeshBlockTree::FindNeighbor (meshblock_tree.cpp:400-490): 0 = beyond a
 * non-periodic face, 1 = a leaf of the same or the next coarser level
 * (*gid), 2 = a refined node whose children are leaves (nl its location). */
static int ml_find(const orc_ml_mesh_t *m, int level, const int64_t *loc, const int o[3],
                   int64_t nl[3], int *gid) {
  for (int a = 0; a < 3; ++a) {
    const int64_t n = (int64_t)m->nroot[a] << (level - m->root_level);
    nl[a] = loc[a] + o[a];
    if (nl[a] < 0) {
      if (m->bc[2 * a] != Z4C_BC_PERIODIC) return 0;
      nl[a] = n - 1;
    }
    if (nl[a] >= n) {
      if (m->bc[2 * a + 1] != Z4C_BC_PERIODIC) return 0;
      nl[a] = 0;
    }
  }
  int b = ml_leaf(m, level, nl);
  if (b >= 0) { *gid = b; return 1; }
  const int64_t pl[3] = {nl[0] >> 1, nl[1] >> 1, nl[2] >> 1};
  b = ml_leaf(m, level - 1, pl);
  if (b >= 0) { *gid = b; return 1; }
  return 2;
}

static int ml_child(const orc_ml_mesh_t *m, int level, const int64_t nl[3], const int c[3]) {
  const int64_t l[3] = {2 * nl[0] + c[0], 2 * nl[1] + c[1], 2 * nl[2] + c[2]};
  return ml_leaf(m, level + 1, l);
}

/* MeshBlock::SearchAndSetNeighbors (mesh_topology.cpp:278-960), 3-D. */
static int ml_neighbours(const orc_ml_mesh_t *m, int b, ml_nb_t *out) {
  const int lev = m->loc[4 * b];
  const int64_t *loc = &m->loc[4 * b + 1];
  int myox[3];
  for (int a = 0; a < 3; ++a) myox[a] = (loc[a] & 1) ? 1 : -1;
  int cnt = 0, gid;
  int64_t nl[3];
  /* faces: x1, x2, x3, each -1 then +1; finer neighbours as 4 leaves with
   * the two transverse child indices (f1 the lower axis) */
  for (int ax = 0; ax < 3; ++ax)
    for (int s = -1; s <= 1; s += 2) {
      int o[3] = {0, 0, 0};
      o[ax] = s;
      const int r = ml_find(m, lev, loc, o, nl, &gid);
      if (r == 0) continue;
      if (r == 2) {
        const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
        for (int f2 = 0; f2 < 2; ++f2)
          for (int f1 = 0; f1 < 2; ++f1) {
            int c[3];
            c[ax] = 1 - (s + 1) / 2;
            c[t1] = f1;
            c[t2] = f2;
            ml_nb_t e = {ml_child(m, lev, nl, c), lev + 1, {o[0], o[1], o[2]}, {f1, f2}};
            out[cnt++] = e;
          }
      } else {
        ml_nb_t e = {gid, m->loc[4 * gid], {o[0], o[1], o[2]}, {0, 0}};
        out[cnt++] = e;
      }
    }
  /* edges x1x2, x1x3, x2x3: the second axis' offset outer, the first's inner */
  static const int pairs[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
  for (int q = 0; q < 3; ++q) {
    const int a0 = pairs[q][0], a1 = pairs[q][1], a2 = pairs[q][2];
    for (int mm = -1; mm <= 1; mm += 2)
      for (int n = -1; n <= 1; n += 2) {
        int o[3] = {0, 0, 0};
        o[a0] = n;
        o[a1] = mm;
        const int r = ml_find(m, lev, loc, o, nl, &gid);
        if (r == 0) continue;
        if (r == 2) {
          for (int f1 = 0; f1 < 2; ++f1) {
            int c[3];
            c[a0] = 1 - (n + 1) / 2;
            c[a1] = 1 - (mm + 1) / 2;
            c[a2] = f1;
            ml_nb_t e = {ml_child(m, lev, nl, c), lev + 1, {o[0], o[1], o[2]}, {f1, 0}};
            out[cnt++] = e;
          }
        } else {
          const int nlev = m->loc[4 * gid];
          if (nlev >= lev || (myox[a0] == n && myox[a1] == mm)) {
            ml_nb_t e = {gid, nlev, {o[0], o[1], o[2]}, {0, 0}};
            out[cnt++] = e;
          }
        }
      }
  }
  /* corners */
  for (int l = -1; l <= 1; l += 2)
    for (int mm = -1; mm <= 1; mm += 2)
      for (int n = -1; n <= 1; n += 2) {
        const int o[3] = {n, mm, l};
        const int r = ml_find(m, lev, loc, o, nl, &gid);
        if (r == 0) continue;
        int nlev;
        if (r == 2) {
          const int c[3] = {1 - (n + 1) / 2, 1 - (mm + 1) / 2, 1 - (l + 1) / 2};
          gid = ml_child(m, lev, nl, c);
          nlev = lev + 1;
        } else {
          nlev = m->loc[4 * gid];
        }
        if (nlev >= lev || (myox[0] == n && myox[1] == mm && myox[2] == l)) {
          ml_nb_t e = {gid, nlev, {n, mm, l}, {0, 0}};
          out[cnt++] = e;
        }
      }
  return cnt;
}

int orc_ml_neighbours(const orc_ml_mesh_t *m, int b, int *out) {
  ml_nb_t nb[56];
  const int cnt = ml_neighbours(m, b, nb);
  for (int q = 0; q < cnt; ++q) {
    int *r = out + 7 * q;
    r[0] = nb[q].gid; r[1] = nb[q].level;
    r[2] = nb[q].ox[0]; r[3] = nb[q].ox[1]; r[4] = nb[q].ox[2];
    r[5] = nb[q].fi[0]; r[6] = nb[q].fi[1];
  }
  return cnt;
}

/* Index ranges of one axis (index_utilities.hpp:124-216) on the fine array
 * (vs = NG, ve = NG + nx, ms = 0, pe = nx + 2 NG) or the coarse buffer
 * (vs = NCG, ve = NCG + nx/2, ...).  fi < 0: the axis is not narrowed. */
typedef struct { int vs, ve, ms, me, ps, pe, gs, ge, ng; } ml_ax_t;
static ml_ax_t ml_axis(int nx, int ng) {
  ml_ax_t a;
  a.ng = ng; a.vs = ng; a.ve = ng + nx; a.ms = 0; a.me = ng - 1;
  a.ps = nx + ng + 1; a.pe = nx + 2 * ng; a.gs = a.vs + ng; a.ge = a.ve - ng;
  return a;
}
/* LoadRangeVC */
static void r_load_same(int ox, ml_ax_t a, int *s, int *e) {
  *s = ox > 0 ? a.ge : a.vs;
  *e = ox < 0 ? a.gs : a.ve;
}
/* SetRangeVC */
static void r_set_same(int ox, ml_ax_t a, int *s, int *e) {
  if (ox == 0) { *s = a.vs; *e = a.ve; }
  else if (ox > 0) { *s = a.ve; *e = a.pe; }
  else { *s = a.ms; *e = a.vs; }
}
/* SetFromCoarserRangeVC (coarse axis) */
static void r_set_from_coarser(int ox, ml_ax_t c, int64_t lx, int *s, int *e) {
  if (ox == 0) {
    *s = c.vs; *e = c.ve;
    if ((lx & 1) == 0) *e = c.pe;
    else *s = c.ms;
  } else if (ox > 0) { *s = c.ps; *e = c.pe; }
  else { *s = c.ms; *e = c.me; }
}
/* LoadToCoarserRangeVC (coarse axis, fine ghost width ng) */
static void r_load_to_coarser(int ox, ml_ax_t c, int ng, int *s, int *e) {
  if (ox > 0) { *s = c.ve - ng; *e = c.ve; }
  else if (ox < 0) { *s = c.vs; *e = c.vs + ng; }
  else { *s = c.vs; *e = c.ve; }
}
/* LoadToFinerRangeVC (fine axis, slab width cng, half size hs) */
static void r_load_to_finer(int ox, ml_ax_t a, int cng, int fi, int hs, int *s, int *e) {
  if (ox > 0) { *s = a.ve - cng; *e = a.ve - 1; }
  else if (ox < 0) { *s = a.vs + 1; *e = a.vs + cng; }
  else {
    *s = a.vs; *e = a.ve;
    if (fi == 1) *s += hs;
    else *e -= hs;
  }
}
/* SetFromFinerRangeVC (fine axis, half size hs) */
static void r_set_from_finer(int ox, ml_ax_t a, int fi, int hs, int *s, int *e) {
  if (ox == 0) {
    *s = a.vs; *e = a.ve;
    if (fi == 1) *s += hs;
    else *e -= hs;
  } else if (ox > 0) { *s = a.ve; *e = a.pe; }
  else { *s = a.ms; *e = a.vs; }
}
/* which of fi1/fi2 narrows axis a (index_utilities.cpp:830-873) */
static int ml_fi(const ml_nb_t *e, int a) {
  if (a == 0) return e->fi[0];
  if (a == 1) return e->ox[0] != 0 ? e->fi[0] : e->fi[1];
  return (e->ox[0] != 0 && e->ox[1] != 0) ? e->fi[0] : e->fi[1];
}

static int64_t box_count(const int bx[6]) {
  return (int64_t)(bx[1] - bx[0] + 1) * (bx[3] - bx[2] + 1) * (bx[5] - bx[4] + 1);
}
/* BufferUtility::PackData / UnpackData(Add) over n, k, j, i */
static void box_pack(const double *a, const int dims[3], int nvar, const int bx[6], double *buf,
                     int64_t *p) {
  const int64_t vol = (int64_t)dims[0] * dims[1] * dims[2];
  for (int n = 0; n < nvar; ++n)
    for (int k = bx[4]; k <= bx[5]; ++k)
      for (int j = bx[2]; j <= bx[3]; ++j)
        for (int i = bx[0]; i <= bx[1]; ++i)
          buf[(*p)++] = a[n * vol + ((int64_t)k * dims[1] + j) * dims[0] + i];
}
static void box_unpack(double *a, const int dims[3], int nvar, const int bx[6], const double *buf,
                       int64_t *p, int add) {
  const int64_t vol = (int64_t)dims[0] * dims[1] * dims[2];
  for (int n = 0; n < nvar; ++n)
    for (int k = bx[4]; k <= bx[5]; ++k)
      for (int j = bx[2]; j <= bx[3]; ++j)
        for (int i = bx[0]; i <= bx[1]; ++i) {
          double *d = &a[n * vol + ((int64_t)k * dims[1] + j) * dims[0] + i];
          if (add) *d += buf[(*p)++];
          else *d = buf[(*p)++];
        }
}

/* ExtrapolateOutflowBC with NEXTRAPOLATE = 5 on the faces need[] of one
 * array, is/ie the interior ends the caller passes and ng the ghost width;
 * transverse limits as ApplyPhysicalBCs / ApplyPhysicalBCsOnCoarseLevel. */
static void ml_bcs(const int need[6], const int is[3], const int ie[3], int ng, const int dims[3],
                   int nvar, double *u) {
  const int64_t vol = (int64_t)dims[0] * dims[1] * dims[2];
  const int64_t st[3] = {1, dims[0], (int64_t)dims[0] * dims[1]};
  int bis = is[0] - ng, bie = ie[0] + ng;
  int bjs = need[2] ? is[1] : is[1] - ng, bje = need[3] ? ie[1] : ie[1] + ng;
  int bks = need[4] ? is[2] : is[2] - ng, bke = need[5] ? ie[2] : ie[2] + ng;
  for (int face = 0; face < 6; ++face) {
    if (!need[face]) continue;
    const int ax = face / 2, outer = face % 2;
    int lo[3], hi[3];
    if (ax == 0) { lo[1] = bjs; hi[1] = bje; lo[2] = bks; hi[2] = bke; }
    else if (ax == 1) { lo[0] = bis; hi[0] = bie; lo[2] = bks; hi[2] = bke; }
    else { lo[0] = bis; hi[0] = bie; lo[1] = is[1] - ng; hi[1] = ie[1] + ng; }
    const int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
    for (int n = 0; n < nvar; ++n)
      for (int t2 = lo[o2]; t2 <= hi[o2]; ++t2)
        for (int t1 = lo[o1]; t1 <= hi[o1]; ++t1)
          for (int g = 1; g <= ng; ++g) {
            const int ia = outer ? ie[ax] + g : is[ax] - g;
            const int dir = outer ? -1 : 1;
            const int64_t p = (int64_t)ia * st[ax] + (int64_t)t1 * st[o1] + (int64_t)t2 * st[o2];
            double v = 0.0;
            for (int q = 0; q < 5; ++q) v += CE[q] * u[n * vol + p + dir * (q + 1) * st[ax]];
            u[n * vol + p] = v;
          }
  }
}

/* ZeroGhosts / ZeroGhostsCoarse: everything outside [vs, ve]^3 */
static void ml_zero_ghosts(double *a, const int dims[3], int nvar, ml_ax_t x, ml_ax_t y,
                           ml_ax_t z) {
  const int64_t vol = (int64_t)dims[0] * dims[1] * dims[2];
  for (int n = 0; n < nvar; ++n)
    for (int k = 0; k < dims[2]; ++k)
      for (int j = 0; j < dims[1]; ++j)
        for (int i = 0; i < dims[0]; ++i)
          if (i < x.vs || i > x.ve || j < y.vs || j > y.ve || k < z.vs || k > z.ve)
            a[n * vol + ((int64_t)k * dims[1] + j) * dims[0] + i] = 0.0;
}

/* ApplyDivisionImpl (node_multiplicity.cpp:364-430): compact zone c of an
 * axis -> physical range */
static void ml_phys(int c, ml_ax_t a, int *lo, int *hi) {
  const int half = (a.ve - a.vs) / 2;
  const int t[7] = {a.ms, a.vs, a.vs + 1, a.vs + half, a.ve - 1, a.ve, a.pe};
  if (c & 1) { *lo = *hi = t[c]; }
  else if (c <= 3) { *lo = t[c]; *hi = t[c + 1] - 1; }
  else { *lo = t[c - 1] + 1; *hi = t[c]; }
}

/* NodeMultiplicity::Precompute (node_multiplicity.cpp:102-180) */
static void ml_multiplicity(const orc_ml_mesh_t *m, int b, const ml_nb_t *nb, int cnt,
                            unsigned short mult[7][7][7]) {
  const int lev = m->loc[4 * b];
  memset(mult, 0, sizeof(unsigned short) * 343);
  for (int k = 1; k <= 5; ++k)
    for (int j = 1; j <= 5; ++j)
      for (int i = 1; i <= 5; ++i) mult[k][j][i] = 1;
  for (int q = 0; q < cnt; ++q) {
    int s[3], e[3];
    for (int a = 0; a < 3; ++a) {
      const int ox = nb[q].ox[a];
      if (nb[q].level == lev) {
        if (ox == 0) { s[a] = 1; e[a] = 5; }
        else if (ox > 0) { s[a] = 5; e[a] = 6; }
        else { s[a] = 0; e[a] = 1; }
      } else if (nb[q].level < lev) {
        if (ox == 0) {
          s[a] = 1; e[a] = 5;
          if ((m->loc[4 * b + 1 + a] & 1) == 0) e[a] = 6;
          else s[a] = 0;
        } else if (ox > 0) { s[a] = e[a] = 6; }
        else { s[a] = e[a] = 0; }
      } else {
        if (ox == 0) {
          s[a] = 1; e[a] = 5;
          if (ml_fi(&nb[q], a) == 1) s[a] += 2;
          else e[a] -= 2;
        } else if (ox > 0) { s[a] = 5; e[a] = 6; }
        else { s[a] = 0; e[a] = 1; }
      }
    }
    for (int k = s[2]; k <= e[2]; ++k)
      for (int j = s[1]; j <= e[1]; ++j)
        for (int i = s[0]; i <= e[0]; ++i) mult[k][j][i] += 1;
  }
}

static void ml_divide(double *a, const int dims[3], int nvar, ml_ax_t x, ml_ax_t y, ml_ax_t z,
                      unsigned short mult[7][7][7]) {
  const int64_t vol = (int64_t)dims[0] * dims[1] * dims[2];
  for (int K = 0; K < 7; ++K) {
    int kl, ku;
    ml_phys(K, z, &kl, &ku);
    for (int J = 0; J < 7; ++J) {
      int jl, ju;
      ml_phys(J, y, &jl, &ju);
      for (int I = 0; I < 7; ++I) {
        const unsigned short mm = mult[K][J][I];
        if (mm <= 1) continue;
        int il, iu;
        ml_phys(I, x, &il, &iu);
        const double inv = 1.0 / (double)mm;
        for (int n = 0; n < nvar; ++n)
          for (int k = kl; k <= ku; ++k)
            for (int j = jl; j <= ju; ++j)
              for (int i = il; i <= iu; ++i) a[n * vol + ((int64_t)k * dims[1] + j) * dims[0] + i] *= inv;
      }
    }
  }
}

/* the faces of block b on a non-periodic mesh boundary */
static void ml_need(const orc_ml_mesh_t *m, int b, int need[6]) {
  const int lev = m->loc[4 * b];
  for (int a = 0; a < 3; ++a) {
    const int64_t n = (int64_t)m->nroot[a] << (lev - m->root_level);
    const int64_t l = m->loc[4 * b + 1 + a];
    need[2 * a] = m->bc[2 * a] != Z4C_BC_PERIODIC && l == 0;
    need[2 * a + 1] = m->bc[2 * a + 1] != Z4C_BC_PERIODIC && l == n - 1;
  }
}

void orc_ml_exchange(const orc_ml_mesh_t *m, int nvar, double *u_all) {
  const int nb = m->nblocks;
  int nn[3], cn[3];
  ml_ax_t F[3], C[3];
  for (int a = 0; a < 3; ++a) {
    nn[a] = m->nx[a] + 1 + 2 * NG;
    cn[a] = m->nx[a] / 2 + 1 + 2 * ORC_NCG;
    F[a] = ml_axis(m->nx[a], NG);
    C[a] = ml_axis(m->nx[a] / 2, ORC_NCG);
  }
  const int64_t fvol = (int64_t)nn[0] * nn[1] * nn[2], cvol = (int64_t)cn[0] * cn[1] * cn[2];
  double *coarse = (double *)calloc((size_t)nb * nvar * cvol, sizeof(double));
  ml_nb_t(*nbs)[56] = (ml_nb_t(*)[56])malloc(sizeof(ml_nb_t) * 56 * nb);
  int *cnt = (int *)malloc(sizeof(int) * nb);
  for (int b = 0; b < nb; ++b) cnt[b] = ml_neighbours(m, b, nbs[b]);
  /* 1. restriction of every interior */
  for (int b = 0; b < nb; ++b) {
    const int box[6] = {C[0].vs, C[0].ve, C[1].vs, C[1].ve, C[2].vs, C[2].ve};
    orc_vc_restrict(m->nx, nvar, u_all + b * nvar * fvol, coarse + b * nvar * cvol, box);
  }
  /* 2. one message per (receiver, neighbour entry), packed by the sender
   * from the entry that points back at the receiver */
  double **msg = (double **)calloc((size_t)nb * 56, sizeof(double *));
  for (int r = 0; r < nb; ++r)
    for (int q = 0; q < cnt[r]; ++q) {
      const int s = nbs[r][q].gid;
      const ml_nb_t *e = NULL;
      for (int t = 0; t < cnt[s]; ++t) {
        const ml_nb_t *c = &nbs[s][t];
        if (c->gid == r && c->ox[0] == -nbs[r][q].ox[0] && c->ox[1] == -nbs[r][q].ox[1] &&
            c->ox[2] == -nbs[r][q].ox[2]) { e = c; break; }
      }
      if (!e) { fprintf(stderr, "orc_ml_exchange: no matching neighbour entry\n"); abort(); }
      const int slev = m->loc[4 * s];
      int fb[6], cb[6];
      int64_t size = 0;
      if (e->level == slev) {
        for (int a = 0; a < 3; ++a) {
          r_load_same(e->ox[a], F[a], &fb[2 * a], &fb[2 * a + 1]);
          r_load_same(e->ox[a], C[a], &cb[2 * a], &cb[2 * a + 1]);
        }
        size = (box_count(fb) + box_count(cb)) * nvar;
      } else if (e->level < slev) {
        for (int a = 0; a < 3; ++a) r_load_to_coarser(e->ox[a], C[a], NG, &cb[2 * a], &cb[2 * a + 1]);
        size = box_count(cb) * nvar;
      } else {
        for (int a = 0; a < 3; ++a)
          r_load_to_finer(e->ox[a], F[a], ORC_NCG, ml_fi(e, a), m->nx[a] / 2 - ORC_NCG,
                          &fb[2 * a], &fb[2 * a + 1]);
        size = box_count(fb) * nvar;
      }
      double *buf = (double *)malloc(sizeof(double) * (size_t)size);
      int64_t p = 0;
      if (e->level == slev) {
        box_pack(u_all + s * nvar * fvol, nn, nvar, fb, buf, &p);
        box_pack(coarse + s * nvar * cvol, cn, nvar, cb, buf, &p);
      } else if (e->level < slev) {
        box_pack(coarse + s * nvar * cvol, cn, nvar, cb, buf, &p);
      } else {
        box_pack(u_all + s * nvar * fvol, nn, nvar, fb, buf, &p);
      }
      msg[r * 56 + q] = buf;
    }
  /* 3. unpack and multiplicity */
  for (int r = 0; r < nb; ++r) {
    double *u = u_all + r * nvar * fvol, *cu = coarse + r * nvar * cvol;
    const int lev = m->loc[4 * r];
    int same = 1;
    for (int q = 0; q < cnt[r]; ++q) same = same && nbs[r][q].level == lev;
    ml_zero_ghosts(u, nn, nvar, F[0], F[1], F[2]);
    ml_zero_ghosts(cu, cn, nvar, C[0], C[1], C[2]);
    for (int q = 0; q < cnt[r]; ++q) {
      const ml_nb_t *e = &nbs[r][q];
      const double *buf = msg[r * 56 + q];
      int64_t p = 0;
      int fb[6], cb[6];
      if (e->level == lev) {
        for (int a = 0; a < 3; ++a) {
          r_set_same(e->ox[a], F[a], &fb[2 * a], &fb[2 * a + 1]);
          r_set_same(e->ox[a], C[a], &cb[2 * a], &cb[2 * a + 1]);
        }
        box_unpack(u, nn, nvar, fb, buf, &p, 1);
        if (!same) box_unpack(cu, cn, nvar, cb, buf, &p, 1);
      } else if (e->level < lev) {
        for (int a = 0; a < 3; ++a)
          r_set_from_coarser(e->ox[a], C[a], m->loc[4 * r + 1 + a], &cb[2 * a], &cb[2 * a + 1]);
        box_unpack(cu, cn, nvar, cb, buf, &p, 0);
      } else {
        for (int a = 0; a < 3; ++a)
          r_set_from_finer(e->ox[a], F[a], ml_fi(e, a), m->nx[a] / 2, &fb[2 * a], &fb[2 * a + 1]);
        box_unpack(u, nn, nvar, fb, buf, &p, 1);
      }
    }
    unsigned short mult[7][7][7];
    ml_multiplicity(m, r, nbs[r], cnt[r], mult);
    ml_divide(u, nn, nvar, F[0], F[1], F[2], mult);
    ml_divide(cu, cn, nvar, C[0], C[1], C[2], mult);
  }
  for (int q = 0; q < nb * 56; ++q) free(msg[q]);
  free(msg);
  /* 4. coarse-level BCs, prolongation from coarser neighbours; 5. fine BCs */
  for (int b = 0; b < nb; ++b) {
    double *u = u_all + b * nvar * fvol, *cu = coarse + b * nvar * cvol;
    int need[6];
    ml_need(m, b, need);
    const int cis[3] = {C[0].vs, C[1].vs, C[2].vs}, cie[3] = {C[0].ve, C[1].ve, C[2].ve};
    ml_bcs(need, cis, cie, ORC_NCG, cn, nvar, cu);
    const int lev = m->loc[4 * b];
    const int pcng = NG / 2 + (NG % 2 != 0);
    for (int q = 0; q < cnt[b]; ++q) {
      const ml_nb_t *e = &nbs[b][q];
      if (e->level >= lev) continue;
      int box[6];
      for (int a = 0; a < 3; ++a) {
        const int ox = e->ox[a];
        int s, t;
        if (ox > 0) { s = C[a].ve + 1; t = C[a].ve + pcng; }
        else if (ox < 0) { s = C[a].vs - pcng; t = C[a].vs - 1; }
        else {
          s = C[a].vs; t = C[a].ve;
          if ((m->loc[4 * b + 1 + a] & 1) == 0) t += pcng;
          else s -= pcng;
        }
        box[2 * a] = s;
        box[2 * a + 1] = t;
      }
      orc_vc_prolongate(m->nx, nvar, cu, u, box);
    }
    const int is[3] = {NG, NG, NG}, ie[3] = {NG + m->nx[0] - 1, NG + m->nx[1] - 1, NG + m->nx[2] - 1};
    ml_bcs(need, is, ie, NG, nn, nvar, u);
  }
  free(coarse);
  free(nbs);
  free(cnt);
}

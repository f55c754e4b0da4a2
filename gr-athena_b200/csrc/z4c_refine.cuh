// Vertex-centred refinement helpers shared by the refinement operators and
// the multilevel ghost exchange: the coarse-array geometry of one
// prolongation or restriction box and the per-vertex prolongation of
// MeshRefinement::ProlongateVertexCenteredValues
// (mesh/mesh_refinement_vc.cpp:283-775, 3-D branch with the
// DBG_SYMMETRIZE_P_OP / DBG_SYMMETRIZE_CHEAP corner sums of
// defs.hpp.in:17-20), in the reference's accumulation order.
#pragma once

#include "../../include/z4c_b200.h"
#include "z4c_common.cuh"

namespace z4c {
int set_error(int code, const char* msg);

namespace refine {

constexpr int NCG = Z4C_NCG;        // coarse ghost vertices (NCGHOST)
constexpr int HSZ = 3;              // H_SZ = (2 NCGHOST - NGHOST)/2 + 1
constexpr int HNC = (2 * NCG - NG) / 2;  // H_NCGHOST

// InterpolateLagrangeUniform<3>::coeff (utils/interp_univariate_stencils.tpp:99-101)
__device__ __forceinline__ double lag3(int q) {
  return q == 0 ? 3. / 256. : (q == 1 ? -25. / 256. : 75. / 128.);
}

struct RefGeom {
  int nn[3], cn[3];
  int64_t fvol, cvol;
  int box[6];           // coarse box {si, ei, sj, ej, sk, ek}
  int sp[3], ep[3];     // interpolation ranges [s_prl, e_prl) per axis
  int f0[3], fe[3];     // fine index range touched per axis
  int nvar;
};

// The value ProlongateVertexCenteredValues writes at fine vertex f from the
// coarse array C of one variable; false where it writes none.
__device__ __forceinline__ bool prolong_value(const RefGeom& G, const double* __restrict__ C,
                                              const int f[3], double& out) {
  // per axis: injected (even fine index, coarse c = f/2 + HNC, s <= c <= e)
  // or interpolated (odd, c = (f-1)/2 + HNC, s_prl <= c < e_prl)
  int c[3];
  bool prl[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    prl[a] = (f[a] & 1) != 0;
    c[a] = (prl[a] ? (f[a] - 1) : f[a]) / 2 + HNC;
    const bool ok = prl[a] ? (c[a] >= G.sp[a] && c[a] < G.ep[a])
                           : (c[a] >= G.box[2 * a] && c[a] <= G.box[2 * a + 1]);
    if (!ok) return false;  // the reference writes no such vertex
  }
  auto co = [&](int k, int j, int i) -> double {
    return __ldg(C + ((int64_t)k * G.cn[1] + j) * G.cn[0] + i);
  };
  const int i = c[0], j = c[1], k = c[2];
  double v = 0.;
  if (prl[2] && prl[1] && prl[0]) {  // (prl, prl, prl)
    for (int dk = 0; dk < HSZ; ++dk) {
      const int ku = k + dk + 1, kl = k - dk;
      const double lck = lag3(HSZ - dk - 1);
      for (int dj = 0; dj < HSZ; ++dj) {
        const int ju = j + dj + 1, jl = j - dj;
        const double lckj = lck * lag3(HSZ - dj - 1);
        for (int di = 0; di < HSZ; ++di) {
          const int iu = i + di + 1, il = i - di;
          const double lckji = lckj * lag3(HSZ - di - 1);
          // FloatingPoint::sum_corners (utils/floating_point.hpp:50-55)
          v += lckji * (((co(ku, ju, iu) + co(kl, jl, il)) + (co(ku, ju, il) + co(kl, jl, iu))) +
                        ((co(kl, ju, il) + co(ku, jl, iu)) + (co(kl, ju, iu) + co(ku, jl, il))));
        }
      }
    }
  } else if (!prl[2] && prl[1] && prl[0]) {  // (inj, prl, prl)
    for (int dj = 0; dj < HSZ; ++dj) {
      const int ju = j + dj + 1, jl = j - dj;
      const double lcj = lag3(HSZ - dj - 1);
      for (int di = 0; di < HSZ; ++di) {
        const int iu = i + di + 1, il = i - di;
        const double lcji = lcj * lag3(HSZ - di - 1);
        v += lcji * ((co(k, ju, iu) + co(k, jl, il)) + (co(k, jl, iu) + co(k, ju, il)));
      }
    }
  } else if (prl[2] && !prl[1] && prl[0]) {  // (prl, inj, prl)
    for (int dk = 0; dk < HSZ; ++dk) {
      const int ku = k + dk + 1, kl = k - dk;
      const double lck = lag3(HSZ - dk - 1);
      for (int di = 0; di < HSZ; ++di) {
        const int iu = i + di + 1, il = i - di;
        const double lcki = lck * lag3(HSZ - di - 1);
        v += lcki * ((co(kl, j, iu) + co(ku, j, il)) + (co(ku, j, iu) + co(kl, j, il)));
      }
    }
  } else if (prl[2] && prl[1] && !prl[0]) {  // (prl, prl, inj)
    for (int dk = 0; dk < HSZ; ++dk) {
      const int ku = k + dk + 1, kl = k - dk;
      const double lck = lag3(HSZ - dk - 1);
      for (int dj = 0; dj < HSZ; ++dj) {
        const int ju = j + dj + 1, jl = j - dj;
        const double lckj = lck * lag3(HSZ - dj - 1);
        v += lckj * ((co(ku, ju, i) + co(kl, jl, i)) + (co(kl, ju, i) + co(ku, jl, i)));
      }
    }
  } else if (!prl[2] && !prl[1] && prl[0]) {  // (inj, inj, prl)
    for (int di = 0; di < HSZ; ++di) v += lag3(HSZ - di - 1) * (co(k, j, i - di) + co(k, j, i + di + 1));
  } else if (!prl[2] && prl[1] && !prl[0]) {  // (inj, prl, inj)
    for (int dj = 0; dj < HSZ; ++dj) v += lag3(HSZ - dj - 1) * (co(k, j - dj, i) + co(k, j + dj + 1, i));
  } else if (prl[2] && !prl[1] && !prl[0]) {  // (prl, inj, inj)
    for (int dk = 0; dk < HSZ; ++dk) v += lag3(HSZ - dk - 1) * (co(k - dk, j, i) + co(k + dk + 1, j, i));
  } else {  // (inj, inj, inj)
    v = co(k, j, i);
  }
  out = v;
  return true;
}

// Transpose of prolong_value: Cb (the coarse array's adjoint, one variable)
// += the weight of every coarse value in the interpolation of fine vertex f
// times a (f's adjoint).  Atomic adds: fine vertices of one box share coarse
// values.  Returns false where prolong_value writes nothing.
__device__ __forceinline__ bool prolong_adj(const RefGeom& G, double* __restrict__ Cb,
                                            const int f[3], double a) {
  int c[3];
  bool prl[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    prl[ax] = (f[ax] & 1) != 0;
    c[ax] = (prl[ax] ? (f[ax] - 1) : f[ax]) / 2 + HNC;
    const bool ok = prl[ax] ? (c[ax] >= G.sp[ax] && c[ax] < G.ep[ax])
                            : (c[ax] >= G.box[2 * ax] && c[ax] <= G.box[2 * ax + 1]);
    if (!ok) return false;
  }
  auto add = [&](int k, int j, int i, double w) {
    atomicAdd(Cb + ((int64_t)k * G.cn[1] + j) * G.cn[0] + i, w);
  };
  // per axis the taps (index, weight): the vertex itself where injected, the
  // 2 HSZ symmetric Lagrange taps where interpolated
  int idx[3][2 * HSZ];
  double wt[3][2 * HSZ];
  int nt[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    if (!prl[ax]) {
      idx[ax][0] = c[ax];
      wt[ax][0] = 1.0;
      nt[ax] = 1;
    } else {
      for (int d = 0; d < HSZ; ++d) {
        idx[ax][2 * d] = c[ax] - d;
        idx[ax][2 * d + 1] = c[ax] + d + 1;
        wt[ax][2 * d] = wt[ax][2 * d + 1] = lag3(HSZ - d - 1);
      }
      nt[ax] = 2 * HSZ;
    }
  }
  for (int tk = 0; tk < nt[2]; ++tk)
    for (int tj = 0; tj < nt[1]; ++tj)
      for (int ti = 0; ti < nt[0]; ++ti)
        add(idx[2][tk], idx[1][tj], idx[0][ti], a * (wt[2][tk] * wt[1][tj] * wt[0][ti]));
  return true;
}

inline int setup(const int nx[3], int nvar, int nblocks, const int box[6], RefGeom& G, bool prolong) {
  if (!nx || !box) return set_error(Z4C_EINVAL, "refinement operator: null argument");
  if (nvar < 1 || nblocks < 1) return set_error(Z4C_EINVAL, "refinement operator: empty input");
  for (int a = 0; a < 3; ++a) {
    if (nx[a] < 2 * NG || nx[a] % 2)
      return set_error(Z4C_EINVAL, "refinement operator: nx must be even and >= 2*ng");
    G.nn[a] = nx[a] + 1 + 2 * NG;
    G.cn[a] = nx[a] / 2 + 1 + 2 * NCG;
  }
  G.fvol = (int64_t)G.nn[0] * G.nn[1] * G.nn[2];
  G.cvol = (int64_t)G.cn[0] * G.cn[1] * G.cn[2];
  G.nvar = nvar;
  for (int q = 0; q < 6; ++q) G.box[q] = box[q];
  for (int a = 0; a < 3; ++a) {
    const int s = box[2 * a], e = box[2 * a + 1];
    if (s > e) return set_error(Z4C_EINVAL, "refinement operator: empty box");
    const int mp = NCG + nx[a] / 4;  // coarse mid-point (MeshBlock::SetIndicialParameters)
    G.sp[a] = (s > mp) ? s - 1 : s;  // :351-356
    G.ep[a] = (e < mp) ? e + 1 : e;
    // every coarse read and fine write must stay inside the arrays
    int clo = s, chi = e, flo = 2 * (s - HNC), fhi = 2 * (e - HNC);
    if (prolong && G.sp[a] < G.ep[a]) {
      clo = G.sp[a] - (HSZ - 1) < clo ? G.sp[a] - (HSZ - 1) : clo;
      chi = G.ep[a] - 1 + HSZ > chi ? G.ep[a] - 1 + HSZ : chi;
      flo = 2 * (G.sp[a] - HNC) + 1 < flo ? 2 * (G.sp[a] - HNC) + 1 : flo;
      fhi = 2 * (G.ep[a] - 1 - HNC) + 1 > fhi ? 2 * (G.ep[a] - 1 - HNC) + 1 : fhi;
    }
    if (!prolong) {
      flo = 2 * (s - NCG) + NG;
      fhi = 2 * (e - NCG) + NG;
    }
    if (clo < 0 || chi >= G.cn[a] || flo < 0 || fhi >= G.nn[a])
      return set_error(Z4C_EINVAL, "refinement operator: box reaches outside the arrays");
    G.f0[a] = flo;
    G.fe[a] = fhi;
  }
  return Z4C_OK;
}


}  // namespace refine
}  // namespace z4c

// Vertex-centred refinement operators of GR-Athena++ for MeshBlocks resident
// in device memory: MeshRefinement::RestrictVertexCenteredValues (injection)
// and MeshRefinement::ProlongateVertexCenteredValues (injection at coincident
// vertices, tensor-product 6-point Lagrange interpolation elsewhere),
// mesh/mesh_refinement_vc.cpp:56-134 and :283-775 (3-D branch, with the
// DBG_SYMMETRIZE_P_OP / DBG_SYMMETRIZE_CHEAP corner sums of
// defs.hpp.in:17-20).  Each output vertex is one thread and keeps the
// reference's accumulation order, so results agree bit for bit.
//
// Fine arrays: [block][nvar][nn3][nn2][nn1], nn = nx + 1 + 2*NG.
// Coarse arrays: [block][nvar][cn3][cn2][cn1], cn = nx/2 + 1 + 2*NCG.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/z4c_b200.h"
#include "z4c_common.cuh"
#include "z4c_kernels.cuh"

namespace z4c {
int set_error(int code, const char* msg);
}

using namespace z4c;

namespace {

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

__global__ void k_vc_restrict(RefGeom G, const double* __restrict__ fine,
                              double* __restrict__ coarse, int nblk) {
  const int e0 = G.box[1] - G.box[0] + 1, e1 = G.box[3] - G.box[2] + 1,
            e2 = G.box[5] - G.box[4] + 1;
  const int64_t per = (int64_t)e0 * e1 * e2;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per * G.nvar * nblk) return;
  const int64_t r = t % per, bn = t / per;  // bn = block * nvar + n
  const int ci = G.box[0] + (int)(r % e0), cj = G.box[2] + (int)((r / e0) % e1),
            ck = G.box[4] + (int)(r / ((int64_t)e0 * e1));
  // RestrictVertexCenteredIndicialHelper (:24-46): fine index 2 (c - cvs) + vs
  const int i = 2 * (ci - NCG) + NG, j = 2 * (cj - NCG) + NG, k = 2 * (ck - NCG) + NG;
  coarse[bn * G.cvol + ((int64_t)ck * G.cn[1] + cj) * G.cn[0] + ci] =
      __ldg(fine + bn * G.fvol + ((int64_t)k * G.nn[1] + j) * G.nn[0] + i);
}

__global__ void k_vc_prolongate(RefGeom G, const double* __restrict__ coarse,
                                double* __restrict__ fine, int nblk) {
  const int e0 = G.fe[0] - G.f0[0] + 1, e1 = G.fe[1] - G.f0[1] + 1, e2 = G.fe[2] - G.f0[2] + 1;
  const int64_t per = (int64_t)e0 * e1 * e2;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per * G.nvar * nblk) return;
  const int64_t r = t % per, bn = t / per;
  const int f[3] = {G.f0[0] + (int)(r % e0), G.f0[1] + (int)((r / e0) % e1),
                    G.f0[2] + (int)(r / ((int64_t)e0 * e1))};
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
    if (!ok) return;  // the reference writes no such vertex
  }
  const double* C = coarse + bn * G.cvol;
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
  fine[bn * G.fvol + ((int64_t)f[2] * G.nn[1] + f[1]) * G.nn[0] + f[0]] = v;
}

int setup(const int nx[3], int nvar, int nblocks, const int box[6], RefGeom& G, bool prolong) {
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

// Regrid transfer copies between a MeshBlock and the coarse buffer, one
// thread per (variable, coarse vertex) of the box lo..hi (inclusive):
// to_coarse: coarse(c) = fine(f0 + c - lo); otherwise fine(f0 + c - lo) = coarse(c).
__global__ void k_regrid_copy(int nvar, int3 nn, int3 cn, int3 lo, int3 hi, int3 f0,
                              const double* __restrict__ src, double* __restrict__ dst,
                              int to_coarse) {
  const int ex = hi.x - lo.x + 1, ey = hi.y - lo.y + 1, ez = hi.z - lo.z + 1;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)ex * ey * ez * nvar) return;
  const int i = (int)(t % ex), j = (int)((t / ex) % ey), k = (int)((t / ((int64_t)ex * ey)) % ez);
  const int n = (int)(t / ((int64_t)ex * ey * ez));
  const int64_t fv = (int64_t)nn.x * nn.y * nn.z, cv = (int64_t)cn.x * cn.y * cn.z;
  const int64_t c = n * cv + ((int64_t)(lo.z + k) * cn.y + (lo.y + j)) * cn.x + (lo.x + i);
  const int64_t f = n * fv + ((int64_t)(f0.z + k) * nn.y + (f0.y + j)) * nn.x + (f0.x + i);
  if (to_coarse) dst[c] = src[f];
  else dst[f] = src[c];
}

int launched(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return Z4C_OK;
  char buf[160];
  snprintf(buf, sizeof(buf), "%s launch: %s", what, cudaGetErrorString(e));
  return set_error(Z4C_ECUDA, buf);
}

}  // namespace

extern "C" int z4c_vc_restrict(const double* fine, double* coarse, int nblocks, int nvar,
                               const int nx[3], const int box[6], void* stream) {
  if (!fine || !coarse) return set_error(Z4C_EINVAL, "z4c_vc_restrict: null array");
  RefGeom G;
  int rc = setup(nx, nvar, nblocks, box, G, false);
  if (rc) return rc;
  const int64_t n = (int64_t)(box[1] - box[0] + 1) * (box[3] - box[2] + 1) *
                    (box[5] - box[4] + 1) * nvar * nblocks;
  k_vc_restrict<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      G, fine, coarse, nblocks);
  add_kernel_launches(1);
  return launched("z4c_vc_restrict");
}

extern "C" int z4c_vc_prolongate(const double* coarse, double* fine, int nblocks, int nvar,
                                 const int nx[3], const int box[6], void* stream) {
  if (!fine || !coarse) return set_error(Z4C_EINVAL, "z4c_vc_prolongate: null array");
  RefGeom G;
  int rc = setup(nx, nvar, nblocks, box, G, true);
  if (rc) return rc;
  const int64_t n = (int64_t)(G.fe[0] - G.f0[0] + 1) * (G.fe[1] - G.f0[1] + 1) *
                    (G.fe[2] - G.f0[2] + 1) * nvar * nblocks;
  k_vc_prolongate<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      G, coarse, fine, nblocks);
  add_kernel_launches(1);
  return launched("z4c_vc_prolongate");
}

namespace {

int regrid_geom(const int nx[3], int nvar, const int oct[3], int3* nn, int3* cn) {
  if (!nx || !oct) return set_error(Z4C_EINVAL, "regrid transfer: null argument");
  if (nvar < 1) return set_error(Z4C_EINVAL, "regrid transfer: nvar < 1");
  for (int a = 0; a < 3; ++a) {
    if (nx[a] < 2 * NG || nx[a] % 2)
      return set_error(Z4C_EINVAL, "regrid transfer: nx must be even and >= 2*ng");
    if (oct[a] != 0 && oct[a] != 1) return set_error(Z4C_EINVAL, "regrid transfer: octant is 0 or 1 per axis");
  }
  *nn = make_int3(nx[0] + 1 + 2 * NG, nx[1] + 1 + 2 * NG, nx[2] + 1 + 2 * NG);
  *cn = make_int3(nx[0] / 2 + 1 + 2 * NCG, nx[1] / 2 + 1 + 2 * NCG, nx[2] / 2 + 1 + 2 * NCG);
  return Z4C_OK;
}

}  // namespace

// AMRRegistry::FillSameRankCoarseToFine (comm/amr_registry.cpp:1015-1233),
// vertex-centred branch: the parent's vertices around the child octant, NCG
// coarse ghosts included, into the coarse buffer, then the prolongation over
// the child's interior vertices.
extern "C" int z4c_regrid_refine(const double* parent, double* child, double* coarse, int nvar,
                                 const int nx[3], const int oct[3], void* stream) {
  if (!parent || !child || !coarse) return set_error(Z4C_EINVAL, "z4c_regrid_refine: null array");
  int3 nn, cn;
  int rc = regrid_geom(nx, nvar, oct, &nn, &cn);
  if (rc) return rc;
  constexpr int ndg = NCG < NG ? NCG : NG;
  const int3 lo = make_int3(NCG - ndg, NCG - ndg, NCG - ndg);
  const int3 hi = make_int3(NCG + nx[0] / 2 + ndg, NCG + nx[1] / 2 + ndg, NCG + nx[2] / 2 + ndg);
  const int3 f0 = make_int3(oct[0] * (nx[0] / 2) + NG - ndg, oct[1] * (nx[1] / 2) + NG - ndg,
                            oct[2] * (nx[2] / 2) + NG - ndg);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = (int64_t)(hi.x - lo.x + 1) * (hi.y - lo.y + 1) * (hi.z - lo.z + 1) * nvar;
  k_regrid_copy<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nvar, nn, cn, lo, hi, f0, parent,
                                                             coarse, 1);
  add_kernel_launches(1);
  if ((rc = launched("z4c_regrid_refine"))) return rc;
  const int box[6] = {NCG, NCG + nx[0] / 2, NCG, NCG + nx[1] / 2, NCG, NCG + nx[2] / 2};
  return z4c_vc_prolongate(coarse, child, 1, nvar, nx, box, stream);
}

// AMRRegistry::FillSameRankFineToCoarse (:814-1012), vertex-centred branch:
// the child's interior restricted (injection) into the coarse buffer, then
// copied into the parent's octant.
extern "C" int z4c_regrid_derefine(const double* child, double* parent, double* coarse, int nvar,
                                   const int nx[3], const int oct[3], void* stream) {
  if (!parent || !child || !coarse) return set_error(Z4C_EINVAL, "z4c_regrid_derefine: null array");
  int3 nn, cn;
  int rc = regrid_geom(nx, nvar, oct, &nn, &cn);
  if (rc) return rc;
  const int box[6] = {NCG, NCG + nx[0] / 2, NCG, NCG + nx[1] / 2, NCG, NCG + nx[2] / 2};
  if ((rc = z4c_vc_restrict(child, coarse, 1, nvar, nx, box, stream))) return rc;
  const int3 lo = make_int3(box[0], box[2], box[4]), hi = make_int3(box[1], box[3], box[5]);
  const int3 f0 = make_int3(NG + oct[0] * (nx[0] / 2), NG + oct[1] * (nx[1] / 2),
                            NG + oct[2] * (nx[2] / 2));
  const int64_t n = (int64_t)(hi.x - lo.x + 1) * (hi.y - lo.y + 1) * (hi.z - lo.z + 1) * nvar;
  k_regrid_copy<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      nvar, nn, cn, lo, hi, f0, coarse, parent, 0);
  add_kernel_launches(1);
  return launched("z4c_regrid_derefine");
}

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
#include "z4c_refine.cuh"

using namespace z4c;
using namespace z4c::refine;

namespace {

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
  double v;
  if (prolong_value(G, coarse + bn * G.cvol, f, v))
    fine[bn * G.fvol + ((int64_t)f[2] * G.nn[1] + f[1]) * G.nn[0] + f[0]] = v;
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

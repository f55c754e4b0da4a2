// Vertex-centred ghost exchange of a statically refined mesh (several
// refinement levels), as the reference runs one ghost fill of the Z4c state
// (task order of task_list/gr/task_list_gr_z4c.cpp:52-64, SEND / RECV / SETB
// / PROLONG / PHY_BVAL):
//   restrict   every block injects its interior into its coarse buffer
//              (CommRegistry::SendBoundaryBuffers, comm_registry.cpp:246-296;
//              RestrictInterior, refinement_ops.cpp:167-195)
//   unpack     per receiving block, in neighbour order, straight from the
//              senders' pre-exchange arrays (the message each would pack,
//              CommChannel::PackAndSend, comm_channel.cpp:733-787; ranges
//              index_utilities.hpp:124-216): the fine and coarse ghosts
//              start at zero and the interiors at the block's own values; same-level
//              data is added into the fine array and its coarse payload into
//              the coarse buffer, data from a coarser block overwrites the
//              coarse buffer, data from a finer block is added into the fine
//              array; then both arrays are multiplied by the inverse node
//              multiplicity (comm_registry.cpp:336-382,
//              comm_channel.cpp:1278-1474, node_multiplicity.cpp:102-430)
//   coarse BC  extrapolation on the coarse buffer's physical faces
//              (physical_bcs.cpp:687-890)
//   prolong    the ghosts next to each coarser neighbour from the coarse
//              buffer (refinement_ops.cpp:24-160)
//   fine BC    extrapolation on the fine array's physical faces
//              (physical_bcs.cpp:506-670)
// The host builds the op lists once (neighbour search of
// mesh/mesh_topology.cpp:278-960 over the blocks' logical locations); each
// receiving block replays its ops in the reference's order, so every vertex
// sees the same additions in the same order and the result agrees bit for
// bit.  Fine arrays [block][var][nn3][nn2][nn1], coarse buffers
// [block][var][cn3][cn2][cn1] with cn = nx/2 + 1 + 2 NCG.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <tuple>
#include <vector>

#include "../../include/z4c_b200.h"
#include "z4c_kernels.cuh"
#include "z4c_multilevel.cuh"

namespace z4c {

using refine::RefGeom;
constexpr int kMlNcg = Z4C_NCG;
constexpr int kMlUnpackThreads = 512;

namespace {

// ---- kernels ---------------------------------------------------------------

// RestrictVertexCenteredValues over the coarse interior [cvs, cve]^3.
__global__ void k_ml_restrict(MlPlan P, const double* __restrict__ src, double* __restrict__ csrc,
                              int nvar, int reg_nvar) {
  const int c0 = P.nx[0] / 2 + 1, c1 = P.nx[1] / 2 + 1, c2 = P.nx[2] / 2 + 1;
  const int64_t per = (int64_t)c0 * c1 * c2;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per * nvar * P.nblocks) return;
  const int64_t r = t % per;
  const int n = (int)((t / per) % nvar), b = (int)(t / (per * nvar));
  const int ci = kMlNcg + (int)(r % c0), cj = kMlNcg + (int)((r / c0) % c1),
            ck = kMlNcg + (int)(r / ((int64_t)c0 * c1));
  const int i = 2 * (ci - kMlNcg) + NG, j = 2 * (cj - kMlNcg) + NG, k = 2 * (ck - kMlNcg) + NG;
  csrc[((int64_t)b * Z4C_NVAR + n) * P.cvol + ((int64_t)ck * P.cn[1] + cj) * P.cn[0] + ci] =
      __ldg(src + ((int64_t)b * reg_nvar + n) * P.fvol + ((int64_t)k * P.nn[1] + j) * P.nn[0] + i);
}

// compact zone (0..6) of index i along one axis: ghosts, the shared vertex,
// the lower half, the midpoint, the upper half, the shared vertex, ghosts
// (NodeMultiplicity::ApplyDivisionImpl's PhysRange, node_multiplicity.cpp:364-430)
__device__ __forceinline__ int ml_zone(int i, int vs, int ve) {
  const int mid = vs + (ve - vs) / 2;
  return i < vs ? 0 : i == vs ? 1 : i < mid ? 2 : i == mid ? 3 : i < ve ? 4 : i == ve ? 5 : 6;
}

// SetBoundaries of one receiving block as a gather, every variable at once:
// each vertex starts at the block's own value (interior) or zero (ghosts),
// takes its zone's contributions in the reference's neighbour order (add, or
// copy for data from a coarser block) and is multiplied by the inverse node
// multiplicity of the zone; blockIdx.y selects the fine array (0) or the
// coarse buffer (1).  The vertex's zone, multiplicity and contribution range
// are found once and serve all nvar variables, whose loads are independent
// of one another; the threads of a warp take consecutive vertices.
__global__ void __launch_bounds__(kMlUnpackThreads)
k_ml_unpack(MlPlan P, const double* __restrict__ src, double* __restrict__ dst, int nvar,
            int reg_nvar) {
  const int b = blockIdx.x, arr = blockIdx.y;  // arr: 0 fine, 1 coarse
  // a coarse buffer that no prolongation reads is not filled
  if (arr == 1 && !P.coarser[b]) return;
  __shared__ unsigned char mult[343];
  __shared__ int zs[344];
  extern __shared__ MlContrib sc[];  // this array's contributions
  for (int q = threadIdx.x; q < 343; q += blockDim.x) mult[q] = P.mult[(int64_t)b * 343 + q];
  for (int q = threadIdx.x; q < 344; q += blockDim.x)
    zs[q] = P.zstart[((int64_t)b * 2 + arr) * 344 + q];
  __syncthreads();
  const int c0 = zs[0], nc = zs[343] - c0;
  for (int q = threadIdx.x; q < nc; q += blockDim.x) sc[q] = P.contrib[c0 + q];
  __syncthreads();
  const int ng = arr ? Z4C_NCG : NG;
  const int d0 = arr ? P.cn[0] : P.nn[0], d1 = arr ? P.cn[1] : P.nn[1];
  const int v0 = ng + (arr ? P.nx[0] / 2 : P.nx[0]), v1 = ng + (arr ? P.nx[1] / 2 : P.nx[1]),
            v2 = ng + (arr ? P.nx[2] / 2 : P.nx[2]);
  const int64_t vol = arr ? P.cvol : P.fvol;
  // variable stride of the arrays read and written
  const int64_t vs = vol;
  const double* own = arr ? P.csrc + (int64_t)b * Z4C_NVAR * vol : src + (int64_t)b * reg_nvar * vol;
  double* out = arr ? P.coarse + (int64_t)b * Z4C_NVAR * vol : dst + (int64_t)b * reg_nvar * vol;
  for (int p = threadIdx.x; p < vol; p += blockDim.x) {
    const int i = p % d0, row = p / d0, j = row % d1, k = row / d1;
    const int zi = ml_zone(i, ng, v0), zj = ml_zone(j, ng, v1), zk = ml_zone(k, ng, v2);
    const int z = (zk * 7 + zj) * 7 + zi;
    const bool in = zi >= 1 && zi <= 5 && zj >= 1 && zj <= 5 && zk >= 1 && zk <= 5;
    const int qb = zs[z] - c0, qe = zs[z + 1] - c0;
    const int m = mult[z];
    const double inv = m > 1 ? P.inv[m] : 1.0;
#pragma unroll 2
    for (int n = 0; n < nvar; ++n) {
      double v = in ? __ldg(own + n * vs + p) : 0.0;
      for (int q = qb; q < qe; ++q) {
        const MlContrib c = sc[q];
        const int64_t sv = c.scoarse ? P.cvol : P.fvol;
        const double* s = c.scoarse ? P.csrc + ((int64_t)c.sblk * Z4C_NVAR + n) * sv
                                    : src + ((int64_t)c.sblk * reg_nvar + n) * sv;
        const int s0 = c.scoarse ? P.cn[0] : P.nn[0], s1 = c.scoarse ? P.cn[1] : P.nn[1];
        const double x = __ldg(s + ((k + c.d[2]) * s1 + j + c.d[1]) * s0 + i + c.d[0]);
        v = c.mode == kMlCopy ? x : v + x;
      }
      if (m > 1) v *= inv;
      out[n * vs + p] = v;
    }
  }
}

// ExtrapolateOutflowBC with NEXTRAPOLATE = 5 (physical_bcs.cpp:187-260),
// InterpolateLagrangeUniformBiasR<5> weights; one CTA per (face, variable),
// a thread per transverse vertex walking its ghosts outwards.
template <int AX>
__global__ void k_ml_bc(const MlBc* __restrict__ items, double* __restrict__ arr, int64_t bstride,
                        int64_t vol, int d0, int d1, int ng) {
  const MlBc it = items[blockIdx.x];
  const int n = blockIdx.y;
  constexpr int o1 = AX == 0 ? 1 : 0, o2 = AX == 2 ? 1 : 2;
  const int64_t st[3] = {1, d0, (int64_t)d0 * d1};
  const int w1 = it.hi[o1] - it.lo[o1] + 1, w2 = it.hi[o2] - it.lo[o2] + 1;
  double* a = arr + (int64_t)it.blk * bstride + (int64_t)n * vol;
  const int dir = it.outer ? -1 : 1;
  for (int t = threadIdx.x; t < w1 * w2; t += blockDim.x) {
    const int t1 = it.lo[o1] + t % w1, t2 = it.lo[o2] + t / w1;
    for (int g = 1; g <= ng; ++g) {
      const int ia = it.outer ? it.hi[AX] + g : it.lo[AX] - g;
      const int64_t p = (int64_t)ia * st[AX] + (int64_t)t1 * st[o1] + (int64_t)t2 * st[o2];
      const int64_t s = dir * st[AX];
      double v = 0.0;
      v += 5. * a[p + s];
      v += -10. * a[p + 2 * s];
      v += 10. * a[p + 3 * s];
      v += -5. * a[p + 4 * s];
      v += 1. * a[p + 5 * s];
      a[p] = v;
    }
  }
}

// ProlongateVertexCenteredValues over one coarse box per CTA row.  The fine
// vertices are taken one parity class (injected or interpolated along each
// axis) at a time, so the threads of a warp run the same interpolation.
__global__ void k_ml_prolong(MlPlan P, double* __restrict__ dst, int reg_nvar) {
  const RefGeom G = P.pro[blockIdx.x];
  const int b = P.pro_blk[blockIdx.x], n = blockIdx.y;
  const double* C = P.coarse + ((int64_t)b * Z4C_NVAR + n) * P.cvol;
  double* F = dst + ((int64_t)b * reg_nvar + n) * P.fvol;
  constexpr int hnc = refine::HNC;
  for (int cls = 0; cls < 8; ++cls) {
    int lo[3], cnt[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      int l, h;
      if ((cls >> a) & 1) {  // interpolated: odd fine index, coarse sp..ep-1
        l = 2 * (G.sp[a] - hnc) + 1;
        h = 2 * (G.ep[a] - 1 - hnc) + 1;
      } else {  // injected: even fine index, coarse box
        l = 2 * (G.box[2 * a] - hnc);
        h = 2 * (G.box[2 * a + 1] - hnc);
      }
      lo[a] = l;
      cnt[a] = h >= l ? (h - l) / 2 + 1 : 0;
    }
    const int total = cnt[0] * cnt[1] * cnt[2];
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int f[3] = {lo[0] + 2 * (t % cnt[0]), lo[1] + 2 * ((t / cnt[0]) % cnt[1]),
                        lo[2] + 2 * (t / (cnt[0] * cnt[1]))};
      double v;
      if (refine::prolong_value(G, C, f, v))
        F[((int64_t)f[2] * G.nn[1] + f[1]) * G.nn[0] + f[0]] = v;
    }
  }
}

// ---- transpose of the ghost fill (the adjoint of a step on refined meshes) --
// The fill is linear in the blocks' interiors.  Its transpose runs the
// pieces backwards: fine BCs, prolongation, coarse BCs, unpack, restriction,
// each transposed.  Adjoint contributions from several receivers meet at one
// source value, so the unpack and the prolongation scatter with atomic adds
// (their sums are exact up to the order of the additions).

// ExtrapolateOutflowBC transposed along one column: the ghosts in reverse
// order push their adjoint to the five values each was formed from, and
// lose it (the forward overwrote them).
template <int AX>
__global__ void k_ml_bc_adj(const MlBc* __restrict__ items, double* __restrict__ arr,
                            int64_t bstride, int64_t vol, int d0, int d1, int ng) {
  const MlBc it = items[blockIdx.x];
  const int n = blockIdx.y;
  constexpr int o1 = AX == 0 ? 1 : 0, o2 = AX == 2 ? 1 : 2;
  const int64_t st[3] = {1, d0, (int64_t)d0 * d1};
  const int w1 = it.hi[o1] - it.lo[o1] + 1, w2 = it.hi[o2] - it.lo[o2] + 1;
  double* a = arr + (int64_t)it.blk * bstride + (int64_t)n * vol;
  const int dir = it.outer ? -1 : 1;
  constexpr double c[5] = {5., -10., 10., -5., 1.};
  for (int t = threadIdx.x; t < w1 * w2; t += blockDim.x) {
    const int t1 = it.lo[o1] + t % w1, t2 = it.lo[o2] + t / w1;
    for (int g = ng; g >= 1; --g) {
      const int ia = it.outer ? it.hi[AX] + g : it.lo[AX] - g;
      const int64_t p = (int64_t)ia * st[AX] + (int64_t)t1 * st[o1] + (int64_t)t2 * st[o2];
      const int64_t s = dir * st[AX];
      const double y = a[p];
      a[p] = 0.0;
#pragma unroll
      for (int q = 0; q < 5; ++q) a[p + (q + 1) * s] += c[q] * y;
    }
  }
}

// For every fine vertex a prolongation box writes, the first box (in plan
// order) of its block that writes it: the one whose transpose carries it.
__global__ void k_ml_prolong_owner(MlPlan P, int* __restrict__ owner) {
  const RefGeom G = P.pro[blockIdx.x];
  const int b = P.pro_blk[blockIdx.x];
  const int nf[3] = {G.fe[0] - G.f0[0] + 1, G.fe[1] - G.f0[1] + 1, G.fe[2] - G.f0[2] + 1};
  const int total = nf[0] * nf[1] * nf[2];
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int f[3] = {G.f0[0] + t % nf[0], G.f0[1] + (t / nf[0]) % nf[1],
                      G.f0[2] + t / (nf[0] * nf[1])};
    int c[3];
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const bool prl = (f[a] & 1) != 0;
      c[a] = (prl ? (f[a] - 1) : f[a]) / 2 + refine::HNC;
      ok &= prl ? (c[a] >= G.sp[a] && c[a] < G.ep[a])
                : (c[a] >= G.box[2 * a] && c[a] <= G.box[2 * a + 1]);
    }
    if (ok)
      atomicMin(owner + (int64_t)b * P.fvol + ((int64_t)f[2] * G.nn[1] + f[1]) * G.nn[0] + f[0],
                (int)blockIdx.x);
  }
}

// ProlongateVertexCenteredValues transposed: each fine vertex a box owns
// moves its adjoint into the coarse buffer's adjoint and loses it.
__global__ void k_ml_prolong_adj(MlPlan P, double* __restrict__ fbar, const int* __restrict__ owner,
                                 int reg_nvar) {
  const RefGeom G = P.pro[blockIdx.x];
  const int b = P.pro_blk[blockIdx.x], n = blockIdx.y;
  double* Cb = P.coarse + ((int64_t)b * Z4C_NVAR + n) * P.cvol;
  double* F = fbar + ((int64_t)b * reg_nvar + n) * P.fvol;
  const int* O = owner + (int64_t)b * P.fvol;
  const int nf[3] = {G.fe[0] - G.f0[0] + 1, G.fe[1] - G.f0[1] + 1, G.fe[2] - G.f0[2] + 1};
  const int total = nf[0] * nf[1] * nf[2];
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int f[3] = {G.f0[0] + t % nf[0], G.f0[1] + (t / nf[0]) % nf[1],
                      G.f0[2] + t / (nf[0] * nf[1])};
    const int64_t q = ((int64_t)f[2] * G.nn[1] + f[1]) * G.nn[0] + f[0];
    if (O[q] != (int)blockIdx.x) continue;
    const double a = F[q];
    if (refine::prolong_adj(G, Cb, f, a)) F[q] = 0.0;
  }
}

// The unpack transposed: the adjoint y of every receiving vertex, times 1/m,
// goes to the contributions in reverse list order until one that copied
// (everything before it was overwritten), and then to the vertex's own value
// when no copy intervened.  Sources are the fine arrays' adjoint (wbar) or
// the restricted snapshot's adjoint (P.csrc); the receiving coarse buffers'
// adjoint is P.coarse.
__global__ void __launch_bounds__(kMlUnpackThreads)
k_ml_unpack_adj(MlPlan P, const double* __restrict__ ybar, double* __restrict__ wbar, int nvar,
                int reg_nvar) {
  const int b = blockIdx.x, arr = blockIdx.y;
  __shared__ unsigned char mult[343];
  __shared__ int zs[344];
  extern __shared__ MlContrib sc[];
  for (int q = threadIdx.x; q < 343; q += blockDim.x) mult[q] = P.mult[(int64_t)b * 343 + q];
  for (int q = threadIdx.x; q < 344; q += blockDim.x)
    zs[q] = P.zstart[((int64_t)b * 2 + arr) * 344 + q];
  __syncthreads();
  const int c0 = zs[0], nc = zs[343] - c0;
  for (int q = threadIdx.x; q < nc; q += blockDim.x) sc[q] = P.contrib[c0 + q];
  __syncthreads();
  const int ng = arr ? Z4C_NCG : NG;
  const int d0 = arr ? P.cn[0] : P.nn[0], d1 = arr ? P.cn[1] : P.nn[1];
  const int v0 = ng + (arr ? P.nx[0] / 2 : P.nx[0]), v1 = ng + (arr ? P.nx[1] / 2 : P.nx[1]),
            v2 = ng + (arr ? P.nx[2] / 2 : P.nx[2]);
  const int64_t vol = arr ? P.cvol : P.fvol;
  const double* yb = arr ? P.coarse + (int64_t)b * Z4C_NVAR * vol : ybar + (int64_t)b * reg_nvar * vol;
  double* own = arr ? P.csrc + (int64_t)b * Z4C_NVAR * vol : wbar + (int64_t)b * reg_nvar * vol;
  for (int p = threadIdx.x; p < vol; p += blockDim.x) {
    const int i = p % d0, row = p / d0, j = row % d1, k = row / d1;
    const int zi = ml_zone(i, ng, v0), zj = ml_zone(j, ng, v1), zk = ml_zone(k, ng, v2);
    const int z = (zk * 7 + zj) * 7 + zi;
    const bool in = zi >= 1 && zi <= 5 && zj >= 1 && zj <= 5 && zk >= 1 && zk <= 5;
    const int qb = zs[z] - c0, qe = zs[z + 1] - c0;
    const int m = mult[z];
    const double inv = m > 1 ? P.inv[m] : 1.0;
    for (int n = 0; n < nvar; ++n) {
      double a = yb[n * vol + p];
      if (a == 0.0) continue;
      if (m > 1) a *= inv;
      bool copied = false;
      for (int q = qe - 1; q >= qb; --q) {
        const MlContrib c = sc[q];
        const int64_t sv = c.scoarse ? P.cvol : P.fvol;
        double* s = c.scoarse ? P.csrc + ((int64_t)c.sblk * Z4C_NVAR + n) * sv
                              : wbar + ((int64_t)c.sblk * reg_nvar + n) * sv;
        const int s0 = c.scoarse ? P.cn[0] : P.nn[0], s1 = c.scoarse ? P.cn[1] : P.nn[1];
        atomicAdd(s + ((k + c.d[2]) * s1 + j + c.d[1]) * s0 + i + c.d[0], a);
        if (c.mode == kMlCopy) {
          copied = true;
          break;
        }
      }
      if (!copied && in) atomicAdd(own + n * vol + p, a);
    }
  }
}

// RestrictInterior transposed: the snapshot's adjoint back onto the fine
// vertices it was injected from.
__global__ void k_ml_restrict_adj(MlPlan P, double* __restrict__ wbar, int nvar, int reg_nvar) {
  const int c0 = P.nx[0] / 2 + 1, c1 = P.nx[1] / 2 + 1, c2 = P.nx[2] / 2 + 1;
  const int64_t per = (int64_t)c0 * c1 * c2;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per * nvar * P.nblocks) return;
  const int64_t r = t % per;
  const int n = (int)((t / per) % nvar), b = (int)(t / (per * nvar));
  const int ci = kMlNcg + (int)(r % c0), cj = kMlNcg + (int)((r / c0) % c1),
            ck = kMlNcg + (int)(r / ((int64_t)c0 * c1));
  const int i = 2 * (ci - kMlNcg) + NG, j = 2 * (cj - kMlNcg) + NG, k = 2 * (ck - kMlNcg) + NG;
  wbar[((int64_t)b * reg_nvar + n) * P.fvol + ((int64_t)k * P.nn[1] + j) * P.nn[0] + i] +=
      P.csrc[((int64_t)b * Z4C_NVAR + n) * P.cvol + ((int64_t)ck * P.cn[1] + cj) * P.cn[0] + ci];
}

// ---- host plan -------------------------------------------------------------

struct Loc {
  int level;
  long long l[3];
  bool operator<(const Loc& o) const {
    return std::tie(level, l[0], l[1], l[2]) < std::tie(o.level, o.l[0], o.l[1], o.l[2]);
  }
};
struct Entry {
  int gid, level, ox[3], fi[2];
};

// Index limits of one axis of the fine array (ng = NG, n = nx) or of the
// coarse buffer (ng = NCG, n = nx/2): MeshBlock::SetIndicialParameters
// (mesh/meshblock.cpp:850-905).
struct Ax {
  int vs, ve, ms, me, ps, pe, gs, ge;
};
Ax axis_limits(int n, int ng) {
  return {ng, ng + n, 0, ng - 1, n + ng + 1, n + 2 * ng, 2 * ng, n};
}

struct Builder {
  int nroot[3], nx[3], bc[6], root_level, nb;
  const long long* locs;
  std::map<Loc, int> leaf;
  std::set<Loc> inner;  // refined nodes (ancestors of leaves)
  std::vector<std::vector<Entry>> nbrs;
  const char* err = nullptr;

  Loc loc(int b) const { return {(int)locs[4 * b], {locs[4 * b + 1], locs[4 * b + 2], locs[4 * b + 3]}}; }

  // MeshBlockTree::FindNeighbor (meshblock_tree.cpp:400-490): 0 beyond a
  // non-periodic face, 1 a leaf of the same or the next coarser level, 2 a
  // refined node (its location in nl); -1 when the 2:1 balance is broken.
  int find(const Loc& me, const int o[3], Loc& nl, int& gid) const {
    nl.level = me.level;
    for (int a = 0; a < 3; ++a) {
      const long long n = (long long)nroot[a] << (me.level - root_level);
      nl.l[a] = me.l[a] + o[a];
      if (nl.l[a] < 0) {
        if (bc[2 * a] != Z4C_BC_PERIODIC) return 0;
        nl.l[a] = n - 1;
      }
      if (nl.l[a] >= n) {
        if (bc[2 * a + 1] != Z4C_BC_PERIODIC) return 0;
        nl.l[a] = 0;
      }
    }
    auto it = leaf.find(nl);
    if (it != leaf.end()) {
      gid = it->second;
      return 1;
    }
    if (nl.level > root_level) {
      const Loc par{nl.level - 1, {nl.l[0] >> 1, nl.l[1] >> 1, nl.l[2] >> 1}};
      it = leaf.find(par);
      if (it != leaf.end()) {
        gid = it->second;
        return 1;
      }
    }
    return inner.count(nl) ? 2 : -1;
  }
  int child(const Loc& nl, const int c[3]) const {
    const Loc ch{nl.level + 1, {2 * nl.l[0] + c[0], 2 * nl.l[1] + c[1], 2 * nl.l[2] + c[2]}};
    auto it = leaf.find(ch);
    return it == leaf.end() ? -1 : it->second;
  }

  // MeshBlock::SearchAndSetNeighbors (mesh_topology.cpp:278-960), 3-D.
  bool neighbours(int b, std::vector<Entry>& out) {
    const Loc me = loc(b);
    int myox[3];
    for (int a = 0; a < 3; ++a) myox[a] = (me.l[a] & 1) ? 1 : -1;
    Loc nl;
    int gid = -1;
    auto add = [&](int g, int lev, const int o[3], int f1, int f2) -> bool {
      if (g < 0) return false;
      out.push_back({g, lev, {o[0], o[1], o[2]}, {f1, f2}});
      return true;
    };
    for (int ax = 0; ax < 3; ++ax)  // faces
      for (int s = -1; s <= 1; s += 2) {
        int o[3] = {0, 0, 0};
        o[ax] = s;
        const int r = find(me, o, nl, gid);
        if (r < 0) return false;
        if (r == 0) continue;
        if (r == 2) {
          const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
          for (int f2 = 0; f2 < 2; ++f2)
            for (int f1 = 0; f1 < 2; ++f1) {
              int c[3];
              c[ax] = 1 - (s + 1) / 2;
              c[t1] = f1;
              c[t2] = f2;
              if (!add(child(nl, c), me.level + 1, o, f1, f2)) return false;
            }
        } else {
          add(gid, (int)locs[4 * gid], o, 0, 0);
        }
      }
    static const int pairs[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
    for (int q = 0; q < 3; ++q) {  // edges x1x2, x1x3, x2x3
      const int a0 = pairs[q][0], a1 = pairs[q][1], a2 = pairs[q][2];
      for (int m = -1; m <= 1; m += 2)
        for (int n = -1; n <= 1; n += 2) {
          int o[3] = {0, 0, 0};
          o[a0] = n;
          o[a1] = m;
          const int r = find(me, o, nl, gid);
          if (r < 0) return false;
          if (r == 0) continue;
          if (r == 2) {
            for (int f1 = 0; f1 < 2; ++f1) {
              int c[3];
              c[a0] = 1 - (n + 1) / 2;
              c[a1] = 1 - (m + 1) / 2;
              c[a2] = f1;
              if (!add(child(nl, c), me.level + 1, o, f1, 0)) return false;
            }
          } else {
            const int lev = (int)locs[4 * gid];
            if (lev >= me.level || (myox[a0] == n && myox[a1] == m)) add(gid, lev, o, 0, 0);
          }
        }
    }
    for (int l = -1; l <= 1; l += 2)  // corners
      for (int m = -1; m <= 1; m += 2)
        for (int n = -1; n <= 1; n += 2) {
          const int o[3] = {n, m, l};
          const int r = find(me, o, nl, gid);
          if (r < 0) return false;
          if (r == 0) continue;
          int lev;
          if (r == 2) {
            const int c[3] = {1 - (n + 1) / 2, 1 - (m + 1) / 2, 1 - (l + 1) / 2};
            gid = child(nl, c);
            if (gid < 0) return false;
            lev = me.level + 1;
          } else {
            lev = (int)locs[4 * gid];
          }
          if (lev >= me.level || (myox[0] == n && myox[1] == m && myox[2] == l))
            add(gid, lev, o, 0, 0);
        }
    return true;
  }
};

// the sub-block index that narrows axis a of a finer neighbour's range
// (index_utilities.cpp:830-873, 1044-1090)
int narrowing_fi(const Entry& e, int a) {
  if (a == 0) return e.fi[0];
  if (a == 1) return e.ox[0] != 0 ? e.fi[0] : e.fi[1];
  return (e.ox[0] != 0 && e.ox[1] != 0) ? e.fi[0] : e.fi[1];
}

MlOp make_op(int blk, int coarse, int mode, const int lo[3], const int hi[3]) {
  MlOp o{};
  o.blk = blk;
  o.coarse = coarse;
  o.mode = mode;
  o.count = 1;
  for (int a = 0; a < 3; ++a) {
    o.lo[a] = lo[a];
    o.hi[a] = hi[a];
    o.count *= hi[a] - lo[a] + 1;
  }
  return o;
}

template <typename T>
int upload(T** dst, const std::vector<T>& v) {
  *dst = nullptr;
  if (v.empty()) return Z4C_OK;
  if (cudaMalloc((void**)dst, sizeof(T) * v.size()) != cudaSuccess) {
    cudaGetLastError();
    return set_error(Z4C_ENOMEM, "multilevel plan: device allocation");
  }
  if (cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return set_error(Z4C_ECUDA, "multilevel plan: upload");
  return Z4C_OK;
}

}  // namespace

int ml_root_level(const int nroot[3]) {
  const int nbmax = std::max(nroot[0], std::max(nroot[1], nroot[2]));
  int r = 0;
  while ((1 << r) < nbmax) ++r;
  return r;
}

void ml_free(MlPlan& p) {
  for (void* q : {(void*)p.csrc, (void*)p.coarse, (void*)p.contrib, (void*)p.zstart, (void*)p.mult,
                  (void*)p.pro, (void*)p.pro_blk, (void*)p.coarser})
    if (q) cudaFree(q);
  for (auto& lv : p.bc)
    for (MlBc*& q : lv) {
      if (q) cudaFree(q);
      q = nullptr;
    }
  p = MlPlan{};
}

int ml_build(const int nroot[3], const int nx[3], const int bcf[6], int nblocks,
             const long long* locs, MlPlan& plan, int query_block, int* query_out) {
  plan = MlPlan{};
  if (nblocks < 1 || !locs) return set_error(Z4C_EINVAL, "multilevel mesh: no blocks");
  Builder B;
  for (int a = 0; a < 3; ++a) {
    B.nroot[a] = nroot[a];
    B.nx[a] = nx[a];
    if (nx[a] % 2 || nx[a] < 2 * NG)
      return set_error(Z4C_EINVAL, "multilevel mesh: block cells must be even and >= 2*ng");
  }
  for (int f = 0; f < 6; ++f) B.bc[f] = bcf[f];
  B.root_level = ml_root_level(nroot);
  B.nb = nblocks;
  B.locs = locs;
  // the blocks must tile the root grid: distinct leaves, none inside
  // another, their volumes summing to the root grid's
  int maxlev = B.root_level;
  for (int b = 0; b < nblocks; ++b) {
    const Loc l = B.loc(b);
    if (l.level < B.root_level || l.level > B.root_level + 12)
      return set_error(Z4C_EINVAL, "multilevel mesh: block level out of range");
    for (int a = 0; a < 3; ++a)
      if (l.l[a] < 0 || l.l[a] >= ((long long)nroot[a] << (l.level - B.root_level)))
        return set_error(Z4C_EINVAL, "multilevel mesh: logical location outside the root grid");
    if (!B.leaf.emplace(l, b).second) return set_error(Z4C_EINVAL, "multilevel mesh: duplicate block");
    maxlev = std::max(maxlev, l.level);
  }
  long long vol = 0;
  for (int b = 0; b < nblocks; ++b) {
    Loc l = B.loc(b);
    vol += 1LL << (3 * (maxlev - l.level));
    while (l.level > B.root_level) {
      l = {l.level - 1, {l.l[0] >> 1, l.l[1] >> 1, l.l[2] >> 1}};
      if (B.leaf.count(l)) return set_error(Z4C_EINVAL, "multilevel mesh: block inside another");
      B.inner.insert(l);
    }
  }
  if (vol != (long long)nroot[0] * nroot[1] * nroot[2] << (3 * (maxlev - B.root_level)))
    return set_error(Z4C_EINVAL, "multilevel mesh: the blocks do not cover the root grid");
  B.nbrs.resize(nblocks);
  for (int b = 0; b < nblocks; ++b)
    if (!B.neighbours(b, B.nbrs[b]))
      return set_error(Z4C_EINVAL, "multilevel mesh: neighbouring levels differ by more than one");
  if (query_out && query_block != -2) {  // the neighbour list of one block, no plan
    if (query_block < 0 || query_block >= nblocks)
      return set_error(Z4C_EINVAL, "multilevel mesh: block out of range");
    int q = 0;
    for (const Entry& e : B.nbrs[query_block]) {
      const int row[7] = {e.gid, e.level, e.ox[0], e.ox[1], e.ox[2], e.fi[0], e.fi[1]};
      std::memcpy(query_out + 7 * q++, row, sizeof(row));
    }
    return q;
  }

  Ax F[3], C[3];
  for (int a = 0; a < 3; ++a) {
    F[a] = axis_limits(nx[a], NG);
    C[a] = axis_limits(nx[a] / 2, kMlNcg);
    plan.nx[a] = nx[a];
    plan.nn[a] = nx[a] + 1 + 2 * NG;
    plan.cn[a] = nx[a] / 2 + 1 + 2 * kMlNcg;
  }
  plan.nblocks = nblocks;
  plan.fvol = (long long)plan.nn[0] * plan.nn[1] * plan.nn[2];
  plan.cvol = (long long)plan.cn[0] * plan.cn[1] * plan.cn[2];

  std::vector<std::vector<MlOp>> unpack(nblocks);
  std::vector<unsigned char> mults((size_t)nblocks * 343);
  long long moved = 0;
  auto push_pair = [&](int sender, int scoarse, const int slo[3], const int shi[3], int receiver,
                       int rcoarse, int mode, const int rlo[3], const int rhi[3]) {
    MlOp r = make_op(receiver, rcoarse, mode, rlo, rhi);
    r.sblk = sender;
    r.scoarse = scoarse;
    int scount = 1;
    for (int a = 0; a < 3; ++a) {
      r.slo[a] = slo[a];
      scount *= shi[a] - slo[a] + 1;
      if (shi[a] - slo[a] != rhi[a] - rlo[a]) return false;
    }
    moved += r.count;
    unpack[receiver].push_back(r);
    return scount == r.count;
  };
  for (int r = 0; r < nblocks; ++r) {
    const int rlev = (int)locs[4 * r];
    bool same = true;
    for (const Entry& e : B.nbrs[r]) same = same && e.level == rlev;
    for (const Entry& e : B.nbrs[r]) {
      const int s = e.gid;
      const Entry* back = nullptr;  // the sender's entry pointing at r
      for (const Entry& c : B.nbrs[s])
        if (c.gid == r && c.ox[0] == -e.ox[0] && c.ox[1] == -e.ox[1] && c.ox[2] == -e.ox[2]) {
          back = &c;
          break;
        }
      if (!back) return set_error(Z4C_EINVAL, "multilevel mesh: asymmetric neighbour lists");
      int slo[3], shi[3], rlo[3], rhi[3];
      bool ok = true;
      if (e.level == rlev) {
        // LoadSameLevel / SetSameLevel (index_utilities.cpp:56-106, 271-318)
        for (int a = 0; a < 3; ++a) {
          const int so = back->ox[a], ro = e.ox[a];
          slo[a] = so > 0 ? F[a].ge : F[a].vs;
          shi[a] = so < 0 ? F[a].gs : F[a].ve;
          rlo[a] = ro == 0 ? F[a].vs : (ro > 0 ? F[a].ve : F[a].ms);
          rhi[a] = ro == 0 ? F[a].ve : (ro > 0 ? F[a].pe : F[a].vs);
        }
        ok = push_pair(s, 0, slo, shi, r, 0, kMlAdd, rlo, rhi);
        if (!same) {  // the coarse payload
          for (int a = 0; a < 3; ++a) {
            const int so = back->ox[a], ro = e.ox[a];
            slo[a] = so > 0 ? C[a].ge : C[a].vs;
            shi[a] = so < 0 ? C[a].gs : C[a].ve;
            rlo[a] = ro == 0 ? C[a].vs : (ro > 0 ? C[a].ve : C[a].ms);
            rhi[a] = ro == 0 ? C[a].ve : (ro > 0 ? C[a].pe : C[a].vs);
          }
          ok = ok && push_pair(s, 1, slo, shi, r, 1, kMlAdd, rlo, rhi);
        }
      } else if (e.level < rlev) {
        // the sender is coarser: LoadToFiner from its fine array, copied into
        // the receiver's coarse buffer (SetFromCoarser)
        for (int a = 0; a < 3; ++a) {
          const int so = back->ox[a], ro = e.ox[a];
          const int hs = nx[a] / 2 - kMlNcg;
          if (so > 0) { slo[a] = F[a].ve - kMlNcg; shi[a] = F[a].ve - 1; }
          else if (so < 0) { slo[a] = F[a].vs + 1; shi[a] = F[a].vs + kMlNcg; }
          else {
            slo[a] = F[a].vs;
            shi[a] = F[a].ve;
            if (narrowing_fi(*back, a) == 1) slo[a] += hs;
            else shi[a] -= hs;
          }
          if (ro == 0) {
            rlo[a] = C[a].vs;
            rhi[a] = C[a].ve;
            if ((locs[4 * r + 1 + a] & 1) == 0) rhi[a] = C[a].pe;
            else rlo[a] = C[a].ms;
          } else if (ro > 0) { rlo[a] = C[a].ps; rhi[a] = C[a].pe; }
          else { rlo[a] = C[a].ms; rhi[a] = C[a].me; }
        }
        ok = push_pair(s, 0, slo, shi, r, 1, kMlCopy, rlo, rhi);
      } else {
        // the sender is finer: LoadToCoarser from its coarse buffer, added
        // into the receiver's fine array (SetFromFiner)
        for (int a = 0; a < 3; ++a) {
          const int so = back->ox[a], ro = e.ox[a];
          if (so > 0) { slo[a] = C[a].ve - NG; shi[a] = C[a].ve; }
          else if (so < 0) { slo[a] = C[a].vs; shi[a] = C[a].vs + NG; }
          else { slo[a] = C[a].vs; shi[a] = C[a].ve; }
          if (ro == 0) {
            rlo[a] = F[a].vs;
            rhi[a] = F[a].ve;
            if (narrowing_fi(e, a) == 1) rlo[a] += nx[a] / 2;
            else rhi[a] -= nx[a] / 2;
          } else if (ro > 0) { rlo[a] = F[a].ve; rhi[a] = F[a].pe; }
          else { rlo[a] = F[a].ms; rhi[a] = F[a].vs; }
        }
        ok = push_pair(s, 1, slo, shi, r, 0, kMlAdd, rlo, rhi);
      }
      if (!ok) return set_error(Z4C_EINVAL, "multilevel mesh: message sizes disagree");
    }
    // node multiplicity in the 7-zone compact space (NodeMultiplicity::
    // Precompute) and its division ops, fine array then coarse buffer
    unsigned short mult[7][7][7];
    std::memset(mult, 0, sizeof(mult));
    for (int k = 1; k <= 5; ++k)
      for (int j = 1; j <= 5; ++j)
        for (int i = 1; i <= 5; ++i) mult[k][j][i] = 1;
    for (const Entry& e : B.nbrs[r]) {
      int s[3], t[3];
      for (int a = 0; a < 3; ++a) {
        const int ox = e.ox[a];
        if (e.level == rlev || e.level > rlev) {
          if (ox == 0) {
            s[a] = 1;
            t[a] = 5;
            if (e.level > rlev) {
              if (narrowing_fi(e, a) == 1) s[a] += 2;
              else t[a] -= 2;
            }
          } else if (ox > 0) { s[a] = 5; t[a] = 6; }
          else { s[a] = 0; t[a] = 1; }
        } else {
          if (ox == 0) {
            s[a] = 1;
            t[a] = 5;
            if ((locs[4 * r + 1 + a] & 1) == 0) t[a] = 6;
            else s[a] = 0;
          } else if (ox > 0) { s[a] = t[a] = 6; }
          else { s[a] = t[a] = 0; }
        }
      }
      for (int k = s[2]; k <= t[2]; ++k)
        for (int j = s[1]; j <= t[1]; ++j)
          for (int i = s[0]; i <= t[0]; ++i) ++mult[k][j][i];
    }
    for (int k = 0; k < 7; ++k)
      for (int j = 0; j < 7; ++j)
        for (int i = 0; i < 7; ++i) {
          if (mult[k][j][i] > 63) return set_error(Z4C_EINVAL, "multilevel plan: multiplicity > 63");
          mults[(size_t)r * 343 + (k * 7 + j) * 7 + i] = (unsigned char)mult[k][j][i];
        }
  }
  // physical faces: extrapolation on the coarse buffer with the vertex
  // interior ends (ApplyPhysicalBCsOnCoarseLevel, called with the Z4c coarse
  // indices civs..cive and NCGHOST) and on the fine array with the cell
  // interior ends (ApplyPhysicalBCs, is..ie)
  std::vector<MlBc> bcs[2][3];
  std::vector<RefGeom> pro;
  std::vector<int> pro_blk;
  std::vector<unsigned char> coarser_of(nblocks, 0);
  for (int b = 0; b < nblocks; ++b) {
    const Loc l = B.loc(b);
    int need[6];
    for (int a = 0; a < 3; ++a) {
      const long long n = (long long)nroot[a] << (l.level - B.root_level);
      need[2 * a] = bcf[2 * a] != Z4C_BC_PERIODIC && l.l[a] == 0;
      need[2 * a + 1] = bcf[2 * a + 1] != Z4C_BC_PERIODIC && l.l[a] == n - 1;
    }
    for (int lv = 0; lv < 2; ++lv) {
      const int ng = lv ? kMlNcg : NG;
      int is[3], ie[3];
      for (int a = 0; a < 3; ++a) {
        is[a] = lv ? C[a].vs : NG;
        ie[a] = lv ? C[a].ve : NG + nx[a] - 1;
      }
      const int bis = is[0] - ng, bie = ie[0] + ng;
      const int bjs = need[2] ? is[1] : is[1] - ng, bje = need[3] ? ie[1] : ie[1] + ng;
      const int bks = need[4] ? is[2] : is[2] - ng, bke = need[5] ? ie[2] : ie[2] + ng;
      for (int face = 0; face < 6; ++face) {
        if (!need[face]) continue;
        const int ax = face / 2;
        MlBc it{};
        it.blk = b;
        it.outer = face % 2;
        it.lo[ax] = is[ax];
        it.hi[ax] = ie[ax];
        if (ax == 0) { it.lo[1] = bjs; it.hi[1] = bje; it.lo[2] = bks; it.hi[2] = bke; }
        else if (ax == 1) { it.lo[0] = bis; it.hi[0] = bie; it.lo[2] = bks; it.hi[2] = bke; }
        else { it.lo[0] = bis; it.hi[0] = bie; it.lo[1] = is[1] - ng; it.hi[1] = ie[1] + ng; }
        bcs[lv][ax].push_back(it);
      }
    }
    // ProlongationIndices (refinement_ops.cpp:24-80) per coarser neighbour
    bool coarser = false;
    for (const Entry& e : B.nbrs[b]) {
      if (e.level >= l.level) continue;
      coarser = true;
      const int pcng = NG / 2 + (NG % 2 != 0);
      int box[6];
      for (int a = 0; a < 3; ++a) {
        const int ox = e.ox[a];
        int s, t;
        if (ox > 0) { s = C[a].ve + 1; t = C[a].ve + pcng; }
        else if (ox < 0) { s = C[a].vs - pcng; t = C[a].vs - 1; }
        else {
          s = C[a].vs;
          t = C[a].ve;
          if ((l.l[a] & 1) == 0) t += pcng;
          else s -= pcng;
        }
        box[2 * a] = s;
        box[2 * a + 1] = t;
      }
      RefGeom G{};
      int rc = refine::setup(nx, 1, 1, box, G, true);
      if (rc) return rc;
      pro.push_back(G);
      pro_blk.push_back(b);
    }
    plan.ncoarser += coarser;
    coarser_of[b] = coarser;
  }
  // every box, ghost write and extrapolation read stays inside its array
  auto inside = [&](const MlOp& o) {
    const int* d = o.coarse ? plan.cn : plan.nn;
    const int* sd = o.scoarse ? plan.cn : plan.nn;
    for (int a = 0; a < 3; ++a) {
      if (o.lo[a] < 0 || o.hi[a] >= d[a] || o.lo[a] > o.hi[a]) return false;
      if (o.slo[a] < 0 || o.slo[a] + (o.hi[a] - o.lo[a]) >= sd[a]) return false;
    }
    return o.blk >= 0 && o.blk < nblocks && o.sblk >= 0 && o.sblk < nblocks;
  };
  for (const auto& v : unpack)
    for (const MlOp& o : v)
      if (!inside(o)) return set_error(Z4C_EINVAL, "multilevel plan: unpack box outside the array");
  for (int lv = 0; lv < 2; ++lv)
    for (int a = 0; a < 3; ++a)
      for (const MlBc& it : bcs[lv][a]) {
        const int* d = lv ? plan.cn : plan.nn;
        const int ng = lv ? kMlNcg : NG;
        for (int t = 0; t < 3; ++t)
          if (t != a && (it.lo[t] < 0 || it.hi[t] >= d[t]))
            return set_error(Z4C_EINVAL, "multilevel plan: boundary face outside the array");
        // ghosts lo-ng..lo-1 read up to lo-1+5; ghosts hi+1..hi+ng read down to hi+1-5
        if (it.lo[a] - ng < 0 || it.hi[a] + ng >= d[a] || it.lo[a] - 1 + 5 >= d[a] ||
            it.hi[a] + 1 - 5 < 0)
          return set_error(Z4C_EINVAL, "multilevel plan: boundary ghosts outside the array");
      }

  // per (block, array, compact zone) the ordered contributions
  std::vector<MlContrib> contrib;
  std::vector<int> zstart((size_t)nblocks * 2 * 344 + 1, 0);
  {
    std::vector<std::vector<MlContrib>> zl(2 * 343);
    for (int b = 0; b < nblocks; ++b) {
      for (auto& v : zl) v.clear();
      for (const MlOp& o : unpack[b]) {
        const Ax* X = o.coarse ? C : F;
        int zlo[3], zhi[3];
        for (int a = 0; a < 3; ++a) {
          const int mid = X[a].vs + (X[a].ve - X[a].vs) / 2;
          auto zone = [&](int i) {
            return i < X[a].vs ? 0 : i == X[a].vs ? 1 : i < mid ? 2 : i == mid ? 3
                 : i < X[a].ve ? 4 : i == X[a].ve ? 5 : 6;
          };
          const int zs[7] = {X[a].ms, X[a].vs, X[a].vs + 1, mid, mid + 1, X[a].ve, X[a].ve + 1};
          const int ze[7] = {X[a].vs - 1, X[a].vs, mid - 1, mid, X[a].ve - 1, X[a].ve, X[a].pe};
          zlo[a] = zone(o.lo[a]);
          zhi[a] = zone(o.hi[a]);
          if (o.lo[a] != zs[zlo[a]] || o.hi[a] != ze[zhi[a]])
            return set_error(Z4C_EINVAL, "multilevel plan: an unpack box splits a compact zone");
        }
        MlContrib c{};
        c.sblk = o.sblk;
        c.scoarse = (short)o.scoarse;
        c.mode = (short)o.mode;
        for (int a = 0; a < 3; ++a) c.d[a] = (short)(o.slo[a] - o.lo[a]);
        for (int zk = zlo[2]; zk <= zhi[2]; ++zk)
          for (int zj = zlo[1]; zj <= zhi[1]; ++zj)
            for (int zi = zlo[0]; zi <= zhi[0]; ++zi)
              zl[o.coarse * 343 + (zk * 7 + zj) * 7 + zi].push_back(c);
      }
      for (int arr = 0; arr < 2; ++arr) {
        for (int z = 0; z < 343; ++z) {
          zstart[((size_t)b * 2 + arr) * 344 + z] = (int)contrib.size();
          contrib.insert(contrib.end(), zl[arr * 343 + z].begin(), zl[arr * 343 + z].end());
        }
        zstart[((size_t)b * 2 + arr) * 344 + 343] = (int)contrib.size();
      }
    }
  }

  if (query_out) {  // query_block == -2: the op counts of the checked plan, no device memory
    size_t nu = 0;
    for (const auto& v : unpack) nu += v.size();
    query_out[0] = (int)nu;  // unpack ops (boxes)
    query_out[1] = (int)std::min(moved, (long long)INT32_MAX);
    query_out[2] = (int)pro.size();
    int nbc = 0;
    for (int lv = 0; lv < 2; ++lv)
      for (int a = 0; a < 3; ++a) nbc += (int)bcs[lv][a].size();
    query_out[3] = nbc;
    return 4;
  }
  int rc = Z4C_OK;
  auto fail_free = [&](int code) {
    ml_free(plan);
    return code;
  };
  for (int m = 1; m < 64; ++m) plan.inv[m] = 1.0 / static_cast<double>(m);
  for (double** q : {&plan.csrc, &plan.coarse}) {
    if (cudaMalloc((void**)q, sizeof(double) * Z4C_NVAR * plan.cvol * nblocks) != cudaSuccess) {
      cudaGetLastError();
      return fail_free(set_error(Z4C_ENOMEM, "multilevel plan: coarse buffers"));
    }
  }
  if ((rc = upload(&plan.contrib, contrib)) || (rc = upload(&plan.zstart, zstart)) ||
      (rc = upload(&plan.mult, mults)) || (rc = upload(&plan.pro, pro)) ||
      (rc = upload(&plan.pro_blk, pro_blk)) || (rc = upload(&plan.coarser, coarser_of)))
    return fail_free(rc);
  plan.ncontrib = (int)contrib.size();
  for (int b = 0; b < nblocks; ++b)
    plan.max_block_contrib = std::max(plan.max_block_contrib,
                                      zstart[((size_t)b * 2 + 1) * 344 + 343] -
                                          zstart[(size_t)b * 2 * 344]);
  plan.npro = (int)pro.size();
  for (int lv = 0; lv < 2; ++lv)
    for (int a = 0; a < 3; ++a) {
      if ((rc = upload(&plan.bc[lv][a], bcs[lv][a]))) return fail_free(rc);
      plan.nbc[lv][a] = (int)bcs[lv][a].size();
    }
  return Z4C_OK;
}

int launch_ml_exchange(const MlPlan& P, const double* src, double* dst, int nvar, int reg_nvar,
                       cudaStream_t st) {
  if (nvar < 1 || nvar > Z4C_NVAR || reg_nvar < nvar)
    return set_error(Z4C_EINVAL, "multilevel exchange: bad variable count");
  long long launches = 0;
  {
    const int64_t n = (int64_t)(P.nx[0] / 2 + 1) * (P.nx[1] / 2 + 1) * (P.nx[2] / 2 + 1) * nvar *
                      P.nblocks;
    k_ml_restrict<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, src, P.csrc, nvar, reg_nvar);
    ++launches;
  }
  const size_t smem = sizeof(MlContrib) * (size_t)std::max(P.max_block_contrib, 1);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_ml_unpack, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return set_error(Z4C_ECUDA, "multilevel exchange: shared memory for the contribution lists");
  k_ml_unpack<<<dim3(P.nblocks, 2), kMlUnpackThreads, smem, st>>>(P, src, dst, nvar, reg_nvar);
  ++launches;
  auto bc_axis = [&](int lv, double* arr, int64_t bstride, int64_t vol, const int* dims, int ng) {
    for (int a = 0; a < 3; ++a) {
      if (!P.nbc[lv][a]) continue;
      const dim3 grid(P.nbc[lv][a], nvar);
      if (a == 0) k_ml_bc<0><<<grid, 128, 0, st>>>(P.bc[lv][a], arr, bstride, vol, dims[0], dims[1], ng);
      else if (a == 1) k_ml_bc<1><<<grid, 128, 0, st>>>(P.bc[lv][a], arr, bstride, vol, dims[0], dims[1], ng);
      else k_ml_bc<2><<<grid, 128, 0, st>>>(P.bc[lv][a], arr, bstride, vol, dims[0], dims[1], ng);
      ++launches;
    }
  };
  bc_axis(1, P.coarse, (int64_t)Z4C_NVAR * P.cvol, P.cvol, P.cn, kMlNcg);
  if (P.npro > 0) {
    k_ml_prolong<<<dim3(P.npro, nvar), 128, 0, st>>>(P, dst, reg_nvar);
    ++launches;
  }
  bc_axis(0, dst, (int64_t)reg_nvar * P.fvol, P.fvol, P.nn, NG);
  add_kernel_launches(launches);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(Z4C_ECUDA, cudaGetErrorString(e));
  return Z4C_OK;
}

int launch_ml_prolong_owner(const MlPlan& P, int* owner, cudaStream_t st) {
  if (cudaMemsetAsync(owner, 0x7f, sizeof(int) * (size_t)P.fvol * P.nblocks, st) != cudaSuccess)
    return set_error(Z4C_ECUDA, "multilevel transpose: owner table");
  if (P.npro > 0) {
    k_ml_prolong_owner<<<P.npro, 128, 0, st>>>(P, owner);
    add_kernel_launches(1);
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? Z4C_OK : set_error(Z4C_ECUDA, cudaGetErrorString(e));
}

int launch_ml_exchange_adj(const MlPlan& P, double* ubar, double* wbar, const int* owner, int nvar,
                           int reg_nvar, cudaStream_t st) {
  if (nvar < 1 || nvar > Z4C_NVAR || reg_nvar < nvar)
    return set_error(Z4C_EINVAL, "multilevel transpose: bad variable count");
  long long launches = 0;
  auto bc_axis = [&](int lv, double* arr, int64_t bstride, int64_t vol, const int* dims, int ng) {
    for (int a = 2; a >= 0; --a) {
      if (!P.nbc[lv][a]) continue;
      const dim3 grid(P.nbc[lv][a], nvar);
      if (a == 0) k_ml_bc_adj<0><<<grid, 128, 0, st>>>(P.bc[lv][a], arr, bstride, vol, dims[0], dims[1], ng);
      else if (a == 1) k_ml_bc_adj<1><<<grid, 128, 0, st>>>(P.bc[lv][a], arr, bstride, vol, dims[0], dims[1], ng);
      else k_ml_bc_adj<2><<<grid, 128, 0, st>>>(P.bc[lv][a], arr, bstride, vol, dims[0], dims[1], ng);
      ++launches;
    }
  };
  // fine BCs, then prolongation, in reverse
  bc_axis(0, ubar, (int64_t)reg_nvar * P.fvol, P.fvol, P.nn, NG);
  const size_t cbytes = sizeof(double) * (size_t)Z4C_NVAR * P.cvol * P.nblocks;
  if (cudaMemsetAsync(P.coarse, 0, cbytes, st) != cudaSuccess ||
      cudaMemsetAsync(P.csrc, 0, cbytes, st) != cudaSuccess ||
      cudaMemsetAsync(wbar, 0, sizeof(double) * (size_t)reg_nvar * P.fvol * P.nblocks, st) !=
          cudaSuccess)
    return set_error(Z4C_ECUDA, "multilevel transpose: clearing the adjoints");
  if (P.npro > 0) {
    k_ml_prolong_adj<<<dim3(P.npro, nvar), 128, 0, st>>>(P, ubar, owner, reg_nvar);
    ++launches;
  }
  bc_axis(1, P.coarse, (int64_t)Z4C_NVAR * P.cvol, P.cvol, P.cn, kMlNcg);
  const size_t smem = sizeof(MlContrib) * (size_t)std::max(P.max_block_contrib, 1);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_ml_unpack_adj, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return set_error(Z4C_ECUDA, "multilevel transpose: shared memory for the contribution lists");
  k_ml_unpack_adj<<<dim3(P.nblocks, 2), kMlUnpackThreads, smem, st>>>(P, ubar, wbar, nvar,
                                                                      reg_nvar);
  ++launches;
  {
    const int64_t n = (int64_t)(P.nx[0] / 2 + 1) * (P.nx[1] / 2 + 1) * (P.nx[2] / 2 + 1) * nvar *
                      P.nblocks;
    k_ml_restrict_adj<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, wbar, nvar, reg_nvar);
    ++launches;
  }
  add_kernel_launches(launches);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(Z4C_ECUDA, cudaGetErrorString(e));
  return Z4C_OK;
}

}  // namespace z4c

extern "C" int z4c_refined_neighbours(const z4c_mesh_desc_t* mesh, int nblocks, const long long* locs,
                                      int block, int* out) {
  using namespace z4c;
  if (!mesh || !locs || !out) return set_error(Z4C_EINVAL, "null argument");
  MlPlan plan;
  return ml_build(mesh->nb, mesh->nx, mesh->bc, nblocks, locs, plan, block, out);
}

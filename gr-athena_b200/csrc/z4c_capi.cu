// C ABI of the B200 Z4c path (include/z4c_b200.h): context, device registers,
// operator launches, stage sequencing and the CUDA-graph-captured step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <tuple>
#include <new>
#include <string>
#include <vector>

#include "../../include/z4c_b200.h"
#include "z4c_common.cuh"
#include "z4c_kernels.cuh"
#include "z4c_multilevel.cuh"
#include "z4c_restart.cuh"
#include "z4c_wave.cuh"
#include "z4c_ctx.cuh"

using namespace z4c;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CUDA_TRY(expr)                                                         \
  do {                                                                         \
    cudaError_t e_ = (expr);                                                   \
    if (e_ != cudaSuccess)                                                     \
      return fail(Z4C_ECUDA, "%s: %s", #expr, cudaGetErrorString(e_));         \
  } while (0)

#define LAUNCH_CHECK(what)                                                     \
  do {                                                                         \
    cudaError_t e_ = cudaGetLastError();                                       \
    if (e_ != cudaSuccess)                                                     \
      return fail(Z4C_ECUDA, "%s launch: %s", what, cudaGetErrorString(e_));   \
  } while (0)


// ComputeMeshGeneratorX with sym_interval (mesh/mesh.hpp:839-863) and
// UniformMeshGeneratorX1 (mesh/mesh.hpp:939-945).
double mesh_gen_x(int64_t index, int64_t nrange, double xmin, double xmax) {
  const int64_t noffset = index - nrange / 2;
  const int64_t noffset_ceil = index - (nrange + 1) / 2;
  const double rx = static_cast<double>(noffset + noffset_ceil) / (2.0 * nrange);
  return 0.5 * (xmin + xmax) + (rx * xmax - rx * xmin);
}

// Vertex coordinates x?f of one block along one axis (nn entries) and its
// spacing, as Coordinates builds them for a uniform mesh
// (coordinates/coordinates.cpp:170-198, mesh/mesh.cpp:2537-2556).
// rlev: the block's level above the root level (nb << rlev blocks per axis).
double block_axis_coords(const z4c_mesh_desc_t* mesh, int64_t loc, int axis, double* xf,
                         int rlev = 0) {
  const int nx = mesh->nx[axis], nn = nx + 1 + 2 * Z4C_NG;
  const int64_t nb = (int64_t)mesh->nb[axis] << rlev;
  const int64_t nroot = (int64_t)nx * nb;
  const double x0 = mesh->xmin[axis], x1 = mesh->xmax[axis];
  const double bmin = (loc == 0) ? x0 : mesh_gen_x((int64_t)loc * nx, nroot, x0, x1);
  const double bmax = (loc == nb - 1) ? x1 : mesh_gen_x((int64_t)(loc + 1) * nx, nroot, x0, x1);
  for (int i = 0; i < nn; ++i)
    xf[i] = mesh_gen_x((int64_t)(i - Z4C_NG) + (int64_t)loc * nx, nroot, x0, x1);
  xf[Z4C_NG] = bmin;
  xf[Z4C_NG + nx] = bmax;
  return (bmax - bmin) / nx;
}

}  // namespace

namespace z4c {
// Records the message z4c_last_error() returns on this thread (used by the
// entry points defined in other translation units).
int set_error(int code, const char* msg) {
  g_err = msg;
  return code;
}
}  // namespace z4c


namespace {

int reg_nvar_(int reg) {
  switch (reg) {
    case Z4C_REG_ADM: return Z4C_NADM;
    case Z4C_REG_ADM_ADJ: return Z4C_NADM;
    case Z4C_REG_CON: return Z4C_NCON;
    case Z4C_REG_WEYL: return Z4C_NWEYL;
    default: return (reg >= 0 && reg < Z4C_NREG) ? Z4C_NVAR : -1;
  }
}

int check_reg(const z4c_ctx* c, int reg) {
  if (reg < 0 || reg >= Z4C_NREG) return fail(Z4C_EINVAL, "register %d out of range", reg);
  if (!c->reg[reg])
    return fail(Z4C_ESTATE, "register %d is not allocated for this integrator", reg);
  return Z4C_OK;
}

int check_block(const z4c_ctx* c, int block, int* b0, int* nb) {
  if (block == -1) {
    *b0 = 0;
    *nb = c->g.nblocks;
    return Z4C_OK;
  }
  if (block < 0 || block >= c->g.nblocks)
    return fail(Z4C_EINVAL, "block %d out of range [0,%d)", block, c->g.nblocks);
  *b0 = block;
  *nb = 1;
  return Z4C_OK;
}

int64_t reg_elems(const z4c_ctx* c, int reg) { return (int64_t)reg_nvar_(reg) * c->g.nvol * c->g.nblocks; }

// Ghost exchange of a 22-variable register, then the physical BCs; the result
// lands in `dst` (all points).  With alg the AlgConstr pass of the task list
// follows; it is folded into the exchange wherever no boundary condition
// reads the values: everywhere on periodic meshes, else on the blocks that
// touch no physical face, the others being constrained after their BCs.
int exchange_into(z4c_ctx* c, const double* src, double* dst, bool alg) {
  const DevParams P = c->dev();
  if (c->ml) {  // multilevel: the plan's exchange, then AlgConstr everywhere
    int rc = launch_ml_exchange(*c->ml, src, dst, Z4C_NVAR, Z4C_NVAR, c->stream);
    if (rc) return rc;
    if (alg) {
      launch_alg_constr(c->g, P, dst, 0, c->g.nblocks, c->stream);
      LAUNCH_CHECK("alg_constr");
    }
    return Z4C_OK;
  }
  const int fuse = !alg ? 0 : (c->has_outflow ? 2 : 1);
  launch_exchange(c->g, P, src, dst, c->nbr, fuse, c->stream);
  LAUNCH_CHECK("exchange");
  if (c->has_outflow) {
    launch_physical_bcs(c->g, dst, Z4C_NVAR, c->stream);
    LAUNCH_CHECK("physical_bcs");
    if (alg) {
      launch_alg_constr_boundary(c->g, P, dst, c->nbr, c->stream);
      LAUNCH_CHECK("alg_constr");
    }
  }
  return Z4C_OK;
}

// One GR_Z4c stage on all blocks.  Batched: fused RHS+KO+stage kernel
// (u -> w interior), then exchange(+AlgConstr) w -> u.  Per-block: the plain
// operator sequence with one RHS launch per block.
int run_stage_body(z4c_ctx* c, int stage, double dt);

// The vertices of one block on its three upper boundary planes (index
// NG + nx along one axis), every variable, from w into out; a thread per
// (variable, axis, vertex of the largest plane).
__global__ void k_save_upper_planes(Grid g, const double* __restrict__ w,
                                    double* __restrict__ out, int64_t plane) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * plane * Z4C_NVAR) return;
  const int64_t q = t % plane;
  const int ax = (int)((t / plane) % 3), n = (int)(t / (3 * plane));
  const int o1 = ax == 0 ? 1 : 0, o2 = ax == 2 ? 1 : 2;
  if (q >= (int64_t)g.nn[o1] * g.nn[o2]) return;
  int idx[3];
  idx[ax] = NG + g.nx[ax];
  idx[o1] = (int)(q % g.nn[o1]);
  idx[o2] = (int)(q / g.nn[o1]);
  const int64_t p = ((int64_t)idx[2] * g.nn[1] + idx[1]) * g.nn[0] + idx[0];
  out[(int64_t)n * g.nvol + p] = w[(int64_t)n * g.nvol + p];
}

// One stage with the puncture trackers around it: the shift is interpolated
// from the state at the start of the step (CalculateZ4cRHS, stage 1,
// task_list_gr_z4c.cpp:147-153) and the positions move after the last stage
// (EvolveTracker, main.hpp:1079-1082).  The last stage also runs the
// Z4C_TO_ADM task, which the task list schedules on every last stage
// (task_list_gr_z4c.cpp:335-344), so the ADM register follows every step.
int run_stage(z4c_ctx* c, int stage, double dt) {
  if (c->ntrk > 0 && stage == 1) {
    launch_track_interp(c->g, c->dev(), c->reg[Z4C_REG_U], c->trk, c->ntrk, c->stream);
    LAUNCH_CHECK("tracker interpolation");
  }
  int rc = run_stage_body(c, stage, dt);
  if (rc) return rc;
  if (stage == 4) {
    const DevParams P = c->dev();
    if (!c->per_block) {
      launch_z4c_to_adm(c->g, P, c->reg[Z4C_REG_U], c->reg[Z4C_REG_ADM], 0, c->g.nblocks,
                        c->stream);
    } else {
      for (int b = 0; b < c->g.nblocks; ++b)
        launch_z4c_to_adm(c->g, P, c->reg[Z4C_REG_U], c->reg[Z4C_REG_ADM], b, 1, c->stream);
    }
    LAUNCH_CHECK("z4c_to_adm");
  }
  if (c->ntrk > 0 && stage == 4) {
    launch_track_update(c->trk, c->ntrk, dt, c->stream);
    LAUNCH_CHECK("tracker update");
  }
  return Z4C_OK;
}

int run_stage_body(z4c_ctx* c, int stage, double dt) {
  const DevParams P = c->dev();
  const Grid& g = c->g;
  double* u = c->reg[Z4C_REG_U];
  double* w = c->reg[Z4C_REG_W];
  if (c->integrator == Z4C_INTEG_RK4) {
    const double* wt = kLsRk4[stage - 1];
    if (!c->per_block) {
      // stage 1 treats u1 as the zero register the task list starts from
      // instead of clearing it first
      LsStage ls{wt[0], wt[1], wt[2], wt[3], wt[4] * dt, stage == 1 ? 1 : 0};
      launch_stage_ls(g, P, u, c->scratch(), c->reg[Z4C_REG_RHS], c->reg[Z4C_REG_U1], w, ls, 0,
                      g.nblocks, c->shape, c->stream);
      LAUNCH_CHECK("stage_ls");
      if (c->in_place_fill) {
        // a single block has no neighbours: its fill is the extrapolation and
        // AlgConstr on every vertex, which run on w itself; the exchange
        // would only copy w's vertices into u.  The last stage's values on
        // the upper boundary planes, which the extrapolation overwrites, are
        // kept in rhs (free until the next step) for the copy back to blocks.
        if (stage == 4) {
          const int64_t plane = std::max({(int64_t)g.nn[1] * g.nn[2], (int64_t)g.nn[0] * g.nn[2],
                                          (int64_t)g.nn[0] * g.nn[1]});
          const int64_t n = 3 * plane * Z4C_NVAR;
          k_save_upper_planes<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
              g, w, c->reg[Z4C_REG_RHS], plane);
          add_kernel_launches(1);
          LAUNCH_CHECK("save planes");
        }
        launch_physical_bcs(g, w, Z4C_NVAR, c->stream);
        LAUNCH_CHECK("physical_bcs");
        launch_alg_constr_boundary(g, P, w, c->nbr, c->stream);
        LAUNCH_CHECK("alg_constr");
        std::swap(c->reg[Z4C_REG_U], c->reg[Z4C_REG_W]);
        return Z4C_OK;
      }
      return exchange_into(c, w, u, true);
    }
    // plain path, every operator launched per block as the task list calls
    // them: u1 = 0 at stage 1, then Z4cRHS, WeightedAve x2, AddZ4cRHS; then
    // exchange, AlgConstr
    if (stage == 1) {
      launch_zero_interior(g, c->reg[Z4C_REG_U1], Z4C_NVAR, c->stream);
      LAUNCH_CHECK("zero u1");
    }
    const double w1[3] = {1.0, wt[0], 0.0};
    const double w2[3] = {wt[1], wt[2], wt[3]};
    for (int b = 0; b < g.nblocks; ++b) {
      launch_rhs(g, P, u, c->scratch(), c->reg[Z4C_REG_RHS], b, 1, c->shape, c->stream);
      launch_boundary_rhs(g, P, u, c->reg[Z4C_REG_RHS], b, 1, c->stream);
      launch_weighted_ave(g, c->reg[Z4C_REG_U1], u, nullptr, w1, b, 1, c->stream);
      launch_weighted_ave(g, u, c->reg[Z4C_REG_U1], nullptr, w2, b, 1, c->stream);
      launch_add_rhs(g, c->reg[Z4C_REG_RHS], wt[4] * dt, u, b, 1, c->stream);
      LAUNCH_CHECK("per-block stage");
    }
    int rc = exchange_into(c, u, w, false);
    if (rc) return rc;
    std::swap(c->reg[Z4C_REG_U], c->reg[Z4C_REG_W]);
    u = c->reg[Z4C_REG_U];
    for (int b = 0; b < g.nblocks; ++b) {
      launch_alg_constr(g, P, u, b, 1, c->stream);
      LAUNCH_CHECK("alg_constr");
    }
    return Z4C_OK;
  }
  // classical Butcher RK4
  if (stage == 1) {
    CUDA_TRY(cudaMemcpyAsync(c->un, u, sizeof(double) * reg_elems(c, Z4C_REG_U),
                             cudaMemcpyDeviceToDevice, c->stream));
  }
  BtStage bs{};
  if (stage < 4) {
    for (int q = 0; q < 4; ++q) bs.coef[q] = kBtA[stage][q] * dt;
    bs.nq = stage + 1;
  } else {
    for (int q = 0; q < 4; ++q) bs.coef[q] = kBtB[q] * dt;
    bs.nq = 4;
  }
  bs.kslot = stage - 1;
  double* K[4] = {c->reg[Z4C_REG_K1], c->reg[Z4C_REG_K2], c->reg[Z4C_REG_K3],
                  c->reg[Z4C_REG_K4]};
  if (!c->per_block) {
    launch_stage_bt(g, P, u, c->scratch(), c->reg[Z4C_REG_RHS], c->un, K, w, bs, 0, g.nblocks,
                    c->shape, c->stream);
    LAUNCH_CHECK("stage_bt");
    return exchange_into(c, w, u, true);
  }
  for (int b = 0; b < g.nblocks; ++b) {
    launch_stage_bt(g, P, u, c->scratch(), c->reg[Z4C_REG_RHS], c->un, K, w, bs, b, 1,
                    c->shape, c->stream);
    LAUNCH_CHECK("stage_bt");
  }
  int rc = exchange_into(c, w, u, false);
  if (rc) return rc;
  for (int b = 0; b < g.nblocks; ++b) {
    launch_alg_constr(g, P, u, b, 1, c->stream);
    LAUNCH_CHECK("alg_constr");
  }
  return Z4C_OK;
}

void free_ctx(z4c_ctx* c) {
  if (c->graph) cudaGraphExecDestroy(c->graph);
  // the tangent and adjoint registers belong to the adjoint buffers
  c->reg[Z4C_REG_TAN] = c->reg[Z4C_REG_ADJ] = c->reg[Z4C_REG_ADM_ADJ] = nullptr;
  for (auto& r : c->reg)
    if (r) cudaFree(r);
  for (void* p : {(void*)c->un, (void*)c->guu, (void*)c->sd, (void*)c->rsum, (void*)c->lv, (void*)c->xf, (void*)c->xv, (void*)c->dxd, (void*)c->fd,
                  (void*)c->nbr, (void*)c->partials, (void*)c->flag, (void*)c->trk})
    if (p) cudaFree(p);
  for (auto& w : c->waves) wave_free(&w);
  if (c->ml) {
    ml_free(*c->ml);
    delete c->ml;
  }
  if (c->som) cudaFree(c->som);
  if (c->adj) adj_free(c->adj);
  if (c->jobs) {
    JobPipe* J = c->jobs;
    for (cudaStream_t s : {J->h2d, J->d2h})
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    for (int k = 0; k < 2; ++k) {
      for (cudaEvent_t e : {J->in_ready[k], J->in_free[k], J->out_ready[k], J->out_free[k]})
        if (e) cudaEventDestroy(e);
      for (void* p : {(void*)J->in[k], (void*)J->out[k], (void*)J->part[k]})
        if (p) cudaFree(p);
      if (J->hpart[k]) cudaFreeHost(J->hpart[k]);
    }
    delete J;
  }
  if (c->merged) free_ctx(c->merged);  // its stream is c's
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // namespace

extern "C" {

void z4c_params_default(z4c_params_t* p) {
  p->chi_psi_power = -4.0;
  p->chi_div_floor = -1000.0;
  p->diss = 0.0;
  p->eps_floor = 1e-12;
  p->damp_kappa1 = 0.0;
  p->damp_kappa2 = 0.0;
  p->lapse_oplog = 2.0;
  p->lapse_harmonicf = 1.0;
  p->lapse_harmonic = 0.0;
  p->lapse_advect = 1.0;
  p->lapse_K = 0.0;
  p->shift_Gamma = 1.0;
  p->shift_alpha2Gamma = 0.0;
  p->shift_H = 0.0;
  p->shift_advect = 1.0;
  p->shift_eta = 2.0;
  p->r_max_con = std::numeric_limits<double>::infinity();
  p->tf_force_regularization = 1;
  p->force_regularization = 0;
}

const char* z4c_last_error(void) { return g_err.c_str(); }

int z4c_reg_nvar(int reg) { return reg_nvar_(reg); }

namespace {
// A context on a uniform block grid (locs == nullptr) or on the nblocks
// blocks of a refined mesh given by their logical locations in gid order.
int create_impl(const z4c_mesh_desc_t* mesh, const z4c_params_t* params, int integrator,
                int nblocks_ml, const long long* locs, z4c_ctx** out) {
  if (!mesh || !params || !out) return fail(Z4C_EINVAL, "null argument");
  *out = nullptr;
  if (integrator != Z4C_INTEG_RK4 && integrator != Z4C_INTEG_BT_RK4)
    return fail(Z4C_EINVAL, "unknown integrator %d", integrator);
  for (int a = 0; a < 3; ++a) {
    if (mesh->nb[a] < 1) return fail(Z4C_EINVAL, "nb[%d] = %d < 1", a, mesh->nb[a]);
    if (mesh->nx[a] < 2 * Z4C_NG)
      return fail(Z4C_EINVAL, "nx[%d] = %d below 2*ng = %d", a, mesh->nx[a], 2 * Z4C_NG);
    if (!(mesh->xmax[a] > mesh->xmin[a])) return fail(Z4C_EINVAL, "empty extent on axis %d", a);
    const int lo = mesh->bc[2 * a], hi = mesh->bc[2 * a + 1];
    auto known = [](int f) {
      return f == Z4C_BC_PERIODIC || f == Z4C_BC_OUTFLOW || f == Z4C_BC_SOMMERFELD;
    };
    if (!known(lo) || !known(hi))
      return fail(Z4C_EINVAL, "unknown boundary flag on axis %d", a);
    if ((lo == Z4C_BC_PERIODIC) != (hi == Z4C_BC_PERIODIC))
      return fail(Z4C_EINVAL, "axis %d: periodic on one face only", a);
  }
  if (locs && nblocks_ml < 1) return fail(Z4C_EINVAL, "refined mesh without blocks");
  const int64_t nblocks_all =
      locs ? (int64_t)nblocks_ml : (int64_t)mesh->nb[0] * mesh->nb[1] * mesh->nb[2];
  {
    // the column passes index (block, variable, interior column) in 32 bits
    const int64_t cols = (int64_t)(mesh->nx[0] + 1) * (mesh->nx[1] + 1) * Z4C_NVAR * nblocks_all;
    if (cols >= (int64_t)std::numeric_limits<int>::max())
      return fail(Z4C_EINVAL, "mesh too large: %lld interior columns x variables", (long long)cols);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(Z4C_ENODEV, "no CUDA device");
  z4c_ctx* c = new (std::nothrow) z4c_ctx();
  if (!c) return fail(Z4C_ENOMEM, "host allocation");
  cudaGetDevice(&c->device);
  c->desc = *mesh;
  c->params = *params;
  c->integrator = integrator;
  Grid& g = c->g;
  for (int a = 0; a < 3; ++a) {
    g.nb[a] = mesh->nb[a];
    g.nx[a] = mesh->nx[a];
    g.nn[a] = mesh->nx[a] + 1 + 2 * Z4C_NG;
  }
  for (int f = 0; f < 6; ++f) {
    g.bc[f] = mesh->bc[f];
    if (g.bc[f] != Z4C_BC_PERIODIC) c->has_outflow = true;
    if (g.bc[f] == Z4C_BC_SOMMERFELD) g.has_sommerfeld = 1;
  }
  g.s[0] = 1;
  g.s[1] = g.nn[0];
  g.s[2] = (int64_t)g.nn[0] * g.nn[1];
  g.nvol = (int64_t)g.nn[0] * g.nn[1] * g.nn[2];
  g.nblocks = g.nb[0] * g.nb[1] * g.nb[2];
  if (locs) {
    // the uniform-grid kernels (exchange, BCs, Sommerfeld faces) never run on
    // a refined mesh; the block row keeps their indexing in range
    g.nb[0] = nblocks_ml;
    g.nb[1] = g.nb[2] = 1;
    g.nblocks = nblocks_ml;
    c->locs.assign(locs, locs + 4 * (size_t)nblocks_ml);
    c->ml = new (std::nothrow) MlPlan();
    if (!c->ml) {
      free_ctx(c);
      return fail(Z4C_ENOMEM, "host allocation");
    }
    const int rc = ml_build(mesh->nb, mesh->nx, mesh->bc, nblocks_ml, locs, *c->ml);
    if (rc) {
      free_ctx(c);
      return rc;
    }
    if (g.has_sommerfeld) {  // the blocks' gr_sommerfeld faces from their logical locations
      const int rl = ml_root_level(mesh->nb);
      std::vector<unsigned char> som(nblocks_ml, 0);
      for (int b = 0; b < nblocks_ml; ++b)
        for (int a = 0; a < 3; ++a) {
          const long long n = (long long)mesh->nb[a] << (locs[4 * b] - rl);
          if (mesh->bc[2 * a] == Z4C_BC_SOMMERFELD && locs[4 * b + 1 + a] == 0)
            som[b] |= (unsigned char)(1u << (2 * a));
          if (mesh->bc[2 * a + 1] == Z4C_BC_SOMMERFELD && locs[4 * b + 1 + a] == n - 1)
            som[b] |= (unsigned char)(1u << (2 * a + 1));
        }
      if (cudaMalloc((void**)&c->som, som.size()) != cudaSuccess ||
          cudaMemcpy(c->som, som.data(), som.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        free_ctx(c);
        return fail(Z4C_ENOMEM, "gr_sommerfeld face table");
      }
    }
  }
  const int root_level = ml_root_level(mesh->nb);

  // block coordinates (coordinates/coordinates.cpp:170-198, cartesian.cpp:29)
  const int nb = g.nblocks;
  const int nsum = g.nn[0] + g.nn[1] + g.nn[2];
  c->h_xf.assign((size_t)nb * nsum, 0.0);
  c->h_xv.assign((size_t)nb * (nsum - 3), 0.0);
  c->h_dx.assign((size_t)nb * 3, 0.0);
  std::vector<FdScale> hfd(nb);
  const double diss_scaling = std::pow(2, -2 * Z4C_NG) * (Z4C_NG % 2 == 0 ? -1 : 1);
  for (int b = 0; b < nb; ++b) {
    int64_t loc[3] = {b % g.nb[0], (b / g.nb[0]) % g.nb[1], b / (g.nb[0] * g.nb[1])};
    int rlev = 0;
    if (locs) {
      rlev = (int)locs[4 * b] - root_level;
      for (int a = 0; a < 3; ++a) loc[a] = locs[4 * b + 1 + a];
    }
    int off = 0, offv = 0;
    for (int a = 0; a < 3; ++a) {
      double* xf = &c->h_xf[(size_t)b * nsum + off];
      const double dx = block_axis_coords(mesh, loc[a], a, xf, rlev);
      double* xv = &c->h_xv[(size_t)b * (nsum - 3) + offv];
      for (int i = 0; i < g.nn[a] - 1; ++i) xv[i] = 0.5 * (xf[i + 1] + xf[i]);
      c->h_dx[(size_t)b * 3 + a] = dx;
      hfd[b].cidx1[a] = 1.0 / (dx * 60.0);
      hfd[b].cidx2[a] = ((1.0 / dx) * (1.0 / dx)) / 180.0;
      hfd[b].cidxd[a] = diss_scaling / (dx * 1.0);
      hfd[b].lidx[a] = 1.0 / (dx * 60.0);
      off += g.nn[a];
      offv += g.nn[a] - 1;
    }
  }
  // neighbour table in the reference's search order (mesh_topology.cpp:329-960)
  static const int dirs[26][3] = {
      {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1},
      {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0},
      {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {1, 0, 1},
      {0, -1, -1}, {0, 1, -1}, {0, -1, 1}, {0, 1, 1},
      {-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
      {-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}};
  std::vector<int> hnbr((size_t)nb * 26);
  for (int b = 0; b < nb; ++b) {
    const int loc[3] = {b % g.nb[0], (b / g.nb[0]) % g.nb[1], b / (g.nb[0] * g.nb[1])};
    for (int d = 0; d < 26; ++d) {
      int l[3];
      bool ok = true;
      for (int a = 0; a < 3; ++a) {
        l[a] = loc[a] + dirs[d][a];
        if (l[a] < 0 || l[a] >= g.nb[a]) {
          if (g.bc[2 * a] == Z4C_BC_PERIODIC) l[a] = (l[a] + g.nb[a]) % g.nb[a];
          else ok = false;
        }
      }
      hnbr[(size_t)b * 26 + d] = ok ? l[0] + g.nb[0] * (l[1] + g.nb[1] * l[2]) : -1;
    }
  }

  auto alloc = [&](void** p, size_t bytes) -> int {
    if (cudaMalloc(p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(Z4C_ENOMEM, "cudaMalloc of %zu bytes failed", bytes);
    }
    return Z4C_OK;
  };
  int rc = Z4C_OK;
  const size_t b22 = sizeof(double) * (size_t)Z4C_NVAR * g.nvol * nb;
  int need[Z4C_NREG] = {};
  need[Z4C_REG_U] = need[Z4C_REG_W] = need[Z4C_REG_RHS] = need[Z4C_REG_ADM] =
      need[Z4C_REG_CON] = need[Z4C_REG_WEYL] = 1;
  if (integrator == Z4C_INTEG_RK4) need[Z4C_REG_U1] = 1;
  else need[Z4C_REG_K1] = need[Z4C_REG_K2] = need[Z4C_REG_K3] = need[Z4C_REG_K4] = 1;
  for (int r = 0; r < Z4C_NREG && rc == Z4C_OK; ++r) {
    if (!need[r]) continue;
    const size_t bytes = sizeof(double) * (size_t)reg_nvar_(r) * g.nvol * nb;
    rc = alloc((void**)&c->reg[r], bytes);
    if (rc == Z4C_OK && cudaMemset(c->reg[r], 0, bytes) != cudaSuccess)
      rc = fail(Z4C_ECUDA, "memset register %d", r);
  }
  if (rc == Z4C_OK && integrator == Z4C_INTEG_BT_RK4) rc = alloc((void**)&c->un, b22);
  if (rc == Z4C_OK) rc = alloc((void**)&c->guu, sizeof(double) * 6 * (size_t)g.nvol * nb);
  if (rc == Z4C_OK)
    rc = alloc((void**)&c->sd, sizeof(double) * kSdComponents * (size_t)g.nvol * nb);
  if (rc == Z4C_OK)
    rc = alloc((void**)&c->rsum, sizeof(double) * 6 * (size_t)interior_count(g) * nb);
  if (rc == Z4C_OK)
    rc = alloc((void**)&c->lv, sizeof(double) * Z4C_NVAR * (size_t)interior_count(g) * nb);
  if (rc == Z4C_OK) rc = alloc((void**)&c->xf, sizeof(double) * c->h_xf.size());
  if (rc == Z4C_OK) rc = alloc((void**)&c->xv, sizeof(double) * c->h_xv.size());
  if (rc == Z4C_OK) rc = alloc((void**)&c->dxd, sizeof(double) * c->h_dx.size());
  if (rc == Z4C_OK) rc = alloc((void**)&c->fd, sizeof(FdScale) * nb);
  if (rc == Z4C_OK) rc = alloc((void**)&c->nbr, sizeof(int) * hnbr.size());
  if (rc == Z4C_OK) rc = alloc((void**)&c->partials, sizeof(double) * 8 * nb);
  if (rc == Z4C_OK) rc = alloc((void**)&c->flag, sizeof(int));
  if (rc == Z4C_OK) rc = alloc((void**)&c->trk, sizeof(double) * 8 * kMaxTrackers);
  if (rc != Z4C_OK) {
    free_ctx(c);
    return rc;
  }
  if (cudaMemcpy(c->xf, c->h_xf.data(), sizeof(double) * c->h_xf.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(c->xv, c->h_xv.data(), sizeof(double) * c->h_xv.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(c->dxd, c->h_dx.data(), sizeof(double) * c->h_dx.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(c->fd, hfd.data(), sizeof(FdScale) * nb, cudaMemcpyHostToDevice) ||
      cudaMemcpy(c->nbr, hnbr.data(), sizeof(int) * hnbr.size(), cudaMemcpyHostToDevice)) {
    free_ctx(c);
    return fail(Z4C_ECUDA, "uploading mesh tables");
  }
  if (allow_slab_smem() != 0) {
    free_ctx(c);
    return fail(Z4C_ECUDA, "raising the shared-memory limit of the slab kernels");
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    free_ctx(c);
    return fail(Z4C_ECUDA, "stream creation");
  }
  c->own_stream = true;
  *out = c;
  return Z4C_OK;
}
}  // namespace

int z4c_create(const z4c_mesh_desc_t* mesh, const z4c_params_t* params, int integrator,
               z4c_ctx** out) {
  return create_impl(mesh, params, integrator, 0, nullptr, out);
}

int z4c_create_refined(const z4c_mesh_desc_t* mesh, int nblocks, const long long* locs,
                       const z4c_params_t* params, int integrator, z4c_ctx** out) {
  if (!locs) return fail(Z4C_EINVAL, "null argument");
  return create_impl(mesh, params, integrator, nblocks, locs, out);
}

int z4c_restart_locs(const char* path, long long* locs, int cap) {
  if (!path) return fail(Z4C_EINVAL, "null argument");
  z4c_restart_info_t info;
  std::string text, err;
  std::vector<long long> l;
  const int rc = restart_read_file(path, &info, &text, nullptr, &err, &l);
  if (rc) return fail(rc, "%s", err.c_str());
  if (locs) {
    if (cap < info.nbtotal) return fail(Z4C_EINVAL, "room for %d MeshBlocks, the file has %d", cap,
                                        info.nbtotal);
    std::memcpy(locs, l.data(), sizeof(long long) * l.size());
  }
  return info.nbtotal;
}

int z4c_mesh_loc_coords(const z4c_mesh_desc_t* mesh, const long long loc[4], int axis,
                        double* x_out, double* dx_out) {
  if (!mesh || !loc || !x_out || axis < 0 || axis > 2) return fail(Z4C_EINVAL, "bad argument");
  const int rlev = (int)loc[0] - ml_root_level(mesh->nb);
  if (rlev < 0 || rlev > 20 || mesh->nx[axis] < 1) return fail(Z4C_EINVAL, "level out of range");
  if (loc[1 + axis] < 0 || loc[1 + axis] >= ((long long)mesh->nb[axis] << rlev))
    return fail(Z4C_EINVAL, "logical location out of range");
  const double dx = block_axis_coords(mesh, loc[1 + axis], axis, x_out, rlev);
  if (dx_out) *dx_out = dx;
  return Z4C_OK;
}

int z4c_destroy(z4c_ctx* ctx) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  cudaStreamSynchronize(ctx->stream);
  free_ctx(ctx);
  return Z4C_OK;
}

int z4c_set_stream(z4c_ctx* ctx, void* stream) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  ctx->own_stream = false;
  ctx->stream = static_cast<cudaStream_t>(stream);
  if (ctx->graph) {
    cudaGraphExecDestroy(ctx->graph);
    ctx->graph = nullptr;
  }
  return Z4C_OK;
}

int z4c_sync(z4c_ctx* ctx) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return Z4C_OK;
}

int z4c_num_blocks(const z4c_ctx* ctx) { return ctx ? ctx->g.nblocks : fail(Z4C_EINVAL, "null context"); }

int z4c_block_nn(const z4c_ctx* ctx, int axis) {
  if (!ctx || axis < 0 || axis > 2) return fail(Z4C_EINVAL, "bad argument");
  return ctx->g.nn[axis];
}

int z4c_dx(const z4c_ctx* ctx, double dx_out[3]) {
  if (!ctx || !dx_out) return fail(Z4C_EINVAL, "null argument");
  for (int a = 0; a < 3; ++a) dx_out[a] = ctx->h_dx[a];
  return Z4C_OK;
}

int z4c_block_coords(const z4c_ctx* ctx, int block, int axis, double* x_out) {
  if (!ctx || !x_out || axis < 0 || axis > 2) return fail(Z4C_EINVAL, "bad argument");
  if (block < 0 || block >= ctx->g.nblocks) return fail(Z4C_EINVAL, "block out of range");
  const int nsum = ctx->g.nn[0] + ctx->g.nn[1] + ctx->g.nn[2];
  int off = 0;
  for (int a = 0; a < axis; ++a) off += ctx->g.nn[a];
  std::memcpy(x_out, &ctx->h_xf[(size_t)block * nsum + off], sizeof(double) * ctx->g.nn[axis]);
  return Z4C_OK;
}

int z4c_mesh_block_coords(const z4c_mesh_desc_t* mesh, int block, int axis, double* x_out,
                          double* dx_out) {
  if (!mesh || !x_out || axis < 0 || axis > 2) return fail(Z4C_EINVAL, "bad argument");
  const int nblocks = mesh->nb[0] * mesh->nb[1] * mesh->nb[2];
  if (block < 0 || block >= nblocks || mesh->nx[axis] < 1)
    return fail(Z4C_EINVAL, "block out of range");
  const int loc[3] = {block % mesh->nb[0], (block / mesh->nb[0]) % mesh->nb[1],
                      block / (mesh->nb[0] * mesh->nb[1])};
  const double dx = block_axis_coords(mesh, loc[axis], axis, x_out);
  if (dx_out) *dx_out = dx;
  return Z4C_OK;
}

int z4c_mesh_new_dt(const z4c_mesh_desc_t* mesh, double cfl, double* dt_out) {
  if (!mesh || !dt_out) return fail(Z4C_EINVAL, "null argument");
  if (!(cfl > 0.0)) return fail(Z4C_EINVAL, "cfl must be positive");
  const int nblocks = mesh->nb[0] * mesh->nb[1] * mesh->nb[2];
  if (nblocks < 1) return fail(Z4C_EINVAL, "empty mesh");
  std::vector<double> x;
  double dt = std::numeric_limits<double>::max();
  for (int b = 0; b < nblocks; ++b) {
    const int loc[3] = {b % mesh->nb[0], (b / mesh->nb[0]) % mesh->nb[1],
                        b / (mesh->nb[0] * mesh->nb[1])};
    // NewBlockTimeStep: the minimum cell width of the block (uniform: dx per
    // axis), times the Courant number; the mesh step is the minimum over
    // blocks (Mesh::NewTimeStep)
    double min_dt = std::numeric_limits<float>::max();
    for (int a = 0; a < 3; ++a) {
      x.resize(mesh->nx[a] + 1 + 2 * Z4C_NG);
      min_dt = std::min(min_dt, block_axis_coords(mesh, loc[a], a, x.data()));
    }
    min_dt *= cfl;
    dt = std::min(dt, min_dt);
  }
  *dt_out = dt;
  return Z4C_OK;
}

int z4c_upload(z4c_ctx* ctx, int reg, int block, const double* host) {
  if (!ctx || !host) return fail(Z4C_EINVAL, "null argument");
  int rc = check_reg(ctx, reg);
  if (rc) return rc;
  int b0, nb;
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  const size_t per = (size_t)reg_nvar_(reg) * ctx->g.nvol;
  CUDA_TRY(cudaMemcpyAsync(ctx->reg[reg] + per * b0, host, sizeof(double) * per * nb,
                           cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return Z4C_OK;
}

int z4c_download(z4c_ctx* ctx, int reg, int block, double* host) {
  if (!ctx || !host) return fail(Z4C_EINVAL, "null argument");
  int rc = check_reg(ctx, reg);
  if (rc) return rc;
  int b0, nb;
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  const size_t per = (size_t)reg_nvar_(reg) * ctx->g.nvol;
  CUDA_TRY(cudaMemcpyAsync(host, ctx->reg[reg] + per * b0, sizeof(double) * per * nb,
                           cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return Z4C_OK;
}

int z4c_device_ptr(z4c_ctx* ctx, int reg, double** dptr) {
  if (!ctx || !dptr) return fail(Z4C_EINVAL, "null argument");
  int rc = check_reg(ctx, reg);
  if (rc) return rc;
  *dptr = ctx->reg[reg];
  return Z4C_OK;
}

int z4c_rhs(z4c_ctx* ctx, int reg_u, int reg_rhs, int block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_u)) || (rc = check_reg(ctx, reg_rhs))) return rc;
  if (reg_nvar_(reg_u) != Z4C_NVAR || reg_nvar_(reg_rhs) != Z4C_NVAR || reg_u == reg_rhs)
    return fail(Z4C_EINVAL, "z4c_rhs needs two distinct 22-variable registers");
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_rhs(ctx->g, ctx->dev(), ctx->reg[reg_u], ctx->scratch(), ctx->reg[reg_rhs], b0, nb,
             ctx->shape, ctx->stream);
  LAUNCH_CHECK("rhs");
  return Z4C_OK;
}

int z4c_boundary_rhs(z4c_ctx* ctx, int reg_u, int reg_rhs, int block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_u)) || (rc = check_reg(ctx, reg_rhs))) return rc;
  if (reg_nvar_(reg_u) != Z4C_NVAR || reg_nvar_(reg_rhs) != Z4C_NVAR || reg_u == reg_rhs)
    return fail(Z4C_EINVAL, "z4c_boundary_rhs needs two distinct 22-variable registers");
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_boundary_rhs(ctx->g, ctx->dev(), ctx->reg[reg_u], ctx->reg[reg_rhs], b0, nb, ctx->stream);
  LAUNCH_CHECK("boundary_rhs");
  return Z4C_OK;
}

int z4c_add_rhs(z4c_ctx* ctx, int reg_rhs, double wght, int reg_out, int block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_rhs)) || (rc = check_reg(ctx, reg_out))) return rc;
  if (reg_nvar_(reg_rhs) != Z4C_NVAR || reg_nvar_(reg_out) != Z4C_NVAR)
    return fail(Z4C_EINVAL, "z4c_add_rhs needs 22-variable registers");
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_add_rhs(ctx->g, ctx->reg[reg_rhs], wght, ctx->reg[reg_out], b0, nb, ctx->stream);
  LAUNCH_CHECK("add_rhs");
  return Z4C_OK;
}

int z4c_weighted_ave(z4c_ctx* ctx, int reg_out, int reg_in1, int reg_in2, const double w[3],
                     int block) {
  if (!ctx || !w) return fail(Z4C_EINVAL, "null argument");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_out)) || (rc = check_reg(ctx, reg_in1))) return rc;
  const double* in2 = nullptr;
  if (w[2] != 0.0) {
    if ((rc = check_reg(ctx, reg_in2))) return rc;
    in2 = ctx->reg[reg_in2];
  }
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_weighted_ave(ctx->g, ctx->reg[reg_out], ctx->reg[reg_in1], in2, w, b0, nb, ctx->stream);
  LAUNCH_CHECK("weighted_ave");
  return Z4C_OK;
}

int z4c_alg_constr(z4c_ctx* ctx, int reg_u, int block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_u))) return rc;
  if (reg_nvar_(reg_u) != Z4C_NVAR) return fail(Z4C_EINVAL, "AlgConstr needs a Z4c register");
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_alg_constr(ctx->g, ctx->dev(), ctx->reg[reg_u], b0, nb, ctx->stream);
  LAUNCH_CHECK("alg_constr");
  return Z4C_OK;
}

int z4c_adm_to_z4c(z4c_ctx* ctx, int reg_adm, int reg_u, int block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_adm)) || (rc = check_reg(ctx, reg_u))) return rc;
  if (reg_nvar_(reg_adm) != Z4C_NADM || reg_nvar_(reg_u) != Z4C_NVAR)
    return fail(Z4C_EINVAL, "ADMToZ4c needs the ADM and a Z4c register");
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_adm_to_z4c(ctx->g, ctx->dev(), ctx->reg[reg_adm], ctx->reg[reg_u], ctx->guu, b0, nb,
                    ctx->stream);
  LAUNCH_CHECK("adm_to_z4c");
  return Z4C_OK;
}

int z4c_z4c_to_adm(z4c_ctx* ctx, int reg_u, int reg_adm, int block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_adm)) || (rc = check_reg(ctx, reg_u))) return rc;
  if (reg_nvar_(reg_adm) != Z4C_NADM || reg_nvar_(reg_u) != Z4C_NVAR)
    return fail(Z4C_EINVAL, "Z4cToADM needs a Z4c and the ADM register");
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_z4c_to_adm(ctx->g, ctx->dev(), ctx->reg[reg_u], ctx->reg[reg_adm], b0, nb, ctx->stream);
  LAUNCH_CHECK("z4c_to_adm");
  return Z4C_OK;
}

int z4c_adm_constraints(z4c_ctx* ctx, int reg_con, int reg_adm, int reg_u, int block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_con)) || (rc = check_reg(ctx, reg_adm)) ||
      (rc = check_reg(ctx, reg_u)))
    return rc;
  if (reg_nvar_(reg_con) != Z4C_NCON || reg_nvar_(reg_adm) != Z4C_NADM ||
      reg_nvar_(reg_u) != Z4C_NVAR)
    return fail(Z4C_EINVAL, "ADMConstraints needs con, adm and a Z4c register");
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_adm_constraints(ctx->g, ctx->dev(), ctx->reg[reg_adm], ctx->reg[reg_u],
                         ctx->reg[reg_con], ctx->xf, b0, nb, ctx->stream);
  LAUNCH_CHECK("adm_constraints");
  return Z4C_OK;
}

int z4c_weyl(z4c_ctx* ctx, int reg_adm, int reg_u, int reg_weyl, int block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc, b0, nb;
  if ((rc = check_reg(ctx, reg_adm)) || (rc = check_reg(ctx, reg_u)) ||
      (rc = check_reg(ctx, reg_weyl)))
    return rc;
  if (reg_nvar_(reg_adm) != Z4C_NADM || reg_nvar_(reg_u) != Z4C_NVAR ||
      reg_nvar_(reg_weyl) != Z4C_NWEYL)
    return fail(Z4C_EINVAL, "Z4cWeyl needs the ADM, a Z4c and the Weyl register");
  if ((rc = check_block(ctx, block, &b0, &nb))) return rc;
  launch_weyl(ctx->g, ctx->dev(), ctx->reg[reg_adm], ctx->reg[reg_u], ctx->sd, ctx->rsum, ctx->lv,
              ctx->reg[reg_weyl], ctx->xf, b0, nb, ctx->stream);
  LAUNCH_CHECK("weyl");
  return Z4C_OK;
}

int z4c_ghost_fill(z4c_ctx* ctx, int reg) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc;
  if ((rc = check_reg(ctx, reg))) return rc;
  if (reg == Z4C_REG_WEYL) {
    // Mesh::CommunicateAuxZ4c: the Aux group exchange and physical BCs of the
    // Weyl register, through the work register
    double* w = ctx->reg[Z4C_REG_W];
    if (ctx->ml) {
      if ((rc = launch_ml_exchange(*ctx->ml, ctx->reg[reg], w, Z4C_NWEYL, Z4C_NWEYL, ctx->stream)))
        return rc;
    } else {
      launch_exchange(ctx->g, ctx->dev(), ctx->reg[reg], w, ctx->nbr, 0, ctx->stream, Z4C_NWEYL);
      LAUNCH_CHECK("exchange");
    }
    if (ctx->has_outflow && !ctx->ml) {
      launch_physical_bcs(ctx->g, w, Z4C_NWEYL, ctx->stream);
      LAUNCH_CHECK("physical_bcs");
    }
    CUDA_TRY(cudaMemcpyAsync(ctx->reg[reg], w, sizeof(double) * reg_elems(ctx, reg),
                             cudaMemcpyDeviceToDevice, ctx->stream));
    return Z4C_OK;
  }
  if (reg_nvar_(reg) != Z4C_NVAR) return fail(Z4C_EINVAL, "ghost fill needs a Z4c register");
  if (reg == Z4C_REG_W) return fail(Z4C_EINVAL, "the work register cannot be ghost-filled");
  if ((rc = exchange_into(ctx, ctx->reg[reg], ctx->reg[Z4C_REG_W], false))) return rc;
  if (reg == Z4C_REG_U) {
    std::swap(ctx->reg[Z4C_REG_U], ctx->reg[Z4C_REG_W]);
    if (ctx->graph) {  // captured pointers are stale
      cudaGraphExecDestroy(ctx->graph);
      ctx->graph = nullptr;
    }
  } else {
    CUDA_TRY(cudaMemcpyAsync(ctx->reg[reg], ctx->reg[Z4C_REG_W],
                             sizeof(double) * reg_elems(ctx, reg), cudaMemcpyDeviceToDevice,
                             ctx->stream));
  }
  return Z4C_OK;
}

int z4c_sphere_grid(int nlev, double rad, int bitant, double* geo) {
  if (nlev < 1 || nlev > 2000) return fail(Z4C_EINVAL, "nlev %d out of range [1, 2000]", nlev);
  if (!(rad > 0.0)) return fail(Z4C_EINVAL, "sphere radius must be positive");
  if (!geo) return fail(Z4C_EINVAL, "null output");
  const std::vector<double> g = sphere_grid(nlev, rad, bitant != 0);
  std::memcpy(geo, g.data(), sizeof(double) * g.size());
  return (int)(g.size() / 6);
}

int z4c_wave_add(z4c_ctx* ctx, double rad, int nlev, int lmax, int bitant, int* id) {
  if (!ctx || !id) return fail(Z4C_EINVAL, "null argument");
  if (nlev < 1 || nlev > 2000) return fail(Z4C_EINVAL, "nlev %d out of range [1, 2000]", nlev);
  if (lmax < 2 || lmax > 16) return fail(Z4C_EINVAL, "lmax %d out of range [2, 16]", lmax);
  if (!(rad > 0.0)) return fail(Z4C_EINVAL, "sphere radius must be positive");
  WaveSphere w;
  char msg[256] = {0};
  const int rc = wave_build(ctx->g, ctx->h_xf, ctx->h_dx, rad, nlev, lmax, bitant != 0, &w, msg,
                            (int)sizeof(msg));
  if (rc) return fail(rc, "%s", msg);
  ctx->waves.push_back(w);
  *id = (int)ctx->waves.size() - 1;
  return Z4C_OK;
}

int z4c_wave_points(const z4c_ctx* ctx, int id) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (id < 0 || id >= (int)ctx->waves.size()) return fail(Z4C_EINVAL, "no sphere %d", id);
  return ctx->waves[id].npts;
}

int z4c_wave_decompose(z4c_ctx* ctx, int id, int reg_weyl, double* psi) {
  if (!ctx || !psi) return fail(Z4C_EINVAL, "null argument");
  if (id < 0 || id >= (int)ctx->waves.size()) return fail(Z4C_EINVAL, "no sphere %d", id);
  int rc;
  if ((rc = check_reg(ctx, reg_weyl))) return rc;
  if (reg_nvar_(reg_weyl) != Z4C_NWEYL) return fail(Z4C_EINVAL, "decomposition needs the Weyl register");
  const WaveSphere& w = ctx->waves[id];
  launch_wave(ctx->g, w, ctx->reg[reg_weyl], ctx->stream);
  LAUNCH_CHECK("wave");
  CUDA_TRY(cudaMemcpyAsync(psi, w.psi, sizeof(double) * 2 * w.nslot, cudaMemcpyDeviceToHost,
                           ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return Z4C_OK;
}

int z4c_init_finalize(z4c_ctx* ctx) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc;
  if ((rc = z4c_ghost_fill(ctx, Z4C_REG_U))) return rc;
  const DevParams P = ctx->dev();
  launch_alg_constr(ctx->g, P, ctx->reg[Z4C_REG_U], 0, ctx->g.nblocks, ctx->stream, 1);
  LAUNCH_CHECK("alg_constr ghosts");
  launch_z4c_to_adm(ctx->g, P, ctx->reg[Z4C_REG_U], ctx->reg[Z4C_REG_ADM], 0, ctx->g.nblocks,
                    ctx->stream, 1);
  LAUNCH_CHECK("z4c_to_adm ghosts");
  return Z4C_OK;
}

int z4c_hst_norms(z4c_ctx* ctx, double out[8]) {
  if (!ctx || !out) return fail(Z4C_EINVAL, "null argument");
  launch_hst(ctx->g, ctx->dev(), ctx->reg[Z4C_REG_CON], ctx->reg[Z4C_REG_U], ctx->xv,
             ctx->partials, ctx->stream);
  LAUNCH_CHECK("hst");
  std::vector<double> h((size_t)8 * ctx->g.nblocks);
  CUDA_TRY(cudaMemcpyAsync(h.data(), ctx->partials, sizeof(double) * h.size(),
                           cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int q = 0; q < 8; ++q) out[q] = 0.0;
  for (int b = 0; b < ctx->g.nblocks; ++b) {
    const double* dx = &ctx->h_dx[(size_t)b * 3];
    const double vol = dx[0] * dx[1] * dx[2];
    for (int q = 0; q < 8; ++q) out[q] += vol * h[(size_t)b * 8 + q];
  }
  return Z4C_OK;
}

int z4c_stage(z4c_ctx* ctx, int stage, double dt) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (stage < 1 || stage > 4) return fail(Z4C_EINVAL, "stage %d outside 1..4", stage);
  return run_stage(ctx, stage, dt);
}

int z4c_rhs_stage(z4c_ctx* ctx, int stage, double dt) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (stage < 1 || stage > 4) return fail(Z4C_EINVAL, "stage %d outside 1..4", stage);
  if (ctx->integrator != Z4C_INTEG_RK4)
    return fail(Z4C_ESTATE, "z4c_rhs_stage runs the low-storage stage only");
  const double* wt = kLsRk4[stage - 1];
  LsStage ls{wt[0], wt[1], wt[2], wt[3], wt[4] * dt, 0};
  launch_stage_ls(ctx->g, ctx->dev(), ctx->reg[Z4C_REG_U], ctx->scratch(),
                  ctx->reg[Z4C_REG_RHS], ctx->reg[Z4C_REG_U1], ctx->reg[Z4C_REG_W], ls, 0,
                  ctx->g.nblocks, ctx->shape, ctx->stream);
  LAUNCH_CHECK("stage_ls");
  return Z4C_OK;
}

int z4c_fp64_probe(z4c_ctx* ctx, double* tflops) {
  if (!ctx || !tflops) return fail(Z4C_EINVAL, "null argument");
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  const int iters = 4096;
  double best = 0.0;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0, ctx->stream);
    const long long flops = launch_fp64_probe(nsm, iters, ctx->partials, 8 * ctx->g.nblocks,
                                              ctx->stream);
    cudaEventRecord(e1, ctx->stream);
    LAUNCH_CHECK("fp64_probe");
    CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *tflops = best;
  return Z4C_OK;
}

int z4c_set_per_block(z4c_ctx* ctx, int per_block) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  ctx->per_block = per_block != 0;
  return Z4C_OK;
}

namespace {
void drop_graph(z4c_ctx* ctx) {
  if (ctx->graph) {
    cudaGraphExecDestroy(ctx->graph);
    ctx->graph = nullptr;
  }
}

// Device time of one fused low-storage stage (u -> w, u1) with the given
// shape: the minimum over reps launches after one warm-up launch.
int time_stage(z4c_ctx* ctx, const LaunchShape& sh, int reps, float* best_ms) {
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  const double* wt = kLsRk4[0];
  const LsStage ls{wt[0], wt[1], wt[2], wt[3], wt[4] * 1e-3, 1};
  const DevParams P = ctx->dev();
  float best = 1e30f;
  int rc = Z4C_OK;
  for (int r = 0; r <= reps && rc == Z4C_OK; ++r) {
    cudaEventRecord(e0, ctx->stream);
    launch_stage_ls(ctx->g, P, ctx->reg[Z4C_REG_U], ctx->scratch(), ctx->reg[Z4C_REG_RHS],
                    ctx->reg[Z4C_REG_U1], ctx->reg[Z4C_REG_W], ls, 0, ctx->g.nblocks, sh,
                    ctx->stream);
    cudaEventRecord(e1, ctx->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
      rc = fail(Z4C_ECUDA, "autotune launch: %s", cudaGetErrorString(e));
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;  // launch 0 is the warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *best_ms = best;
  return rc;
}
}  // namespace

int z4c_set_tile(z4c_ctx* ctx, int ti, int tj, int tk) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  LaunchShape sh = ctx->shape;
  sh.point_threads = ti;
  sh.column_threads = tj;
  sh.column_slabs = tk;
  if (!valid_shape(sh))
    return fail(Z4C_EINVAL, "unsupported launch shape (%d, %d, %d): point threads 64/128/256, "
                "column threads 128/256/512, column slabs 0-4", ti, tj, tk);
  ctx->shape = sh;
  drop_graph(ctx);
  return Z4C_OK;
}

int z4c_set_point_regs(z4c_ctx* ctx, int regs) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (regs != 0 && regs != kPointRegsHigh)
    return fail(Z4C_EINVAL, "register budget %d: 0 or %d", regs, kPointRegsHigh);
  if (ctx->shape.point_regs != regs) {
    ctx->shape.point_regs = regs;
    drop_graph(ctx);
  }
  return Z4C_OK;
}

int z4c_get_point_regs(const z4c_ctx* ctx, int* regs) {
  if (!ctx || !regs) return fail(Z4C_EINVAL, "null argument");
  *regs = ctx->shape.point_regs;
  return Z4C_OK;
}

int z4c_set_contract(z4c_ctx* ctx, int on) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (ctx->shape.contract != (on != 0)) {
    ctx->shape.contract = on != 0;
    drop_graph(ctx);
  }
  return Z4C_OK;
}

int z4c_get_contract(const z4c_ctx* ctx, int* on) {
  if (!ctx || !on) return fail(Z4C_EINVAL, "null argument");
  *on = ctx->shape.contract;
  return Z4C_OK;
}

namespace {
bool merge_eligible(const z4c_ctx* c);
}

int z4c_set_merged(z4c_ctx* ctx, int on) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  ctx->merge = on != 0;
  return Z4C_OK;
}

int z4c_get_merged(const z4c_ctx* ctx, int* on) {
  if (!ctx || !on) return fail(Z4C_EINVAL, "null argument");
  *on = ctx->merge && merge_eligible(ctx);
  return Z4C_OK;
}

int z4c_get_tile(const z4c_ctx* ctx, int tile_out[3]) {
  if (!ctx || !tile_out) return fail(Z4C_EINVAL, "null argument");
  tile_out[0] = ctx->shape.point_threads;
  tile_out[1] = ctx->shape.column_threads;
  tile_out[2] = ctx->shape.column_slabs;
  return Z4C_OK;
}

int z4c_autotune(z4c_ctx* ctx, int reps, float* best_ms_out) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (ctx->integrator != Z4C_INTEG_RK4)
    return fail(Z4C_ESTATE, "the autotuner times the low-storage stage");
  if (reps < 1) reps = 1;
  // greedy: the heavy passes' CTA size first, then the column passes' shape;
  // the stage writes only the work register, u1 and rhs, so u is untouched
  LaunchShape best = ctx->shape;
  float best_ms = 1e30f, ms = 0.f;
  int rc;
  for (int pt : {64, 128, 256})
    for (int regs : {0, kPointRegsHigh}) {
      if (regs && (pt == 256 || !has_fixed_geometry(ctx->g))) continue;
      LaunchShape sh = best;
      sh.point_threads = pt;
      sh.point_regs = regs;
      if ((rc = time_stage(ctx, sh, reps, &ms))) return rc;
      if (ms < best_ms) {
        best_ms = ms;
        best.point_threads = pt;
        best.point_regs = regs;
      }
    }
  for (int ct : {128, 256, 512})
    for (int ns : {0, 1, 2, 3, 4}) {
      LaunchShape sh = best;
      sh.column_threads = ct;
      sh.column_slabs = ns;
      if (ns > 0 && !slabs_fit(ctx->g, sh)) continue;
      // the contracted path has no slab variant
      if (ns > 0 && sh.contract && !ctx->g.has_sommerfeld) continue;
      if ((rc = time_stage(ctx, sh, reps, &ms))) return rc;
      if (ms < best_ms) {
        best_ms = ms;
        best.column_threads = ct;
        best.column_slabs = ns;
      }
    }
  ctx->shape = best;
  drop_graph(ctx);
  if (best_ms_out) *best_ms_out = best_ms;
  return Z4C_OK;
}

namespace {
// ---- merged vertex grid of a uniform mesh ---------------------------------
// The blocks of a uniform mesh tile one vertex grid of nb*nx cells per axis;
// vertex (I, J, K) of that grid (ghosts included) is vertex (I - bx nx,
// J - by nx, K - bz nx) of block (bx, by, bz), bx the highest block whose
// interior starts at or below it (clamped to the mesh), so a vertex on a
// shared face comes from the upper block, one on the mesh's outer ghosts
// from the boundary block.  The merged grid's own step runs the same
// kernels as one block of nb*nx cells.  Block b sits at (b % nb0, (b / nb0) % nb1,
// b / (nb0 nb1)), the order of the uniform context.
__global__ void k_merge_scatter(Grid g, Grid m, const double* __restrict__ blk,
                                double* __restrict__ mg, int nvar) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m.nvol * nvar) return;
  const int n = (int)(t / m.nvol);
  const int64_t p = t % m.nvol;
  const int v[3] = {(int)(p % m.nn[0]), (int)((p / m.nn[0]) % m.nn[1]),
                    (int)(p / ((int64_t)m.nn[0] * m.nn[1]))};
  int bl[3], l[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int q = v[a] - NG;
    int b = q < 0 ? 0 : q / g.nx[a];
    if (b > g.nb[a] - 1) b = g.nb[a] - 1;
    bl[a] = b;
    l[a] = v[a] - b * g.nx[a];
  }
  const int64_t bi = ((int64_t)bl[2] * g.nb[1] + bl[1]) * g.nb[0] + bl[0];
  mg[t] = blk[(bi * nvar + n) * g.nvol + ((int64_t)l[2] * g.nn[1] + l[1]) * g.nn[0] + l[0]];
}
// What the block path's ghost fill leaves at local vertex l of the block at
// loc after a step: 0 nothing (the value stays from step to step), 1 the
// value of the merged grid, 2 a copy the exchange took from the owner before
// the owner's extrapolation overwrote it (the upper boundary vertices are
// extrapolated too, physical_bcs.cpp's cell ranges) and that the block's
// own extrapolation passes do not reach: AlgConstr of the last stage's
// output there.  The block's own vertices and the ghosts another block owns
// are written by the exchange; the extrapolation passes (k_bc_axis) write
// the ghosts below a lower face and the boundary vertex and the ghosts above
// an upper face up to nn - 2, within their transverse ranges.
__device__ int block_fill_class(const Grid& g, const int loc[3], const int l[3]) {
  if (g.bc[0] == Z4C_BC_PERIODIC) return 1;  // periodic: the exchange writes every ghost
  bool own = true, held = true, upper = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    own = own && l[a] >= NG && l[a] <= NG + g.nx[a];
    const int G = l[a] + loc[a] * g.nx[a];
    held = held && G >= NG && G <= NG + g.nb[a] * g.nx[a];
    upper = upper || G == NG + g.nb[a] * g.nx[a];
  }
  if (own) return 1;
  bool need[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    need[2 * a] = loc[a] == 0;
    need[2 * a + 1] = loc[a] == g.nb[a] - 1;
  }
  int lo[3], hi[3];
  lo[0] = 0;
  hi[0] = 2 * NG + g.nx[0] - 1;
  lo[1] = need[2] ? NG : 0;
  hi[1] = need[3] ? NG + g.nx[1] - 1 : 2 * NG + g.nx[1] - 1;
  lo[2] = need[4] ? NG : 0;
  hi[2] = need[5] ? NG + g.nx[2] - 1 : 2 * NG + g.nx[2] - 1;
  bool bc = false;
  for (int ax = 0; ax < 3 && !bc; ++ax) {
    const int o1 = ax == 0 ? 1 : 0, o2 = ax == 2 ? 1 : 2;
    int lo2 = lo[o2], hi2 = hi[o2];
    if (ax == 2) {  // the x3 faces take the whole x2 range
      lo2 = 0;
      hi2 = 2 * NG + g.nx[1] - 1;
    }
    if (l[o1] < lo[o1] || l[o1] > hi[o1] || l[o2] < lo2 || l[o2] > hi2) continue;
    bc = (need[2 * ax] && l[ax] < NG) ||
         (need[2 * ax + 1] && l[ax] >= NG + g.nx[ax] && l[ax] <= 2 * NG + g.nx[ax] - 1);
  }
  if (bc) return 1;
  if (held) return upper ? 2 : 1;
  return 0;
}

__device__ __forceinline__ void block_vertex(const Grid& g, int64_t t, int nvar, int& b, int& n,
                                             int loc[3], int l[3]) {
  const int64_t p = t % g.nvol;
  const int64_t bn = t / g.nvol;
  n = (int)(bn % nvar);
  b = (int)(bn / nvar);
  l[0] = (int)(p % g.nn[0]);
  l[1] = (int)((p / g.nn[0]) % g.nn[1]);
  l[2] = (int)(p / ((int64_t)g.nn[0] * g.nn[1]));
  loc[0] = b % g.nb[0];
  loc[1] = (b / g.nb[0]) % g.nb[1];
  loc[2] = b / (g.nb[0] * g.nb[1]);
}

// The class-1 vertices of every block from the merged grid.
__global__ void k_merge_gather(Grid g, Grid m, const double* __restrict__ mg,
                               double* __restrict__ blk, int nvar) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)g.nblocks * nvar * g.nvol) return;
  int b, n, loc[3], l[3];
  block_vertex(g, t, nvar, b, n, loc, l);
  if (block_fill_class(g, loc, l) != 1) return;
  const int I = loc[0] * g.nx[0] + l[0], J = loc[1] * g.nx[1] + l[1], K = loc[2] * g.nx[2] + l[2];
  blk[t] = mg[(int64_t)n * m.nvol + ((int64_t)K * m.nn[1] + J) * m.nn[0] + I];
}

// The class-2 vertices of the u register: the merged grid's last stage
// output at the vertex (mw: the upper boundary planes kept before the
// extrapolation) with AlgConstr applied, as the block that holds the copy
// constrains it after its own extrapolation.
__global__ void k_merge_gather_copies(Grid g, Grid m, DevParams P, const double* __restrict__ mw,
                                      double* __restrict__ u) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)g.nblocks * g.nvol) return;
  int b, n, loc[3], l[3];
  block_vertex(g, t, 1, b, n, loc, l);
  if (block_fill_class(g, loc, l) != 2) return;
  const int I = loc[0] * g.nx[0] + l[0], J = loc[1] * g.nx[1] + l[1], K = loc[2] * g.nx[2] + l[2];
  const double* src = mw + ((int64_t)K * m.nn[1] + J) * m.nn[0] + I;
  double* dst = u + (int64_t)b * NVAR * g.nvol + t % g.nvol;
  double v[NVAR];
#pragma unroll
  for (int q = 0; q < NVAR; ++q) v[q] = src[(int64_t)q * m.nvol];
  alg_constr_point(P.p, v + Z4C_GXX, v + Z4C_AXX, v + Z4C_CHI, v + Z4C_ALPHA);
#pragma unroll
  for (int q = 0; q < NVAR; ++q) dst[(int64_t)q * g.nvol] = v[q];
}

int merge_launch(const z4c_ctx* c, const z4c_ctx* m, int reg, bool to_merged) {
  const int nv = reg_nvar_(reg);
  const int64_t n = to_merged ? m->g.nvol * nv : (int64_t)c->g.nblocks * nv * c->g.nvol;
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (to_merged)
    k_merge_scatter<<<grid, 256, 0, c->stream>>>(c->g, m->g, c->reg[reg], m->reg[reg], nv);
  else
    k_merge_gather<<<grid, 256, 0, c->stream>>>(c->g, m->g, m->reg[reg], c->reg[reg], nv);
  add_kernel_launches(1);
  LAUNCH_CHECK("merge");
  return Z4C_OK;
}

// Steps of z4c_evolve that run on the merged grid: uniform single-level
// meshes whose faces are all outflow or all periodic, on the contracted
// low-storage path.
bool merge_eligible(const z4c_ctx* c) {
  if (!c->merge || !c->shape.contract || c->ml || c->per_block || c->g.nblocks < 2 ||
      c->integrator != Z4C_INTEG_RK4)
    return false;
  const int kind = c->desc.bc[0];
  if (kind != Z4C_BC_OUTFLOW && kind != Z4C_BC_PERIODIC) return false;
  for (int f = 1; f < 6; ++f)
    if (c->desc.bc[f] != kind) return false;
  return true;
}

int merged_evolve(z4c_ctx* c, double dt, int nsteps, int with_constraints) {
  {  // the merged grid lives on the context's device, which must be current
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != c->device)
      return fail(Z4C_EINVAL, "z4c_evolve: device %d is current, the context lives on %d", cur,
                  c->device);
  }
  if (!c->merged) {
    z4c_mesh_desc_t d = c->desc;
    for (int a = 0; a < 3; ++a) {
      d.nx[a] = c->desc.nx[a] * c->desc.nb[a];
      d.nb[a] = 1;
    }
    z4c_ctx* m = nullptr;
    int rc = create_impl(&d, &c->params, c->integrator, 0, nullptr, &m);
    if (rc) return rc;
    m->merge = false;
    // a periodic single block still runs the exchange (with itself)
    m->in_place_fill = c->desc.bc[0] == Z4C_BC_OUTFLOW;
    c->merged = m;
  }
  z4c_ctx* m = c->merged;
  if (m->stream != c->stream) z4c_set_stream(m, c->stream);
  if (m->shape.point_threads != c->shape.point_threads ||
      m->shape.column_threads != c->shape.column_threads ||
      m->shape.column_slabs != c->shape.column_slabs || m->shape.contract != c->shape.contract ||
      m->shape.point_regs != c->shape.point_regs) {
    m->shape = c->shape;
    drop_graph(m);
  }
  if (m->ntrk != c->ntrk) {
    m->ntrk = c->ntrk;
    drop_graph(m);
  }
  int rc;
  if (c->ntrk > 0)
    CUDA_TRY(cudaMemcpyAsync(m->trk, c->trk, sizeof(double) * 8 * c->ntrk,
                             cudaMemcpyDeviceToDevice, c->stream));
  if ((rc = merge_launch(c, m, Z4C_REG_U, true))) return rc;
  // the constraints are evaluated on the blocks below, not on the merged grid
  if ((rc = z4c_evolve(m, dt, nsteps, 0))) return rc;
  if ((rc = merge_launch(c, m, Z4C_REG_U, false))) return rc;
  {
    const int64_t n = (int64_t)c->g.nblocks * c->g.nvol;
    k_merge_gather_copies<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        c->g, m->g, c->dev(), m->reg[Z4C_REG_RHS], c->reg[Z4C_REG_U]);
    add_kernel_launches(1);
    LAUNCH_CHECK("merge");
  }
  // the ADM variables and the constraints of the final state, on the blocks,
  // as the block path leaves them
  const DevParams P = c->dev();
  launch_z4c_to_adm(c->g, P, c->reg[Z4C_REG_U], c->reg[Z4C_REG_ADM], 0, c->g.nblocks, c->stream);
  LAUNCH_CHECK("z4c_to_adm");
  if (with_constraints) {
    launch_adm_constraints(c->g, P, c->reg[Z4C_REG_ADM], c->reg[Z4C_REG_U],
                           c->reg[Z4C_REG_CON], c->xf, 0, c->g.nblocks, c->stream);
    LAUNCH_CHECK("constraints");
  }
  if (c->ntrk > 0)
    CUDA_TRY(cudaMemcpyAsync(c->trk, m->trk, sizeof(double) * 8 * c->ntrk,
                             cudaMemcpyDeviceToDevice, c->stream));
  return Z4C_OK;
}
}  // namespace

int z4c_evolve(z4c_ctx* ctx, double dt, int nsteps, int with_constraints) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (nsteps < 0) return fail(Z4C_EINVAL, "negative step count");
  if (nsteps > 0 && merge_eligible(ctx)) return merged_evolve(ctx, dt, nsteps, with_constraints);
  // The four stages of a step, captured once into a graph and replayed.  The
  // register pointers inside the graph are fixed: a step leaves u in the same
  // buffer it started from (exchange writes back into u), so replays are
  // valid until a ghost fill swaps the registers (which drops the graph).
  if (nsteps > 0 && (!ctx->graph || ctx->graph_dt != dt || ctx->graph_per_block != ctx->per_block)) {
    if (ctx->graph) {
      cudaGraphExecDestroy(ctx->graph);
      ctx->graph = nullptr;
    }
    double* u_before = ctx->reg[Z4C_REG_U];
    const long long count_before = kernel_launch_count();
    cudaGraph_t graph;
    CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = Z4C_OK;
    for (int s = 1; s <= 4 && rc == Z4C_OK; ++s) rc = run_stage(ctx, s, dt);
    cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc) return rc;
    if (ec != cudaSuccess) return fail(Z4C_ECUDA, "end capture: %s", cudaGetErrorString(ec));
    if (ctx->reg[Z4C_REG_U] != u_before) {
      // per-block path swaps u/w each stage: 4 swaps return to the start
      cudaGraphDestroy(graph);
      return fail(Z4C_ESTATE, "captured step does not return u to its buffer");
    }
    // capture records kernels without running them
    ctx->graph_nodes = kernel_launch_count() - count_before;
    add_kernel_launches(-ctx->graph_nodes);
    ec = cudaGraphInstantiate(&ctx->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ec != cudaSuccess) return fail(Z4C_ECUDA, "graph instantiate: %s", cudaGetErrorString(ec));
    ctx->graph_dt = dt;
    ctx->graph_per_block = ctx->per_block;
  }
  for (int n = 0; n < nsteps; ++n) {
    CUDA_TRY(cudaGraphLaunch(ctx->graph, ctx->stream));
    add_kernel_launches(ctx->graph_nodes);
  }
  if (with_constraints) {
    const DevParams P = ctx->dev();
    // the captured step already ran Z4cToADM on its last stage
    if (nsteps == 0)
      launch_z4c_to_adm(ctx->g, P, ctx->reg[Z4C_REG_U], ctx->reg[Z4C_REG_ADM], 0, ctx->g.nblocks,
                        ctx->stream);
    launch_adm_constraints(ctx->g, P, ctx->reg[Z4C_REG_ADM], ctx->reg[Z4C_REG_U],
                           ctx->reg[Z4C_REG_CON], ctx->xf, 0, ctx->g.nblocks, ctx->stream);
    LAUNCH_CHECK("constraints");
  }
  return Z4C_OK;
}

long long z4c_kernel_launches(void) { return kernel_launch_count(); }

namespace {
// Staging of z4c_evolve_jobs, allocated once per context.
int jobs_setup(z4c_ctx* c) {
  if (c->jobs) return Z4C_OK;
  JobPipe* J = new JobPipe;
  c->jobs = J;  // released by free_ctx whatever happens below
  const size_t reg = sizeof(double) * (size_t)reg_elems(c, Z4C_REG_U);
  const size_t part = sizeof(double) * 8 * (size_t)c->g.nblocks;
  for (int k = 0; k < 2; ++k) {
    CUDA_TRY(cudaMalloc(&J->in[k], reg));
    CUDA_TRY(cudaMalloc(&J->out[k], reg));
    CUDA_TRY(cudaMalloc(&J->part[k], part));
    CUDA_TRY(cudaMallocHost(&J->hpart[k], part));
    for (cudaEvent_t* e : {&J->in_ready[k], &J->in_free[k], &J->out_ready[k], &J->out_free[k]})
      CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&J->h2d, cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamCreateWithFlags(&J->d2h, cudaStreamNonBlocking));
  return Z4C_OK;
}

// Issues job j: its evolution and history partials on the context's stream,
// the download of its result on the download stream.
int jobs_issue(z4c_ctx* c, int j, double* host_out, double dt, int nsteps) {
  JobPipe* J = c->jobs;
  const int s = j & 1;
  const size_t reg = sizeof(double) * (size_t)reg_elems(c, Z4C_REG_U);
  const size_t part = sizeof(double) * 8 * (size_t)c->g.nblocks;
  CUDA_TRY(cudaStreamWaitEvent(c->stream, J->in_ready[s], 0));
  CUDA_TRY(cudaMemcpyAsync(c->reg[Z4C_REG_U], J->in[s], reg, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaEventRecord(J->in_free[s], c->stream));
  int rc = z4c_evolve(c, dt, nsteps, 1);
  if (rc) return rc;
  launch_hst(c->g, c->dev(), c->reg[Z4C_REG_CON], c->reg[Z4C_REG_U], c->xv, c->partials, c->stream);
  LAUNCH_CHECK("hst");
  // the output slot is free once the download of job j - 2 has left it
  CUDA_TRY(cudaStreamWaitEvent(c->stream, J->out_free[s], 0));
  if (host_out)
    CUDA_TRY(cudaMemcpyAsync(J->out[s], c->reg[Z4C_REG_U], reg, cudaMemcpyDeviceToDevice,
                             c->stream));
  CUDA_TRY(cudaMemcpyAsync(J->part[s], c->partials, part, cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaEventRecord(J->out_ready[s], c->stream));
  CUDA_TRY(cudaStreamWaitEvent(J->d2h, J->out_ready[s], 0));
  if (host_out)
    CUDA_TRY(cudaMemcpyAsync(host_out, J->out[s], reg, cudaMemcpyDeviceToHost, J->d2h));
  CUDA_TRY(cudaMemcpyAsync(J->hpart[s], J->part[s], part, cudaMemcpyDeviceToHost, J->d2h));
  CUDA_TRY(cudaEventRecord(J->out_free[s], J->d2h));
  return Z4C_OK;
}

// Issues the upload of job j into its input slot, after the evolution of
// job j - 2 has copied that slot out.  partial: the steps run on the merged
// grid, whose copy from the blocks reads, of a block not on a z face of the
// mesh, only the vertex planes k = NG .. NG + nx; those blocks' planes go up
// as one pitched copy (the other planes of the slot keep older values, which
// nothing reads), the blocks on the z faces whole.
int jobs_upload(z4c_ctx* c, int j, const double* host_in, bool partial) {
  JobPipe* J = c->jobs;
  const int s = j & 1;
  const size_t reg = sizeof(double) * (size_t)reg_elems(c, Z4C_REG_U);
  CUDA_TRY(cudaStreamWaitEvent(J->h2d, J->in_free[s], 0));
  if (!partial) {
    CUDA_TRY(cudaMemcpyAsync(J->in[s], host_in, reg, cudaMemcpyHostToDevice, J->h2d));
  } else {
    const Grid& g = c->g;
    const size_t per = (size_t)Z4C_NVAR * g.nvol;             // values per block
    const size_t layer = (size_t)g.nb[0] * g.nb[1];            // blocks per z layer
    const size_t plane = (size_t)g.nn[0] * g.nn[1];            // values per vertex plane
    const size_t top = layer * (g.nb[2] - 1);                  // first block of the top layer
    CUDA_TRY(cudaMemcpyAsync(J->in[s], host_in, sizeof(double) * per * layer,
                             cudaMemcpyHostToDevice, J->h2d));
    const size_t off = per * layer + plane * NG;
    CUDA_TRY(cudaMemcpy2DAsync(J->in[s] + off, sizeof(double) * g.nvol, host_in + off,
                               sizeof(double) * g.nvol, sizeof(double) * plane * (g.nx[2] + 1),
                               (top - layer) * Z4C_NVAR, cudaMemcpyHostToDevice, J->h2d));
    CUDA_TRY(cudaMemcpyAsync(J->in[s] + per * top, host_in + per * top,
                             sizeof(double) * per * layer, cudaMemcpyHostToDevice, J->h2d));
  }
  CUDA_TRY(cudaEventRecord(J->in_ready[s], J->h2d));
  return Z4C_OK;
}
}  // namespace

// History norms of job j from the page-locked partials of its slot, summed
// as z4c_hst_norms sums them; waits for the slot's download.
static int jobs_hst(z4c_ctx* c, int j, double* hst_out) {
  JobPipe* J = c->jobs;
  CUDA_TRY(cudaEventSynchronize(J->out_free[j & 1]));
  if (!hst_out) return Z4C_OK;
  double* o = hst_out + (size_t)8 * j;
  const double* h = J->hpart[j & 1];
  for (int q = 0; q < 8; ++q) o[q] = 0.0;
  for (int b = 0; b < c->g.nblocks; ++b) {
    const double* dx = &c->h_dx[(size_t)b * 3];
    const double vol = dx[0] * dx[1] * dx[2];
    for (int q = 0; q < 8; ++q) o[q] += vol * h[(size_t)b * 8 + q];
  }
  return Z4C_OK;
}

int z4c_evolve_jobs(z4c_ctx* ctx, int njobs, const double* const* host_in,
                    double* const* host_out, double* hst_out, double dt, int nsteps) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  if (njobs < 1 || !host_in) return fail(Z4C_EINVAL, "need njobs >= 1 and the input array");
  if (nsteps < 0) return fail(Z4C_EINVAL, "negative step count");
  for (int j = 0; j < njobs; ++j)
    if (!host_in[j] || (host_out && !host_out[j]))
      return fail(Z4C_EINVAL, "null host buffer of job %d", j);
  {  // the staging and copy streams live on the context's device
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != ctx->device)
      return fail(Z4C_EINVAL, "z4c_evolve_jobs: device %d is current, the context lives on %d",
                  cur, ctx->device);
  }
  int rc = jobs_setup(ctx);
  if (rc) return rc;
  JobPipe* J = ctx->jobs;
  // norms only, on a merged grid of three or more block layers in z: the
  // planes the merged grid reads
  const bool partial = !host_out && merge_eligible(ctx) && ctx->g.nb[2] > 2;
  // upload j + 1 is issued before evolution j, so that it runs beside it;
  // download j is issued right after it and runs beside evolution j + 1.
  // Job j reuses the slots of job j - 2, whose partials are summed first.
  rc = jobs_upload(ctx, 0, host_in[0], partial);
  int summed = 0;  // jobs whose history norms are taken
  for (int j = 0; j < njobs && rc == Z4C_OK; ++j) {
    if (j + 1 < njobs) rc = jobs_upload(ctx, j + 1, host_in[j + 1], partial);
    if (rc == Z4C_OK && j >= 2) rc = jobs_hst(ctx, summed++, hst_out);
    if (rc == Z4C_OK) rc = jobs_issue(ctx, j, host_out ? host_out[j] : nullptr, dt, nsteps);
  }
  // every job has finished (or failed) before the buffers are handed back
  const cudaError_t e1 = cudaStreamSynchronize(J->h2d);
  const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
  const cudaError_t e3 = cudaStreamSynchronize(J->d2h);
  if (rc) return rc;
  for (cudaError_t e : {e1, e2, e3})
    if (e != cudaSuccess) return fail(Z4C_ECUDA, "evolve_jobs: %s", cudaGetErrorString(e));
  while (summed < njobs)
    if ((rc = jobs_hst(ctx, summed++, hst_out))) return rc;
  return Z4C_OK;
}


namespace {
// {level, lx1, lx2, lx3} of every block of a context in its block order
std::vector<long long> ctx_locs(const z4c_ctx* c) {
  if (c->ml) return c->locs;
  const int rl = ml_root_level(c->desc.nb);
  std::vector<long long> l((size_t)4 * c->g.nblocks);
  for (int b = 0; b < c->g.nblocks; ++b) {
    l[4 * (size_t)b] = rl;
    l[4 * (size_t)b + 1] = b % c->g.nb[0];
    l[4 * (size_t)b + 2] = (b / c->g.nb[0]) % c->g.nb[1];
    l[4 * (size_t)b + 3] = b / (c->g.nb[0] * c->g.nb[1]);
  }
  return l;
}
}  // namespace

int z4c_regrid(z4c_ctx* dst, const z4c_ctx* src) {
  if (!dst || !src) return fail(Z4C_EINVAL, "null context");
  // the kernels below run on dst's stream and read src's registers directly:
  // both contexts must live on the current device
  {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) {
      cudaGetLastError();
      return fail(Z4C_ECUDA, "regrid: no current device");
    }
    if (src->device != dst->device || cur != dst->device)
      return fail(Z4C_EINVAL, "regrid: contexts on devices %d (src) and %d (dst), current "
                              "device %d; both must be on the current device",
                  src->device, dst->device, cur);
  }
  for (int a = 0; a < 3; ++a)
    if (dst->desc.nb[a] != src->desc.nb[a] || dst->desc.nx[a] != src->desc.nx[a] ||
        dst->desc.xmin[a] != src->desc.xmin[a] || dst->desc.xmax[a] != src->desc.xmax[a])
      return fail(Z4C_EINVAL, "regrid: the contexts cover different root grids");
  const std::vector<long long> dl = ctx_locs(dst), sl = ctx_locs(src);
  std::map<std::tuple<long long, long long, long long, long long>, int> sidx;
  for (int b = 0; b < src->g.nblocks; ++b)
    sidx[std::make_tuple(sl[4 * b], sl[4 * b + 1], sl[4 * b + 2], sl[4 * b + 3])] = b;
  // every destination block: the same block, a child of a source block or
  // the parent of eight source blocks (one level per regrid, as the reference)
  struct Move { int kind, from[8], oct[8][3]; };
  std::vector<Move> moves((size_t)dst->g.nblocks);
  for (int b = 0; b < dst->g.nblocks; ++b) {
    const long long lv = dl[4 * b], x = dl[4 * b + 1], y = dl[4 * b + 2], z = dl[4 * b + 3];
    Move& m = moves[b];
    auto it = sidx.find(std::make_tuple(lv, x, y, z));
    if (it != sidx.end()) { m.kind = 0; m.from[0] = it->second; continue; }
    it = sidx.find(std::make_tuple(lv - 1, x >> 1, y >> 1, z >> 1));
    if (it != sidx.end()) {
      m.kind = 1;
      m.from[0] = it->second;
      m.oct[0][0] = (int)(x & 1); m.oct[0][1] = (int)(y & 1); m.oct[0][2] = (int)(z & 1);
      continue;
    }
    m.kind = 2;
    for (int c = 0; c < 8; ++c) {
      const int o[3] = {c & 1, (c >> 1) & 1, (c >> 2) & 1};
      it = sidx.find(std::make_tuple(lv + 1, 2 * x + o[0], 2 * y + o[1], 2 * z + o[2]));
      if (it == sidx.end())
        return fail(Z4C_EINVAL, "regrid: block %d is neither kept, refined nor derefined "
                                "by one level", b);
      m.from[c] = it->second;
      for (int a = 0; a < 3; ++a) m.oct[c][a] = o[a];
    }
  }
  double* scratch = nullptr;
  const int64_t cvol = (int64_t)(dst->g.nx[0] / 2 + 1 + 2 * Z4C_NCG) *
                       (dst->g.nx[1] / 2 + 1 + 2 * Z4C_NCG) * (dst->g.nx[2] / 2 + 1 + 2 * Z4C_NCG);
  if (cudaMalloc((void**)&scratch, sizeof(double) * Z4C_NVAR * cvol) != cudaSuccess) {
    cudaGetLastError();
    return fail(Z4C_ENOMEM, "regrid: coarse scratch");
  }
  // the source's work must be complete before the destination's stream reads it
  if (cudaStreamSynchronize(src->stream) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(scratch);
    return fail(Z4C_ECUDA, "regrid: earlier work on the source context failed");
  }
  const int64_t bs = (int64_t)Z4C_NVAR * dst->g.nvol;
  const double* su = src->reg[Z4C_REG_U];
  double* du = dst->reg[Z4C_REG_U];
  int rc = Z4C_OK;
  for (int b = 0; b < dst->g.nblocks && rc == Z4C_OK; ++b) {
    const Move& m = moves[b];
    if (m.kind == 0) {
      if (cudaMemcpyAsync(du + b * bs, su + m.from[0] * bs, sizeof(double) * bs,
                          cudaMemcpyDeviceToDevice, dst->stream) != cudaSuccess)
        rc = fail(Z4C_ECUDA, "regrid: block copy");
    } else if (m.kind == 1) {
      rc = z4c_regrid_refine(su + m.from[0] * bs, du + b * bs, scratch, Z4C_NVAR, dst->g.nx,
                             m.oct[0], dst->stream);
    } else {
      for (int c = 0; c < 8 && rc == Z4C_OK; ++c)
        rc = z4c_regrid_derefine(su + m.from[c] * bs, du + b * bs, scratch, Z4C_NVAR, dst->g.nx,
                                 m.oct[c], dst->stream);
    }
  }
  // the puncture trackers move with the state
  if (rc == Z4C_OK && src->ntrk > 0 &&
      cudaMemcpyAsync(dst->trk, src->trk, sizeof(double) * 8 * src->ntrk,
                      cudaMemcpyDeviceToDevice, dst->stream) != cudaSuccess)
    rc = fail(Z4C_ECUDA, "regrid: trackers");
  if (cudaStreamSynchronize(dst->stream) != cudaSuccess && rc == Z4C_OK) {
    cudaGetLastError();
    rc = fail(Z4C_ECUDA, "regrid: transfer into the destination context failed");
  }
  cudaFree(scratch);
  if (rc) return rc;
  dst->ntrk = src->ntrk;
  drop_graph(dst);
  return Z4C_OK;
}

int z4c_tracker_add(z4c_ctx* ctx, const double pos[3], int* id) {
  if (!ctx || !pos || !id) return fail(Z4C_EINVAL, "null argument");
  if (ctx->ntrk >= kMaxTrackers) return fail(Z4C_EINVAL, "at most %d trackers", kMaxTrackers);
  const double rec[8] = {pos[0], pos[1], pos[2], NAN, NAN, NAN, 0.0, 0.0};
  CUDA_TRY(cudaMemcpyAsync(ctx->trk + 8 * ctx->ntrk, rec, sizeof(rec), cudaMemcpyHostToDevice,
                           ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *id = ctx->ntrk++;
  drop_graph(ctx);  // the captured step must include the new tracker
  return Z4C_OK;
}

int z4c_restart_load(z4c_ctx* ctx, const char* path, z4c_restart_info_t* info_out) {
  if (!ctx || !path) return fail(Z4C_EINVAL, "null argument");
  z4c_restart_info_t info;
  std::string text, err;
  std::vector<double> u;
  std::vector<long long> locs;
  int rc = restart_read_file(path, &info, &text, &u, &err, &locs);
  if (rc) return fail(rc, "%s", err.c_str());
  for (int a = 0; a < 3; ++a)
    if (info.nb[a] != ctx->desc.nb[a] || info.block_nx[a] != ctx->g.nx[a] ||
        info.xmin[a] != ctx->desc.xmin[a] || info.xmax[a] != ctx->desc.xmax[a])
      return fail(Z4C_EINVAL, "restart file %s holds another mesh than this context's", path);
  if ((info.nlevels > 1) != (ctx->ml != nullptr) || (ctx->ml && locs != ctx->locs))
    return fail(Z4C_EINVAL, "restart file %s holds other MeshBlocks than this context's", path);
  if (ctx->ntrk != 0 && ctx->ntrk != info.ntrackers)
    return fail(Z4C_ESTATE, "the context has %d trackers, the restart file %d", ctx->ntrk,
                info.ntrackers);
  CUDA_TRY(cudaMemcpyAsync(ctx->reg[Z4C_REG_U], u.data(), sizeof(double) * u.size(),
                           cudaMemcpyHostToDevice, ctx->stream));
  for (int t = 0; t < info.ntrackers; ++t) {
    const double* r = info.trackers[t];
    const double rec[8] = {r[0], r[1], r[2], r[3], r[4], r[5], 0.0, 0.0};
    CUDA_TRY(cudaMemcpyAsync(ctx->trk + 8 * t, rec, sizeof(rec), cudaMemcpyHostToDevice,
                             ctx->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->ntrk = info.ntrackers;
  drop_graph(ctx);
  if (info_out) *info_out = info;
  return Z4C_OK;
}

int z4c_restart_save(z4c_ctx* ctx, const char* path, const char* par_text, double time,
                     double dt, int ncycle) {
  if (!ctx || !path) return fail(Z4C_EINVAL, "null argument");
  std::vector<double> u((size_t)reg_elems(ctx, Z4C_REG_U));
  std::vector<double> trk((size_t)8 * (ctx->ntrk > 0 ? ctx->ntrk : 1));
  CUDA_TRY(cudaMemcpyAsync(u.data(), ctx->reg[Z4C_REG_U], sizeof(double) * u.size(),
                           cudaMemcpyDeviceToHost, ctx->stream));
  if (ctx->ntrk > 0)
    CUDA_TRY(cudaMemcpyAsync(trk.data(), ctx->trk, sizeof(double) * 8 * ctx->ntrk,
                             cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  std::vector<double> t6((size_t)6 * (ctx->ntrk > 0 ? ctx->ntrk : 1));
  for (int t = 0; t < ctx->ntrk; ++t)
    for (int q = 0; q < 6; ++q) t6[6 * t + q] = trk[8 * t + q];
  std::string err;
  const int rc = restart_write_file(path, par_text ? par_text : "", ctx->desc, u.data(), time, dt,
                                    ncycle, ctx->ntrk, t6.data(), &err,
                                    ctx->ml ? ctx->locs.data() : nullptr, ctx->g.nblocks);
  if (rc) return fail(rc, "%s", err.c_str());
  return Z4C_OK;
}

int z4c_tracker_get(z4c_ctx* ctx, int id, double out[6]) {
  if (!ctx || !out) return fail(Z4C_EINVAL, "null argument");
  if (id < 0 || id >= ctx->ntrk) return fail(Z4C_EINVAL, "no tracker %d", id);
  double rec[8];
  CUDA_TRY(cudaMemcpyAsync(rec, ctx->trk + 8 * id, sizeof(rec), cudaMemcpyDeviceToHost,
                           ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int q = 0; q < 6; ++q) out[q] = rec[q];
  if (rec[6] != 0.0) return fail(Z4C_ESTATE, "puncture %d has left the grid", id);
  return Z4C_OK;
}

int z4c_check_finite(z4c_ctx* ctx, int reg) {
  if (!ctx) return fail(Z4C_EINVAL, "null context");
  int rc;
  if ((rc = check_reg(ctx, reg))) return rc;
  CUDA_TRY(cudaMemsetAsync(ctx->flag, 0, sizeof(int), ctx->stream));
  launch_check_finite(ctx->g, ctx->reg[reg], reg_nvar_(reg), ctx->flag, ctx->stream);
  LAUNCH_CHECK("check_finite");
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, ctx->flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return h ? fail(Z4C_ENONFINITE, "register %d holds NaN/Inf", reg) : Z4C_OK;
}

}  // extern "C"

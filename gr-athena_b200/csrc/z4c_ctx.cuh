// The context behind the C ABI's z4c_ctx handle, shared by the translation
// units that implement entry points on it (z4c_capi.cu, z4c_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/z4c_b200.h"
#include "z4c_common.cuh"
#include "z4c_kernels.cuh"
#include "z4c_multilevel.cuh"
#include "z4c_wave.cuh"

namespace z4c {
struct AdjState;
// Releases the tangent-linear / adjoint buffers of a context (z4c_adjoint.cu).
void adj_free(AdjState* a);

// Low-storage RK4()4[2S] (task_list_integrators_low_storage.cpp:112-142).
constexpr double kLsRk4[4][5] = {
    {1.0, 0.0, 1.0, 0.0, 1.193743905974738},
    {0.217683334308543, 0.121098479554482, 0.721781678111411, 0.0, 0.099279895495783},
    {1.065841341361089, -3.843833699660025, 2.121209265338722, 0.0, 1.131678018054042},
    {0.0, 0.546370891121863, 0.198653035682705, 0.0, 0.310665766509336}};
// Classical RK4 tableau (task_list_integrators_butcher.cpp:37-48).
constexpr double kBtA[4][4] = {{0, 0, 0, 0}, {0.5, 0, 0, 0}, {0, 0.5, 0, 0}, {0, 0, 1, 0}};
constexpr double kBtB[4] = {1. / 6., 1. / 3., 1. / 3., 1. / 6.};
}  // namespace z4c

using namespace z4c;

// Device staging and copy streams of z4c_evolve_jobs (allocated on its first
// call): two input and two output registers and per-block history partials,
// so that the copies of one job overlap the evolution of the next.
struct JobPipe {
  double* in[2] = {};
  double* out[2] = {};
  double* part[2] = {};
  double* hpart[2] = {};  // page-locked host copies of part
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_free[2] = {};
};

struct z4c_ctx {
  Grid g{};
  MlPlan* ml = nullptr;         // multilevel meshes: the ghost-exchange plan
  unsigned char* som = nullptr; // multilevel meshes: gr_sommerfeld faces per block (device)
  std::vector<long long> locs;  // multilevel meshes: {level, lx1, lx2, lx3} per block
  z4c_mesh_desc_t desc{};
  z4c_params_t params{};
  int integrator = Z4C_INTEG_RK4;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool per_block = false;
  LaunchShape shape;  // launch shape of the RHS passes (autotuner output)
  bool has_outflow = false;

  // device buffers
  double* reg[Z4C_NREG] = {};
  double* un = nullptr;   // Butcher u_n scratch
  double* guu = nullptr;  // ADMToZ4c inverse-metric scratch (6 vars)
  double* sd = nullptr;   // stored first derivatives, 33 values per vertex
  double* rsum = nullptr; // Ricci-pass scratch, 6 values per interior vertex
  double* lv = nullptr;   // advection sums, 22 values per interior vertex
  double* xf = nullptr;   // [nblocks][nn0+nn1+nn2]
  double* xv = nullptr;   // [nblocks][nn0+nn1+nn2-3]
  double* dxd = nullptr;  // [nblocks][3] vertex spacing
  FdScale* fd = nullptr;  // [nblocks]
  int* nbr = nullptr;     // [nblocks][26]
  double* partials = nullptr;
  double* trk = nullptr;  // puncture trackers [kMaxTrackers][8]
  int ntrk = 0;
  int* flag = nullptr;
  std::vector<WaveSphere> waves;  // psi4 extraction spheres
  z4c::AdjState* adj = nullptr;   // tangent-linear / adjoint buffers (z4c_adj_setup)
  JobPipe* jobs = nullptr;        // z4c_evolve_jobs staging
  // Uniform meshes on the contracted path: z4c_evolve runs the steps on one
  // vertex grid holding every block (merged, created on first use); merge
  // switches it (z4c_set_merged).
  z4c_ctx* merged = nullptr;
  bool merge = true;
  // The merged grid itself (one block, every face extrapolated): a stage's
  // fill runs on the stage output, which then becomes u (u and w swap; the
  // four stages of a step return u to its buffer).
  bool in_place_fill = false;

  // host copies
  std::vector<double> h_xf, h_xv, h_dx;  // h_dx: [nblocks][3]

  // kernel nodes of the captured step (graph replays add this many launches)
  long long graph_nodes = 0;

  // captured step
  cudaGraphExec_t graph = nullptr;
  double graph_dt = 0.0;
  bool graph_per_block = false;

  RhsScratch scratch() const { return RhsScratch{sd, rsum, lv}; }

  DevParams dev() const {
    DevParams P;
    P.p = params;
    P.fd = fd;
    P.xf = xf;
    P.dx = dxd;
    P.som = som;
    return P;
  }
};

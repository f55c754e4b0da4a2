// Device kernels of the Z4c path.  Each kernel cites the reference routine it
// replaces; the pointwise arithmetic lives in z4c_common.cuh / z4c_rhs.cuh /
// z4c_adm.cuh.
#pragma once

#include "z4c_common.cuh"

namespace z4c {

// Register view: base pointer, variables per block.
struct Reg {
  double* p;
  int nvar;
  __device__ __forceinline__ double* block(const Grid& g, int b) const {
    return p + (int64_t)b * nvar * g.nvol;
  }
};

// LS stage weights (task_list_integrators_low_storage.cpp:112-142) with the
// step already scaled: beta_dt = beta * dt (time_integrators.hpp:37-40).
// u1_zero: u1 is known to be zero (stage 1 after the task list's u1 = 0,
// task_list_gr_z4c.cpp:115-119), so the kernel does not read it.
struct LsStage {
  double delta, gamma1, gamma2, gamma3, beta_dt;
  int u1_zero;
};

// Butcher stage: u_out = u_n + sum_{q < nq} coef[q] * k_q, coef = a*dt or b*dt
// (task_list_integrators_butcher.cpp:580-680); zero coefficients skipped.
struct BtStage {
  double coef[4];
  int nq;      // number of slopes summed (stage+1 for SumBT_ak, 4 for SumBT_bk)
  int kslot;   // which K register receives this stage's RHS
};

// Interior vertex l of a block -> (i, j, k).
__device__ __forceinline__ void interior_ijk(const Grid& g, int64_t l, int& i, int& j, int& k) {
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1;
  i = NG + (int)(l % n0);
  j = NG + (int)((l / n0) % n1);
  k = NG + (int)(l / ((int64_t)n0 * n1));
}

__host__ __device__ __forceinline__ int64_t interior_count(const Grid& g) {
  return (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
}

// ---- launchers (host side) ----------------------------------------------

// Process-wide count of kernels launched by the launchers below.
long long kernel_launch_count();
void add_kernel_launches(long long n);

// All launches return cudaGetLastError() mapped by the caller.
// Scratch of the right-hand-side passes, indexed by absolute block:
// sd [block][33][vertex] (stored first derivatives of chi, g~, alpha, beta
// along x, y, z), rsum [block][6][interior vertex] (R_ab + Rphi_ab),
// lv [block][22][interior vertex] (advection sums).
struct RhsScratch {
  double* sd;
  double* rsum;
  double* lv;
};
constexpr int kSdComponents = 33;

// Launch shape of the right-hand-side passes: threads per CTA of the heavy
// per-vertex passes (64, 128, 256), threads per CTA of the per-variable
// passes (128, 256, 512) and the number of z-slabs per block in which those
// passes stage a variable in shared memory (1-4; 0 or a slab whose planes do
// not fit: global-memory pencils instead).
// contract: the contracted path (z4c_fast.cu) on meshes without
// gr_sommerfeld faces: floating-point contraction, and the advection sums,
// the Kreiss-Oliger terms and the stage update in one per-variable column
// pass after the main pass; the right-hand side agrees with the exact path to
// round-off instead of bit for bit.
// point_regs: register budget of the heavy per-vertex passes on fixed-geometry
// meshes: 0 (up to 255 per thread, two CTAs of 128 per SM) or
// kPointRegsHigh (168: three CTAs of 128 or six of 64 per SM, 1.5x the
// resident warps); point_threads 256 always takes 255.
constexpr int kPointRegsHigh = 168;
struct LaunchShape {
  int point_threads = 128;
  int column_threads = 128;
  int column_slabs = 0;
  int contract = 0;
  int point_regs = 0;
};
bool valid_shape(const LaunchShape& sh);
// Whether the shape's slabs fit in shared memory on this grid.
bool slabs_fit(const Grid& g, const LaunchShape& sh);
// Raises the dynamic shared-memory limit of the slab kernels (call once per
// device before the first launch, outside stream capture); returns a
// cudaError_t value.
int allow_slab_smem();

// Every RHS launch runs five kernels: stored first derivatives, Ricci pass,
// advection sums, main pass (into rhs, without Kreiss-Oliger), then
// Kreiss-Oliger fused with the consumer: in place for launch_rhs, with the
// stage update for the stage launches (rhs then holds the pre-dissipation
// right-hand side).
void launch_rhs(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                double* rhs, int block0, int nblk, const LaunchShape& sh, cudaStream_t st);
// The first two passes alone: the stored first derivatives of u into sc.sd
// and the Ricci sums into sc.rsum (the linearisation point of the adjoint),
// or the stored first derivatives alone into sd.
void launch_prep_ricci(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                       int block0, int nblk, const LaunchShape& sh, cudaStream_t st);
void launch_prep(const Grid& g, const DevParams& P, const double* u, double* sd, int block0,
                 int nblk, cudaStream_t st);
void launch_stage_ls(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                     double* rhs, double* u1, double* u_out, const LsStage& w, int block0,
                     int nblk, const LaunchShape& sh, cudaStream_t st);
// The contracted path (LaunchShape::contract): four launches, stored first
// derivatives (exact), Ricci, the main pass into rhs without the advection
// sums and Kreiss-Oliger, then one column pass that adds both and runs the
// stage update (launch_stage_ls_fast) or writes the right-hand side back
// (launch_rhs_fast).  Not for meshes with gr_sommerfeld faces (the launchers
// above fall back to the exact path).
void launch_stage_ls_fast(const Grid& g, const DevParams& P, const double* u,
                          const RhsScratch& sc, double* rhs, double* u1, double* u_out,
                          const LsStage& w, int block0, int nblk, const LaunchShape& sh,
                          cudaStream_t st);
void launch_rhs_fast(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                     double* rhs, int block0, int nblk, const LaunchShape& sh, cudaStream_t st);
void launch_stage_bt(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                     double* rhs, const double* un, double* const* k, double* u_out,
                     const BtStage& w, int block0, int nblk, const LaunchShape& sh,
                     cudaStream_t st);
// Ghost exchange of a 22-variable register: src (pre-exchange) -> dst (all
// vertices); src and dst must differ.
// Puncture trackers (records of 8 doubles: pos, betap, lost flag): the
// shift interpolated at each puncture, and pos -= dt * betap.
constexpr int kMaxTrackers = 8;
void launch_track_interp(const Grid& g, const DevParams& P, const double* u, double* trk,
                         int ntrk, cudaStream_t st);
void launch_track_update(double* trk, int ntrk, double dt, cudaStream_t st);
// Z4c::Z4cBoundaryRHS: Sommerfeld right-hand side on gr_sommerfeld faces.
void launch_boundary_rhs(const Grid& g, const DevParams& P, const double* u, double* rhs,
                         int block0, int nblk, cudaStream_t st);
// AlgConstr after the boundary conditions for an exchange run with
// fuse_alg = 2: the blocks that touch a physical face, except the ghosts
// they copied from blocks constrained in the exchange.
void launch_alg_constr_boundary(const Grid& g, const DevParams& P, double* u, const int* nbr,
                                cudaStream_t st);
void launch_exchange(const Grid& g, const DevParams& P, const double* src, double* dst,
                     const int* nbr, int fuse_alg, cudaStream_t st, int nvar = NVAR);
void launch_physical_bcs(const Grid& g, double* u, int nvar, cudaStream_t st);
void launch_alg_constr(const Grid& g, const DevParams& P, double* u, int block0, int nblk,
                       cudaStream_t st, int ghosts_only = 0);
void launch_weighted_ave(const Grid& g, double* out, const double* in1, const double* in2,
                         const double w[3], int block0, int nblk, cudaStream_t st);
void launch_add_rhs(const Grid& g, const double* rhs, double wght, double* out, int block0,
                    int nblk, cudaStream_t st);
void launch_z4c_to_adm(const Grid& g, const DevParams& P, const double* u, double* adm,
                       int block0, int nblk, cudaStream_t st, int ghosts_only = 0);
// alg = 0 leaves out the final AlgConstr (the adjoint's recomputation)
void launch_adm_to_z4c(const Grid& g, const DevParams& P, const double* adm, double* u,
                       double* guu_scratch, int block0, int nblk, cudaStream_t st, int alg = 1);
void launch_adm_constraints(const Grid& g, const DevParams& P, const double* adm,
                            const double* u, double* con, const double* xf, int block0,
                            int nblk, cudaStream_t st);
// Z4cWeyl on blocks [block0, block0+nblk): the stored first derivatives of u
// into sd (k_prep), the curvature terms into the scratch rs (6 values per
// interior vertex) and ks (22), then psi4 (2 variables) into weyl.
void launch_weyl(const Grid& g, const DevParams& P, const double* adm, const double* u,
                 double* sd, double* rs, double* ks, double* weyl, const double* xf, int block0,
                 int nblk, cudaStream_t st);
void launch_hst(const Grid& g, const DevParams& P, const double* con, const double* u,
                const double* xv, double* partials, cudaStream_t st);
void launch_check_finite(const Grid& g, const double* u, int nvar, int* flag, cudaStream_t st);
void launch_zero_interior(const Grid& g, double* u, int nvar, cudaStream_t st);
// FP64 throughput probe: dependent DFMA chains on every SM; returns the
// flops issued (2 per DFMA).  sink receives one value per CTA.
long long launch_fp64_probe(int nsm, int iters, double* sink, int nsink, cudaStream_t st);

}  // namespace z4c

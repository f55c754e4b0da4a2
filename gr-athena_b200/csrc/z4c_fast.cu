// The contracted right-hand side and low-storage stage (LaunchShape::contract).
// Compiled with -fmad=true: the pointwise algebra of z4c_rhs.cuh contracts
// into fused multiply-adds, and the order of the additions that close the
// right-hand side changes, so the values agree with the exact path (and the
// reference) to round-off rather than bit for bit.
//
// Four launches per stage instead of five, and the advection sums never
// cross HBM:
//   k_prep        stored first derivatives (the exact path's kernel)
//   k_ricci_fast  R_ab + Rphi_ab (ricci_point)
//   k_main_fast   the right-hand side without the advection sums and the
//                 Kreiss-Oliger terms (rhs_point<false>) into rhs
//   k_col_fast    per variable and interior column, the advection sum and
//                 the Kreiss-Oliger terms (calculate_z4c_rhs.cpp:184-226,
//                 :908-915) from one sliding z window, added to the main
//                 pass's value with the advection factor the right-hand side
//                 applies (lapse_advect for alpha, shift_advect for beta, 1
//                 otherwise), then the 2S stage update (ls_update) into u1
//                 and the output register, or the right-hand side back into
//                 rhs
#include <cuda_runtime.h>

#include "z4c_common.cuh"
#include "z4c_kernels.cuh"
#include "z4c_rhs.cuh"
#include "z4c_stencil.cuh"

namespace z4c {

namespace {

constexpr int kColThreadsMax = 512;

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Advection factor of variable n in the right-hand side (:860-902).
__device__ __forceinline__ double adv_factor(const z4c_params_t& p, int n) {
  if (n == Z4C_ALPHA) return p.lapse_advect;
  if (n >= Z4C_BETAX && n <= Z4C_BETAZ) return p.shift_advect;
  return 1.0;
}

template <int UNROLL, int NX, bool STAGE>
__global__ void __launch_bounds__(kColThreadsMax)
k_col_fast(Grid gin, DevParams P, const double* __restrict__ u, double* __restrict__ rhs,
           double* __restrict__ u1, double* __restrict__ u_out, LsStage ws, int block0,
           int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  Column c;
  if (!column_index(g, block0, nblk, c)) return;
  const int nn0 = g.nn[0], sk = nn0 * g.nn[1];
  const double* U = u + (int64_t)c.b * NVAR * g.nvol + c.j * nn0 + c.i;
  const double* f = U + (int64_t)c.n * g.nvol;
  const double* bx = U + (int64_t)Z4C_BETAX * g.nvol;
  const double* by = U + (int64_t)Z4C_BETAY * g.nvol;
  const double* bz = U + (int64_t)Z4C_BETAZ * g.nvol;
  const int64_t base = ((int64_t)c.b * NVAR + c.n) * g.nvol + c.j * nn0 + c.i;
  const FdScale& F = P.fd[c.b];
  const double fac = adv_factor(P.p, c.n), diss = P.p.diss;
  double w[9];
  window_init(f, sk, NG, w);
#pragma unroll UNROLL
  for (int k = NG; k <= NG + g.nx[2]; ++k) {
    window_advance(f, sk, k, w);
    const int o = k * sk;
    const int64_t q = base + o;
    double lv = 0;
    lv += fd_lx_side(f + o, 1, __ldg(bx + o), F.lidx[0]);
    lv += fd_lx_side(f + o, nn0, __ldg(by + o), F.lidx[1]);
    lv += fd_lx_window(w, __ldg(bz + o), F.lidx[2]);
    const double r = add_ko_column(rhs[q] + fac * lv, f + o, nn0, w, F, diss);
    if constexpr (STAGE) {
      double v1, v;
      ls_update(ws, w[4], ws.u1_zero ? 0.0 : u1[q], r, v1, v);
      u1[q] = v1;
      u_out[q] = v;
    } else {
      rhs[q] = r;
    }
    window_shift(w);
  }
}

template <int THREADS, int NX, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
k_ricci_fast(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ sd,
             double* __restrict__ rsum, int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = interior_count(g);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * nblk) return;
  const int b = block0 + (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_ijk(g, l, i, j, k);
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  double R[6];
  ricci_point(u + (int64_t)b * NVAR * g.nvol, sd + (int64_t)b * kSdComponents * g.nvol, g.nvol,
              p, g.s, P, P.fd[b], R);
  double* rs = rsum + (int64_t)b * 6 * npts + l;
#pragma unroll
  for (int q = 0; q < 6; ++q) rs[(int64_t)q * npts] = R[q];
}

template <int THREADS, int NX, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
k_main_fast(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ sd,
            const double* __restrict__ rsum, double* __restrict__ rhs, int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = interior_count(g);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * nblk) return;
  const int b = block0 + (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_ijk(g, l, i, j, k);
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  double out[NVAR];
  rhs_point<false>(u + (int64_t)b * NVAR * g.nvol, sd + (int64_t)b * kSdComponents * g.nvol,
                   g.nvol, p, g.s, P, P.fd[b], rsum + (int64_t)b * 6 * npts + l, nullptr, npts,
                   out);
  double* rb = rhs + (int64_t)b * NVAR * g.nvol + p;
#pragma unroll
  for (int n = 0; n < NVAR; ++n) rb[(int64_t)n * g.nvol] = out[n];
}

template <int T, int MINB>
void launch_points(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                   double* rhs, int block0, int nblk, cudaStream_t st) {
  const int64_t n = interior_count(g) * nblk;
  const bool fx = has_fixed_geometry(g), fm = has_merged_geometry(g);
  (fx ? k_ricci_fast<T, kFixedNX, MINB>
      : fm ? k_ricci_fast<T, kMergedNX, 1> : k_ricci_fast<T, 0, 1>)<<<div_up(n, T), T, 0, st>>>(
      g, P, u, sc.sd, sc.rsum, block0, nblk);
  (fx ? k_main_fast<T, kFixedNX, MINB>
      : fm ? k_main_fast<T, kMergedNX, 1> : k_main_fast<T, 0, 1>)<<<div_up(n, T), T, 0, st>>>(
      g, P, u, sc.sd, sc.rsum, rhs, block0, nblk);
}

template <bool STAGE>
void launch_fast(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                 double* rhs, double* u1, double* u_out, const LsStage& w, int block0, int nblk,
                 const LaunchShape& sh, cudaStream_t st) {
  launch_prep(g, P, u, sc.sd, block0, nblk, st);
  const bool hi = sh.point_regs == kPointRegsHigh;
  if (sh.point_threads == 64) {
    if (hi) launch_points<64, 6>(g, P, u, sc, rhs, block0, nblk, st);
    else launch_points<64, 1>(g, P, u, sc, rhs, block0, nblk, st);
  } else {
    if (hi) launch_points<128, 3>(g, P, u, sc, rhs, block0, nblk, st);
    else launch_points<128, 1>(g, P, u, sc, rhs, block0, nblk, st);
  }
  const int ct = sh.column_threads;
  const int64_t cols = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * NVAR * nblk;
  (has_fixed_geometry(g)    ? k_col_fast<kFixedNX + 1, kFixedNX, STAGE>
   : has_merged_geometry(g) ? k_col_fast<4, kMergedNX, STAGE>
                            : k_col_fast<4, 0, STAGE>)<<<div_up(cols, ct), ct, 0, st>>>(
      g, P, u, rhs, u1, u_out, w, block0, nblk);
  add_kernel_launches(3);
}

}  // namespace

void launch_stage_ls_fast(const Grid& g, const DevParams& P, const double* u,
                          const RhsScratch& sc, double* rhs, double* u1, double* u_out,
                          const LsStage& w, int block0, int nblk, const LaunchShape& sh,
                          cudaStream_t st) {
  launch_fast<true>(g, P, u, sc, rhs, u1, u_out, w, block0, nblk, sh, st);
}

void launch_rhs_fast(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                     double* rhs, int block0, int nblk, const LaunchShape& sh, cudaStream_t st) {
  launch_fast<false>(g, P, u, sc, rhs, nullptr, nullptr, LsStage{}, block0, nblk, sh, st);
}

}  // namespace z4c

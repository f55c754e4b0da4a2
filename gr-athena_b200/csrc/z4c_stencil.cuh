// Stencil and stage helpers shared by the translation units that build the
// right-hand side: the exact one (z4c_kernels.cu, compiled without
// floating-point contraction) and the contracted one (z4c_fast.cu).  Each
// unit compiles its own inline copy under its own flags.
#pragma once

#include "z4c_common.cuh"
#include "z4c_kernels.cuh"

namespace z4c {

// ---- per-variable passes: advection sums and Kreiss-Oliger -------------------
// One thread per (block, variable, interior (i, j)) column, looping over the
// interior k.  Stencils along x and y read their lines directly; along z the
// nine-vertex window slides in registers.  Index arithmetic is 32-bit (the
// launcher checks that the thread count fits).
struct Column {
  int b, n, i, j;
};
__device__ __forceinline__ bool column_index(const Grid& g, int block0, int nblk, Column& c) {
  const int n0 = g.nx[0] + 1, per = n0 * (g.nx[1] + 1);
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= per * NVAR * nblk) return false;
  const int ij = t % per, rest = t / per;
  c.n = rest % NVAR;
  c.b = block0 + rest / NVAR;
  c.i = NG + ij % n0;
  c.j = NG + ij / n0;
  return true;
}

// Loads for the stencil helpers below: read-only cache path for global
// memory (GL = true), plain loads for shared memory.
template <bool GL>
__device__ __forceinline__ double ld(const double* p) {
  if (GL) return __ldg(p);
  return *p;
}

// Lop-sided advection along one direction (FDStencilBiased{Left,Right}<1,4,2>,
// finite_differencing.tpp:175-191): only the side the sign of vx selects is
// evaluated; its value is the reference's, which evaluates both and keeps one.
template <bool GL = true>
__device__ __forceinline__ double fd_lx_side(const double* __restrict__ u, int st, double vx,
                                             double lidx) {
  if (vx < 0) {
    double dl = 0.;
    dl += 1. * ld<GL>(u - 4 * st);
    dl += -8. * ld<GL>(u - 3 * st);
    dl += 30. * ld<GL>(u - 2 * st);
    dl += -80. * ld<GL>(u - st);
    dl += 35. * ld<GL>(u);
    dl += 24. * ld<GL>(u + st);
    dl += -2. * ld<GL>(u + 2 * st);
    return (vx * dl) * lidx;
  }
  double dr = 0.;
  dr += -1. * ld<GL>(u + 4 * st);
  dr += 8. * ld<GL>(u + 3 * st);
  dr += -30. * ld<GL>(u + 2 * st);
  dr += 80. * ld<GL>(u + st);
  dr += -35. * ld<GL>(u);
  dr += -24. * ld<GL>(u - st);
  dr += 2. * ld<GL>(u - 2 * st);
  return (vx * dr) * lidx;
}
// The same along z from the window w[0..8] = f(k-4..k+4).
__device__ __forceinline__ double fd_lx_window(const double w[9], double vx, double lidx) {
  if (vx < 0) {
    double dl = 0.;
    dl += 1. * w[0];
    dl += -8. * w[1];
    dl += 30. * w[2];
    dl += -80. * w[3];
    dl += 35. * w[4];
    dl += 24. * w[5];
    dl += -2. * w[6];
    return (vx * dl) * lidx;
  }
  double dr = 0.;
  dr += -1. * w[8];
  dr += 8. * w[7];
  dr += -30. * w[6];
  dr += 80. * w[5];
  dr += -35. * w[4];
  dr += -24. * w[3];
  dr += 2. * w[2];
  return (vx * dr) * lidx;
}

// Kreiss-Oliger along one direction (FDStencilCenteredDegreeEven<8,4>,
// finite_differencing.tpp:335-368) from a line pointer or from the window.
template <bool GL = true>
__device__ __forceinline__ double fd_diss_line(const double* __restrict__ u, int st, double cidxd,
                                               double diss) {
  double out = 0.;
  out += 1. * (ld<GL>(u - 4 * st) + ld<GL>(u + 4 * st));
  out += -8. * (ld<GL>(u - 3 * st) + ld<GL>(u + 3 * st));
  out += 28. * (ld<GL>(u - 2 * st) + ld<GL>(u + 2 * st));
  out += -56. * (ld<GL>(u - st) + ld<GL>(u + st));
  out += 70. * ld<GL>(u);
  return out * cidxd * diss;
}
__device__ __forceinline__ double fd_diss_window(const double w[9], double cidxd, double diss) {
  double out = 0.;
  out += 1. * (w[0] + w[8]);
  out += -8. * (w[1] + w[7]);
  out += 28. * (w[2] + w[6]);
  out += -56. * (w[3] + w[5]);
  out += 70. * w[4];
  return out * cidxd * diss;
}

// Fills the z window of column c at the first interior k.
__device__ __forceinline__ void window_init(const double* __restrict__ f, int sk, int k0,
                                            double w[9]) {
#pragma unroll
  for (int q = 0; q < 8; ++q) w[q] = __ldg(f + (k0 - 4 + q) * sk);
}
__device__ __forceinline__ void window_advance(const double* __restrict__ f, int sk, int k,
                                               double w[9]) {
  w[8] = __ldg(f + (k + 4) * sk);
}
__device__ __forceinline__ void window_shift(double w[9]) {
#pragma unroll
  for (int q = 0; q < 8; ++q) w[q] = w[q + 1];
}

// Kreiss-Oliger added to one right-hand-side value in the reference's
// order, rhs += Diss_x; rhs += Diss_y; rhs += Diss_z (:908-915).
__device__ __forceinline__ double add_ko_column(double r, const double* __restrict__ fo, int nn0,
                                                const double w[9], const FdScale& F,
                                                double diss) {
  r += fd_diss_line(fo, 1, F.cidxd[0], diss);
  r += fd_diss_line(fo, nn0, F.cidxd[1], diss);
  r += fd_diss_window(w, F.cidxd[2], diss);
  return r;
}


// The 2S stage algebra of IntegrateZ4c (task_list_gr_z4c.cpp:176-195):
//   u1 <- u1 + delta u;  u <- gamma1 u + gamma2 u1 (+ gamma3 u2 = 0);
//   u <- u + beta dt rhs
// in the reference's WeightedAve / AddZ4cRHS branch order
// (mesh/weighted_ave.cpp:20-150): un = u, u1_in = u1 (0 at stage 1), r the
// right-hand side; v1 and v are the new u1 and u.
__device__ __forceinline__ void ls_update(const LsStage& w, double un, double u1_in, double r,
                                          double& v1, double& v) {
  v1 = u1_in;
  if (w.delta != 0.0) v1 += w.delta * un;  // w0 == 1, w2 == 0 branch
  if (w.gamma1 == 1.0) {  // gamma3 == 0 for every 2S integrator accepted
    v = un;
    if (w.gamma2 != 0.0) v += w.gamma2 * v1;
  } else if (w.gamma1 == 0.0) {
    if (w.gamma2 == 1.0) v = v1;
    else v = w.gamma2 * v1;
  } else {
    if (w.gamma2 != 0.0) v = w.gamma1 * un + w.gamma2 * v1;
    else v = un * w.gamma1;
  }
  v += w.beta_dt * r;
}

}  // namespace z4c

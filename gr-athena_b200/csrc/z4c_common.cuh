// Shared device helpers for the Z4c kernels: finite-difference stencils and
// 3x3 symmetric linear algebra.
//
// Every expression keeps the evaluation order of the GR-Athena++ reference
// (the reference is compiled with -ffp-contract=off; these kernels are
// compiled with -fmad=false) so that results agree with it to rounding:
//   stencils     utils/finite_differencing.tpp with DBG_SYMMETRIZE_FD
//                (defs.hpp.in:18) and finite_differencing_stencils.tpp
//   det/inverse  utils/linear_algebra.hpp:47-118, TraceRank2 :271-290
//   floors       utils/floating_point.hpp:110-131
#pragma once

#include <cstdint>

#include "../../include/z4c_b200.h"

namespace z4c {

constexpr int NG = Z4C_NG;
constexpr int NVAR = Z4C_NVAR;

// Stencil scalings of one block (finite_differencing.tpp:20-56 with the
// DBG_SYMMETRIZE_FD branch), computed on the host from the block's dx?f(0).
struct FdScale {
  double cidx1[3];  // 1 / (dx * 60)
  double cidx2[3];  // (1/dx)^2 / 180
  double cidxd[3];  // -2^-8 / dx
  double lidx[3];   // 1 / (dx * 60)
};

// Run-time options plus the per-block stencil scalings (device table).
struct DevParams {
  z4c_params_t p;
  const FdScale* fd;  // [nblocks]
  const double* xf;   // [nblocks][nn0+nn1+nn2] vertex coordinates (Sommerfeld faces)
  const double* dx;   // [nblocks][3] vertex spacing (Sommerfeld faces)
  const unsigned char* som;  // refined meshes: [nblocks] gr_sommerfeld faces, bit 2*axis+outer;
                             // null on a uniform block grid (faces from the grid position)
};

// Geometry of the uniform block grid.
struct Grid {
  int nb[3];        // blocks per axis
  int nx[3];        // interior cells per block axis
  int nn[3];        // vertices per block axis (nx + 1 + 2*NG)
  int64_t s[3];     // strides of i, j, k
  int64_t nvol;     // vertices per block
  int nblocks;
  int bc[6];
  int has_sommerfeld;  // some face is Z4C_BC_SOMMERFELD
};

// Block geometry fixed at compile time.  Kernels instantiated with NX > 0 run
// on NX^3 MeshBlocks and see constant vertex counts and strides, so every
// stencil offset folds into the load instruction; NX = 0 reads the geometry
// from the Grid.  kFixedNX is the MeshBlock size that gets the fixed
// instances (0 disables them).
#ifndef Z4C_FIXED_NX
#define Z4C_FIXED_NX 16
#endif
constexpr int kFixedNX = Z4C_FIXED_NX;
template <int NX>
__host__ __device__ __forceinline__ Grid fixed_geometry(const Grid& g) {
  if constexpr (NX == 0) {
    return g;
  } else {
    constexpr int nn = NX + 1 + 2 * NG;
    Grid r = g;
    for (int a = 0; a < 3; ++a) {
      r.nx[a] = NX;
      r.nn[a] = nn;
    }
    r.s[0] = 1;
    r.s[1] = nn;
    r.s[2] = (int64_t)nn * nn;
    r.nvol = (int64_t)nn * nn * nn;
    return r;
  }
}
__host__ __forceinline__ bool has_fixed_geometry(const Grid& g) {
  return kFixedNX > 0 && g.nx[0] == kFixedNX && g.nx[1] == kFixedNX && g.nx[2] == kFixedNX;
}
// The merged vertex grid of a uniform mesh (z4c_evolve on the contracted
// path) is one block of nb * nx cells per axis; kMergedNX is the size whose
// right-hand-side passes get fixed instances as well (0 disables them).
#ifndef Z4C_MERGED_NX
#define Z4C_MERGED_NX 128
#endif
constexpr int kMergedNX = Z4C_MERGED_NX;
__host__ __forceinline__ bool has_merged_geometry(const Grid& g) {
  return kMergedNX > 0 && g.nx[0] == kMergedNX && g.nx[1] == kMergedNX && g.nx[2] == kMergedNX;
}

// ---- stencils -----------------------------------------------------------

#ifdef FD_BARRIER
#define FD_FENCE() asm volatile("" ::: "memory")
#else
#define FD_FENCE()
#endif

// FDStencilCenteredDegreeOdd<1,3>: {-1, 9, -45} / 60
__device__ __forceinline__ double fd_dx(const double* __restrict__ u, int64_t s,
                                        double cidx1) {
  double out = 0.;
  out += -1. * (__ldg(u - 3 * s) - __ldg(u + 3 * s));
  out += 9. * (__ldg(u - 2 * s) - __ldg(u + 2 * s));
  out += -45. * (__ldg(u - s) - __ldg(u + s));
  return out * cidx1;
}

// FDStencilCenteredDegreeEven<2,3>: {2, -27, 270, -490} / 180
__device__ __forceinline__ double fd_dxx(const double* __restrict__ u, int64_t s,
                                         double cidx2) {
  double out = 0.;
  out += 2. * (__ldg(u - 3 * s) + __ldg(u + 3 * s));
  out += -27. * (__ldg(u - 2 * s) + __ldg(u + 2 * s));
  out += 270. * (__ldg(u - s) + __ldg(u + s));
  out += -490. * __ldg(u);
  FD_FENCE();
  return out * cidx2;
}

// Mixed second derivative as the reference forms it: Dx along a of the
// (rounded) Dx along b, evaluated at the six neighbours along a
// (calculate_z4c_rhs.cpp:132,153,174-175).
__device__ __forceinline__ double fd_dxy(const double* __restrict__ u, int64_t sa,
                                         int64_t sb, double cidx1a, double cidx1b) {
  double out = 0.;
  out += -1. * (fd_dx(u - 3 * sa, sb, cidx1b) - fd_dx(u + 3 * sa, sb, cidx1b));
  out += 9. * (fd_dx(u - 2 * sa, sb, cidx1b) - fd_dx(u + 2 * sa, sb, cidx1b));
  out += -45. * (fd_dx(u - sa, sb, cidx1b) - fd_dx(u + sa, sb, cidx1b));
  FD_FENCE();
  return out * cidx1a;
}

// ---- linear algebra -------------------------------------------------------

// index of the symmetric pair (a,b) in xx,xy,xz,yy,yz,zz order
__device__ __forceinline__ constexpr int sidx(int a, int b) {
  return (a == b) ? (a == 0 ? 0 : (a == 1 ? 3 : 5))
                  : ((a + b == 1) ? 1 : ((a + b == 2) ? 2 : 4));
}

__device__ __forceinline__ double det3(double gxx, double gxy, double gxz,
                                       double gyy, double gyz, double gzz) {
  return (-(gxz * gxz) * gyy + 2 * gxy * gxz * gyz - gxx * (gyz * gyz) -
          (gxy * gxy) * gzz + gxx * gyy * gzz);
}

// Inv3Metric; out in xx,xy,xz,yy,yz,zz order
__device__ __forceinline__ void inv3(double oodetg, const double g[6], double gu[6]) {
  const double gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
  gu[0] = (-(gyz * gyz) + gyy * gzz) * oodetg;
  gu[1] = (gxz * gyz - gxy * gzz) * oodetg;
  gu[3] = (-(gxz * gxz) + gxx * gzz) * oodetg;
  gu[2] = (-gxz * gyy + gxy * gyz) * oodetg;
  gu[4] = (gxy * gxz - gxx * gyz) * oodetg;
  gu[5] = (-(gxy * gxy) + gxx * gyy) * oodetg;
}

__device__ __forceinline__ double trace_rank2(double detginv, const double g[6],
                                              const double A[6]) {
  const double gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
  const double Axx = A[0], Axy = A[1], Axz = A[2], Ayy = A[3], Ayz = A[4], Azz = A[5];
  return detginv * (-2. * Ayz * gxx * gyz + Axx * gyy * gzz +
                    gxx * (Azz * gyy + Ayy * gzz) +
                    2. * (gxz * (Ayz * gxy - Axz * gyy + Axy * gyz) +
                          gxy * (Axz * gyz - Axy * gzz)) -
                    Azz * (gxy * gxy) - Ayy * (gxz * gxz) - Axx * (gyz * gyz));
}

__device__ __forceinline__ double regularize_nth_root(double value, double value_reg,
                                                      double eps_floor, double npow) {
  const double eps = value - value_reg;
  return ((eps < eps_floor) ? (1.0 + eps_floor / npow) : pow(value, 1.0 / npow));
}

__device__ __forceinline__ double regularize_near_zero(double value, double value_eps) {
  return (value >= 0) ? ((value < value_eps) ? value_eps : value)
                      : ((value > -value_eps) ? -value_eps : value);
}

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

// AlgConstr on one point (z4c.cpp:677-799); g and A in place.
__device__ __forceinline__ void alg_constr_point(const z4c_params_t& opt, double g[6],
                                                 double A[6], double* chi, double* alpha) {
  if (opt.tf_force_regularization) {
    double detg = det3(g[0], g[1], g[2], g[3], g[4], g[5]);
    detg = detg > 0. ? detg : 1.;
    const double oopsi4 = regularize_nth_root(detg, 1.0, opt.eps_floor, -3.0);
#pragma unroll
    for (int c = 0; c < 6; ++c) g[c] *= oopsi4;
    const double tr = trace_rank2(1.0, g, A);
#pragma unroll
    for (int c = 0; c < 6; ++c) A[c] -= (1.0 / 3.0) * tr * g[c];
  } else {
    const double detg = det3(g[0], g[1], g[2], g[3], g[4], g[5]);
    if (detg > opt.eps_floor) {
      const double oopsi4 = regularize_nth_root(detg, 1.0, opt.eps_floor, -3.0);
#pragma unroll
      for (int c = 0; c < 6; ++c) g[c] *= oopsi4;
      const double tr = trace_rank2(1.0, g, A);
#pragma unroll
      for (int c = 0; c < 6; ++c) A[c] -= (1.0 / 3.0) * tr * g[c];
    }
  }
  if (opt.force_regularization) {
    *chi = dmax(*chi, opt.eps_floor);
    *alpha = regularize_near_zero(*alpha, opt.eps_floor);
  }
}

}  // namespace z4c

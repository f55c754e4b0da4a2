// psi4 extraction on coordinate spheres: WaveExtract / WaveExtractLocal
// (z4c/wave_extract.cpp), SphericalGrid / SphericalPatch
// (mesh/spherical_grid.cpp) and GeodesicGrid (mesh/geodesic_grid.cpp).
//
// The sphere, the ownership of its vertices by MeshBlocks, the Lagrange
// stencils and the spin-weighted harmonics are set up once on the host; each
// extraction then runs three small kernels on the Weyl register: the
// interpolation to the owned vertices, the per-block (l, m) projection and
// the sum over blocks in the reference's MeshBlock (gid) order.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "z4c_common.cuh"

namespace z4c {

// SphericalGrid(nlev, rad, bitant): for each of the 10 nlev^2 + 2 vertices
// (theta, phi, x, y, z, weight), the weight being rad^2 times the area of
// the vertex's dual cell on the unit sphere.
std::vector<double> sphere_grid(int nlev, double rad, bool bitant);

struct WaveSphere {
  double rad = 0;
  int nlev = 0, lmax = 0, bitant = 0;
  int npts = 0;   // vertices owned by some block
  int nseg = 0;   // blocks owning at least one vertex
  int nslot = 0;  // (lmax - 1) (2 lmax + 1): psi(l - 2, m + l) slots
  // device arrays, points grouped by owning block in gid order
  int* blk = nullptr;      // [npts] owning block (context order)
  int* base = nullptr;     // [npts] flat offset of the stencil's first vertex
  double* coef = nullptr;  // [npts][3][8] Lagrange coefficients per axis
  double* pw = nullptr;    // [npts][2] weight, bitant sign
  double* ylm = nullptr;   // [nslot][npts][2] Re, Im of the -2 spin-weighted Y_lm
  int* seg = nullptr;      // [nseg + 1] first point of each block's range
  double* data = nullptr;  // [2][npts] interpolated Re, Im psi4
  double* loc = nullptr;   // [nseg][nslot][2] per-block projections
  double* psi = nullptr;   // [nslot][2] reduced projections
};

// Builds the sphere for the mesh g whose blocks have the vertex coordinates
// xf (nn0 + nn1 + nn2 per block) and spacings dx (3 per block); the blocks'
// logical locations follow the context order b = l0 + nb0 (l1 + nb1 l2).
// Returns 0 or a Z4C_E* code (message in msg).
int wave_build(const Grid& g, const std::vector<double>& xf, const std::vector<double>& dx,
               double rad, int nlev, int lmax, bool bitant, WaveSphere* w, char* msg, int nmsg);
void wave_free(WaveSphere* w);
// Interpolation, projection and reduction on the Weyl register (2 variables,
// ghosts filled); the result is left in w.psi.
void launch_wave(const Grid& g, const WaveSphere& w, const double* weyl, cudaStream_t st);
// The interpolation alone (w.data), and its transpose: databar ([2][npts])
// added onto wbar (a Weyl-shaped register) with the same weights.
void launch_wave_interp(const Grid& g, const WaveSphere& w, const double* weyl, cudaStream_t st);
void launch_wave_interp_adj(const Grid& g, const WaveSphere& w, const double* databar,
                            double* wbar, cudaStream_t st);

}  // namespace z4c

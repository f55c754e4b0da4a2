/* CPU restatement of the GR-Athena++ Z4c hot path: the parity oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arms of bench.py may load this library, and only
 * as the checker or the timed CPU baseline; the product path never calls it.
 *
 * Every function follows the reference file:line cited beside it, including
 * its floating-point evaluation order, so that agreement with the reference
 * CPU build is at the level of rounding (pinned by tests/golden, whose
 * fixtures come from the reference itself built by oracle/ref).
 *
 * Layout (all arrays): one MeshBlock is [var][k][j][i], i fastest, with
 * nn = nx + 1 + 2*ng vertices per axis (vertex-centred, ng = 4).
 */
#ifndef Z4C_ORACLE_H
#define Z4C_ORACLE_H

#include <stdint.h>

#include "../include/z4c_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NG 4

/* Geometry of one vertex-centred MeshBlock. */
typedef struct {
  int nx[3];          /* interior cells per axis */
  double dx[3];       /* grid spacing (the reference's dx?f(0)) */
  const double *x[3]; /* vertex coordinates, nn[a] entries (the reference's x?f) */
  const double *xc[3];/* cell-centre coordinates, nn[a]-1 entries (x?v) */
} orc_block_t;

/* Stored first derivatives used by the RHS and the constraints, computed by
 * orc_prepare_derivs (adm_z4c.cpp:972-1037).  Each array holds nvol values. */
typedef struct {
  double *dalpha[3];      /* d_b alpha */
  double *dchi[3];        /* d_b chi */
  double *dbeta[3][3];    /* [b][c] d_b beta^c */
  double *dg[3][6];       /* [b][cd] d_b g~_cd, cd in xx,xy,xz,yy,yz,zz order */
  double *ddchi[6];       /* d_a d_b chi (interior only) */
} orc_derivs_t;

int64_t orc_nvol(const orc_block_t *b);
/* Allocates / frees the stored-derivative arrays of one block. */
int orc_derivs_alloc(const orc_block_t *b, orc_derivs_t *d);
void orc_derivs_free(orc_derivs_t *d);

/* Z4c::PrepareZ4cDerivatives, adm_z4c.cpp:972-1037. */
void orc_prepare_derivs(const orc_block_t *b, const double *u, orc_derivs_t *d);
/* Z4c::Z4cRHS, calculate_z4c_rhs.cpp:29-916 (constant-eta branch, vacuum:
 * matter terms are evaluated with zero matter fields).  Writes the interior of
 * rhs only.  Requires orc_prepare_derivs(u) first. */
void orc_rhs(const orc_block_t *b, const z4c_params_t *p, const double *u,
             const orc_derivs_t *d, double *rhs);
/* Z4c::Z4cBoundaryRHS, z4c/boundary_conditions.cpp:16-174: on every face
 * with som[face] != 0 (inner_x1, outer_x1, inner_x2, ...) the Sommerfeld
 * right-hand side of Theta, Khat, Gamma^a and A_ab replaces rhs on that
 * face's vertex plane (the interior vertex range of the other axes). */
void orc_boundary_rhs(const orc_block_t *b, const double *u, double *rhs, const int som[6]);
/* Z4c::AlgConstr, z4c.cpp:677-799: all points, in place. */
void orc_algconstr(const orc_block_t *b, const z4c_params_t *p, double *u);
/* Z4c::AlgConstr ranged variant with skip_physical, z4c.cpp:801-991:
 * every point outside the interior [vs..ve]^3. */
void orc_algconstr_ghosts(const orc_block_t *b, const z4c_params_t *p, double *u);
/* Z4c::Z4cToADM, adm_z4c.cpp:200-260: all points.  adm has 17 variables. */
void orc_z4c_to_adm(const orc_block_t *b, const z4c_params_t *p, const double *u,
                    double *adm);
/* Z4c::Z4cToADM ranged variant with skip_physical (ghosts only), :262-365. */
void orc_z4c_to_adm_ghosts(const orc_block_t *b, const z4c_params_t *p,
                           const double *u, double *adm);
/* Z4c::ADMToZ4c, adm_z4c.cpp:46-192 (then AlgConstr).  u is fully written
 * (Gamma^i zero outside the interior). */
void orc_adm_to_z4c(const orc_block_t *b, const z4c_params_t *p, const double *adm,
                    double *u);
/* Z4c::ADMConstraints, adm_z4c.cpp:382-930 (vacuum).  con (7 variables) is
 * zeroed then written on the interior.  Requires orc_prepare_derivs(u). */
void orc_adm_constraints(const orc_block_t *b, const z4c_params_t *p,
                         const double *adm, const double *u, const orc_derivs_t *d,
                         double *con);

/* ---- vertex-centred refinement operators (mesh/mesh_refinement_vc.cpp) ---
 *
 * One MeshBlock of nx[3] cells: fine arrays are [nvar][nn3][nn2][nn1] with
 * nn = nx + 1 + 2*ORC_NG, coarse arrays [nvar][cn3][cn2][cn1] with
 * cn = nx/2 + 1 + 2*ORC_NCG.  Boxes are coarse index ranges
 * {si, ei, sj, ej, sk, ek}, inclusive. */
#define ORC_NCG 4
/* MeshRefinement::RestrictVertexCenteredValues (:56-134), 3-D: injection. */
void orc_vc_restrict(const int nx[3], int nvar, const double *fine, double *coarse,
                     const int box[6]);
/* MeshRefinement::ProlongateVertexCenteredValues (:283-775), 3-D branch with
 * DBG_SYMMETRIZE_P_OP and DBG_SYMMETRIZE_CHEAP (defs.hpp.in:17-20):
 * injection at coincident vertices, tensor-product 6-point Lagrange
 * interpolation (H_SZ = 3) elsewhere. */
void orc_vc_prolongate(const int nx[3], int nvar, const double *coarse, double *fine,
                       const int box[6]);

/* Z4c::Z4cWeyl, z4c/calculate_weyl_scalars.cpp:44-630 (vacuum): the real
 * and imaginary parts of psi4 on the interior from the ADM variables, the Z4c
 * state and the stored derivatives; weyl (2 variables) is NaN elsewhere.
 * Requires orc_prepare_derivs(u). */
void orc_weyl(const orc_block_t *b, const z4c_params_t *p, const double *adm, const double *u,
              const orc_derivs_t *d, double *weyl);

/* ---- psi4 extraction (z4c/wave_extract.cpp, mesh/spherical_grid.cpp,
 * mesh/geodesic_grid.cpp, utils/spherical_harmonics.hpp) ------------------- */
/* Vertices of SphericalGrid(nlev, rad, bitant): 10 nlev^2 + 2 rows of
 * (theta, phi, x, y, z, weight), theta/phi from GeodesicGrid::PositionPolar,
 * x/y/z from SphericalGrid::Position and weight from
 * SphericalGrid::ComputeWeight (rad^2 times the dual-cell area). */
int orc_sphere_grid(int nlev, double rad, int bitant, double *geo);
/* gra::sph_harm::sYlm (spherical_harmonics.hpp:231-255). */
void orc_sylm(int s, int l, int m, double theta, double phi, double *re, double *im);
/* WaveExtractLocal::Decompose_multipole of one MeshBlock on the sphere whose
 * vertices orc_sphere_grid wrote: the SphericalPatch points of the block
 * (their vertex indices into owned, their count returned) and the (l, m)
 * projections of weyl (2 variables, ghosts filled) into psi, laid out
 * psi[l-2][m+l][re/im] with 2 lmax + 1 entries per l. */
int orc_wave_block(const orc_block_t *b, const double *weyl, int np, const double *geo,
                   double rad, int lmax, int bitant, int *owned, double *psi);

/* Regrid-time state transfer between a parent block and one child octant
 * oct[3] (0/1 per axis), one MeshBlock each ([nvar][nn3][nn2][nn1]):
 * AMRRegistry::FillSameRankCoarseToFine, comm/amr_registry.cpp:1015-1233
 * (VC branch: the parent's vertices around the octant, with NCG coarse
 * ghosts, into a coarse buffer, then ProlongateVertexCenteredValues over the
 * child's interior vertices), and FillSameRankFineToCoarse, :814-1012
 * (RestrictVertexCenteredValues of the child's interior, copied into the
 * parent's octant). */
void orc_regrid_refine(const int nx[3], int nvar, const double *parent, double *child,
                       const int oct[3]);
void orc_regrid_derefine(const int nx[3], int nvar, const double *child, double *parent,
                         const int oct[3]);

/* ---- puncture tracker (z4c/puncture_tracker.cpp) ------------------------ */

/* PunctureTracker::InterpolateShift (:95-129): the shift of block b at pos
 * by LagrangeInterpND<2*NGHOST-1, 3> (utils/lagrange_interp.hpp), origin the
 * block's first vertex, spacing dx.  pos must lie in the block. */
void orc_tracker_interp(const orc_block_t *b, const double *u, const double pos[3],
                        double beta[3]);

/* ---- uniform block grid (single level) ---------------------------------- */

/* A uniform mesh of nb[0]*nb[1]*nb[2] blocks, block (l0,l1,l2) at index
 * l0 + nb0*(l1 + nb1*l2) of the arrays.  bc[face] = Z4C_BC_PERIODIC,
 * Z4C_BC_OUTFLOW or Z4C_BC_SOMMERFELD for faces inner_x1, outer_x1, inner_x2,
 * ... (the last two fill ghosts alike). */
typedef struct {
  int nb[3];
  int nx[3];
  int bc[6];
} orc_mesh_t;

/* Same-level vertex-centred ghost exchange (comm_registry.cpp:336-382,
 * node_multiplicity.cpp:102-430, index_utilities.hpp:124-170): every ghost
 * and every block-boundary vertex becomes the mean over all blocks whose
 * interior holds that vertex; then the physical boundary conditions
 * (physical_bcs.cpp:187-260, 506-670).  nvar variables per block. */
void orc_mesh_exchange(const orc_mesh_t *m, int nvar, double *u_all);
/* Only the physical boundary conditions of one block (extrapolate_outflow). */
void orc_block_physical_bcs(const orc_mesh_t *m, const int loc[3], int nvar,
                            double *u);

/* A mesh of MeshBlocks on several refinement levels: nroot blocks per axis
 * at the root level root_level, and per block (gid order) its logical
 * location {level, lx1, lx2, lx3} (levels absolute, as LogicalLocation). */
typedef struct orc_ml_mesh {
  int nroot[3];
  int root_level;
  int nx[3];
  int bc[6];
  int nblocks;
  const int64_t *loc;  /* [nblocks][4] */
} orc_ml_mesh_t;
/* The neighbour list of block b as SearchAndSetNeighbors builds it
 * (mesh/mesh_topology.cpp:278-960): rows {gid, level, ox1, ox2, ox3, fi1,
 * fi2}, at most 56; returns the count. */
int orc_ml_neighbours(const orc_ml_mesh_t *m, int b, int *out);
/* One vertex-centred ghost fill of a multilevel mesh: restriction, pack,
 * additive unpack with node multiplicity, coarse-level BCs, prolongation
 * from coarser neighbours, fine-level BCs (extrapolate_outflow or periodic
 * faces). */
void orc_ml_exchange(const orc_ml_mesh_t *m, int nvar, double *u_all);

/* History-output sums (outputs/history.cpp:168-200) over the cell range of one
 * block: out[8] += {H^2, M, Mx^2, My^2, Mz^2, Z, Theta^2, C} * vol. */
void orc_hst_accumulate(const orc_block_t *b, const z4c_params_t *p,
                        const double *con, const double *u, double out[8]);

#ifdef __cplusplus
}
#endif
#endif

/* z4c_b200: B200-native Z4c spacetime evolution, C ABI.
 *
 * This is the drop-in boundary for the GR-Athena++ Z4c hot path.  Each entry
 * point replaces one member function of the reference `Z4c` class
 * (src/z4c/z4c.hpp:448-539) or one GR_Z4c task (src/task_list/gr/
 * task_list_gr_z4c.cpp); the reference symbol is cited beside it.  All state
 * lives in device memory owned by a context; host pointers are borrowed for
 * the duration of a call only.  No C++ types, no torch types, no exceptions
 * cross this boundary: every call returns Z4C_OK (0) or a negative Z4C_E*
 * code, and z4c_last_error() returns a message for the last failure.
 *
 * Data layout, host and device: one MeshBlock register is the reference's
 * AthenaArray layout [var][k][j][i] (src/athena_arrays.hpp:192-195), i fastest,
 * vertex-centred with nn = nx + 1 + 2*Z4C_NG points per axis; a register over
 * the whole mesh is [block][var][k][j][i] with blocks in the order
 * l0 + nb0*(l1 + nb1*l2) of their logical location.
 *
 * Threading: one context per host thread and CUDA stream; calls on one
 * context must be serialised by the caller.
 */
#ifndef Z4C_B200_H
#define Z4C_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define Z4C_NG 4           /* ghost vertices per side (reference NGHOST=4)  */
#define Z4C_NVAR 22        /* evolved variables (z4c.hpp:63-88)             */
#define Z4C_NADM 17        /* ADM variables (z4c.hpp:100-118)               */
#define Z4C_NCON 7         /* constraint variables (z4c.hpp:128-137)        */
#define Z4C_NWEYL 2        /* Weyl variables: Re, Im psi4 (z4c.hpp:163-171) */

/* Evolved-variable indices, z4c.hpp:63-88. */
enum {
  Z4C_CHI = 0, Z4C_GXX, Z4C_GXY, Z4C_GXZ, Z4C_GYY, Z4C_GYZ, Z4C_GZZ,
  Z4C_KHAT, Z4C_AXX, Z4C_AXY, Z4C_AXZ, Z4C_AYY, Z4C_AYZ, Z4C_AZZ,
  Z4C_GAMX, Z4C_GAMY, Z4C_GAMZ, Z4C_THETA, Z4C_ALPHA,
  Z4C_BETAX, Z4C_BETAY, Z4C_BETAZ
};
/* ADM-variable indices, z4c.hpp:100-118. */
enum {
  Z4C_ADM_ALPHA = 0, Z4C_ADM_BETAX, Z4C_ADM_BETAY, Z4C_ADM_BETAZ,
  Z4C_ADM_GXX, Z4C_ADM_GXY, Z4C_ADM_GXZ, Z4C_ADM_GYY, Z4C_ADM_GYZ, Z4C_ADM_GZZ,
  Z4C_ADM_KXX, Z4C_ADM_KXY, Z4C_ADM_KXZ, Z4C_ADM_KYY, Z4C_ADM_KYZ, Z4C_ADM_KZZ,
  Z4C_ADM_PSI4
};
/* Constraint indices, z4c.hpp:128-137. */
enum {
  Z4C_CON_C = 0, Z4C_CON_H, Z4C_CON_M, Z4C_CON_Z, Z4C_CON_MX, Z4C_CON_MY,
  Z4C_CON_MZ
};

/* Return codes. */
#define Z4C_OK 0
#define Z4C_EINVAL (-1)     /* bad argument                                */
#define Z4C_ENOMEM (-2)     /* device or host allocation failed            */
#define Z4C_ECUDA (-3)      /* a CUDA call failed                          */
#define Z4C_ENONFINITE (-4) /* a NaN/Inf was detected in the state         */
#define Z4C_ETIMEOUT (-5)   /* a bounded device wait gave up               */
#define Z4C_ESTATE (-6)     /* call not valid in the context's state       */
#define Z4C_ENODEV (-7)     /* no usable CUDA device                       */

/* Physical boundary flags per face (inner_x1, outer_x1, inner_x2, ...). */
#define Z4C_BC_PERIODIC 0
/* extrapolate_outflow: polynomial extrapolation of the ghosts
 * (comm/physical_bcs.cpp:187-260). */
#define Z4C_BC_OUTFLOW 1
/* gr_sommerfeld: the same ghost fill for vertex-centred data
 * (comm/physical_bcs.cpp:445-453), plus the Sommerfeld right-hand side of
 * Z4c::Z4cBoundaryRHS on the face's vertex plane (z4c/boundary_conditions.cpp). */
#define Z4C_BC_SOMMERFELD 2

/* Registers held by a context (one value per variable per vertex per block). */
enum {
  Z4C_REG_U = 0,   /* storage.u    (22 vars)                        */
  Z4C_REG_U1,      /* storage.u1   (22 vars, low-storage RK)        */
  Z4C_REG_RHS,     /* storage.rhs  (22 vars)                        */
  Z4C_REG_ADM,     /* storage.adm  (17 vars)                        */
  Z4C_REG_CON,     /* storage.con  (7 vars)                         */
  Z4C_REG_W,       /* work register (22 vars): ping-pong partner of u,
                      and the scratch u_n of the Butcher integrator   */
  Z4C_REG_K1,      /* Butcher stage slopes k_1..k_4 (22 vars each)  */
  Z4C_REG_K2,
  Z4C_REG_K3,
  Z4C_REG_K4,
  Z4C_REG_WEYL,    /* storage.weyl (2 vars: Re psi4, Im psi4)       */
  Z4C_REG_TAN,     /* tangent of u (22 vars; after z4c_adj_setup)   */
  Z4C_REG_ADJ,     /* adjoint of u (22 vars; after z4c_adj_setup)   */
  Z4C_REG_ADM_ADJ, /* adjoint of the ADM register (17 vars; after
                      z4c_adj_setup)                                */
  Z4C_NREG
};

/* Time integrators (task_list/time_integrators.hpp). */
#define Z4C_INTEG_RK4 0     /* low-storage 2S RK4()4[2S], "rk4"  */
#define Z4C_INTEG_BT_RK4 1  /* classical Butcher RK4, "bt_rk4"   */

/* Run-time options of the Z4c class, z4c.hpp:357-431 with the defaults of
 * z4c.cpp:318-410 (set by z4c_params_default). */
typedef struct z4c_params {
  double chi_psi_power;          /* -4 */
  double chi_div_floor;          /* -1000 */
  double diss;                   /* 0 (Kreiss-Oliger strength) */
  double eps_floor;              /* 1e-12 */
  double damp_kappa1;            /* 0 */
  double damp_kappa2;            /* 0 */
  double lapse_oplog;            /* 2 */
  double lapse_harmonicf;        /* 1 */
  double lapse_harmonic;         /* 0 */
  double lapse_advect;           /* 1 */
  double lapse_K;                /* 0 */
  double shift_Gamma;            /* 1 */
  double shift_alpha2Gamma;      /* 0 */
  double shift_H;                /* 0 */
  double shift_advect;           /* 1 */
  double shift_eta;              /* 2 */
  double r_max_con;              /* +inf */
  int tf_force_regularization;   /* 1 */
  int force_regularization;      /* 0 */
} z4c_params_t;

/* A uniform single-level mesh of nb[0]*nb[1]*nb[2] MeshBlocks of nx^3 cells
 * on [xmin, xmax] (reference <mesh> and <meshblock> input blocks). */
typedef struct z4c_mesh_desc {
  int nb[3];
  int nx[3];
  double xmin[3];
  double xmax[3];
  int bc[6];
} z4c_mesh_desc_t;

typedef struct z4c_ctx z4c_ctx;

/* Fills *p with the reference defaults (z4c.cpp:318-410). */
void z4c_params_default(z4c_params_t *p);
/* Message for the last failing call on this thread. */
const char *z4c_last_error(void);

/* Creates a context on the current CUDA device and allocates every register
 * (no reference counterpart: replaces Z4c::Z4c's storage allocation,
 * z4c.cpp:30-217, for all blocks at once). */
int z4c_create(const z4c_mesh_desc_t *mesh, const z4c_params_t *params,
               int integrator, z4c_ctx **out);
/* A context on a statically refined mesh (<refinementN> blocks of the
 * input deck): mesh->nb root blocks per axis of mesh->nx cells, and nblocks
 * MeshBlocks given in gid order by their logical locations
 * locs[b] = {level, lx1, lx2, lx3} (absolute levels, LogicalLocation of
 * mesh/mesh.hpp; the root grid sits at the level ceil(log2(max nb))).  The
 * blocks must tile the root grid with neighbouring levels differing by at
 * most one (MeshBlockTree, mesh/meshblock_tree.cpp:108-260).  Ghost fills
 * run the reference's multilevel vertex-centred exchange
 * (comm/comm_registry.cpp:246-382, 533-570; comm/refinement_ops.cpp:24-195;
 * comm/node_multiplicity.cpp; comm/physical_bcs.cpp:506-890).  Outflow,
 * periodic and gr_sommerfeld faces, puncture trackers, psi4 spheres and
 * restart files. */
int z4c_create_refined(const z4c_mesh_desc_t *mesh, int nblocks, const long long *locs,
                       const z4c_params_t *params, int integrator, z4c_ctx **out);
/* The neighbour list z4c_create_refined builds for one block of a refined
 * mesh (MeshBlock::SearchAndSetNeighbors, mesh/mesh_topology.cpp:278-960),
 * host only: rows {gid, level, ox1, ox2, ox3, fi1, fi2} into out (room for
 * 56 rows); returns the row count, or a negative error code when the blocks
 * do not form a balanced tiling of the root grid.  block = -2 builds and
 * checks the whole exchange plan instead (no device memory) and writes its
 * sizes {pack boxes, unpack ops, prolongation boxes, boundary faces}. */
int z4c_refined_neighbours(const z4c_mesh_desc_t *mesh, int nblocks, const long long *locs,
                           int block, int *out);
int z4c_destroy(z4c_ctx *ctx);
/* Work is enqueued on this CUDA stream (a cudaStream_t; NULL = default). */
int z4c_set_stream(z4c_ctx *ctx, void *stream);
int z4c_sync(z4c_ctx *ctx);
/* Geometry queries: blocks, vertices per block axis, variables of a register,
 * vertex spacing and the per-block vertex coordinates (the reference's x?f). */
int z4c_num_blocks(const z4c_ctx *ctx);
int z4c_block_nn(const z4c_ctx *ctx, int axis);
int z4c_reg_nvar(int reg);
int z4c_dx(const z4c_ctx *ctx, double dx_out[3]);
int z4c_block_coords(const z4c_ctx *ctx, int block, int axis, double *x_out);
/* The same coordinates without a context (host only): vertex coordinates of
 * one block along one axis (nx+1+2*Z4C_NG entries) and its spacing, built as
 * the reference's Coordinates constructor does for a uniform mesh
 * (coordinates/coordinates.cpp:170-198, mesh/mesh.hpp:839-945). */
int z4c_mesh_block_coords(const z4c_mesh_desc_t *mesh, int block, int axis, double *x_out,
                          double *dx_out);

/* Z4c::NewBlockTimeStep (z4c/new_blockdt_z4c.cpp:24-70) over every block and
 * the minimum over blocks of Mesh::NewTimeStep (mesh/mesh.cpp:1753-1803):
 * cfl times the smallest cell width (host only, no context needed). */
/* Vertex coordinates (nx + 1 + 2 NG) and spacing of the block at logical
 * location loc = {level, lx1, lx2, lx3} along one axis
 * (coordinates/coordinates.cpp:125-198, mesh/mesh.cpp:2526-2560). */
/* The MeshBlocks of a restart file, {level, lx1, lx2, lx3} each in gid
 * order, into locs (room for cap); returns their count (locs may be NULL to
 * ask for it).  A refined mesh's file restarts into a z4c_create_refined
 * context over these blocks. */
int z4c_restart_locs(const char *path, long long *locs, int cap);
int z4c_mesh_loc_coords(const z4c_mesh_desc_t *mesh, const long long loc[4], int axis,
                        double *x_out, double *dx_out);
int z4c_mesh_new_dt(const z4c_mesh_desc_t *mesh, double cfl, double *dt_out);

/* Host <-> device copies of a register; block = -1 for the whole mesh.  The
 * host buffer uses the reference layout (see above). */
int z4c_upload(z4c_ctx *ctx, int reg, int block, const double *host);
int z4c_download(z4c_ctx *ctx, int reg, int block, double *host);
/* Device address of a register (whole mesh), for zero-copy interop. */
int z4c_device_ptr(z4c_ctx *ctx, int reg, double **dptr);

/* ---- operators; block = -1 runs every block in one batched launch, a block
 *      index runs that block alone (the per-block launch of the plain path) */

/* Z4c::Z4cRHS (z4c/calculate_z4c_rhs.cpp:29-916), with the 3-D derivative
 * precompute of Z4c::PrepareZ4cDerivatives (z4c/adm_z4c.cpp:972-1037) fused
 * in.  Writes the interior of reg_rhs. */
int z4c_rhs(z4c_ctx *ctx, int reg_u, int reg_rhs, int block);
/* Z4c::Z4cBoundaryRHS (z4c/boundary_conditions.cpp:16-174): on the vertex
 * planes of gr_sommerfeld faces (Z4C_BC_SOMMERFELD), replaces the right-hand
 * side of Theta, Khat, Gamma^a and A_ab in reg_rhs by the Sommerfeld
 * condition evaluated from reg_u.  z4c_stage and z4c_evolve apply it after
 * z4c_rhs, as the CALC_Z4CRHS task does. */
int z4c_boundary_rhs(z4c_ctx *ctx, int reg_u, int reg_rhs, int block);
/* Z4c::AddZ4cRHS (z4c/add_z4c_rhs.cpp:24-35): u_out += wght * rhs, interior. */
int z4c_add_rhs(z4c_ctx *ctx, int reg_rhs, double wght, int reg_out, int block);
/* Z4c::WeightedAve (mesh/weighted_ave.cpp:20-167, VC range):
 * out = w0*out + w1*in1 + w2*in2 on the interior, with the reference's
 * special cases for w0 in {0,1} and zero weights. */
int z4c_weighted_ave(z4c_ctx *ctx, int reg_out, int reg_in1, int reg_in2,
                     const double w[3], int block);
/* Z4c::AlgConstr (z4c/z4c.cpp:677-799): all points, in place. */
int z4c_alg_constr(z4c_ctx *ctx, int reg_u, int block);
/* Z4c::ADMToZ4c (z4c/adm_z4c.cpp:46-192), including the final AlgConstr. */
int z4c_adm_to_z4c(z4c_ctx *ctx, int reg_adm, int reg_u, int block);
/* Z4c::Z4cToADM (z4c/adm_z4c.cpp:200-260). */
int z4c_z4c_to_adm(z4c_ctx *ctx, int reg_u, int reg_adm, int block);
/* Z4c::ADMConstraints (z4c/adm_z4c.cpp:382-930), vacuum. */
int z4c_adm_constraints(z4c_ctx *ctx, int reg_con, int reg_adm, int reg_u,
                        int block);
/* Z4c::Z4cWeyl (z4c/calculate_weyl_scalars.cpp:44-630), vacuum: Re and Im of
 * psi4 into reg_weyl (a Z4C_NWEYL register) on the interior vertices and NaN
 * on every other vertex, from the ADM register (metric and extrinsic
 * curvature) and the Z4c register reg_u (the reference's storage.u, whose
 * first derivatives PrepareZ4cDerivatives stores: this call recomputes
 * them). */
int z4c_weyl(z4c_ctx *ctx, int reg_adm, int reg_u, int reg_weyl, int block);

/* ---- restart files (outputs/restart.cpp:43-352; read back by the Mesh
 * restart constructor, mesh/mesh.cpp:775-1420) -------------------------------
 * The Z4c vacuum build on a uniform mesh: the parameter text, the header,
 * the puncture trackers as the only user Mesh data, the ID list and each
 * MeshBlock's storage.u, blocks in gid order. */
#define Z4C_MAX_TRACKERS 8
typedef struct z4c_restart_info {
  int nbtotal;           /* MeshBlocks */
  int root_level;
  double xmin[3], xmax[3], xrat[3];  /* Mesh::mesh_size */
  int mesh_nx[3];        /* cells of the whole mesh per axis */
  double time, dt;
  int ncycle;
  unsigned long long datasize;  /* bytes per MeshBlock */
  int nb[3];             /* MeshBlocks per axis */
  int block_nx[3];       /* cells per MeshBlock axis */
  int ntrackers;         /* puncture trackers (<z4c> npunct) */
  double trackers[Z4C_MAX_TRACKERS][6];  /* position, shift there (pos, betap) */
  long long text_bytes;  /* parameter text through the byte after <par_end> */
  int nlevels;           /* refinement levels present (1: a uniform mesh) */
} z4c_restart_info_t;
/* Reads the header of a restart file (no context). */
int z4c_restart_info(const char *path, z4c_restart_info_t *info);
/* Copies the parameter text (NUL-terminated, at most cap - 1 bytes) into
 * buf; returns its full length.  buf may be null to ask for the length. */
long long z4c_restart_text(const char *path, char *buf, long long cap);
/* The state of every MeshBlock into the host array u, [block][var][k][j][i]
 * with blocks in context order l0 + nb0 (l1 + nb1 l2) (no context). */
int z4c_restart_read(const char *path, double *u);
/* Writes a restart file from host data (no context): par_text is the
 * parameter text the reference re-reads (an input deck or the text of
 * another restart file; "<par_end>" is appended when missing), u as for
 * z4c_restart_read, trackers[n][6] = position, shift there. */
int z4c_restart_write_host(const char *path, const char *par_text,
                           const z4c_mesh_desc_t *mesh, const double *u, double time,
                           double dt, int ncycle, int ntrackers, const double *trackers);
/* The Mesh restart constructor for this context: checks that the file's mesh
 * is the context's, loads storage.u into Z4C_REG_U and the puncture trackers
 * (added when the context has none); *info receives the header (may be
 * null).  Ghosts are loaded as stored, as the reference does. */
int z4c_restart_load(z4c_ctx *ctx, const char *path, z4c_restart_info_t *info);
/* RestartOutput::WriteOutputFile for this context's Z4C_REG_U and trackers. */
int z4c_restart_save(z4c_ctx *ctx, const char *path, const char *par_text, double time,
                     double dt, int ncycle);

/* ---- psi4 extraction (z4c/wave_extract.cpp, mesh/spherical_grid.cpp,
 * mesh/geodesic_grid.cpp) ---------------------------------------------------
 * A sphere of radius rad carries the geodesic grid of nlev levels
 * (10 nlev^2 + 2 vertices); its multipoles psi(l, m), 2 <= l <= lmax, are
 * laid out as WaveExtract::psi, psi[l-2][m+l][re/im] with 2 lmax + 1 slots
 * per l (slots m + l > 2 l stay 0).  The extraction sequence of the main
 * loop (main.hpp Z4c_DerivedQuantities) is z4c_weyl, then
 * z4c_ghost_fill(Z4C_REG_WEYL) (Mesh::CommunicateAuxZ4c), then
 * z4c_wave_decompose per sphere (Decompose_multipole + ReduceMultipole). */
/* SphericalGrid(nlev, rad, bitant): writes (theta, phi, x, y, z, weight) per
 * vertex into geo (6 (10 nlev^2 + 2) doubles); returns the vertex count.
 * Host only, no context. */
int z4c_sphere_grid(int nlev, double rad, int bitant, double *geo);
/* WaveExtract(pmesh, pin, n) + WaveExtractLocal on every block: sets up a
 * sphere on the context's mesh (vertex ownership, interpolation stencils,
 * spin-weight -2 harmonics); *id numbers the context's spheres from 0. */
int z4c_wave_add(z4c_ctx *ctx, double rad, int nlev, int lmax, int bitant, int *id);
/* Number of sphere vertices owned by some MeshBlock (SphericalPatch sizes). */
int z4c_wave_points(const z4c_ctx *ctx, int id);
/* Decompose_multipole on every block and ReduceMultipole: the multipoles of
 * reg_weyl (ghosts filled) into the host array psi, (lmax-1)(2 lmax+1) 2
 * doubles; returns when psi is written. */
int z4c_wave_decompose(z4c_ctx *ctx, int id, int reg_weyl, double *psi);
/* GR_Z4c SEND/RECV/SETB_Z4C + PHY_BVAL (comm/comm_registry.cpp:336-382,
 * comm/physical_bcs.cpp:506-670): same-level vertex-centred ghost fill by
 * device copy, shared vertices averaged over their owners, then the
 * physical boundary conditions.  Whole mesh. */
int z4c_ghost_fill(z4c_ctx *ctx, int reg);
/* Mesh::FinalizeZ4cADMGhosts (mesh/mesh_communicate.cpp:100-167) for a
 * single-level mesh: ghost fill of u, AlgConstr and Z4cToADM on the ghost
 * vertices only.  Run once after the initial data is in place (after
 * z4c_adm_to_z4c, or after uploading u and adm). */
int z4c_init_finalize(z4c_ctx *ctx);
/* History sums of outputs/history.cpp:168-200 over the whole mesh from the
 * con and u registers: H^2, M, Mx^2, My^2, Mz^2, Z, Theta^2, C (volume
 * weighted). */
int z4c_hst_norms(z4c_ctx *ctx, double out[8]);

/* ---- time stepping ------------------------------------------------------ */

/* One GR_Z4c stage (task_list/gr/task_list_gr_z4c.cpp:142-344) over all
 * blocks: fused RHS + KO + stage update, ghost fill, AlgConstr, and on the
 * last stage (stage 4) Z4cToADM into the ADM register, as the Z4C_TO_ADM task
 * does on every last stage.  stage is 1-based; dt the full step. */
int z4c_stage(z4c_ctx *ctx, int stage, double dt);
/* nsteps full steps (gra::evolve::Z4c_Vacuum, src/main.hpp:906-913); the
 * per-step launch sequence is captured once into a CUDA graph and replayed.
 * Every step ends with Z4cToADM (the last stage's Z4C_TO_ADM task); when
 * with_constraints is non-zero the last step also runs ADMConstraints. */
int z4c_evolve(z4c_ctx *ctx, double dt, int nsteps, int with_constraints);
/* Independent evolutions from host memory (no counterpart in the reference,
 * whose state lives in host memory): for each of njobs jobs, host_in[j] (a
 * whole u register, the layout of z4c_upload) is evolved nsteps steps of dt
 * as z4c_evolve(ctx, dt, nsteps, 1) does, and the final u register is written
 * to host_out[j] and its history norms (those of z4c_hst_norms) to
 * hst_out[8*j .. 8*j+7] (hst_out may be NULL; host_out NULL downloads the
 * norms only, for runs that keep only the diagnostics: then, when the steps
 * run on a merged grid (z4c_set_merged) of three or more block layers in z,
 * only the vertex planes that grid reads are uploaded of the blocks off the
 * mesh's z faces, about three quarters of the register on 8^3 blocks of
 * 16^3, and u keeps older values in the others).  The copies overlap the
 * evolutions: job j+1 is uploaded and job j-1 downloaded while job j
 * evolves, on two copy streams of the library, through two input and two
 * output device registers allocated on the first call and held until
 * z4c_destroy.  Host buffers should be page-locked (cudaHostAlloc or
 * cudaHostRegister) for the copies to overlap; pageable ones give the same
 * results without the overlap.  Returns once every job has finished; u then
 * holds the last job's final state.  For ensembles and parameter sweeps whose
 * states are produced and consumed on the host. */
int z4c_evolve_jobs(z4c_ctx *ctx, int njobs, const double *const *host_in,
                    double *const *host_out, double *hst_out, double dt, int nsteps);
/* Z4c::Z4cRHS + GR_Z4c::IntegrateZ4c of one low-storage stage as a single
 * fused launch over all blocks, without the ghost exchange that follows:
 * reads u and u1, writes the updated interior into the work register and
 * u1.  Used to time the dominant kernel in isolation. */
int z4c_rhs_stage(z4c_ctx *ctx, int stage, double dt);
/* Measured FP64 throughput of the device (dependent DFMA chains on every SM,
 * 2 flops per DFMA), in TFLOP/s; the denominator of the FP64 roofline. */
int z4c_fp64_probe(z4c_ctx *ctx, double *tflops);
/* Selects the per-block launch loop (plain path, one RHS launch per block per
 * stage) instead of the batched launch inside z4c_stage/z4c_evolve. */
int z4c_set_per_block(z4c_ctx *ctx, int per_block);
/* Launch shape of the right-hand-side passes (no reference counterpart):
 * tile = {threads per CTA of the per-vertex Ricci and main passes (64, 128,
 * 256), threads per CTA of the per-variable passes (advection, stored first
 * derivatives, Kreiss-Oliger + stage update: 128, 256, 512), z-slabs per
 * MeshBlock in which those passes stage one variable in shared memory (1-4;
 * 0, or slabs whose vertex planes do not fit, selects global-memory
 * pencils)}.  The default is {128, 128, 0}; unsupported shapes return
 * Z4C_EINVAL.  Results do not depend on the shape. */
int z4c_set_tile(z4c_ctx *ctx, int ti, int tj, int tk);
int z4c_get_tile(const z4c_ctx *ctx, int tile_out[3]);
/* Contracted right-hand side (no reference counterpart): with on != 0 every
 * later z4c_rhs, stage and step of the context takes the contracted path:
 * floating-point contraction (fused multiply-adds), the advection sums and
 * the Kreiss-Oliger terms added in one per-variable pass, and the stage
 * update fused with the main right-hand-side pass, four launches per stage.
 * Its right-hand side agrees with the exact path's (which matches the
 * reference bit for bit) to round-off, within the 1e-12 relative bound per
 * evaluation; meshes with gr_sommerfeld faces and the Butcher integrator keep
 * the exact path.  Off by default; switching drops the captured step graph,
 * and the autotuner times the path that is switched on. */
int z4c_set_contract(z4c_ctx *ctx, int on);
/* Register budget of the heavy per-vertex right-hand-side passes on meshes of
 * 16^3 MeshBlocks (no reference counterpart): 0 lets them use up to 255
 * registers per thread (two CTAs of 128 threads per SM), 168 compiles them
 * for three CTAs of 128 or six of 64 per SM (1.5x the resident warps for a
 * few dozen bytes of spill); 256-thread CTAs always take 255.  The arithmetic
 * is the same either way.  The autotuner tries both; switching drops the
 * captured step graph. */
int z4c_set_point_regs(z4c_ctx *ctx, int regs);
int z4c_get_point_regs(const z4c_ctx *ctx, int *regs);
int z4c_get_contract(const z4c_ctx *ctx, int *on);
/* Merged grid (no reference counterpart): on a uniform single-level mesh
 * whose faces are all outflow or all periodic, the contracted path with the low-storage integrator
 * runs the steps of z4c_evolve on one vertex grid that holds every block
 * (nb*nx cells per axis plus the ghosts), so that no vertex is stored twice
 * and no ghost exchange runs between the blocks; the state (u, and the ADM
 * and constraint registers the step writes) is copied from the blocks at the
 * start of the call and back to them, every vertex and ghost, at its end.
 * The blocks' shared vertices then hold one value where the reference
 * averages its owners' copies (equal up to rounding), so results agree with
 * the block-by-block evolution to round-off, as the contracted path does
 * anyway.  It assumes the state's ghosts are those of a ghost fill (as every
 * state this library or the reference produces).  The merged grid is a
 * second, single-block context (about a third of the blocks' memory on 16^3
 * blocks), created by the first z4c_evolve that uses it and held until
 * z4c_destroy.  on = 1 (the default) allows it, 0 keeps the blocks;
 * z4c_get_merged reports whether the next z4c_evolve will use it. */
int z4c_set_merged(z4c_ctx *ctx, int on);
int z4c_get_merged(const z4c_ctx *ctx, int *on);
/* Autotuner (no reference counterpart): times one fused low-storage stage on
 * the context's current state for each candidate shape (the Ricci/main CTA
 * size first, then the column-pass shape; reps timed launches each after a
 * warm-up), keeps the fastest and drops the captured step graph.  Writes the
 * work register, u1 and rhs (u is untouched); call it between steps.
 * *best_ms (may be NULL) receives the stage time of the chosen shape. */
int z4c_autotune(z4c_ctx *ctx, int reps, float *best_ms);
/* PunctureTracker (z4c/puncture_tracker.cpp): adds a tracker at pos; every
 * following step interpolates the shift at the tracker from the state at the
 * start of the step (InterpolateShift, :95-129, 8-point Lagrange stencils)
 * and moves it, pos -= dt * shift (EvolveTracker, :132-186).  At most 8
 * trackers; adding one drops the captured step graph. */
int z4c_tracker_add(z4c_ctx *ctx, const double pos[3], int *id);
/* Position and interpolated shift of tracker id: out = {x, y, z, beta^x,
 * beta^y, beta^z} (the columns of WriteTracker, :189-203).  Z4C_ESTATE when
 * the puncture has left every MeshBlock. */
int z4c_tracker_get(z4c_ctx *ctx, int id, double out[6]);
/* Kernels launched by this library in this process so far (graph replays
 * count every kernel node); a diagnostic with no reference counterpart. */
long long z4c_kernel_launches(void);
/* Scans a register for NaN/Inf (z4c/z4c_utils.cpp:18-150 is_finite_*):
 * Z4C_OK if all finite, Z4C_ENONFINITE otherwise. */
int z4c_check_finite(z4c_ctx *ctx, int reg);

/* ---- vertex-centred refinement operators ----------------------------------
 *
 * MeshRefinement's vertex-centred operators (mesh/mesh_refinement_vc.cpp) on
 * nblocks MeshBlocks of nx[0] x nx[1] x nx[2] cells held in caller-owned
 * DEVICE arrays: fine [block][nvar][nn3][nn2][nn1] with nn = nx + 1 +
 * 2*Z4C_NG, coarse [block][nvar][cn3][cn2][cn1] with cn = nx/2 + 1 + 2*Z4C_NCG
 * (the reference's coarse_u_ layout, z4c.cpp:78-84).  box = {si, ei, sj, ej,
 * sk, ek} is an inclusive range of coarse vertex indices, the arguments
 * csi..cek / si..ek of the reference functions.  A box whose reads or writes
 * would leave the arrays is rejected with Z4C_EINVAL before any launch.
 * Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default). */
#define Z4C_NCG 4  /* coarse ghost vertices (reference NCGHOST for NGHOST=4) */
/* MeshRefinement::RestrictVertexCenteredValues (:56-134): injection. */
int z4c_vc_restrict(const double *fine, double *coarse, int nblocks, int nvar,
                    const int nx[3], const int box[6], void *stream);
/* MeshRefinement::ProlongateVertexCenteredValues (:283-775, 3-D): injection at
 * coincident vertices, tensor-product 6-point Lagrange interpolation
 * elsewhere (InterpolateLagrangeUniform<3>, utils/interp_univariate.hpp:43). */
int z4c_vc_prolongate(const double *coarse, double *fine, int nblocks, int nvar,
                      const int nx[3], const int box[6], void *stream);
/* Regrid-time state transfer between one parent MeshBlock and its child in
 * octant oct[3] (0 or 1 per axis), one block each in the fine layout above;
 * coarse is a caller-owned device scratch of one coarse block (nvar cn^3).
 * AMRRegistry::FillSameRankCoarseToFine (comm/amr_registry.cpp:1015-1233,
 * vertex-centred): the child's interior vertices prolongated from the
 * parent's vertices around the octant; ghosts are left to the next ghost
 * exchange, as in the reference. */
int z4c_regrid_refine(const double *parent, double *child, double *coarse, int nvar,
                      const int nx[3], const int oct[3], void *stream);
/* AMRRegistry::FillSameRankFineToCoarse (:814-1012, vertex-centred): the
 * child's interior vertices restricted (injection) into the parent's octant. */
int z4c_regrid_derefine(const double *child, double *parent, double *coarse, int nvar,
                        const int nx[3], const int oct[3], void *stream);

/* Regrid (AMRTransfer after MeshBlockTree refinement / derefinement,
 * comm/amr_transfer.cpp:373-412, comm/amr_registry.cpp:814-1233): the Z4c
 * state and the puncture trackers of src carried into dst, a context over the
 * regridded block list of the same root grid (uniform or refined).  Every
 * block of dst is a block of src (copied), a child of one (refined from it)
 * or the parent of eight (derefined from them).  Interiors only; call
 * z4c_init_finalize(dst) after it for the ghosts, as the reference exchanges
 * after a regrid.  Both contexts must live on the current CUDA device
 * (Z4C_EINVAL otherwise, before any work); a failure of earlier work on src,
 * or of the transfer, returns Z4C_ECUDA and leaves dst's state undefined. */
int z4c_regrid(z4c_ctx *dst, const z4c_ctx *src);

/* ---- differentiation (no reference counterpart) ---------------------------
 *
 * The tangent-linear model and the hand-written adjoint of the low-storage
 * RK4 step (Z4cRHS with Kreiss-Oliger, task_list_gr_z4c.cpp:170-213 with the
 * weights of task_list_integrators_low_storage.cpp:112-142, the ghost
 * exchange and AlgConstr), and of the objective J = sum over blocks of the
 * cell volume times the sum over the history cells of H^2, H the Hamiltonian
 * constraint of ADMConstraints after Z4cToADM (the H-norm of
 * outputs/history.cpp:168-200).  Uniform and statically refined meshes
 * (on the latter the transpose of the multilevel ghost fill: fine-level BCs,
 * prolongation, coarse-level BCs, the contribution-list gather and the
 * restriction, transposed; its scatters add atomically, so its sums are
 * ordered differently from run to run) with periodic and
 * extrapolate_outflow faces (gr_sommerfeld faces are rejected), rk4,
 * chi_psi_power = -4.  The state's adjoint lives in Z4C_REG_ADJ and a
 * tangent in Z4C_REG_TAN, each over every vertex (ghosts included); the
 * adjoints of the gauge parameters shift_eta and damp_kappa1 accumulate in
 * the context.  The calls use the context's RHS register as scratch. */
/* Allocates the tangent / adjoint buffers (about 13 state-sized registers
 * plus channel scratch; on refined meshes also an int per vertex for the
 * prolongation's transpose) and zeroes Z4C_REG_TAN and Z4C_REG_ADJ. */
int z4c_adj_setup(z4c_ctx *ctx);
/* One step of u (Z4C_REG_U) and of its tangent (Z4C_REG_TAN) together. */
int z4c_tlm_step(z4c_ctx *ctx, double dt);
/* Adjoint of one step from the state in Z4C_REG_U (left unchanged; the
 * step is recomputed stage by stage): Z4C_REG_ADJ holds the adjoint of the
 * state after the step on entry and of the state in Z4C_REG_U on return. */
int z4c_adj_step(z4c_ctx *ctx, double dt);
/* J of register reg; with reg_tan >= 0 also its directional derivative
 * along the tangent in reg_tan (*Jdot, may be NULL otherwise). */
int z4c_adj_objective(z4c_ctx *ctx, int reg, int reg_tan, double *J, double *Jdot);
/* Z4C_REG_ADJ += scale * dJ/du at the state in reg. */
int z4c_adj_objective_adj(z4c_ctx *ctx, int reg, double scale);
/* Adjoint of the initial data: Z4C_REG_ADJ holds the adjoint of u after
 * z4c_adm_to_z4c(ctx, Z4C_REG_ADM, Z4C_REG_U, -1) and z4c_init_finalize (the
 * reference's ADMToZ4c, adm_z4c.cpp:46-192, and FinalizeZ4cADMGhosts); the
 * ADM register holds the data that mapped; the adjoint of the ADM data is
 * written to Z4C_REG_ADM_ADJ (the lapse and shift through their copies, the
 * metric and extrinsic curvature through the conformal decomposition and
 * Gamma~ = -d_b g~^{ba}).  Z4C_REG_ADJ is overwritten. */
int z4c_adj_adm_to_z4c(z4c_ctx *ctx);
/* The accumulated adjoints of {shift_eta, damp_kappa1}; reset != 0 zeroes
 * them afterwards. */
int z4c_adj_params(z4c_ctx *ctx, double pbar[2], int reset);
/* Gradient of J_total = w_final J(u_n) + w_step sum_{k=1..n} J(u_k) over n
 * steps from the state in Z4C_REG_U (left unchanged) with revolve-style
 * binomial checkpointing: nsnap state snapshots (device memory, kept in the
 * context for later calls; nsnap < 0: as many as z4c_adj_snapshots finds
 * room for), a schedule that minimises the recomputed steps for that
 * count.  On return Z4C_REG_ADJ holds dJ_total/du_0, pbar the parameter
 * adjoints, *J the objective; stats (may be NULL) receives {forward steps
 * (the first sweep and every recomputation), adjoint steps, seconds, the
 * schedule's recomputed steps}. */
int z4c_adj_gradient(z4c_ctx *ctx, double dt, int nsteps, int nsnap, double w_final,
                     double w_step, double *J, double pbar[2], double stats[4]);
/* The Weyl-scalar term of the objective: with sphere >= 0 (a z4c_wave_add
 * sphere, full, not bitant) the objective of z4c_adj_objective,
 * z4c_adj_objective_adj and z4c_adj_gradient becomes J + weight J_W,
 * J_W = sum over the sphere's owned vertices p of w_p |psi4(p)|^2 (w_p the
 * vertex's quadrature weight, rad^2 times its dual cell's area; psi4 of
 * Z4cWeyl after Z4cToADM, the Weyl register's ghost fill and the sphere
 * interpolation).  Its adjoint: the interpolation and the ghost fill
 * transposed, at each interior vertex the adjoints of psi4's local inputs by
 * forward-mode differentiation, then the transposed stencils and Z4cToADM
 * transposed.  sphere < 0 removes the term.  Allocates the term's buffers
 * (an ADM register, three Weyl registers, 30 values per interior vertex). */
int z4c_adj_set_weyl(z4c_ctx *ctx, int sphere, double weight);
/* The number of revolve snapshots a gradient over nsteps steps can hold in
 * the device memory that is free now (state-sized buffers; 2 GiB and 2% of
 * the device are left over), at most nsteps - 1: the checkpointing sized to
 * HBM. */
int z4c_adj_snapshots(z4c_ctx *ctx, int nsteps, int *nsnap);

/* ---- allocation-free variant ----------------------------------------------
 *
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc.  Some host programs own all device memory through their own
 * allocator (a framework's caching allocator, or a pool reserved at start-up)
 * and may not allocate behind its back; others run the right-hand side inside
 * a time-stepping loop that cannot take the device-wide synchronisation a
 * cudaMalloc/cudaFree pair implies.  z4c_rhs needs a context, and creating one
 * allocates, so those callers use this instead.
 *
 * z4c_rhs_noalloc computes what z4c_rhs computes (Z4c::Z4cRHS with the
 * derivative precompute fused, Kreiss-Oliger included) for nblocks MeshBlocks
 * of nx[0] x nx[1] x nx[2] cells and vertex spacing dx, all with the same
 * spacing.  u and rhs are caller-owned DEVICE buffers in the register layout
 * [block][22][nn2][nn1][nn0], nn = nx + 1 + 2*Z4C_NG; only the interior
 * vertices of rhs are written, and u must already carry filled ghosts.  Work is
 * enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream).
 *
 * The scratch of the right-hand-side passes lives in one fixed array of
 * Z4C_NOALLOC_SCRATCH_MIB MiB compiled into the library; every GPU that loads
 * the library holds it until the process exits.  The first call on a device
 * looks the array's device address up (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  With CUDA's lazy
 * module loading (the default) that first lookup is also when the driver
 * loads the library's device code on that device and reserves the array: an
 * allocation of its own.  So make one call (any size) outside the region that
 * must not allocate, e.g. at start-up; every later call on that device
 * allocates nothing.  A CUDA error left pending by earlier work is reported
 * (Z4C_ECUDA) before anything is enqueued, not taken for this call's.  Blocks are
 * processed in chunks that fit the array; a MeshBlock whose scratch alone
 * (33 doubles per vertex, ghosts included, plus 28 per interior vertex)
 * exceeds it -- above roughly 45^3 cells -- is rejected with Z4C_EINVAL
 * before any work is enqueued.  Every call shares
 * the array and it keeps the previous call's contents (nothing in it needs to
 * start at zero); calls whose work overlaps on the GPU race on it, so
 * serialise them (one stream, or events between streams).  No cudaMalloc,
 * cudaFree or allocating library routine is called. */
#define Z4C_NOALLOC_SCRATCH_MIB 64
int z4c_rhs_noalloc(const double *u, double *rhs, int nblocks, const int nx[3],
                    const double dx[3], const z4c_params_t *params, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* Z4C_B200_H */

// Vertex-centred ghost exchange of a mesh whose MeshBlocks sit on several
// refinement levels (static mesh refinement): the plan built once on the
// host from the blocks' logical locations and the kernels that run it.
#pragma once

#include <cuda_runtime.h>

#include "z4c_common.cuh"
#include "z4c_refine.cuh"

namespace z4c {

// One unpack op of a receiving block (host side): a box of its fine array or
// coarse buffer receives (copy or add) the box of the same shape that starts
// at slo in the sending block's fine array or restricted coarse interior.
// Ops of a block run in the reference's neighbour order.
enum MlMode { kMlCopy = 0, kMlAdd = 1 };
struct MlOp {
  int blk, coarse, mode;
  int lo[3], hi[3];  // inclusive
  int count;         // vertices in the box
  int sblk, scoarse;
  int slo[3];
};

// The ops' boxes are unions of the 7 x 7 x 7 compact zones of an array
// (ghosts, shared vertex, lower half, midpoint, upper half, shared vertex,
// ghosts per axis), so every vertex of a zone receives the same ordered
// contributions: the device gathers them per vertex.  d = source index
// minus destination index.
struct MlContrib {
  int sblk;
  short scoarse, mode;
  short d[3];
  short pad;
};

// One physical face of one block: the extrapolation fills the ghosts beyond
// lo[ax] (inner face) or hi[ax] (outer face) along the transverse ranges.
struct MlBc {
  int blk, outer;
  int lo[3], hi[3];
};

struct MlPlan {
  int nblocks = 0;
  int nx[3] = {}, nn[3] = {}, cn[3] = {};
  long long fvol = 0, cvol = 0;
  double* csrc = nullptr;    // restricted interiors [block][Z4C_NVAR][cvol] (read-only in unpack)
  double* coarse = nullptr;  // the receiving coarse buffers, same layout
  MlContrib* contrib = nullptr;
  int* zstart = nullptr;     // contributions of zone z of array a of block b:
                             // [zstart[(b*2+a)*344+z], zstart[(b*2+a)*344+z+1])
  int ncontrib = 0;
  int max_block_contrib = 0;  // the most contributions of one block (shared-memory size)
  unsigned char* mult = nullptr;  // node multiplicity per block in the 7^3 compact zones
  double inv[64] = {};            // 1 / m
  MlBc* bc[2][3] = {};       // [fine, coarse][axis]
  int nbc[2][3] = {};
  refine::RefGeom* pro = nullptr;  // prolongation boxes
  int* pro_blk = nullptr;
  int npro = 0;
  int ncoarser = 0;          // blocks with a coarser neighbour
  unsigned char* coarser = nullptr;  // [block] 1 where a coarser neighbour is prolonged
                                     // from the coarse buffer (no other reads it)
};

// Builds the plan for nblocks MeshBlocks of nx cells given in gid order by
// their logical locations locs[b] = {level, lx1, lx2, lx3} (absolute levels;
// the root grid of nroot blocks per axis sits at the level whose 2^level
// first covers the largest nroot).  Checks that the blocks tile the root
// grid and obey the 2:1 level balance.  Allocates device memory.
// With query_out, only the checks and the neighbour list of query_block are
// made: rows {gid, level, ox1, ox2, ox3, fi1, fi2} (at most 56), the count
// returned; query_block == -2 builds and checks the whole plan without
// device memory and writes its sizes {unpack ops, vertices they move per
// variable, prolongation boxes, boundary faces}.
int ml_build(const int nroot[3], const int nx[3], const int bc[6], int nblocks,
             const long long* locs, MlPlan& plan, int query_block = -1, int* query_out = nullptr);
void ml_free(MlPlan& plan);
// One ghost fill of nvar variables (block stride reg_nvar * fvol): src holds
// the blocks' interiors, dst receives interiors and ghosts.
int launch_ml_exchange(const MlPlan& plan, const double* src, double* dst, int nvar, int reg_nvar,
                       cudaStream_t st);
// The transpose of launch_ml_exchange (the adjoint of a ghost fill): ubar, the
// adjoint of dst (every vertex), is consumed in place; wbar receives the
// adjoint of src (the interiors; ghosts zero).  The plan's coarse buffers
// serve as scratch.  owner: the prolongation owner table that
// launch_ml_prolong_owner fills (an int per fine vertex of every block).
int launch_ml_exchange_adj(const MlPlan& plan, double* ubar, double* wbar, const int* owner,
                           int nvar, int reg_nvar, cudaStream_t st);
int launch_ml_prolong_owner(const MlPlan& plan, int* owner, cudaStream_t st);
// The root level of a root grid of nroot blocks per axis.
int ml_root_level(const int nroot[3]);

}  // namespace z4c

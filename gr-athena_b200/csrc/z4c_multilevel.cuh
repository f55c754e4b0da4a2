// Vertex-centred ghost exchange of a mesh whose MeshBlocks sit on several
// refinement levels (static mesh refinement): the plan built once on the
// host from the blocks' logical locations and the kernels that run it.
#pragma once

#include <cuda_runtime.h>

#include "z4c_common.cuh"
#include "z4c_refine.cuh"

namespace z4c {

// One box of one block's fine array or coarse buffer.  Pack ops copy the box
// into the message buffer; unpack ops of a receiving block run in order:
// copy or add from the buffer, zero the ghosts of the coarse buffer, or
// multiply by the inverse node multiplicity.
enum MlMode { kMlCopy = 0, kMlAdd = 1, kMlZeroGhosts = 2, kMlScale = 3 };
struct MlOp {
  int blk, coarse, mode;
  int lo[3], hi[3];  // inclusive
  int count;         // vertices in the box
  long long off;     // message-buffer offset of variable 0 (variable stride: count)
  double inv;
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
  double* coarse = nullptr;  // [block][Z4C_NVAR][cvol]
  double* buf = nullptr;     // messages of Z4C_NVAR variables
  long long buf_elems = 0;
  MlOp* pack = nullptr;
  int npack = 0;
  MlOp* unpack = nullptr;
  int* ustart = nullptr;     // unpack ops of block b: [ustart[b], ustart[b+1])
  int nunpack = 0;
  MlBc* bc[2][3] = {};       // [fine, coarse][axis]
  int nbc[2][3] = {};
  refine::RefGeom* pro = nullptr;  // prolongation boxes
  int* pro_blk = nullptr;
  int npro = 0;
  int ncoarser = 0;          // blocks with a coarser neighbour
};

// Builds the plan for nblocks MeshBlocks of nx cells given in gid order by
// their logical locations locs[b] = {level, lx1, lx2, lx3} (absolute levels;
// the root grid of nroot blocks per axis sits at the level whose 2^level
// first covers the largest nroot).  Checks that the blocks tile the root
// grid and obey the 2:1 level balance.  Allocates device memory.
// With query_out, only the checks and the neighbour list of query_block are
// made: rows {gid, level, ox1, ox2, ox3, fi1, fi2} (at most 56), the count
// returned; query_block == -2 builds and checks the whole plan without
// device memory and writes its op counts {pack, unpack, prolongation boxes,
// boundary faces}.
int ml_build(const int nroot[3], const int nx[3], const int bc[6], int nblocks,
             const long long* locs, MlPlan& plan, int query_block = -1, int* query_out = nullptr);
void ml_free(MlPlan& plan);
// One ghost fill of nvar variables (block stride reg_nvar * fvol): src holds
// the blocks' interiors, dst receives interiors and ghosts.
int launch_ml_exchange(const MlPlan& plan, const double* src, double* dst, int nvar, int reg_nvar,
                       cudaStream_t st);
// The root level of a root grid of nroot blocks per axis.
int ml_root_level(const int nroot[3]);

}  // namespace z4c

// Reference restart files (outputs/restart.cpp) for the Z4c vacuum state of
// a uniform mesh: host-side reader and writer (see z4c_restart.cu).
#pragma once

#include <string>
#include <vector>

#include "../../include/z4c_b200.h"

namespace z4c {

// Parses path: header fields into *info, the parameter text (through the
// byte after "<par_end>") into *text and, when u_grid is not null, the state
// of every MeshBlock in context (grid) order, [block][var][k][j][i].
// locs (optional) receives {level, lx1, lx2, lx3} per MeshBlock in gid order;
// on a refined mesh (blocks above the root level) u_grid holds the blocks in
// that order, on a uniform one in grid order.
int restart_read_file(const char* path, z4c_restart_info_t* info, std::string* text,
                      std::vector<double>* u_grid, std::string* err,
                      std::vector<long long>* locs = nullptr);
// Writes a restart file the reference can restart from: the parameter text,
// the header, the trackers (6 doubles each), the ID list and the state of
// every MeshBlock, blocks in gid order.
// With locs (a refined mesh of nblocks_refined blocks in gid order, u_grid
// in that order) the ID list carries each block's level.
int restart_write_file(const char* path, const std::string& text, const z4c_mesh_desc_t& mesh,
                       const double* u_grid, double time, double dt, int ncycle, int ntrk,
                       const double* trk6, std::string* err, const long long* locs = nullptr,
                       int nblocks_refined = 0);

}  // namespace z4c

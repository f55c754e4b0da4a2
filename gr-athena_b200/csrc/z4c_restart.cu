// Restart files of the reference (outputs/restart.cpp:43-352 writes them,
// the restart constructor of Mesh, mesh/mesh.cpp:775-1420, and
// ParameterInput::LoadFromFile, parameter_input.cpp:310-348, read them), for
// the Z4c vacuum build on a uniform mesh.
//
// Layout, all little endian as the reference's memcpy/fwrite leave it:
//   parameter text (ParameterInput::ParameterDump) up to and including the
//   first "<par_end>" and the byte after it
//   int nbtotal, int root_level, RegionSize mesh_size (9 doubles, 3 ints,
//   4 bytes of padding), double time, double dt, int ncycle,
//   uint64 datasize (bytes per MeshBlock)
//   user Mesh data: here only the puncture trackers, 6 doubles each
//   (position, shift at the position: PunctureTracker pos, betap)
//   ID list: per MeshBlock in gid order a LogicalLocation (3 int64, int,
//   4 bytes of padding) and its cost (double)
//   per MeshBlock in gid order: Z4c storage.u, [var][k][j][i]
// Host code only; the context entry points that move the state to and from
// the device are in z4c_capi.cu.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/z4c_b200.h"
#include "z4c_restart.cuh"

namespace z4c {

int set_error(int code, const char* msg);

namespace {

constexpr int64_t kHeaderBytes = 4 + 4 + 88 + 8 + 8 + 4 + 8;  // 124
constexpr int64_t kIdBytes = 40;                              // LogicalLocation + cost
constexpr int64_t kTrackerBytes = 6 * 8;

int fail(std::string* err, const std::string& m) {
  *err = m;
  return Z4C_EINVAL;
}

// value of `key` in block <blk> of a parameter text, or "" when absent
std::string param(const std::string& text, const std::string& blk, const std::string& key) {
  const std::string head = "<" + blk + ">";
  size_t p = text.find(head);
  while (p != std::string::npos && p > 0 && text[p - 1] != '\n') p = text.find(head, p + 1);
  if (p == std::string::npos) return "";
  size_t line = text.find('\n', p);
  while (line != std::string::npos && line + 1 < text.size()) {
    const size_t next = text.find('\n', line + 1);
    std::string l = text.substr(line + 1, (next == std::string::npos ? text.size() : next) - line - 1);
    const size_t hash = l.find('#');
    if (hash != std::string::npos) l = l.substr(0, hash);
    size_t a = l.find_first_not_of(" \t");
    if (a != std::string::npos && l[a] == '<') break;  // next block
    const size_t eq = l.find('=');
    if (a != std::string::npos && eq != std::string::npos) {
      std::string k = l.substr(a, eq - a);
      k.erase(k.find_last_not_of(" \t") + 1);
      if (k == key) {
        std::string v = l.substr(eq + 1);
        const size_t b = v.find_first_not_of(" \t");
        if (b == std::string::npos) return "";
        v = v.substr(b);
        v.erase(v.find_last_not_of(" \t\r") + 1);
        return v;
      }
    }
    line = next;
  }
  return "";
}

int level_for(int nb) {
  int l = 0;
  while ((1 << l) < nb) ++l;
  return l;
}

}  // namespace

int restart_read_file(const char* path, z4c_restart_info_t* info, std::string* text,
                      std::vector<double>* u_grid, std::string* err,
                      std::vector<long long>* locs) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(err, std::string("cannot open restart file ") + path);
  std::fseek(fp, 0, SEEK_END);
  const int64_t size = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  // the parameter text ends at the first "<par_end>" (searched within the
  // first 400 kB, as the reference does) plus one byte
  const int64_t scan = size < 409600 ? size : 409600;
  std::string head((size_t)scan, '\0');
  if ((int64_t)std::fread(&head[0], 1, (size_t)scan, fp) != scan) {
    std::fclose(fp);
    return fail(err, "restart file: short read");
  }
  const size_t loc = head.find("<par_end>");
  if (loc == std::string::npos) {
    std::fclose(fp);
    return fail(err, "restart file: <par_end> not found in the first 400 kB");
  }
  const int64_t tbytes = (int64_t)loc + 10;
  *text = head.substr(0, (size_t)tbytes);
  if (tbytes + kHeaderBytes > size) {
    std::fclose(fp);
    return fail(err, "restart file: truncated header");
  }
  unsigned char h[kHeaderBytes];
  std::fseek(fp, (long)tbytes, SEEK_SET);
  if (std::fread(h, 1, kHeaderBytes, fp) != (size_t)kHeaderBytes) {
    std::fclose(fp);
    return fail(err, "restart file: short read");
  }
  z4c_restart_info_t I;
  std::memset(&I, 0, sizeof(I));
  int64_t o = 0;
  std::memcpy(&I.nbtotal, h + o, 4); o += 4;
  std::memcpy(&I.root_level, h + o, 4); o += 4;
  std::memcpy(I.xmin, h + o, 24); o += 24;
  std::memcpy(I.xmax, h + o, 24); o += 24;
  std::memcpy(I.xrat, h + o, 24); o += 24;
  std::memcpy(I.mesh_nx, h + o, 12); o += 12 + 4;
  std::memcpy(&I.time, h + o, 8); o += 8;
  std::memcpy(&I.dt, h + o, 8); o += 8;
  std::memcpy(&I.ncycle, h + o, 4); o += 4;
  uint64_t ds = 0;
  std::memcpy(&ds, h + o, 8);
  I.datasize = ds;
  I.text_bytes = tbytes;
  if (I.nbtotal < 1 || ds == 0) {
    std::fclose(fp);
    return fail(err, "restart file: bad header");
  }
  const int64_t body = (kIdBytes + (int64_t)ds) * I.nbtotal;
  const int64_t udsize = size - body - tbytes - kHeaderBytes;
  if (udsize < 0) {
    std::fclose(fp);
    return fail(err, "restart file: shorter than its header says");
  }
  // user Mesh data: only PunctureTracker records are understood
  const std::string np_s = param(*text, "z4c", "npunct");
  const int npunct = np_s.empty() ? 0 : std::atoi(np_s.c_str());
  if (udsize != kTrackerBytes * npunct || npunct > Z4C_MAX_TRACKERS) {
    std::fclose(fp);
    return fail(err, "restart file: user Mesh data other than " + std::to_string(npunct) +
                         " puncture tracker(s) is not supported");
  }
  I.ntrackers = npunct;
  if (npunct > 0 && std::fread(I.trackers, 1, (size_t)udsize, fp) != (size_t)udsize) {
    std::fclose(fp);
    return fail(err, "restart file: short read");
  }
  // ID list: every block on the root level of a uniform mesh
  std::vector<unsigned char> ids((size_t)(kIdBytes * I.nbtotal));
  if (std::fread(ids.data(), 1, ids.size(), fp) != ids.size()) {
    std::fclose(fp);
    return fail(err, "restart file: short read");
  }
  std::vector<int64_t> loc3((size_t)3 * I.nbtotal);
  std::vector<int> levels((size_t)I.nbtotal);
  for (int a = 0; a < 3; ++a) I.nb[a] = 0;
  I.nlevels = 1;
  int maxlev = I.root_level;
  for (int b = 0; b < I.nbtotal; ++b) {
    std::memcpy(&loc3[3 * (size_t)b], &ids[(size_t)(kIdBytes * b)], 24);
    std::memcpy(&levels[b], &ids[(size_t)(kIdBytes * b) + 24], 4);
    if (levels[b] < I.root_level || levels[b] > I.root_level + 20) {
      std::fclose(fp);
      return fail(err, "restart file: MeshBlock level out of range");
    }
    maxlev = levels[b] > maxlev ? levels[b] : maxlev;
  }
  if (locs) {
    locs->resize((size_t)4 * I.nbtotal);
    for (int b = 0; b < I.nbtotal; ++b) {
      (*locs)[4 * (size_t)b] = levels[b];
      for (int a = 0; a < 3; ++a) (*locs)[4 * (size_t)b + 1 + a] = loc3[3 * (size_t)b + a];
    }
  }
  if (maxlev > I.root_level) {
    // a refined mesh: the root grid from the <meshblock> size of the
    // parameter text, the blocks' data in gid order as stored
    I.nlevels = maxlev - I.root_level + 1;
    for (int a = 0; a < 3; ++a) {
      const std::string v = param(text ? *text : std::string(), "meshblock",
                                  std::string("nx") + char('1' + a));
      I.block_nx[a] = v.empty() ? 0 : std::atoi(v.c_str());
      if (I.block_nx[a] < 1 || I.mesh_nx[a] % I.block_nx[a]) {
        std::fclose(fp);
        return fail(err, "restart file: refined mesh without a <meshblock> size that divides the mesh");
      }
      I.nb[a] = I.mesh_nx[a] / I.block_nx[a];
    }
    const int64_t nvol = (int64_t)(I.block_nx[0] + 1 + 2 * Z4C_NG) *
                         (I.block_nx[1] + 1 + 2 * Z4C_NG) * (I.block_nx[2] + 1 + 2 * Z4C_NG);
    if ((int64_t)ds != (int64_t)Z4C_NVAR * nvol * 8) {
      std::fclose(fp);
      return fail(err, "restart file: MeshBlock data is not exactly the vertex-centred Z4c state "
                       "(other physics or user MeshBlock data)");
    }
    if (u_grid) {
      u_grid->assign((size_t)(Z4C_NVAR * nvol * I.nbtotal), 0.0);
      if (std::fread(u_grid->data(), 1, (size_t)ds * I.nbtotal, fp) != (size_t)ds * I.nbtotal) {
        std::fclose(fp);
        return fail(err, "restart file: short read");
      }
    }
    std::fclose(fp);
    *info = I;
    return Z4C_OK;
  }
  for (int b = 0; b < I.nbtotal; ++b) {
    for (int a = 0; a < 3; ++a) {
      const int64_t l = loc3[3 * (size_t)b + a];
      if (l < 0 || l >= (int64_t)1 << 20) {
        std::fclose(fp);
        return fail(err, "restart file: MeshBlock location out of range");
      }
      if (l + 1 > I.nb[a]) I.nb[a] = (int)(l + 1);
    }
  }
  if ((int64_t)I.nb[0] * I.nb[1] * I.nb[2] != I.nbtotal) {
    std::fclose(fp);
    return fail(err, "restart file: the MeshBlocks do not tile a box");
  }
  for (int a = 0; a < 3; ++a) {
    if (I.mesh_nx[a] % I.nb[a]) {
      std::fclose(fp);
      return fail(err, "restart file: mesh cells not divisible by the block count");
    }
    I.block_nx[a] = I.mesh_nx[a] / I.nb[a];
  }
  const int64_t nvol = (int64_t)(I.block_nx[0] + 1 + 2 * Z4C_NG) * (I.block_nx[1] + 1 + 2 * Z4C_NG) *
                       (I.block_nx[2] + 1 + 2 * Z4C_NG);
  if ((int64_t)ds != (int64_t)Z4C_NVAR * nvol * 8) {
    std::fclose(fp);
    return fail(err, "restart file: MeshBlock data is not exactly the vertex-centred Z4c state "
                     "(other physics or user MeshBlock data)");
  }
  if (u_grid) {
    u_grid->assign((size_t)(Z4C_NVAR * nvol * I.nbtotal), 0.0);
    std::vector<int> seen((size_t)I.nbtotal, 0);
    for (int b = 0; b < I.nbtotal; ++b) {
      const int64_t* l = &loc3[3 * (size_t)b];
      const int g = (int)(l[0] + I.nb[0] * (l[1] + (int64_t)I.nb[1] * l[2]));
      if (seen[g]++) {
        std::fclose(fp);
        return fail(err, "restart file: a MeshBlock location appears twice");
      }
      if (std::fread(&(*u_grid)[(size_t)(Z4C_NVAR * nvol * g)], 1, (size_t)ds, fp) != (size_t)ds) {
        std::fclose(fp);
        return fail(err, "restart file: short read");
      }
    }
  }
  std::fclose(fp);
  *info = I;
  return Z4C_OK;
}

int restart_write_file(const char* path, const std::string& text_in, const z4c_mesh_desc_t& m,
                       const double* u_grid, double time, double dt, int ncycle, int ntrk,
                       const double* trk6, std::string* err, const long long* locs,
                       int nblocks_refined) {
  // the parameter text, cut after the byte that follows its first
  // "<par_end>" (appended when the text has none)
  std::string text = text_in;
  size_t pe = text.find("<par_end>");
  if (pe == std::string::npos) {
    if (!text.empty() && text.back() != '\n') text += '\n';
    pe = text.size();
    text += "<par_end>\n";
  }
  if (text.size() < pe + 10) text += '\n';
  text = text.substr(0, pe + 10);
  const std::string np_s = param(text, "z4c", "npunct");
  const int npunct = np_s.empty() ? 0 : std::atoi(np_s.c_str());
  if (npunct != ntrk)
    return fail(err, "restart write: the parameter text has npunct = " + std::to_string(npunct) +
                         " but the state has " + std::to_string(ntrk) + " tracker(s)");
  const int nbt = locs ? nblocks_refined : m.nb[0] * m.nb[1] * m.nb[2];
  const int64_t nvol = (int64_t)(m.nx[0] + 1 + 2 * Z4C_NG) * (m.nx[1] + 1 + 2 * Z4C_NG) *
                       (m.nx[2] + 1 + 2 * Z4C_NG);
  const uint64_t ds = (uint64_t)(Z4C_NVAR * nvol * 8);
  int root = 0;
  for (int a = 0; a < 3; ++a) root = level_for(m.nb[a]) > root ? level_for(m.nb[a]) : root;
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return fail(err, std::string("cannot create restart file ") + path);
  bool ok = std::fwrite(text.data(), 1, text.size(), fp) == text.size();
  unsigned char h[kHeaderBytes];
  std::memset(h, 0, sizeof(h));
  int64_t o = 0;
  const double rat[3] = {1.0, 1.0, 1.0};
  int mnx[3];
  for (int a = 0; a < 3; ++a) mnx[a] = m.nb[a] * m.nx[a];
  std::memcpy(h + o, &nbt, 4); o += 4;
  std::memcpy(h + o, &root, 4); o += 4;
  std::memcpy(h + o, m.xmin, 24); o += 24;
  std::memcpy(h + o, m.xmax, 24); o += 24;
  std::memcpy(h + o, rat, 24); o += 24;
  std::memcpy(h + o, mnx, 12); o += 12 + 4;
  std::memcpy(h + o, &time, 8); o += 8;
  std::memcpy(h + o, &dt, 8); o += 8;
  std::memcpy(h + o, &ncycle, 4); o += 4;
  std::memcpy(h + o, &ds, 8);
  ok = ok && std::fwrite(h, 1, kHeaderBytes, fp) == (size_t)kHeaderBytes;
  if (ntrk > 0) ok = ok && std::fwrite(trk6, 8, (size_t)(6 * ntrk), fp) == (size_t)(6 * ntrk);
  if (locs) {  // a refined mesh: its blocks are already in gid order
    for (int b = 0; b < nbt; ++b) {
      unsigned char id[kIdBytes];
      std::memset(id, 0, sizeof(id));
      const int64_t l[3] = {locs[4 * b + 1], locs[4 * b + 2], locs[4 * b + 3]};
      const int lev = (int)locs[4 * b];
      const double cost = 1.0;
      std::memcpy(id, l, 24);
      std::memcpy(id + 24, &lev, 4);
      std::memcpy(id + 32, &cost, 8);
      ok = ok && std::fwrite(id, 1, kIdBytes, fp) == (size_t)kIdBytes;
    }
    ok = ok && std::fwrite(u_grid, 1, (size_t)ds * nbt, fp) == (size_t)ds * nbt;
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(err, std::string("restart write failed: ") + path);
    return Z4C_OK;
  }
  // blocks in gid order: the Morton order of the logical locations
  std::vector<int> order;
  for (int64_t key = 0; (int)order.size() < nbt; ++key) {
    int loc[3] = {0, 0, 0};
    for (int bit = 0; bit < 21; ++bit)
      for (int a = 0; a < 3; ++a) loc[a] |= (int)((key >> (3 * bit + a)) & 1) << bit;
    if (loc[0] < m.nb[0] && loc[1] < m.nb[1] && loc[2] < m.nb[2])
      order.push_back(loc[0] + m.nb[0] * (loc[1] + m.nb[1] * loc[2]));
  }
  for (int g : order) {
    unsigned char id[kIdBytes];
    std::memset(id, 0, sizeof(id));
    const int64_t l[3] = {g % m.nb[0], (g / m.nb[0]) % m.nb[1], g / (m.nb[0] * m.nb[1])};
    const double cost = 1.0;
    std::memcpy(id, l, 24);
    std::memcpy(id + 24, &root, 4);
    std::memcpy(id + 32, &cost, 8);
    ok = ok && std::fwrite(id, 1, kIdBytes, fp) == (size_t)kIdBytes;
  }
  for (int g : order)
    ok = ok && std::fwrite(u_grid + (size_t)(Z4C_NVAR * nvol * g), 1, (size_t)ds, fp) == (size_t)ds;
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) return fail(err, std::string("restart write failed: ") + path);
  return Z4C_OK;
}

}  // namespace z4c

using namespace z4c;

extern "C" {

int z4c_restart_info(const char* path, z4c_restart_info_t* info) {
  if (!path || !info) return set_error(Z4C_EINVAL, "null argument");
  std::string text, err;
  const int rc = restart_read_file(path, info, &text, nullptr, &err);
  return rc ? set_error(rc, err.c_str()) : Z4C_OK;
}

long long z4c_restart_text(const char* path, char* buf, long long cap) {
  if (!path) return set_error(Z4C_EINVAL, "null argument");
  z4c_restart_info_t info;
  std::string text, err;
  const int rc = restart_read_file(path, &info, &text, nullptr, &err);
  if (rc) return set_error(rc, err.c_str());
  if (buf && cap > 0) {
    const size_t n = text.size() < (size_t)(cap - 1) ? text.size() : (size_t)(cap - 1);
    std::memcpy(buf, text.data(), n);
    buf[n] = '\0';
  }
  return (long long)text.size();
}

int z4c_restart_read(const char* path, double* u) {
  if (!path || !u) return set_error(Z4C_EINVAL, "null argument");
  z4c_restart_info_t info;
  std::string text, err;
  std::vector<double> st;
  const int rc = restart_read_file(path, &info, &text, &st, &err);
  if (rc) return set_error(rc, err.c_str());
  std::memcpy(u, st.data(), st.size() * sizeof(double));
  return Z4C_OK;
}

int z4c_restart_write_host(const char* path, const char* par_text, const z4c_mesh_desc_t* mesh,
                           const double* u, double time, double dt, int ncycle, int ntrackers,
                           const double* trackers) {
  if (!path || !mesh || !u || (ntrackers > 0 && !trackers))
    return set_error(Z4C_EINVAL, "null argument");
  std::string err;
  const int rc = restart_write_file(path, par_text ? par_text : "", *mesh, u, time, dt, ncycle,
                                    ntrackers, trackers, &err);
  return rc ? set_error(rc, err.c_str()) : Z4C_OK;
}

}  // extern "C"

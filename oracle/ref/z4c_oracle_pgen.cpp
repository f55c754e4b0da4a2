// Problem generator linked into the GR-Athena++ reference build that serves as
// the parity oracle (test infrastructure only).
//
// <problem>/test selects the initial data:
//   gauge_wave1       reference ADMGaugeWave1 + GaugeGaugeWave1 + ADMToZ4c
//                     (pgen/z4c_awa_tests.cpp:52-55)
//   robust_stability  reference ADMRobustStability + GaugeRobStab + ADMToZ4c
//   one_puncture      reference ADMOnePuncture + GaugePreCollapsedLapse +
//                     ADMToZ4c (pgen/z4c_one_puncture.cpp:27-37)
//   minkowski         ADMMinkowski + GaugeGeodesic + ADMToZ4c
//   inject            Z4c state read from <problem>/inject_file (record "u",
//                     shape [nblocks, 22, nn3, nn2, nn1], blocks in gid order);
//                     the ADM register is then filled with Z4cToADM.
//   inject_adm        ADM state read from <problem>/inject_file (record "adm",
//                     [nblocks, 17, ...]) with lapse/shift from it, then
//                     ADMToZ4c.
//   brill_lindquist   conformally flat punctures psi = 1 + sum m_n / (2 r_n)
//                     of masses <problem>/bl_m_<n> at the puncture trackers'
//                     starting points <z4c>/bh_<n>_{x,y,z}, n < <z4c>/npunct
//                     (ADMOnePuncture, z4c/one_puncture_z4c.cpp:22-60, summed
//                     over punctures), pre-collapsed lapse and the constant
//                     shift <problem>/shift_{x,y,z} (default 0), then ADMToZ4c.
//
// Mesh hooks: <problem>/dump_initial and <problem>/dump_final name record files
// that receive the state of every block before the first and after the last
// step (u, adm, con and the block geometry).  <problem>/dump_blocks names a
// record file that receives, after the run, the MeshBlock list at the top of
// every main-loop iteration (after the previous iteration's regrid).
//
// With <mesh>/refinement = adaptive the refinement condition is the
// reference's Z4c_AMR::ShouldIRefine (z4c/z4c_amr.cpp:376-404), the one the
// two-puncture problem generator enrolls (pgen/z4c_two_punctures.cpp:225-237).
#include <cmath>
#include <cstdint>
#include <iostream>
#include <string>
#include <vector>

#include "athena.hpp"
#include "athena_arrays.hpp"
#include "coordinates/coordinates.hpp"
#include "mesh/mesh.hpp"
#include "parameter_input.hpp"
#include "z4c/z4c.hpp"
#include "z4c/puncture_tracker.hpp"
#include "z4c/z4c_amr.hpp"

#include "z4c_oracle_io.hpp"

namespace {

using z4c_oracle::Writer;

void CopyBlockArray(const AthenaArray<Real>& a, int nvar, double* dst) {
  const int nn3 = a.GetDim3(), nn2 = a.GetDim2(), nn1 = a.GetDim1();
  std::int64_t p = 0;
  for (int n = 0; n < nvar; ++n)
    for (int k = 0; k < nn3; ++k)
      for (int j = 0; j < nn2; ++j)
        for (int i = 0; i < nn1; ++i) dst[p++] = a(n, k, j, i);
}

void FillBlockArray(AthenaArray<Real>& a, int nvar, const double* src) {
  const int nn3 = a.GetDim3(), nn2 = a.GetDim2(), nn1 = a.GetDim1();
  std::int64_t p = 0;
  for (int n = 0; n < nvar; ++n)
    for (int k = 0; k < nn3; ++k)
      for (int j = 0; j < nn2; ++j)
        for (int i = 0; i < nn1; ++i) a(n, k, j, i) = src[p++];
}

// Brill-Lindquist data of the brill_lindquist test (see the header).
void BrillLindquist(ParameterInput* pin, Z4c* z) {
  const int np = pin->GetOrAddInteger("z4c", "npunct", 0);
  std::vector<Real> m(np), c(3 * np);
  for (int n = 0; n < np; ++n) {
    const std::string id = std::to_string(n);
    m[n] = pin->GetReal("problem", "bl_m_" + id);
    c[3 * n + 0] = pin->GetReal("z4c", "bh_" + id + "_x");
    c[3 * n + 1] = pin->GetReal("z4c", "bh_" + id + "_y");
    c[3 * n + 2] = pin->GetReal("z4c", "bh_" + id + "_z");
  }
  const Real shift[3] = {pin->GetOrAddReal("problem", "shift_x", 0.0),
                         pin->GetOrAddReal("problem", "shift_y", 0.0),
                         pin->GetOrAddReal("problem", "shift_z", 0.0)};
  AthenaArray<Real>& u_adm = z->storage.adm;
  z->ADMMinkowski(u_adm);
  Z4c::ADM_vars adm;
  Z4c::SetADMAliases(u_adm, adm);
  const int nn3 = z->mbi.nn3, nn2 = z->mbi.nn2, nn1 = z->mbi.nn1;
  for (int k = 0; k < nn3; ++k)
    for (int j = 0; j < nn2; ++j)
      for (int i = 0; i < nn1; ++i) {
        Real psi = 1.0;
        for (int n = 0; n < np; ++n) {
          const Real dx = z->mbi.x1(i) - c[3 * n + 0];
          const Real dy = z->mbi.x2(j) - c[3 * n + 1];
          const Real dz = z->mbi.x3(k) - c[3 * n + 2];
          const Real r = std::sqrt(dx * dx + dy * dy + dz * dz);
          psi = psi + 0.5 * m[n] / r;
        }
        adm.psi4(k, j, i) = z->psi4Regularized(std::pow(psi, 4.));
        for (int a = 0; a < 3; ++a)
          for (int b = a; b < 3; ++b) adm.g_dd(a, b, k, j, i) *= adm.psi4(k, j, i);
      }
  z->GaugePreCollapsedLapse(u_adm, z->storage.u);
  Z4c::Z4c_vars zv;
  Z4c::SetZ4cAliases(z->storage.u, zv);
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < nn3; ++k)
      for (int j = 0; j < nn2; ++j)
        for (int i = 0; i < nn1; ++i) {
          zv.beta_u(a, k, j, i) = shift[a];
          adm.beta_u(a, k, j, i) = shift[a];
        }
}

// Z4c_AMR::ShouldIRefine of the block (1 refine, -1 derefine, 0 keep).
int Z4cRefinementCondition(MeshBlock* pmb) {
  return pmb->pz4c->pz4c_amr->ShouldIRefine(pmb);
}

// MeshBlock lists seen at the top of each main-loop iteration (dump_blocks):
// rows of (ncycle, gid, level, lx1, lx2, lx3), (ncycle, time, dt) and the
// puncture trackers' positions then (the ones the iteration's refinement
// flags see).
std::vector<std::int32_t> g_block_rows;
std::vector<double> g_cycle_rows;
std::vector<double> g_tracker_rows;

void RecordBlocks(Mesh* pm) {
  const auto& blocks = pm->GetMeshBlocksCached();
  std::vector<const MeshBlock*> by_gid(blocks.size(), nullptr);
  for (auto* b : blocks) by_gid.at(b->gid) = b;
  for (const MeshBlock* b : by_gid) {
    g_block_rows.push_back(pm->ncycle);
    g_block_rows.push_back(b->gid);
    g_block_rows.push_back(b->loc.level);
    g_block_rows.push_back(static_cast<std::int32_t>(b->loc.lx1));
    g_block_rows.push_back(static_cast<std::int32_t>(b->loc.lx2));
    g_block_rows.push_back(static_cast<std::int32_t>(b->loc.lx3));
  }
  g_cycle_rows.push_back(pm->ncycle);
  g_cycle_rows.push_back(pm->time);
  g_cycle_rows.push_back(pm->dt);
  for (auto* t : pm->pz4c_tracker)
    for (int a = 0; a < 3; ++a) g_tracker_rows.push_back(t->GetPos(a));
}

}  // namespace

namespace z4c_oracle {

// Writes the geometry of every block (gid order): logical locations, vertex
// and cell-centre coordinates and the spacing used by the FD operators.
void DumpGeometry(Mesh* pm, Writer& w) {
  const auto& blocks = pm->GetMeshBlocksCached();
  const int nb = static_cast<int>(blocks.size());
  Z4c* z0 = blocks[0]->pz4c;
  const int nn1 = z0->mbi.nn1, nn2 = z0->mbi.nn2, nn3 = z0->mbi.nn3;
  std::vector<const MeshBlock*> by_gid(nb, nullptr);
  for (auto* b : blocks) by_gid.at(b->gid) = b;
  std::vector<std::int32_t> meta;
  std::vector<double> geom;
  for (const MeshBlock* b : by_gid) {
    meta.push_back(b->gid);
    meta.push_back(b->loc.level);
    meta.push_back(static_cast<std::int32_t>(b->loc.lx1));
    meta.push_back(static_cast<std::int32_t>(b->loc.lx2));
    meta.push_back(static_cast<std::int32_t>(b->loc.lx3));
    meta.push_back(b->block_size.nx1);
    meta.push_back(b->block_size.nx2);
    meta.push_back(b->block_size.nx3);
  }
  w.i32("meta", {nb, 8}, meta.data());
  {
    std::vector<double> t = {pm->time, pm->dt};
    w.f64("time_dt", {2}, t.data());
  }
  // vertex (x?f) and cell-centre (x?v) coordinates and the FD spacing
  for (const MeshBlock* b : by_gid) {
    const Coordinates* c = b->pcoord;
    for (int i = 0; i < nn1; ++i) geom.push_back(c->x1f(i));
    for (int j = 0; j < nn2; ++j) geom.push_back(c->x2f(j));
    for (int k = 0; k < nn3; ++k) geom.push_back(c->x3f(k));
  }
  w.f64("xf", {nb, nn1 + nn2 + nn3}, geom.data());
  geom.clear();
  for (const MeshBlock* b : by_gid) {
    const Coordinates* c = b->pcoord;
    for (int i = 0; i < nn1 - 1; ++i) geom.push_back(c->x1v(i));
    for (int j = 0; j < nn2 - 1; ++j) geom.push_back(c->x2v(j));
    for (int k = 0; k < nn3 - 1; ++k) geom.push_back(c->x3v(k));
  }
  w.f64("xv", {nb, nn1 + nn2 + nn3 - 3}, geom.data());
  geom.clear();
  for (const MeshBlock* b : by_gid) {
    geom.push_back(b->pcoord->dx1f(0));
    geom.push_back(b->pcoord->dx2f(0));
    geom.push_back(b->pcoord->dx3f(0));
  }
  w.f64("dx", {nb, 3}, geom.data());
}

// Writes the state and geometry of every block (gid order) to a record file.
void DumpMesh(Mesh* pm, const std::string& path) {
  const auto& blocks = pm->GetMeshBlocksCached();
  const int nb = static_cast<int>(blocks.size());
  if (nb == 0) return;
  Z4c* z0 = blocks[0]->pz4c;
  const int nn1 = z0->mbi.nn1, nn2 = z0->mbi.nn2, nn3 = z0->mbi.nn3;
  const std::int64_t nvol = static_cast<std::int64_t>(nn1) * nn2 * nn3;
  std::vector<const MeshBlock*> by_gid(nb, nullptr);
  for (auto* b : blocks) by_gid.at(b->gid) = b;

  Writer w(path);
  DumpGeometry(pm, w);
  std::vector<double> buf;
  auto dump = [&](const char* name, int nvar, auto getter) {
    buf.assign(static_cast<size_t>(nb) * nvar * nvol, 0.0);
    for (int g = 0; g < nb; ++g)
      CopyBlockArray(getter(by_gid[g]->pz4c), nvar, &buf[g * nvar * nvol]);
    w.f64(name, {nb, nvar, nn3, nn2, nn1}, buf.data());
  };
  dump("u", Z4c::N_Z4c, [](Z4c* z) -> AthenaArray<Real>& { return z->storage.u; });
  dump("adm", Z4c::N_ADM, [](Z4c* z) -> AthenaArray<Real>& { return z->storage.adm; });
  dump("con", Z4c::N_CON, [](Z4c* z) -> AthenaArray<Real>& { return z->storage.con; });
}

}  // namespace z4c_oracle

void MeshBlock::ProblemGenerator(ParameterInput* pin) {
  const std::string test = pin->GetOrAddString("problem", "test", "gauge_wave1");
  Z4c* z = pz4c;
  if (test == "gauge_wave1") {
    z->ADMGaugeWave1(z->storage.adm);
    z->GaugeGaugeWave1(z->storage.u);
  } else if (test == "robust_stability") {
    z->ADMRobustStability(z->storage.adm);
    z->GaugeRobStab(z->storage.u);
  } else if (test == "one_puncture") {
    z->ADMOnePuncture(pin, z->storage.adm);
    z->GaugePreCollapsedLapse(z->storage.adm, z->storage.u);
  } else if (test == "minkowski") {
    z->ADMMinkowski(z->storage.adm);
    z->GaugeGeodesic(z->storage.u);
  } else if (test == "brill_lindquist") {
    BrillLindquist(pin, z);
  } else if (test == "inject" || test == "inject_adm") {
    const std::string path = pin->GetString("problem", "inject_file");
    const auto recs = z4c_oracle::read_all(path);
    const bool is_adm = (test == "inject_adm");
    const auto& r = z4c_oracle::find(recs, is_adm ? "adm" : "u");
    const int nvar = is_adm ? Z4c::N_ADM : Z4c::N_Z4c;
    AthenaArray<Real>& dst = is_adm ? z->storage.adm : z->storage.u;
    const std::int64_t per = static_cast<std::int64_t>(nvar) * dst.GetDim3() *
                             dst.GetDim2() * dst.GetDim1();
    if (r.dims.size() != 5 || r.dims[1] != nvar || r.dims[2] != dst.GetDim3() ||
        r.dims[3] != dst.GetDim2() || r.dims[4] != dst.GetDim1() ||
        gid >= r.dims[0]) {
      std::cerr << "inject: shape mismatch for gid " << gid << std::endl;
      std::exit(2);
    }
    FillBlockArray(dst, nvar, &r.f64[gid * per]);
    if (!is_adm) {
      z->storage.mat.ZeroClear();
      z->Z4cToADM(z->storage.u, z->storage.adm);
      return;
    }
    // lapse and shift come from the ADM record
    Z4c::Z4c_vars zv;
    Z4c::SetZ4cAliases(z->storage.u, zv);
    for (int k = 0; k < dst.GetDim3(); ++k)
      for (int j = 0; j < dst.GetDim2(); ++j)
        for (int i = 0; i < dst.GetDim1(); ++i) {
          zv.alpha(k, j, i) = z->storage.adm(Z4c::I_ADM_alpha, k, j, i);
          for (int a = 0; a < 3; ++a)
            zv.beta_u(a, k, j, i) = z->storage.adm(Z4c::I_ADM_betax + a, k, j, i);
        }
  } else {
    std::cerr << "unknown problem/test " << test << std::endl;
    std::exit(2);
  }
  z->storage.mat.ZeroClear();
  z->ADMToZ4c(z->storage.adm, z->storage.u);
}

void Mesh::InitUserMeshData(ParameterInput* pin) {
  if (adaptive) EnrollUserRefinementCondition(Z4cRefinementCondition);
}

// Called at the top of every main-loop iteration (main.cpp:167): only the
// first call sees the initial state.
void Mesh::UserWorkBeforeLoop(ParameterInput* pin) {
  static bool dumped = false;
  const std::string path = pin->GetOrAddString("problem", "dump_initial", "");
  if (!path.empty() && !dumped) z4c_oracle::DumpMesh(this, path);
  dumped = true;
  if (!pin->GetOrAddString("problem", "dump_blocks", "").empty()) RecordBlocks(this);
}

void Mesh::UserWorkAfterLoop(ParameterInput* pin) {
  const std::string path = pin->GetOrAddString("problem", "dump_final", "");
  if (!path.empty()) z4c_oracle::DumpMesh(this, path);
  const std::string blocks = pin->GetOrAddString("problem", "dump_blocks", "");
  if (!blocks.empty()) {
    RecordBlocks(this);  // the list the last iteration's regrid left
    z4c_oracle::Writer w(blocks);
    const std::int64_t nrow = static_cast<std::int64_t>(g_block_rows.size() / 6);
    const std::int64_t ncyc = static_cast<std::int64_t>(g_cycle_rows.size() / 3);
    w.i32("blocks", {nrow, 6}, g_block_rows.data());
    w.f64("cycles", {ncyc, 3}, g_cycle_rows.data());
    const std::int64_t ntr = static_cast<std::int64_t>(pz4c_tracker.size());
    if (ntr > 0) w.f64("trackers", {ncyc, ntr, 3}, g_tracker_rows.data());
  }
}

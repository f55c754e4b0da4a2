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
//
// Mesh hooks: <problem>/dump_initial and <problem>/dump_final name record files
// that receive the state of every block before the first and after the last
// step (u, adm, con and the block geometry).
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

// Called at the top of every main-loop iteration (main.cpp:167): only the
// first call sees the initial state.
void Mesh::UserWorkBeforeLoop(ParameterInput* pin) {
  static bool dumped = false;
  const std::string path = pin->GetOrAddString("problem", "dump_initial", "");
  if (!path.empty() && !dumped) z4c_oracle::DumpMesh(this, path);
  dumped = true;
}

void Mesh::UserWorkAfterLoop(ParameterInput* pin) {
  const std::string path = pin->GetOrAddString("problem", "dump_final", "");
  if (!path.empty()) z4c_oracle::DumpMesh(this, path);
}

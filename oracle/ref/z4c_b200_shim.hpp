// Z4cB200: the reference-side adapter a GR-Athena++ maintainer adds to use
// the B200 library (include/z4c_b200.h, libz4c_b200.so) from the reference's
// own driver.  It keeps the Z4c member-function signatures (z4c/z4c.hpp:
// 448-539) and forwards each call to the C ABI; errors go through the
// reference's ATHENA_ERROR path.  Built against the reference headers by
// oracle/ref/Makefile into the operator driver's shim mode (z4c_ops_shim),
// which calls these in place of Z4c::Z4cRHS, Z4c::AlgConstr and
// Z4c::Z4cToADM, so that the reference's own driver checks the replacement.
//
// Operator-level use: the block's AthenaArray is uploaded, the operator runs
// on the device for that block, and the result is downloaded; the entries
// the reference operator writes are the ones copied back (the interior for
// the right-hand side, every vertex for AlgConstr and Z4cToADM).  A driver
// that keeps the state on the device uses z4c_stage / z4c_evolve instead.
#pragma once

#include <sstream>
#include <vector>

#include "athena.hpp"
#include "athena_arrays.hpp"
#include "mesh/mesh.hpp"
#include "z4c/z4c.hpp"

#include "z4c_b200.h"

class Z4cB200 {
 public:
  // One context over the Mesh's uniform root grid, with the options of pz
  // (Z4c::opt, z4c.hpp:357-431) and the block size of pmb.
  Z4cB200(Mesh* pm, const MeshBlock* pmb, const Z4c* pz, bool butcher) : pm_(pm) {
    const RegionSize& ms = pm->mesh_size;
    const RegionSize& bs = pmb->block_size;
    z4c_mesh_desc_t md{};
    // root grid: the mesh's cells over the block's (Mesh::nrbx1..3)
    md.nb[0] = ms.nx1 / bs.nx1; md.nb[1] = ms.nx2 / bs.nx2; md.nb[2] = ms.nx3 / bs.nx3;
    nb_[0] = md.nb[0];
    nb_[1] = md.nb[1];
    md.nx[0] = bs.nx1; md.nx[1] = bs.nx2; md.nx[2] = bs.nx3;
    md.xmin[0] = ms.x1min; md.xmin[1] = ms.x2min; md.xmin[2] = ms.x3min;
    md.xmax[0] = ms.x1max; md.xmax[1] = ms.x2max; md.xmax[2] = ms.x3max;
    for (int f = 0; f < 6; ++f) {
      switch (pm->mesh_bcs[f]) {
        case BoundaryFlag::periodic: md.bc[f] = Z4C_BC_PERIODIC; break;
        case BoundaryFlag::gr_sommerfeld: md.bc[f] = Z4C_BC_SOMMERFELD; break;
        default: md.bc[f] = Z4C_BC_OUTFLOW; break;
      }
    }
    z4c_params_t p;
    z4c_params_default(&p);
    const auto& o = pz->opt;
    p.chi_psi_power = o.chi_psi_power;
    p.chi_div_floor = o.chi_div_floor;
    p.diss = o.diss;
    p.eps_floor = o.eps_floor;
    p.damp_kappa1 = o.damp_kappa1;
    p.damp_kappa2 = o.damp_kappa2;
    p.lapse_oplog = o.lapse_oplog;
    p.lapse_harmonicf = o.lapse_harmonicf;
    p.lapse_harmonic = o.lapse_harmonic;
    p.lapse_advect = o.lapse_advect;
    p.lapse_K = o.lapse_K;
    p.shift_Gamma = o.shift_Gamma;
    p.shift_alpha2Gamma = o.shift_alpha2Gamma;
    p.shift_H = o.shift_H;
    p.shift_advect = o.shift_advect;
    p.shift_eta = o.shift_eta;
    p.r_max_con = o.r_max_con;
    p.tf_force_regularization = o.tf_force_regularization ? 1 : 0;
    p.force_regularization = o.force_regularization ? 1 : 0;
    Check(z4c_create(&md, &p, butcher ? Z4C_INTEG_BT_RK4 : Z4C_INTEG_RK4, &ctx_), "z4c_create");
    nn_[0] = bs.nx1 + 1 + 2 * Z4C_NG;
    nn_[1] = bs.nx2 + 1 + 2 * Z4C_NG;
    nn_[2] = bs.nx3 + 1 + 2 * Z4C_NG;
  }
  ~Z4cB200() { z4c_destroy(ctx_); }
  Z4cB200(const Z4cB200&) = delete;
  Z4cB200& operator=(const Z4cB200&) = delete;

  // Z4c::Z4cRHS(u, mat, rhs) of block pmb (vacuum: mat is not read); the
  // interior of rhs is written, as the reference writes it.
  void Z4cRHS(MeshBlock* pmb, AthenaArray<Real>& u, AthenaArray<Real>& /*mat*/,
              AthenaArray<Real>& rhs) {
    const int b = Index(pmb);
    Check(z4c_upload(ctx_, Z4C_REG_U, b, u.data()), "z4c_upload");
    Check(z4c_rhs(ctx_, Z4C_REG_U, Z4C_REG_RHS, b), "z4c_rhs");
    buf_.resize((size_t)Z4C_NVAR * nn_[0] * nn_[1] * nn_[2]);
    Check(z4c_download(ctx_, Z4C_REG_RHS, b, buf_.data()), "z4c_download");
    CopyInterior(buf_.data(), rhs, Z4C_NVAR);
  }
  // Z4c::AlgConstr(u): every vertex, in place.
  void AlgConstr(MeshBlock* pmb, AthenaArray<Real>& u) {
    const int b = Index(pmb);
    Check(z4c_upload(ctx_, Z4C_REG_U, b, u.data()), "z4c_upload");
    Check(z4c_alg_constr(ctx_, Z4C_REG_U, b), "z4c_alg_constr");
    Check(z4c_download(ctx_, Z4C_REG_U, b, u.data()), "z4c_download");
  }
  // Z4c::Z4cToADM(u, adm): every vertex.
  void Z4cToADM(MeshBlock* pmb, AthenaArray<Real>& u, AthenaArray<Real>& adm) {
    const int b = Index(pmb);
    Check(z4c_upload(ctx_, Z4C_REG_U, b, u.data()), "z4c_upload");
    Check(z4c_z4c_to_adm(ctx_, Z4C_REG_U, Z4C_REG_ADM, b), "z4c_z4c_to_adm");
    Check(z4c_download(ctx_, Z4C_REG_ADM, b, adm.data()), "z4c_download");
  }
  // Device-resident use: the state of block pmb in or out once, then whole
  // GR_Z4c stages (every block at once) or captured steps in between.
  void Upload(MeshBlock* pmb, const AthenaArray<Real>& u) {
    Check(z4c_upload(ctx_, Z4C_REG_U, Index(pmb), u.data()), "z4c_upload");
  }
  void Download(MeshBlock* pmb, AthenaArray<Real>& u) {
    Check(z4c_download(ctx_, Z4C_REG_U, Index(pmb), u.data()), "z4c_download");
  }
  void Stage(int stage, Real dt) { Check(z4c_stage(ctx_, stage, dt), "z4c_stage"); }
  void Evolve(Real dt, int ncycles, bool with_constraints) {
    Check(z4c_evolve(ctx_, dt, ncycles, with_constraints ? 1 : 0), "z4c_evolve");
  }

 private:
  // the C ABI's block order l0 + nb0 (l1 + nb1 l2) from the block's logical
  // location on the root level (the reference numbers blocks by gid)
  int Index(const MeshBlock* pmb) const {
    return (int)(pmb->loc.lx1 + nb_[0] * (pmb->loc.lx2 + nb_[1] * pmb->loc.lx3));
  }
  void CopyInterior(const double* src, AthenaArray<Real>& dst, int nvar) const {
    const int ng = Z4C_NG;
    for (int n = 0; n < nvar; ++n)
      for (int k = ng; k < nn_[2] - ng; ++k)
        for (int j = ng; j < nn_[1] - ng; ++j)
          for (int i = ng; i < nn_[0] - ng; ++i)
            dst(n, k, j, i) = src[(((size_t)n * nn_[2] + k) * nn_[1] + j) * nn_[0] + i];
  }
  static void Check(int rc, const char* what) {
    if (rc != Z4C_OK) {
      std::stringstream msg;
      msg << "### FATAL ERROR in z4c_b200 (" << what << "): " << z4c_last_error() << std::endl;
      ATHENA_ERROR(msg);
    }
  }
  Mesh* pm_;  // kept for drivers that reach the mesh through the adapter
  z4c_ctx* ctx_ = nullptr;
  int nn_[3], nb_[2];
  std::vector<double> buf_;
};

// Host build of the pointwise tangent-linear and adjoint functions
// (gr-athena_b200/csrc/z4c_ad.cuh) for the CPU tests in test_ad_point.py:
// every reverse sweep against the forward-mode derivative of the same
// forward function (dot-product test), and the forward functions themselves.
#include "../../gr-athena_b200/csrc/z4c_ad.cuh"

using namespace z4c::ad;

extern "C" {

int adp_rhs_size(void) { return RhsLocal<double>::N; }
int adp_ham_size(void) { return HLocal<double>::N; }

// out[22] = the right-hand side (without Kreiss-Oliger) at the local inputs v
void adp_rhs(const double* v, const z4c_params_t* p, double* out) {
  RhsLocal<double> L;
  for (int i = 0; i < RhsLocal<double>::N; ++i) L.data()[i] = v[i];
  rhs_local(*p, L, out);
}

// res = {<ob, J vdot> by forward mode, <J^T ob, vdot> by the reverse sweep,
//        d<ob, F>/d shift_eta, d<ob, F>/d damp_kappa1}; vb_out = J^T ob
void adp_rhs_dot(const double* v, const double* vdot, const double* ob,
                 const z4c_params_t* p, double* res, double* vb_out) {
  const int N = RhsLocal<double>::N;
  RhsLocal<Dual> D;
  RhsLocal<double> L, B;
  for (int i = 0; i < N; ++i) {
    D.data()[i] = Dual(v[i], vdot[i]);
    L.data()[i] = v[i];
    B.data()[i] = 0.;
  }
  Dual out[NV];
  rhs_local(*p, D, out);
  double fwd = 0.;
  for (int n = 0; n < NV; ++n) fwd += ob[n] * out[n].d;
  double Rsum[6], Rsb[6] = {0, 0, 0, 0, 0, 0};
  ricci_local(*p, L, Rsum);
  ParamBar pb{0., 0.};
  main_local_adj(*p, L, Rsum, ob, B, Rsb, pb);
  ricci_local_adj(*p, L, Rsb, B);
  double rev = 0.;
  for (int i = 0; i < N; ++i) rev += B.data()[i] * vdot[i];
  res[0] = fwd;
  res[1] = rev;
  res[2] = pb.shift_eta;
  res[3] = pb.damp_kappa1;
  if (vb_out)
    for (int i = 0; i < N; ++i) vb_out[i] = B.data()[i];
}

// AlgConstr on 22 values in place
void adp_alg(double* u, const z4c_params_t* p) { alg_constr_local(*p, u); }
void adp_alg_dot(const double* u, const double* udot, const double* ub, const z4c_params_t* p,
                 double* res) {
  Dual D[NV];
  double B[NV];
  for (int n = 0; n < NV; ++n) {
    D[n] = Dual(u[n], udot[n]);
    B[n] = ub[n];
  }
  alg_constr_local(*p, D);
  double fwd = 0.;
  for (int n = 0; n < NV; ++n) fwd += ub[n] * D[n].d;
  alg_constr_adj(*p, u, B);
  double rev = 0.;
  for (int n = 0; n < NV; ++n) rev += B[n] * udot[n];
  res[0] = fwd;
  res[1] = rev;
}

double adp_ham(const double* v, const z4c_params_t* p) {
  HLocal<double> L;
  for (int i = 0; i < HLocal<double>::N; ++i) L.data()[i] = v[i];
  return ham_local(*p, L);
}
void adp_ham_dot(const double* v, const double* vdot, const z4c_params_t* p, double* res) {
  const int N = HLocal<double>::N;
  HLocal<Dual> D;
  HLocal<double> L, B;
  for (int i = 0; i < N; ++i) {
    D.data()[i] = Dual(v[i], vdot[i]);
    L.data()[i] = v[i];
    B.data()[i] = 0.;
  }
  res[0] = ham_local(*p, D).d;
  ham_local_adj(*p, L, 1.0, B);
  double rev = 0.;
  for (int i = 0; i < N; ++i) rev += B.data()[i] * vdot[i];
  res[1] = rev;
}

}  // extern "C"

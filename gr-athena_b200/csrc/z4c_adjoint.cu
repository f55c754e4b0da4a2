// Differentiated Z4c time stepping on the device: the tangent-linear model
// and the hand-written adjoint of one RK4 step (low-storage 2S integrator,
// task_list_gr_z4c.cpp:170-213 with the weights of
// task_list_integrators_low_storage.cpp:112-142), of the objective
// J = sum over blocks of vol * sum over cells of H^2 (the H-norm of the
// history output, outputs/history.cpp:168-200), and the revolve-style
// checkpointed gradient of J after n steps (z4c_adj_gradient).
//
// One forward stage maps (u, u1) to (u', u1'):
//   v1 = u1 + delta u,  w = gamma1 u + gamma2 v1 + beta dt (F(u) + KO(u))
//   u_pre = E(w)    ghost exchange (an average over the owners of each vertex,
//                   copies into the ghosts; periodic meshes)
//   u' = AC(u_pre)  AlgConstr at every vertex, u1' = v1
// (u1 = 0 at stage 1).  The reverse of a stage, given the adjoints of u' and
// u1', runs AC^T at u_pre, E^T, and the transposed stage algebra and
// right-hand side at u.  The right-hand side reverse is split as the forward
// is (z4c_ad.cuh): per interior vertex the reverse of the main algebra and of
// the Ricci part write the adjoints of the vertex's local inputs into channel
// arrays; then the transposed stencils gather those channels back onto the
// state (centred first and second derivatives, the mixed second derivatives
// through the stored first derivatives, Kreiss-Oliger and the upwind
// advection with the side fixed at the linearisation point).
//
// Per-stage recomputation: the adjoint of a step recomputes the step from
// the state at its start, keeping each stage's u_pre (4 registers); the
// stage inputs are rebuilt from them (u_s = AC(u_pre_{s-1})) as the reverse
// sweep reaches them.
//
// The adjoint kernels are compiled with floating-point contraction: they
// are not bound to the reference's rounding, only to the transpose of the
// forward map (checked against the tangent-linear model and against finite
// differences of the forward).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "z4c_ad.cuh"
#include "z4c_ctx.cuh"
#include "z4c_rhs.cuh"

namespace z4c {
int set_error(int code, const char* msg);

namespace {

using ad::Dual;
using ad::HLocal;
using ad::RhsLocal;

constexpr int kThreads = 128;
// channels of the right-hand side reverse per interior vertex
constexpr int kChSd = 0;      // 33: the stored first derivatives, slot*3 + direction
constexpr int kChDd = 33;     // 66: second derivatives, slot*6 + pair
constexpr int kChGam = 99;    // 9: d_b Gamma^c, b*3 + c
constexpr int kChKhat = 108;  // 3
constexpr int kChTheta = 111; // 3
constexpr int kNChan = 114;
// per interior vertex from the main reverse to the Ricci reverse: the Ricci
// sums' adjoints (6) and the Christoffel adjoints (27)
constexpr int kNRsb = 33;
// channels of the Hamiltonian-constraint reverse per interior vertex
constexpr int kHChi = 0, kHGt = 1, kHAt = 7, kHKhat = 13, kHTheta = 14;  // point values
constexpr int kHDchi = 15, kHDg = 18, kHDdchi = 36, kHDdg = 42;         // stencil inputs
constexpr int kNHChan = 78;

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

__device__ __forceinline__ void interior_of(const Grid& g, int64_t l, int& i, int& j, int& k) {
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1;
  i = NG + (int)(l % n0);
  j = NG + (int)((l / n0) % n1);
  k = NG + (int)(l / ((int64_t)n0 * n1));
}
__device__ __forceinline__ bool is_interior(const Grid& g, int i, int j, int k) {
  return i >= NG && i <= NG + g.nx[0] && j >= NG && j <= NG + g.nx[1] && k >= NG &&
         k <= NG + g.nx[2];
}
__device__ __forceinline__ int64_t interior_index(const Grid& g, int i, int j, int k) {
  return ((int64_t)(k - NG) * (g.nx[1] + 1) + (j - NG)) * (g.nx[0] + 1) + (i - NG);
}

// stencil weights, offset o = -R..R
__device__ __forceinline__ double w_d1(int o) {  // FDStencilCenteredDegreeOdd<1,3>
  switch (o) {
    case -3: return -1.; case -2: return 9.; case -1: return -45.;
    case 1: return 45.; case 2: return -9.; case 3: return 1.;
    default: return 0.;
  }
}
__device__ __forceinline__ double w_d2(int o) {  // FDStencilCenteredDegreeEven<2,3>
  switch (o) {
    case -3: case 3: return 2.; case -2: case 2: return -27.;
    case -1: case 1: return 270.; case 0: return -490.;
    default: return 0.;
  }
}
__device__ __forceinline__ double w_ko(int o) {  // FDStencilCenteredDegreeEven<8,4>
  switch (o) {
    case -4: case 4: return 1.; case -3: case 3: return -8.; case -2: case 2: return 28.;
    case -1: case 1: return -56.; case 0: return 70.;
    default: return 0.;
  }
}
// lop-sided advection, coefficient of f(p + o): left side (beta < 0) o = -4..2,
// right side (beta >= 0) o = -2..4 (FDStencilBiased{Left,Right}<1,4,2>)
__device__ __forceinline__ double w_lop(bool left, int o) {
  if (left) {
    switch (o) {
      case -4: return 1.; case -3: return -8.; case -2: return 30.; case -1: return -80.;
      case 0: return 35.; case 1: return 24.; case 2: return -2.;
      default: return 0.;
    }
  }
  switch (o) {
    case -2: return 2.; case -1: return -24.; case 0: return -35.; case 1: return 80.;
    case 2: return -30.; case 3: return 8.; case 4: return -1.;
    default: return 0.;
  }
}

// A field for the gathers: value array and, for the tangent-linear model, the
// tangent array at the same offsets.
template <class T>
struct Fld;
template <>
struct Fld<double> {
  const double* v;
  __device__ double at(int64_t o) const { return v[o]; }
};
template <>
struct Fld<Dual> {
  const double* v;
  const double* d;
  __device__ Dual at(int64_t o) const { return Dual(v[o], d[o]); }
};

template <class T>
__device__ __forceinline__ T st_d1(const Fld<T>& f, int64_t p, int64_t s, double c) {
  T out = T(0.);
#pragma unroll
  for (int o = -3; o <= 3; ++o)
    if (o != 0) out += w_d1(o) * f.at(p + o * s);
  return out * c;
}
template <class T>
__device__ __forceinline__ T st_d2(const Fld<T>& f, int64_t p, int64_t s, double c) {
  T out = T(0.);
#pragma unroll
  for (int o = -3; o <= 3; ++o) out += w_d2(o) * f.at(p + o * s);
  return out * c;
}
template <class T>
__device__ __forceinline__ T st_d2x(const Fld<T>& f, int64_t p, int64_t sa, int64_t sb, double ca,
                                   double cb) {
  T out = T(0.);
#pragma unroll
  for (int o = -3; o <= 3; ++o)
    if (o != 0) out += w_d1(o) * st_d1(f, p + o * sa, sb, cb);
  return out * ca;
}
// the side's stencil sum (before the shift and the spacing factor)
template <class T>
__device__ __forceinline__ T st_lop(const Fld<T>& f, int64_t p, int64_t s, bool left) {
  T out = T(0.);
#pragma unroll
  for (int o = -4; o <= 4; ++o) {
    const double w = w_lop(left, o);
    if (w != 0.) out += w * f.at(p + o * s);
  }
  return out;
}

// Which local inputs a gather fills: every one (the tangent-linear model),
// those the main algebra's reverse reads (not the advection sums, whose
// values it does not need), or those of the Ricci part.
enum { kGatherAll = 0, kGatherMain = 1, kGatherRicci = 2 };

// Local inputs of the right-hand side at interior vertex p of a block: U and
// SD point at the block's state and stored first derivatives (and Ud, SDd at
// their tangents for T = Dual).  Inputs a PART does not gather are zero.
template <class T, int PART = kGatherAll>
__device__ void gather_rhs(const Grid& g, const FdScale& F, const double* U, const double* SD,
                           const double* Ud, const double* SDd, int64_t p, RhsLocal<T>& v) {
  const int64_t nv = g.nvol;
  auto fld = [&](const double* base, const double* based, int64_t off) {
    Fld<T> f;
    f.v = base + off;
    if constexpr (sizeof(T) == sizeof(Dual)) f.d = based + off;
    return f;
  };
  #pragma unroll
  for (int n = 0; n < NVAR; ++n) v.u[n] = fld(U, Ud, (int64_t)n * nv).at(p);
  auto sdc = [&](int comp) { return fld(SD, SDd, (int64_t)comp * nv).at(p); };
  #pragma unroll
  for (int a = 0; a < 3; ++a) {
    v.dchi[a] = sdc(a);
    v.dalpha[a] = sdc(7 * 3 + a);
  }
  #pragma unroll
  for (int c = 0; c < 3; ++c)
    #pragma unroll
    for (int q = 0; q < 6; ++q) v.dg[c][q] = sdc((1 + q) * 3 + c);
  #pragma unroll
  for (int a = 0; a < 3; ++a)
    #pragma unroll
    for (int b = 0; b < 3; ++b) v.dbeta[b][a] = sdc((8 + a) * 3 + b);
  #pragma unroll
  for (int b = 0; b < 3; ++b) {
    #pragma unroll
    for (int c = 0; c < 3; ++c)
      v.dGam[b][c] = st_d1(fld(U, Ud, (int64_t)(Z4C_GAMX + c) * nv), p, g.s[b], F.cidx1[b]);
    if (PART != kGatherRicci) {
      v.dKhat[b] = st_d1(fld(U, Ud, (int64_t)Z4C_KHAT * nv), p, g.s[b], F.cidx1[b]);
      v.dTheta[b] = st_d1(fld(U, Ud, (int64_t)Z4C_THETA * nv), p, g.s[b], F.cidx1[b]);
    } else {
      v.dKhat[b] = v.dTheta[b] = T(0.);
    }
  }
  // second derivatives: Dxx on the diagonal, Dx_a of the stored Dx_b (a < b)
  #pragma unroll
  for (int slot = 0; slot < 11; ++slot) {
    const int var = sd_field_var(slot);
    if (PART == kGatherRicci && slot >= 7) {  // alpha, beta: not in the Ricci part
      for (int q = 0; q < 6; ++q) {
        if (slot == 7) v.ddalpha[q] = T(0.);
        else v.ddbeta[slot - 8][q] = T(0.);
      }
      continue;
    }
    #pragma unroll
    for (int a = 0; a < 3; ++a)
      #pragma unroll
      for (int b = a; b < 3; ++b) {
        T d;
        if (a == b) d = st_d2(fld(U, Ud, (int64_t)var * nv), p, g.s[a], F.cidx2[a]);
        else d = st_d1(fld(SD, SDd, (int64_t)(slot * 3 + b) * nv), p, g.s[a], F.cidx1[a]);
        if (slot == 0) v.ddchi[ad::sid(a, b)] = d;
        else if (slot <= 6) v.ddg[slot - 1][ad::sid(a, b)] = d;
        else if (slot == 7) v.ddalpha[ad::sid(a, b)] = d;
        else v.ddbeta[slot - 8][ad::sid(a, b)] = d;
      }
  }
  if (PART != kGatherAll) {
    for (int n = 0; n < NVAR; ++n) v.lv[n] = T(0.);
    return;
  }
  // advection sums beta^a L_a f, the side chosen by the sign of beta^a
  T beta[3];
  #pragma unroll
  for (int a = 0; a < 3; ++a) beta[a] = v.u[Z4C_BETAX + a];
  #pragma unroll
  for (int n = 0; n < NVAR; ++n) {
    T acc = T(0.);
    #pragma unroll
    for (int a = 0; a < 3; ++a) {
      const bool left = ad::val(beta[a]) < 0;
      acc += (beta[a] * st_lop(fld(U, Ud, (int64_t)n * nv), p, g.s[a], left)) * F.lidx[a];
    }
    v.lv[n] = acc;
  }
}

// ---- reverse of the right-hand side ------------------------------------------

struct StageW {
  double delta, gamma1, gamma2, beta_dt;
  int first;  // stage 1: u1 enters as zero
};

// Per interior vertex: the reverse of the main algebra (z4c_ad.cuh
// main_local_adj) for the right-hand side adjoint beta dt * wbar, plus the
// shift adjoint of the advection sums and the stage algebra.  Writes the
// channels, the Ricci-sum adjoints, the direct adjoint of u at the vertex and
// the adjoint of u1; parameter adjoints per CTA into part.
template <int NX>
__global__ void __launch_bounds__(kThreads)
k_adj_main(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ sd,
           const double* __restrict__ rsum, const double* __restrict__ wbar,
           double* __restrict__ u1bar, double* __restrict__ direct, double* __restrict__ chan,
           double* __restrict__ rsb, double* __restrict__ part, StageW W) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double pe = 0., pk = 0.;
  if (t < npts * g.nblocks) {
    const int b = (int)(t / npts);
    const int64_t l = t % npts;
    int i, j, k;
    interior_of(g, l, i, j, k);
    const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
    const int64_t nv = g.nvol;
    const double* U = u + (int64_t)b * NVAR * nv;
    const double* SD = sd + (int64_t)b * kSdComponents * nv;
    const FdScale& F = P.fd[b];
    RhsLocal<double> v;
    gather_rhs<double, kGatherMain>(g, F, U, SD, nullptr, nullptr, p, v);
    double Rs[6];
    const double* RS = rsum + (int64_t)b * 6 * npts + l;
    #pragma unroll
    for (int q = 0; q < 6; ++q) Rs[q] = RS[(int64_t)q * npts];
    double ob[NVAR], wb[NVAR];
    const double* WB = wbar + (int64_t)b * NVAR * nv + p;
    #pragma unroll
    for (int n = 0; n < NVAR; ++n) {
      wb[n] = WB[(int64_t)n * nv];
      ob[n] = W.beta_dt * wb[n];
    }
    RhsLocal<double> vb;
    #pragma unroll
    for (int q = 0; q < RhsLocal<double>::N; ++q) vb.data()[q] = 0.;
    double Rsb[6] = {0, 0, 0, 0, 0, 0};
    ad::ParamBar pb{0., 0.};
    double cb[27];
    ad::main_local_adj(P.p, v, Rs, ob, vb, Rsb, pb, cb);
    pe = pb.shift_eta;
    pk = pb.damp_kappa1;
    // (the advection sums' dependence on the shift at the vertex: k_adj_advbeta)
    // channels
    double* C = chan + (int64_t)b * kNChan * npts + l;
    #pragma unroll
    for (int a = 0; a < 3; ++a) {
      C[(int64_t)(kChSd + a) * npts] = vb.dchi[a];
      C[(int64_t)(kChSd + 7 * 3 + a) * npts] = vb.dalpha[a];
    }
    #pragma unroll
    for (int c = 0; c < 3; ++c)
      #pragma unroll
      for (int q = 0; q < 6; ++q) C[(int64_t)(kChSd + (1 + q) * 3 + c) * npts] = vb.dg[c][q];
    #pragma unroll
    for (int a = 0; a < 3; ++a)
      #pragma unroll
      for (int bb = 0; bb < 3; ++bb) C[(int64_t)(kChSd + (8 + a) * 3 + bb) * npts] = vb.dbeta[bb][a];
    #pragma unroll
    for (int q = 0; q < 6; ++q) {
      C[(int64_t)(kChDd + 0 * 6 + q) * npts] = vb.ddchi[q];
      C[(int64_t)(kChDd + 7 * 6 + q) * npts] = vb.ddalpha[q];
      #pragma unroll
      for (int f = 0; f < 6; ++f) C[(int64_t)(kChDd + (1 + f) * 6 + q) * npts] = vb.ddg[f][q];
      #pragma unroll
      for (int c = 0; c < 3; ++c) C[(int64_t)(kChDd + (8 + c) * 6 + q) * npts] = vb.ddbeta[c][q];
    }
    #pragma unroll
    for (int bb = 0; bb < 3; ++bb) {
      #pragma unroll
      for (int c = 0; c < 3; ++c) C[(int64_t)(kChGam + bb * 3 + c) * npts] = vb.dGam[bb][c];
      C[(int64_t)(kChKhat + bb) * npts] = vb.dKhat[bb];
      C[(int64_t)(kChTheta + bb) * npts] = vb.dTheta[bb];
    }
    double* R = rsb + (int64_t)b * kNRsb * npts + l;
    for (int q = 0; q < 6; ++q) R[(int64_t)q * npts] = Rsb[q];
    for (int q = 0; q < 27; ++q) R[(int64_t)(6 + q) * npts] = cb[q];
    // stage algebra: w = gamma1 u + gamma2 v1 + beta dt r, v1 = u1 + delta u
    double* D = direct + (int64_t)b * NVAR * nv + p;
    double* U1B = u1bar + (int64_t)b * NVAR * nv + p;
    #pragma unroll
    for (int n = 0; n < NVAR; ++n) {
      // the adjoint of v1 = u1 + delta u: that of the stage's u1 output plus
      // gamma2 wbar; the stage's u1 input is the constant 0 at stage 1
      const double v1b = U1B[(int64_t)n * nv] + W.gamma2 * wb[n];
      U1B[(int64_t)n * nv] = W.first ? 0. : v1b;
      D[(int64_t)n * nv] = vb.u[n] + W.gamma1 * wb[n] + W.delta * v1b;
    }
  }
  // parameter adjoints: a fixed-order reduction per CTA
  __shared__ double se[kThreads], sk[kThreads];
  se[threadIdx.x] = pe;
  sk[threadIdx.x] = pk;
  __syncthreads();
  #pragma unroll
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      se[threadIdx.x] += se[threadIdx.x + w];
      sk[threadIdx.x] += sk[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = se[0];
    part[2 * blockIdx.x + 1] = sk[0];
  }
}

// Per interior vertex: the adjoint of the shift through the advection sums,
// sum_n lvbar_n dlv_n/dbeta^a = lidx_a sum_n adv_n beta dt wbar_n L_a f_n,
// added to the direct adjoint (the upwind side of the linearisation point).
template <int NX>
__global__ void __launch_bounds__(kThreads)
k_adj_advbeta(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ wbar,
              double* __restrict__ direct, double beta_dt) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * g.nblocks) return;
  const int b = (int)(t / npts);
  int i, j, k;
  interior_of(g, t % npts, i, j, k);
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  const int64_t nv = g.nvol;
  const double* U = u + (int64_t)b * NVAR * nv;
  const double* WB = wbar + (int64_t)b * NVAR * nv + p;
  const FdScale& F = P.fd[b];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const bool left = U[(int64_t)(Z4C_BETAX + a) * nv + p] < 0;
    double acc = 0.;
#pragma unroll 2
    for (int n = 0; n < NVAR; ++n) {
      const double lb = ad::adv_coef(P.p, n) * beta_dt * WB[(int64_t)n * nv];
      if (lb == 0.) continue;
      Fld<double> f{U + (int64_t)n * nv};
      acc += lb * st_lop(f, p, g.s[a], left);
    }
    direct[(int64_t)b * NVAR * nv + (int64_t)(Z4C_BETAX + a) * nv + p] += acc * F.lidx[a];
  }
}

// Per interior vertex: the reverse of the Ricci part (ricci_local_adj) given
// the Ricci-sum adjoints; adds to the channels and the direct adjoint.
template <int NX>
__global__ void __launch_bounds__(kThreads)
k_adj_ricci(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ sd,
            const double* __restrict__ rsb, double* __restrict__ direct,
            double* __restrict__ chan) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * g.nblocks) return;
  const int b = (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_of(g, l, i, j, k);
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  const int64_t nv = g.nvol;
  const double* U = u + (int64_t)b * NVAR * nv;
  const double* SD = sd + (int64_t)b * kSdComponents * nv;
  RhsLocal<double> v;
  gather_rhs<double, kGatherRicci>(g, P.fd[b], U, SD, nullptr, nullptr, p, v);
  double Rsb[6], cb[27];
  const double* R = rsb + (int64_t)b * kNRsb * npts + l;
  for (int q = 0; q < 6; ++q) Rsb[q] = R[(int64_t)q * npts];
  for (int q = 0; q < 27; ++q) cb[q] = R[(int64_t)(6 + q) * npts];
  RhsLocal<double> vb;
  #pragma unroll
  for (int q = 0; q < RhsLocal<double>::N; ++q) vb.data()[q] = 0.;
  ad::ricci_local_adj(P.p, v, Rsb, vb, cb);
  double* C = chan + (int64_t)b * kNChan * npts + l;
  #pragma unroll
  for (int a = 0; a < 3; ++a) C[(int64_t)(kChSd + a) * npts] += vb.dchi[a];
  #pragma unroll
  for (int c = 0; c < 3; ++c)
    #pragma unroll
    for (int q = 0; q < 6; ++q) C[(int64_t)(kChSd + (1 + q) * 3 + c) * npts] += vb.dg[c][q];
  #pragma unroll
  for (int q = 0; q < 6; ++q) {
    C[(int64_t)(kChDd + 0 * 6 + q) * npts] += vb.ddchi[q];
    #pragma unroll
    for (int f = 0; f < 6; ++f) C[(int64_t)(kChDd + (1 + f) * 6 + q) * npts] += vb.ddg[f][q];
  }
  #pragma unroll
  for (int bb = 0; bb < 3; ++bb)
    #pragma unroll
    for (int c = 0; c < 3; ++c) C[(int64_t)(kChGam + bb * 3 + c) * npts] += vb.dGam[bb][c];
  double* D = direct + (int64_t)b * NVAR * nv + p;
  #pragma unroll
  for (int n = 0; n < NVAR; ++n)
    if (vb.u[n] != 0.) D[(int64_t)n * nv] += vb.u[n];
}

// Region of the stored first derivative along direction dir (as k_prep
// fills it): the interior, extended by 3 along x for dir >= 1 and along y
// for dir == 2.
__device__ __forceinline__ bool in_sd_region(const Grid& g, int dir, int i, int j, int k) {
  const int ex = (dir >= 1) ? 3 : 0, ey = (dir == 2) ? 3 : 0;
  return i >= NG - ex && i <= NG + g.nx[0] + ex && j >= NG - ey && j <= NG + g.nx[1] + ey &&
         k >= NG && k <= NG + g.nx[2];
}

// Adjoint of the stored first derivatives: the vertex's own channel plus the
// transposed outer derivative of every mixed second derivative that reads it.
// One thread per (block, component, vertex of the component's region).
template <int NX>
__global__ void __launch_bounds__(kThreads)
k_adj_sdbar(Grid gin, DevParams P, const double* __restrict__ chan, double* __restrict__ sdbar) {
  const Grid g = fixed_geometry<NX>(gin);
  const int comp = blockIdx.y, b = blockIdx.z;
  const int slot = comp / 3, dir = comp % 3;
  const int ex = (dir >= 1) ? 3 : 0, ey = (dir == 2) ? 3 : 0;
  const int e0 = g.nx[0] + 1 + 2 * ex, e1 = g.nx[1] + 1 + 2 * ey, e2 = g.nx[2] + 1;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)e0 * e1 * e2) return;
  const int i = NG - ex + (int)(t % e0), j = NG - ey + (int)((t / e0) % e1),
            k = NG + (int)(t / ((int64_t)e0 * e1));
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const double* C = chan + (int64_t)b * kNChan * npts;
  const FdScale& F = P.fd[b];
  double acc = 0.;
  if (is_interior(g, i, j, k)) acc = C[(int64_t)(kChSd + comp) * npts + interior_index(g, i, j, k)];
  // D_a(stored D_dir f) for a < dir: p = r - o e_a
  for (int a = 0; a < dir; ++a) {
    const double* dd = C + (int64_t)(kChDd + slot * 6 + ad::sid(a, dir)) * npts;
    double s = 0.;
#pragma unroll
    for (int o = -3; o <= 3; ++o) {
      if (o == 0) continue;
      const int pi = i - (a == 0 ? o : 0), pj = j - (a == 1 ? o : 0);
      if (is_interior(g, pi, pj, k)) s += w_d1(o) * dd[interior_index(g, pi, pj, k)];
    }
    acc += s * F.cidx1[a];
  }
  sdbar[((int64_t)b * kSdComponents + comp) * g.nvol + ((int64_t)k * g.nn[1] + j) * g.nn[0] + i] =
      acc;
}

// Adjoint of the stage input u at every vertex of every block: the direct
// adjoint (interior) plus the transposed stencils of every channel, the
// Kreiss-Oliger terms and the upwind advection.  One thread per (block,
// vertex) for all 22 variables: along each axis the interior points p that
// reach the vertex form one range of offsets, clamped once, and the weights
// that depend on p only (upwind side, shift, Kreiss-Oliger) are shared by
// the variables.
template <int NX>
__global__ void __launch_bounds__(kThreads)
k_adj_gather(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ wbar,
             const double* __restrict__ direct, const double* __restrict__ chan,
             const double* __restrict__ sdbar, double* __restrict__ ubar, double beta_dt) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t nv = g.nvol;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * g.nblocks) return;
  const int64_t q = t % nv;
  const int b = (int)(t / nv);
  const int ijk[3] = {(int)(q % g.nn[0]), (int)((q / g.nn[0]) % g.nn[1]),
                      (int)(q / ((int64_t)g.nn[0] * g.nn[1]))};
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1;
  const int64_t npts = (int64_t)n0 * n1 * (g.nx[2] + 1);
  const int64_t ls[3] = {1, n0, (int64_t)n0 * n1};
  bool inA[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) inA[a] = ijk[a] >= NG && ijk[a] <= NG + g.nx[a];
  const int64_t boff = (int64_t)b * NVAR * nv;
  const double* C = chan + (int64_t)b * kNChan * npts;
  const FdScale& F = P.fd[b];
  double acc[NVAR];
  const bool interior = inA[0] && inA[1] && inA[2];
#pragma unroll
  for (int n = 0; n < NVAR; ++n) acc[n] = interior ? direct[boff + (int64_t)n * nv + q] : 0.;
  double adv[NVAR];
#pragma unroll
  for (int n = 0; n < NVAR; ++n) adv[n] = ad::adv_coef(P.p, n);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!(inA[(a + 1) % 3] && inA[(a + 2) % 3])) continue;
    // interior points p = q - o e_a: NG <= ijk[a] - o <= NG + nx[a]
    const int olo = max(-4, ijk[a] - NG - g.nx[a]), ohi = min(4, ijk[a] - NG);
    int64_t l0 = 0;  // interior index of q with coordinate a at NG
#pragma unroll
    for (int c = 0; c < 3; ++c) l0 += (c == a ? 0 : (int64_t)(ijk[c] - NG)) * ls[c];
    const double ck = F.cidxd[a] * P.p.diss, cl = F.lidx[a], c1 = F.cidx1[a], c2 = F.cidx2[a];
#pragma unroll
    for (int o = -4; o <= 4; ++o) {
      if (o < olo || o > ohi) continue;
      const int64_t pq = q - (int64_t)o * g.s[a];
      const int64_t lp = l0 + (int64_t)(ijk[a] - o - NG) * ls[a];
      const double be = u[boff + (int64_t)(Z4C_BETAX + a) * nv + pq];
      const double wko = w_ko(o) * ck;
      const double wad = w_lop(be < 0, o) * be * cl;
#pragma unroll
      for (int n = 0; n < NVAR; ++n) {
        const double rb = beta_dt * wbar[boff + (int64_t)n * nv + pq];
        acc[n] += (wko + wad * adv[n]) * rb;
      }
      if (o >= -3 && o <= 3) {
        const double w2 = w_d2(o) * c2;
#pragma unroll
        for (int slot = 0; slot < 11; ++slot)
          acc[sd_field_var(slot)] += w2 * C[(int64_t)(kChDd + slot * 6 + ad::sid(a, a)) * npts + lp];
        if (o != 0) {
          const double w1 = w_d1(o) * c1;
#pragma unroll
          for (int c = 0; c < 3; ++c)
            acc[Z4C_GAMX + c] += w1 * C[(int64_t)(kChGam + a * 3 + c) * npts + lp];
          acc[Z4C_KHAT] += w1 * C[(int64_t)(kChKhat + a) * npts + lp];
          acc[Z4C_THETA] += w1 * C[(int64_t)(kChTheta + a) * npts + lp];
        }
      }
    }
  }
  // D_dir^T of the stored first derivatives' adjoints over their regions
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const int ex = (dir >= 1) ? 3 : 0, ey = (dir == 2) ? 3 : 0;
    const int lo[3] = {NG - ex, NG - ey, NG};
    const int hi[3] = {NG + g.nx[0] + ex, NG + g.nx[1] + ey, NG + g.nx[2]};
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (c != dir) ok = ok && ijk[c] >= lo[c] && ijk[c] <= hi[c];
    if (!ok) continue;
    const int olo = max(-3, ijk[dir] - hi[dir]), ohi = min(3, ijk[dir] - lo[dir]);
    const double c1 = F.cidx1[dir];
#pragma unroll
    for (int o = -3; o <= 3; ++o) {
      if (o == 0 || o < olo || o > ohi) continue;
      const int64_t pq = q - (int64_t)o * g.s[dir];
      const double w = w_d1(o) * c1;
#pragma unroll
      for (int slot = 0; slot < 11; ++slot)
        acc[sd_field_var(slot)] +=
            w * sdbar[((int64_t)b * kSdComponents + slot * 3 + dir) * nv + pq];
    }
  }
#pragma unroll
  for (int n = 0; n < NVAR; ++n) ubar[boff + (int64_t)n * nv + q] = acc[n];
}

// AlgConstr^T at every vertex: ubar (adjoint after) -> adjoint before, at the
// pre-constraint state upre.
template <int NX>
__global__ void __launch_bounds__(kThreads)
k_adj_alg(Grid gin, DevParams P, const double* __restrict__ upre, double* __restrict__ ubar) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t nv = g.nvol;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * g.nblocks) return;
  const int b = (int)(t / nv);
  const int64_t q = t % nv;
  double uu[NVAR], ub[NVAR];
  const double* UP = upre + (int64_t)b * NVAR * nv + q;
  double* UB = ubar + (int64_t)b * NVAR * nv + q;
  #pragma unroll
  for (int n = 0; n < NVAR; ++n) {
    uu[n] = UP[(int64_t)n * nv];
    ub[n] = UB[(int64_t)n * nv];
  }
  ad::alg_constr_adj(P.p, uu, ub);
  #pragma unroll
  for (int n = 0; n < NVAR; ++n) UB[(int64_t)n * nv] = ub[n];
}

// Transpose of the extrapolation boundary condition along one axis
// (k_bc_axis: ExtrapolateOutflowBC, comm/physical_bcs.cpp:187-260, with the
// reference's cell-centred index ends).  One thread per line, as the forward:
// the line's ghosts y_1..y_4 (the outer side's y_1 is the boundary vertex)
// were y_g = 5 z1 - 10 z2 + 10 z3 - 5 z4 + z5 over the five values inward of
// it, earlier ghosts included.  Their adjoints flow into those values in
// reverse order; the overwritten values' own adjoints become zero.
template <int AX, int NVB = NVAR>
__global__ void __launch_bounds__(kThreads)
k_adj_bc_axis(Grid g, double* __restrict__ ub) {
  constexpr int ax = AX;
  constexpr int o1 = (ax == 0) ? 1 : 0;
  constexpr int o2 = (ax == 2) ? 1 : 2;
  const int64_t nt = (int64_t)g.nn[o1] * g.nn[o2];
  const int nfb = g.nb[o1] * g.nb[o2];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt * 2 * NVB * nfb) return;
  const int64_t tr = t % nt;
  int64_t r = t / nt;
  const int side = (int)(r % 2);
  r /= 2;
  const int n = (int)(r % NVB);
  const int fb = (int)(r / NVB);
  int loc[3];
  loc[ax] = side ? g.nb[ax] - 1 : 0;
  loc[o1] = fb % g.nb[o1];
  loc[o2] = fb / g.nb[o1];
  if (g.bc[2 * ax + side] == Z4C_BC_PERIODIC) return;
  const int b = loc[0] + g.nb[0] * (loc[1] + g.nb[1] * loc[2]);
  bool need[6];
  for (int a = 0; a < 3; ++a) {
    need[2 * a] = (g.bc[2 * a] != Z4C_BC_PERIODIC) && loc[a] == 0;
    need[2 * a + 1] = (g.bc[2 * a + 1] != Z4C_BC_PERIODIC) && loc[a] == g.nb[a] - 1;
  }
  int is[3], ie[3];
  for (int a = 0; a < 3; ++a) {
    is[a] = NG;
    ie[a] = NG + g.nx[a] - 1;
  }
  int lo[3], hi[3];
  lo[0] = is[0] - NG; hi[0] = ie[0] + NG;
  lo[1] = need[2] ? is[1] : is[1] - NG;
  hi[1] = need[3] ? ie[1] : ie[1] + NG;
  lo[2] = need[4] ? is[2] : is[2] - NG;
  hi[2] = need[5] ? ie[2] : ie[2] + NG;
  if (ax == 2) { lo[1] = is[1] - NG; hi[1] = ie[1] + NG; }
  const int t1 = (int)(tr % g.nn[o1]), t2 = (int)(tr / g.nn[o1]);
  if (t1 < lo[o1] || t1 > hi[o1] || t2 < lo[o2] || t2 > hi[o2]) return;
  double* u = ub + ((int64_t)b * NVB + n) * g.nvol + (int64_t)t1 * g.s[o1] + (int64_t)t2 * g.s[o2];
  const int64_t st = g.s[ax];
  const int dir = side ? -1 : 1;
  const int ia0 = side ? ie[ax] + 1 : is[ax] - 1;
  // sequence s[0..8] = x_4, x_3, x_2, x_1, x_0, y_1, y_2, y_3, y_4 (x_0 the
  // value next to the ghosts); its adjoints
  double sb[9];
  for (int q = 0; q < 5; ++q) sb[4 - q] = u[(int64_t)(ia0 + dir * (q + 1)) * st];
  for (int gh = 1; gh <= NG; ++gh) sb[4 + gh] = u[(int64_t)(side ? ie[ax] + gh : is[ax] - gh) * st];
  constexpr double c[5] = {5., -10., 10., -5., 1.};
  for (int gh = NG; gh >= 1; --gh) {
    const double y = sb[4 + gh];
    for (int k = 0; k < 5; ++k) sb[4 + gh - 1 - k] += c[k] * y;
  }
  for (int q = 0; q < 5; ++q) u[(int64_t)(ia0 + dir * (q + 1)) * st] = sb[4 - q];
  for (int gh = 1; gh <= NG; ++gh) u[(int64_t)(side ? ie[ax] + gh : is[ax] - gh) * st] = 0.;
}

// Block grid neighbour in direction d (periodic wrap; -1 beyond a
// non-periodic face).
__device__ __forceinline__ int grid_neighbour(const Grid& g, int b, const int d[3]) {
  int l[3] = {b % g.nb[0], (b / g.nb[0]) % g.nb[1], b / (g.nb[0] * g.nb[1])};
  for (int a = 0; a < 3; ++a) {
    l[a] += d[a];
    if (l[a] < 0 || l[a] >= g.nb[a]) {
      if (g.bc[2 * a] != Z4C_BC_PERIODIC) return -1;
      l[a] = (l[a] + g.nb[a]) % g.nb[a];
    }
  }
  return l[0] + g.nb[0] * (l[1] + g.nb[1] * l[2]);
}

// E^T of the same-level exchange: the adjoint of every owner copy of a
// vertex is 1/m times the sum of the adjoints of all entries (own, other
// owners', ghosts anywhere) that hold that vertex after the exchange.  Along
// each axis an interior index i has the images i, i + nx and i - nx where
// they lie in [0, nn) (a neighbour's interior or ghost entry); one thread per (block, interior
// vertex) forms the images once and sums all 22 variables.
template <int NX, int NVB = NVAR>
__global__ void __launch_bounds__(kThreads)
k_adj_exchange(Grid gin, const double* __restrict__ ubar, double* __restrict__ wbar) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * g.nblocks) return;
  const int64_t l = t % npts;
  const int b = (int)(t / npts);
  int ijk[3];
  interior_of(g, l, ijk[0], ijk[1], ijk[2]);
  // per axis: the block steps d whose image index i - d nx lies in [0, nn)
  int dlist[3][3], nd[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    nd[a] = 1;
    dlist[a][0] = dlist[a][1] = dlist[a][2] = 0;
    if (ijk[a] + g.nx[a] < g.nn[a]) dlist[a][nd[a]++] = -1;
    if (ijk[a] - g.nx[a] >= 0) dlist[a][nd[a]++] = 1;
  }
  const int64_t nv = g.nvol;
  int64_t off[27];
  int nimg = 0, m = 0;
  for (int z = 0; z < nd[2]; ++z)
    for (int y = 0; y < nd[1]; ++y)
      for (int x = 0; x < nd[0]; ++x) {
        const int d[3] = {dlist[0][x], dlist[1][y], dlist[2][z]};
        const int nb = grid_neighbour(g, b, d);
        if (nb < 0) continue;
        const int li = ijk[0] - d[0] * g.nx[0], lj = ijk[1] - d[1] * g.nx[1],
                  lk = ijk[2] - d[2] * g.nx[2];
        off[nimg++] = (int64_t)nb * NVB * nv + ((int64_t)lk * g.nn[1] + lj) * g.nn[0] + li;
        if (is_interior(g, li, lj, lk)) ++m;
      }
  const double inv = 1.0 / (double)m;
  const int64_t p = ((int64_t)ijk[2] * g.nn[1] + ijk[1]) * g.nn[0] + ijk[0];
  double* W = wbar + (int64_t)b * NVB * nv + p;
  for (int n = 0; n < NVB; ++n) {
    double s = 0.;
    for (int q = 0; q < nimg; ++q) s += ubar[off[q] + (int64_t)n * nv];
    W[(int64_t)n * nv] = s * inv;
  }
}

// ---- the Weyl-scalar objective ---------------------------------------------
// J_W = sum over the sphere's owned vertices p of w_p (Re psi4(p)^2 +
// Im psi4(p)^2), w_p the vertex's quadrature weight: psi4 of Z4cWeyl after
// Z4cToADM, the Weyl register's ghost fill and the sphere interpolation.  Its
// adjoint runs the chain backwards: the interpolation and the ghost fill
// transposed give the adjoint of psi4 at the interior vertices; at each one
// the adjoints of weyl_local's 100 local inputs come from 100 forward-mode
// evaluations (one input seeded each); the inputs that are stored or second
// derivatives of chi and g~ go into the right-hand side's channels (and
// through k_adj_sdbar and k_adj_gather's transposed stencils into u), the
// ADM ones (K, gamma and d K) through Z4cToADM transposed.
constexpr int kNWAdm = 30;  // ADM channels: K_q 6, gamma_q 6, d_c K_q 18

__device__ void gather_weyl(const Grid& g, const FdScale& F, const double* __restrict__ U,
                            const double* __restrict__ ADM, const double* __restrict__ SD,
                            int64_t p, ad::WeylLocal<double>& v) {
  const int64_t nv = g.nvol;
  auto UV = [&](int n) { return U + (int64_t)n * nv + p; };
  auto AV = [&](int n) { return ADM + (int64_t)n * nv + p; };
  auto SDC = [&](int slot, int dir) { return SD + ((int64_t)slot * 3 + dir) * nv + p; };
  v.chi = __ldg(UV(Z4C_CHI));
  for (int q = 0; q < 6; ++q) {
    v.gt[q] = __ldg(UV(Z4C_GXX + q));
    v.Kd[q] = __ldg(AV(Z4C_ADM_KXX + q));
    v.gph[q] = __ldg(AV(Z4C_ADM_GXX + q));
  }
  for (int a = 0; a < 3; ++a) {
    v.dchi[a] = __ldg(SDC(kSdChi, a));
    for (int q = 0; q < 6; ++q) v.dg3[a][q] = __ldg(SDC(kSdG + q, a));
  }
  for (int ab = 0; ab < 6; ++ab) {
    const int a = pair_a(ab), b = pair_b(ab);
    if (a == b) {
      v.ddchi[ab] = fd_dxx(UV(Z4C_CHI), g.s[a], F.cidx2[a]);
      for (int cd = 0; cd < 6; ++cd) v.ddg[ab][cd] = fd_dxx(UV(Z4C_GXX + cd), g.s[a], F.cidx2[a]);
    } else {
      v.ddchi[ab] = fd_dx(SDC(kSdChi, b), g.s[a], F.cidx1[a]);
      for (int cd = 0; cd < 6; ++cd)
        v.ddg[ab][cd] = fd_dx(SDC(kSdG + cd, b), g.s[a], F.cidx1[a]);
    }
  }
  for (int c = 0; c < 3; ++c)
    for (int q = 0; q < 6; ++q) v.dK[c][q] = fd_dx(AV(Z4C_ADM_KXX + q), g.s[c], F.cidx1[c]);
}

// The local inputs' adjoints at every interior vertex whose psi4 adjoint
// (wb2, [block][2][vertex]) is non-zero; channels and direct are cleared
// beforehand.
template <int NX>
__global__ void __launch_bounds__(kThreads)
k_weyl_adj(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ adm,
           const double* __restrict__ sd, const double* __restrict__ xf,
           const double* __restrict__ wb2, double* __restrict__ chan,
           double* __restrict__ direct, double* __restrict__ wadm) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * g.nblocks) return;
  const int b = (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_of(g, l, i, j, k);
  const int64_t nv = g.nvol;
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  const double pr = wb2[(int64_t)b * 2 * nv + p], pi = wb2[((int64_t)b * 2 + 1) * nv + p];
  if (pr == 0.0 && pi == 0.0) return;
  using WL = ad::WeylLocal<double>;
  WL v;
  gather_weyl(g, P.fd[b], u + (int64_t)b * NVAR * nv, adm + (int64_t)b * Z4C_NADM * nv,
              sd + (int64_t)b * kSdComponents * nv, p, v);
  const double* x = xf + (int64_t)b * (g.nn[0] + g.nn[1] + g.nn[2]);
  const double x1 = x[i], x2 = x[g.nn[0] + j], x3 = x[g.nn[0] + g.nn[1] + k];
  double* C = chan + (int64_t)b * kNChan * npts + l;
  double* D = direct + (int64_t)b * NVAR * nv + p;
  double* W = wadm + (int64_t)b * kNWAdm * npts + l;
  const double* src = v.data();
  for (int kk = 0; kk < WL::N; ++kk) {
    ad::WeylLocal<ad::Dual> vd;
    ad::Dual* dst = vd.data();
    for (int m = 0; m < WL::N; ++m) dst[m] = ad::Dual(src[m], m == kk ? 1.0 : 0.0);
    ad::Dual rp, ip;
    ad::weyl_local(P.p, vd, x1, x2, x3, rp, ip);
    const double bar = pr * rp.d + pi * ip.d;
    // the input's place: chi 0, g~ 1-6, K 7-12, gamma 13-18, d chi 19-21,
    // d g~ 22-39 [c][q], dd chi 40-45, dd g~ 46-81 [ab][cd], d K 82-99 [c][q]
    if (kk == 0) D[(int64_t)Z4C_CHI * nv] = bar;
    else if (kk < 7) D[(int64_t)(Z4C_GXX + kk - 1) * nv] = bar;
    else if (kk < 13) W[(int64_t)(kk - 7) * npts] = bar;
    else if (kk < 19) W[(int64_t)(6 + kk - 13) * npts] = bar;
    else if (kk < 22) C[(int64_t)(kChSd + kSdChi * 3 + (kk - 19)) * npts] = bar;
    else if (kk < 40) {
      const int c = (kk - 22) / 6, q = (kk - 22) % 6;
      C[(int64_t)(kChSd + (kSdG + q) * 3 + c) * npts] = bar;
    } else if (kk < 46) {
      C[(int64_t)(kChDd + kSdChi * 6 + (kk - 40)) * npts] = bar;
    } else if (kk < 82) {
      const int ab = (kk - 46) / 6, cd = (kk - 46) % 6;
      C[(int64_t)(kChDd + (kSdG + cd) * 6 + ab) * npts] = bar;
    } else {
      W[(int64_t)(12 + (kk - 82)) * npts] = bar;
    }
  }
}

// The ADM channels' adjoint (K and gamma at the vertex, the transposed
// first-derivative stencil of K) at every vertex, through Z4cToADM
// transposed (chi_psi_power = -4: psi4 = 1/chi, gamma = psi4 g~,
// K = psi4 A~ + (Khat + 2 Theta)/3 gamma), added to ubar.
template <int NX>
__global__ void __launch_bounds__(kThreads)
k_weyl_adm_gather(Grid gin, DevParams P, const double* __restrict__ u,
                  const double* __restrict__ wadm, double* __restrict__ ubar) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t nv = g.nvol;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * g.nblocks) return;
  const int64_t q = t % nv;
  const int b = (int)(t / nv);
  const int ijk[3] = {(int)(q % g.nn[0]), (int)((q / g.nn[0]) % g.nn[1]),
                      (int)(q / ((int64_t)g.nn[0] * g.nn[1]))};
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const double* W = wadm + (int64_t)b * kNWAdm * npts;
  const FdScale& F = P.fd[b];
  double Kb[6], Gb[6];
  const bool interior = is_interior(g, ijk[0], ijk[1], ijk[2]);
  const int64_t lq = interior ? interior_index(g, ijk[0], ijk[1], ijk[2]) : 0;
  for (int c = 0; c < 6; ++c) {
    Kb[c] = interior ? W[(int64_t)c * npts + lq] : 0.0;
    Gb[c] = interior ? W[(int64_t)(6 + c) * npts + lq] : 0.0;
  }
  bool any = interior;
  for (int c = 0; c < 3; ++c) {
    for (int o = -3; o <= 3; ++o) {
      if (o == 0) continue;
      int pp[3] = {ijk[0], ijk[1], ijk[2]};
      pp[c] -= o;
      if (!is_interior(g, pp[0], pp[1], pp[2])) continue;
      const int64_t lp = interior_index(g, pp[0], pp[1], pp[2]);
      const double w = w_d1(o) * F.cidx1[c];
      for (int qq = 0; qq < 6; ++qq) Kb[qq] += w * W[(int64_t)(12 + c * 6 + qq) * npts + lp];
      any = true;
    }
  }
  if (!any) return;
  const double* U = u + (int64_t)b * NVAR * nv + q;
  double* UB = ubar + (int64_t)b * NVAR * nv + q;
  const double chi = U[(int64_t)Z4C_CHI * nv];
  const double psi4 = 1.0 / chi;
  const double Ktr = U[(int64_t)Z4C_KHAT * nv] + 2.0 * U[(int64_t)Z4C_THETA * nv];
  double psi4b = 0.0, trb = 0.0;
  for (int c = 0; c < 6; ++c) {
    const double gt = U[(int64_t)(Z4C_GXX + c) * nv], At = U[(int64_t)(Z4C_AXX + c) * nv];
    const double gph = psi4 * gt;
    UB[(int64_t)(Z4C_AXX + c) * nv] += psi4 * Kb[c];
    psi4b += At * Kb[c];
    trb += (1.0 / 3.0) * gph * Kb[c];
    const double gphb = Gb[c] + (1.0 / 3.0) * Ktr * Kb[c];
    UB[(int64_t)(Z4C_GXX + c) * nv] += psi4 * gphb;
    psi4b += gt * gphb;
  }
  UB[(int64_t)Z4C_KHAT * nv] += trb;
  UB[(int64_t)Z4C_THETA * nv] += 2.0 * trb;
  UB[(int64_t)Z4C_CHI * nv] += -psi4 * psi4 * psi4b;
}

__global__ void k_axpy(int64_t n, double a, const double* __restrict__ x, double* __restrict__ y) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[t] += a * x[t];
}

// Per-CTA partial sums of x . y (added on the host in CTA order).
__global__ void __launch_bounds__(256) k_dot(int64_t n, const double* __restrict__ x,
                                             const double* __restrict__ y, double* __restrict__ part) {
  __shared__ double sm[256];
  double acc = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    acc += x[t] * y[t];
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

// ---- tangent-linear model ------------------------------------------------------

// One low-storage stage of the tangents at every interior vertex: the
// right-hand side's forward-mode derivative (rhs_local on dual numbers) plus
// Kreiss-Oliger of the tangent, then the stage algebra.
__global__ void __launch_bounds__(kThreads)
k_tlm_stage(Grid g, DevParams P, const double* __restrict__ u, const double* __restrict__ sd,
            const double* __restrict__ ud, const double* __restrict__ sdd,
            double* __restrict__ u1d, double* __restrict__ wd, StageW W) {
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * g.nblocks) return;
  const int b = (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_of(g, l, i, j, k);
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  const int64_t nv = g.nvol;
  const int64_t boff = (int64_t)b * NVAR * nv;
  const FdScale& F = P.fd[b];
  RhsLocal<Dual> v;
  gather_rhs<Dual>(g, F, u + boff, sd + (int64_t)b * kSdComponents * nv, ud + boff,
                   sdd + (int64_t)b * kSdComponents * nv, p, v);
  Dual out[NVAR];
  ad::rhs_local(P.p, v, out);
  #pragma unroll
  for (int n = 0; n < NVAR; ++n) {
    const double* fd = ud + boff + (int64_t)n * nv;
    double r = out[n].d;
    #pragma unroll
    for (int a = 0; a < 3; ++a) {
      double s = 0.;
      #pragma unroll
      for (int o = -4; o <= 4; ++o) s += w_ko(o) * fd[p + o * g.s[a]];
      r += s * F.cidxd[a] * P.p.diss;
    }
    const int64_t qn = boff + (int64_t)n * nv + p;
    const double un = ud[qn];
    const double v1 = (W.first ? 0. : u1d[qn]) + W.delta * un;
    u1d[qn] = v1;
    wd[qn] = W.gamma1 * un + W.gamma2 * v1 + W.beta_dt * r;
  }
}

// The tangent of AlgConstr at every vertex: (upre, upre_dot) -> u_dot (the
// value itself comes from the forward kernel, whose rounding this
// translation unit, compiled with contraction, does not reproduce).
__global__ void __launch_bounds__(kThreads)
k_tlm_alg(Grid g, DevParams P, const double* __restrict__ upre, const double* __restrict__ upred,
          double* __restrict__ ud) {
  const int64_t nv = g.nvol;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * g.nblocks) return;
  const int b = (int)(t / nv);
  const int64_t q = t % nv;
  const int64_t base = (int64_t)b * NVAR * nv + q;
  Dual x[NVAR];
  #pragma unroll
  for (int n = 0; n < NVAR; ++n) x[n] = Dual(upre[base + (int64_t)n * nv], upred[base + (int64_t)n * nv]);
  ad::alg_constr_local(P.p, x);
  #pragma unroll
  for (int n = 0; n < NVAR; ++n) ud[base + (int64_t)n * nv] = x[n].d;
}

// ---- the objective: vol * sum over cells of H^2 --------------------------------

template <class T>
__device__ void gather_ham(const Grid& g, const FdScale& F, const double* U, const double* Ud,
                           int64_t p, HLocal<T>& v) {
  const int64_t nv = g.nvol;
  auto fld = [&](int var) {
    Fld<T> f;
    f.v = U + (int64_t)var * nv;
    if constexpr (sizeof(T) == sizeof(Dual)) f.d = Ud + (int64_t)var * nv;
    return f;
  };
  v.chi = fld(Z4C_CHI).at(p);
  #pragma unroll
  for (int c = 0; c < 6; ++c) {
    v.gt[c] = fld(Z4C_GXX + c).at(p);
    v.At[c] = fld(Z4C_AXX + c).at(p);
  }
  v.Khat = fld(Z4C_KHAT).at(p);
  v.Theta = fld(Z4C_THETA).at(p);
  #pragma unroll
  for (int a = 0; a < 3; ++a) {
    v.dchi[a] = st_d1(fld(Z4C_CHI), p, g.s[a], F.cidx1[a]);
    #pragma unroll
    for (int q = 0; q < 6; ++q) v.dg3[a][q] = st_d1(fld(Z4C_GXX + q), p, g.s[a], F.cidx1[a]);
  }
  #pragma unroll
  for (int a = 0; a < 3; ++a)
    #pragma unroll
    for (int b = a; b < 3; ++b) {
      const int pr = ad::sid(a, b);
      if (a == b) {
        v.ddchi[pr] = st_d2(fld(Z4C_CHI), p, g.s[a], F.cidx2[a]);
        #pragma unroll
        for (int q = 0; q < 6; ++q) v.ddg[q][pr] = st_d2(fld(Z4C_GXX + q), p, g.s[a], F.cidx2[a]);
      } else {
        v.ddchi[pr] = st_d2x(fld(Z4C_CHI), p, g.s[a], g.s[b], F.cidx1[a], F.cidx1[b]);
        #pragma unroll
        for (int q = 0; q < 6; ++q)
          v.ddg[q][pr] = st_d2x(fld(Z4C_GXX + q), p, g.s[a], g.s[b], F.cidx1[a], F.cidx1[b]);
      }
    }
}

// Whether interior vertex (i, j, k) of block b is a cell of the history sum
// (cell index range is..ie, cell-centre radius within r_max_con).
__device__ __forceinline__ bool hst_cell(const Grid& g, const DevParams& P, const double* xv,
                                         int b, int i, int j, int k) {
  if (i >= NG + g.nx[0] || j >= NG + g.nx[1] || k >= NG + g.nx[2]) return false;
  const double* x = xv + (int64_t)b * (g.nn[0] + g.nn[1] + g.nn[2] - 3);
  const double x1 = x[i], x2 = x[g.nn[0] - 1 + j], x3 = x[g.nn[0] + g.nn[1] - 2 + k];
  return x1 * x1 + x2 * x2 + x3 * x3 <= P.p.r_max_con * P.p.r_max_con;
}
// H at a vertex as ADMConstraints gives it: zero beyond r_max_con (vertex
// radius).
__device__ __forceinline__ bool con_live(const Grid& g, const DevParams& P, int b, int i, int j,
                                         int k) {
  const double* x = P.xf + (int64_t)b * (g.nn[0] + g.nn[1] + g.nn[2]);
  const double x1 = x[i], x2 = x[g.nn[0] + j], x3 = x[g.nn[0] + g.nn[1] + k];
  return !(x1 * x1 + x2 * x2 + x3 * x3 > P.p.r_max_con * P.p.r_max_con);
}

// Per interior vertex: H (and its tangent when ud is given), vol H^2 (and
// 2 vol H H_dot) summed per CTA into part[2 * cta].
template <bool TAN>
__global__ void __launch_bounds__(kThreads)
k_ham_obj(Grid g, DevParams P, const double* __restrict__ xv, const double* __restrict__ u,
          const double* __restrict__ ud, double* __restrict__ part) {
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double jv = 0., jd = 0.;
  if (t < npts * g.nblocks) {
    const int b = (int)(t / npts);
    int i, j, k;
    interior_of(g, t % npts, i, j, k);
    if (hst_cell(g, P, xv, b, i, j, k) && con_live(g, P, b, i, j, k)) {
      const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
      const int64_t boff = (int64_t)b * NVAR * g.nvol;
      const double vol = P.dx[3 * b] * P.dx[3 * b + 1] * P.dx[3 * b + 2];
      if (TAN) {
        HLocal<Dual> v;
        gather_ham<Dual>(g, P.fd[b], u + boff, ud + boff, p, v);
        const Dual H = ad::ham_local(P.p, v);
        jv = vol * H.v * H.v;
        jd = 2. * vol * H.v * H.d;
      } else {
        HLocal<double> v;
        gather_ham<double>(g, P.fd[b], u + boff, nullptr, p, v);
        const double H = ad::ham_local(P.p, v);
        jv = vol * H * H;
      }
    }
  }
  __shared__ double s0[kThreads], s1[kThreads];
  s0[threadIdx.x] = jv;
  s1[threadIdx.x] = jd;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0[0];
    part[2 * blockIdx.x + 1] = s1[0];
  }
}

// Reverse of the objective per interior vertex: H_bar = scale * 2 vol H, the
// adjoints of H's local inputs into the H channels.
__global__ void __launch_bounds__(kThreads)
k_ham_adj(Grid g, DevParams P, const double* __restrict__ xv, const double* __restrict__ u,
          double scale, double* __restrict__ hchan) {
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * g.nblocks) return;
  const int b = (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_of(g, l, i, j, k);
  HLocal<double> vb;
  #pragma unroll
  for (int q = 0; q < HLocal<double>::N; ++q) vb.data()[q] = 0.;
  if (hst_cell(g, P, xv, b, i, j, k) && con_live(g, P, b, i, j, k)) {
    const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
    HLocal<double> v;
    gather_ham<double>(g, P.fd[b], u + (int64_t)b * NVAR * g.nvol, nullptr, p, v);
    const double H = ad::ham_local(P.p, v);
    const double vol = P.dx[3 * b] * P.dx[3 * b + 1] * P.dx[3 * b + 2];
    ad::ham_local_adj(P.p, v, scale * 2. * vol * H, vb);
  }
  double* C = hchan + (int64_t)b * kNHChan * npts + l;
  #pragma unroll
  for (int q = 0; q < kNHChan; ++q) C[(int64_t)q * npts] = vb.data()[q];
}

// Adds the transposed stencils of the H channels to ubar at every vertex.
__global__ void __launch_bounds__(kThreads)
k_ham_gather(Grid g, DevParams P, const double* __restrict__ hchan, double* __restrict__ ubar) {
  const int64_t nv = g.nvol;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * NVAR * g.nblocks) return;
  const int64_t q = t % nv;
  const int n = (int)((t / nv) % NVAR);
  const int b = (int)(t / (nv * NVAR));
  int pch = -1;  // point-value channel
  int fq = -1;   // chi: -1 -> field index for stencils: 0 chi, 1..6 g~
  if (n == Z4C_CHI) { pch = kHChi; fq = 0; }
  else if (n >= Z4C_GXX && n <= Z4C_GZZ) { pch = kHGt + (n - Z4C_GXX); fq = 1 + (n - Z4C_GXX); }
  else if (n >= Z4C_AXX && n <= Z4C_AZZ) pch = kHAt + (n - Z4C_AXX);
  else if (n == Z4C_KHAT) pch = kHKhat;
  else if (n == Z4C_THETA) pch = kHTheta;
  if (pch < 0) return;
  const int i = (int)(q % g.nn[0]), j = (int)((q / g.nn[0]) % g.nn[1]),
            k = (int)(q / ((int64_t)g.nn[0] * g.nn[1]));
  const int64_t npts = (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1);
  const double* C = hchan + (int64_t)b * kNHChan * npts;
  const FdScale& F = P.fd[b];
  double acc = 0.;
  if (is_interior(g, i, j, k)) acc = C[(int64_t)pch * npts + interior_index(g, i, j, k)];
  if (fq >= 0) {
    for (int a = 0; a < 3; ++a) {
      const double* d1 = C + (int64_t)(fq == 0 ? kHDchi + a : kHDg + a * 6 + (fq - 1)) * npts;
      const double* d2 = C + (int64_t)(fq == 0 ? kHDdchi + ad::sid(a, a)
                                               : kHDdg + (fq - 1) * 6 + ad::sid(a, a)) * npts;
      double s1 = 0., s2 = 0.;
      for (int o = -3; o <= 3; ++o) {
        int pp[3] = {i, j, k};
        pp[a] -= o;
        if (!is_interior(g, pp[0], pp[1], pp[2])) continue;
        const int64_t li = interior_index(g, pp[0], pp[1], pp[2]);
        s1 += w_d1(o) * d1[li];
        s2 += w_d2(o) * d2[li];
      }
      acc += s1 * F.cidx1[a] + s2 * F.cidx2[a];
    }
    for (int a = 0; a < 3; ++a)
      for (int bb = a + 1; bb < 3; ++bb) {
        const double* dx = C + (int64_t)(fq == 0 ? kHDdchi + ad::sid(a, bb)
                                                 : kHDdg + (fq - 1) * 6 + ad::sid(a, bb)) * npts;
        double s = 0.;
        for (int oa = -3; oa <= 3; ++oa) {
          if (oa == 0) continue;
          for (int ob = -3; ob <= 3; ++ob) {
            if (ob == 0) continue;
            int pp[3] = {i, j, k};
            pp[a] -= oa;
            pp[bb] -= ob;
            if (!is_interior(g, pp[0], pp[1], pp[2])) continue;
            s += w_d1(oa) * w_d1(ob) * dx[interior_index(g, pp[0], pp[1], pp[2])];
          }
        }
        acc += s * F.cidx1[a] * F.cidx1[bb];
      }
  }
  ubar[((int64_t)b * NVAR + n) * nv + q] += acc;
}

// ---- adjoint of the initial data (ADMToZ4c + FinalizeZ4cADMGhosts) ---------

// AlgConstr^T at the ghost vertices only (the ghost pass of
// FinalizeZ4cADMGhosts); interior adjoints pass through.
__global__ void __launch_bounds__(kThreads)
k_adj_alg_ghosts(Grid g, DevParams P, const double* __restrict__ upre, double* __restrict__ ubar) {
  const int64_t nv = g.nvol;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * g.nblocks) return;
  const int b = (int)(t / nv);
  const int64_t q = t % nv;
  const int i = (int)(q % g.nn[0]), j = (int)((q / g.nn[0]) % g.nn[1]),
            k = (int)(q / ((int64_t)g.nn[0] * g.nn[1]));
  if (is_interior(g, i, j, k)) return;
  double uu[NVAR], ub[NVAR];
  const double* UP = upre + (int64_t)b * NVAR * nv + q;
  double* UB = ubar + (int64_t)b * NVAR * nv + q;
  for (int n = 0; n < NVAR; ++n) {
    uu[n] = UP[(int64_t)n * nv];
    ub[n] = UB[(int64_t)n * nv];
  }
  ad::alg_constr_adj(P.p, uu, ub);
  for (int n = 0; n < NVAR; ++n) UB[(int64_t)n * nv] = ub[n];
}

// Adjoint of the inverse conformal metric through Gamma~^a = -sum_c
// D_c g~^{ca} on the interior (adm_z4c.cpp:165-176): gub[s] at every vertex,
// s the stored pair of g~^{ca}.
__global__ void __launch_bounds__(kThreads)
k_adj_adm_gam(Grid g, DevParams P, const double* __restrict__ ubar, double* __restrict__ gub) {
  const int64_t nv = g.nvol;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * g.nblocks) return;
  const int b = (int)(t / nv);
  const int64_t q = t % nv;
  const int ijk[3] = {(int)(q % g.nn[0]), (int)((q / g.nn[0]) % g.nn[1]),
                      (int)(q / ((int64_t)g.nn[0] * g.nn[1]))};
  const double* UB = ubar + (int64_t)b * NVAR * nv;
  const FdScale& F = P.fd[b];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int c = 0; c < 3; ++c) {
    bool ok = true;
    for (int e = 0; e < 3; ++e)
      if (e != c) ok = ok && ijk[e] >= NG && ijk[e] <= NG + g.nx[e];
    if (!ok) continue;
    const int olo = max(-3, ijk[c] - NG - g.nx[c]), ohi = min(3, ijk[c] - NG);
#pragma unroll
    for (int o = -3; o <= 3; ++o) {
      if (o == 0 || o < olo || o > ohi) continue;
      const int64_t pq = q - (int64_t)o * g.s[c];
      const double w = -w_d1(o) * F.cidx1[c];
      for (int a = 0; a < 3; ++a) acc[ad::sid(c, a)] += w * UB[(int64_t)(Z4C_GAMX + a) * nv + pq];
    }
  }
  for (int s = 0; s < 6; ++s) gub[((int64_t)b * 6 + s) * nv + q] = acc[s];
}

// Reverse of the pointwise ADMToZ4c at every vertex: the lapse and shift
// through their copies, the metric and curvature through 12 forward-mode
// directions of adm_to_z4c_local.
__global__ void __launch_bounds__(kThreads)
k_adj_adm_pt(Grid g, const double* __restrict__ adm, const double* __restrict__ ubar,
             const double* __restrict__ gub, double* __restrict__ admbar) {
  const int64_t nv = g.nvol;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * g.nblocks) return;
  const int b = (int)(t / nv);
  const int64_t q = t % nv;
  const double* A = adm + (int64_t)b * Z4C_NADM * nv + q;
  const double* UB = ubar + (int64_t)b * NVAR * nv + q;
  double* AB = admbar + (int64_t)b * Z4C_NADM * nv + q;
  AB[(int64_t)Z4C_ADM_ALPHA * nv] = UB[(int64_t)Z4C_ALPHA * nv];
  for (int a = 0; a < 3; ++a) AB[(int64_t)(Z4C_ADM_BETAX + a) * nv] = UB[(int64_t)(Z4C_BETAX + a) * nv];
  AB[(int64_t)Z4C_ADM_PSI4 * nv] = 0.;
  double G[6], K[6], gb[6];
  for (int c = 0; c < 6; ++c) {
    G[c] = A[(int64_t)(Z4C_ADM_GXX + c) * nv];
    K[c] = A[(int64_t)(Z4C_ADM_KXX + c) * nv];
    gb[c] = gub[((int64_t)b * 6 + c) * nv + q];
  }
  double ob_chi = UB[(int64_t)Z4C_CHI * nv], ob_kh = UB[(int64_t)Z4C_KHAT * nv];
  double ob_g[6], ob_a[6];
  for (int c = 0; c < 6; ++c) {
    ob_g[c] = UB[(int64_t)(Z4C_GXX + c) * nv];
    ob_a[c] = UB[(int64_t)(Z4C_AXX + c) * nv];
  }
  for (int dir = 0; dir < 12; ++dir) {
    Dual Gd[6], Kd[6];
    for (int c = 0; c < 6; ++c) {
      Gd[c] = Dual(G[c], dir == c ? 1. : 0.);
      Kd[c] = Dual(K[c], dir == 6 + c ? 1. : 0.);
    }
    Dual chi, gt[6], kh, At[6], guu[6];
    ad::adm_to_z4c_local(Gd, Kd, &chi, gt, &kh, At, guu);
    double s = ob_chi * chi.d + ob_kh * kh.d;
    for (int c = 0; c < 6; ++c) s += ob_g[c] * gt[c].d + ob_a[c] * At[c].d + gb[c] * guu[c].d;
    AB[(int64_t)((dir < 6 ? Z4C_ADM_GXX : Z4C_ADM_KXX - 6) + dir) * nv] = s;
  }
}

// acc[0..1] += the sums of part[2 i], part[2 i + 1] over i < n, in a fixed
// order (one CTA of 256 threads)
__global__ void k_accumulate(const double* __restrict__ part, int n, double* __restrict__ acc) {
  __shared__ double s0[256], s1[256];
  double a = 0., b = 0.;
  for (int i = threadIdx.x; i < n; i += 256) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    acc[0] += s0[0];
    acc[1] += s1[0];
  }
}

}  // namespace

// ---- buffers -------------------------------------------------------------------

struct AdjState {
  int64_t reg_elems = 0;
  double* tan = nullptr;    // tangent of u (Z4C_REG_TAN)
  double* tan1 = nullptr;   // tangent of u1
  double* tanw = nullptr;   // tangent of the stage output / pre-constraint state
  double* sdd = nullptr;    // stored first derivatives of the tangent
  double* adj = nullptr;    // adjoint of u (Z4C_REG_ADJ)
  double* adj1 = nullptr;   // adjoint of u1
  double* wbar = nullptr;   // adjoint of the stage output
  double* direct = nullptr; // direct adjoint of the stage input at interior vertices
  double* upre[4] = {};     // pre-constraint exchanged states of the four stages
  double* us = nullptr;     // recomputed stage input
  double* w = nullptr;      // forward stage output
  double* u1 = nullptr;     // forward u1
  double* chan = nullptr;   // right-hand side reverse channels
  double* rsb = nullptr;    // Ricci-sum adjoints
  double* sdbar = nullptr;  // stored-first-derivative adjoints
  double* hchan = nullptr;  // H reverse channels
  double* part = nullptr;   // per-CTA partial sums
  int npart = 0;
  double* pacc = nullptr;   // device accumulators of the shift_eta, damp_kappa1 adjoints
  double* admbar = nullptr; // adjoint of the ADM register (Z4C_REG_ADM_ADJ)
  double* gub = nullptr;    // adjoint of the inverse conformal metric of ADMToZ4c
  int* pro_owner = nullptr; // refined meshes: the prolongation box that carries each fine vertex
  std::vector<double*> snaps;  // revolve snapshots
  // the Weyl-scalar objective term (z4c_adj_set_weyl)
  int wsphere = -1;         // the psi4 sphere of the term; -1: no term
  double wweight = 0.0;     // its weight in J
  double* admw = nullptr;   // ADM state of the evaluation point
  double* wreg = nullptr;   // psi4 (2 variables) before the ghost fill
  double* wtmp = nullptr;   // psi4 after the fill; its interiors' adjoint on the way back
  double* wregb = nullptr;  // adjoint of the filled psi4 register
  double* wadm = nullptr;   // ADM channels [block][kNWAdm][interior vertex]
  double* databar = nullptr;  // adjoint of the sphere values [2][npts]
  double* dpart = nullptr;  // dot-product partial sums
};

void adj_free(AdjState* a) {
  if (!a) return;
  for (double* p : {a->tan, a->tan1, a->tanw, a->sdd, a->adj, a->adj1, a->wbar, a->direct, a->us,
                    a->w, a->u1, a->chan, a->rsb, a->sdbar, a->hchan, a->part, a->pacc,
                    a->admbar, a->gub})
    if (p) cudaFree(p);
  for (double* p : a->upre)
    if (p) cudaFree(p);
  for (double* p : a->snaps)
    if (p) cudaFree(p);
  if (a->pro_owner) cudaFree(a->pro_owner);
  for (double* p : {a->admw, a->wreg, a->wtmp, a->wregb, a->wadm, a->databar, a->dpart})
    if (p) cudaFree(p);
  delete a;
}

}  // namespace z4c

namespace {

char g_msg[512];
int err(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int err(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return z4c::set_error(code, g_msg);
}

#define ACUDA(expr)                                                                 \
  do {                                                                              \
    cudaError_t e_ = (expr);                                                        \
    if (e_ != cudaSuccess) return err(Z4C_ECUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)
#define ALAUNCH(what)                                                               \
  do {                                                                              \
    cudaError_t e_ = cudaGetLastError();                                            \
    if (e_ != cudaSuccess) return err(Z4C_ECUDA, "%s launch: %s", what, cudaGetErrorString(e_)); \
  } while (0)

int64_t npts_of(const Grid& g) { return (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * (g.nx[2] + 1); }

int check_ctx(z4c_ctx* c) {
  if (!c) return err(Z4C_EINVAL, "null context");
  if (c->integrator != Z4C_INTEG_RK4) return err(Z4C_ESTATE, "the adjoint differentiates rk4 (2S)");
  if (c->g.has_sommerfeld) return err(Z4C_ESTATE, "the adjoint has no gr_sommerfeld faces");

  if (c->params.chi_psi_power != -4.)
    return err(Z4C_ESTATE, "the adjoint objective assumes chi_psi_power = -4");
  if (!c->adj) return err(Z4C_ESTATE, "call z4c_adj_setup first");
  return Z4C_OK;
}

// Transpose of launch_physical_bcs: the axes in reverse order.
template <int NVB = NVAR>
void adj_physical_bcs(const Grid& g, double* ub, cudaStream_t st) {
  for (int ax = 2; ax >= 0; --ax) {
    if (g.bc[2 * ax] == Z4C_BC_PERIODIC && g.bc[2 * ax + 1] == Z4C_BC_PERIODIC) continue;
    const int o1 = (ax == 0) ? 1 : 0, o2 = (ax == 2) ? 1 : 2;
    const int64_t n = (int64_t)g.nn[o1] * g.nn[o2] * 2 * NVB * g.nb[o1] * g.nb[o2];
    auto kern = ax == 0 ? k_adj_bc_axis<0, NVB>
                        : ax == 1 ? k_adj_bc_axis<1, NVB> : k_adj_bc_axis<2, NVB>;
    kern<<<div_up(n, kThreads), kThreads, 0, st>>>(g, ub);
    add_kernel_launches(1);
  }
}

// The ghost fill of the step without AlgConstr (the same-level exchange and
// the physical BCs, or the multilevel fill with its BCs): src's interiors to
// every vertex of dst.
int fill_fwd(z4c_ctx* c, const double* src, double* dst) {
  if (c->ml) return launch_ml_exchange(*c->ml, src, dst, NVAR, NVAR, c->stream);
  launch_exchange(c->g, c->dev(), src, dst, c->nbr, 0, c->stream);
  launch_physical_bcs(c->g, dst, NVAR, c->stream);
  ALAUNCH("exchange");
  return Z4C_OK;
}

// Its transpose: ubar (the adjoint of every vertex after the fill) is
// consumed; wbar receives the adjoint of the interiors, and zero ghosts
// where the caller reads them (clear_ghosts; the multilevel transpose
// clears wbar in any case).
int fill_adj(z4c_ctx* c, double* ubar, double* wbar, bool clear_ghosts) {
  const Grid& g = c->g;
  if (c->ml)
    return launch_ml_exchange_adj(*c->ml, ubar, wbar, c->adj->pro_owner, NVAR, NVAR, c->stream);
  adj_physical_bcs(g, ubar, c->stream);
  if (clear_ghosts)
    ACUDA(cudaMemsetAsync(wbar, 0, sizeof(double) * c->adj->reg_elems, c->stream));
  (has_fixed_geometry(g) ? k_adj_exchange<kFixedNX> : k_adj_exchange<0>)<<<
      div_up(npts_of(g) * g.nblocks, kThreads), kThreads, 0, c->stream>>>(g, ubar, wbar);
  ALAUNCH("adjoint exchange");
  add_kernel_launches(1);
  return Z4C_OK;
}

// Forward stage s (1-based) from u (stage input, all vertices) and u1: w,
// u1 updated, then E(w) -> upre (no constraint), AlgConstr(upre) -> uout.
int fwd_stage(z4c_ctx* c, int s, double dt, const double* u, double* u1, double* w, double* upre,
              double* uout) {
  const double* wt = kLsRk4[s - 1];
  LsStage ls{wt[0], wt[1], wt[2], wt[3], wt[4] * dt, s == 1 ? 1 : 0};
  const DevParams P = c->dev();
  launch_stage_ls(c->g, P, u, c->scratch(), c->reg[Z4C_REG_RHS], u1, w, ls, 0, c->g.nblocks,
                  c->shape, c->stream);
  ALAUNCH("stage");
  int rc = fill_fwd(c, w, upre);
  if (rc) return rc;
  if (uout) {
    if (uout != upre)
      ACUDA(cudaMemcpyAsync(uout, upre, sizeof(double) * c->adj->reg_elems,
                            cudaMemcpyDeviceToDevice, c->stream));
    launch_alg_constr(c->g, P, uout, 0, c->g.nblocks, c->stream);
    ALAUNCH("alg_constr");
  }
  return Z4C_OK;
}

// One forward step of u in place (the captured step's arithmetic, separate
// exchange and constraint passes).
int fwd_step(z4c_ctx* c, double dt, double* u) {
  z4c::AdjState* A = c->adj;
  for (int s = 1; s <= 4; ++s) {
    int rc = fwd_stage(c, s, dt, u, A->u1, A->w, A->us, u);
    if (rc) return rc;
  }
  return Z4C_OK;
}

int reduce_part(z4c_ctx* c, int nblk, double out[2]) {
  std::vector<double> h((size_t)2 * nblk);
  ACUDA(cudaMemcpyAsync(h.data(), c->adj->part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                        c->stream));
  ACUDA(cudaStreamSynchronize(c->stream));
  out[0] = out[1] = 0.;
  for (int i = 0; i < nblk; ++i) {
    out[0] += h[2 * (size_t)i];
    out[1] += h[2 * (size_t)i + 1];
  }
  return Z4C_OK;
}

// Adjoint of one step starting from the state u (not modified): A->adj
// holds the adjoint of the state after the step on entry and of u on return.
int adj_step(z4c_ctx* c, double dt, const double* u) {
  z4c::AdjState* A = c->adj;
  const Grid& g = c->g;
  const DevParams P = c->dev();
  const int64_t bytes = sizeof(double) * A->reg_elems;
  // recompute the step, keeping each stage's pre-constraint state
  ACUDA(cudaMemcpyAsync(A->us, u, bytes, cudaMemcpyDeviceToDevice, c->stream));
  for (int s = 1; s <= 4; ++s) {
    // stage s from us; its constrained output becomes the next stage's input
    int rc = fwd_stage(c, s, dt, A->us, A->u1, A->w, A->upre[s - 1], s < 4 ? A->us : nullptr);
    if (rc) return rc;
  }
  // the adjoint of u1 after the last stage is zero: the next step starts u1 at zero
  ACUDA(cudaMemsetAsync(A->adj1, 0, bytes, c->stream));
  const int64_t npts = npts_of(g);
  const int nthr = div_up(npts * g.nblocks, kThreads);
  for (int s = 4; s >= 1; --s) {
    // AlgConstr^T then E^T: adjoint of this stage's output w
    (has_fixed_geometry(g) ? k_adj_alg<kFixedNX> : k_adj_alg<0>)<<<div_up(g.nvol * g.nblocks, kThreads), kThreads, 0, c->stream>>>(g, P, A->upre[s - 1],
                                                                             A->adj);
    add_kernel_launches(1);
    int rc = fill_adj(c, A->adj, A->wbar, false);
    if (rc) return rc;
    // the stage input
    const double* us = u;
    if (s > 1) {
      ACUDA(cudaMemcpyAsync(A->us, A->upre[s - 2], bytes, cudaMemcpyDeviceToDevice, c->stream));
      launch_alg_constr(g, P, A->us, 0, g.nblocks, c->stream);
      ALAUNCH("alg_constr");
      us = A->us;
    }
    launch_prep_ricci(g, P, us, c->scratch(), 0, g.nblocks, c->shape, c->stream);
    ALAUNCH("prep_ricci");
    const double* wt = kLsRk4[s - 1];
    StageW W{wt[0], wt[1], wt[2], wt[4] * dt, s == 1 ? 1 : 0};
    (has_fixed_geometry(g) ? k_adj_main<kFixedNX> : k_adj_main<0>)<<<nthr, kThreads, 0, c->stream>>>(g, P, us, c->sd, c->rsum, A->wbar, A->adj1,
                                                 A->direct, A->chan, A->rsb, A->part, W);
    k_accumulate<<<1, 256, 0, c->stream>>>(A->part, nthr, A->pacc);
    ALAUNCH("adjoint main");
    (has_fixed_geometry(g) ? k_adj_ricci<kFixedNX> : k_adj_ricci<0>)<<<nthr, kThreads, 0, c->stream>>>(g, P, us, c->sd, A->rsb, A->direct, A->chan);
    (has_fixed_geometry(g) ? k_adj_advbeta<kFixedNX> : k_adj_advbeta<0>)<<<nthr, kThreads, 0, c->stream>>>(g, P, us, A->wbar, A->direct, W.beta_dt);
    const int64_t creg = (int64_t)(g.nx[0] + 7) * (g.nx[1] + 7) * (g.nx[2] + 1);
    (has_fixed_geometry(g) ? k_adj_sdbar<kFixedNX> : k_adj_sdbar<0>)<<<dim3(div_up(creg, kThreads), kSdComponents, g.nblocks), kThreads, 0, c->stream>>>(
        g, P, A->chan, A->sdbar);
    (has_fixed_geometry(g) ? k_adj_gather<kFixedNX> : k_adj_gather<0>)<<<div_up(g.nvol * g.nblocks, kThreads), kThreads, 0, c->stream>>>(
        g, P, us, A->wbar, A->direct, A->chan, A->sdbar, A->adj, W.beta_dt);
    ALAUNCH("adjoint gather");
    add_kernel_launches(6);
  }
  return Z4C_OK;
}

// Revolve-style checkpointing.  cost(n, s): the fewest forward steps that
// reversing n steps needs, given the state at their start and s free
// snapshots: reverse the first m steps after the last n - m, the state after
// m steps kept in a snapshot meanwhile (m advances), so
//   cost(n, s) = min_m [m + cost(n - m, s - 1) + cost(m, s)],
//   cost(1, s) = 0,  cost(n, 0) = n (n - 1) / 2 (re-advance for every step);
// the minimum is the binomial (Griewank-Walther) schedule.
struct Schedule {
  int n, s;
  std::vector<long long> cost;
  std::vector<int> split;
  long long& C(int nn, int ss) { return cost[(size_t)nn * (s + 1) + ss]; }
  int& M(int nn, int ss) { return split[(size_t)nn * (s + 1) + ss]; }
  Schedule(int n_, int s_) : n(n_), s(s_), cost((size_t)(n_ + 1) * (s_ + 1), 0),
                             split((size_t)(n_ + 1) * (s_ + 1), 0) {
    for (int nn = 1; nn <= n; ++nn)
      for (int ss = 0; ss <= s; ++ss) {
        if (nn == 1) { C(nn, ss) = 0; continue; }
        if (ss == 0) { C(nn, ss) = (long long)nn * (nn - 1) / 2; continue; }
        long long best = -1;
        int bm = 1;
        for (int m = 1; m < nn; ++m) {
          const long long v = m + C(nn - m, ss - 1) + C(m, ss);
          if (best < 0 || v < best) { best = v; bm = m; }
        }
        C(nn, ss) = best;
        M(nn, ss) = bm;
      }
  }
};

struct GradRun {
  z4c_ctx* c;
  double dt, w_step;
  Schedule* sch;
  std::vector<double*> free_snaps;
  double* run;  // work state of the snapshot-free recomputation
  double* end;  // the state after the step being reversed (per-step objective)
  long long fwd_steps = 0, adj_steps = 0;
};

int advance(GradRun& R, double* u, int nsteps) {
  for (int i = 0; i < nsteps; ++i) {
    int rc = fwd_step(R.c, R.dt, u);
    if (rc) return rc;
    ++R.fwd_steps;
  }
  return Z4C_OK;
}

// Z4C_REG_ADJ += scale dJ/du at the state u
// ---- the Weyl-scalar objective term (host) ----
// psi4 of the state u at the term's sphere vertices into the sphere's data
// array: Z4cToADM, Z4cWeyl, the Weyl register's ghost fill, the
// interpolation.
int weyl_psi(z4c_ctx* c, const double* u) {
  z4c::AdjState* A = c->adj;
  const Grid& g = c->g;
  const DevParams P = c->dev();
  launch_z4c_to_adm(g, P, u, A->admw, 0, g.nblocks, c->stream);
  launch_weyl(g, P, A->admw, u, c->sd, c->rsum, c->lv, A->wreg, c->xf, 0, g.nblocks, c->stream);
  ALAUNCH("Weyl");
  if (c->ml) {
    int rc = launch_ml_exchange(*c->ml, A->wreg, A->wtmp, Z4C_NWEYL, Z4C_NWEYL, c->stream);
    if (rc) return rc;
  } else {
    launch_exchange(g, P, A->wreg, A->wtmp, c->nbr, 0, c->stream, Z4C_NWEYL);
    if (c->has_outflow) launch_physical_bcs(g, A->wtmp, Z4C_NWEYL, c->stream);
    ALAUNCH("Weyl ghost fill");
  }
  launch_wave_interp(g, c->waves[A->wsphere], A->wtmp, c->stream);
  ALAUNCH("sphere interpolation");
  return Z4C_OK;
}

// J_W at u; with databar, also the adjoint of the sphere values for the
// scale (scale * 2 w_p psi4(p)), uploaded to A->databar.
int weyl_J(z4c_ctx* c, const double* u, double* J, double scale, bool databar) {
  z4c::AdjState* A = c->adj;
  const WaveSphere& w = c->waves[A->wsphere];
  int rc = weyl_psi(c, u);
  if (rc) return rc;
  std::vector<double> d((size_t)2 * w.npts), pw((size_t)2 * w.npts);
  ACUDA(cudaMemcpyAsync(d.data(), w.data, sizeof(double) * d.size(), cudaMemcpyDeviceToHost,
                        c->stream));
  ACUDA(cudaMemcpyAsync(pw.data(), w.pw, sizeof(double) * pw.size(), cudaMemcpyDeviceToHost,
                        c->stream));
  ACUDA(cudaStreamSynchronize(c->stream));
  double s = 0.0;
  for (int p = 0; p < w.npts; ++p) {
    const double dr = d[p], di = d[(size_t)w.npts + p];
    s += pw[2 * (size_t)p] * (dr * dr + di * di);
    if (databar) {
      d[p] = scale * 2.0 * pw[2 * (size_t)p] * dr;
      d[(size_t)w.npts + p] = scale * 2.0 * pw[2 * (size_t)p] * di;
    }
  }
  if (J) *J = s;
  if (databar)
    ACUDA(cudaMemcpyAsync(A->databar, d.data(), sizeof(double) * d.size(),
                          cudaMemcpyHostToDevice, c->stream));
  return Z4C_OK;
}

// out (22 variables, every vertex) = scale dJ_W/du at u.
int weyl_adj(z4c_ctx* c, const double* u, double scale, double* out) {
  z4c::AdjState* A = c->adj;
  const Grid& g = c->g;
  const DevParams P = c->dev();
  int rc = weyl_J(c, u, nullptr, scale, true);
  if (rc) return rc;
  const size_t wbytes = sizeof(double) * Z4C_NWEYL * g.nvol * g.nblocks;
  ACUDA(cudaMemsetAsync(A->wregb, 0, wbytes, c->stream));
  launch_wave_interp_adj(g, c->waves[A->wsphere], A->databar, A->wregb, c->stream);
  ALAUNCH("sphere interpolation transpose");
  // the Weyl register's ghost fill transposed: the interiors' adjoint in wtmp
  if (c->ml) {
    if ((rc = launch_ml_exchange_adj(*c->ml, A->wregb, A->wtmp, A->pro_owner, Z4C_NWEYL,
                                     Z4C_NWEYL, c->stream)))
      return rc;
  } else {
    if (c->has_outflow) adj_physical_bcs<Z4C_NWEYL>(g, A->wregb, c->stream);
    (has_fixed_geometry(g) ? k_adj_exchange<kFixedNX, Z4C_NWEYL> : k_adj_exchange<0, Z4C_NWEYL>)<<<
        div_up(npts_of(g) * g.nblocks, kThreads), kThreads, 0, c->stream>>>(g, A->wregb, A->wtmp);
    ALAUNCH("Weyl ghost fill transpose");
    add_kernel_launches(1);
  }
  const int64_t npts = npts_of(g) * g.nblocks;
  const size_t reg = sizeof(double) * A->reg_elems;
  ACUDA(cudaMemsetAsync(A->chan, 0, sizeof(double) * kNChan * npts, c->stream));
  ACUDA(cudaMemsetAsync(A->direct, 0, reg, c->stream));
  ACUDA(cudaMemsetAsync(A->wadm, 0, sizeof(double) * kNWAdm * npts, c->stream));
  const bool fx = has_fixed_geometry(g);
  (fx ? k_weyl_adj<kFixedNX> : k_weyl_adj<0>)<<<div_up(npts, kThreads), kThreads, 0, c->stream>>>(
      g, P, u, A->admw, c->sd, c->xf, A->wtmp, A->chan, A->direct, A->wadm);
  ALAUNCH("Weyl reverse");
  const int64_t creg = (int64_t)(g.nx[0] + 7) * (g.nx[1] + 7) * (g.nx[2] + 1);
  (fx ? k_adj_sdbar<kFixedNX> : k_adj_sdbar<0>)<<<dim3(div_up(creg, kThreads), kSdComponents,
                                                      g.nblocks), kThreads, 0, c->stream>>>(
      g, P, A->chan, A->sdbar);
  ACUDA(cudaMemsetAsync(A->wbar, 0, reg, c->stream));  // no stage terms
  (fx ? k_adj_gather<kFixedNX> : k_adj_gather<0>)<<<div_up(g.nvol * g.nblocks, kThreads),
                                                    kThreads, 0, c->stream>>>(
      g, P, u, A->wbar, A->direct, A->chan, A->sdbar, out, 0.0);
  (fx ? k_weyl_adm_gather<kFixedNX> : k_weyl_adm_gather<0>)<<<div_up(g.nvol * g.nblocks, kThreads),
                                                              kThreads, 0, c->stream>>>(
      g, P, u, A->wadm, out);
  ALAUNCH("Weyl adjoint gather");
  add_kernel_launches(4);
  return Z4C_OK;
}

// x . y over n values (per-CTA partials added on the host in order).
int dot_dev(z4c_ctx* c, const double* x, const double* y, int64_t n, double* out) {
  z4c::AdjState* A = c->adj;
  const int nb = 1024;
  k_dot<<<nb, 256, 0, c->stream>>>(n, x, y, A->dpart);
  ALAUNCH("dot");
  add_kernel_launches(1);
  std::vector<double> h(nb);
  ACUDA(cudaMemcpyAsync(h.data(), A->dpart, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                        c->stream));
  ACUDA(cudaStreamSynchronize(c->stream));
  double s = 0.0;
  for (double v : h) s += v;
  *out = s;
  return Z4C_OK;
}

bool weyl_on(const z4c_ctx* c) { return c->adj && c->adj->wsphere >= 0 && c->adj->wweight != 0.0; }

int objective_adj(z4c_ctx* c, const double* u, double scale) {
  const Grid& g = c->g;
  const DevParams P = c->dev();
  k_ham_adj<<<div_up(npts_of(g) * g.nblocks, kThreads), kThreads, 0, c->stream>>>(
      g, P, c->xv, u, scale, c->adj->hchan);
  k_ham_gather<<<div_up(g.nvol * NVAR * g.nblocks, kThreads), kThreads, 0, c->stream>>>(
      g, P, c->adj->hchan, c->adj->adj);
  ALAUNCH("objective adjoint");
  add_kernel_launches(2);
  if (weyl_on(c)) {  // REG_ADJ += scale * weight * dJ_W/du
    z4c::AdjState* A = c->adj;
    int rc = weyl_adj(c, u, scale * A->wweight, A->tanw);
    if (rc) return rc;
    k_axpy<<<div_up(A->reg_elems, 256), 256, 0, c->stream>>>(A->reg_elems, 1.0, A->tanw, A->adj);
    ALAUNCH("axpy");
    add_kernel_launches(1);
  }
  return Z4C_OK;
}

// J at the state u and, with ud, its derivative along ud
int objective(z4c_ctx* c, const double* u, const double* ud, double* J, double* Jdot) {
  const Grid& g = c->g;
  const DevParams P = c->dev();
  const int nthr = div_up(npts_of(g) * g.nblocks, kThreads);
  if (ud) k_ham_obj<true><<<nthr, kThreads, 0, c->stream>>>(g, P, c->xv, u, ud, c->adj->part);
  else k_ham_obj<false><<<nthr, kThreads, 0, c->stream>>>(g, P, c->xv, u, nullptr, c->adj->part);
  ALAUNCH("objective");
  add_kernel_launches(1);
  double s2[2];
  int rc = reduce_part(c, nthr, s2);
  if (rc) return rc;
  *J = s2[0];
  if (Jdot) *Jdot = s2[1];
  if (weyl_on(c)) {
    z4c::AdjState* A = c->adj;
    double Jw = 0.0;
    if ((rc = weyl_J(c, u, &Jw, 0.0, false))) return rc;
    *J += A->wweight * Jw;
    if (Jdot && ud) {  // the tangent of J_W: its gradient along ud
      if ((rc = weyl_adj(c, u, A->wweight, A->tanw))) return rc;
      double dj = 0.0;
      if ((rc = dot_dev(c, A->tanw, ud, A->reg_elems, &dj))) return rc;
      *Jdot += dj;
    }
  }
  return Z4C_OK;
}

// Adjoint of the step from u, with the per-step objective's source at its end.
int adj_step_with_source(GradRun& R, const double* u) {
  z4c_ctx* c = R.c;
  if (R.w_step != 0.) {
    ACUDA(cudaMemcpyAsync(R.end, u, sizeof(double) * c->adj->reg_elems,
                          cudaMemcpyDeviceToDevice, c->stream));
    int rc = fwd_step(c, R.dt, R.end);
    if (rc) return rc;
    ++R.fwd_steps;
    rc = objective_adj(c, R.end, R.w_step);
    if (rc) return rc;
  }
  ++R.adj_steps;
  return adj_step(c, R.dt, u);
}

// Reverses steps [l, r) given the state at l in x (unchanged).
int reverse(GradRun& R, const double* x, int l, int r, int s) {
  const int n = r - l;
  z4c::AdjState* A = R.c->adj;
  const size_t bytes = sizeof(double) * A->reg_elems;
  if (n == 1) return adj_step_with_source(R, x);
  if (s == 0) {
    for (int i = r - 1; i >= l; --i) {
      ACUDA(cudaMemcpyAsync(R.run, x, bytes, cudaMemcpyDeviceToDevice, R.c->stream));
      int rc = advance(R, R.run, i - l);
      if (!rc) rc = adj_step_with_source(R, R.run);
      if (rc) return rc;
    }
    return Z4C_OK;
  }
  const int m = R.sch->M(n, s);
  double* snap = R.free_snaps.back();
  R.free_snaps.pop_back();
  ACUDA(cudaMemcpyAsync(snap, x, bytes, cudaMemcpyDeviceToDevice, R.c->stream));
  int rc = advance(R, snap, m);
  if (!rc) rc = reverse(R, snap, l + m, r, s - 1);
  R.free_snaps.push_back(snap);
  if (rc) return rc;
  return reverse(R, x, l, l + m, s);
}

}  // namespace

extern "C" {

int z4c_adj_setup(z4c_ctx* c) {
  if (!c) return err(Z4C_EINVAL, "null context");
  if (c->adj) return Z4C_OK;
  z4c::AdjState* A = new (std::nothrow) z4c::AdjState();
  if (!A) return err(Z4C_ENOMEM, "host allocation");
  const Grid& g = c->g;
  A->reg_elems = (int64_t)NVAR * g.nvol * g.nblocks;
  const int64_t npts = npts_of(g) * g.nblocks;
  const size_t reg = sizeof(double) * A->reg_elems;
  A->npart = div_up(npts, kThreads) + 1;
  struct Buf { double** p; size_t bytes; };
  std::vector<Buf> bufs = {
      {&A->tan, reg}, {&A->tan1, reg}, {&A->tanw, reg}, {&A->adj, reg}, {&A->adj1, reg},
      {&A->wbar, reg}, {&A->direct, reg}, {&A->us, reg}, {&A->w, reg}, {&A->u1, reg},
      {&A->sdd, sizeof(double) * kSdComponents * g.nvol * g.nblocks},
      {&A->sdbar, sizeof(double) * kSdComponents * g.nvol * g.nblocks},
      {&A->chan, sizeof(double) * kNChan * npts}, {&A->rsb, sizeof(double) * kNRsb * npts},
      {&A->hchan, sizeof(double) * kNHChan * npts}, {&A->part, sizeof(double) * 2 * A->npart},
      {&A->pacc, sizeof(double) * 2},
      {&A->admbar, sizeof(double) * Z4C_NADM * g.nvol * g.nblocks},
      {&A->gub, sizeof(double) * 6 * g.nvol * g.nblocks}};
  for (int s = 0; s < 4; ++s) bufs.push_back({&A->upre[s], reg});
  for (auto& b : bufs) {
    if (cudaMalloc((void**)b.p, b.bytes) != cudaSuccess) {
      cudaGetLastError();
      z4c::adj_free(A);
      return err(Z4C_ENOMEM, "adjoint buffers: %zu bytes", b.bytes);
    }
  }
  if (cudaMemsetAsync(A->pacc, 0, sizeof(double) * 2, c->stream) != cudaSuccess) {
    z4c::adj_free(A);
    return err(Z4C_ECUDA, "adjoint buffer clear");
  }
  for (double* p : {A->tan, A->tan1, A->adj, A->adj1})
    if (cudaMemsetAsync(p, 0, reg, c->stream) != cudaSuccess) {
      z4c::adj_free(A);
      return err(Z4C_ECUDA, "adjoint buffer clear");
    }
  if (c->ml) {  // the prolongation owners of the ghost fill's transpose
    if (cudaMalloc((void**)&A->pro_owner, sizeof(int) * g.nvol * g.nblocks) != cudaSuccess) {
      cudaGetLastError();
      z4c::adj_free(A);
      return err(Z4C_ENOMEM, "prolongation owner table");
    }
    if (launch_ml_prolong_owner(*c->ml, A->pro_owner, c->stream) != Z4C_OK) {
      z4c::adj_free(A);
      return err(Z4C_ECUDA, "prolongation owner table");
    }
  }
  c->adj = A;
  c->reg[Z4C_REG_TAN] = A->tan;
  c->reg[Z4C_REG_ADJ] = A->adj;
  c->reg[Z4C_REG_ADM_ADJ] = A->admbar;
  return Z4C_OK;
}

int z4c_tlm_step(z4c_ctx* c, double dt) {
  int rc = check_ctx(c);
  if (rc) return rc;
  z4c::AdjState* A = c->adj;
  const Grid& g = c->g;
  const DevParams P = c->dev();
  double* u = c->reg[Z4C_REG_U];
  const int nthr = div_up(npts_of(g) * g.nblocks, kThreads);
  for (int s = 1; s <= 4; ++s) {
    const double* wt = kLsRk4[s - 1];
    StageW W{wt[0], wt[1], wt[2], wt[4] * dt, s == 1 ? 1 : 0};
    // tangents first (they read the stage input u)
    launch_prep(g, P, u, c->sd, 0, g.nblocks, c->stream);
    launch_prep(g, P, A->tan, A->sdd, 0, g.nblocks, c->stream);
    k_tlm_stage<<<nthr, kThreads, 0, c->stream>>>(g, P, u, c->sd, A->tan, A->sdd, A->tan1, A->tanw,
                                                  W);
    ALAUNCH("tangent stage");
    add_kernel_launches(1);
    // values
    rc = fwd_stage(c, s, dt, u, A->u1, A->w, A->us, nullptr);
    if (rc) return rc;
    rc = fill_fwd(c, A->tanw, A->tan);
    if (rc) return rc;
    // (A->us, A->tan) are the pre-constraint state and its tangent
    ACUDA(cudaMemcpyAsync(A->tanw, A->tan, sizeof(double) * A->reg_elems, cudaMemcpyDeviceToDevice,
                          c->stream));
    k_tlm_alg<<<div_up(g.nvol * g.nblocks, kThreads), kThreads, 0, c->stream>>>(g, P, A->us,
                                                                            A->tanw, A->tan);
    ALAUNCH("tangent alg_constr");
    add_kernel_launches(1);
    ACUDA(cudaMemcpyAsync(u, A->us, sizeof(double) * A->reg_elems, cudaMemcpyDeviceToDevice,
                          c->stream));
    launch_alg_constr(g, P, u, 0, g.nblocks, c->stream);
    ALAUNCH("alg_constr");
  }
  return Z4C_OK;
}

int z4c_adj_step(z4c_ctx* c, double dt) {
  int rc = check_ctx(c);
  if (rc) return rc;
  return adj_step(c, dt, c->reg[Z4C_REG_U]);
}

int z4c_adj_objective(z4c_ctx* c, int reg, int reg_tan, double* J, double* Jdot) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!J || reg < 0 || reg >= Z4C_NREG || !c->reg[reg] ||
      (reg_tan >= 0 && (reg_tan >= Z4C_NREG || !c->reg[reg_tan])))
    return err(Z4C_EINVAL, "bad register or null output");
  if (z4c_reg_nvar(reg) != NVAR || (reg_tan >= 0 && z4c_reg_nvar(reg_tan) != NVAR))
    return err(Z4C_EINVAL, "the objective reads 22-variable registers");
  return objective(c, c->reg[reg], reg_tan >= 0 ? c->reg[reg_tan] : nullptr, J, Jdot);
}

int z4c_adj_objective_adj(z4c_ctx* c, int reg, double scale) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (reg < 0 || reg >= Z4C_NREG || !c->reg[reg] || z4c_reg_nvar(reg) != NVAR)
    return err(Z4C_EINVAL, "bad register");
  return objective_adj(c, c->reg[reg], scale);
}

int z4c_adj_params(z4c_ctx* c, double pbar[2], int reset) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (pbar) {
    ACUDA(cudaMemcpyAsync(pbar, c->adj->pacc, sizeof(double) * 2, cudaMemcpyDeviceToHost,
                          c->stream));
    ACUDA(cudaStreamSynchronize(c->stream));
  }
  if (reset) ACUDA(cudaMemsetAsync(c->adj->pacc, 0, sizeof(double) * 2, c->stream));
  return Z4C_OK;
}

}  // extern "C"

extern "C" int z4c_adj_set_weyl(z4c_ctx* c, int sphere, double weight) {
  int rc = check_ctx(c);
  if (rc) return rc;
  z4c::AdjState* A = c->adj;
  if (sphere < 0) {
    A->wsphere = -1;
    A->wweight = 0.0;
    return Z4C_OK;
  }
  if (sphere >= (int)c->waves.size()) return err(Z4C_EINVAL, "no psi4 sphere %d", sphere);
  if (c->waves[sphere].bitant) return err(Z4C_EINVAL, "the Weyl objective takes full spheres");
  const Grid& g = c->g;
  const int64_t npts = npts_of(g) * g.nblocks;
  const size_t wreg = sizeof(double) * Z4C_NWEYL * g.nvol * g.nblocks;
  struct Buf { double** p; size_t bytes; };
  const Buf bufs[] = {{&A->admw, sizeof(double) * Z4C_NADM * g.nvol * g.nblocks},
                      {&A->wreg, wreg}, {&A->wtmp, wreg}, {&A->wregb, wreg},
                      {&A->wadm, sizeof(double) * kNWAdm * npts}, {&A->dpart, sizeof(double) * 1024}};
  for (const Buf& b : bufs)
    if (!*b.p && cudaMalloc((void**)b.p, b.bytes) != cudaSuccess) {
      cudaGetLastError();
      return err(Z4C_ENOMEM, "Weyl objective buffers: %zu bytes", b.bytes);
    }
  if (A->databar) cudaFree(A->databar);
  A->databar = nullptr;
  if (cudaMalloc((void**)&A->databar, sizeof(double) * 2 * std::max(1, c->waves[sphere].npts)) !=
      cudaSuccess) {
    cudaGetLastError();
    return err(Z4C_ENOMEM, "Weyl objective buffers");
  }
  A->wsphere = sphere;
  A->wweight = weight;
  return Z4C_OK;
}

extern "C" int z4c_adj_snapshots(z4c_ctx* c, int nsteps, int* nsnap) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nsteps < 1 || !nsnap) return err(Z4C_EINVAL, "nsteps >= 1, nsnap non-null");
  const size_t bytes = sizeof(double) * c->adj->reg_elems;
  size_t free_b = 0, total_b = 0;
  ACUDA(cudaMemGetInfo(&free_b, &total_b));
  // keep 2 GiB and 2% of the device free for the library's other scratch
  const size_t margin = (size_t)2 << 30;
  const size_t keep = margin + total_b / 50;
  const long long have = (long long)c->adj->snaps.size();
  long long fit = free_b > keep ? (long long)((free_b - keep) / bytes) : 0;
  fit += have - 2;  // the run and end-state buffers come first
  if (fit < 0) return err(Z4C_ENOMEM, "revolve: no room for the run and end-state buffers");
  *nsnap = (int)std::min<long long>(fit, nsteps - 1);
  return Z4C_OK;
}

extern "C" int z4c_adj_gradient(z4c_ctx* c, double dt, int nsteps, int nsnap, double w_final,
                                double w_step, double* J, double pbar[2], double stats[4]) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nsteps < 1 || !J) return err(Z4C_EINVAL, "nsteps >= 1, J non-null");
  if (nsnap < 0 && (rc = z4c_adj_snapshots(c, nsteps, &nsnap))) return rc;
  z4c::AdjState* A = c->adj;
  const size_t bytes = sizeof(double) * A->reg_elems;
  const int S = std::min(nsnap, nsteps - 1);
  // snapshots: S for the schedule, a run buffer and an end-state buffer
  while ((int)A->snaps.size() < S + 2) {
    double* p = nullptr;
    if (cudaMalloc((void**)&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return err(Z4C_ENOMEM, "revolve snapshots: %d of %zu bytes", S + 2, bytes);
    }
    A->snaps.push_back(p);
  }
  cudaEvent_t e0, e1;
  ACUDA(cudaEventCreate(&e0));
  ACUDA(cudaEventCreate(&e1));
  cudaEventRecord(e0, c->stream);
  Schedule sch(nsteps, S);
  GradRun R{c, dt, w_step, &sch, {}, A->snaps[S], A->snaps[S + 1]};
  for (int i = 0; i < S; ++i) R.free_snaps.push_back(A->snaps[i]);
  ACUDA(cudaMemsetAsync(A->pacc, 0, sizeof(double) * 2, c->stream));
  ACUDA(cudaMemsetAsync(A->adj, 0, bytes, c->stream));
  const double* u0 = c->reg[Z4C_REG_U];
  // forward sweep: the objective along the run
  double Jt = 0.;
  ACUDA(cudaMemcpyAsync(R.run, u0, bytes, cudaMemcpyDeviceToDevice, c->stream));
  for (int i = 1; i <= nsteps; ++i) {
    rc = fwd_step(c, dt, R.run);
    if (rc) return rc;
    ++R.fwd_steps;
    if (w_step != 0. || i == nsteps) {
      double Ji = 0.;
      rc = objective(c, R.run, nullptr, &Ji, nullptr);
      if (rc) return rc;
      if (w_step != 0.) Jt += w_step * Ji;
      if (i == nsteps) Jt += w_final * Ji;
    }
  }
  // the final state's source; every step's end-state source is added as the
  // reverse sweep reaches that step
  if (w_final != 0.) {
    rc = objective_adj(c, R.run, w_final);
    if (rc) return rc;
  }
  rc = reverse(R, u0, 0, nsteps, S);
  if (rc) return rc;
  cudaEventRecord(e1, c->stream);
  ACUDA(cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *J = Jt;
  if (pbar) ACUDA(cudaMemcpy(pbar, A->pacc, sizeof(double) * 2, cudaMemcpyDeviceToHost));
  if (stats) {
    stats[0] = (double)R.fwd_steps;
    stats[1] = (double)R.adj_steps;
    stats[2] = ms * 1e-3;
    stats[3] = (double)sch.C(nsteps, S);
  }
  return Z4C_OK;
}

extern "C" int z4c_adj_adm_to_z4c(z4c_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  z4c::AdjState* A = c->adj;
  const Grid& g = c->g;
  const DevParams P = c->dev();
  const size_t bytes = sizeof(double) * A->reg_elems;
  const int nthr_all = div_up(g.nvol * g.nblocks, kThreads);
  const int64_t npts = npts_of(g);
  // recompute: x1 = the pointwise map and Gamma~ (A->us), x2 = AlgConstr(x1)
  // (A->w), x3 = the ghost fill of x2 (A->upre[0])
  launch_adm_to_z4c(g, P, c->reg[Z4C_REG_ADM], A->us, c->guu, 0, g.nblocks, c->stream, 0);
  ALAUNCH("adm_to_z4c");
  ACUDA(cudaMemcpyAsync(A->w, A->us, bytes, cudaMemcpyDeviceToDevice, c->stream));
  launch_alg_constr(g, P, A->w, 0, g.nblocks, c->stream);
  ALAUNCH("alg_constr");
  if ((rc = fill_fwd(c, A->w, A->upre[0]))) return rc;
  // reverse: AlgConstr on the ghosts, the ghost fill, AlgConstr, the map
  k_adj_alg_ghosts<<<nthr_all, kThreads, 0, c->stream>>>(g, P, A->upre[0], A->adj);
  if ((rc = fill_adj(c, A->adj, A->wbar, true))) return rc;
  (has_fixed_geometry(g) ? k_adj_alg<kFixedNX> : k_adj_alg<0>)<<<nthr_all, kThreads, 0, c->stream>>>(g, P, A->us, A->wbar);
  k_adj_adm_gam<<<nthr_all, kThreads, 0, c->stream>>>(g, P, A->wbar, A->gub);
  k_adj_adm_pt<<<nthr_all, kThreads, 0, c->stream>>>(g, c->reg[Z4C_REG_ADM], A->wbar, A->gub,
                                                     A->admbar);
  ALAUNCH("initial-data adjoint");
  add_kernel_launches(5);
  ACUDA(cudaMemcpyAsync(A->adj, A->wbar, bytes, cudaMemcpyDeviceToDevice, c->stream));
  return Z4C_OK;
}

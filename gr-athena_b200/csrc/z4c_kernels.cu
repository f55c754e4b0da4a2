// Z4c device kernels for sm_100a.  Compiled with -fmad=false so that every
// floating-point expression rounds exactly as the reference's
// -ffp-contract=off build does.
#include <cuda_runtime.h>

#include <atomic>

#include "z4c_adm.cuh"
#include "z4c_common.cuh"
#include "z4c_kernels.cuh"
#include "z4c_rhs.cuh"
#include "z4c_stencil.cuh"
#include "z4c_weyl.cuh"

namespace z4c {

namespace {

// Launch shapes.  The heavy per-vertex passes (k_ricci, k_main) are compiled
// for 64, 128 and 256 threads per CTA (all at the full register file of
// 255 registers per thread); the column passes for k-loop unrolls of 2 and 4
// and up to 512 threads per CTA.  A context's shape comes from the
// autotuner (z4c_autotune) or from z4c_set_tile.
constexpr int kPointThreads = 256;
constexpr int kColumnMaxThreads = 512;

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Rsum scratch: [block][6][interior vertex], interior vertices in i-fastest
// order.
__device__ __forceinline__ double* rsum_at(const Grid& g, double* rsum, int b, int64_t l) {
  return rsum + (int64_t)b * 6 * interior_count(g) + l;
}

// ---- stored first derivatives (Z4c::PrepareZ4cDerivatives) ----------------
// adm_z4c.cpp:972-1037: D_b f for f in chi, g~_ab, alpha, beta^a.  The
// reference fills the interior extended by 3 vertices along both directions
// other than b (:977-985); the passes that read them need D_b f off the
// interior only along the directions a < b of the mixed derivatives
// (Dx_a of the stored Dx_b), so D_x f is computed on the interior, D_y f on
// the interior extended along x, D_z f extended along x and y.  Values are
// the reference's wherever they are computed.
//
// One thread per (i, j) column of a component's region, looping over the
// interior k; D_z keeps the seven-vertex window along k in registers.
// blockIdx.y is the component slot*3 + b, blockIdx.z the block.
__device__ __forceinline__ double fd_dx7(double m3, double m2, double m1, double p1, double p2,
                                         double p3, double cidx1) {
  double out = 0.;
  out += -1. * (m3 - p3);
  out += 9. * (m2 - p2);
  out += -45. * (m1 - p1);
  return out * cidx1;
}

template <int NX>
__global__ void __launch_bounds__(kPointThreads)
k_prep(Grid gin, DevParams P, const double* __restrict__ u, double* __restrict__ sd, int block0) {
  const Grid g = fixed_geometry<NX>(gin);
  constexpr int kUnroll = NX > 0 && NX <= 16 ? NX + 1 : 4;  // the whole z loop of a small block
  const int comp = blockIdx.y;
  const int slot = comp / 3, dir = comp % 3;
  const int b = block0 + (int)blockIdx.z;
  const int ex = (dir >= 1) ? 3 : 0, ey = (dir == 2) ? 3 : 0;
  const int e0 = g.nx[0] + 1 + 2 * ex, e1 = g.nx[1] + 1 + 2 * ey;
  const int c = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (c >= e0 * e1) return;
  const int i = NG - ex + c % e0, j = NG - ey + c / e0;
  const int nn0 = g.nn[0];
  const int sk = nn0 * g.nn[1];
  const int k0 = NG, k1 = NG + g.nx[2];
  const double* f = u + ((int64_t)b * NVAR + sd_field_var(slot)) * g.nvol + j * nn0 + i;
  double* out = sd + ((int64_t)b * kSdComponents + comp) * g.nvol + j * nn0 + i;
  const FdScale& F = P.fd[b];
  if (dir == 2) {
    const double cz = F.cidx1[2];
    double w0 = __ldg(f + (k0 - 3) * sk), w1 = __ldg(f + (k0 - 2) * sk),
           w2 = __ldg(f + (k0 - 1) * sk), w3 = __ldg(f + k0 * sk),
           w4 = __ldg(f + (k0 + 1) * sk), w5 = __ldg(f + (k0 + 2) * sk);
#pragma unroll kUnroll
    for (int k = k0; k <= k1; ++k) {
      const double w6 = __ldg(f + (k + 3) * sk);
      out[k * sk] = fd_dx7(w0, w1, w2, w4, w5, w6, cz);
      w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
    }
  } else {
    const int st = (dir == 0) ? 1 : nn0;
    const double ca = (dir == 0) ? F.cidx1[0] : F.cidx1[1];
#pragma unroll kUnroll
    for (int k = k0; k <= k1; ++k) out[k * sk] = fd_dx(f + k * sk, st, ca);
  }
}

// ---- first pass: Ricci tensor + conformal-factor part per interior vertex --
template <int THREADS, int NX, int MINB = 1>
__global__ void __launch_bounds__(THREADS, MINB)
k_ricci(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ sd,
        double* __restrict__ rsum, int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = interior_count(g);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * nblk) return;
  const int b = block0 + (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_ijk(g, l, i, j, k);
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  double R[6];
  ricci_point(u + (int64_t)b * NVAR * g.nvol, sd + (int64_t)b * kSdComponents * g.nvol, g.nvol,
              p, g.s, P, P.fd[b], R);
  double* rs = rsum_at(g, rsum, b, l);
#pragma unroll
  for (int q = 0; q < 6; ++q) rs[(int64_t)q * npts] = R[q];
}


// ---- Sommerfeld boundary right-hand side (Z4c::Z4cBoundaryRHS) -----------
// z4c/boundary_conditions.cpp:16-174.  On a gr_sommerfeld face's vertex
// plane the right-hand side of Theta, Khat, Gamma^a and A_ab is replaced by
//   rhs = -c u / r - sum_a c s^a Ds_a(u),  s^a = x^a / r,  c = sqrt(2) for
// Khat and 1 otherwise, with the second-order Ds (finite_differencing.tpp:
// 132-150, DBG_SYMMETRIZE_FD branch).  The value depends only on the vertex
// and the variable, so a vertex on several Sommerfeld faces gets it once.
__device__ __forceinline__ bool sommerfeld_var(int n) {
  return n == Z4C_KHAT || n == Z4C_THETA || (n >= Z4C_AXX && n <= Z4C_GAMZ);
}
// Whether vertex (i, j, k) of block b lies on one of its gr_sommerfeld faces.
__device__ __forceinline__ bool on_sommerfeld_face(const Grid& g, const DevParams& P, int b, int i,
                                                   int j, int k) {
  if (P.som) {
    const unsigned m = P.som[b];
    return ((m & 1u) && i == NG) || ((m & 2u) && i == NG + g.nx[0]) || ((m & 4u) && j == NG) ||
           ((m & 8u) && j == NG + g.nx[1]) || ((m & 16u) && k == NG) ||
           ((m & 32u) && k == NG + g.nx[2]);
  }
  const int l0 = b % g.nb[0], l1 = (b / g.nb[0]) % g.nb[1], l2 = b / (g.nb[0] * g.nb[1]);
  return (g.bc[0] == Z4C_BC_SOMMERFELD && l0 == 0 && i == NG) ||
         (g.bc[1] == Z4C_BC_SOMMERFELD && l0 == g.nb[0] - 1 && i == NG + g.nx[0]) ||
         (g.bc[2] == Z4C_BC_SOMMERFELD && l1 == 0 && j == NG) ||
         (g.bc[3] == Z4C_BC_SOMMERFELD && l1 == g.nb[1] - 1 && j == NG + g.nx[1]) ||
         (g.bc[4] == Z4C_BC_SOMMERFELD && l2 == 0 && k == NG) ||
         (g.bc[5] == Z4C_BC_SOMMERFELD && l2 == g.nb[2] - 1 && k == NG + g.nx[2]);
}
template <bool GL = true>
__device__ __forceinline__ double fd_ds(const double* __restrict__ f, int64_t st, double dx) {
  double out = 0.;
  out += -1. * (ld<GL>(f - st) - ld<GL>(f + st));
  return out * (1.0 / (dx * 2));
}
// Sommerfeld value of variable n at vertex (i, j, k) of block b; f points at
// that variable's value there, st holds the strides of f's array.
template <bool GL = true>
__device__ __forceinline__ double sommerfeld_value(const Grid& g, const DevParams& P, int b,
                                                  int n, const double* __restrict__ f, int i,
                                                  int j, int k, const int64_t* st) {
  const double* x = P.xf + (int64_t)b * (g.nn[0] + g.nn[1] + g.nn[2]);
  const double x1 = x[i], x2 = x[g.nn[0] + j], x3 = x[g.nn[0] + g.nn[1] + k];
  double d[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) d[a] = fd_ds<GL>(f, st[a], P.dx[(int64_t)b * 3 + a]);
  const double r = sqrt(x1 * x1 + x2 * x2 + x3 * x3);
  const double s_u[3] = {x1 / r, x2 / r, x3 / r};
  const double sqrt2 = sqrt(2.);
  double v;
  if (n == Z4C_KHAT) {
    v = -sqrt2 * ld<GL>(f) / r;
#pragma unroll
    for (int a = 0; a < 3; ++a) v -= sqrt2 * s_u[a] * d[a];
  } else {
    v = -ld<GL>(f) / r;
#pragma unroll
    for (int a = 0; a < 3; ++a) v -= s_u[a] * d[a];
  }
  return v;
}

// Z4c::Z4cBoundaryRHS on its own: one thread per (block, interior vertex,
// Sommerfeld variable); rhs is overwritten where the vertex lies on a
// gr_sommerfeld face.
__global__ void __launch_bounds__(kPointThreads)
k_sommerfeld(Grid g, DevParams P, const double* __restrict__ u, double* __restrict__ rhs,
             int block0, int nblk) {
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1, per = n0 * n1 * (g.nx[2] + 1);
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= per * 11 * nblk) return;
  const int l = t % per, rest = t / per;
  const int v = rest % 11, b = block0 + rest / 11;
  const int n = (v < 2) ? (v == 0 ? Z4C_KHAT : Z4C_THETA) : Z4C_AXX + (v - 2);  // A, Gamma
  const int i = NG + l % n0, j = NG + (l / n0) % n1, k = NG + l / (n0 * n1);
  if (!on_sommerfeld_face(g, P, b, i, j, k)) return;
  const int64_t q = ((int64_t)b * NVAR + n) * g.nvol + ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  rhs[q] = sommerfeld_value(g, P, b, n, u + q, i, j, k, g.s);
}

// Advection sums (calculate_z4c_rhs.cpp:184-226): lv [block][22][interior vertex]
template <int UNROLL, int NX>
__global__ void __launch_bounds__(kColumnMaxThreads)
k_adv(Grid gin, DevParams P, const double* __restrict__ u, double* __restrict__ lv, int block0,
      int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  Column c;
  if (!column_index(g, block0, nblk, c)) return;
  const int nn0 = g.nn[0], sk = nn0 * g.nn[1];
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1;
  const int64_t npts = interior_count(g);
  const double* U = u + (int64_t)c.b * NVAR * g.nvol + c.j * nn0 + c.i;
  const double* f = U + (int64_t)c.n * g.nvol;
  const double* bx = U + (int64_t)Z4C_BETAX * g.nvol;
  const double* by = U + (int64_t)Z4C_BETAY * g.nvol;
  const double* bz = U + (int64_t)Z4C_BETAZ * g.nvol;
  double* out = lv + ((int64_t)c.b * NVAR + c.n) * npts + (c.j - NG) * n0 + (c.i - NG);
  const FdScale& F = P.fd[c.b];
  double w[9];
  window_init(f, sk, NG, w);
#pragma unroll UNROLL
  for (int k = NG; k <= NG + g.nx[2]; ++k) {
    window_advance(f, sk, k, w);
    const int o = k * sk;
    double acc = 0;
    acc += fd_lx_side(f + o, 1, __ldg(bx + o), F.lidx[0]);
    acc += fd_lx_side(f + o, nn0, __ldg(by + o), F.lidx[1]);
    acc += fd_lx_window(w, __ldg(bz + o), F.lidx[2]);
    out[(k - NG) * n0 * n1] = acc;
    window_shift(w);
  }
}

// Z4cRHS tail: rhs += KO, in place.
template <int UNROLL, int NX>
__global__ void __launch_bounds__(kColumnMaxThreads)
k_ko_rhs(Grid gin, DevParams P, const double* __restrict__ u, double* __restrict__ rhs,
         int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  Column c;
  if (!column_index(g, block0, nblk, c)) return;
  const int nn0 = g.nn[0], sk = nn0 * g.nn[1];
  const int64_t base = ((int64_t)c.b * NVAR + c.n) * g.nvol + c.j * nn0 + c.i;
  const double* f = u + base;
  const FdScale& F = P.fd[c.b];
  double w[9];
  window_init(f, sk, NG, w);
#pragma unroll UNROLL
  for (int k = NG; k <= NG + g.nx[2]; ++k) {
    window_advance(f, sk, k, w);
    const int o = k * sk;
    rhs[base + o] = add_ko_column(rhs[base + o], f + o, nn0, w, F, P.p.diss);
    window_shift(w);
  }
}

// ---- KO + low-storage RK stage ----------------------------------------------
// The right-hand side used is Z4cRHS (main pass + KO) followed by
// Z4cBoundaryRHS, as CALC_Z4CRHS runs them (task_list_gr_z4c.cpp:142-166).
// IntegrateZ4c for 2S integrators (task_list_gr_z4c.cpp:176-195):
//   WeightedAve(u1, u, u2, {1, delta, 0}); WeightedAve(u, u1, u2, {g1, g2, g3});
//   AddZ4cRHS(rhs, beta*dt, u)        (mesh/weighted_ave.cpp:20-150)
// u is read (all points, for the stencils); u_out, u1 are written (interior).
template <int UNROLL, bool SOM, int NX>
__global__ void __launch_bounds__(kColumnMaxThreads)
k_ko_stage_ls(Grid gin, DevParams P, const double* __restrict__ u,
              const double* __restrict__ rhs, double* __restrict__ u1,
              double* __restrict__ u_out, LsStage w, int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  Column c;
  if (!column_index(g, block0, nblk, c)) return;
  const int nn0 = g.nn[0], sk = nn0 * g.nn[1];
  const int64_t base = ((int64_t)c.b * NVAR + c.n) * g.nvol + c.j * nn0 + c.i;
  const double* f = u + base;
  const FdScale& F = P.fd[c.b];
  // Z4cBoundaryRHS replaces this variable's right-hand side on Sommerfeld faces
  const bool som = SOM && sommerfeld_var(c.n);
  double win[9];
  window_init(f, sk, NG, win);
#pragma unroll UNROLL
  for (int k = NG; k <= NG + g.nx[2]; ++k) {
    window_advance(f, sk, k, win);
    const int o = k * sk;
    const int64_t q = base + o;
    const double r = (som && on_sommerfeld_face(g, P, c.b, c.i, c.j, k))
                         ? sommerfeld_value(g, P, c.b, c.n, f + o, c.i, c.j, k, g.s)
                         : add_ko_column(__ldg(rhs + q), f + o, nn0, win, F, P.p.diss);
    double v1, v;
    ls_update(w, win[4], w.u1_zero ? 0.0 : u1[q], r, v1, v);
    u1[q] = v1;
    u_out[q] = v;
    window_shift(win);
  }
}

// ---- KO + Butcher stage (task_list_integrators_butcher.cpp:512-680) ---------
// k_s = RHS(u); u_out = u_n + sum_q coef_q k_q in the reference's order.
struct KPtrs {
  double* k[4];
};
template <int UNROLL, bool SOM, int NX>
__global__ void __launch_bounds__(kColumnMaxThreads)
k_ko_stage_bt(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ rhs,
              const double* __restrict__ un, KPtrs K, double* __restrict__ u_out, BtStage w,
              int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  Column c;
  if (!column_index(g, block0, nblk, c)) return;
  const int nn0 = g.nn[0], sk = nn0 * g.nn[1];
  const int64_t base = ((int64_t)c.b * NVAR + c.n) * g.nvol + c.j * nn0 + c.i;
  const double* f = u + base;
  const FdScale& F = P.fd[c.b];
  // Z4cBoundaryRHS replaces this variable's right-hand side on Sommerfeld faces
  const bool som = SOM && sommerfeld_var(c.n);
  double win[9];
  window_init(f, sk, NG, win);
#pragma unroll UNROLL
  for (int k = NG; k <= NG + g.nx[2]; ++k) {
    window_advance(f, sk, k, win);
    const int o = k * sk;
    const int64_t q = base + o;
    const double r = (som && on_sommerfeld_face(g, P, c.b, c.i, c.j, k))
                         ? sommerfeld_value(g, P, c.b, c.n, f + o, c.i, c.j, k, g.s)
                         : add_ko_column(__ldg(rhs + q), f + o, nn0, win, F, P.p.diss);
    K.k[w.kslot][q] = r;
    double v = __ldg(un + q);
    for (int s = 0; s < w.nq; ++s) {
      if (w.coef[s] != 0.0) {
        const double ks = (s == w.kslot) ? r : K.k[s][q];
        v += w.coef[s] * ks;
      }
    }
    u_out[q] = v;
    window_shift(win);
  }
}

// ---- slab passes: one CTA per (block, variable, z-slab) --------------------
// The per-variable passes read one variable's stencils only, so a CTA takes
// one (block, variable) pair and a slab of its interior planes kl..kh,
// copies the vertex planes kl-4..kh+4 (a contiguous range of the register)
// into shared memory with coalesced loads, and evaluates every stencil of
// the slab's interior vertices from there.  The arithmetic is that of the
// pencil kernels above, vertex by vertex.  Used when the planes fit in
// shared memory (16^3 blocks: 5 kB per plane).
struct SlabGeom {
  int kper;   // interior planes per slab
  int plane;  // vertices per plane, nn0*nn1
};
__device__ __forceinline__ void slab_range(const Grid& g, const SlabGeom& S, int& kl, int& kh) {
  kl = NG + (int)blockIdx.x * S.kper;
  kh = min(NG + g.nx[2], kl + S.kper - 1);
}
// Copies planes kl-4..kh+4 of the variable block f into sm with
// asynchronous global-to-shared copies (cp.async, 8 bytes each): every
// thread issues all of its copies before waiting, so the whole slab is in
// flight at once.
__device__ __forceinline__ void slab_load(double* __restrict__ sm, const double* __restrict__ f,
                                          int kl, int kh, int plane) {
  const double* src = f + (int64_t)(kl - NG) * plane;
  const int n = (kh - kl + 1 + 2 * NG) * plane;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sm + q);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src + q) : "memory");
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
}

// Advection sums, and for chi, g~, alpha, beta the stored first derivatives
// (the work of k_adv and k_prep on one variable).
__global__ void __launch_bounds__(kColumnMaxThreads)
k_adv_prep_slab(Grid g, DevParams P, const double* __restrict__ u, double* __restrict__ lv,
                double* __restrict__ sd, SlabGeom S, int block0) {
  extern __shared__ double sm[];
  const int n = (int)blockIdx.y, b = block0 + (int)blockIdx.z;
  int kl, kh;
  slab_range(g, S, kl, kh);
  if (kl > kh) return;
  const int nn0 = g.nn[0], pl = S.plane;
  const double* U = u + (int64_t)b * NVAR * g.nvol;
  slab_load(sm, U + (int64_t)n * g.nvol, kl, kh, pl);
  // vertex (i, j, k) of the block in shared memory
  const double* s0 = sm - (int64_t)(kl - NG) * pl;
  const FdScale& F = P.fd[b];
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1, nk = kh - kl + 1;
  const int64_t npts = interior_count(g);
  double* out = lv + ((int64_t)b * NVAR + n) * npts;
  for (int q = threadIdx.x; q < n0 * n1 * nk; q += blockDim.x) {
    const int i = NG + q % n0, j = NG + (q / n0) % n1, k = kl + q / (n0 * n1);
    const int o = k * pl + j * nn0 + i;
    double acc = 0;
    acc += fd_lx_side<false>(s0 + o, 1, __ldg(U + (int64_t)Z4C_BETAX * g.nvol + o), F.lidx[0]);
    acc += fd_lx_side<false>(s0 + o, nn0, __ldg(U + (int64_t)Z4C_BETAY * g.nvol + o), F.lidx[1]);
    acc += fd_lx_side<false>(s0 + o, pl, __ldg(U + (int64_t)Z4C_BETAZ * g.nvol + o), F.lidx[2]);
    out[((k - NG) * n1 + (j - NG)) * n0 + (i - NG)] = acc;
  }
  // stored first derivatives (k_prep's regions): D_x on the interior, D_y
  // extended by 3 along x, D_z extended by 3 along x and y
  int slot = -1;
#pragma unroll
  for (int q = 0; q < kSdFields; ++q)
    if (sd_field_var(q) == n) slot = q;
  if (slot < 0) return;
  double* sdb = sd + ((int64_t)b * kSdComponents + slot * 3) * g.nvol;
  for (int dir = 0; dir < 3; ++dir) {
    const int ex = (dir >= 1) ? 3 : 0, ey = (dir == 2) ? 3 : 0;
    const int e0 = n0 + 2 * ex, e1 = n1 + 2 * ey;
    const int st = (dir == 0) ? 1 : (dir == 1 ? nn0 : pl);
    const double c1 = F.cidx1[dir];
    double* o_dir = sdb + (int64_t)dir * g.nvol;
    for (int q = threadIdx.x; q < e0 * e1 * nk; q += blockDim.x) {
      const int i = NG - ex + q % e0, j = NG - ey + (q / e0) % e1, k = kl + q / (e0 * e1);
      const int o = k * pl + j * nn0 + i;
      const double* v = s0 + o;
      o_dir[o] = fd_dx7(v[-3 * st], v[-2 * st], v[-st], v[st], v[2 * st], v[3 * st], c1);
    }
  }
}

// Kreiss-Oliger from shared memory, rhs += Diss_x; += Diss_y; += Diss_z.
__device__ __forceinline__ double add_ko_slab(double r, const double* v, int nn0, int pl,
                                              const FdScale& F, double diss) {
  r += fd_diss_line<false>(v, 1, F.cidxd[0], diss);
  r += fd_diss_line<false>(v, nn0, F.cidxd[1], diss);
  r += fd_diss_line<false>(v, pl, F.cidxd[2], diss);
  return r;
}

// KO + low-storage stage (k_ko_stage_ls) with Z4cBoundaryRHS on
// Sommerfeld faces, from a shared-memory slab.
template <bool SOM>
__global__ void __launch_bounds__(kColumnMaxThreads)
k_ko_stage_ls_slab(Grid g, DevParams P, const double* __restrict__ u,
                   const double* __restrict__ rhs, double* __restrict__ u1,
                   double* __restrict__ u_out, LsStage w, SlabGeom S, int block0) {
  extern __shared__ double sm[];
  const int n = (int)blockIdx.y, b = block0 + (int)blockIdx.z;
  int kl, kh;
  slab_range(g, S, kl, kh);
  if (kl > kh) return;
  const int nn0 = g.nn[0], pl = S.plane;
  const int64_t base = ((int64_t)b * NVAR + n) * g.nvol;
  slab_load(sm, u + base, kl, kh, pl);
  const double* s0 = sm - (int64_t)(kl - NG) * pl;
  const FdScale& F = P.fd[b];
  const bool som = SOM && sommerfeld_var(n);
  const int64_t sst[3] = {1, nn0, pl};
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1, nk = kh - kl + 1;
  for (int q = threadIdx.x; q < n0 * n1 * nk; q += blockDim.x) {
    const int i = NG + q % n0, j = NG + (q / n0) % n1, k = kl + q / (n0 * n1);
    const int o = k * pl + j * nn0 + i;
    const int64_t qq = base + o;
    const double* v = s0 + o;
    const double r = (som && on_sommerfeld_face(g, P, b, i, j, k))
                         ? sommerfeld_value<false>(g, P, b, n, v, i, j, k, sst)
                         : add_ko_slab(__ldg(rhs + qq), v, nn0, pl, F, P.p.diss);
    double v1, x;
    ls_update(w, *v, w.u1_zero ? 0.0 : u1[qq], r, v1, x);
    u1[qq] = v1;
    u_out[qq] = x;
  }
}

// KO + Butcher stage (k_ko_stage_bt) from a shared-memory slab.
template <bool SOM>
__global__ void __launch_bounds__(kColumnMaxThreads)
k_ko_stage_bt_slab(Grid g, DevParams P, const double* __restrict__ u,
                   const double* __restrict__ rhs, const double* __restrict__ un_reg, KPtrs K,
                   double* __restrict__ u_out, BtStage w, SlabGeom S, int block0) {
  extern __shared__ double sm[];
  const int n = (int)blockIdx.y, b = block0 + (int)blockIdx.z;
  int kl, kh;
  slab_range(g, S, kl, kh);
  if (kl > kh) return;
  const int nn0 = g.nn[0], pl = S.plane;
  const int64_t base = ((int64_t)b * NVAR + n) * g.nvol;
  slab_load(sm, u + base, kl, kh, pl);
  const double* s0 = sm - (int64_t)(kl - NG) * pl;
  const FdScale& F = P.fd[b];
  const bool som = SOM && sommerfeld_var(n);
  const int64_t sst[3] = {1, nn0, pl};
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1, nk = kh - kl + 1;
  for (int q = threadIdx.x; q < n0 * n1 * nk; q += blockDim.x) {
    const int i = NG + q % n0, j = NG + (q / n0) % n1, k = kl + q / (n0 * n1);
    const int o = k * pl + j * nn0 + i;
    const int64_t qq = base + o;
    const double* v = s0 + o;
    const double r = (som && on_sommerfeld_face(g, P, b, i, j, k))
                         ? sommerfeld_value<false>(g, P, b, n, v, i, j, k, sst)
                         : add_ko_slab(__ldg(rhs + qq), v, nn0, pl, F, P.p.diss);
    K.k[w.kslot][qq] = r;
    double x = __ldg(un_reg + qq);
    for (int sidx_ = 0; sidx_ < w.nq; ++sidx_) {
      if (w.coef[sidx_] != 0.0) {
        const double ks = (sidx_ == w.kslot) ? r : K.k[sidx_][qq];
        x += w.coef[sidx_] * ks;
      }
    }
    u_out[qq] = x;
  }
}

// Z4cRHS tail (k_ko_rhs) from a shared-memory slab: rhs += KO, in place.
__global__ void __launch_bounds__(kColumnMaxThreads)
k_ko_rhs_slab(Grid g, DevParams P, const double* __restrict__ u, double* __restrict__ rhs,
              SlabGeom S, int block0) {
  extern __shared__ double sm[];
  const int n = (int)blockIdx.y, b = block0 + (int)blockIdx.z;
  int kl, kh;
  slab_range(g, S, kl, kh);
  if (kl > kh) return;
  const int nn0 = g.nn[0], pl = S.plane;
  const int64_t base = ((int64_t)b * NVAR + n) * g.nvol;
  slab_load(sm, u + base, kl, kh, pl);
  const double* s0 = sm - (int64_t)(kl - NG) * pl;
  const FdScale& F = P.fd[b];
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1, nk = kh - kl + 1;
  for (int q = threadIdx.x; q < n0 * n1 * nk; q += blockDim.x) {
    const int i = NG + q % n0, j = NG + (q / n0) % n1, k = kl + q / (n0 * n1);
    const int o = k * pl + j * nn0 + i;
    rhs[base + o] = add_ko_slab(rhs[base + o], s0 + o, nn0, pl, F, P.p.diss);
  }
}

// ---- main pass: the right-hand side without the Kreiss-Oliger terms -------
template <int THREADS, int NX, int MINB = 1>
__global__ void __launch_bounds__(THREADS, MINB)
k_main(Grid gin, DevParams P, const double* __restrict__ u, const double* __restrict__ sd,
       const double* __restrict__ rsum, const double* __restrict__ lv, double* __restrict__ rhs,
       int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = interior_count(g);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * nblk) return;
  const int b = block0 + (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_ijk(g, l, i, j, k);
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  double out[NVAR];
  rhs_point(u + (int64_t)b * NVAR * g.nvol, sd + (int64_t)b * kSdComponents * g.nvol, g.nvol, p,
            g.s, P, P.fd[b], rsum + (int64_t)b * 6 * npts + l, lv + (int64_t)b * NVAR * npts + l,
            npts, out);
  double* rb = rhs + (int64_t)b * NVAR * g.nvol + p;
#pragma unroll
  for (int n = 0; n < NVAR; ++n) rb[(int64_t)n * g.nvol] = out[n];
}

// ---- puncture tracker (z4c/puncture_tracker.cpp) ----------------------------
// Tracker record: pos[3], betap[3], lost flag, padding (8 doubles).
// LagrangeInterp1D<2*NGHOST-1> (utils/lagrange_interp.hpp:33-146): first
// stencil point and the 8 coefficients, in the reference's operation order.
constexpr int kTrkOrder = 2 * NG - 1;
__device__ int trk_lagrange1d(double origin, double delta, int siz, double coord,
                              double coeff[kTrkOrder + 1]) {
  const double delta_inv = 1.0 / delta;
  int point = __double2int_rn(floor((coord - origin) * delta_inv - 0.5 * (kTrkOrder - 1)));
  int shift = point;
  if (shift < 0) point -= shift;
  shift = point + kTrkOrder - (siz - 1);
  if (shift > 0) point -= shift;
  double xp[kTrkOrder + 1];
  for (int i = 0; i <= kTrkOrder; ++i) xp[i] = (point + i) * delta + origin;
  for (int j = 0; j <= kTrkOrder; ++j) {
    double num = 1.0, den = 1.0;
    for (int i = 0; i <= kTrkOrder; ++i) {
      if (i == j) continue;
      num = num * (coord - xp[i]);
      den = den * (xp[j] - xp[i]);
    }
    coeff[j] = num / den;
  }
  return point;
}

// PunctureTracker::InterpolateShift (:95-129): one thread per tracker finds
// the block that holds the puncture exclusively (MeshBlock::
// PointContainedExclusive, mesh/meshblock.cpp:1186-1201) and interpolates
// the shift there (LagrangeInterpND: x innermost, then y, then z).
__global__ void k_track_interp(Grid g, DevParams P, const double* __restrict__ u,
                               double* __restrict__ trk, int ntrk) {
  const int t = (int)threadIdx.x;
  if (t >= ntrk) return;
  double* T = trk + 8 * t;
  const double pos[3] = {T[0], T[1], T[2]};
  const int nsum = g.nn[0] + g.nn[1] + g.nn[2];
  int owner = -1;
  for (int b = 0; b < g.nblocks && owner < 0; ++b) {
    const double* x = P.xf + (int64_t)b * nsum;
    bool in = true;
    int off = 0;
    for (int a = 0; a < 3; ++a) {
      in = in && (x[off + NG] <= pos[a]) && (pos[a] < x[off + NG + g.nx[a]]);
      off += g.nn[a];
    }
    if (in) owner = b;
  }
  if (owner < 0) {  // the puncture has left the grid
    T[6] = 1.0;
    return;
  }
  const double* x = P.xf + (int64_t)owner * nsum;
  double c[3][kTrkOrder + 1];
  int pt[3], off = 0;
  for (int a = 0; a < 3; ++a) {
    pt[a] = trk_lagrange1d(x[off], P.dx[(int64_t)owner * 3 + a], g.nn[a], pos[a], c[a]);
    off += g.nn[a];
  }
  for (int v = 0; v < 3; ++v) {
    const double* f = u + ((int64_t)owner * NVAR + Z4C_BETAX + v) * g.nvol;
    double vz[kTrkOrder + 1];
    for (int ez = 0; ez <= kTrkOrder; ++ez) {
      double vy[kTrkOrder + 1];
      for (int ey = 0; ey <= kTrkOrder; ++ey) {
        const double* row = f + ((int64_t)(pt[2] + ez) * g.nn[1] + (pt[1] + ey)) * g.nn[0] + pt[0];
        double o = 0;
        for (int i = 0; i <= kTrkOrder; ++i) o += c[0][i] * row[i];
        vy[ey] = o;
      }
      double o = 0;
      for (int i = 0; i <= kTrkOrder; ++i) o += c[1][i] * vy[i];
      vz[ez] = o;
    }
    double o = 0;
    for (int i = 0; i <= kTrkOrder; ++i) o += c[2][i] * vz[i];
    T[3 + v] = o;
  }
}

// PunctureTracker::EvolveTracker (:132-186): pos -= dt * betap.
__global__ void k_track_update(double* __restrict__ trk, int ntrk, double dt) {
  const int t = (int)threadIdx.x;
  if (t >= ntrk) return;
  double* T = trk + 8 * t;
  for (int a = 0; a < 3; ++a) T[a] -= dt * T[3 + a];
}

// ---- same-level vertex-centred ghost exchange -------------------------------
// CommRegistry::SetBoundaries (comm/comm_registry.cpp:336-382): ghosts are
// zeroed, every neighbour whose set range (comm/index_utilities.hpp:155-163)
// holds the vertex adds its value in neighbour-list order
// (mesh/mesh_topology.cpp:329-960), and the sum is multiplied by
// 1/multiplicity (comm/node_multiplicity.cpp:396-430).  Strictly interior
// vertices keep their value.
//
// Per axis a vertex is a ghost (below vs or above ve: owned by the neighbour
// on that side only), on a shared plane (vs or ve: owned by this block and
// the neighbour on that side) or inside.  The owners of a vertex are the
// directions whose support U contains every ghost axis and otherwise only
// shared axes; U = {} is the block itself.  The neighbour list orders
// directions by the size of their support and then by the support's axis
// set as a bit mask (x=1, y=2, z=4): faces x, y, z, then edges xy, xz, yz,
// then the corner.  u_order walks the supports in that order.
//
// Two passes.  k_exchange_interior forms every block's own vertices
// [vs, ve]^3 from the owners' pre-exchange copies (src).  For a ghost
// vertex, the owners seen from this block are the ones seen from its
// primary owner (the neighbour across the ghost axes only) plus the ghost
// axes, in the same order, so the reference's sum for the ghost equals the
// primary owner's result for that vertex: k_exchange_ghosts copies it from
// there.  With fuse_alg the AlgConstr pass that follows in the task list is
// applied to the interior results, and the ghosts copy those.
// Whether block b (context order) touches a physical (non-periodic) face.
// Every vertex a boundary condition reads or writes belongs to such a block:
// the extrapolation reads the block's own vertices near the face and its
// ghosts across the faces transverse to it, whose owners sit at the same
// position along the face normal and so touch the same face.
__device__ __forceinline__ bool touches_physical_face(const Grid& g, int b) {
  const int l[3] = {b % g.nb[0], (b / g.nb[0]) % g.nb[1], b / (g.nb[0] * g.nb[1])};
  bool t = false;
#pragma unroll
  for (int a = 0; a < 3; ++a)
    t |= (l[a] == 0 && g.bc[2 * a] != Z4C_BC_PERIODIC) ||
         (l[a] == g.nb[a] - 1 && g.bc[2 * a + 1] != Z4C_BC_PERIODIC);
  return t;
}
// AlgConstr in the exchange: kAlgNone, kAlgAll (no physical faces: every
// vertex constrained in the exchange), kAlgInner (the blocks that touch no
// physical face constrained in the exchange, the others by
// k_alg_constr_boundary after their boundary conditions).
constexpr int kAlgNone = 0, kAlgAll = 1, kAlgInner = 2;

__constant__ int c_dir_index[27];  // (o0+1) + 3(o1+1) + 9(o2+1) -> neighbour slot
// supports in list order: 0, 1, 2, 4, 3, 5, 6, 7
__device__ __forceinline__ constexpr int u_order(int q) { return (q == 3) ? 4 : (q == 4) ? 3 : q; }

template <int NV, int NX>
__global__ void __launch_bounds__(kPointThreads)
k_exchange_interior(Grid gin, DevParams P, const double* __restrict__ src,
                    double* __restrict__ dst, const int* __restrict__ nbr, int fuse_alg) {
  const Grid g = fixed_geometry<NX>(gin);
  const int n0 = g.nx[0] + 1, n1 = g.nx[1] + 1, n2 = g.nx[2] + 1;
  const int per = n0 * n1 * n2;
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= per * g.nblocks) return;
  const int b = t / per, l = t % per;
  const int idx[3] = {NG + l % n0, NG + (l / n0) % n1, NG + l / (n0 * n1)};
  const int p = (idx[2] * g.nn[1] + idx[1]) * g.nn[0] + idx[0];
  int smask = 0, side[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int vs = NG, ve = NG + g.nx[a], x = idx[a];
    side[a] = (x == vs) ? -1 : 1;
    if (x == vs || x == ve) smask |= 1 << a;
  }
  const int64_t bstride = (int64_t)NV * g.nvol;
  // source offset of every owner in list order (-1: not an owner)
  int64_t off[8];
  int mult = 1;
  off[0] = (int64_t)b * bstride + p;
#pragma unroll
  for (int q = 1; q < 8; ++q) {
    const int U = u_order(q);
    off[q] = -1;
    if (smask == 0 || (U & ~smask) != 0) continue;
    int o[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) o[a] = (U >> a & 1) ? side[a] : 0;
    const int nb = __ldg(nbr + b * 26 + c_dir_index[(o[0] + 1) + 3 * (o[1] + 1) + 9 * (o[2] + 1)]);
    if (nb < 0) continue;
    off[q] = (int64_t)nb * bstride + p -
             (((int64_t)o[2] * g.nx[2] * g.nn[1] + (int64_t)o[1] * g.nx[1]) * g.nn[0] +
              (int64_t)o[0] * g.nx[0]);
    ++mult;
  }
  const double inv = (mult > 1) ? 1.0 / (double)mult : 1.0;
  double v[NV];
#pragma unroll
  for (int n = 0; n < NV; ++n) v[n] = __ldg(src + off[0] + (int64_t)n * g.nvol);
  if (mult > 1) {
#pragma unroll
    for (int n = 0; n < NV; ++n) {
      const int64_t vo = (int64_t)n * g.nvol;
      double s = v[n];
#pragma unroll
      for (int q = 1; q < 8; ++q)
        if (off[q] >= 0) s += __ldg(src + off[q] + vo);
      v[n] = s * inv;
    }
  }
  if constexpr (NV == NVAR) {
    if (fuse_alg == kAlgAll || (fuse_alg == kAlgInner && !touches_physical_face(g, b))) {
    double gg[6], AA[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      gg[c] = v[Z4C_GXX + c];
      AA[c] = v[Z4C_AXX + c];
    }
    alg_constr_point(P.p, gg, AA, &v[Z4C_CHI], &v[Z4C_ALPHA]);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      v[Z4C_GXX + c] = gg[c];
      v[Z4C_AXX + c] = AA[c];
    }
    }
  }
  double* db = dst + off[0];
#pragma unroll
  for (int n = 0; n < NV; ++n) db[(int64_t)n * g.nvol] = v[n];
}

// Ghost vertices: copy of the primary owner's result (zero where the primary
// owner lies beyond a physical face; the boundary conditions overwrite those).
template <int NV, int NX>
__global__ void __launch_bounds__(kPointThreads)
k_exchange_ghosts(Grid gin, DevParams P, double* __restrict__ u, const int* __restrict__ nbr,
                  int fuse_alg) {
  const Grid g = fixed_geometry<NX>(gin);
  const int per = (int)g.nvol;
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= per * g.nblocks) return;
  const int b = t / per, p = t % per;
  const int idx[3] = {p % g.nn[0], (p / g.nn[0]) % g.nn[1], p / (g.nn[0] * g.nn[1])};
  int o[3];
  bool ghost = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    o[a] = (idx[a] < NG) ? -1 : (idx[a] > NG + g.nx[a] ? 1 : 0);
    ghost |= (o[a] != 0);
  }
  if (!ghost) return;
  const int64_t bstride = (int64_t)NV * g.nvol;
  double* db = u + (int64_t)b * bstride + p;
  const int nb = __ldg(nbr + b * 26 + c_dir_index[(o[0] + 1) + 3 * (o[1] + 1) + 9 * (o[2] + 1)]);
  if (nb < 0) {
#pragma unroll
    for (int n = 0; n < NV; ++n) db[(int64_t)n * g.nvol] = 0.0;
    return;
  }
  const double* sb = u + (int64_t)nb * bstride + p -
                     (((int64_t)o[2] * g.nx[2] * g.nn[1] + (int64_t)o[1] * g.nx[1]) * g.nn[0] +
                      (int64_t)o[0] * g.nx[0]);
  double v[NV];
#pragma unroll
  for (int n = 0; n < NV; ++n) v[n] = sb[(int64_t)n * g.nvol];
  if constexpr (NV == NVAR) {
    // a block constrained in the exchange receives from an owner constrained
    // only after its boundary conditions: constrain the copy
    if (fuse_alg == kAlgInner && !touches_physical_face(g, b) && touches_physical_face(g, nb)) {
      double gg[6], AA[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        gg[c] = v[Z4C_GXX + c];
        AA[c] = v[Z4C_AXX + c];
      }
      alg_constr_point(P.p, gg, AA, &v[Z4C_CHI], &v[Z4C_ALPHA]);
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        v[Z4C_GXX + c] = gg[c];
        v[Z4C_AXX + c] = AA[c];
      }
    }
  }
#pragma unroll
  for (int n = 0; n < NV; ++n) db[(int64_t)n * g.nvol] = v[n];
}

// AlgConstr after the boundary conditions on the blocks that touch a physical
// face, except their ghosts copied from blocks constrained in the exchange
// (those copies already carry the constrained value).
template <int NX>
__global__ void __launch_bounds__(kPointThreads)
k_alg_constr_boundary(Grid gin, DevParams P, double* __restrict__ u, const int* __restrict__ nbr) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nvol * g.nblocks) return;
  const int b = (int)(t / g.nvol);
  if (!touches_physical_face(g, b)) return;
  const int p = (int)(t % g.nvol);
  const int idx[3] = {p % g.nn[0], (p / g.nn[0]) % g.nn[1], p / (g.nn[0] * g.nn[1])};
  int o[3];
  bool ghost = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    o[a] = (idx[a] < NG) ? -1 : (idx[a] > NG + g.nx[a] ? 1 : 0);
    ghost |= (o[a] != 0);
  }
  if (ghost) {
    const int nb = __ldg(nbr + b * 26 + c_dir_index[(o[0] + 1) + 3 * (o[1] + 1) + 9 * (o[2] + 1)]);
    if (nb >= 0 && !touches_physical_face(g, nb)) return;
  }
  double* ub = u + (int64_t)b * NVAR * g.nvol + p;
  double gg[6], AA[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    gg[c] = ub[(int64_t)(Z4C_GXX + c) * g.nvol];
    AA[c] = ub[(int64_t)(Z4C_AXX + c) * g.nvol];
  }
  double chi = ub[(int64_t)Z4C_CHI * g.nvol], alpha = ub[(int64_t)Z4C_ALPHA * g.nvol];
  alg_constr_point(P.p, gg, AA, &chi, &alpha);
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    ub[(int64_t)(Z4C_GXX + c) * g.nvol] = gg[c];
    ub[(int64_t)(Z4C_AXX + c) * g.nvol] = AA[c];
  }
  if (P.p.force_regularization) {
    ub[(int64_t)Z4C_CHI * g.nvol] = chi;
    ub[(int64_t)Z4C_ALPHA * g.nvol] = alpha;
  }
}

// ---- extrapolate_outflow boundary conditions --------------------------------
// ExtrapolateOutflowBC with NEXTRAPOLATE = 5 (comm/physical_bcs.cpp:187-260),
// also the ghost fill of gr_sommerfeld faces for vertex-centred data (:445-453)
// over the ranges of ApplyPhysicalBCs (:506-670): the cell-centred interior
// end ie = is + nx - 1 bounds the outer faces and the transverse ranges.
// Only the blocks on the two faces of axis ax are visited.  One thread per
// (face block, variable, side, transverse pair) cascades outward; the
// fastest thread index runs along the transverse axis of smallest stride.
template <int NX, int AX>
__global__ void __launch_bounds__(kPointThreads)
k_bc_axis(Grid gin, double* __restrict__ u, int nvar) {
  const Grid g = fixed_geometry<NX>(gin);
  constexpr int ax = AX;                  // one instance per axis: static indexing
  constexpr int o1 = (ax == 0) ? 1 : 0;   // fastest transverse axis
  constexpr int o2 = (ax == 2) ? 1 : 2;   // slowest transverse axis
  const int64_t nt = (int64_t)g.nn[o1] * g.nn[o2];
  const int nfb = g.nb[o1] * g.nb[o2];    // blocks on one face
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt * 2 * nvar * nfb) return;
  const int64_t tr = t % nt;
  int64_t r = t / nt;
  const int side = (int)(r % 2);
  r /= 2;
  const int n = (int)(r % nvar);
  const int fb = (int)(r / nvar);
  int loc[3];
  loc[ax] = side ? g.nb[ax] - 1 : 0;
  loc[o1] = fb % g.nb[o1];
  loc[o2] = fb / g.nb[o1];
  if (g.bc[2 * ax + side] == Z4C_BC_PERIODIC) return;
  const int b = loc[0] + g.nb[0] * (loc[1] + g.nb[1] * loc[2]);
  bool need[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    need[2 * a] = (g.bc[2 * a] != Z4C_BC_PERIODIC) && loc[a] == 0;
    need[2 * a + 1] = (g.bc[2 * a + 1] != Z4C_BC_PERIODIC) && loc[a] == g.nb[a] - 1;
  }
  int is[3], ie[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    is[a] = NG;
    ie[a] = NG + g.nx[a] - 1;
  }
  int lo[3], hi[3];
  // transverse limits, physical_bcs.cpp:516-528, x3 faces :619-621
  lo[0] = is[0] - NG; hi[0] = ie[0] + NG;
  lo[1] = need[2] ? is[1] : is[1] - NG;
  hi[1] = need[3] ? ie[1] : ie[1] + NG;
  lo[2] = need[4] ? is[2] : is[2] - NG;
  hi[2] = need[5] ? ie[2] : ie[2] + NG;
  if (ax == 2) { lo[1] = is[1] - NG; hi[1] = ie[1] + NG; }
  const int t1 = (int)(tr % g.nn[o1]), t2 = (int)(tr / g.nn[o1]);
  if (t1 < lo[o1] || t1 > hi[o1] || t2 < lo[o2] || t2 > hi[o2]) return;
  double* ub = u + ((int64_t)b * nvar + n) * g.nvol + (int64_t)t1 * g.s[o1] + (int64_t)t2 * g.s[o2];
  const int64_t st = g.s[ax];
  // w[q] = the value q + 1 vertices inward of the ghost being filled; each
  // new ghost enters the window, so the cascade stays in registers
  const int dir = side ? -1 : 1;
  const int ia0 = side ? ie[ax] + 1 : is[ax] - 1;
  double w[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) w[q] = ub[(int64_t)(ia0 + dir * (q + 1)) * st];
#pragma unroll
  for (int gh = 1; gh <= NG; ++gh) {
    const int ia = side ? ie[ax] + gh : is[ax] - gh;
    double v = 0.0;  // coefficients 5, -10, 10, -5, 1 (NEXTRAPOLATE = 5)
    v += 5. * w[0];
    v += -10. * w[1];
    v += 10. * w[2];
    v += -5. * w[3];
    v += 1. * w[4];
    ub[(int64_t)ia * st] = v;
#pragma unroll
    for (int q = 4; q > 0; --q) w[q] = w[q - 1];
    w[0] = v;
  }
}

// ---- AlgConstr over all points (z4c.cpp:677-799) ----------------------------
// ghosts_only skips the interior vertices (ranged variant with
// skip_physical, z4c.cpp:801-991).
__device__ __forceinline__ bool is_interior_vertex(const Grid& g, int64_t p) {
  const int i = (int)(p % g.nn[0]);
  const int j = (int)((p / g.nn[0]) % g.nn[1]);
  const int k = (int)(p / ((int64_t)g.nn[0] * g.nn[1]));
  return i >= NG && i <= NG + g.nx[0] && j >= NG && j <= NG + g.nx[1] && k >= NG &&
         k <= NG + g.nx[2];
}

template <int NX>
__global__ void __launch_bounds__(kPointThreads)
k_alg_constr(Grid gin, DevParams P, double* __restrict__ u, int block0, int nblk,
             int ghosts_only) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nvol * nblk) return;
  const int b = block0 + (int)(t / g.nvol);
  if (ghosts_only && is_interior_vertex(g, t % g.nvol)) return;
  double* ub = u + (int64_t)b * NVAR * g.nvol + t % g.nvol;
  double gg[6], AA[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    gg[c] = ub[(int64_t)(Z4C_GXX + c) * g.nvol];
    AA[c] = ub[(int64_t)(Z4C_AXX + c) * g.nvol];
  }
  double chi = ub[(int64_t)Z4C_CHI * g.nvol], alpha = ub[(int64_t)Z4C_ALPHA * g.nvol];
  alg_constr_point(P.p, gg, AA, &chi, &alpha);
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    ub[(int64_t)(Z4C_GXX + c) * g.nvol] = gg[c];
    ub[(int64_t)(Z4C_AXX + c) * g.nvol] = AA[c];
  }
  if (P.p.force_regularization) {
    ub[(int64_t)Z4C_CHI * g.nvol] = chi;
    ub[(int64_t)Z4C_ALPHA * g.nvol] = alpha;
  }
}

// ---- WeightedAve / AddZ4cRHS on the interior (weighted_ave.cpp:20-167) --------
__global__ void k_weighted_ave(Grid g, double* __restrict__ out, const double* __restrict__ in1,
                               const double* __restrict__ in2, double w0, double w1, double w2,
                               int block0, int nblk) {
  const int64_t npts = interior_count(g);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * nblk * NVAR) return;
  const int n = (int)(t % NVAR);
  const int64_t r = t / NVAR;
  const int b = block0 + (int)(r / npts);
  int i, j, k;
  interior_ijk(g, r % npts, i, j, k);
  const int64_t q = ((int64_t)b * NVAR + n) * g.nvol + ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  if (w0 == 1.0) {
    if (w2 != 0.0) out[q] += w1 * in1[q] + w2 * in2[q];
    else if (w1 != 0.0) out[q] += w1 * in1[q];
  } else if (w0 == 0.0) {
    if (w2 != 0.0) out[q] = w1 * in1[q] + w2 * in2[q];
    else if (w1 == 1.0) out[q] = in1[q];
    else out[q] = w1 * in1[q];
  } else {
    if (w2 != 0.0) out[q] = w0 * out[q] + w1 * in1[q] + w2 * in2[q];
    else if (w1 != 0.0) out[q] = w0 * out[q] + w1 * in1[q];
    else out[q] *= w0;
  }
}

__global__ void k_add_rhs(Grid g, const double* __restrict__ rhs, double wght,
                          double* __restrict__ out, int block0, int nblk) {
  const int64_t npts = interior_count(g);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * nblk * NVAR) return;
  const int n = (int)(t % NVAR);
  const int64_t r = t / NVAR;
  const int b = block0 + (int)(r / npts);
  int i, j, k;
  interior_ijk(g, r % npts, i, j, k);
  const int64_t q = ((int64_t)b * NVAR + n) * g.nvol + ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  out[q] += wght * rhs[q];
}

// ---- ADM maps ----------------------------------------------------------------
__global__ void k_z4c_to_adm(Grid g, DevParams P, const double* __restrict__ u,
                             double* __restrict__ adm, int block0, int nblk, int ghosts_only) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nvol * nblk) return;
  const int b = block0 + (int)(t / g.nvol);
  const int64_t p = t % g.nvol;
  if (ghosts_only && is_interior_vertex(g, p)) return;
  z4c_to_adm_point(P.p, u + (int64_t)b * NVAR * g.nvol + p,
                   adm + (int64_t)b * Z4C_NADM * g.nvol + p, g.nvol);
}

__global__ void k_adm_to_z4c_pt(Grid g, DevParams P, const double* __restrict__ adm,
                                double* __restrict__ u, double* __restrict__ guu, int block0,
                                int nblk) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nvol * nblk) return;
  const int b = block0 + (int)(t / g.nvol);
  const int64_t p = t % g.nvol;
  adm_to_z4c_point(P.p, adm + (int64_t)b * Z4C_NADM * g.nvol + p,
                   u + (int64_t)b * NVAR * g.nvol + p, guu + (int64_t)b * 6 * g.nvol + p,
                   g.nvol);
}

// Gamma^a = -sum_b Dx(b, g~^{ba}) on the interior, zero elsewhere (:165-176).
__global__ void k_adm_to_z4c_gam(Grid g, DevParams P, const double* __restrict__ guu,
                                 double* __restrict__ u, int block0, int nblk) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nvol * nblk) return;
  const int b = block0 + (int)(t / g.nvol);
  const int64_t p = t % g.nvol;
  const int i = (int)(p % g.nn[0]);
  const int j = (int)((p / g.nn[0]) % g.nn[1]);
  const int k = (int)(p / ((int64_t)g.nn[0] * g.nn[1]));
  const bool in = i >= NG && i <= NG + g.nx[0] && j >= NG && j <= NG + g.nx[1] && k >= NG &&
                  k <= NG + g.nx[2];
  const double* gb = guu + (int64_t)b * 6 * g.nvol + p;
  double* ub = u + (int64_t)b * NVAR * g.nvol + p;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double v = 0.0;
    if (in) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
        v -= fd_dx(gb + (int64_t)sidx(c, a) * g.nvol, g.s[c], P.fd[b].cidx1[c]);
    }
    ub[(int64_t)(Z4C_GAMX + a) * g.nvol] = v;
  }
}

template <int NX>
__global__ void __launch_bounds__(128, 1)
k_adm_constraints(Grid gin, DevParams P, const double* __restrict__ adm,
                  const double* __restrict__ u, double* __restrict__ con,
                  const double* __restrict__ xf, int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nvol * nblk) return;
  const int b = block0 + (int)(t / g.nvol);
  const int64_t p = t % g.nvol;
  const int i = (int)(p % g.nn[0]);
  const int j = (int)((p / g.nn[0]) % g.nn[1]);
  const int k = (int)(p / ((int64_t)g.nn[0] * g.nn[1]));
  double* cb = con + (int64_t)b * Z4C_NCON * g.nvol + p;
  const bool in = i >= NG && i <= NG + g.nx[0] && j >= NG && j <= NG + g.nx[1] && k >= NG &&
                  k <= NG + g.nx[2];
  double c7[7] = {0, 0, 0, 0, 0, 0, 0};
  if (in) {
    const double* x = xf + (int64_t)b * (g.nn[0] + g.nn[1] + g.nn[2]);
    adm_constraints_point(u + (int64_t)b * NVAR * g.nvol, adm + (int64_t)b * Z4C_NADM * g.nvol,
                          g.nvol, p, g.s, P, P.fd[b], x[i], x[g.nn[0] + j],
                          x[g.nn[0] + g.nn[1] + k], c7);
  }
#pragma unroll
  for (int q = 0; q < 7; ++q) cb[(int64_t)q * g.nvol] = c7[q];
}

// ---- Weyl scalar psi4 (z4c/calculate_weyl_scalars.cpp:44-630) --------------
// One thread per vertex of the requested blocks; interior vertices get psi4,
// every other vertex NaN (the reference fills the register with NaN first).
// In three passes over the interior vertices: the Ricci tensor and its trace
// (k_weyl_curv<NX, 0>: Rd into rs [block][6][interior vertex], R into ks
// [block][22][...] slot 19), K and its covariant derivative (k_weyl_curv<NX,
// 1>: DK into ks slots 0-17, K into slot 18), then the tetrad and the
// contractions per vertex (k_weyl_psi), NaN outside the interior.  The
// single pass spilled; each part holds about half its state.
template <int NX, int PART>
__global__ void __launch_bounds__(128, 1)
k_weyl_curv(Grid gin, DevParams P, const double* __restrict__ adm, const double* __restrict__ u,
            const double* __restrict__ sd, double* __restrict__ rs, double* __restrict__ ks,
            int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t npts = interior_count(g);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * nblk) return;
  const int b = block0 + (int)(t / npts);
  const int64_t l = t % npts;
  int i, j, k;
  interior_ijk(g, l, i, j, k);
  const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
  double Rd[6], R, K, DK[3][6];
  weyl_curvature<PART == 0, PART == 1>(u + (int64_t)b * NVAR * g.nvol,
                                       adm + (int64_t)b * Z4C_NADM * g.nvol,
                                       sd + (int64_t)b * kSdComponents * g.nvol, g.nvol, p, g.s,
                                       P, P.fd[b], Rd, R, K, DK);
  double* q = ks + (int64_t)b * NVAR * npts + l;
  if constexpr (PART == 0) {
    double* r = rs + (int64_t)b * 6 * npts + l;
#pragma unroll
    for (int c = 0; c < 6; ++c) r[(int64_t)c * npts] = Rd[c];
    q[19 * npts] = R;
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 6; ++c) q[(int64_t)(a * 6 + c) * npts] = DK[a][c];
    q[18 * npts] = K;
  }
}

template <int NX>
__global__ void __launch_bounds__(128)
k_weyl_psi(Grid gin, const double* __restrict__ adm, const double* __restrict__ rs,
           const double* __restrict__ ks, double* __restrict__ weyl,
           const double* __restrict__ xf, int block0, int nblk) {
  const Grid g = fixed_geometry<NX>(gin);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nvol * nblk) return;
  const int b = block0 + (int)(t / g.nvol);
  const int64_t p = t % g.nvol;
  const int i = (int)(p % g.nn[0]);
  const int j = (int)((p / g.nn[0]) % g.nn[1]);
  const int k = (int)(p / ((int64_t)g.nn[0] * g.nn[1]));
  double* wb = weyl + (int64_t)b * 2 * g.nvol + p;
  const bool in = i >= NG && i <= NG + g.nx[0] && j >= NG && j <= NG + g.nx[1] && k >= NG &&
                  k <= NG + g.nx[2];
  double rp = __longlong_as_double(0x7ff8000000000000LL), ip = rp;
  if (in) {
    const int64_t npts = interior_count(g);
    const int64_t l = ((int64_t)(k - NG) * (g.nx[1] + 1) + (j - NG)) * (g.nx[0] + 1) + (i - NG);
    const double* r = rs + (int64_t)b * 6 * npts + l;
    const double* q = ks + (int64_t)b * NVAR * npts + l;
    const double* A = adm + (int64_t)b * Z4C_NADM * g.nvol + p;
    double Rd[6], DK[3][6], gph[6], Kd[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      Rd[c] = r[(int64_t)c * npts];
      gph[c] = A[(int64_t)(Z4C_ADM_GXX + c) * g.nvol];
      Kd[c] = A[(int64_t)(Z4C_ADM_KXX + c) * g.nvol];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 6; ++c) DK[a][c] = q[(int64_t)(a * 6 + c) * npts];
    const double* x = xf + (int64_t)b * (g.nn[0] + g.nn[1] + g.nn[2]);
    weyl_contract(gph, Kd, Rd, q[19 * npts], q[18 * npts], DK, x[i], x[g.nn[0] + j],
                  x[g.nn[0] + g.nn[1] + k], &rp, &ip);
  }
  wb[0] = rp;
  wb[g.nvol] = ip;
}

// ---- history sums (outputs/history.cpp:168-200): one CTA per block ---------
__global__ void k_hst(Grid g, DevParams P, const double* __restrict__ con,
                      const double* __restrict__ u, const double* __restrict__ xv,
                      double* __restrict__ partials) {
  const int b = blockIdx.x;
  const int64_t ncell = (int64_t)g.nx[0] * g.nx[1] * g.nx[2];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const double* x = xv + (int64_t)b * (g.nn[0] + g.nn[1] + g.nn[2] - 3);
  for (int64_t c = threadIdx.x; c < ncell; c += blockDim.x) {
    const int i = NG + (int)(c % g.nx[0]);
    const int j = NG + (int)((c / g.nx[0]) % g.nx[1]);
    const int k = NG + (int)(c / ((int64_t)g.nx[0] * g.nx[1]));
    const double x1 = x[i], x2 = x[g.nn[0] - 1 + j], x3 = x[g.nn[0] + g.nn[1] - 2 + k];
    const double R2 = x1 * x1 + x2 * x2 + x3 * x3;
    if (!(R2 <= P.p.r_max_con * P.p.r_max_con)) continue;
    const int64_t p = ((int64_t)k * g.nn[1] + j) * g.nn[0] + i;
    const double* cb = con + (int64_t)b * Z4C_NCON * g.nvol + p;
    const double H = fabs(cb[(int64_t)Z4C_CON_H * g.nvol]);
    acc[0] += H * H;
    acc[1] += fabs(cb[(int64_t)Z4C_CON_M * g.nvol]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double m = fabs(cb[(int64_t)(Z4C_CON_MX + a) * g.nvol]);
      acc[2 + a] += m * m;
    }
    acc[5] += fabs(cb[(int64_t)Z4C_CON_Z * g.nvol]);
    const double th = fabs(u[((int64_t)b * NVAR + Z4C_THETA) * g.nvol + p]);
    acc[6] += th * th;
    acc[7] += fabs(cb[(int64_t)Z4C_CON_C * g.nvol]);
  }
  __shared__ double sh[8][256];
#pragma unroll
  for (int q = 0; q < 8; ++q) sh[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int q = 0; q < 8; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 8; ++q) partials[b * 8 + q] = sh[q][0];
}

__global__ void k_check_finite(int64_t n, const double* __restrict__ u, int* flag) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  bool bad = false;
  for (; t < n; t += stride) bad |= !isfinite(u[t]);
  if (bad) atomicOr(flag, 1);
}

__global__ void k_zero_interior(Grid g, double* __restrict__ u, int nvar) {
  const int64_t npts = interior_count(g);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * g.nblocks * nvar) return;
  const int n = (int)(t % nvar);
  const int64_t r = t / nvar;
  const int b = (int)(r / npts);
  int i, j, k;
  interior_ijk(g, r % npts, i, j, k);
  u[((int64_t)b * nvar + n) * g.nvol + ((int64_t)k * g.nn[1] + j) * g.nn[0] + i] = 0.0;
}

// 8 independent DFMA chains per thread; the result is stored so that the
// compiler keeps the work.  Built with -fmad=false: the fma() intrinsic is an
// explicit DFMA and is not affected.
__global__ void __launch_bounds__(256) k_fp64_probe(int iters, double* sink, int nsink) {
  double a[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) a[q] = 1.0 + 1e-9 * (threadIdx.x + q);
  const double m = 0.999999999, c = 1e-9;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = fma(a[q], m, c);
  }
  double s = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += a[q];
  // never true; keeps the chains live
  if (s == 12345.6789 && (int)blockIdx.x < nsink) sink[blockIdx.x] = s;
}

}  // namespace

// ---- launchers -----------------------------------------------------------------

static std::atomic<long long> g_launches{0};
long long kernel_launch_count() { return g_launches.load(); }
void add_kernel_launches(long long n) { g_launches += n; }
#define COUNTED ++g_launches;

// Unroll of the column passes' z loops (loads in flight per thread): the
// fixed-geometry instances unroll their nx + 1 iterations completely, the
// generic ones by kColUnroll.
constexpr int kColUnroll = 4;

// Threads of the column passes (one per block, variable and interior (i, j)).
static int64_t columns(const Grid& g, int nblk) {
  return (int64_t)(g.nx[0] + 1) * (g.nx[1] + 1) * NVAR * nblk;
}

bool valid_shape(const LaunchShape& sh) {
  return (sh.point_regs == 0 || sh.point_regs == kPointRegsHigh) &&
         (sh.point_threads == 64 || sh.point_threads == 128 || sh.point_threads == 256) &&
         (sh.column_threads == 128 || sh.column_threads == 256 ||
          sh.column_threads == 512) &&
         (sh.column_slabs >= 0 && sh.column_slabs <= 4);
}

// Shared-memory slab geometry of a shape, or kper = 0 when the per-variable
// passes run as pencils (column_slabs = 0, or planes that do not fit).
constexpr int kSlabMaxBytes = 200 * 1024;
static SlabGeom slab_geom(const Grid& g, const LaunchShape& sh, size_t* bytes) {
  SlabGeom S{0, g.nn[0] * g.nn[1]};
  *bytes = 0;
  if (sh.column_slabs <= 0) return S;
  const int nk = g.nx[2] + 1;
  const int kper = (nk + sh.column_slabs - 1) / sh.column_slabs;
  const size_t b = sizeof(double) * (size_t)(kper + 2 * NG) * S.plane;
  if (b > (size_t)kSlabMaxBytes) return S;
  S.kper = kper;
  *bytes = b;
  return S;
}
bool slabs_fit(const Grid& g, const LaunchShape& sh) {
  size_t b;
  return slab_geom(g, sh, &b).kper > 0;
}
// Lets every slab kernel take up to kSlabMaxBytes of dynamic shared memory.
// Runs before any launch (at context creation), never inside a captured
// stream.
int allow_slab_smem() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* k) {
    const cudaError_t r =
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kSlabMaxBytes);
    if (e == cudaSuccess) e = r;
  };
  set((const void*)k_adv_prep_slab);
  set((const void*)k_ko_rhs_slab);
  set((const void*)k_ko_stage_ls_slab<true>);
  set((const void*)k_ko_stage_ls_slab<false>);
  set((const void*)k_ko_stage_bt_slab<true>);
  set((const void*)k_ko_stage_bt_slab<false>);
  return (int)e;
}

// MINB: CTAs per SM the heavy passes are compiled for (1: up to 255
// registers per thread; kPointMinb(T): 168, three resident CTAs of 128 or
// six of 64, for 1.5x the warps at a few dozen bytes of spill).
template <int T, int MINB>
static void launch_point_passes_t(const Grid& g, const DevParams& P, const double* u,
                                  const RhsScratch& sc, double* rhs, int block0, int nblk,
                                  int which, cudaStream_t st) {
  const int64_t n = interior_count(g) * nblk;
  COUNTED
  if (which == 0)
    (has_fixed_geometry(g) ? k_ricci<T, kFixedNX, MINB> : k_ricci<T, 0, MINB>)<<<div_up(n, T), T,
                                                                                0, st>>>(
        g, P, u, sc.sd, sc.rsum, block0, nblk);
  else
    (has_fixed_geometry(g) ? k_main<T, kFixedNX, MINB> : k_main<T, 0, MINB>)<<<div_up(n, T), T,
                                                                              0, st>>>(
        g, P, u, sc.sd, sc.rsum, sc.lv, rhs, block0, nblk);
}
static void launch_point_pass(const Grid& g, const DevParams& P, const double* u,
                              const RhsScratch& sc, double* rhs, int block0, int nblk, int which,
                              const LaunchShape& sh, cudaStream_t st) {
  const bool hi = sh.point_regs == kPointRegsHigh && has_fixed_geometry(g);
  switch (sh.point_threads) {
    case 64:
      if (hi) launch_point_passes_t<64, 6>(g, P, u, sc, rhs, block0, nblk, which, st);
      else launch_point_passes_t<64, 1>(g, P, u, sc, rhs, block0, nblk, which, st);
      break;
    case 256: launch_point_passes_t<256, 1>(g, P, u, sc, rhs, block0, nblk, which, st); break;
    default:
      if (hi) launch_point_passes_t<128, 3>(g, P, u, sc, rhs, block0, nblk, which, st);
      else launch_point_passes_t<128, 1>(g, P, u, sc, rhs, block0, nblk, which, st);
      break;
  }
}

// The right-hand side passes shared by every RHS launch: stored first
// derivatives (sd), Ricci (rsum), advection sums (lv) and the main pass into
// rhs (without KO).
static void launch_rhs_passes(const Grid& g, const DevParams& P, const double* u,
                              const RhsScratch& sc, double* rhs, int block0, int nblk,
                              const LaunchShape& sh, cudaStream_t st) {
  size_t smem;
  const SlabGeom S = slab_geom(g, sh, &smem);
  const int ct = sh.column_threads;
  if (S.kper > 0) {
    // advection sums and stored first derivatives from shared-memory slabs
    const dim3 grid((g.nx[2] + S.kper) / S.kper, NVAR, nblk);
    COUNTED
    k_adv_prep_slab<<<grid, ct, smem, st>>>(g, P, u, sc.lv, sc.sd, S, block0);
    launch_point_pass(g, P, u, sc, rhs, block0, nblk, 0, sh, st);
  } else {
    const int64_t cprep = (int64_t)(g.nx[0] + 7) * (g.nx[1] + 7);  // widest component region
    COUNTED
    (has_fixed_geometry(g) ? k_prep<kFixedNX>
                         : has_merged_geometry(g) ? k_prep<kMergedNX> : k_prep<0>)<<<dim3(div_up(cprep, kPointThreads),
                                                                 kSdComponents, nblk),
                                                            kPointThreads, 0, st>>>(
        g, P, u, sc.sd, block0);
    launch_point_pass(g, P, u, sc, rhs, block0, nblk, 0, sh, st);
    COUNTED
    (has_fixed_geometry(g) ? k_adv<kFixedNX + 1, kFixedNX> : k_adv<kColUnroll, 0>)<<<div_up(columns(g, nblk), ct), ct,
                                                                   0, st>>>(g, P, u, sc.lv, block0,
                                                                            nblk);
  }
  launch_point_pass(g, P, u, sc, rhs, block0, nblk, 1, sh, st);
}

void launch_prep(const Grid& g, const DevParams& P, const double* u, double* sd, int block0,
                 int nblk, cudaStream_t st) {
  const int64_t cprep = (int64_t)(g.nx[0] + 7) * (g.nx[1] + 7);  // widest component region
  COUNTED
  (has_fixed_geometry(g)    ? k_prep<kFixedNX>
   : has_merged_geometry(g) ? k_prep<kMergedNX>
                            : k_prep<0>)<<<dim3(div_up(cprep, kPointThreads), kSdComponents, nblk),
                                            kPointThreads, 0, st>>>(g, P, u, sd, block0);
}

void launch_prep_ricci(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                       int block0, int nblk, const LaunchShape& sh, cudaStream_t st) {
  launch_prep(g, P, u, sc.sd, block0, nblk, st);
  launch_point_pass(g, P, u, sc, nullptr, block0, nblk, 0, sh, st);
}

void launch_rhs(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                double* rhs, int block0, int nblk, const LaunchShape& sh, cudaStream_t st) {
  if (sh.contract && !g.has_sommerfeld) {
    launch_rhs_fast(g, P, u, sc, rhs, block0, nblk, sh, st);
    return;
  }
  launch_rhs_passes(g, P, u, sc, rhs, block0, nblk, sh, st);
  size_t smem;
  const SlabGeom S = slab_geom(g, sh, &smem);
  const int ct = sh.column_threads;
  COUNTED
  if (S.kper > 0) {
    k_ko_rhs_slab<<<dim3((g.nx[2] + S.kper) / S.kper, NVAR, nblk), ct, smem, st>>>(g, P, u, rhs,
                                                                                 S, block0);
  } else {
    (has_fixed_geometry(g) ? k_ko_rhs<kFixedNX + 1, kFixedNX> : k_ko_rhs<kColUnroll, 0>)<<<div_up(columns(g, nblk), ct),
                                                                        ct, 0, st>>>(g, P, u, rhs,
                                                                                     block0, nblk);
  }
}

void launch_stage_ls(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                     double* rhs, double* u1, double* u_out, const LsStage& w, int block0,
                     int nblk, const LaunchShape& sh, cudaStream_t st) {
  if (sh.contract && !g.has_sommerfeld) {
    launch_stage_ls_fast(g, P, u, sc, rhs, u1, u_out, w, block0, nblk, sh, st);
    return;
  }
  launch_rhs_passes(g, P, u, sc, rhs, block0, nblk, sh, st);
  size_t smem;
  const SlabGeom S = slab_geom(g, sh, &smem);
  const int ct = sh.column_threads;
  COUNTED
  if (S.kper > 0) {
    auto kern = g.has_sommerfeld ? k_ko_stage_ls_slab<true> : k_ko_stage_ls_slab<false>;
    kern<<<dim3((g.nx[2] + S.kper) / S.kper, NVAR, nblk), ct, smem, st>>>(g, P, u, rhs, u1, u_out,
                                                                        w, S, block0);
  } else {
    auto kern = has_fixed_geometry(g)
                    ? (g.has_sommerfeld ? k_ko_stage_ls<kFixedNX + 1, true, kFixedNX>
                                        : k_ko_stage_ls<kFixedNX + 1, false, kFixedNX>)
                    : (g.has_sommerfeld ? k_ko_stage_ls<kColUnroll, true, 0> : k_ko_stage_ls<kColUnroll, false, 0>);
    kern<<<div_up(columns(g, nblk), ct), ct, 0, st>>>(g, P, u, rhs, u1, u_out, w, block0, nblk);
  }
}

void launch_stage_bt(const Grid& g, const DevParams& P, const double* u, const RhsScratch& sc,
                     double* rhs, const double* un, double* const* k, double* u_out,
                     const BtStage& w, int block0, int nblk, const LaunchShape& sh,
                     cudaStream_t st) {
  launch_rhs_passes(g, P, u, sc, rhs, block0, nblk, sh, st);
  KPtrs K;
  for (int s = 0; s < 4; ++s) K.k[s] = k[s];
  size_t smem;
  const SlabGeom S = slab_geom(g, sh, &smem);
  const int ct = sh.column_threads;
  COUNTED
  if (S.kper > 0) {
    auto kern = g.has_sommerfeld ? k_ko_stage_bt_slab<true> : k_ko_stage_bt_slab<false>;
    kern<<<dim3((g.nx[2] + S.kper) / S.kper, NVAR, nblk), ct, smem, st>>>(g, P, u, rhs, un, K,
                                                                        u_out, w, S, block0);
  } else {
    auto kern = has_fixed_geometry(g)
                    ? (g.has_sommerfeld ? k_ko_stage_bt<kFixedNX + 1, true, kFixedNX>
                                        : k_ko_stage_bt<kFixedNX + 1, false, kFixedNX>)
                    : (g.has_sommerfeld ? k_ko_stage_bt<kColUnroll, true, 0> : k_ko_stage_bt<kColUnroll, false, 0>);
    kern<<<div_up(columns(g, nblk), ct), ct, 0, st>>>(g, P, u, rhs, un, K, u_out, w, block0,
                                                      nblk);
  }
}

// Slot of every direction in the neighbour list (mesh_topology.cpp:329-960
// order, the c_dirs table of the context), indexed (o0+1) + 3(o1+1) + 9(o2+1).
static int upload_dir_index() {
  static const int dirs[26][3] = {
      {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1},
      {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0},
      {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {1, 0, 1},
      {0, -1, -1}, {0, 1, -1}, {0, -1, 1}, {0, 1, 1},
      {-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
      {-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}};
  int h[27];
  for (int q = 0; q < 27; ++q) h[q] = 0;  // slot 13 (no offset) is never read
  for (int d = 0; d < 26; ++d)
    h[(dirs[d][0] + 1) + 3 * (dirs[d][1] + 1) + 9 * (dirs[d][2] + 1)] = d;
  return (int)cudaMemcpyToSymbol(c_dir_index, h, sizeof(h));
}

void launch_track_interp(const Grid& g, const DevParams& P, const double* u, double* trk,
                         int ntrk, cudaStream_t st) {
  COUNTED
  k_track_interp<<<1, 32, 0, st>>>(g, P, u, trk, ntrk);
}
void launch_track_update(double* trk, int ntrk, double dt, cudaStream_t st) {
  COUNTED
  k_track_update<<<1, 32, 0, st>>>(trk, ntrk, dt);
}

void launch_boundary_rhs(const Grid& g, const DevParams& P, const double* u, double* rhs,
                         int block0, int nblk, cudaStream_t st) {
  if (!g.has_sommerfeld) return;
  COUNTED
  k_sommerfeld<<<div_up(interior_count(g) * 11 * nblk, kPointThreads), kPointThreads, 0, st>>>(
      g, P, u, rhs, block0, nblk);
}

void launch_exchange(const Grid& g, const DevParams& P, const double* src, double* dst,
                     const int* nbr, int fuse_alg, cudaStream_t st, int nvar) {
  static const int dir_rc = upload_dir_index();  // once per process
  (void)dir_rc;
  const int64_t ni = div_up(interior_count(g) * g.nblocks, kPointThreads);
  const int64_t ng = div_up(g.nvol * g.nblocks, kPointThreads);
  const bool fx = has_fixed_geometry(g);
  COUNTED
  if (nvar == Z4C_NWEYL) {
    (fx ? k_exchange_interior<Z4C_NWEYL, kFixedNX> : k_exchange_interior<Z4C_NWEYL, 0>)<<<
        ni, kPointThreads, 0, st>>>(g, P, src, dst, nbr, 0);
  } else {
    (fx ? k_exchange_interior<NVAR, kFixedNX> : k_exchange_interior<NVAR, 0>)<<<
        ni, kPointThreads, 0, st>>>(g, P, src, dst, nbr, fuse_alg);
  }
  COUNTED
  if (nvar == Z4C_NWEYL) {
    (fx ? k_exchange_ghosts<Z4C_NWEYL, kFixedNX> : k_exchange_ghosts<Z4C_NWEYL, 0>)<<<
        ng, kPointThreads, 0, st>>>(g, P, dst, nbr, kAlgNone);
  } else {
    (fx ? k_exchange_ghosts<NVAR, kFixedNX> : k_exchange_ghosts<NVAR, 0>)<<<
        ng, kPointThreads, 0, st>>>(g, P, dst, nbr, fuse_alg);
  }
}

void launch_alg_constr_boundary(const Grid& g, const DevParams& P, double* u, const int* nbr,
                                cudaStream_t st) {
  const int64_t n = g.nvol * g.nblocks;
  COUNTED
  (has_fixed_geometry(g)    ? k_alg_constr_boundary<kFixedNX>
   : has_merged_geometry(g) ? k_alg_constr_boundary<kMergedNX>
                            : k_alg_constr_boundary<0>)<<<div_up(n, kPointThreads), kPointThreads,
                                                         0, st>>>(g, P, u, nbr);
}

void launch_physical_bcs(const Grid& g, double* u, int nvar, cudaStream_t st) {
  bool any = false;
  for (int f = 0; f < 6; ++f) any |= (g.bc[f] != Z4C_BC_PERIODIC);
  if (!any) return;
  for (int ax = 0; ax < 3; ++ax) {
    if (g.bc[2 * ax] == Z4C_BC_PERIODIC && g.bc[2 * ax + 1] == Z4C_BC_PERIODIC) continue;
    const int o1 = (ax == 0) ? 1 : 0, o2 = (ax == 2) ? 1 : 2;
    const int64_t n = (int64_t)g.nn[o1] * g.nn[o2] * 2 * nvar * g.nb[o1] * g.nb[o2];
    COUNTED
    const bool fx = has_fixed_geometry(g), fm = has_merged_geometry(g);
    auto kern = ax == 0   ? (fx ? k_bc_axis<kFixedNX, 0> : fm ? k_bc_axis<kMergedNX, 0> : k_bc_axis<0, 0>)
                : ax == 1 ? (fx ? k_bc_axis<kFixedNX, 1> : fm ? k_bc_axis<kMergedNX, 1> : k_bc_axis<0, 1>)
                          : (fx ? k_bc_axis<kFixedNX, 2> : fm ? k_bc_axis<kMergedNX, 2> : k_bc_axis<0, 2>);
    kern<<<div_up(n, kPointThreads), kPointThreads, 0, st>>>(g, u, nvar);
  }
}

void launch_alg_constr(const Grid& g, const DevParams& P, double* u, int block0, int nblk,
                       cudaStream_t st, int ghosts_only) {
  const int64_t n = g.nvol * nblk;
  COUNTED
  (has_fixed_geometry(g) ? k_alg_constr<kFixedNX> : k_alg_constr<0>)<<<
      div_up(n, kPointThreads), kPointThreads, 0, st>>>(g, P, u, block0, nblk, ghosts_only);
}

void launch_weighted_ave(const Grid& g, double* out, const double* in1, const double* in2,
                         const double w[3], int block0, int nblk, cudaStream_t st) {
  const int64_t n = interior_count(g) * nblk * NVAR;
  COUNTED
  k_weighted_ave<<<div_up(n, kPointThreads), kPointThreads, 0, st>>>(
      g, out, in1, in2, w[0], w[1], w[2], block0, nblk);
}

void launch_add_rhs(const Grid& g, const double* rhs, double wght, double* out, int block0,
                    int nblk, cudaStream_t st) {
  const int64_t n = interior_count(g) * nblk * NVAR;
  COUNTED
  k_add_rhs<<<div_up(n, kPointThreads), kPointThreads, 0, st>>>(g, rhs, wght, out, block0, nblk);
}

void launch_z4c_to_adm(const Grid& g, const DevParams& P, const double* u, double* adm,
                       int block0, int nblk, cudaStream_t st, int ghosts_only) {
  const int64_t n = g.nvol * nblk;
  COUNTED
  k_z4c_to_adm<<<div_up(n, kPointThreads), kPointThreads, 0, st>>>(g, P, u, adm, block0, nblk,
                                                                    ghosts_only);
}

void launch_adm_to_z4c(const Grid& g, const DevParams& P, const double* adm, double* u,
                       double* guu_scratch, int block0, int nblk, cudaStream_t st, int alg) {
  const int64_t n = g.nvol * nblk;
  // guu_scratch is indexed by absolute block number
  COUNTED
  k_adm_to_z4c_pt<<<div_up(n, kPointThreads), kPointThreads, 0, st>>>(g, P, adm, u, guu_scratch,
                                                                      block0, nblk);
  COUNTED
  k_adm_to_z4c_gam<<<div_up(n, kPointThreads), kPointThreads, 0, st>>>(g, P, guu_scratch, u,
                                                                       block0, nblk);
  if (!alg) return;
  COUNTED
  (has_fixed_geometry(g) ? k_alg_constr<kFixedNX> : k_alg_constr<0>)<<<
      div_up(n, kPointThreads), kPointThreads, 0, st>>>(g, P, u, block0, nblk, 0);
}

void launch_adm_constraints(const Grid& g, const DevParams& P, const double* adm,
                            const double* u, double* con, const double* xf, int block0,
                            int nblk, cudaStream_t st) {
  const int64_t n = g.nvol * nblk;
  COUNTED
  (has_fixed_geometry(g) ? k_adm_constraints<kFixedNX> : k_adm_constraints<0>)<<<
      div_up(n, 128), 128, 0, st>>>(g, P, adm, u, con, xf, block0, nblk);
}

void launch_weyl(const Grid& g, const DevParams& P, const double* adm, const double* u,
                 double* sd, double* rs, double* ks, double* weyl, const double* xf, int block0,
                 int nblk, cudaStream_t st) {
  const int64_t cprep = (int64_t)(g.nx[0] + 7) * (g.nx[1] + 7);  // widest component region
  COUNTED
  (has_fixed_geometry(g) ? k_prep<kFixedNX> : k_prep<0>)<<<dim3(div_up(cprep, kPointThreads),
                                                               kSdComponents, nblk),
                                                          kPointThreads, 0, st>>>(
      g, P, u, sd, block0);
  const int64_t m = interior_count(g) * nblk;
  const bool fx = has_fixed_geometry(g);
  COUNTED
  (fx ? k_weyl_curv<kFixedNX, 0> : k_weyl_curv<0, 0>)<<<div_up(m, 128), 128, 0, st>>>(
      g, P, adm, u, sd, rs, ks, block0, nblk);
  COUNTED
  (fx ? k_weyl_curv<kFixedNX, 1> : k_weyl_curv<0, 1>)<<<div_up(m, 128), 128, 0, st>>>(
      g, P, adm, u, sd, rs, ks, block0, nblk);
  const int64_t n = g.nvol * nblk;
  COUNTED
  (has_fixed_geometry(g) ? k_weyl_psi<kFixedNX> : k_weyl_psi<0>)<<<div_up(n, 128), 128, 0, st>>>(
      g, adm, rs, ks, weyl, xf, block0, nblk);
}

void launch_hst(const Grid& g, const DevParams& P, const double* con, const double* u,
                const double* xv, double* partials, cudaStream_t st) {
  COUNTED
  k_hst<<<g.nblocks, 256, 0, st>>>(g, P, con, u, xv, partials);
}

void launch_check_finite(const Grid& g, const double* u, int nvar, int* flag, cudaStream_t st) {
  const int64_t n = g.nvol * g.nblocks * nvar;
  COUNTED
  k_check_finite<<<1184, 256, 0, st>>>(n, u, flag);
}

long long launch_fp64_probe(int nsm, int iters, double* sink, int nsink, cudaStream_t st) {
  const int blocks = nsm * 8;
  COUNTED
  k_fp64_probe<<<blocks, 256, 0, st>>>(iters, sink, nsink);
  return 2LL * 8 * iters * 256LL * blocks;
}

void launch_zero_interior(const Grid& g, double* u, int nvar, cudaStream_t st) {
  const int64_t n = interior_count(g) * g.nblocks * nvar;
  COUNTED
  k_zero_interior<<<div_up(n, kPointThreads), kPointThreads, 0, st>>>(g, u, nvar);
}

}  // namespace z4c

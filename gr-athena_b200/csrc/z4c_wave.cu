// psi4 extraction on coordinate spheres (see z4c_wave.cuh).
//
// Host set-up, once per sphere and mesh:
//   GeodesicGrid           mesh/geodesic_grid.cpp:21-160 (vertices of an
//                          icosahedron refined nlev times: five blocks of
//                          nlev x 2 nlev vertices plus the poles),
//                          :312-360 (dual-cell weights), :463-475
//   SphericalGrid          mesh/spherical_grid.cpp:17-36
//   SphericalPatch         mesh/spherical_grid.cpp:44-116 (vertex
//                          collocation: block ownership over the half-open
//                          box [x1f(is), x1f(ie+1)), LagrangeInterpND<7,3>
//                          stencils from x1f(0) with spacing dx)
//   sYlm                   utils/spherical_harmonics.hpp:231-255
// Device work per extraction (WaveExtractLocal::Decompose_multipole,
// wave_extract.cpp:208-234, and WaveExtract::ReduceMultipole, :95-140):
//   k_wave_interp          Re, Im psi4 at every owned vertex (one thread each)
//   k_wave_project         per (owning block, (l, m)) the sum over the block's
//                          vertices in vertex order
//   k_wave_reduce          per (l, m) the sum over blocks in gid order, i.e.
//                          the Morton order of the blocks' logical locations
//                          (x the lowest bit), which is the order in which the
//                          reference's MeshBlockTree numbers a uniform mesh
// Host arithmetic keeps the reference's evaluation order (the library's host
// code is compiled with -ffp-contract=off), so every table matches it bit for
// bit when the same libm is used.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "z4c_kernels.cuh"
#include "z4c_wave.cuh"

namespace z4c {

namespace {

constexpr double kPi = 3.1415926535897932;  // PI of the reference's configuration
constexpr int kOrder = 2 * NG - 1;          // LagrangeInterpND<2*NGHOST-1, 3>
constexpr int kSten = kOrder + 1;

// ---- GeodesicGrid ----------------------------------------------------------
class Geodesic {
 public:
  explicit Geodesic(int nlev) : n_(nlev), rows_(nlev + 2), cols_(2 * nlev + 2) {
    const size_t sz = (size_t)5 * rows_ * cols_;
    for (auto& c : comp_) c.assign(sz, 0.0);
    idx_.assign(sz, 0);
    const double sa = 2.0 / std::sqrt(5.0), ca = 1.0 / std::sqrt(5.0);
    const double P1[3] = {0.0, 0.0, 1.0};
    const double P2[3] = {sa, 0.0, ca};
    const double P3[3] = {sa * std::cos(0.2 * kPi), sa * std::sin(0.2 * kPi), -ca};
    const double P4[3] = {sa * std::cos(-0.4 * kPi), sa * std::sin(-0.4 * kPi), ca};
    const double P5[3] = {sa * std::cos(-0.2 * kPi), sa * std::sin(-0.2 * kPi), -ca};
    const double P6[3] = {0.0, 0.0, -1.0};
    // block 0 row by row: four runs of vertices, each a normalised weighted
    // sum of three icosahedron vertices
    for (int l = 0; l < n_; ++l) {
      int col = 1;
      for (int m = l; m < n_; ++m) put(l + 1, col++, m - l + 1, P2, n_ - m - 1, P1, l, P4);
      for (int m = n_ - l; m < n_; ++m)
        put(l + 1, col++, n_ - l, P2, m - n_ + l + 1, P5, n_ - m - 1, P4);
      for (int m = l; m < n_; ++m) put(l + 1, col++, m - l + 1, P3, n_ - m - 1, P2, l, P5);
      for (int m = n_ - l; m < n_; ++m)
        put(l + 1, col++, n_ - l, P3, m - n_ + l + 1, P6, n_ - m - 1, P5);
    }
    // blocks 1..4: block 0 rotated by bl * 2 pi / 5 about z
    for (int bl = 1; bl < 5; ++bl)
      for (int l = 1; l <= n_; ++l)
        for (int m = 1; m <= 2 * n_; ++m) {
          const size_t q0 = at(0, l, m), q = at(bl, l, m);
          const double x0 = comp_[0][q0], y0 = comp_[1][q0];
          comp_[0][q] = x0 * std::cos(bl * 0.4 * kPi) + y0 * std::sin(bl * 0.4 * kPi);
          comp_[1][q] = y0 * std::cos(bl * 0.4 * kPi) - x0 * std::sin(bl * 0.4 * kPi);
          comp_[2][q] = comp_[2][q0];
        }
    const double pole[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {1.0, -1.0}};
    for (int a = 0; a < 3; ++a) {
      pole_[a][0] = pole[a][0];
      pole_[a][1] = pole[a][1];
      ghosts(comp_[a], pole_[a]);
    }
    for (int bl = 0; bl < 5; ++bl)
      for (int l = 0; l < n_; ++l)
        for (int m = 0; m < 2 * n_; ++m) idx_[at(bl, l + 1, m + 1)] = bl * 2 * n_ * n_ + l * 2 * n_ + m;
    const int pidx[2] = {10 * n_ * n_, 10 * n_ * n_ + 1};
    ghosts(idx_, pidx);
  }

  int vertices() const { return 10 * n_ * n_ + 2; }

  void position(int ic, double p[3]) const {
    const int b0 = ic / (2 * n_ * n_);
    const int r = ic % (2 * n_ * n_);
    const int b1 = r / (2 * n_), b2 = r % (2 * n_);
    for (int a = 0; a < 3; ++a) p[a] = (b0 == 5) ? pole_[a][b2] : comp_[a][at(b0, b1 + 1, b2 + 1)];
  }

  // area of the dual cell of vertex ic on the unit sphere
  double weight(int ic) const {
    int nv[6];
    const int nn = neighbours(ic, nv);
    double p0[3];
    position(ic, p0);
    double w = 0.0;
    for (int q = 0; q < nn; ++q) {
      double n1[3], n2[3], n3[3], c1[3], c2[3];
      position(nv[(q + nn - 1) % nn], n1);
      position(nv[q], n2);
      position(nv[(q + 1) % nn], n3);
      circumcentre(p0, n1, n2, c1);
      circumcentre(p0, n2, n3, c2);
      const double s1 = p0[0] * c1[0] + p0[1] * c1[1] + p0[2] * c1[2];
      const double s2 = p0[0] * c2[0] + p0[1] * c2[1] + p0[2] * c2[2];
      const double s12 = c1[0] * c2[0] + c1[1] * c2[1] + c1[2] * c2[2];
      const double num = std::abs(p0[0] * (c1[1] * c2[2] - c2[1] * c1[2]) +
                                  p0[1] * (c2[0] * c1[2] - c1[0] * c2[2]) +
                                  p0[2] * (c1[0] * c2[1] - c1[1] * c2[0]));
      const double den = 1.0 + s1 + s2 + s12;
      w += 2.0 * std::atan(num / den);
    }
    return w;
  }

 private:
  size_t at(int bl, int l, int m) const { return ((size_t)bl * rows_ + l) * cols_ + m; }

  void put(int row, int col, int wa, const double* A, int wb, const double* B, int wc,
           const double* C) {
    const double n = (double)n_;
    double v[3];
    for (int a = 0; a < 3; ++a) v[a] = (wa * A[a] + wb * B[a] + wc * C[a]) / n;
    const double norm = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int a = 0; a < 3; ++a) comp_[a][at(0, row, col)] = v[a] / norm;
  }

  // ghost rows/columns of the five blocks (geodesic_grid.hpp:145-160)
  template <class T, class P>
  void ghosts(std::vector<T>& a, const P& pole) const {
    const int n = n_;
    for (int bl = 0; bl < 5; ++bl) {
      const int pv = (bl + 4) % 5, nx = (bl + 1) % 5;
      for (int k = 0; k < n; ++k) {
        a[at(bl, 0, k + 1)] = a[at(pv, k + 1, 1)];
        a[at(bl, 0, k + n + 1)] = a[at(pv, n, k + 1)];
        a[at(bl, k + 1, 2 * n + 1)] = a[at(pv, n, k + n + 1)];
        a[at(bl, k + 2, 0)] = a[at(nx, 1, k + 1)];
        a[at(bl, n + 1, k + 1)] = a[at(nx, 1, k + n + 1)];
        a[at(bl, n + 1, k + n + 1)] = a[at(nx, k + 2, 2 * n)];
      }
      a[at(bl, 1, 0)] = pole[0];
      a[at(bl, n + 1, 2 * n)] = pole[1];
      a[at(bl, 0, 2 * n + 1)] = a[at(bl, 0, 2 * n)];
    }
  }

  int neighbours(int ic, int nb[6]) const {
    const int n = n_;
    if (ic == 10 * n * n) {
      for (int bl = 0; bl < 5; ++bl) nb[bl] = idx_[at(bl, 1, 1)];
      return 5;
    }
    if (ic == 10 * n * n + 1) {
      for (int bl = 0; bl < 5; ++bl) nb[bl] = idx_[at(bl, n, 2 * n)];
      return 5;
    }
    const int b0 = ic / (2 * n * n);
    const int r = ic % (2 * n * n);
    const int b1 = r / (2 * n), b2 = r % (2 * n);
    nb[0] = idx_[at(b0, b1 + 1, b2 + 2)];
    nb[1] = idx_[at(b0, b1 + 2, b2 + 1)];
    nb[2] = idx_[at(b0, b1 + 2, b2)];
    nb[3] = idx_[at(b0, b1 + 1, b2)];
    nb[4] = idx_[at(b0, b1, b2 + 1)];
    if (r == n - 1 || r == 2 * n - 1) return 5;  // the icosahedron's own vertices
    nb[5] = idx_[at(b0, b1, b2 + 2)];
    return 6;
  }

  static void circumcentre(const double p1[3], const double p2[3], const double p3[3],
                           double out[3]) {
    double d23 = 0, d31 = 0, d12 = 0;
    d23 = (p3[0] - p2[0]) * (p3[0] - p2[0]) + (p3[1] - p2[1]) * (p3[1] - p2[1]) +
          (p3[2] - p2[2]) * (p3[2] - p2[2]);
    d31 = (p1[0] - p3[0]) * (p1[0] - p3[0]) + (p1[1] - p3[1]) * (p1[1] - p3[1]) +
          (p1[2] - p3[2]) * (p1[2] - p3[2]);
    d12 = (p2[0] - p1[0]) * (p2[0] - p1[0]) + (p2[1] - p1[1]) * (p2[1] - p1[1]) +
          (p2[2] - p1[2]) * (p2[2] - p1[2]);
    const double a = std::sqrt(d23), b = std::sqrt(d31), c = std::sqrt(d12);
    const double den = 1.0 / ((a + c + b) * (a + c - b) * (a + b - c) * (b + c - a));
    double v[3];
    for (int q = 0; q < 3; ++q)
      v[q] = (p1[q] * a * a * (b * b + c * c - a * a) + p2[q] * b * b * (c * c + a * a - b * b) +
              p3[q] * c * c * (a * a + b * b - c * c)) * den;
    const double nc = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int q = 0; q < 3; ++q) out[q] = v[q] / nc;
  }

  int n_, rows_, cols_;
  std::vector<double> comp_[3];
  std::vector<int> idx_;
  double pole_[3][2];
};

// ---- spin-weighted spherical harmonics --------------------------------------
double factorial(int n) {
  double t = 1.0;
  for (int i = 1; i <= n; ++i) t = t * (double)i;
  return t;
}

void sylm(int s, int l, int m, double theta, double phi, double* re, double* im) {
  double wd = 0;
  const int k1 = std::max(0, m + s), k2 = std::min(l + m, l + s);
  for (int k = k1; k <= k2; ++k) {
    wd += ((k % 2 == 0) ? 1.0 : -1.0) *
          std::sqrt(factorial(l + m) * factorial(l - m) * factorial(l - s) * factorial(l + s)) *
          std::pow(std::cos(theta / 2.0), (double)(2 * l + m + s - 2 * k)) *
          std::pow(std::sin(theta / 2.0), (double)(2 * k - m - s)) /
          (factorial(l + m - k) * factorial(l + s - k) * factorial(k) * factorial(k - m - s));
  }
  const double norm = std::sqrt((2 * l + 1) / (4.0 * kPi));
  *re = norm * wd * std::cos(m * phi);
  *im = norm * wd * std::sin(m * phi);
}

// LagrangeInterp1D<7> (utils/lagrange_interp.hpp:24-150, odd order): the
// first stencil vertex, shifted into [0, siz - 8], and the 8 coefficients
int lagrange_stencil(double origin, double delta, int siz, double coord, double coef[kSten]) {
  const double inv = 1.0 / delta;
  int point = (int)std::lrint(std::floor((coord - origin) * inv - 0.5 * (kOrder - 1)));
  int shift = point;
  if (shift < 0) point -= shift;
  shift = point + kOrder - (siz - 1);
  if (shift > 0) point -= shift;
  double xp[kSten];
  for (int i = 0; i < kSten; ++i) xp[i] = (point + i) * delta + origin;
  for (int j = 0; j < kSten; ++j) {
    double num = 1.0, den = 1.0;
    for (int i = 0; i < kSten; ++i) {
      if (i == j) continue;
      num = num * (coord - xp[i]);
      den = den * (xp[j] - xp[i]);
    }
    coef[j] = num / den;
  }
  return point;
}

uint64_t morton(const int loc[3]) {
  uint64_t key = 0;
  for (int bit = 0; bit < 20; ++bit)
    for (int a = 0; a < 3; ++a) key |= (uint64_t)((loc[a] >> bit) & 1) << (3 * bit + a);
  return key;
}

// ---- kernels ----------------------------------------------------------------
__global__ void k_wave_interp(Grid g, const double* __restrict__ weyl, const int* __restrict__ blk,
                              const int* __restrict__ base, const double* __restrict__ coef,
                              double* __restrict__ data, int npts) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const double* cf = coef + (int64_t)p * 3 * kSten;
  for (int v = 0; v < 2; ++v) {
    const double* f = weyl + ((int64_t)blk[p] * 2 + v) * g.nvol + base[p];
    // LagrangeInterpND::eval: x innermost, then y, then z
    double out = 0;
    for (int ez = 0; ez < kSten; ++ez) {
      double vy = 0;
      for (int ey = 0; ey < kSten; ++ey) {
        const double* row = f + ez * g.s[2] + ey * g.s[1];
        double vx = 0;
#pragma unroll
        for (int i = 0; i < kSten; ++i) vx += cf[i] * __ldg(row + i);
        vy += cf[kSten + ey] * vx;
      }
      out += cf[2 * kSten + ez] * vy;
    }
    data[(int64_t)v * npts + p] = out;
  }
}

__global__ void k_wave_project(const double* __restrict__ data, const double* __restrict__ pw,
                               const double* __restrict__ ylm, const int* __restrict__ seg,
                               double* __restrict__ loc, int npts, int nseg, int nslot,
                               int lmax) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nseg * nslot) return;
  const int sg = t / nslot, slot = t % nslot;
  const int l = 2 + slot / (2 * lmax + 1), mpl = slot % (2 * lmax + 1);
  double pr = 0.0, pi = 0.0;
  if (mpl <= 2 * l) {
    const double* Y = ylm + (int64_t)slot * npts * 2;
    for (int p = seg[sg]; p < seg[sg + 1]; ++p) {
      const double dr = data[p], di = data[npts + p];
      const double wt = pw[2 * p], bz = pw[2 * p + 1];
      const double yr = Y[2 * p], yi = Y[2 * p + 1];
      pr += dr * wt * yr + bz * di * wt * yi;
      pi += bz * di * wt * yr - dr * wt * yi;
    }
  }
  loc[((int64_t)sg * nslot + slot) * 2] = pr;
  loc[((int64_t)sg * nslot + slot) * 2 + 1] = pi;
}

__global__ void k_wave_reduce(const double* __restrict__ loc, double* __restrict__ psi, int nseg,
                              int nslot) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * nslot) return;
  double s = 0.0;
  for (int sg = 0; sg < nseg; ++sg) s += loc[(int64_t)sg * nslot * 2 + t];
  psi[t] = s;
}

template <class T>
cudaError_t upload(T** d, const std::vector<T>& h) {
  cudaError_t e = cudaMalloc((void**)d, sizeof(T) * std::max<size_t>(h.size(), 1));
  if (e != cudaSuccess) return e;
  if (h.empty()) return cudaSuccess;
  return cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
}

}  // namespace

std::vector<double> sphere_grid(int nlev, double rad, bool bitant) {
  Geodesic geo(nlev);
  const int np = geo.vertices();
  std::vector<double> out(6 * (size_t)np);
  for (int ic = 0; ic < np; ++ic) {
    double p[3];
    geo.position(ic, p);
    const double th = std::acos(p[2]), ph = std::atan2(p[1], p[0]);
    double* o = &out[6 * (size_t)ic];
    o[0] = th;
    o[1] = ph;
    o[2] = rad * std::sin(th) * std::cos(ph);
    o[3] = rad * std::sin(th) * std::sin(ph);
    o[4] = rad * std::cos(th);
    if (bitant) o[4] = std::abs(o[4]);
    o[5] = rad * rad * geo.weight(ic);
  }
  return out;
}

int wave_build(const Grid& g, const std::vector<double>& xf, const std::vector<double>& dx,
               double rad, int nlev, int lmax, bool bitant, WaveSphere* w, char* msg, int nmsg) {
  *w = WaveSphere();
  w->rad = rad;
  w->nlev = nlev;
  w->lmax = lmax;
  w->bitant = bitant ? 1 : 0;
  w->nslot = (lmax - 1) * (2 * lmax + 1);
  const std::vector<double> geo = sphere_grid(nlev, rad, bitant);
  const int nv = (int)(geo.size() / 6);
  // blocks in gid order (on a refined mesh the context's blocks already are,
  // and their row g.nb = {nblocks, 1, 1} keeps that order below)
  std::vector<int> order(g.nblocks);
  std::vector<uint64_t> key(g.nblocks);
  for (int b = 0; b < g.nblocks; ++b) {
    const int loc[3] = {b % g.nb[0], (b / g.nb[0]) % g.nb[1], b / (g.nb[0] * g.nb[1])};
    key[b] = morton(loc);
    order[b] = b;
  }
  std::sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
  const int xstride = g.nn[0] + g.nn[1] + g.nn[2];
  std::vector<int> hblk, hbase, hseg;
  std::vector<double> hcoef, hpw;
  std::vector<int> owned;  // vertex index per point
  for (int b : order) {
    const double* x[3] = {&xf[(size_t)b * xstride], &xf[(size_t)b * xstride + g.nn[0]],
                          &xf[(size_t)b * xstride + g.nn[0] + g.nn[1]]};
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = x[a][NG];
      hi[a] = x[a][NG + g.nx[a]];
    }
    const int first = (int)hblk.size();
    for (int ic = 0; ic < nv; ++ic) {
      const double* o = &geo[6 * (size_t)ic];
      if (!(o[2] >= lo[0] && o[2] < hi[0] && o[3] >= lo[1] && o[3] < hi[1] && o[4] >= lo[2] &&
            o[4] < hi[2]))
        continue;
      int pt[3];
      double c[3][kSten];
      for (int a = 0; a < 3; ++a) {
        pt[a] = lagrange_stencil(x[a][0], dx[(size_t)b * 3 + a], g.nn[a], o[2 + a], c[a]);
        if (pt[a] < 0 || pt[a] + kSten > g.nn[a]) {
          snprintf(msg, nmsg, "wave sphere: stencil of vertex %d leaves block %d", ic, b);
          return Z4C_EINVAL;
        }
      }
      hblk.push_back(b);
      hbase.push_back((int)(pt[0] * g.s[0] + pt[1] * g.s[1] + pt[2] * g.s[2]));
      for (int a = 0; a < 3; ++a)
        for (int i = 0; i < kSten; ++i) hcoef.push_back(c[a][i]);
      double wt = o[5];
      wt /= rad * rad;
      hpw.push_back(wt);
      hpw.push_back((bitant && o[0] > kPi / 2) ? -1 : 1);
      owned.push_back(ic);
    }
    if ((int)hblk.size() > first) hseg.push_back(first);
  }
  w->npts = (int)hblk.size();
  w->nseg = (int)hseg.size();
  hseg.push_back(w->npts);
  std::vector<double> hy((size_t)w->nslot * w->npts * 2, 0.0);
  for (int l = 2; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m) {
      const int slot = (l - 2) * (2 * lmax + 1) + (m + l);
      for (int p = 0; p < w->npts; ++p) {
        const double* o = &geo[6 * (size_t)owned[p]];
        sylm(-2, l, m, o[0], o[1], &hy[((size_t)slot * w->npts + p) * 2],
             &hy[((size_t)slot * w->npts + p) * 2 + 1]);
      }
    }
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = upload(&w->blk, hblk);
  if (e == cudaSuccess) e = upload(&w->base, hbase);
  if (e == cudaSuccess) e = upload(&w->coef, hcoef);
  if (e == cudaSuccess) e = upload(&w->pw, hpw);
  if (e == cudaSuccess) e = upload(&w->ylm, hy);
  if (e == cudaSuccess) e = upload(&w->seg, hseg);
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&w->data, sizeof(double) * 2 * std::max(w->npts, 1));
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&w->loc, sizeof(double) * 2 * w->nslot * std::max(w->nseg, 1));
  if (e == cudaSuccess) e = cudaMalloc((void**)&w->psi, sizeof(double) * 2 * w->nslot);
  if (e != cudaSuccess) {
    snprintf(msg, nmsg, "wave sphere: %s", cudaGetErrorString(e));
    cudaGetLastError();
    wave_free(w);
    return Z4C_ENOMEM;
  }
  return Z4C_OK;
}

void wave_free(WaveSphere* w) {
  cudaFree(w->blk);
  cudaFree(w->base);
  cudaFree(w->coef);
  cudaFree(w->pw);
  cudaFree(w->ylm);
  cudaFree(w->seg);
  cudaFree(w->data);
  cudaFree(w->loc);
  cudaFree(w->psi);
  *w = WaveSphere();
}

void launch_wave(const Grid& g, const WaveSphere& w, const double* weyl, cudaStream_t st) {
  if (w.npts > 0) {
    k_wave_interp<<<(w.npts + 127) / 128, 128, 0, st>>>(g, weyl, w.blk, w.base, w.coef, w.data,
                                                       w.npts);
    const int nt = w.nseg * w.nslot;
    k_wave_project<<<(nt + 127) / 128, 128, 0, st>>>(w.data, w.pw, w.ylm, w.seg, w.loc, w.npts,
                                                     w.nseg, w.nslot, w.lmax);
    add_kernel_launches(2);
  }
  k_wave_reduce<<<(2 * w.nslot + 127) / 128, 128, 0, st>>>(w.loc, w.psi, w.nseg, w.nslot);
  add_kernel_launches(1);
}

void launch_wave_interp(const Grid& g, const WaveSphere& w, const double* weyl, cudaStream_t st) {
  if (w.npts <= 0) return;
  k_wave_interp<<<(w.npts + 127) / 128, 128, 0, st>>>(g, weyl, w.blk, w.base, w.coef, w.data,
                                                     w.npts);
  add_kernel_launches(1);
}

// Transpose of k_wave_interp: every sphere vertex's adjoint (databar, Re and
// Im, [2][npts]) scattered onto its 8^3 stencil of the Weyl register's
// adjoint with the interpolation weights; atomic adds (neighbouring sphere
// vertices share stencil vertices).
__global__ void k_wave_interp_adj(Grid g, const int* __restrict__ blk, const int* __restrict__ base,
                                  const double* __restrict__ coef,
                                  const double* __restrict__ databar, double* __restrict__ wbar,
                                  int npts) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const double* cf = coef + (int64_t)p * 3 * kSten;
  for (int v = 0; v < 2; ++v) {
    const double a = databar[(int64_t)v * npts + p];
    if (a == 0.0) continue;
    double* f = wbar + ((int64_t)blk[p] * 2 + v) * g.nvol + base[p];
    for (int ez = 0; ez < kSten; ++ez)
      for (int ey = 0; ey < kSten; ++ey) {
        const double wzy = cf[2 * kSten + ez] * cf[kSten + ey] * a;
        double* row = f + ez * g.s[2] + ey * g.s[1];
        for (int i = 0; i < kSten; ++i) atomicAdd(row + i, cf[i] * wzy);
      }
  }
}

void launch_wave_interp_adj(const Grid& g, const WaveSphere& w, const double* databar,
                            double* wbar, cudaStream_t st) {
  if (w.npts <= 0) return;
  k_wave_interp_adj<<<(w.npts + 127) / 128, 128, 0, st>>>(g, w.blk, w.base, w.coef, databar,
                                                         wbar, w.npts);
  add_kernel_launches(1);
}

}  // namespace z4c

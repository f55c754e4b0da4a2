// z4c_rhs_noalloc: the Z4c right-hand side on caller-owned device buffers,
// with no device allocation anywhere in the call.
//
// Who needs it: a caller whose host program owns every byte of device memory
// through its own allocator (a framework's caching allocator, or a pool
// reserved once at start-up) may not call cudaMalloc behind that allocator's
// back, and a caller inside a time-stepping loop cannot afford the implicit
// device-wide synchronisation that cudaMalloc/cudaFree bring.  z4c_rhs needs a
// context, and a context allocates its registers and scratch.  This entry
// point takes the state and the output as plain device pointers and keeps the
// scratch of the right-hand-side passes (the stored first derivatives, the
// Ricci sums and the advection sums) in a fixed array compiled into the
// library.
//
// The array: kScratchBytes = 64 MiB, a file-scope __device__ array.  Every GPU
// that loads the library holds it until the process exits.  All calls share
// it and it keeps the last call's contents: nothing in it has to start at
// zero (each pass writes every entry it later reads), and two calls whose
// work overlaps on the GPU (different streams, or different host threads)
// race on it.  Blocks are processed in chunks that fit the array; a single
// MeshBlock whose scratch does not fit is rejected.
//
// The first call on a device: with CUDA's lazy module loading the address
// lookup below is when the driver loads this library's device code on that
// device and reserves the array, which is an allocation; callers make one
// call at start-up, outside any stream capture, and every later call
// allocates nothing.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/z4c_b200.h"
#include "z4c_common.cuh"
#include "z4c_kernels.cuh"

namespace z4c {
int set_error(int code, const char* msg);
}

using namespace z4c;

namespace {

constexpr size_t kScratchBytes = (size_t)Z4C_NOALLOC_SCRATCH_MIB << 20;
// The per-block FD scalings sit at the front of the array, the pass scratch
// after them.
constexpr size_t kFdBytes = 64 << 10;
constexpr int kMaxFd = (int)(kFdBytes / sizeof(FdScale));
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kScratchBytes / sizeof(double)];

// Device address of g_noalloc_scratch per device ordinal.  In host code the
// array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
double* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

int scratch_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    char buf[160];
    snprintf(buf, sizeof(buf), "z4c_rhs_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    return set_error(Z4C_ENODEV, buf);
  }
  if (dev < 0 || dev >= kMaxDevices) return set_error(Z4C_ENODEV, "z4c_rhs_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      char buf[160];
      snprintf(buf, sizeof(buf), "z4c_rhs_noalloc: cudaGetSymbolAddress: %s",
               cudaGetErrorString(e));
      return set_error(Z4C_ECUDA, buf);
    }
    g_scratch_addr[dev] = static_cast<double*>(p);
    // the slab kernels launched by the right-hand side take more than the
    // default 48 kB of dynamic shared memory
    e = static_cast<cudaError_t>(allow_slab_smem());
    if (e != cudaSuccess) {
      char buf[160];
      snprintf(buf, sizeof(buf), "z4c_rhs_noalloc: shared-memory limit: %s",
               cudaGetErrorString(e));
      g_scratch_addr[dev] = nullptr;
      return set_error(Z4C_ECUDA, buf);
    }
  }
  *out = g_scratch_addr[dev];
  return Z4C_OK;
}

__global__ void k_fill_fd(FdScale* __restrict__ fd, FdScale v, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) fd[t] = v;
}

}  // namespace

extern "C" int z4c_rhs_noalloc(const double* u, double* rhs, int nblocks, const int nx[3],
                               const double dx[3], const z4c_params_t* params, void* stream) {
  if (!u || !rhs || !nx || !dx || !params)
    return set_error(Z4C_EINVAL, "z4c_rhs_noalloc: null argument");
  if (u == rhs) return set_error(Z4C_EINVAL, "z4c_rhs_noalloc: u and rhs must differ");
  if (nblocks < 1) return set_error(Z4C_EINVAL, "z4c_rhs_noalloc: nblocks < 1");
  for (int a = 0; a < 3; ++a) {
    if (nx[a] < 2 * Z4C_NG)
      return set_error(Z4C_EINVAL, "z4c_rhs_noalloc: nx below 2*ng on some axis");
    if (!(dx[a] > 0.0)) return set_error(Z4C_EINVAL, "z4c_rhs_noalloc: dx must be positive");
  }
  Grid g{};
  for (int a = 0; a < 3; ++a) {
    g.nx[a] = nx[a];
    g.nn[a] = nx[a] + 1 + 2 * Z4C_NG;
  }
  g.s[0] = 1;
  g.s[1] = g.nn[0];
  g.s[2] = (int64_t)g.nn[0] * g.nn[1];
  g.nvol = (int64_t)g.nn[0] * g.nn[1] * g.nn[2];
  const int64_t npts = interior_count(g);
  // scratch per block: 33 stored first derivatives per vertex, 6 Ricci sums
  // and 22 advection sums per interior vertex
  const size_t per_block = sizeof(double) * (kSdComponents * (size_t)g.nvol + 28 * (size_t)npts);
  const size_t room = kScratchBytes - kFdBytes;
  if (per_block > room) {
    char buf[256];
    snprintf(buf, sizeof(buf),
             "z4c_rhs_noalloc: one MeshBlock of %dx%dx%d cells needs %zu bytes of scratch, "
             "above the %zu available in the fixed %d MiB array",
             nx[0], nx[1], nx[2], per_block, room, (int)Z4C_NOALLOC_SCRATCH_MIB);
    return set_error(Z4C_EINVAL, buf);
  }
  int chunk = (int)(room / per_block);
  if (chunk > kMaxFd) chunk = kMaxFd;
  if (chunk > nblocks) chunk = nblocks;

  // a launch failure is read back with cudaGetLastError below; an error left
  // pending by earlier, unrelated work must not be reported as this call's
  {
    const cudaError_t prior = cudaPeekAtLastError();
    if (prior != cudaSuccess) {
      char buf[200];
      snprintf(buf, sizeof(buf),
               "z4c_rhs_noalloc: a CUDA error from earlier work is pending (%s); nothing was "
               "enqueued", cudaGetErrorString(prior));
      return set_error(Z4C_ECUDA, buf);
    }
  }
  double* base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  FdScale* fd = reinterpret_cast<FdScale*>(base);
  RhsScratch sc;
  sc.sd = base + kFdBytes / sizeof(double);
  sc.rsum = sc.sd + (size_t)kSdComponents * g.nvol * chunk;
  sc.lv = sc.rsum + (size_t)6 * npts * chunk;

  // FD scalings of finite_differencing.tpp:20-56, as z4c_create computes them
  FdScale f;
  const double diss_scaling = -1.0 / 256.0;  // 2^(-2*4) * (-1): NGHOST = 4 is even
  for (int a = 0; a < 3; ++a) {
    f.cidx1[a] = 1.0 / (dx[a] * 60.0);
    f.cidx2[a] = ((1.0 / dx[a]) * (1.0 / dx[a])) / 180.0;
    f.cidxd[a] = diss_scaling / (dx[a] * 1.0);
    f.lidx[a] = 1.0 / (dx[a] * 60.0);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_fill_fd<<<(chunk + 127) / 128, 128, 0, st>>>(fd, f, chunk);
  add_kernel_launches(1);
  DevParams P;
  P.p = *params;
  P.fd = fd;
  P.xf = nullptr;  // no Sommerfeld faces: the grid below is periodic
  P.dx = nullptr;
  P.som = nullptr;
  const size_t bstride = (size_t)Z4C_NVAR * g.nvol;
  for (int b0 = 0; b0 < nblocks; b0 += chunk) {
    const int nb = (nblocks - b0 < chunk) ? nblocks - b0 : chunk;
    g.nb[0] = nb;
    g.nb[1] = g.nb[2] = 1;
    g.nblocks = nb;
    launch_rhs(g, P, u + bstride * b0, sc, rhs + bstride * b0, 0, nb, LaunchShape(), st);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char buf[160];
    snprintf(buf, sizeof(buf), "z4c_rhs_noalloc launch: %s", cudaGetErrorString(e));
    return set_error(Z4C_ECUDA, buf);
  }
  return Z4C_OK;
}

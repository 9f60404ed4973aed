// aphid_noalloc.cu -- an operator apply that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code running inside a memory pool or a
// framework allocator that owns all device memory, drivers that must not
// allocate once a run has started, and hosts with no allocator of their own.
// For them, aphid_gpu_inprod_eps_noalloc runs the same operator kernel as
// aphid_gpu_inprod_dev (q = K p with epsilon = p^T q reduced on the device)
// without a context: every input and output is a caller-owned device
// pointer, and the kernel's scratch (coefficient tables, per-block partial
// sums and the last-block ticket) lives in one file-scope __device__ array.
//
// That array is loaded with the library and held by every GPU that uses it
// until the process exits.  All calls share it and it keeps the contents of
// the last call: calls that overlap on the GPU (different streams, or
// different host threads on the same device) race on it.  Every call looks up
// the array's device address in the current context (cudaGetSymbolAddress, a
// host-side lookup), so a context made after cudaDeviceReset, or another
// context current on the device, gets its own copy's address.  The first call
// on a device also loads the library's kernels there: make it before any
// stream capture.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/aphid_gpu.h"
#include "aphid_qmr64.cuh"

using namespace aphid;

namespace {

constexpr int kMaxNodes = APHID_NOALLOC_MAX_NODES;  // per axis
constexpr int kMaxSlots = APHID_NOALLOC_MAX_SLOTS;  // reduction partials
constexpr size_t kAxisStride = 6 * (size_t)(kMaxNodes + 1);
constexpr size_t kPartOff = 3 * kAxisStride;
constexpr size_t kCntOff = kPartOff + 2 * (size_t)kMaxSlots;
constexpr size_t kScratchDoubles = kCntOff + 2;

// tables (3 axes) | partials (2 doubles per slot) | ticket counter
static __device__ __align__(256) double g_scratch[kScratchDoubles];

// Coefficient tables of one axis into the scratch, the same formulas as the
// context path's host-side tables (gen_inprod_*_coefs, src/aphid.f90:750-1185):
// layout d[n+1] dc[n] e2[n-1] e3[n-1] n4[n] n5[n].
__global__ void k_noalloc_tables(const double *__restrict__ dx, const double *__restrict__ dy,
                                 const double *__restrict__ dz, const double *__restrict__ dxc,
                                 const double *__restrict__ dyc, const double *__restrict__ dzc,
                                 int nx, int ny, int nz, double *scratch) {
  const int a = blockIdx.x;
  const int n = a == 0 ? nx : (a == 1 ? ny : nz);
  const double *d = a == 0 ? dx : (a == 1 ? dy : dz);
  const double *dc = a == 0 ? dxc : (a == 1 ? dyc : dzc);
  double *t = scratch + a * kAxisStride;
  for (int m = threadIdx.x; m <= n; m += blockDim.x) {
    t[m] = d[m];
    if (m < n) {
      t[(n + 1) + m] = dc[m];
      t[(n + 1) + n + 2 * (n - 1) + m] = mask_hi(m + 1, n) / d[m + 1] / dc[m];
      t[(n + 1) + n + 2 * (n - 1) + n + m] = mask_lo(m + 1, n) / d[m] / dc[m];
    }
    if (m < n - 1) {
      t[(n + 1) + n + m] = mask_hi(m + 1, n - 1) / dc[m + 1] / d[m + 1];
      t[(n + 1) + n + (n - 1) + m] = mask_lo(m + 1, n) / dc[m] / d[m + 1];
    }
  }
}

}  // namespace

extern "C" int aphid_gpu_inprod_eps_noalloc(int nx, int ny, int nz, const double *d_dx,
                                            const double *d_dy, const double *d_dz,
                                            const double *d_dxc, const double *d_dyc,
                                            const double *d_dzc, const void *d_k2,
                                            const void *d_in, void *d_out, void *d_eps,
                                            void *stream) {
  if (nx < 3 || ny < 3 || nz < 3 || nx > kMaxNodes || ny > kMaxNodes || nz > kMaxNodes)
    return APHID_ERR_BADARG;  // beyond the fixed scratch: APHID_NOALLOC_MAX_NODES per axis
  if (!d_dx || !d_dy || !d_dz || !d_dxc || !d_dyc || !d_dzc || !d_k2 || !d_in || !d_out || !d_eps)
    return APHID_ERR_BADARG;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return APHID_ERR_NODEVICE;
  }
  // the array's address in the context current now (host code cannot use
  // the symbol itself: its host-side name is not a device address)
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return APHID_ERR_CUDA;
  }
  double *scratch = (double *)p;
  cudaStream_t st = (cudaStream_t)stream;

  GridDev g{};
  const int dims[3] = {nx, ny, nz};
  for (int a = 0; a < 3; a++) {
    const int m = dims[a];
    const double *b = scratch + a * kAxisStride;
    g.ax[a].n = m;
    g.ax[a].d = b;
    g.ax[a].dc = b + (m + 1);
    g.ax[a].e2 = b + (m + 1) + m;
    g.ax[a].e3 = b + (m + 1) + m + (m - 1);
    g.ax[a].n4 = b + (m + 1) + m + 2 * (m - 1);
    g.ax[a].n5 = b + (m + 1) + m + 2 * (m - 1) + m;
  }
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.ox = 0;
  g.oy = (long long)(nx - 1) * ny * nz;
  g.oz = g.oy + (long long)nx * (ny - 1) * nz;
  g.op = g.oz + (long long)nx * ny * (nz - 1);
  g.n = g.op + (long long)nx * ny * nz;

  // tiles bounded by the scratch's partial-sum slots
  Tiles t{};
  t.ti = (nx + kTileI - 1) / kTileI;
  t.tj = (ny + kTileJ - 1) / kTileJ;
  const long long cols = (long long)t.ti * t.tj;  // <= 32 * 256 < kMaxSlots
  long long kz = std::min<long long>(32, std::max<long long>(1, cols * nz / (148 * 8)));
  kz = std::max<long long>(kz, (cols * nz + kMaxSlots - 1) / kMaxSlots);
  t.kz = (int)kz;
  t.tk = (nz + t.kz - 1) / t.kz;
  if (t.count() > kMaxSlots) return APHID_ERR_BADARG;

  unsigned *cnt = (unsigned *)(scratch + kCntOff);
  // the ticket counter must start at zero (an earlier failed launch may have
  // left it armed)
  if (cudaMemsetAsync(cnt, 0, sizeof(unsigned), st) != cudaSuccess) return APHID_ERR_CUDA;
  k_noalloc_tables<<<3, 256, 0, st>>>(d_dx, d_dy, d_dz, d_dxc, d_dyc, d_dzc, nx, ny, nz, scratch);
  k_apply64<kApplyEps><<<(unsigned)t.count(), kOpThreads, 0, st>>>(
      g, t, (const double2 *)d_k2, (const double2 *)d_in, (double2 *)d_out, nullptr,
      (double2 *)d_eps, scratch + kPartOff, cnt);
  if (cudaGetLastError() != cudaSuccess) return APHID_ERR_CUDA;
  return APHID_OK;
}

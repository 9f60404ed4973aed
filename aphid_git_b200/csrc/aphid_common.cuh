// aphid_common.cuh -- complex helpers, grid descriptor and deterministic
// two-stage reductions shared by the APhiD kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace aphid {

// ---------------------------------------------------------------- complex
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 rmul(double r, double2 b) { return make_double2(r * b.x, r * b.y); }
__device__ __forceinline__ double2 rdiv(double2 a, double r) { return make_double2(a.x / r, a.y / r); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
// Smith's complex division (the range-reduced form Fortran compilers use).
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, den = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  }
  double r = b.x / b.y, den = b.x * r + b.y;
  return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}
// Uncontracted complex a*b - c*d pieces: the same value wherever computed.
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 csub_rn(double2 a, double2 b) {
  return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}

__device__ __forceinline__ float2 fadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 fsub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 fmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 fscale(float r, float2 b) { return make_float2(r * b.x, r * b.y); }

// ------------------------------------------------------------------ grid
// One axis of the tensor-product mesh.  Tables are indexed 0-based:
//   d[m]   = dx(m)     for m = 0..n     (the reference's dx(0:n))
//   dc[m]  = dxc(m+1)  for m = 0..n-1   (dual lengths at nodes)
//   e2,e3  : coef_2vec/coef_3vec of the component ALONG this axis, per edge
//            e = 0..n-2 (src/aphid.f90:787-795, 905-913, 1044-1052)
//   n4,n5  : coef_4..7vec of components ACROSS this axis and of the node
//            block, per node m = 0..n-1 (src/aphid.f90:767-785, 1152-1183)
struct Axis {
  const double *d, *dc, *e2, *e3, *n4, *n5;
  int n;
};

struct GridDev {
  Axis ax[3];
  int nx, ny, nz;
  long long ox, oy, oz, op, n;  // block offsets in the [Ax|Ay|Az|Phi] vector
};

__device__ __forceinline__ long long ixx(const GridDev &g, int i, int j, int k) {
  return g.ox + i + (long long)(g.nx - 1) * (j + (long long)g.ny * k);
}
__device__ __forceinline__ long long ixy(const GridDev &g, int i, int j, int k) {
  return g.oy + i + (long long)g.nx * (j + (long long)(g.ny - 1) * k);
}
__device__ __forceinline__ long long ixz(const GridDev &g, int i, int j, int k) {
  return g.oz + i + (long long)g.nx * (j + (long long)g.ny * k);
}
__device__ __forceinline__ long long ixp(const GridDev &g, int i, int j, int k) {
  return g.op + i + (long long)g.nx * (j + (long long)g.ny * k);
}

// ------------------------------------------------------------- reductions
// Deterministic two-stage sums: every block reduces in a fixed tree order
// and writes one partial; the last block to arrive (atomic ticket) sums the
// partials in a fixed order.  Same grid => bitwise-identical results.
template <int NV>
struct Vals {
  double v[NV];
};

template <int NV, int NT>
__device__ __forceinline__ Vals<NV> block_reduce(Vals<NV> a) {
  __shared__ double sh[NT / 32][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < NV; c++) {
#pragma unroll
    for (int o = 16; o; o >>= 1) a.v[c] += __shfl_xor_sync(0xffffffffu, a.v[c], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < NV; c++) sh[w][c] = a.v[c];
  }
  __syncthreads();
  Vals<NV> r;
#pragma unroll
  for (int c = 0; c < NV; c++) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < NT / 32; q++) s += sh[q][c];
    r.v[c] = s;
  }
  __syncthreads();
  return r;  // valid in every thread
}

// Stores this block's partial, returns true in the last-arriving block of the
// slot range; that block then calls final_reduce().
template <int NV, int NT>
__device__ __forceinline__ bool arrive(Vals<NV> blk, double *partials, unsigned *counter,
                                       unsigned slot, unsigned nslots) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < NV; c++) partials[(size_t)slot * NV + c] = blk.v[c];
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    last = (t == nslots - 1);
  }
  __syncthreads();
  return last;
}

template <int NV, int NT>
__device__ __forceinline__ Vals<NV> final_reduce(const double *partials, unsigned *counter,
                                                 unsigned nslots) {
  __threadfence();
  Vals<NV> a;
#pragma unroll
  for (int c = 0; c < NV; c++) a.v[c] = 0.0;
  for (unsigned s = threadIdx.x; s < nslots; s += NT) {
#pragma unroll
    for (int c = 0; c < NV; c++) a.v[c] += __ldcg(partials + (size_t)s * NV + c);
  }
  Vals<NV> r = block_reduce<NV, NT>(a);
  if (threadIdx.x == 0) *counter = 0u;  // re-arm for the next launch
  return r;
}

}  // namespace aphid

namespace aphid {
// float2 counterparts of the complex helpers (complex64 inner solver)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 rmul(float r, float2 b) { return make_float2(r * b.x, r * b.y); }
__device__ __forceinline__ float2 rdiv(float2 a, float r) { return make_float2(a.x / r, a.y / r); }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
__device__ __forceinline__ float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }

template <typename R> struct CplxOf;
template <> struct CplxOf<float> { using T = float2; };
template <> struct CplxOf<double> { using T = double2; };
template <typename R>
__device__ __forceinline__ typename CplxOf<R>::T mkc(R a, R b);
template <> __device__ __forceinline__ float2 mkc<float>(float a, float b) { return make_float2(a, b); }
template <> __device__ __forceinline__ double2 mkc<double>(double a, double b) { return make_double2(a, b); }
}  // namespace aphid

// aphid_sweep.cuh -- batched, mixed-precision frequency sweep.
//
// S systems (frequency x source) on one mesh advance together.  Each system
// runs FP64 defect correction (iterative refinement):
//   r = b - K x        complex128 operator, true residual, FP64 norms
//   solve K e = r      complex64 QMR on the symmetrically Jacobi-scaled
//                      operator K~ = D^-1/2 K D^-1/2 (D = gen_diag), FP64
//                      inner products and Lanczos scalars
//   x += D^-1/2 e~     FP64 accumulation
// until ||r|| < target ||b||.  The Jacobi diagonal is FP64; its inverse square
// root is stored once per system in complex64.  k^2 is never stored: it is
// formed per system from the FP64 cell averages sigma-bar (and eps-bar) shared
// by all systems, k^2 = i omega mu0 (sigma-bar + i omega eps0 eps-bar), which
// is gen_k2_*grid (src/aphid.f90:1289-1535) for the linear models R, C, I.
//
// Layout: x and b stay complex128 in the reference's [Ax|Ay|Az|Phi] order.
// The complex64 inner state (v~, p~, q~, d~, x~, D^-1/2) is node-indexed:
// [system][component][k][j][i] with rows padded to a multiple of 4 nodes, so
// all four components of a node share one index, every row starts on a
// 16-byte boundary (TMA-loadable), and components that do not exist at a
// node (x at i = nx-1, ...) are stored zeros.
//
// The inner solver is the reference's coupled two-term QMR recurrence
// (src/aphid_qmr.f90:297-372) with M = I on K~, two kernels per iteration:
//   A  q~_n = K~ p~_n with p~_n = v~_n - k1 p~_{n-1} formed on the fly,
//      epsilon_n = p~_n^T q~_n (= u^T K u with u = D^-1/2 p~_n);
//   B  p~_n stored; vt = q~_n - beta_n v~_n stored unnormalised (v~_{n+1} =
//      vt / rho_{n+1} is applied lazily through a scale factor), ||vt||^2
//      and vt^T vt reduced; d~ and x~ updated one iteration late, because
//      eta_n needs rho_{n+1} from this very reduction.
// It keeps no residual vectors (r, s): the stop test uses the quasi-residual
// norm tau_n = ||r~_0|| prod sqrt(theta_i c_i), an estimate that a
// complex128 true-residual monitor checks once per graph round.
//
// Every system has a phase (OUTER -> INNER -> OUTER ... -> DONE);
// every block first reads its system's phase and returns when the kernel does
// not apply, which masks converged systems out of the remaining launches.
#pragma once
#include <cuda.h>

#include "aphid_qmr64.cuh"

namespace aphid {

enum { PH_OUTER = 0, PH_INNER = 2, PH_DONE = 3 };
enum { CNT_RESID = 0, CNT_APPLY = 2, CNT_UPDATE = 3, CNT_BNORM = 4, CNT_CHECK = 5, CNT_KINDS = 6 };

// An inner cycle ends when the true residual, checked once per graph round,
// falls this far behind its best tracking of the quasi-residual: the complex64
// recurrence has reached its floor and only a restart from the FP64 residual
// makes progress.
constexpr double kStagnation = 16.0;

struct SweepSys {
  double omega, ka, kb;  // k^2 = (-ka * eps-bar, kb * sigma-bar)
  double rho_n, rho_np, c_n, c_nm, theta_n, theta_nm, kap, tau, tau0;
  double2 eps, del, beta, eta, k1;
  double vscale;             // v~_n = vscale * (stored vt)
  double2 eta_pend;          // pending lagged update d = eta p + kap d
  double kap_pend;
  double bnorm, rnorm, inner_tol, target, rt0;
  double ratio_min, mon_rn;  // true-residual monitor of the running inner cycle
  int phase, has_inner, inner_it, total_it, outer_it, max_it, max_outer, status;
  int checks, pending;
};

// plane tile of the complex64 operator pass: 16 x 16 nodes marching along k;
// staged planes cover i0-2 .. i0+17 (20, even start: 16-byte TMA x origin)
// and j0-1 .. j0+16 (18); sigma-bar planes cover i0-4 .. i0+19 (24).
constexpr int kPTI = 16, kPTJ = 16, kPThreads = kPTI * kPTJ;
constexpr int kPW = kPTI + 4, kPH = kPTJ + 2, kPN = kPW * kPH;   // 20 x 18
constexpr int kKW = kPTI + 8, kKN = kKW * kPH;                    // 24 x 18

struct NodeLayout {
  int nxp;      // padded row length (multiple of 4)
  long long N;  // nodes per component: nxp * ny * nz
};

struct SweepDev {
  GridDev g;
  NodeLayout L;
  Tiles t;   // 32 x 4 column tiles (complex128 residual passes)
  Tiles tp;  // 16 x 16 plane tiles (complex64 operator pass)
  long long n;           // unknowns per system (reference layout)
  int nsys, bps;         // systems; blocks per system of the pointwise kernels
  long long slots;       // partial-sum slots per system
  const double *sig;     // sigma-bar per unknown (FP64, reference layout)
  const double *epsr;    // eps-bar per unknown, or null (= 1)
  const float *sig32, *epsr32;    // the same, FP32, node layout [4][N]
  float2 *v, *p, *q, *d, *x, *s;  // [nsys][4][N] complex64, node layout (v holds vt)
  double2 *x64, *b;               // [nsys][n] complex128, reference layout
  SweepSys *sys;
  double *part;                   // [nsys][slots][6]
  unsigned *cnt;                  // [CNT_KINDS][nsys]
  int *ndone;
  int *err;                       // set when a bounded wait gives up
};

__device__ __forceinline__ long long nd_of(const SweepDev &D, int i, int j, int k) {
  return i + (long long)D.L.nxp * (j + (long long)D.g.ny * k);
}
__device__ __forceinline__ bool exists(const GridDev &g, int c, int i, int j, int k) {
  return c == 0 ? i < g.nx - 1 : (c == 1 ? j < g.ny - 1 : (c == 2 ? k < g.nz - 1 : true));
}
__device__ __forceinline__ long long ref_of(const GridDev &g, int c, int i, int j, int k) {
  return c == 0 ? ixx(g, i, j, k) : (c == 1 ? ixy(g, i, j, k) : (c == 2 ? ixz(g, i, j, k) : ixp(g, i, j, k)));
}

// --------------------------------------------------- generic stencil rows
// The rows of rows64 for any precision R, with neighbours addressed as
// (component, i, j, k) so the same code reads either layout; neighbour
// indices are clamped as in the reference (their coefficients are zero
// where the clamp applies).
template <typename R, class IN, class KK>
__device__ __forceinline__ void rowsN(const GridDev &g, int i, int j, int k, const IN &in, const KK &kk,
                                      typename CplxOf<R>::T o[4]) {
  using C = typename CplxOf<R>::T;
  const Axis &X = g.ax[0], &Y = g.ax[1], &Z = g.ax[2];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const R xn4 = (R)X.n4[i], xn5 = (R)X.n5[i], yn4 = (R)Y.n4[j], yn5 = (R)Y.n5[j];
  const R zn4 = (R)Z.n4[k], zn5 = (R)Z.n5[k];
  const R dxc = (R)X.dc[i], dyc = (R)Y.dc[j], dzc = (R)Z.dc[k];
  const int ia = min(i + 1, nx - 1), ib = max(i - 1, 0);
  const int ja = min(j + 1, ny - 1), jb = max(j - 1, 0);
  const int ka = min(k + 1, nz - 1), kb = max(k - 1, 0);
  const C phc = in(3, i, j, k), kpc = kk(3, i, j, k);
  o[0] = o[1] = o[2] = o[3] = mkc<R>((R)0, (R)0);
  if (i < nx - 1) {
    const R c2 = (R)X.e2[i], c3 = (R)X.e3[i], dxi = (R)X.d[i + 1];
    const R vol = dxi * dyc * dzc;
    const C k2 = kk(0, i, j, k), kp2 = kk(3, i + 1, j, k);
    const R sum = c2 + c3 + yn4 + yn5 + zn4 + zn5;
    C s = cmul(mkc<R>(-sum + k2.x, k2.y), in(0, i, j, k));
    s = cadd(s, rmul(c2, in(0, min(i + 1, nx - 2), j, k)));
    s = cadd(s, rmul(c3, in(0, ib, j, k)));
    s = cadd(s, rmul(yn4, in(0, i, ja, k)));
    s = cadd(s, rmul(yn5, in(0, i, jb, k)));
    s = cadd(s, rmul(zn4, in(0, i, j, ka)));
    s = cadd(s, rmul(zn5, in(0, i, j, kb)));
    const C gr = rdiv(csub(cmul(in(3, i + 1, j, k), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dxi);
    o[0] = rmul(vol, cadd(s, gr));
  }
  if (j < ny - 1) {
    const R c2 = (R)Y.e2[j], c3 = (R)Y.e3[j], dyj = (R)Y.d[j + 1];
    const R vol = dxc * dyj * dzc;
    const C k2 = kk(1, i, j, k), kp2 = kk(3, i, j + 1, k);
    const R sum = c2 + c3 + xn4 + xn5 + zn4 + zn5;
    C s = cmul(mkc<R>(-sum + k2.x, k2.y), in(1, i, j, k));
    s = cadd(s, rmul(c2, in(1, i, min(j + 1, ny - 2), k)));
    s = cadd(s, rmul(c3, in(1, i, jb, k)));
    s = cadd(s, rmul(xn4, in(1, ia, j, k)));
    s = cadd(s, rmul(xn5, in(1, ib, j, k)));
    s = cadd(s, rmul(zn4, in(1, i, j, ka)));
    s = cadd(s, rmul(zn5, in(1, i, j, kb)));
    const C gr = rdiv(csub(cmul(in(3, i, j + 1, k), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dyj);
    o[1] = rmul(vol, cadd(s, gr));
  }
  if (k < nz - 1) {
    const R c2 = (R)Z.e2[k], c3 = (R)Z.e3[k], dzk = (R)Z.d[k + 1];
    const R vol = dxc * dyc * dzk;
    const C k2 = kk(2, i, j, k), kp2 = kk(3, i, j, k + 1);
    const R sum = c2 + c3 + xn4 + xn5 + yn4 + yn5;
    C s = cmul(mkc<R>(-sum + k2.x, k2.y), in(2, i, j, k));
    s = cadd(s, rmul(c2, in(2, i, j, min(k + 1, nz - 2))));
    s = cadd(s, rmul(c3, in(2, i, j, kb)));
    s = cadd(s, rmul(xn4, in(2, ia, j, k)));
    s = cadd(s, rmul(xn5, in(2, ib, j, k)));
    s = cadd(s, rmul(yn4, in(2, i, ja, k)));
    s = cadd(s, rmul(yn5, in(2, i, jb, k)));
    const C gr = rdiv(csub(cmul(in(3, i, j, k + 1), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dzk);
    o[2] = rmul(vol, cadd(s, gr));
  }
  if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) {
    const R vol = dxc * dyc * dzc;
    const C s1 = kpc;
    const C s2 = kk(0, i, j, k), s3 = kk(0, i - 1, j, k), s4 = kk(1, i, j, k), s5 = kk(1, i, j - 1, k);
    const C s6 = kk(2, i, j, k), s7 = kk(2, i, j, k - 1);
    const C c2 = rmul(xn4, s2), c3 = rmul(xn5, s3), c4 = rmul(yn4, s4);
    const C c5 = rmul(yn5, s5), c6 = rmul(zn4, s6), c7 = rmul(zn5, s7);
    const C sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
    C s = cmul(cadd(cneg(sum), cmul(s1, s1)), phc);
    s = cadd(s, cmul(c2, in(3, i + 1, j, k)));
    s = cadd(s, cmul(c3, in(3, i - 1, j, k)));
    s = cadd(s, cmul(c4, in(3, i, j + 1, k)));
    s = cadd(s, cmul(c5, in(3, i, j - 1, k)));
    s = cadd(s, cmul(c6, in(3, i, j, k + 1)));
    s = cadd(s, cmul(c7, in(3, i, j, k - 1)));
    C t = cmul(rdiv(csub(s2, s1), dxc), in(0, i, j, k));
    t = cadd(t, cmul(cneg(rdiv(csub(s3, s1), dxc)), in(0, i - 1, j, k)));
    t = cadd(t, cmul(rdiv(csub(s4, s1), dyc), in(1, i, j, k)));
    t = cadd(t, cmul(cneg(rdiv(csub(s5, s1), dyc)), in(1, i, j - 1, k)));
    t = cadd(t, cmul(rdiv(csub(s6, s1), dzc), in(2, i, j, k)));
    t = cadd(t, cmul(cneg(rdiv(csub(s7, s1), dzc)), in(2, i, j, k - 1)));
    o[3] = cadd(rmul(vol, s), rmul(vol, t));
  }
}

// complex128 accessors of the outer passes
struct K2Ref64 {  // k^2 from the FP64 averages (reference layout)
  GridDev g;
  const double *__restrict__ sig, *__restrict__ epsr;
  double ka, kb;
  __device__ __forceinline__ double2 operator()(int c, int i, int j, int k) const {
    const long long t = ref_of(g, c, i, j, k);
    const double e = epsr ? __ldg(epsr + t) : 1.0;
    return make_double2(-ka * e, kb * __ldg(sig + t));
  }
};
struct XRef64 {  // x (reference layout), optionally + D^-1/2 x~ (node layout)
  GridDev g;
  const double2 *__restrict__ x64;
  const float2 *__restrict__ s, *__restrict__ xt;  // null: x only
  int nxp;
  long long N;
  __device__ __forceinline__ double2 operator()(int c, int i, int j, int k) const {
    double2 r = __ldg(x64 + ref_of(g, c, i, j, k));
    if (xt) {
      const long long t = c * N + i + (long long)nxp * (j + (long long)g.ny * k);
      r = cadd(r, cmul(to_d(__ldg(s + t)), to_d(__ldg(xt + t))));
    }
    return r;
  }
};

// p~_n = vscale * vt - k1 p~_{n-1}, uncontracted so that the operator pass and
// the update pass compute the same value
__device__ __forceinline__ float2 vn32(float2 vt, float sc) {
  return make_float2(__fmul_rn(sc, vt.x), __fmul_rn(sc, vt.y));
}
__device__ __forceinline__ float2 pnew32(float2 v, float2 p, float2 k1) {
  const float re = __fsub_rn(__fmul_rn(k1.x, p.x), __fmul_rn(k1.y, p.y));
  const float im = __fadd_rn(__fmul_rn(k1.x, p.y), __fmul_rn(k1.y, p.x));
  return make_float2(__fsub_rn(v.x, re), __fsub_rn(v.y, im));
}

__device__ __forceinline__ void sweep_tile(const SweepDev &D, long long tile, int &i, int &j, int &k0,
                                           int &k1) {
  long long b = tile;
  const int bi = (int)(b % D.t.ti);
  b /= D.t.ti;
  const int bj = (int)(b % D.t.tj);
  const int bk = (int)(b / D.t.tj);
  i = bi * kTileI + (threadIdx.x & 31);
  j = bj * kTileJ + (threadIdx.x >> 5);
  k0 = bk * D.t.kz;
  k1 = min(D.g.nz, k0 + D.t.kz);
}

__device__ __forceinline__ void mark_done(const SweepDev &D, SweepSys *S, int status) {
  S->status = status;
  S->phase = PH_DONE;
  atomicAdd(D.ndone, 1);
}

// ---------------------------------------------------------------- setup
// sigma-bar / eps-bar per unknown: the area- and volume-weighted cell
// averages of gen_k2_*grid before the factor i omega mu0, boundary values
// from the clamped interior index (src/aphid.f90:1289-1535).
static __global__ void k_sw_avg(GridDev g, const float *__restrict__ cell, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz, cx = nx - 1, cy = ny - 1;
  const double *dx = g.ax[0].d, *dy = g.ax[1].d, *dz = g.ax[2].d;
  auto S = [&](int a, int b, int c) { return (double)__ldg(cell + a + (long long)cx * (b + (long long)cy * c)); };
  const int ii = min(max(i, 1), nx - 2), jj = min(max(j, 1), ny - 2), kk = min(max(k, 1), nz - 2);
  if (i < nx - 1) {
    const double dyj = dy[jj + 1], dyjm = dy[jj], dzk = dz[kk + 1], dzkm = dz[kk];
    double s = S(i, jj - 1, kk - 1) * (dyjm * dzkm);
    s += S(i, jj, kk - 1) * (dyj * dzkm);
    s += S(i, jj, kk) * (dyj * dzk);
    s += S(i, jj - 1, kk) * (dyjm * dzk);
    out[ixx(g, i, j, k)] = s / ((dyjm + dyj) * (dzkm + dzk));
  }
  if (j < ny - 1) {
    const double dxi = dx[ii + 1], dxim = dx[ii], dzk = dz[kk + 1], dzkm = dz[kk];
    double s = S(ii - 1, j, kk - 1) * (dxim * dzkm);
    s += S(ii, j, kk - 1) * (dxi * dzkm);
    s += S(ii, j, kk) * (dxi * dzk);
    s += S(ii - 1, j, kk) * (dxim * dzk);
    out[ixy(g, i, j, k)] = s / ((dxim + dxi) * (dzkm + dzk));
  }
  if (k < nz - 1) {
    const double dxi = dx[ii + 1], dxim = dx[ii], dyj = dy[jj + 1], dyjm = dy[jj];
    double s = S(ii - 1, jj - 1, k) * (dxim * dyjm);
    s += S(ii, jj - 1, k) * (dxi * dyjm);
    s += S(ii, jj, k) * (dxi * dyj);
    s += S(ii - 1, jj, k) * (dxim * dyj);
    out[ixz(g, i, j, k)] = s / ((dxim + dxi) * (dyjm + dyj));
  }
  {
    const double dxi = dx[ii + 1], dxim = dx[ii], dyj = dy[jj + 1], dyjm = dy[jj];
    const double dzk = dz[kk + 1], dzkm = dz[kk];
    double s = S(ii - 1, jj - 1, kk) * (dxim * dyjm * dzk);
    s += S(ii, jj - 1, kk) * (dxi * dyjm * dzk);
    s += S(ii, jj, kk) * (dxi * dyj * dzk);
    s += S(ii - 1, jj, kk) * (dxim * dyj * dzk);
    s += S(ii - 1, jj - 1, kk - 1) * (dxim * dyjm * dzkm);
    s += S(ii, jj - 1, kk - 1) * (dxi * dyjm * dzkm);
    s += S(ii, jj, kk - 1) * (dxi * dyj * dzkm);
    s += S(ii - 1, jj, kk - 1) * (dxim * dyj * dzkm);
    out[ixp(g, i, j, k)] = s / ((dxim + dxi) * (dyjm + dyj) * (dzkm + dzk));
  }
}

// k^2 from the FP64 averages at a reference-layout index
struct K2Avg64 {
  const double *__restrict__ sig, *__restrict__ epsr;
  double ka, kb;
  __device__ __forceinline__ double2 operator()(long long t) const {
    const double e = epsr ? __ldg(epsr + t) : 1.0;
    return make_double2(-ka * e, kb * __ldg(sig + t));
  }
};

// complex128 k^2 vector of one system from the averages (for the complex128
// sweep, which runs the reference's own algorithm on it)
static __global__ void k_sw_k2vec(long long n, const double *__restrict__ sig, const double *__restrict__ epsr,
                                  double ka, double kb, double2 *__restrict__ k2) {
  const K2Avg64 K{sig, epsr, ka, kb};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    k2[t] = K(t);
}


// ||b|| per system
static __global__ void __launch_bounds__(kStreamThreads) k_sw_bnorm(SweepDev D) {
  const int sys = blockIdx.x % D.nsys, chunk = blockIdx.x / D.nsys;
  const double2 *b = D.b + (long long)sys * D.n;
  Vals<1> a{{0.0}};
  for (long long t = chunk * (long long)blockDim.x + threadIdx.x; t < D.n; t += (long long)D.bps * blockDim.x)
    a.v[0] += cabs2(b[t]);
  Vals<1> blk = block_reduce<1, kStreamThreads>(a);
  double *part = D.part + (size_t)sys * D.slots * 6;
  if (arrive<1, kStreamThreads>(blk, part, D.cnt + CNT_BNORM * D.nsys + sys, chunk, D.bps)) {
    Vals<1> tot = final_reduce<1, kStreamThreads>(part, D.cnt + CNT_BNORM * D.nsys + sys, D.bps);
    if (threadIdx.x == 0) {
      SweepSys *S = D.sys + sys;
      S->bnorm = sqrt(tot.v[0]);
      if (!(S->bnorm > 0.0)) mark_done(D, S, 2);  // zero source: nothing to solve
    }
  }
}

// reference-layout FP64 per-unknown array -> node-layout FP32 [4][N]
// (zero where a component does not exist; pads are left as initialised)
static __global__ void k_sw_to_node32(GridDev g, NodeLayout L, const double *__restrict__ ref,
                                      float *__restrict__ node) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const long long nd = i + (long long)L.nxp * (j + (long long)g.ny * k);
#pragma unroll
  for (int c = 0; c < 4; c++)
    node[c * L.N + nd] = exists(g, c, i, j, k) ? (float)ref[ref_of(g, c, i, j, k)] : 0.f;
}

// principal complex square root, then its reciprocal
__device__ __forceinline__ double2 cinvsqrt(double2 z) {
  const double m = hypot(z.x, z.y);
  double2 r;
  if (z.x >= 0.0) {
    const double t = sqrt(0.5 * (m + z.x));
    r = make_double2(t, t > 0 ? z.y / (2.0 * t) : 0.0);
  } else {
    const double t = sqrt(0.5 * (m - z.x));
    r = make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
  }
  return cdiv(make_double2(1.0, 0.0), r);
}

// D^-1/2 per node, component and system from the FP64 Jacobi diagonal
// (gen_diag, src/aphid.f90:1542-1725, with k^2 from the averages)
static __global__ void k_sw_scale(SweepDev D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z % D.g.nz;
  const int sys = blockIdx.z / D.g.nz;
  const GridDev &g = D.g;
  if (i >= g.nx) return;
  const SweepSys &S = D.sys[sys];
  const K2Ref64 K{g, D.sig, D.epsr, S.ka, S.kb};
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double *dx = g.ax[0].d, *dy = g.ax[1].d, *dz = g.ax[2].d;
  const int I = i + 1, J = j + 1, KK = k + 1;
  const double dxi = dx[I], dxim = dx[I - 1], dxci = 0.5 * (dxi + dxim);
  const double dyj = dy[J], dyjm = dy[J - 1], dycj = 0.5 * (dyj + dyjm);
  const double dzk = dz[KK], dzkm = dz[KK - 1], dzck = 0.5 * (dzk + dzkm);
  const double xn4 = mask_hi(I, nx) / dxi / dxci, xn5 = mask_lo(I, nx) / dxim / dxci;
  const double yn4 = mask_hi(J, ny) / dyj / dycj, yn5 = mask_lo(J, ny) / dyjm / dycj;
  const double zn4 = mask_hi(KK, nz) / dzk / dzck, zn5 = mask_lo(KK, nz) / dzkm / dzck;
  float2 *s = D.s + (long long)sys * 4 * D.L.N;
  const long long nd = nd_of(D, i, j, k);
  float2 o[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(1.f, 0.f)};
  if (i < nx - 1) {
    const double c2 = mask_hi(I, nx - 1) / (0.5 * (dxi + dx[I + 1])) / dxi, c3 = mask_lo(I, nx) / dxci / dxi;
    const double2 kv = K(0, i, j, k);
    o[0] = to_f(cinvsqrt(rmul(dxi * dycj * dzck, make_double2(-(c2 + c3 + yn4 + yn5 + zn4 + zn5) + kv.x, kv.y))));
  }
  if (j < ny - 1) {
    const double c2 = mask_hi(J, ny - 1) / (0.5 * (dyj + dy[J + 1])) / dyj, c3 = mask_lo(J, ny) / dycj / dyj;
    const double2 kv = K(1, i, j, k);
    o[1] = to_f(cinvsqrt(rmul(dxci * dyj * dzck, make_double2(-(c2 + c3 + xn4 + xn5 + zn4 + zn5) + kv.x, kv.y))));
  }
  if (k < nz - 1) {
    const double c2 = mask_hi(KK, nz - 1) / (0.5 * (dzk + dz[KK + 1])) / dzk, c3 = mask_lo(KK, nz) / dzck / dzk;
    const double2 kv = K(2, i, j, k);
    o[2] = to_f(cinvsqrt(rmul(dxci * dycj * dzk, make_double2(-(c2 + c3 + xn4 + xn5 + yn4 + yn5) + kv.x, kv.y))));
  }
  if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) {
    const double2 s1 = K(3, i, j, k);
    const double2 c2 = rdiv(rdiv(rmul(mask_hi(I, nx), K(0, i, j, k)), dxi), dxci);
    const double2 c3 = rdiv(rdiv(rmul(mask_lo(I, nx), K(0, i - 1, j, k)), dxim), dxci);
    const double2 c4 = rdiv(rdiv(rmul(mask_hi(J, ny), K(1, i, j, k)), dyj), dycj);
    const double2 c5 = rdiv(rdiv(rmul(mask_lo(J, ny), K(1, i, j - 1, k)), dyjm), dycj);
    const double2 c6 = rdiv(rdiv(rmul(mask_hi(KK, nz), K(2, i, j, k)), dzk), dzck);
    const double2 c7 = rdiv(rdiv(rmul(mask_lo(KK, nz), K(2, i, j, k - 1)), dzkm), dzck);
    const double2 sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
    o[3] = to_f(cinvsqrt(rmul(dxci * dycj * dzck, cadd(cneg(sum), cmul(s1, s1)))));
  }
#pragma unroll
  for (int c = 0; c < 4; c++) s[c * D.L.N + nd] = o[c];
}

// ------------------------------------------------------------ outer step
// O1: x += D^-1/2 (x~ + pending lagged update), FP64 accumulation of the
// inner correction into the reference-layout solution
static __global__ void __launch_bounds__(kStreamThreads) k_sw_xupd(SweepDev D) {
  const int sys = blockIdx.x % D.nsys, chunk = blockIdx.x / D.nsys;
  const SweepSys *S = D.sys + sys;
  if (S->phase != PH_OUTER || !S->has_inner) return;
  const long long vb = (long long)sys * 4 * D.L.N;
  const bool pend = S->pending != 0;
  const double2 eta = S->eta_pend;
  const double kap = S->kap_pend;
  const GridDev &g = D.g;
  const long long plane = (long long)D.L.nxp * g.ny;
  double2 *x64 = D.x64 + (long long)sys * D.n;
  for (long long nd = chunk * (long long)blockDim.x + threadIdx.x; nd < D.L.N;
       nd += (long long)D.bps * blockDim.x) {
    const int k = (int)(nd / plane);
    const long long r = nd - k * plane;
    const int j = (int)(r / D.L.nxp), i = (int)(r - (long long)j * D.L.nxp);
    if (i >= g.nx) continue;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      if (!exists(g, c, i, j, k)) continue;
      const long long t = vb + c * D.L.N + nd;
      double2 xt = to_d(D.x[t]);
      if (pend) xt = cadd(xt, cadd(cmul(eta, to_d(D.p[t])), rmul(kap, to_d(D.d[t]))));
      const long long rt = ref_of(g, c, i, j, k);
      x64[rt] = cadd(x64[rt], cmul(to_d(D.s[t]), xt));
    }
  }
}

// O2: r = b - K x in complex128 (true residual); r~ = D^-1/2 r starts the
// next inner cycle: stored (complex64) as the unnormalised first Lanczos
// vector, p~ = d~ = x~ = 0, and the inner scalars of
// src/aphid_qmr.f90:268-285, 299-313 with M = I.
static __global__ void __launch_bounds__(kOpThreads) k_sw_resid(SweepDev D) {
  const int sys = blockIdx.x % D.nsys;
  const long long tile = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (S->phase != PH_OUTER) return;
  int i, j, k0, k1;
  sweep_tile(D, tile, i, j, k0, k1);
  Vals<4> a{{0.0, 0.0, 0.0, 0.0}};
  if (i < D.g.nx && j < D.g.ny) {
    const XRef64 L{D.g, D.x64 + (long long)sys * D.n, nullptr, nullptr, D.L.nxp, D.L.N};
    const K2Ref64 K{D.g, D.sig, D.epsr, S->ka, S->kb};
    const double2 *b = D.b + (long long)sys * D.n;
    const long long vb = (long long)sys * 4 * D.L.N;
    const float2 zero = make_float2(0.f, 0.f);
    for (int k = k0; k < k1; k++) {
      double2 o[4];
      rowsN<double>(D.g, i, j, k, L, K, o);
      const long long nd = nd_of(D, i, j, k);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const long long t = vb + c * D.L.N + nd;
        float2 rt = zero;
        if (exists(D.g, c, i, j, k)) {
          const double2 r = csub(b[ref_of(D.g, c, i, j, k)], o[c]);
          rt = to_f(cmul(to_d(D.s[t]), r));
          const double2 drt = to_d(rt);
          a.v[0] += cabs2(r);
          a.v[1] += cabs2(drt);
          const double2 sq = cmul(drt, drt);
          a.v[2] += sq.x;
          a.v[3] += sq.y;
        }
        D.v[t] = rt;
        D.p[t] = zero;
        D.d[t] = zero;
        D.x[t] = zero;
      }
    }
  }
  Vals<4> blk = block_reduce<4, kOpThreads>(a);
  double *part = D.part + (size_t)sys * D.slots * 6;
  unsigned *cnt = D.cnt + CNT_RESID * D.nsys + sys;
  const unsigned nt = (unsigned)D.t.count();
  if (arrive<4, kOpThreads>(blk, part, cnt, (unsigned)tile, nt)) {
    Vals<4> tot = final_reduce<4, kOpThreads>(part, cnt, nt);
    if (threadIdx.x == 0) {
      S->rnorm = sqrt(tot.v[0]);
      S->has_inner = 0;
      S->pending = 0;
      if (!isfinite(S->rnorm)) {
        mark_done(D, S, 3);
      } else if (S->rnorm < S->target * S->bnorm) {
        mark_done(D, S, 0);
      } else if (S->outer_it >= S->max_outer || S->total_it >= S->max_it) {
        mark_done(D, S, 1);
      } else {
        S->outer_it++;
        const double rt0 = sqrt(tot.v[1]);
        S->rt0 = rt0;
        S->vscale = 1.0 / rt0;
        S->c_n = 1.0;
        S->eps = make_double2(1.0, 0.0);
        S->theta_n = 0.0;
        S->eta = make_double2(-1.0, 0.0);
        S->rho_np = rt0;
        S->c_nm = 1.0;
        S->rho_n = rt0;
        S->theta_nm = 0.0;
        S->del = rmul(S->vscale * S->vscale, make_double2(tot.v[2], tot.v[3]));
        S->k1 = cdiv(rmul(S->rho_n, S->del), S->eps);
        S->tau = S->tau0 = rt0;
        S->ratio_min = 1e300;
        S->inner_it = 0;
        S->has_inner = 1;
        if (finite2(S->del) && !zero2(S->del) && rt0 > 0.0)
          S->phase = PH_INNER;
        else
          mark_done(D, S, 2);
      }
    }
  }
}

// Monitor: the true residual of the running iterate, ||b - K (x + D^-1/2 x~)||
// in complex128 (x~ lags one update), once per graph round.  Ends the inner
// cycle on convergence or on stagnation of the complex64 recurrence (see
// kStagnation); the next round's outer step folds x~ into x and restarts
// from the FP64 residual.
static __global__ void __launch_bounds__(kOpThreads) k_sw_check(SweepDev D) {
  const int sys = blockIdx.x % D.nsys;
  const long long tile = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (S->phase != PH_INNER || S->inner_it < 2) return;
  int i, j, k0, k1;
  sweep_tile(D, tile, i, j, k0, k1);
  Vals<1> a{{0.0}};
  if (i < D.g.nx && j < D.g.ny) {
    const long long vb = (long long)sys * 4 * D.L.N;
    const XRef64 L{D.g, D.x64 + (long long)sys * D.n, D.s + vb, D.x + vb, D.L.nxp, D.L.N};
    const K2Ref64 K{D.g, D.sig, D.epsr, S->ka, S->kb};
    const double2 *b = D.b + (long long)sys * D.n;
    for (int k = k0; k < k1; k++) {
      double2 o[4];
      rowsN<double>(D.g, i, j, k, L, K, o);
#pragma unroll
      for (int c = 0; c < 4; c++)
        if (exists(D.g, c, i, j, k)) a.v[0] += cabs2(csub(__ldg(b + ref_of(D.g, c, i, j, k)), o[c]));
    }
  }
  Vals<1> blk = block_reduce<1, kOpThreads>(a);
  double *part = D.part + (size_t)sys * D.slots * 6;
  unsigned *cnt = D.cnt + CNT_CHECK * D.nsys + sys;
  const unsigned nt = (unsigned)D.t.count();
  if (arrive<1, kOpThreads>(blk, part, cnt, (unsigned)tile, nt)) {
    Vals<1> tot = final_reduce<1, kOpThreads>(part, cnt, nt);
    if (threadIdx.x == 0) {
      const double rn = sqrt(tot.v[0]);
      S->mon_rn = rn;
      S->checks++;
      const double ratio = rn / fmax(S->tau, 1e-300);
      S->ratio_min = fmin(S->ratio_min, ratio);
      if (!isfinite(rn) || rn < S->target * S->bnorm || ratio > kStagnation * S->ratio_min)
        S->phase = PH_OUTER;
    }
  }
}

// ------------------------------------------------------------ inner QMR
// TMA helpers (plain, non-multicast tensor loads into this CTA's shared
// memory; completion through an mbarrier with a bounded wait)
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
// true when the phase completed; gives up after `tries` polls
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned phase, int tries) {
  for (int t = 0; t < tries; t++) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void tma_load5(unsigned dst, const CUtensorMap *map, int x, int y, int z, int c, int s,
                                          unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];\n" ::"r"(dst),
      "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(s), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_load4(unsigned dst, const CUtensorMap *map, int x, int y, int z, int c,
                                          unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(dst),
      "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// tensor maps of the operator pass (kernel parameter, __grid_constant__)
struct ApplyMaps {
  CUtensorMap s, v, p;  // 5-D: (nxp, ny, nz, component, system), 8-byte elements
  CUtensorMap sig, eps; // 4-D: (nxp, ny, nz, component), FP32
};

constexpr unsigned kRawBytes = 4u * kPN * 8u;   // one array, four components, one plane
constexpr unsigned kSigBytes = 4u * kKN * 4u;
constexpr size_t kApplyShm = 3 * (size_t)kRawBytes   // raw s, v, p of one plane
                           + 3 * (size_t)kRawBytes   // U ring (three planes)
                           + 2 * (size_t)kSigBytes   // sigma-bar, two planes
                           + 128;                    // mbarriers (keeps what follows 128-byte aligned)
constexpr size_t kApplyShmEps = 2 * (size_t)kSigBytes;  // eps-bar, two planes (models C, I)
constexpr int kWaitTries = 1 << 24;

// A: q~_n = D^-1/2 K D^-1/2 p~_n and epsilon_n = u^T K u (u = D^-1/2 p~_n),
// then beta_n = epsilon_n / delta_n (src/aphid_qmr.f90:324-330).
//
// A 16 x 16 node tile marches along k.  One thread issues, per z-plane, three
// TMA loads (v~, p~, D^-1/2: all four components, 20 x 18 nodes with halo)
// and one for sigma-bar; the loads of plane k+2 (and sigma-bar of k+1) are in
// flight while plane k is computed.  u = D^-1/2 (vscale vt - k1 p~) is formed
// once per point into a ring of three planes.  TMA fills outside the tensor
// with zeros, pads and non-existent components are stored zeros, so zero
// padding reproduces the reference's clamped neighbours (their coefficients
// are zero at the boundary).
// SCALARS = false: the same pass without the scalar step and the phase test
// (operator timing on resident data; never changes a system's state).
template <bool SCALARS>
__global__ void __launch_bounds__(kPThreads, 2) k_sw_apply(SweepDev D, const __grid_constant__ ApplyMaps M) {
  const int sys = blockIdx.x % D.nsys;
  const long long tile = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (SCALARS && S->phase != PH_INNER) return;
  extern __shared__ __align__(128) unsigned char shm[];
  float2 *RAW = reinterpret_cast<float2 *>(shm);                          // [3][4][kPN]: s, v, p
  float2 *U = reinterpret_cast<float2 *>(shm + 3 * kRawBytes);            // [3][4][kPN]
  float *RK = reinterpret_cast<float *>(shm + 6 * kRawBytes);             // [2][4][kKN]
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(shm + 6 * kRawBytes + 2 * kSigBytes);
  const bool has_eps = D.epsr32 != nullptr;
  float *RE = reinterpret_cast<float *>(shm + kApplyShm);                 // [2][4][kKN]
  const unsigned b_raw = smem_u32(&bar[0]), b_k0 = smem_u32(&bar[1]), b_k1 = smem_u32(&bar[2]);

  const GridDev &g = D.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  long long tb = tile;
  const int bi = (int)(tb % D.tp.ti);
  tb /= D.tp.ti;
  const int bj = (int)(tb % D.tp.tj);
  const int bk = (int)(tb / D.tp.tj);
  const int i0 = bi * kPTI, j0 = bj * kPTJ, k0 = bk * D.tp.kz, k1 = min(nz, k0 + D.tp.kz);
  const int tx = threadIdx.x % kPTI, ty = threadIdx.x / kPTI;
  const int i = i0 + tx, j = j0 + ty;
  const long long N = D.L.N;
  const float2 *__restrict__ sv = D.s + (long long)sys * 4 * N;
  float2 *__restrict__ q = D.q + (long long)sys * 4 * N;
  const float *__restrict__ sig = D.sig32;
  const float *__restrict__ eps = D.epsr32;
  const float2 kone = to_f(S->k1);
  const float vsc = (float)S->vscale;
  const float ka = (float)S->ka, kb = (float)S->kb;
  int *err = D.err;

  // TMA destinations must be 128-byte aligned: refuse to copy otherwise
  if (smem_u32(shm) & 127u) {
    if (threadIdx.x == 0) atomicExch(D.err, 2);
    return;
  }
  if (threadIdx.x == 0) {
    mbar_init(b_raw);
    mbar_init(b_k0);
    mbar_init(b_k1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    fence_async_smem();
  }
  __syncthreads();
  unsigned ph_raw = 0, ph_k[2] = {0, 0};

  auto issue_raw = [&](int kk) {  // thread 0: v~, p~, D^-1/2 of plane kk
    fence_async_smem();
    mbar_expect(b_raw, 3 * kRawBytes);
    tma_load5(smem_u32(RAW), &M.s, i0 - 2, j0 - 1, kk, 0, sys, b_raw);
    tma_load5(smem_u32(RAW + 4 * kPN), &M.v, i0 - 2, j0 - 1, kk, 0, sys, b_raw);
    tma_load5(smem_u32(RAW + 8 * kPN), &M.p, i0 - 2, j0 - 1, kk, 0, sys, b_raw);
  };
  auto issue_k = [&](int kk, int buf) {  // thread 0: sigma-bar (eps-bar) of plane kk
    fence_async_smem();
    const unsigned bb = buf ? b_k1 : b_k0;
    mbar_expect(bb, has_eps ? 2 * kSigBytes : kSigBytes);
    tma_load4(smem_u32(RK + buf * 4 * kKN), &M.sig, i0 - 4, j0 - 1, kk, 0, bb);
    if (has_eps) tma_load4(smem_u32(RE + buf * 4 * kKN), &M.eps, i0 - 4, j0 - 1, kk, 0, bb);
  };
  auto wait_raw = [&]() {
    if (!mbar_wait(b_raw, ph_raw, kWaitTries) && threadIdx.x == 0) atomicExch(err, 1);
    ph_raw ^= 1u;
  };
  auto wait_k = [&](int buf) {
    if (!mbar_wait(buf ? b_k1 : b_k0, ph_k[buf], kWaitTries) && threadIdx.x == 0) atomicExch(err, 1);
    ph_k[buf] ^= 1u;
  };
  auto convert = [&](int kk) {  // raw plane -> u = D^-1/2 (vscale vt - k1 p~) in the ring
    float2 *Us = U + ((kk - k0 + 3) % 3) * 4 * kPN;
    for (int e = threadIdx.x; e < 4 * kPN; e += kPThreads)
      Us[e] = cmul(RAW[e], pnew32(vn32(RAW[4 * kPN + e], vsc), RAW[8 * kPN + e], kone));
  };

  // prologue: planes k0-1, k0, k0+1 into the ring, sigma-bar of k0
  for (int kk = k0 - 1; kk <= k0 + 1; kk++) {
    if (threadIdx.x == 0) issue_raw(kk);
    wait_raw();
    convert(kk);
    __syncthreads();
  }
  if (threadIdx.x == 0) issue_k(k0, 0);

  double ea = 0.0, eb = 0.0;
  const bool live = i < nx && j < ny;
  const int c0 = (ty + 1) * kPW + (tx + 2);  // this node in a staged plane
  const int ck = (ty + 1) * kKW + (tx + 4);  // this node in a sigma-bar plane
  const Axis &X = g.ax[0], &Y = g.ax[1], &Z = g.ax[2];
  const float xn4 = live ? (float)X.n4[i] : 0.f, xn5 = live ? (float)X.n5[i] : 0.f;
  const float yn4 = live ? (float)Y.n4[j] : 0.f, yn5 = live ? (float)Y.n5[j] : 0.f;
  const float dxc = live ? (float)X.dc[i] : 1.f, dyc = live ? (float)Y.dc[j] : 1.f;
  const bool hx = live && i < nx - 1, hy = live && j < ny - 1;
  const float ce2x = hx ? (float)X.e2[i] : 0.f, ce3x = hx ? (float)X.e3[i] : 0.f;
  const float dxi = hx ? (float)X.d[i + 1] : 1.f;
  const float ce2y = hy ? (float)Y.e2[j] : 0.f, ce3y = hy ? (float)Y.e3[j] : 0.f;
  const float dyj = hy ? (float)Y.d[j + 1] : 1.f;
  const bool pin = live && i > 0 && i < nx - 1 && j > 0 && j < ny - 1;
  const long long plane = (long long)D.L.nxp * ny;
  const long long ndc = i + (long long)D.L.nxp * j;  // node index within a plane

  for (int k = k0; k < k1; k++) {
    const int kb_ = (k - k0) & 1;
    const bool more = k + 1 < k1;
    if (more && threadIdx.x == 0) {
      issue_raw(k + 2);
      issue_k(k + 1, kb_ ^ 1);
    }
    wait_k(kb_);
    const float *rk = RK + kb_ * 4 * kKN;
    const float *re = RE + kb_ * 4 * kKN;
    auto kks = [&](int c, int off) {
      const float e = has_eps ? re[c * kKN + ck + off] : 1.0f;
      return make_float2(-ka * e, kb * rk[c * kKN + ck + off]);
    };
    auto kkg = [&](int c, long long nd) {
      const float e = has_eps ? __ldg(eps + c * N + nd) : 1.0f;
      return make_float2(-ka * e, kb * __ldg(sig + c * N + nd));
    };
    if (live) {
      const float2 *Um = U + ((k - 1 - k0 + 3) % 3) * 4 * kPN;
      const float2 *Uc = U + ((k - k0 + 3) % 3) * 4 * kPN;
      const float2 *Up = U + ((k + 1 - k0 + 3) % 3) * 4 * kPN;
      const float zn4 = (float)Z.n4[k], zn5 = (float)Z.n5[k], dzc = (float)Z.dc[k];
      const long long nd = ndc + k * plane;
      const float2 kpc = kks(3, 0), phc = Uc[3 * kPN + c0];
      float2 w[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      if (hx) {
        const float vol = dxi * dyc * dzc;
        const float2 k2 = kks(0, 0), kp2 = kks(3, 1);
        const float sum = ce2x + ce3x + yn4 + yn5 + zn4 + zn5;
        const float2 *u = Uc;
        float2 t = cmul(make_float2(-sum + k2.x, k2.y), u[c0]);
        t = cadd(t, rmul(ce2x, u[c0 + 1]));
        t = cadd(t, rmul(ce3x, u[c0 - 1]));
        t = cadd(t, rmul(yn4, u[c0 + kPW]));
        t = cadd(t, rmul(yn5, u[c0 - kPW]));
        t = cadd(t, rmul(zn4, Up[c0]));
        t = cadd(t, rmul(zn5, Um[c0]));
        const float2 gr = rdiv(csub(cmul(Uc[3 * kPN + c0 + 1], csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dxi);
        w[0] = rmul(vol, cadd(t, gr));
      }
      if (hy) {
        const float vol = dxc * dyj * dzc;
        const float2 k2 = kks(1, 0), kp2 = kks(3, kKW);
        const float sum = ce2y + ce3y + xn4 + xn5 + zn4 + zn5;
        const float2 *u = Uc + kPN;
        float2 t = cmul(make_float2(-sum + k2.x, k2.y), u[c0]);
        t = cadd(t, rmul(ce2y, u[c0 + kPW]));
        t = cadd(t, rmul(ce3y, u[c0 - kPW]));
        t = cadd(t, rmul(xn4, u[c0 + 1]));
        t = cadd(t, rmul(xn5, u[c0 - 1]));
        t = cadd(t, rmul(zn4, Up[kPN + c0]));
        t = cadd(t, rmul(zn5, Um[kPN + c0]));
        const float2 gr = rdiv(csub(cmul(Uc[3 * kPN + c0 + kPW], csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dyj);
        w[1] = rmul(vol, cadd(t, gr));
      }
      if (k < nz - 1) {
        const float c2 = (float)Z.e2[k], c3 = (float)Z.e3[k], dzk = (float)Z.d[k + 1];
        const float vol = dxc * dyc * dzk;
        const float2 k2 = kks(2, 0), kp2 = kkg(3, nd + plane);
        const float sum = c2 + c3 + xn4 + xn5 + yn4 + yn5;
        const float2 *u = Uc + 2 * kPN;
        float2 t = cmul(make_float2(-sum + k2.x, k2.y), u[c0]);
        t = cadd(t, rmul(c2, Up[2 * kPN + c0]));
        t = cadd(t, rmul(c3, Um[2 * kPN + c0]));
        t = cadd(t, rmul(xn4, u[c0 + 1]));
        t = cadd(t, rmul(xn5, u[c0 - 1]));
        t = cadd(t, rmul(yn4, u[c0 + kPW]));
        t = cadd(t, rmul(yn5, u[c0 - kPW]));
        const float2 gr = rdiv(csub(cmul(Up[3 * kPN + c0], csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dzk);
        w[2] = rmul(vol, cadd(t, gr));
      }
      if (pin && k > 0 && k < nz - 1) {
        const float vol = dxc * dyc * dzc;
        const float2 s1 = kpc;
        const float2 s2 = kks(0, 0), s3 = kks(0, -1), s4 = kks(1, 0), s5 = kks(1, -kKW);
        const float2 s6 = kks(2, 0), s7 = kkg(2, nd - plane);
        const float2 c2 = rmul(xn4, s2), c3 = rmul(xn5, s3), c4 = rmul(yn4, s4);
        const float2 c5 = rmul(yn5, s5), c6 = rmul(zn4, s6), c7 = rmul(zn5, s7);
        const float2 sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
        const float2 *u = Uc + 3 * kPN;
        float2 t = cmul(cadd(cneg(sum), cmul(s1, s1)), phc);
        t = cadd(t, cmul(c2, u[c0 + 1]));
        t = cadd(t, cmul(c3, u[c0 - 1]));
        t = cadd(t, cmul(c4, u[c0 + kPW]));
        t = cadd(t, cmul(c5, u[c0 - kPW]));
        t = cadd(t, cmul(c6, Up[3 * kPN + c0]));
        t = cadd(t, cmul(c7, Um[3 * kPN + c0]));
        float2 e = cmul(rdiv(csub(s2, s1), dxc), Uc[c0]);
        e = cadd(e, cmul(cneg(rdiv(csub(s3, s1), dxc)), Uc[c0 - 1]));
        e = cadd(e, cmul(rdiv(csub(s4, s1), dyc), Uc[kPN + c0]));
        e = cadd(e, cmul(cneg(rdiv(csub(s5, s1), dyc)), Uc[kPN + c0 - kPW]));
        e = cadd(e, cmul(rdiv(csub(s6, s1), dzc), Uc[2 * kPN + c0]));
        e = cadd(e, cmul(cneg(rdiv(csub(s7, s1), dzc)), Um[2 * kPN + c0]));
        w[3] = cadd(rmul(vol, t), rmul(vol, e));
      }
      float we_r = 0.f, we_i = 0.f;  // this node's share of u^T w
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const float2 sc = __ldg(sv + c * N + nd);
        q[c * N + nd] = cmul(sc, w[c]);
        const float2 e = cmul(Uc[c * kPN + c0], w[c]);
        we_r += e.x;
        we_i += e.y;
      }
      ea += (double)we_r;
      eb += (double)we_i;
    }
    if (more) wait_raw();  // plane k+2 has landed
    __syncthreads();       // everyone is done with ring slot k-1 and the raw plane
    if (more) {
      convert(k + 2);
      __syncthreads();
    }
  }

  Vals<2> blk = block_reduce<2, kPThreads>(Vals<2>{{ea, eb}});
  double *part = D.part + (size_t)sys * D.slots * 6;
  unsigned *cnt = D.cnt + CNT_APPLY * D.nsys + sys;
  const unsigned nt = (unsigned)D.tp.count();
  if (arrive<2, kPThreads>(blk, part, cnt, (unsigned)tile, nt)) {
    Vals<2> tot = final_reduce<2, kPThreads>(part, cnt, nt);
    if (SCALARS && threadIdx.x == 0) {
      const double2 e = make_double2(tot.v[0], tot.v[1]);
      S->eps = e;
      if (!finite2(e) || zero2(e)) {  // breakdown: restart from the current x
        S->phase = PH_OUTER;
        return;
      }
      S->beta = cdiv(e, S->del);
    }
  }
}

// B: p~_n stored; vt = q~_n - beta_n v~_n stored unnormalised; the lagged
// d~, x~ update of the previous iteration; ||vt||^2 and vt^T vt reduced,
// then rho_{n+1}, delta_{n+1}, theta, c, eta, kappa, the quasi-residual and
// the inner stop test (src/aphid_qmr.f90:332-390).  Two complex64 values per
// 16-byte access over the node-layout vectors (pads and absent components
// are zero and stay zero).
static __global__ void __launch_bounds__(kStreamThreads) k_sw_update(SweepDev D) {
  const int sys = blockIdx.x % D.nsys, chunk = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (S->phase != PH_INNER) return;
  const long long vb = (long long)sys * 4 * D.L.N;
  const float2 k1 = to_f(S->k1), beta = to_f(S->beta);
  const float vsc = (float)S->vscale;
  const bool pend = S->pending != 0;
  const float2 eta = to_f(S->eta_pend);
  const float kap = (float)S->kap_pend;
  float4 *v = reinterpret_cast<float4 *>(D.v + vb), *p = reinterpret_cast<float4 *>(D.p + vb);
  float4 *d = reinterpret_cast<float4 *>(D.d + vb), *x = reinterpret_cast<float4 *>(D.x + vb);
  const float4 *q = reinterpret_cast<const float4 *>(D.q + vb);
  const long long n2 = 2 * D.L.N;  // float4 count: 4N complex values / 2
  Vals<3> a{{0.0, 0.0, 0.0}};
  auto one = [&](float2 vt_old, float2 po, float2 qq, float2 &pn, float2 &vt) {
    const float2 vn = vn32(vt_old, vsc);
    pn = pnew32(vn, po, k1);
    vt = csub(qq, cmul(beta, vn));
    const double2 dv = to_d(vt);
    a.v[0] += cabs2(dv);
    a.v[1] += dv.x * dv.x - dv.y * dv.y;
    a.v[2] += 2.0 * dv.x * dv.y;
  };
  for (long long t = chunk * (long long)blockDim.x + threadIdx.x; t < n2; t += (long long)D.bps * blockDim.x) {
    const float4 v4 = v[t], p4 = p[t], q4 = q[t];
    float2 pa, pb, va, vb2;
    one(make_float2(v4.x, v4.y), make_float2(p4.x, p4.y), make_float2(q4.x, q4.y), pa, va);
    one(make_float2(v4.z, v4.w), make_float2(p4.z, p4.w), make_float2(q4.z, q4.w), pb, vb2);
    p[t] = make_float4(pa.x, pa.y, pb.x, pb.y);
    v[t] = make_float4(va.x, va.y, vb2.x, vb2.y);
    if (pend) {
      const float4 d4 = d[t], x4 = x[t];
      const float2 da = cadd(cmul(eta, make_float2(p4.x, p4.y)), rmul(kap, make_float2(d4.x, d4.y)));
      const float2 db = cadd(cmul(eta, make_float2(p4.z, p4.w)), rmul(kap, make_float2(d4.z, d4.w)));
      d[t] = make_float4(da.x, da.y, db.x, db.y);
      x[t] = make_float4(x4.x + da.x, x4.y + da.y, x4.z + db.x, x4.w + db.y);
    }
  }
  Vals<3> blk = block_reduce<3, kStreamThreads>(a);
  double *part = D.part + (size_t)sys * D.slots * 6;
  unsigned *cnt = D.cnt + CNT_UPDATE * D.nsys + sys;
  if (arrive<3, kStreamThreads>(blk, part, cnt, chunk, D.bps)) {
    Vals<3> tot = final_reduce<3, kStreamThreads>(part, cnt, D.bps);
    if (threadIdx.x == 0) {
      S->inner_it++;
      S->total_it++;
      // from here on p~_n is stored and the previous lagged update is applied
      const double rho = sqrt(tot.v[0]);
      const double2 beta_d = S->beta;
      if (!(rho > 0.0) || !isfinite(rho)) {  // Krylov space exhausted
        S->pending = 0;
        S->phase = PH_OUTER;
        return;
      }
      S->rho_np = rho;
      S->theta_n = rho * rho / S->c_nm / (beta_d.x * beta_d.x + beta_d.y * beta_d.y);
      S->c_n = 1.0 / (1.0 + S->theta_n);
      S->eta = cdiv(rmul(S->c_n, rmul(S->rho_n, cneg(S->eta))), rmul(S->c_nm, beta_d));
      S->kap = S->theta_nm * S->c_n;
      S->tau = S->tau * sqrt(S->theta_n * S->c_n);
      S->eta_pend = S->eta;
      S->kap_pend = S->kap;
      S->pending = 1;
      S->vscale = 1.0 / rho;
      const double2 del = rmul(1.0 / (rho * rho), make_double2(tot.v[1], tot.v[2]));
      if (!finite2(S->eta) || !isfinite(S->tau) || !finite2(del) || zero2(del) ||
          S->tau < S->inner_tol * S->tau0 || S->total_it >= S->max_it) {
        S->phase = PH_OUTER;
        return;
      }
      S->c_nm = S->c_n;
      S->rho_n = rho;
      S->theta_nm = S->theta_n;
      S->del = del;
      S->k1 = cdiv(rmul(S->rho_n, del), S->eps);
    }
  }
}

}  // namespace aphid

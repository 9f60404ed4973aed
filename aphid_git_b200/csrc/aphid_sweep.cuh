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

// plane tile of the complex64 operator pass: 16 (i) x 16 (j) nodes, marching
// along k with a ring of three z-planes in shared memory
constexpr int kPTI = 16, kPTJ = 16, kPThreads = kPTI * kPTJ;
constexpr int kPW = kPTI + 2, kPH = kPTJ + 2, kPN = kPW * kPH;

struct SweepDev {
  GridDev g;
  Tiles t;   // 32 x 4 column tiles (complex128 residual passes)
  Tiles tp;  // 16 x 16 plane tiles (complex64 operator pass)
  long long n;
  int nsys, bps;         // systems; blocks per system of the pointwise kernels
  long long slots;       // partial-sum slots per system
  const double *sig;     // sigma-bar per unknown (FP64, outer residual)
  const double *epsr;    // eps-bar per unknown, or null (= 1)
  const float *sig32, *epsr32;  // the same in FP32 for the inner operator
  float2 *v, *p, *q, *d, *x, *s;  // [nsys][n] complex64 (v holds vt)
  double2 *x64, *b;               // [nsys][n] complex128
  SweepSys *sys;
  double *part;                   // [nsys][slots][6]
  unsigned *cnt;                  // [CNT_KINDS][nsys]
  int *ndone;
};

// --------------------------------------------------- generic stencil rows
// The rows of rows64 for any precision R (float or double); the arithmetic
// order follows the reference, the coefficient tables are FP64 and rounded to
// R where R is float.
template <typename R, class IN, class KK>
__device__ __forceinline__ void rowsT(const GridDev &g, int i, int j, int k, const IN &in, const KK &kk,
                                      typename CplxOf<R>::T &ox, typename CplxOf<R>::T &oy,
                                      typename CplxOf<R>::T &oz, typename CplxOf<R>::T &op) {
  using C = typename CplxOf<R>::T;
  const Axis &X = g.ax[0], &Y = g.ax[1], &Z = g.ax[2];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const R xn4 = (R)X.n4[i], xn5 = (R)X.n5[i], yn4 = (R)Y.n4[j], yn5 = (R)Y.n5[j];
  const R zn4 = (R)Z.n4[k], zn5 = (R)Z.n5[k];
  const R dxc = (R)X.dc[i], dyc = (R)Y.dc[j], dzc = (R)Z.dc[k];
  const int ia = min(i + 1, nx - 1), ib = max(i - 1, 0);
  const int ja = min(j + 1, ny - 1), jb = max(j - 1, 0);
  const int ka = min(k + 1, nz - 1), kb = max(k - 1, 0);
  const long long pc = ixp(g, i, j, k);
  const C phc = in(pc), kpc = kk(pc);
  if (i < nx - 1) {
    const R c2 = (R)X.e2[i], c3 = (R)X.e3[i], dxi = (R)X.d[i + 1];
    const R vol = dxi * dyc * dzc;
    const long long c = ixx(g, i, j, k);
    const C k2 = kk(c), kp2 = kk(pc + 1);
    const R sum = c2 + c3 + yn4 + yn5 + zn4 + zn5;
    C s = cmul(mkc<R>(-sum + k2.x, k2.y), in(c));
    s = cadd(s, rmul(c2, in(ixx(g, min(i + 1, nx - 2), j, k))));
    s = cadd(s, rmul(c3, in(ixx(g, ib, j, k))));
    s = cadd(s, rmul(yn4, in(ixx(g, i, ja, k))));
    s = cadd(s, rmul(yn5, in(ixx(g, i, jb, k))));
    s = cadd(s, rmul(zn4, in(ixx(g, i, j, ka))));
    s = cadd(s, rmul(zn5, in(ixx(g, i, j, kb))));
    const C gr = rdiv(csub(cmul(in(pc + 1), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dxi);
    ox = rmul(vol, cadd(s, gr));
  }
  if (j < ny - 1) {
    const R c2 = (R)Y.e2[j], c3 = (R)Y.e3[j], dyj = (R)Y.d[j + 1];
    const R vol = dxc * dyj * dzc;
    const long long c = ixy(g, i, j, k), pn = pc + nx;
    const C k2 = kk(c), kp2 = kk(pn);
    const R sum = c2 + c3 + xn4 + xn5 + zn4 + zn5;
    C s = cmul(mkc<R>(-sum + k2.x, k2.y), in(c));
    s = cadd(s, rmul(c2, in(ixy(g, i, min(j + 1, ny - 2), k))));
    s = cadd(s, rmul(c3, in(ixy(g, i, jb, k))));
    s = cadd(s, rmul(xn4, in(ixy(g, ia, j, k))));
    s = cadd(s, rmul(xn5, in(ixy(g, ib, j, k))));
    s = cadd(s, rmul(zn4, in(ixy(g, i, j, ka))));
    s = cadd(s, rmul(zn5, in(ixy(g, i, j, kb))));
    const C gr = rdiv(csub(cmul(in(pn), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dyj);
    oy = rmul(vol, cadd(s, gr));
  }
  if (k < nz - 1) {
    const R c2 = (R)Z.e2[k], c3 = (R)Z.e3[k], dzk = (R)Z.d[k + 1];
    const R vol = dxc * dyc * dzk;
    const long long c = ixz(g, i, j, k), pn = pc + (long long)nx * ny;
    const C k2 = kk(c), kp2 = kk(pn);
    const R sum = c2 + c3 + xn4 + xn5 + yn4 + yn5;
    C s = cmul(mkc<R>(-sum + k2.x, k2.y), in(c));
    s = cadd(s, rmul(c2, in(ixz(g, i, j, min(k + 1, nz - 2)))));
    s = cadd(s, rmul(c3, in(ixz(g, i, j, kb))));
    s = cadd(s, rmul(xn4, in(ixz(g, ia, j, k))));
    s = cadd(s, rmul(xn5, in(ixz(g, ib, j, k))));
    s = cadd(s, rmul(yn4, in(ixz(g, i, ja, k))));
    s = cadd(s, rmul(yn5, in(ixz(g, i, jb, k))));
    const C gr = rdiv(csub(cmul(in(pn), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dzk);
    oz = rmul(vol, cadd(s, gr));
  }
  if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) {
    const R vol = dxc * dyc * dzc;
    const C s1 = kpc;
    const long long xc = ixx(g, i, j, k), yc = ixy(g, i, j, k), zc = ixz(g, i, j, k);
    const long long xm = xc - 1, ym = yc - nx, zm = zc - (long long)nx * ny;
    const C s2 = kk(xc), s3 = kk(xm), s4 = kk(yc), s5 = kk(ym), s6 = kk(zc), s7 = kk(zm);
    const C c2 = rmul(xn4, s2), c3 = rmul(xn5, s3), c4 = rmul(yn4, s4);
    const C c5 = rmul(yn5, s5), c6 = rmul(zn4, s6), c7 = rmul(zn5, s7);
    const C sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
    const C c1 = cadd(cneg(sum), cmul(s1, s1));
    C s = cmul(c1, phc);
    s = cadd(s, cmul(c2, in(pc + 1)));
    s = cadd(s, cmul(c3, in(pc - 1)));
    s = cadd(s, cmul(c4, in(pc + nx)));
    s = cadd(s, cmul(c5, in(pc - nx)));
    s = cadd(s, cmul(c6, in(pc + (long long)nx * ny)));
    s = cadd(s, cmul(c7, in(pc - (long long)nx * ny)));
    const C acc = rmul(vol, s);
    C t = cmul(rdiv(csub(s2, s1), dxc), in(xc));
    t = cadd(t, cmul(cneg(rdiv(csub(s3, s1), dxc)), in(xm)));
    t = cadd(t, cmul(rdiv(csub(s4, s1), dyc), in(yc)));
    t = cadd(t, cmul(cneg(rdiv(csub(s5, s1), dyc)), in(ym)));
    t = cadd(t, cmul(rdiv(csub(s6, s1), dzc), in(zc)));
    t = cadd(t, cmul(cneg(rdiv(csub(s7, s1), dzc)), in(zm)));
    op = cadd(acc, rmul(vol, t));
  } else {
    op = mkc<R>((R)0, (R)0);
  }
}

// k^2 from the shared averages, FP64 (outer residual) and FP32 (inner)
struct K2Avg64 {
  const double *__restrict__ sig, *__restrict__ epsr;
  double ka, kb;
  __device__ __forceinline__ double2 operator()(long long t) const {
    const double e = epsr ? __ldg(epsr + t) : 1.0;
    return make_double2(-ka * e, kb * __ldg(sig + t));
  }
};
struct K2Avg32 {
  const float *__restrict__ sig, *__restrict__ epsr;
  float ka, kb;
  __device__ __forceinline__ float2 operator()(long long t) const {
    const float e = epsr ? __ldg(epsr + t) : 1.0f;
    return make_float2(-ka * e, kb * __ldg(sig + t));
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

// FP32 copy of an FP64 per-unknown array
static __global__ void k_sw_to32(long long n, const double *__restrict__ a, float *__restrict__ b) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    b[t] = (float)a[t];
}

// complex128 k^2 vector of one system from the averages (for the complex128
// sweep, which runs the reference's own algorithm on it)
static __global__ void k_sw_k2vec(long long n, const double *__restrict__ sig, const double *__restrict__ epsr,
                                  double ka, double kb, double2 *__restrict__ k2) {
  const K2Avg64 K{sig, epsr, ka, kb};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    k2[t] = K(t);
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

// D^-1/2 per unknown and system from the FP64 Jacobi diagonal (gen_diag,
// src/aphid.f90:1542-1725, with k^2 from the averages)
static __global__ void k_sw_scale(SweepDev D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z % D.g.nz;
  const int sys = blockIdx.z / D.g.nz;
  const GridDev &g = D.g;
  if (i >= g.nx) return;
  const SweepSys &S = D.sys[sys];
  const K2Avg64 K{D.sig, D.epsr, S.ka, S.kb};
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double *dx = g.ax[0].d, *dy = g.ax[1].d, *dz = g.ax[2].d;
  const int I = i + 1, J = j + 1, KK = k + 1;
  const double dxi = dx[I], dxim = dx[I - 1], dxci = 0.5 * (dxi + dxim);
  const double dyj = dy[J], dyjm = dy[J - 1], dycj = 0.5 * (dyj + dyjm);
  const double dzk = dz[KK], dzkm = dz[KK - 1], dzck = 0.5 * (dzk + dzkm);
  const double xn4 = mask_hi(I, nx) / dxi / dxci, xn5 = mask_lo(I, nx) / dxim / dxci;
  const double yn4 = mask_hi(J, ny) / dyj / dycj, yn5 = mask_lo(J, ny) / dyjm / dycj;
  const double zn4 = mask_hi(KK, nz) / dzk / dzck, zn5 = mask_lo(KK, nz) / dzkm / dzck;
  float2 *s = D.s + (long long)sys * D.n;
  if (i < nx - 1) {
    const double c2 = mask_hi(I, nx - 1) / (0.5 * (dxi + dx[I + 1])) / dxi, c3 = mask_lo(I, nx) / dxci / dxi;
    const long long t = ixx(g, i, j, k);
    const double2 kv = K(t);
    s[t] = to_f(cinvsqrt(rmul(dxi * dycj * dzck, make_double2(-(c2 + c3 + yn4 + yn5 + zn4 + zn5) + kv.x, kv.y))));
  }
  if (j < ny - 1) {
    const double c2 = mask_hi(J, ny - 1) / (0.5 * (dyj + dy[J + 1])) / dyj, c3 = mask_lo(J, ny) / dycj / dyj;
    const long long t = ixy(g, i, j, k);
    const double2 kv = K(t);
    s[t] = to_f(cinvsqrt(rmul(dxci * dyj * dzck, make_double2(-(c2 + c3 + xn4 + xn5 + zn4 + zn5) + kv.x, kv.y))));
  }
  if (k < nz - 1) {
    const double c2 = mask_hi(KK, nz - 1) / (0.5 * (dzk + dz[KK + 1])) / dzk, c3 = mask_lo(KK, nz) / dzck / dzk;
    const long long t = ixz(g, i, j, k);
    const double2 kv = K(t);
    s[t] = to_f(cinvsqrt(rmul(dxci * dycj * dzk, make_double2(-(c2 + c3 + xn4 + xn5 + yn4 + yn5) + kv.x, kv.y))));
  }
  const long long pt = ixp(g, i, j, k);
  if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) {
    const double2 s1 = K(pt);
    const double2 c2 = rdiv(rdiv(rmul(mask_hi(I, nx), K(ixx(g, i, j, k))), dxi), dxci);
    const double2 c3 = rdiv(rdiv(rmul(mask_lo(I, nx), K(ixx(g, i - 1, j, k))), dxim), dxci);
    const double2 c4 = rdiv(rdiv(rmul(mask_hi(J, ny), K(ixy(g, i, j, k))), dyj), dycj);
    const double2 c5 = rdiv(rdiv(rmul(mask_lo(J, ny), K(ixy(g, i, j - 1, k))), dyjm), dycj);
    const double2 c6 = rdiv(rdiv(rmul(mask_hi(KK, nz), K(ixz(g, i, j, k))), dzk), dzck);
    const double2 c7 = rdiv(rdiv(rmul(mask_lo(KK, nz), K(ixz(g, i, j, k - 1))), dzkm), dzck);
    const double2 sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
    s[pt] = to_f(cinvsqrt(rmul(dxci * dycj * dzck, cadd(cneg(sum), cmul(s1, s1)))));
  } else {
    s[pt] = make_float2(1.0f, 0.0f);
  }
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

// ------------------------------------------------------------ outer step
// O1: x += D^-1/2 (x~ + pending lagged update), FP64 accumulation of the
// inner correction
static __global__ void __launch_bounds__(kStreamThreads) k_sw_xupd(SweepDev D) {
  const int sys = blockIdx.x % D.nsys, chunk = blockIdx.x / D.nsys;
  const SweepSys *S = D.sys + sys;
  if (S->phase != PH_OUTER || !S->has_inner) return;
  const long long base = (long long)sys * D.n;
  const bool pend = S->pending != 0;
  const double2 eta = S->eta_pend;
  const double kap = S->kap_pend;
  for (long long t = chunk * (long long)blockDim.x + threadIdx.x; t < D.n; t += (long long)D.bps * blockDim.x) {
    double2 xt = to_d(D.x[base + t]);
    if (pend) xt = cadd(xt, cadd(cmul(eta, to_d(D.p[base + t])), rmul(kap, to_d(D.d[base + t]))));
    D.x64[base + t] = cadd(D.x64[base + t], cmul(to_d(D.s[base + t]), xt));
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
  const long long base = (long long)sys * D.n;
  int i, j, k0, k1;
  sweep_tile(D, tile, i, j, k0, k1);
  Vals<4> a{{0.0, 0.0, 0.0, 0.0}};
  if (i < D.g.nx && j < D.g.ny) {
    const LoadVec L{D.x64 + base};
    const K2Avg64 K{D.sig, D.epsr, S->ka, S->kb};
    const double2 *b = D.b + base;
    const float2 *s = D.s + base;
    float2 *v = D.v + base, *p = D.p + base, *d = D.d + base, *x = D.x + base;
    const float2 zero = make_float2(0.f, 0.f);
    for (int k = k0; k < k1; k++) {
      double2 o[4];
      rowsT<double>(D.g, i, j, k, L, K, o[0], o[1], o[2], o[3]);
      const bool has[4] = {i < D.g.nx - 1, j < D.g.ny - 1, k < D.g.nz - 1, true};
      const long long ix[4] = {ixx(D.g, i, j, k), ixy(D.g, i, j, k), ixz(D.g, i, j, k), ixp(D.g, i, j, k)};
#pragma unroll
      for (int c = 0; c < 4; c++) {
        if (!has[c]) continue;
        const long long t = ix[c];
        const double2 r = csub(b[t], o[c]);
        const float2 rt = to_f(cmul(to_d(s[t]), r));
        v[t] = rt;
        p[t] = zero;
        d[t] = zero;
        x[t] = zero;
        const double2 drt = to_d(rt);
        a.v[0] += cabs2(r);
        a.v[1] += cabs2(drt);
        const double2 sq = cmul(drt, drt);
        a.v[2] += sq.x;
        a.v[3] += sq.y;
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
        S->phase = (finite2(S->del) && !zero2(S->del) && rt0 > 0.0) ? PH_INNER : PH_OUTER;
        if (S->phase == PH_OUTER) mark_done(D, S, 2);
      }
    }
  }
}

// Monitor: the true residual of the running iterate, ||b - K (x + D^-1/2 x~)||
// in complex128 (x~ lags one update), once per graph round.  Ends the inner
// cycle on convergence or on stagnation of the complex64 recurrence (see
// kStagnation); the next round's outer step folds x~ into x and restarts
// from the FP64 residual.
struct InXcur {
  const double2 *__restrict__ x64;
  const float2 *__restrict__ s, *__restrict__ x;
  __device__ __forceinline__ double2 operator()(long long t) const {
    return cadd(__ldg(x64 + t), cmul(to_d(__ldg(s + t)), to_d(__ldg(x + t))));
  }
};

static __global__ void __launch_bounds__(kOpThreads) k_sw_check(SweepDev D) {
  const int sys = blockIdx.x % D.nsys;
  const long long tile = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (S->phase != PH_INNER || S->inner_it < 2) return;
  const long long base = (long long)sys * D.n;
  int i, j, k0, k1;
  sweep_tile(D, tile, i, j, k0, k1);
  Vals<1> a{{0.0}};
  if (i < D.g.nx && j < D.g.ny) {
    const InXcur L{D.x64 + base, D.s + base, D.x + base};
    const K2Avg64 K{D.sig, D.epsr, S->ka, S->kb};
    const double2 *b = D.b + base;
    for (int k = k0; k < k1; k++) {
      double2 o[4];
      rowsT<double>(D.g, i, j, k, L, K, o[0], o[1], o[2], o[3]);
      const bool has[4] = {i < D.g.nx - 1, j < D.g.ny - 1, k < D.g.nz - 1, true};
      const long long ix[4] = {ixx(D.g, i, j, k), ixy(D.g, i, j, k), ixz(D.g, i, j, k), ixp(D.g, i, j, k)};
#pragma unroll
      for (int c = 0; c < 4; c++)
        if (has[c]) a.v[0] += cabs2(csub(__ldg(b + ix[c]), o[c]));
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
// A: q~_n = D^-1/2 K D^-1/2 p~_n and epsilon_n = u^T K u (u = D^-1/2 p~_n),
// then beta_n = epsilon_n / delta_n (src/aphid_qmr.f90:324-330).
//
// A 16 x 16 node tile marches along k.  u of the four blocks is formed once
// per mesh point into a ring of three z-planes in shared memory (halo of one
// node in i and j).  The raw inputs of plane k+2 (v~, p~, D^-1/2) and the FP32
// sigma-bar of plane k+1 are copied asynchronously (cp.async, zero-filled
// outside the mesh and for components that do not exist at a point) while
// plane k is computed, so global-memory latency overlaps the arithmetic.
// Zero padding reproduces the reference's clamped neighbour indices, whose
// coefficients are zero at the boundary.  Indices within a system are 32-bit.
// SCALARS = false: the same pass without the scalar step and the phase test
// (operator timing on resident data; never changes a system's state).
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// dynamic shared memory of k_sw_apply: U ring, raw plane, sigma-bar (and
// eps-bar) double buffers
constexpr size_t kApplyShm = sizeof(float2) * 3 * 4 * kPN   // U ring
                           + sizeof(float2) * 3 * 4 * kPN   // raw s, v, p of one plane
                           + sizeof(float) * 2 * 4 * kPN;   // sigma-bar, 2 planes
constexpr size_t kApplyShmEps = sizeof(float) * 2 * 4 * kPN;  // eps-bar, 2 planes (models C, I)

template <bool SCALARS>
__global__ void __launch_bounds__(kPThreads, 3) k_sw_apply(SweepDev D) {
  const int sys = blockIdx.x % D.nsys;
  const long long tile = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (SCALARS && S->phase != PH_INNER) return;
  extern __shared__ __align__(16) unsigned char shm[];
  float2(*U)[4][kPN] = reinterpret_cast<float2(*)[4][kPN]>(shm);                      // [3][4][kPN]
  float2(*R)[4][kPN] = reinterpret_cast<float2(*)[4][kPN]>(shm + sizeof(float2) * 12 * kPN);  // s, v, p
  float(*RK)[4][kPN] = reinterpret_cast<float(*)[4][kPN]>(shm + sizeof(float2) * 24 * kPN);   // [2][4][kPN]
  float(*RE)[4][kPN] = reinterpret_cast<float(*)[4][kPN]>(shm + sizeof(float2) * 24 * kPN + sizeof(float) * 8 * kPN);
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
  const long long base = (long long)sys * D.n;
  const float2 *__restrict__ s = D.s + base;
  const float2 *__restrict__ v = D.v + base;
  const float2 *__restrict__ p = D.p + base;
  float2 *__restrict__ q = D.q + base;
  const float *__restrict__ sig = D.sig32;
  const float *__restrict__ eps = D.epsr32;
  const float2 kone = to_f(S->k1);
  const float vsc = (float)S->vscale;
  const float ka = (float)S->ka, kb = (float)S->kb;
  // 32-bit strides of the four blocks: index = off + i + sj*j + sk*k
  const int oy = (int)g.oy, oz = (int)g.oz, op = (int)g.op;
  const int sjx = nx - 1, skx = (nx - 1) * ny, sjy = nx, sky = nx * (ny - 1), sj = nx, sk = nx * ny;

  // the (at most two) padded-plane points each thread stages
  int qi[2], qj[2];
#pragma unroll
  for (int r = 0; r < 2; r++) {
    const int qd = threadIdx.x + r * kPThreads;
    qi[r] = i0 - 1 + qd % kPW;
    qj[r] = j0 - 1 + qd / kPW;
  }
  // global index of component c at padded point r, plane kk (or -1)
  auto gidx = [&](int c, int r, int kk) -> int {
    const int ii = qi[r], jj = qj[r];
    if (kk < 0 || kk >= nz || ii < 0 || ii >= nx || jj < 0 || jj >= ny) return -1;
    switch (c) {
      case 0: return ii < nx - 1 ? ii + sjx * jj + skx * kk : -1;
      case 1: return jj < ny - 1 ? oy + ii + sjy * jj + sky * kk : -1;
      case 2: return kk < nz - 1 ? oz + ii + sj * jj + sk * kk : -1;
      default: return op + ii + sj * jj + sk * kk;
    }
  };
  auto issue_raw = [&](int kk) {  // s, v, p of plane kk
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int qd = threadIdx.x + r * kPThreads;
      if (qd < kPN) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int t = gidx(c, r, kk);
          const int tt = t < 0 ? 0 : t;
          cp_async8(&R[0][c][qd], s + tt, t >= 0);
          cp_async8(&R[1][c][qd], v + tt, t >= 0);
          cp_async8(&R[2][c][qd], p + tt, t >= 0);
        }
      }
    }
  };
  auto issue_k = [&](int kk, int buf) {  // sigma-bar (and eps-bar) of plane kk
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int qd = threadIdx.x + r * kPThreads;
      if (qd < kPN) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int t = gidx(c, r, kk);
          const int tt = t < 0 ? 0 : t;
          cp_async4(&RK[buf][c][qd], sig + tt, t >= 0);
          if (eps) cp_async4(&RE[buf][c][qd], eps + tt, t >= 0);
        }
      }
    }
  };
  auto convert = [&](int kk) {  // raw plane -> u = D^-1/2 (vscale vt - k1 p) in the ring
    float2(*Us)[kPN] = U[(kk - k0 + 3) % 3];
    for (int e = threadIdx.x; e < 4 * kPN; e += kPThreads) {
      const int c = e / kPN, qd = e % kPN;
      Us[c][qd] = cmul(R[0][c][qd], pnew32(vn32(R[1][c][qd], vsc), R[2][c][qd], kone));
    }
  };

  // prologue: planes k0-1, k0, k0+1 into the ring, sigma-bar of k0
  for (int kk = k0 - 1; kk <= k0 + 1; kk++) {
    issue_raw(kk);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    convert(kk);
    __syncthreads();
  }
  issue_k(k0, 0);
  cp_async_commit();

  double ea = 0.0, eb = 0.0;
  const bool live = i < nx && j < ny;
  const int c0 = (ty + 1) * kPW + (tx + 1);
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
  // k^2 at a padded point of the staged plane, and at an own-column global index
  auto kks = [&](int buf, int c, int qd) {
    const float e = eps ? RE[buf][c][qd] : 1.0f;
    return make_float2(-ka * e, kb * RK[buf][c][qd]);
  };
  auto kkg = [&](int t) {
    const float e = eps ? __ldg(eps + t) : 1.0f;
    return make_float2(-ka * e, kb * __ldg(sig + t));
  };

  for (int k = k0; k < k1; k++) {
    const int kb_ = (k - k0) & 1;
    const bool more = k + 1 < k1;
    if (more) {
      issue_raw(k + 2);
      issue_k(k + 1, kb_ ^ 1);
    }
    cp_async_commit();
    cp_async_wait<1>();  // sigma-bar of plane k has landed
    __syncthreads();
    if (live) {
      const float2(*Um)[kPN] = U[(k - 1 - k0 + 3) % 3];
      const float2(*Uc)[kPN] = U[(k - k0 + 3) % 3];
      const float2(*Up)[kPN] = U[(k + 1 - k0 + 3) % 3];
      const float zn4 = (float)Z.n4[k], zn5 = (float)Z.n5[k], dzc = (float)Z.dc[k];
      const float2 kpc = kks(kb_, 3, c0), phc = Uc[3][c0];
      float2 w;
      float we_r = 0.f, we_i = 0.f;  // this node's share of u^T w
      if (hx) {
        const float vol = dxi * dyc * dzc;
        const float2 k2 = kks(kb_, 0, c0), kp2 = kks(kb_, 3, c0 + 1);
        const float sum = ce2x + ce3x + yn4 + yn5 + zn4 + zn5;
        const float2 uc = Uc[0][c0];
        float2 t = cmul(make_float2(-sum + k2.x, k2.y), uc);
        t = cadd(t, rmul(ce2x, Uc[0][c0 + 1]));
        t = cadd(t, rmul(ce3x, Uc[0][c0 - 1]));
        t = cadd(t, rmul(yn4, Uc[0][c0 + kPW]));
        t = cadd(t, rmul(yn5, Uc[0][c0 - kPW]));
        t = cadd(t, rmul(zn4, Up[0][c0]));
        t = cadd(t, rmul(zn5, Um[0][c0]));
        const float2 gr = rdiv(csub(cmul(Uc[3][c0 + 1], csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dxi);
        w = rmul(vol, cadd(t, gr));
        const int tt = i + sjx * j + skx * k;
        q[tt] = cmul(__ldg(s + tt), w);
        const float2 e = cmul(uc, w);
        we_r += e.x;
        we_i += e.y;
      }
      if (hy) {
        const float vol = dxc * dyj * dzc;
        const float2 k2 = kks(kb_, 1, c0), kp2 = kks(kb_, 3, c0 + kPW);
        const float sum = ce2y + ce3y + xn4 + xn5 + zn4 + zn5;
        const float2 uc = Uc[1][c0];
        float2 t = cmul(make_float2(-sum + k2.x, k2.y), uc);
        t = cadd(t, rmul(ce2y, Uc[1][c0 + kPW]));
        t = cadd(t, rmul(ce3y, Uc[1][c0 - kPW]));
        t = cadd(t, rmul(xn4, Uc[1][c0 + 1]));
        t = cadd(t, rmul(xn5, Uc[1][c0 - 1]));
        t = cadd(t, rmul(zn4, Up[1][c0]));
        t = cadd(t, rmul(zn5, Um[1][c0]));
        const float2 gr = rdiv(csub(cmul(Uc[3][c0 + kPW], csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dyj);
        w = rmul(vol, cadd(t, gr));
        const int tt = oy + i + sjy * j + sky * k;
        q[tt] = cmul(__ldg(s + tt), w);
        const float2 e = cmul(uc, w);
        we_r += e.x;
        we_i += e.y;
      }
      if (k < nz - 1) {
        const float c2 = (float)Z.e2[k], c3 = (float)Z.e3[k], dzk = (float)Z.d[k + 1];
        const float vol = dxc * dyc * dzk;
        const float2 k2 = kks(kb_, 2, c0), kp2 = kkg(op + i + sj * j + sk * (k + 1));
        const float sum = c2 + c3 + xn4 + xn5 + yn4 + yn5;
        const float2 uc = Uc[2][c0];
        float2 t = cmul(make_float2(-sum + k2.x, k2.y), uc);
        t = cadd(t, rmul(c2, Up[2][c0]));
        t = cadd(t, rmul(c3, Um[2][c0]));
        t = cadd(t, rmul(xn4, Uc[2][c0 + 1]));
        t = cadd(t, rmul(xn5, Uc[2][c0 - 1]));
        t = cadd(t, rmul(yn4, Uc[2][c0 + kPW]));
        t = cadd(t, rmul(yn5, Uc[2][c0 - kPW]));
        const float2 gr = rdiv(csub(cmul(Up[3][c0], csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dzk);
        w = rmul(vol, cadd(t, gr));
        const int tt = oz + i + sj * j + sk * k;
        q[tt] = cmul(__ldg(s + tt), w);
        const float2 e = cmul(uc, w);
        we_r += e.x;
        we_i += e.y;
      }
      {
        if (pin && k > 0 && k < nz - 1) {
          const float vol = dxc * dyc * dzc;
          const float2 s1 = kpc;
          const float2 s2 = kks(kb_, 0, c0), s3 = kks(kb_, 0, c0 - 1);
          const float2 s4 = kks(kb_, 1, c0), s5 = kks(kb_, 1, c0 - kPW);
          const float2 s6 = kks(kb_, 2, c0), s7 = kkg(oz + i + sj * j + sk * (k - 1));
          const float2 c2 = rmul(xn4, s2), c3 = rmul(xn5, s3), c4 = rmul(yn4, s4);
          const float2 c5 = rmul(yn5, s5), c6 = rmul(zn4, s6), c7 = rmul(zn5, s7);
          const float2 sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
          float2 t = cmul(cadd(cneg(sum), cmul(s1, s1)), phc);
          t = cadd(t, cmul(c2, Uc[3][c0 + 1]));
          t = cadd(t, cmul(c3, Uc[3][c0 - 1]));
          t = cadd(t, cmul(c4, Uc[3][c0 + kPW]));
          t = cadd(t, cmul(c5, Uc[3][c0 - kPW]));
          t = cadd(t, cmul(c6, Up[3][c0]));
          t = cadd(t, cmul(c7, Um[3][c0]));
          float2 e = cmul(rdiv(csub(s2, s1), dxc), Uc[0][c0]);
          e = cadd(e, cmul(cneg(rdiv(csub(s3, s1), dxc)), Uc[0][c0 - 1]));
          e = cadd(e, cmul(rdiv(csub(s4, s1), dyc), Uc[1][c0]));
          e = cadd(e, cmul(cneg(rdiv(csub(s5, s1), dyc)), Uc[1][c0 - kPW]));
          e = cadd(e, cmul(rdiv(csub(s6, s1), dzc), Uc[2][c0]));
          e = cadd(e, cmul(cneg(rdiv(csub(s7, s1), dzc)), Um[2][c0]));
          w = cadd(rmul(vol, t), rmul(vol, e));
        } else {
          w = make_float2(0.f, 0.f);
        }
        const int tt = op + i + sj * j + sk * k;
        q[tt] = cmul(__ldg(s + tt), w);
        const float2 e = cmul(phc, w);
        we_r += e.x;
        we_i += e.y;
      }
      ea += (double)we_r;
      eb += (double)we_i;
    }
    cp_async_wait<0>();  // raw plane k+2 and sigma-bar of k+1
    __syncthreads();     // everyone is done with ring slot k-1
    if (more) convert(k + 2);
    __syncthreads();
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
// the inner stop test (src/aphid_qmr.f90:332-390).
static __global__ void __launch_bounds__(kStreamThreads) k_sw_update(SweepDev D) {
  const int sys = blockIdx.x % D.nsys, chunk = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (S->phase != PH_INNER) return;
  const long long base = (long long)sys * D.n;
  const float2 k1 = to_f(S->k1), beta = to_f(S->beta);
  const float vsc = (float)S->vscale;
  const bool pend = S->pending != 0;
  const float2 eta = to_f(S->eta_pend);
  const float kap = (float)S->kap_pend;
  float2 *v = D.v + base, *p = D.p + base, *d = D.d + base, *x = D.x + base;
  const float2 *q = D.q + base;
  Vals<3> a{{0.0, 0.0, 0.0}};
  for (long long t = chunk * (long long)blockDim.x + threadIdx.x; t < D.n; t += (long long)D.bps * blockDim.x) {
    const float2 vn = vn32(v[t], vsc);
    const float2 po = p[t];
    const float2 pn = pnew32(vn, po, k1);
    p[t] = pn;
    if (pend) {
      const float2 dd = cadd(cmul(eta, po), rmul(kap, d[t]));
      d[t] = dd;
      x[t] = cadd(x[t], dd);
    }
    const float2 vt = csub(q[t], cmul(beta, vn));
    v[t] = vt;
    const double2 dv = to_d(vt);
    a.v[0] += cabs2(dv);
    a.v[1] += dv.x * dv.x - dv.y * dv.y;
    a.v[2] += 2.0 * dv.x * dv.y;
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

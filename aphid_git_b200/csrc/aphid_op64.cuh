// aphid_op64.cuh -- complex128 operator, wavenumber, Jacobi-diagonal and
// field kernels: the exact-arithmetic counterparts of the reference routines,
// one thread per mesh node (i fastest, coalesced), all four unknown blocks of
// a node handled by the same thread.
#pragma once
#include "aphid_common.cuh"

namespace aphid {

constexpr double kPi = 3.141592653589793;
constexpr double kMu0 = kPi * 4.e-7;           // src/aphid_mod.f90:10
constexpr double kEps0 = 8.8541878176e-12;     // src/aphid_mod.f90:12

// Fortran integer masks of the coefficient tables, 1-based index m:
// (m/n - 1) and ((n-m)/(n-1) - 1) with integer division.
__host__ __device__ __forceinline__ double mask_hi(int m, int n) { return (double)(m / n - 1); }
__host__ __device__ __forceinline__ double mask_lo(int m, int n) { return (double)((n - m) / (n - 1) - 1); }

// Stencil tile: 32 nodes along i (one warp) x 4 along j, KZ planes along k.
constexpr int kTileI = 32, kTileJ = 4, kOpThreads = kTileI * kTileJ;

struct Tiles {
  int ti, tj, tk, kz;
  int ts;  // shape of the plane tiles of the fused passes (0: 16 x 16, 1: 32 x 8); 0 for column tiles
  __host__ __device__ long long count() const { return (long long)ti * tj * tk; }
};

__device__ __forceinline__ void tile_coords(const Tiles &t, int &i, int &j, int &k0, int &k1, int nz) {
  int b = blockIdx.x;
  const int bi = b % t.ti;
  b /= t.ti;
  const int bj = b % t.tj;
  const int bk = b / t.tj;
  i = bi * kTileI + (threadIdx.x & 31);
  j = bj * kTileJ + (threadIdx.x >> 5);
  k0 = bk * t.kz;
  k1 = min(nz, k0 + t.kz);
}

// All four rows of y = K x at node (i,j,k):
//   x-row inprod_x src/aphid.f90:841-865, y-row inprod_y :970-994,
//   z-row inprod_z :1098-1122, node row inprod_p :1227-1276 (0 on the boundary).
// IN(idx) and KK(idx) return the input vector and k^2 at a global index.
template <class IN, class KK>
__device__ __forceinline__ void rows64(const GridDev &g, int i, int j, int k, const IN &in,
                                       const KK &kk, double2 &ox, double2 &oy, double2 &oz,
                                       double2 &op) {
  const Axis &X = g.ax[0], &Y = g.ax[1], &Z = g.ax[2];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double xn4 = X.n4[i], xn5 = X.n5[i], yn4 = Y.n4[j], yn5 = Y.n5[j];
  const double zn4 = Z.n4[k], zn5 = Z.n5[k];
  const double dxc = X.dc[i], dyc = Y.dc[j], dzc = Z.dc[k];
  const int ia = min(i + 1, nx - 1), ib = max(i - 1, 0);
  const int ja = min(j + 1, ny - 1), jb = max(j - 1, 0);
  const int ka = min(k + 1, nz - 1), kb = max(k - 1, 0);
  const long long pc = ixp(g, i, j, k);
  const double2 phc = in(pc), kpc = kk(pc);

  if (i < nx - 1) {
    const double c2 = X.e2[i], c3 = X.e3[i], dxi = X.d[i + 1];
    const double vol = dxi * dyc * dzc;
    const long long c = ixx(g, i, j, k);
    const double2 k2 = kk(c), kp2 = kk(pc + 1);
    const double sum = c2 + c3 + yn4 + yn5 + zn4 + zn5;
    const double2 c1 = make_double2(-sum + k2.x, k2.y);
    double2 s = cmul(c1, in(c));
    s = cadd(s, rmul(c2, in(ixx(g, min(i + 1, nx - 2), j, k))));
    s = cadd(s, rmul(c3, in(ixx(g, ib, j, k))));
    s = cadd(s, rmul(yn4, in(ixx(g, i, ja, k))));
    s = cadd(s, rmul(yn5, in(ixx(g, i, jb, k))));
    s = cadd(s, rmul(zn4, in(ixx(g, i, j, ka))));
    s = cadd(s, rmul(zn5, in(ixx(g, i, j, kb))));
    const double2 gr = rdiv(csub(cmul(in(pc + 1), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dxi);
    ox = rmul(vol, cadd(s, gr));
  }
  if (j < ny - 1) {
    const double c2 = Y.e2[j], c3 = Y.e3[j], dyj = Y.d[j + 1];
    const double vol = dxc * dyj * dzc;
    const long long c = ixy(g, i, j, k);
    const long long pn = pc + nx;
    const double2 k2 = kk(c), kp2 = kk(pn);
    const double sum = c2 + c3 + xn4 + xn5 + zn4 + zn5;
    const double2 c1 = make_double2(-sum + k2.x, k2.y);
    double2 s = cmul(c1, in(c));
    s = cadd(s, rmul(c2, in(ixy(g, i, min(j + 1, ny - 2), k))));
    s = cadd(s, rmul(c3, in(ixy(g, i, jb, k))));
    s = cadd(s, rmul(xn4, in(ixy(g, ia, j, k))));
    s = cadd(s, rmul(xn5, in(ixy(g, ib, j, k))));
    s = cadd(s, rmul(zn4, in(ixy(g, i, j, ka))));
    s = cadd(s, rmul(zn5, in(ixy(g, i, j, kb))));
    const double2 gr = rdiv(csub(cmul(in(pn), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dyj);
    oy = rmul(vol, cadd(s, gr));
  }
  if (k < nz - 1) {
    const double c2 = Z.e2[k], c3 = Z.e3[k], dzk = Z.d[k + 1];
    const double vol = dxc * dyc * dzk;
    const long long c = ixz(g, i, j, k);
    const long long pn = pc + (long long)nx * ny;
    const double2 k2 = kk(c), kp2 = kk(pn);
    const double sum = c2 + c3 + xn4 + xn5 + yn4 + yn5;
    const double2 c1 = make_double2(-sum + k2.x, k2.y);
    double2 s = cmul(c1, in(c));
    s = cadd(s, rmul(c2, in(ixz(g, i, j, min(k + 1, nz - 2)))));
    s = cadd(s, rmul(c3, in(ixz(g, i, j, kb))));
    s = cadd(s, rmul(xn4, in(ixz(g, ia, j, k))));
    s = cadd(s, rmul(xn5, in(ixz(g, ib, j, k))));
    s = cadd(s, rmul(yn4, in(ixz(g, i, ja, k))));
    s = cadd(s, rmul(yn5, in(ixz(g, i, jb, k))));
    const double2 gr = rdiv(csub(cmul(in(pn), csub(kp2, k2)), cmul(phc, csub(kpc, k2))), dzk);
    oz = rmul(vol, cadd(s, gr));
  }
  if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) {
    const double vol = dxc * dyc * dzc;
    const double2 s1 = kpc;
    const long long xc = ixx(g, i, j, k), yc = ixy(g, i, j, k), zc = ixz(g, i, j, k);
    const long long xm = xc - 1, ym = yc - nx, zm = zc - (long long)nx * ny;
    const double2 s2 = kk(xc), s3 = kk(xm), s4 = kk(yc), s5 = kk(ym), s6 = kk(zc), s7 = kk(zm);
    const double2 c2 = rmul(xn4, s2), c3 = rmul(xn5, s3), c4 = rmul(yn4, s4);
    const double2 c5 = rmul(yn5, s5), c6 = rmul(zn4, s6), c7 = rmul(zn5, s7);
    double2 sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
    const double2 c1 = cadd(cneg(sum), cmul(s1, s1));
    double2 s = cmul(c1, phc);
    s = cadd(s, cmul(c2, in(pc + 1)));
    s = cadd(s, cmul(c3, in(pc - 1)));
    s = cadd(s, cmul(c4, in(pc + nx)));
    s = cadd(s, cmul(c5, in(pc - nx)));
    s = cadd(s, cmul(c6, in(pc + (long long)nx * ny)));
    s = cadd(s, cmul(c7, in(pc - (long long)nx * ny)));
    const double2 acc = rmul(vol, s);
    const double2 d2 = rdiv(csub(s2, s1), dxc), d3 = cneg(rdiv(csub(s3, s1), dxc));
    const double2 d4 = rdiv(csub(s4, s1), dyc), d5 = cneg(rdiv(csub(s5, s1), dyc));
    const double2 d6 = rdiv(csub(s6, s1), dzc), d7 = cneg(rdiv(csub(s7, s1), dzc));
    double2 t = cmul(d2, in(xc));
    t = cadd(t, cmul(d3, in(xm)));
    t = cadd(t, cmul(d4, in(yc)));
    t = cadd(t, cmul(d5, in(ym)));
    t = cadd(t, cmul(d6, in(zc)));
    t = cadd(t, cmul(d7, in(zm)));
    op = cadd(acc, rmul(vol, t));
  } else {
    op = make_double2(0.0, 0.0);
  }
}

struct LoadVec {
  const double2 *__restrict__ p;
  __device__ __forceinline__ double2 operator()(long long t) const { return __ldg(p + t); }
};

// ---------------------------------------------------------- wavenumbers
// k^2 at node (i,j,k) of every block, gen_k2_{x,y,z,p}grid
// (src/aphid.f90:1289-1535): the reference fills the boundary by copying the
// nearest interior value, which equals evaluating the interior formula at the
// clamped index.  Result times II*omega*MU0 in the reference's order.
__device__ __forceinline__ double2 times_iwmu(double2 a, double omega) {
  const double2 ii = make_double2(0.0, 1.0);
  return rmul(kMu0, rmul(omega, cmul(a, ii)));
}

static __global__ void k_gen_k2(GridDev g, const double2 *__restrict__ sig, double omega,
                         double2 *__restrict__ k2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz, cx = nx - 1, cy = ny - 1;
  const double *dx = g.ax[0].d, *dy = g.ax[1].d, *dz = g.ax[2].d;
  auto S = [&](int a, int b, int c) { return __ldg(sig + a + (long long)cx * (b + (long long)cy * c)); };
  const int ii = min(max(i, 1), nx - 2), jj = min(max(j, 1), ny - 2), kk = min(max(k, 1), nz - 2);
  if (i < nx - 1) {
    const double dyj = dy[jj + 1], dyjm = dy[jj], dzk = dz[kk + 1], dzkm = dz[kk];
    double2 s = rmul(dyjm * dzkm, S(i, jj - 1, kk - 1));
    s = cadd(s, rmul(dyj * dzkm, S(i, jj, kk - 1)));
    s = cadd(s, rmul(dyj * dzk, S(i, jj, kk)));
    s = cadd(s, rmul(dyjm * dzk, S(i, jj - 1, kk)));
    k2[ixx(g, i, j, k)] = times_iwmu(rdiv(s, (dyjm + dyj) * (dzkm + dzk)), omega);
  }
  if (j < ny - 1) {
    const double dxi = dx[ii + 1], dxim = dx[ii], dzk = dz[kk + 1], dzkm = dz[kk];
    double2 s = rmul(dxim * dzkm, S(ii - 1, j, kk - 1));
    s = cadd(s, rmul(dxi * dzkm, S(ii, j, kk - 1)));
    s = cadd(s, rmul(dxi * dzk, S(ii, j, kk)));
    s = cadd(s, rmul(dxim * dzk, S(ii - 1, j, kk)));
    k2[ixy(g, i, j, k)] = times_iwmu(rdiv(s, (dxim + dxi) * (dzkm + dzk)), omega);
  }
  if (k < nz - 1) {
    const double dxi = dx[ii + 1], dxim = dx[ii], dyj = dy[jj + 1], dyjm = dy[jj];
    double2 s = rmul(dxim * dyjm, S(ii - 1, jj - 1, k));
    s = cadd(s, rmul(dxi * dyjm, S(ii, jj - 1, k)));
    s = cadd(s, rmul(dxi * dyj, S(ii, jj, k)));
    s = cadd(s, rmul(dxim * dyj, S(ii - 1, jj, k)));
    k2[ixz(g, i, j, k)] = times_iwmu(rdiv(s, (dxim + dxi) * (dyjm + dyj)), omega);
  }
  {
    const double dxi = dx[ii + 1], dxim = dx[ii], dyj = dy[jj + 1], dyjm = dy[jj];
    const double dzk = dz[kk + 1], dzkm = dz[kk];
    double2 s = rmul(dxim * dyjm * dzk, S(ii - 1, jj - 1, kk));
    s = cadd(s, rmul(dxi * dyjm * dzk, S(ii, jj - 1, kk)));
    s = cadd(s, rmul(dxi * dyj * dzk, S(ii, jj, kk)));
    s = cadd(s, rmul(dxim * dyj * dzk, S(ii - 1, jj, kk)));
    s = cadd(s, rmul(dxim * dyjm * dzkm, S(ii - 1, jj - 1, kk - 1)));
    s = cadd(s, rmul(dxi * dyjm * dzkm, S(ii, jj - 1, kk - 1)));
    s = cadd(s, rmul(dxi * dyj * dzkm, S(ii, jj, kk - 1)));
    s = cadd(s, rmul(dxim * dyj * dzkm, S(ii - 1, jj, kk - 1)));
    k2[ixp(g, i, j, k)] =
        times_iwmu(rdiv(s, (dxim + dxi) * (dyjm + dyj) * (dzkm + dzk)), omega);
  }
}

// ------------------------------------------------------- Jacobi diagonal
// gen_diag (src/aphid.f90:1542-1725).  It uses 0.5*(d(k)+d(k-1)) where the
// stencils use dxc, and 1 on boundary nodes.
static __global__ void k_gen_diag(GridDev g, const double2 *__restrict__ k2, double2 *__restrict__ dg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double *dx = g.ax[0].d, *dy = g.ax[1].d, *dz = g.ax[2].d;
  const int I = i + 1, J = j + 1, K = k + 1;  // 1-based
  const double dxi = dx[I], dxim = dx[I - 1], dxci = 0.5 * (dxi + dxim);
  const double dyj = dy[J], dyjm = dy[J - 1], dycj = 0.5 * (dyj + dyjm);
  const double dzk = dz[K], dzkm = dz[K - 1], dzck = 0.5 * (dzk + dzkm);
  const double xn4 = mask_hi(I, nx) / dxi / dxci, xn5 = mask_lo(I, nx) / dxim / dxci;
  const double yn4 = mask_hi(J, ny) / dyj / dycj, yn5 = mask_lo(J, ny) / dyjm / dycj;
  const double zn4 = mask_hi(K, nz) / dzk / dzck, zn5 = mask_lo(K, nz) / dzkm / dzck;
  if (i < nx - 1) {
    const double dxcip = 0.5 * (dxi + dx[I + 1]);
    const double c2 = mask_hi(I, nx - 1) / dxcip / dxi, c3 = mask_lo(I, nx) / dxci / dxi;
    const double sum = c2 + c3 + yn4 + yn5 + zn4 + zn5;
    const long long t = ixx(g, i, j, k);
    const double2 kv = k2[t];
    dg[t] = rmul(dxi * dycj * dzck, make_double2(-sum + kv.x, kv.y));
  }
  if (j < ny - 1) {
    const double dycjp = 0.5 * (dyj + dy[J + 1]);
    const double c2 = mask_hi(J, ny - 1) / dycjp / dyj, c3 = mask_lo(J, ny) / dycj / dyj;
    const double sum = c2 + c3 + xn4 + xn5 + zn4 + zn5;
    const long long t = ixy(g, i, j, k);
    const double2 kv = k2[t];
    dg[t] = rmul(dxci * dyj * dzck, make_double2(-sum + kv.x, kv.y));
  }
  if (k < nz - 1) {
    const double dzckp = 0.5 * (dzk + dz[K + 1]);
    const double c2 = mask_hi(K, nz - 1) / dzckp / dzk, c3 = mask_lo(K, nz) / dzck / dzk;
    const double sum = c2 + c3 + xn4 + xn5 + yn4 + yn5;
    const long long t = ixz(g, i, j, k);
    const double2 kv = k2[t];
    dg[t] = rmul(dxci * dycj * dzk, make_double2(-sum + kv.x, kv.y));
  }
  const long long pt = ixp(g, i, j, k);
  if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) {
    const double2 s1 = k2[pt];
    const double2 s2 = k2[ixx(g, i, j, k)], s3 = k2[ixx(g, i - 1, j, k)];
    const double2 s4 = k2[ixy(g, i, j, k)], s5 = k2[ixy(g, i, j - 1, k)];
    const double2 s6 = k2[ixz(g, i, j, k)], s7 = k2[ixz(g, i, j, k - 1)];
    const double2 c2 = rdiv(rdiv(rmul(mask_hi(I, nx), s2), dxi), dxci);
    const double2 c3 = rdiv(rdiv(rmul(mask_lo(I, nx), s3), dxim), dxci);
    const double2 c4 = rdiv(rdiv(rmul(mask_hi(J, ny), s4), dyj), dycj);
    const double2 c5 = rdiv(rdiv(rmul(mask_lo(J, ny), s5), dyjm), dycj);
    const double2 c6 = rdiv(rdiv(rmul(mask_hi(K, nz), s6), dzk), dzck);
    const double2 c7 = rdiv(rdiv(rmul(mask_lo(K, nz), s7), dzkm), dzck);
    const double2 sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
    dg[pt] = rmul(dxci * dycj * dzck, cadd(cneg(sum), cmul(s1, s1)));
  } else {
    dg[pt] = make_double2(1.0, 0.0);
  }
}

// ---------------------------------------------------------------- fields
// gen_fields (src/aphid.f90:2173-2252): B = curl A on faces,
// E = -i omega (A - grad Phi) on edges.
static __global__ void k_fields(GridDev g, double omega, const double2 *__restrict__ a,
                         double2 *__restrict__ bx, double2 *__restrict__ by,
                         double2 *__restrict__ bz, double2 *__restrict__ ex,
                         double2 *__restrict__ ey, double2 *__restrict__ ez) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double dxi = g.ax[0].d[i + 1], dyj = g.ax[1].d[j + 1], dzk = g.ax[2].d[k + 1];
  const long long pc = ixp(g, i, j, k);
  auto E = [&](double2 av, double2 ph1, double2 ph0, double h) {
    const double2 w = csub(av, rdiv(csub(ph1, ph0), h));
    return make_double2(omega * w.y, -(omega * w.x));  // -(i omega w)
  };
  if (bx && j < ny - 1 && k < nz - 1)
    bx[i + (long long)nx * (j + (long long)(ny - 1) * k)] =
        cadd(csub(csub(rdiv(a[ixz(g, i, j + 1, k)], dyj), rdiv(a[ixy(g, i, j, k + 1)], dzk)),
                  rdiv(a[ixz(g, i, j, k)], dyj)),
             rdiv(a[ixy(g, i, j, k)], dzk));
  if (by && i < nx - 1 && k < nz - 1)
    by[i + (long long)(nx - 1) * (j + (long long)ny * k)] =
        cadd(csub(csub(rdiv(a[ixx(g, i, j, k + 1)], dzk), rdiv(a[ixz(g, i + 1, j, k)], dxi)),
                  rdiv(a[ixx(g, i, j, k)], dzk)),
             rdiv(a[ixz(g, i, j, k)], dxi));
  if (bz && i < nx - 1 && j < ny - 1)
    bz[i + (long long)(nx - 1) * (j + (long long)(ny - 1) * k)] =
        cadd(csub(csub(rdiv(a[ixy(g, i + 1, j, k)], dxi), rdiv(a[ixx(g, i, j + 1, k)], dyj)),
                  rdiv(a[ixy(g, i, j, k)], dxi)),
             rdiv(a[ixx(g, i, j, k)], dyj));
  if (ex && i < nx - 1) ex[ixx(g, i, j, k) - g.ox] = E(a[ixx(g, i, j, k)], a[pc + 1], a[pc], dxi);
  if (ey && j < ny - 1) ey[ixy(g, i, j, k) - g.oy] = E(a[ixy(g, i, j, k)], a[pc + nx], a[pc], dyj);
  if (ez && k < nz - 1)
    ez[ixz(g, i, j, k) - g.oz] = E(a[ixz(g, i, j, k)], a[pc + (long long)nx * ny], a[pc], dzk);
}

// ------------------------------------------------------------- receivers
// E and H at mesh nodes with the node interpolation of dump_fields' EM_grid
// output (src/aphid.f90:2012-2165): E along each axis is the mean of the two
// edges through the node, B of each component the mean of the four faces
// around it, H = B / mu0.  (EM_grid's By_grid line repeats the face
// By(i, j, k-1) in place of By(i-1, j, k); the mean here is over the four
// distinct faces.)  The face and edge values are those of k_fields, formed
// with the same operations.
__device__ __forceinline__ double2 face_bx(const GridDev &g, const double2 *a, int i, int j, int k) {
  const double dyj = g.ax[1].d[j + 1], dzk = g.ax[2].d[k + 1];
  return cadd(csub(csub(rdiv(a[ixz(g, i, j + 1, k)], dyj), rdiv(a[ixy(g, i, j, k + 1)], dzk)),
                   rdiv(a[ixz(g, i, j, k)], dyj)),
              rdiv(a[ixy(g, i, j, k)], dzk));
}
__device__ __forceinline__ double2 face_by(const GridDev &g, const double2 *a, int i, int j, int k) {
  const double dxi = g.ax[0].d[i + 1], dzk = g.ax[2].d[k + 1];
  return cadd(csub(csub(rdiv(a[ixx(g, i, j, k + 1)], dzk), rdiv(a[ixz(g, i + 1, j, k)], dxi)),
                   rdiv(a[ixx(g, i, j, k)], dzk)),
              rdiv(a[ixz(g, i, j, k)], dxi));
}
__device__ __forceinline__ double2 face_bz(const GridDev &g, const double2 *a, int i, int j, int k) {
  const double dxi = g.ax[0].d[i + 1], dyj = g.ax[1].d[j + 1];
  return cadd(csub(csub(rdiv(a[ixy(g, i + 1, j, k)], dxi), rdiv(a[ixx(g, i, j + 1, k)], dyj)),
                   rdiv(a[ixy(g, i, j, k)], dxi)),
              rdiv(a[ixx(g, i, j, k)], dyj));
}
// E on the edge of component c (0, 1, 2) that starts at node (i, j, k)
__device__ __forceinline__ double2 edge_e(const GridDev &g, const double2 *a, double omega, int c, int i, int j,
                                          int k) {
  const long long pc = ixp(g, i, j, k);
  const long long t = c == 0 ? ixx(g, i, j, k) : (c == 1 ? ixy(g, i, j, k) : ixz(g, i, j, k));
  const long long step = c == 0 ? 1 : (c == 1 ? (long long)g.nx : (long long)g.nx * g.ny);
  const double h = g.ax[c].d[(c == 0 ? i : (c == 1 ? j : k)) + 1];
  const double2 w = csub(a[t], rdiv(csub(a[pc + step], a[pc]), h));
  return make_double2(omega * w.y, -(omega * w.x));  // -(i omega w)
}

// one thread per (system, receiver): rec holds 0-based interior nodes
// (i, j, k), 1 <= i <= nx-2 etc.; E, H are [nsys][nrec][3]
static __global__ void k_receivers(GridDev g, const double2 *__restrict__ x, long long n, const double *__restrict__ omega,
                                   int nsys, int nrec, const int *__restrict__ rec, double2 *__restrict__ E,
                                   double2 *__restrict__ H) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nsys * nrec) return;
  const int s = (int)(t / nrec), r = (int)(t % nrec);
  const int i = rec[3 * r], j = rec[3 * r + 1], k = rec[3 * r + 2];
  const double2 *a = x + (long long)s * n;
  const double w = omega[s];
  if (E) {
    E[3 * t] = rmul(0.5, cadd(edge_e(g, a, w, 0, i - 1, j, k), edge_e(g, a, w, 0, i, j, k)));
    E[3 * t + 1] = rmul(0.5, cadd(edge_e(g, a, w, 1, i, j - 1, k), edge_e(g, a, w, 1, i, j, k)));
    E[3 * t + 2] = rmul(0.5, cadd(edge_e(g, a, w, 2, i, j, k - 1), edge_e(g, a, w, 2, i, j, k)));
  }
  if (H) {
    const double q = 0.25 / kMu0;
    H[3 * t] = rmul(q, cadd(cadd(face_bx(g, a, i, j - 1, k - 1), face_bx(g, a, i, j, k - 1)),
                            cadd(face_bx(g, a, i, j - 1, k), face_bx(g, a, i, j, k))));
    H[3 * t + 1] = rmul(q, cadd(cadd(face_by(g, a, i - 1, j, k - 1), face_by(g, a, i, j, k - 1)),
                                cadd(face_by(g, a, i - 1, j, k), face_by(g, a, i, j, k))));
    H[3 * t + 2] = rmul(q, cadd(cadd(face_bz(g, a, i - 1, j - 1, k), face_bz(g, a, i, j - 1, k)),
                                cadd(face_bz(g, a, i - 1, j, k), face_bz(g, a, i, j, k))));
  }
}

}  // namespace aphid

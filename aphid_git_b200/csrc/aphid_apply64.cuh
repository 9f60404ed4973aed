// aphid_apply64.cuh -- the complex128 operator y = K x of the plain
// Jacobi-QMR path (aphid_gpu_qmr, the drop-in for `call qmr`), staged
// through shared memory.
//
// The rows are those of rows64 (inprod_x/y/z/p, src/aphid.f90:841-865,
// 970-994, 1098-1122, 1227-1276), with the same arithmetic in the same
// order except that the divisions by cell lengths are multiplications by
// their reciprocals (18 FP64 divides per node were the kernel's critical
// path), on the reference's [Ax|Ay|Az|Phi] layout.  What changes is where the
// neighbours come from.  rows64 reads about 40 complex128 values per node
// straight from global memory, most of them neighbours that other threads
// also read; at 166 registers and 4 warps per block that kernel is
// latency-bound (1.1 TB/s).  Here a 32 x 8 node tile marches along k:
//   - per z-plane, the block stages x, the k^2 of the Ax, Ay and Phi blocks
//     (7 arrays of 34 x 10 values: the tile with a one-node halo, global
//     indices clamped to each block's range, which is exactly the clamping
//     of the reference's neighbour indices), so every x/y neighbour is a
//     shared-memory read;
//   - the z-neighbours of the thread's own node come from the next plane's
//     staging buffer and from registers (plane k-1);
//   - k^2 of Az is only needed at the own node (plane k and k-1): registers.
// Planes are staged by cp.async (global -> shared, no register staging) two
// planes ahead of their use, in a ring of three buffers (planes k, k+1 and
// k+2 in flight), so the loads of the next planes overlap the rows of this
// one.  One block of 256 threads, 112 KB of shared memory, two blocks per SM.
// Global traffic per node and plane: x and k^2 read once (plus the halo,
// 33%), y written once: the 48 B per unknown of the operator.
#pragma once
#include "aphid_qmr64.cuh"

namespace aphid {

constexpr int kAI = 32, kAJ = 8, kAThreads = kAI * kAJ;
constexpr int kAW = kAI + 2, kAH = kAJ + 2, kAN = kAW * kAH;  // staged plane with halo: 34 x 10
constexpr int kAArrays = 7;                                   // x: Ax Ay Az Phi; k^2: Ax Ay Phi
constexpr int kABufs = 3;
constexpr size_t kApplyShm = kABufs * (size_t)kAArrays * kAN * sizeof(double2);
enum { SA_AX = 0, SA_AY, SA_AZ, SA_PH, SK_AX, SK_AY, SK_PH };

// Plane tiles of k_apply64s: kAI x kAJ nodes, kz planes per block.
inline Tiles apply_tiles(int nx, int ny, int nz, int sms) {
  Tiles t{};
  t.ti = (nx + kAI - 1) / kAI;
  t.tj = (ny + kAJ - 1) / kAJ;
  // slab depth: whole waves of 2 blocks per SM, weighed against the extra
  // plane each slab stages
  double best = 1e300;
  for (int kz : {4, 6, 8, 12, 16, 24, 32}) {
    const int tk = (nz + kz - 1) / kz;
    const double waves = (double)t.ti * t.tj * tk / (2.0 * sms);
    const double cost = std::ceil(waves) / waves * (kz + 1.0) / kz;
    if (cost < best - 1e-9) {
      best = cost;
      t.kz = kz;
    }
    if (kz >= nz) break;
  }
  t.kz = std::min(t.kz, nz);
  t.tk = (nz + t.kz - 1) / t.kz;
  return t;
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// MODE: kApplyPlain, kApplyQmr or kApplyEps as for k_apply64.
template <int MODE>
static __global__ void __launch_bounds__(kAThreads, 2) k_apply64s(GridDev g, Tiles tl, const double2 *__restrict__ k2,
                                                                  const double2 *__restrict__ in,
                                                                  double2 *__restrict__ out, Scal64 *sc,
                                                                  double2 *eps_out, double *part, unsigned *cnt) {
  if (MODE == kApplyQmr && sc->done) return;
  extern __shared__ __align__(16) double2 sa[];  // [kABufs][kAArrays][kAN]
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  int b = blockIdx.x;
  const int bi = b % tl.ti;
  b /= tl.ti;
  const int bj = b % tl.tj;
  const int bk = b / tl.tj;
  const int i0 = bi * kAI, j0 = bj * kAJ, k0 = bk * tl.kz, k1 = min(nz, k0 + tl.kz);
  const int tx = threadIdx.x % kAI, ty = threadIdx.x / kAI;
  const int i = i0 + tx, j = j0 + ty;
  const bool live = i < nx && j < ny;
  const int me = (ty + 1) * kAW + (tx + 1);  // own node in a staged plane

  // global index of staged array a at (gi, gj) of plane m, clamped to the
  // block's own range (the reference's min/max neighbour indices)
  auto src = [&](int a, int gi, int gj, int m) -> const double2 * {
    const int c = a < 4 ? a : (a == SK_PH ? 3 : a - 4);
    const int il = c == 0 ? nx - 2 : nx - 1, jl = c == 1 ? ny - 2 : ny - 1;
    gi = min(max(gi, 0), il);
    gj = min(max(gj, 0), jl);
    if (c == 2) m = min(m, nz - 2);
    const long long t = c == 0 ? ixx(g, gi, gj, m) : (c == 1 ? ixy(g, gi, gj, m) : (c == 2 ? ixz(g, gi, gj, m) : ixp(g, gi, gj, m)));
    return (a < 4 ? in : k2) + t;
  };
  // start staging plane m into buffer s (cp.async, one commit group per
  // plane, possibly empty): all arrays with halo, or (own_only) the values at
  // the block's own nodes that the plane below needs; nothing when m is past
  // the slab's last plane + 1 or the mesh
  auto stage = [&](int s, int m) {
    double2 *B = sa + (size_t)s * kAArrays * kAN;
    if (m < nz && m < k1) {
#pragma unroll
      for (int q = 0; q < (kAN + kAThreads - 1) / kAThreads; q++) {
        const int p = threadIdx.x + q * kAThreads;
        if (p < kAN) {
          const int gi = i0 - 1 + p % kAW, gj = j0 - 1 + p / kAW;
#pragma unroll
          for (int a = 0; a < kAArrays; a++) cp_async16(B + a * kAN + p, src(a, gi, gj, m));
        }
      }
    } else if (m < nz && m == k1) {
      const int as[5] = {SA_AX, SA_AY, SA_AZ, SA_PH, SK_PH};
#pragma unroll
      for (int q = 0; q < 5; q++) cp_async16(B + as[q] * kAN + me, src(as[q], i, j, m));
    }
    cp_async_commit();
  };

  const Axis &X = g.ax[0], &Y = g.ax[1], &Z = g.ax[2];
  const int ic = min(i, nx - 1), jc = min(j, ny - 1);
  const double xn4 = X.n4[ic], xn5 = X.n5[ic], yn4 = Y.n4[jc], yn5 = Y.n5[jc];
  const double dxc = X.dc[ic], dyc = Y.dc[jc];
  // reciprocals of the lengths the rows divide by, once per thread (x / d
  // becomes x (1/d): within an ulp, and no FP64 divide in the plane loop)
  const double rdxc = 1.0 / dxc, rdyc = 1.0 / dyc, rdxi = 1.0 / X.d[ic + 1], rdyj = 1.0 / Y.d[jc + 1];
  const bool hx = live && i < nx - 1, hy = live && j < ny - 1;
  const bool pxy = live && i > 0 && i < nx - 1 && j > 0 && j < ny - 1;

  // plane k0-1 (clamped at 0) at the own node: x of the four blocks and k^2 of Az
  double2 axm, aym, azm, phm, kazm;
  {
    const int m = max(k0 - 1, 0);
    axm = __ldg(src(SA_AX, i, j, m));
    aym = __ldg(src(SA_AY, i, j, m));
    azm = __ldg(src(SA_AZ, i, j, m));
    phm = __ldg(src(SA_PH, i, j, m));
    kazm = __ldg(k2 + ixz(g, min(i, nx - 1), min(j, ny - 1), min(m, nz - 2)));
  }
  stage(0, k0);
  stage(1, k0 + 1);

  double ea = 0.0, eb = 0.0;
  for (int k = k0; k < k1; k++) {
    const int s = (k - k0) % kABufs, sn = (k - k0 + 1) % kABufs;
    const bool has_next = k + 1 < nz;
    stage((k - k0 + 2) % kABufs, k + 2);  // into the buffer plane k-1 used
    const double2 kaz = __ldg(k2 + ixz(g, min(i, nx - 1), min(j, ny - 1), min(k, nz - 2)));
    cp_async_wait<1>();  // this thread's copies of planes k and k+1 have landed
    __syncthreads();     // ... and everyone's
    const double2 *C = sa + (size_t)s * kAArrays * kAN;
    const double2 *Nx = has_next ? sa + (size_t)sn * kAArrays * kAN : C;  // plane k+1, clamped at nz-1
    // shared-memory values are read where they are used (short live ranges)
    auto cur = [&](int a, int off) { return C[a * kAN + me + off]; };
    auto nxt = [&](int a) { return Nx[a * kAN + me]; };
    const double2 phc = cur(SA_PH, 0), kpc = cur(SK_PH, 0);
    const double zn4 = Z.n4[k], zn5 = Z.n5[k], dzc = Z.dc[k], rdzc = 1.0 / dzc, rdzk = 1.0 / Z.d[k + 1];
    double2 e = make_double2(0.0, 0.0);
    if (live) {
      const long long pc = ixp(g, i, j, k);
      double2 op = make_double2(0.0, 0.0);
      if (pxy && k > 0 && k < nz - 1) {
        const double vol = dxc * dyc * dzc;
        const double2 s1 = kpc;
        const double2 s2 = cur(SK_AX, 0), s3 = cur(SK_AX, -1), s4 = cur(SK_AY, 0);
        const double2 s5 = cur(SK_AY, -kAW), s6 = kaz, s7 = kazm;
        const double2 c2 = rmul(xn4, s2), c3 = rmul(xn5, s3), c4 = rmul(yn4, s4);
        const double2 c5 = rmul(yn5, s5), c6 = rmul(zn4, s6), c7 = rmul(zn5, s7);
        double2 sum = cadd(cadd(cadd(cadd(cadd(c2, c3), c4), c5), c6), c7);
        const double2 c1 = cadd(cneg(sum), cmul(s1, s1));
        double2 t = cmul(c1, phc);
        t = cadd(t, cmul(c2, cur(SA_PH, 1)));
        t = cadd(t, cmul(c3, cur(SA_PH, -1)));
        t = cadd(t, cmul(c4, cur(SA_PH, kAW)));
        t = cadd(t, cmul(c5, cur(SA_PH, -kAW)));
        t = cadd(t, cmul(c6, nxt(SA_PH)));
        t = cadd(t, cmul(c7, phm));
        const double2 acc = rmul(vol, t);
        const double2 d2 = rmul(rdxc, csub(s2, s1)), d3 = cneg(rmul(rdxc, csub(s3, s1)));
        const double2 d4 = rmul(rdyc, csub(s4, s1)), d5 = cneg(rmul(rdyc, csub(s5, s1)));
        const double2 d6 = rmul(rdzc, csub(s6, s1)), d7 = cneg(rmul(rdzc, csub(s7, s1)));
        double2 u = cmul(d2, cur(SA_AX, 0));
        u = cadd(u, cmul(d3, cur(SA_AX, -1)));
        u = cadd(u, cmul(d4, cur(SA_AY, 0)));
        u = cadd(u, cmul(d5, cur(SA_AY, -kAW)));
        u = cadd(u, cmul(d6, cur(SA_AZ, 0)));
        u = cadd(u, cmul(d7, azm));
        op = cadd(acc, rmul(vol, u));
      }
      out[pc] = op;
      e = cmul(phc, op);
      if (hx) {
        const double c2 = X.e2[i], c3 = X.e3[i], dxi = X.d[i + 1];
        const double vol = dxi * dyc * dzc;
        const double2 kx = cur(SK_AX, 0), kp2 = cur(SK_PH, 1), axc = cur(SA_AX, 0);
        const double sum = c2 + c3 + yn4 + yn5 + zn4 + zn5;
        const double2 c1 = make_double2(-sum + kx.x, kx.y);
        double2 t = cmul(c1, axc);
        t = cadd(t, rmul(c2, cur(SA_AX, 1)));
        t = cadd(t, rmul(c3, cur(SA_AX, -1)));
        t = cadd(t, rmul(yn4, cur(SA_AX, kAW)));
        t = cadd(t, rmul(yn5, cur(SA_AX, -kAW)));
        t = cadd(t, rmul(zn4, nxt(SA_AX)));
        t = cadd(t, rmul(zn5, axm));
        const double2 gr = rmul(rdxi, csub(cmul(cur(SA_PH, 1), csub(kp2, kx)), cmul(phc, csub(kpc, kx))));
        const double2 ox = rmul(vol, cadd(t, gr));
        out[ixx(g, i, j, k)] = ox;
        e = cadd(e, cmul(axc, ox));
      }
      if (hy) {
        const double c2 = Y.e2[j], c3 = Y.e3[j], dyj = Y.d[j + 1];
        const double vol = dxc * dyj * dzc;
        const double2 ky = cur(SK_AY, 0), kp2 = cur(SK_PH, kAW), ayc = cur(SA_AY, 0);
        const double sum = c2 + c3 + xn4 + xn5 + zn4 + zn5;
        const double2 c1 = make_double2(-sum + ky.x, ky.y);
        double2 t = cmul(c1, ayc);
        t = cadd(t, rmul(c2, cur(SA_AY, kAW)));
        t = cadd(t, rmul(c3, cur(SA_AY, -kAW)));
        t = cadd(t, rmul(xn4, cur(SA_AY, 1)));
        t = cadd(t, rmul(xn5, cur(SA_AY, -1)));
        t = cadd(t, rmul(zn4, nxt(SA_AY)));
        t = cadd(t, rmul(zn5, aym));
        const double2 gr = rmul(rdyj, csub(cmul(cur(SA_PH, kAW), csub(kp2, ky)), cmul(phc, csub(kpc, ky))));
        const double2 oy = rmul(vol, cadd(t, gr));
        out[ixy(g, i, j, k)] = oy;
        e = cadd(e, cmul(ayc, oy));
      }
      if (k < nz - 1) {
        const double c2 = Z.e2[k], c3 = Z.e3[k], dzk = Z.d[k + 1];
        const double vol = dxc * dyc * dzk;
        const double2 kz = kaz, kp2 = nxt(SK_PH), azc = cur(SA_AZ, 0);
        const double sum = c2 + c3 + xn4 + xn5 + yn4 + yn5;
        const double2 c1 = make_double2(-sum + kz.x, kz.y);
        double2 t = cmul(c1, azc);
        t = cadd(t, rmul(c2, nxt(SA_AZ)));
        t = cadd(t, rmul(c3, azm));
        t = cadd(t, rmul(xn4, cur(SA_AZ, 1)));
        t = cadd(t, rmul(xn5, cur(SA_AZ, -1)));
        t = cadd(t, rmul(yn4, cur(SA_AZ, kAW)));
        t = cadd(t, rmul(yn5, cur(SA_AZ, -kAW)));
        const double2 gr = rmul(rdzk, csub(cmul(nxt(SA_PH), csub(kp2, kz)), cmul(phc, csub(kpc, kz))));
        const double2 oz = rmul(vol, cadd(t, gr));
        out[ixz(g, i, j, k)] = oz;
        e = cadd(e, cmul(azc, oz));
      }
    }
    ea += e.x;
    eb += e.y;
    axm = cur(SA_AX, 0);
    aym = cur(SA_AY, 0);
    azm = cur(SA_AZ, 0);
    phm = phc;
    kazm = kaz;
    __syncthreads();  // buffer s is free for plane k+3
  }
  cp_async_wait<0>();
  if (MODE == kApplyPlain) return;
  Vals<2> a{{ea, eb}};
  Vals<2> blk = block_reduce<2, kAThreads>(a);
  if (arrive<2, kAThreads>(blk, part, cnt, blockIdx.x, gridDim.x)) {
    Vals<2> tot = final_reduce<2, kAThreads>(part, cnt, gridDim.x);
    if (threadIdx.x == 0) {
      const double2 ev = make_double2(tot.v[0], tot.v[1]);
      if (MODE == kApplyEps) {
        *eps_out = ev;
      } else {
        sc->eps = ev;
        if (guard(sc, finite2(ev), !zero2(ev))) sc->beta = cdiv(ev, sc->del);
      }
    }
  }
}

}  // namespace aphid

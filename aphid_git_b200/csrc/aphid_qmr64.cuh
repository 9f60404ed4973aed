// aphid_qmr64.cuh -- complex128 Jacobi-preconditioned QMR on the device:
// the recurrence of src/aphid_qmr.f90:297-390 as four kernels per iteration,
// each global reduction finished by the last-arriving block, which also runs
// the scalar recurrence, so scalars never leave the GPU.
#pragma once
#include "aphid_op64.cuh"

namespace aphid {

// QMR scalars (src/aphid_qmr.f90:62-68), resident on the device.
struct Scal64 {
  double rho_n, rho_np, c_n, c_nm, theta_n, theta_nm, kap, rnorm, rhsnorm, target;
  double2 eps, del, beta, eta, k1;
  int iter, max_it, conv, done, status, nhist, hist_cap, pad;
};

constexpr int kStreamThreads = 256;

__device__ __forceinline__ bool finite2(double2 a) { return isfinite(a.x) && isfinite(a.y); }
__device__ __forceinline__ bool zero2(double2 a) { return a.x == 0.0 && a.y == 0.0; }

// Ends the solve with a breakdown / non-finite status (the reference would
// carry NaNs to qmr_max_it; we stop and report instead).
__device__ __forceinline__ bool guard(Scal64 *sc, bool ok_finite, bool ok_nonzero) {
  if (!ok_finite) {
    sc->status = 3;  // APHID_NONFINITE
    sc->done = 1;
    return false;
  }
  if (!ok_nonzero) {
    sc->status = 2;  // APHID_BREAKDOWN
    sc->done = 1;
    return false;
  }
  return true;
}

// ||b||^2 -> rhsnorm (src/aphid_qmr.f90:169-172)
static __global__ void __launch_bounds__(kStreamThreads) k_rhsnorm64(long long n, const double2 *__restrict__ b,
                                                            Scal64 *sc, double *part, unsigned *cnt) {
  Vals<1> a{{0.0}};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    a.v[0] += cabs2(b[t]);
  Vals<1> blk = block_reduce<1, kStreamThreads>(a);
  if (arrive<1, kStreamThreads>(blk, part, cnt, blockIdx.x, gridDim.x)) {
    Vals<1> tot = final_reduce<1, kStreamThreads>(part, cnt, gridDim.x);
    if (threadIdx.x == 0) sc->rhsnorm = sqrt(tot.v[0]);
  }
}

// inv_diag = 1/diag (src/aphid_qmr.f90:178-181)
static __global__ void k_invert64(long long n, const double2 *__restrict__ dg, double2 *__restrict__ inv) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    inv[t] = cdiv(make_double2(1.0, 0.0), dg[t]);
}

// r = b - q (q = K x0, or absent for a zero start); ||r|| -> rho_np
// (src/aphid_qmr.f90:245-263)
static __global__ void __launch_bounds__(kStreamThreads) k_init_r64(long long n, const double2 *__restrict__ b,
                                                           const double2 *__restrict__ q,
                                                           double2 *__restrict__ r, Scal64 *sc,
                                                           double *part, unsigned *cnt) {
  Vals<1> a{{0.0}};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const double2 rv = q ? csub(b[t], q[t]) : b[t];
    r[t] = rv;
    a.v[0] += cabs2(rv);
  }
  Vals<1> blk = block_reduce<1, kStreamThreads>(a);
  if (arrive<1, kStreamThreads>(blk, part, cnt, blockIdx.x, gridDim.x)) {
    Vals<1> tot = final_reduce<1, kStreamThreads>(part, cnt, gridDim.x);
    if (threadIdx.x == 0) {
      sc->rho_np = sqrt(tot.v[0]);
      guard(sc, isfinite(sc->rho_np), sc->rho_np != 0.0);
    }
  }
}

// v = r/rho; delta = v^T M^-1 v for the first iteration, then the loop-top
// assignments (src/aphid_qmr.f90:268-285, 299-313)
static __global__ void __launch_bounds__(kStreamThreads) k_init_v64(long long n, const double2 *__restrict__ r,
                                                           const double2 *__restrict__ inv,
                                                           double2 *__restrict__ v, Scal64 *sc,
                                                           double *part, unsigned *cnt) {
  if (sc->done) return;
  const double rho = sc->rho_np;
  Vals<2> a{{0.0, 0.0}};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const double2 vv = rdiv(r[t], rho);
    v[t] = vv;
    const double2 dl = cmul(vv, cmul(vv, inv[t]));
    a.v[0] += dl.x;
    a.v[1] += dl.y;
  }
  Vals<2> blk = block_reduce<2, kStreamThreads>(a);
  if (arrive<2, kStreamThreads>(blk, part, cnt, blockIdx.x, gridDim.x)) {
    Vals<2> tot = final_reduce<2, kStreamThreads>(part, cnt, gridDim.x);
    if (threadIdx.x == 0) {
      sc->c_nm = sc->c_n;
      sc->rho_n = sc->rho_np;
      sc->theta_nm = sc->theta_n;
      sc->del = make_double2(tot.v[0], tot.v[1]);
      if (guard(sc, finite2(sc->del), !zero2(sc->del)))
        sc->k1 = cdiv(rmul(sc->rho_n, sc->del), sc->eps);
    }
  }
}

// step 2: p = M^-1 v - k1 p (src/aphid_qmr.f90:306-320)
static __global__ void __launch_bounds__(kStreamThreads) k_pupd64(long long n, const double2 *__restrict__ v,
                                                         const double2 *__restrict__ inv,
                                                         double2 *__restrict__ p, const Scal64 *sc) {
  if (sc->done) return;
  const double2 k1 = sc->k1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    p[t] = csub(cmul(v[t], inv[t]), cmul(p[t], k1));
}

// step 3a: q = K p with epsilon = p^T q folded in; beta = eps/delta
// (src/aphid_qmr.f90:324-330)
// MODE 0: plain apply; 1: QMR step (epsilon, beta into *sc); 2: epsilon
// written to *eps_out.
enum { kApplyPlain = 0, kApplyQmr = 1, kApplyEps = 2 };
template <int MODE>
static __global__ void __launch_bounds__(kOpThreads) k_apply64(GridDev g, Tiles tl,
                                                      const double2 *__restrict__ k2,
                                                      const double2 *__restrict__ in,
                                                      double2 *__restrict__ out, Scal64 *sc,
                                                      double2 *eps_out, double *part,
                                                      unsigned *cnt) {
  if (MODE == kApplyQmr && sc->done) return;
  int i, j, k0, k1;
  tile_coords(tl, i, j, k0, k1, g.nz);
  Vals<2> a{{0.0, 0.0}};
  if (i < g.nx && j < g.ny) {
    const LoadVec L{in}, KK{k2};
    for (int k = k0; k < k1; k++) {
      double2 ox, oy, oz, op;
      rows64(g, i, j, k, L, KK, ox, oy, oz, op);
      const long long pc = ixp(g, i, j, k);
      out[pc] = op;
      double2 e = cmul(L(pc), op);
      if (i < g.nx - 1) {
        const long long t = ixx(g, i, j, k);
        out[t] = ox;
        e = cadd(e, cmul(L(t), ox));
      }
      if (j < g.ny - 1) {
        const long long t = ixy(g, i, j, k);
        out[t] = oy;
        e = cadd(e, cmul(L(t), oy));
      }
      if (k < g.nz - 1) {
        const long long t = ixz(g, i, j, k);
        out[t] = oz;
        e = cadd(e, cmul(L(t), oz));
      }
      a.v[0] += e.x;
      a.v[1] += e.y;
    }
  }
  if (MODE == kApplyPlain) return;
  Vals<2> blk = block_reduce<2, kOpThreads>(a);
  if (arrive<2, kOpThreads>(blk, part, cnt, blockIdx.x, gridDim.x)) {
    Vals<2> tot = final_reduce<2, kOpThreads>(part, cnt, gridDim.x);
    if (threadIdx.x == 0) {
      const double2 e = make_double2(tot.v[0], tot.v[1]);
      if (MODE == kApplyEps) {
        *eps_out = e;
      } else {
        sc->eps = e;
        if (guard(sc, finite2(e), !zero2(e))) sc->beta = cdiv(e, sc->del);
      }
    }
  }
}

// step 3b + 4: rho = ||q - beta v||; theta, c, eta, kappa
// (src/aphid_qmr.f90:332-345)
static __global__ void __launch_bounds__(kStreamThreads) k_rho64(long long n, const double2 *__restrict__ q,
                                                        const double2 *__restrict__ v, Scal64 *sc,
                                                        double *part, unsigned *cnt) {
  if (sc->done) return;
  const double2 beta = sc->beta;
  Vals<1> a{{0.0}};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    a.v[0] += cabs2(csub(q[t], cmul(v[t], beta)));
  Vals<1> blk = block_reduce<1, kStreamThreads>(a);
  if (arrive<1, kStreamThreads>(blk, part, cnt, blockIdx.x, gridDim.x)) {
    Vals<1> tot = final_reduce<1, kStreamThreads>(part, cnt, gridDim.x);
    if (threadIdx.x == 0) {
      const double rho = sqrt(tot.v[0]);
      sc->rho_np = rho;
      if (guard(sc, isfinite(rho), rho != 0.0)) {
        const double2 b = sc->beta;
        sc->theta_n = rho * rho / sc->c_nm / (b.x * b.x + b.y * b.y);
        sc->c_n = 1.0 / (1.0 + sc->theta_n);
        sc->eta = cdiv(rmul(sc->c_n, rmul(sc->rho_n, cneg(sc->eta))), rmul(sc->c_nm, b));
        sc->kap = sc->theta_nm * sc->c_n;
        guard(sc, finite2(sc->eta) && isfinite(sc->theta_n), true);
      }
    }
  }
}

// step 4 updates + stop test: d, x, s, r, v; ||r||; next delta and k1
// (src/aphid_qmr.f90:347-390, 299-313)
static __global__ void __launch_bounds__(kStreamThreads) k_upd64(long long n, const double2 *__restrict__ p,
                                                        const double2 *__restrict__ q,
                                                        const double2 *__restrict__ inv,
                                                        double2 *__restrict__ d, double2 *__restrict__ x,
                                                        double2 *__restrict__ s, double2 *__restrict__ r,
                                                        double2 *__restrict__ v, Scal64 *sc,
                                                        double *hist, double *part, unsigned *cnt) {
  if (sc->done) return;
  const double2 eta = sc->eta, beta = sc->beta;
  const double kap = sc->kap, rho = sc->rho_np;
  Vals<3> a{{0.0, 0.0, 0.0}};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const double2 qq = q[t];
    const double2 dd = cadd(cmul(p[t], eta), rmul(kap, d[t]));
    d[t] = dd;
    x[t] = cadd(x[t], dd);
    const double2 ss = cadd(cmul(qq, eta), rmul(kap, s[t]));
    s[t] = ss;
    const double2 rr = csub(r[t], ss);
    r[t] = rr;
    const double2 vn = rdiv(csub(qq, cmul(v[t], beta)), rho);
    v[t] = vn;
    a.v[0] += cabs2(rr);
    const double2 dl = cmul(vn, cmul(vn, inv[t]));
    a.v[1] += dl.x;
    a.v[2] += dl.y;
  }
  Vals<3> blk = block_reduce<3, kStreamThreads>(a);
  if (arrive<3, kStreamThreads>(blk, part, cnt, blockIdx.x, gridDim.x)) {
    Vals<3> tot = final_reduce<3, kStreamThreads>(part, cnt, gridDim.x);
    if (threadIdx.x == 0) {
      const double rn = sqrt(tot.v[0]);
      sc->rnorm = rn;
      if (hist && sc->nhist < sc->hist_cap) hist[sc->nhist] = rn;
      sc->nhist++;
      if (!isfinite(rn)) {
        sc->status = 3;
        sc->done = 1;
        return;
      }
      if (rn < sc->target * sc->rhsnorm) sc->conv = 1;
      if (!sc->conv && sc->iter <= sc->max_it) sc->iter++;
      if (sc->conv || sc->iter > sc->max_it) {
        sc->status = sc->conv ? 0 : 1;
        sc->done = 1;
        return;
      }
      sc->c_nm = sc->c_n;
      sc->rho_n = sc->rho_np;
      sc->theta_nm = sc->theta_n;
      sc->del = make_double2(tot.v[1], tot.v[2]);
      if (guard(sc, finite2(sc->del), !zero2(sc->del)))
        sc->k1 = cdiv(rmul(sc->rho_n, sc->del), sc->eps);
    }
  }
}

// ||b - q||^2 for the true residual of the returned solution
static __global__ void __launch_bounds__(kStreamThreads) k_resid64(long long n, const double2 *__restrict__ b,
                                                          const double2 *__restrict__ q, double *out,
                                                          double *part, unsigned *cnt) {
  Vals<1> a{{0.0}};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    a.v[0] += cabs2(csub(b[t], q[t]));
  Vals<1> blk = block_reduce<1, kStreamThreads>(a);
  if (arrive<1, kStreamThreads>(blk, part, cnt, blockIdx.x, gridDim.x)) {
    Vals<1> tot = final_reduce<1, kStreamThreads>(part, cnt, gridDim.x);
    if (threadIdx.x == 0) *out = tot.v[0];
  }
}

}  // namespace aphid

// aphid_sweep.cuh -- batched, mixed-precision frequency sweep.
//
// S systems (frequency x source) on one mesh advance together.  Each system
// runs FP64 defect correction (iterative refinement):
//   r = b - K x        complex128 operator, true residual, FP64 norms
//   solve K e = r      complex64 QMR on the symmetrically Jacobi-scaled
//                      operator K~ = D^-1/2 K D^-1/2 (D = gen_diag), FP64
//                      inner products and Lanczos scalars
//   x += e             FP64 accumulation
// until ||r|| < target ||b||.  The Jacobi diagonal is FP64; its inverse is
// stored once per system in complex64.  k^2 is never stored: it is formed per
// system from the cell averages sigma-bar (and eps-bar) shared by all
// systems, k^2 = i omega mu0 (sigma-bar + i omega eps0 eps-bar), which is
// gen_k2_*grid (src/aphid.f90:1289-1535) for the linear models R, C, I.
//
// Layout: x and b stay complex128 in the reference's [Ax|Ay|Az|Phi] order.
// The complex64 inner state is node-indexed, [component][k][j][i] per vector
// with rows padded to a multiple of 4 nodes, so all four components of a node
// share one index, every row starts on a 16-byte boundary (TMA-loadable), and
// components that do not exist at a node (x at i = nx-1, ...) are stored
// zeros.
//
// Inner solver: the reference's coupled two-term QMR recurrence
// (src/aphid_qmr.f90:297-372) with M = I on K~, carried in "u-space": every
// Krylov vector z~ of the scaled problem is stored as z^ = D^-1/2 z~, so the
// operator is q^ = D^-1 K p^ (no scaling of the stencil's inputs), the
// solution correction is x^ itself, and the scaled-space inner products are
// weighted sums, z~^T y~ = sum D z^ y^ and ||z~||^2 = sum |D| |z^|^2.
//
// One fused pass per QMR iteration n (k_sw_pass).  It reads q^_{n-1},
// v^_{n-1}, p^_{n-1} with halos and forms, per node,
//   vt_n = q^_{n-1} - beta_{n-1} v^_{n-1},  v^_n = vt_n / rho_n,
//   p^_n = v^_n - k1_n p^_{n-1}   (k1_n = rho_n delta_n / epsilon_{n-1}),
// applies the stencil, q^_n = D^-1 K p^_n, and stores v^_n, q^_n into the
// other (q, v) buffer set (the halo reads of the next pass must not see this
// pass's writes) and p^_n into the next slot of a ring of R+1 p^ buffers.  It
// reduces epsilon_n = p~_n^T q~_n and the six inner products of v~_n and q~_n
// from which rho_{n+1} = ||q~_n - beta_n v~_n|| and delta_{n+1} =
// v~_{n+1}^T v~_{n+1} follow without another pass over the vectors (beta_n is
// not known until the pass has finished).  The last block to finish runs the
// scalar recurrences and appends (eta_n, kappa_n, ring slot of p^_n) to the
// system's pending-update list.  The expansions are accumulated in FP64 from
// per-node FP32 products; the cycle restarts from the FP64 residual when they
// lose accuracy (see kCancel and kDrift).  No residual vectors are kept: the
// stop test uses the quasi-residual tau_n = ||r~_0|| prod sqrt(theta_i c_i),
// which a complex128 true-residual monitor checks once per graph round.
//
// The solution update d^_n = eta_n p^_n + kappa_n d^_{n-1}, x += d^_n is not
// in the pass: after every R passes a streaming kernel (k_sw_dxupd) applies
// the pending updates of each system from the ring, accumulating the R
// increments in FP64 straight into the reference-layout solution x.  The pass
// then moves 48 B per unknown instead of 80 B (q^ v^ p^ read and written; d^
// and the solution move once per R iterations, (R + 1) x 8 + 32 B), and it
// keeps no d^ staging in shared memory.
//
// Every system has a phase (OUTER -> INNER -> OUTER ... -> DONE);
// every block first reads its system's phase and returns when the kernel does
// not apply, which masks converged systems out of the remaining launches.
#pragma once
#include <cuda.h>

#include "aphid_qmr64.cuh"

namespace aphid {

enum { PH_OUTER = 0, PH_INNER = 2, PH_DONE = 3 };
enum { CNT_RESID = 0, CNT_PASS = 2, CNT_BNORM = 4, CNT_CHECK = 5, CNT_DX = 6, CNT_KINDS = 7 };
constexpr int kParts = 12;  // partial sums per slot and system

// An inner cycle ends when the true residual, checked once per graph round,
// falls this far behind its best tracking of the quasi-residual: the complex64
// recurrence has reached its floor and only a restart from the FP64 residual
// makes progress.
constexpr double kStagnation = 16.0;
// For complex64 inner solves the monitor runs only once the quasi-residual
// predicts a true residual (rnorm at the cycle start times tau / tau0) below
// this fraction of ||b||, or below 30 x the target: above both, neither
// convergence nor the complex64 floor (about 1e-6 ||b||) can have been
// reached.  Complex128 inner solves track the true residual, so their monitor
// waits for 10 x the target (SweepSys::mon_level).
constexpr double kMonitorLevel = 1e-4;
// Between that level and kCheckNear x the target the monitor checks every
// kCheckEvery inner iterations instead of every graph round: each check is a
// complex128 operator over the system, about a sixth of a round's cost when a
// system runs on alone for thousands of iterations.
constexpr double kCheckNear = 10.0;
constexpr int kCheckEvery = 64;
// rho_{n+1}^2 from the expansion ||q||^2 - 2 Re(conj(beta) v^H q) + |beta|^2
// ||v||^2 is trusted down to this fraction of ||q||^2; below it the new
// Lanczos vector is treated as zero (the iterate is final for this cycle).
constexpr double kCancel = 1e-10;
// the cycle also restarts when the stored v~_n has drifted from ||v~_n|| = 1
// or from v~_n^T v~_n = delta_n by more than this (relative to ||v~_n||^2)
constexpr double kDrift = 1e-3;
// A cycle whose quasi-residual has not halved over this many iterations (the
// default of SweepSys::stall_window) has stalled: the complex64 Lanczos
// process can stagnate outright (seen on seafloor models at 0.27-1.35 Hz,
// where complex128 converges in about 500 iterations).  The cycle ends and
// the next one restarts from the FP64 residual.
constexpr int kStallWindow = 400;
// Complex-symmetric Lanczos normalises v~ in the Hermitian norm but divides by
// the bilinear form delta = v~^T v~.  On strongly conducting layers under air
// |delta| / ||v~||^2 falls to 1e-7 and below within a few dozen iterations
// (seafloor models, 0.27-1.35 Hz), where complex64 storage noise (about 6e-8
// of ||v~||^2) is a sizeable part of delta: the complex64 process loses
// biorthogonality and stalls, while complex128 converges.  With escalation on,
// a system whose |delta_{n+1}| falls below this fraction of ||v~_n||^2 ends
// with kStEscalated and is finished by the complex128 pass (k_sw_pass64).
// Heterogeneous land models stay above 1e-5.
constexpr double kDeltaFloor = 1e-6;
constexpr int kStEscalated = 4;
// A complex64 cycle that lowers the FP64 residual by less than this factor is
// slow; with escalation on, kSlowCycles slow cycles in a row also end the
// system with kStEscalated.  Restarted complex64 cycles can keep stalling at
// the plateau of an unrestarted recurrence (sweep meshes with km cells at
// 1e-3 Hz: 35 cycles in 20000 iterations without reaching 1e-8, while
// complex128 converges) without the bilinear form ever collapsing.
constexpr double kSlowCycle = 0.5;
constexpr int kSlowCycles = 2;
// longest pending-update list (the p^ ring has up to kMaxRing + 1 slots)
constexpr int kMaxRing = 8;

struct SweepSys {
  double omega, ka, kb;  // k^2 = (-ka * eps-bar, kb * sigma-bar)
  double rho_n, rho_np, c_n, c_nm, theta_n, theta_nm, kap, tau, tau0;
  double2 eps, del, beta, eta, k1;
  double vscale;             // 1 / rho_n
  double2 eta_h[kMaxRing];   // pending solution updates d = eta p + kap d, x += d,
  double kap_h[kMaxRing];    //   in order, p^ from ring slot slot_h
  int slot_h[kMaxRing];
  int npend;                 // entries of the pending list
  int pslot;                 // ring slot of the last pass's p^
  double bnorm, rnorm, inner_tol, target, rt0;
  double ratio_min, mon_rn;  // true-residual monitor of the running inner cycle
  int phase, has_inner, inner_it, total_it, outer_it, max_it, max_outer, status;
  int checks;
  int last_check_it;         // total_it at the monitor's last check
  int cur;                   // buffer set holding q^, v^ of the last pass
  int restarts;              // inner cycles ended by kCancel / kDrift / a stall
  double tau_win;            // tau at the start of the current stall window
  int win_it;                // inner iteration at which that window started
  int stall_window;          // window length (INT_MAX: no stall test)
  int escalate;              // 1: end with kStEscalated when the bilinear form collapses
  int escalated;             // set by the pass; the outer step then ends the system
  int slow;                  // slow cycles in a row (see kSlowCycle)
  double rprev;              // FP64 residual norm at the previous outer step
  double mon_level;          // the monitor runs once the predicted true residual is below this x ||b||
};

// Plane tiles of the fused passes, marching along k, in two shapes that the
// autotuner chooses between: TS 0, 16 x 16 nodes (the smallest halo; fastest
// for one system) and TS 1, 32 x 8 (36-node staged rows of 288 B in
// complex64; fastest for large batches, 16.0 against 19.0 ms per pass over 24
// systems of 50.8 M unknowns).  Staged planes cover i0-2 .. i0+I+1 (even
// start: 16-byte TMA x origin) and j0-1 .. j0+J; sigma-bar planes cover
// i0-4 .. i0+I+3.  256 threads, one per node of the tile.
template <int TS>
struct PT {
  static constexpr int I = TS ? 32 : 16, J = TS ? 8 : 16;
  static constexpr int W = I + 4, H = J + 2, N = W * H;  // staged plane: 20 x 18 or 36 x 10
  static constexpr int KW = I + 8, KN = KW * H;          // sigma-bar plane: 24 x 18 or 40 x 10
};
constexpr int kPThreads = 256, kTileShapes = 2;
static_assert(PT<0>::I * PT<0>::J == kPThreads && PT<1>::I * PT<1>::J == kPThreads, "one thread per tile node");

struct NodeLayout {
  int nxp;      // padded row length (multiple of 4)
  long long N;  // nodes per component: nxp * ny * nz
};

struct SweepDev {
  GridDev g;
  NodeLayout L;
  Tiles t;   // 32 x 4 column tiles (complex128 residual passes)
  Tiles tp;  // plane tiles of the fused passes (shape tp.ts, see PT)
  long long n;           // unknowns per system (reference layout)
  int nsys, bps;         // systems; blocks per system of the pointwise kernels
  long long slots;       // partial-sum slots per system
  const double *sig;     // sigma-bar per unknown (FP64, reference layout)
  const double *epsr;    // eps-bar per unknown, or null (= 1)
  const float *sig32, *epsr32;  // the same, FP32, node layout [4][N]
  // per-system model arrays (Cole-Cole: sigma-hat depends on omega): system s
  // reads sig + s mref and the node-layout arrays at + s mnode; 0 when all
  // systems share one model
  long long mref, mnode;
  const float4 *ax32;    // per axis: [n] (n4, n5, dc, 1/dc), then [n] (e2, e3, d, 1/d) of edge m
  float2 *W;             // [2 sets][nsys][q^, v^][4][N] complex64
  float2 *P;             // [ring + 1 slots][nsys][4][N]: p^
  float2 *dd;            // [nsys][4][N]: d^
  int ring;              // R: pending updates between two k_sw_dxupd launches
  double2 *x64, *b;              // [nsys][n] complex128, reference layout
  SweepSys *sys;
  double *part;                  // [nsys][slots][kParts]
  unsigned *cnt;                 // [CNT_KINDS][nsys]
  int *ndone;
  int *err;                      // set when a bounded wait gives up
  float tmix;                    // 1; 0 in timing launches (d^, x^ rewritten unchanged)
  int timing;                    // fused passes: 1 in timing launches (see k_sw_pass)
  int *work;                     // [2]: next work item, blocks finished (complex64 pass)
  const int *order;              // plane tiles in the order the pass takes them
  int *active;                   // [1 + nsys]: count, then the systems in their inner cycle (k_sw_active)
  // complex128 inner storage (k_sw_pass64): same layouts, double2
  double2 *W64, *P64, *dd64;
  int ring64;
  const double *sig64, *epsr64;  // sigma-bar / eps-bar, FP64, node layout [4][N]
  const double4 *ax64;           // the axis tables of ax32 in FP64
};

// q^ (vec 0) or v^ (vec 1) of buffer set `set`; p^ of ring slot `slot`
__device__ __forceinline__ float2 *wvec(const SweepDev &D, int set, int sys, int vec) {
  return D.W + ((long long)(set * D.nsys + sys) * 2 + vec) * 4 * D.L.N;
}
__device__ __forceinline__ float2 *pvec(const SweepDev &D, int slot, int sys) {
  return D.P + (long long)(slot * D.nsys + sys) * 4 * D.L.N;
}
__device__ __forceinline__ double4 ldg4(const double4 *p) {
  const double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ double2 *wvec64(const SweepDev &D, int set, int sys, int vec) {
  return D.W64 + ((long long)(set * D.nsys + sys) * 2 + vec) * 4 * D.L.N;
}
__device__ __forceinline__ double2 *pvec64(const SweepDev &D, int slot, int sys) {
  return D.P64 + (long long)(slot * D.nsys + sys) * 4 * D.L.N;
}
__device__ __forceinline__ long long nd_of(const SweepDev &D, int i, int j, int k) {
  return i + (long long)D.L.nxp * (j + (long long)D.g.ny * k);
}
__device__ __forceinline__ bool exists(const GridDev &g, int c, int i, int j, int k) {
  return c == 0 ? i < g.nx - 1 : (c == 1 ? j < g.ny - 1 : (c == 2 ? k < g.nz - 1 : true));
}
__device__ __forceinline__ long long ref_of(const GridDev &g, int c, int i, int j, int k) {
  return c == 0 ? ixx(g, i, j, k) : (c == 1 ? ixy(g, i, j, k) : (c == 2 ? ixz(g, i, j, k) : ixp(g, i, j, k)));
}

// ------------------------------------------------- complex64 Jacobi scaling
// The Jacobi diagonal D of one node in FP32: the diagonal entries of the
// stencil rows, (-sum of the edge row's coefficients + k^2) vol on edges and
// (k_p^4 - sum_m n_m k^2_m) vol on interior nodes; zero where a component does
// not exist, 1 for boundary Phi (the reference's diag_p = 1, its row being
// zero).  This is gen_diag (src/aphid.f90:1542-1725) except on the outermost
// layers, where gen_diag takes its coefficients from the clamped interior
// index and so is not the operator's own diagonal; any diagonal scaling
// serves the inner solver, and the complex128 path keeps gen_diag exactly.
// Inputs: the FP32 axis tables of the node (x, y, z), sigma-bar (eps-bar)
// of its four components, of the x-edge at i-1, the y-edge at j-1 and the
// z-edge at k-1.  Written with non-contracting operations so that the
// complex64 pass and the residual pass, which call it on the same values,
// get the same bits.
__device__ __forceinline__ void jacobi32(float4 XA, float4 XB, float4 YA, float4 YB, float4 ZA, float4 ZB, float sx,
                                         float sy, float sz, float sp0, float sxm, float sym, float s2m, float ex,
                                         float ey, float ez, float ep0, float exm, float eym, float e2m, bool hx,
                                         bool hy, bool hz, bool pin, float ka, float kb, float2 dg[4]) {
  auto M = [](float a, float b) { return __fmul_rn(a, b); };
  auto A = [](float a, float b) { return __fadd_rn(a, b); };
  // edge row: vol (k^2 - sum) with k^2 = (-ka e, kb s)
  auto edge = [&](float vol, float sum, float s_, float e_) {
    return make_float2(M(vol, __fsub_rn(-M(ka, e_), sum)), M(vol, M(kb, s_)));
  };
  const float xn4 = XA.x, xn5 = XA.y, dxc = XA.z, yn4 = YA.x, yn5 = YA.y, dyc = YA.z, zn4 = ZA.x, zn5 = ZA.y,
              dzc = ZA.z;
  dg[0] = hx ? edge(M(M(XB.z, dyc), dzc), A(A(A(A(A(XB.x, XB.y), yn4), yn5), zn4), zn5), sx, ex)
             : make_float2(0.f, 0.f);
  dg[1] = hy ? edge(M(M(dxc, YB.z), dzc), A(A(A(A(A(YB.x, YB.y), xn4), xn5), zn4), zn5), sy, ey)
             : make_float2(0.f, 0.f);
  dg[2] = hz ? edge(M(M(dxc, dyc), ZB.z), A(A(A(A(A(ZB.x, ZB.y), xn4), xn5), yn4), yn5), sz, ez)
             : make_float2(0.f, 0.f);
  if (pin) {
    const float vol = M(M(dxc, dyc), dzc);
    const float s1r = -M(ka, ep0), s1i = M(kb, sp0);
    // sum_m n_m k^2_m, then k_p^4 - that sum
    const float nr = A(A(A(A(A(M(xn4, ex), M(xn5, exm)), M(yn4, ey)), M(yn5, eym)), M(zn4, ez)), M(zn5, e2m));
    const float ni = A(A(A(A(A(M(xn4, sx), M(xn5, sxm)), M(yn4, sy)), M(yn5, sym)), M(zn4, sz)), M(zn5, s2m));
    const float pr = __fsub_rn(M(s1r, s1r), M(s1i, s1i)), pi = M(2.f, M(s1r, s1i));
    dg[3] = make_float2(M(vol, A(pr, M(ka, nr))), M(vol, __fsub_rn(pi, M(kb, ni))));
  } else {
    dg[3] = make_float2(1.f, 0.f);
  }
}

// 1/D, |D| and 1/|D| of a diagonal entry, scaled against overflow of |D|^2;
// zeros for D = 0
__device__ __forceinline__ void jacobi_weights(float2 z, float2 &inv, float &absd, float &rabsd) {
  const float mz = fmaxf(fabsf(z.x), fabsf(z.y));
  inv = make_float2(0.f, 0.f);
  absd = rabsd = 0.f;
  if (mz > 0.f) {
    const float sc = __frcp_rn(mz), za = __fmul_rn(z.x, sc), zb = __fmul_rn(z.y, sc);
    const float n2 = __fadd_rn(__fmul_rn(za, za), __fmul_rn(zb, zb)), rn = rsqrtf(n2);
    const float t = __fmul_rn(sc, __fmul_rn(rn, rn));
    inv = make_float2(__fmul_rn(za, t), -__fmul_rn(zb, t));
    absd = __fmul_rn(__fmul_rn(mz, n2), rn);
    rabsd = __fmul_rn(sc, rn);
  }
}

// The same two functions in FP64 for the complex128 pass (k_sw_pass64) and
// the kernels that share its state: the diagonal of K from the FP64 axis
// tables and sigma-bar, and D^-1, |D|, 1/|D| -- all with non-contracting
// intrinsics so that every kernel forms bit-identical values.  jacobi64 is
// assembled from its pieces: the entry of one edge component (vol, the sum of
// the row's coefficients, sigma-bar and eps-bar of the edge) and of an
// interior Phi node, so that a kernel forming only some components of a node
// gets the bits that jacobi64 gives.
__device__ __forceinline__ double2 jac64_edge(double vol, double sum, double s_, double e_, double ka, double kb) {
  return make_double2(__dmul_rn(vol, __dsub_rn(-__dmul_rn(ka, e_), sum)), __dmul_rn(vol, __dmul_rn(kb, s_)));
}
__device__ __forceinline__ double2 jac64_x(double4 XA, double4 XB, double4 YA, double4 ZA, double sx, double ex,
                                           double ka, double kb) {
  auto M = [](double a, double b) { return __dmul_rn(a, b); };
  auto A = [](double a, double b) { return __dadd_rn(a, b); };
  return jac64_edge(M(M(XB.z, YA.z), ZA.z), A(A(A(A(A(XB.x, XB.y), YA.x), YA.y), ZA.x), ZA.y), sx, ex, ka, kb);
}
__device__ __forceinline__ double2 jac64_y(double4 XA, double4 YA, double4 YB, double4 ZA, double sy, double ey,
                                           double ka, double kb) {
  auto M = [](double a, double b) { return __dmul_rn(a, b); };
  auto A = [](double a, double b) { return __dadd_rn(a, b); };
  return jac64_edge(M(M(XA.z, YB.z), ZA.z), A(A(A(A(A(YB.x, YB.y), XA.x), XA.y), ZA.x), ZA.y), sy, ey, ka, kb);
}
__device__ __forceinline__ double2 jac64_z(double4 XA, double4 YA, double4 ZA, double4 ZB, double sz, double ez,
                                           double ka, double kb) {
  auto M = [](double a, double b) { return __dmul_rn(a, b); };
  auto A = [](double a, double b) { return __dadd_rn(a, b); };
  return jac64_edge(M(M(XA.z, YA.z), ZB.z), A(A(A(A(A(ZB.x, ZB.y), XA.x), XA.y), YA.x), YA.y), sz, ez, ka, kb);
}
__device__ __forceinline__ double2 jac64_p(double4 XA, double4 YA, double4 ZA, double sx, double sy, double sz,
                                           double sp0, double sxm, double sym, double s2m, double ex, double ey,
                                           double ez, double ep0, double exm, double eym, double e2m, double ka,
                                           double kb) {
  auto M = [](double a, double b) { return __dmul_rn(a, b); };
  auto A = [](double a, double b) { return __dadd_rn(a, b); };
  const double xn4 = XA.x, xn5 = XA.y, dxc = XA.z, yn4 = YA.x, yn5 = YA.y, dyc = YA.z, zn4 = ZA.x, zn5 = ZA.y,
               dzc = ZA.z;
  const double vol = M(M(dxc, dyc), dzc);
  const double s1r = -M(ka, ep0), s1i = M(kb, sp0);
  const double nr = A(A(A(A(A(M(xn4, ex), M(xn5, exm)), M(yn4, ey)), M(yn5, eym)), M(zn4, ez)), M(zn5, e2m));
  const double ni = A(A(A(A(A(M(xn4, sx), M(xn5, sxm)), M(yn4, sy)), M(yn5, sym)), M(zn4, sz)), M(zn5, s2m));
  const double pr = __dsub_rn(M(s1r, s1r), M(s1i, s1i)), pi = M(2.0, M(s1r, s1i));
  return make_double2(M(vol, A(pr, M(ka, nr))), M(vol, __dsub_rn(pi, M(kb, ni))));
}
__device__ __forceinline__ void jacobi64(double4 XA, double4 XB, double4 YA, double4 YB, double4 ZA, double4 ZB,
                                         double sx, double sy, double sz, double sp0, double sxm, double sym,
                                         double s2m, double ex, double ey, double ez, double ep0, double exm,
                                         double eym, double e2m, bool hx, bool hy, bool hz, bool pin, double ka,
                                         double kb, double2 dg[4]) {
  const double2 zero = make_double2(0.0, 0.0);
  dg[0] = hx ? jac64_x(XA, XB, YA, ZA, sx, ex, ka, kb) : zero;
  dg[1] = hy ? jac64_y(XA, YA, YB, ZA, sy, ey, ka, kb) : zero;
  dg[2] = hz ? jac64_z(XA, YA, ZA, ZB, sz, ez, ka, kb) : zero;
  dg[3] = pin ? jac64_p(XA, YA, ZA, sx, sy, sz, sp0, sxm, sym, s2m, ex, ey, ez, ep0, exm, eym, e2m, ka, kb)
              : make_double2(1.0, 0.0);
}
__device__ __forceinline__ void jacobi_weights(double2 z, double2 &inv, double &absd, double &rabsd) {
  // |z|^2 stays far inside the FP64 range here, so no pre-scaling: one
  // reciprocal square root gives D^-1 = conj(z) / |z|^2, |D| and 1/|D|
  const double n2 = __dadd_rn(__dmul_rn(z.x, z.x), __dmul_rn(z.y, z.y));
  inv = make_double2(0.0, 0.0);
  absd = rabsd = 0.0;
  if (n2 > 0.0) {
    const double rn = rsqrt(n2), t = __dmul_rn(rn, rn);
    inv = make_double2(__dmul_rn(z.x, t), -__dmul_rn(z.y, t));
    absd = __dmul_rn(n2, rn);
    rabsd = rn;
  }
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
struct K2Ref64 {  // k^2 from the FP64 averages of one system (reference layout)
  GridDev g;
  const double *__restrict__ sig, *__restrict__ epsr;
  double ka, kb;
  __device__ __forceinline__ double2 operator()(int c, int i, int j, int k) const {
    const long long t = ref_of(g, c, i, j, k);
    const double e = epsr ? __ldg(epsr + t) : 1.0;
    return make_double2(-ka * e, kb * __ldg(sig + t));
  }
};
template <typename T>
struct XRefT {  // x (reference layout), optionally + x^ (node layout, complex64 or complex128)
  GridDev g;
  const double2 *__restrict__ x64;
  const T *__restrict__ xt;  // null: x only
  int nxp;
  long long N;
  __device__ __forceinline__ double2 operator()(int c, int i, int j, int k) const {
    double2 r = __ldg(x64 + ref_of(g, c, i, j, k));
    if (xt) r = cadd(r, to_d(__ldg(xt + c * N + i + (long long)nxp * (j + (long long)g.ny * k))));
    return r;
  }
};
using XRef64 = XRefT<float2>;

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

// sigma-bar / eps-bar per unknown: the area- and volume-weighted cell
// averages of gen_k2_*grid before the factor i omega mu0, boundary values
// from the clamped interior index (src/aphid.f90:1289-1535).
template <typename CT>
static __global__ void k_sw_avg(GridDev g, const CT *__restrict__ cell, double *__restrict__ out) {
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

// Cole-Cole cell conductivity at one frequency (read_mesh model D,
// src/aphid.f90:410-435): sigma-hat = sigma (1 - eta / (1 + (i omega tau)^c))
// from the real(4) cell arrays, in FP64; (i omega tau)^c on the principal
// branch, (omega tau)^c (cos(pi c / 2) + i sin(pi c / 2)).  Real and
// imaginary parts go to re[] and im[].
static __global__ void k_cc_cells(long long ncell, const float *__restrict__ sig, const float *__restrict__ eta,
                                  const float *__restrict__ tau, const float *__restrict__ cee, double omega,
                                  double *__restrict__ re, double *__restrict__ im) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncell;
       t += (long long)gridDim.x * blockDim.x) {
    const double s = sig[t], e = eta[t], ta = tau[t], c = cee[t];
    double sn, cs;
    sincospi(0.5 * c, &sn, &cs);
    const double mag = ta > 0.0 ? pow(omega * ta, c) : 0.0;
    const double2 den = make_double2(1.0 + mag * cs, mag * sn);
    const double2 f = cdiv(make_double2(e, 0.0), den);
    re[t] = s * (1.0 - f.x);
    im[t] = -s * f.y;
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
  double *part = D.part + (size_t)sys * D.slots * kParts;
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
template <typename F>
static __global__ void k_sw_to_node(GridDev g, NodeLayout L, const double *__restrict__ ref, F *__restrict__ node) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const long long nd = i + (long long)L.nxp * (j + (long long)g.ny * k);
#pragma unroll
  for (int c = 0; c < 4; c++)
    node[c * L.N + nd] = exists(g, c, i, j, k) ? (F)ref[ref_of(g, c, i, j, k)] : (F)0;
}


// FP32 axis tables of the complex64 pass, built once per mesh:
// [m] = (n4, n5, dc, 1/dc) of node m and [n + m] = (e2, e3, d, 1/d) of the
// edge (m, m+1) (zeros and ones past the last edge).
static __global__ void k_sw_axis32(GridDev g, float4 *out) {
  const int a = blockIdx.y;
  const Axis A = a == 0 ? g.ax[0] : (a == 1 ? g.ax[1] : g.ax[2]);
  const int n = A.n, m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const int base = a == 0 ? 0 : (a == 1 ? 2 * g.ax[0].n : 2 * (g.ax[0].n + g.ax[1].n));
  out[base + m] = make_float4((float)A.n4[m], (float)A.n5[m], (float)A.dc[m], (float)(1.0 / A.dc[m]));
  const bool e = m < n - 1;
  out[base + n + m] = make_float4(e ? (float)A.e2[m] : 0.f, e ? (float)A.e3[m] : 0.f, e ? (float)A.d[m + 1] : 1.f,
                                  e ? (float)(1.0 / A.d[m + 1]) : 1.f);
}
// the same tables in FP64 (complex128 pass)
static __global__ void k_sw_axis64(GridDev g, double4 *out) {
  const int a = blockIdx.y;
  const Axis A = a == 0 ? g.ax[0] : (a == 1 ? g.ax[1] : g.ax[2]);
  const int n = A.n, m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const int base = a == 0 ? 0 : (a == 1 ? 2 * g.ax[0].n : 2 * (g.ax[0].n + g.ax[1].n));
  out[base + m] = make_double4(A.n4[m], A.n5[m], A.dc[m], 1.0 / A.dc[m]);
  const bool e = m < n - 1;
  out[base + n + m] = make_double4(e ? A.e2[m] : 0.0, e ? A.e3[m] : 0.0, e ? A.d[m + 1] : 1.0, e ? 1.0 / A.d[m + 1] : 1.0);
}


// O2: r = b - K x in complex128 (true residual).  The next inner cycle starts
// from r~_0 = D^-1/2 r (D from jacobi32, as in the pass), stored as
// q^ = D^-1 r with v^ = p^ = d^ = x^ = 0 and
// beta_0 = 0, so that the first pass forms v~_1 = r~_0 / ||r~_0||; scalars of
// src/aphid_qmr.f90:268-285, 299-313 with M = I.
// The Jacobi diagonal of node (i, j, k) exactly as the complex64 pass forms
// it (the same function on the same FP32 values)
__device__ __forceinline__ void node_diag32(const SweepDev &D, const SweepSys *S, int i, int j, int k, float2 dg[4]) {
  const int nx = D.g.nx, ny = D.g.ny, nz = D.g.nz;
  const long long N = D.L.N, plane = (long long)D.L.nxp * ny, nd = nd_of(D, i, j, k);
  const float4 *AX = D.ax32, *AY = D.ax32 + 2 * nx, *AZ = D.ax32 + 2 * (nx + ny);
  const long long mo = (S - D.sys) * D.mnode;
  auto sg = [&](int c, long long q) { return __ldg(D.sig32 + mo + c * N + q); };
  auto ep = [&](int c, long long q) { return D.epsr32 ? __ldg(D.epsr32 + mo + c * N + q) : 1.f; };
  const bool pin = i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1;
  jacobi32(__ldg(AX + i), __ldg(AX + nx + i), __ldg(AY + j), __ldg(AY + ny + j), __ldg(AZ + k), __ldg(AZ + nz + k),
           sg(0, nd), sg(1, nd), sg(2, nd), sg(3, nd), pin ? sg(0, nd - 1) : 0.f, pin ? sg(1, nd - D.L.nxp) : 0.f,
           pin ? sg(2, nd - plane) : 0.f, ep(0, nd), ep(1, nd), ep(2, nd), ep(3, nd), pin ? ep(0, nd - 1) : 1.f,
           pin ? ep(1, nd - D.L.nxp) : 1.f, pin ? ep(2, nd - plane) : 1.f, i < nx - 1, j < ny - 1, k < nz - 1, pin,
           (float)S->ka, (float)S->kb, dg);
}
// ... and the complex128 pass's diagonal from the FP64 tables
__device__ __forceinline__ void node_diag64(const SweepDev &D, const SweepSys *S, int i, int j, int k,
                                            double2 dg[4]) {
  const int nx = D.g.nx, ny = D.g.ny, nz = D.g.nz;
  const long long N = D.L.N, plane = (long long)D.L.nxp * ny, nd = nd_of(D, i, j, k);
  const double4 *AX = D.ax64, *AY = D.ax64 + 2 * nx, *AZ = D.ax64 + 2 * (nx + ny);
  const long long mo = (S - D.sys) * D.mnode;
  auto sg = [&](int c, long long q) { return __ldg(D.sig64 + mo + c * N + q); };
  auto ep = [&](int c, long long q) { return D.epsr64 ? __ldg(D.epsr64 + mo + c * N + q) : 1.0; };
  const bool pin = i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1;
  jacobi64(ldg4(AX + i), ldg4(AX + nx + i), ldg4(AY + j), ldg4(AY + ny + j), ldg4(AZ + k), ldg4(AZ + nz + k),
           sg(0, nd), sg(1, nd), sg(2, nd), sg(3, nd), pin ? sg(0, nd - 1) : 0.0, pin ? sg(1, nd - D.L.nxp) : 0.0,
           pin ? sg(2, nd - plane) : 0.0, ep(0, nd), ep(1, nd), ep(2, nd), ep(3, nd), pin ? ep(0, nd - 1) : 1.0,
           pin ? ep(1, nd - D.L.nxp) : 1.0, pin ? ep(2, nd - plane) : 1.0, i < nx - 1, j < ny - 1, k < nz - 1, pin,
           S->ka, S->kb, dg);
}

// Inner storage of a sweep: complex64 (k_sw_pass) or complex128 (k_sw_pass64)
template <typename T> struct Inner;
template <> struct Inner<float2> {
  using R = float;
  static __device__ __forceinline__ float2 *vec(const SweepDev &D, int set, int sys, int v) {
    return wvec(D, set, sys, v);
  }
  static __device__ __forceinline__ float2 *pv(const SweepDev &D, int slot, int sys) { return pvec(D, slot, sys); }
  static __device__ __forceinline__ float2 *dd(const SweepDev &D) { return D.dd; }
  static __device__ __forceinline__ int ring(const SweepDev &D) { return D.ring; }
  static __device__ __forceinline__ void diag(const SweepDev &D, const SweepSys *S, int i, int j, int k,
                                              float2 dg[4]) {
    node_diag32(D, S, i, j, k, dg);
  }
  static __device__ __forceinline__ float2 from_d(double2 a) { return to_f(a); }
};
template <> struct Inner<double2> {
  using R = double;
  static __device__ __forceinline__ double2 *vec(const SweepDev &D, int set, int sys, int v) {
    return wvec64(D, set, sys, v);
  }
  static __device__ __forceinline__ double2 *pv(const SweepDev &D, int slot, int sys) { return pvec64(D, slot, sys); }
  static __device__ __forceinline__ double2 *dd(const SweepDev &D) { return D.dd64; }
  static __device__ __forceinline__ int ring(const SweepDev &D) { return D.ring64; }
  static __device__ __forceinline__ void diag(const SweepDev &D, const SweepSys *S, int i, int j, int k,
                                              double2 dg[4]) {
    node_diag64(D, S, i, j, k, dg);
  }
  static __device__ __forceinline__ double2 from_d(double2 a) { return a; }
};

// Test hook (aphid_gpu_sweep_apply32): x (reference layout, complex128) as
// the q^ of system 0's read set, with v^ = p^ = 0, so that a timing pass with
// vscale 1, beta 0, k1 0 forms u = x and q^ = D^-1 K u
template <typename T>
static __global__ void k_sw_apply_in(SweepDev D, const double2 *__restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= D.g.nx) return;
  const int cur = D.sys->cur;
  T *Q = Inner<T>::vec(D, cur, 0, 0), *V = Inner<T>::vec(D, cur, 0, 1), *P = Inner<T>::pv(D, D.sys->pslot, 0);
  const long long nd = nd_of(D, i, j, k);
  const T zero = Inner<T>::from_d(make_double2(0.0, 0.0));
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const long long t = c * D.L.N + nd;
    Q[t] = exists(D.g, c, i, j, k) ? Inner<T>::from_d(x[ref_of(D.g, c, i, j, k)]) : zero;
    V[t] = zero;
    P[t] = zero;
  }
}
// ... and y = D q^ of the set that pass wrote (reference layout, complex128)
template <typename T>
static __global__ void k_sw_apply_out(SweepDev D, double2 *__restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= D.g.nx) return;
  const T *Q = Inner<T>::vec(D, D.sys->cur, 0, 0);
  T dg[4];
  Inner<T>::diag(D, D.sys, i, j, k, dg);
  const long long nd = nd_of(D, i, j, k);
#pragma unroll
  for (int c = 0; c < 4; c++)
    if (exists(D.g, c, i, j, k)) y[ref_of(D.g, c, i, j, k)] = cmul(to_d(dg[c]), to_d(Q[c * D.L.N + nd]));
}

// ------------------------------------------------------------ outer step
// The deferred solution update (k_sw_dxupd): for every system with pending
// updates n1 .. nk (eta_j, kappa_j and the ring slot of p^_j, appended by the
// passes), per unknown
//   d^ <- eta_j p^_j + kappa_j d^,  dx += d^   (j = n1 .. nk, in order),
// then x += dx in FP64 (reference layout) and the list is emptied.  d^ stays
// in the inner precision T, the increments of the R passes are summed in
// FP64.  This is the update of src/aphid_qmr.f90:347-354 (d = eta p + kappa
// d, x = x + d), applied R iterations at a time: the graph launches it after
// every R passes, at the start of each round (ending a cycle before its
// residual) and before the true-residual monitor.
// TIMING: the same loads, stores and arithmetic with eta = 0, kappa = 1 over
// R ring slots and x += 0 dx (tmix = 0), leaving d^ and x as they were.
__device__ __forceinline__ float2 dx_link(float2 e, float2 p, float k, float2 d) {  // e p + k d
  return make_float2(fmaf(e.x, p.x, fmaf(-e.y, p.y, k * d.x)), fmaf(e.x, p.y, fmaf(e.y, p.x, k * d.y)));
}
__device__ __forceinline__ double2 dx_link(double2 e, double2 p, double k, double2 d) {
  return make_double2(fma(e.x, p.x, fma(-e.y, p.y, k * d.x)), fma(e.x, p.y, fma(e.y, p.x, k * d.y)));
}
// Every block takes a slice of every system with pending updates (blocks
// stride over the nodes of one system, then go on to the next system), so
// that when only a few systems are still running their updates are spread
// over the whole grid rather than over a fixed per-system share of it.
template <typename T, bool TIMING>
static __global__ void __launch_bounds__(kStreamThreads) k_sw_dxupd(SweepDev D) {
  using R = typename Inner<T>::R;
  const int ring = Inner<T>::ring(D);
  __shared__ int s_np;
  __shared__ T s_eta[kMaxRing];
  __shared__ R s_kap[kMaxRing];
  __shared__ const T *s_p[kMaxRing];
  const double mix = TIMING ? (double)D.tmix : 1.0;
  const GridDev &g = D.g;
  // node indices in 32 bits (the sweep limits a system to 2^31 node-layout
  // values): two 32-bit divisions per node instead of two 64-bit ones
  const unsigned nxp = (unsigned)D.L.nxp, ny = (unsigned)g.ny, nn = (unsigned)D.L.N;
  for (int sys = 0; sys < D.nsys; sys++) {
    SweepSys *S = D.sys + sys;
    __syncthreads();  // the previous system's list is no longer read
    if (threadIdx.x == 0) s_np = TIMING ? ring : S->npend;
    __syncthreads();
    const int np = s_np;
    if (np == 0) continue;
    if (threadIdx.x < np) {
      const int q = threadIdx.x;
      s_eta[q] = TIMING ? Inner<T>::from_d(make_double2(0.0, 0.0)) : Inner<T>::from_d(S->eta_h[q]);
      s_kap[q] = TIMING ? (R)1 : (R)S->kap_h[q];
      s_p[q] = Inner<T>::pv(D, TIMING ? (S->pslot + 1 + q) % (ring + 1) : S->slot_h[q], sys);
    }
    __syncthreads();
    T *dd = Inner<T>::dd(D) + (long long)sys * 4 * D.L.N;
    double2 *x64 = D.x64 + (long long)sys * D.n;
    for (unsigned nd = blockIdx.x * blockDim.x + threadIdx.x; nd < nn; nd += gridDim.x * blockDim.x) {
      const unsigned row = nd / nxp, iu = nd - row * nxp;
      if (iu >= (unsigned)g.nx) continue;
      const unsigned ku = row / ny;
      const int i = (int)iu, j = (int)(row - ku * ny), k = (int)ku;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        if (!exists(g, c, i, j, k)) continue;
        const long long t = c * D.L.N + nd;
        const long long rt = ref_of(g, c, i, j, k);
        // every load of this unknown first (the ring slots, d^, x), then the
        // recurrence: the loads are in flight together instead of one memory
        // latency per pending update
        T pj[kMaxRing];
#pragma unroll
        for (int q = 0; q < kMaxRing; q++)
          if (q < np) pj[q] = __ldg(s_p[q] + t);
        T d = dd[t];
        const double2 x0 = x64[rt];
        double2 dx = make_double2(0.0, 0.0);
#pragma unroll
        for (int q = 0; q < kMaxRing; q++)
          if (q < np) {
            d = dx_link(s_eta[q], pj[q], s_kap[q], d);
            dx = cadd(dx, to_d(d));
          }
        dd[t] = d;
        x64[rt] = make_double2(fma(mix, dx.x, x0.x), fma(mix, dx.y, x0.y));
      }
    }
    // the last block through this system empties its pending list
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      unsigned *cnt = D.cnt + CNT_DX * D.nsys + sys;
      if (atomicAdd(cnt, 1u) == gridDim.x - 1) {
        if (!TIMING) S->npend = 0;
        *cnt = 0;
        __threadfence();
      }
    }
  }
}

template <typename T>
static __global__ void __launch_bounds__(kOpThreads) k_sw_resid(SweepDev D) {
  const int sys = blockIdx.x % D.nsys;
  const long long tile = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (S->phase != PH_OUTER) return;
  int i, j, k0, k1;
  sweep_tile(D, tile, i, j, k0, k1);
  Vals<4> a{{0.0, 0.0, 0.0, 0.0}};
  if (i < D.g.nx && j < D.g.ny) {
    const XRef64 L{D.g, D.x64 + (long long)sys * D.n, nullptr, D.L.nxp, D.L.N};
    const K2Ref64 K{D.g, D.sig + sys * D.mref, D.epsr ? D.epsr + sys * D.mref : nullptr, S->ka, S->kb};
    const double2 *b = D.b + (long long)sys * D.n;
    const long long vb = (long long)sys * 4 * D.L.N;
    T *Q = Inner<T>::vec(D, S->cur, sys, 0), *V = Inner<T>::vec(D, S->cur, sys, 1),
      *P = Inner<T>::pv(D, S->pslot, sys), *dd = Inner<T>::dd(D);
    using R = typename Inner<T>::R;
    const T zero = Inner<T>::from_d(make_double2(0.0, 0.0));
    for (int k = k0; k < k1; k++) {
      double2 o[4];
      rowsN<double>(D.g, i, j, k, L, K, o);
      const long long nd = nd_of(D, i, j, k);
      T dg[4];
      Inner<T>::diag(D, S, i, j, k, dg);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const long long t = c * D.L.N + nd;
        T rq = zero;
        if (exists(D.g, c, i, j, k)) {
          const double2 r = csub(b[ref_of(D.g, c, i, j, k)], o[c]);
          T inv;
          R absd, rabsd;
          jacobi_weights(dg[c], inv, absd, rabsd);
          rq = Inner<T>::from_d(cmul(to_d(inv), r));
          a.v[0] += cabs2(r);
          const double2 q = to_d(rq);
          a.v[1] += (double)absd * cabs2(q);         // ||r~||^2 = sum |D| |q^|^2
          const double2 w = cmul(to_d(dg[c]), cmul(q, q));  // r~^T r~ = sum D q^2
          a.v[2] += w.x;
          a.v[3] += w.y;
        }
        Q[t] = rq;
        V[t] = zero;
        P[t] = zero;
        dd[vb + t] = zero;
      }
    }
  }
  Vals<4> blk = block_reduce<4, kOpThreads>(a);
  double *part = D.part + (size_t)sys * D.slots * kParts;
  unsigned *cnt = D.cnt + CNT_RESID * D.nsys + sys;
  const unsigned nt = (unsigned)D.t.count();
  if (arrive<4, kOpThreads>(blk, part, cnt, (unsigned)tile, nt)) {
    Vals<4> tot = final_reduce<4, kOpThreads>(part, cnt, nt);
    if (threadIdx.x == 0) {
      S->rnorm = sqrt(tot.v[0]);
      S->has_inner = 0;
      S->npend = 0;  // flushed by k_sw_dxupd before this step
      S->slow = (S->outer_it > 0 && S->rnorm > kSlowCycle * S->rprev) ? S->slow + 1 : 0;
      S->rprev = S->rnorm;
      if (!isfinite(S->rnorm)) {
        mark_done(D, S, 3);
      } else if (S->rnorm < S->target * S->bnorm) {
        mark_done(D, S, 0);
      } else if (S->escalated || (S->escalate && S->slow >= kSlowCycles)) {
        mark_done(D, S, kStEscalated);
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
        S->beta = make_double2(0.0, 0.0);
        S->rho_np = rt0;
        S->c_nm = 1.0;
        S->rho_n = rt0;
        S->theta_nm = 0.0;
        S->del = rmul(S->vscale * S->vscale, make_double2(tot.v[2], tot.v[3]));
        S->k1 = cdiv(rmul(S->rho_n, S->del), S->eps);
        S->tau = S->tau0 = rt0;
        S->tau_win = rt0;
        S->win_it = 0;
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

// Monitor: the true residual of the running iterate, ||b - K x|| in
// complex128 (x as k_sw_dxupd left it, every update applied), once per graph
// round once the cycle is near its end (see kMonitorLevel).  Ends the inner
// cycle on convergence or on stagnation of the complex64 recurrence (see
// kStagnation); the next round's outer step restarts from the FP64
// residual.
template <typename T>
static __global__ void __launch_bounds__(kOpThreads) k_sw_check(SweepDev D) {
  const int sys = blockIdx.x % D.nsys;
  const long long tile = blockIdx.x / D.nsys;
  SweepSys *S = D.sys + sys;
  if (S->phase != PH_INNER || S->inner_it < 2) return;
  const double pred = S->rnorm * (S->tau / S->tau0);  // the true residual the quasi-residual predicts
  if (pred > S->mon_level * S->bnorm) return;
  // near the target every round (the check ends the cycle on convergence);
  // further away every kCheckEvery iterations (it ends the cycle when the
  // true residual stops following the quasi-residual)
  if (pred > kCheckNear * S->target * S->bnorm && S->total_it - S->last_check_it < kCheckEvery) return;
  int i, j, k0, k1;
  sweep_tile(D, tile, i, j, k0, k1);
  Vals<1> a{{0.0}};
  if (i < D.g.nx && j < D.g.ny) {
    const XRef64 L{D.g, D.x64 + (long long)sys * D.n, nullptr, D.L.nxp, D.L.N};
    const K2Ref64 K{D.g, D.sig + sys * D.mref, D.epsr ? D.epsr + sys * D.mref : nullptr, S->ka, S->kb};
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
  double *part = D.part + (size_t)sys * D.slots * kParts;
  unsigned *cnt = D.cnt + CNT_CHECK * D.nsys + sys;
  const unsigned nt = (unsigned)D.t.count();
  if (arrive<1, kOpThreads>(blk, part, cnt, (unsigned)tile, nt)) {
    Vals<1> tot = final_reduce<1, kOpThreads>(part, cnt, nt);
    if (threadIdx.x == 0) {
      const double rn = sqrt(tot.v[0]);
      S->mon_rn = rn;
      S->checks++;
      S->last_check_it = S->total_it;
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

// tensor maps of the pass (kernel parameter, __grid_constant__)
struct PassMaps {
  CUtensorMap w;         // 5-D: (nxp, ny, nz, vector x component = 8 (q^ v^), set x system), 8-byte elements
  CUtensorMap p;         // 5-D: (nxp, ny, nz, component, ring slot x system), 8-byte elements
  CUtensorMap sig, eps;  // 4-D: (nxp, ny, nz, component), FP32
  CUtensorMap w64;       // complex128 q^ v^: 5-D (2 nxp, ny, nz, 8, set x system), 8-byte elements
  CUtensorMap p64;       // complex128 p^ ring: 5-D (2 nxp, ny, nz, 4, slot x system), 8-byte elements
};

// Shared memory and occupancy of the pass, in two pipeline configurations
// that the autotuner chooses between per mesh and batch: CFG 0, two load
// stages, with two resident blocks per SM for model R (16 warps, at most 128
// registers per thread); CFG 1, three load stages in one block per SM.
// Models C, I and D stage eps-bar too and fit one block per SM in both.  Each
// stage holds q^ v^ (8 components) and p^ (4) of plane m+1 with halo and
// sigma-bar [eps-bar] of plane m (16 x 16 tiles: 40.5 KB, 47.3 KB with
// eps-bar; 32 x 8: 40.0 KB, 46.3 KB); then two u planes and the mbarriers.
template <bool EPS, int CFG, int TS>
struct PassShm {
  static constexpr unsigned vec_plane = PT<TS>::N * 8u;  // one component of one vector, one staged plane
  static constexpr unsigned raw = 12u * vec_plane;       // q^, v^, p^ with halo, four components each
  static constexpr unsigned sig_bytes = 4u * PT<TS>::KN * 4u;  // sigma-bar with halo, four components
  static constexpr unsigned ubytes = 4u * vec_plane;     // u of one plane
  static constexpr int stages = CFG == 0 ? 2 : 3;
  static constexpr int blocks = (EPS || CFG == 1) ? 1 : 2;  // resident blocks per SM
  static constexpr unsigned sig = raw;
  static constexpr unsigned stage = raw + (EPS ? 2u : 1u) * sig_bytes;
  static constexpr size_t bytes = stages * (size_t)stage + 2 * (size_t)ubytes + 128;
};
constexpr int kWaitTries = 1 << 24;

__device__ __forceinline__ float2 axpy(float a, float2 x, float2 y) {
  return make_float2(fmaf(a, x.x, y.x), fmaf(a, x.y, y.y));
}
__device__ __forceinline__ float2 cfma(float2 a, float2 x, float2 y) {  // y + a x
  return make_float2(fmaf(a.x, x.x, fmaf(-a.y, x.y, y.x)), fmaf(a.x, x.y, fmaf(a.y, x.x, y.y)));
}


// Stencil rows of the complex64 pass in difference form, with the sums as
// trees (see k_sw_pass).  Edge row (Ax, Ay or Az): own value u0, six
// neighbours n_k with real coefficients c_k, the Phi values f1 (ahead along
// the edge) and f0, 1/d of the edge, vol; sigma-bar of the edge (s0), of
// Phi ahead (spn) and at the node (sp0).  Model R: k^2 = (-ka, kb s).
__device__ __forceinline__ float2 edge_row(float2 u0, float2 n1, float c1, float2 n2, float c2, float2 n3, float c3,
                                           float2 n4, float c4, float2 n5, float c5, float2 n6, float c6, float s0,
                                           float spn, float sp0, float2 f1, float2 f0, float rd, float vol, float ka,
                                           float kb) {
  const float2 t1 = axpy(c2, csub(n2, u0), rmul(c1, csub(n1, u0)));
  const float2 t2 = axpy(c4, csub(n4, u0), rmul(c3, csub(n3, u0)));
  const float2 t3 = axpy(c6, csub(n6, u0), rmul(c5, csub(n5, u0)));
  const float2 L = cadd(cadd(t1, t2), axpy(-ka, u0, t3));
  const float2 M = axpy(rd * (spn - sp0), f0, axpy(rd * (spn - s0), csub(f1, f0), rmul(s0, u0)));
  return make_float2(vol * (L.x - kb * M.y), vol * (L.y + kb * M.x));
}
// the same with complex k^2 of the edge (k2), of Phi ahead (kpn) and at the
// node (kp0): models C, I
__device__ __forceinline__ float2 edge_row_c(float2 u0, float2 n1, float c1, float2 n2, float c2, float2 n3, float c3,
                                             float2 n4, float c4, float2 n5, float c5, float2 n6, float c6, float2 k2,
                                             float2 kpn, float2 kp0, float2 f1, float2 f0, float rd, float vol) {
  const float2 t1 = axpy(c2, csub(n2, u0), rmul(c1, csub(n1, u0)));
  const float2 t2 = axpy(c4, csub(n4, u0), rmul(c3, csub(n3, u0)));
  const float2 t3 = axpy(c6, csub(n6, u0), rmul(c5, csub(n5, u0)));
  const float2 g = cfma(make_float2(rd * (kpn.x - kp0.x), rd * (kpn.y - kp0.y)), f0,
                        cfma(make_float2(rd * (kpn.x - k2.x), rd * (kpn.y - k2.y)), csub(f1, f0), cmul(k2, u0)));
  const float2 L = cadd(cadd(t1, t2), cadd(t3, g));
  return make_float2(vol * L.x, vol * L.y);
}
// Node row (Phi): own f, neighbours fx+ fx- fy+ fy- fz+ fz-, axis coefficients
// n4/n5 per axis, the edges of the node (a0, a1, a2) and those behind it
// (a0m, a1m, a2m), 1/dc per axis, sigma-bar of the six edges and of the node:
// k_p^2 Phi + sum c_m (Phi_m - Phi) + sum_a [(k_a - k_p)(A_a - A_a-) +
// (k_a - k_a-) A_a-] / dc_a with c_m = n_m k^2_m.  Model R.
__device__ __forceinline__ float2 node_row(float2 f, float2 fxp, float2 fxm, float2 fyp, float2 fym, float2 fzp,
                                           float2 fzm, float xn4, float xn5, float yn4, float yn5, float zn4,
                                           float zn5, float2 a0, float2 a0m, float2 a1, float2 a1m, float2 a2,
                                           float2 a2m, float rdxc, float rdyc, float rdzc, float sx, float sxm,
                                           float sy, float sym, float sz, float szm, float sp0, float vol, float ka,
                                           float kb) {
  const float2 g1 = csub(fxp, f), g2 = csub(fxm, f), g3 = csub(fyp, f), g4 = csub(fym, f), g5 = csub(fzp, f),
               g6 = csub(fzm, f);
  const float2 T1 = cadd(cadd(axpy(xn5, g2, rmul(xn4, g1)), axpy(yn5, g4, rmul(yn4, g3))),
                         axpy(zn5, g6, rmul(zn4, g5)));
  const float2 T2a = cadd(axpy(xn5 * sxm, g2, rmul(xn4 * sx, g1)), axpy(yn5 * sym, g4, rmul(yn4 * sy, g3)));
  const float2 T2b = axpy(zn5 * szm, g6, rmul(zn4 * sz, g5));
  const float2 Ea = axpy(rdxc * (sx - sxm), a0m, rmul(rdxc * (sx - sp0), csub(a0, a0m)));
  const float2 Eb = axpy(rdyc * (sy - sym), a1m, rmul(rdyc * (sy - sp0), csub(a1, a1m)));
  const float2 Ec = axpy(rdzc * (sz - szm), a2m, rmul(rdzc * (sz - sp0), csub(a2, a2m)));
  const float2 T2 = cadd(cadd(T2a, T2b), cadd(cadd(Ea, Eb), Ec));
  const float2 t = cfma(make_float2(ka * ka - kb * kb * sp0 * sp0, -2.f * ka * kb * sp0), f,
                        make_float2(-ka * T1.x, -ka * T1.y));
  return make_float2(vol * (t.x - kb * T2.y), vol * (t.y + kb * T2.x));
}
// the same with complex k^2 (models C, I)
__device__ __forceinline__ float2 node_row_c(float2 f, float2 fxp, float2 fxm, float2 fyp, float2 fym, float2 fzp,
                                             float2 fzm, float xn4, float xn5, float yn4, float yn5, float zn4,
                                             float zn5, float2 a0, float2 a0m, float2 a1, float2 a1m, float2 a2,
                                             float2 a2m, float rdxc, float rdyc, float rdzc, float2 kx, float2 kxm,
                                             float2 ky, float2 kym, float2 kz, float2 kzm, float2 kp, float vol) {
  const float2 g1 = csub(fxp, f), g2 = csub(fxm, f), g3 = csub(fyp, f), g4 = csub(fym, f), g5 = csub(fzp, f),
               g6 = csub(fzm, f);
  const float2 Ta = cfma(rmul(xn5, kxm), g2, cmul(rmul(xn4, kx), g1));
  const float2 Tb = cfma(rmul(yn5, kym), g4, cmul(rmul(yn4, ky), g3));
  const float2 Tc = cfma(rmul(zn5, kzm), g6, cmul(rmul(zn4, kz), g5));
  const float2 Ea = cfma(rmul(rdxc, csub(kx, kxm)), a0m, cmul(rmul(rdxc, csub(kx, kp)), csub(a0, a0m)));
  const float2 Eb = cfma(rmul(rdyc, csub(ky, kym)), a1m, cmul(rmul(rdyc, csub(ky, kp)), csub(a1, a1m)));
  const float2 Ec = cfma(rmul(rdzc, csub(kz, kzm)), a2m, cmul(rmul(rdzc, csub(kz, kp)), csub(a2, a2m)));
  const float2 t = cadd(cadd(cadd(Ta, Tb), cadd(Tc, cmul(cmul(kp, kp), f))), cadd(cadd(Ea, Eb), Ec));
  return make_float2(vol * t.x, vol * t.y);
}

// Scalar step at the end of pass n (one thread): epsilon_n, beta_n,
// rho_{n+1} and delta_{n+1} from the pipelined inner products, then theta,
// c, eta, kappa, tau and k1 as in src/aphid_qmr.f90:324-372.
__device__ __noinline__ void pass_scalars(SweepSys *S, const double *T, int ring) {
  S->cur ^= 1;
  S->pslot = (S->pslot + 1) % (ring + 1);
  S->inner_it++;
  S->total_it++;
  const double2 e = make_double2(T[0], T[1]);
  S->eps = e;
  if (!finite2(e) || zero2(e)) {  // breakdown: restart from the current x
    S->phase = PH_OUTER;
    return;
  }
  const double2 beta = cdiv(e, S->del);
  const double A1 = T[2], A3 = T[5];
  const double2 A2 = make_double2(T[3], T[4]), B1 = make_double2(T[6], T[7]);
  const double2 B2 = make_double2(T[8], T[9]), B3 = make_double2(T[10], T[11]);
  const double bb = cabs2(beta);
  double rho2 = A1 - 2.0 * (beta.x * A2.x + beta.y * A2.y) + bb * A3;
  if (!isfinite(rho2) || !(bb > 0.0)) {
    S->phase = PH_OUTER;
    return;
  }
  const bool exhausted = !(rho2 > kCancel * A1);  // Krylov space exhausted (or below the expansion's accuracy)
  if (exhausted) rho2 = 0.0;
  const double rho = sqrt(rho2);
  S->beta = beta;
  S->rho_np = rho;
  S->theta_n = rho2 / S->c_nm / bb;
  S->c_n = 1.0 / (1.0 + S->theta_n);
  S->eta = cdiv(rmul(S->c_n, rmul(S->rho_n, cneg(S->eta))), rmul(S->c_nm, beta));
  S->kap = S->theta_nm * S->c_n;
  S->tau = S->tau * sqrt(S->theta_n * S->c_n);
  // the solution update of this iteration, d = eta p^_n + kappa d, x += d, for
  // k_sw_dxupd (the graph flushes the list before it can exceed the ring)
  const bool update = finite2(S->eta) && isfinite(S->kap) && S->npend < kMaxRing;
  if (update) {
    S->eta_h[S->npend] = S->eta;
    S->kap_h[S->npend] = S->kap;
    S->slot_h[S->npend] = S->pslot;
    S->npend++;
  }
  if (exhausted) {
    S->phase = PH_OUTER;
    return;
  }
  const double2 vtv = cadd(csub(B1, rmul(2.0, cmul(beta, B2))), cmul(cmul(beta, beta), B3));
  const double2 del = rmul(1.0 / rho2, vtv);
  // |v~^T v~ - delta| is measured against ||v~||^2 (about 1), not against
  // delta, which may be small in complex-symmetric Lanczos without any loss
  const bool drift = fabs(A3 - 1.0) > kDrift || sqrt(cabs2(csub(B3, S->del))) > kDrift * A3;
  if (drift) S->restarts++;
  bool stall = false;
  if (S->inner_it - S->win_it >= S->stall_window) {
    stall = S->tau > 0.5 * S->tau_win;
    S->tau_win = S->tau;
    S->win_it = S->inner_it;
  }
  if (stall) S->restarts++;
  if (S->escalate && sqrt(cabs2(del)) < kDeltaFloor * A3) S->escalated = 1;
  if (S->escalated || !update || !isfinite(S->tau) || !finite2(del) || zero2(del) || drift || stall ||
      S->tau < S->inner_tol * S->tau0 || S->total_it >= S->max_it) {
    S->phase = PH_OUTER;
    return;
  }
  S->c_nm = S->c_n;
  S->rho_n = rho;
  S->theta_nm = S->theta_n;
  S->del = del;
  S->k1 = cdiv(rmul(rho, del), e);
  S->vscale = 1.0 / rho;
}

// The fused QMR pass (see the file comment).  One persistent block per SM
// takes (tile, system) work items from a counter, tiles with the most live
// nodes first.  A 16 x 16 node tile marches along k.  Thread 0 issues, per
// z-plane, one TMA transaction into a kStages-deep ring: q^, v^, p^ of plane
// m+1 (q^ v^ of the read set and p^ of the last ring slot, all four
// components, 20 x 18 nodes with halo) and sigma-bar (eps-bar) of plane m,
// kStages-1 planes ahead of their use; the kernel makes no synchronous global
// load in its steady state.  Each thread forms u = p^_n of its own node (which also gives v^_n
// and the stored outputs) and halo values into the u plane of the next step;
// the z-neighbours of its own node stay in registers.  The Jacobi diagonal D
// is formed in FP32 from the same coefficients as the rows (it is their
// diagonal term) instead of being read.  TMA fills outside the tensor with
// zeros, and pads and absent components are stored zeros, so zero padding
// reproduces the reference's clamped neighbours (their coefficients are zero
// at the boundary).
// EPS: models C, I and D (eps-bar not 1).  D.timing: the same pass over
// resident data without the phase test and the scalar step; it flips the
// buffer set and advances the ring like an iteration does, so consecutive
// timing launches read what the previous one wrote (d^ and the x64 solution
// are untouched).  A run-time switch rather than a second instance, so that
// timing launches run the very code (and register allocation) of the solve.
// One work item (a tile's z-slab of one system) of the complex64 pass, on
// the mesh and buffers of D with the tensor maps M.  shm: the pass's dynamic
// shared memory; bar, phase: its stage mbarriers and their wait parities.
template <bool EPS, int CFG, int TS>
__device__ __forceinline__ void pass_item(const SweepDev &D, const PassMaps &M, int sys, long long tile,
                                          unsigned char *shm, unsigned long long *bar, unsigned &phase) {
  using SH = PassShm<EPS, CFG, TS>;
  constexpr int kStages = SH::stages;
  constexpr unsigned kStage = SH::stage, kVecPlane = SH::vec_plane, kSigBytes = SH::sig_bytes;
  constexpr int kPTI = PT<TS>::I, kPTJ = PT<TS>::J, kPW = PT<TS>::W, kPN = PT<TS>::N, kKW = PT<TS>::KW,
                kKN = PT<TS>::KN;
  float2 *Ub = reinterpret_cast<float2 *>(shm + kStages * kStage);  // [2][4][kPN]
  SweepSys *S = D.sys + sys;
  if (!D.timing && S->phase != PH_INNER) return;

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
  const bool live = i < nx && j < ny;
  const long long N = D.L.N, plane = (long long)D.L.nxp * ny;
  const long long ndc = i + (long long)D.L.nxp * j;  // this node within a plane
  const int cur = S->cur, pslot = S->pslot;
  float2 *__restrict__ Qw = wvec(D, cur ^ 1, sys, 0);
  float2 *__restrict__ Vw = wvec(D, cur ^ 1, sys, 1);
  float2 *__restrict__ Pw = pvec(D, (pslot + 1) % (D.ring + 1), sys);
  const float *__restrict__ sig = D.sig32 + sys * D.mnode;
  const float *__restrict__ eps = D.epsr32 ? D.epsr32 + sys * D.mnode : nullptr;
  const int msig = D.mnode ? 4 * sys : 0;  // TMA component coordinate of this system's sigma-bar
  // u = ca q^ + cb v^ + cc p^ and v = ca q^ + cb v^
  const float ca = (float)S->vscale;
  const float2 cb = to_f(rmul(-S->vscale, S->beta));
  const float2 cc = to_f(cneg(S->k1));
  const float ka = (float)S->ka, kb = (float)S->kb;
  const int wset = cur * D.nsys + sys;    // TMA coordinate of the read (q^, v^) set
  const int pset = pslot * D.nsys + sys;  // ... and of the p^ read

  // thread 0: the loads of step m into stage st
  auto issue = [&](int st, int m) {
    const unsigned bb = smem_u32(&bar[st]);
    unsigned char *base = shm + st * kStage;
    fence_async_smem();
    mbar_expect(bb, kStage);
    tma_load5(smem_u32(base), &M.w, i0 - 2, j0 - 1, m + 1, 0, wset, bb);
    tma_load5(smem_u32(base + 8u * kVecPlane), &M.p, i0 - 2, j0 - 1, m + 1, 0, pset, bb);
    tma_load4(smem_u32(base + SH::sig), &M.sig, i0 - 4, j0 - 1, m, msig, bb);
    if (EPS) tma_load4(smem_u32(base + SH::sig + kSigBytes), &M.eps, i0 - 4, j0 - 1, m, msig, bb);
  };
  auto wait = [&](int st) {
    if (!mbar_wait(smem_u32(&bar[st]), (phase >> st) & 1u, kWaitTries) && threadIdx.x == 0) atomicExch(D.err, 1);
    phase ^= 1u << st;
  };
  auto combine = [&](float2 q, float2 v, float2 p, float2 &vo) {
    vo = cfma(cb, v, make_float2(ca * q.x, ca * q.y));
    return cfma(cc, p, vo);
  };

  const int eo = (ty + 1) * kPW + (tx + 2);  // this node in a staged plane
  const int ck = (ty + 1) * kKW + (tx + 4);  // this node in a sigma-bar plane
  // halo values of a plane: 4 components x (2 columns of kPTJ + 2 rows of
  // kPTI) positions, dealt to the threads in order
  constexpr int kHaloPos = 2 * (kPTI + kPTJ), kHalo = 4 * kHaloPos;
  auto halo_at = [](int h) {  // staged-plane index of halo position h
    return h < 2 * kPTJ ? (h % kPTJ + 1) * kPW + (h < kPTJ ? 1 : kPTI + 2)
                        : (h < 2 * kPTJ + kPTI ? 0 : (kPTJ + 1) * kPW) + (h - 2 * kPTJ) % kPTI + 2;
  };

  float2 um[4], uc[4], up[4], vc[4], vn[4];
  // own node of plane m1 from stage st: u (into the u plane and registers),
  // v^_n; v^_n and p^_n stored when the node is this item's
  auto own_step = [&](int st, int m1, float2 *Us, float2 (&uo)[4], float2 (&vo)[4]) {
    const float2 *R = reinterpret_cast<const float2 *>(shm + st * kStage);
    const bool owned = live && m1 < k1;
    const long long nd = ndc + m1 * plane;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      uo[c] = combine(R[c * kPN + eo], R[(4 + c) * kPN + eo], R[(8 + c) * kPN + eo], vo[c]);
      Us[c * kPN + eo] = uo[c];
      if (owned) {
        const long long t = c * N + nd;
        Vw[t] = vo[c];
        Pw[t] = uo[c];
      }
    }
  };
  auto halo = [&](int st, float2 *Us) {
    const float2 *R = reinterpret_cast<const float2 *>(shm + st * kStage);
    float2 vt;
#pragma unroll
    for (int h = threadIdx.x; h < kHalo; h += kPThreads) {
      const int hc = h / kHaloPos, he = halo_at(h % kHaloPos);
      Us[hc * kPN + he] = combine(R[hc * kPN + he], R[(4 + hc) * kPN + he], R[(8 + hc) * kPN + he], vt);
    }
  };

  // axis coefficients of the tile's columns and rows, staged in shared
  // memory and read where used (not held in registers through the plane
  // loop: the two-blocks-per-SM configuration has 128 registers per thread)
  const int ic = min(i, nx - 1), jc = min(j, ny - 1);
  const float4 *AX = D.ax32, *AY = D.ax32 + 2 * nx, *AZ = D.ax32 + 2 * (nx + ny);
  __shared__ float4 s_axis[2 * PT<1>::I + 2 * PT<0>::J];  // XA XB per column, YA YB per row
  if (ty == 0) {
    s_axis[tx] = __ldg(AX + ic);
    s_axis[kPTI + tx] = __ldg(AX + nx + ic);
  }
  if (tx == 0) {
    s_axis[2 * kPTI + ty] = __ldg(AY + jc);
    s_axis[2 * kPTI + kPTJ + ty] = __ldg(AY + ny + jc);
  }
  const bool hx = live && i < nx - 1, hy = live && j < ny - 1;
  const bool pxy = live && i > 0 && i < nx - 1 && j > 0 && j < ny - 1;

  // ---- prologue: step k0-1 (stage 0); the next kStages-1 steps in flight
  if (threadIdx.x == 0) {
    issue(0, k0 - 1);
    issue(1, k0);
#pragma unroll
    for (int q = 2; q < kStages; q++)
      if (k0 + q - 1 <= k1 - 1) issue(q, k0 + q - 1);
  }
#pragma unroll
  for (int c = 0; c < 4; c++) um[c] = make_float2(0.f, 0.f);
  if (live && k0 > 0) {  // u of plane k0-1, own node: the first plane's z-neighbour
    const float2 *Qr = wvec(D, cur, sys, 0), *Vr = wvec(D, cur, sys, 1), *Pr = pvec(D, pslot, sys);
    const long long nd = ndc + (k0 - 1) * plane;
    float2 vt;
#pragma unroll
    for (int c = 0; c < 4; c++) um[c] = combine(__ldg(Qr + c * N + nd), __ldg(Vr + c * N + nd), __ldg(Pr + c * N + nd), vt);
  }
  wait(0);
  own_step(0, k0, Ub, uc, vc);
  halo(0, Ub);
  float s2m = reinterpret_cast<const float *>(shm + SH::sig)[2 * kKN + ck];  // sigma-bar of Az at k0-1
  float e2m = EPS ? reinterpret_cast<const float *>(shm + SH::sig + kSigBytes)[2 * kKN + ck] : 1.f;
  __syncthreads();
  if (threadIdx.x == 0 && k0 + kStages - 1 <= k1 - 1) issue(0, k0 + kStages - 1);

  double acc[kParts];
#pragma unroll
  for (int q = 0; q < kParts; q++) acc[q] = 0.0;

  for (int m = k0; m < k1; m++) {
    const int st = (m - k0 + 1) % kStages;
    const float2 *Uc = Ub + ((m - k0) & 1) * 4 * kPN;
    float2 *Un = Ub + ((m - k0 + 1) & 1) * 4 * kPN;
    const long long nd = ndc + m * plane;
    float s3p = 0.f, e3p = 1.f;
    if (live && m + 1 < nz) {
      s3p = __ldg(sig + 3 * N + nd + plane);
      if (EPS) e3p = __ldg(eps + 3 * N + nd + plane);
    }
    const float4 ZA = __ldg(AZ + m), ZB = __ldg(AZ + nz + m);
    wait(st);
    own_step(st, m + 1, Un, up, vn);

    const float *rk = reinterpret_cast<const float *>(shm + st * kStage + SH::sig);
    const float *re = reinterpret_cast<const float *>(shm + st * kStage + SH::sig + kSigBytes);
    const float sx = rk[ck], sy = rk[kKN + ck], sz = rk[2 * kKN + ck], sp0 = rk[3 * kKN + ck];
    const float ex = EPS ? re[ck] : 1.f, ey = EPS ? re[kKN + ck] : 1.f;
    const float ez = EPS ? re[2 * kKN + ck] : 1.f, ep0 = EPS ? re[3 * kKN + ck] : 1.f;
    const float4 XA = s_axis[tx], XB = s_axis[kPTI + tx], YA = s_axis[2 * kPTI + ty], YB = s_axis[2 * kPTI + kPTJ + ty];
    if (live) {
      const float xn4 = XA.x, xn5 = XA.y, dxc = XA.z, rdxc = XA.w, ce2x = XB.x, ce3x = XB.y, dxi = XB.z,
                  rdxi = XB.w;
      const float yn4 = YA.x, yn5 = YA.y, dyc = YA.z, rdyc = YA.w, ce2y = YB.x, ce3y = YB.y, dyj = YB.z,
                  rdyj = YB.w;
      const float zn4 = ZA.x, zn5 = ZA.y, dzc = ZA.z, rdzc = ZA.w, ce2z = ZB.x, ce3z = ZB.y, dzk = ZB.z,
                  rdzk = ZB.w;
      const float2 *U0 = Uc, *U1 = Uc + kPN, *U2 = Uc + 2 * kPN, *U3 = Uc + 3 * kPN;
      // Rows in difference form: k^2 u0 + sum c (u_nb - u0) for
      // (-sum c + k^2) u0 + sum c u_nb, and (kp' - k^2)(Phi' - Phi) +
      // (kp' - kp) Phi for Phi' (kp' - k^2) - Phi (kp - k^2): equal in exact
      // arithmetic, and in FP32 free of the cancellation between the diagonal
      // and the neighbours that a smooth field causes.  All four rows are
      // formed without branches (boundary rows are zeroed after) and summed
      // as trees, so that the rows interleave.
      const float spx = rk[3 * kKN + ck + 1], spy = rk[3 * kKN + ck + kKW];
      const float sxm = rk[ck - 1], sym = rk[kKN + ck - kKW];
      const float2 f0 = uc[3];
      float2 w0, w1, w2, w3;
      if (!EPS) {
        w0 = edge_row(uc[0], U0[eo + 1], ce2x, U0[eo - 1], ce3x, U0[eo + kPW], yn4, U0[eo - kPW], yn5, up[0], zn4,
                      um[0], zn5, sx, spx, sp0, U3[eo + 1], f0, rdxi, dxi * dyc * dzc, ka, kb);
        w1 = edge_row(uc[1], U1[eo + kPW], ce2y, U1[eo - kPW], ce3y, U1[eo + 1], xn4, U1[eo - 1], xn5, up[1], zn4,
                      um[1], zn5, sy, spy, sp0, U3[eo + kPW], f0, rdyj, dxc * dyj * dzc, ka, kb);
        w2 = edge_row(uc[2], up[2], ce2z, um[2], ce3z, U2[eo + 1], xn4, U2[eo - 1], xn5, U2[eo + kPW], yn4,
                      U2[eo - kPW], yn5, sz, s3p, sp0, up[3], f0, rdzk, dxc * dyc * dzk, ka, kb);
        w3 = node_row(f0, U3[eo + 1], U3[eo - 1], U3[eo + kPW], U3[eo - kPW], up[3], um[3], xn4, xn5, yn4, yn5, zn4,
                      zn5, uc[0], U0[eo - 1], uc[1], U1[eo - kPW], uc[2], um[2], rdxc, rdyc, rdzc, sx, sxm, sy, sym,
                      sz, s2m, sp0, dxc * dyc * dzc, ka, kb);
      } else {
        auto K2 = [&](float s_, float e_) { return make_float2(-ka * e_, kb * s_); };
        const float2 kp0 = K2(sp0, ep0);
        const float2 kx = K2(sx, ex), ky = K2(sy, ey), kz = K2(sz, ez);
        w0 = edge_row_c(uc[0], U0[eo + 1], ce2x, U0[eo - 1], ce3x, U0[eo + kPW], yn4, U0[eo - kPW], yn5, up[0], zn4,
                        um[0], zn5, kx, K2(spx, re[3 * kKN + ck + 1]), kp0, U3[eo + 1], f0, rdxi, dxi * dyc * dzc);
        w1 = edge_row_c(uc[1], U1[eo + kPW], ce2y, U1[eo - kPW], ce3y, U1[eo + 1], xn4, U1[eo - 1], xn5, up[1], zn4,
                        um[1], zn5, ky, K2(spy, re[3 * kKN + ck + kKW]), kp0, U3[eo + kPW], f0, rdyj,
                        dxc * dyj * dzc);
        w2 = edge_row_c(uc[2], up[2], ce2z, um[2], ce3z, U2[eo + 1], xn4, U2[eo - 1], xn5, U2[eo + kPW], yn4,
                        U2[eo - kPW], yn5, kz, K2(s3p, e3p), kp0, up[3], f0, rdzk, dxc * dyc * dzk);
        w3 = node_row_c(f0, U3[eo + 1], U3[eo - 1], U3[eo + kPW], U3[eo - kPW], up[3], um[3], xn4, xn5, yn4, yn5, zn4,
                        zn5, uc[0], U0[eo - 1], uc[1], U1[eo - kPW], uc[2], um[2], rdxc, rdyc, rdzc, kx,
                        K2(sxm, re[ck - 1]), ky, K2(sym, re[kKN + ck - kKW]), kz, K2(s2m, e2m), kp0,
                        dxc * dyc * dzc);
      }
      const float2 zero2 = make_float2(0.f, 0.f);
      float2 w[4] = {hx ? w0 : zero2, hy ? w1 : zero2, m < nz - 1 ? w2 : zero2,
                     (pxy && m > 0 && m < nz - 1) ? w3 : zero2};
      // the Jacobi diagonal of this node (the same function the residual
      // pass uses, on the same values)
      float2 dg[4];
      jacobi32(XA, XB, YA, YB, ZA, ZB, sx, sy, sz, sp0, rk[ck - 1], rk[kKN + ck - kKW], s2m, ex, ey, ez, ep0,
               EPS ? re[ck - 1] : 1.f, EPS ? re[kKN + ck - kKW] : 1.f, e2m, hx, hy, m < nz - 1,
               pxy && m > 0 && m < nz - 1, ka, kb, dg);
      // q^ = D^-1 w; this node's shares of epsilon and of the six products
      float r[kParts];
#pragma unroll
      for (int q = 0; q < kParts; q++) r[q] = 0.f;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const float2 z = dg[c];
        float2 d;
        float rs, mag;  // |D|, |D^-1|
        jacobi_weights(z, d, rs, mag);
        const float2 ww = w[c], u = uc[c], v = vc[c];
        const float2 qh = cmul(d, ww);
        Qw[c * N + nd] = qh;
        r[0] += u.x * ww.x - u.y * ww.y;                // epsilon = u^T K u
        r[1] += u.x * ww.y + u.y * ww.x;
        r[2] += mag * (ww.x * ww.x + ww.y * ww.y);      // ||q~||^2
        r[3] += rs * (v.x * qh.x + v.y * qh.y);         // v~^H q~
        r[4] += rs * (v.x * qh.y - v.y * qh.x);
        r[5] += rs * (v.x * v.x + v.y * v.y);           // ||v~||^2
        r[6] += ww.x * qh.x - ww.y * qh.y;              // q~^T q~
        r[7] += ww.x * qh.y + ww.y * qh.x;
        r[8] += ww.x * v.x - ww.y * v.y;                // v~^T q~
        r[9] += ww.x * v.y + ww.y * v.x;
        const float v2r = v.x * v.x - v.y * v.y, v2i = 2.f * v.x * v.y;
        r[10] += v2r * z.x - v2i * z.y;                 // v~^T v~ = sum D v^2
        r[11] += v2r * z.y + v2i * z.x;
      }
#pragma unroll
      for (int q = 0; q < kParts; q++) acc[q] += (double)r[q];
    }
    if (m + 1 < k1) halo(st, Un);
    __syncthreads();  // everyone is done with stage st and with u plane m
    if (threadIdx.x == 0 && m + kStages <= k1 - 1) issue(st, m + kStages);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      um[c] = uc[c];
      uc[c] = up[c];
      vc[c] = vn[c];
    }
    s2m = sz;
    e2m = ez;
  }

  Vals<kParts> blk;
#pragma unroll
  for (int q = 0; q < kParts; q++) blk.v[q] = acc[q];
  blk = block_reduce<kParts, kPThreads>(blk);
  double *part = D.part + (size_t)sys * D.slots * kParts;
  unsigned *cnt = D.cnt + CNT_PASS * D.nsys + sys;
  const unsigned nt = (unsigned)D.tp.count();
  if (arrive<kParts, kPThreads>(blk, part, cnt, (unsigned)tile, nt)) {
    Vals<kParts> tot = final_reduce<kParts, kPThreads>(part, cnt, nt);
    if (threadIdx.x == 0) {
      if (D.timing) {
        S->cur ^= 1;
        S->pslot = (S->pslot + 1) % (D.ring + 1);
      } else {
        pass_scalars(S, tot.v, D.ring);
      }
    }
  }
}

// The systems a fused pass serves.  A persistent pass takes (tile, system)
// work items from a counter; items of systems that have left their inner
// cycle cost a counter round trip, two barriers and a phase read each, which
// on a batch whose last few systems run on alone is a large part of every
// pass.  So before each pass k_sw_active lists the systems still in their
// inner cycle, and the pass numbers its items over those only.  Timing
// launches (and the several-mesh group pass) serve every system.
static __global__ void __launch_bounds__(1024) k_sw_active(SweepDev D) {
  __shared__ int s_warp[32], s_base;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int s0 = 0; s0 < D.nsys; s0 += blockDim.x) {
    const int s = s0 + threadIdx.x;
    const bool on = s < D.nsys && D.sys[s].phase == PH_INNER;
    const unsigned b = __ballot_sync(0xffffffffu, on);
    if (lane == 0) s_warp[w] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {  // exclusive scan over the warps, ascending systems
      int acc = s_base;
      for (int q = 0; q < nw; q++) {
        const int c = s_warp[q];
        s_warp[q] = acc;
        acc += c;
      }
      s_base = acc;
    }
    __syncthreads();
    if (on) D.active[1 + s_warp[w] + __popc(b & ((1u << lane) - 1u))] = s;
    __syncthreads();
  }
  if (threadIdx.x == 0) D.active[0] = s_base;
}
struct ActiveSet {
  const int *list;  // null: every system, in order
  long long n;      // systems served
  // system of work item `item` (items are tile-major, systems fastest)
  __device__ __forceinline__ int sys(long long item, long long total) const {
    return list ? (item < total ? list[item % n] : 0) : (int)(item % n);
  }
};
__device__ __forceinline__ ActiveSet active_set(const SweepDev &D) {
  ActiveSet A;
  if (D.active && !D.timing) {
    A.list = D.active + 1;
    A.n = *(volatile const int *)D.active;
  } else {
    A.list = nullptr;
    A.n = D.nsys;
  }
  return A;
}

// set-up of a pass block: the stage mbarriers; false when the dynamic shared
// memory is not 128-byte aligned (TMA destinations must be; the block then
// takes no work and the launch reports the error)
template <int kStages>
__device__ __forceinline__ bool pass_block_init(unsigned char *shm, unsigned long long *bar, int *err) {
  const bool aligned = (smem_u32(shm) & 127u) == 0;
  if (!aligned && threadIdx.x == 0) atomicExch(err, 2);
  if (threadIdx.x == 0 && aligned) {
#pragma unroll
    for (int q = 0; q < kStages; q++) mbar_init(smem_u32(&bar[q]));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    fence_async_smem();
  }
  return aligned;
}
// the last block out of a persistent launch re-arms its work counter
__device__ __forceinline__ void pass_block_done(int *work) {
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(work + 1, 1) == gridDim.x - 1) {
      work[0] = 0;
      work[1] = 0;
      __threadfence();
    }
  }
}

template <bool EPS, int CFG, int TS>
__global__ void __launch_bounds__(kPThreads, PassShm<EPS, CFG, TS>::blocks) k_sw_pass(SweepDev D,
                                                                                     const __grid_constant__ PassMaps M) {
  using SH = PassShm<EPS, CFG, TS>;
  extern __shared__ __align__(128) unsigned char shm[];
  __shared__ int s_item;
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(shm + SH::stages * SH::stage + 2 * SH::ubytes);
  // the host launches the instance of D.tp.ts (launch_pass); no device check:
  // a test here pushed the two-blocks-per-SM instance into spilling registers
  __shared__ int s_sys;
  const bool aligned = pass_block_init<SH::stages>(shm, bar, D.err);
  unsigned phase = 0;  // bit q: parity of the next wait on stage q
  const ActiveSet A = active_set(D);
  const long long total = aligned ? D.tp.count() * A.n : 0;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      s_item = atomicAdd(D.work, 1);
      s_sys = A.sys(s_item, total);
    }
    __syncthreads();
    const long long item = s_item;
    if (item >= total) break;
    pass_item<EPS, CFG, TS>(D, M, s_sys, __ldg(D.order + item / A.n), shm, bar, phase);
  }
  pass_block_done(D.work);
}

// Several meshes in one persistent launch (aphid_gpu_sweep_group): the
// complex64 passes of up to kMaxGroup sweeps, each with its own mesh, model,
// buffers and tile order, take work items from one counter.  Items are
// numbered mesh after mesh (first[m] .. first[m+1]-1), the larger meshes
// first, so that the smaller ones fill the tail of the launch.
constexpr int kMaxGroup = 8;
struct PassGroup {
  int n;
  int *work;  // [2]: next item, blocks finished
  long long first[kMaxGroup + 1];
  SweepDev D[kMaxGroup];
  PassMaps M[kMaxGroup];
};

template <bool EPS, int CFG, int TS>
__global__ void __launch_bounds__(kPThreads, PassShm<EPS, CFG, TS>::blocks) k_sw_pass_group(const __grid_constant__ PassGroup G) {
  using SH = PassShm<EPS, CFG, TS>;
  extern __shared__ __align__(128) unsigned char shm[];
  __shared__ int s_item;
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(shm + SH::stages * SH::stage + 2 * SH::ubytes);
  const bool aligned = pass_block_init<SH::stages>(shm, bar, G.D[0].err);  // all meshes in tile shape TS (run_group)
  unsigned phase = 0;
  const long long total = aligned ? G.first[G.n] : 0;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(G.work, 1);
    __syncthreads();
    const long long item = s_item;
    if (item >= total) break;
    int m = 0;
    while (m + 1 < G.n && item >= G.first[m + 1]) m++;
    const long long it = item - G.first[m];
    pass_item<EPS, CFG, TS>(G.D[m], G.M[m], (int)(it % G.D[m].nsys), __ldg(G.D[m].order + it / G.D[m].nsys), shm,
                            bar, phase);
  }
  pass_block_done(G.work);
}


// ------------------------------------------------------------ complex128 pass
// k_sw_pass64: the fused QMR iteration of k_sw_pass with complex128 vectors,
// FP64 coefficients (sigma-bar, eps-bar, axis tables) and FP64 arithmetic, for
// systems on which complex64 storage cannot carry the Lanczos process (see
// kDeltaFloor).  Same tiles, same work order, same inner products, the same
// p^ ring and deferred solution update (k_sw_dxupd<double2>) and scalar step
// (pass_scalars); 2 TMA stages of q^ v^ p^ planes (69 KB each); sigma-bar is
// read with plain loads, prefetched into L1 a plane ahead.
constexpr int kStages64 = 2;
template <int TS>
struct Pass64Shm {
  static constexpr unsigned raw = 12u * PT<TS>::N * 16u;  // q^, v^, p^ with halo, four components, complex128
  static constexpr unsigned ubytes = 4u * PT<TS>::N * 16u;
  static constexpr size_t bytes = kStages64 * (size_t)raw + 2 * (size_t)ubytes + 128;
};

// pull a line towards this SM's L1 ahead of its use (no register, no wait)
__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

__device__ __forceinline__ double2 daxpy(double a, double2 x, double2 y) {
  return make_double2(fma(a, x.x, y.x), fma(a, x.y, y.y));
}
__device__ __forceinline__ double2 dcfma(double2 a, double2 x, double2 y) {  // y + a x
  return make_double2(fma(a.x, x.x, fma(-a.y, x.y, y.x)), fma(a.x, x.y, fma(a.y, x.x, y.y)));
}
// the rows of edge_row / edge_row_c / node_row / node_row_c in FP64
__device__ __forceinline__ double2 edge_row64(double2 u0, double2 n1, double c1, double2 n2, double c2, double2 n3,
                                              double c3, double2 n4, double c4, double2 n5, double c5, double2 n6,
                                              double c6, double s0, double spn, double sp0, double2 f1, double2 f0,
                                              double rd, double vol, double ka, double kb) {
  const double2 t1 = daxpy(c2, csub(n2, u0), rmul(c1, csub(n1, u0)));
  const double2 t2 = daxpy(c4, csub(n4, u0), rmul(c3, csub(n3, u0)));
  const double2 t3 = daxpy(c6, csub(n6, u0), rmul(c5, csub(n5, u0)));
  const double2 L = cadd(cadd(t1, t2), daxpy(-ka, u0, t3));
  const double2 M = daxpy(rd * (spn - sp0), f0, daxpy(rd * (spn - s0), csub(f1, f0), rmul(s0, u0)));
  return make_double2(vol * (L.x - kb * M.y), vol * (L.y + kb * M.x));
}
__device__ __forceinline__ double2 edge_row64_c(double2 u0, double2 n1, double c1, double2 n2, double c2,
                                                double2 n3, double c3, double2 n4, double c4, double2 n5, double c5,
                                                double2 n6, double c6, double2 k2, double2 kpn, double2 kp0,
                                                double2 f1, double2 f0, double rd, double vol) {
  const double2 t1 = daxpy(c2, csub(n2, u0), rmul(c1, csub(n1, u0)));
  const double2 t2 = daxpy(c4, csub(n4, u0), rmul(c3, csub(n3, u0)));
  const double2 t3 = daxpy(c6, csub(n6, u0), rmul(c5, csub(n5, u0)));
  const double2 g = dcfma(rmul(rd, csub(kpn, kp0)), f0, dcfma(rmul(rd, csub(kpn, k2)), csub(f1, f0), cmul(k2, u0)));
  const double2 L = cadd(cadd(t1, t2), cadd(t3, g));
  return rmul(vol, L);
}
__device__ __forceinline__ double2 node_row64(double2 f, double2 fxp, double2 fxm, double2 fyp, double2 fym,
                                              double2 fzp, double2 fzm, double xn4, double xn5, double yn4,
                                              double yn5, double zn4, double zn5, double2 a0, double2 a0m,
                                              double2 a1, double2 a1m, double2 a2, double2 a2m, double rdxc,
                                              double rdyc, double rdzc, double sx, double sxm, double sy, double sym,
                                              double sz, double szm, double sp0, double vol, double ka, double kb) {
  const double2 g1 = csub(fxp, f), g2 = csub(fxm, f), g3 = csub(fyp, f), g4 = csub(fym, f), g5 = csub(fzp, f),
                g6 = csub(fzm, f);
  const double2 T1 = cadd(cadd(daxpy(xn5, g2, rmul(xn4, g1)), daxpy(yn5, g4, rmul(yn4, g3))),
                          daxpy(zn5, g6, rmul(zn4, g5)));
  const double2 T2a = cadd(daxpy(xn5 * sxm, g2, rmul(xn4 * sx, g1)), daxpy(yn5 * sym, g4, rmul(yn4 * sy, g3)));
  const double2 T2b = daxpy(zn5 * szm, g6, rmul(zn4 * sz, g5));
  const double2 Ea = daxpy(rdxc * (sx - sxm), a0m, rmul(rdxc * (sx - sp0), csub(a0, a0m)));
  const double2 Eb = daxpy(rdyc * (sy - sym), a1m, rmul(rdyc * (sy - sp0), csub(a1, a1m)));
  const double2 Ec = daxpy(rdzc * (sz - szm), a2m, rmul(rdzc * (sz - sp0), csub(a2, a2m)));
  const double2 T2 = cadd(cadd(T2a, T2b), cadd(cadd(Ea, Eb), Ec));
  const double2 t = dcfma(make_double2(ka * ka - kb * kb * sp0 * sp0, -2.0 * ka * kb * sp0), f,
                          make_double2(-ka * T1.x, -ka * T1.y));
  return make_double2(vol * (t.x - kb * T2.y), vol * (t.y + kb * T2.x));
}
__device__ __forceinline__ double2 node_row64_c(double2 f, double2 fxp, double2 fxm, double2 fyp, double2 fym,
                                                double2 fzp, double2 fzm, double xn4, double xn5, double yn4,
                                                double yn5, double zn4, double zn5, double2 a0, double2 a0m,
                                                double2 a1, double2 a1m, double2 a2, double2 a2m, double rdxc,
                                                double rdyc, double rdzc, double2 kx, double2 kxm, double2 ky,
                                                double2 kym, double2 kz, double2 kzm, double2 kp, double vol) {
  const double2 g1 = csub(fxp, f), g2 = csub(fxm, f), g3 = csub(fyp, f), g4 = csub(fym, f), g5 = csub(fzp, f),
                g6 = csub(fzm, f);
  const double2 Ta = dcfma(rmul(xn5, kxm), g2, cmul(rmul(xn4, kx), g1));
  const double2 Tb = dcfma(rmul(yn5, kym), g4, cmul(rmul(yn4, ky), g3));
  const double2 Tc = dcfma(rmul(zn5, kzm), g6, cmul(rmul(zn4, kz), g5));
  const double2 Ea = dcfma(rmul(rdxc, csub(kx, kxm)), a0m, cmul(rmul(rdxc, csub(kx, kp)), csub(a0, a0m)));
  const double2 Eb = dcfma(rmul(rdyc, csub(ky, kym)), a1m, cmul(rmul(rdyc, csub(ky, kp)), csub(a1, a1m)));
  const double2 Ec = dcfma(rmul(rdzc, csub(kz, kzm)), a2m, cmul(rmul(rdzc, csub(kz, kp)), csub(a2, a2m)));
  const double2 t = cadd(cadd(cadd(Ta, Tb), cadd(Tc, cmul(cmul(kp, kp), f))), cadd(cadd(Ea, Eb), Ec));
  return rmul(vol, t);
}

template <bool EPS, int TS>
__global__ void __launch_bounds__(kPThreads, 1) k_sw_pass64(SweepDev D, const __grid_constant__ PassMaps M) {
  constexpr unsigned kStage = Pass64Shm<TS>::raw;
  constexpr int kPTI = PT<TS>::I, kPTJ = PT<TS>::J, kPW = PT<TS>::W, kPN = PT<TS>::N;
  extern __shared__ __align__(128) unsigned char shm[];
  __shared__ int s_item;
  double2 *Ub = reinterpret_cast<double2 *>(shm + kStages64 * kStage);  // [2][4][kPN]
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(shm + kStages64 * kStage + 2 * Pass64Shm<TS>::ubytes);
  const bool aligned = (smem_u32(shm) & 127u) == 0;  // tile shape TS: launch_pass64
  if (!aligned && threadIdx.x == 0) atomicExch(D.err, 2);
  if (threadIdx.x == 0 && aligned) {
#pragma unroll
    for (int q = 0; q < kStages64; q++) mbar_init(smem_u32(&bar[q]));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    fence_async_smem();
  }
  unsigned phase = 0;  // bit q: parity of the next wait on stage q
  __shared__ int s_sys;
  const ActiveSet A = active_set(D);
  const long long total = aligned ? D.tp.count() * A.n : 0;

  for (;;) {
  __syncthreads();
  if (threadIdx.x == 0) {
    s_item = atomicAdd(D.work, 1);
    s_sys = A.sys(s_item, total);
  }
  __syncthreads();
  const long long item = s_item;
  if (item >= total) break;
  const int sys = s_sys;
  const long long tile = __ldg(D.order + item / A.n);
  SweepSys *S = D.sys + sys;
  if (!D.timing && S->phase != PH_INNER) continue;

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
  const bool live = i < nx && j < ny;
  const long long N = D.L.N, plane = (long long)D.L.nxp * ny;
  const long long ndc = i + (long long)D.L.nxp * j;
  const int cur = S->cur, pslot = S->pslot;
  double2 *__restrict__ Qw = wvec64(D, cur ^ 1, sys, 0);
  double2 *__restrict__ Vw = wvec64(D, cur ^ 1, sys, 1);
  double2 *__restrict__ Pw = pvec64(D, (pslot + 1) % (D.ring64 + 1), sys);
  const double *__restrict__ sig = D.sig64 + sys * D.mnode;
  const double *__restrict__ eps = D.epsr64 ? D.epsr64 + sys * D.mnode : nullptr;
  const double ca = S->vscale;
  const double2 cb = rmul(-S->vscale, S->beta);
  const double2 cc = cneg(S->k1);
  const double ka = S->ka, kb = S->kb;
  const int wset = cur * D.nsys + sys, pset = pslot * D.nsys + sys;

  // thread 0: the q^ v^ p^ plane m+1 into stage st (x in 8-byte units: even)
  auto issue = [&](int st, int m) {
    const unsigned bb = smem_u32(&bar[st]);
    fence_async_smem();
    mbar_expect(bb, kStage);
    tma_load5(smem_u32(shm + st * kStage), &M.w64, 2 * (i0 - 2), j0 - 1, m + 1, 0, wset, bb);
    tma_load5(smem_u32(shm + st * kStage + 8u * kPN * 16u), &M.p64, 2 * (i0 - 2), j0 - 1, m + 1, 0, pset, bb);
  };
  auto wait = [&](int st) {
    if (!mbar_wait(smem_u32(&bar[st]), (phase >> st) & 1u, kWaitTries) && threadIdx.x == 0) atomicExch(D.err, 1);
    phase ^= 1u << st;
  };
  auto combine = [&](double2 q, double2 v, double2 p, double2 &vo) {
    vo = dcfma(cb, v, rmul(ca, q));
    return dcfma(cc, p, vo);
  };
  const int eo = (ty + 1) * kPW + (tx + 2);
  constexpr int kHaloPos = 2 * (kPTI + kPTJ), kHalo = 4 * kHaloPos;
  auto halo_at = [](int h) {
    return h < 2 * kPTJ ? (h % kPTJ + 1) * kPW + (h < kPTJ ? 1 : kPTI + 2)
                        : (h < 2 * kPTJ + kPTI ? 0 : (kPTJ + 1) * kPW) + (h - 2 * kPTJ) % kPTI + 2;
  };

  double2 um[4], uc[4], up[4], vc[4], vn[4];
  auto own_step = [&](int st, int m1, double2 *Us, double2 (&uo)[4], double2 (&vo)[4]) {
    const double2 *R = reinterpret_cast<const double2 *>(shm + st * kStage);
    const bool owned = live && m1 < k1;
    const long long nd = ndc + m1 * plane;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      uo[c] = combine(R[c * kPN + eo], R[(4 + c) * kPN + eo], R[(8 + c) * kPN + eo], vo[c]);
      Us[c * kPN + eo] = uo[c];
      if (owned) {
        const long long t = c * N + nd;
        Vw[t] = vo[c];
        Pw[t] = uo[c];
      }
    }
  };
  auto halo = [&](int st, double2 *Us) {
    const double2 *R = reinterpret_cast<const double2 *>(shm + st * kStage);
    double2 vt;
#pragma unroll
    for (int h = threadIdx.x; h < kHalo; h += kPThreads) {
      const int hc = h / kHaloPos, he = halo_at(h % kHaloPos);
      Us[hc * kPN + he] = combine(R[hc * kPN + he], R[(4 + hc) * kPN + he], R[(8 + hc) * kPN + he], vt);
    }
  };

  const int ic = min(i, nx - 1), jc = min(j, ny - 1);
  const double4 *AX = D.ax64, *AY = D.ax64 + 2 * nx, *AZ = D.ax64 + 2 * (nx + ny);
  const double4 XA = ldg4(AX + ic), XB = ldg4(AX + nx + ic), YA = ldg4(AY + jc), YB = ldg4(AY + ny + jc);
  const bool hx = live && i < nx - 1, hy = live && j < ny - 1;
  const bool pxy = live && i > 0 && i < nx - 1 && j > 0 && j < ny - 1;
  // sigma-bar / eps-bar of component c at node offset q from this column (0
  // outside the mesh)
  auto sgl = [&](int c, long long q, bool in) { return in ? __ldg(sig + c * N + q) : 0.0; };
  auto epl = [&](int c, long long q, bool in) { return !EPS ? 1.0 : (in ? __ldg(eps + c * N + q) : 1.0); };

  if (threadIdx.x == 0) {
    issue(0, k0 - 1);
    issue(1, k0);
  }
#pragma unroll
  for (int c = 0; c < 4; c++) um[c] = make_double2(0.0, 0.0);
  if (live && k0 > 0) {
    const double2 *Qr = wvec64(D, cur, sys, 0), *Vr = wvec64(D, cur, sys, 1), *Pr = pvec64(D, pslot, sys);
    const long long nd = ndc + (k0 - 1) * plane;
    double2 vt;
#pragma unroll
    for (int c = 0; c < 4; c++) um[c] = combine(__ldg(Qr + c * N + nd), __ldg(Vr + c * N + nd), __ldg(Pr + c * N + nd), vt);
  }
  wait(0);
  own_step(0, k0, Ub, uc, vc);
  halo(0, Ub);
  const long long nd0 = ndc + k0 * plane;
  double s2m = sgl(2, nd0 - plane, live && k0 > 0);  // sigma-bar of Az at k0-1
  double e2m = epl(2, nd0 - plane, live && k0 > 0);
  __syncthreads();
  if (threadIdx.x == 0 && k0 + 1 <= k1 - 1) issue(0, k0 + 1);

  double acc[kParts];
#pragma unroll
  for (int q = 0; q < kParts; q++) acc[q] = 0.0;

  for (int m = k0; m < k1; m++) {
    const int st = (m - k0 + 1) % kStages64;
    const double2 *Uc = Ub + ((m - k0) & 1) * 4 * kPN;
    double2 *Un = Ub + ((m - k0 + 1) & 1) * 4 * kPN;
    const long long nd = ndc + m * plane;
    if (live) {
      // the plain loads of the next plane (sigma-bar) and of the lagged
      // update one plane further (d^, x^) start now, under this plane's work
      if (m + 1 < k1) {
        const long long n1 = nd + plane;
#pragma unroll
        for (int c = 0; c < 4; c++) prefetch_l1(sig + c * N + n1);
        if (j + 1 < ny) prefetch_l1(sig + 3 * N + n1 + D.L.nxp);
        if (j > 0) prefetch_l1(sig + N + n1 - D.L.nxp);
        if (EPS) {
#pragma unroll
          for (int c = 0; c < 4; c++) prefetch_l1(eps + c * N + n1);
        }
      }
    }
    wait(st);
    own_step(st, m + 1, Un, up, vn);
    const double4 ZA = ldg4(AZ + m), ZB = ldg4(AZ + nz + m);
    if (live) {
      const double sx = sgl(0, nd, true), sy = sgl(1, nd, true), sz = sgl(2, nd, true), sp0 = sgl(3, nd, true);
      const double spx = sgl(3, nd + 1, i + 1 < nx), spy = sgl(3, nd + D.L.nxp, j + 1 < ny);
      const double sxm = sgl(0, nd - 1, i > 0), sym = sgl(1, nd - D.L.nxp, j > 0);
      const double s3p = sgl(3, nd + plane, m + 1 < nz);
      const double xn4 = XA.x, xn5 = XA.y, dxc = XA.z, rdxc = XA.w, ce2x = XB.x, ce3x = XB.y, dxi = XB.z,
                   rdxi = XB.w;
      const double yn4 = YA.x, yn5 = YA.y, dyc = YA.z, rdyc = YA.w, ce2y = YB.x, ce3y = YB.y, dyj = YB.z,
                   rdyj = YB.w;
      const double zn4 = ZA.x, zn5 = ZA.y, dzc = ZA.z, rdzc = ZA.w, ce2z = ZB.x, ce3z = ZB.y, dzk = ZB.z,
                   rdzk = ZB.w;
      const double2 *U0 = Uc, *U1 = Uc + kPN, *U2 = Uc + 2 * kPN, *U3 = Uc + 3 * kPN;
      const double2 f0 = uc[3];
      double2 w0, w1, w2, w3;
      double ex = 1.0, ey = 1.0, ez = 1.0, ep0 = 1.0, exm = 1.0, eym = 1.0;
      if (!EPS) {
        w0 = edge_row64(uc[0], U0[eo + 1], ce2x, U0[eo - 1], ce3x, U0[eo + kPW], yn4, U0[eo - kPW], yn5, up[0], zn4,
                        um[0], zn5, sx, spx, sp0, U3[eo + 1], f0, rdxi, dxi * dyc * dzc, ka, kb);
        w1 = edge_row64(uc[1], U1[eo + kPW], ce2y, U1[eo - kPW], ce3y, U1[eo + 1], xn4, U1[eo - 1], xn5, up[1], zn4,
                        um[1], zn5, sy, spy, sp0, U3[eo + kPW], f0, rdyj, dxc * dyj * dzc, ka, kb);
        w2 = edge_row64(uc[2], up[2], ce2z, um[2], ce3z, U2[eo + 1], xn4, U2[eo - 1], xn5, U2[eo + kPW], yn4,
                        U2[eo - kPW], yn5, sz, s3p, sp0, up[3], f0, rdzk, dxc * dyc * dzk, ka, kb);
        w3 = node_row64(f0, U3[eo + 1], U3[eo - 1], U3[eo + kPW], U3[eo - kPW], up[3], um[3], xn4, xn5, yn4, yn5,
                        zn4, zn5, uc[0], U0[eo - 1], uc[1], U1[eo - kPW], uc[2], um[2], rdxc, rdyc, rdzc, sx, sxm,
                        sy, sym, sz, s2m, sp0, dxc * dyc * dzc, ka, kb);
      } else {
        ex = epl(0, nd, true), ey = epl(1, nd, true), ez = epl(2, nd, true), ep0 = epl(3, nd, true);
        exm = epl(0, nd - 1, i > 0), eym = epl(1, nd - D.L.nxp, j > 0);
        auto K2 = [&](double s_, double e_) { return make_double2(-ka * e_, kb * s_); };
        const double2 kp0 = K2(sp0, ep0);
        const double2 kx = K2(sx, ex), ky = K2(sy, ey), kz = K2(sz, ez);
        w0 = edge_row64_c(uc[0], U0[eo + 1], ce2x, U0[eo - 1], ce3x, U0[eo + kPW], yn4, U0[eo - kPW], yn5, up[0],
                          zn4, um[0], zn5, kx, K2(spx, epl(3, nd + 1, i + 1 < nx)), kp0, U3[eo + 1], f0, rdxi,
                          dxi * dyc * dzc);
        w1 = edge_row64_c(uc[1], U1[eo + kPW], ce2y, U1[eo - kPW], ce3y, U1[eo + 1], xn4, U1[eo - 1], xn5, up[1],
                          zn4, um[1], zn5, ky, K2(spy, epl(3, nd + D.L.nxp, j + 1 < ny)), kp0, U3[eo + kPW], f0,
                          rdyj, dxc * dyj * dzc);
        w2 = edge_row64_c(uc[2], up[2], ce2z, um[2], ce3z, U2[eo + 1], xn4, U2[eo - 1], xn5, U2[eo + kPW], yn4,
                          U2[eo - kPW], yn5, kz, K2(s3p, epl(3, nd + plane, m + 1 < nz)), kp0, up[3], f0, rdzk,
                          dxc * dyc * dzk);
        w3 = node_row64_c(f0, U3[eo + 1], U3[eo - 1], U3[eo + kPW], U3[eo - kPW], up[3], um[3], xn4, xn5, yn4, yn5,
                          zn4, zn5, uc[0], U0[eo - 1], uc[1], U1[eo - kPW], uc[2], um[2], rdxc, rdyc, rdzc, kx,
                          K2(sxm, exm), ky, K2(sym, eym), kz, K2(s2m, e2m), kp0, dxc * dyc * dzc);
      }
      const double2 zero2 = make_double2(0.0, 0.0);
      double2 w[4] = {hx ? w0 : zero2, hy ? w1 : zero2, m < nz - 1 ? w2 : zero2,
                      (pxy && m > 0 && m < nz - 1) ? w3 : zero2};
      double2 dg[4];
      const bool pin = pxy && m > 0 && m < nz - 1;
      jacobi64(XA, XB, YA, YB, ZA, ZB, sx, sy, sz, sp0, pin ? sxm : 0.0, pin ? sym : 0.0, pin ? s2m : 0.0, ex, ey,
               ez, ep0, pin ? exm : 1.0, pin ? eym : 1.0, pin ? e2m : 1.0, hx, hy, m < nz - 1, pin, ka, kb, dg);
      double r[kParts];
#pragma unroll
      for (int q = 0; q < kParts; q++) r[q] = 0.0;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const double2 z = dg[c];
        double2 d;
        double rs, mag;
        jacobi_weights(z, d, rs, mag);
        const double2 ww = w[c], u = uc[c], v = vc[c];
        const double2 qh = cmul(d, ww);
        Qw[c * N + nd] = qh;
        r[0] += u.x * ww.x - u.y * ww.y;
        r[1] += u.x * ww.y + u.y * ww.x;
        r[2] += mag * (ww.x * ww.x + ww.y * ww.y);
        r[3] += rs * (v.x * qh.x + v.y * qh.y);
        r[4] += rs * (v.x * qh.y - v.y * qh.x);
        r[5] += rs * (v.x * v.x + v.y * v.y);
        r[6] += ww.x * qh.x - ww.y * qh.y;
        r[7] += ww.x * qh.y + ww.y * qh.x;
        r[8] += ww.x * v.x - ww.y * v.y;
        r[9] += ww.x * v.y + ww.y * v.x;
        const double v2r = v.x * v.x - v.y * v.y, v2i = 2.0 * v.x * v.y;
        r[10] += v2r * z.x - v2i * z.y;
        r[11] += v2r * z.y + v2i * z.x;
      }
#pragma unroll
      for (int q = 0; q < kParts; q++) acc[q] += r[q];
      s2m = sz;
      e2m = ez;
    }
    if (m + 1 < k1) halo(st, Un);
    __syncthreads();  // everyone is done with stage st and u plane m
    if (threadIdx.x == 0 && m + 2 <= k1 - 1) issue(st, m + 2);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      um[c] = uc[c];
      uc[c] = up[c];
      vc[c] = vn[c];
    }
  }

  Vals<kParts> blk;
#pragma unroll
  for (int q = 0; q < kParts; q++) blk.v[q] = acc[q];
  blk = block_reduce<kParts, kPThreads>(blk);
  double *part = D.part + (size_t)sys * D.slots * kParts;
  unsigned *cnt = D.cnt + CNT_PASS * D.nsys + sys;
  const unsigned nt = (unsigned)D.tp.count();
  if (arrive<kParts, kPThreads>(blk, part, cnt, (unsigned)tile, nt)) {
    Vals<kParts> tot = final_reduce<kParts, kPThreads>(part, cnt, nt);
    if (threadIdx.x == 0) {
      if (D.timing) {
        S->cur ^= 1;
        S->pslot = (S->pslot + 1) % (D.ring64 + 1);
      } else {
        pass_scalars(S, tot.v, D.ring64);
      }
    }
  }
  }  // work items
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(D.work + 1, 1) == gridDim.x - 1) {
      D.work[0] = 0;
      D.work[1] = 0;
      __threadfence();
    }
  }
}


}  // namespace aphid

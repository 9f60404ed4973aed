/*
 * aphid_gpu.h -- C ABI of the B200 (sm_100a) implementation of APhiD's
 * frequency-domain solve: the matrix-free Lorenz-gauged A-Phi operator on the
 * staggered Yee grid and the Jacobi-preconditioned complex-symmetric QMR
 * that inverts it.
 *
 * The ABI uses plain C types only, so a Fortran host can bind it with
 * ISO_C_BINDING (aphid_git_b200/fortran/aphid_gpu_mod.f90) and Python with
 * ctypes (aphid_git_b200/abi.py).
 *
 * Conventions
 *   - aphid_z is layout-identical to Fortran complex(c_double_complex) and to
 *     C99 double _Complex.
 *   - Every array is Fortran column-major with the reference's shapes:
 *       Ax, k2_x, diag_x, rhs_x : (nx-1, ny,   nz  )   x-directed edges
 *       Ay, ...                 : (nx,   ny-1, nz  )   y-directed edges
 *       Az, ...                 : (nx,   ny,   nz-1)   z-directed edges
 *       Phi, ...                : (nx,   ny,   nz  )   nodes
 *       cells (sigma)           : (nx-1, ny-1, nz-1)
 *     (nx, ny, nz are NODE counts, as in the reference's aphid.mesh.)
 *   - dx, dy, dz are dx(0:nx) etc. (nx+1 values); dxc, dyc, dzc are
 *     dxc(1:nx) etc. (nx values), exactly the module mesh arrays
 *     (src/aphid_mod.f90:44-45, filled by src/aphid.f90:341-361).
 *   - Host pointers belong to the caller; the library copies in and out and
 *     keeps no host pointer after a call returns.
 *   - Calls are synchronous and never abort the process.  They return
 *     APHID_OK (0) or a negative APHID_ERR_* code; aphid_gpu_last_error()
 *     gives the message.  Solver outcomes (converged, iteration cap,
 *     breakdown) are reported in aphid_info.status, not as errors, because
 *     the reference only warns on non-convergence
 *     (src/aphid_qmr.f90:394-401).
 *   - One context per host thread.
 */
#ifndef APHID_GPU_H
#define APHID_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } aphid_z;
typedef struct aphid_ctx aphid_ctx;

/* call results */
#define APHID_OK             0
#define APHID_ERR_BADARG    -1   /* invalid argument (sizes, pointers, flags) */
#define APHID_ERR_CUDA      -2   /* CUDA runtime error, message in last_error */
#define APHID_ERR_NOMEM     -3   /* device allocation failed */
#define APHID_ERR_STATE     -4   /* call order: e.g. solve before set_mesh */
#define APHID_ERR_NODEVICE  -5   /* no usable sm_100 device */

/* aphid_info.status */
#define APHID_CONVERGED      0   /* residual below target */
#define APHID_MAXIT          1   /* iteration cap reached (reference warns) */
#define APHID_BREAKDOWN      2   /* QMR breakdown: delta, epsilon, beta or rho = 0 */
#define APHID_NONFINITE      3   /* NaN/Inf in a recurrence scalar */

/* precision of aphid_gpu_sweep */
#define APHID_PREC_FP64      0   /* plain complex128 Jacobi-QMR, the reference's algorithm */
#define APHID_PREC_MIXED     1   /* complex64 inner QMR inside FP64 defect correction */
#define APHID_PREC_FUSED64   2   /* complex128 inner QMR, the batched fused pass in FP64 */
#define APHID_PREC_AUTO      3   /* MIXED; a system whose complex-symmetric Lanczos form
                                    v^T v collapses below complex64 resolution, or whose
                                    complex64 cycles twice in a row lower the FP64 residual
                                    by less than 2x, is finished by FUSED64 from its
                                    current iterate */

typedef struct {
  int device;        /* CUDA device ordinal */
  void *stream;      /* cudaStream_t to run on; NULL = a stream owned by the context */
  int graph_iters;   /* QMR iterations per CUDA-graph launch; 0 = default (16) */
  int verbose;       /* 1 = progress lines on stderr */
  int plane_kz;      /* z-planes per work item of the complex64 pass (>= 4);
                        0 = autotuned: timed on the device for each new
                        (mesh, batch, model kind) and cached, in the process
                        and in the file named by APHID_TUNE_CACHE if set */
} aphid_opts;

typedef struct {
  int status;               /* APHID_CONVERGED / MAXIT / BREAKDOWN / NONFINITE */
  int iters;                /* iteration count as the reference reports it */
  int inner_iters;          /* total inner (complex64) iterations, mixed path */
  int outer_iters;          /* defect-correction steps, mixed path */
  double rhs_norm;          /* ||b||_2 */
  double recur_resid;       /* last recurrence residual norm ||r|| (absolute) */
  double true_rel_resid;    /* ||b - K x||_2 / ||b||_2 recomputed in FP64 */
  double seconds;           /* device time of the solve (CUDA events) */
  long long kernel_launches; /* kernels this call launched (graph nodes included) */
  int inner64_iters;        /* of inner_iters, those run in complex128 (FUSED64, or
                               AUTO after escalation) */
} aphid_info;

/* ---- context --------------------------------------------------------- */

/* Create a context on opts->device (opts may be NULL: device 0, own stream). */
int aphid_gpu_create(aphid_ctx **ctx, const aphid_opts *opts);
int aphid_gpu_destroy(aphid_ctx *ctx);
/* Message of the last failed call on this context (never NULL). */
const char *aphid_gpu_last_error(const aphid_ctx *ctx);

/* Mesh geometry: the module mesh arrays (src/aphid_mod.f90:40-45).
 * Requires nx, ny, nz >= 3 and positive spacings. */
int aphid_gpu_set_mesh(aphid_ctx *ctx, int nx, int ny, int nz,
                       const double *dx, const double *dy, const double *dz,
                       const double *dxc, const double *dyc, const double *dzc);

/* ---- operator-level entry points -------------------------------------- */

/* out = K in for all four blocks: replaces inprod_x/inprod_y/inprod_z/
 * inprod_p (src/aphid.f90:803-871, 932-1000, 1061-1128, 1191-1282) with the
 * coefficient tables of gen_inprod_*_coefs (src/aphid.f90:750-1185). */
int aphid_gpu_inprod(aphid_ctx *ctx,
                     const aphid_z *k2_x, const aphid_z *k2_y,
                     const aphid_z *k2_z, const aphid_z *k2_p,
                     const aphid_z *in_x, const aphid_z *in_y,
                     const aphid_z *in_z, const aphid_z *in_p,
                     aphid_z *out_x, aphid_z *out_y, aphid_z *out_z,
                     aphid_z *out_p);

/* k^2 grids from cell sigma-hat: replaces gen_k2_xgrid/_ygrid/_zgrid/_pgrid
 * (src/aphid.f90:1289-1535).  sig: complex cell array (nx-1,ny-1,nz-1). */
int aphid_gpu_gen_k2(aphid_ctx *ctx, const aphid_z *sig, double omega,
                     aphid_z *k2_x, aphid_z *k2_y, aphid_z *k2_z,
                     aphid_z *k2_p);

/* Jacobi diagonal: replaces gen_diag (src/aphid.f90:1542-1725). */
int aphid_gpu_gen_diag(aphid_ctx *ctx,
                       const aphid_z *k2_x, const aphid_z *k2_y,
                       const aphid_z *k2_z, const aphid_z *k2_p,
                       aphid_z *diag_x, aphid_z *diag_y, aphid_z *diag_z,
                       aphid_z *diag_p);

/* ---- the solve ---------------------------------------------------------- */

/* Drop-in for `call qmr` / `call qmr_mthread` (src/aphid.f90:102-104;
 * solver src/aphid_qmr.f90:5-434).  rhs_* hold b on entry and the solution on
 * return, exactly as the reference overwrites rhs_* (src/aphid_qmr.f90:225-240).
 * Same recurrence, same stopping rule (recurrence residual
 * < qmr_target * ||b||, src/aphid_qmr.f90:386-390) and the same iteration
 * count semantics, in complex128 on the GPU.
 * x0_* (all NULL, or all non-NULL) is an optional initial guess; the
 * reference starts from zero (src/aphid_qmr.f90:230-233).
 * hist (nullable) receives the recurrence residual of each iteration (the
 * content of qmr.iter, src/aphid_qmr.f90:381), up to hist_cap values;
 * info->iters tells how many were written (min(iters, hist_cap) when
 * converged).  info may be NULL. */
int aphid_gpu_qmr(aphid_ctx *ctx,
                  const aphid_z *k2_x, const aphid_z *k2_y,
                  const aphid_z *k2_z, const aphid_z *k2_p,
                  const aphid_z *diag_x, const aphid_z *diag_y,
                  const aphid_z *diag_z, const aphid_z *diag_p,
                  aphid_z *rhs_x, aphid_z *rhs_y, aphid_z *rhs_z,
                  aphid_z *rhs_p,
                  const aphid_z *x0_x, const aphid_z *x0_y,
                  const aphid_z *x0_z, const aphid_z *x0_p,
                  double qmr_target, int qmr_max_it,
                  double *hist, int hist_cap, aphid_info *info);

/* The same solve split in three, for callers that keep a problem resident
 * on the device and re-solve it (benchmarks, restarts):
 *   aphid_gpu_qmr_load   copies k2_*, diag_* and rhs_* (= b) to the device,
 *   aphid_gpu_qmr_run    runs the solve on the resident copies (x0 = 0, or
 *                        the resident solution when use_previous_x != 0),
 *   aphid_gpu_qmr_fetch  copies the solution back into sol_*.
 * aphid_gpu_qmr is exactly load + run + fetch. */
int aphid_gpu_qmr_load(aphid_ctx *ctx,
                       const aphid_z *k2_x, const aphid_z *k2_y,
                       const aphid_z *k2_z, const aphid_z *k2_p,
                       const aphid_z *diag_x, const aphid_z *diag_y,
                       const aphid_z *diag_z, const aphid_z *diag_p,
                       const aphid_z *rhs_x, const aphid_z *rhs_y,
                       const aphid_z *rhs_z, const aphid_z *rhs_p);
int aphid_gpu_qmr_run(aphid_ctx *ctx, double qmr_target, int qmr_max_it,
                      int use_previous_x, double *hist, int hist_cap,
                      aphid_info *info);
int aphid_gpu_qmr_fetch(aphid_ctx *ctx, aphid_z *sol_x, aphid_z *sol_y,
                        aphid_z *sol_z, aphid_z *sol_p);

/* Device-pointer form of aphid_gpu_inprod for callers whose vectors already
 * live on this context's device (e.g. framework tensors): d_k2, d_in, d_out
 * are concatenated [x|y|z|p] complex128 vectors of the mesh's unknown count.
 * When d_eps is non-NULL the bilinear form in^T out (unconjugated, the
 * epsilon of src/aphid_qmr.f90:329) is reduced on the device and written
 * there as one aphid_z.  The reduction uses the context's scratch buffers.
 * All four pointers must be 16-byte aligned (APHID_ERR_BADARG otherwise).
 * Runs on the context's stream; returns after the launch (asynchronous). */
int aphid_gpu_inprod_dev(aphid_ctx *ctx, const void *d_k2, const void *d_in,
                         void *d_out, void *d_eps);

/* ---- batched frequency sweep ------------------------------------------- */

/* Cell model for the sweep: csig_flag 'R' (sig_re; sigma-hat = sigma +
 * i omega eps0), 'C' (sig_re and eps_rel; sigma + i omega eps0 eps_rel) or
 * 'I' (eps_rel only; i omega eps0 eps_rel), the linear models of read_mesh
 * (src/aphid.f90:379-449), real(4) cell arrays (nx-1,ny-1,nz-1).  The
 * area/volume-weighted averages of gen_k2_*grid are formed once on the device
 * in FP64; every system's k^2 follows from them and its omega.  'D'
 * (Cole-Cole) has four cell arrays: aphid_gpu_set_model_cole_cole. */
int aphid_gpu_set_model(aphid_ctx *ctx, char csig_flag, const float *sig_re,
                        const float *eps_rel);

/* Cole-Cole cell model (read_mesh csig_flag 'D', src/aphid.f90:410-435):
 * sigma-hat = sigma (1 - eta / (1 + (i omega tau)^c)), real(4) cell arrays
 * sig_re, eta (chargeability), tau (time constant) and cee (frequency
 * exponent).  sigma-hat is not linear in omega, so each sweep forms one
 * averaged model per system on the device (gen_k2_*grid's averages of the
 * complex sigma-hat at that system's omega): about 80 bytes per unknown and
 * system beyond the linear models. */
int aphid_gpu_set_model_cole_cole(aphid_ctx *ctx, const float *sig_re,
                                  const float *eta, const float *tau,
                                  const float *cee);

typedef struct {
  int precision;      /* APHID_PREC_FP64, _MIXED, _FUSED64 or _AUTO */
  double target;      /* MIXED, FUSED64, AUTO: stop when ||b - K x||_2 <
                         target ||b||_2 (FP64 true residual); FP64: the
                         reference's recurrence stop test with this
                         qmr_target */
  int max_it;         /* iteration cap per system (inner iterations, MIXED) */
  double inner_tol;   /* MIXED: cap on the inner quasi-residual reduction per
                         defect-correction step (0 = 1e-10); a cycle also
                         ends when the true residual, checked every graph
                         round, converges or stagnates */
  int max_outer;      /* MIXED: cap on defect-correction steps (0 = 40) */
  int stall_window;   /* MIXED, AUTO: a cycle whose quasi-residual has not
                         halved over this many inner iterations restarts from
                         the FP64 residual (0 = 400, < 0 = never); FUSED64:
                         0 = never */
  int reserved[2];
} aphid_sweep_opts;

/* Solve nsys systems (frequency x source) on the context's mesh and model:
 * the MPI farm of src/aphid_parallel.f90 as one batched GPU solve.  System s
 * has angular frequency omega[s] and source source_of_system[s]; source q is
 * an oper_mode-5 dipole list (src/aphid.f90:638-741) of src_ndip[q] dipoles,
 * stored consecutively in dip_dir (2 chars each, "+X" ... "-Z") and dip_ijk
 * (1-based tail-end node, 3 ints each).  Out-of-range or invalid dipoles are
 * skipped, as the reference does.
 * x0 (nullable): nsys concatenated [x|y|z|p] initial guesses.
 * x_out (nullable): nsys concatenated solutions; when NULL the solutions stay
 * on the device for aphid_gpu_sweep_fetch.  info: nsys records. */
int aphid_gpu_sweep(aphid_ctx *ctx, int nsys, const double *omega,
                    const int *source_of_system, int nsrc, const int *src_ndip,
                    const char *dip_dir, const int *dip_ijk, const aphid_z *x0,
                    const aphid_sweep_opts *opts, aphid_z *x_out,
                    aphid_info *info);

/* A source of the batched sweep, as gen_rhs forms it (src/aphid.f90:534-743):
 *   oper_mode 2: x-polarised MT plane-wave source, a sheet current on every
 *                x-edge of node layer k = 2 (src/aphid.f90:590-603);
 *   oper_mode 3: y-polarised MT source on the y-edges of layer 2 (:607-619);
 *   oper_mode 5: a dipole list (:638-741): ndip dipoles, 2 chars each in
 *                dip_dir ("+X" ... "-Z") and their 1-based tail-end nodes,
 *                3 ints each, in dip_ijk; invalid or out-of-range dipoles are
 *                skipped as the reference skips them.
 * The MPI farm's aphid_mpi.input chooses between the two kinds: MT sweeps
 * run modes 2 and 3 per frequency, CS sweeps one mode-5 list per dipole
 * array (src/aphid_parallel.f90:75-103). */
typedef struct {
  int oper_mode;
  int ndip;
  const char *dip_dir;
  const int *dip_ijk;
} aphid_source;

/* aphid_gpu_sweep with sources of any of the kinds above: system s solves
 * for source srcs[source_of_system[s]] at omega[s].  aphid_gpu_sweep is this
 * call with every source a dipole list. */
int aphid_gpu_sweep_sources(aphid_ctx *ctx, int nsys, const double *omega,
                            const int *source_of_system, int nsrc,
                            const aphid_source *srcs, const aphid_z *x0,
                            const aphid_sweep_opts *opts, aphid_z *x_out,
                            aphid_info *info);

/* Several meshes in one batched solve.  Each job is one context (its own
 * mesh and model, set with aphid_gpu_set_mesh / aphid_gpu_set_model) with
 * its own systems, sources, optional x0, optional x_out and info records,
 * exactly the arguments of aphid_gpu_sweep_sources.  With precision MIXED or
 * AUTO and models of one kind (R, or C and I), the complex64 QMR passes of
 * all jobs run as one persistent launch per iteration whose blocks take work
 * items from every mesh, so systems of uneven mesh sizes share the GPU
 * without a launch per mesh; escalated systems (AUTO) then finish per
 * context.  Other precisions, Cole-Cole models, mixed model kinds or a single
 * job run the jobs one after another.  All contexts must be on one device;
 * the shared work runs on the first job's stream, and info->seconds is the
 * group's time.  At most 8 jobs. */
typedef struct {
  aphid_ctx *ctx;
  int nsys;
  const double *omega;
  const int *source_of_system;
  int nsrc;
  const aphid_source *srcs;
  const aphid_z *x0;   /* nullable */
  aphid_z *x_out;      /* nullable */
  aphid_info *info;    /* nullable */
} aphid_group_job;
int aphid_gpu_sweep_group(int njob, const aphid_group_job *jobs,
                          const aphid_sweep_opts *opts);

/* Receiver gather after a sweep: E and H = B / mu0 at nrec mesh nodes for
 * every system of the last sweep, without moving the solutions to the host.
 * The node values are dump_fields' EM_grid interpolation
 * (src/aphid.f90:2012-2165): E is the mean of the two edges through the node
 * along each axis (E = -i omega (A - grad Phi), gen_fields
 * src/aphid.f90:2225-2250), B the mean of the four faces around the node
 * (B = curl A, :2191-2216).  rec_ijk: 1-based node indices, 3 ints per
 * receiver, each in 2..n-1 as EM_grid's nodes are.  E, H (either may be
 * NULL): [nsys][nrec][3] values (x, y, z components). */
int aphid_gpu_sweep_receivers(aphid_ctx *ctx, int nrec, const int *rec_ijk,
                              aphid_z *E, aphid_z *H);

/* z-planes per work item of the fused pass that ran last (the autotuner's
 * choice unless aphid_opts.plane_kz fixed it): the complex128 pass's after
 * an AUTO sweep that escalated systems or a FUSED64 sweep, else the
 * complex64 pass's; 0 before the first mixed sweep. */
int aphid_gpu_sweep_plane_kz(aphid_ctx *ctx);

/* Pipeline configuration of the complex64 pass in use: 0 = two load stages
 * (two resident blocks per SM for model R), 1 = three load stages in one
 * block per SM; chosen with the slab depth by the autotuner (0 when
 * aphid_opts.plane_kz fixes the depth). */
int aphid_gpu_sweep_pass_config(aphid_ctx *ctx);

/* Plane-tile shape of the fused passes in use: 0 = 16 x 16 nodes, 1 = 32 x 8;
 * chosen with the slab depth by the autotuner (0 when aphid_opts.plane_kz
 * fixes the depth). */
int aphid_gpu_sweep_tile_shape(aphid_ctx *ctx);

/* Copy system `sys` of the last sweep into x (one [x|y|z|p] vector). */
int aphid_gpu_sweep_fetch(aphid_ctx *ctx, int sys, aphid_z *x);

/* Benchmarking hook, no counterpart in the reference: launch the fused
 * QMR iteration pass -- complex64, or complex128 after a FUSED64 sweep --
 * (p update, q^ = D^-1 K p^, the lagged d/x update with zero weights, the
 * inner products) `reps` times over all systems of the last batched sweep,
 * on the context's stream, without
 * the scalar recurrence.  The solutions (aphid_gpu_sweep_fetch) are not
 * changed; the inner Krylov vectors are, as by an iteration.  An AUTO sweep
 * that escalated systems releases its inner buffers, so after one this returns
 * APHID_ERR_STATE until the next MIXED, AUTO or FUSED64 sweep.  Returns after
 * the launches (asynchronous). */
int aphid_gpu_sweep_time_apply(aphid_ctx *ctx, int reps);

/* Testing hook, no counterpart in the reference: y = K x with the operator of
 * the fused pass of the last batched sweep -- the complex64 pass (x rounded
 * to complex64, the rows in FP32 arithmetic) after MIXED or AUTO, the
 * complex128 pass after FUSED64 -- for its system 0 (that frequency, on the
 * context's model), so that tests can hold each pass to the reference's K
 * (src/aphid_qmr.f90 inprod_*) row by row.  x and y are host arrays of n
 * complex128.  Like aphid_gpu_sweep_time_apply it overwrites the inner
 * Krylov vectors of that sweep; the solutions are kept.  Synchronises the
 * stream. */
int aphid_gpu_sweep_apply(aphid_ctx *ctx, const aphid_z *x, aphid_z *y);

/* ---- allocation-free operator apply -------------------------------------- */

/* No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc -- code that runs inside a memory pool or a framework allocator
 * owning all device memory, or a host that must not allocate once a run has
 * started.  It computes what aphid_gpu_inprod_dev with a non-NULL d_eps
 * computes (out = K in, and the epsilon in^T out written to *d_eps as one
 * aphid_z; the same rows, the epsilon summed in another order), but needs no
 * context and allocates nothing: every argument
 * is a caller-owned device pointer on the current device (d_dx..d_dzc hold
 * dx(0:n) and dxc(1:n) as in aphid_gpu_set_mesh; d_k2, d_in, d_out are the
 * concatenated [x|y|z|p] complex128 vectors).  Its scratch is one fixed
 * file-scope device array of about 400 KB, held by every GPU that loads the
 * library until the process exits; meshes larger than
 * APHID_NOALLOC_MAX_NODES nodes per axis are rejected with APHID_ERR_BADARG.
 * All calls share that array: calls that overlap on the GPU race on it.  Each
 * call looks up the array's address in the current context; the first call
 * on a device also loads the library's kernels there, so make it before any
 * stream capture.  Runs on `stream` (a cudaStream_t, NULL = legacy default)
 * and returns after the launch. */
#define APHID_NOALLOC_MAX_NODES 1024
#define APHID_NOALLOC_MAX_SLOTS 16384
int aphid_gpu_inprod_eps_noalloc(int nx, int ny, int nz,
                                 const double *d_dx, const double *d_dy,
                                 const double *d_dz, const double *d_dxc,
                                 const double *d_dyc, const double *d_dzc,
                                 const void *d_k2, const void *d_in,
                                 void *d_out, void *d_eps, void *stream);

/* ---- post-processing ---------------------------------------------------- */

/* B = curl A on cell faces and E = -i omega (A - grad Phi) on edges:
 * replaces gen_fields (src/aphid.f90:2173-2252).  Shapes:
 * Bx (nx,ny-1,nz-1), By (nx-1,ny,nz-1), Bz (nx-1,ny-1,nz); Ex/Ey/Ez the edge
 * shapes.  Any output pointer may be NULL to skip it. */
int aphid_gpu_fields(aphid_ctx *ctx, double omega,
                     const aphid_z *a_x, const aphid_z *a_y,
                     const aphid_z *a_z, const aphid_z *phi,
                     aphid_z *b_x, aphid_z *b_y, aphid_z *b_z,
                     aphid_z *e_x, aphid_z *e_y, aphid_z *e_z);

#ifdef __cplusplus
}
#endif
#endif /* APHID_GPU_H */

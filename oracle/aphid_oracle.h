/*
 * aphid_oracle.h -- CPU restatement of APhiD's frequency-domain solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline legs may load it.
 * The product path (aphid_git_b200) never links or calls it.
 *
 * Parity status: parity unpinned against a reference binary.  The
 * reference is Fortran 90 (+OpenMP, +MPI for mpi_wtime) and neither this
 * machine nor the GPU machine has a Fortran compiler, and the reference
 * ships no tests, fixtures or sample outputs.  The restatement is pinned
 * instead by an independent NumPy/SciPy assembly of the same operator
 * (tests/golden/make_golden.py), by structural identities of the operator,
 * by a sparse direct solve, and by the 1-D magnetotelluric analytic
 * solution the reference's paper validates against.
 *
 * Conventions
 *   - Arrays are Fortran column-major: 1-based (i,j,k) of an (n1,n2,n3)
 *     block lives at (i-1) + n1*((j-1) + n2*(k-1)).
 *   - A "vector" is the concatenation [Ax | Ay | Az | Phi] with block shapes
 *     (nx-1,ny,nz), (nx,ny-1,nz), (nx,ny,nz-1), (nx,ny,nz): the unknown
 *     ordering of the reference (src/aphid_qmr.f90:157).
 *   - d[0..n] is dx(0:n) and dc[0..n-1] is dxc(1:n) (src/aphid_mod.f90:44-45).
 *   - Complex numbers are C99 double _Complex, layout-identical to Fortran
 *     complex(8); the file is compiled with -fcx-fortran-rules.
 */
#ifndef APHID_ORACLE_H
#define APHID_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } orc_z;   /* ABI view of double _Complex */

/* node coordinates -> dx(0:n), dxc(1:n)   (src/aphid.f90:341-361) */
void orc_spacings(int n, const double *xn, double *d, double *dc);

/* cell sigma-hat for csig_flag R/C/D/I (src/aphid.f90:379-449).  Inputs are
 * real(4) as in the reference (src/aphid.f90:288).  Returns 0 or -1. */
int orc_sigma_hat(char mode, size_t ncell, double omega,
                  const float *sig_re, const float *eps_rel, const float *eta,
                  const float *tau, const float *cee, orc_z *sig);

/* k^2 on x/y/z edges and nodes (src/aphid.f90:1289-1535).  out = concat
 * vector of nunk complex values in [x|y|z|p] order. */
void orc_gen_k2(int nx, int ny, int nz, const double *dx, const double *dy,
                const double *dz, const orc_z *sig, double omega, orc_z *k2);

/* Jacobi diagonal (src/aphid.f90:1542-1725).  k2, diag: concat vectors. */
void orc_gen_diag(int nx, int ny, int nz, const double *dx, const double *dy,
                  const double *dz, const orc_z *k2, orc_z *diag);

/* y = K x for all four blocks (coefficient tables src/aphid.f90:750-797,
 * 878-925, 1007-1054, 1135-1185; stencils inprod_x/y/z/p
 * src/aphid.f90:803-871, 932-1000, 1061-1128, 1191-1282). */
void orc_inprod(int nx, int ny, int nz, const double *dx, const double *dy,
                const double *dz, const double *dxc, const double *dyc,
                const double *dzc, const orc_z *k2, const orc_z *x, orc_z *y);

/* RHS for oper_mode 1,2,3,4,5 (src/aphid.f90:534-743).  Mode 5 takes ndip
 * dipoles: dirs[2*d..2*d+1] in {"+X","-X","+Y","-Y","+Z","-Z"} and
 * ijk[3*d..3*d+2] the tail-end node.  Out-of-range or invalid dipoles are
 * skipped as the reference does; *nskipped counts them.  Returns 0, or -1
 * when mode 1 finds no node at the origin or mode 4 does not fit. */
int orc_gen_rhs(int mode, int nx, int ny, int nz, const double *xn,
                const double *yn, const double *zn, const double *dx,
                const double *dy, const double *dz, int ndip,
                const char *dirs, const int *ijk, orc_z *rhs, int *nskipped);

/* Jacobi-preconditioned complex-symmetric QMR (src/aphid_qmr.f90:5-434).
 * rhs: in b, out x (overwritten, as the reference does with rhs_*).
 * x0 (nullable) is an initial guess; the reference always starts from 0.
 * nthreads 1 = qmr (single thread); 4 = qmr_mthread's component split
 * (src/aphid_qmr.f90:744-928) without its delta race.
 * hist[] receives rnorm per iteration (capacity hist_cap).
 * Returns the iteration count as the reference reports it. */
int orc_qmr(int nx, int ny, int nz, const double *dx, const double *dy,
            const double *dz, const double *dxc, const double *dyc,
            const double *dzc, const orc_z *k2, const orc_z *diag,
            orc_z *rhs, const orc_z *x0, double target, int max_it,
            int nthreads, double *hist, int hist_cap, double *rnorm_out,
            double *rhsnorm_out, int *converged, double *seconds);

/* B = curl A on faces and E = -i omega (A - grad Phi) on edges
 * (src/aphid.f90:2173-2252).  B = concat [Bx(nx,ny-1,nz-1) |
 * By(nx-1,ny,nz-1) | Bz(nx-1,ny-1,nz)], E = concat [Ex | Ey | Ez] with the
 * edge shapes of A. */
void orc_gen_fields(int nx, int ny, int nz, const double *dx,
                    const double *dy, const double *dz, double omega,
                    const orc_z *sol, orc_z *B, orc_z *E);

/* vector length (src/aphid_qmr.f90:157) */
size_t orc_nunk(int nx, int ny, int nz);

#ifdef __cplusplus
}
#endif
#endif

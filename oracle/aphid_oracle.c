/*
 * aphid_oracle.c -- CPU restatement of APhiD's frequency-domain solve.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the
 * product never links it.  Parity against a reference binary is unpinned
 * (no Fortran compiler exists here); see aphid_oracle.h for how the
 * restatement is pinned instead.
 *
 * Every routine follows one reference routine, cited by file:line, keeping
 * its loop order, its sequential left-to-right sums (gfortran's SUM) and its
 * operation order, so that results agree with the Fortran to rounding.
 * Build: see oracle/Makefile (-O2 -fno-fast-math -ffp-contract=off
 * -fcx-fortran-rules).
 */
#include "aphid_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex zc;

/* constants of module general (src/aphid_mod.f90:9-12) */
static const double PI = 3.141592653589793;
#define MU0 (PI * 4.e-7)
static const double EPS0 = 8.8541878176e-12;

/* 1-based Fortran index into an (n1,n2,*) block */
#define F3(i, j, k, n1, n2) \
  ((size_t)((i)-1) + (size_t)(n1) * ((size_t)((j)-1) + (size_t)(n2) * (size_t)((k)-1)))

typedef struct {
  int nx, ny, nz;
  size_t nxe, nye, nze, np;   /* block lengths */
  size_t ox, oy, oz, op;      /* block offsets in the concat vector */
  size_t n;                   /* total unknowns */
} layout_t;

static layout_t mk_layout(int nx, int ny, int nz) {
  layout_t L;
  L.nx = nx; L.ny = ny; L.nz = nz;
  L.nxe = (size_t)(nx - 1) * ny * nz;
  L.nye = (size_t)nx * (ny - 1) * nz;
  L.nze = (size_t)nx * ny * (nz - 1);
  L.np = (size_t)nx * ny * nz;
  L.ox = 0; L.oy = L.nxe; L.oz = L.oy + L.nye; L.op = L.oz + L.nze;
  L.n = L.op + L.np;
  return L;
}

size_t orc_nunk(int nx, int ny, int nz) { return mk_layout(nx, ny, nz).n; }

/* src/aphid.f90:341-361 */
void orc_spacings(int n, const double *xn, double *d, double *dc) {
  for (int i = 1; i <= n - 1; i++) d[i] = xn[i] - xn[i - 1];
  d[0] = d[1];
  d[n] = d[n - 1];
  for (int i = 2; i <= n - 1; i++) dc[i - 1] = 0.5 * (d[i - 1] + d[i]);
  dc[0] = dc[1];
  dc[n - 1] = dc[n - 2];
}

/* src/aphid.f90:379-449: sig = sig_re + II*omega*EPS0 (R);
 * sig_re + II*omega*EPS0*eps_rel (C);
 * sig_re*(1 - eta/(1 + (II*omega*tau)**cee)) (D); II*omega*EPS0*eps_rel (I) */
int orc_sigma_hat(char mode, size_t ncell, double omega, const float *sig_re,
                  const float *eps_rel, const float *eta, const float *tau,
                  const float *cee, orc_z *out) {
  zc *sig = (zc *)out;
  const zc II = I;
  for (size_t c = 0; c < ncell; c++) {
    switch (mode) {
      case 'R': sig[c] = (double)sig_re[c] + II * omega * EPS0; break;
      case 'C': sig[c] = (double)sig_re[c] + II * omega * EPS0 * (double)eps_rel[c]; break;
      case 'D': {
        zc z = II * omega * (double)tau[c];
        zc zp = cpow(z, (zc)(double)cee[c]);
        sig[c] = (double)sig_re[c] * (1.0 - (double)eta[c] / (1.0 + zp));
        break;
      }
      case 'I': sig[c] = II * omega * EPS0 * (double)eps_rel[c]; break;
      default: return -1;
    }
  }
  return 0;
}

/* gen_k2_xgrid/_ygrid/_zgrid/_pgrid, src/aphid.f90:1289-1535 */
void orc_gen_k2(int nx, int ny, int nz, const double *dx, const double *dy,
                const double *dz, const orc_z *sig_, double omega, orc_z *k2_) {
  const layout_t L = mk_layout(nx, ny, nz);
  const zc *sig = (const zc *)sig_;
  zc *kx = (zc *)k2_ + L.ox, *ky = (zc *)k2_ + L.oy;
  zc *kz = (zc *)k2_ + L.oz, *kp = (zc *)k2_ + L.op;
  const int cx = nx - 1, cy = ny - 1;   /* sig is (nx-1,ny-1,nz-1) */
#define SIG(i, j, k) sig[F3(i, j, k, cx, cy)]
  const zc II = I;

  /* x-edges (nx-1,ny,nz), :1304-1336 */
  for (size_t t = 0; t < L.nxe; t++) kx[t] = (double)1.e30f;
  for (int i = 1; i <= nx - 1; i++)
    for (int j = 2; j <= ny - 1; j++)
      for (int k = 2; k <= nz - 1; k++) {
        double dyj = dy[j], dyjm = dy[j - 1], dzk = dz[k], dzkm = dz[k - 1];
        double c1 = dyjm * dzkm, c2 = dyj * dzkm, c3 = dyj * dzk, c4 = dyjm * dzk;
        zc s = SIG(i, j - 1, k - 1) * c1;
        s += SIG(i, j, k - 1) * c2;
        s += SIG(i, j, k) * c3;
        s += SIG(i, j - 1, k) * c4;
        kx[F3(i, j, k, nx - 1, ny)] = s / ((dyjm + dyj) * (dzkm + dzk));
      }
  for (int i = 1; i <= nx - 1; i++)
    for (int j = 2; j <= ny - 1; j++) {
      kx[F3(i, j, 1, nx - 1, ny)] = kx[F3(i, j, 2, nx - 1, ny)];
      kx[F3(i, j, nz, nx - 1, ny)] = kx[F3(i, j, nz - 1, nx - 1, ny)];
    }
  for (int i = 1; i <= nx - 1; i++)
    for (int k = 1; k <= nz; k++) {
      kx[F3(i, 1, k, nx - 1, ny)] = kx[F3(i, 2, k, nx - 1, ny)];
      kx[F3(i, ny, k, nx - 1, ny)] = kx[F3(i, ny - 1, k, nx - 1, ny)];
    }
  for (size_t t = 0; t < L.nxe; t++) kx[t] = kx[t] * II * omega * MU0;

  /* y-edges (nx,ny-1,nz), :1359-1389 */
  for (int i = 2; i <= nx - 1; i++)
    for (int j = 1; j <= ny - 1; j++)
      for (int k = 2; k <= nz - 1; k++) {
        double dxi = dx[i], dxim = dx[i - 1], dzk = dz[k], dzkm = dz[k - 1];
        double c1 = dxim * dzkm, c2 = dxi * dzkm, c3 = dxi * dzk, c4 = dxim * dzk;
        zc s = SIG(i - 1, j, k - 1) * c1;
        s += SIG(i, j, k - 1) * c2;
        s += SIG(i, j, k) * c3;
        s += SIG(i - 1, j, k) * c4;
        ky[F3(i, j, k, nx, ny - 1)] = s / ((dxim + dxi) * (dzkm + dzk));
      }
  for (int i = 2; i <= nx - 1; i++)
    for (int j = 1; j <= ny - 1; j++) {
      ky[F3(i, j, 1, nx, ny - 1)] = ky[F3(i, j, 2, nx, ny - 1)];
      ky[F3(i, j, nz, nx, ny - 1)] = ky[F3(i, j, nz - 1, nx, ny - 1)];
    }
  for (int j = 1; j <= ny - 1; j++)
    for (int k = 1; k <= nz; k++) {
      ky[F3(1, j, k, nx, ny - 1)] = ky[F3(2, j, k, nx, ny - 1)];
      ky[F3(nx, j, k, nx, ny - 1)] = ky[F3(nx - 1, j, k, nx, ny - 1)];
    }
  for (size_t t = 0; t < L.nye; t++) ky[t] = ky[t] * II * omega * MU0;

  /* z-edges (nx,ny,nz-1), :1412-1442 */
  for (int i = 2; i <= nx - 1; i++)
    for (int j = 2; j <= ny - 1; j++)
      for (int k = 1; k <= nz - 1; k++) {
        double dxi = dx[i], dxim = dx[i - 1], dyj = dy[j], dyjm = dy[j - 1];
        double c1 = dxim * dyjm, c2 = dxi * dyjm, c3 = dxi * dyj, c4 = dxim * dyj;
        zc s = SIG(i - 1, j - 1, k) * c1;
        s += SIG(i, j - 1, k) * c2;
        s += SIG(i, j, k) * c3;
        s += SIG(i - 1, j, k) * c4;
        kz[F3(i, j, k, nx, ny)] = s / ((dxim + dxi) * (dyjm + dyj));
      }
  for (int j = 2; j <= ny - 1; j++)
    for (int k = 1; k <= nz - 1; k++) {
      kz[F3(1, j, k, nx, ny)] = kz[F3(2, j, k, nx, ny)];
      kz[F3(nx, j, k, nx, ny)] = kz[F3(nx - 1, j, k, nx, ny)];
    }
  for (int i = 1; i <= nx; i++)
    for (int k = 1; k <= nz - 1; k++) {
      kz[F3(i, 1, k, nx, ny)] = kz[F3(i, 2, k, nx, ny)];
      kz[F3(i, ny, k, nx, ny)] = kz[F3(i, ny - 1, k, nx, ny)];
    }
  for (size_t t = 0; t < L.nze; t++) kz[t] = kz[t] * II * omega * MU0;

  /* nodes (nx,ny,nz), :1465-1533 */
#define KP(i, j, k) kp[F3(i, j, k, nx, ny)]
  for (int i = 2; i <= nx - 1; i++)
    for (int j = 2; j <= ny - 1; j++)
      for (int k = 2; k <= nz - 1; k++) {
        double dxi = dx[i], dxim = dx[i - 1], dyj = dy[j], dyjm = dy[j - 1];
        double dzk = dz[k], dzkm = dz[k - 1];
        double c[8] = {dxim * dyjm * dzk,  dxi * dyjm * dzk,  dxi * dyj * dzk,
                       dxim * dyj * dzk,   dxim * dyjm * dzkm, dxi * dyjm * dzkm,
                       dxi * dyj * dzkm,   dxim * dyj * dzkm};
        zc s = SIG(i - 1, j - 1, k) * c[0];
        s += SIG(i, j - 1, k) * c[1];
        s += SIG(i, j, k) * c[2];
        s += SIG(i - 1, j, k) * c[3];
        s += SIG(i - 1, j - 1, k - 1) * c[4];
        s += SIG(i, j - 1, k - 1) * c[5];
        s += SIG(i, j, k - 1) * c[6];
        s += SIG(i - 1, j, k - 1) * c[7];
        KP(i, j, k) = s / ((dxim + dxi) * (dyjm + dyj) * (dzkm + dzk));
      }
  for (int j = 2; j <= ny - 1; j++)
    for (int k = 2; k <= nz - 1; k++) {
      KP(1, j, k) = KP(2, j, k);
      KP(nx, j, k) = KP(nx - 1, j, k);
    }
  for (int i = 2; i <= nx - 1; i++)
    for (int k = 2; k <= nz - 1; k++) {
      KP(i, 1, k) = KP(i, 2, k);
      KP(i, ny, k) = KP(i, ny - 1, k);
    }
  for (int i = 2; i <= nx - 1; i++)
    for (int j = 2; j <= ny - 1; j++) {
      KP(i, j, 1) = KP(i, j, 2);
      KP(i, j, nz) = KP(i, j, nz - 1);
    }
  for (int k = 2; k <= nz - 1; k++) {
    KP(1, 1, k) = KP(2, 2, k);
    KP(1, ny, k) = KP(2, ny - 1, k);
    KP(nx, 1, k) = KP(nx - 1, 2, k);
    KP(nx, ny, k) = KP(nx - 1, ny - 1, k);
  }
  for (int i = 2; i <= nx - 1; i++) {
    KP(i, 1, 1) = KP(i, 2, 2);
    KP(i, ny, 1) = KP(i, ny - 1, 2);
    KP(i, 1, nz) = KP(i, 2, nz - 1);
    KP(i, ny, nz) = KP(i, ny - 1, nz - 1);
  }
  for (int j = 2; j <= ny - 1; j++) {
    KP(1, j, 1) = KP(2, j, 2);
    KP(nx, j, 1) = KP(nx - 1, j, 2);
    KP(1, j, nz) = KP(2, j, nz - 1);
    KP(nx, j, nz) = KP(nx - 1, j, nz - 1);
  }
  KP(1, 1, 1) = KP(2, 2, 2);
  KP(nx, 1, 1) = KP(nx - 1, 2, 2);
  KP(1, ny, 1) = KP(2, ny - 1, 2);
  KP(nx, ny, 1) = KP(nx - 1, ny - 1, 2);
  KP(1, 1, nz) = KP(2, 2, nz - 1);
  KP(nx, 1, nz) = KP(nx - 1, 2, nz - 1);
  KP(1, ny, nz) = KP(2, ny - 1, nz - 1);
  KP(nx, ny, nz) = KP(nx - 1, ny - 1, nz - 1);
  for (size_t t = 0; t < L.np; t++) kp[t] = kp[t] * II * omega * MU0;
#undef KP
#undef SIG
}

/* Fortran integer masks used by the coefficient tables:
 * (i/n - 1) and ((n-i)/(n-1) - 1) with integer division. */
static inline double mask_hi(int i, int n) { return (double)(i / n - 1); }
static inline double mask_lo(int i, int n) { return (double)((n - i) / (n - 1) - 1); }

/* gen_diag, src/aphid.f90:1542-1725 */
void orc_gen_diag(int nx, int ny, int nz, const double *dx, const double *dy,
                  const double *dz, const orc_z *k2_, orc_z *diag_) {
  const layout_t L = mk_layout(nx, ny, nz);
  const zc *k2 = (const zc *)k2_;
  zc *diag = (zc *)diag_;
  for (size_t t = 0; t < L.n; t++) diag[t] = 1.0;
  const zc *kx = k2 + L.ox, *ky = k2 + L.oy, *kz = k2 + L.oz, *kp = k2 + L.op;
  zc *gx = diag + L.ox, *gy = diag + L.oy, *gz = diag + L.oz, *gp = diag + L.op;

  /* x-edges, :1571-1604 */
  for (int k = 1; k <= nz; k++) {
    double dzk = dz[k], dzkm = dz[k - 1], dzck = 0.5 * (dzk + dzkm);
    zc c6 = mask_hi(k, nz) / dzk / dzck;
    zc c7 = mask_lo(k, nz) / dzkm / dzck;
    for (int j = 1; j <= ny; j++) {
      double dyj = dy[j], dyjm = dy[j - 1], dycj = 0.5 * (dyj + dyjm);
      zc c4 = mask_hi(j, ny) / dyj / dycj;
      zc c5 = mask_lo(j, ny) / dyjm / dycj;
      for (int i = 1; i <= nx - 1; i++) {
        double dxip = dx[i + 1], dxi = dx[i], dxim = dx[i - 1];
        double dxcip = 0.5 * (dxi + dxip), dxci = 0.5 * (dxi + dxim);
        double vol = dxi * dycj * dzck;
        zc c2 = mask_hi(i, nx - 1) / dxcip / dxi;
        zc c3 = mask_lo(i, nx) / dxci / dxi;
        zc sum = c2 + c3 + c4 + c5 + c6 + c7;
        gx[F3(i, j, k, nx - 1, ny)] = (-sum + kx[F3(i, j, k, nx - 1, ny)]) * vol;
      }
    }
  }
  /* y-edges, :1609-1642 */
  for (int k = 1; k <= nz; k++) {
    double dzk = dz[k], dzkm = dz[k - 1], dzck = 0.5 * (dzk + dzkm);
    zc c6 = mask_hi(k, nz) / dzk / dzck;
    zc c7 = mask_lo(k, nz) / dzkm / dzck;
    for (int j = 1; j <= ny - 1; j++) {
      double dyjp = dy[j + 1], dyj = dy[j], dyjm = dy[j - 1];
      double dycjp = 0.5 * (dyj + dyjp), dycj = 0.5 * (dyj + dyjm);
      zc c2 = mask_hi(j, ny - 1) / dycjp / dyj;
      zc c3 = mask_lo(j, ny) / dycj / dyj;
      for (int i = 1; i <= nx; i++) {
        double dxi = dx[i], dxim = dx[i - 1], dxci = 0.5 * (dxi + dxim);
        double vol = dxci * dyj * dzck;
        zc c4 = mask_hi(i, nx) / dxi / dxci;
        zc c5 = mask_lo(i, nx) / dxim / dxci;
        zc sum = c2 + c3 + c4 + c5 + c6 + c7;
        gy[F3(i, j, k, nx, ny - 1)] = (-sum + ky[F3(i, j, k, nx, ny - 1)]) * vol;
      }
    }
  }
  /* z-edges, :1647-1679 */
  for (int k = 1; k <= nz - 1; k++) {
    double dzkp = dz[k + 1], dzk = dz[k], dzkm = dz[k - 1];
    double dzckp = 0.5 * (dzk + dzkp), dzck = 0.5 * (dzk + dzkm);
    zc c2 = mask_hi(k, nz - 1) / dzckp / dzk;
    zc c3 = mask_lo(k, nz) / dzck / dzk;
    for (int j = 1; j <= ny; j++) {
      double dyj = dy[j], dyjm = dy[j - 1], dycj = 0.5 * (dyj + dyjm);
      zc c6 = mask_hi(j, ny) / dyj / dycj;
      zc c7 = mask_lo(j, ny) / dyjm / dycj;
      for (int i = 1; i <= nx; i++) {
        double dxi = dx[i], dxim = dx[i - 1], dxci = 0.5 * (dxi + dxim);
        double vol = dxci * dycj * dzk;
        zc c4 = mask_hi(i, nx) / dxi / dxci;
        zc c5 = mask_lo(i, nx) / dxim / dxci;
        zc sum = c2 + c3 + c4 + c5 + c6 + c7;
        gz[F3(i, j, k, nx, ny)] = (-sum + kz[F3(i, j, k, nx, ny)]) * vol;
      }
    }
  }
  /* nodes, interior only, :1684-1723 */
  for (int k = 2; k <= nz - 1; k++) {
    double dzk = dz[k], dzkm = dz[k - 1], dzck = 0.5 * (dzk + dzkm);
    for (int j = 2; j <= ny - 1; j++) {
      double dyj = dy[j], dyjm = dy[j - 1], dycj = 0.5 * (dyj + dyjm);
      for (int i = 2; i <= nx - 1; i++) {
        double dxi = dx[i], dxim = dx[i - 1], dxci = 0.5 * (dxi + dxim);
        double vol = dxci * dycj * dzck;
        zc k2 = kp[F3(i, j, k, nx, ny)];
        zc s2 = kx[F3(i < nx - 1 ? i : nx - 1, j, k, nx - 1, ny)];
        zc s3 = kx[F3(i - 1 > 1 ? i - 1 : 1, j, k, nx - 1, ny)];
        zc s4 = ky[F3(i, j < ny - 1 ? j : ny - 1, k, nx, ny - 1)];
        zc s5 = ky[F3(i, j - 1 > 1 ? j - 1 : 1, k, nx, ny - 1)];
        zc s6 = kz[F3(i, j, k < nz - 1 ? k : nz - 1, nx, ny)];
        zc s7 = kz[F3(i, j, k - 1 > 1 ? k - 1 : 1, nx, ny)];
        zc c2 = mask_hi(i, nx) * s2 / dxi / dxci;
        zc c3 = mask_lo(i, nx) * s3 / dxim / dxci;
        zc c4 = mask_hi(j, ny) * s4 / dyj / dycj;
        zc c5 = mask_lo(j, ny) * s5 / dyjm / dycj;
        zc c6 = mask_hi(k, nz) * s6 / dzk / dzck;
        zc c7 = mask_lo(k, nz) * s7 / dzkm / dzck;
        zc sum = c2 + c3 + c4 + c5 + c6 + c7;
        gp[F3(i, j, k, nx, ny)] = (-sum + k2 * k2) * vol;
      }
    }
  }
}

/* ---------------------------------------------------------------------- */
/* operator: coefficient tables (gen_inprod_*_coefs) and stencils           */
/* ---------------------------------------------------------------------- */

typedef struct {
  layout_t L;
  const double *dx, *dy, *dz, *dxc, *dyc, *dzc;
  /* per-axis tables, 1-based index stored at [i] (entry 0 unused) */
  double *xe2, *xe3, *xn4, *xn5;   /* x-axis: edge (len nx-1) and node (len nx) */
  double *ye2, *ye3, *yn4, *yn5;
  double *ze2, *ze3, *zn4, *zn5;
  const zc *k2;
  double *buf;
} op_t;

/* Edge-type coefficients (coef_2vec/coef_3vec of the component along an
 * axis, e.g. src/aphid.f90:787-795) and node-type coefficients (coef_4..7
 * of the transverse components and of the node block, e.g. :777-785,
 * :1152-1161; the node block uses the same formula on 2..n-1). */
static void axis_tables(int n, const double *d, const double *dc, double *e2,
                        double *e3, double *n4, double *n5) {
  for (int i = 1; i <= n - 1; i++) {
    e2[i] = mask_hi(i, n - 1) / dc[i] / d[i];       /* /dxc(i+1)/dx(i) */
    e3[i] = mask_lo(i, n) / dc[i - 1] / d[i];   /* /dxc(i)/dx(i)   */
  }
  for (int i = 1; i <= n; i++) {
    n4[i] = mask_hi(i, n) / d[i] / dc[i - 1];       /* /dx(i)/dxc(i)   */
    n5[i] = mask_lo(i, n) / d[i - 1] / dc[i - 1];   /* /dx(i-1)/dxc(i) */
  }
}

static void op_init(op_t *o, int nx, int ny, int nz, const double *dx,
                    const double *dy, const double *dz, const double *dxc,
                    const double *dyc, const double *dzc, const zc *k2) {
  o->L = mk_layout(nx, ny, nz);
  o->dx = dx; o->dy = dy; o->dz = dz; o->dxc = dxc; o->dyc = dyc; o->dzc = dzc;
  o->k2 = k2;
  size_t tot = 4 * (size_t)(nx + 1) + 4 * (size_t)(ny + 1) + 4 * (size_t)(nz + 1);
  o->buf = (double *)calloc(tot, sizeof(double));
  double *b = o->buf;
  o->xe2 = b; b += nx + 1; o->xe3 = b; b += nx + 1; o->xn4 = b; b += nx + 1; o->xn5 = b; b += nx + 1;
  o->ye2 = b; b += ny + 1; o->ye3 = b; b += ny + 1; o->yn4 = b; b += ny + 1; o->yn5 = b; b += ny + 1;
  o->ze2 = b; b += nz + 1; o->ze3 = b; b += nz + 1; o->zn4 = b; b += nz + 1; o->zn5 = b; b += nz + 1;
  axis_tables(nx, dx, dxc, o->xe2, o->xe3, o->xn4, o->xn5);
  axis_tables(ny, dy, dyc, o->ye2, o->ye3, o->yn4, o->yn5);
  axis_tables(nz, dz, dzc, o->ze2, o->ze3, o->zn4, o->zn5);
}

static void op_free(op_t *o) { free(o->buf); }

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* inprod_x, src/aphid.f90:803-871 */
static void op_x(const op_t *o, const zc *in, zc *out) {
  const int nx = o->L.nx, ny = o->L.ny, nz = o->L.nz;
  const zc *ax = in + o->L.ox, *ph = in + o->L.op;
  const zc *kx = o->k2 + o->L.ox, *kp = o->k2 + o->L.op;
  for (int k = 1; k <= nz; k++) {
    double dzck = o->dzc[k - 1];
    zc c6 = o->zn4[k], c7 = o->zn5[k];
    int ka = imin(k + 1, nz), kb = imax(1, k - 1);
    for (int j = 1; j <= ny; j++) {
      double dycj = o->dyc[j - 1];
      zc c4 = o->yn4[j], c5 = o->yn5[j];
      int ja = imin(j + 1, ny), jb = imax(1, j - 1);
      for (int i = 1; i <= nx - 1; i++) {
        double dxi = o->dx[i];
        zc c2 = o->xe2[i], c3 = o->xe3[i];
        int ia = imin(i + 1, nx - 1), ib = imax(1, i - 1);
        double vol = dxi * dycj * dzck;
        zc k2 = kx[F3(i, j, k, nx - 1, ny)];
        zc kp1 = kp[F3(i, j, k, nx, ny)], kp2 = kp[F3(i + 1, j, k, nx, ny)];
        zc c1 = -(c2 + c3 + c4 + c5 + c6 + c7) + k2;
        zc s = c1 * ax[F3(i, j, k, nx - 1, ny)];
        s += c2 * ax[F3(ia, j, k, nx - 1, ny)];
        s += c3 * ax[F3(ib, j, k, nx - 1, ny)];
        s += c4 * ax[F3(i, ja, k, nx - 1, ny)];
        s += c5 * ax[F3(i, jb, k, nx - 1, ny)];
        s += c6 * ax[F3(i, j, ka, nx - 1, ny)];
        s += c7 * ax[F3(i, j, kb, nx - 1, ny)];
        out[F3(i, j, k, nx - 1, ny)] =
            (s + (ph[F3(i + 1, j, k, nx, ny)] * (kp2 - k2) -
                  ph[F3(i, j, k, nx, ny)] * (kp1 - k2)) / dxi) * vol;
      }
    }
  }
}

/* inprod_y, src/aphid.f90:932-1000 */
static void op_y(const op_t *o, const zc *in, zc *out) {
  const int nx = o->L.nx, ny = o->L.ny, nz = o->L.nz;
  const zc *ay = in + o->L.oy, *ph = in + o->L.op;
  const zc *ky = o->k2 + o->L.oy, *kp = o->k2 + o->L.op;
  for (int k = 1; k <= nz; k++) {
    double dzck = o->dzc[k - 1];
    int ka = imin(k + 1, nz), kb = imax(1, k - 1);
    zc c6 = o->zn4[k], c7 = o->zn5[k];
    for (int j = 1; j <= ny - 1; j++) {
      double dyj = o->dy[j];
      int ja = imin(j + 1, ny - 1), jb = imax(1, j - 1);
      zc c2 = o->ye2[j], c3 = o->ye3[j];
      for (int i = 1; i <= nx; i++) {
        double dxci = o->dxc[i - 1];
        int ia = imin(i + 1, nx), ib = imax(1, i - 1);
        zc c4 = o->xn4[i], c5 = o->xn5[i];
        double vol = dxci * dyj * dzck;
        zc k2 = ky[F3(i, j, k, nx, ny - 1)];
        zc kp1 = kp[F3(i, j, k, nx, ny)], kp2 = kp[F3(i, j + 1, k, nx, ny)];
        zc c1 = -(c2 + c3 + c4 + c5 + c6 + c7) + k2;
        zc s = c1 * ay[F3(i, j, k, nx, ny - 1)];
        s += c2 * ay[F3(i, ja, k, nx, ny - 1)];
        s += c3 * ay[F3(i, jb, k, nx, ny - 1)];
        s += c4 * ay[F3(ia, j, k, nx, ny - 1)];
        s += c5 * ay[F3(ib, j, k, nx, ny - 1)];
        s += c6 * ay[F3(i, j, ka, nx, ny - 1)];
        s += c7 * ay[F3(i, j, kb, nx, ny - 1)];
        out[F3(i, j, k, nx, ny - 1)] =
            (s + (ph[F3(i, j + 1, k, nx, ny)] * (kp2 - k2) -
                  ph[F3(i, j, k, nx, ny)] * (kp1 - k2)) / dyj) * vol;
      }
    }
  }
}

/* inprod_z, src/aphid.f90:1061-1128 */
static void op_z(const op_t *o, const zc *in, zc *out) {
  const int nx = o->L.nx, ny = o->L.ny, nz = o->L.nz;
  const zc *az = in + o->L.oz, *ph = in + o->L.op;
  const zc *kz = o->k2 + o->L.oz, *kp = o->k2 + o->L.op;
  for (int k = 1; k <= nz - 1; k++) {
    double dzk = o->dz[k];
    int ka = imin(k + 1, nz - 1), kb = imax(1, k - 1);
    zc c2 = o->ze2[k], c3 = o->ze3[k];
    for (int j = 1; j <= ny; j++) {
      double dycj = o->dyc[j - 1];
      int ja = imin(j + 1, ny), jb = imax(1, j - 1);
      zc c6 = o->yn4[j], c7 = o->yn5[j];
      for (int i = 1; i <= nx; i++) {
        double dxci = o->dxc[i - 1];
        int ia = imin(i + 1, nx), ib = imax(1, i - 1);
        zc c4 = o->xn4[i], c5 = o->xn5[i];
        double vol = dxci * dycj * dzk;
        zc k2 = kz[F3(i, j, k, nx, ny)];
        zc kp1 = kp[F3(i, j, k, nx, ny)], kp2 = kp[F3(i, j, k + 1, nx, ny)];
        zc c1 = -(c2 + c3 + c4 + c5 + c6 + c7) + k2;
        zc s = c1 * az[F3(i, j, k, nx, ny)];
        s += c2 * az[F3(i, j, ka, nx, ny)];
        s += c3 * az[F3(i, j, kb, nx, ny)];
        s += c4 * az[F3(ia, j, k, nx, ny)];
        s += c5 * az[F3(ib, j, k, nx, ny)];
        s += c6 * az[F3(i, ja, k, nx, ny)];
        s += c7 * az[F3(i, jb, k, nx, ny)];
        out[F3(i, j, k, nx, ny)] =
            (s + (ph[F3(i, j, k + 1, nx, ny)] * (kp2 - k2) -
                  ph[F3(i, j, k, nx, ny)] * (kp1 - k2)) / dzk) * vol;
      }
    }
  }
}

/* inprod_p, src/aphid.f90:1191-1282 (boundary nodes give 0) */
static void op_p(const op_t *o, const zc *in, zc *out) {
  const int nx = o->L.nx, ny = o->L.ny, nz = o->L.nz;
  const zc *ax = in + o->L.ox, *ay = in + o->L.oy, *az = in + o->L.oz, *ph = in + o->L.op;
  const zc *kx = o->k2 + o->L.ox, *ky = o->k2 + o->L.oy, *kz = o->k2 + o->L.oz,
           *kp = o->k2 + o->L.op;
  for (size_t t = 0; t < o->L.np; t++) out[t] = 0.0;
  for (int k = 2; k <= nz - 1; k++) {
    double dzck = o->dzc[k - 1];
    int ka = imin(k + 1, nz), kb = imax(1, k - 1), kc = imin(k, nz - 1);
    for (int j = 2; j <= ny - 1; j++) {
      double dycj = o->dyc[j - 1];
      int ja = imin(j + 1, ny), jb = imax(1, j - 1), jc = imin(j, ny - 1);
      for (int i = 2; i <= nx - 1; i++) {
        double dxci = o->dxc[i - 1];
        int ia = imin(i + 1, nx), ib = imax(1, i - 1), ic = imin(i, nx - 1);
        double vol = dxci * dycj * dzck;
        zc k2 = kp[F3(i, j, k, nx, ny)];
        zc s1 = kp[F3(i, j, k, nx, ny)];
        zc s2 = kx[F3(ic, j, k, nx - 1, ny)];
        zc s3 = kx[F3(ib, j, k, nx - 1, ny)];
        zc s4 = ky[F3(i, jc, k, nx, ny - 1)];
        zc s5 = ky[F3(i, jb, k, nx, ny - 1)];
        zc s6 = kz[F3(i, j, kc, nx, ny)];
        zc s7 = kz[F3(i, j, kb, nx, ny)];
        zc c2 = o->xn4[i] * s2, c3 = o->xn5[i] * s3;
        zc c4 = o->yn4[j] * s4, c5 = o->yn5[j] * s5;
        zc c6 = o->zn4[k] * s6, c7 = o->zn5[k] * s7;
        zc c1 = -(c2 + c3 + c4 + c5 + c6 + c7) + k2 * k2;
        zc s = c1 * ph[F3(i, j, k, nx, ny)];
        s += c2 * ph[F3(ia, j, k, nx, ny)];
        s += c3 * ph[F3(ib, j, k, nx, ny)];
        s += c4 * ph[F3(i, ja, k, nx, ny)];
        s += c5 * ph[F3(i, jb, k, nx, ny)];
        s += c6 * ph[F3(i, j, ka, nx, ny)];
        s += c7 * ph[F3(i, j, kb, nx, ny)];
        zc acc = s * vol;
        zc d2 = (s2 - s1) / dxci, d3 = -(s3 - s1) / dxci;
        zc d4 = (s4 - s1) / dycj, d5 = -(s5 - s1) / dycj;
        zc d6 = (s6 - s1) / dzck, d7 = -(s7 - s1) / dzck;
        zc t = d2 * ax[F3(ic, j, k, nx - 1, ny)];
        t += d3 * ax[F3(ib, j, k, nx - 1, ny)];
        t += d4 * ay[F3(i, jc, k, nx, ny - 1)];
        t += d5 * ay[F3(i, jb, k, nx, ny - 1)];
        t += d6 * az[F3(i, j, kc, nx, ny)];
        t += d7 * az[F3(i, j, kb, nx, ny)];
        out[F3(i, j, k, nx, ny)] = acc + t * vol;
      }
    }
  }
}

static void op_apply(const op_t *o, const zc *in, zc *out) {
  op_x(o, in, out + o->L.ox);
  op_y(o, in, out + o->L.oy);
  op_z(o, in, out + o->L.oz);
  op_p(o, in, out + o->L.op);
}

void orc_inprod(int nx, int ny, int nz, const double *dx, const double *dy,
                const double *dz, const double *dxc, const double *dyc,
                const double *dzc, const orc_z *k2, const orc_z *x, orc_z *y) {
  op_t o;
  op_init(&o, nx, ny, nz, dx, dy, dz, dxc, dyc, dzc, (const zc *)k2);
  op_apply(&o, (const zc *)x, (zc *)y);
  op_free(&o);
}

/* gen_rhs, src/aphid.f90:534-743 */
int orc_gen_rhs(int mode, int nx, int ny, int nz, const double *xn,
                const double *yn, const double *zn, const double *dx,
                const double *dy, const double *dz, int ndip, const char *dirs,
                const int *ijk, orc_z *rhs_, int *nskipped) {
  const layout_t L = mk_layout(nx, ny, nz);
  zc *rhs = (zc *)rhs_;
  zc *rx = rhs + L.ox, *ry = rhs + L.oy, *rz = rhs + L.oz, *rp = rhs + L.op;
  for (size_t t = 0; t < L.n; t++) rhs[t] = 0.0;
  if (nskipped) *nskipped = 0;
#define RX(i, j, k) rx[F3(i, j, k, nx - 1, ny)]
#define RY(i, j, k) ry[F3(i, j, k, nx, ny - 1)]
#define RZ(i, j, k) rz[F3(i, j, k, nx, ny)]
#define RP(i, j, k) rp[F3(i, j, k, nx, ny)]
  if (mode == 1) {  /* :566-587; last node within 1e-4 (real(4)) of 0 */
    const double tol = (double)1.e-4f;
    int ip = -1, jp = -1, kp = -1;
    for (int k = 1; k <= nz; k++) {
      if (fabs(zn[k - 1] - 0.) < tol) kp = k;
      for (int j = 1; j <= ny; j++) {
        if (fabs(yn[j - 1] - 0.) < tol) jp = j;
        for (int i = 1; i <= nx; i++)
          if (fabs(xn[i - 1] - 0.) < tol) ip = i;
      }
    }
    if (ip < 1 || jp < 1 || kp < 1 || ip > nx - 1) return -1;
    RX(ip, jp, kp) = 1.0 * MU0;
    RP(ip, jp, kp) = 1.0 * MU0 / dx[ip];
    RP(ip + 1, jp, kp) = -1.0 * MU0 / dx[ip];
  } else if (mode == 2) {  /* :592-604 */
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx - 1; i++) RX(i, j, 2) = 1.0 * MU0;
    for (int i = 1; i <= nx - 1; i++)
      for (int j = 1; j <= ny; j++) RX(i, j, 2) = RX(i, j, 2) * dx[i];
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx - 1; i++) RX(i, j, 2) = RX(i, j, 2) * (0.5 * (dy[j - 1] + dy[j]));
  } else if (mode == 3) {  /* :608-620 */
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++) RY(i, j, 2) = 1.0 * MU0;
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++) RY(i, j, 2) = RY(i, j, 2) * dy[j];
    for (int i = 1; i <= nx; i++)
      for (int j = 1; j <= ny - 1; j++) RY(i, j, 2) = RY(i, j, 2) * (0.5 * (dx[i - 1] + dx[i]));
  } else if (mode == 4) {  /* :624-631, fixed 40x40 loop centred at (51,51,51) */
    const int n = 20;
    if (nx < 51 + n || ny < 51 + n || nz < 51) return -1;
    for (int i = 51 - n; i <= 51 + n - 1; i++) {
      RX(i, 51 + n, 51) = 1.0 * MU0 * dx[i];
      RX(i, 51 - n, 51) = -1.0 * MU0 * dx[i];
    }
    for (int j = 51 - n; j <= 51 + n - 1; j++) {
      RY(51 - n, j, 51) = 1.0 * MU0 * dy[j];
      RY(51 + n, j, 51) = -1.0 * MU0 * dy[j];
    }
  } else if (mode == 5) {  /* :638-741 */
    for (int d = 0; d < ndip; d++) {
      char s0 = dirs[2 * d], s1 = dirs[2 * d + 1];
      int ip = ijk[3 * d], jp = ijk[3 * d + 1], kp = ijk[3 * d + 2];
      int ok = 0;
      if ((s0 == '+' || s0 == '-') && (s1 == 'X' || s1 == 'Y' || s1 == 'Z')) {
        if (s0 == '+' && s1 == 'X') {
          if (!(ip < 1 || ip > nx - 1 || jp < 1 || jp > ny || kp < 1 || kp > nz)) {
            RX(ip, jp, kp) = RX(ip, jp, kp) + 1.0 * MU0 * dx[ip];
            RP(ip, jp, kp) = RP(ip, jp, kp) + 1.0 * MU0;
            RP(ip + 1, jp, kp) = RP(ip + 1, jp, kp) - 1.0 * MU0;
            ok = 1;
          }
        } else if (s0 == '-' && s1 == 'X') {
          if (!(ip < 2 || ip > nx || jp < 1 || jp > ny || kp < 1 || kp > nz)) {
            RX(ip - 1, jp, kp) = RX(ip - 1, jp, kp) - 1.0 * MU0 * dx[ip - 1];
            RP(ip - 1, jp, kp) = RP(ip - 1, jp, kp) - 1.0 * MU0;
            RP(ip, jp, kp) = RP(ip, jp, kp) + 1.0 * MU0;
            ok = 1;
          }
        } else if (s0 == '+' && s1 == 'Y') {
          if (!(ip < 1 || ip > nx || jp < 1 || jp > ny - 1 || kp < 1 || kp > nz)) {
            RY(ip, jp, kp) = RY(ip, jp, kp) + 1.0 * MU0 * dy[jp];
            RP(ip, jp, kp) = RP(ip, jp, kp) + 1.0 * MU0;
            RP(ip, jp + 1, kp) = RP(ip, jp + 1, kp) - 1.0 * MU0;
            ok = 1;
          }
        } else if (s0 == '-' && s1 == 'Y') {
          if (!(ip < 1 || ip > nx || jp < 2 || jp > ny || kp < 1 || kp > nz)) {
            RY(ip, jp - 1, kp) = RY(ip, jp - 1, kp) - 1.0 * MU0 * dy[jp - 1];
            RP(ip, jp - 1, kp) = RP(ip, jp - 1, kp) - 1.0 * MU0;
            RP(ip, jp, kp) = RP(ip, jp, kp) + 1.0 * MU0;
            ok = 1;
          }
        } else if (s0 == '+' && s1 == 'Z') {
          if (!(ip < 1 || ip > nx || jp < 1 || jp > ny || kp < 1 || kp > nz - 1)) {
            RZ(ip, jp, kp) = RZ(ip, jp, kp) + 1.0 * MU0 * dz[kp];
            RP(ip, jp, kp) = RP(ip, jp, kp) + 1.0 * MU0;
            RP(ip, jp, kp + 1) = RP(ip, jp, kp + 1) - 1.0 * MU0;
            ok = 1;
          }
        } else {  /* -Z */
          if (!(ip < 1 || ip > nx || jp < 1 || jp > ny || kp < 2 || kp > nz)) {
            RZ(ip, jp, kp - 1) = RZ(ip, jp, kp - 1) - 1.0 * MU0 * dz[kp - 1];
            RP(ip, jp, kp - 1) = RP(ip, jp, kp - 1) - 1.0 * MU0;
            RP(ip, jp, kp) = RP(ip, jp, kp) + 1.0 * MU0;
            ok = 1;
          }
        }
      }
      if (!ok && nskipped) (*nskipped)++;
    }
  } else {
    return -1;
  }
#undef RX
#undef RY
#undef RZ
#undef RP
  return 0;
}

/* ---------------------------------------------------------------------- */
/* QMR, src/aphid_qmr.f90:5-434 (nthreads=4: :744-928 component split)      */
/* ---------------------------------------------------------------------- */

/* block b of a concat vector: [lo, hi) */
static void blk(const layout_t *L, int b, size_t *lo, size_t *hi) {
  size_t o[5] = {L->ox, L->oy, L->oz, L->op, L->n};
  *lo = o[b];
  *hi = o[b + 1];
}

/* sum(a*b) over one block, sequential */
static zc bdot(const zc *a, const zc *b, size_t lo, size_t hi) {
  zc s = 0.0;
  for (size_t t = lo; t < hi; t++) s += a[t] * b[t];
  return s;
}
/* sum(a*conjg(a)) over one block, sequential */
static zc bnrm2(const zc *a, size_t lo, size_t hi) {
  zc s = 0.0;
  for (size_t t = lo; t < hi; t++) s += a[t] * conj(a[t]);
  return s;
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void op_apply_block(const op_t *o, int b, const zc *in, zc *out) {
  switch (b) {
    case 0: op_x(o, in, out + o->L.ox); break;
    case 1: op_y(o, in, out + o->L.oy); break;
    case 2: op_z(o, in, out + o->L.oz); break;
    default: op_p(o, in, out + o->L.op); break;
  }
}

int orc_qmr(int nx, int ny, int nz, const double *dx, const double *dy,
            const double *dz, const double *dxc, const double *dyc,
            const double *dzc, const orc_z *k2_, const orc_z *diag_,
            orc_z *rhs_, const orc_z *x0_, double target, int max_it,
            int nthreads, double *hist, int hist_cap, double *rnorm_out,
            double *rhsnorm_out, int *converged, double *seconds) {
  const layout_t L = mk_layout(nx, ny, nz);
  const size_t n = L.n;
  const zc *diag = (const zc *)diag_;
  zc *x = (zc *)rhs_;
  op_t o;
  op_init(&o, nx, ny, nz, dx, dy, dz, dxc, dyc, dzc, (const zc *)k2_);

  zc *W = (zc *)malloc(8 * n * sizeof(zc));
  zc *inv = W, *tmp = W + n, *r = W + 2 * n, *s = W + 3 * n;
  zc *p = W + 4 * n, *d = W + 5 * n, *vt = W + 6 * n, *v = W + 7 * n;
  int nt = (nthreads == 4) ? 4 : 1;

  double t1 = now_s();
  /* :169-172 */
  zc rn = 0.0;
  for (int b = 0; b < 4; b++) {
    size_t lo, hi;
    blk(&L, b, &lo, &hi);
    rn += bnrm2(x, lo, hi);
  }
  double rhsnorm = sqrt(creal(rn));
  /* :178-181 */
  for (size_t t = 0; t < n; t++) inv[t] = 1.0 / diag[t];
  /* :211-233 */
  for (size_t t = 0; t < n; t++) {
    p[t] = 0.0;
    d[t] = 0.0;
    s[t] = x[t];
    x[t] = x0_ ? ((const zc *)x0_)[t] : 0.0;
  }
  /* :245-263 */
  op_apply(&o, x, tmp);
  for (size_t t = 0; t < n; t++) {
    vt[t] = s[t] - tmp[t];
    r[t] = s[t] - tmp[t];
  }
  zc rr = 0.0;
  for (int b = 0; b < 4; b++) {
    size_t lo, hi;
    blk(&L, b, &lo, &hi);
    rr += bnrm2(r, lo, hi);
  }
  double rho_np = sqrt(creal(rr));
  /* :268-285 */
  for (size_t t = 0; t < n; t++) {
    v[t] = vt[t] / rho_np;
    s[t] = 0.0;
  }
  double c_n = 1.0, theta_n = 0.0, c_nm, rho_n, theta_nm, k2s, rnorm = 0.0;
  zc eps = 1.0, eta = -1.0, del, k1, beta;
  int conv = 0, iter = 1, nh = 0;
  zc part[4];
  double partr[4];

  for (;;) {
    /* :299-302 */
    c_nm = c_n;
    rho_n = rho_np;
    theta_nm = theta_n;
    /* step 1, :306-313 */
#pragma omp parallel for num_threads(nt) schedule(static, 1) if (nt > 1)
    for (int b = 0; b < 4; b++) {
      size_t lo, hi;
      blk(&L, b, &lo, &hi);
      for (size_t t = lo; t < hi; t++) tmp[t] = v[t] * inv[t];
      part[b] = bdot(v, tmp, lo, hi);
    }
    del = part[0] + part[1] + part[2] + part[3];
    k1 = rho_n * del / eps;
    /* step 2, :317-320 */
#pragma omp parallel for num_threads(nt) schedule(static, 1) if (nt > 1)
    for (int b = 0; b < 4; b++) {
      size_t lo, hi;
      blk(&L, b, &lo, &hi);
      for (size_t t = lo; t < hi; t++) p[t] = tmp[t] - p[t] * k1;
    }
    /* step 3, :324-338 */
#pragma omp parallel for num_threads(nt) schedule(static, 1) if (nt > 1)
    for (int b = 0; b < 4; b++) {
      size_t lo, hi;
      blk(&L, b, &lo, &hi);
      op_apply_block(&o, b, p, tmp);
      part[b] = bdot(p, tmp, lo, hi);
    }
    eps = part[0] + part[1] + part[2] + part[3];
    beta = eps / del;
#pragma omp parallel for num_threads(nt) schedule(static, 1) if (nt > 1)
    for (int b = 0; b < 4; b++) {
      size_t lo, hi;
      blk(&L, b, &lo, &hi);
      for (size_t t = lo; t < hi; t++) vt[t] = tmp[t] - v[t] * beta;
      partr[b] = creal(bnrm2(vt, lo, hi));
    }
    rho_np = sqrt(partr[0] + partr[1] + partr[2] + partr[3]);
    /* step 4, :342-345 */
    theta_n = rho_np * rho_np / c_nm / (creal(beta) * creal(beta) + cimag(beta) * cimag(beta));
    c_n = 1.0 / (1.0 + theta_n);
    eta = -eta * rho_n * c_n / (beta * c_nm);
    k2s = theta_nm * c_n;
    /* :347-372 */
#pragma omp parallel for num_threads(nt) schedule(static, 1) if (nt > 1)
    for (int b = 0; b < 4; b++) {
      size_t lo, hi;
      blk(&L, b, &lo, &hi);
      for (size_t t = lo; t < hi; t++) {
        d[t] = p[t] * eta + d[t] * k2s;
        x[t] = x[t] + d[t];
        s[t] = tmp[t] * eta + s[t] * k2s;
        r[t] = r[t] - s[t];
        v[t] = vt[t] / rho_np;
      }
      partr[b] = creal(bnrm2(r, lo, hi));
    }
    rnorm = sqrt(partr[0] + partr[1] + partr[2] + partr[3]);
    if (hist && nh < hist_cap) hist[nh] = rnorm;
    nh++;
    /* :386-390 */
    if (rnorm < target * rhsnorm) conv = 1;
    if (!conv && iter <= max_it) iter++;
    if (!(!conv && iter <= max_it)) break;
  }
  double t2 = now_s();
  if (rnorm_out) *rnorm_out = rnorm;
  if (rhsnorm_out) *rhsnorm_out = rhsnorm;
  if (converged) *converged = conv;
  if (seconds) *seconds = t2 - t1;
  free(W);
  op_free(&o);
  return iter;
}

/* gen_fields, src/aphid.f90:2173-2252 */
void orc_gen_fields(int nx, int ny, int nz, const double *dx, const double *dy,
                    const double *dz, double omega, const orc_z *sol_,
                    orc_z *B_, orc_z *E_) {
  const layout_t L = mk_layout(nx, ny, nz);
  const zc *sol = (const zc *)sol_;
  const zc *ax = sol + L.ox, *ay = sol + L.oy, *az = sol + L.oz, *ph = sol + L.op;
  zc *B = (zc *)B_, *E = (zc *)E_;
  const size_t nbx = (size_t)nx * (ny - 1) * (nz - 1);
  const size_t nby = (size_t)(nx - 1) * ny * (nz - 1);
  zc *bx = B, *by = B + nbx, *bz = B + nbx + nby;
  zc *ex = E + L.ox, *ey = E + L.oy, *ez = E + L.oz;
  const zc II = I;
#define AX(i, j, k) ax[F3(i, j, k, nx - 1, ny)]
#define AY(i, j, k) ay[F3(i, j, k, nx, ny - 1)]
#define AZ(i, j, k) az[F3(i, j, k, nx, ny)]
#define PH(i, j, k) ph[F3(i, j, k, nx, ny)]
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++)
        bx[F3(i, j, k, nx, ny - 1)] = AZ(i, j + 1, k) / dy[j] - AY(i, j, k + 1) / dz[k] -
                                      AZ(i, j, k) / dy[j] + AY(i, j, k) / dz[k];
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx - 1; i++)
        by[F3(i, j, k, nx - 1, ny)] = AX(i, j, k + 1) / dz[k] - AZ(i + 1, j, k) / dx[i] -
                                      AX(i, j, k) / dz[k] + AZ(i, j, k) / dx[i];
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++)
        bz[F3(i, j, k, nx - 1, ny - 1)] = AY(i + 1, j, k) / dx[i] - AX(i, j + 1, k) / dy[j] -
                                          AY(i, j, k) / dx[i] + AX(i, j, k) / dy[j];
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx - 1; i++)
        ex[F3(i, j, k, nx - 1, ny)] =
            -(II * omega * (AX(i, j, k) - (PH(i + 1, j, k) - PH(i, j, k)) / dx[i]));
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++)
        ey[F3(i, j, k, nx, ny - 1)] =
            -(II * omega * (AY(i, j, k) - (PH(i, j + 1, k) - PH(i, j, k)) / dy[j]));
  for (int k = 1; k <= nz - 1; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++)
        ez[F3(i, j, k, nx, ny)] =
            -(II * omega * (AZ(i, j, k) - (PH(i, j, k + 1) - PH(i, j, k)) / dz[k]));
#undef AX
#undef AY
#undef AZ
#undef PH
}

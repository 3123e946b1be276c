/*
 * ocfd_oracle.c -- CPU oracle (test infrastructure) for the OpenCFD-SC RHS and
 * RK3 time advance: a single-rank C restatement of the reference's Fortran.
 *
 * Every routine cites the reference routine it restates (paths relative to the
 * OpenCFD-SC source tree) and keeps that routine's operation order, so that a
 * build with -ffp-contract=off reproduces the reference's double-precision
 * arithmetic operation by operation.  Parity against a reference binary is
 * unpinned (no Fortran compiler or MPI is available); see ocfd_oracle.h.
 *
 * Used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 */
#include "ocfd_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define LAP 4
#define DEL_NONE 0
#define DEL_LIFT 1
#define DEL_RIGHT 2

struct pwork {
  double *pc, *pd, *pu, *pv, *pw, *pa1, *pa2, *pa3;
  double *pfp[5], *pfm[5];
  double *ph1, *ph2, *phh[5];
  int* scm;
};

struct ocfd_oracle {
  ocfd_params p;
  int nx, ny, nz, nxh, nyh, nzh;
  size_t n, nh;
  double *f, *fn, *du, *amu;
  double *d, *u, *v, *w, *T;
  double *met[OCFD_N_METRICS];
  double *rhybrid;
  double *cc;
  double *ev[3];  /* Ev1..Ev3, each 4 haloed arrays */
  double *g[12];  /* uk ui us vk vi vs wk wi ws Tk Ti Ts (interior) */
  /* pencil work arrays (OCFD_inviscous.f90:6-12), one set per OpenMP thread */
  int npen, nthreads;
  struct pwork* pw;
  int istep;
  double tt;
  /* BC_BoundaryLayer / BC_SweptCorner data (BC_data, OCFD_BC_Boundarylayers.f90:3-15) */
  double *bl_inlet, *bl_upper, *bl_pertb, *bl_tm, *bl_fait;
  int *bl_dirichlet;
  int bl_mt;
  double bl_beta;
};

/* ---------------------------------------------------------------- indexing */
static inline size_t IH(const ocfd_oracle* o, int i, int j, int k) {
  return (size_t)(i + LAP - 1) + (size_t)o->nxh * ((size_t)(j + LAP - 1) + (size_t)o->nyh * (size_t)(k + LAP - 1));
}
static inline size_t I3(const ocfd_oracle* o, int i, int j, int k) {
  return (size_t)(i - 1) + (size_t)o->nx * ((size_t)(j - 1) + (size_t)o->ny * (size_t)(k - 1));
}
static inline size_t IF(const ocfd_oracle* o, int i, int j, int k, int m) {
  return I3(o, i, j, k) + o->n * (size_t)(m - 1);
}
static inline double sq(double x) { return x * x; }
static inline double fsign1(double b) { return copysign(1.0, b); }
static inline double fmin2(double a, double b) { return a < b ? a : b; }
static inline double fmax2(double a, double b) { return a > b ? a : b; }
static inline double fmin3(double a, double b, double c) { return fmin2(fmin2(a, b), c); }
static inline double fmax3(double a, double b, double c) { return fmax2(fmax2(a, b), c); }

/* ---------------------------------------------------------------- parameters */
/* Namelist defaults: OCFD_readpara.f90:28-65 */
void orc_default_params(ocfd_params* p) {
  memset(p, 0, sizeof(*p));
  p->gamma = 1.4;
  p->re = 100.0;
  p->ma = 1.0;
  p->pr = 0.7;
  p->lap = 4;
  p->scheme_invis = OCFD_SCHEME_WENO5;
  p->scheme_vis = OCFD_SCHEME_CD6;
  p->ref_amu_t0 = 288.15;
  p->dt = 1.0e-4;
  p->end_time = 100.0;
  p->iflag_gridtype = OCFD_GRID3D;
  p->ibc = OCFD_BC_NONE;
  p->istep_show = 1;
  p->istep_save = 1000;
  p->if_viscous = 1;
  p->ud7l_diss = 1.0;
  for (int i = 0; i < 100; i++) p->hybrid_para[i] = 1.0;
  p->flux_splitting = OCFD_SPLIT_SW;
}

/* set_parameters + set_scheme_para for one rank: OCFD_readpara.f90:261-341 */
int orc_set_parameters(ocfd_params* p) {
  p->hx = 1.0 / (p->nx - 1.0);
  p->hy = 1.0 / (p->ny - 1.0);
  p->hz = 1.0 / (p->nz - 1.0);
  p->cv = 1.0 / (p->gamma * (p->gamma - 1.0) * p->ma * p->ma);
  p->cp = p->cv * p->gamma;
  for (int d = 0; d < 3; d++) {
    p->bound_index[2 * d] = p->iperiodic[d] == 0 ? 1 : 0;
    p->bound_index[2 * d + 1] = p->iperiodic[d] == 0 ? 1 : 0;
  }
  switch (p->scheme_invis) {
    case OCFD_SCHEME_WENO5: p->ka1 = -2; p->kb1 = 2; p->ka2 = -1; p->kb2 = 3; break;
    case OCFD_SCHEME_WENO7: p->ka1 = -3; p->kb1 = 3; p->ka2 = -2; p->kb2 = 4; break;
    case OCFD_SCHEME_OMP6:
    case OCFD_SCHEME_UD7L:
    case OCFD_SCHEME_HYBRID: p->ka1 = -3; p->kb1 = 4; p->ka2 = -3; p->kb2 = 4; break;
    default: return -1;
  }
  {
    const double UD7[8] = {-3.0, 25.0, -101.0, 319.0, 214.0, -38.0, 4.0, 0.0};
    const double CD8[8] = {-3.0, 29.0, -139.0, 533.0, 533.0, -139.0, 29.0, -3.0};
    for (int k = 0; k < 8; k++)
      p->ud7l[k] = p->ud7l_diss * UD7[k] / 420.0 + (1.0 - p->ud7l_diss) * CD8[k] / 840.0;
  }
  return 0;
}

/* ---------------------------------------------------------------- schemes
 * Point forms of OCFD_Schemes_1.f90; v points at the stencil's centre v(0).
 * The array forms of OCFD_Schemes.f90 perform the same operations per face. */

/* hh_weno5P: OCFD_Schemes_1.f90:9-29 (= OCFD_weno5P, OCFD_Schemes.f90:6-28) */
static double hh_weno5P(const double* v) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double S0 = 13.0 / 12.0 * sq(v[0] - 2.0 * v[1] + v[2]) + 1.0 / 4.0 * sq(3.0 * v[0] - 4.0 * v[1] + v[2]);
  double S1 = 13.0 / 12.0 * sq(v[-1] - 2.0 * v[0] + v[1]) + 1.0 / 4.0 * sq(v[-1] - v[1]);
  double S2 = 13.0 / 12.0 * sq(v[-2] - 2.0 * v[-1] + v[0]) + 1.0 / 4.0 * sq(v[-2] - 4.0 * v[-1] + 3.0 * v[0]);
  double a0 = C03 / sq(ep + S0);
  double a1 = C13 / sq(ep + S1);
  double a2 = C23 / sq(ep + S2);
  double am = a0 + a1 + a2;
  double q03 = 1.0 / 3.0 * v[0] + 5.0 / 6.0 * v[1] - 1.0 / 6.0 * v[2];
  double q13 = -1.0 / 6.0 * v[-1] + 5.0 / 6.0 * v[0] + 1.0 / 3.0 * v[1];
  double q23 = 1.0 / 3.0 * v[-2] - 7.0 / 6.0 * v[-1] + 11.0 / 6.0 * v[0];
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

/* hh_weno5M: OCFD_Schemes_1.f90:31-52 (= OCFD_weno5M, OCFD_Schemes.f90:30-53) */
static double hh_weno5M(const double* v) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double S0 = 13.0 / 12.0 * sq(v[1] - 2.0 * v[0] + v[-1]) + 1.0 / 4.0 * sq(3.0 * v[1] - 4.0 * v[0] + v[-1]);
  double S1 = 13.0 / 12.0 * sq(v[2] - 2.0 * v[1] + v[0]) + 1.0 / 4.0 * sq(v[2] - v[0]);
  double S2 = 13.0 / 12.0 * sq(v[3] - 2.0 * v[2] + v[1]) + 1.0 / 4.0 * sq(v[3] - 4.0 * v[2] + 3.0 * v[1]);
  double a0 = C03 / sq(ep + S0);
  double a1 = C13 / sq(ep + S1);
  double a2 = C23 / sq(ep + S2);
  double am = a0 + a1 + a2;
  double q03 = 1.0 / 3.0 * v[1] + 5.0 / 6.0 * v[0] - 1.0 / 6.0 * v[-1];
  double q13 = -1.0 / 6.0 * v[2] + 5.0 / 6.0 * v[1] + 1.0 / 3.0 * v[0];
  double q23 = 1.0 / 3.0 * v[3] - 7.0 / 6.0 * v[2] + 11.0 / 6.0 * v[1];
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

/* WENO7 coefficients: OCFD_Schemes_1.f90:65-79 */
#define W7_COEFFS                                                                                          \
  const double C0 = 1.0 / 35.0, C1 = 12.0 / 35.0, C2 = 18.0 / 35.0, C3 = 4.0 / 35.0;                      \
  const double a11 = -2.0 / 6.0, a12 = 9.0 / 6.0, a13 = -18.0 / 6.0, a14 = 11.0 / 6.0;                    \
  const double a21 = 1.0 / 6.0, a23 = 3.0 / 6.0, a24 = 2.0 / 6.0;                                        \
  const double a31 = -2.0 / 6.0, a32 = -3.0 / 6.0, a34 = -1.0 / 6.0;                                      \
  const double a41 = -11.0 / 6.0, a42 = 18.0 / 6.0, a43 = -9.0 / 6.0, a44 = 2.0 / 6.0;                    \
  const double b12 = 4.0, b13 = -5.0, b14 = 2.0, b22 = -2.0, b41 = 2.0, b42 = -5.0, b43 = 4.0, c12 = 3.0; \
  const double d12 = 13.0 / 12.0, d13 = 1043.0 / 960.0, d14 = 1.0 / 12.0;                                 \
  const double e11 = -3.0 / 12.0, e12 = 13.0 / 12.0, e13 = -23.0 / 12.0, e14 = 25.0 / 12.0;               \
  const double e21 = 1.0 / 12.0, e22 = -5.0 / 12.0, e23 = 13.0 / 12.0, e24 = 3.0 / 12.0;                  \
  const double e31 = -1.0 / 12.0, e32 = 7.0 / 12.0, e33 = 7.0 / 12.0, e34 = -1.0 / 12.0;                  \
  const double e41 = 3.0 / 12.0, e42 = 13.0 / 12.0, e43 = -5.0 / 12.0, e44 = 1.0 / 12.0;                  \
  const double ep = 1.0e-8

/* hh_weno7P: OCFD_Schemes_1.f90:58-121 (= OCFD_weno7P, OCFD_Schemes.f90:59-124) */
static double hh_weno7P(const double* v) {
  W7_COEFFS;
  double S10 = a11 * v[-3] + a12 * v[-2] + a13 * v[-1] + a14 * v[0];
  double S11 = a21 * v[-2] - v[-1] + a23 * v[0] + a24 * v[1];
  double S12 = a31 * v[-1] + a32 * v[0] + v[1] + a34 * v[2];
  double S13 = a41 * v[0] + a42 * v[1] + a43 * v[2] + a44 * v[3];
  double S20 = -v[-3] + b12 * v[-2] + b13 * v[-1] + b14 * v[0];
  double S21 = v[-1] + b22 * v[0] + v[1];
  double S22 = v[0] + b22 * v[1] + v[2];
  double S23 = b41 * v[0] + b42 * v[1] + b43 * v[2] - v[3];
  double S30 = -v[-3] + c12 * (v[-2] - v[-1]) + v[0];
  double S31 = -v[-2] + c12 * (v[-1] - v[0]) + v[1];
  double S32 = -v[-1] + c12 * (v[0] - v[1]) + v[2];
  double S33 = -v[0] + c12 * (v[1] - v[2]) + v[3];
  double S0 = S10 * S10 + d12 * S20 * S20 + d13 * S30 * S30 + d14 * S10 * S30;
  double S1 = S11 * S11 + d12 * S21 * S21 + d13 * S31 * S31 + d14 * S11 * S31;
  double S2 = S12 * S12 + d12 * S22 * S22 + d13 * S32 * S32 + d14 * S12 * S32;
  double S3 = S13 * S13 + d12 * S23 * S23 + d13 * S33 * S33 + d14 * S13 * S33;
  double a0 = C0 / sq(ep + S0);
  double a1 = C1 / sq(ep + S1);
  double a2 = C2 / sq(ep + S2);
  double a3 = C3 / sq(ep + S3);
  double am = a0 + a1 + a2 + a3;
  double q0 = e11 * v[-3] + e12 * v[-2] + e13 * v[-1] + e14 * v[0];
  double q1 = e21 * v[-2] + e22 * v[-1] + e23 * v[0] + e24 * v[1];
  double q2 = e31 * v[-1] + e32 * v[0] + e33 * v[1] + e34 * v[2];
  double q3 = e41 * v[0] + e42 * v[1] + e43 * v[2] + e44 * v[3];
  return (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / am;
}

/* hh_weno7M: OCFD_Schemes_1.f90:124-187 (= OCFD_weno7M, OCFD_Schemes.f90:127-193) */
static double hh_weno7M(const double* v) {
  W7_COEFFS;
  double S10 = a11 * v[4] + a12 * v[3] + a13 * v[2] + a14 * v[1];
  double S11 = a21 * v[3] - v[2] + a23 * v[1] + a24 * v[0];
  double S12 = a31 * v[2] + a32 * v[1] + v[0] + a34 * v[-1];
  double S13 = a41 * v[1] + a42 * v[0] + a43 * v[-1] + a44 * v[-2];
  double S20 = -v[4] + b12 * v[3] + b13 * v[2] + b14 * v[1];
  double S21 = v[2] + b22 * v[1] + v[0];
  double S22 = v[1] + b22 * v[0] + v[-1];
  double S23 = b41 * v[1] + b42 * v[0] + b43 * v[-1] - v[-2];
  double S30 = -v[4] + c12 * (v[3] - v[2]) + v[1];
  double S31 = -v[3] + c12 * (v[2] - v[1]) + v[0];
  double S32 = -v[2] + c12 * (v[1] - v[0]) + v[-1];
  double S33 = -v[1] + c12 * (v[0] - v[-1]) + v[-2];
  double S0 = S10 * S10 + d12 * S20 * S20 + d13 * S30 * S30 + d14 * S10 * S30;
  double S1 = S11 * S11 + d12 * S21 * S21 + d13 * S31 * S31 + d14 * S11 * S31;
  double S2 = S12 * S12 + d12 * S22 * S22 + d13 * S32 * S32 + d14 * S12 * S32;
  double S3 = S13 * S13 + d12 * S23 * S23 + d13 * S33 * S33 + d14 * S13 * S33;
  double a0 = C0 / sq(ep + S0);
  double a1 = C1 / sq(ep + S1);
  double a2 = C2 / sq(ep + S2);
  double a3 = C3 / sq(ep + S3);
  double am = a0 + a1 + a2 + a3;
  double q0 = e11 * v[4] + e12 * v[3] + e13 * v[2] + e14 * v[1];
  double q1 = e21 * v[3] + e22 * v[2] + e23 * v[1] + e24 * v[0];
  double q2 = e31 * v[2] + e32 * v[1] + e33 * v[0] + e34 * v[-1];
  double q3 = e41 * v[1] + e42 * v[0] + e43 * v[-1] + e44 * v[-2];
  return (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / am;
}

/* minmod2 / minmod4: OCFD_Schemes.f90:274-289 */
static double minmod2(double x1, double x2) {
  return 0.5 * (fsign1(x1) + fsign1(x2)) * fmin2(fabs(x1), fabs(x2));
}
static double minmod4(double x1, double x2, double x3, double x4) {
  double r = 0.5 * (fsign1(x1) + fsign1(x2));
  r = r * fabs(0.5 * (fsign1(x1) + fsign1(x3)));
  r = r * fabs(0.5 * (fsign1(x1) + fsign1(x4)));
  r = r * fmin2(fmin2(fmin2(fabs(x1), fabs(x2)), fabs(x3)), fabs(x4));
  return r;
}

/* OMP6 constants: OCFD_Schemes_1.f90:203-209.  ep is the single-precision
 * literal 1.e-10 of the reference, widened to double. */
typedef struct { double a1, a2, a3, a4, a5, a6, a7, a8, kappa, ep; } omp6_c;
static omp6_c omp6_consts(void) {
  omp6_c c;
  const double OMP_m = 0.015, OMP_n = 0.0;
  const double OMP_a = 0.5 * (OMP_m + OMP_n), OMP_b = 0.5 * (OMP_m - OMP_n);
  c.a1 = OMP_a;
  c.a2 = 1.0 / 60.0 - OMP_b - 6.0 * OMP_a;
  c.a3 = -2.0 / 15.0 + 6.0 * OMP_b + 15.0 * OMP_a;
  c.a4 = 37.0 / 60.0 - 15.0 * OMP_b - 20.0 * OMP_a;
  c.a5 = 37.0 / 60.0 + 20.0 * OMP_b + 15.0 * OMP_a;
  c.a6 = -2.0 / 15.0 - 6.0 * OMP_a - 15.0 * OMP_b;
  c.a7 = 1.0 / 60.0 + OMP_a + 6.0 * OMP_b;
  c.a8 = -OMP_b;
  c.kappa = 4.0;
  c.ep = (double)1.e-10f;
  return c;
}

/* hh_OMP6P: OCFD_Schemes_1.f90:195-226 (= OCFD_OMP6P, OCFD_Schemes.f90:201-234) */
static double hh_omp6P(const double* v) {
  const omp6_c c = omp6_consts();
  double mid_nf = c.a1 * v[4] + c.a2 * v[3] + c.a3 * v[2] + c.a4 * v[1] + c.a5 * v[0] + c.a6 * v[-1] +
                  c.a7 * v[-2] + c.a8 * v[-3];
  double mp = v[0] + minmod2((v[1] - v[0]), c.kappa * (v[0] - v[-1]));
  if ((mid_nf - v[0]) * (mid_nf - mp) >= c.ep) {
    double d1 = v[-2] + v[0] - 2.0 * v[-1];
    double d2 = v[-1] + v[1] - 2.0 * v[0];
    double d3 = v[0] + v[2] - 2.0 * v[1];
    double ul = v[0] + c.kappa * (v[0] - v[-1]);
    double md = 0.5 * (v[0] + v[1]) - 0.5 * minmod4(4.0 * d2 - d3, 4.0 * d3 - d2, d2, d3);
    double lc = v[0] + 0.5 * (v[0] - v[-1]) + c.kappa * minmod4(4.0 * d1 - d2, 4.0 * d2 - d1, d2, d1) / 3.0;
    double fmin = fmax2(fmin3(v[0], v[1], md), fmin3(v[0], ul, lc));
    double fmax = fmin2(fmax3(v[0], v[1], md), fmax3(v[0], ul, lc));
    mid_nf = mid_nf + minmod2(fmax - mid_nf, fmin - mid_nf);
  }
  return mid_nf;
}

/* hh_OMP6M: OCFD_Schemes_1.f90:228-260 (= OCFD_OMP6M, OCFD_Schemes.f90:236-271) */
static double hh_omp6M(const double* v) {
  const omp6_c c = omp6_consts();
  double mid_nf = c.a1 * v[-3] + c.a2 * v[-2] + c.a3 * v[-1] + c.a4 * v[0] + c.a5 * v[1] + c.a6 * v[2] +
                  c.a7 * v[3] + c.a8 * v[4];
  double mp = v[1] + minmod2((v[0] - v[1]), c.kappa * (v[1] - v[2]));
  if ((mid_nf - v[1]) * (mid_nf - mp) >= c.ep) {
    double d1 = v[3] + v[1] - 2.0 * v[2];
    double d2 = v[2] + v[0] - 2.0 * v[1];
    double d3 = v[1] + v[-1] - 2.0 * v[0];
    double ul = v[1] + c.kappa * (v[1] - v[2]);
    double md = 0.5 * (v[1] + v[0]) - 0.5 * minmod4(4.0 * d2 - d3, 4.0 * d3 - d2, d2, d3);
    double lc = v[1] + 0.5 * (v[1] - v[0]) + c.kappa * minmod4(4.0 * d1 - d2, 4.0 * d2 - d1, d2, d1) / 3.0;
    double fmin = fmax2(fmin3(v[1], v[0], md), fmin3(v[1], ul, lc));
    double fmax = fmin2(fmax3(v[1], v[0], md), fmax3(v[1], ul, lc));
    mid_nf = mid_nf + minmod2(fmax - mid_nf, fmin - mid_nf);
  }
  return mid_nf;
}

/* hh_weno5P_boundary: OCFD_Schemes_1.f90:266-295 */
static double hh_weno5P_boundary(const double* v, int del) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double a0 = 0.0, q03 = 0.0, a2 = 0.0, q23 = 0.0;
  if (del != DEL_RIGHT) {
    double S0 = 13.0 / 12.0 * sq(v[0] - 2.0 * v[1] + v[2]) + 1.0 / 4.0 * sq(3.0 * v[0] - 4.0 * v[1] + v[2]);
    a0 = C03 / sq(ep + S0);
    q03 = 1.0 / 3.0 * v[0] + 5.0 / 6.0 * v[1] - 1.0 / 6.0 * v[2];
  }
  double S1 = 13.0 / 12.0 * sq(v[-1] - 2.0 * v[0] + v[1]) + 1.0 / 4.0 * sq(v[-1] - v[1]);
  double a1 = C13 / sq(ep + S1);
  double q13 = -1.0 / 6.0 * v[-1] + 5.0 / 6.0 * v[0] + 1.0 / 3.0 * v[1];
  if (del != DEL_LIFT) {
    double S2 = 13.0 / 12.0 * sq(v[-2] - 2.0 * v[-1] + v[0]) + 1.0 / 4.0 * sq(v[-2] - 4.0 * v[-1] + 3.0 * v[0]);
    a2 = C23 / sq(ep + S2);
    q23 = 1.0 / 3.0 * v[-2] - 7.0 / 6.0 * v[-1] + 11.0 / 6.0 * v[0];
  }
  double am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

/* hh_weno5M_boundary: OCFD_Schemes_1.f90:297-325 */
static double hh_weno5M_boundary(const double* v, int del) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double a0 = 0.0, q03 = 0.0, a2 = 0.0, q23 = 0.0;
  if (del != DEL_LIFT) {
    double S0 = 13.0 / 12.0 * sq(v[1] - 2.0 * v[0] + v[-1]) + 1.0 / 4.0 * sq(3.0 * v[1] - 4.0 * v[0] + v[-1]);
    a0 = C03 / sq(ep + S0);
    q03 = 1.0 / 3.0 * v[1] + 5.0 / 6.0 * v[0] - 1.0 / 6.0 * v[-1];
  }
  double S1 = 13.0 / 12.0 * sq(v[2] - 2.0 * v[1] + v[0]) + 1.0 / 4.0 * sq(v[2] - v[0]);
  double a1 = C13 / sq(ep + S1);
  double q13 = -1.0 / 6.0 * v[2] + 5.0 / 6.0 * v[1] + 1.0 / 3.0 * v[0];
  if (del != DEL_RIGHT) {
    double S2 = 13.0 / 12.0 * sq(v[3] - 2.0 * v[2] + v[1]) + 1.0 / 4.0 * sq(v[3] - 4.0 * v[2] + 3.0 * v[1]);
    a2 = C23 / sq(ep + S2);
    q23 = 1.0 / 3.0 * v[3] - 7.0 / 6.0 * v[2] + 11.0 / 6.0 * v[1];
  }
  double am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

/* hh_UD7L_P / _M: OCFD_Schemes_1.f90:328-348 (= OCFD_UD7L_P/M, OCFD_Schemes.f90:292-316) */
static double hh_ud7lP(const double* U, const double* v) {
  return U[0] * v[-3] + U[1] * v[-2] + U[2] * v[-1] + U[3] * v[0] + U[4] * v[1] + U[5] * v[2] + U[6] * v[3] +
         U[7] * v[4];
}
static double hh_ud7lM(const double* U, const double* v) {
  return U[0] * v[4] + U[1] * v[3] + U[2] * v[2] + U[3] * v[1] + U[4] * v[0] + U[5] * v[-1] + U[6] * v[-2] +
         U[7] * v[-3];
}

/* Interior scheme dispatch for F+ (OCFD2d_flux1 select, OCFD_inviscous.f90:230-244;
 * hybrid: OCFD_HybridP, OCFD_Schemes.f90:319-337 / hh_HybridP, OCFD_Schemes_1.f90:351-365) */
static double scheme_P(const ocfd_params* p, const double* v, int ihy) {
  switch (p->scheme_invis) {
    case OCFD_SCHEME_OMP6: return hh_omp6P(v);
    case OCFD_SCHEME_WENO7: return hh_weno7P(v);
    case OCFD_SCHEME_WENO5: return hh_weno5P(v);
    case OCFD_SCHEME_UD7L: return hh_ud7lP(p->ud7l, v);
    case OCFD_SCHEME_HYBRID:
      if (ihy == 1) return hh_ud7lP(p->ud7l, v);
      if (ihy == 2) return hh_weno7P(v);
      return hh_weno5P(v);
  }
  return 0.0;
}
/* ... and for F- (OCFD_inviscous.f90:307-320; OCFD_HybridM, OCFD_Schemes.f90:339-358) */
static double scheme_M(const ocfd_params* p, const double* v, int ihy) {
  switch (p->scheme_invis) {
    case OCFD_SCHEME_OMP6: return hh_omp6M(v);
    case OCFD_SCHEME_WENO7: return hh_weno7M(v);
    case OCFD_SCHEME_WENO5: return hh_weno5M(v);
    case OCFD_SCHEME_UD7L: return hh_ud7lM(p->ud7l, v);
    case OCFD_SCHEME_HYBRID:
      if (ihy == 1) return hh_ud7lM(p->ud7l, v);
      if (ihy == 2) return hh_weno7M(v);
      return hh_weno5M(v);
  }
  return 0.0;
}

/* OCFD2d_flux1: OCFD_inviscous.f90:210-283.  f1d[i] valid for 1-LAP..n+LAP. */
static void ocfd2d_flux1(const ocfd_params* p, const double* f1d, double* hh, int n, const int* bi,
                         const int* scm, const int* sb) {
  int Ka = p->ka1, Kb = p->kb1, ib, ie, i;
  ib = (bi[0] == 0 || sb[0] == -1) ? 0 : -Ka + 1;
  ie = (bi[1] == 0 || sb[1] == -1) ? n : n - Kb;
  for (i = ib; i <= ie; i++) hh[i] = scheme_P(p, f1d + i, scm[i]);
  if (bi[0] == 1) {
    if (sb[0] == 0) {
      for (i = 0; i <= -Ka; i++) {
        if (i == 0 || i == 1)
          hh[i] = (2.0 * f1d[1] + 5.0 * f1d[2] - f1d[3]) / 6.0;
        else if (i == 2)
          hh[i] = hh_weno5P_boundary(f1d + i, DEL_LIFT);
        else
          hh[i] = hh_weno5P(f1d + i);
      }
    } else if (sb[0] == 1) {
      for (i = 0; i <= -Ka; i++) hh[i] = hh_weno5P(f1d + i);
    }
  }
  if (bi[1] == 1) {
    if (sb[1] == 0) {
      for (i = n - Kb + 1; i <= n; i++) {
        if (i == n)
          hh[i] = (2.0 * f1d[n - 2] - 7.0 * f1d[n - 1] + 11.0 * f1d[n]) / 6.0;
        else if (i == n - 1)
          hh[i] = hh_weno5P_boundary(f1d + i, DEL_RIGHT);
        else
          hh[i] = hh_weno5P(f1d + i);
      }
    } else if (sb[1] == 1) {
      for (i = n - Kb + 1; i <= n; i++) hh[i] = hh_weno5P(f1d + i);
    }
  }
}

/* OCFD2d_flux2: OCFD_inviscous.f90:287-361 */
static void ocfd2d_flux2(const ocfd_params* p, const double* f1d, double* hh, int n, const int* bi,
                         const int* scm, const int* sb) {
  int Ka = p->ka2, Kb = p->kb2, ib, ie, i;
  ib = (bi[0] == 0 || sb[0] == -1) ? 0 : -Ka + 1;
  ie = (bi[1] == 0 || sb[1] == -1) ? n : n - Kb;
  for (i = ib; i <= ie; i++) hh[i] = scheme_M(p, f1d + i, scm[i]);
  if (bi[0] == 1) {
    if (sb[0] == 0) {
      for (i = 0; i <= -Ka; i++) {
        if (i == 0)
          hh[i] = (2.0 * f1d[3] - 7.0 * f1d[2] + 11.0 * f1d[1]) / 6.0;
        else if (i == 1)
          hh[i] = hh_weno5M_boundary(f1d + i, DEL_LIFT);
        else
          hh[i] = hh_weno5M(f1d + i);
      }
    } else if (sb[0] == 1) {
      for (i = 0; i <= -Ka; i++) hh[i] = hh_weno5M(f1d + i);
    }
  }
  if (bi[1] == 1) {
    if (sb[1] == 0) {
      for (i = n - Kb + 1; i <= n; i++) {
        if (i == n || i == n - 1)
          hh[i] = (2.0 * f1d[n] + 5.0 * f1d[n - 1] - f1d[n - 2]) / 6.0;
        else if (i == n - 2)
          hh[i] = hh_weno5M_boundary(f1d + i, DEL_RIGHT);
        else
          hh[i] = hh_weno5M(f1d + i);
      }
    } else if (sb[1] == 1) {
      for (i = n - Kb + 1; i <= n; i++) hh[i] = hh_weno5M(f1d + i);
    }
  }
}

/* ---------------------------------------------------------------- splitting */
/* split_Stager_Warming: OCFD_flux_split.f90:5-70 (the P2 term is dropped as in :51-60) */
static void split_sw(const ocfd_params* p, int n, const double* c1, const double* d1, const double* u1,
                     const double* v1, const double* w1, const double* A1, const double* A2, const double* A3,
                     double* const* fp, double* const* fm) {
  double g = p->gamma;
  double tmp1 = 2.0 * (g - 1.0);
  double tmp3 = (3.0 - g) / (2.0 * (g - 1.0));
  for (int i = 1 - LAP; i <= n + LAP; i++) {
    double ss = sqrt(A1[i] * A1[i] + A2[i] * A2[i] + A3[i] * A3[i]);
    double ss1 = 1.0 / ss;
    double ak1 = A1[i] * ss1, ak2 = A2[i] * ss1, ak3 = A3[i] * ss1;
    double vs = A1[i] * u1[i] + A2[i] * v1[i] + A3[i] * w1[i];
    double E1 = vs, E2 = vs - c1[i] * ss, E3 = vs + c1[i] * ss;
    double E1P = (E1 + fabs(E1)) * 0.5, E2P = (E2 + fabs(E2)) * 0.5, E3P = (E3 + fabs(E3)) * 0.5;
    double E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    double tmp0 = d1[i] / (2.0 * g);
    double uc1 = u1[i] - c1[i] * ak1, uc2 = u1[i] + c1[i] * ak1;
    double vc1 = v1[i] - c1[i] * ak2, vc2 = v1[i] + c1[i] * ak2;
    double wc1 = w1[i] - c1[i] * ak3, wc2 = w1[i] + c1[i] * ak3;
    double vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.5;
    double vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.5;
    double vv = (g - 1.0) * (u1[i] * u1[i] + v1[i] * v1[i] + w1[i] * w1[i]);
    double W2 = tmp3 * c1[i] * c1[i];
    fp[0][i] = tmp0 * (tmp1 * E1P + E2P + E3P);
    fp[1][i] = tmp0 * (tmp1 * E1P * u1[i] + E2P * uc1 + E3P * uc2);
    fp[2][i] = tmp0 * (tmp1 * E1P * v1[i] + E2P * vc1 + E3P * vc2);
    fp[3][i] = tmp0 * (tmp1 * E1P * w1[i] + E2P * wc1 + E3P * wc2);
    fp[4][i] = tmp0 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
    fm[0][i] = tmp0 * (tmp1 * E1M + E2M + E3M);
    fm[1][i] = tmp0 * (tmp1 * E1M * u1[i] + E2M * uc1 + E3M * uc2);
    fm[2][i] = tmp0 * (tmp1 * E1M * v1[i] + E2M * vc1 + E3M * vc2);
    fm[3][i] = tmp0 * (tmp1 * E1M * w1[i] + E2M * wc1 + E3M * wc2);
    fm[4][i] = tmp0 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
  }
}

/* split_Local_LaxFriedrichs: OCFD_flux_split.f90:73-104 */
static void split_llf(const ocfd_params* p, int n, const double* c1, const double* d1, const double* u1,
                      const double* v1, const double* w1, const double* A1, const double* A2, const double* A3,
                      double* const* fp, double* const* fm) {
  double tmp0 = 1.0 / p->gamma;
  double tmp1 = 1.0 / (p->gamma - 1.0);
  for (int i = 1 - LAP; i <= n + LAP; i++) {
    double ss = sqrt(A1[i] * A1[i] + A2[i] * A2[i] + A3[i] * A3[i]);
    double un = A1[i] * u1[i] + A2[i] * v1[i] + A3[i] * w1[i];
    double lamda0 = fabs(un) + ss * c1[i];
    double p1 = tmp0 * d1[i] * c1[i] * c1[i];
    double E0 = tmp1 * p1 + 0.5 * d1[i] * (u1[i] * u1[i] + v1[i] * v1[i] + w1[i] * w1[i]);
    double h0 = E0 + p1;
    fp[0][i] = 0.5 * (d1[i] * un + lamda0 * d1[i]);
    fp[1][i] = 0.5 * (d1[i] * u1[i] * un + A1[i] * p1 + lamda0 * d1[i] * u1[i]);
    fp[2][i] = 0.5 * (d1[i] * v1[i] * un + A2[i] * p1 + lamda0 * d1[i] * v1[i]);
    fp[3][i] = 0.5 * (d1[i] * w1[i] * un + A3[i] * p1 + lamda0 * d1[i] * w1[i]);
    fp[4][i] = 0.5 * (h0 * un + lamda0 * E0);
    fm[0][i] = 0.5 * (d1[i] * un - lamda0 * d1[i]);
    fm[1][i] = 0.5 * (d1[i] * u1[i] * un + A1[i] * p1 - lamda0 * d1[i] * u1[i]);
    fm[2][i] = 0.5 * (d1[i] * v1[i] * un + A2[i] * p1 - lamda0 * d1[i] * v1[i]);
    fm[3][i] = 0.5 * (d1[i] * w1[i] * un + A3[i] * p1 - lamda0 * d1[i] * w1[i]);
    fm[4][i] = 0.5 * (h0 * un - lamda0 * E0);
  }
}

/* ---------------------------------------------------------------- lifetime */
static double* alloc_fill(size_t n, double v) {
  double* a = (double*)malloc(n * sizeof(double));
  for (size_t i = 0; i < n; i++) a[i] = v;
  return a;
}

/* allocate_flow_data / allocate_inviscous_data / allocate_vicous_data:
 * OCFD_NS_Solver.f90:93-151, OCFD_inviscous.f90:15-40, OCFD_viscous.f90:16-25 */
ocfd_oracle* orc_create(const ocfd_params* p) {
  ocfd_oracle* o = (ocfd_oracle*)calloc(1, sizeof(ocfd_oracle));
  o->p = *p;
  o->nx = p->nx; o->ny = p->ny; o->nz = p->nz;
  o->nxh = o->nx + 2 * LAP; o->nyh = o->ny + 2 * LAP; o->nzh = o->nz + 2 * LAP;
  o->n = (size_t)o->nx * o->ny * o->nz;
  o->nh = (size_t)o->nxh * o->nyh * o->nzh;
  o->f = alloc_fill(5 * o->n, 0.0);
  o->fn = alloc_fill(5 * o->n, 0.0);
  o->du = alloc_fill(5 * o->n, 0.0);
  o->amu = alloc_fill(o->n, 0.0);
  o->d = alloc_fill(o->nh, 1.0); o->u = alloc_fill(o->nh, 1.0); o->v = alloc_fill(o->nh, 1.0);
  o->w = alloc_fill(o->nh, 1.0); o->T = alloc_fill(o->nh, 1.0);
  for (int m = 0; m < OCFD_N_METRICS; m++) o->met[m] = alloc_fill(o->nh, 1.0);
  o->rhybrid = alloc_fill(o->nh, 0.0);
  o->cc = alloc_fill(o->nh, 0.0);
  for (int m = 0; m < 3; m++) o->ev[m] = alloc_fill(4 * o->nh, 0.0);
  for (int m = 0; m < 12; m++) o->g[m] = alloc_fill(o->n, 0.0);
  int nmax = o->nx; if (o->ny > nmax) nmax = o->ny; if (o->nz > nmax) nmax = o->nz;
  o->npen = nmax;
  o->nthreads = omp_get_max_threads();
  o->pw = (struct pwork*)calloc(o->nthreads, sizeof(struct pwork));
  size_t pl = (size_t)nmax + 2 * LAP;
  for (int t = 0; t < o->nthreads; t++) {
    struct pwork* w = &o->pw[t];
    double** pens[8] = {&w->pc, &w->pd, &w->pu, &w->pv, &w->pw, &w->pa1, &w->pa2, &w->pa3};
    for (int m = 0; m < 8; m++) *pens[m] = alloc_fill(pl, 0.0);
    for (int m = 0; m < 5; m++) { w->pfp[m] = alloc_fill(pl, 0.0); w->pfm[m] = alloc_fill(pl, 0.0); }
    w->ph1 = alloc_fill(nmax + 1, 0.0);
    w->ph2 = alloc_fill(nmax + 1, 0.0);
    for (int m = 0; m < 5; m++) w->phh[m] = alloc_fill(nmax + 1, 0.0);
    w->scm = (int*)calloc(nmax + 1, sizeof(int));
  }
  return o;
}

void orc_destroy(ocfd_oracle* o) {
  if (!o) return;
  free(o->f); free(o->fn); free(o->du); free(o->amu);
  free(o->d); free(o->u); free(o->v); free(o->w); free(o->T);
  for (int m = 0; m < OCFD_N_METRICS; m++) free(o->met[m]);
  free(o->rhybrid); free(o->cc);
  for (int m = 0; m < 3; m++) free(o->ev[m]);
  for (int m = 0; m < 12; m++) free(o->g[m]);
  for (int t = 0; t < o->nthreads; t++) {
    struct pwork* w = &o->pw[t];
    free(w->pc); free(w->pd); free(w->pu); free(w->pv); free(w->pw); free(w->pa1); free(w->pa2); free(w->pa3);
    for (int m = 0; m < 5; m++) { free(w->pfp[m]); free(w->pfm[m]); free(w->phh[m]); }
    free(w->ph1); free(w->ph2); free(w->scm);
  }
  free(o->pw);
  free(o->bl_inlet); free(o->bl_upper); free(o->bl_pertb); free(o->bl_tm); free(o->bl_fait);
  free(o->bl_dirichlet);
  free(o);
}

double* orc_array(ocfd_oracle* o, int id) {
  switch (id) {
    case ORC_F: return o->f;
    case ORC_FN: return o->fn;
    case ORC_DU: return o->du;
    case ORC_AMU: return o->amu;
    case ORC_D: return o->d;
    case ORC_U: return o->u;
    case ORC_V: return o->v;
    case ORC_W: return o->w;
    case ORC_T: return o->T;
    case ORC_RHYBRID: return o->rhybrid;
  }
  if (id >= ORC_METRIC0 && id < ORC_METRIC0 + OCFD_N_METRICS) return o->met[id - ORC_METRIC0];
  return NULL;
}
void orc_get_time(const ocfd_oracle* o, int* istep, double* tt) { *istep = o->istep; *tt = o->tt; }
void orc_set_time(ocfd_oracle* o, int istep, double tt) { o->istep = istep; o->tt = tt; }

/* ---------------------------------------------------------------- halos */
/* exchange_boundary_x/y/z with one rank (OCFD_mpi.f90:198-233 with the
 * neighbour ids of :70-89): a periodic direction wraps its 4-layer face halo
 * onto itself over the interior of the other two directions; a non-periodic
 * one sends to MPI_PROC_NULL, i.e. nothing happens. */
static void exchange_x(ocfd_oracle* o, double* a) {
  if (!o->p.iperiodic[0]) return;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int l = 1; l <= LAP; l++) {
        a[IH(o, o->nx + l, j, k)] = a[IH(o, l, j, k)];
        a[IH(o, 1 - l, j, k)] = a[IH(o, o->nx + 1 - l, j, k)];
      }
}
static void exchange_y(ocfd_oracle* o, double* a) {
  if (!o->p.iperiodic[1]) return;
  for (int k = 1; k <= o->nz; k++)
    for (int l = 1; l <= LAP; l++)
      for (int i = 1; i <= o->nx; i++) {
        a[IH(o, i, o->ny + l, k)] = a[IH(o, i, l, k)];
        a[IH(o, i, 1 - l, k)] = a[IH(o, i, o->ny + 1 - l, k)];
      }
}
static void exchange_z(ocfd_oracle* o, double* a) {
  if (!o->p.iperiodic[2]) return;
  for (int l = 1; l <= LAP; l++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        a[IH(o, i, j, o->nz + l)] = a[IH(o, i, j, l)];
        a[IH(o, i, j, 1 - l)] = a[IH(o, i, j, o->nz + 1 - l)];
      }
}
void orc_exchange_xyz(ocfd_oracle* o, double* a) {
  exchange_x(o, a);
  exchange_y(o, a);
  exchange_z(o, a);
}
void orc_halo_prims(ocfd_oracle* o) {
  orc_exchange_xyz(o, o->d);
  orc_exchange_xyz(o, o->u);
  orc_exchange_xyz(o, o->v);
  orc_exchange_xyz(o, o->w);
  orc_exchange_xyz(o, o->T);
}

/* ---------------------------------------------------------------- central derivatives */
/* OCFD_dx0 / OCFD_dy0 / OCFD_dz0: OCFD_dxyz_viscous.f90:3-239 */
void orc_d0(ocfd_oracle* o, int dir, const double* f, double* fx) {
  const ocfd_params* p = &o->p;
  int scheme = p->scheme_vis;
  double h = dir == 0 ? p->hx : (dir == 1 ? p->hy : p->hz);
  double a1 = 1.0 / (60.0 * h), a2 = -3.0 / (20.0 * h), a3 = 3.0 / (4.0 * h);
  double c1 = 0.8 / h, c2 = -0.2 / h, c3 = 3.80952380952380952e-2 / h, c4 = -3.571428571428571428e-3 / h;
  int nn = dir == 0 ? o->nx : (dir == 1 ? o->ny : o->nz);
  /* stride of the derivative direction in the haloed array */
  ptrdiff_t s = dir == 0 ? 1 : (dir == 1 ? (ptrdiff_t)o->nxh : (ptrdiff_t)o->nxh * o->nyh);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        const double* q = f + IH(o, i, j, k);
        double r;
        if (scheme == OCFD_SCHEME_CD6)
          r = a1 * (q[3 * s] - q[-3 * s]) + a2 * (q[2 * s] - q[-2 * s]) + a3 * (q[s] - q[-s]);
        else
          r = c1 * (q[s] - q[-s]) + c2 * (q[2 * s] - q[-2 * s]) + c3 * (q[3 * s] - q[-3 * s]) +
              c4 * (q[4 * s] - q[-4 * s]);
        fx[I3(o, i, j, k)] = r;
      }
  if (p->iperiodic[dir]) return;
  /* boundary closures: OCFD_dxyz_viscous.f90:43-77 (x), :123-157 (y), :203-237 (z) */
  int n1 = dir == 0 ? o->ny : o->nx, n2 = dir == 2 ? o->ny : o->nz;
  for (int b = 0; b < n2; b++)
    for (int a = 0; a < n1; a++) {
      int i0, j0, k0;
      if (dir == 0) { j0 = a + 1; k0 = b + 1; i0 = 1; }
      else if (dir == 1) { i0 = a + 1; k0 = b + 1; j0 = 1; }
      else { i0 = a + 1; j0 = b + 1; k0 = 1; }
      const double* q = f + IH(o, i0, j0, k0) - s; /* q[l*s] = f at index l along dir */
      size_t o0 = I3(o, i0, j0, k0);
      ptrdiff_t so = dir == 0 ? 1 : (dir == 1 ? (ptrdiff_t)o->nx : (ptrdiff_t)o->nx * o->ny);
      double* out = fx + o0 - so; /* out[l*so] = fx at index l */
#define Q(l) q[(ptrdiff_t)(l) * s]
#define OUT(l) out[(ptrdiff_t)(l) * so]
      OUT(1) = (-3.0 * Q(1) + 4.0 * Q(2) - Q(3)) / (2.0 * h);
      OUT(2) = (Q(3) - Q(1)) / (2.0 * h);
      OUT(3) = (8.0 * (Q(4) - Q(2)) - (Q(5) - Q(1))) / (12.0 * h);
      if (scheme == OCFD_SCHEME_CD8) OUT(4) = a1 * (Q(7) - Q(1)) + a2 * (Q(6) - Q(2)) + a3 * (Q(5) - Q(3));
      OUT(nn) = (Q(nn - 2) - 4.0 * Q(nn - 1) + 3.0 * Q(nn)) / (2.0 * h);
      OUT(nn - 1) = (Q(nn) - Q(nn - 2)) / (2.0 * h);
      OUT(nn - 2) = (8.0 * (Q(nn - 1) - Q(nn - 3)) - (Q(nn) - Q(nn - 4))) / (12.0 * h);
      if (scheme == OCFD_SCHEME_CD8)
        OUT(nn - 3) = a1 * (Q(nn) - Q(nn - 6)) + a2 * (Q(nn - 1) - Q(nn - 5)) + a3 * (Q(nn - 2) - Q(nn - 4));
#undef Q
#undef OUT
    }
}

/* ---------------------------------------------------------------- mesh */
/* comput_Jacobian3d: OCFD_mesh.f90:61-107 */
static void comput_jacobian3d(ocfd_oracle* o) {
  double* xi = (double*)malloc(9 * o->n * sizeof(double));
  double *xj = xi + o->n, *xk = xj + o->n, *yi = xk + o->n, *yj = yi + o->n, *yk = yj + o->n;
  double *zi = yk + o->n, *zj = zi + o->n, *zk = zj + o->n;
  double** M = o->met;
  orc_d0(o, 0, M[OCFD_M_AXX], xi); orc_d0(o, 0, M[OCFD_M_AYY], yi); orc_d0(o, 0, M[OCFD_M_AZZ], zi);
  orc_d0(o, 1, M[OCFD_M_AXX], xj); orc_d0(o, 1, M[OCFD_M_AYY], yj); orc_d0(o, 1, M[OCFD_M_AZZ], zj);
  orc_d0(o, 2, M[OCFD_M_AXX], xk); orc_d0(o, 2, M[OCFD_M_AYY], yk); orc_d0(o, 2, M[OCFD_M_AZZ], zk);
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t c = I3(o, i, j, k), h = IH(o, i, j, k);
        double xi1 = xi[c], xj1 = xj[c], xk1 = xk[c], yi1 = yi[c], yj1 = yj[c], yk1 = yk[c];
        double zi1 = zi[c], zj1 = zj[c], zk1 = zk[c];
        double Jac1 = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1 - zi1 * yj1 * xk1 -
                             yi1 * xj1 * zk1 - xi1 * zj1 * yk1);
        M[OCFD_M_AJAC][h] = Jac1;
        M[OCFD_M_AKX][h] = Jac1 * (yj1 * zk1 - zj1 * yk1);
        M[OCFD_M_AKY][h] = Jac1 * (zj1 * xk1 - xj1 * zk1);
        M[OCFD_M_AKZ][h] = Jac1 * (xj1 * yk1 - yj1 * xk1);
        M[OCFD_M_AIX][h] = Jac1 * (yk1 * zi1 - zk1 * yi1);
        M[OCFD_M_AIY][h] = Jac1 * (zk1 * xi1 - xk1 * zi1);
        M[OCFD_M_AIZ][h] = Jac1 * (xk1 * yi1 - yk1 * xi1);
        M[OCFD_M_ASX][h] = Jac1 * (yi1 * zj1 - zi1 * yj1);
        M[OCFD_M_ASY][h] = Jac1 * (zi1 * xj1 - xi1 * zj1);
        M[OCFD_M_ASZ][h] = Jac1 * (xi1 * yj1 - yi1 * xj1);
      }
  free(xi);
}

/* updata_Axyz_periodic: OCFD_mesh.f90:109-185 */
static void updata_axyz_periodic(ocfd_oracle* o) {
  double** M = o->met;
  const ocfd_params* p = &o->p;
  for (int c = 0; c < 3; c++) {
    double* A = M[OCFD_M_AXX + c];
    if (p->iperiodic[0])
      for (int k = 1; k <= o->nz; k++)
        for (int j = 1; j <= o->ny; j++)
          for (int l = 1; l <= LAP; l++) {
            A[IH(o, 1 - l, j, k)] = A[IH(o, 1 - l, j, k)] - p->periodic_span[0][c];
            A[IH(o, o->nx + l, j, k)] = A[IH(o, o->nx + l, j, k)] + p->periodic_span[0][c];
          }
    if (p->iperiodic[1])
      for (int k = 1; k <= o->nz; k++)
        for (int l = 1; l <= LAP; l++)
          for (int i = 1; i <= o->nx; i++) {
            A[IH(o, i, 1 - l, k)] = A[IH(o, i, 1 - l, k)] - p->periodic_span[1][c];
            A[IH(o, i, o->ny + l, k)] = A[IH(o, i, o->ny + l, k)] + p->periodic_span[1][c];
          }
    if (p->iperiodic[2])
      for (int l = 1; l <= LAP; l++)
        for (int j = 1; j <= o->ny; j++)
          for (int i = 1; i <= o->nx; i++) {
            A[IH(o, i, j, 1 - l)] = A[IH(o, i, j, 1 - l)] - p->periodic_span[2][c];
            A[IH(o, i, j, o->nz + l)] = A[IH(o, i, j, o->nz + l)] + p->periodic_span[2][c];
          }
  }
}

/* Jac_Ghost_Extent_1st: OCFD_GhostCell.f90:18-160 */
static void jac_ghost_extent_1st(ocfd_oracle* o) {
  double** M = o->met;
  const int* gc = o->p.ghost_cell;
  int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int face = 0; face < 6; face++) {
    if (gc[face] != 1) continue;
    int dir = face / 2, hi = face % 2;
    int n1 = dir == 0 ? ny : nx, n2 = dir == 2 ? ny : nz, nn = dir == 0 ? nx : (dir == 1 ? ny : nz);
    for (int b = 1; b <= n2; b++)
      for (int l = 1; l <= LAP; l++)
        for (int a = 1; a <= n1; a++) {
          int g = hi ? nn + l : 1 - l;          /* ghost index along dir */
          int e = hi ? nn : 1, e2 = hi ? nn - 1 : 2; /* edge point and its neighbour */
          /* map (along, a, b) to (i,j,k) */
#define MAP(idx, along) \
  do { if (dir == 0) { idx[0] = along; idx[1] = a; idx[2] = b; } \
       else if (dir == 1) { idx[0] = a; idx[1] = along; idx[2] = b; } \
       else { idx[0] = a; idx[1] = b; idx[2] = along; } } while (0)
          int ig[3], ie_[3], ie2[3];
          MAP(ig, g); MAP(ie_, e); MAP(ie2, e2);
          size_t hg = IH(o, ig[0], ig[1], ig[2]), he = IH(o, ie_[0], ie_[1], ie_[2]), he2 = IH(o, ie2[0], ie2[1], ie2[2]);
          for (int m = OCFD_M_AKX; m <= OCFD_M_AJAC; m++) M[m][hg] = M[m][he];
          double fac = hi ? (double)(g - nn) : (1.0 - g);
          for (int m = OCFD_M_AXX; m <= OCFD_M_AZZ; m++) M[m][hg] = M[m][he] + fac * (M[m][he] - M[m][he2]);
        }
  }
}

/* comput_Jacobian3d_Ghost: OCFD_GhostCell.f90:394-500 */
static void comput_jacobian3d_ghost(ocfd_oracle* o, int nb) {
  int nx = o->nx, ny = o->ny, nz = o->nz;
  int ib, ie, jb, je, kb, ke, ib1, ie1, jb1, je1, kb1, ke1;
  double** M = o->met;
  const ocfd_params* p = &o->p;
  if (nb == 1) { ib = 1 - LAP; ie = 0; jb = 1; je = ny; kb = 1; ke = nz; ib1 = ib; ie1 = 1; jb1 = jb; je1 = je; kb1 = kb; ke1 = ke; }
  else if (nb == 2) { ib = nx + 1; ie = nx + LAP; jb = 1; je = ny; kb = 1; ke = nz; ib1 = nx; ie1 = ie; jb1 = jb; je1 = je; kb1 = kb; ke1 = ke; }
  else if (nb == 3) { ib = 1; ie = nx; jb = 1 - LAP; je = 0; kb = 1; ke = nz; ib1 = ib; ie1 = ie; jb1 = jb; je1 = 1; kb1 = kb; ke1 = ke; }
  else if (nb == 4) { ib = 1; ie = nx; jb = ny + 1; je = ny + LAP; kb = 1; ke = nz; ib1 = ib; ie1 = ie; jb1 = ny; je1 = je; kb1 = kb; ke1 = ke; }
  else if (nb == 5) { ib = 1; ie = nx; jb = 1; je = ny; kb = 1 - LAP; ke = 0; ib1 = ib; ie1 = ie; jb1 = jb; je1 = je; kb1 = kb; ke1 = 1; }
  else { ib = 1; ie = nx; jb = 1; je = ny; kb = nz + 1; ke = nz + LAP; ib1 = ib; ie1 = ie; jb1 = jb; je1 = je; kb1 = nz; ke1 = ke; }
  const double *X = M[OCFD_M_AXX], *Y = M[OCFD_M_AYY], *Z = M[OCFD_M_AZZ];
  double hx = p->hx, hy = p->hy, hz = p->hz;
  for (int k = kb; k <= ke; k++)
    for (int j = jb; j <= je; j++)
      for (int i = ib; i <= ie; i++) {
        double xi1, yi1, zi1, xj1, yj1, zj1, xk1, yk1, zk1;
        size_t c = IH(o, i, j, k);
        ptrdiff_t s;
        /* i direction */
        s = 1;
#define D_ONE_L(A, h) ((-3.0 * A[c] + 4.0 * A[c + s] - A[c + 2 * s]) / (2.0 * h))
#define D_ONE_R(A, h) ((A[c - 2 * s] - 4.0 * A[c - s] + 3.0 * A[c]) / (2.0 * h))
#define D_C2(A, h) ((A[c + s] - A[c - s]) / (2.0 * h))
#define D_C4(A, h) ((8.0 * (A[c + s] - A[c - s]) - (A[c + 2 * s] - A[c - 2 * s])) / (12.0 * h))
        if (i == ib1) { xi1 = D_ONE_L(X, hx); yi1 = D_ONE_L(Y, hx); zi1 = D_ONE_L(Z, hx); }
        else if (i == ie1) { xi1 = D_ONE_R(X, hx); yi1 = D_ONE_R(Y, hx); zi1 = D_ONE_R(Z, hx); }
        else if (i == ib1 + 1 || i == ie1 - 1) { xi1 = D_C2(X, hx); yi1 = D_C2(Y, hx); zi1 = D_C2(Z, hx); }
        else { xi1 = D_C4(X, hx); yi1 = D_C4(Y, hx); zi1 = D_C4(Z, hx); }
        s = o->nxh;
        if (j == jb1) { xj1 = D_ONE_L(X, hy); yj1 = D_ONE_L(Y, hy); zj1 = D_ONE_L(Z, hy); }
        else if (j == je1) { xj1 = D_ONE_R(X, hy); yj1 = D_ONE_R(Y, hy); zj1 = D_ONE_R(Z, hy); }
        else if (j == jb1 + 1 || j == je1 - 1) { xj1 = D_C2(X, hy); yj1 = D_C2(Y, hy); zj1 = D_C2(Z, hy); }
        else { xj1 = D_C4(X, hy); yj1 = D_C4(Y, hy); zj1 = D_C4(Z, hy); }
        s = (ptrdiff_t)o->nxh * o->nyh;
        if (k == kb1) { xk1 = D_ONE_L(X, hz); yk1 = D_ONE_L(Y, hz); zk1 = D_ONE_L(Z, hz); }
        else if (k == ke1) { xk1 = D_ONE_R(X, hz); yk1 = D_ONE_R(Y, hz); zk1 = D_ONE_R(Z, hz); }
        else if (k == kb1 + 1 || k == ke1 - 1) { xk1 = D_C2(X, hz); yk1 = D_C2(Y, hz); zk1 = D_C2(Z, hz); }
        else { xk1 = D_C4(X, hz); yk1 = D_C4(Y, hz); zk1 = D_C4(Z, hz); }
#undef D_ONE_L
#undef D_ONE_R
#undef D_C2
#undef D_C4
        double Jac1 = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1 - zi1 * yj1 * xk1 -
                             yi1 * xj1 * zk1 - xi1 * zj1 * yk1);
        M[OCFD_M_AJAC][c] = Jac1;
        M[OCFD_M_AKX][c] = Jac1 * (yj1 * zk1 - zj1 * yk1);
        M[OCFD_M_AKY][c] = Jac1 * (zj1 * xk1 - xj1 * zk1);
        M[OCFD_M_AKZ][c] = Jac1 * (xj1 * yk1 - yj1 * xk1);
        M[OCFD_M_AIX][c] = Jac1 * (yk1 * zi1 - zk1 * yi1);
        M[OCFD_M_AIY][c] = Jac1 * (zk1 * xi1 - xk1 * zi1);
        M[OCFD_M_AIZ][c] = Jac1 * (xk1 * yi1 - yk1 * xi1);
        M[OCFD_M_ASX][c] = Jac1 * (yi1 * zj1 - zi1 * yj1);
        M[OCFD_M_ASY][c] = Jac1 * (zi1 * xj1 - xi1 * zj1);
        M[OCFD_M_ASZ][c] = Jac1 * (xi1 * yj1 - yi1 * xj1);
      }
}

/* Jac_Ghost_Extent_2nd: OCFD_GhostCell.f90:290-391 */
static void jac_ghost_extent_2nd(ocfd_oracle* o) {
  double** M = o->met;
  const int* gc = o->p.ghost_cell;
  int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int face = 0; face < 6; face++) {
    if (gc[face] != 2) continue;
    int dir = face / 2, hi = face % 2;
    int n1 = dir == 0 ? ny : nx, n2 = dir == 2 ? ny : nz, nn = dir == 0 ? nx : (dir == 1 ? ny : nz);
    for (int b = 1; b <= n2; b++)
      for (int l = 1; l <= LAP; l++)
        for (int a = 1; a <= n1; a++) {
          int g = hi ? nn + l : 1 - l;
          int g1 = hi ? 2 * nn - g : 2 - g;
          int e = hi ? nn : 1;
          int ig[3], ie_[3], ig1[3];
          MAP(ig, g); MAP(ie_, e); MAP(ig1, g1);
          size_t hg = IH(o, ig[0], ig[1], ig[2]), he = IH(o, ie_[0], ie_[1], ie_[2]), hg1 = IH(o, ig1[0], ig1[1], ig1[2]);
          for (int m = OCFD_M_AXX; m <= OCFD_M_AZZ; m++) M[m][hg] = 2.0 * M[m][he] - M[m][hg1];
        }
    comput_jacobian3d_ghost(o, face + 1);
  }
}
#undef MAP

/* init_mesh: OCFD_mesh.f90:1-58.  x,y,z NULL -> mesh_gen('box') (:319-354);
 * otherwise interior coordinates as read by read_mesh1d/2d_plane/3d. */
static void jac_ghost_user(ocfd_oracle* o);

/* init_mesh (OCFD_mesh.f90:1-58).  jac == NULL: the metrics and Jacobian are
 * computed from the coordinates (comput_Jacobian3d, :24-26); otherwise jac
 * holds the interior Akx, Aky, Akz, Aix, Aiy, Aiz, Asx, Asy, Asz, Ajac read
 * from the grid file (Iflag_Gridtype = GRID_AND_JACOBIAN3D, read_mesh3d :187-217)
 * and only their halos, ghost values and the /Ajac copies are formed. */
static void init_mesh_common(ocfd_oracle* o, const double* x, const double* y, const double* z,
                             const double* const jac[10]) {
  double** M = o->met;
  const double PI = 3.1415926535897932;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t h = IH(o, i, j, k), c = I3(o, i, j, k);
        if (x == NULL) {
          M[OCFD_M_AXX][h] = 2.0 * PI / (double)o->nx * (double)i;
          M[OCFD_M_AYY][h] = 2.0 * PI / (double)o->ny * (double)j;
          M[OCFD_M_AZZ][h] = 2.0 * PI / (double)o->nz * (double)k;
        } else {
          M[OCFD_M_AXX][h] = x[c];
          M[OCFD_M_AYY][h] = y[c];
          M[OCFD_M_AZZ][h] = z[c];
        }
      }
  orc_exchange_xyz(o, M[OCFD_M_AXX]);
  orc_exchange_xyz(o, M[OCFD_M_AYY]);
  orc_exchange_xyz(o, M[OCFD_M_AZZ]);
  updata_axyz_periodic(o);
  if (jac == NULL) {
    comput_jacobian3d(o);
  } else {
    for (int m = 0; m < 10; m++)
      for (int k = 1; k <= o->nz; k++)
        for (int j = 1; j <= o->ny; j++)
          for (int i = 1; i <= o->nx; i++) M[OCFD_M_AKX + m][IH(o, i, j, k)] = jac[m][I3(o, i, j, k)];
  }
  for (int m = OCFD_M_AKX; m <= OCFD_M_AJAC; m++) orc_exchange_xyz(o, M[m]);
  /* Jac_Ghost_boundary: OCFD_GhostCell.f90:1-7 */
  jac_ghost_extent_1st(o);
  jac_ghost_extent_2nd(o);
  jac_ghost_user(o);
  for (size_t h = 0; h < o->nh; h++) {
    double J = M[OCFD_M_AJAC][h];
    for (int m = 0; m < 9; m++) M[OCFD_M_AKX1 + m][h] = M[OCFD_M_AKX + m][h] / J;
  }
}

void orc_init_mesh(ocfd_oracle* o, const double* x, const double* y, const double* z) {
  init_mesh_common(o, x, y, z, NULL);
}

void orc_init_mesh_jacobian(ocfd_oracle* o, const double* x, const double* y, const double* z,
                            const double* const jac[10]) {
  init_mesh_common(o, x, y, z, jac);
}

/* Jac_Ghost_Userdef: OCFD_GhostCell_UserDef.f90:4-11 with Jac_Ghost_Sweptcorner
 * (:23-49, k- symmetry about z = 0) and Jac_Ghost_flatplate (:76-102, j-
 * symmetry about y = 0): mirrored metrics, sign flips of the reflected components */
static void jac_ghost_user(ocfd_oracle* o) {
  double** M = o->met;
  if (o->p.ibc == OCFD_BC_SWEPTCORNER && o->p.ghost_cell[4] == -1) {
    /* sign of Akx..Ajac, Axx..Azz under z -> -z */
    const int ids[13] = {OCFD_M_AKX, OCFD_M_AKY, OCFD_M_AKZ, OCFD_M_AIX, OCFD_M_AIY, OCFD_M_AIZ, OCFD_M_ASX,
                         OCFD_M_ASY, OCFD_M_ASZ, OCFD_M_AJAC, OCFD_M_AXX, OCFD_M_AYY, OCFD_M_AZZ};
    const double sg[13] = {1, 1, -1, 1, 1, -1, -1, -1, 1, 1, 1, 1, -1};
    for (int k = 1 - LAP; k <= 0; k++) {
      int k1 = 1 - k;
      for (int j = 1; j <= o->ny; j++)
        for (int i = 1; i <= o->nx; i++)
          for (int q = 0; q < 13; q++) {
            double x = M[ids[q]][IH(o, i, j, k1)];
            M[ids[q]][IH(o, i, j, k)] = sg[q] < 0 ? -x : x;
          }
    }
  } else if (o->p.ibc == OCFD_BC_BOUNDARYLAYER && o->p.ghost_cell[2] == -1) {
    const int ids[13] = {OCFD_M_AKX, OCFD_M_AKY, OCFD_M_AKZ, OCFD_M_AIX, OCFD_M_AIY, OCFD_M_AIZ, OCFD_M_ASX,
                         OCFD_M_ASY, OCFD_M_ASZ, OCFD_M_AJAC, OCFD_M_AXX, OCFD_M_AYY, OCFD_M_AZZ};
    const double sg[13] = {1, -1, 1, -1, 1, -1, 1, -1, 1, 1, 1, -1, 1};
    for (int k = 1; k <= o->nz; k++)
      for (int j = 1 - LAP; j <= 0; j++) {
        int j1 = 2 - j;
        for (int i = 1; i <= o->nx; i++)
          for (int q = 0; q < 13; q++) {
            double x = M[ids[q]][IH(o, i, j1, k)];
            M[ids[q]][IH(o, i, j, k)] = sg[q] < 0 ? -x : x;
          }
      }
  }
}

/* ---------------------------------------------------------------- BC */
/* ocfd_bc_blunt2d: OCFD_BC_Def.f90:4-33 */
static void bc_blunt2d(ocfd_oracle* o) {
  for (int k = 1; k <= o->nz; k++)
    for (int i = 1; i <= o->nx; i++) {
      size_t h1 = IH(o, i, 1, k), h2 = IH(o, i, 2, k);
      o->d[h1] = o->d[h2];
      o->u[h1] = 0.0; o->v[h1] = 0.0; o->w[h1] = 0.0;
      o->T[h1] = o->T[h2];
    }
  for (int k = 1; k <= o->nz; k++)
    for (int i = 1; i <= o->nx; i++) {
      size_t h = IH(o, i, o->ny, k);
      o->d[h] = 1.0; o->u[h] = 1.0; o->v[h] = 0.0; o->w[h] = 0.0; o->T[h] = 1.0;
    }
}

/* BC_User_Def slot (OCFD_User_Def.f90:12-18) filled with an isothermal wall at
 * j=1, modelled on OCFD_BC_Boundarylayers.f90:125-133 (no perturbation), and
 * the free stream of ocfd_bc_blunt2d at j=ny. */
static void bc_user_isothermal(ocfd_oracle* o) {
  double Tw = o->p.bc_para[0];
  for (int k = 1; k <= o->nz; k++)
    for (int i = 1; i <= o->nx; i++) {
      size_t h1 = IH(o, i, 1, k), h2 = IH(o, i, 2, k), h3 = IH(o, i, 3, k);
      o->u[h1] = 0.0; o->v[h1] = 0.0; o->w[h1] = 0.0;
      o->T[h1] = Tw;
      o->d[h1] = (4.0 * o->d[h2] * o->T[h2] - o->d[h3] * o->T[h3]) / (3.0 * Tw);
    }
  for (int k = 1; k <= o->nz; k++)
    for (int i = 1; i <= o->nx; i++) {
      size_t h = IH(o, i, o->ny, k);
      o->d[h] = 1.0; o->u[h] = 1.0; o->v[h] = 0.0; o->w[h] = 0.0; o->T[h] = 1.0;
    }
}

/* ---- BC_BoundaryLayer / BC_SweptCorner (OCFD_BC_Boundarylayers.f90) ----
 * The boundary data that the reference builds at its first call
 * (init_bcdata_boundarylayer :171-270 reads the inlet / upper files,
 * init_bc_wall_perturbation :313-400 draws random phases) arrive from the host:
 * inlet (ny,nz,5), upper (nx,nz,5), wall perturbation shape (nx,nz), and the
 * amplitudes TM / phases fait of the time factor (get_ht_multifrequancy
 * :404-440).  init_bc_nonRef (:273-311) is computed here from the grid. */
void orc_set_bc_layer(ocfd_oracle* o, const double* inlet, const double* upper, const double* pertb, int mt,
                      double beta, const double* tm, const double* fait) {
  const size_t ni = (size_t)o->ny * o->nz * 5, nu = (size_t)o->nx * o->nz * 5, np = (size_t)o->nx * o->nz;
  free(o->bl_inlet); free(o->bl_upper); free(o->bl_pertb); free(o->bl_tm); free(o->bl_fait);
  free(o->bl_dirichlet);
  o->bl_inlet = (double*)calloc(ni, sizeof(double));
  o->bl_upper = (double*)calloc(nu, sizeof(double));
  o->bl_pertb = (double*)calloc(np, sizeof(double));
  o->bl_dirichlet = (int*)calloc(np, sizeof(int));
  o->bl_mt = mt > 0 ? mt : 0;
  o->bl_beta = beta;
  o->bl_tm = (double*)calloc((size_t)o->bl_mt + 1, sizeof(double));
  o->bl_fait = (double*)calloc((size_t)o->bl_mt + 1, sizeof(double));
  if (inlet) memcpy(o->bl_inlet, inlet, ni * sizeof(double));
  if (upper) memcpy(o->bl_upper, upper, nu * sizeof(double));
  if (pertb) memcpy(o->bl_pertb, pertb, np * sizeof(double));
  for (int m = 0; m < o->bl_mt; m++) { o->bl_tm[m] = tm[m]; o->bl_fait[m] = fait[m]; }
  /* init_bc_nonRef: mode 0 auto (Dirichlet where the upper boundary rises faster
   * than the free stream, tan(AoA)), 1 non-reflecting, 2 Dirichlet */
  const int mode = o->p.ibc == OCFD_BC_SWEPTCORNER ? 0 : (int)lround(o->p.bc_para[2]);
  const double sy0 = tan(o->p.aoa), epsl = 1.0e-6;
  double** M = o->met;
  for (int k = 1; k <= o->nz; k++)
    for (int i = 1; i <= o->nx; i++) {
      int dir = 0;
      if (mode == 2) dir = 1;
      else if (mode == 0) {
        double sy;
        if (i == 1)
          sy = (M[OCFD_M_AYY][IH(o, i + 1, o->ny, k)] - M[OCFD_M_AYY][IH(o, i, o->ny, k)]) /
               (M[OCFD_M_AXX][IH(o, i + 1, o->ny, k)] - M[OCFD_M_AXX][IH(o, i, o->ny, k)]);
        else
          sy = (M[OCFD_M_AYY][IH(o, i, o->ny, k)] - M[OCFD_M_AYY][IH(o, i - 1, o->ny, k)]) /
               (M[OCFD_M_AXX][IH(o, i, o->ny, k)] - M[OCFD_M_AXX][IH(o, i - 1, o->ny, k)]);
        dir = sy >= sy0 + epsl;
      }
      o->bl_dirichlet[(size_t)(i - 1) + (size_t)o->nx * (k - 1)] = dir;
    }
}

/* get_ht_multifrequancy: OCFD_BC_Boundarylayers.f90:404-440 */
static double bl_ht(const ocfd_oracle* o) {
  const double PI = 3.14159265358979;
  if (!(o->bl_beta > 0.0)) return 1.0;
  double ht = 0.0;
  for (int m = 1; m <= o->bl_mt; m++) ht = ht + o->bl_tm[m - 1] * sin(m * o->bl_beta * o->tt + 2.0 * PI * o->bl_fait[m - 1]);
  return ht;
}

static void bl_set(ocfd_oracle* o, size_t h, double d, double u, double v, double w, double T) {
  o->d[h] = d; o->u[h] = u; o->v[h] = v; o->w[h] = w; o->T[h] = T;
}

/* the j=1 wall of both BCs (:123-141, :525-551) for point (i,k) */
static void bl_wall(ocfd_oracle* o, int i, int k, double Tw, double A, double ht) {
  double** M = o->met;
  size_t h1 = IH(o, i, 1, k), h2 = IH(o, i, 2, k), h3 = IH(o, i, 3, k);
  double aix = M[OCFD_M_AIX][h1], aiy = M[OCFD_M_AIY][h1], aiz = M[OCFD_M_AIZ][h1];
  double tmp = 1.0 / (sqrt(aix * aix + aiy * aiy + aiz * aiz));
  double A0 = A * ht * o->bl_pertb[(size_t)(i - 1) + (size_t)o->nx * (k - 1)];
  o->u[h1] = A0 * aix * tmp;
  o->v[h1] = A0 * aiy * tmp;
  o->w[h1] = A0 * aiz * tmp;
  if (Tw > 0.0) {
    o->T[h1] = Tw;
    o->d[h1] = (4.0 * o->d[h2] * o->T[h2] - o->d[h3] * o->T[h3]) / (3.0 * Tw);
  } else {
    o->T[h1] = (4.0 * o->T[h2] - o->T[h3]) / 3.0;
    o->d[h1] = (4.0 * o->d[h2] - o->d[h3]) / 3.0;
  }
}

/* outlet i=nx (:143-167): 1 first-order, 2 second-order extrapolation */
static void bl_outlet(ocfd_oracle* o, int mode) {
  double* Q[5] = {o->d, o->u, o->v, o->w, o->T};
  if (mode != 1 && mode != 2) return;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++) {
      size_t h = IH(o, o->nx, j, k), h1 = IH(o, o->nx - 1, j, k), h2 = IH(o, o->nx - 2, j, k);
      for (int q = 0; q < 5; q++) Q[q][h] = mode == 1 ? Q[q][h1] : 2.0 * Q[q][h1] - Q[q][h2];
    }
}

static void bl_upper(ocfd_oracle* o, int data) {
  const double u0 = cos(o->p.aoa), v0 = sin(o->p.aoa);
  for (int k = 1; k <= o->nz; k++)
    for (int i = 1; i <= o->nx; i++) {
      const size_t c = (size_t)(i - 1) + (size_t)o->nx * (k - 1), nxz = (size_t)o->nx * o->nz;
      if (!o->bl_dirichlet[c]) continue;
      size_t h = IH(o, i, o->ny, k);
      if (data == 0)
        bl_set(o, h, 1.0, u0, v0, 0.0, 1.0);
      else {
        const double* U = o->bl_upper;
        bl_set(o, h, U[c], U[c + nxz], U[c + 2 * nxz], U[c + 3 * nxz], U[c + 4 * nxz]);
      }
    }
}

/* ocfd_bc_BoundaryLayer: OCFD_BC_Boundarylayers.f90:17-169 */
static void bc_boundary_layer(ocfd_oracle* o) {
  const double* bp = o->p.bc_para;
  const int inlet = (int)lround(bp[0]), upper = (int)lround(bp[1]), outlet = (int)lround(bp[3]);
  const double Tw = bp[4], A = bp[7];
  const double u0 = cos(o->p.aoa), v0 = sin(o->p.aoa);
  /* inlet i=1: the free stream of the reference sets T = 0 there (:58-66) */
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++) {
      size_t h = IH(o, 1, j, k);
      if (inlet == 0)
        bl_set(o, h, 1.0, u0, v0, 0.0, 0.0);
      else {
        const size_t c = (size_t)(j - 1) + (size_t)o->ny * (k - 1), nyz = (size_t)o->ny * o->nz;
        const double* I = o->bl_inlet;
        bl_set(o, h, I[c], I[c + nyz], I[c + 2 * nyz], I[c + 3 * nyz], I[c + 4 * nyz]);
      }
    }
  bl_upper(o, upper);
  const double ht = bl_ht(o);
  for (int k = 1; k <= o->nz; k++)
    for (int i = 1; i <= o->nx; i++) bl_wall(o, i, k, Tw, A, ht);
  bl_outlet(o, outlet);
}

/* ocfd_bc_swept_corner: OCFD_BC_Boundarylayers.f90:443-618 (1-D inlet data,
 * free-stream upper boundary with the automatic Dirichlet mask) */
static void bc_swept_corner(ocfd_oracle* o) {
  const double* bp = o->p.bc_para;
  const int outlet = (int)lround(bp[0]), z1 = (int)lround(bp[10]), z2 = (int)lround(bp[11]);
  const double Tw = bp[1], wall_zl = bp[2], A = bp[4], epsl = 1.0e-7;
  double** M = o->met;
  double* Q[5] = {o->d, o->u, o->v, o->w, o->T};
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++) {
      const size_t c = (size_t)(j - 1) + (size_t)o->ny * (k - 1), nyz = (size_t)o->ny * o->nz;
      const double* I = o->bl_inlet;
      bl_set(o, IH(o, 1, j, k), I[c], I[c + nyz], I[c + 2 * nyz], I[c + 3 * nyz], I[c + 4 * nyz]);
    }
  bl_upper(o, 0);
  const double ht = bl_ht(o);
  for (int k = 1; k <= o->nz; k++)
    for (int i = 1; i <= o->nx; i++) {
      size_t h1 = IH(o, i, 1, k), h2 = IH(o, i, 2, k);
      double zz = M[OCFD_M_AZZ][h1], yy = M[OCFD_M_AYY][h1];
      if ((zz >= -epsl && zz <= wall_zl + epsl) || yy <= epsl)
        bl_wall(o, i, k, Tw, A, ht);
      else
        for (int q = 0; q < 5; q++) Q[q][h1] = Q[q][h2];
    }
  bl_outlet(o, outlet);
  if (z1 == 1)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++)
        for (int q = 0; q < 5; q++) Q[q][IH(o, i, j, 1)] = Q[q][IH(o, i, j, 2)];
  if (z2 == 1)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++)
        for (int q = 0; q < 5; q++) Q[q][IH(o, i, j, o->nz)] = Q[q][IH(o, i, j, o->nz - 1)];
}

/* Flow_Ghost_Userdef: OCFD_GhostCell_UserDef.f90:13-20, 54-73 (swept corner,
 * k- symmetry) and 106-136 (flat plate, j- extrapolation with limiter) */
static void flow_ghost_user(ocfd_oracle* o) {
  if (o->p.ibc == OCFD_BC_SWEPTCORNER && o->p.ghost_cell[4] == -1) {
    for (int k = 1 - LAP; k <= 0; k++) {
      int k1 = 1 - k;
      for (int j = 1; j <= o->ny; j++)
        for (int i = 1; i <= o->nx; i++) {
          size_t h = IH(o, i, j, k), h1 = IH(o, i, j, k1);
          o->u[h] = o->u[h1]; o->v[h] = o->v[h1]; o->w[h] = -o->w[h1]; o->d[h] = o->d[h1]; o->T[h] = o->T[h1];
        }
    }
  } else if (o->p.ibc == OCFD_BC_BOUNDARYLAYER && o->p.ghost_cell[2] == -1) {
    const double s1 = 0.5, s2 = 2.0;
    for (int k = 1; k <= o->nz; k++)
      for (int j = 1 - LAP; j <= 0; j++) {
        int j1 = 2 - j;
        for (int i = 1; i <= o->nx; i++) {
          size_t h = IH(o, i, j, k), hw = IH(o, i, 1, k), h1 = IH(o, i, j1, k);
          o->u[h] = 2.0 * o->u[hw] - o->u[h1];
          o->v[h] = 2.0 * o->v[hw] - o->v[h1];
          o->w[h] = 2.0 * o->w[hw] - o->w[h1];
          o->d[h] = 2.0 * o->d[hw] - o->d[h1];
          o->T[h] = 2.0 * o->T[hw] - o->T[h1];
          if (o->d[h] < s1 * o->d[hw]) o->d[h] = s1 * o->d[hw];
          if (o->d[h] > s2 * o->d[hw]) o->d[h] = s2 * o->d[hw];
          if (o->T[h] < s1 * o->T[hw]) o->T[h] = s1 * o->T[hw];
          if (o->T[h] > s2 * o->T[hw]) o->T[h] = s2 * o->T[hw];
        }
      }
  }
}

/* Flow_Ghost_Extent_2nd: OCFD_GhostCell.f90:164-286 */
static void flow_ghost_extent_2nd(ocfd_oracle* o) {
  const double s1 = 0.8, s2 = 1.2;
  const int* gc = o->p.ghost_cell;
  double* Q[5] = {o->u, o->v, o->w, o->d, o->T};
  for (int face = 0; face < 6; face++) {
    if (!(gc[face] == 1 || gc[face] == 2)) continue;
    int dir = face / 2, hi = face % 2;
    int n1 = dir == 0 ? o->ny : o->nx, n2 = dir == 2 ? o->ny : o->nz;
    int nn = dir == 0 ? o->nx : (dir == 1 ? o->ny : o->nz);
    for (int b = 1; b <= n2; b++)
      for (int l = 1; l <= LAP; l++)
        for (int a = 1; a <= n1; a++) {
          int g = hi ? nn + l : 1 - l;
          int g1 = hi ? 2 * nn - g : 2 - g;
          int e = hi ? nn : 1;
          int ig[3], ie_[3], ig1[3];
#define MAP2(idx, along) \
  do { if (dir == 0) { idx[0] = along; idx[1] = a; idx[2] = b; } \
       else if (dir == 1) { idx[0] = a; idx[1] = along; idx[2] = b; } \
       else { idx[0] = a; idx[1] = b; idx[2] = along; } } while (0)
          MAP2(ig, g); MAP2(ie_, e); MAP2(ig1, g1);
#undef MAP2
          size_t hg = IH(o, ig[0], ig[1], ig[2]), he = IH(o, ie_[0], ie_[1], ie_[2]), hg1 = IH(o, ig1[0], ig1[1], ig1[2]);
          for (int q = 0; q < 5; q++) Q[q][hg] = 2.0 * Q[q][he] - Q[q][hg1];
          double* dd = o->d;
          double* TT = o->T;
          if (dd[hg] < s1 * dd[he]) dd[hg] = s1 * dd[he];
          if (dd[hg] > s2 * dd[he]) dd[hg] = s2 * dd[he];
          if (TT[hg] < s1 * TT[he]) TT[hg] = s1 * TT[he];
          if (TT[hg] > s2 * TT[he]) TT[hg] = s2 * TT[he];
        }
  }
}

/* OCFD_bc: OCFD_BC.f90:2-99 (one rank: all six faces are global boundaries) */
void orc_bc(ocfd_oracle* o) {
  if (o->p.ibc == OCFD_BC_BLUNT2D) bc_blunt2d(o);
  else if (o->p.ibc == OCFD_BC_USER_DEF) bc_user_isothermal(o);
  else if (o->p.ibc == OCFD_BC_BOUNDARYLAYER) bc_boundary_layer(o);
  else if (o->p.ibc == OCFD_BC_SWEPTCORNER) bc_swept_corner(o);
  const double Cv = o->p.cv;
  /* f refresh on the six faces, in the reference's order */
  for (int face = 0; face < 6; face++) {
    int dir = face / 2, hi = face % 2;
    int nn = dir == 0 ? o->nx : (dir == 1 ? o->ny : o->nz);
    int n1 = dir == 0 ? o->ny : o->nx, n2 = dir == 2 ? o->ny : o->nz;
    int e = hi ? nn : 1;
    for (int b = 1; b <= n2; b++)
      for (int a = 1; a <= n1; a++) {
        int i, j, k;
        if (dir == 0) { i = e; j = a; k = b; } else if (dir == 1) { i = a; j = e; k = b; } else { i = a; j = b; k = e; }
        size_t h = IH(o, i, j, k);
        double d = o->d[h], u = o->u[h], v = o->v[h], w = o->w[h], T = o->T[h];
        o->f[IF(o, i, j, k, 1)] = d;
        o->f[IF(o, i, j, k, 2)] = d * u;
        o->f[IF(o, i, j, k, 3)] = d * v;
        o->f[IF(o, i, j, k, 4)] = d * w;
        o->f[IF(o, i, j, k, 5)] = d * (Cv * T + (u * u + v * v + w * w) * 0.5);
      }
  }
  flow_ghost_extent_2nd(o);
  flow_ghost_user(o);
}

/* init3d: OCFD_init.f90:1-20, then the OCFD_bc of OCFD_NS_Solver.f90:15 */
void orc_init3d(ocfd_oracle* o, const double* const prims[5]) {
  double* Q[5] = {o->d, o->u, o->v, o->w, o->T};
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++)
        for (int q = 0; q < 5; q++) Q[q][IH(o, i, j, k)] = prims[q][I3(o, i, j, k)];
  const double Cv = o->p.cv;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t h = IH(o, i, j, k);
        double d = o->d[h], u = o->u[h], v = o->v[h], w = o->w[h], T = o->T[h];
        o->f[IF(o, i, j, k, 1)] = d;
        o->f[IF(o, i, j, k, 2)] = d * u;
        o->f[IF(o, i, j, k, 3)] = d * v;
        o->f[IF(o, i, j, k, 4)] = d * w;
        o->f[IF(o, i, j, k, 5)] = d * ((u * u + v * v + w * w) * 0.5 + Cv * T);
      }
  orc_bc(o);
}

/* ---------------------------------------------------------------- hybrid sensor */
/* set_hybrid_scheme: OCFD_SetHybrid.f90:2-15 */
static int set_hybrid_scheme(const ocfd_params* p, double R0) {
  if (R0 <= p->hybrid_para[1]) return 1;
  if (R0 <= p->hybrid_para[2]) return 2;
  return 3;
}

/* comput_Rhybrid: OCFD_SetHybrid.f90:17-152 (statistics print omitted).
 * The patch loop of :88-110 assigns Hybrid_para(8) to ie (the reference's
 * :93) and leaves je undefined; this restatement uses Hybrid_para(8) for both. */
void orc_comput_rhybrid(ocfd_oracle* o) {
  const ocfd_params* p = &o->p;
  double* P = alloc_fill(o->nh, 0.0);
  double p00 = 1.0 / (p->gamma * p->ma * p->ma);
  double epsl = 1.0e-30;
  for (size_t h = 0; h < o->nh; h++) P[h] = p00 * o->d[h] * o->T[h];
  int sensor = (int)lround(p->hybrid_para[0]);
  if (sensor == 1) {
    for (int k = 1; k <= o->nz; k++)
      for (int j = 1; j <= o->ny; j++)
        for (int i = 1; i <= o->nx; i++) {
          size_t c = IH(o, i, j, k);
          size_t sx = 1, sy = o->nxh, sz = (size_t)o->nxh * o->nyh;
          o->rhybrid[c] = fabs((P[c - sx] - 2.0 * P[c] + P[c + sx]) / (P[c - sx] + 2.0 * P[c] + P[c + sx])) +
                          fabs((P[c - sy] - 2.0 * P[c] + P[c + sy]) / (P[c - sy] + 2.0 * P[c] + P[c + sy])) +
                          fabs((P[c - sz] - 2.0 * P[c] + P[c + sz]) / (P[c - sz] + 2.0 * P[c] + P[c + sz]));
        }
  } else {
    double* pk = (double*)malloc(3 * o->n * sizeof(double));
    double *pi = pk + o->n, *ps = pi + o->n;
    orc_d0(o, 0, P, pk);
    orc_d0(o, 1, P, pi);
    orc_d0(o, 2, P, ps);
    double dp0 = 0.0;
    double** M = o->met;
    for (int k = 1; k <= o->nz; k++)
      for (int j = 1; j <= o->ny; j++)
        for (int i = 1; i <= o->nx; i++) {
          size_t c = I3(o, i, j, k), h = IH(o, i, j, k);
          double px = pk[c] * M[OCFD_M_AKX][h] + pi[c] * M[OCFD_M_AIX][h] + ps[c] * M[OCFD_M_ASX][h];
          double py = pk[c] * M[OCFD_M_AKY][h] + pi[c] * M[OCFD_M_AIY][h] + ps[c] * M[OCFD_M_ASY][h];
          double pz = pk[c] * M[OCFD_M_AKZ][h] + pi[c] * M[OCFD_M_AIZ][h] + ps[c] * M[OCFD_M_ASZ][h];
          o->rhybrid[h] = sqrt(px * px + py * py + pz * pz);
          dp0 = dp0 + o->rhybrid[h];
        }
    double dp_av = dp0 / (1.0 * o->nx * o->ny * o->nz);
    double dp_av1 = 1.0 / (dp_av + epsl);
    for (int k = 1; k <= o->nz; k++)
      for (int j = 1; j <= o->ny; j++)
        for (int i = 1; i <= o->nx; i++) o->rhybrid[IH(o, i, j, k)] = o->rhybrid[IH(o, i, j, k)] * dp_av1;
    free(pk);
  }
  int mpatch = (int)lround(p->hybrid_para[3]);
  for (int m = 1; m <= mpatch; m++) {
    int ib = (int)lround(p->hybrid_para[4 + (m - 1) * 6]);
    int ie = (int)lround(p->hybrid_para[7 + (m - 1) * 6]);
    int jb = (int)lround(p->hybrid_para[6 + (m - 1) * 6]);
    int je = (int)lround(p->hybrid_para[7 + (m - 1) * 6]);
    int kb = (int)lround(p->hybrid_para[8 + (m - 1) * 6]);
    int ke = (int)lround(p->hybrid_para[9 + (m - 1) * 6]);
    if (ib < 1) ib = 1;
    if (ie > o->nx) ie = o->nx;
    if (jb < 1) jb = 1;
    if (je > o->ny) je = o->ny;
    if (kb < 1) kb = 1;
    if (ke > o->nz) ke = o->nz;
    for (int k = kb; k <= ke; k++)
      for (int j = jb; j <= je; j++)
        for (int i = ib; i <= ie; i++) o->rhybrid[IH(o, i, j, k)] = o->rhybrid[IH(o, i, j, k)] + 100.0;
  }
  orc_exchange_xyz(o, o->rhybrid);
  free(P);
}

/* ---------------------------------------------------------------- inviscous */
/* gather one pencil (OCFD_inviscous.f90:83-92 / :123-132 / :161-170) */
static void gather_pencil(ocfd_oracle* o, int dir, int a, int b, double** pen) {
  int nn = dir == 0 ? o->nx : (dir == 1 ? o->ny : o->nz);
  const double* src[8];
  src[0] = o->cc; src[1] = o->d; src[2] = o->u; src[3] = o->v; src[4] = o->w;
  int mb = dir == 0 ? OCFD_M_AKX1 : (dir == 1 ? OCFD_M_AIX1 : OCFD_M_ASX1);
  src[5] = o->met[mb]; src[6] = o->met[mb + 1]; src[7] = o->met[mb + 2];
  for (int l = 1 - LAP; l <= nn + LAP; l++) {
    size_t h = dir == 0 ? IH(o, l, a, b) : (dir == 1 ? IH(o, a, l, b) : IH(o, a, b, l));
    for (int q = 0; q < 8; q++) pen[q][l] = src[q][h];
  }
}

static void compute_cc(ocfd_oracle* o) {
  /* OCFD_inviscous.f90:64-70 */
  for (size_t h = 0; h < o->nh; h++) o->cc[h] = sqrt(o->T[h]) / o->p.ma;
}

static void hybrid_index(ocfd_oracle* o, int dir, int a, int b, int nn, int* scm) {
  /* OCFD_inviscous.f90:76-81 / :116-121 / :154-159 */
  for (int l = 0; l <= nn; l++) {
    size_t h0, h1;
    if (dir == 0) { h0 = IH(o, l, a, b); h1 = IH(o, l + 1, a, b); }
    else if (dir == 1) { h0 = IH(o, a, l, b); h1 = IH(o, a, l + 1, b); }
    else { h0 = IH(o, a, b, l); h1 = IH(o, a, b, l + 1); }
    double Rhb0 = fmax2(o->rhybrid[h0], o->rhybrid[h1]);
    scm[l] = set_hybrid_scheme(&o->p, Rhb0);
  }
}

static void pencil_ptrs(struct pwork* w, double** pen, double** fp, double** fm) {
  double* base[8] = {w->pc, w->pd, w->pu, w->pv, w->pw, w->pa1, w->pa2, w->pa3};
  for (int q = 0; q < 8; q++) pen[q] = base[q] + LAP - 1;
  for (int m = 0; m < 5; m++) { fp[m] = w->pfp[m] + LAP - 1; fm[m] = w->pfm[m] + LAP - 1; }
}

/* du_inviscous: OCFD_inviscous.f90:53-203.  Pencils are independent: OpenMP
 * over the pencils of one direction (the directions stay in order). */
void orc_du_inviscous(ocfd_oracle* o) {
  const ocfd_params* p = &o->p;
  double hx_1 = 1.0 / p->hx, hy_1 = 1.0 / p->hy, hz_1 = 1.0 / p->hz;
  compute_cc(o);
  int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int dir = 0; dir < 3; dir++) {
    int nn = dir == 0 ? nx : (dir == 1 ? ny : nz);
    int na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
    const int* bi = p->bound_index + 2 * dir;
    const int* sb = p->scheme_boundary + 2 * dir;
    double h_1 = dir == 0 ? hx_1 : (dir == 1 ? hy_1 : hz_1);
#pragma omp parallel for schedule(static)
    for (int b = 1; b <= nb; b++) {
      struct pwork* w = &o->pw[omp_get_thread_num()];
      double* pen[8];
      double *fp[5], *fm[5];
      pencil_ptrs(w, pen, fp, fm);
      for (int a = 1; a <= na; a++) {
        if (p->scheme_invis == OCFD_SCHEME_HYBRID) hybrid_index(o, dir, a, b, nn, w->scm);
        else memset(w->scm, 0, sizeof(int) * (nn + 1));
        gather_pencil(o, dir, a, b, pen);
        if (p->flux_splitting == OCFD_SPLIT_SW) split_sw(p, nn, pen[0], pen[1], pen[2], pen[3], pen[4], pen[5], pen[6], pen[7], fp, fm);
        else split_llf(p, nn, pen[0], pen[1], pen[2], pen[3], pen[4], pen[5], pen[6], pen[7], fp, fm);
        for (int m = 1; m <= 5; m++) {
          ocfd2d_flux1(p, fp[m - 1], w->ph1, nn, bi, w->scm, sb);
          ocfd2d_flux2(p, fm[m - 1], w->ph2, nn, bi, w->scm, sb);
          for (int l = 1; l <= nn; l++) {
            int i, j, k;
            if (dir == 0) { i = l; j = a; k = b; } else if (dir == 1) { i = a; j = l; k = b; } else { i = a; j = b; k = l; }
            size_t c = IF(o, i, j, k, m);
            double dd = (w->ph1[l] - w->ph1[l - 1] + w->ph2[l] - w->ph2[l - 1]) * h_1;
            if (dir == 0) o->du[c] = dd;
            else if (dir == 1) o->du[c] = o->du[c] + dd;
            else o->du[c] = -(o->du[c] + dd) * o->met[OCFD_M_AJAC][IH(o, i, j, k)];
          }
        }
      }
    }
  }
  if (p->if_mass_force == 1) {
    /* OCFD_inviscous.f90:189-201 */
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          size_t h = IH(o, i, j, k);
          double d = o->d[h];
          o->du[IF(o, i, j, k, 2)] = o->du[IF(o, i, j, k, 2)] + d * p->mass_force[0];
          o->du[IF(o, i, j, k, 3)] = o->du[IF(o, i, j, k, 3)] + d * p->mass_force[1];
          o->du[IF(o, i, j, k, 4)] = o->du[IF(o, i, j, k, 4)] + d * p->mass_force[2];
          o->du[IF(o, i, j, k, 5)] = o->du[IF(o, i, j, k, 5)] +
                                     d * (o->u[h] * p->mass_force[0] + o->v[h] * p->mass_force[1] + o->w[h] * p->mass_force[2]);
        }
  }
}

/* flux_x1: OCFD_inviscous_character.f90:313-364.  ff points at ff(0). */
static double flux_x1(const ocfd_params* p, int Ka, int Kb, const double* ff, const int* bi, int i, int nn, int ihy,
                      const int* sb) {
  if ((bi[0] == 0 || i > -Ka || sb[0] == -1) && (bi[1] == 0 || i <= nn - Kb || sb[1] == -1)) {
    return scheme_P(p, ff, ihy);
  } else if (i <= -Ka && bi[0] == 1 && sb[0] != -1) {
    if (sb[0] == 0) {
      if (i == 1) return (2.0 * ff[0] + 5.0 * ff[1] - ff[2]) / 6.0;
      if (i == 2) return hh_weno5P_boundary(ff, DEL_LIFT);
      return hh_weno5P(ff);
    } else if (sb[0] == 1) {
      return hh_weno5P(ff);
    }
  } else if (i > nn - Kb && bi[1] == 1 && sb[1] != -1) {
    if (sb[1] == 0) {
      if (i == nn - 1) return hh_weno5P_boundary(ff, DEL_RIGHT);
      return hh_weno5P(ff);
    } else if (sb[1] == 1) {
      return hh_weno5P(ff);
    }
  }
  return 0.0;
}

/* flux_x2: OCFD_inviscous_character.f90:367-416 */
static double flux_x2(const ocfd_params* p, int Ka, int Kb, const double* ff, const int* bi, int i, int nn, int ihy,
                      const int* sb) {
  if ((bi[0] == 0 || i > -Ka || sb[0] == -1) && (bi[1] == 0 || i <= nn - Kb || sb[1] == -1)) {
    return scheme_M(p, ff, ihy);
  } else if (i <= -Ka && bi[0] == 1 && sb[0] != -1) {
    if (sb[0] == 0) {
      if (i == 1) return hh_weno5M_boundary(ff, DEL_LIFT);
      return hh_weno5M(ff);
    } else if (sb[0] == 1) {
      return hh_weno5M(ff);
    }
  } else if (i > nn - Kb && bi[1] == 1 && sb[1] != -1) {
    if (sb[1] == 0) {
      if (i == nn - 1) return (2.0 * ff[1] + 5.0 * ff[0] - ff[-1]) / 6.0;
      if (i == nn - 2) return hh_weno5M_boundary(ff, DEL_RIGHT);
      return hh_weno5M(ff);
    } else if (sb[1] == 1) {
      return hh_weno5M(ff);
    }
  }
  return 0.0;
}

/* The L = S and R = S^-1 matrices of flux_charteric
 * (OCFD_inviscous_character.f90:205-248), row-major S[r*5+c]. */
static void char_matrices(double gamma, double u1, double v1, double w1, double c1, double a1, double a2, double a3,
                          double* S, double* S1) {
  double ss = sqrt(a1 * a1 + a2 * a2 + a3 * a3);
  double n1 = a1 / ss, n2 = a2 / ss, n3 = a3 / ss, l1, l2, l3;
  if (fabs(n3) <= fabs(n2)) {
    ss = sqrt(n1 * n1 + n2 * n2);
    l1 = -n2 / ss; l2 = n1 / ss; l3 = 0.0;
  } else {
    ss = sqrt(n1 * n1 + n3 * n3);
    l1 = -n3 / ss; l2 = 0.0; l3 = n1 / ss;
  }
  double m1 = n2 * l3 - n3 * l2, m2 = n3 * l1 - n1 * l3, m3 = n1 * l2 - n2 * l1;
  double un = u1 * n1 + v1 * n2 + w1 * n3;
  double ul = u1 * l1 + v1 * l2 + w1 * l3;
  double um = u1 * m1 + v1 * m2 + w1 * m3;
  double V2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5;
  double KK = (gamma - 1.0) / (c1 * c1);
  double KK1 = KK * 0.5;
  double X1 = 1.0 / (2.0 * c1);
  double H = V2 + 1.0 / KK;
  double L[25] = {1.0 - KK * V2, KK * u1, KK * v1, KK * w1, -KK,
                  -ul, l1, l2, l3, 0.0,
                  -um, m1, m2, m3, 0.0,
                  KK1 * V2 + X1 * un, -X1 * n1 - KK1 * u1, -X1 * n2 - KK1 * v1, -X1 * n3 - KK1 * w1, KK1,
                  KK1 * V2 - X1 * un, X1 * n1 - KK1 * u1, X1 * n2 - KK1 * v1, X1 * n3 - KK1 * w1, KK1};
  double R[25] = {1.0, 0.0, 0.0, 1.0, 1.0,
                  u1, l1, m1, u1 - c1 * n1, u1 + c1 * n1,
                  v1, l2, m2, v1 - c1 * n2, v1 + c1 * n2,
                  w1, l3, m3, w1 - c1 * n3, w1 + c1 * n3,
                  V2, ul, um, H - c1 * un, H + c1 * un};
  memcpy(S, L, sizeof(L));
  memcpy(S1, R, sizeof(R));
}

void orc_char_matrices(double gamma, const double uvwc[4], const double a123[3], double S[25], double S1[25]) {
  char_matrices(gamma, uvwc[0], uvwc[1], uvwc[2], uvwc[3], a123[0], a123[1], a123[2], S, S1);
}

/* flux_charteric: OCFD_inviscous_character.f90:162-310 */
static void flux_charteric(ocfd_oracle* o, int nn, double** hh, double** fp, double** fm, double** pen,
                           const int* bi, const int* scm, const int* sb) {
  const ocfd_params* p = &o->p;
  int Ka1 = p->ka1, Kb1 = p->kb1, Ka2 = p->ka2, Kb2 = p->kb2;
  const double *cc = pen[0], *uu = pen[2], *vv = pen[3], *ww = pen[4];
  const double *AA1 = pen[5], *AA2 = pen[6], *AA3 = pen[7];
  /* fpc(Ka1:Kb1,5), fmc(Ka2:Kb2,5) persist across faces, as in the reference */
  double fpc_s[5][16] = {{0}}, fmc_s[5][16] = {{0}};
  double S[25] = {0}, S1[25] = {0};
  int ia = (bi[0] == 0 || sb[0] != 0) ? 0 : 1;
  int ib = (bi[1] == 0 || sb[1] != 0) ? nn : nn - 1;
  for (int i = ia; i <= ib; i++) {
    double* fpc[5];
    double* fmc[5];
    for (int m = 0; m < 5; m++) { fpc[m] = fpc_s[m] + 8; fmc[m] = fmc_s[m] + 8; }
    if (scm[i] == 1) {
      for (int mm = Ka1; mm <= Kb1; mm++)
        for (int m = 0; m < 5; m++) fpc[m][mm] = fp[m][i + mm];
      for (int mm = Ka2; mm <= Kb2; mm++)
        for (int m = 0; m < 5; m++) fmc[m][mm] = fm[m][i + mm];
    } else {
      int Ka1h, Kb1h, Ka2h, Kb2h;
      if (scm[i] == 0) { Ka1h = Ka1; Kb1h = Kb1; Ka2h = Ka2; Kb2h = Kb2; }
      else if (scm[i] == 2) { Ka1h = -3; Kb1h = 3; Ka2h = -2; Kb2h = 4; }
      else { Ka1h = -2; Kb1h = 2; Ka2h = -1; Kb2h = 3; }
      double u1 = (uu[i] + uu[i + 1]) * 0.5;
      double v1 = (vv[i] + vv[i + 1]) * 0.5;
      double w1 = (ww[i] + ww[i + 1]) * 0.5;
      double c1 = (cc[i] + cc[i + 1]) * 0.5;
      double a1 = (AA1[i] + AA1[i + 1]) * 0.5;
      double a2 = (AA2[i] + AA2[i + 1]) * 0.5;
      double a3 = (AA3[i] + AA3[i + 1]) * 0.5;
      char_matrices(p->gamma, u1, v1, w1, c1, a1, a2, a3, S, S1);
      for (int mm = Ka1h; mm <= Kb1h; mm++) {
        int m = i + mm;
        for (int r = 0; r < 5; r++)
          fpc[r][mm] = S[r * 5 + 0] * fp[0][m] + S[r * 5 + 1] * fp[1][m] + S[r * 5 + 2] * fp[2][m] +
                       S[r * 5 + 3] * fp[3][m] + S[r * 5 + 4] * fp[4][m];
      }
      for (int mm = Ka2h; mm <= Kb2h; mm++) {
        int m = i + mm;
        for (int r = 0; r < 5; r++)
          fmc[r][mm] = S[r * 5 + 0] * fm[0][m] + S[r * 5 + 1] * fm[1][m] + S[r * 5 + 2] * fm[2][m] +
                       S[r * 5 + 3] * fm[3][m] + S[r * 5 + 4] * fm[4][m];
      }
    }
    double h0[5];
    for (int m = 0; m < 5; m++) {
      double h1 = flux_x1(p, Ka1, Kb1, fpc[m], bi, i, nn, scm[i], sb);
      double h2 = flux_x2(p, Ka2, Kb2, fmc[m], bi, i, nn, scm[i], sb);
      h0[m] = h1 + h2;
    }
    if (scm[i] == 1) {
      for (int m = 0; m < 5; m++) hh[m][i] = h0[m];
    } else {
      for (int r = 0; r < 5; r++)
        hh[r][i] = S1[r * 5 + 0] * h0[0] + S1[r * 5 + 1] * h0[1] + S1[r * 5 + 2] * h0[2] + S1[r * 5 + 3] * h0[3] +
                   S1[r * 5 + 4] * h0[4];
    }
  }
  if (bi[0] == 1 && sb[0] == 0)
    for (int m = 0; m < 5; m++)
      hh[m][0] = (2.0 * fp[m][1] + 5.0 * fp[m][2] - fp[m][3] + 2.0 * fm[m][3] - 7.0 * fm[m][2] + 11.0 * fm[m][1]) / 6.0;
  if (bi[1] == 1 && sb[1] == 0)
    for (int m = 0; m < 5; m++)
      hh[m][nn] = (2.0 * fp[m][nn - 2] - 7.0 * fp[m][nn - 1] + 11.0 * fp[m][nn] + 2.0 * fm[m][nn] +
                   5.0 * fm[m][nn - 1] - fm[m][nn - 2]) / 6.0;
}

/* du_inviscous_Character: OCFD_inviscous_character.f90:3-159 */
void orc_du_inviscous_character(ocfd_oracle* o) {
  const ocfd_params* p = &o->p;
  double hx_1 = 1.0 / p->hx, hy_1 = 1.0 / p->hy, hz_1 = 1.0 / p->hz;
  compute_cc(o);
  int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int dir = 0; dir < 3; dir++) {
    int nn = dir == 0 ? nx : (dir == 1 ? ny : nz);
    int na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
    const int* bi = p->bound_index + 2 * dir;
    const int* sb = p->scheme_boundary + 2 * dir;
    double h_1 = dir == 0 ? hx_1 : (dir == 1 ? hy_1 : hz_1);
#pragma omp parallel for schedule(static)
    for (int b = 1; b <= nb; b++) {
      struct pwork* w = &o->pw[omp_get_thread_num()];
      double* pen[8];
      double *fp[5], *fm[5];
      pencil_ptrs(w, pen, fp, fm);
      for (int a = 1; a <= na; a++) {
        if (p->scheme_invis == OCFD_SCHEME_HYBRID) hybrid_index(o, dir, a, b, nn, w->scm);
        else memset(w->scm, 0, sizeof(int) * (nn + 1));
        gather_pencil(o, dir, a, b, pen);
        if (p->flux_splitting == OCFD_SPLIT_SW) split_sw(p, nn, pen[0], pen[1], pen[2], pen[3], pen[4], pen[5], pen[6], pen[7], fp, fm);
        else split_llf(p, nn, pen[0], pen[1], pen[2], pen[3], pen[4], pen[5], pen[6], pen[7], fp, fm);
        flux_charteric(o, nn, w->phh, fp, fm, pen, bi, w->scm, sb);
        for (int m = 1; m <= 5; m++)
          for (int l = 1; l <= nn; l++) {
            int i, j, k;
            if (dir == 0) { i = l; j = a; k = b; } else if (dir == 1) { i = a; j = l; k = b; } else { i = a; j = b; k = l; }
            size_t c = IF(o, i, j, k, m);
            double dd = (w->phh[m - 1][l] - w->phh[m - 1][l - 1]) * h_1;
            if (dir == 0) o->du[c] = dd;
            else if (dir == 1) o->du[c] = o->du[c] + dd;
            else o->du[c] = -(o->du[c] + dd) * o->met[OCFD_M_AJAC][IH(o, i, j, k)];
          }
      }
    }
  }
  if (p->if_mass_force == 1) {
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          size_t h = IH(o, i, j, k);
          double d = o->d[h];
          o->du[IF(o, i, j, k, 2)] = o->du[IF(o, i, j, k, 2)] + d * p->mass_force[0];
          o->du[IF(o, i, j, k, 3)] = o->du[IF(o, i, j, k, 3)] + d * p->mass_force[1];
          o->du[IF(o, i, j, k, 4)] = o->du[IF(o, i, j, k, 4)] + d * p->mass_force[2];
          o->du[IF(o, i, j, k, 5)] = o->du[IF(o, i, j, k, 5)] +
                                     d * (o->u[h] * p->mass_force[0] + o->v[h] * p->mass_force[1] + o->w[h] * p->mass_force[2]);
        }
  }
}

void orc_flux1d(ocfd_oracle* o, int dir, int sign, const double* f1d, int n, const int* scm, double* hh) {
  const ocfd_params* p = &o->p;
  const int* bi = p->bound_index + 2 * dir;
  const int* sb = p->scheme_boundary + 2 * dir;
  if (sign > 0) ocfd2d_flux1(p, f1d + LAP - 1, hh, n, bi, scm, sb);
  else ocfd2d_flux2(p, f1d + LAP - 1, hh, n, bi, scm, sb);
}

/* ---------------------------------------------------------------- viscous */
/* comput_Amu: OCFD_viscous.f90:135-149 */
static void comput_amu(ocfd_oracle* o) {
  double Tsb = 110.4 / o->p.ref_amu_t0;
  double TmpR = 1.0 / o->p.re;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        double T = o->T[IH(o, i, j, k)];
        o->amu[I3(o, i, j, k)] = TmpR * (1.0 + Tsb) * sqrt(T * T * T) / (Tsb + T);
      }
}

/* du_viscous: OCFD_viscous.f90:29-131 */
void orc_du_viscous(ocfd_oracle* o) {
  const ocfd_params* p = &o->p;
  const double tmp2_3 = 2.0 / 3.0;
  double** g = o->g;
  double** M = o->met;
  comput_amu(o);
  orc_d0(o, 0, o->u, g[0]); orc_d0(o, 0, o->v, g[3]); orc_d0(o, 0, o->w, g[6]); orc_d0(o, 0, o->T, g[9]);
  orc_d0(o, 1, o->u, g[1]); orc_d0(o, 1, o->v, g[4]); orc_d0(o, 1, o->w, g[7]); orc_d0(o, 1, o->T, g[10]);
  orc_d0(o, 2, o->u, g[2]); orc_d0(o, 2, o->v, g[5]); orc_d0(o, 2, o->w, g[8]); orc_d0(o, 2, o->T, g[11]);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t c = I3(o, i, j, k), h = IH(o, i, j, k);
        double Akx = M[OCFD_M_AKX][h], Aky = M[OCFD_M_AKY][h], Akz = M[OCFD_M_AKZ][h];
        double Aix = M[OCFD_M_AIX][h], Aiy = M[OCFD_M_AIY][h], Aiz = M[OCFD_M_AIZ][h];
        double Asx = M[OCFD_M_ASX][h], Asy = M[OCFD_M_ASY][h], Asz = M[OCFD_M_ASZ][h];
        double uk = g[0][c], ui = g[1][c], us = g[2][c], vk = g[3][c], vi = g[4][c], vs = g[5][c];
        double wk = g[6][c], wi = g[7][c], ws = g[8][c], Tk = g[9][c], Ti = g[10][c], Ts = g[11][c];
        double ux = uk * Akx + ui * Aix + us * Asx;
        double vx = vk * Akx + vi * Aix + vs * Asx;
        double wx = wk * Akx + wi * Aix + ws * Asx;
        double Tx = Tk * Akx + Ti * Aix + Ts * Asx;
        double uy = uk * Aky + ui * Aiy + us * Asy;
        double vy = vk * Aky + vi * Aiy + vs * Asy;
        double wy = wk * Aky + wi * Aiy + ws * Asy;
        double Ty = Tk * Aky + Ti * Aiy + Ts * Asy;
        double uz = uk * Akz + ui * Aiz + us * Asz;
        double vz = vk * Akz + vi * Aiz + vs * Asz;
        double wz = wk * Akz + wi * Aiz + ws * Asz;
        double Tz = Tk * Akz + Ti * Aiz + Ts * Asz;
        double div = ux + vy + wz;
        double Amu1 = o->amu[c];
        double Amuk = p->cp * o->amu[c] / p->pr;
        double s11 = (2.0 * ux - tmp2_3 * div) * Amu1;
        double s22 = (2.0 * vy - tmp2_3 * div) * Amu1;
        double s33 = (2.0 * wz - tmp2_3 * div) * Amu1;
        double s12 = (uy + vx) * Amu1;
        double s13 = (uz + wx) * Amu1;
        double s23 = (vz + wy) * Amu1;
        double uu = o->u[h], vv = o->v[h], ww = o->w[h];
        double E1 = uu * s11 + vv * s12 + ww * s13 + Amuk * Tx;
        double E2 = uu * s12 + vv * s22 + ww * s23 + Amuk * Ty;
        double E3 = uu * s13 + vv * s23 + ww * s33 + Amuk * Tz;
        for (int d = 0; d < 3; d++) {
          int mb = OCFD_M_AKX1 + 3 * d;
          double A1 = M[mb][h], A2 = M[mb + 1][h], A3 = M[mb + 2][h];
          double* Ev = o->ev[d];
          Ev[h + 0 * o->nh] = A1 * s11 + A2 * s12 + A3 * s13;
          Ev[h + 1 * o->nh] = A1 * s12 + A2 * s22 + A3 * s23;
          Ev[h + 2 * o->nh] = A1 * s13 + A2 * s23 + A3 * s33;
          Ev[h + 3 * o->nh] = A1 * E1 + A2 * E2 + A3 * E3;
        }
      }
  for (int m = 1; m <= 4; m++) {
    double* E1 = o->ev[0] + (size_t)(m - 1) * o->nh;
    double* E2 = o->ev[1] + (size_t)(m - 1) * o->nh;
    double* E3 = o->ev[2] + (size_t)(m - 1) * o->nh;
    exchange_x(o, E1);
    exchange_y(o, E2);
    exchange_z(o, E3);
    orc_d0(o, 0, E1, g[0]);
    orc_d0(o, 1, E2, g[1]);
    orc_d0(o, 2, E3, g[2]);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= o->nz; k++)
      for (int j = 1; j <= o->ny; j++)
        for (int i = 1; i <= o->nx; i++) {
          size_t c = I3(o, i, j, k);
          o->du[IF(o, i, j, k, m + 1)] =
              o->du[IF(o, i, j, k, m + 1)] + (g[0][c] + g[1][c] + g[2][c]) * M[OCFD_M_AJAC][IH(o, i, j, k)];
        }
  }
}

/* ---------------------------------------------------------------- RK3 + primitives */
/* OCFD_time_adv_RK3: OCFD_Time_Adv.f90:4-36 */
void orc_rk3(ocfd_oracle* o, int krk) {
  const double Ralfa[3] = {1.0, 3.0 / 4.0, 1.0 / 3.0}, Rbeta[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  double dt = o->p.dt;
  size_t n5 = 5 * o->n;
  if (krk == 1) {
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < n5; c++) o->f[c] = o->fn[c] + dt * o->du[c];
  } else {
    double a = Ralfa[krk - 1], b = Rbeta[krk - 1];
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < n5; c++) o->f[c] = a * o->fn[c] + b * (o->f[c] + dt * o->du[c]);
  }
}

/* comput_duvwT + handle_NegativeT: OCFD_Time_Adv.f90:40-63,
 * OCFD_handle_NegativeT.f90:1-17 (in-place, i fastest). */
int orc_duvwt(ocfd_oracle* o) {
  int num_negt = 0;
  const double Cv = o->p.cv;
  size_t sy = o->nxh, sz = (size_t)o->nxh * o->nyh;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t h = IH(o, i, j, k);
        double f1 = o->f[IF(o, i, j, k, 1)], f2 = o->f[IF(o, i, j, k, 2)], f3 = o->f[IF(o, i, j, k, 3)];
        double f4 = o->f[IF(o, i, j, k, 4)], f5 = o->f[IF(o, i, j, k, 5)];
        o->d[h] = f1;
        o->u[h] = f2 / f1;
        o->v[h] = f3 / f1;
        o->w[h] = f4 / f1;
        o->T[h] = (f5 - (f2 * o->u[h] + f3 * o->v[h] + f4 * o->w[h]) * 0.5) / (f1 * Cv);
        if (o->T[h] <= 0) {
          double* T = o->T;
          T[h] = (T[h + 1] + T[h - 1] + T[h + sy] + T[h - sy] + T[h + sz] + T[h - sz]) / 6.0;
          num_negt = num_negt + 1;
          if (num_negt > 10) return -1;
        }
      }
  return num_negt;
}

/* ---------------------------------------------------------------- filter */
/* filter_x3d / filter_y3d / filter_z3d: OCFD_filtering.f90:73-183 */
static void filter_dir(ocfd_oracle* o, int dir, double* f0, double s0, int lo[3], int hi[3]) {
  const double d0 = 0.243527493120, d1 = -0.204788880640, d2 = 0.120007591680, d3 = -0.045211119360,
               d4 = 0.008228661760;
  int nn = dir == 0 ? o->nx : (dir == 1 ? o->ny : o->nz);
  int b1 = lo[dir], e1 = hi[dir];
  if (!o->p.iperiodic[dir]) {
    if (b1 < 6) b1 = 6;
    if (e1 > nn - 5) e1 = nn - 5;
  }
  ptrdiff_t s = dir == 0 ? 1 : (dir == 1 ? (ptrdiff_t)o->nxh : (ptrdiff_t)o->nxh * o->nyh);
  for (int m = 1; m <= 5; m++) {
    for (int k = 1; k <= o->nz; k++)
      for (int j = 1; j <= o->ny; j++)
        for (int i = 1; i <= o->nx; i++) f0[IH(o, i, j, k)] = o->f[IF(o, i, j, k, m)];
    if (dir == 0) exchange_x(o, f0); else if (dir == 1) exchange_y(o, f0); else exchange_z(o, f0);
    int kb = dir == 2 ? b1 : lo[2], ke = dir == 2 ? e1 : hi[2];
    int jb = dir == 1 ? b1 : lo[1], je = dir == 1 ? e1 : hi[1];
    int ib = dir == 0 ? b1 : lo[0], ie = dir == 0 ? e1 : hi[0];
    for (int k = kb; k <= ke; k++)
      for (int j = jb; j <= je; j++)
        for (int i = ib; i <= ie; i++) {
          const double* q = f0 + IH(o, i, j, k);
          o->f[IF(o, i, j, k, m)] =
              q[0] - s0 * (d0 * q[0] + d1 * (q[-s] + q[s]) + d2 * (q[-2 * s] + q[2 * s]) + d3 * (q[-3 * s] + q[3 * s]) +
                           d4 * (q[-4 * s] + q[4 * s]));
        }
  }
}

/* filter_x3d_shock / _y3d_shock / _z3d_shock: OCFD_filtering.f90:188-363 */
static void filter_dir_shock(ocfd_oracle* o, int dir, double* f0, double* P, double s0, double rth, int lo[3],
                             int hi[3]) {
  const double c1 = -0.210383, c2 = 0.039617;
  int nn = dir == 0 ? o->nx : (dir == 1 ? o->ny : o->nz);
  int b1 = lo[dir], e1 = hi[dir];
  if (!o->p.iperiodic[dir]) {
    if (b1 < 4) b1 = 4;
    if (e1 > nn - 3) e1 = nn - 3;
  }
  ptrdiff_t s = dir == 0 ? 1 : (dir == 1 ? (ptrdiff_t)o->nxh : (ptrdiff_t)o->nxh * o->nyh);
  double g1 = o->p.gamma - 1.0;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        double f1 = o->f[IF(o, i, j, k, 1)], f2 = o->f[IF(o, i, j, k, 2)], f3 = o->f[IF(o, i, j, k, 3)];
        double f4 = o->f[IF(o, i, j, k, 4)], f5 = o->f[IF(o, i, j, k, 5)];
        P[IH(o, i, j, k)] = (f5 - 0.5 * (f2 * f2 + f3 * f3 + f4 * f4) / f1) * g1;
      }
  if (dir == 0) exchange_x(o, P); else if (dir == 1) exchange_y(o, P); else exchange_z(o, P);
  double* sc0 = (double*)malloc((size_t)(nn + 2) * sizeof(double)); /* sc0(0:nn+1) */
  for (int m = 1; m <= 5; m++) {
    for (int k = 1; k <= o->nz; k++)
      for (int j = 1; j <= o->ny; j++)
        for (int i = 1; i <= o->nx; i++) f0[IH(o, i, j, k)] = o->f[IF(o, i, j, k, m)];
    if (dir == 0) exchange_x(o, f0); else if (dir == 1) exchange_y(o, f0); else exchange_z(o, f0);
    /* transverse loops over the filter box, pencil along dir */
    int ta0 = dir == 0 ? 1 : 0, tb0 = dir == 2 ? 1 : 2; /* transverse dims */
    for (int b = lo[tb0]; b <= hi[tb0]; b++)
      for (int a = lo[ta0]; a <= hi[ta0]; a++) {
        int ijk[3];
        ijk[ta0] = a; ijk[tb0] = b;
        for (int l = b1 - 1; l <= e1 + 1; l++) {
          ijk[dir] = l;
          const double* pp = P + IH(o, ijk[0], ijk[1], ijk[2]);
          double dp0 = 0.25 * (-pp[s] + 2.0 * pp[0] - pp[-s]);
          double dp1 = 0.25 * (-pp[2 * s] + 2.0 * pp[s] - pp[0]);
          double dp2 = 0.25 * (-pp[0] + 2.0 * pp[-s] - pp[-2 * s]);
          double ri = 0.5 * (sq(dp0 - dp1) + sq(dp0 - dp2)) / (pp[0] * pp[0]) + 1.0e-16;
          sc0[l] = 0.5 * (1.0 - rth / ri + fabs(1.0 - rth / ri));
        }
        for (int l = b1; l <= e1; l++) {
          ijk[dir] = l;
          double sc1 = 0.5 * (sc0[l] + sc0[l + 1]);
          double sc2 = 0.5 * (sc0[l] + sc0[l - 1]);
          const double* q = f0 + IH(o, ijk[0], ijk[1], ijk[2]);
          o->f[IF(o, ijk[0], ijk[1], ijk[2], m)] =
              q[0] - s0 * (sc1 * (c1 * (q[s] - q[0]) + c2 * (q[2 * s] - q[-s])) -
                           sc2 * (c1 * (q[0] - q[-s]) + c2 * (q[s] - q[-2 * s])));
        }
      }
  }
  free(sc0);
}

/* filtering: OCFD_filtering.f90:4-70 */
void orc_filtering(ocfd_oracle* o) {
  const ocfd_params* p = &o->p;
  int any = 0;
  for (int m = 0; m < p->nfiltering; m++)
    if (o->istep % (int)lround(p->filter_para[m][0]) == 0) any = 1;
  if (!any) return;
  double* f0 = alloc_fill(o->nh, 0.0);
  double* P = alloc_fill(o->nh, 0.0);
  for (int m = 0; m < p->nfiltering; m++) {
    const double* F = p->filter_para[m];
    if (o->istep % (int)lround(F[0]) != 0) continue;
    int fx = (int)lround(F[1]), fy = (int)lround(F[2]), fz = (int)lround(F[3]);
    int lo[3] = {(int)lround(F[4]), (int)lround(F[6]), (int)lround(F[8])};
    int hi[3] = {(int)lround(F[5]), (int)lround(F[7]), (int)lround(F[9])};
    int nn[3] = {o->nx, o->ny, o->nz};
    for (int d = 0; d < 3; d++) {
      if (lo[d] < 1) lo[d] = 1;
      if (hi[d] > nn[d]) hi[d] = nn[d];
    }
    int scheme = (int)lround(F[10]);
    double s0 = F[11], rth = F[12];
    int on[3] = {fx, fy, fz};
    for (int d = 0; d < 3; d++) {
      if (on[d] != 1) continue;
      if (scheme == 1) filter_dir(o, d, f0, s0, lo, hi);
      else if (scheme == 2) filter_dir_shock(o, d, f0, P, s0, rth, lo, hi);
    }
  }
  free(f0);
  free(P);
}

/* ---------------------------------------------------------------- the step */
/* One pass of the NS_solver time loop: OCFD_NS_Solver.f90:21-67 */
int orc_step(ocfd_oracle* o) {
  const ocfd_params* p = &o->p;
  memcpy(o->fn, o->f, 5 * o->n * sizeof(double));
  for (int krk = 1; krk <= 3; krk++) {
    orc_halo_prims(o);
    if (krk == 1 && p->scheme_invis == OCFD_SCHEME_HYBRID) orc_comput_rhybrid(o);
    if (p->if_scheme_character == 0) orc_du_inviscous(o);
    else orc_du_inviscous_character(o);
    if (p->if_viscous == 1) orc_du_viscous(o);
    orc_rk3(o, krk);
    if (orc_duvwt(o) < 0) return -1;
    orc_bc(o);
  }
  o->istep = o->istep + 1;
  o->tt = o->tt + p->dt;
  orc_filtering(o);
  return 0;
}

/* ---------------------------------------------------------------- diagnostics */
/* show_flow_msg sums: OCFD_Time_Adv.f90:65-104 */
void orc_show_flow_msg(ocfd_oracle* o, double E0[3]) {
  const ocfd_params* p = &o->p;
  double p00 = 1.0 / (p->gamma * p->ma * p->ma);
  double tmp1 = 1.0 - p->gamma;
  double E1[3] = {0.0, 0.0, 0.0};
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t h = IH(o, i, j, k);
        double tmp0 = 1.0 / o->met[OCFD_M_AJAC][h];
        double d = o->d[h], u = o->u[h], v = o->v[h], w = o->w[h];
        E1[0] = E1[0] + o->f[IF(o, i, j, k, 5)] * tmp0;
        E1[1] = E1[1] + d * (u * u + v * v + w * w) * 0.5 * tmp0;
        E1[2] = E1[2] + p00 * pow(d, tmp1) * o->T[h] * tmp0;
      }
  double N = (double)(o->nx * o->ny * o->nz);
  for (int q = 0; q < 3; q++) E0[q] = E1[q] / N;
}

/* ana_getQ: OCFD_ANA.f90:127-171 (g[0..8] hold uk ui us vk vi vs wk wi ws) */
void orc_ana_q(ocfd_oracle* o, double* q) {
  double** g = o->g;
  double** M = o->met;
  orc_exchange_xyz(o, o->u);
  orc_exchange_xyz(o, o->v);
  orc_exchange_xyz(o, o->w);
  orc_d0(o, 0, o->u, g[0]); orc_d0(o, 0, o->v, g[3]); orc_d0(o, 0, o->w, g[6]);
  orc_d0(o, 1, o->u, g[1]); orc_d0(o, 1, o->v, g[4]); orc_d0(o, 1, o->w, g[7]);
  orc_d0(o, 2, o->u, g[2]); orc_d0(o, 2, o->v, g[5]); orc_d0(o, 2, o->w, g[8]);
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t c = I3(o, i, j, k), h = IH(o, i, j, k);
        double Akx = M[OCFD_M_AKX][h], Aky = M[OCFD_M_AKY][h], Akz = M[OCFD_M_AKZ][h];
        double Aix = M[OCFD_M_AIX][h], Aiy = M[OCFD_M_AIY][h], Aiz = M[OCFD_M_AIZ][h];
        double Asx = M[OCFD_M_ASX][h], Asy = M[OCFD_M_ASY][h], Asz = M[OCFD_M_ASZ][h];
        double ux = g[0][c] * Akx + g[1][c] * Aix + g[2][c] * Asx;
        double vx = g[3][c] * Akx + g[4][c] * Aix + g[5][c] * Asx;
        double wx = g[6][c] * Akx + g[7][c] * Aix + g[8][c] * Asx;
        double uy = g[0][c] * Aky + g[1][c] * Aiy + g[2][c] * Asy;
        double vy = g[3][c] * Aky + g[4][c] * Aiy + g[5][c] * Asy;
        double wy = g[6][c] * Aky + g[7][c] * Aiy + g[8][c] * Asy;
        double uz = g[0][c] * Akz + g[1][c] * Aiz + g[2][c] * Asz;
        double vz = g[3][c] * Akz + g[4][c] * Aiz + g[5][c] * Asz;
        double wz = g[6][c] * Akz + g[7][c] * Aiz + g[8][c] * Asz;
        q[c] = ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy;
      }
}

/* ana_time_average: OCFD_ANA.f90:34-125, the running-mean update of the
 * means held by the caller (5 interior arrays), K samples so far */
void orc_ana_time_average(ocfd_oracle* o, double* mean, int K) {
  const double* Q[5] = {o->d, o->u, o->v, o->w, o->T};
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t c = I3(o, i, j, k), h = IH(o, i, j, k);
        for (int a = 0; a < 5; a++) mean[c + a * o->n] = (K * mean[c + a * o->n] + Q[a][h]) / (K + 1.0);
      }
}

/* Ana_corner: OCFD_ANA.f90:316-384 for one rank (npx = npx0 - 1) */
void orc_ana_corner(ocfd_oracle* o, double* out) {
  double** M = o->met;
  const double p00 = 1.0 / (o->p.gamma * o->p.ma * o->p.ma);
  for (int i = 1; i <= o->nx; i++) {
    double sx, sy;
    if (i < o->nx) {
      sx = M[OCFD_M_AXX][IH(o, i + 1, 1, 1)] - M[OCFD_M_AXX][IH(o, i, 1, 1)];
      sy = M[OCFD_M_AYY][IH(o, i + 1, 1, 1)] - M[OCFD_M_AYY][IH(o, i, 1, 1)];
    } else {
      sx = M[OCFD_M_AXX][IH(o, o->nx, 1, 1)] - M[OCFD_M_AXX][IH(o, o->nx - 1, 1, 1)];
      sy = M[OCFD_M_AYY][IH(o, o->nx, 1, 1)] - M[OCFD_M_AYY][IH(o, o->nx - 1, 1, 1)];
    }
    double tmp = 1.0 / sqrt(sx * sx + sy * sy);
    sx = sx * tmp;
    sy = sy * tmp;
    double us = 0.0, Ts = 0.0, ps = 0.0;
    for (int k = 1; k <= o->nz; k++) {
      size_t c2 = IH(o, i, 2, k), c1 = IH(o, i, 1, k);
      us = us + o->u[c2] * sx + o->v[c2] * sy;
      Ts = Ts + o->T[c2];
      ps = ps + p00 * o->d[c1] * o->T[c1];
    }
    double r = 1.0 / o->nz;
    out[i - 1] = us * r;
    out[o->nx + i - 1] = Ts * r;
    out[2 * o->nx + i - 1] = ps * r;
  }
}

/* ana_box: OCFD_ANA.f90:178-311 */
void orc_ana_box(ocfd_oracle* o, double out[20]) {
  const ocfd_params* p = &o->p;
  double** g = o->g;
  double** M = o->met;
  orc_exchange_xyz(o, o->u);
  orc_d0(o, 0, o->u, g[0]); orc_d0(o, 1, o->u, g[1]); orc_d0(o, 2, o->u, g[2]);
  orc_exchange_xyz(o, o->v);
  orc_d0(o, 0, o->v, g[3]); orc_d0(o, 1, o->v, g[4]); orc_d0(o, 2, o->v, g[5]);
  orc_exchange_xyz(o, o->w);
  orc_d0(o, 0, o->w, g[6]); orc_d0(o, 1, o->w, g[7]); orc_d0(o, 2, o->w, g[8]);
  comput_amu(o);
  double c_aver = 0, d_aver = 0, Amu_aver = 0, T_aver = 0, u_rms = 0, v_rms = 0, w_rms = 0, Ux_rms = 0;
  double Ux_skewness = 0, Ux_flatness = 0, u_skewness = 0, u_flatness = 0, E_kinetic = 0, ens = 0;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) {
        size_t c = I3(o, i, j, k), h = IH(o, i, j, k);
        double Akx = M[OCFD_M_AKX][h], Aky = M[OCFD_M_AKY][h], Akz = M[OCFD_M_AKZ][h];
        double Aix = M[OCFD_M_AIX][h], Aiy = M[OCFD_M_AIY][h], Aiz = M[OCFD_M_AIZ][h];
        double Asx = M[OCFD_M_ASX][h], Asy = M[OCFD_M_ASY][h], Asz = M[OCFD_M_ASZ][h];
        double ux = g[0][c] * Akx + g[1][c] * Aix + g[2][c] * Asx;
        double uy = g[0][c] * Aky + g[1][c] * Aiy + g[2][c] * Asy;
        double uz = g[0][c] * Akz + g[1][c] * Aiz + g[2][c] * Asz;
        double vx = g[3][c] * Akx + g[4][c] * Aix + g[5][c] * Asx;
        double vy = g[3][c] * Aky + g[4][c] * Aiy + g[5][c] * Asy;
        double vz = g[3][c] * Akz + g[4][c] * Aiz + g[5][c] * Asz;
        double wx = g[6][c] * Akx + g[7][c] * Aix + g[8][c] * Asx;
        double wy = g[6][c] * Aky + g[7][c] * Aiy + g[8][c] * Asy;
        double wz = g[6][c] * Akz + g[7][c] * Aiz + g[8][c] * Asz;
        (void)wz;
        double u = o->u[h], v = o->v[h], w = o->w[h], d = o->d[h], T = o->T[h];
        c_aver = c_aver + sqrt(T) / p->ma;
        d_aver = d_aver + d;
        Amu_aver = Amu_aver + o->amu[c];
        T_aver = T_aver + T;
        u_rms = u_rms + u * u;
        v_rms = v_rms + v * v;
        w_rms = w_rms + w * w;
        Ux_rms = Ux_rms + ux * ux;
        Ux_skewness = Ux_skewness + ux * ux * ux; /* ux**3 = (ux*ux)*ux */
        Ux_flatness = Ux_flatness + sq(ux) * sq(ux); /* ux**4 = (ux*ux)*(ux*ux) */
        u_skewness = u_skewness + u * u * u;
        u_flatness = u_flatness + sq(u) * sq(u);
        E_kinetic = E_kinetic + (u * u + v * v + w * w) * d * 0.5;
        ens = ens + sq(wy - vz) + sq(uz - wx) + sq(vx - uy);
      }
  double N = (double)(o->nx * o->ny * o->nz);
  u_rms /= N; v_rms /= N; w_rms /= N; Ux_rms /= N; Ux_skewness /= N; Ux_flatness /= N; d_aver /= N;
  c_aver /= N; Amu_aver /= N; E_kinetic /= N; T_aver /= N; u_skewness /= N; u_flatness /= N;
  ens = 0.5 * (ens / N);
  double VV_rms = sqrt((u_rms + v_rms + w_rms) / 3.0);
  double Amt = sqrt(u_rms + v_rms + w_rms) / c_aver;
  u_rms = sqrt(u_rms); v_rms = sqrt(v_rms); w_rms = sqrt(w_rms); Ux_rms = sqrt(Ux_rms);
  double Alamda = VV_rms / Ux_rms;
  double Alamdax = u_rms / Ux_rms;
  double Re_lamda = VV_rms * Alamda * d_aver / Amu_aver;
  double Re_lamdax = VV_rms * Alamdax * d_aver / Amu_aver;
  Ux_skewness = Ux_skewness / (Ux_rms * Ux_rms * Ux_rms);
  Ux_flatness = Ux_flatness / (sq(Ux_rms) * sq(Ux_rms));
  u_skewness = u_skewness / (u_rms * u_rms * u_rms);
  u_flatness = u_flatness / (sq(u_rms) * sq(u_rms));
  double d_rms = 0.0;
  for (int k = 1; k <= o->nz; k++)
    for (int j = 1; j <= o->ny; j++)
      for (int i = 1; i <= o->nx; i++) d_rms = d_rms + sq(o->d[IH(o, i, j, k)] - d_aver);
  d_rms = sqrt(d_rms / N);
  double r[20] = {o->tt, Re_lamda, Re_lamdax, Amt, VV_rms, u_rms, v_rms, w_rms, u_skewness, u_flatness,
                  Ux_skewness, Ux_flatness, E_kinetic, ens, d_rms, T_aver, Amu_aver, d_aver, Ux_rms, Alamdax};
  memcpy(out, r, sizeof(r));
}

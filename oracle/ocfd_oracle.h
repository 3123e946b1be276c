/*
 * ocfd_oracle.h -- CPU oracle for the OpenCFD-SC RHS / RK3 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a single-rank C restatement of the
 * reference's Fortran routines, compiled with -O2 -ffp-contract=off so that
 * every floating-point operation happens in the reference's order and without
 * FMA contraction (the reference's gfortran Release build, -O3
 * -funroll-all-loops with no -march, has none either).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the
 * checker; the GPU library never calls it.
 *
 * Parity status: the reference is Fortran 90 + MPI and no Fortran compiler or
 * MPI exists on the build or GPU machines, so the reference itself cannot be
 * run.  The reference ships no stored golden vectors.  The oracle is pinned
 * against the reference's own known-answer harnesses (test-dx-invis.f90:
 * scheme derivative of cos; test-dxyz0.f90: CD6/CD8 derivative of
 * cos*cos*cos; test_S in OCFD_inviscous_character.f90:420-443: S*S^-1 = I) and
 * against invariants (free-stream preservation, conservation of the periodic
 * sums).  Parity against a reference binary is therefore unpinned.
 */
#ifndef OCFD_ORACLE_H
#define OCFD_ORACLE_H
#include "ocfd_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ocfd_oracle ocfd_oracle;

/* Array ids for orc_array() */
enum {
  ORC_F = 0, ORC_FN, ORC_DU, ORC_AMU,
  ORC_D, ORC_U, ORC_V, ORC_W, ORC_T,
  ORC_RHYBRID,
  ORC_METRIC0 /* + OCFD_M_* */
};

void orc_default_params(ocfd_params* p);
int orc_set_parameters(ocfd_params* p);

ocfd_oracle* orc_create(const ocfd_params* p);
void orc_destroy(ocfd_oracle* o);
double* orc_array(ocfd_oracle* o, int id);
void orc_get_time(const ocfd_oracle* o, int* istep, double* tt);
void orc_set_time(ocfd_oracle* o, int istep, double tt);

/* init_mesh; x,y,z interior coordinates (Fortran order) or NULL for 'box'. */
void orc_init_mesh(ocfd_oracle* o, const double* x, const double* y, const double* z);
/* init_mesh for Iflag_Gridtype = GRID_AND_JACOBIAN3D: jac = interior Akx, Aky,
 * Akz, Aix, Aiy, Aiz, Asx, Asy, Asz, Ajac from the grid file (no
 * comput_Jacobian3d, OCFD_mesh.f90:24-26). */
void orc_init_mesh_jacobian(ocfd_oracle* o, const double* x, const double* y, const double* z,
                            const double* const jac[10]);
/* init3d from interior primitives + the initial OCFD_bc. */
void orc_init3d(ocfd_oracle* o, const double* const prims[5]);

void orc_exchange_xyz(ocfd_oracle* o, double* a);
void orc_halo_prims(ocfd_oracle* o);
void orc_comput_rhybrid(ocfd_oracle* o);
void orc_du_inviscous(ocfd_oracle* o);
void orc_du_inviscous_character(ocfd_oracle* o);
void orc_du_viscous(ocfd_oracle* o);
void orc_rk3(ocfd_oracle* o, int krk);
/* returns number of repaired points, or -1 when the reference would stop */
int orc_duvwt(ocfd_oracle* o);
void orc_bc(ocfd_oracle* o);
/* BC_BoundaryLayer / BC_SweptCorner boundary data (after orc_init_mesh):
 * inlet (ny,nz,5), upper (nx,nz,5), wall perturbation (nx,nz) -- each may be
 * NULL for zeros -- and the time factor's amplitudes / phases (mt each). */
void orc_set_bc_layer(ocfd_oracle* o, const double* inlet, const double* upper, const double* pertb, int mt,
                      double beta, const double* tm, const double* fait);
void orc_filtering(ocfd_oracle* o);
/* one full time step; returns 0 or -1 (negative-T stop) */
int orc_step(ocfd_oracle* o);
void orc_show_flow_msg(ocfd_oracle* o, double E0[3]);
void orc_ana_box(ocfd_oracle* o, double out[20]);
void orc_ana_q(ocfd_oracle* o, double* q);
void orc_ana_time_average(ocfd_oracle* o, double* mean, int K);
void orc_ana_corner(ocfd_oracle* o, double* out);

/* Scheme-level entry points for the known-answer harnesses.
 * f1d has n+2*LAP values (index 1-LAP..n+LAP), hh receives n+1 faces.
 * sign = +1: OCFD2d_flux1, -1: OCFD2d_flux2, with the parameters' scheme
 * and the direction dir's boundary settings. */
void orc_flux1d(ocfd_oracle* o, int dir, int sign, const double* f1d, int n, const int* scm, double* hh);
/* S and S^-1 of flux_charteric for one face state (test_S) */
void orc_char_matrices(double gamma, const double uvwc[4], const double a123[3], double S[25], double S1[25]);
/* OCFD_dx0/dy0/dz0 of a haloed array into an interior array */
void orc_d0(ocfd_oracle* o, int dir, const double* f, double* fx);

#ifdef __cplusplus
}
#endif
#endif

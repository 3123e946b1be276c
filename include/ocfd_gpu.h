/*
 * ocfd_gpu.h -- C ABI of the B200 (sm_100a) implementation of OpenCFD-SC's
 * right-hand side and RK3 time advance.
 *
 * The Fortran driver of OpenCFD-SC (opencfd.f90, OCFD_readpara, OCFD_init, the
 * opencfd2.in deck and the OCFD%08d.dat files) stays the host.  It owns the
 * parameters and the initial field; this library owns the flow state on the
 * GPU between synchronisation points (show / analysis / save steps).
 *
 * Every entry point below replaces one subroutine of the reference; the
 * reference routine is named in the comment as file:line (paths relative to
 * the OpenCFD-SC source tree).  The reference routines take no arguments and
 * work on module globals (flow_data, inviscous_data, viscous_data); here the
 * globals live in an opaque handle.
 *
 * Conventions
 *   - All functions return 0 on success and a negative OCFD_E* code on error,
 *     except where stated.  ocfd_gpu_last_error() returns a message.
 *   - Arrays cross the boundary in the reference's own Fortran layout:
 *       f(nx,ny,nz,5)                 f(i,j,k,m) at (i-1)+nx*((j-1)+ny*((k-1)+nz*(m-1)))
 *       haloed q(1-LAP:nx+LAP, ...)   q(i,j,k)   at (i+LAP-1)+NXH*((j+LAP-1)+NYH*(k+LAP-1))
 *     with NXH = nx+2*LAP etc. and LAP = 4 (OCFD_readpara.f90:35).
 *   - One handle = one solver instance with its own CUDA stream.  A handle is
 *     used from one host thread at a time; separate handles may be driven from
 *     separate threads.
 *   - Every call is asynchronous on the handle's stream unless it returns host
 *     data (download, diagnostics, negative-T count) or is ocfd_gpu_sync().
 */
#ifndef OCFD_GPU_H
#define OCFD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OCFD_LAP 4
#define OCFD_ABI_VERSION 1

/* Scheme / splitting / boundary / grid enums: OCFD_parameters.f90:23-33 */
enum {
  OCFD_SCHEME_WENO5 = 1,
  OCFD_SCHEME_WENO7 = 2,
  OCFD_SCHEME_OMP6 = 3,
  OCFD_SCHEME_UD7L = 4,
  OCFD_SCHEME_CD6 = 5,
  OCFD_SCHEME_CD8 = 6,
  OCFD_SCHEME_HYBRID = 10,
  OCFD_SCHEME_USER = 99
};
enum { OCFD_SPLIT_SW = 1, OCFD_SPLIT_LLF = 2 };
enum {
  OCFD_BC_NONE = 0,
  OCFD_BC_BLUNT2D = 1,
  OCFD_BC_BOUNDARYLAYER = 2,
  OCFD_BC_SWEPTCORNER = 3,
  /* BC_User_Def (OCFD_BC.f90:141, slot OCFD_User_Def.f90:12-18).  This build
   * fills the slot with an isothermal no-slip wall at j=1 (T=bc_para[0]) and a
   * free stream (1,1,0,0,1) at j=ny, the wall modelled on the isothermal branch
   * of OCFD_BC_Boundarylayers.f90:129-133. */
  OCFD_BC_USER_DEF = 99
};
enum {
  OCFD_GRIDGEN = 0,
  OCFD_GRID1D = 10,
  OCFD_GRID2D_PLANE = 20,
  OCFD_GRID2D_AXIAL_SYMM = 21,
  OCFD_GRID3D = 30,
  OCFD_GRID_AND_JACOBIAN3D = 31
};
enum { OCFD_PRECISION_FP64 = 0, OCFD_PRECISION_MIXED = 1 };

/* Error codes */
enum {
  OCFD_OK = 0,
  OCFD_E_PARAM = -1,     /* unsupported or inconsistent parameter */
  OCFD_E_CUDA = -2,      /* CUDA runtime error (message via last_error) */
  OCFD_E_NEGT = -3,      /* > 10 negative-temperature points: the reference stops
                            (OCFD_handle_NegativeT.f90:13-16 / OCFD_Time_Adv.f90:118-121) */
  OCFD_E_STATE = -4,     /* call out of order (e.g. step before metrics) */
  OCFD_E_NOMEM = -5,
  OCFD_E_TIMEOUT = -6    /* a bounded device wait gave up: the results of the steps since the
                            last synchronisation are invalid (restart from a kept state); the
                            handle stages its face tiles with plain loads from then on */
};

/*
 * Parameters.  The first block mirrors the namelist /control_opencfd/
 * (OCFD_readpara.f90:14-22) with the reference defaults of :28-65; the second
 * block is filled by ocfd_set_parameters() exactly as set_parameters /
 * set_scheme_para do (OCFD_readpara.f90:261-341).  TYPE_Para and TYPE_Scheme:
 * OCFD_parameters.f90:55-90.
 */
typedef struct ocfd_params {
  int32_t nx, ny, nz;              /* nx_global, ny_global, nz_global        */
  int32_t lap;                     /* LAP, must be 4                         */
  int32_t iperiodic[3];            /* Iperiodic_X/Y/Z                        */
  int32_t iflag_gridtype;          /* Iflag_Gridtype                         */
  double periodic_span[3][3];      /* Periodic_ISpan, _JSpan, _KSpan         */
  int32_t scheme_invis;            /* Scheme_Invis (OCFD_SCHEME_*)           */
  int32_t scheme_vis;              /* Scheme_Vis (CD6 / CD8)                 */
  int32_t if_scheme_character;     /* IF_Scheme_Character                    */
  int32_t flux_splitting;          /* Flux_Splitting (SW / LLF)              */
  int32_t scheme_boundary[6];      /* Scheme_boundary(6): 0, 1 or -1         */
  int32_t if_viscous;              /* IF_Viscous                             */
  int32_t if_mass_force;           /* IF_Mass_Force                          */
  int32_t ibc;                     /* BoundaryCondition (OCFD_BC_*)          */
  int32_t ghost_cell[6];           /* Ghost_Cell(6)                          */
  int32_t nfiltering;              /* NFiltering (<= 10)                     */
  int32_t istep_show, istep_save;  /* Istep_Show, Istep_Save                 */
  int32_t precision;               /* OCFD_PRECISION_FP64 / _MIXED           */
  double ma, re, gamma, pr, ref_amu_t0, dt, end_time, aoa;
  double ud7l_diss;                /* UD7L_Diss                              */
  double mass_force[3];            /* Mass_Force(3)                          */
  double hybrid_para[100];         /* Hybrid_para(100)                       */
  double bc_para[100];             /* BC_Para(100)                           */
  double filter_para[10][100];     /* Filter_Para(100,10): filter_para[m][c] = Filter(c+1,m+1) */
  /* ---- derived: ocfd_set_parameters() ---- */
  double hx, hy, hz;               /* 1/(n_global-1)                          */
  double cv, cp;                   /* Cv = 1/(gamma(gamma-1)Ma^2), Cp = gamma Cv */
  double ud7l[8];                  /* Scheme%UD7L                            */
  int32_t bound_index[6];          /* Scheme%Bound_index(2,3) flattened (i-,i+,j-,j+,k-,k+) */
  int32_t ka1, kb1, ka2, kb2;      /* Scheme%Ka1.. stencil of F+(i+1/2), F-(i+1/2) */
  int32_t reserved[8];
} ocfd_params;

typedef struct ocfd_handle ocfd_handle;

/* Index of the 22 haloed metric arrays in ocfd_gpu_upload_metrics(), in the
 * order of flow_data (OCFD_parameters.f90:103-105). */
enum {
  OCFD_M_AXX = 0, OCFD_M_AYY, OCFD_M_AZZ,
  OCFD_M_AKX, OCFD_M_AKY, OCFD_M_AKZ, OCFD_M_AIX, OCFD_M_AIY, OCFD_M_AIZ,
  OCFD_M_ASX, OCFD_M_ASY, OCFD_M_ASZ, OCFD_M_AJAC,
  OCFD_M_AKX1, OCFD_M_AKY1, OCFD_M_AKZ1, OCFD_M_AIX1, OCFD_M_AIY1, OCFD_M_AIZ1,
  OCFD_M_ASX1, OCFD_M_ASY1, OCFD_M_ASZ1,
  OCFD_N_METRICS
};

/* ---------------------------------------------------------------------------
 * Host-side parameter handling
 * ------------------------------------------------------------------------- */

/* Fill p with the namelist defaults of OCFD_readpara.f90:28-65. */
void ocfd_default_params(ocfd_params* p);

/* set_parameters + set_scheme_para (OCFD_readpara.f90:261-341) for one rank
 * owning the whole grid.  Validates the configuration; returns OCFD_E_PARAM for
 * anything this library does not implement (SCHEME_USER, LAP != 4, grids
 * smaller than the stencils, BC_BoundaryLayer / BC_SweptCorner with a periodic
 * x or y direction). */
int ocfd_set_parameters(ocfd_params* p);

/* Bytes of device memory an instance with these parameters needs (admission). */
size_t ocfd_gpu_footprint(const ocfd_params* p);

/* ---------------------------------------------------------------------------
 * Instance lifetime.  Replaces allocate_flow_data / allocate_inviscous_data /
 * allocate_vicous_data (OCFD_NS_Solver.f90:93-151, OCFD_inviscous.f90:15-40,
 * OCFD_viscous.f90:16-25).  Haloed arrays start at 1.0 and Rhybrid at 0.0, as
 * in the reference.
 * ------------------------------------------------------------------------- */
int ocfd_gpu_create(const ocfd_params* p, int device, ocfd_handle** out);
void ocfd_gpu_destroy(ocfd_handle* h);
const char* ocfd_gpu_last_error(const ocfd_handle* h);
int ocfd_gpu_sync(ocfd_handle* h);
/* The handle's cudaStream_t, as void* (for callers that interleave their own work). */
void* ocfd_gpu_stream(ocfd_handle* h);

/* ---------------------------------------------------------------------------
 * Mesh and metrics (init time)
 * ------------------------------------------------------------------------- */

/* Upload the 22 haloed metric arrays computed by the host (init_mesh,
 * OCFD_mesh.f90:1-58).  metrics[OCFD_M_*] in Fortran haloed order. */
int ocfd_gpu_upload_metrics(ocfd_handle* h, const double* const metrics[OCFD_N_METRICS]);

/* init_mesh on the device (OCFD_mesh.f90:1-58): coordinates -> face-halo
 * exchange -> periodic span shift (updata_Axyz_periodic :109-185) ->
 * comput_Jacobian3d (:61-107) -> metric halos -> Jac_Ghost_boundary
 * (OCFD_GhostCell.f90:1-160,290-500) -> A?1 = A?/Ajac.
 * xyz: three interior coordinate arrays (nx,ny,nz) in Fortran order; NULL
 * means mesh_gen('box') (OCFD_mesh.f90:319-354). */
int ocfd_gpu_init_mesh(ocfd_handle* h, const double* x, const double* y, const double* z);

/* init_mesh for Iflag_Gridtype = GRID_AND_JACOBIAN3D (31): read_mesh3d reads
 * the metrics and the Jacobian from the grid file with the coordinates
 * (OCFD_mesh.f90:187-217) and init_mesh skips comput_Jacobian3d (:24-26); the
 * rest is ocfd_gpu_init_mesh.  jac: ten interior (nx,ny,nz) arrays in Fortran
 * order, Akx, Aky, Akz, Aix, Aiy, Aiz, Asx, Asy, Asz, Ajac. */
int ocfd_gpu_init_mesh_jacobian(ocfd_handle* h, const double* x, const double* y, const double* z,
                                const double* const jac[10]);

/* Download the 22 haloed metric arrays (for checks and for the host's analysis). */
int ocfd_gpu_download_metrics(ocfd_handle* h, double* const metrics[OCFD_N_METRICS]);

/* Bit m set: metric array m (OCFD_M_*) holds +0.0 at every point the kernels
 * read (interior and face halos), so its loads are skipped -- the off-diagonal
 * metrics of box and 1-D grids.  Known after init_mesh / upload_metrics.  No
 * counterpart in the reference (an internal optimisation made visible for
 * tests and byte accounting). */
unsigned int ocfd_gpu_metric_zero_mask(const ocfd_handle* h);

/* ---------------------------------------------------------------------------
 * State transfer (sync points of NS_solver: init3d, show, analysis, save)
 * ------------------------------------------------------------------------- */

/* Upload conserved f(nx,ny,nz,5) and/or the haloed primitives d,u,v,w,T
 * (either may be NULL).  istep/tt are the restart counters. */
int ocfd_gpu_upload_state(ocfd_handle* h, const double* f, const double* const prims[5],
                          int istep, double tt);
/* init3d (OCFD_init.f90:10-20): f from the interior primitives (d,u,v,w,T as
 * nx*ny*nz Fortran arrays), then OCFD_bc (OCFD_NS_Solver.f90:15). */
int ocfd_gpu_init3d(ocfd_handle* h, const double* const prims_interior[5], int istep, double tt);
/* Download f and/or haloed primitives (either may be NULL); synchronous. */
int ocfd_gpu_download_state(ocfd_handle* h, double* f, double* const prims[5]);
/* Download du(nx,ny,nz,5) (the right-hand side of the last stage); synchronous. */
int ocfd_gpu_download_du(ocfd_handle* h, double* du);
/* Download Rhybrid (haloed); synchronous. */
int ocfd_gpu_download_rhybrid(ocfd_handle* h, double* rh);
/* Current Istep and tt. */
int ocfd_gpu_get_time(ocfd_handle* h, int* istep, double* tt);

/* ---------------------------------------------------------------------------
 * The stage operators -- one per reference subroutine, same call order as
 * NS_solver (OCFD_NS_Solver.f90:21-78).
 * ------------------------------------------------------------------------- */

/* fn = f (OCFD_NS_Solver.f90:23-31). */
int ocfd_gpu_save_fn(ocfd_handle* h);
/* exchange_boundary_xyz(d,u,v,w,T) for one rank (OCFD_NS_Solver.f90:35-39,
 * OCFD_mpi.f90:183-233): periodic face halos, edges and corners untouched. */
int ocfd_gpu_halo_prims(ocfd_handle* h);
/* comput_Rhybrid (OCFD_SetHybrid.f90:17-152), sensor 1 or 2, patches, halo. */
int ocfd_gpu_rhybrid(ocfd_handle* h);
/* du_inviscous (OCFD_inviscous.f90:53-203). */
int ocfd_gpu_du_inviscous(ocfd_handle* h);
/* du_inviscous_Character (OCFD_inviscous_character.f90:3-159). */
int ocfd_gpu_du_inviscous_character(ocfd_handle* h);
/* du_viscous (OCFD_viscous.f90:29-131) incl. comput_Amu (:135-149). */
int ocfd_gpu_du_viscous(ocfd_handle* h);
/* OCFD_time_adv_RK3(KRK) (OCFD_Time_Adv.f90:4-36), krk in 1..3. */
int ocfd_gpu_rk3(ocfd_handle* h, int krk);
/* comput_duvwT + handle_NegativeT (OCFD_Time_Adv.f90:40-63,
 * OCFD_handle_NegativeT.f90:1-17).  Synchronous: *num_negt receives the number
 * of repaired points; returns OCFD_E_NEGT when it exceeds 10. */
int ocfd_gpu_duvwt(ocfd_handle* h, int* num_negt);
/* OCFD_bc (OCFD_BC.f90:2-99): BC dispatch, f refresh on the six faces,
 * Flow_Ghost_boundary (OCFD_GhostCell.f90:9-14,164-286, user ghost cells
 * OCFD_GhostCell_UserDef.f90:13-20). */
int ocfd_gpu_bc(ocfd_handle* h);

/* Boundary data of BC_BoundaryLayer (ocfd_bc_BoundaryLayer,
 * OCFD_BC_Boundarylayers.f90:17-169) and BC_SweptCorner (ocfd_bc_swept_corner,
 * :443-618), which the reference builds at its first BC call:
 * init_bcdata_boundarylayer (:171-270) reads flow1d/flow2d-inlet.dat and
 * -upper.dat, init_bc_wall_perturbation (:313-400) and get_ht_multifrequancy
 * (:404-440) draw random phases.  The host passes the results; the library
 * computes init_bc_nonRef (:273-311) from the mesh.  Arrays in Fortran order,
 * NULL for zeros:
 *   inlet (ny,nz,5)  d,u,v,w,T at i = 1 (used when BC_Para(1) != 0, and always
 *                    by BC_SweptCorner)
 *   upper (nx,nz,5)  at j = ny (used when BC_Para(2) != 0)
 *   pertb (nx,nz)    wall blowing/suction shape wall_pertb
 *   mt, beta, tm, fait: time factor ht = sum_m tm[m-1] sin(m beta tt + 2 pi fait[m-1])
 *                    (beta <= 0: ht = 1)
 * Call after the mesh is set.  With the free-stream inlet and upper boundary
 * and no perturbation it may be omitted (the first BC call sets the mask).
 * A wall perturbation that varies in time disables the captured step graphs. */
typedef struct ocfd_bc_layer {
  const double* inlet;
  const double* upper;
  const double* pertb;
  int32_t mt;
  double beta;
  const double* tm;
  const double* fait;
} ocfd_bc_layer;
int ocfd_gpu_set_bc_layer(ocfd_handle* h, const ocfd_bc_layer* d);
/* filtering(f) (OCFD_filtering.f90:4-70) for the current Istep. */
int ocfd_gpu_filter(ocfd_handle* h);
/* Istep += 1, tt += dt (OCFD_NS_Solver.f90:64-65). */
int ocfd_gpu_advance_clock(ocfd_handle* h);

/* nsteps full time steps of NS_solver (OCFD_NS_Solver.f90:21-78 without
 * show/analysis/save), launched from a captured CUDA graph.  The negative-T
 * status of every stage is checked on the device; a failure is reported by
 * the next synchronous call (and by this one when sync != 0). */
int ocfd_gpu_step(ocfd_handle* h, int nsteps, int sync);
/* Kernels launched by one captured time step of ocfd_gpu_step (the kernel
 * nodes of its CUDA graph), or -1 before the first captured step or when the
 * step runs without a graph (filtering, time-dependent wall data).  The
 * reference has no counterpart (launch accounting of the device path). */
int ocfd_gpu_step_kernels(const ocfd_handle* h);

/* Run nsteps fused steps eagerly (no graph) with CUDA events around each kernel
 * group on the instance's stream; ms[] receives the average milliseconds per
 * step of: [0] shock sensor, [1] x faces, [2] y faces, [3] z faces, [4]
 * viscous gradients, [5] fused stage tail, [6] negative-T repair + BC +
 * halos, [7] the whole step.  Advances the solution like ocfd_gpu_step.
 * (Timing instrumentation: the reference only times the whole loop with
 * MPI_wtime, OCFD_NS_Solver.f90:18-19,79-80.) */
int ocfd_gpu_profile_steps(ocfd_handle* h, int nsteps, double ms[8]);

/* ---------------------------------------------------------------------------
 * Diagnostics on the device
 * ------------------------------------------------------------------------- */

/* show_flow_msg sums (OCFD_Time_Adv.f90:65-104): E0[0] total energy, E0[1]
 * kinetic energy, E0[2] p/rho^gamma, all /(nx*ny*nz), weighted by 1/Ajac. */
int ocfd_gpu_show_flow_msg(ocfd_handle* h, double E0[3]);

/* ana_box statistics (OCFD_ANA.f90:178-311).  out[20] in the column order of
 * statistics.dat: tt, Re_lamda, Re_lamdax, Amt, vv_rms, u_rms, v_rms, w_rms,
 * u_skewness, u_flatness, ux_skewness, ux_flatness, E_kinetic, Enstrophy,
 * d_rms, T_aver, Amu_aver, d_aver, Ux_rms, Alamdax. */
int ocfd_gpu_ana_box(ocfd_handle* h, double out[20]);

/* The other analyses of OCFD_analysis (OCFD_ANA.f90:3-31); the host keeps the
 * schedule (ANA_Para) and the files.
 * ana_getQ (OCFD_ANA.f90:127-171): q receives Q = II(grad u), nx*ny*nz. */
int ocfd_gpu_ana_q(ocfd_handle* h, double* q);
/* ana_time_average (OCFD_ANA.f90:34-125): adds the current d,u,v,w,T to the
 * running means (K_average += 1, t_average += dt).  The means start at zero,
 * or from ocfd_gpu_upload_average (the reference's opencfd.dat.average). */
int ocfd_gpu_ana_time_average(ocfd_handle* h);
int ocfd_gpu_download_average(ocfd_handle* h, double* const mean[5], int* k_average, double* t_average);
int ocfd_gpu_upload_average(ocfd_handle* h, const double* const mean[5], int k_average, double t_average);
/* Ana_corner (OCFD_ANA.f90:316-384): out[3*nx] = span averages of the
 * wall-tangential velocity at j=2, of T at j=2 and of the wall pressure. */
int ocfd_gpu_ana_corner(ocfd_handle* h, double* out);
/* The interior box [ib,ie]x[jb,je]x[kb,ke] (1-based, inclusive) of d,u,v,w,T,
 * i fastest (entries of out may be NULL): the data of ana_savedata's planes,
 * points and blocks (OCFD_ANA_savedata.f90:3-196, write_2d_*a / write_points /
 * write_blockdata, OCFD_IO_mpi.f90:7-130,286-326). */
int ocfd_gpu_download_block(ocfd_handle* h, int ib, int ie, int jb, int je, int kb, int ke, double* const out[5]);

/* show_flow_msg on arrays the caller owns, allocating nothing.  No counterpart
 * in the reference: it is for callers that cannot allocate device memory (a
 * host solver whose device memory all belongs to its own pool, or code that
 * must not trigger cudaFree's device-wide synchronisation while other streams
 * run), so they cannot create an ocfd_handle.
 *   p      parameters after ocfd_set_parameters (nx, ny, nz, gamma, Ma are read)
 *   f      device (nx,ny,nz,5) conserved variables, Fortran order
 *   prims  device haloed d, u, v, w, T ((nx+8)(ny+8)(nz+8) each, LAP = 4)
 *   ajac   device haloed Jacobian, same layout
 *   stream cudaStream_t (NULL: the default stream); the call waits for it
 * E0 receives the same three averages as ocfd_gpu_show_flow_msg (equal within
 * rounding: the summation order differs).  Every call copies its three sums to
 * host memory and waits for the stream before it returns.  The partial sums
 * live in a fixed static device array of OCFD_NOALLOC_MAX_PLANES partial
 * blocks: nz above OCFD_NOALLOC_MAX_PLANES is rejected with OCFD_E_PARAM.
 * Nothing in that array has to start at zero.  The first call on a device,
 * made with that device current, looks up the array's address (once per
 * device) and keeps it for the life of the process.  No call may be made
 * while its stream is capturing (the call copies to host memory and waits):
 * a capturing stream is refused with OCFD_E_PARAM before anything is
 * enqueued.  A cudaDeviceReset of that device makes
 * the kept address stale: do not use this entry point on a device after
 * resetting it.  There is one array per device, so overlapping calls on the
 * same device (from several streams or host threads) race: serialise them. */
#define OCFD_NOALLOC_MAX_PLANES 4096
int ocfd_show_flow_msg_noalloc(const ocfd_params* p, const double* f, const double* const prims[5],
                               const double* ajac, void* stream, double E0[3]);

/* ---------------------------------------------------------------------------
 * Ensemble (batched) mode: several independent instances advanced together.
 * No counterpart in the reference (which runs one case per process); used by
 * the serving loop.  Members keep their own state, grid size and physical
 * parameters (Re, Ma, dt, splitting).  When all members are periodic in the
 * three directions (BC_None, no ghost cells, no filter) and share precision,
 * flux form, inviscid scheme and the viscous flag, a time step is one launch
 * per kernel and per RK stage for the whole batch (18 launches, ragged grids
 * in the same launch), captured as a CUDA graph; the face-sweep tile shape per
 * direction is chosen by timing the candidates on the first step
 * (autotuning).  For the flux-vector WENO7 and the characteristic OMP6 forms
 * (viscous) a stage is instead ONE persistent launch for the whole batch
 * (3 launches per step): resident blocks take the tiles of every member's face
 * sweeps, viscous gradients, stage tail and negative-T repair from one work
 * list, a member's tail starting as soon as its own fluxes are complete.
 * Otherwise the members advance concurrently on their own streams.  Results
 * are bit-identical to stepping each member alone.
 * Between batch steps a member may be used on its own (downloads,
 * diagnostics, single steps); the batch rebuilds its tables when needed.
 * ------------------------------------------------------------------------- */
typedef struct ocfd_batch ocfd_batch;
int ocfd_batch_create(ocfd_handle* const* members, int count, ocfd_batch** out);
/* nsteps time steps of every member; sync = 1 waits and checks every member's
 * negative-temperature status (OCFD_E_NEGT if any member exceeded the limit). */
int ocfd_batch_step(ocfd_batch* b, int nsteps, int sync);
/* Force the face tile variant per direction (0 or 1; -1 = autotune). */
int ocfd_batch_set_tiles(ocfd_batch* b, const int variants[3]);
/* *fused = 1 when the batch runs one launch per kernel for all members;
 * variants[3] = the tile variants in use (after the first step). */
int ocfd_batch_info(const ocfd_batch* b, int* fused, int variants[3]);
/* Launch mode where the persistent stage kernel exists: on = -1 (the
 * default) times two steps in each mode at the first batch step of at least
 * four steps and keeps the faster (those steps are real steps: both modes give
 * the same bits); 0: one launch per kernel and stage; 1: the persistent
 * kernel. */
int ocfd_batch_set_persistent(ocfd_batch* b, int on);
/* 0: members advance on their own graphs; 1: one batched launch per kernel
 * and stage; 2: one persistent launch per stage.  OCFD_E_TIMEOUT from a batch
 * step (sync = 1) or from a member's ocfd_gpu_sync after mode 2: a bounded
 * dependency wait inside the persistent kernel gave up (about a second); the
 * steps since the last synchronisation are invalid and the batch continues in
 * mode 1. */
int ocfd_batch_mode(const ocfd_batch* b);
/* ms[0], ms[1]: device time of the two steps timed in mode 1 and in mode 2 by
 * the launch-mode choice; OCFD_E_STATE before that choice was timed. */
int ocfd_batch_mode_times(const ocfd_batch* b, float ms[2]);
const char* ocfd_batch_last_error(const ocfd_batch* b);
void ocfd_batch_destroy(ocfd_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* OCFD_GPU_H */

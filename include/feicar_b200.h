/*
 * feicar_b200.h -- C ABI of the B200 (sm_100a) pressure-Poisson path of
 * FEICAR3D: immersed-boundary tagging, ghost-cell pressure boundary
 * condition and the multigrid Poisson solve.
 *
 * Every entry point takes plain pointers and sizes, returns an fg_status
 * and never aborts; host arrays are the reference's Fortran module arrays
 * passed by c_loc (column-major, i fastest, lower bound 0):
 *     field(0:nx+1, 0:ny+1, 0:nz+1)   nx, ny, nz = NODE counts
 * which is how one MPI rank with nProcs = 1 lays them out
 * (CORE_MEMORY_ALLOCATE.F90:23-96, CORE_PARALLEL.F90:170-185).
 * The library keeps device-resident copies of the grid hierarchy, masks,
 * ghost/dead lists and solver state per handle across time steps.
 *
 * One handle is used from one host thread; every call is ordered on the
 * handle's CUDA stream.
 */
#ifndef FEICAR_B200_H
#define FEICAR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fg_status {
  FG_OK = 0,
  FG_NOT_CONVERGED = 1,          /* CORE_POISSON.F90:195-198 prints      */
  FG_GEOMETRY_NO_HOST_CELL = 2,  /* GCM_SET_BOUNDARY.F90:476-492         */
  FG_ALLOC_FAIL = 3,
  FG_TIMEOUT = 4,
  FG_BAD_INPUT = 5,
  FG_GEOMETRY_DEAD_NO_BODY = 6,  /* GCM_SET_BOUNDARY.F90:1061-1066       */
  FG_CUDA_ERROR = 7,
  FG_NO_DEVICE = 8,
  FG_REJECTED = 9,               /* serving admission refused            */
  FG_IO_ERROR = 10               /* a file could not be opened, read or
                                    written, or its layout is not the one
                                    expected                             */
} fg_status;

enum { FG_PBC_DIRICHLET = 1, FG_PBC_NEUMANN = 2 };
enum { FG_SOLID = 1, FG_MEMBRANE = 2 };
enum { FG_PREC_FP64 = 0, FG_PREC_MIXED = 1 };
/* outer iteration: V-cycles on p, FGMRES preconditioned by a V-cycle, or
 * the reference's single-grid line SOR (solver type 1, CORE_POISSON.F90
 * :205-456; FP64 on the finest level, max_cycles counts sweeps) */
enum { FG_OUTER_RICHARDSON = 0, FG_OUTER_FGMRES = 1, FG_OUTER_LSOR = 2 };

/* Solver settings: the input.dat keys of MAIN.F90:214-254 that the pressure
 * path reads, plus the knobs of the multigrid run on the GPU. */
typedef struct fg_solver_config {
  int    precision;          /* FG_PREC_FP64 or FG_PREC_MIXED              */
  int    outer;              /* FG_OUTER_RICHARDSON: V-cycles on p;
                                FG_OUTER_FGMRES: flexible GMRES(restart)
                                preconditioned by one V-cycle            */
  int    nu1, nu2;           /* pre/post smoothing steps (x, y, z lines)   */
  double omega;              /* line relaxation factor (omega_pson)        */
  double rtol;               /* ||f - A p||_2 / ||f||_2 on fluid rows       */
  int    max_cycles;         /* outer iterations (itermax_pson)            */
  int    pbc[6];             /* pbcx1..pbcz2                               */
  double ppp[6];             /* pppx1..pppz2 (Dirichlet values)            */
  int    mgrids[3];          /* mgrids_x/y/z, 0 = automatic (CORE_MG:69-102)*/
  double probe_length;       /* probeLengthNormalized                      */
  double probe_length_dead;  /* probeLengthNormalizedD                     */
  double membrane_tkns_factor;
  int    gauge_corner;       /* 1: subtract p(1,1,1) when all-Neumann      */
  int    restart;            /* FGMRES restart length (2..15)              */
} fg_solver_config;

typedef struct fg_solve_stats {
  int    cycles;             /* outer iterations used                       */
  double relres;             /* final relative residual (fluid rows)        */
  double ghost_res;          /* final max |ghost/dead row residual|         */
  double seconds;            /* device time of the solve                    */
  double vcycle_ms;          /* mean device time of one V-cycle             */
} fg_solve_stats;

typedef struct fg_case fg_case;

/* Library. */
const char *fg_version(void);
fg_status fg_device_count(int *count);
void fg_default_config(fg_solver_config *cfg);
const char *fg_status_string(fg_status s);

/* Replaces make_grid/metrics (CORE_GRID.F90:29-205) and MG_initial
 * (CORE_MG.F90:22-599): xn/yn/zn are the node coordinates x(1..nx),
 * y(1..ny), z(1..nz).  Allocates the device hierarchy on `device`. */
fg_status fg_case_create(int nx, int ny, int nz, const double *xn,
                         const double *yn, const double *zn,
                         const fg_solver_config *cfg, int device,
                         fg_case **out);
fg_status fg_case_destroy(fg_case *c);
/* node counts of level lev (mgrid_I/J/K) and the number of levels */
fg_status fg_case_levels(const fg_case *c, int *mlevel, int *dims /*3*MAX*/);

/* Body surfaces (BOUNDARY_MARKER_INIT / BOUNDARY_SET_ARCLENGTH_NORM input):
 * xyz[3*nvert], tri[3*ntri] 0-based, normals (v2-v1)x(v3-v2) into body. */
fg_status fg_case_add_body(fg_case *c, int nvert, int ntri, const double *xyz,
                           const int32_t *tri, int surface_type,
                           double membrane_tkns, int body_dim);
/* Moves body `ibody` (BOUNDARY_MOVE.F90:151-186 output). */
fg_status fg_case_update_body(fg_case *c, int ibody, const double *xyz);

/* Prescribed rigid motion of a body (boundary_motion_type
 * PRESCRIBED_RIGID): the input.dat parameters forced_motion reads
 * (BOUNDARY_MARKER_VEL.F90:5-33) and the state the next step needs
 * (centroid, the previous step's angular velocity), updated by each move. */
typedef struct fg_rigid_motion {
  double vcent_trans[3];  /* vxcentTrans, vycentTrans, vzcentTrans   */
  double amp[3], freq[3]; /* ampx.., freqx.. (translation)           */
  double angv_init[3];    /* angvxinit..                             */
  double ampang[3], freqang[3], angphase[3];
  double cent[3];         /* xcent, ycent, zcent                     */
  double angv_old[3];     /* angvx_old..                             */
} fg_rigid_motion;
/* Replaces move_boundary for a PRESCRIBED_RIGID body (BOUNDARY_MOVE.F90
 * :3-186 with forced_motion / compute_marker_vel, BOUNDARY_MARKER_VEL.F90
 * :5-125, and compute_marker_poisition, BOUNDARY_MOVE.F90:151-186) on the
 * device: the marker velocities of time `time`, the markers moved by dt,
 * the surface normals (calculate_arclength_norm_ds) and the marker dp/dn
 * (-Du_n/Dt, 0 when ntime <= 1) recomputed on the device, where the next
 * tagging reads them.  *ds_max: the largest marker displacement since the
 * last re-tag snapshot; *iblank_reset = 1 when it exceeds 0.05 of the
 * smallest cell width (the snapshot then moves to the new positions). */
fg_status fg_move_body(fg_case *c, int ibody, fg_rigid_motion *m, int ntime, double time, double dt,
                       double *ds_max, int *iblank_reset);
/* The markers of body ibody: positions xyz[3n], velocities uvw[3n] and
 * dp/dn[n] (any may be NULL). */
fg_status fg_get_body_markers(fg_case *c, int ibody, double *xyz, double *uvw, double *dpdn);

/* Replaces set_iblank_body_fast (BOUNDARY_IBLANK_FAST.F90:2-854) on the
 * device.  iblank (host, int8, the field above) may be NULL. */
fg_status fg_set_iblank_body_fast(fg_case *c, int8_t *iblank);
/* Replaces GCM_set_internal_boundary (GCM_SET_BOUNDARY.F90:2-604,
 * :880-1491): smoothing, ghost and dead lists, image points, weights.
 * Any output pointer may be NULL. */
fg_status fg_gcm_set_internal_boundary(fg_case *c, int8_t *iblank,
                                       int8_t *ghostCellMark,
                                       int8_t *dead_cell, int *nGhost,
                                       int *nDead);
/* Copies of the ghost / dead lists (1 row each, k-j-i list order):
 * ijk[3n], cell[3n] (host cell lower corner), coefN[8n], coefD[8n],
 * bi[3n] body intercept, ip[3n] image point, probe[n], closest[n]. */
fg_status fg_get_ghost_rows(const fg_case *c, int32_t *ijk, int32_t *cell,
                            double *coefN, double *coefD, double *bi,
                            double *ip, double *probe, int32_t *closest,
                            double *alpha);
fg_status fg_get_dead_rows(const fg_case *c, int32_t *ijk, int32_t *cell,
                           double *coefN, double *coefD, double *bi,
                           double *ip, double *probe, int32_t *closest);
/* band flag of the last tagging (1 = cell of the triangle-box band) */
fg_status fg_get_band(const fg_case *c, int8_t *band);

/* Supplies masks and interpolation rows computed by the caller instead of
 * the two calls above (a host that keeps its own GCM setup). */
fg_status fg_case_set_geometry(fg_case *c, const int8_t *iblank,
                               const int8_t *ghostCellMark,
                               const int8_t *dead_cell, int nGhost,
                               const int32_t *ghost_ijk,
                               const int32_t *ghost_cell,
                               const double *ghost_coefN, int nDead,
                               const int32_t *dead_ijk,
                               const int32_t *dead_cell_idx,
                               const double *dead_coefN,
                               const double *dead_probe,
                               const double *dead_ip);

/* Replaces mg_prepare (CORE_MG.F90:1365-1555): coarse masks. */
fg_status fg_mg_prepare(fg_case *c);

/* Replaces solve_poisson (CORE_POISSON.F90:83-200) with its ghost-cell
 * update (GCM_GHOSTCELL_UPDATE.F90:361-739) and mg_solve: p (in: initial
 * guess, out: converged pressure) and div are host fields; p_old is the
 * previous time step's pressure read by the dead-cell fallback (NULL = 0);
 * dpdn_ghost[nGhost], dpdn_dead[nDead] may be NULL (homogeneous).
 * Host<->device copies happen inside the call. */
fg_status fg_solve_poisson(fg_case *c, double *p, const double *div,
                           const double *p_old, const double *dpdn_ghost,
                           const double *dpdn_dead, fg_solve_stats *st);
/* Same with device pointers on the handle's layout-compatible arrays
 * (Fortran field layout, double, on the handle's device); d_p_old (NULL =
 * 0) feeds the dead-cell fallback. */
fg_status fg_solve_poisson_device(fg_case *c, double *d_p,
                                  const double *d_div, const double *d_p_old,
                                  fg_solve_stats *st);
/* The same with device dp/dn data, d_dpdn_ghost[nGhost] and
 * d_dpdn_dead[nDead] (NULL: homogeneous): the rows' constants (dp/dn
 * terms, the p_old fallback) are formed by a kernel, so a time step's
 * pressure data stay on the device. */
fg_status fg_solve_poisson_device_bc(fg_case *c, double *d_p, const double *d_div, const double *d_p_old,
                                     const double *d_dpdn_ghost, const double *d_dpdn_dead,
                                     fg_solve_stats *st);
/* Outer-face pressure gradients, the reference's module arrays pgradx1,
 * pgradx2, pgrady1, pgrady2, pgradz1, pgradz2 (face 0..5) read by
 * set_outer_pressure_bc (CORE_SET_OUTER_BC.F90:831-1042): x faces
 * (0:ny+1, 0:nz+1), y faces (0:nx+1, 0:nz+1), z faces (0:nx+1, 0:ny+1),
 * node counts, column-major.  Kept on the device (zero until set); a
 * Neumann face's gradient enters the finest-level right-hand side. */
fg_status fg_set_pressure_gradient(fg_case *c, int face, const double *values);
fg_status fg_get_pressure_gradient(fg_case *c, int face, double *values);
/* Replaces GCM_enforce_p_compatibility (GCM_GHOSTCELL_UPDATE.F90:865-1003)
 * on the device: with no Dirichlet face and some face whose velocity is
 * ZERO_GRADIENT (vel_zero_gradient[6] != 0), the net pressure-gradient
 * flux of p out of the fluid non-ghost cells, divided by the fluid area of
 * those faces, shifts their gradients (lower faces -, upper faces +).
 * p: host field. */
fg_status fg_enforce_p_compatibility(fg_case *c, const double *p, const int *vel_zero_gradient);
/* The faces whose velocity is ZERO_GRADIENT: every later solve on c first
 * applies the compatibility step to its initial pressure (the reference
 * applies it at the top of each outer iteration, CORE_POISSON.F90:160).
 * NULL clears. */
fg_status fg_case_set_zero_gradient_faces(fg_case *c, const int *vel_zero_gradient);
/* Replaces calc_residual (CORE_POISSON.F90:460-551) on the device:
 * *maxres = sqrt(sum r^2 / (nx ny nz)), r = div - A p over the fluid,
 * non-ghost interior cells, p read with its own outer ghost layers; the
 * normalisation by node counts is the reference's.  Host fields. */
fg_status fg_calc_residual(fg_case *c, const double *p, const double *div, double *maxres);
/* Replaces calc_residual2 (CORE_POISSON.F90:679-724) on the device:
 * *maxres2 = max |p - p_temp| over the non-iblank interior cells. */
fg_status fg_calc_residual2(fg_case *c, const double *p, const double *p_temp, double *maxres2);
/* One ghost/dead-cell update pass on a host field (GCM_ghostcell_pressure
 * with itermax_gc iterations). */
fg_status fg_ghostcell_pressure(fg_case *c, double *p, const double *p_old,
                                int iterations);

/* ----- the projection steps either side of the solve, on device fields
 * (reference layout, on the case's device; each call waits for its
 * kernels).  Face-velocity boundary arrays as the reference keeps them:
 * bcxu(0:1, 0:ny+1, 0:nz+1), bcyv(0:nx+1, 0:1, 0:nz+1),
 * bczw(0:nx+1, 0:ny+1, 0:1). ----- */
/* Replaces face_vel (CORE_FRAC_STEP_ROUTINES.F90:1-130): face velocities
 * interpolated from the cell velocities with the factors of
 * CORE_GRID.F90:194-202, the outer faces from the boundary arrays. */
fg_status fg_face_vel_device(fg_case *c, const double *u, const double *v, const double *w, const double *bcxu,
                             const double *bcyv, const double *bczw, double *face_u, double *face_v,
                             double *face_w);
/* Replaces rhs_poisson (CORE_POISSON.F90:9-79) with the
 * enforce_global_mass_consv it calls first (CORE_SET_OUTER_BC.F90:515-735,
 * mix_GC_form = 0): with zero-gradient faces (vel_zero_gradient[6], may be
 * NULL) the net mass flux is spread over their fluid area (boundary arrays
 * and boundary face velocities corrected); then div = (du/dx + dv/dy +
 * dw/dz)/dt on the fluid non-ghost cells, 0 elsewhere.  *sumd: the mass
 * flux; *resdiv: max |div| dt (either may be NULL). */
fg_status fg_rhs_poisson_device(fg_case *c, double *face_u, double *face_v, double *face_w, double *bcxu,
                                double *bcyv, double *bczw, const int *vel_zero_gradient, double dt, double *div,
                                double *sumd, double *resdiv);
/* Replaces correct_vel (CORE_FRAC_STEP_ROUTINES.F90:132-190: u -= dt grad
 * p' on the non-iblank cells) and calc_pres_grad (:270-320: the gradient
 * itself); either triple may be NULL. */
fg_status fg_correct_vel_device(fg_case *c, const double *pPrime, double dt, double *u, double *v, double *w,
                                double *dpdx, double *dpdy, double *dpdz);
/* GCM_SetBodyInterceptValues (GCM_BODYINTERCEPT_VALUES.F90:22-388) on the
 * rows of the last fg_gcm_set_internal_boundary: per ghost and dead row the
 * velocity at its body intercept, interpolated linearly over the closest
 * element's markers (the element's three vertices and its normal), from
 * the marker velocities fg_move_body keeps (zero before the first move),
 * this and the previous step's, and dp/dn = -(du/dt . n) at the intercept
 * (0 when ntime <= 1) -- the dp/dn data of fg_solve_poisson_device_bc.
 * Device outputs: ubi_*[3 * rows], dpdn_*[rows]; any may be NULL.
 * FG_BAD_INPUT when the rows came from fg_case_set_geometry. */
fg_status fg_body_intercept_values_device(fg_case *c, int ntime, double dt, double *ubi_ghost, double *ubi_dead,
                                          double *dpdn_ghost, double *dpdn_dead);
/* GCM_ghostcell_velocity (GCM_GHOSTCELL_UPDATE.F90:1-359) for iOpt = 2 and
 * mix_GC_form = 0 on device fields u, v, w (the reference updates the dead
 * cells of its arguments and the ghost cells of the module arrays, the
 * same arrays in solve_ad): dead cells u_BI w_BI - u_IP w_IP, ghost cells
 * the Dirichlet interpolation with the intercept velocity in their own
 * slot, iterated (Jacobi sweeps; the reference's in-place sweeps reach the
 * same values) while a sweep changes some row by more than restol_gcv and
 * fewer than itermax_gc sweeps ran.  FG_NOT_CONVERGED when the limit ran
 * out. */
fg_status fg_ghostcell_velocity_device(fg_case *c, double *u, double *v, double *w, const double *ubi_ghost,
                                       const double *ubi_dead, int itermax_gc, double restol_gcv, int *iterations);
/* The momentum equation's line SOR on device fields (one rank):
 * set_solve_ad's diffusion coefficients with viscosity reinv
 * (CORE_SET_SOLVERS.F90:591-677), then one pass of itsolv_ad
 * (CORE_SOLVE_AD.F90:131-776): x, y and z line sweeps of one velocity
 * component var with right-hand side r, the implicit convection terms
 * from face_u/v/w when crank_nicolson (advec_scheme == CRANK_NICOLSON2;
 * central for 25 <= i <= 375, first-order upwind elsewhere, as the
 * reference), relaxation omega_ad.  The lines of each direction are
 * solved one anti-diagonal at a time, which gives the reference's
 * lexicographic Gauss-Seidel sweep bit for bit.  The ghost-cell
 * coefficients the z sweep stores (ghostNScoeff) are not kept: the
 * velocity ghost-cell update stays with the caller. */
typedef struct fg_ad_params {
  double dt, reinv, omega_ad;
  int crank_nicolson;
} fg_ad_params;
fg_status fg_itsolv_ad_device(fg_case *c, double *var, const double *r, const double *face_u,
                              const double *face_v, const double *face_w, const fg_ad_params *prm);
/* calc_residual_ad (CORE_SOLVE_AD.F90:780-964): max |res| over the fluid
 * non-ghost cells and its first location (i, j, k) in the reference's
 * loop order ((1,1,1) when every residual is 0). */
fg_status fg_calc_residual_ad_device(fg_case *c, const double *var, const double *r, const double *face_u,
                                     const double *face_v, const double *face_w, const fg_ad_params *prm,
                                     double *resm, int *loc);
/* Outer velocity boundary data: the input.dat keys of MAIN.F90:196-207.
 * type per face x1, x2, y1, y2, z1, z2 (bcx1 ... bcz2): 1 Dirichlet, 2
 * zero gradient, 3 pulsatile inflow, 4 symmetry, 5 periodic, 6 user
 * specified; val the face's (u, v, w) (ux1, vx1, wx1, ...), freq their
 * frequencies (freq_ux1, ...), time the flow time, and the bounds of the
 * user-specified channel profiles. */
typedef struct fg_velocity_bc {
  int type[6];
  double val[6][3];
  double freq[6][3];
  double time, yOrigin, yout, zOrigin, zout;
} fg_velocity_bc;
/* The nine outer boundary arrays in the reference layout: bcxu, bcxv,
 * bcxw (0:1, 0:ny+1, 0:nz+1), bcyu, bcyv, bcyw (0:nx+1, 0:1, 0:nz+1),
 * bczu, bczv, bczw (0:nx+1, 0:ny+1, 0:1), device memory. */
typedef struct fg_velocity_bc_arrays {
  double *bcxu, *bcxv, *bcxw, *bcyu, *bcyv, *bcyw, *bczu, *bczv, *bczw;
} fg_velocity_bc_arrays;
/* Replaces set_outer_velocity_bc (CORE_SET_OUTER_BC.F90:18-509) for one
 * rank: x faces over j = 0..ny+1, k = 0..nz+1, then y faces over
 * i = 0..nx, k = 0..nz+1, then z faces over i = 0..nx, j = 0..ny+1, each
 * face by its type as the reference (the user-specified y and z faces
 * write the x2 arrays at (1, j, k), as it does).  A shear face (7) or an
 * unknown type returns FG_BAD_INPUT: the reference stops there. */
fg_status fg_set_outer_velocity_bc_device(fg_case *c, const double *u, const double *v, const double *w,
                                          const fg_velocity_bc_arrays *bc, const fg_velocity_bc *vb);
/* Replaces set_outer_ghost_velocity (CORE_SET_OUTER_BC.F90:739-823): the
 * outer ghost layer u = 2 bc - u(first interior), x faces, then y, then z
 * (the corners take the later face's value, as the reference). */
fg_status fg_set_outer_ghost_velocity_device(fg_case *c, double *u, double *v, double *w,
                                             const fg_velocity_bc_arrays *bc);
/* Replaces enforce_global_mass_consv (CORE_SET_OUTER_BC.F90:515-735) for
 * one rank: when a face of vel_zero_gradient[6] is set, the net mass flux
 * out of the fluid non-ghost cells is removed by a uniform outflow
 * correction on those faces (bcxu/bcyv/bczw and the boundary face
 * velocities). */
fg_status fg_enforce_global_mass_consv_device(fg_case *c, double *face_u, double *face_v, double *face_w,
                                              double *bcxu, double *bcyv, double *bczw,
                                              const int *vel_zero_gradient);
/* Replaces solve_ad (CORE_SOLVE_AD.F90:11-127) for one rank: while
 * iterations < itermax_ad and the residual > restol_ad, one itsolv_ad pass
 * of u, v, w (right-hand sides nlu, nlv, nlw), the velocity ghost and dead
 * cells (fg_ghostcell_velocity_device with the intercept velocities
 * ubi_ghost, ubi_dead), face_vel, enforce_global_mass_consv on vb's
 * zero-gradient faces, the outer velocity boundaries and their ghost
 * layer, and the largest of the three components' calc_residual_ad with
 * its location.  An iteration count that reaches itermax_ad is reported
 * in the outputs, not as an error (the reference prints it and goes on);
 * ghost velocities that do not converge return FG_NOT_CONVERGED (the
 * reference stops the run there). */
typedef struct fg_solve_ad_stats {
  int iterations;
  double residual;
  int loc[3];
} fg_solve_ad_stats;
fg_status fg_solve_ad_device(fg_case *c, double *u, double *v, double *w, const double *nlu, const double *nlv,
                             const double *nlw, double *face_u, double *face_v, double *face_w,
                             const fg_velocity_bc_arrays *bc, const double *ubi_ghost, const double *ubi_dead,
                             const fg_ad_params *prm, const fg_velocity_bc *vb, int itermax_gc, double restol_gcv,
                             int itermax_ad, double restol_ad, fg_solve_ad_stats *stats);
/* update_pressure (CORE_FRAC_STEP_ROUTINES.F90:212-299) for one rank:
 * pPrime = 0 on the solid cells (iblank) not dead-marked -1, for
 * i = 0..nx, j = 0..ny+1, k = 0..nz+1, and on the domain edge lines the
 * reference's twelve edge assignments name (its plane k = -1, outside
 * the array, is left out); then p = pPrime when p is not NULL. */
fg_status fg_update_pressure_device(fg_case *c, double *pPrime, double *p);

/* ----- stream, launch count and timing (no reference counterpart: the
 * reference prints wall time per solve_poisson call only,
 * CORE_TIME_STEP.F90:180-185) ----- */
/* Orders the handle's work on the caller's cudaStream_t (NULL: back to a
 * stream of the handle's own). */
fg_status fg_case_set_stream(fg_case *c, void *stream);
/* Kernels this process has launched through the library so far. */
fg_status fg_launch_count(long long *count);

enum {
  FG_PROF_LINE_X0 = 0,     /* finest-level x line sweeps (one colour each) */
  FG_PROF_LINE_Y0 = 1,     /* finest-level y line sweeps                   */
  FG_PROF_LINE_Z0 = 2,     /* finest-level z line sweeps                   */
  FG_PROF_LINE_COARSE = 3, /* line sweeps of the coarse levels             */
  FG_PROF_RESIDUAL = 4,    /* finest residual / correction / norms         */
  FG_PROF_TRANSFER = 5,    /* residual, restriction, prolongation (coarse) */
  FG_PROF_ROWS = 6,        /* ghost / dead row relaxation                  */
  FG_PROF_COARSEST = 7,    /* coarsest dense solve                         */
  FG_PROF_NCLASS = 8
};
typedef struct fg_profile {
  long long class_launches[FG_PROF_NCLASS]; /* timed launch groups       */
  double class_ms[FG_PROF_NCLASS];          /* CUDA-event device time    */
  double class_bytes[FG_PROF_NCLASS];       /* algorithmic bytes (line
                                               sweeps: 3s+1 per cell per
                                               direction, +s if omega!=1) */
} fg_profile;
/* Relative residual after each cycle of the last solve on c (the
 * reference prints its per-cycle MG residuals with infoconv = 1,
 * CORE_MG.F90:1811-1813): *count = cycles, relres[0..capacity-1] filled. */
fg_status fg_case_history(const fg_case *c, double *relres, int capacity, int *count);
/* How the last solve on c ran: *mode = 1 when the whole FGMRES solve was
 * one CUDA graph launch (its loops are graph conditional nodes decided on
 * the device, the host waits once at the end), 0 when the host drove the
 * same kernels step by step (launch-class timing on, the caller's stream
 * being captured, Richardson outer iteration, or a failed capture). */
fg_status fg_case_solve_mode(const fg_case *c, int *mode);
/* enable != 0: later solves on c bracket each launch group with CUDA
 * events on the handle's stream; resets the totals. */
fg_status fg_case_profile(fg_case *c, int enable);
fg_status fg_case_profile_read(const fg_case *c, fg_profile *out);

/* ----- ghost/dead row relaxation without any allocation (no counterpart
 * in the reference) -----
 * For callers that cannot call cudaMalloc -- code that only gets device
 * memory from a pool or framework it does not own, code where an
 * allocation would stall the device or a latency budget, Fortran hosts
 * passing arrays they manage themselves.  Runs `iterations` Jacobi passes
 * of the interpolation rows (the update fg_ghostcell_pressure performs) on
 * the caller's device field d_p, laid out like the reference arrays
 * (0:nx+1, 0:ny+1, 0:nz+1), nx/ny/nz node counts.  Row r sets
 *     p[tgt[r]] = sum_q w[8r+q] * p[cell[r] + corner_q] + c0[r]
 * with corner_q the 8 corners of the host cell whose lower corner is the
 * element cell[r], in the order of GCM_MEMORY_ALLOCATE.F90:593-623 (a
 * target's own corner carries weight 0); all rows of a pass read the
 * field before any row writes it.  tgt and cell are element indices of
 * the field; rows whose indices leave the field are skipped, and the call
 * does not report them (it returns FG_OK): the caller validates its row
 * lists.  d_c0 may be NULL (all zero).  Work is queued on `stream` (a
 * cudaStream_t of the current device, NULL for the default stream; a
 * stream of another device returns FG_BAD_INPUT) and the call returns
 * without waiting.
 * Scratch: a fixed device array of FG_NOALLOC_MAX_ROWS doubles (2 MiB),
 * present on every GPU that loads the library until the process exits;
 * nrows > FG_NOALLOC_MAX_ROWS returns FG_BAD_INPUT.  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress) and
 * keeps it for the life of the process, so make the first call on each
 * device before any stream capture, and do not call cudaDeviceReset on a
 * device after its first call (the kept address would be stale).  Every
 * call on a device shares the one array: calls that overlap on the GPU
 * (other streams, other host threads) race and must be ordered by the
 * caller.  Nothing in it needs to start at zero -- each pass writes every
 * value it reads. */
#define FG_NOALLOC_MAX_ROWS 262144
fg_status fg_rows_relax_noalloc(int nx, int ny, int nz, double *d_p, int nrows,
                                const int64_t *d_tgt, const int64_t *d_cell,
                                const double *d_w, const double *d_c0,
                                int iterations, void *stream);

/* ----- batched uneven solves: many cases per launch per MG stage ----- */
typedef struct fg_batch fg_batch;
fg_status fg_batch_create(int device, const fg_solver_config *cfg,
                          fg_batch **out);
fg_status fg_batch_add(fg_batch *b, fg_case *c);
/* Solves every case of the batch; p[i] and div[i] are device fields of
 * case i (as for fg_solve_poisson_device). */
fg_status fg_batch_solve_device(fg_batch *b, double **d_p,
                                const double **d_div, fg_solve_stats *st);
fg_status fg_batch_destroy(fg_batch *b);

/* ----- autotuner (no reference counterpart: the reference's smoother and
 * sweep counts are fixed in CORE_MG.F90) -----
 * Measures, on the batch's own levels, every line-kernel family that can
 * take each level set's lines along each axis (x: lines in registers with
 * lanes by line length, in registers with 32 lanes, or staged in shared
 * memory; y/z: tiles in registers with a Thomas over the chunks, tiles with
 * a block-wide cyclic reduction over the chunks, or one warp per line) and
 * keeps the fastest; then times whole solves of the batch's problems with
 * (nu1, nu2) = (1,1), (2,1), (2,2), (3,3) and keeps the fastest one that
 * converges.  The choices hold for later solves of the batch (and across
 * new geometries of the same grids).  d_p / d_div as for
 * fg_batch_solve_device; the tuning solves start from zero and leave the
 * last solution in d_p. */
#define FG_TUNE_MAXLEVELS 12
enum { FG_LV_XREG = 1, FG_LV_XREG32 = 2, FG_LV_XSMEM = 3 };   /* x sweeps   */
enum { FG_LV_YREG = 1, FG_LV_YPCR = 2, FG_LV_YWARP = 3,       /* y/z sweeps */
       FG_LV_YPCR_HOISTED = 4, FG_LV_YPCR_4ROWS = 5, FG_LV_YWAVE = 6 };
typedef struct fg_tuning {
  int nlevels;
  int line_variant[FG_TUNE_MAXLEVELS][3];  /* family that runs, per level and axis (0: no line launches) */
  double line_us[FG_TUNE_MAXLEVELS][3];    /* its measured time per sweep (both colours), us */
  int nu1, nu2;                            /* smoothing steps in use */
  double solve_ms[4];                      /* solve time of each (nu1,nu2) candidate, -1 = not converged */
  int tuned;                               /* 1 once fg_*_autotune ran */
  /* smoothing steps of the levels from level coarse_from (1 or 2; 0: 2)
   * down (0, 0: nu1, nu2 as the finer levels), set by fg_*_set_tuning
   * only: fewer coarse steps shorten a solve to a given rtol but leave a
   * residual with a larger error to the exact discrete solution, so the
   * autotuner (which sees only the time to rtol) leaves them at (0, 0) */
  int nu1_coarse, nu2_coarse;
  double solve_ms_coarse[2];               /* reserved (0) */
  int coarse_from;
} fg_tuning;
fg_status fg_batch_autotune(fg_batch *b, double **d_p, const double **d_div, fg_tuning *out);
fg_status fg_batch_get_tuning(const fg_batch *b, fg_tuning *out);
/* The same for a single case's solves (d_p, d_div: device fields in the
 * reference layout, as for fg_solve_poisson_device). */
fg_status fg_case_autotune(fg_case *c, double *d_p, const double *d_div, fg_tuning *out);
/* Sets the families and smoothing steps of an earlier tuning (a tuning
 * kept from another process or run on the same problems): line_variant
 * per level and axis (0 or a family that cannot take that level's lines:
 * the default), nu1/nu2 when their sum is positive.  The tables are built
 * first if needed; the captured graphs are dropped. */
fg_status fg_batch_set_tuning(fg_batch *b, const fg_tuning *t);
fg_status fg_case_set_tuning(fg_case *c, const fg_tuning *t);

/* ----- serving: a stream of solve requests over many cases (no reference
 * counterpart: the reference runs one case per process and calls
 * rhs_poisson -> solve_poisson once per time step, CORE_TIME_STEP.F90
 * :171-178) -----
 * An engine thread admits requests first come, first served while at most
 * max_active cases are resident and their estimated device memory
 * (fg_case_estimate_bytes) stays within budget_bytes; a request that
 * arrives while others run is admitted as soon as a slot and memory free
 * up.  Each admitted request gets its own case (hierarchy, device
 * tagging, lists) on its own stream, resident across its steps; every
 * step is the right-hand side's copy in, the FGMRES solve as one CUDA
 * graph launch and the pressure's copy out, and the steps of different
 * requests overlap on the device.  Step s starts from step s-1's pressure
 * (step 0 from p0, NULL = zero).  The host fields div[s] (and p[s], if
 * given) belong to the caller until the request's result is polled;
 * page-locked buffers keep the copies asynchronous. */
typedef struct fg_server fg_server;
typedef struct fg_serve_request {
  long long id;                   /* the caller's tag, echoed in the result */
  int nx, ny, nz;                 /* node counts                            */
  const double *xn, *yn, *zn;     /* node coordinates (copied at submit)    */
  int nvert, ntri;                /* one body surface (copied at submit)    */
  const double *xyz;
  const int32_t *tri;
  int surface_type;               /* FG_SOLID or FG_MEMBRANE                */
  double membrane_tkns;
  int nsteps;                     /* time steps of the request              */
  const double *const *div;       /* nsteps right-hand sides (reference layout) */
  double *const *p;               /* nsteps outputs, or NULL (no copy out)  */
  const double *p0;               /* initial pressure of step 0, or NULL    */
} fg_serve_request;
typedef struct fg_serve_result {
  long long id;
  fg_status status;               /* FG_OK, FG_NOT_CONVERGED or an error    */
  int steps_done;
  int cycles_max;                 /* most cycles of a step                  */
  double relres_max;              /* worst final relative residual          */
  double t_submit, t_admit, t_done;  /* server clock (s): latency = t_done - t_submit */
} fg_serve_result;
typedef struct fg_server_stats {
  long long submitted, finished, pending;
  int active, active_peak;
  size_t bytes_in_use;            /* estimated device bytes of active cases */
} fg_server_stats;
/* Device memory a case of this grid and configuration holds (levels,
 * Krylov vectors, staging, tagging), the admission estimate. */
fg_status fg_case_estimate_bytes(int nx, int ny, int nz, const fg_solver_config *cfg, size_t *bytes);
fg_status fg_server_create(int device, const fg_solver_config *cfg, size_t budget_bytes, int max_active,
                           fg_server **out);
/* Queues a request (FG_REJECTED if it alone exceeds the budget). */
fg_status fg_server_submit(fg_server *s, const fg_serve_request *req);
/* Results of finished requests, oldest first (up to capacity). */
fg_status fg_server_poll(fg_server *s, fg_serve_result *out, int capacity, int *count);
/* Waits until every submitted request has finished (FG_TIMEOUT after
 * timeout_s seconds). */
fg_status fg_server_wait_idle(fg_server *s, double timeout_s);
fg_status fg_server_info(const fg_server *s, fg_server_stats *out);
/* Seconds since the server was created (the clock of the results). */
double fg_server_clock(const fg_server *s);
/* Finishes every submitted request, then stops the engine. */
fg_status fg_server_destroy(fg_server *s);

/* ----- formats around the path (host code; no device is touched) ----- */

/* Gmsh MSH 2.2 ASCII body surface, the unstructured surface input of the
 * marker initialisation (BOUNDARY_MARKER_INIT.F90:247-296).  The reference
 * skips a fixed number of lines and reads every element line as
 * `elm type ntags tag tag n1 n2 n3`; here the sections are found by name,
 * the tags are counted, elements other than 3-node triangles (type 2) are
 * skipped and counted in *nskipped, and node tags are mapped to 0-based
 * vertex indices (the reference's marker index is the tag itself; files
 * whose tags run 1..n in order give the same triangles).  Call with
 * xyz = tri = NULL for the counts, then with xyz[3*cap_vert] and
 * tri[3*cap_tri].  FG_IO_ERROR: no file, not ASCII 2.x, a short section;
 * FG_BAD_INPUT: buffers too small, a triangle naming a node not listed. */
fg_status fg_read_msh22(const char *path, int *nvert, int *ntri, double *xyz, int cap_vert, int *tri,
                        int cap_tri, int *nskipped);

/* The restart file of write_restart / read_restart (MAIN.F90:1049-1122,
 * 983-1040) for one rank (nProcs = 1): an unformatted sequential file of
 * records with 4-byte length markers (time, ntime), (every flow array), then
 * one record per body.  A record longer than the maximum subrecord length
 * is split: every subrecord but the last carries a negative leading marker,
 * every one but the first a negative trailing marker (the layout of
 * gfortran and of Intel Fortran's variable-length records).  NULL arrays
 * are written as zeros and skipped on reading.  Arrays are the reference's
 * Fortran arrays (column-major, lower bounds 0). */
typedef struct fg_restart_flow {
  int nx, ny, nz;                 /* node counts                            */
  double time;
  int ntime;
  /* (0:nx+1, 0:ny+1, 0:nz+1) */
  double *u, *v, *w, *p, *face_u, *face_v, *face_w, *pPrime;
  double *bcxu, *bcxv, *bcxw, *bcxp;  /* (0:1, 0:ny+1, 0:nz+1)              */
  double *bcyu, *bcyv, *bcyw, *bcyp;  /* (0:nx+1, 0:1, 0:nz+1)              */
  double *bczu, *bczv, *bczw, *bczp;  /* (0:nx+1, 0:ny+1, 0:1)              */
  /* pgradx1, pgradx2 (0:ny+1,0:nz+1); pgrady1, pgrady2 (0:nx+1,0:nz+1);
   * pgradz1, pgradz2 (0:nx+1,0:ny+1) -- the order of fg_get_pressure_gradient */
  double *pgrad[6];
  int8_t *iblank, *ghostcellmark;     /* (0:nx+1, 0:ny+1, 0:nz+1)           */
} fg_restart_flow;
typedef struct fg_restart_body {
  int npts, nelm;
  double *x, *y, *z, *u, *v, *w;  /* marker positions and velocities [npts] */
  double *fx, *fy, *fz;           /* marker forces [npts]                   */
  int *tri;                       /* [3*nelm] 0-based; stored 1-based       */
  double cent[3], ang[3], vcent[3], angv[3];
} fg_restart_body;
fg_status fg_write_restart(const char *path, const fg_restart_flow *f, int nbody, const fg_restart_body *b);
/* Reads into the arrays of f and b, whose sizes (nx, ny, nz, npts, nelm)
 * must be those of the file (FG_IO_ERROR otherwise); sets time and ntime. */
fg_status fg_read_restart(const char *path, fg_restart_flow *f, int nbody, fg_restart_body *b);
/* The longest subrecord written (bytes, 16 .. 2**31-9; other values give
 * the default 2**31-9), the counterpart of gfortran's
 * -fmax-subrecord-length.  Process-wide. */
void fg_set_max_subrecord(long long bytes);

/* The Tecplot POINT dump of write_flowfield for nDim = 3
 * (UTIL_GENERAL.F90:167-247): a VARIABLES line, a ZONE line of
 * I = nx+1, J = ny+1, K = nz+1 points, then for k = 0..nz, j = 0..ny,
 * i = 0..nx one line in format 11(2x,1PE12.5),5(2x,I2) of
 * xc, yc, zc, u, v, w, p, ox, oy, oz, lmd, iblank, ghost, dead, body, goa.
 * xc[0..nx], yc[0..ny], zc[0..nz] are the cell centres with the ghost
 * layers; fields are (0:nx+1, 0:ny+1, 0:nz+1); a NULL field is written as
 * zeros.  The reference gzips the file afterwards; this does not. */
typedef struct fg_tecplot_fields {
  const double *u, *v, *w, *p, *ox, *oy, *oz, *lmd;
  const int8_t *iblank, *ghost, *dead, *bodynum, *goa;
} fg_tecplot_fields;
fg_status fg_write_tecplot(const char *path, int nx, int ny, int nz, const double *xc, const double *yc,
                           const double *zc, const fg_tecplot_fields *f);

#ifdef __cplusplus
}
#endif
#endif

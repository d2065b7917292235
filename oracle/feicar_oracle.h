/*
 * feicar_oracle.h -- CPU restatement (FP64) of the FEICAR3D pressure-Poisson
 * path, used ONLY as test infrastructure: the checker that the CUDA path is
 * compared against, and the timed CPU baseline in bench.py.  Nothing in the
 * product library links or calls this code.
 *
 * Parity status: the reference is Fortran + MPI + MKL and cannot be compiled
 * in this image (no Fortran compiler, no MPI, no MKL); it ships no tests, no
 * fixtures and no golden vectors.  This restatement is therefore pinned only
 * by known answers: the manufactured-solution Poisson test of
 * CORE_POISSON.F90:565-674 (test_mg) with its closed-form solution, the
 * discrete-residual identity, geometric invariants of the tagging, and the
 * 8x8 Vandermonde inverse checked against scipy.  Parity against reference
 * OUTPUTS is unpinned.
 *
 * Layout: every 3-D field is the reference's column-major array
 * (0:nx+1, 0:ny+1, 0:nz+1) for one MPI rank (nProcs = 1), i fastest,
 * index  i + (nx+2)*(j + (ny+2)*k).  nx, ny, nz are NODE counts
 * (cells = n-1), exactly as in CORE_GRID.F90:29-205.
 */
#ifndef FEICAR_ORACLE_H
#define FEICAR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* pressure boundary types (AMODULES PBC_DIRICHLET / PBC_NEUMANN) */
enum { OR_PBC_DIRICHLET = 1, OR_PBC_NEUMANN = 2 };
/* surface types (AMODULES SOLID_BODY / MEMBRANE) */
enum { OR_SOLID = 1, OR_MEMBRANE = 2 };
/* Poisson solver types (AMODULES IT_SOLVER_TYPE_LSOR / _MG) */
enum { OR_SOLVER_LSOR = 1, OR_SOLVER_MG = 3 };

/* status codes shared with the product C-ABI */
enum {
  OR_OK = 0,
  OR_NOT_CONVERGED = 1,
  OR_GEOMETRY_NO_HOST_CELL = 2,
  OR_ALLOC_FAIL = 3,
  OR_BAD_INPUT = 5,
  OR_GEOMETRY_DEAD_NO_BODY = 6
};

/* Poisson parameters: the input.dat keys of MAIN.F90:214-254 that the
 * pressure path reads. */
typedef struct or_params {
  int    it_solver_type;    /* OR_SOLVER_MG or OR_SOLVER_LSOR            */
  int    itermax_pson;      /* outer iterations (CORE_POISSON.F90:126)   */
  double restol_pson;       /* V-cycle residual tolerance (CORE_MG:1613) */
  double restol_gcp;        /* outer iterate-change / ghost tolerance    */
  int    itermax_gc;        /* ghost Gauss-Seidel iterations             */
  double omega_pson;        /* line-SOR relaxation                       */
  int    iterInter;         /* max V-cycles per mg_solve = iterInter+1   */
  int    pbc[6];            /* x1,x2,y1,y2,z1,z2 pressure BC types        */
  double ppp[6];            /* Dirichlet values                           */
  int    vel_zero_gradient[6]; /* velocity BC == ZERO_GRADIENT per face  */
  int    mix_GC_form;
  int    is_PBC_homogeneous;
  int    freeze_solid;      /* 1: the per-iteration gauge shift skips
                               pure-solid (iblank, non-dead) cells         */
} or_params;

/* statistics of one solve_poisson call */
typedef struct or_stats {
  int    outer_iterations;
  int    vcycles;           /* total V-cycles (or LSOR sweeps)            */
  double maxres;            /* calc_residual of the last iteration        */
  double maxres2;           /* calc_residual2 of the last iteration       */
  double relres;            /* ||f - A p||_2 / ||f||_2 on fluid rows       */
  double seconds;
} or_stats;

typedef struct or_case or_case;

/* CORE_GRID.F90:29-205 + CORE_MG.F90:22-599.  xn/yn/zn hold x(1..nx) etc.
 * mgrids = 0 selects the automatic level count. */
or_case *or_case_create(int nx, int ny, int nz, const double *xn,
                        const double *yn, const double *zn, int mgrids_x,
                        int mgrids_y, int mgrids_z);
void or_case_destroy(or_case *c);
int  or_case_dims(const or_case *c, int *out /* nx,ny,nz,mLevel */);
int  or_case_level_dims(const or_case *c, int lev, int *out /* I,J,K */);
int  or_case_grid(const or_case *c, int axis, int what, double *out);

/* add one triangulated body; tri is 0-based, 3 per triangle.
 * BOUNDARY_SET_ARCLENGTH_NORM.F90:46-175 normals are computed here. */
int  or_case_add_body(or_case *c, int nvert, int ntri, const double *xyz,
                      const int32_t *tri, int surface_type,
                      double membrane_tkns, int body_dim);
int  or_case_update_body(or_case *c, int ibody, const double *xyz);

/* BOUNDARY_IBLANK_FAST.F90:2-854 */
int  or_set_iblank_body_fast(or_case *c, int ntime, int ntime_start);
/* GCM_SET_BOUNDARY.F90:2-604 (+ smooth, ghost, dead cells) */
int  or_gcm_set_internal_boundary(or_case *c, double probeLengthNormalized,
                                  double probeLengthNormalizedD);
/* CORE_MG.F90:1365-1555 */
int  or_mg_prepare(or_case *c);

/* field export: 0 iblank, 1 ghostCellMark, 2 dead_cell, 3 bodyNum,
 * 4 iblankUndecided band flag (1 = band cell) */
int  or_get_field_i8(const or_case *c, int which, int8_t *out);
/* counts: nGhost, nDead, nWarnSide, nHostFail, nStencilSolid, nFallbackDead */
int  or_get_counts(const or_case *c, int *out);
/* GCM_GHOSTCELL_UPDATE.F90:865-1003 on p (updates the face gradients) and
 * the face gradient arrays it reads and writes (face 0..5: x1..z2) */
int  or_enforce_p_compatibility(or_case *c, const double *p, const or_params *prm);
/* prescribed rigid motion of a body (BOUNDARY_MOVE.F90 move_boundary,
 * BOUNDARY_MARKER_VEL.F90 forced_motion / compute_marker_vel) */
typedef struct or_rigid_motion {
  double vcent_trans[3], amp[3], freq[3];
  double angv_init[3], ampang[3], freqang[3], angphase[3];
  double cent[3], angv_old[3];
} or_rigid_motion;
int  or_move_body(or_case *c, int ibody, or_rigid_motion *m, int ntime, double time, double dt,
                  double *ds_max, int *iblank_reset);
int  or_get_body_markers(or_case *c, int ibody, double *xyz, double *uvw, double *dpdn);
int  or_get_pgrad(or_case *c, int face, double *out);
int  or_set_pgrad(or_case *c, int face, const double *in);
/* the fractional-step projection either side of the solve:
 * CORE_FRAC_STEP_ROUTINES.F90 face_vel, correct_vel / calc_pres_grad,
 * CORE_SET_OUTER_BC.F90 enforce_global_mass_consv + CORE_POISSON.F90
 * rhs_poisson */
int  or_face_vel(or_case *c, const double *u, const double *v, const double *w, const double *bcxu,
                 const double *bcyv, const double *bczw, double *fu, double *fv, double *fw);
int  or_rhs_poisson(or_case *c, double *fu, double *fv, double *fw, double *bcxu, double *bcyv,
                    double *bczw, const int *vzg, double dt, double *div, double *sumd, double *resdiv);
int  or_correct_vel(or_case *c, const double *pp, double dt, double *u, double *v, double *w,
                    double *dpdx, double *dpdy, double *dpdz);
int  or_update_pressure(or_case *c, double *pp, double *p);
/* body-intercept velocities (3 per row) and dp/dn of the ghost and dead
 * rows (GCM_BODYINTERCEPT_VALUES.F90:22-388); any output may be NULL */
int  or_body_intercept_values(or_case *c, int ntime, double dt, double *ubi_g, double *ubi_d, double *dpdn_g,
                              double *dpdn_d);
/* velocity ghost and dead cells (GCM_GHOSTCELL_UPDATE.F90:1-359, mix_GC_form 0) */
int  or_ghostcell_velocity(or_case *c, double *u, double *v, double *w, const double *ubi_g, const double *ubi_d,
                           double pld, int itermax_gc, double restol_gcv, int *iterations);
/* outer velocity boundary data (CORE_SET_OUTER_BC.F90:18-509): type per
 * face x1,x2,y1,y2,z1,z2 (1 Dirichlet, 2 zero gradient, 3 pulsatile
 * inflow, 4 symmetry, 5 periodic, 6 user specified), (u,v,w) values and
 * frequencies per face, the time, the channel-profile bounds */
typedef struct or_velocity_bc {
  int type[6];
  double val[6][3], freq[6][3];
  double time, yOrigin, yout, zOrigin, zout;
} or_velocity_bc;
int  or_enforce_global_mass_consv(or_case *c, double *fu, double *fv, double *fw, double *bcxu, double *bcyv,
                                  double *bczw, const int *vzg);
/* bc: bcxu, bcxv, bcxw, bcyu, bcyv, bcyw, bczu, bczv, bczw */
int  or_set_outer_velocity_bc(or_case *c, const double *u, const double *v, const double *w, double *const *bc,
                              const or_velocity_bc *p);
int  or_set_outer_ghost_velocity(or_case *c, double *u, double *v, double *w, double *const *bc);
int  or_solve_ad(or_case *c, const double *ad, double *u, double *v, double *w, const double *nlu,
                 const double *nlv, const double *nlw, double *fu, double *fv, double *fw, double *const *bc,
                 const double *ubi_g, const double *ubi_d, double half_dt, double omega_ad,
                 const or_velocity_bc *vb, double pld, int itermax_gc, double restol_gcv, int itermax_ad,
                 double restol_ad, int *iterations, double *resm, int *loc);
/* momentum line SOR (CORE_SET_SOLVERS.F90:591-677, CORE_SOLVE_AD.F90):
 * ad holds amx_ad, apx_ad (nx+2 each), amy_ad, apy_ad (ny+2), amz_ad,
 * apz_ad (nz+2) */
int  or_set_solve_ad(or_case *c, double dt, double reinv, double *ad);
int  or_itsolv_ad(or_case *c, const double *ad, double *var, const double *r, const double *fu,
                  const double *fv, const double *fw, double half_dt, double omega_ad);
int  or_calc_residual_ad(or_case *c, const double *ad, const double *var, const double *r, const double *fu,
                         const double *fv, const double *fw, double half_dt, double *resm, int *loc);
int  or_get_ghosts(const or_case *c, int32_t *ijk, int32_t *cell,
                   double *coeffN, double *coeffD, double *bi, double *ip,
                   double *probeLength, int32_t *closestElem, double *alpha);
int  or_get_deads(const or_case *c, int32_t *ijk, int32_t *cell,
                  double *coeffN, double *coeffD, double *bi, double *ip,
                  double *probeLengthDead, int32_t *closestElem);
int  or_get_mg_mask(const or_case *c, int lev, int which, int8_t *out);

/* CORE_POISSON.F90:83-200.  p (in/out), div (in), p_old (in: the previous
 * time step's pressure read by the dead-cell fallback), dpdn arrays may be
 * NULL (homogeneous). */
int  or_solve_poisson(or_case *c, double *p, const double *div,
                      const double *p_old, const double *dpdn_ghost,
                      const double *dpdn_dead, const or_params *prm,
                      or_stats *st);
/* pieces exported for unit tests */
int  or_ghostcell_pressure(or_case *c, double *p, const double *div,
                           const double *p_old, const double *dpdn_ghost,
                           const double *dpdn_dead, const or_params *prm,
                           int *iterations);
double or_calc_residual(const or_case *c, const double *p, const double *r);
double or_relres(const or_case *c, const double *p, const double *r);
int  or_tdma(const double *a, const double *b, const double *cc,
             const double *r, double *u, int n1, int n2);
int  or_invert8(const double *a /* 8x8 column-major */, double *inv,
                int *info);
/* OpenMP timing variant of the V-cycle loop (block-Jacobi over z slabs, the
 * shared-memory analogue of the reference's MPI pencils). */
int  or_set_threads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif

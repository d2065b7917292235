/*
 * feicar_oracle.c -- CPU FP64 restatement of the FEICAR3D pressure-Poisson
 * path.  TEST INFRASTRUCTURE ONLY: the checker the CUDA library is compared
 * against and the CPU baseline timed by bench.py.  The product library never
 * links this file.
 *
 * Parity status: pinned by known answers only (see feicar_oracle.h); the
 * reference (Fortran/MPI/MKL) cannot be compiled in this image, so parity
 * against reference outputs is unpinned.
 *
 * Compiled with -O2 -ffp-contract=off and without -ffast-math, so every
 * floating-point expression below is evaluated in the order it is written,
 * one IEEE-754 double operation at a time, which is how the Fortran
 * expressions it restates read left to right.
 *
 * Restated reference files (nProcs = 1, so halo exchanges and MPI reductions
 * are identities):
 *   CORE_GRID.F90:29-205, CORE_MG.F90:22-1848, CORE_TDMA.F90:10-34,
 *   CORE_POISSON.F90:83-551,679-724, CORE_SET_OUTER_BC.F90:831-1186,
 *   GCM_GHOSTCELL_UPDATE.F90:361-739,865-1003,
 *   BOUNDARY_IBLANK_FAST.F90:2-1555, GCM_SET_BOUNDARY.F90:2-1491,1618-1697,
 *   GCM_MEMORY_ALLOCATE.F90:565-650, BOUNDARY_SET_ARCLENGTH_NORM.F90:46-175.
 */
#include "feicar_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXLEV 16
#define MAXBODY 8
#define UNDECIDED 100
/* The reference is compiled without a default-real-8 flag (makefile:34-45),
 * so literals written without a kind suffix are single precision and enter
 * double expressions as their float values: 1.0e-12 (CORE_MG.F90:690),
 * 0.01 (CORE_MG.F90:1168) and 0.1 (GCM_SET_BOUNDARY.F90:1144). */
#define TINY_F32 ((double)1.0e-12f)
#define CENTI_F32 ((double)0.01f)
#define TENTH_F32 ((double)0.1f)

typedef struct or_body {
  int nvert, ntri, type, body_dim;
  double membrane_tkns;
  double *xv, *yv, *zv;
  int32_t *tri;
  double *enx, *eny, *enz, *ecx, *ecy, *ecz, *earea;
  double *vnx, *vny, *vnz;
  /* vertex -> incident triangles in ascending triangle order: the same
   * sequence the full scan of BOUNDARY_IBLANK_FAST.F90:992-999 produces */
  int32_t *v2t_off, *v2t;
  /* prescribed motion: marker velocities (this and the previous step),
   * positions at the last re-tag, marker dp/dn (made on the first move) */
  double *mu, *mv, *mw, *muo, *mvo, *mwo, *sx, *sy, *sz, *dpdn;
} or_body;

typedef struct or_level {
  int I, J, K;
  double *x, *y, *z, *xc, *yc, *zc;
  double *dxinv, *dyinv, *dzinv, *dxcinv, *dycinv, *dzcinv;
  double *rhs, *phi, *res;
  int8_t *ibk, *igk;
} or_level;

struct or_case {
  int nx, ny, nz;
  long NX, NY, NZ, ntot;
  double *x, *y, *z, *xc, *yc, *zc;
  double *dx, *dy, *dz, *dxinv, *dyinv, *dzinv;
  double *dxc, *dyc, *dzc, *dxcinv, *dycinv, *dzcinv;
  double dxMin, dyMin, dzMin;
  int mLevel, mgx, mgy, mgz;
  or_level lev[MAXLEV];
  int nbody;
  or_body body[MAXBODY];
  int8_t *iblank, *ghost, *dead, *bodyNum, *undecided, *igmark, *ps1, *ps2;
  int8_t *iblankTemp;
  int32_t *ghostIndex;
  /* ghost cells */
  int nGhost;
  int32_t *gijk, *gcell, *gclosest;
  double *gcoefN, *gcoefD, *gbi, *gip, *gprobe, *galpha, *gnrm;
  /* dead cells */
  int nDead;
  int32_t *dijk, *dcell, *dclosest;
  double *dcoefN, *dcoefD, *dbi, *dip, *dprobe, *dnrm;
  /* outer BC state (CORE_SET_OUTER_BC.F90): persistent like the module
   * arrays bcxp/bcyp/bczp and pgrad* */
  double *bcxp, *bcyp, *bczp;
  double *pgradx1, *pgradx2, *pgrady1, *pgrady2, *pgradz1, *pgradz2;
  /* diagnostics */
  int nWarnSide, nHostFail, nStencilSolid, nFallbackDead;
  /* solver scratch: 1-D line arrays (solver_arrays) and p_temp */
  double *am, *ac, *ap, *rr, *dum;
  double *p_temp;
};

static int g_threads = 1;

int or_set_threads(int nthreads) {
  g_threads = nthreads > 0 ? nthreads : 1;
  return OR_OK;
}

#define IDX(c, i, j, k) ((long)(i) + (c)->NX * ((long)(j) + (c)->NY * (long)(k)))
#define LIDX(L, i, j, k) \
  ((long)(i) + (long)((L)->I + 2) * ((long)(j) + (long)((L)->J + 2) * (long)(k)))

static double *dzalloc(long n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }
static int8_t *bzalloc(long n) { return (int8_t *)calloc((size_t)(n > 0 ? n : 1), 1); }
static int32_t *izalloc(long n) { return (int32_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t)); }

/* ------------------------------------------------------------------ grid */
/* CORE_GRID.F90:29-170 make_grid, given x(1..n) (uniform or file grid). */
static void make_axis(int n, const double *xn, double *x, double *xc,
                      double *dx, double *dxinv, double *dxc,
                      double *dxcinv) {
  for (int i = 1; i <= n; ++i) x[i] = xn[i - 1];
  x[0] = x[1] * 2.0 - x[2];
  x[n + 1] = x[n] + x[n] - x[n - 1];
  for (int i = 0; i <= n; ++i) {
    xc[i] = 0.5 * (x[i + 1] + x[i]);
    dx[i] = x[i + 1] - x[i];
    dxinv[i] = 1.0 / dx[i];
  }
  xc[n + 1] = x[n + 1];
  for (int i = 1; i <= n; ++i) {
    dxc[i] = xc[i] - xc[i - 1];
    dxcinv[i] = 1.0 / dxc[i];
  }
}

/* CORE_MG.F90:69-102: number of halvings until fewer than 4 cells. */
static int auto_levels(int n) {
  int II = n - 1, N;
  for (N = 1; N <= 10; ++N) {
    II = II / 2;
    if (II >= 4) continue;
    break;
  }
  if (N > 10) N = 10;
  return N;
}

static void level_alloc(or_level *L) {
  L->x = dzalloc(L->I + 2); L->y = dzalloc(L->J + 2); L->z = dzalloc(L->K + 2);
  L->xc = dzalloc(L->I + 2); L->yc = dzalloc(L->J + 2); L->zc = dzalloc(L->K + 2);
  L->dxinv = dzalloc(L->I + 2); L->dyinv = dzalloc(L->J + 2); L->dzinv = dzalloc(L->K + 2);
  L->dxcinv = dzalloc(L->I + 2); L->dycinv = dzalloc(L->J + 2); L->dzcinv = dzalloc(L->K + 2);
  long n = (long)(L->I + 2) * (L->J + 2) * (L->K + 2);
  L->rhs = dzalloc(n); L->phi = dzalloc(n); L->res = dzalloc(n);
  L->ibk = bzalloc(n); L->igk = bzalloc(n);
}

/* CORE_MG.F90:231-332 coarse coordinates of one axis */
static void coarse_axis(int nC, int nF, const double *xF, double *x,
                        double *dxinv, double *xc, double *dxcinv,
                        double x1fine, double xnfine) {
  for (int i = 1; i <= nC - 1; ++i) {
    int iim = (nC == nF) ? i : 2 * i - 1;
    x[i] = xF[iim];
  }
  x[nC] = xF[nF];
  for (int i = 1; i <= nC - 1; ++i) {
    dxinv[i] = 1.0 / (x[i + 1] - x[i]);
    xc[i] = 0.5 * (x[i] + x[i + 1]);
  }
  xc[0] = 2.0 * x1fine - xc[1];
  xc[nC] = 2.0 * xnfine - xc[nC - 1];
  for (int i = 1; i <= nC; ++i) dxcinv[i] = 1.0 / (xc[i] - xc[i - 1]);
}

static int coarsen_count(int n) { return (n % 2 == 0) ? n / 2 + 1 : (n + 1) / 2; }

or_case *or_case_create(int nx, int ny, int nz, const double *xn,
                        const double *yn, const double *zn, int mgx, int mgy,
                        int mgz) {
  if (nx < 3 || ny < 3 || nz < 3) return NULL;
  or_case *c = (or_case *)calloc(1, sizeof(or_case));
  if (!c) return NULL;
  c->nx = nx; c->ny = ny; c->nz = nz;
  c->NX = nx + 2; c->NY = ny + 2; c->NZ = nz + 2;
  c->ntot = c->NX * c->NY * c->NZ;
  c->x = dzalloc(nx + 2); c->xc = dzalloc(nx + 2); c->dx = dzalloc(nx + 2);
  c->dxinv = dzalloc(nx + 2); c->dxc = dzalloc(nx + 2); c->dxcinv = dzalloc(nx + 2);
  c->y = dzalloc(ny + 2); c->yc = dzalloc(ny + 2); c->dy = dzalloc(ny + 2);
  c->dyinv = dzalloc(ny + 2); c->dyc = dzalloc(ny + 2); c->dycinv = dzalloc(ny + 2);
  c->z = dzalloc(nz + 2); c->zc = dzalloc(nz + 2); c->dz = dzalloc(nz + 2);
  c->dzinv = dzalloc(nz + 2); c->dzc = dzalloc(nz + 2); c->dzcinv = dzalloc(nz + 2);
  make_axis(nx, xn, c->x, c->xc, c->dx, c->dxinv, c->dxc, c->dxcinv);
  make_axis(ny, yn, c->y, c->yc, c->dy, c->dyinv, c->dyc, c->dycinv);
  make_axis(nz, zn, c->z, c->zc, c->dz, c->dzinv, c->dzc, c->dzcinv);
  c->dxMin = c->dx[1]; c->dyMin = c->dy[1]; c->dzMin = c->dz[1];
  for (int i = 1; i <= nx - 1; ++i) if (c->dx[i] < c->dxMin) c->dxMin = c->dx[i];
  for (int i = 1; i <= ny - 1; ++i) if (c->dy[i] < c->dyMin) c->dyMin = c->dy[i];
  for (int i = 1; i <= nz - 1; ++i) if (c->dz[i] < c->dzMin) c->dzMin = c->dz[i];

  /* MG_initial, CORE_MG.F90:71-332 */
  c->mgx = (mgx <= 0 || mgx > 10) ? auto_levels(nx) : mgx;
  c->mgy = (mgy <= 0 || mgy > 10) ? auto_levels(ny) : mgy;
  c->mgz = (mgz <= 0 || mgz > 10) ? auto_levels(nz) : mgz;
  int mL = c->mgx;
  if (c->mgy > mL) mL = c->mgy;
  if (c->mgz > mL) mL = c->mgz;
  c->mLevel = mL;
  c->lev[0].I = nx; c->lev[0].J = ny; c->lev[0].K = nz;
  for (int n = 1; n < mL; ++n) {
    or_level *P = &c->lev[n - 1], *L = &c->lev[n];
    L->I = (n + 1 <= c->mgx) ? coarsen_count(P->I) : P->I;
    L->J = (n + 1 <= c->mgy) ? coarsen_count(P->J) : P->J;
    L->K = (n + 1 <= c->mgz) ? coarsen_count(P->K) : P->K;
  }
  for (int n = 0; n < mL; ++n) level_alloc(&c->lev[n]);
  or_level *L1 = &c->lev[0];
  for (int i = 0; i <= nx; ++i) { L1->dxcinv[i] = c->dxcinv[i]; L1->dxinv[i] = c->dxinv[i]; L1->xc[i] = c->xc[i]; }
  for (int j = 0; j <= ny; ++j) { L1->dycinv[j] = c->dycinv[j]; L1->dyinv[j] = c->dyinv[j]; L1->yc[j] = c->yc[j]; }
  for (int k = 0; k <= nz; ++k) { L1->dzcinv[k] = c->dzcinv[k]; L1->dzinv[k] = c->dzinv[k]; L1->zc[k] = c->zc[k]; }
  for (int i = 0; i <= nx + 1; ++i) L1->x[i] = c->x[i];
  for (int j = 0; j <= ny + 1; ++j) L1->y[j] = c->y[j];
  for (int k = 0; k <= nz + 1; ++k) L1->z[k] = c->z[k];
  for (int n = 1; n < mL; ++n) {
    or_level *P = &c->lev[n - 1], *L = &c->lev[n];
    coarse_axis(L->I, P->I, P->x, L->x, L->dxinv, L->xc, L->dxcinv, c->x[1], c->x[nx]);
    coarse_axis(L->J, P->J, P->y, L->y, L->dyinv, L->yc, L->dycinv, c->y[1], c->y[ny]);
    coarse_axis(L->K, P->K, P->z, L->z, L->dzinv, L->zc, L->dzcinv, c->z[1], c->z[nz]);
  }

  long nt = c->ntot;
  c->iblank = bzalloc(nt); c->ghost = bzalloc(nt); c->dead = bzalloc(nt);
  c->bodyNum = bzalloc(nt); c->undecided = bzalloc(nt); c->igmark = bzalloc(nt);
  c->ps1 = bzalloc(nt); c->ps2 = bzalloc(nt); c->iblankTemp = bzalloc(nt);
  c->ghostIndex = izalloc(nt);
  c->bcxp = dzalloc(2 * c->NY * c->NZ);
  c->bcyp = dzalloc(c->NX * 2 * c->NZ);
  c->bczp = dzalloc(c->NX * c->NY * 2);
  c->pgradx1 = dzalloc(c->NY * c->NZ); c->pgradx2 = dzalloc(c->NY * c->NZ);
  c->pgrady1 = dzalloc(c->NX * c->NZ); c->pgrady2 = dzalloc(c->NX * c->NZ);
  c->pgradz1 = dzalloc(c->NX * c->NY); c->pgradz2 = dzalloc(c->NX * c->NY);
  int nmax = nx; if (ny > nmax) nmax = ny; if (nz > nmax) nmax = nz;
  c->am = dzalloc(nmax + 2); c->ac = dzalloc(nmax + 2); c->ap = dzalloc(nmax + 2);
  c->rr = dzalloc(nmax + 2); c->dum = dzalloc(nmax + 2);
  c->p_temp = dzalloc(nt);
  return c;
}

static void free_ghosts(or_case *c) {
  free(c->gijk); free(c->gcell); free(c->gclosest); free(c->gcoefN); free(c->gcoefD);
  free(c->gbi); free(c->gip); free(c->gprobe); free(c->galpha); free(c->gnrm);
  c->gijk = c->gcell = c->gclosest = NULL;
  c->gcoefN = c->gcoefD = c->gbi = c->gip = c->gprobe = c->galpha = c->gnrm = NULL;
}
static void free_deads(or_case *c) {
  free(c->dijk); free(c->dcell); free(c->dclosest); free(c->dcoefN); free(c->dcoefD);
  free(c->dbi); free(c->dip); free(c->dprobe); free(c->dnrm);
  c->dijk = c->dcell = c->dclosest = NULL;
  c->dcoefN = c->dcoefD = c->dbi = c->dip = c->dprobe = c->dnrm = NULL;
}

void or_case_destroy(or_case *c) {
  if (!c) return;
  double *d1[] = {c->x, c->y, c->z, c->xc, c->yc, c->zc, c->dx, c->dy, c->dz,
                  c->dxinv, c->dyinv, c->dzinv, c->dxc, c->dyc, c->dzc,
                  c->dxcinv, c->dycinv, c->dzcinv, c->bcxp, c->bcyp, c->bczp,
                  c->pgradx1, c->pgradx2, c->pgrady1, c->pgrady2, c->pgradz1,
                  c->pgradz2, c->am, c->ac, c->ap, c->rr, c->dum, c->p_temp};
  for (size_t q = 0; q < sizeof(d1) / sizeof(d1[0]); ++q) free(d1[q]);
  int8_t *b1[] = {c->iblank, c->ghost, c->dead, c->bodyNum, c->undecided,
                  c->igmark, c->ps1, c->ps2, c->iblankTemp};
  for (size_t q = 0; q < sizeof(b1) / sizeof(b1[0]); ++q) free(b1[q]);
  free(c->ghostIndex);
  for (int n = 0; n < c->mLevel; ++n) {
    or_level *L = &c->lev[n];
    double *d2[] = {L->x, L->y, L->z, L->xc, L->yc, L->zc, L->dxinv, L->dyinv,
                    L->dzinv, L->dxcinv, L->dycinv, L->dzcinv, L->rhs, L->phi, L->res};
    for (size_t q = 0; q < sizeof(d2) / sizeof(d2[0]); ++q) free(d2[q]);
    free(L->ibk); free(L->igk);
  }
  for (int b = 0; b < c->nbody; ++b) {
    or_body *B = &c->body[b];
    free(B->xv); free(B->yv); free(B->zv); free(B->tri);
    free(B->enx); free(B->eny); free(B->enz); free(B->ecx); free(B->ecy); free(B->ecz);
    free(B->earea); free(B->vnx); free(B->vny); free(B->vnz);
    free(B->v2t_off); free(B->v2t);
    free(B->mu); free(B->mv); free(B->mw); free(B->muo); free(B->mvo); free(B->mwo);
    free(B->sx); free(B->sy); free(B->sz); free(B->dpdn);
  }
  free_ghosts(c); free_deads(c);
  free(c);
}

int or_case_dims(const or_case *c, int *out) {
  out[0] = c->nx; out[1] = c->ny; out[2] = c->nz; out[3] = c->mLevel;
  return OR_OK;
}
int or_case_level_dims(const or_case *c, int lev, int *out) {
  if (lev < 0 || lev >= c->mLevel) return OR_BAD_INPUT;
  out[0] = c->lev[lev].I; out[1] = c->lev[lev].J; out[2] = c->lev[lev].K;
  return OR_OK;
}
/* what: 0 x, 1 xc, 2 dx, 3 dxinv, 4 dxc, 5 dxcinv (n+2 values) */
int or_case_grid(const or_case *c, int axis, int what, double *out) {
  const double *src[3][6] = {
      {c->x, c->xc, c->dx, c->dxinv, c->dxc, c->dxcinv},
      {c->y, c->yc, c->dy, c->dyinv, c->dyc, c->dycinv},
      {c->z, c->zc, c->dz, c->dzinv, c->dzc, c->dzcinv}};
  int n = axis == 0 ? c->nx : axis == 1 ? c->ny : c->nz;
  if (axis < 0 || axis > 2 || what < 0 || what > 5) return OR_BAD_INPUT;
  memcpy(out, src[axis][what], sizeof(double) * (size_t)(n + 2));
  return OR_OK;
}

/* ------------------------------------------------------------ surfaces */
/* BOUNDARY_SET_ARCLENGTH_NORM.F90:46-175: unit element normals (pointing
 * into the body), centroids, areas, vertex normals = normalised sums. */
static void body_normals(or_body *B) {
  for (int v = 0; v < B->nvert; ++v) { B->vnx[v] = 0.0; B->vny[v] = 0.0; B->vnz[v] = 0.0; }
  for (int m = 0; m < B->ntri; ++m) {
    int n1 = B->tri[3 * m], n2 = B->tri[3 * m + 1], n3 = B->tri[3 * m + 2];
    double ax = B->xv[n2] - B->xv[n1], ay = B->yv[n2] - B->yv[n1], az = B->zv[n2] - B->zv[n1];
    double bx = B->xv[n3] - B->xv[n2], by = B->yv[n3] - B->yv[n2], bz = B->zv[n3] - B->zv[n2];
    double nxv = (ay * bz - az * by);
    double nyv = (az * bx - ax * bz);
    double nzv = (ax * by - ay * bx);
    double mag = sqrt(nxv * nxv + nyv * nyv + nzv * nzv);
    B->earea[m] = 0.5 * mag;
    B->enx[m] = nxv / mag; B->eny[m] = nyv / mag; B->enz[m] = nzv / mag;
    B->vnx[n1] = B->vnx[n1] + B->enx[m];
    B->vnx[n2] = B->vnx[n2] + B->enx[m];
    B->vnx[n3] = B->vnx[n3] + B->enx[m];
    B->vny[n1] = B->vny[n1] + B->eny[m];
    B->vny[n2] = B->vny[n2] + B->eny[m];
    B->vny[n3] = B->vny[n3] + B->eny[m];
    B->vnz[n1] = B->vnz[n1] + B->enz[m];
    B->vnz[n2] = B->vnz[n2] + B->enz[m];
    B->vnz[n3] = B->vnz[n3] + B->enz[m];
    B->ecx[m] = (B->xv[n1] + B->xv[n2] + B->xv[n3]) / 3.0;
    B->ecy[m] = (B->yv[n1] + B->yv[n2] + B->yv[n3]) / 3.0;
    B->ecz[m] = (B->zv[n1] + B->zv[n2] + B->zv[n3]) / 3.0;
  }
  for (int v = 0; v < B->nvert; ++v) {
    double mag = sqrt(B->vnx[v] * B->vnx[v] + B->vny[v] * B->vny[v] + B->vnz[v] * B->vnz[v]);
    B->vnx[v] = B->vnx[v] / mag; B->vny[v] = B->vny[v] / mag; B->vnz[v] = B->vnz[v] / mag;
  }
}

static void body_adjacency(or_body *B) {
  free(B->v2t_off); free(B->v2t);
  B->v2t_off = izalloc(B->nvert + 1);
  int32_t *cnt = izalloc(B->nvert);
  for (int m = 0; m < B->ntri; ++m) {
    int a = B->tri[3 * m], b = B->tri[3 * m + 1], d = B->tri[3 * m + 2];
    cnt[a]++;
    if (b != a) cnt[b]++;
    if (d != a && d != b) cnt[d]++;
  }
  for (int v = 0; v < B->nvert; ++v) B->v2t_off[v + 1] = B->v2t_off[v] + cnt[v];
  B->v2t = izalloc(B->v2t_off[B->nvert]);
  memset(cnt, 0, sizeof(int32_t) * (size_t)B->nvert);
  for (int m = 0; m < B->ntri; ++m) {
    int a = B->tri[3 * m], b = B->tri[3 * m + 1], d = B->tri[3 * m + 2];
    B->v2t[B->v2t_off[a] + cnt[a]++] = m;
    if (b != a) B->v2t[B->v2t_off[b] + cnt[b]++] = m;
    if (d != a && d != b) B->v2t[B->v2t_off[d] + cnt[d]++] = m;
  }
  free(cnt);
}

int or_case_add_body(or_case *c, int nvert, int ntri, const double *xyz,
                     const int32_t *tri, int surface_type,
                     double membrane_tkns, int body_dim) {
  if (c->nbody >= MAXBODY || nvert < 3 || ntri < 1) return OR_BAD_INPUT;
  for (int m = 0; m < 3 * ntri; ++m)
    if (tri[m] < 0 || tri[m] >= nvert) return OR_BAD_INPUT;
  or_body *B = &c->body[c->nbody];
  memset(B, 0, sizeof(*B));
  B->nvert = nvert; B->ntri = ntri; B->type = surface_type;
  B->membrane_tkns = membrane_tkns; B->body_dim = body_dim;
  B->xv = dzalloc(nvert); B->yv = dzalloc(nvert); B->zv = dzalloc(nvert);
  B->tri = izalloc(3 * ntri);
  memcpy(B->tri, tri, sizeof(int32_t) * 3 * (size_t)ntri);
  B->enx = dzalloc(ntri); B->eny = dzalloc(ntri); B->enz = dzalloc(ntri);
  B->ecx = dzalloc(ntri); B->ecy = dzalloc(ntri); B->ecz = dzalloc(ntri);
  B->earea = dzalloc(ntri);
  B->vnx = dzalloc(nvert); B->vny = dzalloc(nvert); B->vnz = dzalloc(nvert);
  for (int v = 0; v < nvert; ++v) {
    B->xv[v] = xyz[3 * v]; B->yv[v] = xyz[3 * v + 1]; B->zv[v] = xyz[3 * v + 2];
  }
  body_normals(B);
  body_adjacency(B);
  c->nbody++;
  return OR_OK;
}

int or_case_update_body(or_case *c, int ibody, const double *xyz) {
  if (ibody < 0 || ibody >= c->nbody) return OR_BAD_INPUT;
  or_body *B = &c->body[ibody];
  for (int v = 0; v < B->nvert; ++v) {
    B->xv[v] = xyz[3 * v]; B->yv[v] = xyz[3 * v + 1]; B->zv[v] = xyz[3 * v + 2];
  }
  body_normals(B);
  return OR_OK;
}

/* ------------------------------------------------ prescribed rigid motion
 * BOUNDARY_MOVE.F90:3-186 (move_boundary, PRESCRIBED_RIGID) with
 * BOUNDARY_MARKER_VEL.F90:5-33 forced_motion, :60-125 compute_marker_vel
 * and BOUNDARY_MOVE.F90:151-186 compute_marker_poisition; the normals of
 * calculate_arclength_norm_ds; dp/dn at the markers (:96-110); the re-tag
 * test (:122-145). */
int or_move_body(or_case *c, int ibody, or_rigid_motion *m, int ntime, double time, double dt,
                 double *ds_max, int *iblank_reset) {
  if (ibody < 0 || ibody >= c->nbody || !(dt > 0.0)) return OR_BAD_INPUT;
  or_body *B = &c->body[ibody];
  const int nv = B->nvert;
  if (!B->mu) {
    B->mu = dzalloc(nv); B->mv = dzalloc(nv); B->mw = dzalloc(nv);
    B->muo = dzalloc(nv); B->mvo = dzalloc(nv); B->mwo = dzalloc(nv);
    B->sx = dzalloc(nv); B->sy = dzalloc(nv); B->sz = dzalloc(nv); B->dpdn = dzalloc(nv);
    for (int v = 0; v < nv; ++v) { B->sx[v] = B->xv[v]; B->sy[v] = B->yv[v]; B->sz[v] = B->zv[v]; }
  }
  const double PI = 3.14159265358979323846;
  double vc[3], av[3], ta[3];
  for (int a = 0; a < 3; ++a) {
    vc[a] = m->vcent_trans[a] + m->amp[a] * sin(2.0 * PI * m->freq[a] * time);
    av[a] = m->angv_init[a] + m->ampang[a] * sin(2.0 * PI * m->freqang[a] * time + m->angphase[a]);
  }
  for (int a = 0; a < 3; ++a) ta[a] = 0.5 * (m->angv_old[a] + av[a]);
  const double ax = av[0], ay = av[1], az = av[2];
  const double tot = 1.0 / (1.0 + 0.25 * (dt * dt) * (ax * ax + ay * ay + az * az));
  const double q = 0.25 * (dt * dt), h = 0.5 * dt;
  double ds = 0.0;
  for (int i = 0; i < nv; ++i) {
    const double tu = (ta[1] * (B->zv[i] - m->cent[2]) - ta[2] * (B->yv[i] - m->cent[1]));
    const double tv = -(ta[0] * (B->zv[i] - m->cent[2]) - ta[2] * (B->xv[i] - m->cent[0]));
    const double tw = (ta[0] * (B->yv[i] - m->cent[1]) - ta[1] * (B->xv[i] - m->cent[0]));
    const double uB = vc[0] + tot * (tu * (1.0 + q * (ax * ax)) + tv * (-h * az - q * ax * ay) + tw * (-h * ay + q * ax * az));
    const double vB = vc[1] + tot * (tu * (h * az - q * ax * ay) + tv * (1.0 + q * (ay * ay)) + tw * (-h * ax - q * ay * az));
    const double wB = vc[2] + tot * (tu * (h * ay + q * ax * az) + tv * (h * ax - q * ay * az) + tw * (1.0 + q * (az * az)));
    B->muo[i] = B->mu[i]; B->mvo[i] = B->mv[i]; B->mwo[i] = B->mw[i];
    B->mu[i] = uB; B->mv[i] = vB; B->mw[i] = wB;
    B->xv[i] = B->xv[i] + dt * uB;
    B->yv[i] = B->yv[i] + dt * vB;
    B->zv[i] = B->zv[i] + dt * wB;
    const double dx = B->xv[i] - B->sx[i], dy = B->yv[i] - B->sy[i], dz = B->zv[i] - B->sz[i];
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d > ds) ds = d;
  }
  for (int a = 0; a < 3; ++a) {
    m->cent[a] = m->cent[a] + dt * vc[a];
    m->angv_old[a] = av[a];
  }
  body_normals(B);
  for (int i = 0; i < nv; ++i)
    B->dpdn[i] = ntime > 1 ? -((B->mu[i] - B->muo[i]) / dt * B->vnx[i] + (B->mv[i] - B->mvo[i]) / dt * B->vny[i] +
                               (B->mw[i] - B->mwo[i]) / dt * B->vnz[i])
                           : 0.0;
  double hmin = 1e300;
  for (int i = 1; i <= c->nx - 1; ++i) if (c->dx[i] < hmin) hmin = c->dx[i];
  for (int j = 1; j <= c->ny - 1; ++j) if (c->dy[j] < hmin) hmin = c->dy[j];
  for (int k = 1; k <= c->nz - 1; ++k) if (c->dz[k] < hmin) hmin = c->dz[k];
  const int reset = ds > 0.05 * hmin;
  if (reset)
    for (int v = 0; v < nv; ++v) { B->sx[v] = B->xv[v]; B->sy[v] = B->yv[v]; B->sz[v] = B->zv[v]; }
  if (ds_max) *ds_max = ds;
  if (iblank_reset) *iblank_reset = reset;
  return OR_OK;
}

int or_get_body_markers(or_case *c, int ibody, double *xyz, double *uvw, double *dpdn) {
  if (ibody < 0 || ibody >= c->nbody) return OR_BAD_INPUT;
  or_body *B = &c->body[ibody];
  for (int v = 0; v < B->nvert; ++v) {
    if (xyz) { xyz[3 * v] = B->xv[v]; xyz[3 * v + 1] = B->yv[v]; xyz[3 * v + 2] = B->zv[v]; }
    if (uvw) {
      uvw[3 * v] = B->mu ? B->mu[v] : 0.0;
      uvw[3 * v + 1] = B->mv ? B->mv[v] : 0.0;
      uvw[3 * v + 2] = B->mw ? B->mw[v] : 0.0;
    }
    if (dpdn) dpdn[v] = B->dpdn ? B->dpdn[v] : 0.0;
  }
  return OR_OK;
}

/* ------------------------------------------------ body intercept query */
static void cross3(const double *r, const double *s, double *o) {
  /* BOUNDARY_IBLANK_FAST.F90:1539-1555 */
  o[0] = r[1] * s[2] - s[1] * r[2];
  o[1] = r[2] * s[0] - s[2] * r[0];
  o[2] = r[0] * s[1] - s[0] * r[1];
}

/* BOUNDARY_IBLANK_FAST.F90:1220-1313 (Heron areas) */
static void bi_inside_triangle(const double *xv, const double *yv,
                               const double *zv, double xb, double yb,
                               double zb, double *area123, double *areaDiff) {
  double s12 = sqrt((xv[1] - xv[0]) * (xv[1] - xv[0]) + (yv[1] - yv[0]) * (yv[1] - yv[0]) + (zv[1] - zv[0]) * (zv[1] - zv[0]));
  double s23 = sqrt((xv[2] - xv[1]) * (xv[2] - xv[1]) + (yv[2] - yv[1]) * (yv[2] - yv[1]) + (zv[2] - zv[1]) * (zv[2] - zv[1]));
  double s31 = sqrt((xv[0] - xv[2]) * (xv[0] - xv[2]) + (yv[0] - yv[2]) * (yv[0] - yv[2]) + (zv[0] - zv[2]) * (zv[0] - zv[2]));
  double s14 = sqrt((xb - xv[0]) * (xb - xv[0]) + (yb - yv[0]) * (yb - yv[0]) + (zb - zv[0]) * (zb - zv[0]));
  double s24 = sqrt((xb - xv[1]) * (xb - xv[1]) + (yb - yv[1]) * (yb - yv[1]) + (zb - zv[1]) * (zb - zv[1]));
  double s34 = sqrt((xb - xv[2]) * (xb - xv[2]) + (yb - yv[2]) * (yb - yv[2]) + (zb - zv[2]) * (zb - zv[2]));
  double p123 = 0.5 * (s12 + s23 + s31);
  double p124 = 0.5 * (s12 + s24 + s14);
  double p234 = 0.5 * (s23 + s24 + s34);
  double p314 = 0.5 * (s31 + s34 + s14);
  double a123 = sqrt(p123 * fabs(p123 - s12) * fabs(p123 - s23) * fabs(p123 - s31));
  double a124 = sqrt(p124 * fabs(p124 - s12) * fabs(p124 - s24) * fabs(p124 - s14));
  double a234 = sqrt(p234 * fabs(p234 - s23) * fabs(p234 - s24) * fabs(p234 - s34));
  double a314 = sqrt(p314 * fabs(p314 - s31) * fabs(p314 - s34) * fabs(p314 - s14));
  *area123 = a123;
  *areaDiff = a124 + a234 + a314 - a123;
}

/* BOUNDARY_IBLANK_FAST.F90:1316-1536.  When no side passes the sign test
 * the reference leaves isideSelect undefined (:1383-1416); here the side
 * with the smallest dot value is taken and *warn is raised. */
static void bi_outside_triangle(const double *xv, const double *yv,
                                const double *zv, double xcg, double ycg,
                                double zcg, const double *xvn,
                                const double *yvn, const double *zvn,
                                double *xb, double *yb, double *zb,
                                double *dist, double *nx_, double *ny_,
                                double *nz_, int *warn) {
  double v4[3] = {*xb, *yb, *zb};
  int sel = -1;
  double best = 0.0;
  int bestside = 1;
  for (int iside = 1; iside <= 3; ++iside) {
    int mside = iside + 1;
    if (iside == 3) mside = 1;
    int kside = iside == 1 ? 3 : (iside == 2 ? 1 : 2);
    double v1[3] = {xv[iside - 1], yv[iside - 1], zv[iside - 1]};
    double v2[3] = {xv[mside - 1], yv[mside - 1], zv[mside - 1]};
    double v3[3] = {xv[kside - 1], yv[kside - 1], zv[kside - 1]};
    double a[3] = {v3[0] - v1[0], v3[1] - v1[1], v3[2] - v1[2]};
    double b[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
    double cc[3] = {v4[0] - v1[0], v4[1] - v1[1], v4[2] - v1[2]};
    double axb[3], cxb[3];
    cross3(a, b, axb);
    cross3(cc, b, cxb);
    double dotVal = cxb[0] * axb[0] + cxb[1] * axb[1] + cxb[2] * axb[2];
    if (iside == 1 || dotVal < best) { best = dotVal; bestside = iside; }
    if (dotVal <= 0.0) { sel = iside; break; }
  }
  if (sel < 0) { sel = bestside; (*warn)++; }
  int s1 = sel == 1 ? 0 : (sel == 2 ? 1 : 2);
  int s2 = sel == 1 ? 1 : (sel == 2 ? 2 : 0);
  double n12x = xv[s2] - xv[s1], n12y = yv[s2] - yv[s1], n12z = zv[s2] - zv[s1];
  double mag = sqrt(n12x * n12x + n12y * n12y + n12z * n12z);
  n12x = n12x / mag; n12y = n12y / mag; n12z = n12z / mag;
  double plen = (*xb - xv[s1]) * n12x + (*yb - yv[s1]) * n12y + (*zb - zv[s1]) * n12z;
  double xB = xv[s1] + plen * n12x, yB = yv[s1] + plen * n12y, zB = zv[s1] + plen * n12z;
  double d1 = sqrt((xv[s1] - xB) * (xv[s1] - xB) + (yv[s1] - yB) * (yv[s1] - yB) + (zv[s1] - zB) * (zv[s1] - zB)) / mag;
  double d2 = sqrt((xv[s2] - xB) * (xv[s2] - xB) + (yv[s2] - yB) * (yv[s2] - yB) + (zv[s2] - zB) * (zv[s2] - zB)) / mag;
  if (d1 <= 1.0 && d2 <= 1.0) {
    *xb = xB; *yb = yB; *zb = zB;
    *nx_ = 0.5 * (xvn[s1] + xvn[s2]);
    *ny_ = 0.5 * (yvn[s1] + yvn[s2]);
    *nz_ = 0.5 * (zvn[s1] + zvn[s2]);
  } else if (d2 > 1.0) {
    *xb = xv[s1]; *yb = yv[s1]; *zb = zv[s1];
    *nx_ = xvn[s1]; *ny_ = yvn[s1]; *nz_ = zvn[s1];
  } else {
    *xb = xv[s2]; *yb = yv[s2]; *zb = zv[s2];
    *nx_ = xvn[s2]; *ny_ = yvn[s2]; *nz_ = zvn[s2];
  }
  *dist = sqrt((xcg - *xb) * (xcg - *xb) + (ycg - *yb) * (ycg - *yb) + (zcg - *zb) * (zcg - *zb));
}

/* BOUNDARY_IBLANK_FAST.F90:857-1216 calc_bodyIntercept_Unstruc with
 * nCheck = 1: closest vertex (first index of the minimum), then the
 * elements sharing it in ascending order, last element with dist <= min. */
static void body_intercept(or_case *c, int ib, double xC, double yC,
                           double zC, double *xBI, double *yBI, double *zBI,
                           int *closest, double *distOut, double *dotNorm) {
  or_body *B = &c->body[ib];
  double dmin = 0.0;
  int vmin = 0;
  for (int m = 0; m < B->nvert; ++m) {
    double dd = (B->xv[m] - xC) * (B->xv[m] - xC) + (B->yv[m] - yC) * (B->yv[m] - yC) +
                (B->zv[m] - zC) * (B->zv[m] - zC);
    if (m == 0 || dd < dmin) { dmin = dd; vmin = m; }
  }
  double distMin = 1.0e16, xb = 0.0, yb = 0.0, zb = 0.0, bnx = 0.0, bny = 0.0, bnz = 0.0;
  int cel = -1;
  for (int q = B->v2t_off[vmin]; q < B->v2t_off[vmin + 1]; ++q) {
    int e = B->v2t[q];
    int n1 = B->tri[3 * e], n2 = B->tri[3 * e + 1], n3 = B->tri[3 * e + 2];
    double xv[3] = {B->xv[n1], B->xv[n2], B->xv[n3]};
    double yv[3] = {B->yv[n1], B->yv[n2], B->yv[n3]};
    double zv[3] = {B->zv[n1], B->zv[n2], B->zv[n3]};
    double xn = B->enx[e], yn = B->eny[e], zn = B->enz[e];
    double xvn[3] = {B->vnx[n1], B->vnx[n2], B->vnx[n3]};
    double yvn[3] = {B->vny[n1], B->vny[n2], B->vny[n3]};
    double zvn[3] = {B->vnz[n1], B->vnz[n2], B->vnz[n3]};
    double planeConst = -xn * xv[0] - yn * yv[0] - zn * zv[0];
    double dtp = -(xn * xC + yn * yC + zn * zC + planeConst);
    double xt = xC + xn * dtp, yt = yC + yn * dtp, zt = zC + zn * dtp;
    double a123, adiff;
    bi_inside_triangle(xv, yv, zv, xt, yt, zt, &a123, &adiff);
    double dist = sqrt((xC - xt) * (xC - xt) + (yC - yt) * (yC - yt) + (zC - zt) * (zC - zt));
    double tnx, tny, tnz;
    if (fabs(adiff) < 1.0e-6 * a123) {
      tnx = xn; tny = yn; tnz = zn;
    } else {
      bi_outside_triangle(xv, yv, zv, xC, yC, zC, xvn, yvn, zvn, &xt, &yt, &zt,
                          &dist, &tnx, &tny, &tnz, &c->nWarnSide);
    }
    if (dist <= distMin) {
      distMin = dist; cel = e; xb = xt; yb = yt; zb = zt;
      bnx = tnx; bny = tny; bnz = tnz;
    }
  }
  double d = sqrt((xb - xC) * (xb - xC) + (yb - yC) * (yb - yC) + (zb - zC) * (zb - zC));
  *xBI = xb; *yBI = yb; *zBI = zb; *closest = cel; *distOut = d;
  *dotNorm = (xC - xb) * bnx + (yC - yb) * bny + (zC - zb) * bnz;
}

/* ------------------------------------------------------------- tagging */
int or_set_iblank_body_fast(or_case *c, int ntime, int ntime_start) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  if (c->nbody < 1) return OR_BAD_INPUT;
  memset(c->bodyNum, 0, (size_t)c->ntot);
  memset(c->iblankTemp, 0, (size_t)c->ntot);
  /* iblankUndecided = UNDECIDED over (0:nx, yb1:yb2, zb1:zb2) (:88-94);
   * stored here as a band flag: 1 = -UNDECIDED (band), 0 = +UNDECIDED */
  memset(c->undecided, 0, (size_t)c->ntot);
  const int yc_start = 1, yc_end = ny - 1, zc_start = 1, zc_end = nz - 1;
  const int y_start = 1, y_end = ny, z_start = 1, z_end = nz;
  /* :153-396 band marking */
  for (int ib = c->nbody - 1; ib >= 0; --ib) {
    or_body *B = &c->body[ib];
    int Nm = (B->type == OR_MEMBRANE) ? 3 : 0;
    double mt = B->membrane_tkns;
    for (int m = 0; m < B->ntri; ++m) {
      int v1 = B->tri[3 * m], v2 = B->tri[3 * m + 1], v3 = B->tri[3 * m + 2];
      double xv[3] = {B->xv[v1], B->xv[v2], B->xv[v3]};
      double yv[3] = {B->yv[v1], B->yv[v2], B->yv[v3]};
      double zv[3] = {B->zv[v1], B->zv[v2], B->zv[v3]};
      double mtN = mt * (double)Nm;
      if ((xv[0] <= c->x[1] && xv[1] <= c->x[1] && xv[2] <= c->x[1]) ||
          (xv[0] >= c->x[nx] && xv[1] >= c->x[nx] && xv[2] >= c->x[nx]) ||
          (yv[0] + mtN <= c->y[y_start] && yv[1] + mtN <= c->y[y_start] && yv[2] + mtN <= c->y[y_start]) ||
          (yv[0] - mtN >= c->y[y_end] && yv[1] - mtN >= c->y[y_end] && yv[2] - mtN >= c->y[y_end]) ||
          (zv[0] + mtN <= c->z[z_start] && zv[1] + mtN <= c->z[z_start] && zv[2] + mtN <= c->z[z_start]) ||
          (zv[0] - mtN >= c->z[z_end] && zv[1] - mtN >= c->z[z_end] && zv[2] - mtN >= c->z[z_end]))
        continue;
      double xmn = xv[0], xmx = xv[0], ymn = yv[0], ymx = yv[0], zmn = zv[0], zmx = zv[0];
      for (int q = 1; q < 3; ++q) {
        if (xv[q] < xmn) xmn = xv[q];
        if (xv[q] > xmx) xmx = xv[q];
        if (yv[q] < ymn) ymn = yv[q];
        if (yv[q] > ymx) ymx = yv[q];
        if (zv[q] < zmn) zmn = zv[q];
        if (zv[q] > zmx) zmx = zv[q];
      }
      if (B->type == OR_MEMBRANE) {
        xmn = xmn - mtN; xmx = xmx + mtN; ymn = ymn - mtN; ymx = ymx + mtN;
        zmn = zmn - mtN; zmx = zmx + mtN;
      }
      int iMin = 0, iMax = 0, jMin = yc_start - 1, jMax = yc_start - 1;
      int kMin = zc_start - 1, kMax = zc_start - 1;
      for (int i = 0; i <= nx - 1; ++i) {
        if ((c->xc[i] - xmn) * (c->xc[i + 1] - xmn) <= 0.0) iMin = i;
        if ((c->xc[i] - xmx) * (c->xc[i + 1] - xmx) <= 0.0) iMax = i + 1;
      }
      if (iMin == 0) iMin = 1;
      if (iMax == 0 || iMax == nx) iMax = nx - 1;
      for (int j = yc_start - 1; j <= yc_end; ++j) {
        if ((c->yc[j] - ymn) * (c->yc[j + 1] - ymn) <= 0.0) jMin = j;
        if ((c->yc[j] - ymx) * (c->yc[j + 1] - ymx) <= 0.0) jMax = j + 1;
      }
      if (jMin == yc_start - 1) jMin = yc_start;
      if (jMax == yc_start - 1 || jMax == yc_end + 1) jMax = yc_end;
      for (int k = zc_start - 1; k <= zc_end; ++k) {
        if ((c->zc[k] - zmn) * (c->zc[k + 1] - zmn) <= 0.0) kMin = k;
        if ((c->zc[k] - zmx) * (c->zc[k + 1] - zmx) <= 0.0) kMax = k + 1;
      }
      if (kMin == zc_start - 1) kMin = zc_start;
      if (kMax == zc_start - 1 || kMax == zc_end + 1) kMax = zc_end;
      for (int k = kMin; k <= kMax; ++k)
        for (int j = jMin; j <= jMax; ++j)
          for (int i = iMin; i <= iMax; ++i) c->undecided[IDX(c, i, j, k)] = 1;
    }
  }
  /* :417-474 dot-normal classification of band cells */
  for (int k = zc_start; k <= zc_end; ++k)
    for (int j = yc_start; j <= yc_end; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        long id = IDX(c, i, j, k);
        if (!c->undecided[id]) continue;
        double xP = c->xc[i], yP = c->yc[j], zP = c->zc[k];
        int hit = 0;
        for (int ib = c->nbody - 1; ib >= 0; --ib) {
          double xb, yb, zb, dist, dn;
          int ce;
          body_intercept(c, ib, xP, yP, zP, &xb, &yb, &zb, &ce, &dist, &dn);
          if (c->body[ib].type == OR_MEMBRANE) {
            double de = sqrt((xP - xb) * (xP - xb) + (yP - yb) * (yP - yb) + (zP - zb) * (zP - zb));
            if (de < c->body[ib].membrane_tkns / 2.0) { hit = ib + 1; break; }
          } else {
            if (dn >= 0.0) { hit = ib + 1; break; }
          }
        }
        c->iblankTemp[id] = hit ? 1 : 0;
        if (hit) c->bodyNum[id] = (int8_t)hit;
      }
  /* :509-536 i-direction fill */
  for (int k = zc_start; k <= zc_end; ++k)
    for (int j = yc_start; j <= yc_end; ++j) {
      for (int ii = 1; ii <= nx - 1; ++ii) {
        long id = IDX(c, ii, j, k);
        if (!c->undecided[id]) continue;
        c->iblankTemp[IDX(c, 0, j, k)] = c->iblankTemp[id];
        c->bodyNum[IDX(c, 0, j, k)] = c->bodyNum[id];
        break;
      }
      for (int i = 1; i <= nx - 1; ++i) {
        long id = IDX(c, i, j, k);
        if (c->undecided[id]) continue;
        c->iblankTemp[id] = c->iblankTemp[id - 1];
        if (c->iblankTemp[id] == 1) c->bodyNum[id] = c->bodyNum[id - 1];
      }
    }
  /* :725-730 outflow copy */
  for (int j = yc_start; j <= yc_end; ++j)
    for (int k = zc_start; k <= zc_end; ++k) {
      c->iblankTemp[IDX(c, nx, j, k)] = c->iblankTemp[IDX(c, nx - 1, j, k)];
      c->bodyNum[IDX(c, nx, j, k)] = c->bodyNum[IDX(c, nx - 1, j, k)];
    }
  /* :763-787 commit */
  for (int k = zc_start; k <= zc_end; ++k)
    for (int j = yc_start; j <= yc_end; ++j)
      for (int i = 0; i <= nx; ++i) {
        long id = IDX(c, i, j, k);
        (void)ntime; (void)ntime_start;
        c->iblank[id] = c->iblankTemp[id];
      }
  return OR_OK;
}

/* ---------------------------------------------------- 8x8 inverse (LAPACK
 * DGETRF + DGETRI semantics: partial pivoting on max |a|, first index on
 * ties, inverse of U then solve inv(A) L = inv(U), column interchanges).
 * MKL's exact operation order is not published; weights built from this
 * inverse are compared to the CUDA path to a relative tolerance. */
static int invert_n(int N, const double *a_in, double *inv, int *info) {
  double a[64];
  int ipiv[8];
  memcpy(a, a_in, sizeof(double) * (size_t)(N * N));
#define A(i, j) a[(i) + N * (j)]
  *info = 0;
  for (int j = 0; j < N; ++j) {
    int p = j;
    double mx = fabs(A(j, j));
    for (int i = j + 1; i < N; ++i)
      if (fabs(A(i, j)) > mx) { mx = fabs(A(i, j)); p = i; }
    ipiv[j] = p;
    if (A(p, j) == 0.0) { if (*info == 0) *info = j + 1; continue; }
    if (p != j)
      for (int q = 0; q < N; ++q) { double t = A(j, q); A(j, q) = A(p, q); A(p, q) = t; }
    double r = 1.0 / A(j, j);
    for (int i = j + 1; i < N; ++i) A(i, j) = A(i, j) * r;
    for (int q = j + 1; q < N; ++q)
      for (int i = j + 1; i < N; ++i) A(i, q) = A(i, q) - A(i, j) * A(j, q);
  }
  if (*info != 0) { memcpy(inv, a, sizeof(double) * (size_t)(N * N)); return OR_BAD_INPUT; }
  /* DTRTRI: inverse of upper-triangular U in place */
  for (int j = 0; j < N; ++j) {
    A(j, j) = 1.0 / A(j, j);
    double ajj = -A(j, j);
    /* x = triu(A(0:j-1,0:j-1)) * A(0:j-1, j) */
    for (int i = 0; i < j; ++i) {
      double s = 0.0;
      for (int q = i; q < j; ++q) s = s + A(i, q) * A(q, j);
      inv[i] = s;
    }
    for (int i = 0; i < j; ++i) A(i, j) = inv[i] * ajj;
  }
  /* DGETRI: solve inv(A)*L = inv(U) column by column from the right */
  double work[8];
  for (int j = N - 1; j >= 0; --j) {
    for (int i = j + 1; i < N; ++i) { work[i] = A(i, j); A(i, j) = 0.0; }
    for (int q = j + 1; q < N; ++q)
      for (int i = 0; i < N; ++i) A(i, j) = A(i, j) - A(i, q) * work[q];
  }
  for (int j = N - 2; j >= 0; --j) {
    int jp = ipiv[j];
    if (jp != j)
      for (int i = 0; i < N; ++i) { double t = A(i, j); A(i, j) = A(i, jp); A(i, jp) = t; }
  }
#undef A
  memcpy(inv, a, sizeof(double) * (size_t)(N * N));
  return OR_OK;
}

int or_invert8(const double *a_in, double *inv, int *info) { return invert_n(8, a_in, inv, info); }

static const int incI[8] = {0, 0, 1, 1, 0, 0, 1, 1}; /* GCM_MEMORY_ALLOCATE.F90:593-623 */
static const int incJ[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int incK[8] = {0, 0, 0, 0, 1, 1, 1, 1};

/* GCM_SET_BOUNDARY.F90:607-797 */
static int van_matrix_dn(or_case *c, int iG, int jG, int kG, int ic, int jc,
                         int kc, double xIP, double yIP, double zIP,
                         double xBI, double yBI, double zBI, double xN,
                         double yN, double zN, double *cD, double *cN) {
  double vD[64], vN[64], iD[64], iN[64];
  for (int r = 0; r < 8; ++r) {
    int i = ic + incI[r], j = jc + incJ[r], k = kc + incK[r];
    double x1 = c->xc[i], x2 = c->yc[j], x3 = c->zc[k];
    double rowD[8] = {x1 * x2 * x3, x1 * x2, x1 * x3, x2 * x3, x1, x2, x3, 1.0};
    double rowN[8];
    memcpy(rowN, rowD, sizeof(rowD));
    if (i == iG && j == jG && k == kG) {
      x1 = xBI; x2 = yBI; x3 = zBI;
      rowD[0] = x1 * x2 * x3; rowD[1] = x1 * x2; rowD[2] = x1 * x3; rowD[3] = x2 * x3;
      rowD[4] = x1; rowD[5] = x2; rowD[6] = x3; rowD[7] = 1.0;
      rowN[0] = xN * x2 * x3 + yN * x1 * x3 + zN * x1 * x2;
      rowN[1] = xN * x2 + yN * x1;
      rowN[2] = xN * x3 + zN * x1;
      rowN[3] = yN * x3 + zN * x2;
      rowN[4] = xN; rowN[5] = yN; rowN[6] = zN; rowN[7] = 0.0;
    }
    for (int q = 0; q < 8; ++q) { vD[r + 8 * q] = rowD[q]; vN[r + 8 * q] = rowN[q]; }
  }
  int info1, info2;
  or_invert8(vD, iD, &info1);
  or_invert8(vN, iN, &info2);
  for (int r = 0; r < 8; ++r) {
    cD[r] = iD[0 + 8 * r] * xIP * yIP * zIP + iD[1 + 8 * r] * xIP * yIP + iD[2 + 8 * r] * xIP * zIP +
            iD[3 + 8 * r] * yIP * zIP + iD[4 + 8 * r] * xIP + iD[5 + 8 * r] * yIP +
            iD[6 + 8 * r] * zIP + iD[7 + 8 * r];
    cN[r] = iN[0 + 8 * r] * xIP * yIP * zIP + iN[1 + 8 * r] * xIP * yIP + iN[2 + 8 * r] * xIP * zIP +
            iN[3 + 8 * r] * yIP * zIP + iN[4 + 8 * r] * xIP + iN[5 + 8 * r] * yIP +
            iN[6 + 8 * r] * zIP + iN[7 + 8 * r];
  }
  return (info1 || info2) ? OR_BAD_INPUT : OR_OK;
}

/* NINT: round half away from zero */
static int nint(double v) { return (int)(v >= 0.0 ? floor(v + 0.5) : -floor(-v + 0.5)); }

/* GCM_SET_BOUNDARY.F90:1618-1697 smooth_iblank (in place, k-j-i order) */
static int smooth_iblank(or_case *c) {
  int nb = 0;
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  int ibody = 0;
  for (int it = 0; it < 5; ++it)
    for (int k = 1; k <= nz - 1; ++k)
      for (int j = 1; j <= ny - 1; ++j)
        for (int i = 1; i <= nx - 1; ++i) {
          long id = IDX(c, i, j, k);
          if (c->iblank[id] == 1) continue;
          int s = 0;
          long nb6[6] = {IDX(c, i, j, k - 1), IDX(c, i, j - 1, k), IDX(c, i - 1, j, k),
                         IDX(c, i + 1, j, k), IDX(c, i, j + 1, k), IDX(c, i, j, k + 1)};
          for (int q = 0; q < 6; ++q)
            if (c->iblank[nb6[q]] == 1) {
              s++;
              if (c->bodyNum[nb6[q]] > 0) ibody = c->bodyNum[nb6[q]];
            }
          if (s >= 5) { c->iblank[id] = 1; c->bodyNum[id] = (int8_t)ibody; nb++; }
        }
  return nb;
}

static int ghost_dead_setup(or_case *c, double pln, double plnD);

int or_gcm_set_internal_boundary(or_case *c, double pln, double plnD) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  smooth_iblank(c);
  int ibody = 0;
  /* GCM_SET_BOUNDARY.F90:132-169: 2-D passes in x planes (i outer, j, k) */
  for (int it = 0; it < 5; ++it)
    for (int i = 1; i <= nx - 1; ++i)
      for (int j = 1; j <= ny - 1; ++j)
        for (int k = 1; k <= nz - 1; ++k) {
          long id = IDX(c, i, j, k);
          if (c->iblank[id] == 1) continue;
          int s = 0;
          long nb4[4] = {IDX(c, i, j, k - 1), IDX(c, i, j - 1, k), IDX(c, i, j + 1, k), IDX(c, i, j, k + 1)};
          for (int q = 0; q < 4; ++q)
            if (c->iblank[nb4[q]] == 1) {
              s++;
              if (c->bodyNum[nb4[q]] > 0) ibody = c->bodyNum[nb4[q]];
            }
          if (s >= 3) { c->iblank[id] = 1; c->bodyNum[id] = (int8_t)ibody; }
        }
  /* :188-223: 2-D passes in y planes (j outer, i, k) */
  for (int it = 0; it < 5; ++it)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        for (int k = 1; k <= nz - 1; ++k) {
          long id = IDX(c, i, j, k);
          if (c->iblank[id] == 1) continue;
          int s = 0;
          long nb4[4] = {IDX(c, i, j, k - 1), IDX(c, i - 1, j, k), IDX(c, i + 1, j, k), IDX(c, i, j, k + 1)};
          for (int q = 0; q < 4; ++q)
            if (c->iblank[nb4[q]] == 1) {
              s++;
              if (c->bodyNum[nb4[q]] > 0) ibody = c->bodyNum[nb4[q]];
            }
          if (s >= 3) { c->iblank[id] = 1; c->bodyNum[id] = (int8_t)ibody; }
        }
  /* :800-876 GCM_define_ghostcells */
  memset(c->ghost, 0, (size_t)c->ntot);
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        long id = IDX(c, i, j, k);
        if (c->iblank[id] != 1) continue;
        int off[6][3] = {{0, 0, -1}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        for (int q = 0; q < 6; ++q) {
          int i2 = i + off[q][0], j2 = j + off[q][1], k2 = k + off[q][2];
          if (i2 < 1 || i2 > nx - 1) continue;
          if (j2 < 1 || j2 > ny - 1) continue;
          if (k2 < 1 || k2 > nz - 1) continue;
          long id2 = IDX(c, i2, j2, k2);
          if (c->iblank[id2] == 0 && c->ghost[id2] == 0) {
            c->ghost[id2] = 1;
            c->bodyNum[id2] = c->bodyNum[id];
          }
        }
      }
  return ghost_dead_setup(c, pln, plnD);
}

static int ghost_dead_setup(or_case *c, double pln, double plnD) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  int status = OR_OK;
  c->nHostFail = 0; c->nStencilSolid = 0;
  /* :270-310 ghost list in k-j-i order */
  int ng = 0;
  memset(c->ghostIndex, 0, sizeof(int32_t) * (size_t)c->ntot);
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        if (c->ghost[IDX(c, i, j, k)] == 1) ng++;
  free_ghosts(c);
  c->nGhost = ng;
  c->gijk = izalloc(3L * ng); c->gcell = izalloc(3L * ng); c->gclosest = izalloc(ng);
  c->gcoefN = dzalloc(8L * ng); c->gcoefD = dzalloc(8L * ng);
  c->gbi = dzalloc(3L * ng); c->gip = dzalloc(3L * ng); c->gprobe = dzalloc(ng); c->gnrm = dzalloc(3L * ng);
  c->galpha = dzalloc(ng);
  ng = 0;
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        if (c->ghost[IDX(c, i, j, k)] == 1) {
          c->gijk[3 * ng] = i; c->gijk[3 * ng + 1] = j; c->gijk[3 * ng + 2] = k;
          ng++;
          c->ghostIndex[IDX(c, i, j, k)] = ng;
        }
  /* :321-537 body intercept, image point, host cell, weights */
  for (int n = 0; n < c->nGhost; ++n) {
    int iG = c->gijk[3 * n], jG = c->gijk[3 * n + 1], kG = c->gijk[3 * n + 2];
    int ib = c->bodyNum[IDX(c, iG, jG, kG)] - 1;
    if (ib < 0) ib = 0;
    double xGC = c->xc[iG], yGC = c->yc[jG], zGC = c->zc[kG];
    double xBI, yBI, zBI, dist, dn;
    int ce;
    body_intercept(c, ib, xGC, yGC, zGC, &xBI, &yBI, &zBI, &ce, &dist, &dn);
    if (c->body[ib].body_dim == 2) zBI = zGC;
    c->gclosest[n] = ce;
    c->gbi[3 * n] = xBI; c->gbi[3 * n + 1] = yBI; c->gbi[3 * n + 2] = zBI;
    double ds = sqrt((xGC - xBI) * (xGC - xBI) + (yGC - yBI) * (yGC - yBI) + (zGC - zBI) * (zGC - zBI));
    double sx = (xGC - xBI) / ds, sy = (yGC - yBI) / ds, sz = (zGC - zBI) / ds;
    if (c->body[ib].type == OR_MEMBRANE) {
      double mt = c->body[ib].membrane_tkns;
      xBI = xBI + mt / 2.0 * sx; yBI = yBI + mt / 2.0 * sy; zBI = zBI + mt / 2.0 * sz;
      ds = sqrt((xGC - xBI) * (xGC - xBI) + (yGC - yBI) * (yGC - yBI) + (zGC - zBI) * (zGC - zBI));
    }
    double bnx = -sx, bny = -sy, bnz = -sz;
    c->gnrm[3 * n] = bnx; c->gnrm[3 * n + 1] = bny; c->gnrm[3 * n + 2] = bnz;  /* xBodyInterceptNorm (:386-388) */
    c->gprobe[n] = ds * pln;
    double xIP = xBI - (xBI - xGC) * pln;
    double yIP = yBI - (yBI - yGC) * pln;
    double zIP = zBI - (zBI - zGC) * pln;
    c->gip[3 * n] = xIP; c->gip[3 * n + 1] = yIP; c->gip[3 * n + 2] = zIP;
    double maxDelta = c->dx[iG];
    if (c->dy[jG] > maxDelta) maxDelta = c->dy[jG];
    if (c->dz[kG] > maxDelta) maxDelta = c->dz[kG];
    int iR = 2 * nint(maxDelta / c->dx[iG] + 0.5);
    int jR = 2 * nint(maxDelta / c->dy[jG] + 0.5);
    int kR = 2 * nint(maxDelta / c->dz[kG] + 0.5);
    int ic = -1, jc = -1, kc = -1;
    int lo = iG - iR, hi = iG + iR;
    if (lo < 0) lo = 0;
    if (hi > nx) hi = nx;
    for (int i = lo; i <= hi; ++i)
      if (c->xc[i] <= xIP && c->xc[i + 1] > xIP) ic = i;
    lo = jG - jR; hi = jG + jR;
    if (lo < 0) lo = 0; /* yc(-1) lies outside the array; the clause
                           yc(0) > yIP is false for image points inside the
                           domain, so j = -1 can never match there */
    if (hi > ny) hi = ny;
    for (int j = lo; j <= hi; ++j)
      if (c->yc[j] <= yIP && c->yc[j + 1] > yIP) jc = j;
    lo = kG - kR; hi = kG + kR;
    if (lo < 0) lo = 0;
    if (hi > nz) hi = nz;
    for (int k = lo; k <= hi; ++k)
      if (c->zc[k] <= zIP && c->zc[k + 1] > zIP) kc = k;
    c->gcell[3 * n] = ic; c->gcell[3 * n + 1] = jc; c->gcell[3 * n + 2] = kc;
    if (ic < 0 || jc < 0 || kc < 0) {
      c->nHostFail++;
      status = OR_GEOMETRY_NO_HOST_CELL;
      continue;
    }
    van_matrix_dn(c, iG, jG, kG, ic, jc, kc, xGC, yGC, zGC, xBI, yBI, zBI, bnx, bny, bnz,
                  &c->gcoefD[8 * n], &c->gcoefN[8 * n]);
  }

  /* GCM_set_deadcells :880-1491 */
  memset(c->dead, 0, (size_t)c->ntot);
  memset(c->ps1, 0, (size_t)c->ntot);
  memset(c->ps2, 0, (size_t)c->ntot);
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        if (c->ghost[IDX(c, i, j, k)] != 1) continue;
        if (c->iblank[IDX(c, i + 1, j, k)] == 1) c->dead[IDX(c, i + 1, j, k)] = -1;
        if (c->iblank[IDX(c, i - 1, j, k)] == 1) c->dead[IDX(c, i - 1, j, k)] = -1;
        if (c->iblank[IDX(c, i, j + 1, k)] == 1) c->dead[IDX(c, i, j + 1, k)] = -1;
        if (c->iblank[IDX(c, i, j - 1, k)] == 1) c->dead[IDX(c, i, j - 1, k)] = -1;
        if (c->iblank[IDX(c, i, j, k + 1)] == 1) c->dead[IDX(c, i, j, k + 1)] = -1;
        if (c->iblank[IDX(c, i, j, k - 1)] == 1) c->dead[IDX(c, i, j, k - 1)] = -1;
      }
  int nd = 0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        if (abs(c->dead[IDX(c, i, j, k)]) == 1) nd++;
  free_deads(c);
  c->nDead = nd;
  c->dijk = izalloc(3L * nd); c->dcell = izalloc(3L * nd); c->dclosest = izalloc(nd);
  c->dcoefN = dzalloc(8L * nd); c->dcoefD = dzalloc(8L * nd);
  c->dbi = dzalloc(3L * nd); c->dip = dzalloc(3L * nd); c->dprobe = dzalloc(nd); c->dnrm = dzalloc(3L * nd);
  nd = 0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        if (abs(c->dead[IDX(c, i, j, k)]) == 1) {
          c->dijk[3 * nd] = i; c->dijk[3 * nd + 1] = j; c->dijk[3 * nd + 2] = k;
          nd++;
        }
  for (int n = 0; n < c->nGhost; ++n) c->galpha[n] = 0.0;
  for (int n = 0; n < c->nDead; ++n) {
    int iG = c->dijk[3 * n], jG = c->dijk[3 * n + 1], kG = c->dijk[3 * n + 2];
    int ib = c->bodyNum[IDX(c, iG, jG, kG)] - 1;
    if (ib < 0) { status = OR_GEOMETRY_DEAD_NO_BODY; c->dcell[3 * n] = -1; continue; }
    double xDC = c->xc[iG], yDC = c->yc[jG], zDC = c->zc[kG];
    double xBI, yBI, zBI, dist, dn;
    int ce;
    body_intercept(c, ib, xDC, yDC, zDC, &xBI, &yBI, &zBI, &ce, &dist, &dn);
    if (c->body[ib].body_dim == 2) zBI = zDC;
    c->dclosest[n] = ce;
    c->dbi[3 * n] = xBI; c->dbi[3 * n + 1] = yBI; c->dbi[3 * n + 2] = zBI;
    double ds = sqrt((xDC - xBI) * (xDC - xBI) + (yDC - yBI) * (yDC - yBI) + (zDC - zBI) * (zDC - zBI));
    double sx = (xBI - xDC) / ds, sy = (yBI - yDC) / ds, sz = (zBI - zDC) / ds;
    double bnx = -sx, bny = -sy, bnz = -sz;
    c->dnrm[3 * n] = bnx; c->dnrm[3 * n + 1] = bny; c->dnrm[3 * n + 2] = bnz;  /* xNormInterceptDead (:1109-1111) */
    double xIP, yIP, zIP;
    if (c->body[ib].type == OR_MEMBRANE) {
      /* :1115-1216.  The reference tests yIP before assigning it in this
       * branch (its value is left over from the previous dead cell); here
       * the y and z shifts start from the current dead cell's image point. */
      double mt = c->body[ib].membrane_tkns;
      sx = -sx; sy = -sy; sz = -sz;
      if (ds >= mt / 2.0) {
        double s = ds + TENTH_F32 * (ds - mt / 2.0);
        xBI = xBI + s * sx; yBI = yBI + s * sy; zBI = zBI + s * sz;
      } else {
        xBI = xBI + mt / 2.0 * sx; yBI = yBI + mt / 2.0 * sy; zBI = zBI + mt / 2.0 * sz;
      }
      zIP = zDC + (zBI - zDC) * plnD;
      yIP = yDC + (yBI - yDC) * plnD;
      int guard = 0;
      while ((yIP < c->yc[0] || yIP > c->yc[ny + 1]) && guard++ < 200) {
        double d1 = sqrt((xDC - xBI) * (xDC - xBI) + (yDC - yBI) * (yDC - yBI) + (zDC - zBI) * (zDC - zBI));
        double t = -0.5 * d1;
        xBI = xBI + t * sx; yBI = yBI + t * sy; zBI = zBI + t * sz;
        yIP = yDC + (yBI - yDC) * plnD;
      }
      guard = 0;
      while ((zIP < c->zc[0] || zIP > c->zc[nz + 1]) && guard++ < 200) {
        double d1 = sqrt((xDC - xBI) * (xDC - xBI) + (yDC - yBI) * (yDC - yBI) + (zDC - zBI) * (zDC - zBI));
        double t = -0.5 * d1;
        xBI = xBI + t * sx; yBI = yBI + t * sy; zBI = zBI + t * sz;
        zIP = zDC + (zBI - zDC) * plnD;
      }
      ds = sqrt((xDC - xBI) * (xDC - xBI) + (yDC - yBI) * (yDC - yBI) + (zDC - zBI) * (zDC - zBI));
    }
    /* alphaGhost accumulation :1220-1277 */
    int gi;
    if (abs(c->ghost[IDX(c, iG + 1, jG, kG)]) == 1) {
      double t = ds / c->dxc[iG + 1];
      gi = c->ghostIndex[IDX(c, iG + 1, jG, kG)];
      if (gi > 0) c->galpha[gi - 1] = c->galpha[gi - 1] + t * t;
    }
    if (abs(c->ghost[IDX(c, iG - 1, jG, kG)]) == 1) {
      double t = ds / c->dxc[iG];
      gi = c->ghostIndex[IDX(c, iG - 1, jG, kG)];
      if (gi > 0) c->galpha[gi - 1] = c->galpha[gi - 1] + t * t;
    }
    if (abs(c->ghost[IDX(c, iG, jG + 1, kG)]) == 1) {
      double t = ds / c->dyc[jG + 1];
      gi = c->ghostIndex[IDX(c, iG, jG + 1, kG)];
      if (gi > 0) c->galpha[gi - 1] = c->galpha[gi - 1] + t * t;
    }
    if (abs(c->ghost[IDX(c, iG, jG - 1, kG)]) == 1) {
      double t = ds / c->dyc[jG];
      gi = c->ghostIndex[IDX(c, iG, jG - 1, kG)];
      if (gi > 0) c->galpha[gi - 1] = c->galpha[gi - 1] + t * t;
    }
    if (abs(c->ghost[IDX(c, iG, jG, kG + 1)]) == 1) {
      double t = ds / c->dzc[kG + 1];
      gi = c->ghostIndex[IDX(c, iG, jG, kG + 1)];
      if (gi > 0) c->galpha[gi - 1] = c->galpha[gi - 1] + t * t;
    }
    if (abs(c->ghost[IDX(c, iG, jG, kG - 1)]) == 1) {
      double t = ds / c->dzc[kG];
      gi = c->ghostIndex[IDX(c, iG, jG, kG - 1)];
      if (gi > 0) c->galpha[gi - 1] = c->galpha[gi - 1] + t * t;
    }
    xIP = xDC + (xBI - xDC) * plnD;
    yIP = yDC + (yBI - yDC) * plnD;
    zIP = zDC + (zBI - zDC) * plnD;
    c->dprobe[n] = ds * plnD;
    if (yIP < c->yc[0] || yIP > c->yc[ny + 1]) {
      yIP = (fabs(yIP - c->yc[0]) < fabs(yIP - c->yc[ny + 1])) ? c->yc[0] : c->yc[ny + 1];
      c->dprobe[n] = sqrt((xDC - xIP) * (xDC - xIP) + (yDC - yIP) * (yDC - yIP) + (zDC - zIP) * (zDC - zIP));
    }
    if (zIP < c->zc[0] || zIP > c->zc[nz + 1]) {
      zIP = (fabs(zIP - c->zc[0]) < fabs(zIP - c->zc[nz + 1])) ? c->zc[0] : c->zc[nz + 1];
      c->dprobe[n] = sqrt((xDC - xIP) * (xDC - xIP) + (yDC - yIP) * (yDC - yIP) + (zDC - zIP) * (zDC - zIP));
    }
    c->dip[3 * n] = xIP; c->dip[3 * n + 1] = yIP; c->dip[3 * n + 2] = zIP;
    double maxDelta = c->dx[iG];
    if (c->dy[jG] > maxDelta) maxDelta = c->dy[jG];
    if (c->dz[kG] > maxDelta) maxDelta = c->dz[kG];
    int iR = 2 * nint(maxDelta / c->dx[iG] + 0.5);
    int jR = 2 * nint(maxDelta / c->dy[jG] + 0.5);
    int kR = 2 * nint(maxDelta / c->dz[kG] + 0.5);
    int ic = -1, jc = -1, kc = -1;
    int lo = iG - iR, hi = iG + iR;
    if (lo < 0) lo = 0;
    if (hi > nx) hi = nx;
    for (int i = lo; i <= hi; ++i)
      if (c->xc[i] <= xIP && c->xc[i + 1] >= xIP) ic = i;
    lo = jG - jR; hi = jG + jR;
    if (lo < 0) lo = 0;
    if (hi > ny) hi = ny;
    for (int j = lo; j <= hi; ++j)
      if (c->yc[j] <= yIP && c->yc[j + 1] >= yIP) jc = j;
    lo = kG - kR; hi = kG + kR;
    if (lo < 0) lo = 0;
    if (hi > nz) hi = nz;
    for (int k = lo; k <= hi; ++k)
      if (c->zc[k] <= zIP && c->zc[k + 1] >= zIP) kc = k;
    c->dcell[3 * n] = ic; c->dcell[3 * n + 1] = jc; c->dcell[3 * n + 2] = kc;
    if (ic < 0 || jc < 0 || kc < 0) {
      c->nHostFail++;
      status = OR_GEOMETRY_NO_HOST_CELL;
      continue;
    }
    for (int r = 0; r < 8; ++r) {
      long q = IDX(c, ic + incI[r], jc + incJ[r], kc + incK[r]);
      if (c->iblank[q] == 1 && c->dead[q] != -1) c->ps1[IDX(c, iG, jG, kG)] = 10;
    }
    if (c->ps1[IDX(c, iG, jG, kG)] == 10) {
      if (iG - 1 >= 0 && c->ghost[IDX(c, iG - 1, jG, kG)] == 1) c->ps2[IDX(c, iG - 1, jG, kG)] = 10;
      if (iG + 1 <= nx && c->ghost[IDX(c, iG + 1, jG, kG)] == 1) c->ps2[IDX(c, iG + 1, jG, kG)] = 10;
      if (jG - 1 >= 0 && c->ghost[IDX(c, iG, jG - 1, kG)] == 1) c->ps2[IDX(c, iG, jG - 1, kG)] = 10;
      if (jG + 1 <= ny && c->ghost[IDX(c, iG, jG + 1, kG)] == 1) c->ps2[IDX(c, iG, jG + 1, kG)] = 10;
      if (kG - 1 >= 1 && c->ghost[IDX(c, iG, jG, kG - 1)] == 1) c->ps2[IDX(c, iG, jG, kG - 1)] = 10;
      if (kG + 1 <= nz - 1 && c->ghost[IDX(c, iG, jG, kG + 1)] == 1) c->ps2[IDX(c, iG, jG, kG + 1)] = 10;
    }
    van_matrix_dn(c, iG, jG, kG, ic, jc, kc, xIP, yIP, zIP, xBI, yBI, zBI, bnx, bny, bnz,
                  &c->dcoefD[8 * n], &c->dcoefN[8 * n]);
  }
  for (int n = 0; n < c->nGhost; ++n) c->galpha[n] = 1.0 - sqrt(c->galpha[n]);
  /* stencil corners of ghost cells that are pure solid (iblank, not dead):
   * their pressure is never updated by the solver */
  for (int n = 0; n < c->nGhost; ++n) {
    if (c->gcell[3 * n] < 0) continue;
    for (int r = 0; r < 8; ++r) {
      long q = IDX(c, c->gcell[3 * n] + incI[r], c->gcell[3 * n + 1] + incJ[r], c->gcell[3 * n + 2] + incK[r]);
      if (c->iblank[q] == 1 && c->dead[q] != -1) c->nStencilSolid++;
    }
  }
  return status;
}

int or_get_field_i8(const or_case *c, int which, int8_t *out) {
  const int8_t *src = which == 0 ? c->iblank : which == 1 ? c->ghost : which == 2 ? c->dead
                      : which == 3 ? c->bodyNum : which == 4 ? c->undecided
                      : which == 5 ? c->igmark : NULL;
  if (!src) return OR_BAD_INPUT;
  memcpy(out, src, (size_t)c->ntot);
  return OR_OK;
}

int or_get_counts(const or_case *c, int *out) {
  out[0] = c->nGhost; out[1] = c->nDead; out[2] = c->nWarnSide;
  out[3] = c->nHostFail; out[4] = c->nStencilSolid; out[5] = c->nFallbackDead;
  return OR_OK;
}

int or_get_ghosts(const or_case *c, int32_t *ijk, int32_t *cell, double *cN,
                  double *cD, double *bi, double *ip, double *probe,
                  int32_t *closest, double *alpha) {
  int n = c->nGhost;
  if (ijk) memcpy(ijk, c->gijk, sizeof(int32_t) * 3 * (size_t)n);
  if (cell) memcpy(cell, c->gcell, sizeof(int32_t) * 3 * (size_t)n);
  if (cN) memcpy(cN, c->gcoefN, sizeof(double) * 8 * (size_t)n);
  if (cD) memcpy(cD, c->gcoefD, sizeof(double) * 8 * (size_t)n);
  if (bi) memcpy(bi, c->gbi, sizeof(double) * 3 * (size_t)n);
  if (ip) memcpy(ip, c->gip, sizeof(double) * 3 * (size_t)n);
  if (probe) memcpy(probe, c->gprobe, sizeof(double) * (size_t)n);
  if (closest) memcpy(closest, c->gclosest, sizeof(int32_t) * (size_t)n);
  if (alpha) memcpy(alpha, c->galpha, sizeof(double) * (size_t)n);
  return OR_OK;
}

int or_get_deads(const or_case *c, int32_t *ijk, int32_t *cell, double *cN,
                 double *cD, double *bi, double *ip, double *probe,
                 int32_t *closest) {
  int n = c->nDead;
  if (ijk) memcpy(ijk, c->dijk, sizeof(int32_t) * 3 * (size_t)n);
  if (cell) memcpy(cell, c->dcell, sizeof(int32_t) * 3 * (size_t)n);
  if (cN) memcpy(cN, c->dcoefN, sizeof(double) * 8 * (size_t)n);
  if (cD) memcpy(cD, c->dcoefD, sizeof(double) * 8 * (size_t)n);
  if (bi) memcpy(bi, c->dbi, sizeof(double) * 3 * (size_t)n);
  if (ip) memcpy(ip, c->dip, sizeof(double) * 3 * (size_t)n);
  if (probe) memcpy(probe, c->dprobe, sizeof(double) * (size_t)n);
  if (closest) memcpy(closest, c->dclosest, sizeof(int32_t) * (size_t)n);
  return OR_OK;
}

/* ------------------------------------------------------------- MG prep */
int or_mg_prepare(or_case *c) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  memset(c->igmark, 0, (size_t)c->ntot);
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 0; i <= nx; ++i) {
        long id = IDX(c, i, j, k);
        if (c->iblank[id] == 1 || c->ghost[id] == 1) c->igmark[id] = 1;
      }
  or_level *L1 = &c->lev[0];
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 0; i <= nx; ++i) {
        long id = IDX(c, i, j, k);
        L1->ibk[id] = c->iblank[id];
        L1->igk[id] = c->igmark[id];
      }
  for (int N = 1; N < c->mLevel; ++N) {
    or_level *P = &c->lev[N - 1], *L = &c->lev[N];
    int ic = (L->I != P->I), jc = (L->J != P->J), kc = (L->K != P->K);
    long nL = (long)(L->I + 2) * (L->J + 2) * (L->K + 2);
    memset(L->igk, 0, (size_t)nL);
    memset(L->ibk, 0, (size_t)nL);
    for (int k = 1; k <= L->K - 1; ++k)
      for (int j = 1; j <= L->J - 1; ++j)
        for (int i = 1; i <= L->I - 1; ++i) {
          int i1 = (1 - ic) * i + ic * (2 * i - 1), i2 = (1 - ic) * i + ic * (2 * i);
          int j1 = (1 - jc) * j + jc * (2 * j - 1), j2 = (1 - jc) * j + jc * (2 * j);
          int k1 = (1 - kc) * k + kc * (2 * k - 1), k2 = (1 - kc) * k + kc * (2 * k);
          double vol0 = 0.0, volb = 0.0;
          for (int kk = k1; kk <= k2; ++kk)
            for (int jj = j1; jj <= j2; ++jj)
              for (int ii = i1; ii <= i2; ++ii) {
                long q = LIDX(P, ii, jj, kk);
                if (P->igk[q] == 1) L->igk[LIDX(L, i, j, k)] = 1;
                double dX = P->x[ii + 1] - P->x[ii];
                double dY = P->y[jj + 1] - P->y[jj];
                double dZ = P->z[kk + 1] - P->z[kk];
                double v = dX * dY * dZ;
                vol0 = vol0 + v;
                if (P->ibk[q] == 1) volb = volb + v;
              }
          if (volb / vol0 >= 0.5) L->ibk[LIDX(L, i, j, k)] = 1;
        }
    memset(L->rhs, 0, sizeof(double) * (size_t)nL);
    memset(L->phi, 0, sizeof(double) * (size_t)nL);
  }
  return OR_OK;
}

int or_get_mg_mask(const or_case *c, int lev, int which, int8_t *out) {
  if (lev < 0 || lev >= c->mLevel) return OR_BAD_INPUT;
  const or_level *L = &c->lev[lev];
  long nL = (long)(L->I + 2) * (L->J + 2) * (L->K + 2);
  memcpy(out, which == 0 ? L->ibk : L->igk, (size_t)nL);
  return OR_OK;
}

/* ------------------------------------------------------- Poisson pieces */
/* CORE_TDMA.F90:10-34 */
int or_tdma(const double *a, const double *b, const double *cc,
            const double *r, double *u, int n1, int n2) {
  double *gam = (double *)malloc(sizeof(double) * (size_t)(n2 + 1));
  double binv = 1.0 / b[n1];
  u[n1] = r[n1] * binv;
  for (int j = n1 + 1; j <= n2; ++j) {
    gam[j] = cc[j - 1] * binv;
    binv = 1.0 / (b[j] - a[j] * gam[j]);
    u[j] = (r[j] - a[j] * u[j - 1]) * binv;
  }
  for (int j = n2 - 1; j >= n1; --j) u[j] = u[j] - gam[j + 1] * u[j + 1];
  free(gam);
  return OR_OK;
}

static void tdma_ws(const double *a, const double *b, const double *cc,
                    const double *r, double *u, int n1, int n2, double *gam) {
  double binv = 1.0 / b[n1];
  u[n1] = r[n1] * binv;
  for (int j = n1 + 1; j <= n2; ++j) {
    gam[j] = cc[j - 1] * binv;
    binv = 1.0 / (b[j] - a[j] * gam[j]);
    u[j] = (r[j] - a[j] * u[j - 1]) * binv;
  }
  for (int j = n2 - 1; j >= n1; --j) u[j] = u[j] - gam[j + 1] * u[j + 1];
}

/* CORE_SET_OUTER_BC.F90:831-1042 then :1044-1186 for a level array */
static void outer_bc(or_case *c, double *pres, int lev, const or_params *prm) {
  const or_level *L = &c->lev[lev];
  const int nxm = L->I;
  const long NXl = L->I + 2, NYl = L->J + 2;
#define PL(i, j, k) pres[(long)(i) + NXl * ((long)(j) + NYl * (long)(k))]
#define BCXP(s, j, k) c->bcxp[(long)(s) + 2 * ((long)(j) + c->NY * (long)(k))]
#define BCYP(i, s, k) c->bcyp[(long)(i) + c->NX * ((long)(s) + 2 * (long)(k))]
#define BCZP(i, j, s) c->bczp[(long)(i) + c->NX * ((long)(j) + c->NY * (long)(s))]
  int iHomo = (lev != 0);
  double pp[6];
  for (int f = 0; f < 6; ++f) pp[f] = iHomo ? 0.0 : prm->ppp[f];
  const int zk1 = 1, zk2 = L->K - 1, yj1 = 1, yj2 = L->J - 1;
  const double hom = (double)(1 - iHomo);
  for (int k = zk1; k <= zk2; ++k)
    for (int j = yj1; j <= yj2; ++j) {
      if (prm->pbc[0] == OR_PBC_DIRICHLET) BCXP(0, j, k) = pp[0];
      else BCXP(0, j, k) = PL(1, j, k) - c->pgradx1[j + c->NY * k] * c->dxc[1] / 2.0 * hom;
      if (prm->pbc[1] == OR_PBC_DIRICHLET) BCXP(1, j, k) = pp[1];
      else BCXP(1, j, k) = PL(nxm - 1, j, k) + c->pgradx2[j + c->NY * k] * c->dxc[nxm] / 2.0 * hom;
    }
  for (int k = zk1; k <= zk2; ++k)
    for (int i = 1; i <= nxm - 1; ++i) {
      if (prm->pbc[2] == OR_PBC_DIRICHLET) BCYP(i, 0, k) = pp[2];
      else BCYP(i, 0, k) = PL(i, 1, k) - c->pgrady1[i + c->NX * k] * c->dyc[1] / 2.0 * hom;
      if (prm->pbc[3] == OR_PBC_DIRICHLET) BCYP(i, 1, k) = pp[3];
      else BCYP(i, 1, k) = PL(i, yj2, k) + c->pgrady2[i + c->NX * k] * c->dyc[c->ny] / 2.0 * hom;
    }
  for (int j = yj1; j <= yj2; ++j)
    for (int i = 1; i <= nxm - 1; ++i) {
      if (prm->pbc[4] == OR_PBC_DIRICHLET) BCZP(i, j, 0) = pp[4];
      else BCZP(i, j, 0) = PL(i, j, 1) - c->pgradz1[i + c->NX * j] * c->dzc[1] / 2.0 * hom;
      if (prm->pbc[5] == OR_PBC_DIRICHLET) BCZP(i, j, 1) = pp[5];
      else BCZP(i, j, 1) = PL(i, j, zk2) + c->pgradz2[i + c->NX * j] * c->dzc[c->nz] / 2.0 * hom;
    }
  /* set_outer_ghost_pressure */
  for (int k = zk1; k <= zk2; ++k)
    for (int j = yj1; j <= yj2; ++j) {
      PL(0, j, k) = 2.0 * BCXP(0, j, k) - PL(1, j, k);
      PL(nxm, j, k) = 2.0 * BCXP(1, j, k) - PL(nxm - 1, j, k);
    }
  for (int k = zk1; k <= zk2; ++k)
    for (int i = 0; i <= nxm; ++i) PL(i, 0, k) = 2.0 * BCYP(i, 0, k) - PL(i, 1, k);
  for (int k = zk1; k <= zk2; ++k)
    for (int i = 0; i <= nxm; ++i) PL(i, yj2 + 1, k) = 2.0 * BCYP(i, 1, k) - PL(i, yj2, k);
  for (int j = yj1; j <= yj2; ++j)
    for (int i = 0; i <= nxm; ++i) PL(i, j, 0) = 2.0 * BCZP(i, j, 0) - PL(i, j, 1);
  for (int j = yj1; j <= yj2; ++j)
    for (int i = 0; i <= nxm; ++i) PL(i, j, zk2 + 1) = 2.0 * BCZP(i, j, 1) - PL(i, j, zk2);
#undef BCXP
#undef BCYP
#undef BCZP
#undef PL
}

/* itsolv_mg on `ns` z-slabs at once (ns = threads), as the reference runs
 * it on nProcZ MPI ranks (CORE_PARALLEL pencils, one plane of halo): inside
 * a slab the sweeps are the sequential ones above; across slab faces the
 * neighbour's plane is its value before the sweep (a copy taken after each
 * outer_bc, as the ranks exchange halos), and z lines are solved per slab
 * segment with those halo values as fixed end rows.  ns = 1 is exactly the
 * sequential sweep.  Used only for the timed CPU baseline. */
static void itsolv_mg_slabs(or_case *c, int lev, double *var, const double *r,
                            const int8_t *igk, const or_params *prm, int ns) {
  const or_level *L = &c->lev[lev];
  const int nxm = L->I, JL1 = 1, JL2 = L->J - 1, KL1 = 1, KL2 = L->K - 1;
  const long NXl = L->I + 2, NYl = L->J + 2, PL = NXl * NYl;
  const double om = prm->omega_pson;
  const int nk = KL2 - KL1 + 1;
  int nmax = L->I > L->J ? L->I : L->J;
  if (L->K > nmax) nmax = L->K;
  double *halo = dzalloc(2L * ns * PL);  /* slab s: [2s] plane lo-1, [2s+1] plane hi+1 */
#define V(i, j, k) var[(long)(i) + NXl * ((long)(j) + NYl * (long)(k))]
#define R(i, j, k) r[(long)(i) + NXl * ((long)(j) + NYl * (long)(k))]
#define G(i, j, k) igk[(long)(i) + NXl * ((long)(j) + NYl * (long)(k))]
#define SLO(s) (KL1 + (int)(((long)nk * (s)) / ns))
#define SHI(s) (KL1 + (int)(((long)nk * ((s) + 1)) / ns) - 1)
#define VH(i, j, k)                                                                              \
  ((k) < lo ? halo[(2L * s) * PL + (i) + NXl * (long)(j)]                                       \
            : (k) > hi ? halo[(2L * s + 1) * PL + (i) + NXl * (long)(j)] : V(i, j, k))
#define TAKE_HALOS()                                                                             \
  for (int s = 0; s < ns; ++s) {                                                                 \
    memcpy(halo + (2L * s) * PL, var + (long)(SLO(s) - 1) * PL, sizeof(double) * (size_t)PL);    \
    memcpy(halo + (2L * s + 1) * PL, var + (long)(SHI(s) + 1) * PL, sizeof(double) * (size_t)PL); \
  }
  /* x lines */
  outer_bc(c, var, lev, prm);
  TAKE_HALOS();
#pragma omp parallel for num_threads(ns) schedule(static, 1)
  for (int s = 0; s < ns; ++s) {
    const int lo = SLO(s), hi = SHI(s);
    double *w = dzalloc(6L * (nmax + 2));
    double *am = w, *ac = w + (nmax + 2), *ap = w + 2 * (nmax + 2), *rh = w + 3 * (nmax + 2);
    double *du = w + 4 * (nmax + 2), *g = w + 5 * (nmax + 2);
    for (int k = lo; k <= hi; ++k) {
      double amz = L->dzcinv[k] * L->dzinv[k];
      double apz = L->dzcinv[k + 1] * L->dzinv[k];
      double acz = -(amz + apz);
      for (int j = JL1; j <= JL2; ++j) {
        double amy = L->dycinv[j] * L->dyinv[j];
        double apy = L->dycinv[j + 1] * L->dyinv[j];
        double acy = -(amy + apy);
        for (int i = 1; i <= nxm - 1; ++i) {
          am[i] = L->dxcinv[i] * L->dxinv[i];
          ap[i] = L->dxcinv[i + 1] * L->dxinv[i];
          ac[i] = -(am[i] + ap[i]);
          rh[i] = R(i, j, k) - V(i, j - 1, k) * amy - V(i, j + 1, k) * apy - VH(i, j, k - 1) * amz -
                  VH(i, j, k + 1) * apz;
          double flag = (double)(1 - G(i, j, k));
          am[i] = am[i] * flag;
          ap[i] = ap[i] * flag;
          ac[i] = (ac[i] + acy + acz) * flag + (1.0 - flag);
          rh[i] = rh[i] * flag + (1.0 - flag) * V(i, j, k);
          if (fabs(ac[i]) < TINY_F32) { am[i] = 0.0; ap[i] = 0.0; ac[i] = 1.0; rh[i] = V(i, j, k); }
        }
        am[0] = 0.0; ap[0] = 0.0; ac[0] = 1.0; rh[0] = V(0, j, k);
        am[nxm] = 0.0; ap[nxm] = 0.0; ac[nxm] = 1.0; rh[nxm] = V(nxm, j, k);
        tdma_ws(am, ac, ap, rh, du, 0, nxm, g);
        for (int i = 0; i <= nxm; ++i) V(i, j, k) = V(i, j, k) * (1.0 - om) + om * du[i];
      }
    }
    free(w);
  }
  /* y lines, zebra in i */
  const int j0 = JL1 - 1, j1 = JL2 + 1;
  for (int col = 1; col <= 2; ++col) {
    outer_bc(c, var, lev, prm);
    TAKE_HALOS();
#pragma omp parallel for num_threads(ns) schedule(static, 1)
    for (int s = 0; s < ns; ++s) {
      const int lo = SLO(s), hi = SHI(s);
      double *w = dzalloc(6L * (nmax + 2));
      double *am = w, *ac = w + (nmax + 2), *ap = w + 2 * (nmax + 2), *rh = w + 3 * (nmax + 2);
      double *du = w + 4 * (nmax + 2), *g = w + 5 * (nmax + 2);
      for (int k = lo; k <= hi; ++k) {
        double amz = L->dzcinv[k] * L->dzinv[k];
        double apz = L->dzcinv[k + 1] * L->dzinv[k];
        double acz = -(amz + apz);
        for (int i = col; i <= nxm - 1; i += 2) {
          double amx = L->dxcinv[i] * L->dxinv[i];
          double apx = L->dxcinv[i + 1] * L->dxinv[i];
          double acx = -(amx + apx);
          for (int j = JL1; j <= JL2; ++j) {
            am[j] = L->dycinv[j] * L->dyinv[j];
            ap[j] = L->dycinv[j + 1] * L->dyinv[j];
            ac[j] = -(am[j] + ap[j]);
            rh[j] = R(i, j, k) - V(i - 1, j, k) * amx - V(i + 1, j, k) * apx - VH(i, j, k - 1) * amz -
                    VH(i, j, k + 1) * apz;
            double flag = (double)(1 - G(i, j, k));
            am[j] = am[j] * flag;
            ap[j] = ap[j] * flag;
            ac[j] = (acx + ac[j] + acz) * flag + (1.0 - flag);
            rh[j] = rh[j] * flag + (1.0 - flag) * V(i, j, k);
            if (fabs(ac[j]) < TINY_F32) { am[j] = 0.0; ap[j] = 0.0; ac[j] = 1.0; rh[j] = V(i, j, k); }
          }
          am[j0] = 0.0; ap[j0] = 0.0; ac[j0] = 1.0; rh[j0] = V(i, JL1 - 1, k);
          am[j1] = 0.0; ap[j1] = 0.0; ac[j1] = 1.0; rh[j1] = V(i, JL2 + 1, k);
          tdma_ws(am, ac, ap, rh, du, j0, j1, g);
          for (int j = j0; j <= j1; ++j) V(i, j, k) = V(i, j, k) * (1.0 - om) + om * du[j];
        }
      }
      free(w);
    }
  }
  /* z lines, one segment per slab between the halo planes */
  outer_bc(c, var, lev, prm);
  TAKE_HALOS();
#pragma omp parallel for num_threads(ns) schedule(static, 1)
  for (int s = 0; s < ns; ++s) {
    const int lo = SLO(s), hi = SHI(s);
    double *w = dzalloc(6L * (nmax + 2));
    double *am = w, *ac = w + (nmax + 2), *ap = w + 2 * (nmax + 2), *rh = w + 3 * (nmax + 2);
    double *du = w + 4 * (nmax + 2), *g = w + 5 * (nmax + 2);
    for (int j = JL1; j <= JL2; ++j) {
      double amy = L->dycinv[j] * L->dyinv[j];
      double apy = L->dycinv[j + 1] * L->dyinv[j];
      double acy = -(amy + apy);
      for (int i = 1; i <= nxm - 1; ++i) {
        double amx = L->dxcinv[i] * L->dxinv[i];
        double apx = L->dxcinv[i + 1] * L->dxinv[i];
        double acx = -(amx + apx);
        for (int k = lo; k <= hi; ++k) {
          am[k] = L->dzcinv[k] * L->dzinv[k];
          ap[k] = L->dzcinv[k + 1] * L->dzinv[k];
          ac[k] = -(am[k] + ap[k]);
          rh[k] = R(i, j, k) - V(i - 1, j, k) * amx - V(i + 1, j, k) * apx - V(i, j - 1, k) * amy -
                  V(i, j + 1, k) * apy;
          double flag = (double)(1 - G(i, j, k));
          am[k] = am[k] * flag;
          ap[k] = ap[k] * flag;
          ac[k] = (acx + acy + ac[k]) * flag + (1.0 - flag);
          rh[k] = rh[k] * flag + (1.0 - flag) * V(i, j, k);
          if (fabs(ac[k]) < TINY_F32) { am[k] = 0.0; ap[k] = 0.0; ac[k] = 1.0; rh[k] = V(i, j, k); }
        }
        am[lo - 1] = 0.0; ap[lo - 1] = 0.0; ac[lo - 1] = 1.0; rh[lo - 1] = VH(i, j, lo - 1);
        am[hi + 1] = 0.0; ap[hi + 1] = 0.0; ac[hi + 1] = 1.0; rh[hi + 1] = VH(i, j, hi + 1);
        tdma_ws(am, ac, ap, rh, du, lo - 1, hi + 1, g);
        for (int k = lo; k <= hi; ++k) V(i, j, k) = V(i, j, k) * (1.0 - om) + om * du[k];
      }
    }
    free(w);
  }
#undef TAKE_HALOS
#undef VH
#undef SLO
#undef SHI
#undef V
#undef R
#undef G
  free(halo);
}

/* CORE_MG.F90:615-938 itsolv_mg (one line-SOR sweep x, zebra y, z) */
static void itsolv_mg(or_case *c, int lev, double *var, const double *r,
                      const int8_t *igk, const or_params *prm) {
  {
    const int nk = c->lev[lev].K - 1;
    const int ns = g_threads < nk ? g_threads : nk;
    if (ns > 1) { itsolv_mg_slabs(c, lev, var, r, igk, prm, ns); return; }
  }
  const or_level *L = &c->lev[lev];
  const int nxm = L->I, JL1 = 1, JL2 = L->J - 1, KL1 = 1, KL2 = L->K - 1;
  const long NXl = L->I + 2, NYl = L->J + 2;
  const double om = prm->omega_pson;
  double *am = c->am, *ac = c->ac, *ap = c->ap, *rh = c->rr, *du = c->dum;
  double gam[1100];
  double *g = gam;
  double *gbig = NULL;
  int nmax = L->I > L->J ? L->I : L->J;
  if (L->K > nmax) nmax = L->K;
  if (nmax + 2 > 1100) { gbig = (double *)malloc(sizeof(double) * (size_t)(nmax + 2)); g = gbig; }
#define V(i, j, k) var[(long)(i) + NXl * ((long)(j) + NYl * (long)(k))]
#define R(i, j, k) r[(long)(i) + NXl * ((long)(j) + NYl * (long)(k))]
#define G(i, j, k) igk[(long)(i) + NXl * ((long)(j) + NYl * (long)(k))]
  /* x lines */
  outer_bc(c, var, lev, prm);
  for (int k = KL1; k <= KL2; ++k) {
    double amz = L->dzcinv[k] * L->dzinv[k];
    double apz = L->dzcinv[k + 1] * L->dzinv[k];
    double acz = -(amz + apz);
    for (int j = JL1; j <= JL2; ++j) {
      double amy = L->dycinv[j] * L->dyinv[j];
      double apy = L->dycinv[j + 1] * L->dyinv[j];
      double acy = -(amy + apy);
      for (int i = 1; i <= nxm - 1; ++i) {
        am[i] = L->dxcinv[i] * L->dxinv[i];
        ap[i] = L->dxcinv[i + 1] * L->dxinv[i];
        ac[i] = -(am[i] + ap[i]);
        rh[i] = R(i, j, k) - V(i, j - 1, k) * amy - V(i, j + 1, k) * apy - V(i, j, k - 1) * amz -
                V(i, j, k + 1) * apz;
        double flag = (double)(1 - G(i, j, k));
        am[i] = am[i] * flag;
        ap[i] = ap[i] * flag;
        ac[i] = (ac[i] + acy + acz) * flag + (1.0 - flag);
        rh[i] = rh[i] * flag + (1.0 - flag) * V(i, j, k);
        if (fabs(ac[i]) < TINY_F32) { am[i] = 0.0; ap[i] = 0.0; ac[i] = 1.0; rh[i] = V(i, j, k); }
      }
      am[0] = 0.0; ap[0] = 0.0; ac[0] = 1.0; rh[0] = V(0, j, k);
      am[nxm] = 0.0; ap[nxm] = 0.0; ac[nxm] = 1.0; rh[nxm] = V(nxm, j, k);
      tdma_ws(am, ac, ap, rh, du, 0, nxm, g);
      for (int i = 0; i <= nxm; ++i) V(i, j, k) = V(i, j, k) * (1.0 - om) + om * du[i];
    }
  }
  /* y lines, zebra in i */
  const int j0 = JL1 - 1, j1 = JL2 + 1;
  for (int col = 1; col <= 2; ++col) {
    outer_bc(c, var, lev, prm);
    for (int k = KL1; k <= KL2; ++k) {
      double amz = L->dzcinv[k] * L->dzinv[k];
      double apz = L->dzcinv[k + 1] * L->dzinv[k];
      double acz = -(amz + apz);
      for (int i = col; i <= nxm - 1; i += 2) {
        double amx = L->dxcinv[i] * L->dxinv[i];
        double apx = L->dxcinv[i + 1] * L->dxinv[i];
        double acx = -(amx + apx);
        for (int j = JL1; j <= JL2; ++j) {
          am[j] = L->dycinv[j] * L->dyinv[j];
          ap[j] = L->dycinv[j + 1] * L->dyinv[j];
          ac[j] = -(am[j] + ap[j]);
          rh[j] = R(i, j, k) - V(i - 1, j, k) * amx - V(i + 1, j, k) * apx - V(i, j, k - 1) * amz -
                  V(i, j, k + 1) * apz;
          double flag = (double)(1 - G(i, j, k));
          am[j] = am[j] * flag;
          ap[j] = ap[j] * flag;
          ac[j] = (acx + ac[j] + acz) * flag + (1.0 - flag);
          rh[j] = rh[j] * flag + (1.0 - flag) * V(i, j, k);
          if (fabs(ac[j]) < TINY_F32) { am[j] = 0.0; ap[j] = 0.0; ac[j] = 1.0; rh[j] = V(i, j, k); }
        }
        am[j0] = 0.0; ap[j0] = 0.0; ac[j0] = 1.0; rh[j0] = V(i, JL1 - 1, k);
        am[j1] = 0.0; ap[j1] = 0.0; ac[j1] = 1.0; rh[j1] = V(i, JL2 + 1, k);
        tdma_ws(am, ac, ap, rh, du, j0, j1, g);
        for (int j = j0; j <= j1; ++j) V(i, j, k) = V(i, j, k) * (1.0 - om) + om * du[j];
      }
    }
  }
  /* z lines */
  const int k0 = KL1 - 1, k1 = KL2 + 1;
  outer_bc(c, var, lev, prm);
  for (int j = JL1; j <= JL2; ++j) {
    double amy = L->dycinv[j] * L->dyinv[j];
    double apy = L->dycinv[j + 1] * L->dyinv[j];
    double acy = -(amy + apy);
    for (int i = 1; i <= nxm - 1; ++i) {
      double amx = L->dxcinv[i] * L->dxinv[i];
      double apx = L->dxcinv[i + 1] * L->dxinv[i];
      double acx = -(amx + apx);
      for (int k = KL1; k <= KL2; ++k) {
        am[k] = L->dzcinv[k] * L->dzinv[k];
        ap[k] = L->dzcinv[k + 1] * L->dzinv[k];
        ac[k] = -(am[k] + ap[k]);
        rh[k] = R(i, j, k) - V(i - 1, j, k) * amx - V(i + 1, j, k) * apx - V(i, j - 1, k) * amy -
                V(i, j + 1, k) * apy;
        double flag = (double)(1 - G(i, j, k));
        am[k] = am[k] * flag;
        ap[k] = ap[k] * flag;
        ac[k] = (acx + acy + ac[k]) * flag + (1.0 - flag);
        rh[k] = rh[k] * flag + (1.0 - flag) * V(i, j, k);
        if (fabs(ac[k]) < TINY_F32) { am[k] = 0.0; ap[k] = 0.0; ac[k] = 1.0; rh[k] = V(i, j, k); }
      }
      am[k0] = 0.0; ap[k0] = 0.0; ac[k0] = 1.0; rh[k0] = V(i, j, k0);
      am[k1] = 0.0; ap[k1] = 0.0; ac[k1] = 1.0; rh[k1] = V(i, j, k1);
      tdma_ws(am, ac, ap, rh, du, k0, k1, g);
      for (int k = k0; k <= k1; ++k) V(i, j, k) = V(i, j, k) * (1.0 - om) + om * du[k];
    }
  }
#undef V
#undef R
#undef G
  free(gbig);
}

/* CORE_MG.F90:956-1043 residual_mg: rrr <- (rrr - A var) * flag */
static void residual_mg(const or_case *c, int lev, const double *var,
                        double *rrr, const int8_t *igk) {
  const or_level *L = &c->lev[lev];
  const long NXl = L->I + 2, NYl = L->J + 2;
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1)
  for (int k = 1; k <= L->K - 1; ++k)
    for (int j = 1; j <= L->J - 1; ++j)
      for (int i = 1; i <= L->I - 1; ++i) {
        double bmz = L->dzcinv[k] * L->dzinv[k], bpz = L->dzcinv[k + 1] * L->dzinv[k];
        double bcz = -(bmz + bpz);
        double bmy = L->dycinv[j] * L->dyinv[j], bpy = L->dycinv[j + 1] * L->dyinv[j];
        double bcy = -(bmy + bpy);
        double bmx = L->dxcinv[i] * L->dxinv[i], bpx = L->dxcinv[i + 1] * L->dxinv[i];
        double bcx = -(bmx + bpx);
        long id = i + NXl * (j + NYl * (long)k);
        double flag = 1.0 - (double)igk[id];
        double bc = (bcx + bcy + bcz);
        double res = rrr[id] - var[id] * bc - var[id - 1] * bmx - var[id + 1] * bpx -
                     var[id - NXl] * bmy - var[id + NXl] * bpy - var[id - NXl * NYl] * bmz -
                     var[id + NXl * NYl] * bpz;
        rrr[id] = res * flag;
      }
}

/* CORE_MG.F90:1061-1183 mg_inject (including the sum0 assignment that
 * keeps only the last non-iblank child, :1159) */
static void mg_inject(const or_case *c, int N, const double *rr1, double *rr2) {
  const or_level *F = &c->lev[N], *C = &c->lev[N + 1];
  long nC = (long)(C->I + 2) * (C->J + 2) * (C->K + 2);
  memset(rr2, 0, sizeof(double) * (size_t)nC);
  int ic = (F->I != C->I), jc = (F->J != C->J), kc = (F->K != C->K);
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1)
  for (int k = 1; k <= C->K - 1; ++k)
    for (int j = 1; j <= C->J - 1; ++j)
      for (int i = 1; i <= C->I - 1; ++i) {
        double xc0 = C->xc[i], yc0 = C->yc[j], zc0 = C->zc[k];
        int i1 = (1 - ic) * i + ic * (2 * i - 1), i2 = (1 - ic) * i + ic * (2 * i);
        int j1 = (1 - jc) * j + jc * (2 * j - 1), j2 = (1 - jc) * j + jc * (2 * j);
        int k1 = (1 - kc) * k + kc * (2 * k - 1), k2 = (1 - kc) * k + kc * (2 * k);
        double aX = (xc0 - F->xc[i1]) * F->dxcinv[i1 + 1];
        double aY = (yc0 - F->yc[j1]) * F->dycinv[j1 + 1];
        double aZ = (zc0 - F->zc[k1]) * F->dzcinv[k1 + 1];
#define RF(a, b, d) rr1[LIDX(F, a, b, d)]
        double rt = RF(i1, j1, k1) * (1.0 - aX) * (1.0 - aY) * (1.0 - aZ) +
                    RF(i1 + 1, j1, k1) * aX * (1.0 - aY) * (1.0 - aZ) +
                    RF(i1, j1 + 1, k1) * (1.0 - aX) * aY * (1.0 - aZ) +
                    RF(i1, j1, k1 + 1) * (1.0 - aX) * (1.0 - aY) * aZ +
                    RF(i1 + 1, j1 + 1, k1) * aX * aY * (1.0 - aZ) +
                    RF(i1 + 1, j1, k1 + 1) * aX * (1.0 - aY) * aZ +
                    RF(i1, j1 + 1, k1 + 1) * (1.0 - aX) * aY * aZ +
                    RF(i1 + 1, j1 + 1, k1 + 1) * aX * aY * aZ;
        double vol0 = 0.0, sum0 = 0.0;
        int inside = 0;
        for (int kk = k1; kk <= k2; ++kk)
          for (int jj = j1; jj <= j2; ++jj)
            for (int ii = i1; ii <= i2; ++ii) {
              if (F->ibk[LIDX(F, ii, jj, kk)] == 1) inside = 1;
              else {
                double v = (F->x[ii + 1] - F->x[ii]) * (F->y[jj + 1] - F->y[jj]) * (F->z[kk + 1] - F->z[kk]);
                vol0 = vol0 + v;
                sum0 = RF(ii, jj, kk) * v;
              }
            }
#undef RF
        double volc = 1.0 / F->dxinv[i1] / F->dyinv[j1] / F->dzinv[k1];
        double ravg = (vol0 > CENTI_F32 * volc) ? sum0 / vol0 : 0.0;
        rr2[LIDX(C, i, j, k)] = rt * (double)(1 - inside) + ravg * (double)inside;
      }
}

/* CORE_MG.F90:1200-1351 mg_interp */
static void mg_interp(const or_case *c, int N, const double *phi1,
                      double *phi2, double *dphi) {
  const or_level *C = &c->lev[N], *F = &c->lev[N - 1];
  long nF = (long)(F->I + 2) * (F->J + 2) * (F->K + 2);
  memset(dphi, 0, sizeof(double) * (size_t)nF);
  int ic = (F->I != C->I), jc = (F->J != C->J), kc = (F->K != C->K);
  const int nx2 = F->I, ny2 = F->J, nz2 = F->K, JL1 = 1, JL2 = F->J - 1, KL1 = 1, KL2 = F->K - 1;
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1)
  for (int k = KL1; k <= KL2; ++k)
    for (int j = JL1; j <= JL2; ++j)
      for (int i = 1; i <= nx2 - 1; ++i) {
        if ((i - 1) + (j - 1) == 0) continue;
        if ((i - 1) + (ny2 - 1 - j) == 0) continue;
        if ((nx2 - 1 - i) + (j - 1) == 0) continue;
        if ((nx2 - 1 - i) + (ny2 - 1 - j) == 0) continue;
        if ((i - 1) + (k - KL1) == 0) continue;
        if ((i - 1) + (KL2 - k) == 0) continue;
        if ((nx2 - 1 - i) + (k - KL1) == 0) continue;
        if ((nx2 - 1 - i) + (KL2 - k) == 0) continue;
        if ((j - 1) + (k - KL1) == 0) continue;
        if ((j - 1) + (KL2 - k) == 0) continue;
        if ((ny2 - 1 - j) + (k - KL1) == 0) continue;
        if ((ny2 - 1 - j) + (KL2 - k) == 0) continue;
        if ((k - 1) + (j - JL1) == 0) continue;
        if ((k - 1) + (JL2 - j) == 0) continue;
        if ((nz2 - 1 - k) + (j - JL1) == 0) continue;
        if ((nz2 - 1 - k) + (JL2 - j) == 0) continue;
        if (F->ibk[LIDX(F, i, j, k)] == 1) continue;
        double xc0 = F->xc[i], yc0 = F->yc[j], zc0 = F->zc[k];
        int i1 = (1 - ic) * i + ic * (i / 2), i2 = (1 - ic) * i + ic * (i / 2 + 1);
        int j1 = (1 - jc) * j + jc * (j / 2), j2 = (1 - jc) * j + jc * (j / 2 + 1);
        int k1 = (1 - kc) * k + kc * (k / 2), k2 = (1 - kc) * k + kc * (k / 2 + 1);
        double aX = (xc0 - C->xc[i1]) * C->dxcinv[i1 + 1];
        double aY = (yc0 - C->yc[j1]) * C->dycinv[j1 + 1];
        double aZ = (zc0 - C->zc[k1]) * C->dzcinv[k1 + 1];
#define PC(a, b, d) phi1[LIDX(C, a, b, d)]
        double rt = PC(i1, j1, k1) * (1.0 - aX) * (1.0 - aY) * (1.0 - aZ) +
                    PC(i1 + 1, j1, k1) * aX * (1.0 - aY) * (1.0 - aZ) +
                    PC(i1, j1 + 1, k1) * (1.0 - aX) * aY * (1.0 - aZ) +
                    PC(i1, j1, k1 + 1) * (1.0 - aX) * (1.0 - aY) * aZ +
                    PC(i1 + 1, j1 + 1, k1) * aX * aY * (1.0 - aZ) +
                    PC(i1 + 1, j1, k1 + 1) * aX * (1.0 - aY) * aZ +
                    PC(i1, j1 + 1, k1 + 1) * (1.0 - aX) * aY * aZ +
                    PC(i1 + 1, j1 + 1, k1 + 1) * aX * aY * aZ;
        double vol0 = 0.0, sum0 = 0.0;
        int inside = 0;
        for (int kk = k1; kk <= k2; ++kk)
          for (int jj = j1; jj <= j2; ++jj)
            for (int ii = i1; ii <= i2; ++ii) {
              if (C->ibk[LIDX(C, ii, jj, kk)] == 1) inside = 1;
              else {
                double v = (C->x[ii + 1] - C->x[ii]) * (C->y[jj + 1] - C->y[jj]) * (C->z[kk + 1] - C->z[kk]);
                vol0 = vol0 + v;
                sum0 = PC(ii, jj, kk) * v;
              }
            }
#undef PC
        double volc = 1.0 / C->dxinv[i1] / C->dyinv[j1] / C->dzinv[k1];
        double ravg = (vol0 > CENTI_F32 * volc) ? sum0 / vol0 : 0.0;
        long id = LIDX(F, i, j, k);
        dphi[id] = rt * (double)(1 - inside) + ravg * (double)inside;
        phi2[id] = phi2[id] + dphi[id];
      }
}

/* CORE_POISSON.F90:460-551 calc_residual (L2 / sqrt(nx*ny*nz)) */
double or_calc_residual(const or_case *c, const double *var, const double *r) {
  double res2 = 0.0;
  for (int k = 1; k <= c->nz - 1; ++k)
    for (int j = 1; j <= c->ny - 1; ++j)
      for (int i = 1; i <= c->nx - 1; ++i) {
        double bmx = c->dxcinv[i] * c->dxinv[i], bpx = c->dxcinv[i + 1] * c->dxinv[i];
        double bcx = -(bmx + bpx);
        double bmy = c->dycinv[j] * c->dyinv[j], bpy = c->dycinv[j + 1] * c->dyinv[j];
        double bcy = -(bmy + bpy);
        double bmz = c->dzcinv[k] * c->dzinv[k], bpz = c->dzcinv[k + 1] * c->dzinv[k];
        double bcz = -(bmz + bpz);
        long id = IDX(c, i, j, k);
        double flag = (1.0 - (double)c->iblank[id]) * (1.0 - (double)c->ghost[id]);
        double bc = (bcx + bcy + bcz);
        double res = r[id] - var[id] * bc - var[id - 1] * bmx - var[id + 1] * bpx -
                     var[id - c->NX] * bmy - var[id + c->NX] * bpy -
                     var[id - c->NX * c->NY] * bmz - var[id + c->NX * c->NY] * bpz;
        res = res * flag;
        res2 = res2 + res * res;
      }
  return sqrt(res2 / (double)((long)c->nx * c->ny * c->nz));
}

/* ||f - A p||_2 / ||f||_2 over fluid non-ghost rows: the convergence
 * measure of the synthetic workloads (relative residual 1e-8) */
double or_relres(const or_case *c, const double *var, const double *r) {
  double res2 = 0.0, f2 = 0.0;
  for (int k = 1; k <= c->nz - 1; ++k)
    for (int j = 1; j <= c->ny - 1; ++j)
      for (int i = 1; i <= c->nx - 1; ++i) {
        long id = IDX(c, i, j, k);
        if (c->iblank[id] || c->ghost[id]) continue;
        double bmx = c->dxcinv[i] * c->dxinv[i], bpx = c->dxcinv[i + 1] * c->dxinv[i];
        double bmy = c->dycinv[j] * c->dyinv[j], bpy = c->dycinv[j + 1] * c->dyinv[j];
        double bmz = c->dzcinv[k] * c->dzinv[k], bpz = c->dzcinv[k + 1] * c->dzinv[k];
        double bc = -(bmx + bpx) + -(bmy + bpy) + -(bmz + bpz);
        double res = r[id] - var[id] * bc - var[id - 1] * bmx - var[id + 1] * bpx -
                     var[id - c->NX] * bmy - var[id + c->NX] * bpy -
                     var[id - c->NX * c->NY] * bmz - var[id + c->NX * c->NY] * bpz;
        res2 += res * res;
        f2 += r[id] * r[id];
      }
  return f2 > 0.0 ? sqrt(res2 / f2) : sqrt(res2);
}

/* GCM_GHOSTCELL_UPDATE.F90:361-739 (mix_GC_form == 0 and 1) */
int or_ghostcell_pressure(or_case *c, double *pres, const double *r,
                          const double *p_old, const double *dpdn_g,
                          const double *dpdn_d, const or_params *prm,
                          int *iterations) {
  int it = 0;
  double resMax = 1.0e10;
  while (it < prm->itermax_gc && resMax > prm->restol_gcp) {
    resMax = 0.0;
    for (int n = 0; n < c->nDead; ++n) {
      int iG = c->dijk[3 * n], jG = c->dijk[3 * n + 1], kG = c->dijk[3 * n + 2];
      if (jG < 1 || jG > c->ny - 1 || kG < 1 || kG > c->nz - 1) continue;
      if (c->dcell[3 * n] < 0) continue;
      long idG = IDX(c, iG, jG, kG);
      double pPrev = pres[idG];
      double pIP = 0.0;
      double dpdn = (prm->is_PBC_homogeneous || !dpdn_d) ? 0.0 : dpdn_d[n];
      double xIP = c->dip[3 * n], yIP = c->dip[3 * n + 1], zIP = c->dip[3 * n + 2];
      double pinv = 0.0, dint = 0.0;
      int sumk = 0;
      for (int q = 0; q < 8; ++q) {
        int ii = c->dcell[3 * n] + incI[q], jj = c->dcell[3 * n + 1] + incJ[q], kk = c->dcell[3 * n + 2] + incK[q];
        if (ii == iG && jj == jG && kk == kG) continue;
        double dist = (c->xc[ii] - xIP) * (c->xc[ii] - xIP) + (c->yc[jj] - yIP) * (c->yc[jj] - yIP) +
                      (c->zc[kk] - zIP) * (c->zc[kk] - zIP);
        long id = IDX(c, ii, jj, kk);
        if (c->iblank[id] == 0 || c->dead[id] == -1) {
          sumk++;
          dint = dint + (1.0 / dist);
          pinv = pinv + (1.0 / dist) * (p_old ? p_old[id] : 0.0);
        }
      }
      int fallback = 0;
      for (int q = 0; q < 8; ++q) {
        int ii = c->dcell[3 * n] + incI[q], jj = c->dcell[3 * n + 1] + incJ[q], kk = c->dcell[3 * n + 2] + incK[q];
        long id = IDX(c, ii, jj, kk);
        if (c->iblank[id] == 1 && c->dead[id] == 0) {
          if (dint < 0.000001 || sumk == 1) {
            pIP = 0.0;
          } else {
            pIP = pinv / dint;
            fallback = 1;
            break;
          }
        }
      }
      if (!fallback) {
        for (int q = 0; q < 8; ++q) {
          int ii = c->dcell[3 * n] + incI[q], jj = c->dcell[3 * n + 1] + incJ[q], kk = c->dcell[3 * n + 2] + incK[q];
          if (ii == iG && jj == jG && kk == kG) pIP = pIP + c->dcoefN[8 * n + q] * dpdn;
          else pIP = pIP + c->dcoefN[8 * n + q] * pres[IDX(c, ii, jj, kk)];
        }
      }
      pres[idG] = pIP + dpdn * c->dprobe[n];
      double rp = fabs(pres[idG] - pPrev);
      if (rp > resMax) resMax = rp;
    }
    for (int n = 0; n < c->nGhost; ++n) {
      int iG = c->gijk[3 * n], jG = c->gijk[3 * n + 1], kG = c->gijk[3 * n + 2];
      if (c->gcell[3 * n] < 0) continue;
      long idG = IDX(c, iG, jG, kG);
      double pPrev = pres[idG];
      double pG = 0.0;
      double dpdn = (prm->is_PBC_homogeneous || !dpdn_g) ? 0.0 : dpdn_g[n];
      for (int q = 0; q < 8; ++q) {
        int ii = c->gcell[3 * n] + incI[q], jj = c->gcell[3 * n + 1] + incJ[q], kk = c->gcell[3 * n + 2] + incK[q];
        if (ii == iG && jj == jG && kk == kG) pG = pG + c->gcoefN[8 * n + q] * dpdn;
        else pG = pG + c->gcoefN[8 * n + q] * pres[IDX(c, ii, jj, kk)];
      }
      if (prm->mix_GC_form == 1) {
        const long NX = c->NX, NXY = c->NX * c->NY;
        double dW = (pres[idG] - pres[idG - 1]) * c->dxcinv[iG];
        double dE = (pres[idG + 1] - pres[idG]) * c->dxcinv[iG + 1];
        double dS = (pres[idG] - pres[idG - NX]) * c->dycinv[jG];
        double dN = (pres[idG + NX] - pres[idG]) * c->dycinv[jG + 1];
        double dB = (pres[idG] - pres[idG - NXY]) * c->dzcinv[kG];
        double dF = (pres[idG + NXY] - pres[idG]) * c->dzcinv[kG + 1];
        double flag = c->galpha[n];
        double coeffG = -(c->dxcinv[iG] + c->dxcinv[iG + 1]) * c->dxinv[iG] -
                        (c->dycinv[jG] + c->dycinv[jG + 1]) * c->dyinv[jG] -
                        (c->dzcinv[kG] + c->dzcinv[kG + 1]) * c->dzinv[kG];
        double rp = (dE - dW) * c->dxinv[iG] + (dN - dS) * c->dyinv[jG] + (dF - dB) * c->dzinv[kG] - r[idG];
        double pG2 = pres[idG] + rp / (-coeffG);
        pres[idG] = (1.0 - flag) * pG + flag * pG2;
      } else {
        pres[idG] = pG;
      }
      double rp = fabs(pres[idG] - pPrev);
      if (rp > resMax) resMax = rp;
    }
    it++;
  }
  if (iterations) *iterations = it;
  return (it == prm->itermax_gc && resMax > prm->restol_gcp) ? OR_NOT_CONVERGED : OR_OK;
}

/* GCM_GHOSTCELL_UPDATE.F90:865-1003 (mix_GC_form == 0 branch) */
static void enforce_p_compatibility(or_case *c, const double *pres, const or_params *prm) {
  for (int f = 0; f < 6; ++f)
    if (prm->pbc[f] == OR_PBC_DIRICHLET) return;
  int any = 0;
  for (int f = 0; f < 6; ++f) any |= prm->vel_zero_gradient[f];
  if (!any) return; /* no face receives the correction */
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  double flux = 0.0;
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        long id = IDX(c, i, j, k);
        const long NX = c->NX, NXY = c->NX * c->NY;
        double pxw = (pres[id] - pres[id - 1]) * c->dxcinv[i];
        double pxe = (pres[id + 1] - pres[id]) * c->dxcinv[i + 1];
        double pys = (pres[id] - pres[id - NX]) * c->dycinv[j];
        double pyn = (pres[id + NX] - pres[id]) * c->dycinv[j + 1];
        double pzb = (pres[id] - pres[id - NXY]) * c->dzcinv[k];
        double pzf = (pres[id + NXY] - pres[id]) * c->dzcinv[k + 1];
        double flag = (1.0 - (double)c->iblank[id]) * (1.0 - (double)c->ghost[id]);
        flux = flux + flag * ((-pxw + pxe) * c->dy[j] * c->dz[k] + (-pys + pyn) * c->dx[i] * c->dz[k] +
                              (-pzb + pzf) * c->dx[i] * c->dy[j]);
      }
  /* outflow area, CORE_SET_OUTER_BC.F90:585-643 */
  double aL = 0, aR = 0, aB = 0, aT = 0, aK = 0, aF = 0, area = 0.0;
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j) {
      aL = aL + c->dy[j] * c->dz[k] * (1.0 - c->iblank[IDX(c, 1, j, k)]);
      aR = aR + c->dy[j] * c->dz[k] * (1.0 - c->iblank[IDX(c, nx - 1, j, k)]);
    }
  for (int k = 1; k <= nz - 1; ++k)
    for (int i = 1; i <= nx - 1; ++i) {
      aB = aB + c->dx[i] * c->dz[k] * (1.0 - c->iblank[IDX(c, i, 1, k)]);
      aT = aT + c->dx[i] * c->dz[k] * (1.0 - c->iblank[IDX(c, i, ny - 1, k)]);
    }
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      aK = aK + c->dx[i] * c->dy[j] * (1.0 - c->iblank[IDX(c, i, j, 1)]);
      aF = aF + c->dx[i] * c->dy[j] * (1.0 - c->iblank[IDX(c, i, j, nz - 1)]);
    }
  if (prm->vel_zero_gradient[0]) area += aL;
  if (prm->vel_zero_gradient[1]) area += aR;
  if (prm->vel_zero_gradient[2]) area += aB;
  if (prm->vel_zero_gradient[3]) area += aT;
  if (prm->vel_zero_gradient[4]) area += aK;
  if (prm->vel_zero_gradient[5]) area += aF;
  double corr = -flux / area;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j) {
      if (prm->vel_zero_gradient[0]) c->pgradx1[j + c->NY * k] -= corr;
      if (prm->vel_zero_gradient[1]) c->pgradx2[j + c->NY * k] += corr;
    }
  for (int k = 0; k <= nz; ++k)
    for (int i = 0; i <= nx; ++i) {
      if (prm->vel_zero_gradient[2]) c->pgrady1[i + c->NX * k] -= corr;
      if (prm->vel_zero_gradient[3]) c->pgrady2[i + c->NX * k] += corr;
    }
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      if (prm->vel_zero_gradient[4]) c->pgradz1[i + c->NX * j] -= corr;
      if (prm->vel_zero_gradient[5]) c->pgradz2[i + c->NX * j] += corr;
    }
}

/* exported for the tests: one GCM_enforce_p_compatibility step on p, and
 * access to the outer-face pressure gradients it updates (face 0..5 =
 * x1, x2, y1, y2, z1, z2; x faces (0:ny+1, 0:nz+1), y faces (0:nx+1,
 * 0:nz+1), z faces (0:nx+1, 0:ny+1)) */
int or_enforce_p_compatibility(or_case *c, const double *p, const or_params *prm) {
  enforce_p_compatibility(c, p, prm);
  return OR_OK;
}
static double *pgrad_face(or_case *c, int face, long *n) {
  double *a[6] = {c->pgradx1, c->pgradx2, c->pgrady1, c->pgrady2, c->pgradz1, c->pgradz2};
  const long ext[3] = {(long)c->NY * c->NZ, (long)c->NX * c->NZ, (long)c->NX * c->NY};
  if (face < 0 || face > 5) return NULL;
  *n = ext[face / 2];
  return a[face];
}
int or_get_pgrad(or_case *c, int face, double *out) {
  long n = 0;
  double *a = pgrad_face(c, face, &n);
  if (!a) return OR_BAD_INPUT;
  memcpy(out, a, sizeof(double) * (size_t)n);
  return OR_OK;
}
int or_set_pgrad(or_case *c, int face, const double *in) {
  long n = 0;
  double *a = pgrad_face(c, face, &n);
  if (!a) return OR_BAD_INPUT;
  memcpy(a, in, sizeof(double) * (size_t)n);
  return OR_OK;
}

/* ------------------------------------------------------------------
 * The steps either side of the pressure solve (fractional-step
 * projection), restated for nProcs = 1.  Face-velocity boundary arrays as
 * the reference keeps them: bcxu(0:1, 0:ny+1, 0:nz+1), bcyv(0:nx+1, 0:1,
 * 0:nz+1), bczw(0:nx+1, 0:ny+1, 0:1), column-major.  vzg: the faces whose
 * velocity is ZERO_GRADIENT (x1 x2 y1 y2 z1 z2).
 * ------------------------------------------------------------------ */
#define BCXU(s, j, k) bcxu[(long)(s) + 2 * ((long)(j) + c->NY * (long)(k))]
#define BCYV(i, s, k) bcyv[(long)(i) + c->NX * ((long)(s) + 2 * (long)(k))]
#define BCZW(i, j, s) bczw[(long)(i) + c->NX * ((long)(j) + c->NY * (long)(s))]
/* CORE_GRID.F90:194-202: face interpolation factor of node i */
static double fint(const double *x, const double *xc, int i) { return (x[i] - xc[i - 1]) / (xc[i] - xc[i - 1]); }

/* CORE_FRAC_STEP_ROUTINES.F90:1-130 face_vel */
int or_face_vel(or_case *c, const double *u, const double *v, const double *w, const double *bcxu,
                const double *bcyv, const double *bczw, double *fu, double *fv, double *fw) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const double f = fint(c->x, c->xc, i);
        fu[IDX(c, i, j, k)] = f * u[IDX(c, i, j, k)] + (1.0 - f) * u[IDX(c, i - 1, j, k)];
      }
  for (int j = 2; j <= ny - 1; ++j)
    for (int k = 1; k <= nz - 1; ++k)
      for (int i = 1; i <= nx - 1; ++i) {
        const double f = fint(c->y, c->yc, j);
        fv[IDX(c, i, j, k)] = f * v[IDX(c, i, j, k)] + (1.0 - f) * v[IDX(c, i, j - 1, k)];
      }
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        const double f = fint(c->z, c->zc, k);
        fw[IDX(c, i, j, k)] = f * w[IDX(c, i, j, k)] + (1.0 - f) * w[IDX(c, i, j, k - 1)];
      }
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j) {
      fu[IDX(c, 1, j, k)] = BCXU(0, j, k);
      fu[IDX(c, nx, j, k)] = BCXU(1, j, k);
    }
  for (int k = 1; k <= nz - 1; ++k)
    for (int i = 1; i <= nx - 1; ++i) {
      fv[IDX(c, i, 1, k)] = BCYV(i, 0, k);
      fv[IDX(c, i, ny, k)] = BCYV(i, 1, k);
    }
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      fw[IDX(c, i, j, 1)] = BCZW(i, j, 0);
      fw[IDX(c, i, j, nz)] = BCZW(i, j, 1);
    }
  return OR_OK;
}

/* CORE_SET_OUTER_BC.F90:515-735 enforce_global_mass_consv (mix_GC_form =
 * 0) then CORE_POISSON.F90:9-79 rhs_poisson: div = (du/dx + dv/dy +
 * dw/dz) / dt on fluid non-ghost cells; *sumd = the mass flux (dt removed),
 * *resdiv = max |div| dt */
int or_enforce_global_mass_consv(or_case *c, double *fu, double *fv, double *fw, double *bcxu, double *bcyv,
                                 double *bczw, const int *vzg) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  int any = 0;
  for (int f = 0; f < 6; ++f) any |= vzg[f];
  if (any) {
    double massflux = 0.0;
    for (int k = 1; k <= nz - 1; ++k)
      for (int j = 1; j <= ny - 1; ++j)
        for (int i = 1; i <= nx - 1; ++i) {
          const long id = IDX(c, i, j, k);
          const double flag = (1.0 - (double)c->iblank[id]) * (1.0 - (double)c->ghost[id]);
          massflux = massflux + flag * ((-fu[id] + fu[IDX(c, i + 1, j, k)]) * c->dy[j] * c->dz[k] +
                                        (-fv[id] + fv[IDX(c, i, j + 1, k)]) * c->dx[i] * c->dz[k] +
                                        (-fw[id] + fw[IDX(c, i, j, k + 1)]) * c->dx[i] * c->dy[j]);
        }
    double aL = 0, aR = 0, aB = 0, aT = 0, aK = 0, aF = 0, area = 0.0;
    for (int k = 1; k <= nz - 1; ++k)
      for (int j = 1; j <= ny - 1; ++j) {
        aL = aL + c->dy[j] * c->dz[k] * (1.0 - c->iblank[IDX(c, 1, j, k)]);
        aR = aR + c->dy[j] * c->dz[k] * (1.0 - c->iblank[IDX(c, nx - 1, j, k)]);
      }
    for (int k = 1; k <= nz - 1; ++k)
      for (int i = 1; i <= nx - 1; ++i) {
        aB = aB + c->dx[i] * c->dz[k] * (1.0 - c->iblank[IDX(c, i, 1, k)]);
        aT = aT + c->dx[i] * c->dz[k] * (1.0 - c->iblank[IDX(c, i, ny - 1, k)]);
      }
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        aK = aK + c->dx[i] * c->dy[j] * (1.0 - c->iblank[IDX(c, i, j, 1)]);
        aF = aF + c->dx[i] * c->dy[j] * (1.0 - c->iblank[IDX(c, i, j, nz - 1)]);
      }
    if (vzg[0]) area += aL;
    if (vzg[1]) area += aR;
    if (vzg[2]) area += aB;
    if (vzg[3]) area += aT;
    if (vzg[4]) area += aK;
    if (vzg[5]) area += aF;
    const double cv = -massflux / area;
    for (int k = 0; k <= nz; ++k)
      for (int j = 0; j <= ny; ++j) {
        if (vzg[0]) BCXU(0, j, k) = BCXU(0, j, k) - cv;
        if (vzg[1]) BCXU(1, j, k) = BCXU(1, j, k) + cv;
      }
    for (int k = 0; k <= nz; ++k)
      for (int i = 0; i <= nx; ++i) {
        if (vzg[2]) BCYV(i, 0, k) = BCYV(i, 0, k) - cv;
        if (vzg[3]) BCYV(i, 1, k) = BCYV(i, 1, k) + cv;
      }
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        if (vzg[4]) BCZW(i, j, 0) = BCZW(i, j, 0) - cv;
        if (vzg[5]) BCZW(i, j, 1) = BCZW(i, j, 1) + cv;
      }
    for (int k = 1; k <= nz - 1; ++k)
      for (int j = 1; j <= ny - 1; ++j) {
        if (vzg[0]) fu[IDX(c, 1, j, k)] = fu[IDX(c, 1, j, k)] - cv;
        if (vzg[1]) fu[IDX(c, nx, j, k)] = fu[IDX(c, nx, j, k)] + cv;
      }
    for (int k = 1; k <= nz - 1; ++k)
      for (int i = 1; i <= nx - 1; ++i) {
        if (vzg[2]) fv[IDX(c, i, 1, k)] = fv[IDX(c, i, 1, k)] - cv;
        if (vzg[3]) fv[IDX(c, i, ny, k)] = fv[IDX(c, i, ny, k)] + cv;
      }
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        if (vzg[4]) fw[IDX(c, i, j, 1)] = fw[IDX(c, i, j, 1)] - cv;
        if (vzg[5]) fw[IDX(c, i, j, nz)] = fw[IDX(c, i, j, nz)] + cv;
      }
  }
  return OR_OK;
}

int or_rhs_poisson(or_case *c, double *fu, double *fv, double *fw, double *bcxu, double *bcyv, double *bczw,
                   const int *vzg, double dt, double *div, double *sumd, double *resdiv) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  or_enforce_global_mass_consv(c, fu, fv, fw, bcxu, bcyv, bczw, vzg);
  const double dtinv = 1.0 / dt;
  double sd = 0.0, rd = 0.0;
  memset(div, 0, sizeof(double) * (size_t)c->ntot);
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        const long id = IDX(c, i, j, k);
        const double flag = (1.0 - (double)c->iblank[id]) * (1.0 - (double)c->ghost[id]);
        double d = dtinv * ((fu[IDX(c, i + 1, j, k)] - fu[id]) * c->dxinv[i] +
                            (fv[IDX(c, i, j + 1, k)] - fv[id]) * c->dyinv[j] +
                            (fw[IDX(c, i, j, k + 1)] - fw[id]) * c->dzinv[k]);
        d = d * flag;
        div[id] = d;
        sd = sd + d * c->dx[i] * c->dy[j] * c->dz[k];
        const double a = fabs(d / dtinv);
        if (a > rd) rd = a;
      }
  *sumd = sd / dtinv;
  *resdiv = rd;
  return OR_OK;
}

/* CORE_FRAC_STEP_ROUTINES.F90:132-190 correct_vel (u -= dt grad p' on
 * non-iblank cells) and :270-320 calc_pres_grad (grad p' on non-iblank
 * cells); either output set may be NULL */
int or_correct_vel(or_case *c, const double *pp, double dt, double *u, double *v, double *w, double *dpdx,
                   double *dpdy, double *dpdz) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        const long id = IDX(c, i, j, k);
        const double fx1 = fint(c->x, c->xc, i + 1), fx0 = fint(c->x, c->xc, i);
        const double fy1 = fint(c->y, c->yc, j + 1), fy0 = fint(c->y, c->yc, j);
        const double fz1 = fint(c->z, c->zc, k + 1), fz0 = fint(c->z, c->zc, k);
        const double pe = fx1 * pp[IDX(c, i + 1, j, k)] + (1.0 - fx1) * pp[id];
        const double pw = fx0 * pp[id] + (1.0 - fx0) * pp[IDX(c, i - 1, j, k)];
        const double pn = fy1 * pp[IDX(c, i, j + 1, k)] + (1.0 - fy1) * pp[id];
        const double ps = fy0 * pp[id] + (1.0 - fy0) * pp[IDX(c, i, j - 1, k)];
        const double pf = fz1 * pp[IDX(c, i, j, k + 1)] + (1.0 - fz1) * pp[id];
        const double pb = fz0 * pp[id] + (1.0 - fz0) * pp[IDX(c, i, j, k - 1)];
        const double pgx = (pe - pw) * c->dxinv[i], pgy = (pn - ps) * c->dyinv[j], pgz = (pf - pb) * c->dzinv[k];
        const double flag = 1.0 - (double)c->iblank[id];
        if (u) {
          u[id] = u[id] - dt * pgx * flag;
          v[id] = v[id] - dt * pgy * flag;
          w[id] = w[id] - dt * pgz * flag;
        }
        if (dpdx) {
          dpdx[id] = pgx * flag;
          dpdy[id] = pgy * flag;
          dpdz[id] = pgz * flag;
        }
      }
  return OR_OK;
}
#undef BCXU
#undef BCYV
#undef BCZW

/* CORE_FRAC_STEP_ROUTINES.F90:212-299 update_pressure for one rank
 * (jProc = kProc = 0 = nProcY-1 = nProcZ-1): p' = 0 on the solid cells
 * that are not dead-marked -1 (k, j from 0 to n+1, i from 0 to nx), p' = 0
 * on the domain edge lines of its twelve assignments, then p = p'.  The
 * assignment !07 names plane k = zc_start-2 = -1, outside the array
 * (lower bound 0); its plane 0 part is kept, the rest is not restated. */
int or_update_pressure(or_case *c, double *pp, double *p) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 0; i <= nx; ++i) {
        const long id = IDX(c, i, j, k);
        if (c->iblank[id] == 0 || c->dead[id] == -1) continue;
        pp[id] = 0.0;
      }
  /* !01-!04: i = 0..nx on the lines j = 0 and j = ny, planes 0 and nz..nz+1 */
  for (int jj = 0; jj < 2; ++jj) {
    const int j = jj ? ny : 0;
    for (int i = 0; i <= nx; ++i) {
      pp[IDX(c, i, j, 0)] = 0.0;
      pp[IDX(c, i, j, nz)] = 0.0;
      pp[IDX(c, i, j, nz + 1)] = 0.0;
    }
  }
  /* !05-!08: i = 0 and nx, j = 0..ny+1, planes 0 and nz..nz+1 */
  for (int ii = 0; ii < 2; ++ii) {
    const int i = ii ? nx : 0;
    for (int j = 0; j <= ny + 1; ++j) {
      pp[IDX(c, i, j, 0)] = 0.0;
      pp[IDX(c, i, j, nz)] = 0.0;
      pp[IDX(c, i, j, nz + 1)] = 0.0;
    }
  }
  /* !09-!12: the four lines along k at (i, j) in {0, nx} x {0, ny} */
  for (int k = 0; k <= nz + 1; ++k) {
    pp[IDX(c, 0, 0, k)] = 0.0;
    pp[IDX(c, nx, 0, k)] = 0.0;
    pp[IDX(c, 0, ny, k)] = 0.0;
    pp[IDX(c, nx, ny, k)] = 0.0;
  }
  if (p) memcpy(p, pp, sizeof(double) * (size_t)c->NX * c->NY * c->NZ);
  return OR_OK;
}

/* ------------------------------------------ body-intercept values
 * GCM_BODYINTERCEPT_VALUES.F90:22-178 GCM_SetBodyInterceptValues with
 * :198-388 GCM_calc_BIVelocity_Unstruc: per ghost and dead row the marker
 * velocities of the closest element interpolated linearly to the body
 * intercept (the 4x4 system of the element's three vertices and its normal,
 * inverted with LAPACK DGETRF/DGETRI semantics), this step's and the
 * previous step's, and dp/dn = -(du/dt . n) at the intercept (0 on the
 * first step). */
static void bi_velocity(const or_case *c, int ib, int elem, double xB, double yB, double zB, double *uvw,
                        double *uvw_old) {
  const or_body *B = &c->body[ib];
  const int n1 = B->tri[3 * elem], n2 = B->tri[3 * elem + 1], n3 = B->tri[3 * elem + 2];
  double van[16], inv[16];
  const int nd[3] = {n1, n2, n3};
  for (int r = 0; r < 3; ++r) {
    van[r + 4 * 0] = B->xv[nd[r]]; van[r + 4 * 1] = B->yv[nd[r]]; van[r + 4 * 2] = B->zv[nd[r]];
    van[r + 4 * 3] = 1.0;
  }
  van[3 + 4 * 0] = B->enx[elem]; van[3 + 4 * 1] = B->eny[elem]; van[3 + 4 * 2] = B->enz[elem];
  van[3 + 4 * 3] = 0.0;
  int info;
  invert_n(4, van, inv, &info);
  const double *src[6] = {B->mu, B->mv, B->mw, B->muo, B->mvo, B->mwo};
  for (int q = 0; q < 6; ++q) {
    double rhs[4] = {0.0, 0.0, 0.0, 0.0};
    if (src[q]) { rhs[0] = src[q][n1]; rhs[1] = src[q][n2]; rhs[2] = src[q][n3]; }
    double cX = 0.0, cY = 0.0, cZ = 0.0, cC = 0.0;
    for (int i = 0; i < 4; ++i) {
      cX = cX + inv[0 + 4 * i] * rhs[i];
      cY = cY + inv[1 + 4 * i] * rhs[i];
      cZ = cZ + inv[2 + 4 * i] * rhs[i];
      cC = cC + inv[3 + 4 * i] * rhs[i];
    }
    const double v = cX * xB + cY * yB + cZ * zB + cC;
    if (q < 3) uvw[q] = v; else uvw_old[q - 3] = v;
  }
}

int or_body_intercept_values(or_case *c, int ntime, double dt, double *ubi_g, double *ubi_d, double *dpdn_g,
                             double *dpdn_d) {
  for (int pass = 0; pass < 2; ++pass) {
    const int nr = pass == 0 ? c->nGhost : c->nDead;
    const int32_t *ijk = pass == 0 ? c->gijk : c->dijk, *ce = pass == 0 ? c->gclosest : c->dclosest;
    const double *bi = pass == 0 ? c->gbi : c->dbi, *nrm = pass == 0 ? c->gnrm : c->dnrm;
    double *ub = pass == 0 ? ubi_g : ubi_d, *dp = pass == 0 ? dpdn_g : dpdn_d;
    for (int n = 0; n < nr; ++n) {
      int ib = c->bodyNum[IDX(c, ijk[3 * n], ijk[3 * n + 1], ijk[3 * n + 2])] - 1;
      double u[3] = {0.0, 0.0, 0.0}, uo[3] = {0.0, 0.0, 0.0};
      if (ib >= 0 && ib < c->nbody && ce[n] >= 0)
        bi_velocity(c, ib, ce[n], bi[3 * n], bi[3 * n + 1], bi[3 * n + 2], u, uo);
      if (ub) { ub[3 * n] = u[0]; ub[3 * n + 1] = u[1]; ub[3 * n + 2] = u[2]; }
      if (dp) {
        double d = 0.0;
        if (ntime > 1) {
          d = (u[0] - uo[0]) / dt * nrm[3 * n] + (u[1] - uo[1]) / dt * nrm[3 * n + 1] +
              (u[2] - uo[2]) / dt * nrm[3 * n + 2];
          d = -d;
        }
        dp[n] = d;
      }
    }
  }
  return OR_OK;
}

/* GCM_GHOSTCELL_UPDATE.F90:1-359 GCM_ghostcell_velocity for iOpt = 2 and
 * mix_GC_form = 0, one rank: Gauss-Seidel over the dead rows, then the
 * ghost rows, until the largest |du|+|dv|+|dw| of a sweep is at most
 * restol_gcv or itermax_gc sweeps ran.  A dead row takes the intercept
 * velocity through the Dirichlet weights (or the inverse-distance average
 * of its fluid corners when a corner is pure solid) and is set to
 * u_BI w_BI - u_IP w_IP with w_BI = pLD/(pLD-1), w_IP = 1/(pLD-1), pLD =
 * probeLengthNormalizedD; a ghost row is the Dirichlet interpolation with
 * the intercept velocity in its own slot. */
int or_ghostcell_velocity(or_case *c, double *u, double *v, double *w, const double *ubi_g, const double *ubi_d,
                          double pld, int itermax_gc, double restol_gcv, int *iterations) {
  const double bw = pld / (pld - 1.0), iw = 1.0 / (pld - 1.0);
  double *fld[3] = {u, v, w};
  int it = 0;
  double resMax = 1.0e10;
  while (it < itermax_gc && resMax > restol_gcv) {
    resMax = 0.0;
    for (int n = 0; n < c->nDead; ++n) {
      const int i = c->dijk[3 * n], j = c->dijk[3 * n + 1], k = c->dijk[3 * n + 2];
      if (j < 1 || j > c->ny - 1 || k < 1 || k > c->nz - 1) continue;
      if (c->dcell[3 * n] < 0) continue;
      const long id = IDX(c, i, j, k);
      const double xIP = c->dip[3 * n], yIP = c->dip[3 * n + 1], zIP = c->dip[3 * n + 2];
      double prev[3], ip[3] = {0.0, 0.0, 0.0}, inv[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < 3; ++q) prev[q] = fld[q][id];
      double dint = 0.0;
      int sumk = 0;
      for (int r = 0; r < 8; ++r) {
        const int ii = c->dcell[3 * n] + incI[r], jj = c->dcell[3 * n + 1] + incJ[r], kk = c->dcell[3 * n + 2] + incK[r];
        if (ii == i && jj == j && kk == k) continue;
        const double dist = (c->xc[ii] - xIP) * (c->xc[ii] - xIP) + (c->yc[jj] - yIP) * (c->yc[jj] - yIP) +
                            (c->zc[kk] - zIP) * (c->zc[kk] - zIP);
        const long q2 = IDX(c, ii, jj, kk);
        if (c->iblank[q2] == 0 || c->dead[q2] == -1) {
          sumk++;
          dint = dint + (1.0 / dist);
          for (int q = 0; q < 3; ++q) inv[q] = inv[q] + (1.0 / dist) * fld[q][q2];
        }
      }
      int fallback = 0;
      for (int r = 0; r < 8 && !fallback; ++r) {
        const int ii = c->dcell[3 * n] + incI[r], jj = c->dcell[3 * n + 1] + incJ[r], kk = c->dcell[3 * n + 2] + incK[r];
        const long q2 = IDX(c, ii, jj, kk);
        if (c->iblank[q2] == 1 && c->dead[q2] == 0) {
          if (dint < 0.000001 || sumk == 1) {
            ip[0] = ip[1] = ip[2] = 0.0;
          } else {
            for (int q = 0; q < 3; ++q) ip[q] = inv[q] / dint;
            fallback = 1;
          }
        }
      }
      if (!fallback)
        for (int r = 0; r < 8; ++r) {
          const int ii = c->dcell[3 * n] + incI[r], jj = c->dcell[3 * n + 1] + incJ[r], kk = c->dcell[3 * n + 2] + incK[r];
          for (int q = 0; q < 3; ++q) {
            if (ii != i || jj != j || kk != k) ip[q] = ip[q] + c->dcoefD[8 * n + r] * fld[q][IDX(c, ii, jj, kk)];
            else ip[q] = ip[q] + c->dcoefD[8 * n + r] * ubi_d[3 * n + q];
          }
        }
      for (int q = 0; q < 3; ++q) fld[q][id] = ubi_d[3 * n + q] * bw - ip[q] * iw;
      const double rv = fabs(u[id] - prev[0]) + fabs(v[id] - prev[1]) + fabs(w[id] - prev[2]);
      if (rv > resMax) resMax = rv;
    }
    for (int n = 0; n < c->nGhost; ++n) {
      const int i = c->gijk[3 * n], j = c->gijk[3 * n + 1], k = c->gijk[3 * n + 2];
      if (c->gcell[3 * n] < 0) continue;
      const long id = IDX(c, i, j, k);
      double prev[3], g[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < 3; ++q) prev[q] = fld[q][id];
      for (int r = 0; r < 8; ++r) {
        const int ii = c->gcell[3 * n] + incI[r], jj = c->gcell[3 * n + 1] + incJ[r], kk = c->gcell[3 * n + 2] + incK[r];
        for (int q = 0; q < 3; ++q) {
          if (ii != i || jj != j || kk != k) g[q] = g[q] + c->gcoefD[8 * n + r] * fld[q][IDX(c, ii, jj, kk)];
          else g[q] = g[q] + c->gcoefD[8 * n + r] * ubi_g[3 * n + q];
        }
      }
      const double flag = c->galpha[n];
      for (int q = 0; q < 3; ++q) fld[q][id] = (1.0 - flag) * g[q] + flag * g[q];
      const double rv = fabs(u[id] - prev[0]) + fabs(v[id] - prev[1]) + fabs(w[id] - prev[2]);
      if (rv > resMax) resMax = rv;
    }
    it++;
  }
  if (iterations) *iterations = it;
  return (it == itermax_gc && resMax > restol_gcv) ? OR_NOT_CONVERGED : OR_OK;
}

/* ------------------------------------------ outer velocity boundaries
 * CORE_SET_OUTER_BC.F90:18-509 set_outer_velocity_bc and :739-823
 * set_outer_ghost_velocity, one rank.  bc holds bcxu, bcxv, bcxw
 * (0:1,0:ny+1,0:nz+1), bcyu, bcyv, bcyw (0:nx+1,0:1,0:nz+1), bczu, bczv, bczw
 * (0:nx+1,0:ny+1,0:1).  The user-specified case of the y and z faces writes
 * the x-face arrays at (1, j, k), as the reference does. */
#define BX(a, s, j, k) bc[a][(long)(s) + 2 * ((long)(j) + c->NY * (long)(k))]
#define BY(a, i, s, k) bc[3 + (a)][(long)(i) + c->NX * ((long)(s) + 2 * (long)(k))]
#define BZ(a, i, j, s) bc[6 + (a)][(long)(i) + c->NX * ((long)(j) + c->NY * (long)(s))]
int or_set_outer_velocity_bc(or_case *c, const double *u, const double *v, const double *w, double *const *bc,
                             const or_velocity_bc *p) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const double pi = 4.0 * atan(1.0), t = p->time;
  const double *f3[3] = {u, v, w};
  for (int f = 0; f < 6; ++f)
    if (p->type[f] < 1 || p->type[f] > 6) return OR_BAD_INPUT;  /* shear: not implemented (:102-105) */
  /* x faces */
  for (int side = 0; side < 2; ++side) {
    const int i = side == 0 ? 1 : nx - 1, io = side == 0 ? nx - 1 : 1, f = side;
    const double *val = p->val[f], *fr = p->freq[f];
    for (int k = 0; k <= nz + 1; ++k)
      for (int j = 0; j <= ny + 1; ++j)
        switch (p->type[f]) {
          case 1: for (int a = 0; a < 3; ++a) BX(a, side, j, k) = val[a]; break;
          case 2: for (int a = 0; a < 3; ++a) BX(a, side, j, k) = f3[a][IDX(c, i, j, k)]; break;
          case 3:
            BX(0, side, j, k) = side == 0 ? val[0] * t / 30.0 : val[0] * sin(2.0 * pi * fr[0] * t);
            BX(1, side, j, k) = val[1] * sin(2.0 * pi * fr[1] * t);
            BX(2, side, j, k) = val[2] * sin(2.0 * pi * fr[2] * t);
            break;
          case 4:
            BX(0, side, j, k) = 0.0;
            BX(1, side, j, k) = v[IDX(c, i, j, k)];
            BX(2, side, j, k) = w[IDX(c, i, j, k)];
            break;
          case 5:
            for (int a = 0; a < 3; ++a) BX(a, side, j, k) = 0.5 * (f3[a][IDX(c, i, j, k)] + f3[a][IDX(c, io, j, k)]);
            break;
          case 6: {
            const double e = p->yout - p->yOrigin;
            BX(0, side, j, k) = val[0] * 6.0 * (c->y[j] - p->yOrigin) * (p->yout - c->y[j]) / (e * e);
            if (side == 1) { BX(1, side, j, k) = val[1]; BX(2, side, j, k) = val[2]; }
            break;
          }
        }
  }
  /* y faces */
  for (int side = 0; side < 2; ++side) {
    const int j = side == 0 ? 1 : ny - 1, jo = side == 0 ? ny - 1 : 1, f = 2 + side;
    const double *val = p->val[f], *fr = p->freq[f];
    for (int k = 0; k <= nz + 1; ++k)
      for (int i = 0; i <= nx; ++i)
        switch (p->type[f]) {
          case 1: for (int a = 0; a < 3; ++a) BY(a, i, side, k) = val[a]; break;
          case 2: for (int a = 0; a < 3; ++a) BY(a, i, side, k) = f3[a][IDX(c, i, j, k)]; break;
          case 3: for (int a = 0; a < 3; ++a) BY(a, i, side, k) = val[a] * sin(2.0 * pi * fr[a] * t); break;
          case 4:
            BY(0, i, side, k) = u[IDX(c, i, j, k)];
            BY(1, i, side, k) = 0.0;
            BY(2, i, side, k) = w[IDX(c, i, j, k)];
            break;
          case 5:
            for (int a = 0; a < 3; ++a) BY(a, i, side, k) = 0.5 * (f3[a][IDX(c, i, j, k)] + f3[a][IDX(c, i, jo, k)]);
            break;
          case 6: {
            const double e = p->zout - p->zOrigin;
            BX(0, 1, j, k) = val[0];
            BX(1, 1, j, k) = val[1] * 6.0 * (c->z[k] - p->zOrigin) * (p->zout - c->z[k]) / (e * e);
            BX(2, 1, j, k) = val[2];
            break;
          }
        }
  }
  /* z faces */
  for (int side = 0; side < 2; ++side) {
    const int k = side == 0 ? 1 : nz - 1, ko = side == 0 ? nz - 1 : 1, f = 4 + side;
    const double *val = p->val[f], *fr = p->freq[f];
    for (int i = 0; i <= nx; ++i)
      for (int j = 0; j <= ny + 1; ++j)
        switch (p->type[f]) {
          case 1: for (int a = 0; a < 3; ++a) BZ(a, i, j, side) = val[a]; break;
          case 2: for (int a = 0; a < 3; ++a) BZ(a, i, j, side) = f3[a][IDX(c, i, j, k)]; break;
          case 3: for (int a = 0; a < 3; ++a) BZ(a, i, j, side) = val[a] * sin(2.0 * pi * fr[a] * t); break;
          case 4:
            BZ(0, i, j, side) = u[IDX(c, i, j, k)];
            BZ(2, i, j, side) = 0.0;
            BZ(1, i, j, side) = v[IDX(c, i, j, k)];
            break;
          case 5:
            for (int a = 0; a < 3; ++a) BZ(a, i, j, side) = 0.5 * (f3[a][IDX(c, i, j, k)] + f3[a][IDX(c, i, j, ko)]);
            break;
          case 6: {
            const double e = p->yout - p->yOrigin;
            BX(0, 1, j, k) = val[0];
            BX(1, 1, j, k) = val[1];
            BX(2, 1, j, k) = val[2] * 6.0 * (c->y[j] - p->yOrigin) * (p->yout - c->y[j]) / (e * e);
            break;
          }
        }
  }
  return OR_OK;
}

int or_set_outer_ghost_velocity(or_case *c, double *u, double *v, double *w, double *const *bc) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  double *f3[3] = {u, v, w};
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j)
      for (int a = 0; a < 3; ++a) {
        f3[a][IDX(c, 0, j, k)] = 2.0 * BX(a, 0, j, k) - f3[a][IDX(c, 1, j, k)];
        f3[a][IDX(c, nx, j, k)] = 2.0 * BX(a, 1, j, k) - f3[a][IDX(c, nx - 1, j, k)];
      }
  for (int k = 0; k <= nz + 1; ++k)
    for (int i = 0; i <= nx; ++i)
      for (int a = 0; a < 3; ++a) {
        f3[a][IDX(c, i, 0, k)] = 2.0 * BY(a, i, 0, k) - f3[a][IDX(c, i, 1, k)];
        f3[a][IDX(c, i, ny, k)] = 2.0 * BY(a, i, 1, k) - f3[a][IDX(c, i, ny - 1, k)];
      }
  for (int i = 0; i <= nx; ++i)
    for (int j = 0; j <= ny + 1; ++j)
      for (int a = 0; a < 3; ++a) {
        f3[a][IDX(c, i, j, 0)] = 2.0 * BZ(a, i, j, 0) - f3[a][IDX(c, i, j, 1)];
        f3[a][IDX(c, i, j, nz)] = 2.0 * BZ(a, i, j, 1) - f3[a][IDX(c, i, j, nz - 1)];
      }
  return OR_OK;
}
#undef BX
#undef BY
#undef BZ

/* ---------------------------------------------- momentum line SOR
 * CORE_SET_SOLVERS.F90:591-677 set_solve_ad (diffusion coefficients with
 * nu = reinv), CORE_SOLVE_AD.F90:162-776 itsolv_ad_x/y/z (one Gauss-Seidel
 * line sweep per direction, lexicographic, with the implicit convection
 * terms: central for 25 <= i <= 375, first-order upwind elsewhere) and
 * :780-964 calc_residual_ad, for one rank. */
typedef struct {
  double amx, apx, acx, amy, apy, acy, amz, apz, acz;
} ad_coef;

static double fsign1(double x) { return copysign(1.0, x); }

/* the coefficients of cell (i,j,k) as each sweep forms them (:215-330) */
static void ad_cell(const or_case *c, const double *ad, const double *fu, const double *fv, const double *fw,
                    double half_dt, int i, int j, int k, ad_coef *q) {
  const int nx = c->nx, ny = c->ny;
  const double *amx_ad = ad, *apx_ad = ad + (nx + 2), *amy_ad = ad + 2 * (nx + 2),
               *apy_ad = ad + 2 * (nx + 2) + (ny + 2), *amz_ad = ad + 2 * (nx + 2) + 2 * (ny + 2),
               *apz_ad = amz_ad + (c->nz + 2);
  const long id = IDX(c, i, j, k);
  const long ip = IDX(c, i + 1, j, k), jp = IDX(c, i, j + 1, k), kp = IDX(c, i, j, k + 1);
  const int central = (i >= 25) && (i <= 375);
  double hyb1, hyb2, tmp1, tmp2;
  q->amx = amx_ad[i]; q->apx = apx_ad[i]; q->acx = -(q->amx + q->apx);
  q->amy = amy_ad[j]; q->apy = apy_ad[j]; q->acy = -(q->amy + q->apy);
  q->amz = amz_ad[k]; q->apz = apz_ad[k]; q->acz = -(q->amz + q->apz);
  /* x */
  hyb1 = 0.5 * (1.0 + fsign1(fu[id])); hyb2 = 0.5 * (1.0 - fsign1(fu[ip]));
  tmp1 = 1.0 - fint(c->x, c->xc, i); tmp2 = fint(c->x, c->xc, i + 1);
  if (central) {
    q->amx = q->amx - half_dt * fu[id] * tmp1 * c->dxinv[i];
    q->apx = q->apx + half_dt * fu[ip] * tmp2 * c->dxinv[i];
  } else {
    q->amx = q->amx - half_dt * hyb1 * fu[id] * c->dxinv[i];
    q->apx = q->apx + half_dt * hyb2 * fu[ip] * c->dxinv[i];
  }
  hyb1 = 0.5 * (1.0 - fsign1(fu[id])); hyb2 = 0.5 * (1.0 + fsign1(fu[ip]));
  tmp1 = fint(c->x, c->xc, i); tmp2 = 1.0 - fint(c->x, c->xc, i + 1);
  if (central) q->acx = q->acx + half_dt * (fu[ip] * tmp2 - fu[id] * tmp1) * c->dxinv[i];
  else q->acx = q->acx + half_dt * (fu[ip] * hyb2 - fu[id] * hyb1) * c->dxinv[i];
  /* y */
  hyb1 = 0.5 * (1.0 + fsign1(fv[id])); hyb2 = 0.5 * (1.0 - fsign1(fv[jp]));
  tmp1 = 1.0 - fint(c->y, c->yc, j); tmp2 = fint(c->y, c->yc, j + 1);
  if (central) {
    q->amy = q->amy - half_dt * fv[id] * tmp1 * c->dyinv[j];
    q->apy = q->apy + half_dt * fv[jp] * tmp2 * c->dyinv[j];
  } else {
    q->amy = q->amy - half_dt * hyb1 * fv[id] * c->dyinv[j];
    q->apy = q->apy + half_dt * hyb2 * fv[jp] * c->dyinv[j];
  }
  hyb1 = 0.5 * (1.0 - fsign1(fv[id])); hyb2 = 0.5 * (1.0 + fsign1(fv[jp]));
  tmp1 = fint(c->y, c->yc, j); tmp2 = 1.0 - fint(c->y, c->yc, j + 1);
  if (central) q->acy = q->acy + half_dt * (fv[jp] * tmp2 - fv[id] * tmp1) * c->dyinv[j];
  else q->acy = q->acy + half_dt * (fv[jp] * hyb2 - fv[id] * hyb1) * c->dyinv[j];
  /* z */
  hyb1 = 0.5 * (1.0 + fsign1(fw[id])); hyb2 = 0.5 * (1.0 - fsign1(fw[kp]));
  tmp1 = 1.0 - fint(c->z, c->zc, k); tmp2 = fint(c->z, c->zc, k + 1);
  if (central) {
    q->amz = q->amz - half_dt * fw[id] * tmp1 * c->dzinv[k];
    q->apz = q->apz + half_dt * fw[kp] * tmp2 * c->dzinv[k];
  } else {
    q->amz = q->amz - half_dt * hyb1 * fw[id] * c->dzinv[k];
    q->apz = q->apz + half_dt * hyb2 * fw[kp] * c->dzinv[k];
  }
  hyb1 = 0.5 * (1.0 - fsign1(fw[id])); hyb2 = 0.5 * (1.0 + fsign1(fw[kp]));
  tmp1 = fint(c->z, c->zc, k); tmp2 = 1.0 - fint(c->z, c->zc, k + 1);
  if (central) q->acz = q->acz + half_dt * (fw[kp] * tmp2 - fw[id] * tmp1) * c->dzinv[k];
  else q->acz = q->acz + half_dt * (fw[kp] * hyb2 - fw[id] * hyb1) * c->dzinv[k];
}

/* CORE_TDMA.F90:11-34 on a[n1..n2] (gam in g, result in u) */
static void tdma_ad(const double *a, const double *b, const double *cc, const double *r, double *u, double *g, int n1,
                    int n2) {
  double binv = 1.0 / b[n1];
  u[n1] = r[n1] * binv;
  for (int j = n1 + 1; j <= n2; ++j) {
    g[j] = cc[j - 1] * binv;
    binv = 1.0 / (b[j] - a[j] * g[j]);
    u[j] = (r[j] - a[j] * u[j - 1]) * binv;
  }
  for (int j = n2 - 1; j >= n1; --j) u[j] = u[j] - g[j + 1] * u[j + 1];
}

int or_set_solve_ad(or_case *c, double dt, double reinv, double *ad) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  double *amx = ad, *apx = ad + (nx + 2), *amy = ad + 2 * (nx + 2), *apy = amy + (ny + 2),
         *amz = apy + (ny + 2), *apz = amz + (nz + 2);
  memset(ad, 0, sizeof(double) * (size_t)(2 * (nx + 2) + 2 * (ny + 2) + 2 * (nz + 2)));
  for (int i = 1; i <= nx - 1; ++i) {
    amx[i] = (c->dxcinv[i]) * c->dxinv[i];
    apx[i] = (c->dxcinv[i + 1]) * c->dxinv[i];
    amx[i] = -(0.50 * dt * reinv) * amx[i];
    apx[i] = -(0.50 * dt * reinv) * apx[i];
  }
  for (int j = 1; j <= ny - 1; ++j) {
    amy[j] = c->dycinv[j] * c->dyinv[j];
    apy[j] = c->dycinv[j + 1] * c->dyinv[j];
    amy[j] = -(0.50 * dt * reinv) * amy[j];
    apy[j] = -(0.50 * dt * reinv) * apy[j];
  }
  for (int k = 1; k <= nz - 1; ++k) {
    amz[k] = c->dzcinv[k] * c->dzinv[k];
    apz[k] = c->dzcinv[k + 1] * c->dzinv[k];
    amz[k] = -(0.50 * dt * reinv) * amz[k];
    apz[k] = -(0.50 * dt * reinv) * apz[k];
  }
  return OR_OK;
}

int or_itsolv_ad(or_case *c, const double *ad, double *var, const double *r, const double *fu, const double *fv,
                 const double *fw, double half_dt, double omega_ad) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const int nmax = (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)) + 2;
  double *am = dzalloc(nmax), *ac = dzalloc(nmax), *ap = dzalloc(nmax), *rh = dzalloc(nmax), *u = dzalloc(nmax),
         *g = dzalloc(nmax);
  ad_coef q;
  /* x lines (CORE_SOLVE_AD.F90:162-349): k, then j */
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j) {
      for (int i = 1; i <= nx - 1; ++i) {
        const long id = IDX(c, i, j, k);
        ad_cell(c, ad, fu, fv, fw, half_dt, i, j, k, &q);
        rh[i] = r[id] - (var[IDX(c, i, j - 1, k)] * q.amy + var[IDX(c, i, j + 1, k)] * q.apy +
                         var[IDX(c, i, j, k - 1)] * q.amz + var[IDX(c, i, j, k + 1)] * q.apz);
        const double rib = (1.0 - (double)c->iblank[id]) * (1.0 - (double)abs(c->ghost[id]));
        am[i] = q.amx * rib;
        ap[i] = q.apx * rib;
        ac[i] = 1.0 + (q.acx + q.acy + q.acz) * rib;
        rh[i] = rh[i] * rib + var[id] * (1.0 - rib);
      }
      am[0] = 0.0; ap[0] = 0.0; ac[0] = 1.0; rh[0] = var[IDX(c, 0, j, k)];
      am[nx] = 0.0; ap[nx] = 0.0; ac[nx] = 1.0; rh[nx] = var[IDX(c, nx, j, k)];
      tdma_ad(am, ac, ap, rh, u, g, 0, nx);
      for (int i = 1; i <= nx - 1; ++i) {
        const long id = IDX(c, i, j, k);
        var[id] = var[id] + omega_ad * (u[i] - var[id]);
      }
    }
  /* y lines (:353-549): k, then i */
  for (int k = 1; k <= nz - 1; ++k)
    for (int i = 1; i <= nx - 1; ++i) {
      for (int j = 1; j <= ny - 1; ++j) {
        const long id = IDX(c, i, j, k);
        ad_cell(c, ad, fu, fv, fw, half_dt, i, j, k, &q);
        rh[j] = r[id] - (var[IDX(c, i - 1, j, k)] * q.amx + var[IDX(c, i + 1, j, k)] * q.apx +
                         var[IDX(c, i, j, k - 1)] * q.amz + var[IDX(c, i, j, k + 1)] * q.apz);
        const double rib = (1.0 - (double)c->iblank[id]) * (1.0 - (double)abs(c->ghost[id]));
        am[j] = q.amy * rib;
        ap[j] = q.apy * rib;
        ac[j] = 1.0 + (q.acx + q.acy + q.acz) * rib;
        rh[j] = rh[j] * rib + var[id] * (1.0 - rib);
      }
      am[0] = 0.0; ap[0] = 0.0; ac[0] = 1.0; rh[0] = var[IDX(c, i, 0, k)];
      am[ny] = 0.0; ap[ny] = 0.0; ac[ny] = 1.0; rh[ny] = var[IDX(c, i, ny, k)];
      tdma_ad(am, ac, ap, rh, u, g, 0, ny);
      for (int j = 1; j <= ny - 1; ++j) {
        const long id = IDX(c, i, j, k);
        var[id] = var[id] + omega_ad * (u[j] - var[id]);
      }
    }
  /* z lines (:553-776): j, then i */
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      for (int k = 1; k <= nz - 1; ++k) {
        const long id = IDX(c, i, j, k);
        ad_cell(c, ad, fu, fv, fw, half_dt, i, j, k, &q);
        rh[k] = r[id] - (var[IDX(c, i - 1, j, k)] * q.amx + var[IDX(c, i + 1, j, k)] * q.apx +
                         var[IDX(c, i, j - 1, k)] * q.amy + var[IDX(c, i, j + 1, k)] * q.apy);
        const double rib = (1.0 - (double)c->iblank[id]) * (1.0 - (double)abs(c->ghost[id]));
        am[k] = q.amz * rib;
        ap[k] = q.apz * rib;
        ac[k] = 1.0 + (q.acx + q.acy + q.acz) * rib;
        rh[k] = rh[k] * rib + var[id] * (1.0 - rib);
      }
      am[0] = 0.0; ap[0] = 0.0; ac[0] = 1.0; rh[0] = var[IDX(c, i, j, 0)];
      am[nz] = 0.0; ap[nz] = 0.0; ac[nz] = 1.0; rh[nz] = var[IDX(c, i, j, nz)];
      tdma_ad(am, ac, ap, rh, u, g, 0, nz);
      for (int k = 1; k <= nz - 1; ++k) {
        const long id = IDX(c, i, j, k);
        var[id] = var[id] + omega_ad * (u[k] - var[id]);
      }
    }
  free(am); free(ac); free(ap); free(rh); free(u); free(g);
  return OR_OK;
}

int or_calc_residual_ad(or_case *c, const double *ad, const double *var, const double *r, const double *fu,
                        const double *fv, const double *fw, double half_dt, double *resm, int *loc) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  ad_coef q;
  double m = 0.0;
  int li = 1, lj = 1, lk = 1;
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        const long id = IDX(c, i, j, k);
        ad_cell(c, ad, fu, fv, fw, half_dt, i, j, k, &q);
        double res = r[id] - var[id] * (1.0 + q.acx + q.acy + q.acz) - var[IDX(c, i - 1, j, k)] * q.amx -
                     var[IDX(c, i + 1, j, k)] * q.apx - var[IDX(c, i, j - 1, k)] * q.amy -
                     var[IDX(c, i, j + 1, k)] * q.apy - var[IDX(c, i, j, k - 1)] * q.amz -
                     var[IDX(c, i, j, k + 1)] * q.apz;
        res = res * (1.0 - (double)c->iblank[id]) * (1.0 - (double)c->ghost[id]);
        if (fabs(res) > m) { m = fabs(res); li = i; lj = j; lk = k; }
      }
  if (resm) *resm = m;
  if (loc) { loc[0] = li; loc[1] = lj; loc[2] = lk; }
  return OR_OK;
}

/* CORE_SOLVE_AD.F90:11-127 solve_ad, one rank: while iter < itermax_ad and
 * the largest of the three components' max residual exceeds restol_ad:
 * itsolv_ad of u, v, w; the velocity ghost cells; face_vel;
 * enforce_global_mass_consv; the outer velocity BCs and their ghost layer;
 * calc_residual_ad of the three components.  The zero-gradient faces of vb
 * are the ones whose outflow enforce_global_mass_consv corrects. */
int or_solve_ad(or_case *c, const double *ad, double *u, double *v, double *w, const double *nlu, const double *nlv,
                const double *nlw, double *fu, double *fv, double *fw, double *const *bc, const double *ubi_g,
                const double *ubi_d, double half_dt, double omega_ad, const or_velocity_bc *vb, double pld,
                int itermax_gc, double restol_gcv, int itermax_ad, double restol_ad, int *iterations, double *resm,
                int *loc) {
  int vzg[6];
  for (int f = 0; f < 6; ++f) vzg[f] = vb->type[f] == 2;
  int iter = 0;
  double res2 = 1.0e10;
  int l[3] = {1, 1, 1};
  while (iter < itermax_ad && res2 > restol_ad) {
    or_itsolv_ad(c, ad, u, nlu, fu, fv, fw, half_dt, omega_ad);
    or_itsolv_ad(c, ad, v, nlv, fu, fv, fw, half_dt, omega_ad);
    or_itsolv_ad(c, ad, w, nlw, fu, fv, fw, half_dt, omega_ad);
    /* the reference stops the run when the ghost velocities do not converge
       (GCM_GHOSTCELL_UPDATE.F90:344-356) */
    if (or_ghostcell_velocity(c, u, v, w, ubi_g, ubi_d, pld, itermax_gc, restol_gcv, NULL) != OR_OK)
      return OR_NOT_CONVERGED;
    or_face_vel(c, u, v, w, bc[0], bc[4], bc[8], fu, fv, fw);
    or_enforce_global_mass_consv(c, fu, fv, fw, bc[0], bc[4], bc[8], vzg);
    int st = or_set_outer_velocity_bc(c, u, v, w, bc, vb);
    if (st != OR_OK) return st;
    or_set_outer_ghost_velocity(c, u, v, w, bc);
    double ru, rv, rw;
    int lu[3], lv[3], lw[3];
    or_calc_residual_ad(c, ad, u, nlu, fu, fv, fw, half_dt, &ru, lu);
    or_calc_residual_ad(c, ad, v, nlv, fu, fv, fw, half_dt, &rv, lv);
    or_calc_residual_ad(c, ad, w, nlw, fu, fv, fw, half_dt, &rw, lw);
    res2 = fabs(ru);
    memcpy(l, lu, sizeof(l));
    if (fabs(rv) > res2) { res2 = fabs(rv); memcpy(l, lv, sizeof(l)); }
    if (fabs(rw) > res2) { res2 = fabs(rw); memcpy(l, lw, sizeof(l)); }
    iter++;
  }
  if (iterations) *iterations = iter;
  if (resm) *resm = res2;
  if (loc) memcpy(loc, l, sizeof(l));
  return OR_OK;  /* an unconverged sweep count is reported, not an error (CORE_SOLVE_AD.F90:110-114) */
}

/* CORE_POISSON.F90:205-456 itsolv (LSOR: x lexicographic, y zebra, z) on
 * the fine grid with the iblank/ghost flag */
static void itsolv_lsor(or_case *c, double *var, const double *r, const or_params *prm) {
  /* identical to itsolv_mg on level 1 except: relaxation only on interior
   * rows, no |ac| guard, and no outer-BC refresh between directions; the
   * level-1 igk equals iblank|ghost after or_mg_prepare */
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const long NX = c->NX, NXY = c->NX * c->NY;
  const double om = prm->omega_pson;
  double *am = c->am, *ac = c->ac, *ap = c->ap, *rh = c->rr, *du = c->dum;
  double *g = (double *)malloc(sizeof(double) * (size_t)(c->nx + c->ny + c->nz + 4));
  for (int k = 1; k <= nz - 1; ++k)
    for (int j = 1; j <= ny - 1; ++j) {
      double amy = c->dycinv[j] * c->dyinv[j], apy = c->dycinv[j + 1] * c->dyinv[j], acy = -(amy + apy);
      double amz = c->dzcinv[k] * c->dzinv[k], apz = c->dzcinv[k + 1] * c->dzinv[k], acz = -(amz + apz);
      for (int i = 1; i <= nx - 1; ++i) {
        long id = IDX(c, i, j, k);
        am[i] = c->dxcinv[i] * c->dxinv[i];
        ap[i] = c->dxcinv[i + 1] * c->dxinv[i];
        ac[i] = -(am[i] + ap[i]);
        rh[i] = r[id] - var[id - NX] * amy - var[id + NX] * apy - var[id - NXY] * amz - var[id + NXY] * apz;
        double flag = (1.0 - (double)c->iblank[id]) * (1.0 - (double)c->ghost[id]);
        am[i] = am[i] * flag; ap[i] = ap[i] * flag;
        ac[i] = (ac[i] + acy + acz) * flag + (1.0 - flag);
        rh[i] = rh[i] * flag + (1.0 - flag) * var[id];
      }
      am[0] = 0.0; ap[0] = 0.0; ac[0] = 1.0; rh[0] = var[IDX(c, 0, j, k)];
      am[nx] = 0.0; ap[nx] = 0.0; ac[nx] = 1.0; rh[nx] = var[IDX(c, nx, j, k)];
      tdma_ws(am, ac, ap, rh, du, 0, nx, g);
      for (int i = 1; i <= nx - 1; ++i) {
        long id = IDX(c, i, j, k);
        var[id] = var[id] + om * (du[i] - var[id]);
      }
    }
  for (int col = 1; col <= 2; ++col)
    for (int k = 1; k <= nz - 1; ++k)
      for (int i = col; i <= nx - 1; i += 2) {
        double amx = c->dxcinv[i] * c->dxinv[i], apx = c->dxcinv[i + 1] * c->dxinv[i], acx = -(amx + apx);
        double amz = c->dzcinv[k] * c->dzinv[k], apz = c->dzcinv[k + 1] * c->dzinv[k], acz = -(amz + apz);
        for (int j = 1; j <= ny - 1; ++j) {
          long id = IDX(c, i, j, k);
          am[j] = c->dycinv[j] * c->dyinv[j];
          ap[j] = c->dycinv[j + 1] * c->dyinv[j];
          ac[j] = -(am[j] + ap[j]);
          rh[j] = r[id] - var[id - 1] * amx - var[id + 1] * apx - var[id - NXY] * amz - var[id + NXY] * apz;
          double flag = (1.0 - (double)c->iblank[id]) * (1.0 - (double)c->ghost[id]);
          am[j] = am[j] * flag; ap[j] = ap[j] * flag;
          ac[j] = (acx + ac[j] + acz) * flag + (1.0 - flag);
          rh[j] = rh[j] * flag + (1.0 - flag) * var[id];
        }
        am[0] = 0.0; ap[0] = 0.0; ac[0] = 1.0; rh[0] = var[IDX(c, i, 0, k)];
        am[ny] = 0.0; ap[ny] = 0.0; ac[ny] = 1.0; rh[ny] = var[IDX(c, i, ny, k)];
        tdma_ws(am, ac, ap, rh, du, 0, ny, g);
        for (int j = 1; j <= ny - 1; ++j) {
          long id = IDX(c, i, j, k);
          var[id] = var[id] + om * (du[j] - var[id]);
        }
      }
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i) {
      double amx = c->dxcinv[i] * c->dxinv[i], apx = c->dxcinv[i + 1] * c->dxinv[i], acx = -(amx + apx);
      double amy = c->dycinv[j] * c->dyinv[j], apy = c->dycinv[j + 1] * c->dyinv[j], acy = -(amy + apy);
      for (int k = 1; k <= nz - 1; ++k) {
        long id = IDX(c, i, j, k);
        am[k] = c->dzcinv[k] * c->dzinv[k];
        ap[k] = c->dzcinv[k + 1] * c->dzinv[k];
        ac[k] = -(am[k] + ap[k]);
        rh[k] = r[id] - var[id - 1] * amx - var[id + 1] * apx - var[id - NX] * amy - var[id + NX] * apy;
        double flag = (1.0 - (double)c->iblank[id]) * (1.0 - (double)c->ghost[id]);
        am[k] = am[k] * flag; ap[k] = ap[k] * flag;
        ac[k] = (acx + acy + ac[k]) * flag + (1.0 - flag);
        rh[k] = rh[k] * flag + (1.0 - flag) * var[id];
      }
      am[0] = 0.0; ap[0] = 0.0; ac[0] = 1.0; rh[0] = var[IDX(c, i, j, 0)];
      am[nz] = 0.0; ap[nz] = 0.0; ac[nz] = 1.0; rh[nz] = var[IDX(c, i, j, nz)];
      tdma_ws(am, ac, ap, rh, du, 0, nz, g);
      for (int k = 1; k <= nz - 1; ++k) {
        long id = IDX(c, i, j, k);
        var[id] = var[id] + om * (du[k] - var[id]);
      }
    }
  free(g);
}

/* CORE_MG.F90:1572-1848 mg_solve */
static int mg_solve(or_case *c, double *var, const double *rr, const or_params *prm) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  or_level *L1 = &c->lev[0];
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 0; i <= nx; ++i) {
        long id = IDX(c, i, j, k);
        L1->phi[id] = var[id];
        L1->rhs[id] = rr[id];
      }
  int iter = 0;
  double resm = 1.0e6;
  while (iter <= prm->iterInter && resm > prm->restol_pson) {
    for (int N = 0; N < c->mLevel; ++N) {
      or_level *L = &c->lev[N];
      long nL = (long)(L->I + 2) * (L->J + 2) * (L->K + 2);
      if (N > 0) memset(L->phi, 0, sizeof(double) * (size_t)nL);
      itsolv_mg(c, N, L->phi, L->rhs, L->igk, prm);
      for (int k = 1; k <= L->K - 1; ++k)
        for (int j = 1; j <= L->J - 1; ++j)
          for (int i = 1; i <= L->I; ++i) L->res[LIDX(L, i, j, k)] = L->rhs[LIDX(L, i, j, k)];
      residual_mg(c, N, L->phi, L->res, L->igk);
      if (N != c->mLevel - 1) mg_inject(c, N, L->res, c->lev[N + 1].rhs);
    }
    for (int N = c->mLevel - 1; N >= 1; --N) {
      or_level *L = &c->lev[N];
      if (N != c->mLevel - 1) itsolv_mg(c, N, L->phi, L->rhs, L->igk, prm);
      mg_interp(c, N, L->phi, c->lev[N - 1].phi, c->lev[N - 1].res);
    }
    resm = or_calc_residual(c, L1->phi, L1->rhs);
    iter++;
  }
  for (int k = 0; k <= nz + 1; ++k)
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 0; i <= nx; ++i) {
        long id = IDX(c, i, j, k);
        var[id] = L1->phi[id];
      }
  return iter;
}

/* CORE_POISSON.F90:679-724 calc_residual2 */
static double calc_residual2(const or_case *c, const double *var, const double *ptemp) {
  double r1 = 0.0;
  for (int k = 1; k <= c->nz - 1; ++k)
    for (int j = 1; j <= c->ny - 1; ++j)
      for (int i = 1; i <= c->nx - 1; ++i) {
        long id = IDX(c, i, j, k);
        double flag = 1.0 - (double)c->iblank[id];
        double res = fabs(var[id] - ptemp[id]) * flag;
        if (res > r1) r1 = res;
      }
  return r1;
}

int or_solve_poisson(or_case *c, double *p, const double *div,
                     const double *p_old, const double *dpdn_g,
                     const double *dpdn_d, const or_params *prm,
                     or_stats *st) {
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  int iter = 0, vc = 0;
  double maxres = 1.0e10, maxres2 = 1.0e10;
  int allN = 1;
  for (int f = 0; f < 6; ++f) allN &= (prm->pbc[f] == OR_PBC_NEUMANN);
  if (prm->it_solver_type == OR_SOLVER_MG) or_mg_prepare(c);
  while (iter < prm->itermax_pson && maxres2 > prm->restol_gcp) {
    if (allN) {
      double pAvg = p[IDX(c, 1, 1, 1)];
      for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
          for (int i = 0; i <= nx; ++i) {
            long id = IDX(c, i, j, k);
            if (prm->freeze_solid && c->iblank[id] == 1 && c->dead[id] != -1) continue;
            p[id] = p[id] - pAvg;
          }
    }
    outer_bc(c, p, 0, prm);
    enforce_p_compatibility(c, p, prm);
    memcpy(c->p_temp, p, sizeof(double) * (size_t)c->ntot);
    or_ghostcell_pressure(c, p, div, p_old, dpdn_g, dpdn_d, prm, NULL);
    if (prm->it_solver_type == OR_SOLVER_LSOR) {
      itsolv_lsor(c, p, div, prm);
      vc++;
    } else {
      vc += mg_solve(c, p, div, prm);
    }
    maxres = or_calc_residual(c, p, div);
    maxres2 = calc_residual2(c, p, c->p_temp);
    iter++;
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  if (st) {
    st->outer_iterations = iter;
    st->vcycles = vc;
    st->maxres = maxres;
    st->maxres2 = maxres2;
    st->relres = or_relres(c, p, div);
    st->seconds = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
  }
  return (maxres2 > prm->restol_gcp) ? OR_NOT_CONVERGED : OR_OK;
}

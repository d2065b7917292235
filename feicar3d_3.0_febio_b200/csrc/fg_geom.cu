// fg_geom.cu -- immersed-boundary tagging and ghost/dead-cell geometry on the
// device (sm_100a).  Compiled with --fmad=false: every FP64 expression is
// evaluated one IEEE operation at a time in the written order, so iblank,
// the ghost and dead lists and their host cells are bit-identical to the
// CPU restatement of BOUNDARY_IBLANK_FAST.F90 and GCM_SET_BOUNDARY.F90.
//
// Fields here use the reference layout (0:nx+1, 0:ny+1, 0:nz+1), nx, ny, nz
// node counts, index i + (nx+2)*(j + (ny+2)*k).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "fg_case.h"

namespace fg {

void geom_free(Geom &g) {
  for (auto &b : g.bodies) {
    fg::dev_free(b.d_xyz); fg::dev_free(b.d_en); fg::dev_free(b.d_vn); fg::dev_free(b.d_tri);
    fg::dev_free(b.d_uvw); fg::dev_free(b.d_uvw_old); fg::dev_free(b.d_snap); fg::dev_free(b.d_dpdn);
    fg::dev_free(b.d_v2t_off); fg::dev_free(b.d_v2t);
  }
  g.bodies.clear();
  fg::dev_free(g.d_iblank); fg::dev_free(g.d_ghost); fg::dev_free(g.d_dead); fg::dev_free(g.d_body);
  fg::dev_free(g.d_band); fg::dev_free(g.d_tmp); fg::dev_free(g.d_xc);
  g.d_iblank = g.d_ghost = g.d_dead = g.d_body = g.d_band = g.d_tmp = nullptr;
  g.d_xc = nullptr;
  for (DevScratch *b : {&g.cub_tmp, &g.sel_out, &g.sel_count, &g.cells, &g.glist, &g.dlist, &g.alpha,
                        &g.rank, &g.flags})
    b->release();
  g.rg.release();
  g.rd.release();
}

namespace geo {

// grid arrays in reference indexing, all length n+2
struct Grid {
  int nx, ny, nz;
  long long NX, NY;
  const double *x, *y, *z, *xc, *yc, *zc, *dx, *dy, *dz, *dxc, *dyc, *dzc;
};

struct Body {
  int nvert, ntri, type, dim;
  double mt;  // membrane thickness
  const double *vx, *vy, *vz;  // vertices
  const double *enx, *eny, *enz;  // element unit normals
  const double *vnx, *vny, *vnz;  // vertex unit normals
  const int *tri;
  const int *v2t_off, *v2t;
};

__device__ __forceinline__ long long ridx(const Grid &g, int i, int j, int k) {
  return (long long)i + g.NX * ((long long)j + g.NY * (long long)k);
}

// ------------------------------------------------- body intercept query
__device__ void cross3(const double *r, const double *s, double *o) {
  o[0] = r[1] * s[2] - s[1] * r[2];
  o[1] = r[2] * s[0] - s[2] * r[0];
  o[2] = r[0] * s[1] - s[0] * r[1];
}

// BOUNDARY_IBLANK_FAST.F90:1220-1313
__device__ void bi_inside(const double *xv, const double *yv, const double *zv, double xb,
                          double yb, double zb, double *a123o, double *adiffo) {
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
  *a123o = a123;
  *adiffo = a124 + a234 + a314 - a123;
}

// BOUNDARY_IBLANK_FAST.F90:1316-1536 (side fallback as in the restatement)
__device__ void bi_outside(const double *xv, const double *yv, const double *zv, double xcg,
                           double ycg, double zcg, const double *xvn, const double *yvn,
                           const double *zvn, double *xb, double *yb, double *zb, double *dist,
                           double *nx_, double *ny_, double *nz_, int *warn) {
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

struct BIResult {
  double x, y, z, dist, dot;
  int elem;
};

// BOUNDARY_IBLANK_FAST.F90:857-1216 for one point, by one warp: the
// nearest vertex (first index of the minimum) by a lane-parallel scan, then
// the incident triangles of that vertex one per lane, the kept element being
// the last one (in triangle order) at the minimum distance -- the element
// the sequential "dist <= distMin" loop keeps.
__device__ BIResult body_intercept_warp(const Body &B, double xC, double yC, double zC,
                                        int lane, int *warn) {
  double dmin = 0.0;
  int vmin = 0x7fffffff;
  for (int m = lane; m < B.nvert; m += 32) {
    const double dd = (B.vx[m] - xC) * (B.vx[m] - xC) + (B.vy[m] - yC) * (B.vy[m] - yC) +
                      (B.vz[m] - zC) * (B.vz[m] - zC);
    if (vmin == 0x7fffffff || dd < dmin) { dmin = dd; vmin = m; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double od = __shfl_down_sync(0xffffffffu, dmin, o);
    const int ov = __shfl_down_sync(0xffffffffu, vmin, o);
    const bool take = (ov != 0x7fffffff) &&
                      (vmin == 0x7fffffff || od < dmin || (od == dmin && ov < vmin));
    if (take) { dmin = od; vmin = ov; }
  }
  vmin = __shfl_sync(0xffffffffu, vmin, 0);
  const int t0 = B.v2t_off[vmin], t1 = B.v2t_off[vmin + 1];
  double bestd = 1.0e16, bx = 0, by = 0, bz = 0, bnx = 0, bny = 0, bnz = 0;
  int bel = -1;
  int lw = 0;
  for (int q0 = t0; q0 < t1; q0 += 32) {
    const int q = q0 + lane;
    double dist = 1.0e300, xt = 0, yt = 0, zt = 0, tnx = 0, tny = 0, tnz = 0;
    int e = -1;
    if (q < t1) {
      e = B.v2t[q];
      const int n1 = B.tri[3 * e], n2 = B.tri[3 * e + 1], n3 = B.tri[3 * e + 2];
      double xv[3] = {B.vx[n1], B.vx[n2], B.vx[n3]};
      double yv[3] = {B.vy[n1], B.vy[n2], B.vy[n3]};
      double zv[3] = {B.vz[n1], B.vz[n2], B.vz[n3]};
      const double xn = B.enx[e], yn = B.eny[e], zn = B.enz[e];
      double xvn[3] = {B.vnx[n1], B.vnx[n2], B.vnx[n3]};
      double yvn[3] = {B.vny[n1], B.vny[n2], B.vny[n3]};
      double zvn[3] = {B.vnz[n1], B.vnz[n2], B.vnz[n3]};
      const double planeConst = -xn * xv[0] - yn * yv[0] - zn * zv[0];
      const double dtp = -(xn * xC + yn * yC + zn * zC + planeConst);
      xt = xC + xn * dtp; yt = yC + yn * dtp; zt = zC + zn * dtp;
      double a123, adiff;
      bi_inside(xv, yv, zv, xt, yt, zt, &a123, &adiff);
      dist = sqrt((xC - xt) * (xC - xt) + (yC - yt) * (yC - yt) + (zC - zt) * (zC - zt));
      if (fabs(adiff) < 1.0e-6 * a123) {
        tnx = xn; tny = yn; tnz = zn;
      } else {
        bi_outside(xv, yv, zv, xC, yC, zC, xvn, yvn, zvn, &xt, &yt, &zt, &dist, &tnx, &tny, &tnz, &lw);
      }
    }
    // minimum distance over the batch, then the last position holding it
    double md = dist;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) md = fmin(md, __shfl_xor_sync(0xffffffffu, md, o));
    const unsigned hit = __ballot_sync(0xffffffffu, q < t1 && dist == md);
    if (hit && md <= bestd) {
      const int src = 31 - __clz(hit);
      bestd = md;
      bel = __shfl_sync(0xffffffffu, e, src);
      bx = __shfl_sync(0xffffffffu, xt, src); by = __shfl_sync(0xffffffffu, yt, src);
      bz = __shfl_sync(0xffffffffu, zt, src);
      bnx = __shfl_sync(0xffffffffu, tnx, src); bny = __shfl_sync(0xffffffffu, tny, src);
      bnz = __shfl_sync(0xffffffffu, tnz, src);
    }
  }
  // the side-selection fallback count of the lanes
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lw += __shfl_down_sync(0xffffffffu, lw, o);
  if (lane == 0 && warn) *warn += lw;
  BIResult r;
  r.x = bx; r.y = by; r.z = bz; r.elem = bel;
  r.dist = sqrt((bx - xC) * (bx - xC) + (by - yC) * (by - yC) + (bz - zC) * (bz - zC));
  r.dot = (xC - bx) * bnx + (yC - by) * bny + (zC - bz) * bnz;
  return r;
}

// ------------------------------------------------------------- band
// :153-396.  One thread per triangle: index box of the vertices (last
// bracketing index on each side, as the sequential scans), then marks it.
__global__ void k_band(Grid g, Body B, int8_t *band) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= B.ntri) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int v1 = B.tri[3 * m], v2 = B.tri[3 * m + 1], v3 = B.tri[3 * m + 2];
  const double xv[3] = {B.vx[v1], B.vx[v2], B.vx[v3]};
  const double yv[3] = {B.vy[v1], B.vy[v2], B.vy[v3]};
  const double zv[3] = {B.vz[v1], B.vz[v2], B.vz[v3]};
  const int Nm = (B.type == 2) ? 3 : 0;
  const double mtN = B.mt * (double)Nm;
  if ((xv[0] <= g.x[1] && xv[1] <= g.x[1] && xv[2] <= g.x[1]) ||
      (xv[0] >= g.x[nx] && xv[1] >= g.x[nx] && xv[2] >= g.x[nx]) ||
      (yv[0] + mtN <= g.y[1] && yv[1] + mtN <= g.y[1] && yv[2] + mtN <= g.y[1]) ||
      (yv[0] - mtN >= g.y[ny] && yv[1] - mtN >= g.y[ny] && yv[2] - mtN >= g.y[ny]) ||
      (zv[0] + mtN <= g.z[1] && zv[1] + mtN <= g.z[1] && zv[2] + mtN <= g.z[1]) ||
      (zv[0] - mtN >= g.z[nz] && zv[1] - mtN >= g.z[nz] && zv[2] - mtN >= g.z[nz]))
    return;
  double xmn = xv[0], xmx = xv[0], ymn = yv[0], ymx = yv[0], zmn = zv[0], zmx = zv[0];
  for (int q = 1; q < 3; ++q) {
    if (xv[q] < xmn) xmn = xv[q];
    if (xv[q] > xmx) xmx = xv[q];
    if (yv[q] < ymn) ymn = yv[q];
    if (yv[q] > ymx) ymx = yv[q];
    if (zv[q] < zmn) zmn = zv[q];
    if (zv[q] > zmx) zmx = zv[q];
  }
  if (B.type == 2) {
    xmn = xmn - mtN; xmx = xmx + mtN; ymn = ymn - mtN; ymx = ymx + mtN;
    zmn = zmn - mtN; zmx = zmx + mtN;
  }
  int iMin = 0, iMax = 0, jMin = 0, jMax = 0, kMin = 0, kMax = 0;
  for (int i = 0; i <= nx - 1; ++i) {
    if ((g.xc[i] - xmn) * (g.xc[i + 1] - xmn) <= 0.0) iMin = i;
    if ((g.xc[i] - xmx) * (g.xc[i + 1] - xmx) <= 0.0) iMax = i + 1;
  }
  if (iMin == 0) iMin = 1;
  if (iMax == 0 || iMax == nx) iMax = nx - 1;
  for (int j = 0; j <= ny - 1; ++j) {
    if ((g.yc[j] - ymn) * (g.yc[j + 1] - ymn) <= 0.0) jMin = j;
    if ((g.yc[j] - ymx) * (g.yc[j + 1] - ymx) <= 0.0) jMax = j + 1;
  }
  if (jMin == 0) jMin = 1;
  if (jMax == 0 || jMax == ny) jMax = ny - 1;
  for (int k = 0; k <= nz - 1; ++k) {
    if ((g.zc[k] - zmn) * (g.zc[k + 1] - zmn) <= 0.0) kMin = k;
    if ((g.zc[k] - zmx) * (g.zc[k + 1] - zmx) <= 0.0) kMax = k + 1;
  }
  if (kMin == 0) kMin = 1;
  if (kMax == 0 || kMax == nz) kMax = nz - 1;
  for (int k = kMin; k <= kMax; ++k)
    for (int j = jMin; j <= jMax; ++j)
      for (int i = iMin; i <= iMax; ++i) band[ridx(g, i, j, k)] = 1;
}

// :417-474 dot-normal (or membrane distance) classification of band cells,
// one warp per band cell; bodies are tested from the last to the first
struct Bodies {
  int n;
  Body b[8];
};

__global__ void k_classify(Grid g, Bodies BB, const int *cells, int ncells, int8_t *ibt,
                           int8_t *body, int *warn) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= ncells) return;
  const long long id = cells[w];
  const int i = (int)(id % g.NX), j = (int)((id / g.NX) % g.NY), k = (int)(id / (g.NX * g.NY));
  const double xP = g.xc[i], yP = g.yc[j], zP = g.zc[k];
  int hit = 0;
  int lw = 0;
  for (int ib = BB.n - 1; ib >= 0; --ib) {
    const BIResult r = body_intercept_warp(BB.b[ib], xP, yP, zP, lane, &lw);
    if (BB.b[ib].type == 2) {
      const double de = sqrt((xP - r.x) * (xP - r.x) + (yP - r.y) * (yP - r.y) + (zP - r.z) * (zP - r.z));
      if (de < BB.b[ib].mt / 2.0) { hit = ib + 1; break; }
    } else {
      if (r.dot >= 0.0) { hit = ib + 1; break; }
    }
  }
  if (lane == 0) {
    ibt[id] = hit ? 1 : 0;
    if (hit) body[id] = (int8_t)hit;
    if (lw) atomicAdd(warn, lw);
  }
}

// :509-536 i-direction fill, one thread per (j,k) line; :725-730 outflow copy
__global__ void k_fill(Grid g, const int8_t *band, int8_t *ibt, int8_t *body) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nyl = g.ny - 1;
  if (t >= nyl * (g.nz - 1)) return;
  const int j = 1 + t % nyl, k = 1 + t / nyl;
  const long long r0 = ridx(g, 0, j, k);
  for (int ii = 1; ii <= g.nx - 1; ++ii)
    if (band[r0 + ii]) { ibt[r0] = ibt[r0 + ii]; body[r0] = body[r0 + ii]; break; }
  for (int i = 1; i <= g.nx - 1; ++i) {
    if (band[r0 + i]) continue;
    ibt[r0 + i] = ibt[r0 + i - 1];
    if (ibt[r0 + i] == 1) body[r0 + i] = body[r0 + i - 1];
  }
  ibt[r0 + g.nx] = ibt[r0 + g.nx - 1];
  body[r0 + g.nx] = body[r0 + g.nx - 1];
}

// :763-787 commit over i = 0..nx of the interior (j,k)
__global__ void k_commit(Grid g, const int8_t *ibt, int8_t *ib) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)(g.nx + 1) * (g.ny - 1) * (g.nz - 1);
  if (e >= n) return;
  const int i = (int)(e % (g.nx + 1));
  const int j = 1 + (int)((e / (g.nx + 1)) % (g.ny - 1));
  const int k = 1 + (int)(e / ((long long)(g.nx + 1) * (g.ny - 1)));
  const long long id = ridx(g, i, j, k);
  ib[id] = ibt[id];
}

// ------------------------------------------------------- smoothing
// In-place passes of GCM_SET_BOUNDARY.F90:132-223 and :1639-1692 give every
// cell the count over its "backward" neighbours (already visited in the
// loop order) in their UPDATED state and over the forward ones in their
// state at the start of the pass.  Flags only go 0 -> 1, so iterating
//   X(c) = old(c) OR [count(X over backward) + count(old over forward) >= thr]
// from X = old reaches the sequential result in at most (longest chain)
// steps; each step is a Jacobi update from cur to nxt.
// mode 0: 3-D pass (k,j,i order, 6 faces, >= 5); mode 1: x planes (j,k
// order within an i plane, >= 3); mode 2: y planes (i,k order, >= 3).
// Only interior cells (1..n-1 on every axis) are updated and written; a
// backward neighbour on the boundary layer is never updated, so it is read
// from old, and cur/nxt need no boundary values.
__global__ void k_smooth_step(Grid g, int mode, const int8_t *old, const int8_t *cur, int8_t *nxt,
                              const int8_t *bold, const int8_t *bcur, int8_t *bnxt, int *changed) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)(g.nx - 1) * (g.ny - 1) * (g.nz - 1);
  if (e >= n) return;
  const int i = 1 + (int)(e % (g.nx - 1));
  const int j = 1 + (int)((e / (g.nx - 1)) % (g.ny - 1));
  const int k = 1 + (int)(e / ((long long)(g.nx - 1) * (g.ny - 1)));
  const long long id = ridx(g, i, j, k);
  if (old[id] == 1) { nxt[id] = 1; bnxt[id] = bcur[id]; return; }
  const long long sx = 1, sy = g.NX, sz = g.NX * g.NY;
  // neighbour offsets in the reference enumeration order, and which are
  // backward in the loop order and updated (backward and not on the boundary)
  long long off[6];
  bool upd[6];
  int nn, thr;
  if (mode == 0) {
    off[0] = -sz; off[1] = -sy; off[2] = -sx; off[3] = sx; off[4] = sy; off[5] = sz;
    upd[0] = k > 1; upd[1] = j > 1; upd[2] = i > 1; upd[3] = upd[4] = upd[5] = false;
    nn = 6; thr = 5;
  } else if (mode == 1) {
    off[0] = -sz; off[1] = -sy; off[2] = sy; off[3] = sz;
    upd[0] = k > 1; upd[1] = j > 1; upd[2] = false; upd[3] = false;
    nn = 4; thr = 3;
  } else {
    off[0] = -sz; off[1] = -sx; off[2] = sx; off[3] = sz;
    upd[0] = k > 1; upd[1] = i > 1; upd[2] = false; upd[3] = false;
    nn = 4; thr = 3;
  }
  int s = 0, ibody = 0;
  for (int q = 0; q < nn; ++q) {
    const long long nb = id + off[q];
    const int8_t v = upd[q] ? cur[nb] : old[nb];
    const int8_t bv = upd[q] ? bcur[nb] : bold[nb];
    if (v == 1) {
      s++;
      if (bv > 0) ibody = bv;
    }
  }
  int8_t nv = 0, nb = bcur[id];
  if (s >= thr) { nv = 1; nb = (int8_t)(ibody > 0 ? ibody : 1); }
  nxt[id] = nv;
  bnxt[id] = nb;
  if (nv != cur[id] || nb != bcur[id]) atomicOr(changed, 1);
}

// interior cells of the fixed point back into the case's iblank and body
__global__ void k_smooth_commit(Grid g, const int8_t *cur, const int8_t *bcur, int8_t *iblank,
                                int8_t *body) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)(g.nx - 1) * (g.ny - 1) * (g.nz - 1);
  if (e >= n) return;
  const int i = 1 + (int)(e % (g.nx - 1));
  const int j = 1 + (int)((e / (g.nx - 1)) % (g.ny - 1));
  const int k = 1 + (int)(e / ((long long)(g.nx - 1) * (g.ny - 1)));
  const long long id = ridx(g, i, j, k);
  iblank[id] = cur[id];
  body[id] = bcur[id];
}

// ---------------------------------------------------------- ghosts
// GCM_SET_BOUNDARY.F90:800-876: fluid interior cells face-adjacent to an
// iblank cell; their body is that of the first such iblank cell in (k,j,i)
// order among the cells the reference loop visits (i in [1,nx-1]).
__global__ void k_ghost_mark(Grid g, const int8_t *ib, int8_t *ghost, int8_t *body) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)(g.nx - 1) * (g.ny - 1) * (g.nz - 1);
  if (e >= n) return;
  const int i = 1 + (int)(e % (g.nx - 1));
  const int j = 1 + (int)((e / (g.nx - 1)) % (g.ny - 1));
  const int k = 1 + (int)(e / ((long long)(g.nx - 1) * (g.ny - 1)));
  const long long id = ridx(g, i, j, k);
  if (ib[id] != 0) { ghost[id] = 0; return; }
  const long long sy = g.NX, sz = g.NX * g.NY;
  // ascending linear index: -z, -y, -x, +x, +y, +z
  const long long off[6] = {-sz, -sy, -1, 1, sy, sz};
  const int ii[6] = {i, i, i - 1, i + 1, i, i};
  int8_t gb = 0, is_g = 0;
  for (int q = 0; q < 6; ++q) {
    if (ii[q] < 1 || ii[q] > g.nx - 1) continue;
    const long long nb = id + off[q];
    if (ib[nb] == 1) { is_g = 1; gb = body[nb]; break; }
  }
  ghost[id] = is_g;
  if (is_g) body[id] = gb;  // each ghost reads only iblank cells' bodies
}

// GCM_SET_BOUNDARY.F90:946-964: iblank face neighbours of ghost cells
__global__ void k_dead_mark(Grid g, const int8_t *ib, const int8_t *ghost, int8_t *dead) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)(g.nx + 2) * (g.ny + 2) * (g.nz + 2);
  if (e >= n) return;
  const int i = (int)(e % g.NX);
  const int j = (int)((e / g.NX) % g.NY);
  const int k = (int)(e / (g.NX * g.NY));
  if (ib[e] != 1) { dead[e] = 0; return; }
  const long long sy = g.NX, sz = g.NX * g.NY;
  const int ci[6] = {i - 1, i + 1, i, i, i, i};
  const int cj[6] = {j, j, j - 1, j + 1, j, j};
  const int ck[6] = {k, k, k, k, k - 1, k + 1};
  const long long off[6] = {-1, 1, -sy, sy, -sz, sz};
  int8_t d = 0;
  for (int q = 0; q < 6; ++q) {
    if (ci[q] < 1 || ci[q] > g.nx - 1 || cj[q] < 1 || cj[q] > g.ny - 1 || ck[q] < 1 || ck[q] > g.nz - 1)
      continue;
    if (ghost[e + off[q]] == 1) { d = -1; break; }
  }
  dead[e] = d;
}

// -------------------------------------------------- image points
__device__ __forceinline__ int nint_d(double v) {
  return (int)(v >= 0.0 ? floor(v + 0.5) : -floor(-v + 0.5));
}

// GCM_SET_BOUNDARY.F90:607-797 (inverse: LAPACK getrf/getri semantics as in
// the restatement)
__device__ int invert8(double *a, double *inv) {
  int ipiv[8];
  int info = 0;
#define A(i, j) a[(i) + 8 * (j)]
  for (int j = 0; j < 8; ++j) {
    int p = j;
    double mx = fabs(A(j, j));
    for (int i = j + 1; i < 8; ++i)
      if (fabs(A(i, j)) > mx) { mx = fabs(A(i, j)); p = i; }
    ipiv[j] = p;
    if (A(p, j) == 0.0) { if (info == 0) info = j + 1; continue; }
    if (p != j)
      for (int q = 0; q < 8; ++q) { double t = A(j, q); A(j, q) = A(p, q); A(p, q) = t; }
    double r = 1.0 / A(j, j);
    for (int i = j + 1; i < 8; ++i) A(i, j) = A(i, j) * r;
    for (int q = j + 1; q < 8; ++q)
      for (int i = j + 1; i < 8; ++i) A(i, q) = A(i, q) - A(i, j) * A(j, q);
  }
  if (info) return info;
  for (int j = 0; j < 8; ++j) {
    A(j, j) = 1.0 / A(j, j);
    double ajj = -A(j, j);
    for (int i = 0; i < j; ++i) {
      double s = 0.0;
      for (int q = i; q < j; ++q) s = s + A(i, q) * A(q, j);
      inv[i] = s;
    }
    for (int i = 0; i < j; ++i) A(i, j) = inv[i] * ajj;
  }
  double work[8];
  for (int j = 7; j >= 0; --j) {
    for (int i = j + 1; i < 8; ++i) { work[i] = A(i, j); A(i, j) = 0.0; }
    for (int q = j + 1; q < 8; ++q)
      for (int i = 0; i < 8; ++i) A(i, j) = A(i, j) - A(i, q) * work[q];
  }
  for (int j = 6; j >= 0; --j) {
    int jp = ipiv[j];
    if (jp != j)
      for (int i = 0; i < 8; ++i) { double t = A(i, j); A(i, j) = A(i, jp); A(i, jp) = t; }
  }
#undef A
  for (int q = 0; q < 64; ++q) inv[q] = a[q];
  return 0;
}

__constant__ int c_incI[8] = {0, 0, 1, 1, 0, 0, 1, 1};
__constant__ int c_incJ[8] = {0, 1, 1, 0, 0, 1, 1, 0};
__constant__ int c_incK[8] = {0, 0, 0, 0, 1, 1, 1, 1};

__device__ void van_matrix(const Grid &g, int iG, int jG, int kG, int ic, int jc, int kc, double xIP,
                           double yIP, double zIP, double xBI, double yBI, double zBI, double xN,
                           double yN, double zN, double *cD, double *cN) {
  double vD[64], vN[64], iD[64], iN[64];
  for (int r = 0; r < 8; ++r) {
    int i = ic + c_incI[r], j = jc + c_incJ[r], k = kc + c_incK[r];
    double x1 = g.xc[i], x2 = g.yc[j], x3 = g.zc[k];
    double rowD[8] = {x1 * x2 * x3, x1 * x2, x1 * x3, x2 * x3, x1, x2, x3, 1.0};
    double rowN[8];
    for (int q = 0; q < 8; ++q) rowN[q] = rowD[q];
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
  invert8(vD, iD);
  invert8(vN, iN);
  for (int r = 0; r < 8; ++r) {
    cD[r] = iD[0 + 8 * r] * xIP * yIP * zIP + iD[1 + 8 * r] * xIP * yIP + iD[2 + 8 * r] * xIP * zIP +
            iD[3 + 8 * r] * yIP * zIP + iD[4 + 8 * r] * xIP + iD[5 + 8 * r] * yIP +
            iD[6 + 8 * r] * zIP + iD[7 + 8 * r];
    cN[r] = iN[0 + 8 * r] * xIP * yIP * zIP + iN[1 + 8 * r] * xIP * yIP + iN[2 + 8 * r] * xIP * zIP +
            iN[3 + 8 * r] * yIP * zIP + iN[4 + 8 * r] * xIP + iN[5 + 8 * r] * yIP +
            iN[6 + 8 * r] * zIP + iN[7 + 8 * r];
  }
}

// Per ghost cell (warp): body intercept, image point, host cell
// (GCM_SET_BOUNDARY.F90:321-475).  Writes bi, ip, probe, cell, closest, the
// intercept normal and ds.
struct RowOut {
  double *bi;  // body intercept (before the membrane shift)
  double *bw;  // intercept the interpolation weights use
  double *ip, *probe, *nrm, *ds;
  int *cell, *closest;
};

__global__ void k_ghost_geom(Grid g, Bodies BB, const int *list, int n, const int8_t *body,
                             double pln, RowOut out, int *warn) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const long long id = list[w];
  const int iG = (int)(id % g.NX), jG = (int)((id / g.NX) % g.NY), kG = (int)(id / (g.NX * g.NY));
  int ib = body[id] - 1;
  if (ib < 0) ib = 0;
  if (ib >= BB.n) ib = BB.n - 1;
  const double xGC = g.xc[iG], yGC = g.yc[jG], zGC = g.zc[kG];
  int lw = 0;
  BIResult r = body_intercept_warp(BB.b[ib], xGC, yGC, zGC, lane, &lw);
  if (lane != 0) return;
  if (lw) atomicAdd(warn, lw);
  double xBI = r.x, yBI = r.y, zBI = r.z;
  if (BB.b[ib].dim == 2) zBI = zGC;
  out.closest[w] = r.elem;
  out.bi[3 * w] = xBI; out.bi[3 * w + 1] = yBI; out.bi[3 * w + 2] = zBI;
  double ds = sqrt((xGC - xBI) * (xGC - xBI) + (yGC - yBI) * (yGC - yBI) + (zGC - zBI) * (zGC - zBI));
  const double sx = (xGC - xBI) / ds, sy = (yGC - yBI) / ds, sz = (zGC - zBI) / ds;
  if (BB.b[ib].type == 2) {
    const double mt = BB.b[ib].mt;
    xBI = xBI + mt / 2.0 * sx; yBI = yBI + mt / 2.0 * sy; zBI = zBI + mt / 2.0 * sz;
    ds = sqrt((xGC - xBI) * (xGC - xBI) + (yGC - yBI) * (yGC - yBI) + (zGC - zBI) * (zGC - zBI));
  }
  out.nrm[3 * w] = -sx; out.nrm[3 * w + 1] = -sy; out.nrm[3 * w + 2] = -sz;
  out.ds[w] = ds;
  out.probe[w] = ds * pln;
  const double xIP = xBI - (xBI - xGC) * pln;
  const double yIP = yBI - (yBI - yGC) * pln;
  const double zIP = zBI - (zBI - zGC) * pln;
  out.ip[3 * w] = xIP; out.ip[3 * w + 1] = yIP; out.ip[3 * w + 2] = zIP;
  out.bw[3 * w] = xBI; out.bw[3 * w + 1] = yBI; out.bw[3 * w + 2] = zBI;
  double maxDelta = g.dx[iG];
  if (g.dy[jG] > maxDelta) maxDelta = g.dy[jG];
  if (g.dz[kG] > maxDelta) maxDelta = g.dz[kG];
  const int iR = 2 * nint_d(maxDelta / g.dx[iG] + 0.5);
  const int jR = 2 * nint_d(maxDelta / g.dy[jG] + 0.5);
  const int kR = 2 * nint_d(maxDelta / g.dz[kG] + 0.5);
  int ic = -1, jc = -1, kc = -1;
  int lo = iG - iR, hi = iG + iR;
  if (lo < 0) lo = 0;
  if (hi > g.nx) hi = g.nx;
  for (int i = lo; i <= hi; ++i)
    if (g.xc[i] <= xIP && g.xc[i + 1] > xIP) ic = i;
  lo = jG - jR; hi = jG + jR;
  if (lo < 0) lo = 0;
  if (hi > g.ny) hi = g.ny;
  for (int j = lo; j <= hi; ++j)
    if (g.yc[j] <= yIP && g.yc[j + 1] > yIP) jc = j;
  lo = kG - kR; hi = kG + kR;
  if (lo < 0) lo = 0;
  if (hi > g.nz) hi = g.nz;
  for (int k = lo; k <= hi; ++k)
    if (g.zc[k] <= zIP && g.zc[k + 1] > zIP) kc = k;
  out.cell[3 * w] = ic; out.cell[3 * w + 1] = jc; out.cell[3 * w + 2] = kc;
}

// Per dead cell (warp): GCM_SET_BOUNDARY.F90:1053-1409 up to the host cell
__global__ void k_dead_geom(Grid g, Bodies BB, const int *list, int n, const int8_t *body,
                            double plnD, RowOut out, int *warn, int *nobody) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const long long id = list[w];
  const int iG = (int)(id % g.NX), jG = (int)((id / g.NX) % g.NY), kG = (int)(id / (g.NX * g.NY));
  const int ib = body[id] - 1;
  if (ib < 0 || ib >= BB.n) {
    if (lane == 0) {
      atomicAdd(nobody, 1);
      out.cell[3 * w] = -1; out.cell[3 * w + 1] = -1; out.cell[3 * w + 2] = -1;
      out.ds[w] = -1.0;  // contributes nothing to alphaGhost
    }
    return;
  }
  const double xDC = g.xc[iG], yDC = g.yc[jG], zDC = g.zc[kG];
  int lw = 0;
  BIResult r = body_intercept_warp(BB.b[ib], xDC, yDC, zDC, lane, &lw);
  if (lane != 0) return;
  if (lw) atomicAdd(warn, lw);
  double xBI = r.x, yBI = r.y, zBI = r.z;
  if (BB.b[ib].dim == 2) zBI = zDC;
  out.closest[w] = r.elem;
  out.bi[3 * w] = xBI; out.bi[3 * w + 1] = yBI; out.bi[3 * w + 2] = zBI;
  double ds = sqrt((xDC - xBI) * (xDC - xBI) + (yDC - yBI) * (yDC - yBI) + (zDC - zBI) * (zDC - zBI));
  double sx = (xBI - xDC) / ds, sy = (yBI - yDC) / ds, sz = (zBI - zDC) / ds;
  const double bnx = -sx, bny = -sy, bnz = -sz;
  if (BB.b[ib].type == 2) {
    const double mt = BB.b[ib].mt;
    sx = -sx; sy = -sy; sz = -sz;
    if (ds >= mt / 2.0) {
      const double s = ds + (double)0.1f * (ds - mt / 2.0);
      xBI = xBI + s * sx; yBI = yBI + s * sy; zBI = zBI + s * sz;
    } else {
      xBI = xBI + mt / 2.0 * sx; yBI = yBI + mt / 2.0 * sy; zBI = zBI + mt / 2.0 * sz;
    }
    double zIP = zDC + (zBI - zDC) * plnD;
    double yIP = yDC + (yBI - yDC) * plnD;
    int guard = 0;
    while ((yIP < g.yc[0] || yIP > g.yc[g.ny + 1]) && guard++ < 200) {
      const double d1 = sqrt((xDC - xBI) * (xDC - xBI) + (yDC - yBI) * (yDC - yBI) + (zDC - zBI) * (zDC - zBI));
      const double t = -0.5 * d1;
      xBI = xBI + t * sx; yBI = yBI + t * sy; zBI = zBI + t * sz;
      yIP = yDC + (yBI - yDC) * plnD;
    }
    guard = 0;
    while ((zIP < g.zc[0] || zIP > g.zc[g.nz + 1]) && guard++ < 200) {
      const double d1 = sqrt((xDC - xBI) * (xDC - xBI) + (yDC - yBI) * (yDC - yBI) + (zDC - zBI) * (zDC - zBI));
      const double t = -0.5 * d1;
      xBI = xBI + t * sx; yBI = yBI + t * sy; zBI = zBI + t * sz;
      zIP = zDC + (zBI - zDC) * plnD;
    }
    ds = sqrt((xDC - xBI) * (xDC - xBI) + (yDC - yBI) * (yDC - yBI) + (zDC - zBI) * (zDC - zBI));
  }
  out.ds[w] = ds;
  out.nrm[3 * w] = bnx; out.nrm[3 * w + 1] = bny; out.nrm[3 * w + 2] = bnz;
  double xIP = xDC + (xBI - xDC) * plnD;
  double yIP = yDC + (yBI - yDC) * plnD;
  double zIP = zDC + (zBI - zDC) * plnD;
  double probe = ds * plnD;
  if (yIP < g.yc[0] || yIP > g.yc[g.ny + 1]) {
    yIP = (fabs(yIP - g.yc[0]) < fabs(yIP - g.yc[g.ny + 1])) ? g.yc[0] : g.yc[g.ny + 1];
    probe = sqrt((xDC - xIP) * (xDC - xIP) + (yDC - yIP) * (yDC - yIP) + (zDC - zIP) * (zDC - zIP));
  }
  if (zIP < g.zc[0] || zIP > g.zc[g.nz + 1]) {
    zIP = (fabs(zIP - g.zc[0]) < fabs(zIP - g.zc[g.nz + 1])) ? g.zc[0] : g.zc[g.nz + 1];
    probe = sqrt((xDC - xIP) * (xDC - xIP) + (yDC - yIP) * (yDC - yIP) + (zDC - zIP) * (zDC - zIP));
  }
  out.probe[w] = probe;
  out.ip[3 * w] = xIP; out.ip[3 * w + 1] = yIP; out.ip[3 * w + 2] = zIP;
  out.bw[3 * w] = xBI; out.bw[3 * w + 1] = yBI; out.bw[3 * w + 2] = zBI;
  double maxDelta = g.dx[iG];
  if (g.dy[jG] > maxDelta) maxDelta = g.dy[jG];
  if (g.dz[kG] > maxDelta) maxDelta = g.dz[kG];
  const int iR = 2 * nint_d(maxDelta / g.dx[iG] + 0.5);
  const int jR = 2 * nint_d(maxDelta / g.dy[jG] + 0.5);
  const int kR = 2 * nint_d(maxDelta / g.dz[kG] + 0.5);
  int ic = -1, jc = -1, kc = -1;
  int lo = iG - iR, hi = iG + iR;
  if (lo < 0) lo = 0;
  if (hi > g.nx) hi = g.nx;
  for (int i = lo; i <= hi; ++i)
    if (g.xc[i] <= xIP && g.xc[i + 1] >= xIP) ic = i;
  lo = jG - jR; hi = jG + jR;
  if (lo < 0) lo = 0;
  if (hi > g.ny) hi = g.ny;
  for (int j = lo; j <= hi; ++j)
    if (g.yc[j] <= yIP && g.yc[j + 1] >= yIP) jc = j;
  lo = kG - kR; hi = kG + kR;
  if (lo < 0) lo = 0;
  if (hi > g.nz) hi = g.nz;
  for (int k = lo; k <= hi; ++k)
    if (g.zc[k] <= zIP && g.zc[k + 1] >= zIP) kc = k;
  out.cell[3 * w] = ic; out.cell[3 * w + 1] = jc; out.cell[3 * w + 2] = kc;
}

// weights of one row (thread per row): ghost rows evaluate the interpolant
// at the ghost cell centre (GCM_SET_BOUNDARY.F90:521-523), dead rows at the
// image point (:1451-1453)
__global__ void k_weights(Grid g, const int *list, int n, RowOut out, int at_image, double *cD,
                          double *cN, int *hostfail) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n) return;
  const int ic = out.cell[3 * w], jc = out.cell[3 * w + 1], kc = out.cell[3 * w + 2];
  if (ic < 0 || jc < 0 || kc < 0) {
    atomicAdd(hostfail, 1);
    for (int q = 0; q < 8; ++q) { cD[8 * w + q] = 0.0; cN[8 * w + q] = 0.0; }
    return;
  }
  const long long id = list[w];
  const int iG = (int)(id % g.NX), jG = (int)((id / g.NX) % g.NY), kG = (int)(id / (g.NX * g.NY));
  double X, Y, Z;
  if (at_image) { X = out.ip[3 * w]; Y = out.ip[3 * w + 1]; Z = out.ip[3 * w + 2]; }
  else { X = g.xc[iG]; Y = g.yc[jG]; Z = g.zc[kG]; }
  van_matrix(g, iG, jG, kG, ic, jc, kc, X, Y, Z, out.bw[3 * w], out.bw[3 * w + 1], out.bw[3 * w + 2],
             out.nrm[3 * w], out.nrm[3 * w + 1], out.nrm[3 * w + 2], cD + 8 * w, cN + 8 * w);
}

// alphaGhost (GCM_SET_BOUNDARY.F90:1218-1277, 1477-1489): per ghost, the sum
// over its face-adjacent dead cells, in dead-list (k,j,i) order, of
// (ds / dxc)^2, then 1 - sqrt(sum)
__global__ void k_alpha(Grid g, const int *glist, int ng, const int8_t *dead, const int *dead_rank,
                        const double *dead_ds, double *alpha) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= ng) return;
  const long long id = glist[w];
  const int i = (int)(id % g.NX), j = (int)((id / g.NX) % g.NY), k = (int)(id / (g.NX * g.NY));
  const long long sy = g.NX, sz = g.NX * g.NY;
  // dead neighbours in ascending linear index: -z, -y, -x, +x, +y, +z; the
  // ghost is the dead cell's (+z, +y, +x, -x, -y, -z) neighbour and the
  // reference divides by dzc(k_dead+1)=dzc(k), dyc(j), dxc(i), dxc(i+1)...
  const long long off[6] = {-sz, -sy, -1, 1, sy, sz};
  const double h[6] = {g.dzc[k], g.dyc[j], g.dxc[i], g.dxc[i + 1], g.dyc[j + 1], g.dzc[k + 1]};
  const int ci[6] = {i, i, i - 1, i + 1, i, i};
  double s = 0.0;
  for (int q = 0; q < 6; ++q) {
    if (ci[q] < 1 || ci[q] > g.nx - 1) continue;
    const long long nb = id + off[q];
    if (dead[nb] != -1) continue;
    const int rk = dead_rank[nb];
    if (rk < 0 || dead_ds[rk] < 0.0) continue;
    const double t = dead_ds[rk] / h[q];
    s = s + t * t;
  }
  alpha[w] = 1.0 - sqrt(s);
}

__global__ void k_rank(const int *list, int n, int *rank) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w < n) rank[list[w]] = w;
}

struct IsFlag {
  const int8_t *f;
  int8_t want;
  __host__ __device__ bool operator()(const int &i) const { return f[i] == want; }
};

// dead cells that get a row: i in [1, nx-1], j in [0, ny], k in [0, nz]
// (GCM_SET_BOUNDARY.F90:1036-1047)
struct IsDeadRow {
  const int8_t *f;
  int NX, NY, nx, ny, nz;
  __host__ __device__ bool operator()(const int &e) const {
    if (f[e] != -1) return false;
    const int i = e % NX, j = (e / NX) % NY, k = e / (NX * NY);
    return i >= 1 && i <= nx - 1 && j <= ny && k <= nz;
  }
};

}  // namespace geo

// ---------------------------------------------------------------- host
static fg_status geom_grid(fg_case *c, geo::Grid &g) {
  Geom &G = *c->geom;
  const int n3[3] = {c->nx, c->ny, c->nz};
  if (!G.d_xc) {
    std::vector<double> all;
    const HLevel &L = c->lev[0];
    const std::vector<double> *xs[3] = {&L.x, &L.y, &L.z};
    const std::vector<double> *xcs[3] = {&L.xc, &L.yc, &L.zc};
    for (int a = 0; a < 3; ++a) {
      const int n = n3[a];
      std::vector<double> dx(n + 2, 0.0), dxc(n + 2, 0.0);
      for (int i = 0; i <= n; ++i) dx[i] = (*xs[a])[i + 1] - (*xs[a])[i];
      for (int i = 1; i <= n; ++i) dxc[i] = (*xcs[a])[i] - (*xcs[a])[i - 1];
      all.insert(all.end(), xs[a]->begin(), xs[a]->end());
      all.insert(all.end(), xcs[a]->begin(), xcs[a]->end());
      all.insert(all.end(), dx.begin(), dx.end());
      all.insert(all.end(), dxc.begin(), dxc.end());
    }
    FG_CUDA(fg::dev_alloc(&G.d_xc, all.size() * sizeof(double)));
    FG_CUDA(cudaMemcpy(G.d_xc, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  const double *p = G.d_xc;
  const double *ax[3][4];
  for (int a = 0; a < 3; ++a)
    for (int w = 0; w < 4; ++w) { ax[a][w] = p; p += n3[a] + 2; }
  g.nx = c->nx; g.ny = c->ny; g.nz = c->nz;
  g.NX = c->nx + 2; g.NY = c->ny + 2;
  g.x = ax[0][0]; g.xc = ax[0][1]; g.dx = ax[0][2]; g.dxc = ax[0][3];
  g.y = ax[1][0]; g.yc = ax[1][1]; g.dy = ax[1][2]; g.dyc = ax[1][3];
  g.z = ax[2][0]; g.zc = ax[2][1]; g.dz = ax[2][2]; g.dzc = ax[2][3];
  return FG_OK;
}

// BOUNDARY_SET_ARCLENGTH_NORM.F90:46-175 on the host (same operation order
// as the restatement; host code is compiled without FMA contraction)
static void host_normals(const DevBody &B, std::vector<double> &en, std::vector<double> &vn) {
  const int nt = B.ntri, nv = B.nvert;
  en.assign(3 * (size_t)nt, 0.0);
  vn.assign(3 * (size_t)nv, 0.0);
  const double *X = B.xyz.data();
  double *vnx = vn.data(), *vny = vn.data() + nv, *vnz = vn.data() + 2 * nv;
  double *enx = en.data(), *eny = en.data() + nt, *enz = en.data() + 2 * nt;
  for (int m = 0; m < nt; ++m) {
    const int n1 = B.tri[3 * m], n2 = B.tri[3 * m + 1], n3 = B.tri[3 * m + 2];
    const double ax = X[3 * n2] - X[3 * n1], ay = X[3 * n2 + 1] - X[3 * n1 + 1], az = X[3 * n2 + 2] - X[3 * n1 + 2];
    const double bx = X[3 * n3] - X[3 * n2], by = X[3 * n3 + 1] - X[3 * n2 + 1], bz = X[3 * n3 + 2] - X[3 * n2 + 2];
    const double nxv = (ay * bz - az * by);
    const double nyv = (az * bx - ax * bz);
    const double nzv = (ax * by - ay * bx);
    const double mag = sqrt(nxv * nxv + nyv * nyv + nzv * nzv);
    enx[m] = nxv / mag; eny[m] = nyv / mag; enz[m] = nzv / mag;
    vnx[n1] = vnx[n1] + enx[m]; vnx[n2] = vnx[n2] + enx[m]; vnx[n3] = vnx[n3] + enx[m];
    vny[n1] = vny[n1] + eny[m]; vny[n2] = vny[n2] + eny[m]; vny[n3] = vny[n3] + eny[m];
    vnz[n1] = vnz[n1] + enz[m]; vnz[n2] = vnz[n2] + enz[m]; vnz[n3] = vnz[n3] + enz[m];
  }
  for (int v = 0; v < nv; ++v) {
    const double mag = sqrt(vnx[v] * vnx[v] + vny[v] * vny[v] + vnz[v] * vnz[v]);
    vnx[v] = vnx[v] / mag; vny[v] = vny[v] / mag; vnz[v] = vnz[v] / mag;
  }
}

static fg_status upload_body(DevBody &B) {
  std::vector<double> en, vn;
  host_normals(B, en, vn);
  std::vector<double> soa(3 * (size_t)B.nvert);
  for (int v = 0; v < B.nvert; ++v) {
    soa[v] = B.xyz[3 * v]; soa[B.nvert + v] = B.xyz[3 * v + 1]; soa[2 * B.nvert + v] = B.xyz[3 * v + 2];
  }
  if (!B.d_xyz) {
    FG_CUDA(fg::dev_alloc(&B.d_xyz, soa.size() * sizeof(double)));
    FG_CUDA(fg::dev_alloc(&B.d_en, en.size() * sizeof(double)));
    FG_CUDA(fg::dev_alloc(&B.d_vn, vn.size() * sizeof(double)));
  }
  FG_CUDA(cudaMemcpy(B.d_xyz, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice));
  FG_CUDA(cudaMemcpy(B.d_en, en.data(), en.size() * sizeof(double), cudaMemcpyHostToDevice));
  FG_CUDA(cudaMemcpy(B.d_vn, vn.data(), vn.size() * sizeof(double), cudaMemcpyHostToDevice));
  return FG_OK;
}

static geo::Body dev_body(const DevBody &B) {
  geo::Body b;
  b.nvert = B.nvert; b.ntri = B.ntri; b.type = B.type; b.dim = B.body_dim; b.mt = B.membrane_tkns;
  b.vx = B.d_xyz; b.vy = B.d_xyz + B.nvert; b.vz = B.d_xyz + 2 * B.nvert;
  b.enx = B.d_en; b.eny = B.d_en + B.ntri; b.enz = B.d_en + 2 * B.ntri;
  b.vnx = B.d_vn; b.vny = B.d_vn + B.nvert; b.vnz = B.d_vn + 2 * B.nvert;
  b.tri = B.d_tri; b.v2t_off = B.d_v2t_off; b.v2t = B.d_v2t;
  return b;
}

static fg_status ensure_fields(fg_case *c) {
  Geom &G = *c->geom;
  const size_t n = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  if (!G.d_iblank) {
    FG_CUDA(fg::dev_alloc(&G.d_iblank, n));
    FG_CUDA(fg::dev_alloc(&G.d_ghost, n));
    FG_CUDA(fg::dev_alloc(&G.d_dead, n));
    FG_CUDA(fg::dev_alloc(&G.d_body, n));
    FG_CUDA(fg::dev_alloc(&G.d_band, n));
    FG_CUDA(fg::dev_alloc(&G.d_tmp, 4 * n));  // iblankTemp, smoothing buffers
    FG_CUDA(cudaMemset(G.d_iblank, 0, n));
  }
  return FG_OK;
}

// stream compaction of the cell indices satisfying pred, in linear (k,j,i)
// order, into `out` (grown to the count); the case's grow-only scratch holds
// the temporaries, so a call allocates nothing once the sizes are known.
// One synchronisation (the count).
template <typename Pred>
static fg_status compact(Geom &G, Pred pred, size_t n, DevScratch &out, int *count, cudaStream_t s) {
  size_t tmp = 0;
  thrust::counting_iterator<int> it(0);
  FG_CUDA(cub::DeviceSelect::If(nullptr, tmp, it, (int *)nullptr, (int *)nullptr, (int)n, pred, s));
  FG_CUDA(G.cub_tmp.ensure(tmp));
  FG_CUDA(G.sel_out.ensure(n * sizeof(int)));
  FG_CUDA(G.sel_count.ensure(sizeof(int)));
  FG_CUDA(cub::DeviceSelect::If(G.cub_tmp.p, tmp, it, G.sel_out.as<int>(), G.sel_count.as<int>(), (int)n,
                                pred, s));
  FG_CUDA(cudaMemcpyAsync(count, G.sel_count.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  FG_CUDA(cudaStreamSynchronize(s));
  FG_CUDA(out.ensure((size_t)std::max(1, *count) * sizeof(int)));
  if (*count > 0)
    FG_CUDA(cudaMemcpyAsync(out.p, G.sel_out.p, (size_t)(*count) * sizeof(int), cudaMemcpyDeviceToDevice, s));
  return FG_OK;
}

}  // namespace fg

using namespace fg;

extern "C" {

fg_status fg_case_add_body(fg_case *c, int nvert, int ntri, const double *xyz, const int32_t *tri,
                           int surface_type, double membrane_tkns, int body_dim) {
  if (!c || nvert < 3 || ntri < 1 || !xyz || !tri) return FG_BAD_INPUT;
  if (c->geom->bodies.size() >= 8) return FG_BAD_INPUT;
  for (long long m = 0; m < 3LL * ntri; ++m)
    if (tri[m] < 0 || tri[m] >= nvert) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  DevBody B;
  B.nvert = nvert; B.ntri = ntri; B.type = surface_type; B.body_dim = body_dim;
  B.membrane_tkns = membrane_tkns;
  B.xyz.assign(xyz, xyz + 3 * (size_t)nvert);
  B.tri.assign(tri, tri + 3 * (size_t)ntri);
  // vertex -> triangles in ascending triangle order (the full scan of
  // BOUNDARY_IBLANK_FAST.F90:992-999 visits them in that order)
  std::vector<int32_t> cnt(nvert, 0), off(nvert + 1, 0), v2t;
  for (int m = 0; m < ntri; ++m) {
    int a = tri[3 * m], b = tri[3 * m + 1], d = tri[3 * m + 2];
    cnt[a]++;
    if (b != a) cnt[b]++;
    if (d != a && d != b) cnt[d]++;
  }
  for (int v = 0; v < nvert; ++v) off[v + 1] = off[v] + cnt[v];
  v2t.assign(off[nvert], 0);
  std::fill(cnt.begin(), cnt.end(), 0);
  for (int m = 0; m < ntri; ++m) {
    int a = tri[3 * m], b = tri[3 * m + 1], d = tri[3 * m + 2];
    v2t[off[a] + cnt[a]++] = m;
    if (b != a) v2t[off[b] + cnt[b]++] = m;
    if (d != a && d != b) v2t[off[d] + cnt[d]++] = m;
  }
  FG_CUDA(fg::dev_alloc(&B.d_tri, 3 * (size_t)ntri * sizeof(int32_t)));
  FG_CUDA(cudaMemcpy(B.d_tri, tri, 3 * (size_t)ntri * sizeof(int32_t), cudaMemcpyHostToDevice));
  FG_CUDA(fg::dev_alloc(&B.d_v2t_off, (nvert + 1) * sizeof(int32_t)));
  FG_CUDA(cudaMemcpy(B.d_v2t_off, off.data(), (nvert + 1) * sizeof(int32_t), cudaMemcpyHostToDevice));
  FG_CUDA(fg::dev_alloc(&B.d_v2t, std::max<size_t>(1, v2t.size()) * sizeof(int32_t)));
  FG_CUDA(cudaMemcpy(B.d_v2t, v2t.data(), v2t.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  fg_status st = upload_body(B);
  if (st != FG_OK) return st;
  c->geom->bodies.push_back(B);
  return FG_OK;
}

fg_status fg_case_update_body(fg_case *c, int ibody, const double *xyz) {
  if (!c || !xyz || ibody < 0 || ibody >= (int)c->geom->bodies.size()) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  DevBody &B = c->geom->bodies[ibody];
  B.xyz.assign(xyz, xyz + 3 * (size_t)B.nvert);
  B.host_stale = false;
  return upload_body(B);
}

static geo::Bodies make_bodies(fg_case *c) {
  geo::Bodies BB;
  memset(&BB, 0, sizeof(BB));
  BB.n = (int)c->geom->bodies.size();
  for (int b = 0; b < BB.n; ++b) BB.b[b] = dev_body(c->geom->bodies[b]);
  return BB;
}

fg_status fg_set_iblank_body_fast(fg_case *c, int8_t *iblank) {
  if (!c || c->geom->bodies.empty()) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  Geom &G = *c->geom;
  fg_status st = ensure_fields(c);
  if (st != FG_OK) return st;
  geo::Grid g;
  if ((st = geom_grid(c, g)) != FG_OK) return st;
  const size_t n = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  int8_t *ibt = G.d_tmp;
  FG_CUDA(cudaMemsetAsync(G.d_band, 0, n, s));
  FG_CUDA(cudaMemsetAsync(ibt, 0, n, s));
  FG_CUDA(cudaMemsetAsync(G.d_body, 0, n, s));
  geo::Bodies BB = make_bodies(c);
  for (int b = BB.n - 1; b >= 0; --b)
    geo::k_band<<<(BB.b[b].ntri + 127) / 128, 128, 0, s>>>(g, BB.b[b], G.d_band);
  FG_CUDA(cudaGetLastError());
  // band cells of the interior classification range (j, k in [1, n-1])
  int ncell = 0;
  if ((st = compact(G, geo::IsFlag{G.d_band, 1}, n, G.cells, &ncell, s)) != FG_OK) return st;
  int *d_cells = G.cells.as<int>();
  FG_CUDA(G.flags.ensure(16 * sizeof(int)));
  int *d_warn = G.flags.as<int>();
  FG_CUDA(cudaMemsetAsync(d_warn, 0, sizeof(int), s));
  if (ncell > 0) {
    const int wpb = 4;
    geo::k_classify<<<(ncell + wpb - 1) / wpb, 32 * wpb, 0, s>>>(g, BB, d_cells, ncell, ibt, G.d_body, d_warn);
    FG_CUDA(cudaGetLastError());
  }
  const int nl = (c->ny - 1) * (c->nz - 1);
  geo::k_fill<<<(nl + 127) / 128, 128, 0, s>>>(g, G.d_band, ibt, G.d_body);
  const long long nc = (long long)(c->nx + 1) * (c->ny - 1) * (c->nz - 1);
  geo::k_commit<<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(g, ibt, G.d_iblank);
  FG_CUDA(cudaGetLastError());
  int hw = 0;
  FG_CUDA(cudaMemcpyAsync(&hw, d_warn, sizeof(int), cudaMemcpyDeviceToHost, s));
  FG_CUDA(cudaStreamSynchronize(s));
  G.nWarnSide = hw;
  if (iblank) {
    G.h_stage.resize(std::max(G.h_stage.size(), n));
    FG_CUDA(cudaMemcpyAsync(G.h_stage.data(), G.d_iblank, n, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    fg::host_copy(iblank, G.h_stage.data(), n);
  }
  G.tagged = true;
  return FG_OK;
}

fg_status fg_get_band(const fg_case *c, int8_t *band) {
  if (!c || !band || !c->geom->d_band) return FG_BAD_INPUT;
  const size_t n = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  FG_CUDA(cudaMemcpy(band, c->geom->d_band, n, cudaMemcpyDeviceToHost));
  return FG_OK;
}

// One in-place smoothing pass (mode 0: 3-D, 1: x planes, 2: y planes) as a
// Jacobi fixed-point iteration.  Every dependency chain of the sequential
// pass steps backward along x, y or z, so the iteration is exact after at
// most nx + ny + nz steps.  The first step reads the case's iblank and body
// as both old and cur; later steps alternate between two scratch pairs.
// *identity is set when the first step changes nothing: the pass then maps
// its input to itself and leaves iblank and body untouched.
static fg_status smooth_pass(fg_case *c, const geo::Grid &g, int mode, int *d_changed,
                             bool *identity) {
  Geom &G = *c->geom;
  cudaStream_t s = c->stream;
  const size_t n = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  const int8_t *old = G.d_iblank, *bold = G.d_body;
  int8_t *buf[2] = {G.d_tmp, G.d_tmp + n}, *bbuf[2] = {G.d_tmp + 2 * n, G.d_tmp + 3 * n};
  const long long ni = (long long)(c->nx - 1) * (c->ny - 1) * (c->nz - 1);
  const unsigned blocks = (unsigned)((ni + 255) / 256);
  const int cap = c->nx + c->ny + c->nz + 2;
  // batches of 1, 2, 4 then 8 steps per host check, step q flagging into
  // slot q: most passes reach their fixed point in one or two steps; the
  // fixed point is the first step that changes nothing, and the steps after
  // it change nothing either
  constexpr int SMOOTH_BATCH = 8;
  bool done = false;
  int it = 0, w = 0;  // steps taken; buffer the next step writes
  *identity = false;
  for (int nb_want = 1; it < cap && !done; nb_want = std::min(2 * nb_want, SMOOTH_BATCH)) {
    int h[SMOOTH_BATCH];
    const int nb = std::min(nb_want, cap - it);
    FG_CUDA(cudaMemsetAsync(d_changed, 0, nb * sizeof(int), s));
    for (int q = 0; q < nb; ++q) {
      const bool first = (it + q == 0);
      const int8_t *cur = first ? old : buf[1 - w], *bcur = first ? bold : bbuf[1 - w];
      geo::k_smooth_step<<<blocks, 256, 0, s>>>(g, mode, old, cur, buf[w], bold, bcur, bbuf[w],
                                                d_changed + q);
      w = 1 - w;
    }
    FG_CUDA(cudaGetLastError());
    FG_CUDA(cudaMemcpyAsync(h, d_changed, nb * sizeof(int), cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    if (it == 0 && h[0] == 0) {
      *identity = true;
      return FG_OK;
    }
    it += nb;
    done = (h[nb - 1] == 0);
  }
  if (!done) {
    set_last_error("iblank smoothing did not reach its fixed point", __FILE__, __LINE__);
    return FG_TIMEOUT;
  }
  geo::k_smooth_commit<<<blocks, 256, 0, s>>>(g, buf[1 - w], bbuf[1 - w], G.d_iblank, G.d_body);
  FG_CUDA(cudaGetLastError());
  return FG_OK;
}

}  // extern "C"

namespace {
// device outputs of one row list (ghost or dead): a view of the case's
// grow-only row scratch, sized for m rows
struct RowBufs {
  geo::RowOut o{};
  double *cD = nullptr, *cN = nullptr;
  fg_status bind(RowScratch &r, int m) {
    const size_t mm = (size_t)std::max(1, m), d = sizeof(double);
    FG_CUDA(r.bi.ensure(3 * mm * d)); FG_CUDA(r.bw.ensure(3 * mm * d));
    FG_CUDA(r.ip.ensure(3 * mm * d)); FG_CUDA(r.nrm.ensure(3 * mm * d));
    FG_CUDA(r.probe.ensure(mm * d)); FG_CUDA(r.ds.ensure(mm * d));
    FG_CUDA(r.cell.ensure(3 * mm * sizeof(int))); FG_CUDA(r.closest.ensure(mm * sizeof(int)));
    FG_CUDA(r.cD.ensure(8 * mm * d)); FG_CUDA(r.cN.ensure(8 * mm * d));
    o.bi = r.bi.as<double>(); o.bw = r.bw.as<double>(); o.ip = r.ip.as<double>();
    o.nrm = r.nrm.as<double>(); o.probe = r.probe.as<double>(); o.ds = r.ds.as<double>();
    o.cell = r.cell.as<int>(); o.closest = r.closest.as<int>();
    cD = r.cD.as<double>(); cN = r.cN.as<double>();
    return FG_OK;
  }
};

void list_ijk(const std::vector<int> &l, long long NX, long long NY, std::vector<int32_t> &ijk) {
  ijk.resize(3 * l.size());
  for (size_t r = 0; r < l.size(); ++r) {
    ijk[3 * r] = (int32_t)(l[r] % NX);
    ijk[3 * r + 1] = (int32_t)((l[r] / NX) % NY);
    ijk[3 * r + 2] = (int32_t)(l[r] / (NX * NY));
  }
}

}  // namespace

extern "C" {

fg_status fg_gcm_set_internal_boundary(fg_case *c, int8_t *iblank, int8_t *ghostCellMark,
                                       int8_t *dead_cell, int *nGhost, int *nDead) {
  if (!c || !c->geom->tagged) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  Geom &G = *c->geom;
  geo::Grid g;
  fg_status st = geom_grid(c, g);
  if (st != FG_OK) return st;
  const size_t n = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  FG_CUDA(G.flags.ensure(16 * sizeof(int)));
  int *flagp = G.flags.as<int>();
  // smoothing: 5 x 3-D, 5 x x-planes, 5 x y-planes (GCM_SET_BOUNDARY.F90:115-223, :1618-1697)
  // a pass that maps its input to itself does so again, so the passes of a
  // mode stop at the first one that changes nothing
  for (int mode = 0; mode < 3; ++mode)
    for (int it = 0; it < 5; ++it) {
      bool identity = false;
      if ((st = smooth_pass(c, g, mode, flagp + 4, &identity)) != FG_OK) return st;
      if (identity) break;
    }
  const long long ni = (long long)(c->nx - 1) * (c->ny - 1) * (c->nz - 1);
  FG_CUDA(cudaMemsetAsync(G.d_ghost, 0, n, s));
  geo::k_ghost_mark<<<(unsigned)((ni + 255) / 256), 256, 0, s>>>(g, G.d_iblank, G.d_ghost, G.d_body);
  FG_CUDA(cudaGetLastError());
  geo::k_dead_mark<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, G.d_iblank, G.d_ghost, G.d_dead);
  FG_CUDA(cudaGetLastError());
  int ng = 0, nd = 0;
  if ((st = compact(G, geo::IsFlag{G.d_ghost, 1}, n, G.glist, &ng, s)) != FG_OK) return st;
  geo::IsDeadRow dpred{G.d_dead, c->nx + 2, c->ny + 2, c->nx, c->ny, c->nz};
  if ((st = compact(G, dpred, n, G.dlist, &nd, s)) != FG_OK) return st;
  const int *glp = G.glist.as<int>(), *dlp = G.dlist.as<int>();
  geo::Bodies BB = make_bodies(c);
  RowBufs gb, db;
  if ((st = gb.bind(G.rg, ng)) != FG_OK) return st;
  if ((st = db.bind(G.rd, nd)) != FG_OK) return st;
  FG_CUDA(G.alpha.ensure((size_t)std::max(1, ng) * sizeof(double)));
  double *alpha = G.alpha.as<double>();
  FG_CUDA(cudaMemsetAsync(flagp, 0, 4 * sizeof(int), s));
  const double pln = c->cfg.probe_length, plnD = c->cfg.probe_length_dead;
  if (ng > 0) {
    geo::k_ghost_geom<<<(ng + 3) / 4, 128, 0, s>>>(g, BB, glp, ng, G.d_body, pln, gb.o, flagp);
    geo::k_weights<<<(ng + 63) / 64, 64, 0, s>>>(g, glp, ng, gb.o, 0, gb.cD, gb.cN, flagp + 1);
  }
  if (nd > 0) {
    geo::k_dead_geom<<<(nd + 3) / 4, 128, 0, s>>>(g, BB, dlp, nd, G.d_body, plnD, db.o, flagp,
                                                  flagp + 2);
    geo::k_weights<<<(nd + 63) / 64, 64, 0, s>>>(g, dlp, nd, db.o, 1, db.cD, db.cN, flagp + 1);
  }
  FG_CUDA(cudaGetLastError());
  FG_CUDA(G.rank.ensure(n * sizeof(int)));
  int *rankp = G.rank.as<int>();
  FG_CUDA(cudaMemsetAsync(rankp, 0xff, n * sizeof(int), s));
  if (nd > 0) geo::k_rank<<<(nd + 255) / 256, 256, 0, s>>>(dlp, nd, rankp);
  if (ng > 0) geo::k_alpha<<<(ng + 255) / 256, 256, 0, s>>>(g, glp, ng, G.d_dead, rankp, db.o.ds, alpha);
  FG_CUDA(cudaGetLastError());
  int flags[4] = {0, 0, 0, 0};
  FG_CUDA(cudaMemcpyAsync(flags, flagp, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
  FG_CUDA(cudaStreamSynchronize(s));
  G.nWarnSide += flags[0];
  G.nHostFail = flags[1];
  // host copies of the masks (straight into the case's page-locked copies)
  // and of the rows
  c->iblank.resize(n);
  c->ghost.resize(n);
  c->dead.resize(n);
  FG_CUDA(cudaMemcpyAsync(c->iblank.data(), G.d_iblank, n, cudaMemcpyDeviceToHost, s));
  FG_CUDA(cudaMemcpyAsync(c->ghost.data(), G.d_ghost, n, cudaMemcpyDeviceToHost, s));
  FG_CUDA(cudaMemcpyAsync(c->dead.data(), G.d_dead, n, cudaMemcpyDeviceToHost, s));
  FG_CUDA(cudaStreamSynchronize(s));
  // the row lists and row outputs: one landing area, one synchronisation
  std::vector<int> hgl, hdl;
  std::vector<int32_t> g_ijk, d_ijk, g_cell, d_cell;
  std::vector<double> g_coefN, d_coefN, d_probe, d_ip;
  {
    struct Piece { const void *src; size_t bytes; size_t off; };
    std::vector<Piece> pieces;
    size_t tot = 0;
    auto add = [&](const void *src, size_t bytes) {
      pieces.push_back({src, bytes, tot});
      tot += (bytes + 15) & ~size_t(15);
      return pieces.size() - 1;
    };
    const size_t ngs = (size_t)ng, nds = (size_t)nd, I = sizeof(int32_t), D = sizeof(double);
    const size_t p_gl = add(glp, ngs * I), p_dl = add(dlp, nds * I);
    const size_t p_gcell = add(gb.o.cell, 3 * ngs * I), p_dcell = add(db.o.cell, 3 * nds * I);
    const size_t p_gcN = add(gb.cN, 8 * ngs * D), p_dcN = add(db.cN, 8 * nds * D);
    const size_t p_dprobe = add(db.o.probe, nds * D), p_dip = add(db.o.ip, 3 * nds * D);
    const size_t p_gcD = add(gb.cD, 8 * ngs * D), p_gbi = add(gb.o.bi, 3 * ngs * D);
    const size_t p_gip = add(gb.o.ip, 3 * ngs * D), p_gprobe = add(gb.o.probe, ngs * D);
    const size_t p_alpha = add(alpha, ngs * D), p_gcl = add(gb.o.closest, ngs * I);
    const size_t p_dcD = add(db.cD, 8 * nds * D), p_dbi = add(db.o.bi, 3 * nds * D);
    const size_t p_dcl = add(db.o.closest, nds * I);
    G.h_stage.resize(std::max(G.h_stage.size(), tot));
    char *h = G.h_stage.data();
    for (const Piece &q : pieces)
      if (q.bytes) FG_CUDA(cudaMemcpyAsync(h + q.off, q.src, q.bytes, cudaMemcpyDeviceToHost, s));
    FG_CUDA(cudaStreamSynchronize(s));
    auto take = [&](size_t pi, auto &v, size_t count) {
      using E = typename std::remove_reference<decltype(v)>::type::value_type;
      v.resize(count);
      if (count) memcpy(v.data(), h + pieces[pi].off, count * sizeof(E));
    };
    take(p_gl, hgl, ngs); take(p_dl, hdl, nds);
    take(p_gcell, g_cell, 3 * ngs); take(p_dcell, d_cell, 3 * nds);
    take(p_gcN, g_coefN, 8 * ngs); take(p_dcN, d_coefN, 8 * nds);
    take(p_dprobe, d_probe, nds); take(p_dip, d_ip, 3 * nds);
    take(p_gcD, G.g_coefD, 8 * ngs); take(p_gbi, G.g_bi, 3 * ngs);
    take(p_gip, G.g_ip, 3 * ngs); take(p_gprobe, G.g_probe, ngs);
    take(p_alpha, G.g_alpha, ngs); take(p_gcl, G.g_closest, ngs);
    take(p_dcD, G.d_coefD, 8 * nds); take(p_dbi, G.d_bi, 3 * nds);
    take(p_dcl, G.d_closest, nds);
  }
  list_ijk(hgl, c->nx + 2, c->ny + 2, g_ijk);
  list_ijk(hdl, c->nx + 2, c->ny + 2, d_ijk);
  // hand the rows to the solver (same path as caller-supplied geometry,
  // which also marks the dead rows using the fallback)
  st = fg::geometry_rows(c, ng, g_ijk.data(), g_cell.data(), g_coefN.data(), nd, d_ijk.data(),
                         d_cell.data(), d_coefN.data(), d_probe.data(), d_ip.data());
  if (st != FG_OK) return st;
  if (iblank) fg::host_copy(iblank, c->iblank.data(), n);
  if (ghostCellMark) fg::host_copy(ghostCellMark, c->ghost.data(), n);
  if (dead_cell) fg::host_copy(dead_cell, c->dead.data(), n);
  if (nGhost) *nGhost = ng;
  if (nDead) *nDead = nd;
  G.rows_ng = ng;
  G.rows_nd = nd;
  if (flags[2]) return FG_GEOMETRY_DEAD_NO_BODY;
  if (G.nHostFail) return FG_GEOMETRY_NO_HOST_CELL;
  return FG_OK;
}

fg_status fg_get_ghost_rows(const fg_case *c, int32_t *ijk, int32_t *cell, double *coefN,
                            double *coefD, double *bi, double *ip, double *probe,
                            int32_t *closest, double *alpha) {
  if (!c) return FG_BAD_INPUT;
  const Geom &G = *c->geom;
  const size_t n = (size_t)c->nGhost;
  if (ijk) memcpy(ijk, c->g_ijk.data(), 3 * n * sizeof(int32_t));
  if (cell) memcpy(cell, c->g_cell.data(), 3 * n * sizeof(int32_t));
  if (coefN) memcpy(coefN, c->g_coefN.data(), 8 * n * sizeof(double));
  if (coefD && G.g_coefD.size() >= 8 * n) memcpy(coefD, G.g_coefD.data(), 8 * n * sizeof(double));
  if (bi && G.g_bi.size() >= 3 * n) memcpy(bi, G.g_bi.data(), 3 * n * sizeof(double));
  if (ip && G.g_ip.size() >= 3 * n) memcpy(ip, G.g_ip.data(), 3 * n * sizeof(double));
  if (probe && G.g_probe.size() >= n) memcpy(probe, G.g_probe.data(), n * sizeof(double));
  if (closest && G.g_closest.size() >= n) memcpy(closest, G.g_closest.data(), n * sizeof(int32_t));
  if (alpha && G.g_alpha.size() >= n) memcpy(alpha, G.g_alpha.data(), n * sizeof(double));
  return FG_OK;
}

fg_status fg_get_dead_rows(const fg_case *c, int32_t *ijk, int32_t *cell, double *coefN,
                           double *coefD, double *bi, double *ip, double *probe,
                           int32_t *closest) {
  if (!c) return FG_BAD_INPUT;
  const Geom &G = *c->geom;
  const size_t n = (size_t)c->nDead;
  if (ijk) memcpy(ijk, c->d_ijk.data(), 3 * n * sizeof(int32_t));
  if (cell) memcpy(cell, c->d_cell.data(), 3 * n * sizeof(int32_t));
  if (coefN) memcpy(coefN, c->d_coefN.data(), 8 * n * sizeof(double));
  if (coefD && G.d_coefD.size() >= 8 * n) memcpy(coefD, G.d_coefD.data(), 8 * n * sizeof(double));
  if (bi && G.d_bi.size() >= 3 * n) memcpy(bi, G.d_bi.data(), 3 * n * sizeof(double));
  if (ip && c->d_ipv.size() >= 3 * n) memcpy(ip, c->d_ipv.data(), 3 * n * sizeof(double));
  if (probe && c->d_probe.size() >= n) memcpy(probe, c->d_probe.data(), n * sizeof(double));
  if (closest && G.d_closest.size() >= n) memcpy(closest, G.d_closest.data(), n * sizeof(int32_t));
  return FG_OK;
}

}  // extern "C"


// ===================================================== prescribed body motion
// BOUNDARY_MOVE.F90:3-186 (move_boundary for PRESCRIBED_RIGID bodies) with
// BOUNDARY_MARKER_VEL.F90:5-125 (forced_motion, compute_marker_vel) and
// BOUNDARY_MOVE.F90:151-186 (compute_marker_poisition), on the device.  The
// body's scalars of the step (centroid velocity, angular velocity, the
// length-preserving rotation coefficients) are formed on the host in the
// reference's order; every marker's velocity, position, displacement since
// the last re-tag and dp/dn, and the surface normals
// (BOUNDARY_SET_ARCLENGTH_NORM.F90:2-189), are computed here without fused
// multiply-adds, so the markers are the same doubles as a sequential run.
namespace fg {
namespace mv {

struct Step {
  double vc[3];     // vxcent, vycent, vzcent
  double ta[3];     // the half-sum of the old and new angular velocities
  double cent[3];   // xcent, ycent, zcent before the step
  double co[3][3];  // coefficient of temp_(u,v,w)B in (u,v,w)B, times total_omega applied after
  double tot;       // total_omega
  double dt;
  int with_dpdn;    // ntime > 1
};

// marker velocities (the old ones kept), positions, displacement from the
// re-tag snapshot (max into *dsmax as the bits of a non-negative double)
__global__ void k_markers(int nv, double *x, double *uvw, double *uvw_old, const double *snap, Step st,
                          unsigned long long *dsmax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double *y = x + nv, *z = y + nv;
  const double xi = x[i], yi = y[i], zi = z[i];
  const double tu = (st.ta[1] * (zi - st.cent[2]) - st.ta[2] * (yi - st.cent[1]));
  const double tv = -(st.ta[0] * (zi - st.cent[2]) - st.ta[2] * (xi - st.cent[0]));
  const double tw = (st.ta[0] * (yi - st.cent[1]) - st.ta[1] * (xi - st.cent[0]));
  double b[3];
  for (int r = 0; r < 3; ++r)
    b[r] = st.vc[r] + st.tot * (tu * st.co[r][0] + tv * st.co[r][1] + tw * st.co[r][2]);
  for (int r = 0; r < 3; ++r) {
    uvw_old[r * nv + i] = uvw[r * nv + i];
    uvw[r * nv + i] = b[r];
  }
  const double nx = xi + st.dt * b[0], ny = yi + st.dt * b[1], nz = zi + st.dt * b[2];
  x[i] = nx; y[i] = ny; z[i] = nz;
  const double dx = nx - snap[i], dy = ny - snap[nv + i], dz = nz - snap[2 * nv + i];
  const double ds = sqrt(dx * dx + dy * dy + dz * dz);
  atomicMax(dsmax, (unsigned long long)__double_as_longlong(ds));
}

// element unit normals (v2-v1) x (v3-v2) / |.| (host_normals' arithmetic)
__global__ void k_elem_normals(int nt, int nv, const double *x, const int32_t *tri, double *en) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nt) return;
  const double *y = x + nv, *z = y + nv;
  const int n1 = tri[3 * m], n2 = tri[3 * m + 1], n3 = tri[3 * m + 2];
  const double ax = x[n2] - x[n1], ay = y[n2] - y[n1], az = z[n2] - z[n1];
  const double bx = x[n3] - x[n2], by = y[n3] - y[n2], bz = z[n3] - z[n2];
  const double nxv = (ay * bz - az * by);
  const double nyv = (az * bx - ax * bz);
  const double nzv = (ax * by - ay * bx);
  const double mag = sqrt(nxv * nxv + nyv * nyv + nzv * nzv);
  en[m] = nxv / mag; en[nt + m] = nyv / mag; en[2 * nt + m] = nzv / mag;
}

// vertex unit normals: the incident element normals summed in ascending
// element order (once per occurrence of the vertex in the element, as the
// sequential loop does), normalised; then dp/dn at the marker
// (BOUNDARY_MOVE.F90:96-110: -D u_n / Dt, 0 on the first step)
__global__ void k_vert_normals(int nt, int nv, const int32_t *tri, const int32_t *off, const int32_t *v2t,
                               const double *en, double *vn, const double *uvw, const double *uvw_old, double dt,
                               int with_dpdn, double *dpdn) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int q = off[v]; q < off[v + 1]; ++q) {
    const int m = v2t[q];
    const int mult = (tri[3 * m] == v) + (tri[3 * m + 1] == v) + (tri[3 * m + 2] == v);
    for (int r = 0; r < mult; ++r) { sx = sx + en[m]; sy = sy + en[nt + m]; sz = sz + en[2 * nt + m]; }
  }
  const double mag = sqrt(sx * sx + sy * sy + sz * sz);
  const double nx = sx / mag, ny = sy / mag, nz = sz / mag;
  vn[v] = nx; vn[nv + v] = ny; vn[2 * nv + v] = nz;
  if (dpdn) {
    double d = 0.0;
    if (with_dpdn)
      d = -((uvw[v] - uvw_old[v]) / dt * nx + (uvw[nv + v] - uvw_old[nv + v]) / dt * ny +
            (uvw[2 * nv + v] - uvw_old[2 * nv + v]) / dt * nz);
    dpdn[v] = d;
  }
}

}  // namespace mv
}  // namespace fg

namespace {

fg_status ensure_motion(DevBody &B, cudaStream_t s) {
  if (B.d_uvw) return FG_OK;
  const size_t n3 = 3 * (size_t)B.nvert * sizeof(double);
  FG_CUDA(fg::dev_alloc(&B.d_uvw, n3));
  FG_CUDA(fg::dev_alloc(&B.d_uvw_old, n3));
  FG_CUDA(fg::dev_alloc(&B.d_snap, n3));
  FG_CUDA(fg::dev_alloc(&B.d_dpdn, (size_t)B.nvert * sizeof(double)));
  FG_CUDA(cudaMemsetAsync(B.d_uvw, 0, n3, s));
  FG_CUDA(cudaMemsetAsync(B.d_uvw_old, 0, n3, s));
  FG_CUDA(cudaMemcpyAsync(B.d_snap, B.d_xyz, n3, cudaMemcpyDeviceToDevice, s));
  FG_CUDA(cudaMemsetAsync(B.d_dpdn, 0, (size_t)B.nvert * sizeof(double), s));
  return FG_OK;
}

// the host copy of the vertices from the device (after device moves)
fg_status sync_host_body(DevBody &B, cudaStream_t s) {
  if (!B.host_stale) return FG_OK;
  std::vector<double> soa(3 * (size_t)B.nvert);
  FG_CUDA(cudaMemcpyAsync(soa.data(), B.d_xyz, soa.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  FG_CUDA(cudaStreamSynchronize(s));
  for (int v = 0; v < B.nvert; ++v) {
    B.xyz[3 * v] = soa[v]; B.xyz[3 * v + 1] = soa[B.nvert + v]; B.xyz[3 * v + 2] = soa[2 * B.nvert + v];
  }
  B.host_stale = false;
  return FG_OK;
}

}  // namespace

extern "C" {

fg_status fg_move_body(fg_case *c, int ibody, fg_rigid_motion *m, int ntime, double time, double dt,
                       double *ds_max, int *iblank_reset) {
  if (!c || !m || ibody < 0 || ibody >= (int)c->geom->bodies.size() || !(dt > 0.0)) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  DevBody &B = c->geom->bodies[ibody];
  fg_status st = ensure_motion(B, s);
  if (st != FG_OK) return st;
  // forced_motion (BOUNDARY_MARKER_VEL.F90:5-33)
  const double PI = 3.14159265358979323846;
  double vc[3], av[3];
  for (int a = 0; a < 3; ++a) {
    vc[a] = m->vcent_trans[a] + m->amp[a] * sin(2.0 * PI * m->freq[a] * time);
    av[a] = m->angv_init[a] + m->ampang[a] * sin(2.0 * PI * m->freqang[a] * time + m->angphase[a]);
  }
  // compute_marker_vel's scalars (BOUNDARY_MARKER_VEL.F90:60-125)
  mv::Step S{};
  for (int a = 0; a < 3; ++a) {
    S.vc[a] = vc[a];
    S.ta[a] = 0.5 * (m->angv_old[a] + av[a]);
    S.cent[a] = m->cent[a];
  }
  const double ax = av[0], ay = av[1], az = av[2];
  S.tot = 1.0 / (1.0 + 0.25 * (dt * dt) * (ax * ax + ay * ay + az * az));
  const double q = 0.25 * (dt * dt), h = 0.5 * dt;
  S.co[0][0] = 1.0 + q * (ax * ax);  S.co[0][1] = -h * az - q * ax * ay;  S.co[0][2] = -h * ay + q * ax * az;
  S.co[1][0] = h * az - q * ax * ay; S.co[1][1] = 1.0 + q * (ay * ay);   S.co[1][2] = -h * ax - q * ay * az;
  S.co[2][0] = h * ay + q * ax * az; S.co[2][1] = h * ax - q * ay * az;  S.co[2][2] = 1.0 + q * (az * az);
  S.dt = dt;
  S.with_dpdn = ntime > 1 ? 1 : 0;
  unsigned long long *d_ds = nullptr;
  FG_CUDA(fg::dev_alloc(&d_ds, sizeof(unsigned long long)));
  cudaError_t e = cudaMemsetAsync(d_ds, 0, sizeof(unsigned long long), s);
  const int nv = B.nvert, nt = B.ntri;
  if (e == cudaSuccess) {
    mv::k_markers<<<(nv + 255) / 256, 256, 0, s>>>(nv, B.d_xyz, B.d_uvw, B.d_uvw_old, B.d_snap, S, d_ds);
    mv::k_elem_normals<<<(nt + 255) / 256, 256, 0, s>>>(nt, nv, B.d_xyz, B.d_tri, B.d_en);
    mv::k_vert_normals<<<(nv + 255) / 256, 256, 0, s>>>(nt, nv, B.d_tri, B.d_v2t_off, B.d_v2t, B.d_en, B.d_vn,
                                                        B.d_uvw, B.d_uvw_old, dt, S.with_dpdn, B.d_dpdn);
    note_launches(3);
    e = cudaGetLastError();
  }
  unsigned long long bits = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, d_ds, sizeof(bits), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  fg::dev_free(d_ds);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return FG_CUDA_ERROR;
  }
  B.host_stale = true;
  // compute_marker_poisition's centroid, and the state the next step reads
  for (int a = 0; a < 3; ++a) {
    m->cent[a] = m->cent[a] + dt * vc[a];
    m->angv_old[a] = av[a];
  }
  // the re-tag policy (BOUNDARY_MOVE.F90:122-145): a marker moved more than
  // 0.05 of the smallest cell width since the last snapshot
  double ds;
  memcpy(&ds, &bits, sizeof(ds));
  double hmin = 1e300;
  const HLevel &L = c->lev[0];
  for (const std::vector<double> *xv : {&L.x, &L.y, &L.z})
    for (size_t i = 1; i + 2 < xv->size(); ++i) hmin = std::min(hmin, (*xv)[i + 1] - (*xv)[i]);
  const int reset = ds > 0.05 * hmin ? 1 : 0;
  if (reset) FG_CUDA(cudaMemcpyAsync(B.d_snap, B.d_xyz, 3 * (size_t)nv * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (ds_max) *ds_max = ds;
  if (iblank_reset) *iblank_reset = reset;
  return FG_OK;
}

fg_status fg_get_body_markers(fg_case *c, int ibody, double *xyz, double *uvw, double *dpdn) {
  if (!c || ibody < 0 || ibody >= (int)c->geom->bodies.size()) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  DevBody &B = c->geom->bodies[ibody];
  const int nv = B.nvert;
  if (xyz) {
    fg_status st = sync_host_body(B, c->stream);
    if (st != FG_OK) return st;
    memcpy(xyz, B.xyz.data(), 3 * (size_t)nv * sizeof(double));
  }
  if ((uvw || dpdn) && !B.d_uvw) {
    if (uvw) memset(uvw, 0, 3 * (size_t)nv * sizeof(double));
    if (dpdn) memset(dpdn, 0, (size_t)nv * sizeof(double));
    return FG_OK;
  }
  std::vector<double> soa(3 * (size_t)nv);
  if (uvw) {
    FG_CUDA(cudaMemcpyAsync(soa.data(), B.d_uvw, soa.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FG_CUDA(cudaStreamSynchronize(c->stream));
    for (int v = 0; v < nv; ++v) {
      uvw[3 * v] = soa[v]; uvw[3 * v + 1] = soa[nv + v]; uvw[3 * v + 2] = soa[2 * nv + v];
    }
  }
  if (dpdn) {
    FG_CUDA(cudaMemcpyAsync(dpdn, B.d_dpdn, (size_t)nv * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FG_CUDA(cudaStreamSynchronize(c->stream));
  }
  return FG_OK;
}

}  // extern "C"

// ------------------------------------------------ body-intercept values
// and the velocity ghost cells (GCM_BODYINTERCEPT_VALUES.F90,
// GCM_GHOSTCELL_UPDATE.F90:1-359), on the rows of the last device tagging
namespace fg {
namespace bi {

struct BodyVel {
  int n;
  const double *u[8], *uo[8];  // marker velocities (SoA, nvert each), this and the previous step; may be null
};

// LAPACK getrf/getri semantics on a 4x4 column-major matrix (partial
// pivoting on the largest |a|, first index on ties; inverse of U, then
// inv(A) L = inv(U), column interchanges)
__device__ void invert4(double *a) {
  int ipiv[4];
#define A(i, j) a[(i) + 4 * (j)]
  for (int j = 0; j < 4; ++j) {
    int p = j;
    double mx = fabs(A(j, j));
    for (int i = j + 1; i < 4; ++i)
      if (fabs(A(i, j)) > mx) { mx = fabs(A(i, j)); p = i; }
    ipiv[j] = p;
    if (A(p, j) == 0.0) continue;
    if (p != j)
      for (int q = 0; q < 4; ++q) { const double t = A(j, q); A(j, q) = A(p, q); A(p, q) = t; }
    const double r = 1.0 / A(j, j);
    for (int i = j + 1; i < 4; ++i) A(i, j) = A(i, j) * r;
    for (int q = j + 1; q < 4; ++q)
      for (int i = j + 1; i < 4; ++i) A(i, q) = A(i, q) - A(i, j) * A(j, q);
  }
  double t4[4];
  for (int j = 0; j < 4; ++j) {
    A(j, j) = 1.0 / A(j, j);
    const double ajj = -A(j, j);
    for (int i = 0; i < j; ++i) {
      double s = 0.0;
      for (int q = i; q < j; ++q) s = s + A(i, q) * A(q, j);
      t4[i] = s;
    }
    for (int i = 0; i < j; ++i) A(i, j) = t4[i] * ajj;
  }
  double work[4];
  for (int j = 3; j >= 0; --j) {
    for (int i = j + 1; i < 4; ++i) { work[i] = A(i, j); A(i, j) = 0.0; }
    for (int q = j + 1; q < 4; ++q)
      for (int i = 0; i < 4; ++i) A(i, j) = A(i, j) - A(i, q) * work[q];
  }
  for (int j = 2; j >= 0; --j) {
    const int jp = ipiv[j];
    if (jp != j)
      for (int i = 0; i < 4; ++i) { const double t = A(i, j); A(i, j) = A(i, jp); A(i, jp) = t; }
  }
#undef A
}

// one thread per row: the intercept velocity of this and the previous
// step (GCM_calc_BIVelocity_Unstruc, :198-388) and dp/dn (:80-95, :141-156)
__global__ void k_bi_values(int n, const int *list, const double *bi, const double *nrm, const int *closest,
                            const int8_t *body, geo::Bodies BB, BodyVel V, int ntime, double dt, double *ubi,
                            double *dpdn) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int ib = body[list[r]] - 1, e = closest[r];
  double u[3] = {0.0, 0.0, 0.0}, uo[3] = {0.0, 0.0, 0.0};
  if (ib >= 0 && ib < BB.n && e >= 0) {
    const geo::Body &B = BB.b[ib];
    const int n1 = B.tri[3 * e], n2 = B.tri[3 * e + 1], n3 = B.tri[3 * e + 2];
    const int nd[3] = {n1, n2, n3};
    double a[16];
    for (int q = 0; q < 3; ++q) {
      a[q] = B.vx[nd[q]]; a[q + 4] = B.vy[nd[q]]; a[q + 8] = B.vz[nd[q]]; a[q + 12] = 1.0;
    }
    a[3] = B.enx[e]; a[7] = B.eny[e]; a[11] = B.enz[e]; a[15] = 0.0;
    invert4(a);
    const double xB = bi[3 * r], yB = bi[3 * r + 1], zB = bi[3 * r + 2];
    for (int q = 0; q < 6; ++q) {
      const double *src = q < 3 ? V.u[ib] : V.uo[ib];
      const int comp = q % 3;
      double rhs[4] = {0.0, 0.0, 0.0, 0.0};
      if (src) {
        const double *sc = src + (size_t)comp * B.nvert;
        rhs[0] = sc[n1]; rhs[1] = sc[n2]; rhs[2] = sc[n3];
      }
      double cX = 0.0, cY = 0.0, cZ = 0.0, cC = 0.0;
      for (int i = 0; i < 4; ++i) {
        cX = cX + a[0 + 4 * i] * rhs[i];
        cY = cY + a[1 + 4 * i] * rhs[i];
        cZ = cZ + a[2 + 4 * i] * rhs[i];
        cC = cC + a[3 + 4 * i] * rhs[i];
      }
      const double v = cX * xB + cY * yB + cZ * zB + cC;
      if (q < 3) u[comp] = v; else uo[comp] = v;
    }
  }
  if (ubi) { ubi[3 * r] = u[0]; ubi[3 * r + 1] = u[1]; ubi[3 * r + 2] = u[2]; }
  if (dpdn) {
    double d = 0.0;
    if (ntime > 1) {
      d = (u[0] - uo[0]) / dt * nrm[3 * r] + (u[1] - uo[1]) / dt * nrm[3 * r + 1] + (u[2] - uo[2]) / dt * nrm[3 * r + 2];
      d = -d;
    }
    dpdn[r] = d;
  }
}

__constant__ int c_incI[8] = {0, 0, 1, 1, 0, 0, 1, 1};  // GCM_MEMORY_ALLOCATE.F90:593-623
__constant__ int c_incJ[8] = {0, 1, 1, 0, 0, 1, 1, 0};
__constant__ int c_incK[8] = {0, 0, 0, 0, 1, 1, 1, 1};

struct VelRows {
  int nd, ng;
  const int *dlist, *glist;     // cell ids
  const int *dcell, *gcell;     // host cells (3 per row)
  const double *dip;            // dead image points (3 per row)
  const double *dcD, *gcD;      // Dirichlet weights (8 per row)
  const double *alpha;          // ghost blending factors
  const double *ubi_d, *ubi_g;  // intercept velocities (3 per row)
};

// one Jacobi step of the velocity ghost and dead cells: new values of
// every row from the current fields into nv (3 per row; dead rows first)
__global__ void k_vel_rows(geo::Grid g, VelRows R, const int8_t *iblank, const int8_t *dead, double bw, double iw,
                           const double *u, const double *v, const double *w, double *nv, int *skip) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R.nd + R.ng) return;
  const double *fld[3] = {u, v, w};
  const bool isdead = r < R.nd;
  const int q = isdead ? r : r - R.nd;
  const long long id = isdead ? R.dlist[q] : R.glist[q];
  const int i = (int)(id % g.NX), j = (int)((id / g.NX) % g.NY), k = (int)(id / (g.NX * g.NY));
  const int *cell = isdead ? R.dcell + 3 * q : R.gcell + 3 * q;
  double out[3];
  if (cell[0] < 0 || (isdead && (j < 1 || j > g.ny - 1 || k < 1 || k > g.nz - 1))) {
    skip[r] = 1;  // rows the reference leaves out keep their value
    for (int c = 0; c < 3; ++c) nv[3 * r + c] = fld[c][id];
    return;
  }
  skip[r] = 0;
  if (isdead) {
    const double xIP = R.dip[3 * q], yIP = R.dip[3 * q + 1], zIP = R.dip[3 * q + 2];
    double ip[3] = {0.0, 0.0, 0.0}, inv[3] = {0.0, 0.0, 0.0}, dint = 0.0;
    int sumk = 0;
    bool solid = false;
    for (int t = 0; t < 8; ++t) {
      const int ii = cell[0] + c_incI[t], jj = cell[1] + c_incJ[t], kk = cell[2] + c_incK[t];
      const long long q2 = ii + g.NX * (jj + g.NY * (long long)kk);
      if (iblank[q2] == 1 && dead[q2] == 0) solid = true;
      if (ii == i && jj == j && kk == k) continue;
      const double dist = (g.xc[ii] - xIP) * (g.xc[ii] - xIP) + (g.yc[jj] - yIP) * (g.yc[jj] - yIP) +
                          (g.zc[kk] - zIP) * (g.zc[kk] - zIP);
      if (iblank[q2] == 0 || dead[q2] == -1) {
        sumk++;
        dint = dint + (1.0 / dist);
        for (int c = 0; c < 3; ++c) inv[c] = inv[c] + (1.0 / dist) * fld[c][q2];
      }
    }
    const bool fallback = solid && !(dint < 0.000001 || sumk == 1);
    if (fallback) {
      for (int c = 0; c < 3; ++c) ip[c] = inv[c] / dint;
    } else {
      for (int t = 0; t < 8; ++t) {
        const int ii = cell[0] + c_incI[t], jj = cell[1] + c_incJ[t], kk = cell[2] + c_incK[t];
        const long long q2 = ii + g.NX * (jj + g.NY * (long long)kk);
        const bool own = ii == i && jj == j && kk == k;
        for (int c = 0; c < 3; ++c)
          ip[c] = ip[c] + R.dcD[8 * q + t] * (own ? R.ubi_d[3 * q + c] : fld[c][q2]);
      }
    }
    for (int c = 0; c < 3; ++c) out[c] = R.ubi_d[3 * q + c] * bw - ip[c] * iw;
  } else {
    double gg[3] = {0.0, 0.0, 0.0};
    for (int t = 0; t < 8; ++t) {
      const int ii = cell[0] + c_incI[t], jj = cell[1] + c_incJ[t], kk = cell[2] + c_incK[t];
      const long long q2 = ii + g.NX * (jj + g.NY * (long long)kk);
      const bool own = ii == i && jj == j && kk == k;
      for (int c = 0; c < 3; ++c) gg[c] = gg[c] + R.gcD[8 * q + t] * (own ? R.ubi_g[3 * q + c] : fld[c][q2]);
    }
    const double flag = R.alpha[q];
    for (int c = 0; c < 3; ++c) out[c] = (1.0 - flag) * gg[c] + flag * gg[c];
  }
  for (int c = 0; c < 3; ++c) nv[3 * r + c] = out[c];
}

// the new values into the fields and the largest |du|+|dv|+|dw| (as the
// bits of a non-negative double, which order like the values)
__global__ void k_vel_scatter(VelRows R, long long NX, long long NY, const double *nv, const int *skip, double *u,
                              double *v, double *w, unsigned long long *res) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R.nd + R.ng || skip[r]) return;
  const long long id = r < R.nd ? R.dlist[r] : R.glist[r - R.nd];
  const double d = fabs(nv[3 * r] - u[id]) + fabs(nv[3 * r + 1] - v[id]) + fabs(nv[3 * r + 2] - w[id]);
  u[id] = nv[3 * r];
  v[id] = nv[3 * r + 1];
  w[id] = nv[3 * r + 2];
  atomicMax(res, (unsigned long long)__double_as_longlong(d));
  (void)NX; (void)NY;
}

}  // namespace bi
}  // namespace fg

namespace {

fg_status bi_rows_ready(fg_case *c) {
  const Geom &G = *c->geom;
  if (G.rows_ng < 0 || G.rows_nd < 0 || G.rows_ng != c->nGhost || G.rows_nd != c->nDead) return FG_BAD_INPUT;
  return FG_OK;
}

}  // namespace

extern "C" {

fg_status fg_body_intercept_values_device(fg_case *c, int ntime, double dt, double *ubi_ghost, double *ubi_dead,
                                          double *dpdn_ghost, double *dpdn_dead) {
  if (!c || !(dt > 0.0)) return FG_BAD_INPUT;
  fg_status st = bi_rows_ready(c);
  if (st != FG_OK) return st;
  cudaSetDevice(c->device);
  Geom &G = *c->geom;
  cudaStream_t s = c->stream;
  geo::Bodies BB = make_bodies(c);
  bi::BodyVel V{};
  V.n = BB.n;
  for (int b = 0; b < BB.n && b < 8; ++b) {
    V.u[b] = G.bodies[b].d_uvw;
    V.uo[b] = G.bodies[b].d_uvw_old;
  }
  const int ng = G.rows_ng, nd = G.rows_nd;
  if (ng > 0)
    bi::k_bi_values<<<(ng + 127) / 128, 128, 0, s>>>(ng, G.glist.as<int>(), G.rg.bi.as<double>(), G.rg.nrm.as<double>(),
                                                     G.rg.closest.as<int>(), G.d_body, BB, V, ntime, dt, ubi_ghost,
                                                     dpdn_ghost);
  if (nd > 0)
    bi::k_bi_values<<<(nd + 127) / 128, 128, 0, s>>>(nd, G.dlist.as<int>(), G.rd.bi.as<double>(), G.rd.nrm.as<double>(),
                                                     G.rd.closest.as<int>(), G.d_body, BB, V, ntime, dt, ubi_dead,
                                                     dpdn_dead);
  note_launches((ng > 0) + (nd > 0));
  FG_CUDA(cudaGetLastError());
  FG_CUDA(cudaStreamSynchronize(s));
  return FG_OK;
}

fg_status fg_ghostcell_velocity_device(fg_case *c, double *u, double *v, double *w, const double *ubi_ghost,
                                       const double *ubi_dead, int itermax_gc, double restol_gcv, int *iterations) {
  if (!c || !u || !v || !w || itermax_gc < 0) return FG_BAD_INPUT;
  fg_status st = bi_rows_ready(c);
  if (st != FG_OK) return st;
  Geom &G = *c->geom;
  const int ng = G.rows_ng, nd = G.rows_nd;
  if ((ng > 0 && !ubi_ghost) || (nd > 0 && !ubi_dead)) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  geo::Grid g;
  if ((st = geom_grid(c, g)) != FG_OK) return st;
  bi::VelRows R{};
  R.nd = nd; R.ng = ng;
  R.dlist = G.dlist.as<int>(); R.glist = G.glist.as<int>();
  R.dcell = G.rd.cell.as<int>(); R.gcell = G.rg.cell.as<int>();
  R.dip = G.rd.ip.as<double>();
  R.dcD = G.rd.cD.as<double>(); R.gcD = G.rg.cD.as<double>();
  R.alpha = G.alpha.as<double>();
  R.ubi_d = ubi_dead; R.ubi_g = ubi_ghost;
  const double pld = c->cfg.probe_length_dead;
  const double bw = pld / (pld - 1.0), iw = 1.0 / (pld - 1.0);
  const int nr = nd + ng;
  int it = 0;
  double res = 1.0e10;
  if (nr > 0) {
    double *nv = nullptr;
    int *skip = nullptr;
    unsigned long long *d_res = nullptr;
    FG_CUDA(fg::dev_alloc(&nv, 3 * (size_t)nr * sizeof(double)));
    cudaError_t e = fg::dev_alloc(&skip, (size_t)nr * sizeof(int));
    if (e == cudaSuccess) e = fg::dev_alloc(&d_res, sizeof(unsigned long long));
    // GCM_GHOSTCELL_UPDATE.F90:73: iterate while iterGC < itermax_gc and
    // the last sweep changed some row by more than restol_gcv
    while (e == cudaSuccess && it < itermax_gc && res > restol_gcv) {
      e = cudaMemsetAsync(d_res, 0, sizeof(unsigned long long), s);
      if (e != cudaSuccess) break;
      bi::k_vel_rows<<<(nr + 127) / 128, 128, 0, s>>>(g, R, G.d_iblank, G.d_dead, bw, iw, u, v, w, nv, skip);
      bi::k_vel_scatter<<<(nr + 127) / 128, 128, 0, s>>>(R, g.NX, g.NY, nv, skip, u, v, w, d_res);
      note_launches(2);
      unsigned long long bits = 0;
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, d_res, sizeof(bits), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      memcpy(&res, &bits, sizeof(res));
      ++it;
    }
    fg::dev_free(nv);
    fg::dev_free(skip);
    fg::dev_free(d_res);
    if (e != cudaSuccess) {
      set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
      return FG_CUDA_ERROR;
    }
  }
  if (iterations) *iterations = it;
  return (nr > 0 && it == itermax_gc && res > restol_gcv) ? FG_NOT_CONVERGED : FG_OK;
}

}  // extern "C"

// fg_ad.cu -- the momentum equation's line SOR on device fields:
// set_solve_ad's diffusion coefficients (CORE_SET_SOLVERS.F90:591-677),
// one pass of itsolv_ad (CORE_SOLVE_AD.F90:131-776: x, then y, then z line
// sweeps with the implicit convection terms) and calc_residual_ad
// (:780-964), the outer velocity boundaries (CORE_SET_OUTER_BC.F90
// set_outer_velocity_bc, set_outer_ghost_velocity) and the solve_ad
// iteration around them (CORE_SOLVE_AD.F90:11-127).  Fields are device
// arrays in the reference layout (0:nx+1, 0:ny+1, 0:nz+1), node counts.
//
// The reference sweeps the lines of each direction in lexicographic order,
// Gauss-Seidel style: an x line (j,k) reads the new values of lines (j-1,k)
// and (j,k-1) and the old values of (j+1,k) and (j,k+1).  Lines on one
// anti-diagonal j + k = d read only lines of d-1 (new) and d+1 (old), so
// one launch per anti-diagonal, in increasing d, solves every line of it at
// once and reproduces the lexicographic sweep exactly (y lines: i + k, z
// lines: i + j).  Each thread solves one line by the reference's Thomas
// recursion with the coefficients formed row by row in the reference's
// operation order; this file is compiled without FMA contraction, so the
// result is bit-identical to the sequential sweep.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "fg_case.h"
#include "fg_internal.h"

namespace fg {
namespace ad {

struct Met {
  const double *x, *y, *z, *xc, *yc, *zc, *dxi, *dyi, *dzi;
  const double *amx, *apx, *amy, *apy, *amz, *apz;  // set_solve_ad
};

struct Dims {
  int nx, ny, nz;
  long long NX, NY;
  __device__ __forceinline__ long long id(int i, int j, int k) const { return i + NX * (j + NY * (long long)k); }
};

struct Coef {
  double amx, apx, acx, amy, apy, acy, amz, apz, acz;
};

__device__ __forceinline__ double fint(const double *x, const double *xc, int i) {
  return (x[i] - xc[i - 1]) / (xc[i] - xc[i - 1]);
}

// the coefficients of cell (i,j,k) as every sweep and the residual form
// them (CORE_SOLVE_AD.F90:215-330): diffusion, then the implicit
// convection of each direction, central for 25 <= i <= 375 (the
// reference's switch is on i for all three directions), first-order
// upwind elsewhere
__device__ void cell(const Dims &d, const Met &m, const double *fu, const double *fv, const double *fw,
                     double half_dt, int i, int j, int k, Coef &q) {
  const long long id = d.id(i, j, k);
  const long long ip = id + 1, jp = id + d.NX, kp = id + d.NX * d.NY;
  const bool central = (i >= 25) && (i <= 375);
  double hyb1, hyb2, tmp1, tmp2;
  q.amx = m.amx[i]; q.apx = m.apx[i]; q.acx = -(q.amx + q.apx);
  q.amy = m.amy[j]; q.apy = m.apy[j]; q.acy = -(q.amy + q.apy);
  q.amz = m.amz[k]; q.apz = m.apz[k]; q.acz = -(q.amz + q.apz);
  const double fu0 = fu[id], fu1 = fu[ip], fv0 = fv[id], fv1 = fv[jp], fw0 = fw[id], fw1 = fw[kp];
  hyb1 = 0.5 * (1.0 + copysign(1.0, fu0)); hyb2 = 0.5 * (1.0 - copysign(1.0, fu1));
  tmp1 = 1.0 - fint(m.x, m.xc, i); tmp2 = fint(m.x, m.xc, i + 1);
  if (central) {
    q.amx = q.amx - half_dt * fu0 * tmp1 * m.dxi[i];
    q.apx = q.apx + half_dt * fu1 * tmp2 * m.dxi[i];
  } else {
    q.amx = q.amx - half_dt * hyb1 * fu0 * m.dxi[i];
    q.apx = q.apx + half_dt * hyb2 * fu1 * m.dxi[i];
  }
  hyb1 = 0.5 * (1.0 - copysign(1.0, fu0)); hyb2 = 0.5 * (1.0 + copysign(1.0, fu1));
  tmp1 = fint(m.x, m.xc, i); tmp2 = 1.0 - fint(m.x, m.xc, i + 1);
  if (central) q.acx = q.acx + half_dt * (fu1 * tmp2 - fu0 * tmp1) * m.dxi[i];
  else q.acx = q.acx + half_dt * (fu1 * hyb2 - fu0 * hyb1) * m.dxi[i];

  hyb1 = 0.5 * (1.0 + copysign(1.0, fv0)); hyb2 = 0.5 * (1.0 - copysign(1.0, fv1));
  tmp1 = 1.0 - fint(m.y, m.yc, j); tmp2 = fint(m.y, m.yc, j + 1);
  if (central) {
    q.amy = q.amy - half_dt * fv0 * tmp1 * m.dyi[j];
    q.apy = q.apy + half_dt * fv1 * tmp2 * m.dyi[j];
  } else {
    q.amy = q.amy - half_dt * hyb1 * fv0 * m.dyi[j];
    q.apy = q.apy + half_dt * hyb2 * fv1 * m.dyi[j];
  }
  hyb1 = 0.5 * (1.0 - copysign(1.0, fv0)); hyb2 = 0.5 * (1.0 + copysign(1.0, fv1));
  tmp1 = fint(m.y, m.yc, j); tmp2 = 1.0 - fint(m.y, m.yc, j + 1);
  if (central) q.acy = q.acy + half_dt * (fv1 * tmp2 - fv0 * tmp1) * m.dyi[j];
  else q.acy = q.acy + half_dt * (fv1 * hyb2 - fv0 * hyb1) * m.dyi[j];

  hyb1 = 0.5 * (1.0 + copysign(1.0, fw0)); hyb2 = 0.5 * (1.0 - copysign(1.0, fw1));
  tmp1 = 1.0 - fint(m.z, m.zc, k); tmp2 = fint(m.z, m.zc, k + 1);
  if (central) {
    q.amz = q.amz - half_dt * fw0 * tmp1 * m.dzi[k];
    q.apz = q.apz + half_dt * fw1 * tmp2 * m.dzi[k];
  } else {
    q.amz = q.amz - half_dt * hyb1 * fw0 * m.dzi[k];
    q.apz = q.apz + half_dt * hyb2 * fw1 * m.dzi[k];
  }
  hyb1 = 0.5 * (1.0 - copysign(1.0, fw0)); hyb2 = 0.5 * (1.0 + copysign(1.0, fw1));
  tmp1 = fint(m.z, m.zc, k); tmp2 = 1.0 - fint(m.z, m.zc, k + 1);
  if (central) q.acz = q.acz + half_dt * (fw1 * tmp2 - fw0 * tmp1) * m.dzi[k];
  else q.acz = q.acz + half_dt * (fw1 * hyb2 - fw0 * hyb1) * m.dzi[k];
}

// the lines of anti-diagonal `diag` along AXIS (0: x lines (j,k), j + k =
// diag; 1: y lines (i,k); 2: z lines (i,j)); one thread per line, gam and
// the forward values in the thread's slot of `scr` (2 (n+1) doubles)
template <int AXIS>
__global__ void k_ad_diag(Dims d, Met m, const int8_t *ib, const int8_t *gh, double *var, const double *r,
                          const double *fu, const double *fv, const double *fw, double half_dt, double omega,
                          int diag, double *scr) {
  // the two transverse indices a (first) and b (second) of the line
  const int amax = AXIS == 0 ? d.ny - 1 : d.nx - 1;
  const int bmax = AXIS == 2 ? d.ny - 1 : d.nz - 1;
  const int a0 = max(1, diag - bmax), a1 = min(amax, diag - 1);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = a0 + t;
  if (a > a1) return;
  const int b = diag - a;
  const int n = AXIS == 0 ? d.nx : AXIS == 1 ? d.ny : d.nz;  // rows 0..n, unknowns 1..n-1
  double *g = scr + (size_t)t * 2 * (n + 1), *u = g + (n + 1);
  auto at = [&](int s) -> long long {
    return AXIS == 0 ? d.id(s, a, b) : AXIS == 1 ? d.id(a, s, b) : d.id(a, b, s);
  };
  // row 0: the trivial equation u = var (diagonal 1)
  double binv = 1.0 / 1.0;
  u[0] = var[at(0)] * binv;
  double c_prev = 0.0;
  for (int s = 1; s <= n; ++s) {
    double am, ac, ap, rh;
    const long long id = at(s);
    if (s == n) {
      am = 0.0; ap = 0.0; ac = 1.0; rh = var[id];
    } else {
      const int i = AXIS == 0 ? s : a;
      const int j = AXIS == 1 ? s : AXIS == 0 ? a : b;
      const int k = AXIS == 2 ? s : b;
      Coef q;
      cell(d, m, fu, fv, fw, half_dt, i, j, k, q);
      double lo, hi;  // the line's own couplings
      if (AXIS == 0) {
        rh = r[id] - (var[id - d.NX] * q.amy + var[id + d.NX] * q.apy + var[id - d.NX * d.NY] * q.amz +
                      var[id + d.NX * d.NY] * q.apz);
        lo = q.amx; hi = q.apx;
      } else if (AXIS == 1) {
        rh = r[id] - (var[id - 1] * q.amx + var[id + 1] * q.apx + var[id - d.NX * d.NY] * q.amz +
                      var[id + d.NX * d.NY] * q.apz);
        lo = q.amy; hi = q.apy;
      } else {
        rh = r[id] - (var[id - 1] * q.amx + var[id + 1] * q.apx + var[id - d.NX] * q.amy + var[id + d.NX] * q.apy);
        lo = q.amz; hi = q.apz;
      }
      const double rib = (1.0 - (double)ib[id]) * (1.0 - (double)abs((int)gh[id]));
      am = lo * rib;
      ap = hi * rib;
      ac = 1.0 + (q.acx + q.acy + q.acz) * rib;
      rh = rh * rib + var[id] * (1.0 - rib);
    }
    // CORE_TDMA.F90:22-27
    const double gam = c_prev * binv;
    binv = 1.0 / (ac - am * gam);
    u[s] = (rh - am * u[s - 1]) * binv;
    g[s] = gam;
    c_prev = ap;
  }
  for (int s = n - 1; s >= 0; --s) u[s] = u[s] - g[s + 1] * u[s + 1];
  for (int s = 1; s <= n - 1; ++s) {
    const long long id = at(s);
    var[id] = var[id] + omega * (u[s] - var[id]);
  }
}

// calc_residual_ad: per block the largest |res| and the first cell (in the
// reference's k, j, i loop order) that has it
__global__ void __launch_bounds__(256)
k_ad_resid(Dims d, Met m, const int8_t *ib, const int8_t *gh, const double *var, const double *r, const double *fu,
           const double *fv, const double *fw, double half_dt, double *pval, long long *pidx) {
  const long long ni = d.nx - 1, nj = d.ny - 1, nt = ni * nj * (d.nz - 1);
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double v = -1.0;
  long long at = e;
  if (e < nt) {
    const int i = 1 + (int)(e % ni), j = 1 + (int)((e / ni) % nj), k = 1 + (int)(e / (ni * nj));
    const long long id = d.id(i, j, k), sz = d.NX * d.NY;
    Coef q;
    cell(d, m, fu, fv, fw, half_dt, i, j, k, q);
    double res = r[id] - var[id] * (1.0 + q.acx + q.acy + q.acz) - var[id - 1] * q.amx - var[id + 1] * q.apx -
                 var[id - d.NX] * q.amy - var[id + d.NX] * q.apy - var[id - sz] * q.amz - var[id + sz] * q.apz;
    res = res * (1.0 - (double)ib[id]) * (1.0 - (double)gh[id]);
    v = fabs(res);
  }
  // larger value wins; equal values: the earlier cell
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_down_sync(0xffffffffu, v, o);
    const long long oa = __shfl_down_sync(0xffffffffu, at, o);
    if (ov > v || (ov == v && oa < at)) { v = ov; at = oa; }
  }
  __shared__ double sv[8];
  __shared__ long long sa[8];
  if ((threadIdx.x & 31) == 0) { sv[threadIdx.x >> 5] = v; sa[threadIdx.x >> 5] = at; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w)
      if (sv[w] > v || (sv[w] == v && sa[w] < at)) { v = sv[w]; at = sa[w]; }
    pval[blockIdx.x] = v;
    pidx[blockIdx.x] = at;
  }
}

// ---- outer velocity boundaries (CORE_SET_OUTER_BC.F90:18-509, :739-823)
// Face order f: x1, x2, y1, y2, z1, z2.  puls holds the pulsatile values
// val * sin(2 pi freq t) (x1's u: val t / 30), formed on the host with the
// host's libm as the reference.
struct VelBC {
  int type[6];
  double val[6][3], puls[6][3];
  double yOrigin, yout, zOrigin, zout;
};
struct BCArr {
  double *a[9];  // bcxu, bcxv, bcxw, bcyu, bcyv, bcyw, bczu, bczv, bczw
};
struct Vel {
  const double *f[3];
};

// the user-specified channel profile val 6 (s - lo)(hi - s) / (hi - lo)^2
__device__ __forceinline__ double channel(double val, double s, double lo, double hi) {
  const double e = hi - lo;
  return val * 6.0 * (s - lo) * (hi - s) / (e * e);
}

// x faces: one thread per (side, j, k), j = 0..ny+1, k = 0..nz+1
__global__ void k_outer_bc_x(Dims d, VelBC p, const double *y, Vel U, BCArr B) {
  const long long n = d.NY * (long long)(d.nz + 2), e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2 * n) return;
  const int side = (int)(e / n), j = (int)((e % n) % d.NY), k = (int)((e % n) / d.NY);
  const int i = side ? d.nx - 1 : 1, io = side ? 1 : d.nx - 1;
  const long long b = side + 2 * (j + d.NY * (long long)k), id = d.id(i, j, k), ido = d.id(io, j, k);
  const double *val = p.val[side];
  switch (p.type[side]) {
    case 1: for (int a = 0; a < 3; ++a) B.a[a][b] = val[a]; break;
    case 2: for (int a = 0; a < 3; ++a) B.a[a][b] = U.f[a][id]; break;
    case 3: for (int a = 0; a < 3; ++a) B.a[a][b] = p.puls[side][a]; break;
    case 4: B.a[0][b] = 0.0; B.a[1][b] = U.f[1][id]; B.a[2][b] = U.f[2][id]; break;
    case 5: for (int a = 0; a < 3; ++a) B.a[a][b] = 0.5 * (U.f[a][id] + U.f[a][ido]); break;
    case 6:
      B.a[0][b] = channel(val[0], y[j], p.yOrigin, p.yout);
      if (side) { B.a[1][b] = val[1]; B.a[2][b] = val[2]; }
      break;
  }
}

// y faces: one thread per (side, i, k), i = 0..nx, k = 0..nz+1; the
// user-specified profile goes into the x2 arrays at (1, j, k), written by
// the i = 0 thread alone (the reference writes the same value for each i)
__global__ void k_outer_bc_y(Dims d, VelBC p, const double *z, Vel U, BCArr B) {
  const long long ni = d.nx + 1, n = ni * (d.nz + 2), e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2 * n) return;
  const int side = (int)(e / n), i = (int)((e % n) % ni), k = (int)((e % n) / ni), f = 2 + side;
  const int j = side ? d.ny - 1 : 1, jo = side ? 1 : d.ny - 1;
  const long long b = i + d.NX * (side + 2 * (long long)k), id = d.id(i, j, k), ido = d.id(i, jo, k);
  const double *val = p.val[f];
  switch (p.type[f]) {
    case 1: for (int a = 0; a < 3; ++a) B.a[3 + a][b] = val[a]; break;
    case 2: for (int a = 0; a < 3; ++a) B.a[3 + a][b] = U.f[a][id]; break;
    case 3: for (int a = 0; a < 3; ++a) B.a[3 + a][b] = p.puls[f][a]; break;
    case 4: B.a[3][b] = U.f[0][id]; B.a[4][b] = 0.0; B.a[5][b] = U.f[2][id]; break;
    case 5: for (int a = 0; a < 3; ++a) B.a[3 + a][b] = 0.5 * (U.f[a][id] + U.f[a][ido]); break;
    case 6:
      if (i == 0) {
        const long long bx = 1 + 2 * (j + d.NY * (long long)k);
        B.a[0][bx] = val[0];
        B.a[1][bx] = channel(val[1], z[k], p.zOrigin, p.zout);
        B.a[2][bx] = val[2];
      }
      break;
  }
}

// z faces: one thread per (side, i, j), i = 0..nx, j = 0..ny+1
__global__ void k_outer_bc_z(Dims d, VelBC p, const double *y, Vel U, BCArr B) {
  const long long ni = d.nx + 1, n = ni * d.NY, e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2 * n) return;
  const int side = (int)(e / n), i = (int)((e % n) % ni), j = (int)((e % n) / ni), f = 4 + side;
  const int k = side ? d.nz - 1 : 1, ko = side ? 1 : d.nz - 1;
  const long long b = i + d.NX * (j + d.NY * (long long)side), id = d.id(i, j, k), ido = d.id(i, j, ko);
  const double *val = p.val[f];
  switch (p.type[f]) {
    case 1: for (int a = 0; a < 3; ++a) B.a[6 + a][b] = val[a]; break;
    case 2: for (int a = 0; a < 3; ++a) B.a[6 + a][b] = U.f[a][id]; break;
    case 3: for (int a = 0; a < 3; ++a) B.a[6 + a][b] = p.puls[f][a]; break;
    case 4: B.a[6][b] = U.f[0][id]; B.a[7][b] = U.f[1][id]; B.a[8][b] = 0.0; break;
    case 5: for (int a = 0; a < 3; ++a) B.a[6 + a][b] = 0.5 * (U.f[a][id] + U.f[a][ido]); break;
    case 6:
      if (i == 0) {
        const long long bx = 1 + 2 * (j + d.NY * (long long)k);
        B.a[0][bx] = val[0];
        B.a[1][bx] = val[1];
        B.a[2][bx] = channel(val[2], y[j], p.yOrigin, p.yout);
      }
      break;
  }
}

// the outer ghost layer of one axis: u(ghost) = 2 bc - u(first interior);
// x over (j, k) of 0..ny+1 x 0..nz+1, y over (i, k) of 0..nx x 0..nz+1,
// z over (i, j) of 0..nx x 0..ny+1
template <int AXIS>
__global__ void k_outer_ghost(Dims d, double *u, double *v, double *w, BCArr B) {
  const long long n1 = AXIS == 0 ? d.NY : d.nx + 1, n2 = AXIS == 2 ? d.NY : d.nz + 2;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n1 * n2) return;
  const int p = (int)(e % n1), q = (int)(e / n1);
  double *F[3] = {u, v, w};
  long long g0, g1, i0, i1, b0, b1;
  if (AXIS == 0) {
    g0 = d.id(0, p, q); i0 = d.id(1, p, q); g1 = d.id(d.nx, p, q); i1 = d.id(d.nx - 1, p, q);
    b0 = 2 * (p + d.NY * (long long)q); b1 = b0 + 1;
  } else if (AXIS == 1) {
    g0 = d.id(p, 0, q); i0 = d.id(p, 1, q); g1 = d.id(p, d.ny, q); i1 = d.id(p, d.ny - 1, q);
    b0 = p + d.NX * (2 * (long long)q); b1 = b0 + d.NX;
  } else {
    g0 = d.id(p, q, 0); i0 = d.id(p, q, 1); g1 = d.id(p, q, d.nz); i1 = d.id(p, q, d.nz - 1);
    b0 = p + d.NX * (long long)q; b1 = b0 + d.NX * d.NY;
  }
  for (int a = 0; a < 3; ++a) {
    const double *bc = B.a[3 * AXIS + a];
    F[a][g0] = 2.0 * bc[b0] - F[a][i0];
    F[a][g1] = 2.0 * bc[b1] - F[a][i1];
  }
}

}  // namespace ad
}  // namespace fg

using namespace fg;

namespace {

// set_solve_ad on the host (CORE_SET_SOLVERS.F90:650-675) and the metric
// arrays, uploaded into the case's buffer
fg_status ad_setup(fg_case *c, const fg_ad_params *prm, ad::Met &m, ad::Dims &d) {
  if (!c->prepared) {
    fg_status st = fg_mg_prepare(c);
    if (st != FG_OK) return st;
  }
  const HLevel &L = c->lev[0];
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  std::vector<double> amx(nx + 2, 0.0), apx(nx + 2, 0.0), amy(ny + 2, 0.0), apy(ny + 2, 0.0), amz(nz + 2, 0.0),
      apz(nz + 2, 0.0);
  const double nu = prm->reinv, dt = prm->dt;
  for (int i = 1; i <= nx - 1; ++i) {
    amx[i] = (L.dxcinv[i]) * L.dxinv[i];
    apx[i] = (L.dxcinv[i + 1]) * L.dxinv[i];
    amx[i] = -(0.50 * dt * nu) * amx[i];
    apx[i] = -(0.50 * dt * nu) * apx[i];
  }
  for (int j = 1; j <= ny - 1; ++j) {
    amy[j] = L.dycinv[j] * L.dyinv[j];
    apy[j] = L.dycinv[j + 1] * L.dyinv[j];
    amy[j] = -(0.50 * dt * nu) * amy[j];
    apy[j] = -(0.50 * dt * nu) * apy[j];
  }
  for (int k = 1; k <= nz - 1; ++k) {
    amz[k] = L.dzcinv[k] * L.dzinv[k];
    apz[k] = L.dzcinv[k + 1] * L.dzinv[k];
    amz[k] = -(0.50 * dt * nu) * amz[k];
    apz[k] = -(0.50 * dt * nu) * apz[k];
  }
  std::vector<double> v;
  const std::vector<double> *parts[] = {&L.x,     &L.y, &L.z,   &L.xc, &L.yc, &L.zc, &L.dxinv, &L.dyinv,
                                        &L.dzinv, &amx, &apx,   &amy,  &apy,  &amz,  &apz};
  for (const std::vector<double> *a : parts) v.insert(v.end(), a->begin(), a->end());
  if (!c->d_admet) FG_CUDA(fg::dev_alloc(&c->d_admet, v.size() * sizeof(double)));
  FG_CUDA(cudaMemcpyAsync(c->d_admet, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FG_CUDA(cudaStreamSynchronize(c->stream));  // v is pageable and goes out of scope
  const size_t NX = (size_t)nx + 2, NY = (size_t)ny + 2, NZ = (size_t)nz + 2;
  const double *p = c->d_admet;
  m.x = p; m.y = m.x + NX; m.z = m.y + NY;
  m.xc = m.z + NZ; m.yc = m.xc + NX; m.zc = m.yc + NY;
  m.dxi = m.zc + NZ; m.dyi = m.dxi + NX; m.dzi = m.dyi + NY;
  m.amx = m.dzi + NZ; m.apx = m.amx + NX; m.amy = m.apx + NX; m.apy = m.amy + NY; m.amz = m.apy + NY;
  m.apz = m.amz + NZ;
  d.nx = nx; d.ny = ny; d.nz = nz;
  d.NX = (long long)NX; d.NY = (long long)NY;
  return FG_OK;
}

bool ad_params_ok(const fg_ad_params *p) {
  return p && p->dt > 0.0 && std::isfinite(p->reinv) && std::isfinite(p->omega_ad);
}

bool bc_arrays_ok(const fg_velocity_bc_arrays *b) {
  return b && b->bcxu && b->bcxv && b->bcxw && b->bcyu && b->bcyv && b->bcyw && b->bczu && b->bczv && b->bczw;
}

ad::BCArr bc_arr(const fg_velocity_bc_arrays *b) {
  ad::BCArr B;
  double *const src[9] = {b->bcxu, b->bcxv, b->bcxw, b->bcyu, b->bcyv, b->bcyw, b->bczu, b->bczv, b->bczw};
  for (int q = 0; q < 9; ++q) B.a[q] = src[q];
  return B;
}

// the grid dimensions alone (the boundary kernels need no coefficients)
fg_status dims_setup(fg_case *c, ad::Dims &d) {
  if (!c->prepared) {
    fg_status st = fg_mg_prepare(c);
    if (st != FG_OK) return st;
  }
  d.nx = c->nx; d.ny = c->ny; d.nz = c->nz;
  d.NX = (long long)c->nx + 2; d.NY = (long long)c->ny + 2;
  return FG_OK;
}

unsigned blocks_of(long long n) { return (unsigned)((n + 255) / 256); }

// set_outer_velocity_bc's face data; the pulsatile values with the host's
// sin, pi = 4 atan(1) (CORE_SET_OUTER_BC.F90:40-42)
bool vel_bc(const fg_velocity_bc *vb, ad::VelBC &p) {
  const double pi = 4.0 * std::atan(1.0), t = vb->time;
  for (int f = 0; f < 6; ++f) {
    if (vb->type[f] < 1 || vb->type[f] > 6) return false;
    p.type[f] = vb->type[f];
    for (int a = 0; a < 3; ++a) {
      p.val[f][a] = vb->val[f][a];
      p.puls[f][a] = vb->val[f][a] * std::sin(2.0 * pi * vb->freq[f][a] * t);
    }
  }
  p.puls[0][0] = vb->val[0][0] * t / 30.0;
  p.yOrigin = vb->yOrigin; p.yout = vb->yout; p.zOrigin = vb->zOrigin; p.zout = vb->zout;
  return true;
}

// the three face kernels of set_outer_velocity_bc, in the reference's order
fg_status enqueue_outer_bc(fg_case *c, const ad::Dims &d, const double *u, const double *v, const double *w,
                           const fg_velocity_bc_arrays *bc, const fg_velocity_bc *vb) {
  ad::VelBC p;
  if (!vel_bc(vb, p)) return FG_BAD_INPUT;
  const HLevel &L = c->lev[0];
  if (!c->d_vbcmet) {
    std::vector<double> yz(L.y);
    yz.insert(yz.end(), L.z.begin(), L.z.end());
    FG_CUDA(fg::dev_alloc(&c->d_vbcmet, yz.size() * sizeof(double)));
    FG_CUDA(cudaMemcpy(c->d_vbcmet, yz.data(), yz.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  const double *y = c->d_vbcmet, *z = c->d_vbcmet + d.NY;
  const ad::Vel U = {{u, v, w}};
  const ad::BCArr B = bc_arr(bc);
  cudaStream_t s = c->stream;
  ad::k_outer_bc_x<<<blocks_of(2 * d.NY * (d.nz + 2)), 256, 0, s>>>(d, p, y, U, B);
  ad::k_outer_bc_y<<<blocks_of(2 * (long long)(d.nx + 1) * (d.nz + 2)), 256, 0, s>>>(d, p, z, U, B);
  ad::k_outer_bc_z<<<blocks_of(2 * (long long)(d.nx + 1) * d.NY), 256, 0, s>>>(d, p, y, U, B);
  note_launches(3);
  FG_CUDA(cudaGetLastError());
  return FG_OK;
}

fg_status enqueue_outer_ghost(fg_case *c, const ad::Dims &d, double *u, double *v, double *w,
                              const fg_velocity_bc_arrays *bc) {
  const ad::BCArr B = bc_arr(bc);
  cudaStream_t s = c->stream;
  ad::k_outer_ghost<0><<<blocks_of(d.NY * (d.nz + 2)), 256, 0, s>>>(d, u, v, w, B);
  ad::k_outer_ghost<1><<<blocks_of((long long)(d.nx + 1) * (d.nz + 2)), 256, 0, s>>>(d, u, v, w, B);
  ad::k_outer_ghost<2><<<blocks_of((long long)(d.nx + 1) * d.NY), 256, 0, s>>>(d, u, v, w, B);
  note_launches(3);
  FG_CUDA(cudaGetLastError());
  return FG_OK;
}

}  // namespace

extern "C" {

fg_status fg_itsolv_ad_device(fg_case *c, double *var, const double *r, const double *face_u, const double *face_v,
                              const double *face_w, const fg_ad_params *prm) {
  if (!c || !var || !r || !face_u || !face_v || !face_w || !ad_params_ok(prm)) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  ad::Met m;
  ad::Dims d;
  fg_status st = ad_setup(c, prm, m, d);
  if (st != FG_OK) return st;
  const size_t nref = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  const int8_t *ib = c->d_refmask, *gh = c->d_refmask + nref;
  const double half_dt = prm->crank_nicolson ? 0.5 * prm->dt : 0.0;
  // scratch: the longest anti-diagonal of any direction times the longest line
  const int nmax = std::max(c->nx, std::max(c->ny, c->nz));
  const int lmax = std::max(std::min(c->ny, c->nz), std::max(std::min(c->nx, c->nz), std::min(c->nx, c->ny)));
  double *scr = nullptr;
  FG_CUDA(fg::dev_alloc(&scr, (size_t)lmax * 2 * (nmax + 1) * sizeof(double)));
  cudaStream_t s = c->stream;
  cudaError_t e = cudaSuccess;
  long long launches = 0;
  for (int axis = 0; axis < 3 && e == cudaSuccess; ++axis) {
    const int amax = axis == 0 ? c->ny - 1 : c->nx - 1;
    const int bmax = axis == 2 ? c->ny - 1 : c->nz - 1;
    for (int diag = 2; diag <= amax + bmax && e == cudaSuccess; ++diag) {
      const int nl = std::min(amax, diag - 1) - std::max(1, diag - bmax) + 1;
      if (nl <= 0) continue;
      const unsigned nb = (unsigned)((nl + 63) / 64);
      if (axis == 0)
        ad::k_ad_diag<0><<<nb, 64, 0, s>>>(d, m, ib, gh, var, r, face_u, face_v, face_w, half_dt, prm->omega_ad, diag,
                                           scr);
      else if (axis == 1)
        ad::k_ad_diag<1><<<nb, 64, 0, s>>>(d, m, ib, gh, var, r, face_u, face_v, face_w, half_dt, prm->omega_ad, diag,
                                           scr);
      else
        ad::k_ad_diag<2><<<nb, 64, 0, s>>>(d, m, ib, gh, var, r, face_u, face_v, face_w, half_dt, prm->omega_ad, diag,
                                           scr);
      ++launches;
      e = cudaGetLastError();
    }
  }
  note_launches(launches);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  fg::dev_free(scr);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return FG_CUDA_ERROR;
  }
  return FG_OK;
}

fg_status fg_calc_residual_ad_device(fg_case *c, const double *var, const double *r, const double *face_u,
                                     const double *face_v, const double *face_w, const fg_ad_params *prm,
                                     double *resm, int *loc) {
  if (!c || !var || !r || !face_u || !face_v || !face_w || !ad_params_ok(prm) || !resm) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  ad::Met m;
  ad::Dims d;
  fg_status st = ad_setup(c, prm, m, d);
  if (st != FG_OK) return st;
  const size_t nref = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  const int8_t *ib = c->d_refmask, *gh = c->d_refmask + nref;
  const double half_dt = prm->crank_nicolson ? 0.5 * prm->dt : 0.0;
  const long long nt = (long long)(c->nx - 1) * (c->ny - 1) * (c->nz - 1);
  const unsigned nb = (unsigned)((nt + 255) / 256);
  double *pv = nullptr;
  long long *pi = nullptr;
  FG_CUDA(fg::dev_alloc(&pv, (size_t)nb * sizeof(double)));
  cudaError_t e = fg::dev_alloc(&pi, (size_t)nb * sizeof(long long));
  std::vector<double> hv(nb);
  std::vector<long long> hi(nb);
  if (e == cudaSuccess) {
    ad::k_ad_resid<<<nb, 256, 0, c->stream>>>(d, m, ib, gh, var, r, face_u, face_v, face_w, half_dt, pv, pi);
    note_launches(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(hv.data(), pv, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hi.data(), pi, nb * sizeof(long long), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  fg::dev_free(pv);
  fg::dev_free(pi);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return FG_CUDA_ERROR;
  }
  // the reference starts from resm = 0 and keeps the first cell whose |res|
  // exceeds the running maximum
  double v = 0.0;
  long long at = 0;
  for (unsigned q = 0; q < nb; ++q)
    if (hv[q] > v || (hv[q] == v && hv[q] > 0.0 && hi[q] < at)) { v = hv[q]; at = hi[q]; }
  *resm = v;
  if (loc) {
    const long long ni = c->nx - 1, nj = c->ny - 1;
    loc[0] = v > 0.0 ? 1 + (int)(at % ni) : 1;
    loc[1] = v > 0.0 ? 1 + (int)((at / ni) % nj) : 1;
    loc[2] = v > 0.0 ? 1 + (int)(at / (ni * nj)) : 1;
  }
  return FG_OK;
}

fg_status fg_set_outer_velocity_bc_device(fg_case *c, const double *u, const double *v, const double *w,
                                          const fg_velocity_bc_arrays *bc, const fg_velocity_bc *vb) {
  if (!c || !u || !v || !w || !bc_arrays_ok(bc) || !vb) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  ad::Dims d;
  fg_status st = dims_setup(c, d);
  if (st == FG_OK) st = enqueue_outer_bc(c, d, u, v, w, bc, vb);
  if (st != FG_OK) return st;
  FG_CUDA(cudaStreamSynchronize(c->stream));
  return FG_OK;
}

fg_status fg_set_outer_ghost_velocity_device(fg_case *c, double *u, double *v, double *w,
                                             const fg_velocity_bc_arrays *bc) {
  if (!c || !u || !v || !w || !bc_arrays_ok(bc)) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  ad::Dims d;
  fg_status st = dims_setup(c, d);
  if (st == FG_OK) st = enqueue_outer_ghost(c, d, u, v, w, bc);
  if (st != FG_OK) return st;
  FG_CUDA(cudaStreamSynchronize(c->stream));
  return FG_OK;
}

fg_status fg_solve_ad_device(fg_case *c, double *u, double *v, double *w, const double *nlu, const double *nlv,
                             const double *nlw, double *face_u, double *face_v, double *face_w,
                             const fg_velocity_bc_arrays *bc, const double *ubi_ghost, const double *ubi_dead,
                             const fg_ad_params *prm, const fg_velocity_bc *vb, int itermax_gc, double restol_gcv,
                             int itermax_ad, double restol_ad, fg_solve_ad_stats *stats) {
  if (!c || !u || !v || !w || !nlu || !nlv || !nlw || !face_u || !face_v || !face_w || !bc_arrays_ok(bc) ||
      !ad_params_ok(prm) || !vb || itermax_ad < 0)
    return FG_BAD_INPUT;
  ad::VelBC chk;
  if (!vel_bc(vb, chk)) return FG_BAD_INPUT;
  int vzg[6];
  for (int f = 0; f < 6; ++f) vzg[f] = vb->type[f] == 2;
  int iter = 0, loc[3] = {1, 1, 1};
  double res2 = 1.0e10;
  fg_status st = FG_OK;
  while (st == FG_OK && iter < itermax_ad && res2 > restol_ad) {
    st = fg_itsolv_ad_device(c, u, nlu, face_u, face_v, face_w, prm);
    if (st == FG_OK) st = fg_itsolv_ad_device(c, v, nlv, face_u, face_v, face_w, prm);
    if (st == FG_OK) st = fg_itsolv_ad_device(c, w, nlw, face_u, face_v, face_w, prm);
    if (st == FG_OK) st = fg_ghostcell_velocity_device(c, u, v, w, ubi_ghost, ubi_dead, itermax_gc, restol_gcv, nullptr);
    if (st == FG_OK) st = fg_face_vel_device(c, u, v, w, bc->bcxu, bc->bcyv, bc->bczw, face_u, face_v, face_w);
    if (st == FG_OK)
      st = fg_enforce_global_mass_consv_device(c, face_u, face_v, face_w, bc->bcxu, bc->bcyv, bc->bczw, vzg);
    if (st == FG_OK) st = fg_set_outer_velocity_bc_device(c, u, v, w, bc, vb);
    if (st == FG_OK) st = fg_set_outer_ghost_velocity_device(c, u, v, w, bc);
    double r[3] = {0.0, 0.0, 0.0};
    int l[3][3];
    const double *var[3] = {u, v, w}, *rhs[3] = {nlu, nlv, nlw};
    for (int a = 0; a < 3 && st == FG_OK; ++a)
      st = fg_calc_residual_ad_device(c, var[a], rhs[a], face_u, face_v, face_w, prm, &r[a], l[a]);
    if (st != FG_OK) break;
    int best = 0;
    res2 = std::fabs(r[0]);
    for (int a = 1; a < 3; ++a)
      if (std::fabs(r[a]) > res2) { res2 = std::fabs(r[a]); best = a; }
    std::memcpy(loc, l[best], sizeof(loc));
    ++iter;
  }
  if (stats) {
    stats->iterations = iter;
    stats->residual = res2;
    std::memcpy(stats->loc, loc, sizeof(loc));
  }
  return st;
}

}  // extern "C"

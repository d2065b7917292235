// fg_proj.cu -- the steps either side of the pressure solve on the device:
// face velocities (CORE_FRAC_STEP_ROUTINES.F90 face_vel), global mass
// conservation on zero-gradient outflow faces and the Poisson right-hand
// side (CORE_SET_OUTER_BC.F90 enforce_global_mass_consv, CORE_POISSON.F90
// rhs_poisson), and the velocity correction with the pressure gradient
// (CORE_FRAC_STEP_ROUTINES.F90 correct_vel, calc_pres_grad).  Fields are
// device arrays in the reference layout (0:nx+1, 0:ny+1, 0:nz+1), node
// counts; the face-velocity boundary arrays are the reference's bcxu(0:1,
// 0:ny+1, 0:nz+1), bcyv(0:nx+1, 0:1, 0:nz+1), bczw(0:nx+1, 0:ny+1, 0:1).
// With these, a time step's div and pPrime stay on the device from the
// face velocities to the corrected velocity.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "fg_case.h"
#include "fg_internal.h"

namespace fg {
namespace proj {

// the reference's 1-D grid arrays of the finest level, reference indexing
// (n+2 entries each): nodes, cell centres, widths and their inverses
struct Met {
  const double *x, *y, *z, *xc, *yc, *zc, *dx, *dy, *dz, *dxi, *dyi, *dzi;
};

struct Dims {
  int nx, ny, nz;  // node counts
  long long NX, NY;
  __device__ __forceinline__ long long id(int i, int j, int k) const { return i + NX * (j + NY * (long long)k); }
};

// CORE_GRID.F90:194-202: face interpolation factor of node i
__device__ __forceinline__ double fint(const double *x, const double *xc, int i) {
  return (x[i] - xc[i - 1]) / (xc[i] - xc[i - 1]);
}

// interior cells (1..n-1 per axis) of e, false past the last
__device__ __forceinline__ bool interior(const Dims &d, long long e, int &i, int &j, int &k) {
  const long long ni = d.nx - 1, nj = d.ny - 1;
  if (e >= ni * nj * (d.nz - 1)) return false;
  i = 1 + (int)(e % ni);
  j = 1 + (int)((e / ni) % nj);
  k = 1 + (int)(e / (ni * nj));
  return true;
}

// face_vel: face_u(i) for i = 2..nx-1 from the cell velocities, i = 1 and
// nx from bcxu (faces v, w alike); one thread per interior cell, which
// writes its own faces and, on the last cell of a line, the far boundary
__global__ void k_face_vel(Dims d, Met m, const double *u, const double *v, const double *w, const double *bcxu,
                           const double *bcyv, const double *bczw, double *fu, double *fv, double *fw) {
  int i, j, k;
  if (!interior(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const long long id = d.id(i, j, k);
  if (i >= 2) {
    const double f = fint(m.x, m.xc, i);
    fu[id] = f * u[id] + (1.0 - f) * u[id - 1];
  } else {
    fu[id] = bcxu[0 + 2 * (j + d.NY * (long long)k)];
  }
  if (i == d.nx - 1) fu[d.id(d.nx, j, k)] = bcxu[1 + 2 * (j + d.NY * (long long)k)];
  if (j >= 2) {
    const double f = fint(m.y, m.yc, j);
    fv[id] = f * v[id] + (1.0 - f) * v[id - d.NX];
  } else {
    fv[id] = bcyv[i + d.NX * (0 + 2 * (long long)k)];
  }
  if (j == d.ny - 1) fv[d.id(i, d.ny, k)] = bcyv[i + d.NX * (1 + 2 * (long long)k)];
  if (k >= 2) {
    const double f = fint(m.z, m.zc, k);
    fw[id] = f * w[id] + (1.0 - f) * w[id - d.NX * d.NY];
  } else {
    fw[id] = bczw[i + d.NX * (j + d.NY * 0)];
  }
  if (k == d.nz - 1) fw[d.id(i, j, d.nz)] = bczw[i + d.NX * (j + d.NY * 1)];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// the net mass flux out of the fluid non-ghost cells (block partials)
__global__ void __launch_bounds__(256)
k_massflux(Dims d, Met m, const int8_t *ib, const int8_t *gh, const double *fu, const double *fv, const double *fw,
           double *part) {
  int i, j, k;
  double f = 0.0;
  if (interior(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) {
    const long long id = d.id(i, j, k);
    const double flag = (1.0 - (double)ib[id]) * (1.0 - (double)gh[id]);
    f = flag * ((-fu[id] + fu[id + 1]) * m.dy[j] * m.dz[k] + (-fv[id] + fv[id + d.NX]) * m.dx[i] * m.dz[k] +
                (-fw[id] + fw[id + d.NX * d.NY]) * m.dx[i] * m.dy[j]);
  }
  f = warp_sum(f);
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = f;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < 8; ++q) t += red[q];
    part[blockIdx.x] = t;
  }
}

// one block: the flux summed, the fluid area of the zero-gradient faces,
// the outflow velocity correction -flux/area into *cv
__global__ void __launch_bounds__(1024)
k_massflux_corr(Dims d, Met m, const int8_t *ib, const double *part, int nb, int vzg, double *cv) {
  double flux = 0.0, area = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) flux += part[b];
  for (int f = 0; f < 6; ++f) {
    if (!((vzg >> f) & 1)) continue;
    const int a = f >> 1, up = f & 1;
    const int nu = a == 0 ? d.ny - 1 : d.nx - 1, nv = a == 2 ? d.ny - 1 : d.nz - 1;
    const int layer = a == 0 ? (up ? d.nx - 1 : 1) : a == 1 ? (up ? d.ny - 1 : 1) : (up ? d.nz - 1 : 1);
    for (long long e = threadIdx.x; e < (long long)nu * nv; e += blockDim.x) {
      const int u = 1 + (int)(e % nu), v = 1 + (int)(e / nu);
      long long id;
      double w;
      if (a == 0) { id = d.id(layer, u, v); w = m.dy[u] * m.dz[v]; }
      else if (a == 1) { id = d.id(u, layer, v); w = m.dx[u] * m.dz[v]; }
      else { id = d.id(u, v, layer); w = m.dx[u] * m.dy[v]; }
      area += w * (1.0 - (double)ib[id]);
    }
  }
  __shared__ double rf[32], ra[32];
  flux = warp_sum(flux);
  area = warp_sum(area);
  if ((threadIdx.x & 31) == 0) { rf[threadIdx.x >> 5] = flux; ra[threadIdx.x >> 5] = area; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double F = 0.0, A = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { F += rf[q]; A += ra[q]; }
    *cv = -F / A;
  }
}

// the correction on the zero-gradient faces: the boundary arrays over
// every entry 0..n, the boundary face velocities over the interior
// (lower faces -, upper faces +); blockIdx.y = face
__global__ void k_massflux_apply(Dims d, int vzg, const double *cv, double *bcxu, double *bcyv, double *bczw,
                                 double *fu, double *fv, double *fw) {
  const int f = blockIdx.y;
  if (!((vzg >> f) & 1)) return;
  const int a = f >> 1, up = f & 1;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int u1 = a == 0 ? d.ny : d.nx, v1 = a == 2 ? d.ny : d.nz;  // boundary array indices 0..u1, 0..v1
  if (e >= (long long)(u1 + 1) * (v1 + 1)) return;
  const int u = (int)(e % (u1 + 1)), v = (int)(e / (u1 + 1));
  const double c = up ? *cv : -*cv;
  if (a == 0) bcxu[up + 2 * (u + d.NY * (long long)v)] += c;
  else if (a == 1) bcyv[u + d.NX * (up + 2 * (long long)v)] += c;
  else bczw[u + d.NX * (v + d.NY * (long long)up)] += c;
  const bool in = u >= 1 && v >= 1 && u <= u1 - 1 && v <= v1 - 1;
  if (!in) return;
  if (a == 0) fu[d.id(up ? d.nx : 1, u, v)] += c;
  else if (a == 1) fv[d.id(u, up ? d.ny : 1, v)] += c;
  else fw[d.id(u, v, up ? d.nz : 1)] += c;
}

// rhs_poisson: div on the fluid non-ghost cells (0 elsewhere, also the
// boundary layers: the caller's array is cleared first), block partials of
// the mass flux and of max |div| dt
__global__ void __launch_bounds__(256)
k_div(Dims d, Met m, const int8_t *ib, const int8_t *gh, const double *fu, const double *fv, const double *fw,
      double dtinv, double *div, double *psum, double *pmax) {
  int i, j, k;
  double s = 0.0, mx = 0.0;
  if (interior(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) {
    const long long id = d.id(i, j, k);
    const double flag = (1.0 - (double)ib[id]) * (1.0 - (double)gh[id]);
    double v = dtinv * ((fu[id + 1] - fu[id]) * m.dxi[i] + (fv[id + d.NX] - fv[id]) * m.dyi[j] +
                        (fw[id + d.NX * d.NY] - fw[id]) * m.dzi[k]);
    v = v * flag;
    div[id] = v;
    s = v * m.dx[i] * m.dy[j] * m.dz[k];
    mx = fabs(v / dtinv);
  }
  s = warp_sum(s);
  mx = warp_max(mx);
  __shared__ double rs[8], rm[8];
  if ((threadIdx.x & 31) == 0) { rs[threadIdx.x >> 5] = s; rm[threadIdx.x >> 5] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ts = 0.0, tm = 0.0;
    for (int q = 0; q < 8; ++q) { ts += rs[q]; tm = fmax(tm, rm[q]); }
    psum[blockIdx.x] = ts;
    pmax[blockIdx.x] = tm;
  }
}

// correct_vel / calc_pres_grad: the face-interpolated gradient of p' on
// the non-iblank cells; u -= dt grad p' and/or the gradient stored
__global__ void k_correct(Dims d, Met m, const int8_t *ib, const double *pp, double dt, double *u, double *v,
                          double *w, double *gx, double *gy, double *gz) {
  int i, j, k;
  if (!interior(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const long long id = d.id(i, j, k), sy = d.NX, sz = d.NX * d.NY;
  const double fx1 = fint(m.x, m.xc, i + 1), fx0 = fint(m.x, m.xc, i);
  const double fy1 = fint(m.y, m.yc, j + 1), fy0 = fint(m.y, m.yc, j);
  const double fz1 = fint(m.z, m.zc, k + 1), fz0 = fint(m.z, m.zc, k);
  const double pc = pp[id];
  const double pe = fx1 * pp[id + 1] + (1.0 - fx1) * pc, pw = fx0 * pc + (1.0 - fx0) * pp[id - 1];
  const double pn = fy1 * pp[id + sy] + (1.0 - fy1) * pc, ps = fy0 * pc + (1.0 - fy0) * pp[id - sy];
  const double pf = fz1 * pp[id + sz] + (1.0 - fz1) * pc, pb = fz0 * pc + (1.0 - fz0) * pp[id - sz];
  const double pgx = (pe - pw) * m.dxi[i], pgy = (pn - ps) * m.dyi[j], pgz = (pf - pb) * m.dzi[k];
  const double flag = 1.0 - (double)ib[id];
  if (u) {
    u[id] = u[id] - dt * pgx * flag;
    v[id] = v[id] - dt * pgy * flag;
    w[id] = w[id] - dt * pgz * flag;
  }
  if (gx) {
    gx[id] = pgx * flag;
    gy[id] = pgy * flag;
    gz[id] = pgz * flag;
  }
}

// update_pressure: p' = 0 on the solid cells not dead-marked -1, i = 0..nx,
// j = 0..ny+1, k = 0..nz+1
__global__ void k_zero_solid(Dims d, const int8_t *ib, const int8_t *dead, double *pp) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ni = d.nx + 1, nj = d.NY;
  if (e >= ni * nj * (d.nz + 2)) return;
  const int i = (int)(e % ni), j = (int)((e / ni) % nj), k = (int)(e / (ni * nj));
  const long long id = d.id(i, j, k);
  if (ib[id] == 0 || dead[id] == -1) return;
  pp[id] = 0.0;
}

// update_pressure's domain edge lines for one rank: i = 0..nx on j in
// {0, ny} and j = 0..ny+1 on i in {0, nx}, each in the planes 0, nz, nz+1;
// the four k lines at (i, j) in {0, nx} x {0, ny}
__global__ void k_zero_edges(Dims d, double *pp) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int na = 6 * (d.nx + 1), nb = 6 * (d.ny + 2), nc = 4 * (d.nz + 2);
  const int pl[3] = {0, d.nz, d.nz + 1};
  if (t < na) {
    const int i = t % (d.nx + 1), q = t / (d.nx + 1);
    pp[d.id(i, (q & 1) ? d.ny : 0, pl[q >> 1])] = 0.0;
  } else if (t < na + nb) {
    const int u = t - na, j = u % (d.ny + 2), q = u / (d.ny + 2);
    pp[d.id((q & 1) ? d.nx : 0, j, pl[q >> 1])] = 0.0;
  } else if (t < na + nb + nc) {
    const int u = t - na - nb, k = u % (d.nz + 2), q = u / (d.nz + 2);
    pp[d.id((q & 1) ? d.nx : 0, (q & 2) ? d.ny : 0, k)] = 0.0;
  }
}

}  // namespace proj
}  // namespace fg

using namespace fg;

namespace {

// the case's projection metrics (uploaded on first use) and its masks
fg_status proj_setup(fg_case *c, proj::Met &m, proj::Dims &d) {
  if (!c->prepared) {
    fg_status st = fg_mg_prepare(c);
    if (st != FG_OK) return st;
  }
  if (!c->d_pmet) {
    const HLevel &L = c->lev[0];
    std::vector<double> v;
    for (const std::vector<double> *a : {&L.x, &L.y, &L.z, &L.xc, &L.yc, &L.zc}) v.insert(v.end(), a->begin(), a->end());
    for (const std::vector<double> *a : {&L.x, &L.y, &L.z}) {
      const size_t n = a->size();
      for (size_t i = 0; i < n; ++i) v.push_back(i + 1 < n ? (*a)[i + 1] - (*a)[i] : 0.0);
    }
    for (const std::vector<double> *a : {&L.dxinv, &L.dyinv, &L.dzinv}) v.insert(v.end(), a->begin(), a->end());
    FG_CUDA(fg::dev_alloc(&c->d_pmet, v.size() * sizeof(double)));
    FG_CUDA(cudaMemcpy(c->d_pmet, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  const size_t NX = (size_t)c->nx + 2, NY = (size_t)c->ny + 2, NZ = (size_t)c->nz + 2;
  const double *p = c->d_pmet;
  m.x = p; m.y = m.x + NX; m.z = m.y + NY;
  m.xc = m.z + NZ; m.yc = m.xc + NX; m.zc = m.yc + NY;
  m.dx = m.zc + NZ; m.dy = m.dx + NX; m.dz = m.dy + NY;
  m.dxi = m.dz + NZ; m.dyi = m.dxi + NX; m.dzi = m.dyi + NY;
  d.nx = c->nx; d.ny = c->ny; d.nz = c->nz;
  d.NX = (long long)NX; d.NY = (long long)NY;
  return FG_OK;
}

unsigned cells_blocks(const fg_case *c) {
  return (unsigned)(((long long)(c->nx - 1) * (c->ny - 1) * (c->nz - 1) + 255) / 256);
}

int zero_gradient_faces(const int *vel_zero_gradient) {
  int vzg = 0;
  if (vel_zero_gradient)
    for (int f = 0; f < 6; ++f)
      if (vel_zero_gradient[f]) vzg |= 1 << f;
  return vzg;
}

// enforce_global_mass_consv on the stream: the flux partials into part
// (nb entries), the correction into part[2 nb], then applied
void enqueue_mass_consv(fg_case *c, const proj::Met &m, const proj::Dims &d, int vzg, double *fu, double *fv,
                        double *fw, double *bcxu, double *bcyv, double *bczw, double *part, unsigned nb,
                        long long &launches) {
  const size_t nref = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  const int8_t *ib = c->d_refmask, *gh = c->d_refmask + nref;
  cudaStream_t s = c->stream;
  proj::k_massflux<<<nb, 256, 0, s>>>(d, m, ib, gh, fu, fv, fw, part);
  proj::k_massflux_corr<<<1, 1024, 0, s>>>(d, m, ib, part, (int)nb, vzg, part + 2 * nb);
  const long long big = (long long)(std::max(c->nx, c->ny) + 1) * (std::max(c->ny, c->nz) + 1);
  proj::k_massflux_apply<<<dim3((unsigned)((big + 255) / 256), 6), 256, 0, s>>>(d, vzg, part + 2 * nb, bcxu, bcyv,
                                                                              bczw, fu, fv, fw);
  launches += 3;
}

}  // namespace

extern "C" {

fg_status fg_face_vel_device(fg_case *c, const double *u, const double *v, const double *w, const double *bcxu,
                             const double *bcyv, const double *bczw, double *face_u, double *face_v,
                             double *face_w) {
  if (!c || !u || !v || !w || !bcxu || !bcyv || !bczw || !face_u || !face_v || !face_w) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  proj::Met m;
  proj::Dims d;
  fg_status st = proj_setup(c, m, d);
  if (st != FG_OK) return st;
  proj::k_face_vel<<<cells_blocks(c), 256, 0, c->stream>>>(d, m, u, v, w, bcxu, bcyv, bczw, face_u, face_v, face_w);
  note_launches(1);
  FG_CUDA(cudaGetLastError());
  FG_CUDA(cudaStreamSynchronize(c->stream));
  return FG_OK;
}

fg_status fg_rhs_poisson_device(fg_case *c, double *face_u, double *face_v, double *face_w, double *bcxu,
                                double *bcyv, double *bczw, const int *vel_zero_gradient, double dt, double *div,
                                double *sumd, double *resdiv) {
  if (!c || !face_u || !face_v || !face_w || !div || !(dt > 0.0)) return FG_BAD_INPUT;
  const int vzg = zero_gradient_faces(vel_zero_gradient);
  if (vzg && (!bcxu || !bcyv || !bczw)) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  proj::Met m;
  proj::Dims d;
  fg_status st = proj_setup(c, m, d);
  if (st != FG_OK) return st;
  const size_t nref = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  const int8_t *ib = c->d_refmask, *gh = c->d_refmask + nref;
  const unsigned nb = cells_blocks(c);
  double *part = nullptr;
  FG_CUDA(fg::dev_alloc(&part, (2 * (size_t)nb + 1) * sizeof(double)));
  cudaStream_t s = c->stream;
  cudaError_t e = cudaSuccess;
  long long launches = 0;
  if (vzg) enqueue_mass_consv(c, m, d, vzg, face_u, face_v, face_w, bcxu, bcyv, bczw, part, nb, launches);
  e = cudaMemsetAsync(div, 0, nref * sizeof(double), s);
  if (e == cudaSuccess) {
    proj::k_div<<<nb, 256, 0, s>>>(d, m, ib, gh, face_u, face_v, face_w, 1.0 / dt, div, part, part + nb);
    launches += 1;
    e = cudaGetLastError();
  }
  note_launches(launches);
  std::vector<double> h(2 * (size_t)nb);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  fg::dev_free(part);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return FG_CUDA_ERROR;
  }
  double sd = 0.0, rd = 0.0;
  for (unsigned b = 0; b < nb; ++b) { sd += h[b]; rd = std::max(rd, h[nb + b]); }
  if (sumd) *sumd = sd / (1.0 / dt);  // the mass flux, dt removed
  if (resdiv) *resdiv = rd;
  return FG_OK;
}

fg_status fg_enforce_global_mass_consv_device(fg_case *c, double *face_u, double *face_v, double *face_w,
                                              double *bcxu, double *bcyv, double *bczw,
                                              const int *vel_zero_gradient) {
  if (!c || !face_u || !face_v || !face_w) return FG_BAD_INPUT;
  const int vzg = zero_gradient_faces(vel_zero_gradient);
  if (!vzg) return FG_OK;
  if (!bcxu || !bcyv || !bczw) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  proj::Met m;
  proj::Dims d;
  fg_status st = proj_setup(c, m, d);
  if (st != FG_OK) return st;
  const unsigned nb = cells_blocks(c);
  double *part = nullptr;
  FG_CUDA(fg::dev_alloc(&part, (2 * (size_t)nb + 1) * sizeof(double)));
  long long launches = 0;
  enqueue_mass_consv(c, m, d, vzg, face_u, face_v, face_w, bcxu, bcyv, bczw, part, nb, launches);
  note_launches(launches);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  fg::dev_free(part);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return FG_CUDA_ERROR;
  }
  return FG_OK;
}

fg_status fg_correct_vel_device(fg_case *c, const double *pPrime, double dt, double *u, double *v, double *w,
                                double *dpdx, double *dpdy, double *dpdz) {
  if (!c || !pPrime) return FG_BAD_INPUT;
  if ((u || v || w) && !(u && v && w)) return FG_BAD_INPUT;
  if ((dpdx || dpdy || dpdz) && !(dpdx && dpdy && dpdz)) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  proj::Met m;
  proj::Dims d;
  fg_status st = proj_setup(c, m, d);
  if (st != FG_OK) return st;
  proj::k_correct<<<cells_blocks(c), 256, 0, c->stream>>>(d, m, c->d_refmask, pPrime, dt, u, v, w, dpdx, dpdy, dpdz);
  note_launches(1);
  FG_CUDA(cudaGetLastError());
  FG_CUDA(cudaStreamSynchronize(c->stream));
  return FG_OK;
}

fg_status fg_update_pressure_device(fg_case *c, double *pPrime, double *p) {
  if (!c || !pPrime) return FG_BAD_INPUT;
  cudaSetDevice(c->device);
  proj::Met m;
  proj::Dims d;
  fg_status st = proj_setup(c, m, d);
  if (st != FG_OK) return st;
  const size_t nref = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  const int8_t *ib = c->d_refmask, *dead = c->d_refmask + 2 * nref;
  cudaStream_t s = c->stream;
  const long long ncell = (long long)(c->nx + 1) * (c->ny + 2) * (c->nz + 2);
  proj::k_zero_solid<<<(unsigned)((ncell + 255) / 256), 256, 0, s>>>(d, ib, dead, pPrime);
  const int nedge = 6 * (c->nx + 1) + 6 * (c->ny + 2) + 4 * (c->nz + 2);
  proj::k_zero_edges<<<(nedge + 255) / 256, 256, 0, s>>>(d, pPrime);
  note_launches(2);
  FG_CUDA(cudaGetLastError());
  if (p && p != pPrime) FG_CUDA(cudaMemcpyAsync(p, pPrime, nref * sizeof(double), cudaMemcpyDeviceToDevice, s));
  FG_CUDA(cudaStreamSynchronize(s));
  return FG_OK;
}

}  // extern "C"

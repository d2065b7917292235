// fg_mg.cu -- multigrid kernels of the pressure-Poisson path (sm_100a).
//
// All kernels are batched: one launch covers one multigrid level of every
// problem of a batch (a single solve is a batch of one).  Block b works for
// the problem p with off[p] <= b < off[p+1].
//
// The discrete system is the reference's fine-grid fixed point
// (CORE_POISSON.F90:494-521 rows on fluid cells, GCM_GHOSTCELL_UPDATE.F90
// :563-641 rows on ghost cells); the smoother is a zebra line relaxation
// (CORE_MG.F90:615-938 relaxes lines lexicographically; here lines of one
// colour are solved in parallel, one warp per line).
#include <cuda_runtime.h>
#include <stdint.h>

#include "fg_internal.h"

namespace fg {
namespace k {

constexpr int XL_WARPS = 4;    // x-lines per block
constexpr int TILE_I = 32;     // i-extent of a y/z tile
constexpr int YZ_WARPS = 16;   // lines of one colour per y/z tile
constexpr int CELL_BLOCK = 256;

__device__ __forceinline__ int find_entry(const int *off, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// 1 = coupled neighbour, 2 = Dirichlet boundary face (diagonal doubled,
// CORE_SET_OUTER_BC.F90:901-904 with :1093), 0 = face dropped (Neumann
// boundary, CORE_SET_OUTER_BC.F90:907-911 with pgrad = 0, or OFF cell)
__device__ __forceinline__ int face_w(int8_t nt, int bc) {
  return (nt == T_ACTIVE || nt == T_GHOST || nt == T_SOLID) ? 1 : ((nt == T_BOUND && bc) ? 2 : 0);
}

// padded position of row r of a line split into P chunks (base, rem): one
// unused slot after every chunk keeps the per-lane chunk reads of the
// solver off a single shared-memory bank
__device__ __forceinline__ int padpos(int r, int base, int rem) {
  int big = rem * (base + 1);
  int c = r < big ? r / (base + 1) : rem + (r - big) / base;
  return r + c;
}

__host__ __device__ __forceinline__ void chunking(int n, int &P, int &base, int &rem) {
  P = n / 2 < 32 ? n / 2 : 32;
  if (P < 1) P = 1;
  base = n / P;
  rem = n % P;
}

// ------------------------------------------------------- row staging
// Coefficients of row (cell id) of a line along AXIS: b = diagonal,
// d = rhs minus the transverse couplings, flags bit0 active, bit1 coupled to
// the previous cell of the line, bit2 coupled to the next one.  Non-active
// cells become identity rows holding their current value.
template <typename T, int AXIS>
__device__ __forceinline__ void stage_row(const DevLevel &L, long long id, int i, int j, int k,
                                          const T *__restrict__ x, const T *__restrict__ rhs,
                                          T &b, T &d, uint8_t &f) {
  const int8_t t = L.type[id];
  if (t != T_ACTIVE) {
    b = T(1); d = x[id]; f = 0;
    return;
  }
  double diag = 0.0;
  T acc = rhs[id];
  uint8_t fl = 1;
  const long long off[6] = {-1, 1, -L.sy, L.sy, -L.sz, L.sz};
  const double a[6] = {L.amx[i], L.apx[i], L.amy[j], L.apy[j], L.amz[k], L.apz[k]};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int w = face_w(L.type[id + off[q]], L.bc[q]);
    diag -= a[q] * (double)w;
    if (q / 2 == AXIS) {
      if (w == 1) fl |= (q & 1) ? 4 : 2;
    } else if (w == 1) {
      acc -= (T)a[q] * x[id + off[q]];
    }
  }
  if (diag == 0.0) {  // no face left: keep the value (CORE_MG.F90:690-695)
    b = T(1); d = x[id]; f = 0;
    return;
  }
  b = (T)diag; d = acc; f = fl;
}

// ------------------------------------------------------ warp line solve
template <typename T> struct Eq { T a, b, c, d; };

template <typename T>
__device__ __forceinline__ Eq<T> pcr_combine(const Eq<T> &e, const Eq<T> &l, const Eq<T> &r) {
  const T k1 = e.a / l.b, k2 = e.c / r.b;
  Eq<T> o;
  o.a = -l.a * k1;
  o.c = -r.c * k2;
  o.b = e.b - l.c * k1 - r.a * k2;
  o.d = e.d - l.d * k1 - r.d * k2;
  return o;
}

template <typename T>
__device__ __forceinline__ Eq<T> shfl_eq_up(const Eq<T> &e, int t, int lane) {
  Eq<T> o;
  o.a = __shfl_up_sync(0xffffffffu, e.a, t);
  o.b = __shfl_up_sync(0xffffffffu, e.b, t);
  o.c = __shfl_up_sync(0xffffffffu, e.c, t);
  o.d = __shfl_up_sync(0xffffffffu, e.d, t);
  if (lane < t) { o.a = T(0); o.b = T(1); o.c = T(0); o.d = T(0); }
  return o;
}
template <typename T>
__device__ __forceinline__ Eq<T> shfl_eq_down(const Eq<T> &e, int t, int lane) {
  Eq<T> o;
  o.a = __shfl_down_sync(0xffffffffu, e.a, t);
  o.b = __shfl_down_sync(0xffffffffu, e.b, t);
  o.c = __shfl_down_sync(0xffffffffu, e.c, t);
  o.d = __shfl_down_sync(0xffffffffu, e.d, t);
  if (lane + t >= 32) { o.a = T(0); o.b = T(1); o.c = T(0); o.d = T(0); }
  return o;
}

// Solves one tridiagonal line of n rows held in shared memory (b, d,
// flags at padded positions; sub/super diagonals from the axis coefficient
// arrays am/ap gated by the flags) with the whole warp: each lane
// eliminates a chunk of >= 2 rows down and up (the partition method), the
// 2P chunk-end unknowns form a tridiagonal system solved by parallel cyclic
// reduction across lanes, and each lane back-substitutes its chunk.  The
// solution overwrites d.
template <typename T, int MAXM>
__device__ __forceinline__ void warp_solve(int n, const double *__restrict__ am, const double *__restrict__ ap,
                           const T *sb, T *sd, const uint8_t *sf, int lane) {
  if (n == 1) {
    if (lane == 0) sd[0] = sd[0] / sb[0];
    __syncwarp();
    return;
  }
  int P, base, rem;
  chunking(n, P, base, rem);
  const bool own = lane < P;
  const int m = own ? base + (lane < rem ? 1 : 0) : 0;
  const int s = lane * base + (lane < rem ? lane : rem);
  const int ps = s + lane;
  T al[MAXM], ga[MAXM], de[MAXM];
  Eq<T> F{T(0), T(1), T(0), T(0)}, L{T(0), T(1), T(0), T(0)};
  T a0 = T(0), b0 = T(1), c0 = T(0), d0 = T(0);
  if (own) {
    {
      const uint8_t f0 = sf[ps];
      a0 = (f0 & 2) ? (T)am[s + 1] : T(0);
      c0 = (f0 & 4) ? (T)ap[s + 1] : T(0);
      b0 = sb[ps];
      d0 = sd[ps];
    }
#pragma unroll
    for (int q = 1; q < MAXM; ++q) {
      if (q < m) {
        const uint8_t fq = sf[ps + q];
        const T aq = (fq & 2) ? (T)am[s + q + 1] : T(0);
        const T cq = (fq & 4) ? (T)ap[s + q + 1] : T(0);
        const T bq = sb[ps + q], dq = sd[ps + q];
        if (q == 1) {
          const T r = T(1) / bq;
          al[1] = aq * r; ga[1] = cq * r; de[1] = dq * r;
        } else {
          const T r = T(1) / (bq - aq * ga[q - 1]);
          al[q] = -aq * al[q - 1] * r;
          ga[q] = cq * r;
          de[q] = (dq - aq * de[q - 1]) * r;
        }
        // the last row of the chunk (q = m-1) gives the L equation
        L.a = al[q]; L.b = T(1); L.c = ga[q]; L.d = de[q];
      }
    }
    T pa = T(0), pb = T(-1), pd = T(0);
#pragma unroll
    for (int q = MAXM - 2; q >= 1; --q) {
      if (q <= m - 2) {
        const T nd = de[q] - ga[q] * pd;
        const T na = al[q] - ga[q] * pa;
        const T nb = -ga[q] * pb;
        al[q] = na; ga[q] = nb; de[q] = nd;
        pa = na; pb = nb; pd = nd;
      }
    }
    F.a = a0; F.b = b0 - c0 * pa; F.c = -c0 * pb; F.d = d0 - c0 * pd;
  }
  // parallel cyclic reduction over the 2*32 chunk-end equations
  {
    const Eq<T> Lm = shfl_eq_up(L, 1, lane);
    const Eq<T> Fp = shfl_eq_down(F, 1, lane);
    const Eq<T> nF = pcr_combine(F, Lm, L);
    const Eq<T> nL = pcr_combine(L, F, Fp);
    F = nF; L = nL;
  }
#pragma unroll
  for (int t = 1; t < 32; t <<= 1) {
    const Eq<T> Fm = shfl_eq_up(F, t, lane), Fp = shfl_eq_down(F, t, lane);
    const Eq<T> Lm = shfl_eq_up(L, t, lane), Lp = shfl_eq_down(L, t, lane);
    const Eq<T> nF = pcr_combine(F, Fm, Fp);
    const Eq<T> nL = pcr_combine(L, Lm, Lp);
    F = nF; L = nL;
  }
  if (own) {
    const T xF = F.d / F.b, xL = L.d / L.b;
#pragma unroll
    for (int q = 1; q < MAXM; ++q)
      if (q <= m - 2) sd[ps + q] = de[q] - al[q] * xF - ga[q] * xL;
    sd[ps] = xF;
    sd[ps + m - 1] = xL;
  }
  __syncwarp();
}

template <typename T> struct PrecOf;
template <> struct PrecOf<double> {
  static __device__ __forceinline__ double *x(const DevLevel &L) { return L.x64; }
  static __device__ __forceinline__ double *rhs(const DevLevel &L) { return L.rhs64; }
  static __device__ __forceinline__ double *res(const DevLevel &L) { return L.res64; }
};
template <> struct PrecOf<float> {
  static __device__ __forceinline__ float *x(const DevLevel &L) { return L.x32; }
  static __device__ __forceinline__ float *rhs(const DevLevel &L) { return L.rhs32; }
  static __device__ __forceinline__ float *res(const DevLevel &L) { return L.res32; }
};

__host__ __device__ __forceinline__ int line_pad(int n) { return n + 33; }
__host__ __device__ __forceinline__ size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

// ------------------------------------------------------- x-line kernel
// Lines (j,k) with (j+k)%2 == color; one warp per line.
template <typename T, int MAXM>
__global__ void __launch_bounds__(XL_WARPS * 32)
k_xline(const int *off, int nent, const DevLevel *levs, int color, T omega) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nyh = (L.ny + 1) >> 1;
  const int q = lb * XL_WARPS + warp;
  const int k = 1 + q / nyh;
  const int jj = q % nyh;
  const int n = L.nx;
  const int np = line_pad(n);
  const size_t per = align16(np * sizeof(T)) * 2 + align16(np);
  T *sb = reinterpret_cast<T *>(smem + per * warp);
  T *sd = reinterpret_cast<T *>(smem + per * warp + align16(np * sizeof(T)));
  uint8_t *sf = smem + per * warp + 2 * align16(np * sizeof(T));
  if (k > L.nz) return;
  const int j0 = (((1 + k) & 1) == color) ? 1 : 2;
  const int j = j0 + 2 * jj;
  if (j > L.ny) return;
  T *x = PrecOf<T>::x(L);
  const T *rhs = PrecOf<T>::rhs(L);
  int P, base, rem;
  chunking(n, P, base, rem);
  const long long row = L.sy * j + L.sz * k;
  for (int r = lane; r < n; r += 32) {
    T b, d; uint8_t f;
    stage_row<T, 0>(L, row + r + 1, r + 1, j, k, x, rhs, b, d, f);
    const int pp = padpos(r, base, rem);
    sb[pp] = b; sd[pp] = d; sf[pp] = f;
  }
  __syncwarp();
  warp_solve<T, MAXM>(n, L.amx, L.apx, sb, sd, sf, lane);
  for (int r = lane; r < n; r += 32) {
    const int pp = padpos(r, base, rem);
    if (sf[pp] & 1) {
      const long long id = row + r + 1;
      x[id] = (omega == T(1)) ? sd[pp] : x[id] + omega * (sd[pp] - x[id]);
    }
  }
}

// ----------------------------------------------------- y/z-line kernel
// AXIS 1: lines (i,k) along j, colour (i+k)%2, tiles of 32 i at fixed k.
// AXIS 2: lines (i,j) along k, colour (i+j)%2, tiles of 32 i at fixed j.
template <typename T, int MAXM, int AXIS>
__global__ void __launch_bounds__(YZ_WARPS * 32)
k_yzline(const int *off, int nent, const DevLevel *levs, int color, T omega) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  const int ntx = (L.nx + TILE_I - 1) / TILE_I;
  const int ti = lb % ntx;
  const int o = 1 + lb / ntx;  // fixed index: k for AXIS 1, j for AXIS 2
  const int i0 = 1 + TILE_I * ti;
  const int n = AXIS == 1 ? L.ny : L.nz;
  const long long ls = AXIS == 1 ? L.sy : L.sz;
  const long long os = AXIS == 1 ? L.sz : L.sy;
  const int np = line_pad(n);
  const int lstride = np + 1;  // per-line stride (elements), odd in words
  T *sb = reinterpret_cast<T *>(smem);
  T *sd = reinterpret_cast<T *>(smem + align16((size_t)YZ_WARPS * lstride * sizeof(T)));
  uint8_t *sf = smem + 2 * align16((size_t)YZ_WARPS * lstride * sizeof(T));
  const int il0 = (color + i0 + o) & 1;  // tile-local i of the first line of this colour
  T *x = PrecOf<T>::x(L);
  const T *rhs = PrecOf<T>::rhs(L);
  int P, base, rem;
  chunking(n, P, base, rem);
  const int tid = threadIdx.x;
  const int total = TILE_I * n;
  for (int e = tid; e < total; e += YZ_WARPS * 32) {
    const int il = e & (TILE_I - 1), r = e / TILE_I;
    if ((il & 1) != il0) continue;
    const int i = i0 + il;
    if (i > L.nx) continue;
    const int slot = il >> 1;
    const int jj = AXIS == 1 ? r + 1 : o;
    const int kk = AXIS == 1 ? o : r + 1;
    const long long id = i + L.sy * jj + L.sz * kk;
    T b, d; uint8_t f;
    stage_row<T, AXIS>(L, id, i, jj, kk, x, rhs, b, d, f);
    const int pp = slot * lstride + padpos(r, base, rem);
    sb[pp] = b; sd[pp] = d; sf[pp] = f;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  {
    const int i = i0 + il0 + 2 * warp;
    if (i <= L.nx) {
      const double *am = AXIS == 1 ? L.amy : L.amz;
      const double *ap = AXIS == 1 ? L.apy : L.apz;
      warp_solve<T, MAXM>(n, am, ap, sb + warp * lstride, sd + warp * lstride,
                          sf + warp * lstride, lane);
    }
  }
  __syncthreads();
  for (int e = tid; e < total; e += YZ_WARPS * 32) {
    const int il = e & (TILE_I - 1), r = e / TILE_I;
    if ((il & 1) != il0) continue;
    const int i = i0 + il;
    if (i > L.nx) continue;
    const int pp = (il >> 1) * lstride + padpos(r, base, rem);
    if (sf[pp] & 1) {
      const long long id = i + ls * (r + 1) + os * o;
      x[id] = (omega == T(1)) ? sd[pp] : x[id] + omega * (sd[pp] - x[id]);
    }
  }
}

int blocks_cells(const DevLevel &L) {
  long long c = (long long)L.nx * L.ny * L.nz;
  return (int)((c + CELL_BLOCK - 1) / CELL_BLOCK);
}
int blocks_xline(const DevLevel &L) {
  long long lines = (long long)((L.ny + 1) / 2) * L.nz;
  return (int)((lines + XL_WARPS - 1) / XL_WARPS);
}
int blocks_tile(const DevLevel &L, int axis) {
  int ntx = (L.nx + TILE_I - 1) / TILE_I;
  return ntx * (axis == 1 ? L.nz : L.ny);
}
size_t smem_line(int n, int tsize, int lines) {
  const int np = line_pad(n);
  if (lines == XL_WARPS) {
    const size_t per = align16((size_t)np * tsize) * 2 + align16(np);
    return per * XL_WARPS;
  }
  const int lstride = np + 1;
  return 2 * align16((size_t)YZ_WARPS * lstride * tsize) + align16((size_t)YZ_WARPS * lstride);
}

template <typename T, int MAXM>
static cudaError_t launch_line(const Launch &Lr, int axis, int color, double omega, int maxn,
                               cudaStream_t s) {
  const T om = (T)omega;
  if (axis == 0) {
    const size_t sm = smem_line(maxn, sizeof(T), XL_WARPS);
    auto kern = k_xline<T, MAXM>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<Lr.blocks, XL_WARPS * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, om);
  } else {
    const size_t sm = smem_line(maxn, sizeof(T), YZ_WARPS);
    if (axis == 1) {
      auto kern = k_yzline<T, MAXM, 1>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      kern<<<Lr.blocks, YZ_WARPS * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, om);
    } else {
      auto kern = k_yzline<T, MAXM, 2>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      kern<<<Lr.blocks, YZ_WARPS * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, om);
    }
  }
  return cudaGetLastError();
}

// maxn: the longest line of this launch along `axis`
template <typename T>
cudaError_t line_sweep(const Launch &Lr, int axis, int color, double omega, int maxn,
                       cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  int P, base, rem;
  chunking(maxn, P, base, rem);
  const int m = base + (rem ? 1 : 0);
  if (m <= 4) return launch_line<T, 4>(Lr, axis, color, omega, maxn, s);
  if (m <= 8) return launch_line<T, 8>(Lr, axis, color, omega, maxn, s);
  if (m <= 16) return launch_line<T, 16>(Lr, axis, color, omega, maxn, s);
  if (m <= 32) return launch_line<T, 32>(Lr, axis, color, omega, maxn, s);
  return cudaErrorInvalidValue;  // lines longer than 1024 cells
}

// ---------------------------------------------------------- residual
template <typename T>
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[CELL_BLOCK / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = l < CELL_BLOCK / 32 ? red[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;
}

template <typename T>
__device__ __forceinline__ T apply_row(const DevLevel &L, long long id, int i, int j, int k,
                                       const T *__restrict__ x) {
  double diag = 0.0;
  T acc = T(0);
  const long long off[6] = {-1, 1, -L.sy, L.sy, -L.sz, L.sz};
  const double a[6] = {L.amx[i], L.apx[i], L.amy[j], L.apy[j], L.amz[k], L.apz[k]};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int w = face_w(L.type[id + off[q]], L.bc[q]);
    diag -= a[q] * (double)w;
    if (w == 1) acc += (T)a[q] * x[id + off[q]];
  }
  return acc + (T)diag * x[id];
}

template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_residual(const int *off, int nent, const DevLevel *levs, double *norm2) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const long long e = (long long)(blockIdx.x - off[p]) * CELL_BLOCK + threadIdx.x;
  const long long nc = (long long)L.nx * L.ny * L.nz;
  double r2 = 0.0;
  if (e < nc) {
    const int i = 1 + (int)(e % L.nx);
    const int j = 1 + (int)((e / L.nx) % L.ny);
    const int k = 1 + (int)(e / ((long long)L.nx * L.ny));
    const long long id = i + L.sy * j + L.sz * k;
    T r = T(0);
    if (L.type[id] == T_ACTIVE) {
      const T *x = PrecOf<T>::x(L);
      r = PrecOf<T>::rhs(L)[id] - apply_row<T>(L, id, i, j, k, x);
    }
    PrecOf<T>::res(L)[id] = r;
    r2 = (double)r * (double)r;
  }
  if (norm2) {
    const double t = block_sum<T>(r2);
    if (threadIdx.x == 0) atomicAdd(norm2 + p, t);
  }
}

template <typename T>
cudaError_t residual(const Launch &Lr, double *norm2, cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  k_residual<T><<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev, norm2);
  return cudaGetLastError();
}

// ||f||^2 over active cells of level 0 (FP64 rhs)
__global__ void __launch_bounds__(CELL_BLOCK)
k_fluid_norm(const int *off, int nent, const DevLevel *levs, double *norm2) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const long long e = (long long)(blockIdx.x - off[p]) * CELL_BLOCK + threadIdx.x;
  const long long nc = (long long)L.nx * L.ny * L.nz;
  double r2 = 0.0;
  if (e < nc) {
    const int i = 1 + (int)(e % L.nx);
    const int j = 1 + (int)((e / L.nx) % L.ny);
    const int k = 1 + (int)(e / ((long long)L.nx * L.ny));
    const long long id = i + L.sy * j + L.sz * k;
    if (L.type[id] == T_ACTIVE) r2 = L.rhs64[id] * L.rhs64[id];
  }
  const double t = block_sum<double>(r2);
  if (threadIdx.x == 0) atomicAdd(norm2 + p, t);
}

cudaError_t fluid_norm(const Launch &Lr, double *norm2, cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  k_fluid_norm<<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev, norm2);
  return cudaGetLastError();
}

// Mixed precision outer step, part 1: p += e (FP64 += FP32) and e = 0.
// Part 2 is k_residual<double>-like but writes the FP32 residual.
__global__ void __launch_bounds__(CELL_BLOCK)
k_correct(const int *off, int nent, const DevLevel *levs) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const long long e = (long long)(blockIdx.x - off[p]) * CELL_BLOCK + threadIdx.x;
  const long long nc = (long long)L.nx * L.ny * L.nz;
  if (e >= nc) return;
  const int i = 1 + (int)(e % L.nx);
  const int j = 1 + (int)((e / L.nx) % L.ny);
  const int k = 1 + (int)(e / ((long long)L.nx * L.ny));
  const long long id = i + L.sy * j + L.sz * k;
  const float ev = L.x32[id];
  L.x64[id] = L.x64[id] + (double)ev;
  L.x32[id] = 0.0f;
}

__global__ void __launch_bounds__(CELL_BLOCK)
k_residual_mixed(const int *off, int nent, const DevLevel *levs, double *norm2) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const long long e = (long long)(blockIdx.x - off[p]) * CELL_BLOCK + threadIdx.x;
  const long long nc = (long long)L.nx * L.ny * L.nz;
  double r2 = 0.0;
  if (e < nc) {
    const int i = 1 + (int)(e % L.nx);
    const int j = 1 + (int)((e / L.nx) % L.ny);
    const int k = 1 + (int)(e / ((long long)L.nx * L.ny));
    const long long id = i + L.sy * j + L.sz * k;
    double r = 0.0;
    if (L.type[id] == T_ACTIVE) r = L.rhs64[id] - apply_row<double>(L, id, i, j, k, L.x64);
    L.rhs32[id] = (float)r;
    r2 = r * r;
  }
  const double t = block_sum<double>(r2);
  if (threadIdx.x == 0) atomicAdd(norm2 + p, t);
}

cudaError_t correct_residual(const Launch &Lr, const DevLevel *unused, double *norm2,
                             cudaStream_t s) {
  (void)unused;
  if (Lr.empty()) return cudaSuccess;
  k_correct<<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev);
  k_residual_mixed<<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev, norm2);
  return cudaGetLastError();
}

// ------------------------------------------------------- restriction
// coarse rhs = volume-weighted mean of the children's residuals on active
// coarse cells (the sum of the children's finite-volume equations)
template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_restrict(const int *off, int nent, const DevLevel *coarse, const DevLevel *fine) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &C = coarse[p];
  const DevLevel &F = fine[p];
  const long long e = (long long)(blockIdx.x - off[p]) * CELL_BLOCK + threadIdx.x;
  const long long nc = (long long)C.nx * C.ny * C.nz;
  if (e >= nc) return;
  const int I = 1 + (int)(e % C.nx);
  const int J = 1 + (int)((e / C.nx) % C.ny);
  const int K = 1 + (int)(e / ((long long)C.nx * C.ny));
  const long long id = I + C.sy * J + C.sz * K;
  T *rc = PrecOf<T>::rhs(C);
  if (C.type[id] != T_ACTIVE) { rc[id] = T(0); return; }
  const T *rf = PrecOf<T>::res(F);
  double s = 0.0, v = 0.0;
  for (int k = C.clz[K]; k <= C.chz[K]; ++k)
    for (int j = C.cly[J]; j <= C.chy[J]; ++j) {
      const double wyz = F.wy[j] * F.wz[k];
      const long long rb = F.sy * j + F.sz * k;
      for (int i = C.clx[I]; i <= C.chx[I]; ++i) {
        const double w = F.wx[i] * wyz;
        s += w * (double)rf[rb + i];
        v += w;
      }
    }
  rc[id] = (T)(s / v);
}

template <typename T>
cudaError_t restrict_to(const Launch &Lc, const DevLevel *fine, cudaStream_t s) {
  if (Lc.empty()) return cudaSuccess;
  k_restrict<T><<<Lc.blocks, CELL_BLOCK, 0, s>>>(Lc.off, Lc.n, Lc.lev, fine);
  return cudaGetLastError();
}

// ------------------------------------------------------ prolongation
// fine x += trilinear interpolation of the coarse correction at the fine
// cell centre, over the active coarse corners only (renormalised)
template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_prolong(const int *off, int nent, const DevLevel *fine, const DevLevel *coarse) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &F = fine[p];
  const DevLevel &C = coarse[p];
  const long long e = (long long)(blockIdx.x - off[p]) * CELL_BLOCK + threadIdx.x;
  const long long nc = (long long)F.nx * F.ny * F.nz;
  if (e >= nc) return;
  const int i = 1 + (int)(e % F.nx);
  const int j = 1 + (int)((e / F.nx) % F.ny);
  const int k = 1 + (int)(e / ((long long)F.nx * F.ny));
  const long long id = i + F.sy * j + F.sz * k;
  const int8_t t = F.type[id];
  if (t != T_ACTIVE && t != T_GHOST) return;
  const int i0 = F.plx[i], j0 = F.ply[j], k0 = F.plz[k];
  const int i1 = i0 < C.nx ? i0 + 1 : i0, j1 = j0 < C.ny ? j0 + 1 : j0, k1 = k0 < C.nz ? k0 + 1 : k0;
  const double wx1 = F.pwx[i], wy1 = F.pwy[j], wz1 = F.pwz[k];
  const T *xc = PrecOf<T>::x(C);
  double s = 0.0, ws = 0.0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int ci = (c & 1) ? i1 : i0, cj = (c & 2) ? j1 : j0, ck = (c & 4) ? k1 : k0;
    const double w = ((c & 1) ? wx1 : 1.0 - wx1) * ((c & 2) ? wy1 : 1.0 - wy1) *
                     ((c & 4) ? wz1 : 1.0 - wz1);
    const long long cid = ci + C.sy * cj + C.sz * ck;
    if (w > 0.0 && C.type[cid] == T_ACTIVE) {
      s += w * (double)xc[cid];
      ws += w;
    }
  }
  if (ws > 1e-12) {
    T *x = PrecOf<T>::x(F);
    x[id] = x[id] + (T)(s / ws);
  }
}

template <typename T>
cudaError_t prolong_add(const Launch &Lf, const DevLevel *coarse, cudaStream_t s) {
  if (Lf.empty()) return cudaSuccess;
  k_prolong<T><<<Lf.blocks, CELL_BLOCK, 0, s>>>(Lf.off, Lf.n, Lf.lev, coarse);
  return cudaGetLastError();
}

template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_zero(const int *off, int nent, const DevLevel *levs) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const long long e = (long long)(blockIdx.x - off[p]) * CELL_BLOCK + threadIdx.x;
  const long long nc = (long long)L.nx * L.ny * L.nz;
  if (e >= nc) return;
  const int i = 1 + (int)(e % L.nx);
  const int j = 1 + (int)((e / L.nx) % L.ny);
  const int k = 1 + (int)(e / ((long long)L.nx * L.ny));
  PrecOf<T>::x(L)[i + L.sy * j + L.sz * k] = T(0);
}

template <typename T>
cudaError_t zero_x(const Launch &Lr, cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  k_zero<T><<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev);
  return cudaGetLastError();
}

// ------------------------------------------------- interpolation rows
// x_t = sum_q w_q x_(cell + inc_q) + c  (GCM_GHOSTCELL_UPDATE.F90:582-601,
// corner order of GCM_MEMORY_ALLOCATE.F90:593-623); c is the row constant
// (solution form) or the row residual (correction form).  Rows read other
// rows' targets, so the update is a Jacobi step: all new values are formed
// from the current field first (k_rows), then written (k_rows_scatter).
template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_rows(DevRows R, const DevLevel *lev0, int corr, double *tmp) {
  const int r = blockIdx.x * CELL_BLOCK + threadIdx.x;
  if (r >= R.n) return;
  const DevLevel &L = lev0[R.prob[r]];
  const T *x = PrecOf<T>::x(L);
  const long long b = R.cell[r], sy = L.sy, sz = L.sz;
  const long long o[8] = {0, sy, sy + 1, 1, sz, sz + sy, sz + sy + 1, sz + 1};
  double acc = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) acc += R.w[8 * r + q] * (double)x[b + o[q]];
  double c;
  if (!corr) c = R.c0[r];
  else c = sizeof(T) == 4 ? (double)R.rf[r] : R.rd[r];
  tmp[r] = acc + c;
}

template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_rows_scatter(DevRows R, const DevLevel *lev0, const double *tmp) {
  const int r = blockIdx.x * CELL_BLOCK + threadIdx.x;
  if (r >= R.n) return;
  const DevLevel &L = lev0[R.prob[r]];
  PrecOf<T>::x(L)[R.tgt[r]] = (T)tmp[r];
}

template <typename T>
cudaError_t rows_relax(const DevRows &R, const DevLevel *lev0, int corr, double *tmp,
                       cudaStream_t s) {
  if (R.n <= 0) return cudaSuccess;
  const int nb = (R.n + CELL_BLOCK - 1) / CELL_BLOCK;
  k_rows<T><<<nb, CELL_BLOCK, 0, s>>>(R, lev0, corr, tmp);
  k_rows_scatter<T><<<nb, CELL_BLOCK, 0, s>>>(R, lev0, tmp);
  return cudaGetLastError();
}

// row residual (FP64 solution): r_t = sum w p + c0 - p_t; stores it in
// FP64 and FP32 and the max |r_t| per problem (as ordered bits)
__global__ void __launch_bounds__(CELL_BLOCK)
k_rows_residual(DevRows R, const DevLevel *lev0, double *maxabs) {
  const int r = blockIdx.x * CELL_BLOCK + threadIdx.x;
  if (r >= R.n) return;
  const int p = R.prob[r];
  const DevLevel &L = lev0[p];
  const double *x = L.x64;
  const long long b = R.cell[r], sy = L.sy, sz = L.sz;
  const long long o[8] = {0, sy, sy + 1, 1, sz, sz + sy, sz + sy + 1, sz + 1};
  double acc = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) acc += R.w[8 * r + q] * x[b + o[q]];
  const double rt = acc + R.c0[r] - x[R.tgt[r]];
  R.rd[r] = rt;
  R.rf[r] = (float)rt;
  if (maxabs)
    atomicMax(reinterpret_cast<unsigned long long *>(maxabs + p),
              (unsigned long long)__double_as_longlong(fabs(rt)));
}

cudaError_t rows_residual(const DevRows &R, const DevLevel *lev0, double *maxabs,
                          cudaStream_t s) {
  if (R.n <= 0) return cudaSuccess;
  k_rows_residual<<<(R.n + CELL_BLOCK - 1) / CELL_BLOCK, CELL_BLOCK, 0, s>>>(R, lev0, maxabs);
  return cudaGetLastError();
}

// ---------------------------------------------------- coarsest solve
// x = G rhs over the active cells of a problem's coarsest level, G the
// generalised inverse of the coarsest operator (FP64)
template <typename T>
__global__ void __launch_bounds__(256)
k_coarsest(const DevLevel *levs, const double *const *G, const int *const *gidx, const int *gn) {
  extern __shared__ double sr[];
  const int p = blockIdx.x;
  const DevLevel &L = levs[p];
  const int n = gn[p];
  const int *idx = gidx[p];
  const double *g = G[p];
  const T *rhs = PrecOf<T>::rhs(L);
  T *x = PrecOf<T>::x(L);
  for (int c = threadIdx.x; c < n; c += blockDim.x) sr[c] = (double)rhs[idx[c]];
  __syncthreads();
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    double acc = 0.0;
    const double *gr = g + (size_t)r * n;
    for (int c = 0; c < n; ++c) acc += gr[c] * sr[c];
    x[idx[r]] = (T)acc;
  }
}

template <typename T>
cudaError_t coarsest_solve(int nprob, const DevLevel *lev, const double *const *G,
                           const int *const *gidx, const int *gn, int maxn, cudaStream_t s) {
  if (nprob <= 0) return cudaSuccess;
  const size_t sm = (size_t)maxn * sizeof(double);
  if (sm > 48 * 1024)
    cudaFuncSetAttribute(k_coarsest<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_coarsest<T><<<nprob, 256, sm, s>>>(lev, G, gidx, gn);
  return cudaGetLastError();
}

// ----------------------------------------- layout conversion (boundary)
// reference field (0:nx+1 nodes) <-> device level-0 layout, nx ny nz cells
__global__ void k_copy_in(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                          long long sz) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long X = nx + 2, Y = ny + 2, Z = nz + 2;
  if (e >= X * Y * Z) return;
  const long long i = e % X, j = (e / X) % Y, k = e / (X * Y);
  dst[i + sy * j + sz * k] = src[i + (nx + 3) * (j + (long long)(ny + 3) * k)];
}
__global__ void k_copy_out(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                           long long sz) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long X = nx + 2, Y = ny + 2, Z = nz + 2;
  if (e >= X * Y * Z) return;
  const long long i = e % X, j = (e / X) % Y, k = e / (X * Y);
  dst[i + (nx + 3) * (j + (long long)(ny + 3) * k)] = src[i + sy * j + sz * k];
}
cudaError_t copy_in(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                    long long sz, cudaStream_t s) {
  const long long n = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  k_copy_in<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dst, src, nx, ny, nz, sy, sz);
  return cudaGetLastError();
}
cudaError_t copy_out(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                     long long sz, cudaStream_t s) {
  const long long n = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  k_copy_out<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dst, src, nx, ny, nz, sy, sz);
  return cudaGetLastError();
}

template cudaError_t line_sweep<double>(const Launch &, int, int, double, int, cudaStream_t);
template cudaError_t line_sweep<float>(const Launch &, int, int, double, int, cudaStream_t);
template cudaError_t residual<double>(const Launch &, double *, cudaStream_t);
template cudaError_t residual<float>(const Launch &, double *, cudaStream_t);
template cudaError_t restrict_to<double>(const Launch &, const DevLevel *, cudaStream_t);
template cudaError_t restrict_to<float>(const Launch &, const DevLevel *, cudaStream_t);
template cudaError_t prolong_add<double>(const Launch &, const DevLevel *, cudaStream_t);
template cudaError_t prolong_add<float>(const Launch &, const DevLevel *, cudaStream_t);
template cudaError_t zero_x<double>(const Launch &, cudaStream_t);
template cudaError_t zero_x<float>(const Launch &, cudaStream_t);
template cudaError_t rows_relax<double>(const DevRows &, const DevLevel *, int, double *,
                                        cudaStream_t);
template cudaError_t rows_relax<float>(const DevRows &, const DevLevel *, int, double *,
                                       cudaStream_t);
template cudaError_t coarsest_solve<double>(int, const DevLevel *, const double *const *,
                                            const int *const *, const int *, int, cudaStream_t);
template cudaError_t coarsest_solve<float>(int, const DevLevel *, const double *const *,
                                           const int *const *, const int *, int, cudaStream_t);

}  // namespace k
}  // namespace fg

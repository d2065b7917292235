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

#include <algorithm>
#include <atomic>
#include <type_traits>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#include "fg_internal.h"

namespace fg {

static std::atomic<long long> g_launches{0};
static thread_local long long t_launches = 0;  // this thread's share
void note_launches(long long n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}
long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }
long long thread_launches() { return t_launches; }

namespace k {

constexpr int XL_WARPS = 8;    // x-lines per block
constexpr int TILE_I = 16;     // i-extent of a y/z tile
constexpr int YZ_WARPS = 8;    // lines of one colour per y/z tile
constexpr int CELL_BLOCK = 128;

// Cell kernels tile each level by rows: block lb covers cells
// i = 1 + 128 t + threadIdx.x of row (j,k), so no thread divides by a
// runtime extent (only one 32-bit division per block).
constexpr int CELL_ROWS = 4;  // rows (j,k) per block
struct CellIdx { int i, j, k; bool ok; };
// cell of row r (0..CELL_ROWS-1) of block lb
__device__ __forceinline__ CellIdx cell_of(const DevLevel &L, int lb, int r) {
  const int tpr = (L.nx + CELL_BLOCK - 1) / CELL_BLOCK;
  const int rb = lb / tpr;
  const int t = lb - rb * tpr;
  const int row = rb * CELL_ROWS + r;
  CellIdx c;
  c.j = 1 + row % L.ny;
  c.k = 1 + row / L.ny;
  c.i = 1 + t * CELL_BLOCK + (int)threadIdx.x;
  c.ok = c.i <= L.nx && c.k <= L.nz;
  return c;
}

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

// Reciprocal by Newton-Raphson refinement of the hardware estimate
// (rcp.approx): each step y <- y + y (1 - x y) doubles the number of correct
// bits, two steps take the FP64 estimate to full double precision and one
// the FP32 estimate to full single precision.  Used for the pivots of the
// line solves (diagonally dominant, no denormals).
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}
__device__ __forceinline__ float rcp_nr(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  const float e = fmaf(-x, y, 1.0f);
  return fmaf(y, e, y);
}

// Row -> padded position for a line split into P chunks of base or base+1
// rows: one unused slot after every chunk keeps the per-lane chunk reads
// of the solver on distinct shared-memory banks.  The chunk of a row is
// found with multiply-high by ceil(2^32/d), exact for r, d < 2^16.
struct PadMap {
  int big, rem;
  unsigned m0, m1;  // magic numbers for base and base+1
};
__host__ __device__ __forceinline__ unsigned magic_u32(int d) {
  return (unsigned)((0xffffffffull + (unsigned long long)d) / (unsigned long long)d);
}
__device__ __forceinline__ PadMap padmap(int base, int rem) {
  PadMap pm;
  pm.big = rem * (base + 1);
  pm.rem = rem;
  pm.m0 = magic_u32(base);
  pm.m1 = magic_u32(base + 1);
  return pm;
}
__device__ __forceinline__ int padpos(int r, const PadMap &pm) {
  const int c = r < pm.big ? (int)__umulhi((unsigned)r, pm.m1)
                           : pm.rem + (int)__umulhi((unsigned)(r - pm.big), pm.m0);
  return r + c;
}

__host__ __device__ __forceinline__ void chunking(int n, int &P, int &base, int &rem) {
  P = n / 2 < 32 ? n / 2 : 32;
  if (P < 1) P = 1;
  base = n / P;
  rem = n % P;
}

// ------------------------------------------------------- row staging
// A line along axis A has two faces on its own axis (qm = 2A, qp = 2A+1)
// and four transverse faces whose coefficients are constant along it.
struct LineCoef {
  double tq[4];   // transverse face coefficients
  long long to[4];  // element offsets of the transverse neighbours
  int qt[4];      // transverse face ids
  double tdir;    // 2a over transverse Dirichlet boundary faces of the line
  int qm, qp;     // own-axis face ids
  int dirm, dirp; // Dirichlet boundary at the first / last row
};

__device__ __forceinline__ LineCoef line_coef(const DevLevel &L, int axis, int i, int j, int k) {
  LineCoef c;
  const double am[3] = {glob(L.amx)[i], glob(L.amy)[j], glob(L.amz)[k]};
  const double ap[3] = {glob(L.apx)[i], glob(L.apy)[j], glob(L.apz)[k]};
  const long long st[3] = {1, L.sy, L.sz};
  const int idx[3] = {i, j, k};
  const int nn[3] = {L.nx, L.ny, L.nz};
  int t = 0;
  c.tdir = 0.0;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    if (ax == axis) continue;
    c.qt[t] = 2 * ax; c.tq[t] = am[ax]; c.to[t] = -st[ax];
    if (idx[ax] == 1 && L.bc[2 * ax]) c.tdir += 2.0 * am[ax];
    ++t;
    c.qt[t] = 2 * ax + 1; c.tq[t] = ap[ax]; c.to[t] = st[ax];
    if (idx[ax] == nn[ax] && L.bc[2 * ax + 1]) c.tdir += 2.0 * ap[ax];
    ++t;
  }
  c.qm = 2 * axis; c.qp = 2 * axis + 1;
  c.dirm = L.bc[2 * axis]; c.dirp = L.bc[2 * axis + 1];
  return c;
}

// The coefficients of line_coef in the arithmetic type T of a sweep along
// AXIS, with the face ids fixed at compile time: transverse faces t = 0..3
// are the lower and upper faces of the first, then the second axis other
// than AXIS, at element offsets -s0, +s0, -s1, +s1.
template <typename T, int AXIS>
struct LineCoefT {
  static constexpr int A0 = AXIS == 0 ? 1 : 0;
  static constexpr int A1 = AXIS == 2 ? 1 : 2;
  __host__ __device__ static constexpr int qt(int t) { return t < 2 ? 2 * A0 + t : 2 * A1 + t - 2; }
  static constexpr int qm = 2 * AXIS, qp = 2 * AXIS + 1;
  T tq[4];
  T tdir;
  bool dirm, dirp;
  __device__ __forceinline__ explicit LineCoefT(const LineCoef &c)
      : tq{(T)c.tq[0], (T)c.tq[1], (T)c.tq[2], (T)c.tq[3]}, tdir((T)c.tdir), dirm(c.dirm != 0),
        dirp(c.dirp != 0) {}
  __device__ __forceinline__ bool iso() const { return tdir == T(0) && !dirm && !dirp; }
};

// Row coefficients from the staged mask: a couples to the previous row, c
// to the next, b the diagonal (sum over the kept faces, doubled on
// Dirichlet boundary faces).  Non-active rows are identities.
template <typename T>
__device__ __forceinline__ void row_coef(uint8_t mk, int r, int n, double am, double ap,
                                         const LineCoef &lc, T &a, T &b, T &c) {
  if (!(mk & 64)) { a = T(0); c = T(0); b = T(1); return; }
  double diag = -lc.tdir;
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if ((mk >> lc.qt[q]) & 1) diag -= lc.tq[q];
  const bool cm = (mk >> lc.qm) & 1, cp = (mk >> lc.qp) & 1;
  if (cm) diag -= am; else if (r == 0 && lc.dirm) diag -= 2.0 * am;
  if (cp) diag -= ap; else if (r == n - 1 && lc.dirp) diag -= 2.0 * ap;
  a = cm ? (T)am : T(0);
  c = cp ? (T)ap : T(0);
  b = (T)diag;
}

// Right-hand side of a row: rhs minus the transverse couplings; rows that
// are not active (or have no face left, CORE_MG.F90:690-695) hold their
// value.  All loads are issued unconditionally.
template <typename T>
__device__ __forceinline__ void stage(const DevLevel &L, long long id, const LineCoef &lc,
                                      dptr<const T> FG_RESTRICT x,
                                      dptr<const T> FG_RESTRICT rhs, T &d, uint8_t &mk) {
  mk = glob(L.mask)[id];
  const T r = rhs[id], xo = x[id];
  const T x0 = x[id + lc.to[0]], x1 = x[id + lc.to[1]], x2 = x[id + lc.to[2]], x3 = x[id + lc.to[3]];
  T acc = r;
  if ((mk >> lc.qt[0]) & 1) acc -= (T)lc.tq[0] * x0;
  if ((mk >> lc.qt[1]) & 1) acc -= (T)lc.tq[1] * x1;
  if ((mk >> lc.qt[2]) & 1) acc -= (T)lc.tq[2] * x2;
  if ((mk >> lc.qt[3]) & 1) acc -= (T)lc.tq[3] * x3;
  const bool isolated = ((mk & 63) == 0) && lc.tdir == 0.0 && !lc.dirm && !lc.dirp;
  if (!(mk & 64) || isolated) { d = xo; mk = (uint8_t)(mk & ~64); }
  else d = acc;
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
__device__ __forceinline__ void warp_solve(int n, dptr<const double> FG_RESTRICT am,
                                           dptr<const double> FG_RESTRICT ap, const LineCoef &lc,
                                           dptr<T> sd, dptr<const uint8_t> sf, int lane) {
  if (n == 1) {
    if (lane == 0) {
      T a, b, c;
      row_coef<T>(sf[0], 0, 1, am[1], ap[1], lc, a, b, c);
      sd[0] = sd[0] / b;
    }
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
  // chunk-end equations: F (first row)   aF L_{l-1} + bF F_l + cF L_l = dF
  //                      L (last row)    aL F_l + L_l + cL F_{l+1} = dL
  T aF = T(0), bF = T(1), cF = T(0), dF = T(0), aL = T(0), cL = T(0), dL = T(0);
  if (own) {
    T a0, b0, c0;
    row_coef<T>(sf[ps], s, n, am[s + 1], ap[s + 1], lc, a0, b0, c0);
    const T d0 = sd[ps];
    // operands of every row of the chunk are loaded up front (clamped to the
    // chunk so the loads are unconditional and leave the elimination chain)
    uint8_t fq_[MAXM];
    double amq_[MAXM], apq_[MAXM];
    T dq_[MAXM];
#pragma unroll
    for (int q = 1; q < MAXM; ++q) {
      const int qq = q < m ? q : m - 1;
      fq_[q] = sf[ps + qq];
      amq_[q] = am[s + qq + 1];
      apq_[q] = ap[s + qq + 1];
      dq_[q] = sd[ps + qq];
    }
#pragma unroll
    for (int q = 1; q < MAXM; ++q) {
      if (q < m) {
        T aq, bq, cq;
        row_coef<T>(fq_[q], s + q, n, amq_[q], apq_[q], lc, aq, bq, cq);
        const T dq = dq_[q];
        if (q == 1) {
          const T r = rcp_nr(bq);
          al[1] = aq * r; ga[1] = cq * r; de[1] = dq * r;
        } else {
          const T r = rcp_nr(bq - aq * ga[q - 1]);
          al[q] = -aq * al[q - 1] * r;
          ga[q] = cq * r;
          de[q] = (dq - aq * de[q - 1]) * r;
        }
        aL = al[q]; cL = ga[q]; dL = de[q];  // last row of the chunk
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
    aF = a0; bF = b0 - c0 * pa; cF = -c0 * pb; dF = d0 - c0 * pd;
  }
  // eliminate the L unknowns: L_l = dL - aL F_l - cL F_{l+1}, so each lane
  // holds one equation of a tridiagonal system in F_0 .. F_31
  T aLp = __shfl_up_sync(0xffffffffu, aL, 1);
  T cLp = __shfl_up_sync(0xffffffffu, cL, 1);
  T dLp = __shfl_up_sync(0xffffffffu, dL, 1);
  if (lane == 0) { aLp = T(0); cLp = T(0); dLp = T(0); }
  T A = -aF * aLp;
  T B = bF - aF * cLp - cF * aL;
  T Cc = -cF * cL;
  T D = dF - aF * dLp - cF * dL;
  if (!own) { A = T(0); B = T(1); Cc = T(0); D = T(0); }
  // parallel cyclic reduction over 32 equations, one reciprocal per step
#pragma unroll
  for (int t = 1; t < 32; t <<= 1) {
    const T ib = rcp_nr(B);
    T la = __shfl_up_sync(0xffffffffu, A, t), lc2 = __shfl_up_sync(0xffffffffu, Cc, t);
    T ld = __shfl_up_sync(0xffffffffu, D, t), lib = __shfl_up_sync(0xffffffffu, ib, t);
    T ra = __shfl_down_sync(0xffffffffu, A, t), rc = __shfl_down_sync(0xffffffffu, Cc, t);
    T rd = __shfl_down_sync(0xffffffffu, D, t), rib = __shfl_down_sync(0xffffffffu, ib, t);
    if (lane < t) { la = T(0); lc2 = T(0); ld = T(0); lib = T(0); }
    if (lane + t >= 32) { ra = T(0); rc = T(0); rd = T(0); rib = T(0); }
    const T k1 = A * lib, k2 = Cc * rib;
    const T nA = -la * k1, nC = -rc * k2;
    const T nB = B - lc2 * k1 - ra * k2;
    const T nD = D - ld * k1 - rd * k2;
    A = nA; Cc = nC; B = nB; D = nD;
  }
  const T xF = D / B;
  const T xFn = __shfl_down_sync(0xffffffffu, xF, 1);
  if (own) {
    const T xL = dL - aL * xF - cL * (lane + 1 < 32 ? xFn : T(0));
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
  static __device__ __forceinline__ dptr<double> x(const DevLevel &L) { return glob(L.x64); }
  static __device__ __forceinline__ dptr<double> rhs(const DevLevel &L) { return glob(L.rhs64); }
  static __device__ __forceinline__ dptr<double> res(const DevLevel &L) { return glob(L.res64); }
};
template <> struct PrecOf<float> {
  static __device__ __forceinline__ dptr<float> x(const DevLevel &L) { return glob(L.x32); }
  static __device__ __forceinline__ dptr<float> rhs(const DevLevel &L) { return glob(L.rhs32); }
  static __device__ __forceinline__ dptr<float> res(const DevLevel &L) { return glob(L.res32); }
};

// bytes of dynamic shared memory of the launch (checked builds bound the
// staging arrays by it)
__device__ __forceinline__ long long dyn_smem_bytes() {
#ifdef FG_CHECKED
  unsigned v;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
  return (long long)v;
#else
  return 0;
#endif
}

__host__ __device__ __forceinline__ int line_pad(int n) { return n + 33; }
__host__ __device__ __forceinline__ size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

// ------------------------------------------- register-staged line kernels
// M consecutive elements of a row (16-byte aligned start, see the field
// padding of the allocator) into registers.
template <typename T, int M, typename P>
__device__ __forceinline__ void load_run(T (&v)[M], const P &base, long long off) {
#ifdef FG_CHECKED
#pragma unroll
  for (int q = 0; q < M; ++q) v[q] = base[off + q];
#else
  static_assert((M * sizeof(T)) % 4 == 0, "run of at least 4 bytes");
  const T *src = &base[off];
  if constexpr ((M * sizeof(T)) % 16 == 0) {
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int u = 0; u < (int)(M * sizeof(T) / 16); ++u) {
      const uint4 w = s4[u];
      memcpy(&v[u * (16 / sizeof(T))], &w, 16);
    }
  } else if constexpr ((M * sizeof(T)) % 8 == 0) {
    const uint2 *s2 = reinterpret_cast<const uint2 *>(src);
#pragma unroll
    for (int u = 0; u < (int)(M * sizeof(T) / 8); ++u) {
      const uint2 w = s2[u];
      memcpy(&v[u * (8 / sizeof(T))], &w, 8);
    }
  } else {
    const unsigned w = *reinterpret_cast<const unsigned *>(src);
    memcpy(&v[0], &w, 4);
  }
#endif
}

template <typename T, int M, typename P>
__device__ __forceinline__ void store_run(const P &base, long long off, const T (&v)[M], int valid) {
#ifndef FG_CHECKED
  if (valid >= M) {
    T *dst = &base[off];
    if constexpr ((M * sizeof(T)) % 16 == 0) {
      uint4 *d4 = reinterpret_cast<uint4 *>(dst);
#pragma unroll
      for (int u = 0; u < (int)(M * sizeof(T) / 16); ++u) {
        uint4 w;
        memcpy(&w, &v[u * (16 / sizeof(T))], 16);
        d4[u] = w;
      }
      return;
    }
  }
#endif
#pragma unroll
  for (int q = 0; q < M; ++q)
    if (q < valid) base[off + q] = v[q];
}

// Parallel cyclic reduction of W equations A x_{l-1} + B x_l + C x_{l+1}
// = D held one per lane of a W-lane segment of the warp (sl = lane within
// the segment; A of the first and C of the last are zero); returns x of
// this lane.  One reciprocal per step (rcp_nr).
template <typename T, int W>
__device__ __forceinline__ T pcr_seg(T A, T B, T Cc, T D, int sl) {
#pragma unroll
  for (int t = 1; t < W; t <<= 1) {
    const T ib = rcp_nr(B);
    T la = __shfl_up_sync(0xffffffffu, A, t, W), lc2 = __shfl_up_sync(0xffffffffu, Cc, t, W);
    T ld = __shfl_up_sync(0xffffffffu, D, t, W), lib = __shfl_up_sync(0xffffffffu, ib, t, W);
    T ra = __shfl_down_sync(0xffffffffu, A, t, W), rc = __shfl_down_sync(0xffffffffu, Cc, t, W);
    T rd = __shfl_down_sync(0xffffffffu, D, t, W), rib = __shfl_down_sync(0xffffffffu, ib, t, W);
    if (sl < t) { la = T(0); lc2 = T(0); ld = T(0); lib = T(0); }
    if (sl + t >= W) { ra = T(0); rc = T(0); rd = T(0); rib = T(0); }
    const T k1 = A * lib, k2 = Cc * rib;
    const T nA = -la * k1, nC = -rc * k2;
    const T nB = B - lc2 * k1 - ra * k2;
    const T nD = D - ld * k1 - rd * k2;
    A = nA; Cc = nC; B = nB; D = nD;
  }
  return D / B;
}

// One chunk of M consecutive rows of a line, held by one thread: the rows'
// right-hand sides d (held rows: their current value) and masks mk (0 for
// held rows) are given; the row coefficients come from the mask and the
// axis coefficients am/ap.  Eliminates the chunk down and up (partition
// method): afterwards x_u = d_u - al_u F - ga_u L for 0 < u < M-1, with F
// = x_0 and L = x_{M-1}, and the chunk's F/L equations are
//     aF L_prev + bF F + cF L = dF,   L = dL - aL F - cL F_next.
// Rows r >= n (past the line end) are identities.
template <typename T, int M, typename PA>
__device__ __forceinline__ void chunk_eliminate(int r0, int n, const uint8_t (&mk)[M], T (&d)[M],
                                                T (&al)[M], T (&ga)[M], const PA &am_,
                                                const PA &ap_, const LineCoef &lc, T &aF, T &bF,
                                                T &cF, T &dF, T &aL, T &cL, T &dL) {
  T a0 = T(0), b0 = T(1), c0 = T(0), d0 = T(0);
#pragma unroll
  for (int u = 0; u < M; ++u) {
    const int r = r0 + u;
    T a = T(0), b = T(1), c = T(0), dd = T(0);
    if (r < n) {
      const uint8_t m8 = mk[u];
      dd = d[u];
      if (m8 & 64) {
        const double am = am_[1 + r], ap = ap_[1 + r];
        double diag = -lc.tdir;
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if ((m8 >> lc.qt[t]) & 1) diag -= lc.tq[t];
        const bool cm = (m8 >> lc.qm) & 1, cp = (m8 >> lc.qp) & 1;
        if (cm) diag -= am; else if (r == 0 && lc.dirm) diag -= 2.0 * am;
        if (cp) diag -= ap; else if (r == n - 1 && lc.dirp) diag -= 2.0 * ap;
        a = cm ? (T)am : T(0);
        c = cp ? (T)ap : T(0);
        b = (T)diag;
      }
    }
    if (u == 0) {
      a0 = a; b0 = b; c0 = c; d0 = dd;
    } else if (u == 1) {
      const T rr = rcp_nr(b);
      al[1] = a * rr; ga[1] = c * rr; d[1] = dd * rr;
    } else {
      const T rr = rcp_nr(b - a * ga[u - 1]);
      al[u] = -a * al[u - 1] * rr;
      ga[u] = c * rr;
      d[u] = (dd - a * d[u - 1]) * rr;
    }
  }
  aL = al[M - 1]; cL = ga[M - 1]; dL = d[M - 1];
  T pa = T(0), pb = T(-1), pd = T(0);
#pragma unroll
  for (int u = M - 2; u >= 1; --u) {
    const T nd = d[u] - ga[u] * pd;
    const T na = al[u] - ga[u] * pa;
    const T nb = -ga[u] * pb;
    al[u] = na; ga[u] = nb; d[u] = nd;
    pa = na; pb = nb; pd = nd;
  }
  aF = a0; bF = b0 - c0 * pa; cF = -c0 * pb; dF = d0 - c0 * pd;
}

// chunk_eliminate with coefficients in T (LineCoefT) and the couplings
// along the line staged as am_[r], ap_[r] for line row r (0-based).
// REG: every row but the line's first and last has all six faces coupled
// and is active (a regular tile), so those rows skip the mask decode
template <typename T, int M, typename LC, bool REG = false>
__device__ __forceinline__ void chunk_eliminate_t(int r0, int n, const uint8_t (&mk)[M], T (&d)[M],
                                                  T (&al)[M], T (&ga)[M], const T *am_, const T *ap_,
                                                  const LC &lc, T &aF, T &bF, T &cF, T &dF, T &aL,
                                                  T &cL, T &dL) {
  T a0 = T(0), b0 = T(1), c0 = T(0), d0 = T(0);
#pragma unroll
  for (int u = 0; u < M; ++u) {
    const int r = r0 + u;
    T a = T(0), b = T(1), c = T(0), dd = T(0);
    if (r < n) {
      const uint8_t m8 = mk[u];
      dd = d[u];
      if (REG && r != 0 && r != n - 1) {
        const T am = am_[r], ap = ap_[r];
        T diag = -lc.tdir;
#pragma unroll
        for (int t = 0; t < 4; ++t) diag -= lc.tq[t];
        diag -= am;
        diag -= ap;
        a = am;
        c = ap;
        b = diag;
      } else if (m8 & 64) {
        const T am = am_[r], ap = ap_[r];
        T diag = -lc.tdir;
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if ((m8 >> LC::qt(t)) & 1) diag -= lc.tq[t];
        const bool cm = (m8 >> LC::qm) & 1, cp = (m8 >> LC::qp) & 1;
        if (cm) diag -= am; else if (r == 0 && lc.dirm) diag -= T(2) * am;
        if (cp) diag -= ap; else if (r == n - 1 && lc.dirp) diag -= T(2) * ap;
        a = cm ? am : T(0);
        c = cp ? ap : T(0);
        b = diag;
      }
    }
    if (u == 0) {
      a0 = a; b0 = b; c0 = c; d0 = dd;
    } else if (u == 1) {
      const T rr = rcp_nr(b);
      al[1] = a * rr; ga[1] = c * rr; d[1] = dd * rr;
    } else {
      const T rr = rcp_nr(b - a * ga[u - 1]);
      al[u] = -a * al[u - 1] * rr;
      ga[u] = c * rr;
      d[u] = (dd - a * d[u - 1]) * rr;
    }
  }
  aL = al[M - 1]; cL = ga[M - 1]; dL = d[M - 1];
  T pa = T(0), pb = T(-1), pd = T(0);
#pragma unroll
  for (int u = M - 2; u >= 1; --u) {
    const T nd = d[u] - ga[u] * pd;
    const T na = al[u] - ga[u] * pa;
    const T nb = -ga[u] * pb;
    al[u] = na; ga[u] = nb; d[u] = nd;
    pa = na; pb = nb; pd = nd;
  }
  aF = a0; bF = b0 - c0 * pa; cF = -c0 * pb; dF = d0 - c0 * pd;
}

// chunk_eliminate with the per-row state in shared memory: row u of the
// calling thread's chunk at sal[u*st], sga[u*st], sd[u*st] (sd holds the
// right-hand sides on entry); am_[r], ap_[r] couple line row r (0-based) to
// rows r-1 and r+1.
template <typename T, int M, typename LC>
__device__ __forceinline__ void chunk_eliminate_smem(int r0, int n, const uint8_t (&mk)[M], T *sd, T *sal,
                                                     T *sga, int st, const T *am_, const T *ap_,
                                                     const LC &lc, T &aF, T &bF, T &cF, T &dF,
                                                     T &aL, T &cL, T &dL) {
  T a0 = T(0), b0 = T(1), c0 = T(0), d0 = T(0);
  T alp = T(0), gap = T(0), dp = T(0);
#pragma unroll
  for (int u = 0; u < M; ++u) {
    const int r = r0 + u;
    T a = T(0), b = T(1), c = T(0), dd = T(0);
    if (r < n) {
      const uint8_t m8 = mk[u];
      dd = sd[u * st];
      if (m8 & 64) {
        const T am = am_[r], ap = ap_[r];
        T diag = -lc.tdir;
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if ((m8 >> LC::qt(t)) & 1) diag -= lc.tq[t];
        const bool cm = (m8 >> LC::qm) & 1, cp = (m8 >> LC::qp) & 1;
        if (cm) diag -= am; else if (r == 0 && lc.dirm) diag -= T(2) * am;
        if (cp) diag -= ap; else if (r == n - 1 && lc.dirp) diag -= T(2) * ap;
        a = cm ? am : T(0);
        c = cp ? ap : T(0);
        b = diag;
      }
    }
    if (u == 0) {
      a0 = a; b0 = b; c0 = c; d0 = dd;
    } else {
      const T rr = u == 1 ? rcp_nr(b) : rcp_nr(b - a * gap);
      const T nal = u == 1 ? a * rr : -a * alp * rr;
      const T nga = c * rr;
      const T nd = u == 1 ? dd * rr : (dd - a * dp) * rr;
      sal[u * st] = nal; sga[u * st] = nga; sd[u * st] = nd;
      alp = nal; gap = nga; dp = nd;
    }
  }
  aL = alp; cL = gap; dL = dp;
  T pa = T(0), pb = T(-1), pd = T(0);
#pragma unroll
  for (int u = M - 2; u >= 1; --u) {
    const T du = sd[u * st], au = sal[u * st], gu = sga[u * st];
    const T nd = du - gu * pd;
    const T na = au - gu * pa;
    const T nb = -gu * pb;
    sal[u * st] = na; sga[u * st] = nb; sd[u * st] = nd;
    pa = na; pb = nb; pd = nd;
  }
  aF = a0; bF = b0 - c0 * pa; cF = -c0 * pb; dF = d0 - c0 * pd;
}

// Zebra x-line relaxation, lines (j,k) with (j+k)%2 == color, W lanes per
// line (32/W lines per warp).  Lane l of a line owns rows [M l, M l + M),
// loaded straight into registers with 16-byte loads (rows past the line
// end are identity equations), eliminates them down and up, and the W
// chunk-first unknowns are solved by PCR across the line's lanes.  One
// pass over rhs, mask, the line's own values and its four neighbour
// lines; no shared memory.
template <typename T, int M, int W>
__global__ void __launch_bounds__(XL_WARPS * 32, 1)
k_xline_reg(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, int color, T omega) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sl = lane % W;
  const int nyh = (L.ny + 1) >> 1;
  const int q = (lb * XL_WARPS + warp) * (32 / W) + lane / W;
  int k = 1 + q / nyh;
  const int jj = q % nyh;
  int j = ((((1 + k) & 1) == color) ? 1 : 2) + 2 * jj;
  const bool line_ok = k <= L.nz && j <= L.ny;
  if (!line_ok) { k = 1; j = 1; }  // idle segment: identity rows, no loads or stores
  const int n = L.nx;
  auto x = PrecOf<T>::x(L);
  auto rhs = PrecOf<T>::rhs(L);
  const LineCoef lc = line_coef(L, 0, 1, j, k);
  const long long row = L.sy * j + L.sz * k + 1;  // cell i = 1
  const int r0 = sl * M;
  const bool any = line_ok && r0 < n;
  T d[M], al[M], ga[M];
  uint8_t mk[M];
#pragma unroll
  for (int u = 0; u < M; ++u) { d[u] = T(0); mk[u] = 0; }
  const bool iso_line = lc.tdir == 0.0 && !lc.dirm && !lc.dirp;
  if (any) {
    // every load of the chunk is issued before the first use
    T nb[4][M], xv[M];
    load_run<T, M>(d, rhs, row + r0);
    load_run<uint8_t, M>(mk, glob(L.mask), row + r0);
#pragma unroll
    for (int t = 0; t < 4; ++t) load_run<T, M>(nb[t], x, row + r0 + lc.to[t]);
    load_run<T, M>(xv, x, row + r0);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const T cq = (T)lc.tq[t];
#pragma unroll
      for (int u = 0; u < M; ++u)
        if ((mk[u] >> lc.qt[t]) & 1) d[u] -= cq * nb[t][u];
    }
#pragma unroll
    for (int u = 0; u < M; ++u) {
      const bool held = !(mk[u] & 64) || (((mk[u] & 63) == 0) && iso_line);
      if (held) { d[u] = xv[u]; mk[u] = 0; }
    }
  }
  T aF, bF, cF, dF, aL, cL, dL;
  chunk_eliminate<T, M>(r0, any ? n : r0, mk, d, al, ga, L.amx, L.apx, lc, aF, bF, cF, dF, aL, cL, dL);
  // reduced system in the chunk-first unknowns F_l
  T aLp = __shfl_up_sync(0xffffffffu, aL, 1, W);
  T cLp = __shfl_up_sync(0xffffffffu, cL, 1, W);
  T dLp = __shfl_up_sync(0xffffffffu, dL, 1, W);
  if (sl == 0) { aLp = T(0); cLp = T(0); dLp = T(0); }
  const T xF = pcr_seg<T, W>(-aF * aLp, bF - aF * cLp - cF * aL, -cF * cL, dF - aF * dLp - cF * dL, sl);
  const T xFn = __shfl_down_sync(0xffffffffu, xF, 1, W);
  if (!any) return;
  const T xL = dL - aL * xF - cL * (sl + 1 < W ? xFn : T(0));
  T out[M];
  out[0] = xF;
#pragma unroll
  for (int u = 1; u < M - 1; ++u) out[u] = d[u] - al[u] * xF - ga[u] * xL;
  out[M - 1] = xL;
  if (omega != T(1)) {
    T xo[M];
    load_run<T, M>(xo, x, row + r0);
#pragma unroll
    for (int u = 0; u < M; ++u) out[u] = xo[u] + omega * (out[u] - xo[u]);
  }
  const int valid = n - r0 < M ? n - r0 : M;
  store_run<T, M>(x, row + r0, out, valid);
}

// A lane's chunk of M values (or M mask bytes) moved between registers and
// shared memory as 16-byte (8-byte) pieces: with the chunk stride a multiple
// of 16 bytes, 8 lanes of a phase hit distinct bank groups.
template <typename T, int M>
__device__ __forceinline__ void lds_chunk(const unsigned char *p, T (&v)[M]) {
  constexpr int W = 16 / sizeof(T);
#pragma unroll
  for (int c = 0; c < M / W; ++c) {
    const uint4 q = reinterpret_cast<const uint4 *>(p)[c];
    memcpy(&v[c * W], &q, 16);
  }
}
template <typename T, int M>
__device__ __forceinline__ void sts_chunk(unsigned char *p, const T (&v)[M]) {
  constexpr int W = 16 / sizeof(T);
#pragma unroll
  for (int c = 0; c < M / W; ++c) {
    uint4 q;
    memcpy(&q, &v[c * W], 16);
    reinterpret_cast<uint4 *>(p)[c] = q;
  }
}
template <int M>
__device__ __forceinline__ void lds_mask(const unsigned char *p, uint8_t (&m)[M]) {
  if constexpr (M == 8) {
    const uint2 q = *reinterpret_cast<const uint2 *>(p);
    memcpy(m, &q, 8);
  } else {
#pragma unroll
    for (int c = 0; c < M / 16; ++c) {
      const uint4 q = reinterpret_cast<const uint4 *>(p)[c];
      memcpy(&m[16 * c], &q, 16);
    }
  }
}

// Zebra x-line relaxation for lines of 129..1024 cells: one warp per line,
// XS_WARPS lines per block.  Consecutive lanes load consecutive 4-cell
// pieces of the line (rhs, mask, own values, four neighbour lines: every
// load instruction reads whole 32-byte sectors) and form each row's
// right-hand side; the rows go to shared memory in chunk order (lane l's M
// rows at a padded stride), each lane eliminates its chunk in registers,
// the 32 chunk-first unknowns are solved by PCR, and the results return
// through shared memory to coalesced stores.
constexpr int XS_WARPS = 4;
constexpr int XS_PIECE = 4;  // cells per piece of the coalesced phases
template <typename T, int M>
struct XsLayout {
  static constexpr int CT = M * (int)sizeof(T) + 16;  // padded chunk of T
  static constexpr int LT = 32 * CT;                  // right-hand sides, then results
  static constexpr int PER_WARP = LT + 32 * M;        // + mask bytes in line order
};

// Line (j,k) of warp `warp` in block `lb` of a level's x sweep; false when
// the warp has no line.  Colour 1 walks the k planes backward, so its first
// blocks meet the planes the colour-0 launch left in L2.
__device__ __forceinline__ bool xs_line(const DevLevel &L, int lb, int warp, int color, int &j, int &k) {
  const int nyh = (L.ny + 1) >> 1;
  const int q = lb * XS_WARPS + warp;
  k = 1 + q / nyh;
  const int jj = q % nyh;
  if (k > L.nz) return false;
  if (color == 1) k = L.nz + 1 - k;
  j = ((((1 + k) & 1) == color) ? 1 : 2) + 2 * jj;
  return j <= L.ny;
}

template <typename T, int M>
__global__ void __launch_bounds__(XS_WARPS * 32)
k_xline_smem(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, int color, T omega) {
  using LY = XsLayout<T, M>;
  using LC = LineCoefT<T, 0>;
  constexpr int P = XS_PIECE;
  extern __shared__ __align__(16) unsigned char xs_smem[];
  // couplings along x (one level per block), row r at r + r / M: lane l's
  // chunk starts at l (M + 1), so the lanes' reads fall in distinct banks
  __shared__ T s_am[32 * (M + 1)], s_ap[32 * (M + 1)];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  const int n = L.nx;
  for (int r = threadIdx.x; r < n; r += XS_WARPS * 32) {
    s_am[r + r / M] = (T)glob(L.amx)[1 + r];
    s_ap[r + r / M] = (T)glob(L.apx)[1 + r];
  }
  __syncthreads();
  int j, k;
  if (!xs_line(L, lb, warp, color, j, k)) return;  // uniform over the warp
  auto x = PrecOf<T>::x(L);
  auto rhs = PrecOf<T>::rhs(L);
  const LC lc(line_coef(L, 0, 1, j, k));
  const bool iso_line = lc.iso();
  const long long row = L.sy * j + L.sz * k + 1;  // cell i = 1
  const long long to[4] = {-L.sy, L.sy, -L.sz, L.sz};
  unsigned char *sw = xs_smem + (size_t)warp * LY::PER_WARP;
  unsigned char *s_d = sw, *s_mk = sw + LY::LT;
  // right-hand sides of the line's rows, piece by piece (pieces past the
  // line end are not read by the elimination)
#pragma unroll
  for (int c = 0; c < M / P; ++c) {
    const int e = (lane + 32 * c) * P;
    if (e < n) {
      T rv[P], xo[P], dv[P];
      uint8_t m4[P];
      load_run<T, P>(rv, rhs, row + e);
      load_run<T, P>(xo, x, row + e);
      load_run<uint8_t, P>(m4, glob(L.mask), row + e);
      T nb[4][P];
#pragma unroll
      for (int t = 0; t < 4; ++t) load_run<T, P>(nb[t], x, row + e + to[t]);
#pragma unroll
      for (int v = 0; v < P; ++v) {
        uint8_t m8 = m4[v];
        T acc = rv[v];
#pragma unroll
        for (int t = 0; t < 4; ++t) acc -= ((m8 >> LC::qt(t)) & 1) ? lc.tq[t] * nb[t][v] : T(0);
        const bool held = !(m8 & 64) || (((m8 & 63) == 0) && iso_line);
        if (held) { acc = xo[v]; m8 = 0; }
        dv[v] = acc;
        m4[v] = m8;
      }
      sts_chunk<T, P>(s_d + (e / M) * LY::CT + (e % M) * sizeof(T), dv);
      unsigned w4;
      memcpy(&w4, m4, 4);
      *reinterpret_cast<unsigned *>(s_mk + e) = w4;
    }
  }
  __syncwarp();
  const int r0 = lane * M;
  T d[M], al[M], ga[M];
  uint8_t mk[M];
  lds_chunk<T, M>(s_d + lane * LY::CT, d);
  lds_mask<M>(s_mk + lane * M, mk);
  T aF, bF, cF, dF, aL, cL, dL;
  chunk_eliminate_t<T, M>(r0, r0 < n ? n : r0, mk, d, al, ga, s_am + lane, s_ap + lane, lc, aF, bF, cF, dF,
                          aL, cL, dL);
  T aLp = __shfl_up_sync(0xffffffffu, aL, 1);
  T cLp = __shfl_up_sync(0xffffffffu, cL, 1);
  T dLp = __shfl_up_sync(0xffffffffu, dL, 1);
  if (lane == 0) { aLp = T(0); cLp = T(0); dLp = T(0); }
  const T xF = pcr_seg<T, 32>(-aF * aLp, bF - aF * cLp - cF * aL, -cF * cL, dF - aF * dLp - cF * dL, lane);
  const T xFn = __shfl_down_sync(0xffffffffu, xF, 1);
  const T xL = dL - aL * xF - cL * (lane + 1 < 32 ? xFn : T(0));
#pragma unroll
  for (int u = 0; u < M; ++u) d[u] = u == 0 ? xF : (u == M - 1 ? xL : d[u] - al[u] * xF - ga[u] * xL);
  __syncwarp();
  sts_chunk<T, M>(s_d + lane * LY::CT, d);
  __syncwarp();
#pragma unroll
  for (int c = 0; c < M / P; ++c) {
    const int e = (lane + 32 * c) * P;
    if (e < n) {
      T v[P];
      lds_chunk<T, P>(s_d + (e / M) * LY::CT + (e % M) * sizeof(T), v);
      if (omega != T(1)) {
        T xo[P];
        load_run<T, P>(xo, x, row + e);
#pragma unroll
        for (int q = 0; q < P; ++q) v[q] = xo[q] + omega * (v[q] - xo[q]);
      }
      store_run<T, P>(x, row + e, v, n - e);
    }
  }
}

// Zebra line relaxation along y (AXIS 1, lines (i,k), colour (i+k)%2) or z
// (AXIS 2, lines (i,j), colour (i+j)%2).  A block takes the 32 lines of
// one colour in a 64-cell i-tile (lane l: i = i0 + par + 2l, so every
// load of a warp spans 64 consecutive cells) and CH warps, warp w holding
// rows [M w, M w + M) of all 32 lines in registers.  Each thread
// eliminates its chunk down and up; the CH chunk equations of a line go
// through shared memory and one thread per line solves them (Thomas),
// then every thread back-substitutes its rows.
constexpr int YZ_MAXROWS = 256;  // longest line of k_yzline_reg (M 16 x CH 16)
constexpr int YP_LINES = 8;      // lines per block of k_yzline_pcr
constexpr int YP_MINROWS = 65;   // shortest line of k_yzline_pcr
template <typename T>
struct ChunkEq { T a, b, c, d; };
template <typename T>
struct Eq3 { T a, c, d; };  // a x_prev + x + c x_next = d

template <typename T, int M, int CH, int AXIS>
__global__ void __launch_bounds__(CH * 32, (sizeof(T) == 4 && CH == 16) ? (M <= 8 ? 3 : 2) : 1)
k_yzline_reg(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, int color, T omega) {
  using LC = LineCoefT<T, AXIS>;
  __shared__ ChunkEq<T> s_eq[CH][32];
  __shared__ T s_f[CH + 1][32];   // chunk-first unknowns
  __shared__ T s_am[M * CH], s_ap[M * CH];  // couplings along the line
  extern __shared__ __align__(16) unsigned char yz_smem[];
  constexpr int NT = CH * 32;     // per-row stride of the state arrays
  T *s_d = reinterpret_cast<T *>(yz_smem);
  T *s_al = s_d + M * NT;
  T *s_ga = s_al + M * NT;
  const int tid = threadIdx.x;
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  const int ntx = (L.nx + 63) >> 6;
  const int ti = lb % ntx;
  const int o = 1 + lb / ntx;  // k for AXIS 1, j for AXIS 2
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i0 = 1 + 64 * ti;
  const int par = (color + i0 + o) & 1;
  const int i = i0 + par + 2 * lane;
  const bool valid = i <= L.nx;
  const int n = AXIS == 1 ? L.ny : L.nz;
  const long long ls = AXIS == 1 ? L.sy : L.sz;  // row stride along the line
  const long long os = AXIS == 1 ? L.sz : L.sy;  // stride of the fixed index
  auto x = PrecOf<T>::x(L);
  auto rhs = PrecOf<T>::rhs(L);
  const LC lc(line_coef(L, AXIS, valid ? i : L.nx, AXIS == 1 ? 1 : o, AXIS == 1 ? o : 1));
  const long long base = (long long)(valid ? i : L.nx) + os * o;  // row index 0 of the line
  const int r0 = w * M;
  const bool any = valid && r0 < n;
  uint8_t mk[M];
  const bool iso_line = lc.iso();
  {
    auto am = AXIS == 1 ? L.amy : L.amz;
    auto ap = AXIS == 1 ? L.apy : L.apz;
    for (int r = tid; r < n; r += NT) { s_am[r] = (T)am[1 + r]; s_ap[r] = (T)ap[1 + r]; }
  }
  __syncthreads();
  // all loads of a row are issued unconditionally (none waits on the mask)
#pragma unroll
  for (int u = 0; u < M; ++u) {
    const int r = r0 + u;
    T dv = T(0);
    mk[u] = 0;
    if (any && r < n) {
      const long long id = base + ls * (r + 1);
      uint8_t m8 = glob(L.mask)[id];
      const T rv = rhs[id];
      const T xv = x[id];
      T nb[4];
      nb[0] = x[id - 1];
      nb[1] = x[id + 1];
      nb[2] = x[id - os];
      nb[3] = x[id + os];
      T acc = rv;
#pragma unroll
      for (int t = 0; t < 4; ++t) acc -= ((m8 >> LC::qt(t)) & 1) ? lc.tq[t] * nb[t] : T(0);
      const bool held = !(m8 & 64) || (((m8 & 63) == 0) && iso_line);
      if (held) { acc = xv; m8 = 0; }
      dv = acc;
      mk[u] = m8;
    }
    s_d[u * NT + tid] = dv;
  }
  T aF, bF, cF, dF, aL, cL, dL;
  chunk_eliminate_smem<T, M>(r0, any ? n : r0, mk, s_d + tid, s_al + tid, s_ga + tid, NT,
                             s_am, s_ap, lc, aF, bF, cF, dF, aL, cL, dL);
  __syncthreads();
  {
    T aLp = T(0), cLp = T(0), dLp = T(0);
    if (w > 0) {  // last-row equation of the previous chunk (row M-1 is not touched upward)
      const int tp = tid - 32;
      aLp = s_al[(M - 1) * NT + tp]; cLp = s_ga[(M - 1) * NT + tp]; dLp = s_d[(M - 1) * NT + tp];
    }
    ChunkEq<T> e;
    e.a = -aF * aLp;
    e.b = bF - aF * cLp - cF * aL;
    e.c = -cF * cL;
    e.d = dF - aF * dLp - cF * dL;
    s_eq[w][lane] = e;
  }
  __syncthreads();
  if (w == 0) {
    // Thomas over the chunk equations of line `lane` (chunks past the line
    // end are identities); the forward sweep is kept in place
    T cprev = T(0), dprev = T(0);
    for (int q = 0; q < CH; ++q) {
      const ChunkEq<T> e = s_eq[q][lane];
      const T rr = rcp_nr(e.b - e.a * cprev);
      cprev = e.c * rr;
      dprev = (e.d - e.a * dprev) * rr;
      s_eq[q][lane].c = cprev;
      s_eq[q][lane].d = dprev;
    }
    T xn = T(0);
    for (int q = CH - 1; q >= 0; --q) {
      xn = s_eq[q][lane].d - s_eq[q][lane].c * xn;
      s_f[q][lane] = xn;
    }
    s_f[CH][lane] = T(0);
  }
  __syncthreads();
  if (!any) return;
  const T xF = s_f[w][lane];
  const T xFn = s_f[w + 1][lane];
  const T xL = dL - aL * xF - cL * xFn;
#pragma unroll
  for (int u = 0; u < M; ++u) {
    const int r = r0 + u;
    if (r >= n) break;
    T v = u == 0 ? xF : (u == M - 1 ? xL : s_d[u * NT + tid] - s_al[u * NT + tid] * xF - s_ga[u * NT + tid] * xL);
    const long long id = base + ls * (r + 1);
    if (omega != T(1)) v = x[id] + omega * (v - x[id]);
    x[id] = v;
  }
}

// ------------------------------------------------------- x-line kernel
// Lines (j,k) with (j+k)%2 == color; one warp per line.
template <typename T, int MAXM>
__global__ void __launch_bounds__(XL_WARPS * 32, 2)
k_xline(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, int color, T omega) {
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
  const size_t per = align16(np * sizeof(T)) + align16(np);
  const long long dyn = dyn_smem_bytes();
  dptr<T> sd = mkptr(reinterpret_cast<T *>(smem + per * warp),
                     (dyn - (long long)(per * warp)) / (long long)sizeof(T), K_SMEM_D);
  dptr<uint8_t> sf = mkptr(smem + per * warp + align16(np * sizeof(T)),
                           dyn - (long long)(per * warp + align16(np * sizeof(T))), K_SMEM_F);
  if (k > L.nz) return;
  const int j0 = (((1 + k) & 1) == color) ? 1 : 2;
  const int j = j0 + 2 * jj;
  if (j > L.ny) return;
  auto x = PrecOf<T>::x(L);
  auto rhs = PrecOf<T>::rhs(L);
  int P, base, rem;
  chunking(n, P, base, rem);
  const PadMap pm = padmap(base, rem);
  const LineCoef lc = line_coef(L, 0, 1, j, k);
  const long long row = L.sy * j + L.sz * k + 1;
  for (int r0 = lane; r0 < n; r0 += 128) {
    T d[4]; uint8_t f[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = r0 + 32 * u;
      if (r < n) stage<T>(L, row + r, lc, x, rhs, d[u], f[u]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = r0 + 32 * u;
      if (r < n) { const int pp = padpos(r, pm); sd[pp] = d[u]; sf[pp] = f[u]; }
    }
  }
  __syncwarp();
  warp_solve<T, MAXM>(n, L.amx, L.apx, lc, sd, sf, lane);
  for (int r = lane; r < n; r += 32) {
    const int pp = padpos(r, pm);
    if (sf[pp] & 64) {
      const long long id = row + r;
      x[id] = (omega == T(1)) ? sd[pp] : x[id] + omega * (sd[pp] - x[id]);
    }
  }
}

// ----------------------------------------------------- y/z-line kernel
// AXIS 1: lines (i,k) along j, colour (i+k)%2, tiles of 16 i at fixed k.
// AXIS 2: lines (i,j) along k, colour (i+j)%2, tiles of 16 i at fixed j.
// The 8 lines of the colour in a tile are staged together (cell e of the
// tile: line slot e%8, row e/8), then one warp solves each line.
template <typename T, int MAXM, int AXIS>
__global__ void __launch_bounds__(YZ_WARPS * 32, 2)
k_yzline(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, int color, T omega) {
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
  const long long dyn = dyn_smem_bytes();
  const size_t fo = align16((size_t)YZ_WARPS * lstride * sizeof(T));
  dptr<T> sd = mkptr(reinterpret_cast<T *>(smem), (long long)fo / (long long)sizeof(T), K_SMEM_D);
  dptr<uint8_t> sf = mkptr(smem + fo, dyn - (long long)fo, K_SMEM_F);
  const int il0 = (color + i0 + o) & 1;  // tile-local i of the first line of this colour
  auto x = PrecOf<T>::x(L);
  auto rhs = PrecOf<T>::rhs(L);
  int P, base, rem;
  chunking(n, P, base, rem);
  const PadMap pm = padmap(base, rem);
  const int tid = threadIdx.x;
  const int total = YZ_WARPS * n;
  constexpr int NT = YZ_WARPS * 32;
  {
    // each thread stages one line (slot fixed per thread) for rows r0, r0+2, ...
    const int slot = tid % YZ_WARPS;
    const int i = i0 + il0 + 2 * slot;
    const bool valid = i <= L.nx;
    const LineCoef lc = line_coef(L, AXIS, valid ? i : L.nx, AXIS == 1 ? 1 : o, AXIS == 1 ? o : 1);
    const long long base_id = i + os * o;
    for (int e0 = tid; e0 < total; e0 += 4 * NT) {
      T d[4]; uint8_t f[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * NT;
        if (valid && e < total) stage<T>(L, base_id + ls * (e / YZ_WARPS + 1), lc, x, rhs, d[u], f[u]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = e0 + u * NT;
        if (valid && e < total) {
          const int pp = slot * lstride + padpos(e / YZ_WARPS, pm);
          sd[pp] = d[u]; sf[pp] = f[u];
        }
      }
    }
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  {
    const int i = i0 + il0 + 2 * warp;
    if (i <= L.nx) {
      const auto am = AXIS == 1 ? L.amy : L.amz;
      const auto ap = AXIS == 1 ? L.apy : L.apz;
      const LineCoef lc = line_coef(L, AXIS, i, AXIS == 1 ? 1 : o, AXIS == 1 ? o : 1);
      warp_solve<T, MAXM>(n, am, ap, lc, sd + warp * lstride, sf + warp * lstride, lane);
    }
  }
  __syncthreads();
  {
    const int slot = tid % YZ_WARPS;
    const int i = i0 + il0 + 2 * slot;
    if (i <= L.nx) {
      const long long base_id = i + os * o;
      for (int e = tid; e < total; e += NT) {
        const int r = e / YZ_WARPS;
        const int pp = slot * lstride + padpos(r, pm);
        if (sf[pp] & 64) {
          const long long id = base_id + ls * (r + 1);
          x[id] = (omega == T(1)) ? sd[pp] : x[id] + omega * (sd[pp] - x[id]);
        }
      }
    }
  }
}

int blocks_cells(const DevLevel &L) {
  return ((L.nx + CELL_BLOCK - 1) / CELL_BLOCK) * ((L.ny * L.nz + CELL_ROWS - 1) / CELL_ROWS);
}
// lanes per x line of k_xline_reg for a level set whose longest x line is maxn
int xline_lanes(int maxn) { return maxn <= 16 ? 4 : maxn <= 32 ? 8 : maxn <= 64 ? 16 : 32; }
// The line kernel family a level set's sweep along `axis` takes (LV_*):
// the requested one when it can take lines of maxn cells, else the
// default (the family measured fastest for that line length on the
// 512x256x256 case).
int line_variant(int axis, int maxn, int v) {
  if (axis == 0) {
    if (v == LV_XREG && maxn > 128) v = LV_DEFAULT;
    if (v == LV_XREG32 && maxn > 128) v = LV_DEFAULT;
    if (v == LV_XSMEM && maxn > 1024) v = LV_DEFAULT;
    if (v != LV_XREG && v != LV_XREG32 && v != LV_XSMEM) v = maxn <= 128 ? LV_XREG : LV_XSMEM;
    return v;
  }
  const bool pcr = v == LV_YPCR || v == LV_YPCRH || v == LV_YPCR4 || v == LV_YWAVE;
  if ((v == LV_YREG || pcr) && maxn > YZ_MAXROWS) v = LV_DEFAULT;
  if (pcr && v != LV_YPCR && v != LV_YWAVE && maxn < YP_MINROWS) v = LV_DEFAULT;
  if (v != LV_YREG && v != LV_YWARP && !pcr)
    v = (maxn >= YP_MINROWS && maxn <= YZ_MAXROWS) ? LV_YPCR : maxn <= YZ_MAXROWS ? LV_YREG : LV_YWARP;
  return v;
}
int blocks_xline(const DevLevel &L, int maxn, int variant) {
  const long long lines = (long long)((L.ny + 1) / 2) * L.nz;
  const int v = line_variant(0, maxn, variant);
  // k_xline_smem: one line per warp; k_xline_reg: 32 / lanes lines per warp
  const long long per_block = v == LV_XSMEM ? (long long)XS_WARPS
                              : v == LV_XREG32 ? (long long)XL_WARPS
                                               : (long long)XL_WARPS * (32 / xline_lanes(maxn));
  return (int)((lines + per_block - 1) / per_block);
}
int blocks_tile(const DevLevel &L, int axis, int maxn, int variant) {
  // i-tile of k_yzline_reg (64 cells), k_yzline_pcr (16) or k_yzline (16)
  const int v = line_variant(axis, maxn, variant);
  const int w = v == LV_YREG ? 64 : (v == LV_YPCR || v == LV_YPCRH || v == LV_YPCR4 || v == LV_YWAVE) ? 2 * YP_LINES : TILE_I;
  const int ntx = (L.nx + w - 1) / w;
  return ntx * (axis == 1 ? L.nz : L.ny);
}
// dynamic shared memory of a line launch: axis 0 uses the per-warp layout
// of k_xline, axes 1 and 2 the interleaved tile layout of k_yzline
size_t smem_line(int n, int tsize, int axis) {
  const int np = line_pad(n);
  if (axis == 0) {
    const size_t per = align16((size_t)np * tsize) + align16(np);
    return per * XL_WARPS;
  }
  const int lstride = np + 1;
  return align16((size_t)YZ_WARPS * lstride * tsize) + align16((size_t)YZ_WARPS * lstride);
}

template <typename T, int MAXM>
static cudaError_t launch_line(const Launch &Lr, int axis, int color, double omega, int maxn,
                               cudaStream_t s) {
  const T om = (T)omega;
  if (axis == 0) {
    const size_t sm = smem_line(maxn, sizeof(T), 0);
    auto kern = k_xline<T, MAXM>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<Lr.blocks, XL_WARPS * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, om);
    note_launches(1);
  } else {
    const size_t sm = smem_line(maxn, sizeof(T), axis);
    if (axis == 1) {
      auto kern = k_yzline<T, MAXM, 1>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      kern<<<Lr.blocks, YZ_WARPS * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, om);
      note_launches(1);
    } else {
      auto kern = k_yzline<T, MAXM, 2>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      kern<<<Lr.blocks, YZ_WARPS * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, om);
      note_launches(1);
    }
  }
  return cudaGetLastError();
}

// maxn: the longest line of this launch along `axis`
template <typename T, int M, int W>
static cudaError_t launch_xreg(const Launch &Lr, int color, double omega, cudaStream_t s) {
  k_xline_reg<T, M, W><<<Lr.blocks, XL_WARPS * 32, 0, s>>>(Lr.off, Lr.n, Lr.lev, color, (T)omega);
  note_launches(1);
  return cudaGetLastError();
}

// x loads of a tile: through L1, or (COH) from L2 only, for values other
// blocks of the same launch may have written since this launch began
template <bool COH, typename P>
__device__ __forceinline__ auto ldx(const P &x, long long i)
    -> std::remove_cv_t<std::remove_reference_t<decltype(x[i])>> {
  if constexpr (COH) return __ldcg(&x[i]);
  else return x[i];
}

// One tile of zebra y/z line relaxation in short chunks, for lines of
// YP_MINROWS..YZ_MAXROWS cells: YP_LINES lines of one colour in the i-tile
// ti (2 YP_LINES cells) of plane o (k for AXIS 1, j for AXIS 2); thread t
// takes line t % YP_LINES at i = i0 + par + 2 (t % YP_LINES) and chunk
// t / YP_LINES of CH chunks of M rows.  Every thread issues the loads of
// all its rows at once, eliminates its chunk in registers, the CH chunk
// equations of each line are solved by parallel cyclic reduction across
// the block (log2 CH steps through shared memory), and every thread
// back-substitutes its rows.
// NB > 0: the loads of all of a thread's rows are issued before the first
// row's arithmetic (the kernels give NB blocks per SM, more registers).
template <typename T, int M, int CH, int AXIS, int NB, bool COH, bool REG>
__device__ __forceinline__ void yz_pcr_tile_impl(const DevLevel &L, int ti, int o, int color, T omega) {
  using LC = LineCoefT<T, AXIS>;
  constexpr int NT = CH * YP_LINES;
  __shared__ T s_am[M * CH], s_ap[M * CH];  // couplings along the line
  // two buffers of unit-diagonal chunk equations (a, c, d); the last-row
  // equations of the chunks (aL, cL, dL) use the second before the reduction
  extern __shared__ __align__(16) unsigned char yp_smem[];
  auto s_eq = reinterpret_cast<Eq3<T>(*)[CH][YP_LINES]>(yp_smem);
  auto s_last = reinterpret_cast<T(*)[CH][YP_LINES]>(&s_eq[1][0][0]);
  const int tid = threadIdx.x;
  const int l = tid % YP_LINES, c = tid / YP_LINES;
  constexpr int TW = 2 * YP_LINES;  // cells of an i-tile
  const int i0 = 1 + TW * ti;
  const int par = (color + i0 + o) & 1;
  const int i = i0 + par + 2 * l;
  const bool valid = i <= L.nx;
  const int n = AXIS == 1 ? L.ny : L.nz;
  const long long ls = AXIS == 1 ? L.sy : L.sz;  // row stride along the line
  const long long os = AXIS == 1 ? L.sz : L.sy;  // stride of the fixed index
  auto x = glob(PrecOf<T>::x(L));
  auto rhs = glob(PrecOf<T>::rhs(L));
  {
    auto am = glob(AXIS == 1 ? L.amy : L.amz);
    auto ap = glob(AXIS == 1 ? L.apy : L.apz);
    for (int r = tid; r < n; r += NT) { s_am[r] = (T)am[1 + r]; s_ap[r] = (T)ap[1 + r]; }
  }
  auto mask = glob(L.mask);
  const LC lc(line_coef(L, AXIS, valid ? i : L.nx, AXIS == 1 ? 1 : o, AXIS == 1 ? o : 1));
  const bool iso_line = lc.iso();
  const long long base = (long long)(valid ? i : L.nx) + os * o;  // row index 0 of the line
  const int r0 = c * M;
  const bool any = valid && r0 < n;
  T d[M], al[M], ga[M];
  uint8_t mk[M];
  if constexpr (NB > 0) {
    // every load of the thread's rows first, then the arithmetic
    T rv[M], xv[M], nb[M][4];
#pragma unroll
    for (int u = 0; u < M; ++u) {
      const int r = r0 + u;
      mk[u] = 0;
      rv[u] = xv[u] = T(0);
      nb[u][0] = nb[u][1] = nb[u][2] = nb[u][3] = T(0);
      if (any && r < n) {
        const long long id = base + ls * (r + 1);
        mk[u] = mask[id];
        rv[u] = rhs[id];
        xv[u] = ldx<COH>(x, id);
        nb[u][0] = ldx<COH>(x, id - 1);
        nb[u][1] = ldx<COH>(x, id + 1);
        nb[u][2] = ldx<COH>(x, id - os);
        nb[u][3] = ldx<COH>(x, id + os);
      }
    }
#pragma unroll
    for (int u = 0; u < M; ++u) {
      uint8_t m8 = mk[u];
      T acc = rv[u];
#pragma unroll
      for (int t = 0; t < 4; ++t) acc -= ((m8 >> LC::qt(t)) & 1) ? lc.tq[t] * nb[u][t] : T(0);
      const bool held = !(m8 & 64) || (((m8 & 63) == 0) && iso_line);
      if (held) { acc = xv[u]; m8 = 0; }
      d[u] = (any && r0 + u < n) ? acc : T(0);
      mk[u] = (any && r0 + u < n) ? m8 : (uint8_t)0;
    }
  } else {
#pragma unroll
    for (int u = 0; u < M; ++u) {
      const int r = r0 + u;
      d[u] = T(0);
      mk[u] = 0;
      if (any && r < n) {
        const long long id = base + ls * (r + 1);
        const T rv = rhs[id];
        const T nb[4] = {ldx<COH>(x, id - 1), ldx<COH>(x, id + 1), ldx<COH>(x, id - os), ldx<COH>(x, id + os)};
        if (REG && r != 0 && r != n - 1) {
          // a regular tile's inner row: active, all faces coupled (no mask read)
          T acc = rv;
#pragma unroll
          for (int t = 0; t < 4; ++t) acc -= lc.tq[t] * nb[t];
          d[u] = acc;
          mk[u] = 0x7F;
        } else {
          uint8_t m8 = mask[id];
          const T xv = ldx<COH>(x, id);
          T acc = rv;
#pragma unroll
          for (int t = 0; t < 4; ++t) acc -= ((m8 >> LC::qt(t)) & 1) ? lc.tq[t] * nb[t] : T(0);
          const bool held = !(m8 & 64) || (((m8 & 63) == 0) && iso_line);
          if (held) { acc = xv; m8 = 0; }
          d[u] = acc;
          mk[u] = m8;
        }
      }
    }
  }
  __syncthreads();  // s_am, s_ap
  T aF, bF, cF, dF, aL, cL, dL;
  chunk_eliminate_t<T, M, LC, REG>(r0, any ? n : r0, mk, d, al, ga, s_am, s_ap, lc, aF, bF, cF, dF, aL, cL, dL);
  s_last[0][c][l] = aL;
  s_last[1][c][l] = cL;
  s_last[2][c][l] = dL;
  __syncthreads();
  {
    // equation of the chunk-first unknowns (previous chunk's last row
    // eliminated), normalised to a unit diagonal
    T aLp = T(0), cLp = T(0), dLp = T(0);
    if (c > 0) { aLp = s_last[0][c - 1][l]; cLp = s_last[1][c - 1][l]; dLp = s_last[2][c - 1][l]; }
    const T rb = rcp_nr(bF - aF * cLp - cF * aL);
    Eq3<T> e;
    e.a = -aF * aLp * rb;
    e.c = -cF * cL * rb;
    e.d = (dF - aF * dLp - cF * dL) * rb;
    __syncthreads();  // every s_last read before the buffers are written
    s_eq[0][c][l] = e;
  }
  __syncthreads();
  int buf = 0;
#pragma unroll
  for (int st = 1; st < CH; st <<= 1) {
    const Eq3<T> cur = s_eq[buf][c][l];
    Eq3<T> lo{T(0), T(0), T(0)}, hi{T(0), T(0), T(0)};
    if (c >= st) lo = s_eq[buf][c - st][l];
    if (c + st < CH) hi = s_eq[buf][c + st][l];
    const T rn = rcp_nr(T(1) - cur.a * lo.c - cur.c * hi.a);
    Eq3<T> ne;
    ne.a = -cur.a * lo.a * rn;
    ne.c = -cur.c * hi.c * rn;
    ne.d = (cur.d - cur.a * lo.d - cur.c * hi.d) * rn;
    s_eq[buf ^ 1][c][l] = ne;
    buf ^= 1;
    __syncthreads();
  }
  const T xF = s_eq[buf][c][l].d;
  const T xFn = c + 1 < CH ? s_eq[buf][c + 1][l].d : T(0);
  if (!any) return;
  const T xL = dL - aL * xF - cL * xFn;
#pragma unroll
  for (int u = 0; u < M; ++u) {
    const int r = r0 + u;
    if (r >= n) break;
    T v = u == 0 ? xF : (u == M - 1 ? xL : d[u] - al[u] * xF - ga[u] * xL);
    const long long id = base + ls * (r + 1);
    if (omega != T(1)) {
      const T xo = ldx<COH>(x, id);
      v = xo + omega * (v - xo);
    }
    x[id] = v;
  }
}


// A tile runs the regular form when its flag says so (every inner row of
// its 16 lines active with all faces coupled, set when the level's masks
// are built); otherwise the general one.  The loads-first variants always
// take the general form.
template <typename T, int M, int CH, int AXIS, int NB, bool COH>
__device__ __forceinline__ void yz_pcr_tile(const DevLevel &L, int ti, int o, int color, T omega) {
  if constexpr (NB > 0) {
    yz_pcr_tile_impl<T, M, CH, AXIS, NB, COH, false>(L, ti, o, color, omega);
  } else {
    const int ntx = (L.nx + 2 * YP_LINES - 1) / (2 * YP_LINES);
    const auto reg = AXIS == 1 ? L.regy : L.regz;
    if (reg && reg[ti + (long long)ntx * (o - 1)])
      yz_pcr_tile_impl<T, M, CH, AXIS, NB, COH, true>(L, ti, o, color, omega);
    else
      yz_pcr_tile_impl<T, M, CH, AXIS, NB, COH, false>(L, ti, o, color, omega);
  }
}

// Regular-tile flags of a level's y (AXIS 1) or z (AXIS 2) PCR tiles, one
// block per (tile, plane): 1 when all 16 cells of the tile lie inside the
// level and every row but the first and last of each of its lines is active
// with all six faces coupled.
template <int AXIS>
__global__ void k_reg_tiles(DevLevel L, uint8_t *flags) {
  const int ntx = (L.nx + 2 * YP_LINES - 1) / (2 * YP_LINES);
  const int ti = blockIdx.x % ntx, o = 1 + blockIdx.x / ntx;
  const int i0 = 1 + 2 * YP_LINES * ti;
  const int n = AXIS == 1 ? L.ny : L.nz;
  const long long ls = AXIS == 1 ? L.sy : L.sz, os = AXIS == 1 ? L.sz : L.sy;
  bool ok = i0 + 2 * YP_LINES - 1 <= L.nx;
  const int inner = n > 2 ? n - 2 : 0;
  for (int e = threadIdx.x; ok && e < 2 * YP_LINES * inner; e += blockDim.x) {
    const int i = i0 + e % (2 * YP_LINES), r = 1 + e / (2 * YP_LINES);
    const long long id = (long long)i + os * o + ls * (r + 1);
    if ((glob(L.mask)[id] & 0x7F) != 0x7F) ok = false;
  }
  ok = __syncthreads_and(ok);
  if (threadIdx.x == 0) flags[blockIdx.x] = ok ? 1 : 0;
}

cudaError_t reg_tiles(const DevLevel &L, uint8_t *flags_y, uint8_t *flags_z, cudaStream_t s) {
  const int ntx = (L.nx + 2 * YP_LINES - 1) / (2 * YP_LINES);
  if (ntx * L.nz > 0) k_reg_tiles<1><<<ntx * L.nz, 256, 0, s>>>(L, flags_y);
  if (ntx * L.ny > 0) k_reg_tiles<2><<<ntx * L.ny, 256, 0, s>>>(L, flags_z);
  note_launches(2);
  return cudaGetLastError();
}

// occupancy bound of the y/z PCR kernels: the resident threads per SM the
// register budget is sized for.  The kernels wait on their row loads, so
// more resident blocks at fewer registers pay until the spills grow:
// measured on the 512x256x256 case, FP32 256-thread tiles run fastest at
// 1536 threads (40 registers; 288 -> 242 us per level-0 y sweep against
// 1024), 128-thread tiles at 1280 (1536 spills more and is slower), FP64
// at 1024 (450 -> 387 us against 768)
template <typename T, int CH, int NB>
struct YpBound {
  static constexpr int budget = sizeof(T) == 4 ? (CH * YP_LINES >= 256 ? 1536 : 1280) : 1024;
  static constexpr int def = (budget / (CH * YP_LINES)) > 0 ? budget / (CH * YP_LINES) : 1;
  static constexpr int v = NB > 0 ? NB : def;
};

// one colour of a sweep: block -> (problem, tile, plane); a colour-1
// launch walks the planes backward, so its first blocks meet the planes
// the colour-0 launch left in L2
template <typename T, int M, int CH, int AXIS, int NB>
__global__ void __launch_bounds__(CH * YP_LINES, YpBound<T, CH, NB>::v)
k_yzline_pcr(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, int color, T omega) {
  const int p = find_entry(off, nent, blockIdx.x);
  const int lb = blockIdx.x - off[p];
  const DevLevel &L = levs[p];
  const int ntx = (L.nx + 2 * YP_LINES - 1) / (2 * YP_LINES);
  const int ti = lb % ntx;
  const int o = color == 1 ? (AXIS == 1 ? L.nz : L.ny) - lb / ntx : 1 + lb / ntx;
  yz_pcr_tile<T, M, CH, AXIS, NB, false>(L, ti, o, color, omega);
}

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Both colours of a y/z sweep in one launch.  Each block draws a ticket
// (in the order blocks start) that names one tile of one plane and colour;
// per problem the tickets run through the plane groups C0(0) .. C0(D),
// then C0(D+1), C1(0), C0(D+2), C1(1), ..., then C1(N-D-1) .. C1(N-1): a
// colour-1 plane comes D planes after the colour-0 plane it needs last,
// with D (at most N-1) such that D planes of tiles fill the GPU's resident
// blocks (`resident`), so a colour-1 tile rarely finds them unfinished.  A colour-0 tile
// reads only values no block of the launch writes before it; a colour-1
// tile of plane q waits until every colour-0 tile of planes q-1, q, q+1
// has stored its lines (a per-plane count), so it reads their new values
// (from L2, where the colour-0 tiles left them) and none of its writes
// reaches a colour-0 tile that still reads the old ones.  Every wait is on
// tiles with earlier tickets, whose blocks have started, so all waits end;
// each is also bounded, and one that gives up sets *err and goes on.
// wave: [0] the ticket counter, [2 + off[p] + q ntx] the colour-0 count of
// plane q of problem p; zeroed before each launch.
template <typename T, int M, int CH, int AXIS>
__global__ void __launch_bounds__(CH * YP_LINES, YpBound<T, CH, 0>::v)
k_yzline_wave(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, T omega, int *wave, int *err, int resident) {
  __shared__ int s_ticket;
  if (threadIdx.x == 0) s_ticket = atomicAdd(wave, 1);
  __syncthreads();
  const int t = s_ticket;
  const int p = find_entry(off, nent, t >> 1);
  const DevLevel &L = levs[p];
  const int ntx = (L.nx + 2 * YP_LINES - 1) / (2 * YP_LINES);
  const int N = AXIS == 1 ? L.nz : L.ny;
  const int u = t - 2 * off[p];
  const int g = u / ntx, ti = u % ntx;
  const int D = min(N - 1, (resident + ntx - 1) / ntx);
  const int npair = 2 * (N - 1 - D);  // groups of the interleaved middle
  int color, q;
  if (g <= D) { color = 0; q = g; }
  else if (g - (D + 1) < npair) {
    const int h = g - (D + 1);
    if (h & 1) { color = 1; q = h >> 1; }
    else { color = 0; q = D + 1 + (h >> 1); }
  } else { color = 1; q = N - 1 - D + (g - (D + 1) - npair); }
  int *cnt = wave + 2 + off[p];
  if (color == 1) {
    if (threadIdx.x == 0) {
      for (int dq = -1; dq <= 1; ++dq) {
        const int qq = q + dq;
        if (qq < 0 || qq >= N) continue;
        unsigned spins = 0;
        while (ld_acquire_gpu(cnt + qq * ntx) < ntx) {
          if (++spins > (1u << 22)) { atomicOr(err, 1); break; }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    __syncthreads();
    yz_pcr_tile<T, M, CH, AXIS, 0, true>(L, ti, 1 + q, 1, omega);
  } else {
    yz_pcr_tile<T, M, CH, AXIS, 0, false>(L, ti, 1 + q, 0, omega);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(cnt + q * ntx, 1);
  }
}

template <typename T, int M>
static cudaError_t launch_xsmem(const Launch &Lr, int color, double omega, cudaStream_t s) {
  const size_t sm = (size_t)XS_WARPS * XsLayout<T, M>::PER_WARP;
  auto kern = k_xline_smem<T, M>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  kern<<<Lr.blocks, XS_WARPS * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, (T)omega);
  note_launches(1);
  return cudaGetLastError();
}

template <typename T, int M, int CH, int NB = 0>
static cudaError_t launch_yzpcr(const Launch &Lr, int axis, int color, double omega, cudaStream_t s) {
  const size_t sm = (size_t)2 * CH * YP_LINES * sizeof(Eq3<T>);
  if (axis == 1) {
    auto kern = k_yzline_pcr<T, M, CH, 1, NB>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<Lr.blocks, CH * YP_LINES, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, (T)omega);
  } else {
    auto kern = k_yzline_pcr<T, M, CH, 2, NB>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<Lr.blocks, CH * YP_LINES, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, (T)omega);
  }
  note_launches(1);
  return cudaGetLastError();
}



__global__ void k_row_consts(int n, RowConstGeo g, const double *p_old, const double *dpdn_g, const double *dpdn_d,
                             int nd, double *c0) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int q = g.src[r];
  const double *dp = q < nd ? dpdn_d : dpdn_g;
  const double dpdn = dp ? dp[q < nd ? q : q - nd] : 0.0;
  double v = 0.0;
  if (g.fb[r]) {
    double num = 0.0, den = 0.0;
    for (int t = 0; t < 8; ++t) {
      const long long id = g.fid[8 * (long long)r + t];
      if (id < 0) continue;
      const double w = g.fw[8 * (long long)r + t];
      den += w;
      num += w * (p_old ? p_old[id] : 0.0);
    }
    v = num / den;
  }
  v += g.a[r] * dpdn;
  v += dpdn * g.b[r];
  c0[r] = v;
}

cudaError_t row_constants_device(int n, RowConstGeo g, const double *p_old, const double *dpdn_g,
                                 const double *dpdn_d, int nd, double *c0, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_row_consts<<<(n + 127) / 128, 128, 0, s>>>(n, g, p_old, dpdn_g, dpdn_d, nd, c0);
  note_launches(1);
  return cudaGetLastError();
}

__device__ int g_wave_err;  // set by a k_yzline_wave wait that gave up

template <typename T, int M, int CH>
static cudaError_t launch_yzwave(const Launch &Lr, int axis, double omega, cudaStream_t s) {
  if (!Lr.wave) return cudaErrorInvalidValue;
  int *err = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&err, g_wave_err);
  if (e == cudaSuccess) e = cudaMemsetAsync(Lr.wave, 0, (size_t)(Lr.blocks + 2) * sizeof(int), s);
  if (e != cudaSuccess) return e;
  const size_t sm = (size_t)2 * CH * YP_LINES * sizeof(Eq3<T>);
  auto kern = axis == 1 ? k_yzline_wave<T, M, CH, 1> : k_yzline_wave<T, M, CH, 2>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  // blocks resident on the whole GPU at once (the lag of the colour-1 planes)
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, CH * YP_LINES, sm);
  const int resident = std::max(1, sms * per_sm);
  kern<<<2 * Lr.blocks, CH * YP_LINES, sm, s>>>(Lr.off, Lr.n, Lr.lev, (T)omega, Lr.wave, err, resident);
  note_launches(1);
  return cudaGetLastError();
}

fg_status wave_error_take() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_wave_err, sizeof(int)) != cudaSuccess) return FG_CUDA_ERROR;
  if (!v) return FG_OK;
  const int zero = 0;
  cudaMemcpyToSymbol(g_wave_err, &zero, sizeof(int));
  set_last_error("a y/z line sweep gave up waiting for its neighbour planes", __FILE__, __LINE__);
  return FG_TIMEOUT;
}

bool line_both_colours(int axis, int maxn, int variant) {
  return axis != 0 && line_variant(axis, maxn, variant) == LV_YWAVE;
}

template <typename T, int M, int CH>
static cudaError_t launch_yzreg(const Launch &Lr, int axis, int color, double omega, cudaStream_t s) {
  const size_t sm = (size_t)3 * M * CH * 32 * sizeof(T);  // row state: d, al, ga
  if (axis == 1) {
    auto kern = k_yzline_reg<T, M, CH, 1>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<Lr.blocks, CH * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, (T)omega);
  } else {
    auto kern = k_yzline_reg<T, M, CH, 2>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<Lr.blocks, CH * 32, sm, s>>>(Lr.off, Lr.n, Lr.lev, color, (T)omega);
  }
  note_launches(1);
  return cudaGetLastError();
}

// x lines always take the register kernel (lines up to 1024 cells; lines
// per warp as xline_lanes); y/z lines up to YZ_MAXROWS cells take
// k_yzline_reg, longer ones the shared-memory tile kernel (blocks_tile and
// blocks_xline count blocks the same way)
template <typename T>
cudaError_t line_sweep(const Launch &Lr, int axis, int color, double omega, int maxn, int variant,
                       cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  const int v = line_variant(axis, maxn, variant);
  if (axis == 0) {
    if (v == LV_XREG) {
      if (maxn <= 16) return launch_xreg<T, 4, 4>(Lr, color, omega, s);
      if (maxn <= 32) return launch_xreg<T, 4, 8>(Lr, color, omega, s);
      if (maxn <= 64) return launch_xreg<T, 4, 16>(Lr, color, omega, s);
      return launch_xreg<T, 4, 32>(Lr, color, omega, s);
    }
    if (v == LV_XREG32) return launch_xreg<T, 4, 32>(Lr, color, omega, s);
    if (maxn <= 256) return launch_xsmem<T, 8>(Lr, color, omega, s);
    if (maxn <= 512) return launch_xsmem<T, 16>(Lr, color, omega, s);
    if (maxn <= 1024) return launch_xsmem<T, 32>(Lr, color, omega, s);
    return cudaErrorInvalidValue;  // lines longer than 1024 cells
  }
  if (v == LV_YPCR) {  // lines shorter than YP_MINROWS only when chosen (autotuner)
    if (maxn <= 32) return launch_yzpcr<T, 4, 8>(Lr, axis, color, omega, s);
    if (maxn <= 64) return launch_yzpcr<T, 4, 16>(Lr, axis, color, omega, s);
    if (maxn <= 128) return launch_yzpcr<T, 8, 16>(Lr, axis, color, omega, s);
    return launch_yzpcr<T, 8, 32>(Lr, axis, color, omega, s);
  }
  if (v == LV_YPCRH) {
    if (maxn <= 128) return launch_yzpcr<T, 8, 16, 4>(Lr, axis, color, omega, s);
    return launch_yzpcr<T, 8, 32, 2>(Lr, axis, color, omega, s);
  }
  if (v == LV_YWAVE) {  // both colours in the colour-0 call
    if (color == 1) return cudaSuccess;
    if (maxn <= 32) return launch_yzwave<T, 4, 8>(Lr, axis, omega, s);
    if (maxn <= 64) return launch_yzwave<T, 4, 16>(Lr, axis, omega, s);
    if (maxn <= 128) return launch_yzwave<T, 8, 16>(Lr, axis, omega, s);
    return launch_yzwave<T, 8, 32>(Lr, axis, omega, s);
  }
  if (v == LV_YPCR4) {
    if (maxn <= 128) return launch_yzpcr<T, 4, 32, 4>(Lr, axis, color, omega, s);
    return launch_yzpcr<T, 4, 64, 2>(Lr, axis, color, omega, s);
  }
  if (v == LV_YREG) {
    if (maxn <= 16) return launch_yzreg<T, 4, 4>(Lr, axis, color, omega, s);
    if (maxn <= 32) return launch_yzreg<T, 4, 8>(Lr, axis, color, omega, s);
    if (maxn <= 64) return launch_yzreg<T, 4, 16>(Lr, axis, color, omega, s);
    if (maxn <= 128) return launch_yzreg<T, 8, 16>(Lr, axis, color, omega, s);
    return launch_yzreg<T, 16, 16>(Lr, axis, color, omega, s);
  }
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

// (A x) at an active cell from its mask: sum over the kept faces of
// a (x_n - x_c), Dirichlet boundary faces contributing -2 a x_c
// (A x) at an active cell from its own value xc and its six neighbours xn
// (faces -x,+x,-y,+y,-z,+z) and the axis coefficients a
template <typename T>
__device__ __forceinline__ T apply_vals(const DevLevel &L, int i, int j, int k, uint8_t mk, T xc,
                                        const T (&xn)[6], const double (&a)[6]) {
  const bool atb[6] = {i == 1, i == L.nx, j == 1, j == L.ny, k == 1, k == L.nz};
  T acc = T(0);
  double diag = 0.0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    if ((mk >> q) & 1) { acc += (T)a[q] * xn[q]; diag -= a[q]; }
    else if (atb[q] && L.bc[q]) diag -= 2.0 * a[q];
  }
  return acc + (T)diag * xc;
}

template <typename T>
__device__ __forceinline__ T apply_row(const DevLevel &L, long long id, int i, int j, int k,
                                       uint8_t mk, dptr<const T> FG_RESTRICT x) {
  const T xc = x[id];
  const T xn[6] = {x[id - 1], x[id + 1], x[id - L.sy], x[id + L.sy], x[id - L.sz], x[id + L.sz]};
  const double a[6] = {glob(L.amx)[i], glob(L.apx)[i], glob(L.amy)[j], glob(L.apy)[j], glob(L.amz)[k], glob(L.apz)[k]};
  return apply_vals<T>(L, i, j, k, mk, xc, xn, a);
}

// per-entry sum of the block partials of a launch (1024 threads, eight
// independent loads in flight per thread)
__global__ void __launch_bounds__(1024) k_reduce_parts(const int *off, const double *part, double *out) {
  const int p = blockIdx.x;
  const int b0 = off[p], b1 = off[p + 1];
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = b0 + threadIdx.x; b < b1; b += 8 * 1024) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int q = b + u * 1024;
      if (q < b1) v[u] += part[q];
    }
  }
  double t = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = red[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) out[p] += w;
  }
}

template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_residual(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, double *part) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  auto x = PrecOf<T>::x(L);
  auto rhs = PrecOf<T>::rhs(L);
  auto res = PrecOf<T>::res(L);
  double r2 = 0.0;
#pragma unroll 2
  for (int rr = 0; rr < CELL_ROWS; ++rr) {
    const CellIdx c = cell_of(L, lb, rr);
    if (!c.ok) continue;
    const long long id = c.i + L.sy * c.j + L.sz * c.k;
    const uint8_t mk = glob(L.mask)[id];
    T r = T(0);
    if (mk & 64) r = rhs[id] - apply_row<T>(L, id, c.i, c.j, c.k, mk, x);
    if (res) res[id] = r;  // norm only where the level keeps no residual array
    r2 += (double)r * (double)r;
  }
  if (part) {
    const double t = block_sum(r2);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

template <typename T>
cudaError_t residual(const Launch &Lr, double *norm2, double *part, cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  k_residual<T><<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev, norm2 ? part : nullptr);
  note_launches(1);
  if (norm2) {
    k_reduce_parts<<<Lr.n, 1024, 0, s>>>(Lr.off, part, norm2);
    note_launches(1);
  }
  return cudaGetLastError();
}

// ||f||^2 over active cells of level 0 (FP64 rhs)
__global__ void __launch_bounds__(CELL_BLOCK)
k_fluid_norm(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, double *part) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  double r2 = 0.0;
  for (int rr = 0; rr < CELL_ROWS; ++rr) {
    const CellIdx c = cell_of(L, lb, rr);
    if (!c.ok) continue;
    const long long id = c.i + L.sy * c.j + L.sz * c.k;
    if (glob(L.mask)[id] & 64) r2 += L.rhs64[id] * L.rhs64[id];
  }
  const double t = block_sum(r2);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

cudaError_t fluid_norm(const Launch &Lr, double *norm2, double *part, cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  k_fluid_norm<<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev, part);
  note_launches(1);
  k_reduce_parts<<<Lr.n, 1024, 0, s>>>(Lr.off, part, norm2);
  note_launches(1);
  return cudaGetLastError();
}

// Mixed precision outer step, part 1: p += e (FP64 += FP32) and e = 0.
__global__ void __launch_bounds__(CELL_BLOCK)
k_correct(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  for (int rr = 0; rr < CELL_ROWS; ++rr) {
    const CellIdx c = cell_of(L, lb, rr);
    if (!c.ok) continue;
    const long long id = c.i + L.sy * c.j + L.sz * c.k;
    const float ev = L.x32[id];
    L.x64[id] = L.x64[id] + (double)ev;
    L.x32[id] = 0.0f;
  }
}

// part 2: FP64 residual of the corrected field, stored as the FP32 rhs of
// the next correction V-cycle
__global__ void __launch_bounds__(CELL_BLOCK)
k_residual_mixed(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, double *part) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  double r2 = 0.0;
#pragma unroll 2
  for (int rr = 0; rr < CELL_ROWS; ++rr) {
    const CellIdx c = cell_of(L, lb, rr);
    if (!c.ok) continue;
    const long long id = c.i + L.sy * c.j + L.sz * c.k;
    double r = 0.0;
    const uint8_t mk = glob(L.mask)[id];
    if (mk & 64) r = L.rhs64[id] - apply_row<double>(L, id, c.i, c.j, c.k, mk, L.x64);
    L.rhs32[id] = (float)r;
    r2 += r * r;
  }
  const double t = block_sum(r2);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

cudaError_t correct_residual(const Launch &Lr, double *norm2, double *part, cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  k_correct<<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev);
  note_launches(1);
  k_residual_mixed<<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev, part);
  note_launches(1);
  k_reduce_parts<<<Lr.n, 1024, 0, s>>>(Lr.off, part, norm2);
  note_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------------ quad kernels
// Cell kernels that take 4 consecutive cells of a row per thread: 16-byte
// vector loads of the row and of its four transverse neighbour rows (cell 1
// of every row is 16-byte aligned, so every quad starting at i = 1 + 4q is),
// the row's two end neighbours as scalars.  A block has QBLOCK threads: QW
// threads per row (one per quad, at most QBLOCK) and QBLOCK/QW rows at a
// time, QROWS times.
constexpr int QBLOCK = 128;
constexpr int QROWS = 4;
__host__ __device__ inline int quad_w(int nx) {
  int q = ((nx + 3) / 4 + 31) / 32 * 32;
  return q < QBLOCK ? q : QBLOCK;
}
int blocks_quads(const DevLevel &L) {
  const int qw = quad_w(L.nx), rpb = QBLOCK / qw;
  const int nseg = ((L.nx + 3) / 4 + qw - 1) / qw;
  const long long rows = (long long)L.ny * L.nz, per = (long long)rpb * QROWS;
  return (int)(nseg * ((rows + per - 1) / per));
}
struct QuadIdx { int i0, j, k; bool ok; };
__device__ __forceinline__ QuadIdx quad_of(const DevLevel &L, int lb, int r) {
  const int qw = quad_w(L.nx), rpb = QBLOCK / qw;
  const int nseg = ((L.nx + 3) / 4 + qw - 1) / qw;
  const int seg = lb % nseg, rg = lb / nseg;
  const int t = threadIdx.x;
  const long long row = ((long long)rg * QROWS + r) * rpb + t / qw;
  QuadIdx q;
  q.i0 = 1 + 4 * (seg * qw + t % qw);
  q.j = 1 + (int)(row % L.ny);
  q.k = 1 + (int)(row / L.ny);
  q.ok = q.i0 <= L.nx && q.k <= L.nz;
  return q;
}

// A quad's own values, its four transverse neighbour rows and its two end
// neighbours
template <typename T>
struct QuadVals {
  T c[4], ym[4], yp[4], zm[4], zp[4];
  T xl, xr;
  template <typename P>
  __device__ __forceinline__ void load(const DevLevel &L, const P &x, long long id) {
    load_run<T, 4>(c, x, id);
    load_run<T, 4>(ym, x, id - L.sy);
    load_run<T, 4>(yp, x, id + L.sy);
    load_run<T, 4>(zm, x, id - L.sz);
    load_run<T, 4>(zp, x, id + L.sz);
    xl = x[id - 1];
    xr = x[id + 4];
  }
  // neighbours of cell v (faces -x,+x,-y,+y,-z,+z)
  __device__ __forceinline__ void nbrs(int v, T (&xn)[6]) const {
    xn[0] = v == 0 ? xl : c[v - 1];
    xn[1] = v == 3 ? xr : c[v + 1];
    xn[2] = ym[v]; xn[3] = yp[v]; xn[4] = zm[v]; xn[5] = zp[v];
  }
};

// r = f - A x on active cells, 0 on the other interior cells (the V-cycle's
// restriction input); the arithmetic of k_residual, per quad
template <typename T>
__global__ void __launch_bounds__(QBLOCK)
k_residual_q(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  auto x = PrecOf<T>::x(L);
  auto rhs = PrecOf<T>::rhs(L);
  auto res = PrecOf<T>::res(L);
#pragma unroll
  for (int r = 0; r < QROWS; ++r) {
    const QuadIdx q = quad_of(L, lb, r);
    if (!q.ok) continue;
    const long long id = q.i0 + L.sy * q.j + L.sz * q.k;
    QuadVals<T> xv;
    xv.load(L, x, id);
    T f[4];
    uint8_t m4[4];
    load_run<T, 4>(f, rhs, id);
    load_run<uint8_t, 4>(m4, glob(L.mask), id);
    const double ay0 = glob(L.amy)[q.j], ay1 = glob(L.apy)[q.j], az0 = glob(L.amz)[q.k], az1 = glob(L.apz)[q.k];
    T out[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = q.i0 + v;
      T rv = T(0);
      if (i <= L.nx && (m4[v] & 64)) {
        T xn[6];
        xv.nbrs(v, xn);
        const double a[6] = {glob(L.amx)[i], glob(L.apx)[i], ay0, ay1, az0, az1};
        rv = f[v] - apply_vals<T>(L, i, q.j, q.k, m4[v], xv.c[v], xn, a);
      }
      out[v] = rv;
    }
    store_run<T, 4>(res, id, out, L.nx - q.i0 + 1);
  }
}

template <typename T>
cudaError_t residual_q(const Launch &Lq, cudaStream_t s) {
  if (Lq.empty()) return cudaSuccess;
  k_residual_q<T><<<Lq.blocks, QBLOCK, 0, s>>>(Lq.off, Lq.n, Lq.lev);
  note_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------------- restriction
// coarse rhs = volume-weighted mean of the children's residuals on active
// coarse cells (the sum of the children's finite-volume equations)
// the restriction into coarse cell (I,J,K)
template <typename T>
__device__ __forceinline__ void restrict_cell(const DevLevel &C, const DevLevel &F, int I, int J, int K) {
  auto rc = PrecOf<T>::rhs(C);
  auto rf = PrecOf<T>::res(F);
  const long long id = I + C.sy * J + C.sz * K;
  if (!(glob(C.mask)[id] & 64)) { rc[id] = T(0); return; }
  double s = 0.0, v = 0.0;
  for (int k = glob(C.clz)[K]; k <= glob(C.chz)[K]; ++k)
    for (int j = glob(C.cly)[J]; j <= glob(C.chy)[J]; ++j) {
      const double wyz = glob(F.wy)[j] * glob(F.wz)[k];
      const long long rb = F.sy * j + F.sz * k;
      for (int i = glob(C.clx)[I]; i <= glob(C.chx)[I]; ++i) {
        const double w = glob(F.wx)[i] * wyz;
        s += w * (double)rf[rb + i];
        v += w;
      }
    }
  rc[id] = (T)(s / v);
}

template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_restrict(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT coarse, const DevLevel *FG_RESTRICT fine) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &C = coarse[p];
  const DevLevel &F = fine[p];
  const int lb = blockIdx.x - off[p];
  // the arithmetic of restrict_cell with the thread's i-children and their
  // widths kept over the block's CELL_ROWS rows (at most two children per
  // axis: cl = 2I-1, ch = min(2I, n))
  const int tpr = (C.nx + CELL_BLOCK - 1) / CELL_BLOCK;
  const int rb = lb / tpr;
  const int I = 1 + (lb - rb * tpr) * CELL_BLOCK + (int)threadIdx.x;
  if (I > C.nx) return;
  dptr<T> FG_RESTRICT rc = PrecOf<T>::rhs(C);
  dptr<const T> FG_RESTRICT rf = PrecOf<T>::res(F);
  dptr<const uint8_t> FG_RESTRICT cm = C.mask;
  const long long csy = C.sy, csz = C.sz, fsy = F.sy, fsz = F.sz;
  const int cny = C.ny, cnz = C.nz;
  const int il = glob(C.clx)[I], ih = glob(C.chx)[I];
  const double wx0 = glob(F.wx)[il], wx1 = glob(F.wx)[ih];
  // every child's value is loaded before the coarse mask decides (the
  // children exist for every coarse cell), so the rows' loads are in
  // flight together; the sums take the valid children in the order of
  // restrict_cell
  const int row0 = rb * CELL_ROWS;
  int J = 1 + row0 % cny, K = 1 + row0 / cny;
#pragma unroll
  for (int rr = 0; rr < CELL_ROWS; ++rr) {
    if (rr > 0 && ++J > cny) { J = 1; ++K; }
    if (K > cnz) break;  // rows only grow with rr
    const long long id = I + csy * J + csz * K;
    const int kl = glob(C.clz)[K], kh = glob(C.chz)[K], jl = glob(C.cly)[J], jh = glob(C.chy)[J];
    const double wy0 = glob(F.wy)[jl], wy1 = glob(F.wy)[jh], wz0 = glob(F.wz)[kl], wz1 = glob(F.wz)[kh];
    const long long b00 = fsy * jl + fsz * kl, b10 = fsy * jh + fsz * kl, b01 = fsy * jl + fsz * kh,
                    b11 = fsy * jh + fsz * kh;
    const T f[8] = {rf[b00 + il], rf[b00 + ih], rf[b10 + il], rf[b10 + ih],
                    rf[b01 + il], rf[b01 + ih], rf[b11 + il], rf[b11 + ih]};
    if (!(cm[id] & 64)) { rc[id] = T(0); continue; }
    double s = 0.0, v = 0.0;
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) {
      if (kk == 1 && kh == kl) break;
      const double wz = kk ? wz1 : wz0;
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        if (jj == 1 && jh == jl) break;
        const double wyz = (jj ? wy1 : wy0) * wz;
        {
          const double w = wx0 * wyz;
          s += w * (double)f[4 * kk + 2 * jj];
          v += w;
        }
        if (ih > il) {
          const double w = wx1 * wyz;
          s += w * (double)f[4 * kk + 2 * jj + 1];
          v += w;
        }
      }
    }
    rc[id] = (T)(s / v);
  }
}

template <typename T>
cudaError_t restrict_to(const Launch &Lc, const DevLevel *fine, cudaStream_t s) {
  if (Lc.empty()) return cudaSuccess;
  k_restrict<T><<<Lc.blocks, CELL_BLOCK, 0, s>>>(Lc.off, Lc.n, Lc.lev, fine);
  note_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------------ prolongation
// fine x += trilinear interpolation of the coarse correction at the fine
// cell centre, over the active coarse corners only (renormalised)
// the prolongation into fine cell (i,j,k), in the arithmetic of the cycle
// (FP32 weights and sums in the mixed path: the correction itself is FP32)
template <typename T>
__device__ __forceinline__ void prolong_cell(const DevLevel &F, const DevLevel &C, int i, int j, int k) {
  auto xc = PrecOf<T>::x(C);
  auto x = PrecOf<T>::x(F);
  const long long id = i + F.sy * j + F.sz * k;
  if (!(glob(F.mask)[id] & 128)) return;
  const int i0 = glob(F.plx)[i], j0 = glob(F.ply)[j], k0 = glob(F.plz)[k];
  const int i1 = i0 < C.nx ? i0 + 1 : i0, j1 = j0 < C.ny ? j0 + 1 : j0, k1 = k0 < C.nz ? k0 + 1 : k0;
  const T wx1 = (T)glob(F.pwx)[i], wy1 = (T)glob(F.pwy)[j], wz1 = (T)glob(F.pwz)[k];
  const T wx[2] = {T(1) - wx1, wx1};
  const T wyz[4] = {(T(1) - wy1) * (T(1) - wz1), wy1 * (T(1) - wz1), (T(1) - wy1) * wz1, wy1 * wz1};
  T s = T(0), ws = T(0);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int ci = (q & 1) ? i1 : i0, cj = (q & 2) ? j1 : j0, ck = (q & 4) ? k1 : k0;
    const T w = wx[q & 1] * wyz[q >> 1];
    const long long cid = ci + C.sy * cj + C.sz * ck;
    const T act = (glob(C.mask)[cid] & 64) ? w : T(0);
    s += act * xc[cid];
    ws += act;
  }
  if (ws > T(1e-12)) x[id] = x[id] + s / ws;
}

// A block prolongs PT_I consecutive fine cells of i in PT_J consecutive
// rows of j of one fine plane k.  The coarse corners those cells read (the
// lower coarse cell never decreases with the fine index, so they form a box
// of at most PT_I + 2 by PT_J + 2 by 2 coarse cells) and their mask bytes
// are copied into shared memory by asynchronous copies (no registers
// held), while the thread's own fine column is loaded into registers; then
// each fine cell reads its eight corners from shared memory, with the
// arithmetic of prolong_cell.
constexpr int PT_I = 128, PT_J = 8;
constexpr int PT_CI = PT_I + 2, PT_CJ = PT_J + 2;
constexpr int PT_MW = (PT_CI + 3 + 3) / 4;  // mask words of a tile row (from a word boundary)
int blocks_ptile(const DevLevel &L) {
  return ((L.nx + PT_I - 1) / PT_I) * ((L.ny + PT_J - 1) / PT_J) * L.nz;
}

// global -> shared copy of B bytes (4, 8 or 16, both addresses aligned to B)
template <int B>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <typename T>
__global__ void __launch_bounds__(PT_I)
k_prolong(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT fine, const DevLevel *FG_RESTRICT coarse) {
  __shared__ T sv[2 * PT_CJ * PT_CI];
  __shared__ uint32_t smw[2 * PT_CJ * PT_MW];
  __shared__ T swy[PT_J];
  __shared__ int sr0[PT_J], sr1[PT_J];
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &F = fine[p];
  const DevLevel &C = coarse[p];
  const int lb = blockIdx.x - off[p];
  const int nti = (F.nx + PT_I - 1) / PT_I, ntj = (F.ny + PT_J - 1) / PT_J;
  const int ti = lb % nti, rest = lb / nti, tj = rest % ntj, k = 1 + rest / ntj;
  const int ia = 1 + ti * PT_I, ib = min(F.nx, ia + PT_I - 1);
  const int ja = 1 + tj * PT_J, jb = min(F.ny, ja + PT_J - 1);
  const int ca = glob(F.plx)[ia], cb = min(glob(F.plx)[ib] + 1, C.nx);
  const int da = glob(F.ply)[ja], db = min(glob(F.ply)[jb] + 1, C.ny);
  const int k0 = glob(F.plz)[k], k1 = k0 < C.nz ? k0 + 1 : k0;
  const int ni = cb - ca + 1, nj = db - da + 1;
  const int i = ia + (int)threadIdx.x;
  if (ni > PT_CI || nj > PT_CJ) {  // a box larger than the tile (no level builds one): per cell
    if (i <= ib)
      for (int j = ja; j <= jb; ++j) prolong_cell<T>(F, C, i, j, k);
    return;
  }
  // the coarse box: tile row r = (plane kk, row jj) at r = kk PT_CJ + jj;
  // the mask words from the word holding cell ca (cell 1 of a row starts a
  // word), so byte sh of a row is cell ca
  const int ca4 = ca - ((ca - 1) & 3), sh = ca - ca4, nw = (sh + ni + 3) >> 2;
  {
    dptr<const T> xc = PrecOf<T>::x(C);
    dptr<const uint8_t> cm = C.mask;
    const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
    for (int r = warp; r < 2 * nj; r += PT_I / 32) {
      const int kk = r >= nj ? 1 : 0, jj = r - kk * nj;
      const long long rb = C.sy * (da + jj) + C.sz * (kk ? k1 : k0);
      const int srow = kk * PT_CJ + jj;
      for (int c = lane; c < ni; c += 32) cp_async<sizeof(T)>(&sv[srow * PT_CI + c], &xc[rb + ca + c]);
      for (int w = lane; w < nw; w += 32) cp_async<4>(&smw[srow * PT_MW + w], &cm[rb + ca4 + 4 * w]);
    }
  }
  // the thread's fine column: masks packed four to a word, values
  dptr<T> FG_RESTRICT x = PrecOf<T>::x(F);
  const long long fsy = F.sy, id0 = i + fsy * ja + F.sz * k;
  uint32_t mp[2] = {0u, 0u};
  T xf[PT_J];
  if (i <= ib) {
    dptr<const uint8_t> FG_RESTRICT fm = F.mask;
#pragma unroll
    for (int jj = 0; jj < PT_J; ++jj) {
      xf[jj] = T(0);
      if (ja + jj <= jb) {
        mp[jj >> 2] |= (uint32_t)fm[id0 + fsy * jj] << (8 * (jj & 3));
        xf[jj] = x[id0 + fsy * jj];
      }
    }
  }
  if (threadIdx.x < PT_J && ja + (int)threadIdx.x <= jb) {
    const int j = ja + (int)threadIdx.x, cj0 = glob(F.ply)[j];
    sr0[threadIdx.x] = cj0 - da;
    sr1[threadIdx.x] = (cj0 < C.ny ? cj0 + 1 : cj0) - da;
    swy[threadIdx.x] = (T)glob(F.pwy)[j];
  }
  cp_async_wait_all();
  __syncthreads();
  if (i > ib) return;
  const uint8_t *smb = reinterpret_cast<const uint8_t *>(smw);
  const int ci0 = glob(F.plx)[i];
  const int i0 = ci0 - ca, i1 = (ci0 < C.nx ? ci0 + 1 : ci0) - ca;
  const T wx1 = (T)glob(F.pwx)[i], wz1 = (T)glob(F.pwz)[k];
  const T wx[2] = {T(1) - wx1, wx1};
#pragma unroll
  for (int jj = 0; jj < PT_J; ++jj) {
    if (ja + jj > jb) break;
    if (!((mp[jj >> 2] >> (8 * (jj & 3))) & 128)) continue;
    const int r0 = sr0[jj], r1 = sr1[jj];
    const T wy1 = swy[jj];
    const T wyz[4] = {(T(1) - wy1) * (T(1) - wz1), wy1 * (T(1) - wz1), (T(1) - wy1) * wz1, wy1 * wz1};
    T s = T(0), ws = T(0);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int row = ((q & 4) ? PT_CJ : 0) + ((q & 2) ? r1 : r0), col = (q & 1) ? i1 : i0;
      const T w = wx[q & 1] * wyz[q >> 1];
      const T act = (smb[row * (4 * PT_MW) + sh + col] & 64) ? w : T(0);
      s += act * sv[row * PT_CI + col];
      ws += act;
    }
    if (ws > T(1e-12)) x[id0 + fsy * jj] = xf[jj] + s / ws;
  }
}

template <typename T>
cudaError_t prolong_add(const Launch &Lf, const DevLevel *coarse, cudaStream_t s) {
  if (Lf.empty()) return cudaSuccess;
  k_prolong<T><<<Lf.blocks, CELL_BLOCK, 0, s>>>(Lf.off, Lf.n, Lf.lev, coarse);
  note_launches(1);
  return cudaGetLastError();
}

template <typename T>
__global__ void __launch_bounds__(CELL_BLOCK)
k_zero(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  auto x = PrecOf<T>::x(L);
  for (int rr = 0; rr < CELL_ROWS; ++rr) {
    const CellIdx c = cell_of(L, lb, rr);
    if (c.ok) x[c.i + L.sy * c.j + L.sz * c.k] = T(0);
  }
}

template <typename T>
cudaError_t zero_x(const Launch &Lr, cudaStream_t s) {
  if (Lr.empty()) return cudaSuccess;
  k_zero<T><<<Lr.blocks, CELL_BLOCK, 0, s>>>(Lr.off, Lr.n, Lr.lev);
  note_launches(1);
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
  auto x = PrecOf<T>::x(L);
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
  note_launches(1);
  k_rows_scatter<T><<<nb, CELL_BLOCK, 0, s>>>(R, lev0, tmp);
  note_launches(1);
  return cudaGetLastError();
}

// row residual (FP64 solution): r_t = sum w p + c0 - p_t; stores it in
// FP64 and FP32 and the max |r_t| per problem (as ordered bits)
__global__ void __launch_bounds__(CELL_BLOCK)
k_rows_residual(DevRows R, const DevLevel *lev0, double *maxabs) {
  const int r = blockIdx.x * CELL_BLOCK + threadIdx.x;
  const bool valid = r < R.n;
  const int p = valid ? R.prob[r] : -1;
  unsigned long long v = 0ull;
  if (valid) {
    const DevLevel &L = lev0[p];
    const auto x = L.x64;
    const long long b = R.cell[r], sy = L.sy, sz = L.sz;
    const long long o[8] = {0, sy, sy + 1, 1, sz, sz + sy, sz + sy + 1, sz + 1};
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += R.w[8 * r + q] * x[b + o[q]];
    const double rt = acc + R.c0[r] - x[R.tgt[r]];
    R.rd[r] = rt;
    R.rf[r] = (float)rt;
    v = (unsigned long long)__double_as_longlong(fabs(rt));  // order-preserving for >= 0
  }
  if (!maxabs) return;
  // rows of one problem are contiguous: one atomic per warp when the warp's
  // valid rows share a problem
  const int p0 = __shfl_sync(0xffffffffu, p, 0);
  const bool same = __all_sync(0xffffffffu, !valid || p == p0);
  if (same) {
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long w = __shfl_down_sync(0xffffffffu, v, o);
      v = v > w ? v : w;
    }
    if ((threadIdx.x & 31) == 0 && p0 >= 0)
      atomicMax(reinterpret_cast<unsigned long long *>(maxabs + p0), v);
  } else if (valid) {
    atomicMax(reinterpret_cast<unsigned long long *>(maxabs + p), v);
  }
}

cudaError_t rows_residual(const DevRows &R, const DevLevel *lev0, double *maxabs,
                          cudaStream_t s) {
  if (R.n <= 0) return cudaSuccess;
  k_rows_residual<<<(R.n + CELL_BLOCK - 1) / CELL_BLOCK, CELL_BLOCK, 0, s>>>(R, lev0, maxabs);
  note_launches(1);
  return cudaGetLastError();
}

// ---------------------------------------------------- coarsest solve
// x = G rhs over the active cells of a problem's coarsest level, G the
// generalised inverse of the coarsest operator (FP64)
template <typename T>
__global__ void __launch_bounds__(256)
k_coarsest(const DevLevel *FG_RESTRICT levs, const double *const *G, const int *const *gidx, const int *gn) {
  extern __shared__ double sr[];
  const int p = blockIdx.x;
  const DevLevel &L = levs[p];
  const int n = gn[p];
  const int *idx = gidx[p];
  const double *g = G[p];
  auto rhs = PrecOf<T>::rhs(L);
  auto x = PrecOf<T>::x(L);
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
  note_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------ small levels, one block
// The V-cycle from the first level whose every line has at most SC_MAXN
// cells and every level at most SC_MAXCELLS cells down to the coarsest, as
// one block per problem.  On such levels each launch of the level-by-level
// cycle (six line sweeps per smoothing step, residual, restriction,
// prolongation, coarsest solve) is a few microseconds of fixed cost for a
// few hundred cells; here they are phases of one kernel separated by
// __syncthreads, on data that stays in the SM's L1.  The line sweeps keep
// the line kernels' colours ((transverse index sum) & 1), rows, held rows,
// couplings and omega, one line per thread solved by the Thomas algorithm;
// residual, restriction, prolongation and coarsest solve use the
// arithmetic of their kernels.
template <typename T>
__device__ void sc_sweep(const DevLevel &L, int axis, int color, T omega) {
  const int n = axis == 0 ? L.nx : axis == 1 ? L.ny : L.nz;
  const int n1 = axis == 0 ? L.ny : L.nx;  // first transverse extent
  const int n2 = axis == 2 ? L.ny : L.nz;  // second transverse extent
  const long long ls = axis == 0 ? 1 : axis == 1 ? L.sy : L.sz;
  auto x = PrecOf<T>::x(L);
  auto rhs = PrecOf<T>::rhs(L);
  auto am_ = axis == 0 ? L.amx : axis == 1 ? L.amy : L.amz;
  auto ap_ = axis == 0 ? L.apx : axis == 1 ? L.apy : L.apz;
  for (int line = threadIdx.x; line < n1 * n2; line += blockDim.x) {
    const int a = 1 + line % n1, b = 1 + line / n1;  // transverse indices
    if (((a + b) & 1) != color) continue;
    const int i = axis == 0 ? 1 : a, j = axis == 0 ? a : axis == 1 ? 1 : b, k = axis == 2 ? 1 : b;
    const LineCoef lc = line_coef(L, axis, i, j, k);
    const bool iso_line = lc.tdir == 0.0 && !lc.dirm && !lc.dirp;
    const long long base = (long long)i + L.sy * j + L.sz * k - ls;  // row r at base + ls (r + 1)
    T cpa[SC_MAXN], dpa[SC_MAXN];
    T cprev = T(0), dprev = T(0);
    for (int r = 0; r < n; ++r) {
      const long long id = base + ls * (r + 1);
      const uint8_t m8 = glob(L.mask)[id];
      T aa = T(0), bb = T(1), cc = T(0), dd;
      const bool held = !(m8 & 64) || (((m8 & 63) == 0) && iso_line);
      if (held) {
        dd = x[id];
      } else {
        T acc = rhs[id];
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if ((m8 >> lc.qt[t]) & 1) acc -= (T)lc.tq[t] * x[id + lc.to[t]];
        dd = acc;
        row_coef<T>(m8, r, n, am_[1 + r], ap_[1 + r], lc, aa, bb, cc);
      }
      const T den = bb - aa * cprev;
      cprev = cc / den;
      dprev = (dd - aa * dprev) / den;
      cpa[r] = cprev;
      dpa[r] = dprev;
    }
    T xn = T(0);
    for (int r = n - 1; r >= 0; --r) {
      xn = dpa[r] - cpa[r] * xn;
      const long long id = base + ls * (r + 1);
      T v = xn;
      if (omega != T(1)) v = x[id] + omega * (v - x[id]);
      x[id] = v;
    }
  }
  __syncthreads();
}

template <typename T>
__device__ void sc_smooth(const DevLevel &L, int nu, T omega) {
  for (int s_ = 0; s_ < nu; ++s_)
    for (int axis = 0; axis < 3; ++axis)
      for (int color = 0; color < 2; ++color) sc_sweep<T>(L, axis, color, omega);
}

// residual of fine level F restricted into coarse level C, coarse x = 0
template <typename T>
__device__ void sc_down(const DevLevel &F, const DevLevel &C) {
  auto x = PrecOf<T>::x(F);
  auto rhs = PrecOf<T>::rhs(F);
  auto res = PrecOf<T>::res(F);
  const int nf = F.nx * F.ny * F.nz;
  for (int c = threadIdx.x; c < nf; c += blockDim.x) {
    const int i = 1 + c % F.nx, j = 1 + (c / F.nx) % F.ny, k = 1 + c / (F.nx * F.ny);
    const long long id = i + F.sy * j + F.sz * k;
    const uint8_t mk = glob(F.mask)[id];
    T r = T(0);
    if (mk & 64) r = rhs[id] - apply_row<T>(F, id, i, j, k, mk, x);
    res[id] = r;
  }
  __syncthreads();
  auto xc = PrecOf<T>::x(C);
  const int ncc = C.nx * C.ny * C.nz;
  for (int c = threadIdx.x; c < ncc; c += blockDim.x) {
    const int I = 1 + c % C.nx, J = 1 + (c / C.nx) % C.ny, K = 1 + c / (C.nx * C.ny);
    restrict_cell<T>(C, F, I, J, K);
    xc[I + C.sy * J + C.sz * K] = T(0);
  }
  __syncthreads();
}

template <typename T>
__device__ void sc_up(const DevLevel &F, const DevLevel &C) {
  const int nf = F.nx * F.ny * F.nz;
  for (int c = threadIdx.x; c < nf; c += blockDim.x) {
    const int i = 1 + c % F.nx, j = 1 + (c / F.nx) % F.ny, k = 1 + c / (F.nx * F.ny);
    prolong_cell<T>(F, C, i, j, k);
  }
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(SC_THREADS)
k_small_cycle(const SmallProb *probs, const DevLevel *FG_RESTRICT levs, int nu1, int nu2, T omega) {
  extern __shared__ double sc_sr[];  // coarsest right-hand side (gn values)
  const SmallProb P = probs[blockIdx.x];
  for (int l = 0; l < P.nl - 1; ++l) {
    sc_smooth<T>(levs[P.l0 + l], nu1, omega);
    sc_down<T>(levs[P.l0 + l], levs[P.l0 + l + 1]);
  }
  {
    const DevLevel &L = levs[P.l0 + P.nl - 1];
    auto rhs = PrecOf<T>::rhs(L);
    auto x = PrecOf<T>::x(L);
    for (int c = threadIdx.x; c < P.gn; c += blockDim.x) sc_sr[c] = (double)rhs[P.gidx[c]];
    __syncthreads();
    for (int r = threadIdx.x; r < P.gn; r += blockDim.x) {
      double acc = 0.0;
      const double *gr = P.G + (size_t)r * P.gn;
      for (int c = 0; c < P.gn; ++c) acc += gr[c] * sc_sr[c];
      x[P.gidx[r]] = (T)acc;
    }
    __syncthreads();
  }
  for (int l = P.nl - 2; l >= 0; --l) {
    sc_up<T>(levs[P.l0 + l], levs[P.l0 + l + 1]);
    sc_smooth<T>(levs[P.l0 + l], nu2, omega);
  }
}

template <typename T>
cudaError_t small_cycle(int nprob, const SmallProb *probs, const DevLevel *levs, int maxgn, int nu1,
                        int nu2, double omega, cudaStream_t s) {
  if (nprob <= 0) return cudaSuccess;
  const size_t sm = (size_t)std::max(1, maxgn) * sizeof(double);
  if (sm > 48 * 1024)
    cudaFuncSetAttribute(k_small_cycle<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_small_cycle<T><<<nprob, SC_THREADS, sm, s>>>(probs, levs, nu1, nu2, (T)omega);
  note_launches(1);
  return cudaGetLastError();
}
template cudaError_t small_cycle<float>(int, const SmallProb *, const DevLevel *, int, int, int, double,
                                        cudaStream_t);
template cudaError_t small_cycle<double>(int, const SmallProb *, const DevLevel *, int, int, int, double,
                                         cudaStream_t);

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
  note_launches(1);
  return cudaGetLastError();
}
cudaError_t copy_out(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                     long long sz, cudaStream_t s) {
  const long long n = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  k_copy_out<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dst, src, nx, ny, nz, sy, sz);
  note_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------ output finishing
__global__ void k_gauge_save(const double *ref, long long id111, double *pa) { *pa = ref[id111]; }

__global__ void k_gauge(double *ref, const DevLevel L, int nx, int ny, int nz, const double *pa) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long X = nx + 1, Y = ny + 1, Z = nz + 1;  // indices 0..n
  if (e >= X * Y * Z) return;
  const int i = (int)(e % X), j = (int)((e / X) % Y), k = (int)(e / (X * Y));
  if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 1 &&
      glob(L.type)[i + L.sy * j + L.sz * k] == T_SOLID)
    return;  // pure-solid values are held
  ref[i + (long long)(nx + 2) * (j + (long long)(ny + 2) * k)] -= *pa;
}

struct FaceBC {
  int pbc[6];
  double ppp[6];
};

// face pair of one axis; a = 0: x faces over j,k in 1..n-1; a = 1: y faces
// over i in 0..nx, k in 1..nz-1; a = 2: z faces over i in 0..nx, j in 1..ny-1
__global__ void k_faces(double *ref, int nx, int ny, int nz, int a, FaceBC bc) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long RX = nx + 2, RY = ny + 2;
  long long lo, hi, in0, in1;
  if (a == 0) {
    const long long nj = ny - 1;
    if (e >= nj * (nz - 1)) return;
    const long long j = 1 + e % nj, k = 1 + e / nj;
    const long long b = RX * (j + RY * k);
    lo = b; in0 = b + 1; hi = b + nx; in1 = b + nx - 1;
  } else if (a == 1) {
    const long long ni = nx + 1;
    if (e >= ni * (nz - 1)) return;
    const long long i = e % ni, k = 1 + e / ni;
    lo = i + RX * (RY * k); in0 = lo + RX;
    hi = i + RX * (ny + RY * k); in1 = hi - RX;
  } else {
    const long long ni = nx + 1;
    if (e >= ni * (ny - 1)) return;
    const long long i = e % ni, j = 1 + e / ni;
    lo = i + RX * j; in0 = lo + RX * RY;
    hi = i + RX * (j + RY * (long long)nz); in1 = hi - RX * RY;
  }
  const double v0 = ref[in0], v1 = ref[in1];
  ref[lo] = bc.pbc[2 * a] == 1 ? 2.0 * bc.ppp[2 * a] - v0 : v0;
  ref[hi] = bc.pbc[2 * a + 1] == 1 ? 2.0 * bc.ppp[2 * a + 1] - v1 : v1;
}

cudaError_t finish_field(double *ref, const DevLevel *lev0, int nx, int ny, int nz, const int *pbc,
                         const double *ppp, int gauge, double *scratch, cudaStream_t s) {
  if (gauge) {
    const long long id111 = 1 + (long long)(nx + 2) * (1 + (long long)(ny + 2));
    k_gauge_save<<<1, 1, 0, s>>>(ref, id111, scratch);
    note_launches(1);
    const long long n = (long long)(nx + 1) * (ny + 1) * (nz + 1);
    k_gauge<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ref, *lev0, nx, ny, nz, scratch);
    note_launches(1);
  }
  FaceBC bc;
  for (int f = 0; f < 6; ++f) { bc.pbc[f] = pbc[f]; bc.ppp[f] = ppp[f]; }
  const long long nf[3] = {(long long)(ny - 1) * (nz - 1), (long long)(nx + 1) * (nz - 1),
                           (long long)(nx + 1) * (ny - 1)};
  for (int a = 0; a < 3; ++a) {
    k_faces<<<(unsigned)((nf[a] + 255) / 256), 256, 0, s>>>(ref, nx, ny, nz, a, bc);
    note_launches(1);
  }
  return cudaGetLastError();
}

// Known boundary terms of the rows next to the outer faces, moved into the
// right-hand side of the finest level (solution form).  A Dirichlet face
// (CORE_SET_OUTER_BC.F90:1093-1170: ghost value 2 ppp - p(1)) couples the
// row by a (p_ghost - p) = 2 a ppp - 2 a p: the operator holds -2 a p, the
// right-hand side loses 2 a ppp.  A Neumann face with gradient data
// (CORE_SET_OUTER_BC.F90:831-1042: ghost value p(1) -+ pgrad dxc) adds
// +- pgrad / w, w the cell width along the face normal; pgrad arrays are
// the reference's face arrays, (0:ny+1, 0:nz+1) for x faces, (0:nx+1,
// 0:nz+1) for y faces, (0:nx+1, 0:ny+1) for z faces (node counts),
// indexed by the face cell's two transverse reference indices.
//
// The known term of face f at the face cell idx:
__device__ __forceinline__ double face_term(const DevLevel &L, const FaceData &fd, int f, const int (&idx)[3]) {
  const int a = f >> 1, up = f & 1;
  if (fd.pbc[f] == FG_PBC_DIRICHLET) {
    const double am[3] = {glob(L.amx)[idx[0]], glob(L.amy)[idx[1]], glob(L.amz)[idx[2]]};
    const double ap[3] = {glob(L.apx)[idx[0]], glob(L.apy)[idx[1]], glob(L.apz)[idx[2]]};
    return -2.0 * (up ? ap[a] : am[a]) * fd.ppp[f];
  }
  if (fd.pgrad[f]) {
    const int n[3] = {L.nx, L.ny, L.nz};
    const int u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;  // transverse axes
    const double w[3] = {glob(L.wx)[idx[0]], glob(L.wy)[idx[1]], glob(L.wz)[idx[2]]};
    const long long stride = (long long)n[u] + 3;  // reference extent of the first transverse index
    const double g = fd.pgrad[f][idx[u] + stride * idx[v]];
    return up ? -g / w[a] : g / w[a];
  }
  return 0.0;
}

// blockIdx.y = face; threads cover the face's cells.  A cell on an edge or
// corner of the box lies on two or three faces: the thread of the lowest
// of them adds all their terms, in face order (one writer, the same sum
// on every run).
__global__ void k_face_rhs(double *rhs, const DevLevel L, FaceData fd) {
  const int f = blockIdx.y, a = f >> 1, up = f & 1;
  const int n[3] = {L.nx, L.ny, L.nz};
  const int u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;  // transverse axes
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n[u] * n[v]) return;
  int idx[3];
  idx[u] = 1 + (int)(e % n[u]);
  idx[v] = 1 + (int)(e / n[u]);
  idx[a] = up ? n[a] : 1;
  const long long id = idx[0] + L.sy * idx[1] + L.sz * idx[2];
  if (!(glob(L.mask)[id] & 64)) return;
  int on = 0;  // faces the cell lies on
  for (int q = 0; q < 3; ++q) {
    if (idx[q] == 1) on |= 1 << (2 * q);
    if (idx[q] == n[q]) on |= 1 << (2 * q + 1);
  }
  if ((on & -on) != (1 << f)) return;  // a lower face owns the cell
  double add = 0.0;
  for (int q = 0; q < 6; ++q)
    if ((on >> q) & 1) add += face_term(L, fd, q, idx);
  if (add != 0.0) rhs[id] += add;
}

cudaError_t face_rhs(double *rhs, const DevLevel &L0, const FaceData &fd, cudaStream_t s) {
  bool any = false;
  for (int f = 0; f < 6; ++f)
    any |= (fd.pbc[f] == FG_PBC_DIRICHLET && fd.ppp[f] != 0.0) || (fd.pbc[f] != FG_PBC_DIRICHLET && fd.pgrad[f]);
  if (!any) return cudaSuccess;
  const long long m = std::max((long long)L0.ny * L0.nz, std::max((long long)L0.nx * L0.nz, (long long)L0.nx * L0.ny));
  k_face_rhs<<<dim3((unsigned)((m + 255) / 256), 6), 256, 0, s>>>(rhs, L0, fd);
  note_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------ reference residual norms
// CORE_POISSON.F90:460-551 (calc_residual): r = div - A p on the fluid,
// non-ghost interior cells of a reference-layout field (its own outer ghost
// layers as stored), block sums of r^2 into part[b].  CORE_POISSON.F90
// :679-724 (calc_residual2): block maxima of |p - p_temp| over the
// non-iblank interior cells into part[b].  mask: iblank then ghostCellMark
// (reference layout); lev0 supplies the axis coefficients.
__global__ void __launch_bounds__(256)
k_ref_residual(const double *p, const double *div, const int8_t *ib, const int8_t *gh, const DevLevel L,
               int nx, int ny, int nz, double *part) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ni = nx - 1, nj = ny - 1, n = ni * nj * (nz - 1);
  double r2 = 0.0;
  if (e < n) {
    const int i = 1 + (int)(e % ni), j = 1 + (int)((e / ni) % nj), k = 1 + (int)(e / (ni * nj));
    const long long NX = nx + 2, NXY = NX * (ny + 2), id = i + NX * j + NXY * k;
    const double bmx = glob(L.amx)[i], bpx = glob(L.apx)[i], bmy = glob(L.amy)[j], bpy = glob(L.apy)[j], bmz = glob(L.amz)[k], bpz = glob(L.apz)[k];
    const double bc = -(bmx + bpx) + -(bmy + bpy) + -(bmz + bpz);
    const double res = div[id] - p[id] * bc - p[id - 1] * bmx - p[id + 1] * bpx - p[id - NX] * bmy -
                       p[id + NX] * bpy - p[id - NXY] * bmz - p[id + NXY] * bpz;
    const double flag = (1.0 - (double)ib[id]) * (1.0 - (double)gh[id]);
    r2 = res * flag * (res * flag);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(256)
k_ref_change(const double *p, const double *pt, const int8_t *ib, int nx, int ny, int nz, double *part) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ni = nx - 1, nj = ny - 1, n = ni * nj * (nz - 1);
  double v = 0.0;
  if (e < n) {
    const int i = 1 + (int)(e % ni), j = 1 + (int)((e / ni) % nj), k = 1 + (int)(e / (ni * nj));
    const long long id = i + (long long)(nx + 2) * (j + (long long)(ny + 2) * k);
    v = fabs(p[id] - pt[id]) * (1.0 - (double)ib[id]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t = fmax(t, red[w]);
    part[blockIdx.x] = t;
  }
}

// GCM_GHOSTCELL_UPDATE.F90:865-1003 (GCM_enforce_p_compatibility), on a
// reference-layout field: the net pressure-gradient flux out of the fluid,
// non-ghost cells, block partials into part.  met: the reference's 1-D
// arrays dx, dy, dz, dxcinv, dycinv, dzcinv back to back (n+2 each).
struct RefMet {
  const double *dx, *dy, *dz, *dxci, *dyci, *dzci;
};
__global__ void __launch_bounds__(256)
k_compat_flux(const double *p, const int8_t *ib, const int8_t *gh, RefMet m, int nx, int ny, int nz,
              double *part) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ni = nx - 1, nj = ny - 1, n = ni * nj * (nz - 1);
  double f = 0.0;
  if (e < n) {
    const int i = 1 + (int)(e % ni), j = 1 + (int)((e / ni) % nj), k = 1 + (int)(e / (ni * nj));
    const long long NX = nx + 2, NXY = NX * (ny + 2), id = i + NX * j + NXY * k;
    const double pc = p[id];
    const double pxw = (pc - p[id - 1]) * m.dxci[i], pxe = (p[id + 1] - pc) * m.dxci[i + 1];
    const double pys = (pc - p[id - NX]) * m.dyci[j], pyn = (p[id + NX] - pc) * m.dyci[j + 1];
    const double pzb = (pc - p[id - NXY]) * m.dzci[k], pzf = (p[id + NXY] - pc) * m.dzci[k + 1];
    const double flag = (1.0 - (double)ib[id]) * (1.0 - (double)gh[id]);
    f = flag * ((-pxw + pxe) * m.dy[j] * m.dz[k] + (-pys + pyn) * m.dx[i] * m.dz[k] +
                (-pzb + pzf) * m.dx[i] * m.dy[j]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) f += __shfl_down_sync(0xffffffffu, f, o);
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = f;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

// one block: the flux partials summed, the fluid area of the faces whose
// velocity is zero-gradient (CORE_SET_OUTER_BC.F90:585-643: the first
// interior layer's non-iblank cells), corr = -flux / area into *corr
__global__ void __launch_bounds__(1024)
k_compat_corr(const double *part, int nb, const int8_t *ib, RefMet m, int nx, int ny, int nz, int vzg,
              double *corr) {
  const long long NX = nx + 2, NXY = NX * (ny + 2);
  double flux = 0.0, area = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) flux += part[b];
  // x faces over (j,k), y faces over (i,k), z faces over (i,j): interior cells
  for (int f = 0; f < 6; ++f) {
    if (!((vzg >> f) & 1)) continue;
    const int a = f >> 1, up = f & 1;
    const int nu = a == 0 ? ny - 1 : nx - 1, nv = a == 2 ? ny - 1 : nz - 1;
    const int layer = a == 0 ? (up ? nx - 1 : 1) : a == 1 ? (up ? ny - 1 : 1) : (up ? nz - 1 : 1);
    for (long long e = threadIdx.x; e < (long long)nu * nv; e += blockDim.x) {
      const int u = 1 + (int)(e % nu), v = 1 + (int)(e / nu);
      long long id;
      double w;
      if (a == 0) { id = layer + NX * u + NXY * v; w = m.dy[u] * m.dz[v]; }
      else if (a == 1) { id = u + NX * layer + NXY * v; w = m.dx[u] * m.dz[v]; }
      else { id = u + NX * v + NXY * layer; w = m.dx[u] * m.dy[v]; }
      area += w * (1.0 - (double)ib[id]);
    }
  }
  __shared__ double rf[32], ra[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    flux += __shfl_down_sync(0xffffffffu, flux, o);
    area += __shfl_down_sync(0xffffffffu, area, o);
  }
  if ((threadIdx.x & 31) == 0) { rf[threadIdx.x >> 5] = flux; ra[threadIdx.x >> 5] = area; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double F = 0.0, A = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { F += rf[w]; A += ra[w]; }
    *corr = -F / A;
  }
}

// pgrad -= corr on the lower faces, += corr on the upper faces whose
// velocity is zero-gradient, over every entry (0..n) of the face arrays;
// blockIdx.y = face
__global__ void k_compat_apply(double *pg, int nx, int ny, int nz, int vzg, const double *corr) {
  const int f = blockIdx.y;
  if (!((vzg >> f) & 1)) return;
  const long long NX = nx + 2, NY = ny + 2, NZ = nz + 2;
  const long long ext[3] = {NY * NZ, NX * NZ, NX * NY};
  long long off = 0;
  for (int q = 0; q < f; ++q) off += ext[q >> 1];
  const int a = f >> 1;
  const long long n0 = a == 0 ? NY : NX;  // first index extent
  const long long u1 = a == 0 ? ny : nx, v1 = a == 2 ? ny : nz;  // indices 0..u1, 0..v1
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (u1 + 1) * (v1 + 1)) return;
  const long long u = e % (u1 + 1), v = e / (u1 + 1);
  const double c = *corr;
  double &g = pg[off + u + n0 * v];
  g = (f & 1) ? g + c : g - c;
}

cudaError_t compat(const double *p, const int8_t *ib, const int8_t *gh, const double *met, int nx, int ny,
                   int nz, int vzg, double *part, double *corr, double *pgrad, cudaStream_t s) {
  RefMet m;
  m.dx = met; m.dy = met + (nx + 2); m.dz = m.dy + (ny + 2);
  m.dxci = m.dz + (nz + 2); m.dyci = m.dxci + (nx + 2); m.dzci = m.dyci + (ny + 2);
  const int nb = ref_blocks(nx, ny, nz);
  k_compat_flux<<<nb, 256, 0, s>>>(p, ib, gh, m, nx, ny, nz, part);
  k_compat_corr<<<1, 1024, 0, s>>>(part, nb, ib, m, nx, ny, nz, vzg, corr);
  const long long big = (long long)(std::max(nx, ny) + 1) * (std::max(ny, nz) + 1);
  k_compat_apply<<<dim3((unsigned)((big + 255) / 256), 6), 256, 0, s>>>(pgrad, nx, ny, nz, vzg, corr);
  note_launches(3);
  return cudaGetLastError();
}

int ref_blocks(int nx, int ny, int nz) {
  return (int)(((long long)(nx - 1) * (ny - 1) * (nz - 1) + 255) / 256);
}
cudaError_t ref_residual(const double *p, const double *div, const int8_t *ib, const int8_t *gh,
                         const DevLevel &L0, int nx, int ny, int nz, double *part, cudaStream_t s) {
  k_ref_residual<<<ref_blocks(nx, ny, nz), 256, 0, s>>>(p, div, ib, gh, L0, nx, ny, nz, part);
  note_launches(1);
  return cudaGetLastError();
}
cudaError_t ref_change(const double *p, const double *pt, const int8_t *ib, int nx, int ny, int nz, double *part,
                       cudaStream_t s) {
  k_ref_change<<<ref_blocks(nx, ny, nz), 256, 0, s>>>(p, pt, ib, nx, ny, nz, part);
  note_launches(1);
  return cudaGetLastError();
}

// ------------------------------------------------------------- FGMRES
// Vector v of a Krylov set (basis V or preconditioned Z) of one problem.
template <typename B>
__device__ __forceinline__ dptr<B> kvec(const KDesc &d, void *base, int v) {
  return glob(mkptr(reinterpret_cast<B *>(base) + (long long)v * d.stride, d.n, K_X));
}

__device__ __forceinline__ bool is_row(const DevLevel &L, long long id, uint8_t mk) {
  return (mk & 64) || glob(L.type)[id] == T_GHOST;
}

// (A x) at an active cell in FP64 from values of type T: the sum of
// apply_row (kept faces a (x_n - x_c), Dirichlet boundary faces -2 a x_c)
template <typename T, typename P>
__device__ __forceinline__ double apply_row_d(const DevLevel &L, long long id, int i, int j, int k,
                                              uint8_t mk, const P &x) {
  const double xc = (double)x[id];
  const double xn[6] = {(double)x[id - 1],    (double)x[id + 1],    (double)x[id - L.sy],
                        (double)x[id + L.sy], (double)x[id - L.sz], (double)x[id + L.sz]};
  const double a[6] = {glob(L.amx)[i], glob(L.apx)[i], glob(L.amy)[j], glob(L.apy)[j], glob(L.amz)[k], glob(L.apz)[k]};
  const bool atb[6] = {i == 1, i == L.nx, j == 1, j == L.ny, k == 1, k == L.nz};
  double acc = 0.0, diag = 0.0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    if ((mk >> q) & 1) { acc += a[q] * xn[q]; diag -= a[q]; }
    else if (atb[q] && L.bc[q]) diag -= 2.0 * a[q];
  }
  return acc + diag * xc;
}

// Vector indices of a Krylov pass: the immediates, or, with ctl, those of
// phase `ph` at the step counters of ctl (one captured launch then serves
// every step of a device-side loop).
struct KSel {
  int vz, vw, nv, vd, s0, ns, stage;
};
__device__ __forceinline__ KSel kidx(const KCtl *ctl, int ph, KSel s) {
  if (!ctl) return s;
  const int j = ctl->j, jl = ctl->jlast;
  switch (ph) {
    case KPH_RESTART: s.vw = 0; s.nv = 0; s.vd = 0; s.s0 = 0; s.ns = 0; s.stage = 1; break;
    case KPH_APPLY: s.vz = j; s.vw = j + 1; s.nv = j + 1; break;
    case KPH_REORTH: s.vd = j + 1; s.s0 = 0; s.ns = j + 1; s.stage = 0; break;
    case KPH_NORMALIZE: s.vd = jl; s.s0 = 0; s.ns = jl; s.stage = ctl->more; break;
    default: s.ns = jl; break;  // KPH_UPDATE
  }
  return s;
}

// V_vd = F - A P on active rows, 0 on every other interior cell; part[b] =
// block sum of the squared active-row residuals (fluid-row norm).  Per quad
// (4 cells of a row per thread, vector loads), FP64 arithmetic.
template <typename B>
__global__ void __launch_bounds__(QBLOCK)
k_kr_resid(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, const KDesc *kd, int vd, double *part) {
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  const KDesc &d = kd[p];
  auto P = glob(mkptr<const double>(d.P, d.n, K_X));
  auto F = glob(mkptr<const double>(d.F, d.n, K_RHS));
  auto D = kvec<B>(d, d.V, vd);
  double r2 = 0.0;
#pragma unroll
  for (int r = 0; r < QROWS; ++r) {
    const QuadIdx q = quad_of(L, lb, r);
    if (!q.ok) continue;
    const long long id = q.i0 + L.sy * q.j + L.sz * q.k;
    QuadVals<double> pv;
    pv.load(L, P, id);
    double f[4];
    uint8_t m4[4];
    load_run<double, 4>(f, F, id);
    load_run<uint8_t, 4>(m4, glob(L.mask), id);
    const double ay0 = glob(L.amy)[q.j], ay1 = glob(L.apy)[q.j], az0 = glob(L.amz)[q.k], az1 = glob(L.apz)[q.k];
    B out[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = q.i0 + v;
      double rv = 0.0;
      if (i <= L.nx && (m4[v] & 64)) {
        double xn[6];
        pv.nbrs(v, xn);
        const double a[6] = {glob(L.amx)[i], glob(L.apx)[i], ay0, ay1, az0, az1};
        rv = f[v] - apply_vals<double>(L, i, q.j, q.k, m4[v], pv.c[v], xn, a);
      }
      out[v] = (B)rv;
      r2 += rv * rv;
    }
    store_run<B, 4>(D, id, out, L.nx - q.i0 + 1);
  }
  const double t = block_sum(r2);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// Preconditioner output x_T into Z_vz (rows; 0 elsewhere) and W = A x_T
// into V_vw on active rows (0 on every other interior cell), per quad (4
// cells of a row per thread, vector loads), in the FP64 arithmetic of
// apply_row_d.  x_T is zero on the pure-solid cells an active row may
// couple to (they are held at the staged zero), so A x_T equals A Z_vz.
template <typename B, typename T>
__global__ void __launch_bounds__(QBLOCK)
k_kr_apply_q(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, const KDesc *kd, int vz, int vw,
             const KCtl *ctl) {
  if (ctl) { vz = ctl->j; vw = ctl->j + 1; }
  const int p = find_entry(off, nent, blockIdx.x);
  const DevLevel &L = levs[p];
  const int lb = blockIdx.x - off[p];
  const KDesc &d = kd[p];
  auto x = PrecOf<T>::x(L);
  auto Z = kvec<B>(d, d.Z, vz);
  auto W = kvec<B>(d, d.V, vw);
#pragma unroll
  for (int r = 0; r < QROWS; ++r) {
    const QuadIdx q = quad_of(L, lb, r);
    if (!q.ok) continue;
    const long long id = q.i0 + L.sy * q.j + L.sz * q.k;
    QuadVals<T> xv;
    xv.load(L, x, id);
    uint8_t m4[4];
    int8_t t4[4];
    load_run<uint8_t, 4>(m4, glob(L.mask), id);
    load_run<int8_t, 4>(t4, glob(L.type), id);
    const double ay0 = glob(L.amy)[q.j], ay1 = glob(L.apy)[q.j], az0 = glob(L.amz)[q.k], az1 = glob(L.apz)[q.k];
    B z4[4], w4[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = q.i0 + v;
      const bool row = (m4[v] & 64) || t4[v] == T_GHOST;
      z4[v] = row ? (B)xv.c[v] : B(0);
      double wv = 0.0;
      if (i <= L.nx && (m4[v] & 64)) {
        T xn[6];
        xv.nbrs(v, xn);
        const double a[6] = {glob(L.amx)[i], glob(L.apx)[i], ay0, ay1, az0, az1};
        const bool atb[6] = {i == 1, i == L.nx, q.j == 1, q.j == L.ny, q.k == 1, q.k == L.nz};
        double acc = 0.0, diag = 0.0;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
          if ((m4[v] >> f) & 1) { acc += a[f] * (double)xn[f]; diag -= a[f]; }
          else if (atb[f] && L.bc[f]) diag -= 2.0 * a[f];
        }
        wv = acc + diag * (double)xv.c[v];
      }
      w4[v] = (B)wv;
    }
    store_run<B, 4>(Z, id, z4, L.nx - q.i0 + 1);
    store_run<B, 4>(W, id, w4, L.nx - q.i0 + 1);
  }
}

// interpolation rows: mode 0 -> V_vd[t] = c0 + sum w P[corner] - P[t] (the
// row's residual in solution form), mode 1 -> V_vd[t] = Z_vs[t] - sum w
// Z_vs[corner] (the row of A), mode 2 -> correction constants of the
// preconditioner: rd = rf = V_vs[t]
template <typename B>
__global__ void __launch_bounds__(CELL_BLOCK)
k_kr_rows(DevRows R, const DevLevel *lev0, const KDesc *kd, int mode, int vs, int vd, const KCtl *ctl,
          int ph) {
  if (ctl) {
    if (mode == 1) { vs = ctl->j; vd = ctl->j + 1; }
    if (mode == 2) {
      if (ph == KPH_NORMALIZE && !ctl->more) return;  // nothing staged
      vs = vd = ph == KPH_RESTART ? 0 : ctl->jlast;
    }
  }
  const int r = blockIdx.x * CELL_BLOCK + threadIdx.x;
  if (r >= R.n) return;
  const int p = R.prob[r];
  const DevLevel &L = lev0[p];
  const KDesc &d = kd[p];
  const long long t = R.tgt[r];
  if (mode == 2) {
    const B v = kvec<B>(d, d.V, vs)[t];
    R.rd[r] = (double)v;
    R.rf[r] = (float)v;
    return;
  }
  auto D = kvec<B>(d, d.V, vd);
  const long long b = R.cell[r], sy = L.sy, sz = L.sz;
  const long long o[8] = {0, sy, sy + 1, 1, sz, sz + sy, sz + sy + 1, sz + 1};
  double acc = 0.0;
  if (mode == 0) {
    auto S = glob(mkptr<const double>(d.P, d.n, K_X));
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += R.w[8 * r + q] * S[b + o[q]];
    D[t] = (B)(R.c0[r] + acc - S[t]);
  } else {
    auto S = kvec<B>(d, d.Z, vs);
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += R.w[8 * r + q] * (double)S[b + o[q]];
    D[t] = (B)((double)S[t] - acc);
  }
}

// Flat passes over Krylov vectors: 4-element pieces starting at element 1
// (16-byte aligned by the padding), FLAT_PPT pieces per thread interleaved
// across the block so every load instruction covers consecutive pieces.
// Elements 0 and past the last piece are boundary cells, zero in every
// vector and never written.
constexpr int FLAT_THREADS = 256;
constexpr int FLAT_PPT = 4;
int blocks_flat(long long n) {
  const long long nq = (n - 1) / 4;
  return (int)((nq + FLAT_THREADS * FLAT_PPT - 1) / (FLAT_THREADS * FLAT_PPT));
}
__device__ __forceinline__ long long flat_elem(int lb, int u) {
  return 1 + 4 * (((long long)lb * FLAT_PPT + u) * FLAT_THREADS + threadIdx.x);
}
__device__ __forceinline__ long long flat_end(long long n) { return 1 + 4 * ((n - 1) / 4); }

// block partials of (V_vw, V_i) for i < nv and of (V_vw, V_vw):
// part[i * nblk + b], part[nv * nblk + b]
template <typename B>
__global__ void __launch_bounds__(FLAT_THREADS)
k_kr_dots(const int *off, int nent, const KDesc *kd, int vw, int nv, int nblk, double *part,
          const KCtl *ctl, int ph) {
  {
    const KSel ks = kidx(ctl, ph, KSel{0, vw, nv, 0, 0, 0, 0});
    vw = ks.vw;
    nv = ks.nv;
  }
  const int p = find_entry(off, nent, blockIdx.x);
  const int lb = blockIdx.x - off[p];
  const KDesc &d = kd[p];
  const long long lim = flat_end(d.n);
  B w[FLAT_PPT][4];
  bool ok[FLAT_PPT];
  double acc[KR_MAXV + 1];
#pragma unroll
  for (int i = 0; i <= KR_MAXV; ++i) acc[i] = 0.0;
  {
    auto W = kvec<B>(d, d.V, vw);
#pragma unroll
    for (int u = 0; u < FLAT_PPT; ++u) {
      const long long e = flat_elem(lb, u);
      ok[u] = e < lim;
      if (ok[u]) load_run<B, 4>(w[u], W, e);
      else
#pragma unroll
        for (int q = 0; q < 4; ++q) w[u][q] = B(0);
    }
  }
#pragma unroll
  for (int u = 0; u < FLAT_PPT; ++u)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[KR_MAXV] += (double)w[u][q] * (double)w[u][q];
#pragma unroll
  for (int i = 0; i < KR_MAXV; ++i) {
    if (i < nv) {
      auto V = kvec<B>(d, d.V, i);
      B v[FLAT_PPT][4];
#pragma unroll
      for (int u = 0; u < FLAT_PPT; ++u) {
        if (ok[u]) load_run<B, 4>(v[u], V, flat_elem(lb, u));
        else
#pragma unroll
          for (int q = 0; q < 4; ++q) v[u][q] = B(0);
      }
#pragma unroll
      for (int u = 0; u < FLAT_PPT; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i] += (double)w[u][q] * (double)v[u][q];
    }
  }
  __shared__ double red[FLAT_THREADS / 32][KR_MAXV + 1];
  const int wi = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i <= KR_MAXV; ++i) {
    if (i < nv || i == KR_MAXV) {
      double v = acc[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (ln == 0) red[wi][i] = v;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x <= nv) {
    const int slot = (int)threadIdx.x < nv ? (int)threadIdx.x : KR_MAXV;
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < FLAT_THREADS / 32; ++q) t += red[q][slot];
    part[(size_t)threadIdx.x * nblk + blockIdx.x] = t;
  }
}

// out[p * ostride + i] = sum of part[i * nblk + off[p] .. off[p+1]) for
// i < nsum (grid: problems x nsum)
__global__ void __launch_bounds__(256)
k_kr_reduce(const int *off, const double *part, int nblk, double *out, int ostride, const KCtl *ctl,
            int ph) {
  const int p = blockIdx.x, i = blockIdx.y;
  if (ctl && i > kidx(ctl, ph, KSel{0, 0, 0, 0, 0, 0, 0}).nv) return;  // grid sized for the most vectors
  double v = 0.0;
  for (int b = off[p] + threadIdx.x; b < off[p + 1]; b += 256) v += part[(size_t)i * nblk + b];
  __shared__ double red[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w];
    out[(size_t)p * ostride + i] = t;
  }
}

// V_vd = c0 V_vd + sum_{i<ns} c_{1+i} V_{s0+i} (FP64 arithmetic); with
// stage, rhs_T = V_vd on active rows (0 elsewhere) and x_T = 0
template <typename B, typename T>
__global__ void __launch_bounds__(FLAT_THREADS)
k_kr_vaxpy(const int *FG_RESTRICT off, int nent, const DevLevel *FG_RESTRICT levs, const KDesc *kd, int vd, int s0, int ns,
           const double *coef, int cs, int stage, const KCtl *ctl, int ph) {
  {
    const KSel ks = kidx(ctl, ph, KSel{0, 0, 0, vd, s0, ns, stage});
    vd = ks.vd; s0 = ks.s0; ns = ks.ns; stage = ks.stage;
  }
  const int p = find_entry(off, nent, blockIdx.x);
  const int lb = blockIdx.x - off[p];
  const KDesc &d = kd[p];
  const long long lim = flat_end(d.n);
  const double *cf = coef + (size_t)p * cs;
  auto D = kvec<B>(d, d.V, vd);
  double acc[FLAT_PPT][4];
  bool ok[FLAT_PPT];
  {
    const double c0 = cf[0];
#pragma unroll
    for (int u = 0; u < FLAT_PPT; ++u) {
      const long long e = flat_elem(lb, u);
      ok[u] = e < lim;
      B v[4] = {B(0), B(0), B(0), B(0)};
      if (ok[u]) load_run<B, 4>(v, D, e);
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[u][q] = c0 * (double)v[q];
    }
  }
  for (int i = 0; i < ns; ++i) {
    const double ci = cf[1 + i];
    auto S = kvec<B>(d, d.V, s0 + i);
    B v[FLAT_PPT][4];
#pragma unroll
    for (int u = 0; u < FLAT_PPT; ++u) {
      if (ok[u]) load_run<B, 4>(v[u], S, flat_elem(lb, u));
      else
#pragma unroll
        for (int q = 0; q < 4; ++q) v[u][q] = B(0);
    }
#pragma unroll
    for (int u = 0; u < FLAT_PPT; ++u)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[u][q] += ci * (double)v[u][q];
  }
  const DevLevel &L = levs[p];
#pragma unroll
  for (int u = 0; u < FLAT_PPT; ++u) {
    if (!ok[u]) continue;
    const long long e = flat_elem(lb, u);
    B o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = (B)acc[u][q];
    store_run<B, 4>(D, e, o, 4);
    if (stage) {
      uint8_t m4[4];
      load_run<uint8_t, 4>(m4, glob(L.mask), e);
      T r4[4], z4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) { r4[q] = (m4[q] & 64) ? (T)o[q] : T(0); z4[q] = T(0); }
      store_run<T, 4>(PrecOf<T>::rhs(L), e, r4, 4);
      store_run<T, 4>(PrecOf<T>::x(L), e, z4, 4);
    }
  }
}

// P += sum_{i<ns} c_{1+i} Z_i (c_0 is 1)
template <typename B>
__global__ void __launch_bounds__(FLAT_THREADS)
k_kr_update(const int *off, int nent, const KDesc *kd, int ns, const double *coef, int cs,
            const KCtl *ctl) {
  if (ctl) ns = ctl->jlast;
  if (ns == 0) return;
  const int p = find_entry(off, nent, blockIdx.x);
  const int lb = blockIdx.x - off[p];
  const KDesc &d = kd[p];
  const long long lim = flat_end(d.n);
  const double *cf = coef + (size_t)p * cs;
  auto P = glob(mkptr<double>(d.P, d.n, K_X));
  double acc[FLAT_PPT][4];
  bool ok[FLAT_PPT];
#pragma unroll
  for (int u = 0; u < FLAT_PPT; ++u) {
    const long long e = flat_elem(lb, u);
    ok[u] = e < lim;
    if (ok[u]) load_run<double, 4>(acc[u], P, e);
  }
  for (int i = 0; i < ns; ++i) {
    const double ci = cf[1 + i];
    auto S = kvec<B>(d, d.Z, i);
#pragma unroll
    for (int u = 0; u < FLAT_PPT; ++u) {
      if (!ok[u]) continue;
      B v[4];
      load_run<B, 4>(v, S, flat_elem(lb, u));
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[u][q] += ci * (double)v[q];
    }
  }
#pragma unroll
  for (int u = 0; u < FLAT_PPT; ++u)
    if (ok[u]) store_run<double, 4>(P, flat_elem(lb, u), acc[u], 4);
}

static int rows_blocks(const DevRows &R) { return (R.n + CELL_BLOCK - 1) / CELL_BLOCK; }

template <typename B>
cudaError_t kr_resid(const Launch &quads, const DevRows &R, const DevLevel *lev0, const KDesc *kd, int vd,
                     double *part, double *norm2, cudaStream_t s) {
  if (quads.empty()) return cudaSuccess;
  k_kr_resid<B><<<quads.blocks, QBLOCK, 0, s>>>(quads.off, quads.n, quads.lev, kd, vd, part);
  k_reduce_parts<<<quads.n, 1024, 0, s>>>(quads.off, part, norm2);
  note_launches(2);
  if (R.n > 0) {
    k_kr_rows<B><<<rows_blocks(R), CELL_BLOCK, 0, s>>>(R, lev0, kd, 0, 0, vd, nullptr, 0);
    note_launches(1);
  }
  return cudaGetLastError();
}

template <typename B, typename T>
cudaError_t kr_apply(const Launch &quads, const DevRows &R, const DevLevel *lev0, const KDesc *kd, int vz,
                     int vw, cudaStream_t s) {
  if (quads.empty()) return cudaSuccess;
  k_kr_apply_q<B, T><<<quads.blocks, QBLOCK, 0, s>>>(quads.off, quads.n, quads.lev, kd, vz, vw, nullptr);
  note_launches(1);
  if (R.n > 0) {
    k_kr_rows<B><<<rows_blocks(R), CELL_BLOCK, 0, s>>>(R, lev0, kd, 1, vz, vw, nullptr, 0);
    note_launches(1);
  }
  return cudaGetLastError();
}

template <typename B>
cudaError_t kr_dots(const Launch &flat, const KDesc *kd, int vw, int nv, double *part, double *out,
                    int ostride, cudaStream_t s) {
  if (flat.empty()) return cudaSuccess;
  if (nv > KR_MAXV) return cudaErrorInvalidValue;
  k_kr_dots<B><<<flat.blocks, FLAT_THREADS, 0, s>>>(flat.off, flat.n, kd, vw, nv, flat.blocks, part,
                                                    nullptr, 0);
  k_kr_reduce<<<dim3(flat.n, nv + 1), 256, 0, s>>>(flat.off, part, flat.blocks, out, ostride, nullptr, 0);
  note_launches(2);
  return cudaGetLastError();
}

template <typename B, typename T>
cudaError_t kr_vaxpy(const Launch &flat, const DevRows &R, const DevLevel *lev0, const KDesc *kd, int vd,
                     int s0, int ns, const double *coef, int cs, bool stage, cudaStream_t s) {
  if (flat.empty()) return cudaSuccess;
  if (ns > KR_MAXV) return cudaErrorInvalidValue;
  k_kr_vaxpy<B, T><<<flat.blocks, FLAT_THREADS, 0, s>>>(flat.off, flat.n, flat.lev, kd, vd, s0, ns, coef,
                                                        cs, stage ? 1 : 0, nullptr, 0);
  note_launches(1);
  if (stage && R.n > 0) {
    k_kr_rows<B><<<rows_blocks(R), CELL_BLOCK, 0, s>>>(R, lev0, kd, 2, vd, vd, nullptr, 0);
    note_launches(1);
  }
  return cudaGetLastError();
}

template <typename B>
cudaError_t kr_update(const Launch &flat, const KDesc *kd, int ns, const double *coef, int cs,
                      cudaStream_t s) {
  if (flat.empty() || ns == 0) return cudaSuccess;
  if (ns > KR_MAXV) return cudaErrorInvalidValue;
  k_kr_update<B><<<flat.blocks, FLAT_THREADS, 0, s>>>(flat.off, flat.n, kd, ns, coef, cs, nullptr);
  note_launches(1);
  return cudaGetLastError();
}

template cudaError_t kr_resid<float>(const Launch &, const DevRows &, const DevLevel *, const KDesc *, int,
                                     double *, double *, cudaStream_t);
template cudaError_t kr_resid<double>(const Launch &, const DevRows &, const DevLevel *, const KDesc *, int,
                                      double *, double *, cudaStream_t);
template cudaError_t kr_apply<float, float>(const Launch &, const DevRows &, const DevLevel *, const KDesc *,
                                            int, int, cudaStream_t);
template cudaError_t kr_apply<double, double>(const Launch &, const DevRows &, const DevLevel *,
                                              const KDesc *, int, int, cudaStream_t);
template cudaError_t kr_dots<float>(const Launch &, const KDesc *, int, int, double *, double *, int,
                                    cudaStream_t);
template cudaError_t kr_dots<double>(const Launch &, const KDesc *, int, int, double *, double *, int,
                                     cudaStream_t);
template cudaError_t kr_vaxpy<float, float>(const Launch &, const DevRows &, const DevLevel *, const KDesc *,
                                            int, int, int, const double *, int, bool, cudaStream_t);
template cudaError_t kr_vaxpy<double, double>(const Launch &, const DevRows &, const DevLevel *,
                                              const KDesc *, int, int, int, const double *, int, bool,
                                              cudaStream_t);
template cudaError_t kr_update<float>(const Launch &, const KDesc *, int, const double *, int, cudaStream_t);
template cudaError_t kr_update<double>(const Launch &, const KDesc *, int, const double *, int, cudaStream_t);

// ---- the same passes with their indices read on the device (phase KPH_*)
template <typename B, typename T>
cudaError_t krd_apply(const Launch &quads, const DevRows &R, const DevLevel *lev0, const KDesc *kd,
                      const KCtl *ctl, cudaStream_t s) {
  if (quads.empty()) return cudaSuccess;
  k_kr_apply_q<B, T><<<quads.blocks, QBLOCK, 0, s>>>(quads.off, quads.n, quads.lev, kd, 0, 0, ctl);
  note_launches(1);
  if (R.n > 0) {
    k_kr_rows<B><<<rows_blocks(R), CELL_BLOCK, 0, s>>>(R, lev0, kd, 1, 0, 0, ctl, KPH_APPLY);
    note_launches(1);
  }
  return cudaGetLastError();
}

template <typename B>
cudaError_t krd_dots(const Launch &flat, const KDesc *kd, const KCtl *ctl, int phase, double *part,
                     double *out, cudaStream_t s) {
  if (flat.empty()) return cudaSuccess;
  k_kr_dots<B><<<flat.blocks, FLAT_THREADS, 0, s>>>(flat.off, flat.n, kd, 0, 0, flat.blocks, part, ctl,
                                                    phase);
  k_kr_reduce<<<dim3(flat.n, KR_MAXV + 1), 256, 0, s>>>(flat.off, part, flat.blocks, out, KR_CS, ctl, phase);
  note_launches(2);
  return cudaGetLastError();
}

template <typename B, typename T>
cudaError_t krd_vaxpy(const Launch &flat, const DevRows &R, const DevLevel *lev0, const KDesc *kd,
                      const KCtl *ctl, int phase, const double *coef, cudaStream_t s) {
  if (flat.empty()) return cudaSuccess;
  k_kr_vaxpy<B, T><<<flat.blocks, FLAT_THREADS, 0, s>>>(flat.off, flat.n, flat.lev, kd, 0, 0, 0, coef, KR_CS,
                                                        0, ctl, phase);
  note_launches(1);
  if (phase != KPH_REORTH && R.n > 0) {  // staged row constants (skipped on the device when not staged)
    k_kr_rows<B><<<rows_blocks(R), CELL_BLOCK, 0, s>>>(R, lev0, kd, 2, 0, 0, ctl, phase);
    note_launches(1);
  }
  return cudaGetLastError();
}

template <typename B>
cudaError_t krd_update(const Launch &flat, const KDesc *kd, const KCtl *ctl, const double *coef,
                       cudaStream_t s) {
  if (flat.empty()) return cudaSuccess;
  k_kr_update<B><<<flat.blocks, FLAT_THREADS, 0, s>>>(flat.off, flat.n, kd, 0, coef, KR_CS, ctl);
  note_launches(1);
  return cudaGetLastError();
}

template cudaError_t krd_apply<float, float>(const Launch &, const DevRows &, const DevLevel *, const KDesc *,
                                             const KCtl *, cudaStream_t);
template cudaError_t krd_apply<double, double>(const Launch &, const DevRows &, const DevLevel *,
                                               const KDesc *, const KCtl *, cudaStream_t);
template cudaError_t krd_dots<float>(const Launch &, const KDesc *, const KCtl *, int, double *, double *,
                                     cudaStream_t);
template cudaError_t krd_dots<double>(const Launch &, const KDesc *, const KCtl *, int, double *, double *,
                                      cudaStream_t);
template cudaError_t krd_vaxpy<float, float>(const Launch &, const DevRows &, const DevLevel *, const KDesc *,
                                             const KCtl *, int, const double *, cudaStream_t);
template cudaError_t krd_vaxpy<double, double>(const Launch &, const DevRows &, const DevLevel *,
                                               const KDesc *, const KCtl *, int, const double *, cudaStream_t);
template cudaError_t krd_update<float>(const Launch &, const KDesc *, const KCtl *, const double *,
                                       cudaStream_t);
template cudaError_t krd_update<double>(const Launch &, const KDesc *, const KCtl *, const double *,
                                        cudaStream_t);

// ---- scalar FGMRES steps: one block, problem p on thread p (mod 256)
constexpr int FG_SCALAR_THREADS = 256;

// Second Gram-Schmidt pass when the first leaves less than this fraction of
// |w|^2.  With a V-cycle preconditioner w = A M^-1 v_j lies mostly in the
// span of the basis, so the usual 1/2 test asks for the second pass on
// almost every step; at 1e-4 the FP32 basis of small sphere and ellipsoid
// problems loses enough orthogonality to cost two extra cycles, at 1e-2
// they keep theirs and the large box case its time; without any second
// pass the strict convergence cases stall.
constexpr double kReorth = 1e-2;

__device__ __forceinline__ void hist_push(KCtl *ctl, double v) {
  if (ctl->nhist < KR_HIST) ctl->hist[ctl->nhist] = v;
  ctl->nhist++;
}

// block-wide AND of `flag` and max of `v` (non-negative) over the threads
__device__ __forceinline__ void block_all_max(int &flag, double &v) {
  __shared__ int s_flag[FG_SCALAR_THREADS / 32];
  __shared__ double s_v[FG_SCALAR_THREADS / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  flag = __all_sync(0xffffffffu, flag);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  if (l == 0) { s_flag[w] = flag; s_v[w] = v; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < FG_SCALAR_THREADS / 32; ++q) { flag = flag && s_flag[q]; v = fmax(v, s_v[q]); }
  }
}

__global__ void __launch_bounds__(FG_SCALAR_THREADS) k_fg_begin(KCtl *ctl, int np, int m, int max_cycles,
                                                                 double rtol) {
  if (threadIdx.x != 0) return;
  ctl->np = np; ctl->m = m; ctl->max_cycles = max_cycles; ctl->rtol = rtol;
  ctl->cycles = 0; ctl->j = 0; ctl->jlast = 0; ctl->first = 1; ctl->status = FG_NOT_CONVERGED;
  ctl->outer = 1; ctl->inner = 0; ctl->reorth = 0; ctl->more = 0;
  ctl->n_restart = 0; ctl->n_body = 0; ctl->n_inner = 0; ctl->n_reorth = 0;
  ctl->relres_max = 0.0; ctl->nhist = 0;
}

// After the true residual V_0 = F - A P: per problem |f|^2 (first restart),
// the relative residual, beta = |V_0| and whether it is done; the solve
// continues unless every problem meets rtol or the cycles are used up.
// Stages the coefficients of V_0 / beta and resets the rotated system.
__global__ void __launch_bounds__(FG_SCALAR_THREADS)
k_fg_restart(KCtl *ctl, KProb *kp, const double *kout, const double *norm, double *coef, int use_cond,
             cudaGraphConditionalHandle h_outer, cudaGraphConditionalHandle h_body,
             cudaGraphConditionalHandle h_inner) {
  const int np = ctl->np, m = ctl->m;
  const int first = ctl->first;
  const double rtol = ctl->rtol;
  int all = 1;
  double worst = 0.0;
  for (int p = threadIdx.x; p < np; p += FG_SCALAR_THREADS) {
    KProb &q = kp[p];
    if (first) q.f2 = norm[np + p];
    q.relres = q.f2 > 0.0 ? sqrt(norm[p] / q.f2) : sqrt(norm[p]);
    q.beta = sqrt(fmax(0.0, kout[(size_t)p * KR_CS]));
    q.done = (q.relres <= rtol || q.beta == 0.0) ? 1 : 0;
    worst = fmax(worst, q.relres);
    if (!q.done) all = 0;
    double *cf = coef + (size_t)p * KR_CS;
    cf[0] = q.done ? 0.0 : 1.0 / q.beta;
    q.ncol = 0;
    for (int i = 0; i <= m; ++i) q.g[i] = 0.0;
    q.g[0] = q.beta;
  }
  block_all_max(all, worst);
  if (threadIdx.x == 0) {
    ctl->first = 0;
    hist_push(ctl, worst);
    ctl->relres_max = worst;
    ctl->n_restart++;
    int outer = 1;
    if (all) { ctl->status = FG_OK; outer = 0; }
    else if (ctl->cycles >= ctl->max_cycles) outer = 0;
    ctl->outer = outer;
    ctl->inner = outer;
    ctl->j = 0;
    ctl->jlast = 0;
    if (outer) ctl->n_body++;
    if (use_cond) {
      cudaGraphSetConditional(h_outer, outer);
      cudaGraphSetConditional(h_body, outer);
      cudaGraphSetConditional(h_inner, outer);
    }
  }
}

// After the first Gram-Schmidt dots of step j: the Hessenberg column, and
// whether any problem needs the second pass (its coefficients staged).
__global__ void __launch_bounds__(FG_SCALAR_THREADS)
k_fg_reorth_test(KCtl *ctl, KProb *kp, const double *kout, double *coef, int use_cond,
                 cudaGraphConditionalHandle h_reorth) {
  const int np = ctl->np, j = ctl->j;
  int none = 1;
  double dummy = 0.0;
  for (int p = threadIdx.x; p < np; p += FG_SCALAR_THREADS) {
    KProb &q = kp[p];
    const double *o = kout + (size_t)p * KR_CS;
    double sum = 0.0;
    for (int i = 0; i <= j; ++i) { q.hcol[i] = o[i]; sum += o[i] * o[i]; }
    const double ww = o[j + 1];
    if (!q.done && ww - sum < kReorth * ww) none = 0;
    double *cf = coef + (size_t)p * KR_CS;
    cf[0] = 1.0;
    for (int i = 0; i <= j; ++i) cf[1 + i] = q.done ? 0.0 : -q.hcol[i];
  }
  block_all_max(none, dummy);
  if (threadIdx.x == 0) {
    ctl->cycles++;  // the V-cycle of this step
    ctl->reorth = none ? 0 : 1;
    if (!none) ctl->n_reorth++;
    if (use_cond) cudaGraphSetConditional(h_reorth, none ? 0u : 1u);
  }
}

// Normalises step j: h_{j+1,j}, the rotations, the rotated right-hand
// side, the residual estimate; stages the coefficients of
// V_{j+1} = (W - sum h_i V_i) / h_{j+1,j}; decides whether another inner
// step follows.
__global__ void __launch_bounds__(FG_SCALAR_THREADS)
k_fg_arnoldi(KCtl *ctl, KProb *kp, const double *kout, double *coef, int use_cond,
             cudaGraphConditionalHandle h_inner) {
  const int np = ctl->np, j = ctl->j, m = ctl->m, reorth = ctl->reorth;
  const double rtol = ctl->rtol;
  int inner_done = 1;
  double west = 0.0;
  for (int p = threadIdx.x; p < np; p += FG_SCALAR_THREADS) {
    KProb &q = kp[p];
    double *cf = coef + (size_t)p * KR_CS;
    const double *o = kout + (size_t)p * KR_CS;
    double sum = 0.0;
    for (int i = 0; i <= j; ++i) {
      const double hi = o[i];  // second-pass corrections when reorthogonalised
      if (reorth) q.hcol[i] += hi;
      sum += hi * hi;
    }
    const double h2 = o[j + 1] - sum;
    const double hn = h2 > 0.0 ? sqrt(h2) : 0.0;
    q.hcol[j + 1] = hn;
    const bool brk = q.done || !(hn > 1e-14 * q.beta);
    cf[0] = brk ? 0.0 : 1.0 / hn;
    for (int i = 0; i <= j; ++i) cf[1 + i] = brk ? 0.0 : -o[i] / hn;
    if (!q.done) {
      for (int i = 0; i <= j + 1; ++i) q.H[i * KR_MAXV + j] = q.hcol[i];
      for (int i = 0; i < j; ++i) {
        const double c = q.cs[i], sv = q.sn[i];
        const double h0 = q.H[i * KR_MAXV + j], h1 = q.H[(i + 1) * KR_MAXV + j];
        q.H[i * KR_MAXV + j] = c * h0 + sv * h1;
        q.H[(i + 1) * KR_MAXV + j] = -sv * h0 + c * h1;
      }
      const double a = q.H[j * KR_MAXV + j], bb = q.H[(j + 1) * KR_MAXV + j];
      const double rr = hypot(a, bb);
      const double c = rr > 0.0 ? a / rr : 1.0, sv = rr > 0.0 ? bb / rr : 0.0;
      q.cs[j] = c; q.sn[j] = sv;
      q.H[j * KR_MAXV + j] = rr; q.H[(j + 1) * KR_MAXV + j] = 0.0;
      q.g[j + 1] = -sv * q.g[j];
      q.g[j] = c * q.g[j];
      q.ncol = j + 1;
      if (brk) q.done = 1;
    }
    // residual estimate |g_ncol| (all rows) over the fluid-row |f|
    const double est = fabs(q.g[q.ncol]);
    const double rel = q.f2 > 0.0 ? est / sqrt(q.f2) : est;
    west = fmax(west, rel);
    if (!(q.done || rel <= 0.5 * rtol)) inner_done = 0;
  }
  block_all_max(inner_done, west);
  if (threadIdx.x == 0) {
    hist_push(ctl, west);
    ctl->jlast = j + 1;
    ctl->j = j + 1;
    const int more = (!inner_done && j + 1 < m && ctl->cycles < ctl->max_cycles) ? 1 : 0;
    ctl->more = more;
    ctl->inner = more;
    ctl->n_inner++;
    if (use_cond) cudaGraphSetConditional(h_inner, more);
  }
}

// End of a restart cycle: y from the rotated Hessenberg system (back
// substitution), staged as the coefficients of P += sum y_i Z_i.
__global__ void __launch_bounds__(FG_SCALAR_THREADS) k_fg_lsq(KCtl *ctl, KProb *kp, double *coef) {
  const int np = ctl->np;
  for (int p = threadIdx.x; p < np; p += FG_SCALAR_THREADS) {
    const KProb &q = kp[p];
    double *cf = coef + (size_t)p * KR_CS;
    for (int i = 0; i < KR_CS; ++i) cf[i] = 0.0;
    cf[0] = 1.0;
    const int nc = q.ncol;
    double y[KR_MAXV];
    for (int i = nc - 1; i >= 0; --i) {
      double v = q.g[i];
      for (int r = i + 1; r < nc; ++r) v -= q.H[i * KR_MAXV + r] * y[r];
      y[i] = q.H[i * KR_MAXV + i] != 0.0 ? v / q.H[i * KR_MAXV + i] : 0.0;
    }
    for (int i = 0; i < nc; ++i) cf[1 + i] = y[i];
  }
}

cudaError_t fg_begin(KCtl *ctl, int np, int m, int max_cycles, double rtol, cudaStream_t s) {
  k_fg_begin<<<1, FG_SCALAR_THREADS, 0, s>>>(ctl, np, m, max_cycles, rtol);
  note_launches(1);
  return cudaGetLastError();
}
cudaError_t fg_restart(KCtl *ctl, KProb *kp, const double *kout, const double *norm, double *coef,
                       int use_cond, unsigned long long h_outer, unsigned long long h_body,
                       unsigned long long h_inner, cudaStream_t s) {
  k_fg_restart<<<1, FG_SCALAR_THREADS, 0, s>>>(ctl, kp, kout, norm, coef, use_cond, h_outer, h_body, h_inner);
  note_launches(1);
  return cudaGetLastError();
}
cudaError_t fg_reorth_test(KCtl *ctl, KProb *kp, const double *kout, double *coef, int use_cond,
                           unsigned long long h_reorth, cudaStream_t s) {
  k_fg_reorth_test<<<1, FG_SCALAR_THREADS, 0, s>>>(ctl, kp, kout, coef, use_cond, h_reorth);
  note_launches(1);
  return cudaGetLastError();
}
cudaError_t fg_arnoldi(KCtl *ctl, KProb *kp, const double *kout, double *coef, int use_cond,
                       unsigned long long h_inner, cudaStream_t s) {
  k_fg_arnoldi<<<1, FG_SCALAR_THREADS, 0, s>>>(ctl, kp, kout, coef, use_cond, h_inner);
  note_launches(1);
  return cudaGetLastError();
}
cudaError_t fg_lsq(KCtl *ctl, KProb *kp, double *coef, cudaStream_t s) {
  k_fg_lsq<<<1, FG_SCALAR_THREADS, 0, s>>>(ctl, kp, coef);
  note_launches(1);
  return cudaGetLastError();
}

#ifdef FG_CHECKED
// first recorded out-of-range access of a checked build: {hits, index,
// limit, kind, kinds bitmask}; resets the record
extern "C" fg_status fg_debug_check(long long *out) {
  CheckRec h{};
  if (cudaMemcpyFromSymbol(&h, g_check, sizeof(h)) != cudaSuccess) return FG_CUDA_ERROR;
  out[0] = (long long)h.hits; out[1] = h.idx; out[2] = h.lim; out[3] = h.kid; out[4] = h.kinds;
  const CheckRec z{};
  if (cudaMemcpyToSymbol(g_check, &z, sizeof(z)) != cudaSuccess) return FG_CUDA_ERROR;
  return FG_OK;
}
#endif

template cudaError_t line_sweep<double>(const Launch &, int, int, double, int, int, cudaStream_t);
template cudaError_t line_sweep<float>(const Launch &, int, int, double, int, int, cudaStream_t);
template cudaError_t residual<double>(const Launch &, double *, double *, cudaStream_t);
template cudaError_t residual_q<double>(const Launch &, cudaStream_t);
template cudaError_t residual_q<float>(const Launch &, cudaStream_t);
template cudaError_t prolong_add<double>(const Launch &, const DevLevel *, cudaStream_t);
template cudaError_t prolong_add<float>(const Launch &, const DevLevel *, cudaStream_t);
template cudaError_t residual<float>(const Launch &, double *, double *, cudaStream_t);
template cudaError_t restrict_to<double>(const Launch &, const DevLevel *, cudaStream_t);
template cudaError_t restrict_to<float>(const Launch &, const DevLevel *, cudaStream_t);
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

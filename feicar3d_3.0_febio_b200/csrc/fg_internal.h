// fg_internal.h -- shared declarations of the B200 pressure-Poisson library.
//
// Device layout of one multigrid level (every level of every problem):
//   value(i, j, k) at  base[i + sy*j + sz*k],  i in [0, nx+1], j in [0, ny+1],
//   k in [0, nz+1]; nx, ny, nz are CELL counts (reference node count - 1),
//   interior cells are 1..n, index 0 and n+1 are the boundary layers of the
//   reference arrays (its indices 0 and the node count).  sy is rounded up
//   to a multiple of 32 elements so every row starts on a 256-byte boundary.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/feicar_b200.h"

namespace fg {

// cell types of a level
enum : int8_t {
  T_ACTIVE = 0,  // fluid row of the 7-point operator
  T_GHOST = 1,   // ghost or dead cell: value from its interpolation row
  T_OFF = 2,     // coarse cell with >= 50 % solid volume: excluded, no flux
  T_BOUND = 3,   // boundary layer (outside the interior)
  T_SOLID = 4    // pure solid cell (iblank, not dead): value held
};

constexpr int kMaxLevels = 12;
constexpr int kRowPitch = 32;  // elements

// Device arrays of the level and row descriptors.  In a checked build
// (-DFG_CHECKED, for diagnosing a memory fault) each one carries its length:
// an index outside it is recorded (first offender, hit count, kinds hit) and
// the access goes to a scratch slot, so the faulting access never happens.
// Normal builds use plain pointers and generate the same code as without.
#ifdef FG_CHECKED
struct CheckRec {
  unsigned long long hits;
  long long idx, lim;
  int kid;
  unsigned kinds;
};
static __device__ CheckRec g_check;
static __device__ double g_check_sink[8];
__device__ __forceinline__ void check_record(long long i, long long n, int kid) {
  if (atomicAdd(&g_check.hits, 1ull) == 0ull) {
    g_check.idx = i;
    g_check.lim = n;
    g_check.kid = kid;
  }
  atomicOr(&g_check.kinds, 1u << (kid & 31));
}
template <class T>
struct DPtr {
  T *p;
  long long n;
  int kid;
  __host__ __device__ DPtr() : p(nullptr), n(0), kid(0) {}
  __host__ __device__ DPtr(T *q, long long m, int k) : p(q), n(m), kid(k) {}
  template <class U>
  __host__ __device__ DPtr(const DPtr<U> &o) : p(o.p), n(o.n), kid(o.kid) {}
  __device__ T &operator[](long long i) const {
    if (p != nullptr && i >= 0 && i < n) return p[i];
    check_record(i, p ? n : -1, kid);
    return *reinterpret_cast<T *>(g_check_sink);
  }
  __host__ __device__ DPtr operator+(long long o) const { return DPtr(p + o, n - o, kid); }
  __host__ __device__ explicit operator bool() const { return p != nullptr; }
};
template <class T> using dptr = DPtr<T>;
template <class T>
__host__ __device__ inline DPtr<T> mkptr(T *p, long long n, int kid) { return DPtr<T>(p, n, kid); }
#define FG_RESTRICT
#else
template <class T> using dptr = T *;
template <class T>
__host__ __device__ inline T *mkptr(T *p, long long, int) { return p; }
#define FG_RESTRICT __restrict__
#endif

// A level array's pointer marked as global memory (the pointers are read
// from the level descriptors, so the compiler cannot tell their address
// space): loads and stores through it take the global forms, not the
// generic ones.  Checked builds keep their bounds-checked pointers.
#ifdef FG_CHECKED
template <class P> __device__ __forceinline__ P glob(P p) { return p; }
#else
template <class T> __device__ __forceinline__ T *glob(T *p) {
  __builtin_assume(__isGlobal(p));
  return p;
}
#endif

// array kinds reported by a checked build
enum : int {
  K_TYPE = 1, K_MASK = 2, K_AXIS = 3, K_WIDTH = 4, K_CHILD = 5, K_PROL = 6, K_X = 7, K_RHS = 8,
  K_RES = 9, K_ROWS = 10, K_SMEM_D = 11, K_SMEM_F = 12
};

struct DevLevel {
  int nx, ny, nz;        // interior cells per axis
  int pad_;
  long long sy, sz;      // strides in elements
  long long ntot;        // elements of one field
  dptr<const int8_t> type;
  // per-cell operator mask: bit q (0..5) = face q coupled (neighbour
  // active, ghost or solid; faces -x,+x,-y,+y,-z,+z), bit 6 = active row,
  // bit 7 = receives the coarse correction (active or ghost)
  dptr<const uint8_t> mask;
  // per-axis operator coefficients indexed by cell 1..n (arrays of n+2):
  // am(i) couples cell i to i-1, ap(i) to i+1 (CORE_MG.F90:674-676)
  dptr<const double> amx, apx, amy, apy, amz, apz;
  // cell widths indexed by cell 1..n
  dptr<const double> wx, wy, wz;
  // children (in the next finer level) of each cell of THIS level: [lo, hi]
  dptr<const int> clx, chx, cly, chy, clz, chz;
  // prolongation into THIS level from the next coarser one: lower coarse
  // cell and the weight of the upper one, per fine cell (1..n)
  dptr<const int> plx, ply, plz;
  dptr<const double> pwx, pwy, pwz;
  // y/z line tiles (16 cells of i, one plane) whose inner rows are all
  // active with every face coupled: flag[ti + ntx (plane - 1)], ntx =
  // ceil(nx / 16); such tiles skip the mask decode
  dptr<const uint8_t> regy, regz;
  int bc[6];             // 0 Neumann (face dropped), 1 Dirichlet
  // value arrays (only those of the level's precision are set)
  dptr<double> x64, rhs64, res64;
  dptr<float> x32, rhs32, res32;
};

// interpolation rows of the fine level (ghost or dead cells) of a batch
struct DevRows {
  int n;
  dptr<const int> prob;        // problem of each row
  dptr<const long long> tgt;   // target element index
  dptr<const long long> cell;  // host-cell lower-corner element index
  dptr<const double> w;        // 8 weights per row (own slot zeroed)
  dptr<const double> c0;       // constant term per row (solution form)
  dptr<double> rd;             // row residual, FP64 (correction form constant)
  dptr<float> rf;              // row residual, FP32
};

// one launch over a set of problems: block b belongs to entry p with
// off[p] <= b < off[p+1]; lev[p] is that problem's level descriptor
struct Launch {
  int n = 0;
  int blocks = 0;
  const int *off = nullptr;
  const DevLevel *lev = nullptr;
  int *wave = nullptr;  // y/z sweeps: ticket and plane counters (blocks + 2 ints)
  bool empty() const { return n == 0 || blocks == 0; }
};

void set_last_error(const char *msg, const char *file, int line);
const char *last_error_msg();

// Device memory of the library, through a per-process cache: a freed block
// waits (after a device synchronisation, as cudaFree's own) for the next
// request of its rounded size on its device, so cases that live one
// request, and buffers that grow, map and unmap no memory in steady state.
// The cache holds at most a few GB per device and is emptied when an
// allocation fails.
// host memcpy split over the host threads for large copies (the masks
// handed to the caller: several MB of freshly mapped pages)
void host_copy(void *dst, const void *src, size_t bytes);

cudaError_t dev_alloc_raw(void **p, size_t bytes);
void dev_free(void *p);
// while one lives on a thread, dev_free on that thread skips the
// device-wide wait (the caller has drained every stream that used the
// blocks it frees)
struct IdleFree {
  bool prev;
  IdleFree();
  ~IdleFree();
  IdleFree(const IdleFree &) = delete;
  IdleFree &operator=(const IdleFree &) = delete;
};
template <class T>
inline cudaError_t dev_alloc(T **p, size_t bytes) {
  return dev_alloc_raw(reinterpret_cast<void **>(p), bytes);
}

// kernels launched by this process (every launch site adds its count)
void note_launches(long long n);
long long launches_so_far();
long long thread_launches();  // launches noted by the calling thread

#define FG_CUDA(call)                                                  \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      fg::set_last_error(cudaGetErrorString(e_), __FILE__, __LINE__);  \
      return FG_CUDA_ERROR;                                            \
    }                                                                  \
  } while (0)

// Krylov vectors of one problem (FGMRES outer iteration), all in the finest
// level's layout with the field padding (element 1 on a 16-byte boundary):
// the solution P and right-hand side F in FP64, the basis V_0..V_m and the
// preconditioned vectors Z_0..Z_{m-1} in the basis type B (FP32 in the
// mixed path, FP64 otherwise).  Vector v of a kind starts at its base +
// v*stride.  Every vector is zero outside the rows of the system.
struct KDesc {
  double *P, *F;
  void *V, *Z;
  long long n;       // elements of one vector (the level's ntot)
  long long stride;  // elements from one vector to the next
};
constexpr int KR_MAXV = 16;  // most vectors one dot-product pass reads
constexpr int KR_CS = KR_MAXV + 2;  // stride of the per-problem dot results and coefficients

// The scalar side of FGMRES, kept on the device so a whole solve runs
// without the host: per problem the Hessenberg matrix, the Givens rotations
// and the rotated right-hand side; per batch the step counters and the
// decisions the loop takes (which the host reads in direct mode, and CUDA
// graph conditional nodes read in graph mode).
struct KProb {
  double H[KR_MAXV * KR_MAXV];  // H(i, j) at i * KR_MAXV + j, i <= j + 1 < m + 1
  double g[KR_MAXV + 1];
  double cs[KR_MAXV], sn[KR_MAXV];
  double hcol[KR_MAXV + 1];  // column j of the current Arnoldi step
  double f2, beta, relres;
  int done, ncol;
};
constexpr int KR_HIST = 1024;
struct KCtl {
  int np, m;
  int cycles, max_cycles;  // preconditioner applications so far / allowed
  int j;                   // inner step in progress (vectors V_j -> V_{j+1})
  int jlast;               // basis columns of the current restart cycle
  int first;               // the next restart is the first (records |f|^2)
  int status;              // FG_OK once every problem meets rtol
  int outer;               // the restart just taken continues the solve
  int inner;               // another inner step follows
  int reorth;              // the current step takes a second Gram-Schmidt pass
  int more;                // the next basis vector is staged as preconditioner input
  int n_restart, n_body, n_inner, n_reorth;  // executed sections (launch counting)
  double rtol;
  double relres_max;       // worst true relative residual at the last restart
  int nhist, pad_;
  double hist[KR_HIST];    // worst residual (estimate) after each restart / step
};
// what a Krylov vector kernel reads its vector indices from (the step
// counters of KCtl): see kidx() in fg_mg.cu
enum : int {
  KPH_RESTART = 0,    // resid into V_0, dots of V_0, stage V_0 / beta
  KPH_APPLY = 1,      // Z_j, V_{j+1} = A Z_j, dots of V_{j+1} with V_0..V_j
  KPH_REORTH = 2,     // V_{j+1} -= sum h_i V_i (second pass), no staging
  KPH_NORMALIZE = 3,  // V_jlast = (W - sum h_i V_i) / h, staged when `more`
  KPH_UPDATE = 4      // P += sum y_i Z_i over jlast columns
};

// A problem's small levels that one block cycles through (k_small_cycle):
// levels [l0, l0 + nl) of a packed DevLevel table, the last one the
// coarsest, with its generalised inverse G (gn x gn) over the cells gidx.
constexpr int SC_THREADS = 256;           // threads of the block
constexpr int SC_MAXN = 32;               // longest line of such a level
constexpr long long SC_MAXCELLS = 2048;   // most cells of any such level
struct SmallProb {
  int l0, nl;
  const double *G;
  const int *gidx;
  int gn;
};

// kernel launchers (fg_mg.cu)
namespace k {
// blocks needed by one problem's level for each kernel family
int blocks_cells(const DevLevel &L);
// flat passes over the n elements of a level-0 field (Krylov vectors)
int blocks_flat(long long n);
// quad kernels (4 cells of a row per thread)
int blocks_quads(const DevLevel &L);
// the prolongation into a level (shared-memory tiles of PT_I x PT_J cells
// of one plane)
int blocks_ptile(const DevLevel &L);
// line kernel families of a sweep (chosen per level set and axis, by
// default or by the autotuner): x lines in registers (lanes by line
// length, or always 32), x lines staged in shared memory (one warp per
// line); y/z tiles in registers with a per-line Thomas over the chunks,
// with a block-wide PCR over the chunks, or one warp per line; the PCR
// tile with every row's loads issued first at fewer blocks per SM (8 rows
// per thread), with 4 rows per thread and twice the chunks, or both
// colours of a sweep in one launch (plane-ordered tickets)
enum : int {
  LV_DEFAULT = 0,
  LV_XREG = 1, LV_XREG32 = 2, LV_XSMEM = 3,
  LV_YREG = 1, LV_YPCR = 2, LV_YWARP = 3, LV_YPCRH = 4, LV_YPCR4 = 5, LV_YWAVE = 6
};
constexpr int LV_NX = 3, LV_NYZ = 6;  // families per axis kind
// the family does both colours in the colour-0 call of line_sweep (the
// colour-1 call launches nothing)
bool line_both_colours(int axis, int maxn, int variant);
// FG_TIMEOUT (once) if a both-colour y/z sweep gave up a wait since the
// last call
fg_status wave_error_take();
int line_variant(int axis, int maxn, int v);  // the family that runs
int blocks_xline(const DevLevel &L, int maxn, int variant);
// y/z tiles: blocks depend on the kernel the level set's longest line picks
int blocks_tile(const DevLevel &L, int axis, int maxn, int variant);
size_t smem_line(int n, int tsize, int axis);

template <typename T>
cudaError_t line_sweep(const Launch &L, int axis, int color, double omega, int maxn, int variant,
                       cudaStream_t s);
// norm2[p] += ||r||^2 of entry p when norm2 != null (part: one double per block)
template <typename T>
cudaError_t residual(const Launch &L, double *norm2, double *part, cudaStream_t s);
template <typename T>
cudaError_t restrict_to(const Launch &fine_cells_of_coarse, const DevLevel *fine,
                        cudaStream_t s);
template <typename T>
cudaError_t prolong_add(const Launch &fine, const DevLevel *coarse, cudaStream_t s);
// the residual (no norm) with quads: Launch over the level's quads
// (blocks_quads)
template <typename T>
cudaError_t residual_q(const Launch &quads, cudaStream_t s);
template <typename T>
cudaError_t zero_x(const Launch &L, cudaStream_t s);
// the V-cycle of each problem's small levels, one block per problem
template <typename T>
cudaError_t small_cycle(int nprob, const SmallProb *probs, const DevLevel *levs, int maxgn, int nu1,
                        int nu2, double omega, cudaStream_t s);
template <typename T>
cudaError_t rows_relax(const DevRows &R, const DevLevel *lev0, int correction_form,
                       double *tmp, cudaStream_t s);
cudaError_t rows_residual(const DevRows &R, const DevLevel *lev0, double *maxabs,
                          cudaStream_t s);
template <typename T>
cudaError_t coarsest_solve(int nprob, const DevLevel *lev, const double *const *ginv,
                           const int *const *gidx, const int *gn, int maxn, cudaStream_t s);
cudaError_t correct_residual(const Launch &L0, double *norm2, double *part, cudaStream_t s);
cudaError_t fluid_norm(const Launch &L, double *norm2, double *part, cudaStream_t s);
// row constants on the device (one thread per interpolation row):
// c0[r] = (fallback ? sum w p_old / sum w : 0) + a dpdn + dpdn b, with dpdn =
// dpdn[src[r]] (ghost rows after the nd dead ones) or 0 without dp/dn data
struct RowConstGeo {
  const int *src;
  const int8_t *fb;
  const double *a, *b;
  const long long *fid;  // 8 per row, -1 = not a fallback corner
  const double *fw;      // 8 per row
};
cudaError_t row_constants_device(int n, RowConstGeo g, const double *p_old, const double *dpdn_g,
                                 const double *dpdn_d, int nd, double *c0, cudaStream_t s);
// the regular-tile flags of a level (DevLevel::regy, regz) from its masks
cudaError_t reg_tiles(const DevLevel &L, uint8_t *flags_y, uint8_t *flags_z, cudaStream_t s);
cudaError_t copy_in(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                    long long sz, cudaStream_t s);
cudaError_t copy_out(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                     long long sz, cudaStream_t s);
// gauge shift and outer boundary layers of a reference-layout field
// (CORE_POISSON.F90:129-149, CORE_SET_OUTER_BC.F90:1088-1170): with all
// faces Neumann and gauge set, p -= p(1,1,1) on every cell of 0..n except
// pure-solid interior cells; then the faces x, y, z in that order copy
// (Neumann) or reflect about ppp (Dirichlet) the first interior layer.
// nx, ny, nz are node counts; lev0 is the host copy of the level-0
// descriptor (its type array marks the pure-solid cells).
// the known outer-face terms of the finest level's right-hand side
// (Dirichlet values, Neumann gradient data); see k_face_rhs
struct FaceData {
  int pbc[6];
  double ppp[6];
  const double *pgrad[6];  // device face arrays or null (zero gradient)
};
cudaError_t face_rhs(double *rhs, const DevLevel &L0, const FaceData &fd, cudaStream_t s);
// the reference's own residual measures on reference-layout fields
// (block partials into part, ref_blocks of them): squared residuals of
// calc_residual, maxima of |p - p_temp| of calc_residual2
int ref_blocks(int nx, int ny, int nz);
// GCM_enforce_p_compatibility on the device: pgrad (the six face arrays
// back to back, x1 x2 y1 y2 z1 z2) shifted by the flux correction of p on
// the faces flagged in the bit mask vzg; met: dx, dy, dz, dxcinv, dycinv,
// dzcinv (n+2 each, reference indexing); part: ref_blocks doubles
cudaError_t compat(const double *p, const int8_t *ib, const int8_t *gh, const double *met, int nx, int ny,
                   int nz, int vzg, double *part, double *corr, double *pgrad, cudaStream_t s);
cudaError_t ref_residual(const double *p, const double *div, const int8_t *ib, const int8_t *gh,
                         const DevLevel &L0, int nx, int ny, int nz, double *part, cudaStream_t s);
cudaError_t ref_change(const double *p, const double *pt, const int8_t *ib, int nx, int ny, int nz, double *part,
                       cudaStream_t s);
cudaError_t finish_field(double *ref, const DevLevel *lev0, int nx, int ny, int nz,
                         const int *pbc, const double *ppp, int gauge, double *scratch,
                         cudaStream_t s);
// FGMRES pieces over the finest level of a batch: `cells` launches over
// the level-0 cells of all problems, `flat` over their vector elements
// (blocks_flat); rows of all problems.  B is the basis type, T the type of
// the preconditioner's level-0 arrays.
//  kr_resid:  V_vd = F - A P (rows included), norm2[p] += fluid-row |r|^2
//  kr_apply:  Z_vz = preconditioner output x_T on rows (0 elsewhere),
//             V_vw = A Z_vz (rows included); launched over the level-0 quads
//  kr_dots:   out[p*ostride + i] = (V_vw, V_i) for i < nv,
//             out[p*ostride + nv] = (V_vw, V_vw)
//  kr_vaxpy:  V_vd = c0 V_vd + sum_{i<ns} c_{1+i} V_{s0+i} (c = coef + p*cs);
//             with stage, also the preconditioner input: rhs_T = V_vd on
//             active rows (0 elsewhere), x_T = 0, row constants = V_vd
//  kr_update: P += sum_{i<ns} c_{1+i} Z_i
template <typename B>
cudaError_t kr_resid(const Launch &cells, const DevRows &R, const DevLevel *lev0, const KDesc *kd, int vd,
                     double *part, double *norm2, cudaStream_t s);
template <typename B, typename T>
cudaError_t kr_apply(const Launch &cells, const DevRows &R, const DevLevel *lev0, const KDesc *kd, int vz,
                     int vw, cudaStream_t s);
template <typename B>
cudaError_t kr_dots(const Launch &flat, const KDesc *kd, int vw, int nv, double *part, double *out,
                    int ostride, cudaStream_t s);
template <typename B, typename T>
cudaError_t kr_vaxpy(const Launch &flat, const DevRows &R, const DevLevel *lev0, const KDesc *kd, int vd,
                     int s0, int ns, const double *coef, int cs, bool stage, cudaStream_t s);
template <typename B>
cudaError_t kr_update(const Launch &flat, const KDesc *kd, int ns, const double *coef, int cs,
                      cudaStream_t s);
// The same vector passes with their vector indices taken on the device from
// ctl (phase KPH_*), so one captured launch serves every step of a loop.
template <typename B, typename T>
cudaError_t krd_apply(const Launch &quads, const DevRows &R, const DevLevel *lev0, const KDesc *kd,
                      const KCtl *ctl, cudaStream_t s);
template <typename B>
cudaError_t krd_dots(const Launch &flat, const KDesc *kd, const KCtl *ctl, int phase, double *part,
                     double *out, cudaStream_t s);
template <typename B, typename T>
cudaError_t krd_vaxpy(const Launch &flat, const DevRows &R, const DevLevel *lev0, const KDesc *kd,
                      const KCtl *ctl, int phase, const double *coef, cudaStream_t s);
template <typename B>
cudaError_t krd_update(const Launch &flat, const KDesc *kd, const KCtl *ctl, const double *coef,
                       cudaStream_t s);
// scalar FGMRES steps (one block over all problems); with use_cond the
// decisions are also written to the CUDA graph conditional handles
cudaError_t fg_begin(KCtl *ctl, int np, int m, int max_cycles, double rtol, cudaStream_t s);
cudaError_t fg_restart(KCtl *ctl, KProb *kp, const double *kout, const double *norm, double *coef,
                       int use_cond, unsigned long long h_outer, unsigned long long h_body,
                       unsigned long long h_inner, cudaStream_t s);
cudaError_t fg_reorth_test(KCtl *ctl, KProb *kp, const double *kout, double *coef, int use_cond,
                           unsigned long long h_reorth, cudaStream_t s);
cudaError_t fg_arnoldi(KCtl *ctl, KProb *kp, const double *kout, double *coef, int use_cond,
                       unsigned long long h_inner, cudaStream_t s);
cudaError_t fg_lsq(KCtl *ctl, KProb *kp, double *coef, cudaStream_t s);
}  // namespace k

}  // namespace fg

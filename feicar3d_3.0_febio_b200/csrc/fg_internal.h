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

struct DevLevel {
  int nx, ny, nz;        // interior cells per axis
  int pad_;
  long long sy, sz;      // strides in elements
  long long ntot;        // elements of one field
  const int8_t *type;
  // per-cell operator mask: bit q (0..5) = face q coupled (neighbour
  // active, ghost or solid; faces -x,+x,-y,+y,-z,+z), bit 6 = active row,
  // bit 7 = receives the coarse correction (active or ghost)
  const uint8_t *mask;
  // per-axis operator coefficients indexed by cell 1..n (arrays of n+2):
  // am(i) couples cell i to i-1, ap(i) to i+1 (CORE_MG.F90:674-676)
  const double *amx, *apx, *amy, *apy, *amz, *apz;
  // cell widths indexed by cell 1..n
  const double *wx, *wy, *wz;
  // children (in the next finer level) of each cell of THIS level: [lo, hi]
  const int *clx, *chx, *cly, *chy, *clz, *chz;
  // prolongation into THIS level from the next coarser one: lower coarse
  // cell and the weight of the upper one, per fine cell (1..n)
  const int *plx, *ply, *plz;
  const double *pwx, *pwy, *pwz;
  int bc[6];             // 0 Neumann (face dropped), 1 Dirichlet
  // value arrays (only those of the level's precision are set)
  double *x64, *rhs64, *res64;
  float *x32, *rhs32, *res32;
};

// interpolation rows of the fine level (ghost or dead cells) of a batch
struct DevRows {
  int n;
  const int *prob;        // problem of each row
  const long long *tgt;   // target element index
  const long long *cell;  // host-cell lower-corner element index
  const double *w;        // 8 weights per row (own slot zeroed)
  const double *c0;       // constant term per row (solution form)
  double *rd;             // row residual, FP64 (correction form constant)
  float *rf;              // row residual, FP32
};

// one launch over a set of problems: block b belongs to entry p with
// off[p] <= b < off[p+1]; lev[p] is that problem's level descriptor
struct Launch {
  int n = 0;
  int blocks = 0;
  const int *off = nullptr;
  const DevLevel *lev = nullptr;
  bool empty() const { return n == 0 || blocks == 0; }
};

void set_last_error(const char *msg, const char *file, int line);
const char *last_error_msg();

#define FG_CUDA(call)                                                  \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      fg::set_last_error(cudaGetErrorString(e_), __FILE__, __LINE__);  \
      return FG_CUDA_ERROR;                                            \
    }                                                                  \
  } while (0)

// kernel launchers (fg_mg.cu)
namespace k {
// blocks needed by one problem's level for each kernel family
int blocks_cells(const DevLevel &L);
int blocks_xline(const DevLevel &L);
int blocks_tile(const DevLevel &L, int axis);
size_t smem_line(int n, int tsize, int lines_per_block);

template <typename T>
cudaError_t line_sweep(const Launch &L, int axis, int color, double omega, int maxn,
                       cudaStream_t s);
// norm2[p] += ||r||^2 of entry p when norm2 != null (part: one double per block)
template <typename T>
cudaError_t residual(const Launch &L, double *norm2, double *part, cudaStream_t s);
template <typename T>
cudaError_t restrict_to(const Launch &fine_cells_of_coarse, const DevLevel *fine,
                        cudaStream_t s);
template <typename T>
cudaError_t prolong_add(const Launch &fine, const DevLevel *coarse, cudaStream_t s);
template <typename T>
cudaError_t zero_x(const Launch &L, cudaStream_t s);
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
cudaError_t copy_in(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                    long long sz, cudaStream_t s);
cudaError_t copy_out(double *dst, const double *src, int nx, int ny, int nz, long long sy,
                     long long sz, cudaStream_t s);
}  // namespace k

}  // namespace fg

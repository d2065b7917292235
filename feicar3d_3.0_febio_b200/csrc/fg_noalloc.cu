// fg_noalloc.cu -- ghost/dead-cell row relaxation that allocates no memory.
//
// Some callers cannot call cudaMalloc: code that only receives device
// memory from a pool or framework it does not own, code running where an
// allocation would synchronise the device or break a latency budget, and
// Fortran hosts that hand over arrays they manage themselves. For them
// fg_rows_relax_noalloc runs the same Jacobi update of the interpolation
// rows as fg_ghostcell_pressure, on a field the caller owns, with its
// scratch buffer in a fixed static device array instead of a handle.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "fg_internal.h"

namespace fg {
namespace {

// One scratch value per row. The array exists on every GPU that loads the
// library, for the life of the process: FG_NOALLOC_MAX_ROWS doubles (2 MiB).
static __device__ __align__(256) double g_rows_scratch[FG_NOALLOC_MAX_ROWS];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up
// once per device (host code may not use the array's name as an address).
fg_status scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return FG_CUDA_ERROR;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_last_error("device index beyond the no-alloc table", __FILE__, __LINE__);
    return FG_BAD_INPUT;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    double *p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_rows_scratch);
    if (e != cudaSuccess || !p) {
      set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "no address for the scratch array",
                     __FILE__, __LINE__);
      return FG_CUDA_ERROR;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return FG_OK;
}

// corner order of GCM_MEMORY_ALLOCATE.F90:593-623 in a layout of row stride
// sy and plane stride sz
__device__ __forceinline__ void corners(long long sy, long long sz, long long *o) {
  o[0] = 0; o[1] = sy; o[2] = sy + 1; o[3] = 1;
  o[4] = sz; o[5] = sz + sy; o[6] = sz + sy + 1; o[7] = sz + 1;
}

// scratch[r] = sum_q w[8r+q] p[cell[r] + corner_q] + c0[r]; rows whose
// indices fall outside the field are left out (scratch untouched, no write)
__global__ void k_gather(const double *p, long long nref, long long sy, long long sz, int nrows,
                         const int64_t *tgt, const int64_t *cell, const double *w,
                         const double *c0, double *scratch) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  long long o[8];
  corners(sy, sz, o);
  const long long b = cell[r];
  if (b < 0 || b + o[6] >= nref || tgt[r] < 0 || tgt[r] >= nref) return;
  double acc = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) acc += w[8 * r + q] * p[b + o[q]];
  scratch[r] = acc + (c0 ? c0[r] : 0.0);
}

__global__ void k_scatter(double *p, long long nref, long long sy, long long sz, int nrows,
                          const int64_t *tgt, const int64_t *cell, const double *scratch) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  const long long b = cell[r];
  if (b < 0 || b + sz + sy + 1 >= nref || tgt[r] < 0 || tgt[r] >= nref) return;
  p[tgt[r]] = scratch[r];
}

}  // namespace
}  // namespace fg

extern "C" fg_status fg_rows_relax_noalloc(int nx, int ny, int nz, double *d_p, int nrows,
                                           const int64_t *d_tgt, const int64_t *d_cell,
                                           const double *d_w, const double *d_c0,
                                           int iterations, void *stream) {
  if (nx < 1 || ny < 1 || nz < 1 || nrows < 0 || iterations < 0) return FG_BAD_INPUT;
  if (nrows > FG_NOALLOC_MAX_ROWS) {
    fg::set_last_error("more rows than the static scratch array holds (FG_NOALLOC_MAX_ROWS)",
                       __FILE__, __LINE__);
    return FG_BAD_INPUT;
  }
  if (nrows == 0 || iterations == 0) return FG_OK;
  if (!d_p || !d_tgt || !d_cell || !d_w) return FG_BAD_INPUT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (s) {
    // the scratch address below is the current device's: a stream of
    // another device would run the kernels where that address means nothing
    int cur = 0, sdev = 0;
    cudaError_t e = cudaGetDevice(&cur);
    if (e == cudaSuccess) e = cudaStreamGetDevice(s, &sdev);
    if (e != cudaSuccess) {
      fg::set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
      return FG_CUDA_ERROR;
    }
    if (sdev != cur) {
      fg::set_last_error("stream belongs to another device than the current one", __FILE__, __LINE__);
      return FG_BAD_INPUT;
    }
  }
  double *scratch = nullptr;
  fg_status st = fg::scratch_address(&scratch);
  if (st != FG_OK) return st;
  const long long sy = (long long)nx + 2, sz = sy * ((long long)ny + 2);
  const long long nref = sz * ((long long)nz + 2);
  const int threads = 128, blocks = (nrows + threads - 1) / threads;
  for (int it = 0; it < iterations; ++it) {
    fg::k_gather<<<blocks, threads, 0, s>>>(d_p, nref, sy, sz, nrows, d_tgt, d_cell, d_w, d_c0, scratch);
    fg::k_scatter<<<blocks, threads, 0, s>>>(d_p, nref, sy, sz, nrows, d_tgt, d_cell, scratch);
    fg::note_launches(2);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fg::set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return FG_CUDA_ERROR;
  }
  return FG_OK;
}

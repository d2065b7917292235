// fg_case.h -- host-side state of one case (grid, hierarchy, geometry).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <new>
#include <vector>

#include "fg_internal.h"

namespace fg {

struct Geom;
void geom_free(Geom &g);

// ------------------------------------------------------------ host level
struct HLevel {
  int I = 0, J = 0, K = 0;   // node counts (mgrid_I/J/K)
  int nx = 0, ny = 0, nz = 0;  // cells
  long long sy = 0, sz = 0, ntot = 0;
  std::vector<double> x, y, z, xc, yc, zc;          // 0..n+1 (reference level arrays)
  std::vector<double> dxinv, dyinv, dzinv, dxcinv, dycinv, dzcinv;
  std::vector<int8_t> type;  // device layout, host copy of the coarsest level only
  // device
  int8_t *d_type = nullptr;
  uint8_t *d_mask = nullptr;
  uint8_t *d_reg = nullptr;     // regular-tile flags of the y then the z line tiles
  int8_t *d_ibk = nullptr;      // solid flag (interior cells)
  double *d_nodes = nullptr;    // x, y, z node arrays back to back
  double *d_coef = nullptr;  // packed 1-D double arrays
  int *d_int = nullptr;      // packed 1-D int arrays
  double *d_x64 = nullptr, *d_rhs64 = nullptr, *d_res64 = nullptr;
  float *d_x32 = nullptr, *d_rhs32 = nullptr, *d_res32 = nullptr;
  std::vector<void *> raw;   // allocations behind the offset field pointers
  DevLevel dl{};
};

// page-locked host storage for the masks that cross between host and device
// on every re-tag (copies at full link speed, no staging).  Blocks come
// from a process-wide pool and go back to it: pinning and unpinning pages
// costs milliseconds per call and serialises with the device, too much for
// a case that lives one request.
void *pinned_get(size_t bytes);
void pinned_put(void *p);
template <class T>
struct PinnedAlloc {
  using value_type = T;
  PinnedAlloc() = default;
  template <class U>
  PinnedAlloc(const PinnedAlloc<U> &) {}
  T *allocate(size_t n) {
    void *p = pinned_get(n * sizeof(T));
    if (!p) throw std::bad_alloc();
    return static_cast<T *>(p);
  }
  void deallocate(T *p, size_t) { pinned_put(p); }
};
template <class T, class U>
bool operator==(const PinnedAlloc<T> &, const PinnedAlloc<U> &) { return true; }
template <class T, class U>
bool operator!=(const PinnedAlloc<T> &, const PinnedAlloc<U> &) { return false; }
template <class T>
using pinned_vector = std::vector<T, PinnedAlloc<T>>;

struct RowsHost {
  std::vector<long long> tgt, cell;
  std::vector<double> w, c0;
};

}  // namespace fg

// ---------------------------------------------------------------- case
#include "fg_geom.h"

struct fg_case {
  int device = 0;
  fg_solver_config cfg{};
  int nx = 0, ny = 0, nz = 0;  // node counts
  int nlev = 0;
  fg::HLevel lev[fg::kMaxLevels];
  cudaStream_t stream = nullptr;
  bool own_stream = true;  // false after fg_case_set_stream(c, caller's stream)
  // geometry
  std::unique_ptr<fg::Geom> geom;
  std::vector<double> d_ipv;           // dead-cell image points (3 per row)
  fg::pinned_vector<int8_t> iblank, ghost, dead;  // reference layout (host copies)
  bool has_geometry = false;
  bool prepared = false;
  // interpolation rows (dead rows first, then ghost rows, like the
  // reference's update order)
  int nGhost = 0, nDead = 0;
  std::vector<int32_t> g_ijk, g_cell, d_ijk, d_cell;
  std::vector<double> g_coefN, d_coefN, d_probe;
  std::vector<int8_t> d_fallback;   // dead rows using the inverse-distance fallback
  fg::RowsHost rows;                // device-layout rows
  // coarsest generalised inverse
  std::vector<double> G;
  std::vector<int> gidx;
  double *d_G = nullptr;
  int *d_gidx = nullptr;
  size_t G_cap = 0, gidx_cap = 0;  // elements the two device arrays hold
  long long geom_version = 0;      // bumped by every prepare
  // per interpolation row, for row constants formed on the device: the
  // dp/dn index, its two factors, the fallback corners and weights
  double *d_admet = nullptr;          // momentum sweeps: metrics and set_solve_ad coefficients
  double *d_vbcmet = nullptr;         // outer velocity boundaries: node coordinates y, z
  void *d_rcg = nullptr;
  long long rcg_version = -1;
  int rcg_n = 0;
  fg::k::RowConstGeo rcg_ptrs{};
  // reference-layout staging buffers on the device
  double *d_pin = nullptr, *d_fin = nullptr;
  int8_t *d_refmask = nullptr;      // iblank, ghostCellMark, dead_cell (reference layout)
  long long *d_rowtgt = nullptr;    // level-0 element of every row
  size_t rowtgt_cap = 0;
  double *d_gauge = nullptr;  // p(1,1,1) of the output gauge
  bool batch_dirty = true;
  struct fg_batch *solo = nullptr;
  // outer-face pressure gradients (the reference's pgradx1..pgradz2, six
  // face arrays back to back), the faces whose velocity is zero-gradient
  // (bit mask: solves first apply GCM_enforce_p_compatibility), and the
  // reference 1-D metrics and scratch the compatibility step reads
  double *d_pgrad = nullptr;
  int vzg = 0;
  double *d_met = nullptr;
  double *d_cpart = nullptr;  // flux partials, then the correction
  double *d_pmet = nullptr;   // grid arrays of the projection steps (fg_proj.cu)
};

namespace fg {
// the interpolation rows of a geometry whose masks are already in
// c->iblank / c->ghost / c->dead (argument meaning as fg_case_set_geometry)
fg_status geometry_rows(fg_case *c, int nGhost, const int32_t *ghost_ijk, const int32_t *ghost_cell,
                        const double *ghost_coefN, int nDead, const int32_t *dead_ijk,
                        const int32_t *dead_cell_idx, const double *dead_coefN,
                        const double *dead_probe, const double *dead_ip);
// a solve of the fields staged in c->d_pin / c->d_fin queued on the case's
// stream (output finished into d_pin), and the wait for its outcome
fg_status solve_enqueue(fg_case *c, const double *p_old, const double *dpdn_g, const double *dpdn_d);
// the same with the row constants formed on the device from device p_old
// and dp/dn arrays (each may be NULL)
fg_status solve_enqueue_dev(fg_case *c, const double *d_p_old, const double *d_dpdn_g, const double *d_dpdn_d);
fg_status solve_collect(fg_case *c, fg_solve_stats *st);
}  // namespace fg

// fg_geom.h -- device state of the immersed-boundary tagging of one case.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace fg {

struct DevBody {
  int nvert = 0, ntri = 0, type = 1, body_dim = 3;
  double membrane_tkns = 0.0;
  std::vector<double> xyz;     // host copy, 3 per vertex
  std::vector<int32_t> tri;    // host copy, 3 per triangle (0-based)
  double *d_xyz = nullptr;     // SoA: x[nvert], y[nvert], z[nvert]
  double *d_en = nullptr;      // element normals (3*ntri, SoA)
  double *d_vn = nullptr;      // vertex normals (3*nvert, SoA)
  int32_t *d_tri = nullptr;    // 3*ntri
  int32_t *d_v2t_off = nullptr, *d_v2t = nullptr;  // vertex -> triangles
  // prescribed motion on the device (fg_move_body): marker velocities of
  // this and the previous step, positions at the last re-tag, dp/dn at
  // the markers (all SoA, nvert each); the host copy xyz is brought up to
  // date only when asked for
  double *d_uvw = nullptr, *d_uvw_old = nullptr, *d_snap = nullptr, *d_dpdn = nullptr;
  bool host_stale = false;
};

// Device buffer that only grows: kept across calls, so re-tagging a moving
// body on every time step allocates (and synchronises on a free) only while
// the lists are still growing.
struct DevScratch {
  void *p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    fg::dev_free(p);
    p = nullptr;
    cap = 0;
    const cudaError_t e = fg::dev_alloc(&p, bytes > 0 ? bytes : 1);
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
  void release() { fg::dev_free(p); p = nullptr; cap = 0; }
};

// device outputs of one row list (ghost or dead) of the tagging
struct RowScratch {
  DevScratch bi, bw, ip, nrm, probe, ds, cell, closest, cD, cN;
  void release() {
    bi.release(); bw.release(); ip.release(); nrm.release(); probe.release(); ds.release();
    cell.release(); closest.release(); cD.release(); cN.release();
  }
};

struct Geom {
  std::vector<DevBody> bodies;
  // grow-only scratch of the tagging calls: compaction (CUB temporary
  // storage, selection, count), the band cells, the ghost and dead lists and
  // their row outputs, alpha, the dead-row rank map and the status flags
  DevScratch cub_tmp, sel_out, sel_count, cells, glist, dlist, alpha, rank, flags;
  RowScratch rg, rd;
  int8_t *d_iblank = nullptr, *d_ghost = nullptr, *d_dead = nullptr, *d_body = nullptr;
  int8_t *d_band = nullptr, *d_tmp = nullptr;
  double *d_xc = nullptr;      // xc[0..nx+1], yc, zc concatenated
  int nWarnSide = 0, nHostFail = 0;
  // ghost and dead rows of the last device tagging (-1: the case's rows
  // came from the caller, fg_case_set_geometry, and have no device copy)
  int rows_ng = -1, rows_nd = -1;
  // lists (host copies after fg_gcm_set_internal_boundary)
  std::vector<double> g_coefD, g_bi, g_ip, g_probe, g_alpha, d_coefD, d_bi, d_probe;
  std::vector<int32_t> g_closest, d_closest;
  pinned_vector<char> h_stage;  // page-locked landing area of device -> host copies
  bool tagged = false;
};

}  // namespace fg

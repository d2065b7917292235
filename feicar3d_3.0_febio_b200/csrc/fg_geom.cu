// fg_geom.cu -- immersed-boundary tagging on the device (placeholder entry
// points; the kernels follow).
#include <cuda_runtime.h>

#include "fg_case.h"

namespace fg {
void geom_free(Geom &g) {
  for (auto &b : g.bodies) {
    cudaFree(b.d_xyz); cudaFree(b.d_en); cudaFree(b.d_vn); cudaFree(b.d_tri);
    cudaFree(b.d_v2t_off); cudaFree(b.d_v2t);
  }
  g.bodies.clear();
  cudaFree(g.d_iblank); cudaFree(g.d_ghost); cudaFree(g.d_dead); cudaFree(g.d_body);
  cudaFree(g.d_band); cudaFree(g.d_tmp); cudaFree(g.d_xc);
}
}  // namespace fg

extern "C" {
fg_status fg_case_add_body(fg_case *, int, int, const double *, const int32_t *, int, double, int) { return FG_BAD_INPUT; }
fg_status fg_case_update_body(fg_case *, int, const double *) { return FG_BAD_INPUT; }
fg_status fg_set_iblank_body_fast(fg_case *, int8_t *) { return FG_BAD_INPUT; }
fg_status fg_gcm_set_internal_boundary(fg_case *, int8_t *, int8_t *, int8_t *, int *, int *) { return FG_BAD_INPUT; }
fg_status fg_get_ghost_rows(const fg_case *, int32_t *, int32_t *, double *, double *, double *, double *, double *, int32_t *, double *) { return FG_BAD_INPUT; }
fg_status fg_get_dead_rows(const fg_case *, int32_t *, int32_t *, double *, double *, double *, double *, double *, int32_t *) { return FG_BAD_INPUT; }
fg_status fg_get_band(const fg_case *, int8_t *) { return FG_BAD_INPUT; }
}

// fields_f32.cu -- the grid half of the mixed-precision path: fold, Yee,
// smooth2, Poisson/CG and energies on the FP32 field block, with the CG dot
// products and the energies accumulated in FP64 (grid_kernels.cuh).
#include "fields_impl.cuh"

namespace em2g {

int smooth2_f32(em2g_ctx *c, float *a) { return grid::smooth2_t<float>(c, a, c->smooth_tmp32); }

int cg_init_f32(em2g_ctx *c) { return grid::cg_init_t<float>(c); }

int tma_init_f32(em2g_ctx *c) { return grid::tma_init_t<float>(c, c->fld32, c->smooth_tmp32); }

int fields_f32(em2g_ctx *c, int it, bool want_energies) {
  return grid::fields_t<float>(c, c->fld32, c->smooth_tmp32, it, want_energies);
}

}  // namespace em2g

// fields_f64.cu -- the grid half of the FP64 drop-in path: fold, Yee,
// smooth2, Poisson/CG and energies (pic/fields.f90, pic/smooth.f90) on the
// FP64 field block.  Compiled with -fmad=false: every stencil cell is
// rounded as em2 rounds it, so these sweeps are bitwise em2's for equal
// inputs; the CG dot products and the energies are FP64 tree sums
// (deterministic for a given grid, summed in another order than em2's loops).
#include "fields_impl.cuh"

namespace em2g {

int smooth2_f64(em2g_ctx *c, double *a) {
  return grid::smooth2_t<double>(c, a, c->smooth_tmp);
}

int cg_init(em2g_ctx *c) { return grid::cg_init_t<double>(c); }

int tma_init_f64(em2g_ctx *c) { return grid::tma_init_t<double>(c, c->fld, c->smooth_tmp); }

void cg_free(em2g_ctx *c) {
  cudaFree(c->cg.u);
  cudaFree(c->cg.partial);
  cudaFree(c->cg.bar);
  cudaFree(c->cg.status);
  c->cg = CgWork();
}

// Both bounded device waits made to run out on purpose (the probes of
// grid_kernels.cuh and tma_stencil.cuh), on the context's stream and with
// its CG workspace, which is left as the solver expects it.
int selftest_waits(em2g_ctx *c, int *cg_status, int *tma_status) {
  int st = 0;
  EM2G_CUDA(cudaMemsetAsync(c->cg.bar, 0, sizeof(unsigned) * 2, c->stream));
  EM2G_CUDA(cudaMemsetAsync(c->cg.status, 0, sizeof(int) * 2, c->stream));
  grid::k_barrier_wait_probe<<<1, 32, 0, c->stream>>>(c->cg.bar, c->cg.status);
  EM2G_CUDA(cudaGetLastError());
  EM2G_CUDA(cudaMemcpyAsync(&st, c->cg.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  *cg_status = st;
  EM2G_CUDA(cudaMemsetAsync(c->cg.status, 0, sizeof(int) * 2, c->stream));
  tma::k_tma_wait_probe<<<1, 32, 0, c->stream>>>(c->cg.status);
  EM2G_CUDA(cudaGetLastError());
  EM2G_CUDA(cudaMemcpyAsync(&st, c->cg.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  *tma_status = st;
  EM2G_CUDA(cudaMemsetAsync(c->cg.bar, 0, sizeof(unsigned) * 2, c->stream));
  EM2G_CUDA(cudaMemsetAsync(c->cg.status, 0, sizeof(int) * 2, c->stream));
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  return EM2G_OK;
}

int fields_f64(em2g_ctx *c, int it, bool want_energies, int *cg_iters) {
  (void)cg_iters;  // read from cg.status by the caller after its last launch
  return grid::fields_t<double>(c, c->fld, c->smooth_tmp, it, want_energies);
}

}  // namespace em2g

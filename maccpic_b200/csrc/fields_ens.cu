// fields_ens.cu -- em2's fields (pic/fields.f90:2-366) for every run of an
// ensemble, each stage one launch over all runs.
//
// A stage's blocks are numbered run after run: run r owns blocks
// t0[r] .. t0[r+1]-1 of the launch (its own tile grid, row-major), and a
// block finds its run by a binary search of t0.  The per-cell arithmetic is
// the single-run FP32 path's (the *_at device functions of
// grid_kernels.cuh), so a run of an ensemble computes what an em2g context
// of the same parameters computes.  The CG runs every run's solve in one
// cooperative launch: run r owns its own range of blocks, its own partial
// sums and its own bounded grid barrier, and stops at its own tolerance.
// Stages that apply only every isav steps (the E/B filter, the energies)
// read the step counter from device memory, so one captured graph serves
// every step.
#include <algorithm>
#include <memory>

#include "ens_fields.cuh"

namespace em2g {
namespace {

__global__ void k_ens_tick(int *it) { *it += 1; }

// E and B times ae of species blockIdx.y into the run's (E, B) pairs
// (pic/move.f90:52-64), as k_prescale_f32
__global__ void k_ens_prescale(const __grid_constant__ EnsGrid32 e) {
  const int r = find_run(e.wblk0, e.nruns, blockIdx.x);
  const EnsRunDev &R = e.run[r];
  const int s = blockIdx.y;
  const int64_t w = R.g.w;
  const int64_t k = (int64_t)(blockIdx.x - e.wblk0[r]) * blockDim.x + threadIdx.x;
  if (s >= R.nsp || k >= w) return;
  const float *f = R.fld;
  float2 *o = reinterpret_cast<float2 *>(R.sc + (int64_t)s * 6 * w);
  const float ae = R.ae[s];
  o[k] = make_float2(ae * f[EM2G_EX * w + k], ae * f[EM2G_BX * w + k] + R.tx[s]);
  o[w + k] = make_float2(ae * f[EM2G_EZ * w + k], ae * f[EM2G_BZ * w + k]);
  o[2 * w + k] = make_float2(ae * f[EM2G_EY * w + k], ae * f[EM2G_BY * w + k] + R.ty[s]);
}

__global__ void k_ens_fold_x(const __grid_constant__ EnsGrid32 e) {
  const int r = find_run(e.foldx0, e.nruns, blockIdx.x);
  const EnsRunDev &R = e.run[r];
  grid::fold_x_at(R.g, R.fld, (int)((blockIdx.x - e.foldx0[r]) * blockDim.x + threadIdx.x),
                  (int)blockIdx.y);
}

__global__ void k_ens_fold_y(const __grid_constant__ EnsGrid32 e) {
  const int r = find_run(e.foldy0, e.nruns, blockIdx.x);
  const EnsRunDev &R = e.run[r];
  grid::fold_y_at(R.g, R.fld, (int)((blockIdx.x - e.foldy0[r]) * blockDim.x + threadIdx.x),
                  (int)blockIdx.y);
}

template <int OP>
__global__ void __launch_bounds__(TX *TY) k_ens_sten(const __grid_constant__ EnsGrid32 e,
                                                     int set) {
  const int r = find_run(e.sten0, e.nruns, blockIdx.x);
  const EnsRunDev &R = e.run[r];
  const int lb = blockIdx.x - e.sten0[r];
  const int tby = lb / R.tiles_x, tbx = lb - tby * R.tiles_x;
  const int64_t N = (int64_t)R.g.nx * R.g.ny;
  if (OP == OP_BHALF) {
    grid::b_half_at(R.g, R.fld, R.ctxh, R.ctyh, tbx, tby);
  } else if (OP == OP_EFULL) {
    grid::e_full_at(R.g, R.fld, R.ctx, R.cty, R.tem, tbx, tby);
  } else if (OP == OP_SMOOTH_B || OP == OP_SMOOTH_C) {
    int arr;
    if (!smooth_target(e, R, set, (int)blockIdx.y, &arr)) return;
    float *a = R.fld + arr * R.g.w, *d = R.tmp + blockIdx.y * R.g.w;
    if (OP == OP_SMOOTH_B)
      grid::smooth_binomial_at(R.g, a, d, tbx, tby);
    else
      grid::smooth_compensate_at(R.g, d, a, tbx, tby);
  } else if (OP == OP_RHS) {
    grid::poisson_rhs_at(R.g, R.fld, R.dx, R.dy, R.cgu + N, R.cgu + 2 * N, tbx, tby);
  } else {
    grid::poisson_correct_at(R.g, R.fld, R.cgu, R.dx, R.dy, tbx, tby);
  }
}

__global__ void __launch_bounds__(256) k_ens_cg(const __grid_constant__ EnsCg32 e) {
  __shared__ double sh[33];
  const int r = find_run(e.blk0, e.nruns, blockIdx.x);
  grid::cg_body(e.a[r], (int)blockIdx.x - e.blk0[r], (unsigned)(e.blk0[r + 1] - e.blk0[r]), sh);
}

// field energies of run blockIdx.x, component blockIdx.y, on isav steps
// (pic/fields.f90:267-347 over the whole grid), summed in a fixed order
__global__ void __launch_bounds__(256) k_ens_energy(const __grid_constant__ EnsGrid32 e) {
  __shared__ double sh[32];
  const EnsRunDev &R = e.run[blockIdx.x];
  if ((*e.it % R.isav) != 0) return;
  const float *a = R.fld + blockIdx.y * R.g.w;
  const int nx = R.g.nx;
  const int64_t N = (int64_t)nx * R.g.ny;
  double loc = 0.0;
  for (int64_t t = threadIdx.x; t < N; t += blockDim.x) {
    const int ix = 1 + (int)(t % nx), iy = 1 + (int)(t / nx);
    const double v = (double)a[(int64_t)iy * R.g.nxg + ix];
    loc += v * v;
  }
  loc = grid::block_sum(loc, sh);
  if (threadIdx.x == 0) R.out[4 + blockIdx.y] = loc * R.anorml1;
}

// rho and J back to zero (pic/fields.f90:353-365)
__global__ void k_ens_zero(const __grid_constant__ EnsGrid32 e) {
  const int r = find_run(e.wblk0, e.nruns, blockIdx.x);
  const EnsRunDev &R = e.run[r];
  const int64_t k = (int64_t)(blockIdx.x - e.wblk0[r]) * blockDim.x + threadIdx.x;
  if (k < R.g.w) R.fld[(EM2G_RHO + blockIdx.y) * R.g.w + k] = 0.0f;
}

}  // namespace

int ens_cg_setup(em2g_ens *e) {
  int per_sm = 0;
  EM2G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_cg, 256, 0));
  if (per_sm < 1) return fail(EM2G_ERR_CUDA, "ensemble cg kernel cannot be resident");
  const int nr = (int)e->runs.size();
  const int total = per_sm * e->num_sms;
  if (total < nr) return fail(EM2G_ERR_RANGE, "more runs than co-resident CG blocks");
  double sum = 0.0;
  for (const EnsRun &R : e->runs) sum += (double)R.g.nx * R.g.ny;
  // blocks in proportion to the run's cells, at least one, at most one per
  // 256 cells; then trim the largest shares until the sum fits
  std::vector<int> b(nr);
  int used = 0;
  for (int r = 0; r < nr; ++r) {
    const double cells = (double)e->runs[r].g.nx * e->runs[r].g.ny;
    const int most = (int)std::max(1.0, std::ceil(cells / 256.0));
    b[r] = std::min(most, std::max(1, (int)(total * cells / sum)));
    used += b[r];
  }
  while (used > total) {
    int k = (int)(std::max_element(b.begin(), b.end()) - b.begin());
    --b[k];
    --used;
  }
  int b0 = 0;
  for (int r = 0; r < nr; ++r) {
    e->runs[r].cg_block0 = b0;
    e->runs[r].cg_blocks = b[r];
    b0 += b[r];
  }
  e->cg_blocks = b0;
  EM2G_CUDA(cudaMalloc(&e->cg_partial, sizeof(double) * 2 * b0));
  EM2G_CUDA(cudaMalloc(&e->cg_bar, sizeof(unsigned) * 2 * nr));
  EM2G_CUDA(cudaMalloc(&e->cg_status, sizeof(int) * 2 * nr));
  EM2G_CUDA(cudaMemset(e->cg_bar, 0, sizeof(unsigned) * 2 * nr));
  EM2G_CUDA(cudaMemset(e->cg_status, 0, sizeof(int) * 2 * nr));
  return EM2G_OK;
}

int ens_tick(em2g_ens *e) {
  k_ens_tick<<<1, 1, 0, e->stream>>>(e->d_it);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int ens_prescale(em2g_ens *e) {
  auto t = make_grid_table(e);
  const int nr = t->nruns;
  k_ens_prescale<<<dim3(t->wblk0[nr], max_nsp(e)), 256, 0, e->stream>>>(*t);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int ens_fields(em2g_ens *e) {
  auto t = make_grid_table(e);
  const int nr = t->nruns;
  const dim3 blk(TX, TY);
  const unsigned ns = (unsigned)t->sten0[nr];
  cudaStream_t st = e->stream;
  k_ens_fold_x<<<dim3(t->foldx0[nr], 7), 128, 0, st>>>(*t);
  k_ens_fold_y<<<dim3(t->foldy0[nr], 7), 128, 0, st>>>(*t);
  if (e->any_smooth_current) {  // optional current filter (no em2 counterpart)
    k_ens_sten<OP_SMOOTH_B><<<dim3(ns, 3), blk, 0, st>>>(*t, SET_J);
    k_ens_sten<OP_SMOOTH_C><<<dim3(ns, 3), blk, 0, st>>>(*t, SET_J);
  }
  k_ens_sten<OP_BHALF><<<ns, blk, 0, st>>>(*t, 0);
  k_ens_sten<OP_EFULL><<<ns, blk, 0, st>>>(*t, 0);
  k_ens_sten<OP_BHALF><<<ns, blk, 0, st>>>(*t, 0);
  k_ens_sten<OP_SMOOTH_B><<<ns, blk, 0, st>>>(*t, SET_RHO);
  k_ens_sten<OP_SMOOTH_C><<<ns, blk, 0, st>>>(*t, SET_RHO);
  k_ens_sten<OP_SMOOTH_B><<<dim3(ns, 6), blk, 0, st>>>(*t, SET_EB);
  k_ens_sten<OP_SMOOTH_C><<<dim3(ns, 6), blk, 0, st>>>(*t, SET_EB);
  k_ens_sten<OP_RHS><<<ns, blk, 0, st>>>(*t, 0);
  EM2G_CUDA(cudaGetLastError());
  // every run's CG (pic/fields.f90:508-651) in one cooperative launch
  std::unique_ptr<EnsCg32> cg(new EnsCg32());
  cg->nruns = nr;
  for (int r = 0; r < nr; ++r) {
    const EnsRun &R = e->runs[r];
    const int64_t N = (int64_t)R.g.nx * R.g.ny;
    grid::CgArgs<float> &a = cg->a[r];
    a.nx = R.g.nx;
    a.ny = R.g.ny;
    a.u = e->cgv + R.cg_off;
    a.r = a.u + N;
    a.p = a.u + 2 * N;
    a.ap = a.u + 3 * N;
    a.partial = e->cg_partial + 2 * R.cg_block0;
    a.bar = e->cg_bar + 2 * r;
    a.status = e->cg_status + 2 * r;
    a.res = e->dev_out + (int64_t)r * kEnsOut + 10;
    a.maxits = R.P.cg_maxits;
    a.eps = R.P.cg_eps;
    cg->blk0[r] = R.cg_block0;
  }
  cg->blk0[nr] = e->cg_blocks;
  EM2G_CUDA(cudaMemsetAsync(e->cg_bar, 0, sizeof(unsigned) * 2 * nr, st));
  void *args[] = {cg.get()};
  EM2G_CUDA(cudaLaunchCooperativeKernel((const void *)k_ens_cg, dim3(e->cg_blocks), dim3(256),
                                        args, 0, st));
  k_ens_sten<OP_CORRECT><<<ns, blk, 0, st>>>(*t, 0);
  k_ens_energy<<<dim3(nr, 6), 256, 0, st>>>(*t);
  k_ens_zero<<<dim3(t->wblk0[nr], 7), 256, 0, st>>>(*t);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int ens_fields_kernels(const em2g_ens *e) { return e->any_smooth_current ? 16 : 14; }

}  // namespace em2g

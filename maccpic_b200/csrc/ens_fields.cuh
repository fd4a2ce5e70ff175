// ens_fields.cuh -- the per-run tables of an ensemble's field stages
// (fields_ens.cu) and of its fused step (ens_step.cu): every run's grid,
// arrays and constants, the block ranges that number each stage's blocks
// run after run, and the CG's per-run block ranges.
#pragma once
#include <algorithm>
#include <memory>

#include "ens_internal.cuh"
#include "grid_kernels.cuh"

namespace em2g {
namespace {

using grid::G;
using grid::TX;
using grid::TY;

struct EnsRunDev {
  G g;
  float *fld, *tmp, *cgu, *sc;
  float ctx, cty, ctxh, ctyh, tem, dx, dy;
  float ae[EM2G_MAX_SPECIES], tx[EM2G_MAX_SPECIES], ty[EM2G_MAX_SPECIES];
  int nsp, isav, smooth_current, tiles_x;
  double anorml1;
  double *out;
};

struct EnsGrid32 {
  int nruns;
  const int *it;
  int sten0[kEnsMaxRuns + 1];   // TX x TY tiles over (nx+1) x (ny+1)
  int foldx0[kEnsMaxRuns + 1];  // blocks of 128 rows (0..ny+2)
  int foldy0[kEnsMaxRuns + 1];  // blocks of 128 columns (0..nx+2)
  int wblk0[kEnsMaxRuns + 1];   // blocks of 256 elements of one array
  EnsRunDev run[kEnsMaxRuns];
};

struct EnsCg32 {
  int nruns;
  int blk0[kEnsMaxRuns + 1];
  grid::CgArgs<float> a[kEnsMaxRuns];
};

// the last r with t0[r] <= b
__device__ __forceinline__ int find_run(const int *t0, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t0[mid] <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

enum { OP_BHALF, OP_EFULL, OP_SMOOTH_B, OP_SMOOTH_C, OP_RHS, OP_CORRECT };
// arrays a smooth2 stage filters (blockIdx.y indexes the set)
enum { SET_RHO, SET_J, SET_EB };

__device__ __forceinline__ bool smooth_target(const EnsGrid32 &e, const EnsRunDev &R, int set,
                                              int y, int *arr) {
  if (set == SET_RHO) {
    *arr = EM2G_RHO;
    return y == 0;
  }
  if (set == SET_J) {  // the ensemble deposits the whole current into jm
    *arr = y == 0 ? EM2G_JXM : (y == 1 ? EM2G_JYM : EM2G_JZM);
    return y < 3 && R.smooth_current;
  }
  *arr = EM2G_EX + y;  // SET_EB: every isav steps (pic/fields.f90:252-260)
  return y < 6 && (*e.it % R.isav) == 0;
}

std::unique_ptr<EnsGrid32> make_grid_table(em2g_ens *e) {
  std::unique_ptr<EnsGrid32> t(new EnsGrid32());
  const int nr = (int)e->runs.size();
  t->nruns = nr;
  t->it = e->d_it;
  int s0 = 0, fx = 0, fy = 0, wb = 0;
  for (int r = 0; r < nr; ++r) {
    const EnsRun &R = e->runs[r];
    EnsRunDev &D = t->run[r];
    D.g = G{R.g.nx, R.g.ny, R.g.nxg, R.g.w};
    D.fld = e->fld + R.fld_off;
    D.tmp = e->tmp + R.tmp_off;
    D.cgu = e->cgv + R.cg_off;
    D.sc = e->scaled + R.sc_off;
    const double ctx = R.P.dt * R.P.c / R.P.dx, cty = R.P.dt * R.P.c / R.P.dy;
    D.ctx = (float)ctx;
    D.cty = (float)cty;
    D.ctxh = (float)(ctx * 0.5);
    D.ctyh = (float)(cty * 0.5);
    D.tem = (float)(0.5 * R.P.dt);
    D.dx = (float)R.P.dx;
    D.dy = (float)R.P.dy;
    for (int s = 0; s < EM2G_MAX_SPECIES; ++s) {
      D.ae[s] = s < R.P.nsp ? (float)(0.5 * R.P.qm[s] * R.P.dt / R.P.c) : 0.0f;
      D.tx[s] = (float)R.P.tx[s];
      D.ty[s] = (float)R.P.ty[s];
    }
    D.nsp = R.P.nsp;
    D.isav = R.P.isav;
    D.smooth_current = R.P.smooth_current;
    D.tiles_x = (R.g.nx + 1 + TX - 1) / TX;
    const double alx = R.P.dx * R.g.nx, aly = R.P.dy * R.g.ny;
    const double q = R.P.qme / R.P.wpe / R.P.c;
    D.anorml1 = 0.5 * R.P.dx * R.P.dy * (q * q / (alx * aly));  // pic/global.f90:26-27
    D.out = e->dev_out + (int64_t)r * kEnsOut;
    t->sten0[r] = s0;
    t->foldx0[r] = fx;
    t->foldy0[r] = fy;
    t->wblk0[r] = wb;
    s0 += D.tiles_x * ((R.g.ny + 1 + TY - 1) / TY);
    fx += (R.g.ny + 3 + 127) / 128;
    fy += (R.g.nx + 3 + 127) / 128;
    wb += (int)((R.g.w + 255) / 256);
  }
  t->sten0[nr] = s0;
  t->foldx0[nr] = fx;
  t->foldy0[nr] = fy;
  t->wblk0[nr] = wb;
  return t;
}

int max_nsp(const em2g_ens *e) {
  int m = 1;
  for (const EnsRun &R : e->runs) m = std::max(m, R.P.nsp);
  return m;
}

}  // namespace
}  // namespace em2g

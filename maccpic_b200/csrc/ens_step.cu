// ens_step.cu -- one ensemble step in one persistent, cooperative launch.
//
// The same step as the stage-by-stage launches of push_fast_f32.cu and
// fields_ens.cu -- prescale; for a regrouping step the scan of all pairs'
// cell counts; the persistent push of every pair; the kinetic energies;
// em2's fields for every run (pic/fields.f90:2-366): fold, the optional
// current filter, Yee B/2 - E - B/2, smooth2 of rho and, every isav steps,
// of E and B, the Poisson right-hand side, the CG, the correction, the
// energies, rho and J back to zero -- here as phases of one kernel whose
// blocks stay resident and meet at a grid barrier between phases.  Each
// barrier's wait is bounded: a block that gives up records a timeout in the
// step's status word and every block leaves at its next barrier; the host
// reads the status after the step (EM2G_ERR_TIMEOUT).
//
// Phases read data that other blocks wrote in earlier phases of the same
// launch, so those reads go through L2 (ld.global.cg): a line an SM cached
// in L1 earlier in the launch may since have been rewritten by another SM.
// The stencils are grid_kernels.cuh's own, with its L2 load policy; the
// push is push_f32_body.cuh's, reading
// only data written by earlier launches or, for the (E, B) pairs, written in
// the first phase before any read of them.  The block shape is the push
// variant's (TCX*G threads); a 32x8 stencil tile takes 256/(TCX*G) passes.
#include "ens_fields.cuh"
#include "push_f32_body.cuh"

namespace em2g {
namespace {

template <typename T>
__device__ __forceinline__ T ld(const T *p) {
  return __ldcg(p);
}

// exclusive scan of all pairs' cell counts (regrouping steps), in chunks
constexpr int kScanChunk = 4096;

struct EnsScanArgs {
  const int32_t *in;  // counts of the current positions, all pairs
  int32_t *out;       // offsets of the next grouping (n + 1 values)
  int64_t n;
  int32_t *sums;      // one per chunk
  int nchunks;
};

// The step's tables besides the push's, which travel as a kernel parameter
// (the constant bank, as for the stage-by-stage push: the segment loop
// reads a pair's arguments without loads that stores could invalidate).
struct EnsStepTab {
  EnsAke ake;
  int npairs;
  EnsGrid32 grid;
  EnsCg32 cg;
  EnsScanArgs scan;
  int32_t *cnt_next;  // counts of the new positions, zeroed first
  int32_t *cursor;    // back-fill cursors of a regrouping push, zeroed first
  int64_t ncell;
  int nsp_max;
  int any_smooth_current;
  unsigned *bar;      // the step's grid barrier: arrival count, generation
  int *status;        // 1 when a barrier wait gave up
  unsigned long long *marks;  // the global timer at the start and after each barrier
};

constexpr int kMaxMarks = 32;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- the per-cell stages: grid_kernels.cuh's, reading through L2 ---------

__device__ __forceinline__ void f_fold_x(const G &g, float *fld, int iy, int k) {
  grid::fold_x_at<float, grid::LdL2>(g, fld, iy, k);
}
__device__ __forceinline__ void f_fold_y(const G &g, float *fld, int ix, int k) {
  grid::fold_y_at<float, grid::LdL2>(g, fld, ix, k);
}
__device__ __forceinline__ void f_b_half(const G &g, float *fld, float ctxh, float ctyh, int ix,
                                         int iy) {
  grid::b_half_cell<float, grid::LdL2>(g, fld, ctxh, ctyh, ix, iy);
}
__device__ __forceinline__ void f_e_full(const G &g, float *fld, float ctx, float cty, float tem,
                                         int ix, int iy) {
  grid::e_full_cell<float, grid::LdL2>(g, fld, ctx, cty, tem, ix, iy);
}
__device__ __forceinline__ void f_smooth_b(const G &g, const float *s, float *d, int ix, int iy) {
  grid::smooth_binomial_cell<float, grid::LdL2>(g, s, d, ix, iy);
}
__device__ __forceinline__ void f_smooth_c(const G &g, const float *d, float *s, int ix, int iy) {
  grid::smooth_compensate_cell<float, grid::LdL2>(g, d, s, ix, iy);
}
__device__ __forceinline__ void f_rhs(const G &g, const float *fld, float dx, float dy, float *r,
                                      float *p, int ix, int iy) {
  grid::poisson_rhs_cell<float, grid::LdL2>(g, fld, dx, dy, r, p, ix, iy);
}
__device__ __forceinline__ void f_correct(const G &g, float *fld, const float *u, float dx,
                                          float dy, int ix, int iy) {
  grid::poisson_correct_cell<float, grid::LdL2>(g, fld, u, dx, dy, ix, iy);
}

// one stencil stage over every run: 32x8 tiles numbered run after run
// (grid.sten0), each covered by this block in 256 / blockDim.x passes
template <typename F>
__device__ __forceinline__ void for_tiles(const EnsGrid32 &e, F f) {
  const int nt = e.sten0[e.nruns];
  const int passes = (TX * TY) / (int)blockDim.x;
  for (int vb = blockIdx.x; vb < nt; vb += gridDim.x) {
    const int r = find_run(e.sten0, e.nruns, vb);
    const EnsRunDev &R = e.run[r];
    const int lb = vb - e.sten0[r];
    const int tby = lb / R.tiles_x, tbx = lb - tby * R.tiles_x;
    for (int q = 0; q < passes; ++q) {
      const int t = threadIdx.x + q * blockDim.x;
      f(R, 1 + tbx * TX + (t % TX), 1 + tby * TY + (t / TX));
    }
  }
}

template <int TCX, int G, int NC, int MINB, bool INPLACE>
__global__ void __launch_bounds__(TCX * G, MINB)
    k_ens_step(const __grid_constant__ EnsPush32 e, const EnsStepTab *tp) {
  __shared__ float4 win[3][WY][NC * TCX + 5];
  __shared__ WarpScratch ws[TCX * G / 32];
  __shared__ int s_tile;
  __shared__ double sh[33];
  const EnsStepTab &t = *tp;
  const EnsGrid32 &eg = t.grid;
  // Nothing computed here stays live across the push phase, whose register
  // budget is the push's own: the run count, the global thread index and
  // stride are re-read or recomputed from the builtins where used.
#define nr (eg.nruns)
#define gtid ((int64_t)blockIdx.x * blockDim.x + threadIdx.x)
#define gstride ((int64_t)gridDim.x * blockDim.x)
  // block 0's thread 0 notes the time at the start and after each barrier
  // (mark k after the k-th barrier): the phases' durations, for the design
  // notes (em2g_ens_get_phase_ns)
  if (gtid == 0) {
    for (int k = 1; k < kMaxMarks; ++k) t.marks[k] = 0;  // a step in place skips two
    t.marks[0] = global_ns();
  }
#define EM2G_SYNC_ALL(k)                                                \
  do {                                                                  \
    if (!grid::grid_barrier(t.bar, gridDim.x, t.status)) return;        \
    if (gtid == 0) t.marks[k] = global_ns();                            \
  } while (0)

  // ---- (E, B) pairs of every species, counters to zero, the first pass
  // of a regrouping step's scan
  {
    const int nwb = eg.wblk0[nr];
    for (int vb = blockIdx.x; vb < nwb * t.nsp_max; vb += gridDim.x) {
      const int s = vb / nwb, b = vb - s * nwb;
      const int r = find_run(eg.wblk0, nr, b);
      const EnsRunDev &R = eg.run[r];
      if (s >= R.nsp) continue;
      const int64_t w = R.g.w;
      const float *f = R.fld;
      float2 *o = reinterpret_cast<float2 *>(R.sc + (int64_t)s * 6 * w);
      const float ae = R.ae[s];
      const int64_t k0 = (int64_t)(b - eg.wblk0[r]) * 256;
      for (int64_t k = k0 + threadIdx.x; k < w && k < k0 + 256; k += blockDim.x) {
        o[k] = make_float2(ae * f[EM2G_EX * w + k], ae * f[EM2G_BX * w + k] + R.tx[s]);
        o[w + k] = make_float2(ae * f[EM2G_EZ * w + k], ae * f[EM2G_BZ * w + k]);
        o[2 * w + k] = make_float2(ae * f[EM2G_EY * w + k], ae * f[EM2G_BY * w + k] + R.ty[s]);
      }
    }
    for (int64_t k = gtid; k < t.ncell; k += gstride) {
      t.cnt_next[k] = 0;
      if (!INPLACE) t.cursor[k] = 0;
    }
    if (gtid == 0) *e.counter = 0;
    for (int r = (int)gtid; r < nr; r += (int)gstride) t.cg.a[r].bar[0] = 0u;
    if (!INPLACE) {
      // each chunk's exclusive scan, its total aside
      const EnsScanArgs &sc = t.scan;
      int32_t *wt = reinterpret_cast<int32_t *>(sh);  // warp totals, then the block's
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      for (int c = blockIdx.x; c < sc.nchunks; c += gridDim.x) {
        const int64_t lo = (int64_t)c * kScanChunk, hi = min(lo + kScanChunk, sc.n);
        int32_t carry = 0;
        for (int64_t base = lo; base < hi; base += blockDim.x) {
          const int64_t i = base + threadIdx.x;
          const int32_t v = i < hi ? sc.in[i] : 0;
          int32_t incl = v;
          for (int o = 1; o < 32; o <<= 1) {
            const int32_t u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
          }
          if (lane == 31) wt[wid] = incl;
          __syncthreads();
          if (threadIdx.x == 0) {
            int32_t run = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
              const int32_t x = wt[k];
              wt[k] = run;
              run += x;
            }
            wt[32] = run;
          }
          __syncthreads();
          if (i < hi) sc.out[i] = carry + wt[wid] + incl - v;
          carry += wt[32];
          __syncthreads();
        }
        if (threadIdx.x == 0) sc.sums[c] = carry;
      }
    }
  }
  EM2G_SYNC_ALL(1);
  if (!INPLACE) {
    // the chunk totals scanned by block 0, then added to every chunk
    const EnsScanArgs &sc = t.scan;
    if (blockIdx.x == 0) {
      int32_t *wt = reinterpret_cast<int32_t *>(sh);
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      int32_t carry = 0;
      for (int base = 0; base < sc.nchunks; base += blockDim.x) {
        const int c = base + threadIdx.x;
        const int32_t v = c < sc.nchunks ? ld(sc.sums + c) : 0;
        int32_t incl = v;
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t u = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += u;
        }
        if (lane == 31) wt[wid] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
          int32_t run = 0;
          for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            const int32_t x = wt[k];
            wt[k] = run;
            run += x;
          }
          wt[32] = run;
        }
        __syncthreads();
        if (c < sc.nchunks) sc.sums[c] = carry + wt[wid] + incl - v;
        carry += wt[32];
        __syncthreads();
      }
      if (threadIdx.x == 0) sc.out[sc.n] = carry;
    }
    EM2G_SYNC_ALL(2);
    for (int c = blockIdx.x; c < sc.nchunks; c += gridDim.x) {
      const int32_t add = ld(sc.sums + c);
      const int64_t lo = (int64_t)c * kScanChunk, hi = min(lo + kScanChunk, sc.n);
      for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) sc.out[i] = ld(sc.out + i) + add;
    }
    EM2G_SYNC_ALL(3);
  }

  // ---- the push of every pair, row segments claimed from a counter
  {
    for (;;) {
      if (threadIdx.x == 0) s_tile = atomicAdd(e.counter, 1);
      __syncthreads();  // also: every thread is done with the last segment
      const int tl = s_tile;
      if (tl >= e.ntiles) break;
      int lo = 0, hi = e.npairs - 1;  // last pair p with tile0[p] <= tl
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (e.tile0[mid] <= tl) lo = mid; else hi = mid - 1;
      }
      const int lt = tl - e.tile0[lo];
      const int segs = e.segs[lo];
      const int row = lt / segs;
      push_segment<TCX, G, NC, INPLACE>(e.pair[lo], (lt - row * segs) * (NC * TCX), row, lt,
                                        win, ws);
    }
  }
  EM2G_SYNC_ALL(4);

  // ---- kinetic energies, the step counter, the fold in x, then in y
  {
    const EnsAke &a = t.ake;
    for (int p = blockIdx.x; p < t.npairs; p += gridDim.x) {
      double v = 0.0;
      for (int i = threadIdx.x; i < a.count[p]; i += blockDim.x) v += ld(a.partial[p] + i);
      v = grid::block_sum(v, sh);
      if (threadIdx.x == 0) *a.out[p] = v * a.scale[p];
    }
    if (gtid == 0) atomicAdd(const_cast<int *>(eg.it), 1);
    const int64_t nfx = (int64_t)eg.foldx0[nr] * 128;
    for (int64_t v = gtid; v < nfx * 7; v += gstride) {
      const int k = (int)(v / nfx), rem = (int)(v - k * nfx), b = rem / 128;
      const int r = find_run(eg.foldx0, nr, b);
      f_fold_x(eg.run[r].g, eg.run[r].fld, (b - eg.foldx0[r]) * 128 + (rem % 128), k);
    }
  }
  EM2G_SYNC_ALL(5);
  {
    const int64_t nfy = (int64_t)eg.foldy0[nr] * 128;
    for (int64_t v = gtid; v < nfy * 7; v += gstride) {
      const int k = (int)(v / nfy), rem = (int)(v - k * nfy), b = rem / 128;
      const int r = find_run(eg.foldy0, nr, b);
      f_fold_y(eg.run[r].g, eg.run[r].fld, (b - eg.foldy0[r]) * 128 + (rem % 128), k);
    }
  }
  EM2G_SYNC_ALL(6);
  const int it = ld(eg.it);
  // ---- the optional current filter after the fold (no em2 counterpart)
  if (t.any_smooth_current) {
    for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
      if (!R.smooth_current) return;
      for (int y = 0; y < 3; ++y) {
        const int arr = y == 0 ? EM2G_JXM : (y == 1 ? EM2G_JYM : EM2G_JZM);
        f_smooth_b(R.g, R.fld + arr * R.g.w, R.tmp + y * R.g.w, ix, iy);
      }
    });
    EM2G_SYNC_ALL(7);
    for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
      if (!R.smooth_current) return;
      for (int y = 0; y < 3; ++y) {
        const int arr = y == 0 ? EM2G_JXM : (y == 1 ? EM2G_JYM : EM2G_JZM);
        f_smooth_c(R.g, R.tmp + y * R.g.w, R.fld + arr * R.g.w, ix, iy);
      }
    });
    EM2G_SYNC_ALL(8);
  }
  // ---- Yee: B/2, E, B/2 (pic/fields.f90:184-247)
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    f_b_half(R.g, R.fld, R.ctxh, R.ctyh, ix, iy);
  });
  EM2G_SYNC_ALL(9);
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    f_e_full(R.g, R.fld, R.ctx, R.cty, R.tem, ix, iy);
  });
  EM2G_SYNC_ALL(10);
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    f_b_half(R.g, R.fld, R.ctxh, R.ctyh, ix, iy);
  });
  EM2G_SYNC_ALL(11);
  // ---- smooth2 of rho every step, of E and B every isav steps
  // (pic/fields.f90:252-260)
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    f_smooth_b(R.g, R.fld + EM2G_RHO * R.g.w, R.tmp, ix, iy);
  });
  EM2G_SYNC_ALL(12);
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    f_smooth_c(R.g, R.tmp, R.fld + EM2G_RHO * R.g.w, ix, iy);
  });
  EM2G_SYNC_ALL(13);
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    if (it % R.isav != 0) return;
    for (int y = 0; y < 6; ++y)
      f_smooth_b(R.g, R.fld + (EM2G_EX + y) * R.g.w, R.tmp + y * R.g.w, ix, iy);
  });
  EM2G_SYNC_ALL(14);
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    if (it % R.isav != 0) return;
    for (int y = 0; y < 6; ++y)
      f_smooth_c(R.g, R.tmp + y * R.g.w, R.fld + (EM2G_EX + y) * R.g.w, ix, iy);
  });
  EM2G_SYNC_ALL(15);
  // ---- Poisson: right-hand side, every run's CG on its own blocks, the
  // correction (pic/fields.f90:370-651)
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    const int64_t N = (int64_t)R.g.nx * R.g.ny;
    f_rhs(R.g, R.fld, R.dx, R.dy, R.cgu + N, R.cgu + 2 * N, ix, iy);
  });
  EM2G_SYNC_ALL(16);
  if ((int)blockIdx.x < t.cg.blk0[nr]) {
    const int r = find_run(t.cg.blk0, nr, blockIdx.x);
    grid::cg_body(t.cg.a[r], (int)blockIdx.x - t.cg.blk0[r],
                  (unsigned)(t.cg.blk0[r + 1] - t.cg.blk0[r]), sh);
  }
  EM2G_SYNC_ALL(17);
  for_tiles(eg, [&](const EnsRunDev &R, int ix, int iy) {
    f_correct(R.g, R.fld, R.cgu, R.dx, R.dy, ix, iy);
  });
  EM2G_SYNC_ALL(18);
  // ---- energies on isav steps (pic/fields.f90:267-347, whole grid), rho
  // and J back to zero (pic/fields.f90:353-365)
  for (int vb = blockIdx.x; vb < nr * 6; vb += gridDim.x) {
    const int r = vb / 6, comp = vb - r * 6;
    const EnsRunDev &R = eg.run[r];
    if (it % R.isav != 0) continue;
    const float *a = R.fld + comp * R.g.w;
    const int nx = R.g.nx;
    const int64_t N = (int64_t)nx * R.g.ny;
    double loc = 0.0;
    for (int64_t q = threadIdx.x; q < N; q += blockDim.x) {
      const int ix = 1 + (int)(q % nx), iy = 1 + (int)(q / nx);
      const double v = (double)ld(a + (int64_t)iy * R.g.nxg + ix);
      loc += v * v;
    }
    loc = grid::block_sum(loc, sh);
    if (threadIdx.x == 0) R.out[4 + comp] = loc * R.anorml1;
  }
  {
    const int64_t nw = (int64_t)eg.wblk0[nr] * 256;
    for (int64_t v = gtid; v < nw * 7; v += gstride) {
      const int k = (int)(v / nw), rem = (int)(v - k * nw), b = rem / 256;
      const int r = find_run(eg.wblk0, nr, b);
      const EnsRunDev &R = eg.run[r];
      const int64_t q = (int64_t)(b - eg.wblk0[r]) * 256 + (rem % 256);
      if (q < R.g.w) R.fld[(EM2G_RHO + k) * R.g.w + q] = 0.0f;
    }
  }
#undef EM2G_SYNC_ALL
#undef nr
#undef gtid
#undef gstride
}

struct FusedVariant {
  void (*regroup)(const EnsPush32, const EnsStepTab *);
  void (*inplace)(const EnsPush32, const EnsStepTab *);
  int threads, cells;
};
#define EM2G_FUSED(T, GG, N, M) \
  {k_ens_step<T, GG, N, M, false>, k_ens_step<T, GG, N, M, true>, T * GG, T * N},
const FusedVariant kFused[] = {EM2G_F32_VARIANTS(EM2G_FUSED)};
#undef EM2G_FUSED

const FusedVariant &fused_variant(const em2g_ens *e) {
  const int n = (int)(sizeof(kFused) / sizeof(kFused[0]));
  return kFused[e->variant >= 0 && e->variant < n ? e->variant : 0];
}

// blocks of the cooperative launch: as many as fit on every SM at once
int fused_blocks(const em2g_ens *e, int *blocks) {
  const FusedVariant &F = fused_variant(e);
  int a = 0, b = 0;
  EM2G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, F.regroup, F.threads, 0));
  EM2G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, F.inplace, F.threads, 0));
  const int per_sm = std::min(a, b);
  if (per_sm < 1) return fail(EM2G_ERR_CUDA, "the fused ensemble step cannot be resident");
  *blocks = per_sm * e->num_sms;
  return EM2G_OK;
}

}  // namespace

// Device tables, barrier and scratch of the fused step, allocated on first
// use: one table per kind of step (in place or regrouping x buffer parity x
// count parity), the CG's partial sums for every block of the launch, the
// scan's chunk totals.
static int fused_alloc(em2g_ens *e) {
  if (e->fused_tab) return EM2G_OK;
  e->fused_push = ::operator new(sizeof(EnsPush32) * 8);
  EM2G_CUDA(cudaMalloc(&e->fused_tab, sizeof(EnsStepTab) * 8));
  EM2G_CUDA(cudaMalloc((void **)&e->step_sync, sizeof(unsigned) * 4));
  EM2G_CUDA(cudaMemset(e->step_sync, 0, sizeof(unsigned) * 4));
  const int64_t max_blocks = 64 * (int64_t)e->num_sms;  // 2048 threads per SM, 32 per block
  EM2G_CUDA(cudaMalloc((void **)&e->fused_partial, sizeof(double) * 2 * max_blocks));
  const int64_t nchunks = (e->ncell + kScanChunk - 1) / kScanChunk;
  EM2G_CUDA(cudaMalloc((void **)&e->fused_sums, sizeof(int32_t) * (nchunks + 1)));
  EM2G_CUDA(cudaMalloc((void **)&e->fused_marks, sizeof(unsigned long long) * kMaxMarks));
  EM2G_CUDA(cudaMemset(e->fused_marks, 0, sizeof(unsigned long long) * kMaxMarks));
  return EM2G_OK;
}

// The table of step kind `key` (in place, parity, cparity as graph keys
// number them), written to the device before the step is launched or
// captured: the push's and the kinetic energies' tables, the field stages',
// every run's CG on its share of the launch's blocks, the scan.
int ens_fused_prepare(em2g_ens *e, int key, bool inplace) {
  if (e->fused_ready[key]) return EM2G_OK;  // written for this variant already
  int rc = fused_alloc(e);
  if (rc) return rc;
  const FusedVariant &F = fused_variant(e);
  int blocks = 0;
  if ((rc = fused_blocks(e, &blocks))) return rc;
  const int nr = (int)e->runs.size();
  if (blocks < nr) return fail(EM2G_ERR_RANGE, "more runs than blocks of the fused step");
  std::unique_ptr<EnsStepTab> T(new EnsStepTab());
  const int bp = e->parity, cp = e->cparity;
  EnsPush32 *P = static_cast<EnsPush32 *>(e->fused_push) + key;
  ens_push_tables(e, bp, cp, inplace, F.cells, F.threads, P, &T->ake);
  P->counter = e->counter;
  T->npairs = P->npairs;
  T->grid = *make_grid_table(e);
  // every run's CG: blocks in proportion to its cells (at least one, at
  // most one per blockDim cells), summing to at most the launch's blocks
  {
    double sum = 0.0;
    for (const EnsRun &R : e->runs) sum += (double)R.g.nx * R.g.ny;
    std::vector<int> b(nr);
    int used = 0;
    for (int r = 0; r < nr; ++r) {
      const double cells = (double)e->runs[r].g.nx * e->runs[r].g.ny;
      const int most = (int)std::max(1.0, std::ceil(cells / F.threads));
      b[r] = std::min(most, std::max(1, (int)(blocks * cells / sum)));
      used += b[r];
    }
    while (used > blocks) {
      const int k = (int)(std::max_element(b.begin(), b.end()) - b.begin());
      --b[k];
      --used;
    }
    EnsCg32 &cg = T->cg;
    cg.nruns = nr;
    int b0 = 0;
    for (int r = 0; r < nr; ++r) {
      const EnsRun &R = e->runs[r];
      const int64_t N = (int64_t)R.g.nx * R.g.ny;
      grid::CgArgs<float> &a = cg.a[r];
      a.nx = R.g.nx;
      a.ny = R.g.ny;
      a.u = e->cgv + R.cg_off;
      a.r = a.u + N;
      a.p = a.u + 2 * N;
      a.ap = a.u + 3 * N;
      a.partial = e->fused_partial + 2 * b0;
      a.bar = e->cg_bar + 2 * r;
      a.status = e->cg_status + 2 * r;
      a.res = e->dev_out + (int64_t)r * kEnsOut + 10;
      a.maxits = R.P.cg_maxits;
      a.eps = R.P.cg_eps;
      cg.blk0[r] = b0;
      b0 += b[r];
    }
    cg.blk0[nr] = b0;
  }
  int32_t *offB = bp ? e->off : e->off_alt;
  int32_t *cntA = cp ? e->cnt_alt : e->cnt, *cntB = cp ? e->cnt : e->cnt_alt;
  T->scan.in = cntA;
  T->scan.out = offB;
  T->scan.n = e->ncell;
  T->scan.sums = e->fused_sums;
  T->scan.nchunks = (int)((e->ncell + kScanChunk - 1) / kScanChunk);
  T->cnt_next = cntB;
  T->cursor = e->cursor;
  T->ncell = e->ncell;
  int nsp = 1;
  for (const EnsRun &R : e->runs) nsp = std::max(nsp, R.P.nsp);
  T->nsp_max = nsp;
  T->any_smooth_current = e->any_smooth_current ? 1 : 0;
  T->bar = e->step_sync;
  T->status = reinterpret_cast<int *>(e->step_sync + 2);
  T->marks = e->fused_marks;
  EM2G_CUDA(cudaMemcpyAsync(static_cast<EnsStepTab *>(e->fused_tab) + key, T.get(),
                            sizeof(EnsStepTab), cudaMemcpyHostToDevice, e->stream));
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  e->fused_blocks = blocks;
  e->fused_ready[key] = true;
  return EM2G_OK;
}

// the step of kind `key`, whose table ens_fused_prepare wrote, as one
// cooperative launch on the ensemble's stream
int ens_fused_launch(em2g_ens *e, int key, bool inplace) {
  const FusedVariant &F = fused_variant(e);
  const EnsStepTab *tab = static_cast<const EnsStepTab *>(e->fused_tab) + key;
  EnsPush32 *push = static_cast<EnsPush32 *>(e->fused_push) + key;
  void *args[] = {(void *)push, (void *)&tab};
  EM2G_CUDA(cudaLaunchCooperativeKernel(
      inplace ? (const void *)F.inplace : (const void *)F.regroup, dim3(e->fused_blocks),
      dim3(F.threads), args, 0, e->stream));
  return EM2G_OK;
}

// the durations between the marks of the last fused step (ns)
int ens_fused_phase_ns(em2g_ens *e, int64_t *out, int n) {
  if (!e->fused_marks) return fail(EM2G_ERR_INVALID, "no fused step has run");
  unsigned long long h[kMaxMarks];
  EM2G_CUDA(cudaMemcpyAsync(h, e->fused_marks, sizeof(h), cudaMemcpyDeviceToHost, e->stream));
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  // marks left at zero belong to phases the step skipped
  int m = 0;
  unsigned long long last = h[0];
  for (int k = 1; k < kMaxMarks && m < n; ++k) {
    if (h[k] == 0) continue;
    out[m++] = h[k] >= last ? (int64_t)(h[k] - last) : 0;
    last = h[k];
  }
  for (; m < n; ++m) out[m] = 0;
  return EM2G_OK;
}

}  // namespace em2g

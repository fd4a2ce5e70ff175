// grid_kernels.cuh -- the grid kernels of em2's fields / smooth2 / Poisson
// (pic/fields.f90, pic/smooth.f90), templated on the storage type T:
// double for the drop-in FP64 path (fields_f64.cu, compiled with
// -fmad=false so each cell is rounded as em2 rounds it) and float for the
// mixed path (fields_f32.cu).  Dot products and energies always accumulate
// in FP64.
//
// Every stencil sweep of the reference ends with guard copies, columns 0 and
// nx+2 from nx and 2, then rows 0 and ny+2 from ny and 2
// (pic/fields.f90:192-200).  Here the thread that computes a cell also
// stores it into the guard positions that copy it, so no second pass is
// needed and the values are the same.
#pragma once
#include "em2g_internal.cuh"

namespace em2g {
namespace grid {
namespace {

constexpr int TX = 32, TY = 8;

struct G {
  int nx, ny, nxg;
  int64_t w;
};

__device__ __forceinline__ int64_t at(const G &g, int ix, int iy) {
  return (int64_t)iy * g.nxg + ix;
}

// How a stage reads the arrays: plainly in a launch of its own, through L2
// (ld.global.cg) inside a persistent launch whose earlier phases other SMs
// wrote -- an L1 line cached before such a write would be stale.  The
// arithmetic is the same expression for expression either way.
struct LdPlain {
  template <typename T>
  __device__ __forceinline__ static T ld(const T *p) { return *p; }
};
struct LdL2 {
  template <typename T>
  __device__ __forceinline__ static T ld(const T *p) { return __ldcg(p); }
};

// store v at (ix,iy), 1<=ix<=nx+1, 1<=iy<=ny+1, and at its guard copies
template <typename T>
__device__ __forceinline__ void store_with_guards(const G &g, T *a, int ix, int iy, T v) {
  a[at(g, ix, iy)] = v;
  const int mx = (ix == g.nx) ? 0 : ((ix == 2) ? g.nx + 2 : -1);
  const int my = (iy == g.ny) ? 0 : ((iy == 2) ? g.ny + 2 : -1);
  if (mx >= 0) a[at(g, mx, iy)] = v;
  if (my >= 0) a[at(g, ix, my)] = v;
  if (mx >= 0 && my >= 0) a[at(g, mx, my)] = v;
}

// ---- guard fold of rho and the 6 current arrays (pic/fields.f90:44-137)
// x pass: row iy in 0..ny+2 of array k (the six positions are distinct for
// nx >= 3; the library asks nx, ny >= 4)
template <typename T, typename L = LdPlain>
__device__ __forceinline__ void fold_x_at(const G &g, T *fld, int iy, int k) {
  if (iy > g.ny + 2) return;
  T *a = fld + (EM2G_RHO + k) * g.w + (int64_t)iy * g.nxg;
  const int nx = g.nx;
  const T a1 = L::ld(a + 1) + L::ld(a + nx + 1);
  const T a2 = L::ld(a + 2) + L::ld(a + nx + 2);
  const T an = L::ld(a + nx) + L::ld(a);
  a[1] = a1;
  a[2] = a2;
  a[nx] = an;
  a[nx + 1] = a1;
  a[nx + 2] = a2;
  a[0] = an;
}
template <typename T>
__global__ void k_fold_x(G g, T *fld) {
  fold_x_at(g, fld, (int)(blockIdx.x * blockDim.x + threadIdx.x), (int)blockIdx.y);
}
// y pass: column ix in 0..nx+2 of array k
template <typename T, typename L = LdPlain>
__device__ __forceinline__ void fold_y_at(const G &g, T *fld, int ix, int k) {
  if (ix > g.nx + 2) return;
  T *a = fld + (EM2G_RHO + k) * g.w + ix;
  const int64_t s = g.nxg;
  const int ny = g.ny;
  const T a1 = L::ld(a + 1 * s) + L::ld(a + (ny + 1) * s);
  const T a2 = L::ld(a + 2 * s) + L::ld(a + (ny + 2) * s);
  const T an = L::ld(a + ny * s) + L::ld(a);
  a[1 * s] = a1;
  a[2 * s] = a2;
  a[ny * s] = an;
  a[(ny + 1) * s] = a1;
  a[(ny + 2) * s] = a2;
  a[0] = an;
}
template <typename T>
__global__ void k_fold_y(G g, T *fld) {
  fold_y_at(g, fld, (int)(blockIdx.x * blockDim.x + threadIdx.x), (int)blockIdx.y);
}

// The cell stages take the cell (ix, iy); the *_at forms take a 32x8 tile
// (tbx, tby) whose cell is given by the thread index.

// ---- the stencils' arithmetic on loaded values.  Every implementation of
// a stage (direct loads here, the TMA-staged tiles of tma_stencil.cuh, the
// ensemble's kernels) calls these, so each rounds a cell as em2 does, in
// the same order.  Suffixes name neighbours: _w (ix-1), _e (ix+1), _s
// (iy-1), _n (iy+1).
// pic/fields.f90:188-190
template <typename T>
__device__ __forceinline__ void b_half_vals(T bx, T by, T bz, T ezc, T ez_s, T ez_w, T ey_e,
                                            T eyc, T ex_n, T exc, T ctxh, T ctyh, T &vbx,
                                            T &vby, T &vbz) {
  vbx = bx - ctyh * (ezc - ez_s);
  vby = by + ctxh * (ezc - ez_w);
  vbz = bz - ctxh * (ey_e - eyc) + ctyh * (ex_n - exc);
}
// pic/fields.f90:211-215
template <typename T>
__device__ __forceinline__ void e_full_vals(T ex, T ey, T ez, T bzc, T bz_s, T bz_w, T by_e,
                                            T byc, T bx_n, T bxc, T jxm, T jxp, T jym, T jyp,
                                            T jzm, T jzp, T ctx, T cty, T tem, T &vex, T &vey,
                                            T &vez) {
  vex = ex + cty * (bzc - bz_s) - tem * (jxm + jxp);
  vey = ey - ctx * (bzc - bz_w) - tem * (jym + jyp);
  vez = ez + ctx * (by_e - byc) - cty * (bx_n - bxc) - tem * (jzm + jzp);
}
// pic/smooth.f90:145-146 (c: the cell; then w, e, s, n; then sw, nw, se, ne)
template <typename T>
__device__ __forceinline__ T binomial_val(T c, T w, T e, T s, T n, T sw, T nw, T se, T ne) {
  return (4 * c + 2 * (w + e + s + n) + sw + nw + se + ne) / T(16.0);
}
// pic/smooth.f90:163-164 (same order)
template <typename T>
__device__ __forceinline__ T compensate_val(T c, T w, T e, T s, T n, T sw, T nw, T se, T ne) {
  return (20 * c - w - e - s - n - sw - nw - se - ne) / T(12.0);
}

// ---- Yee half step of B (pic/fields.f90:184-200, :231-247)
template <typename T, typename L = LdPlain>
__device__ __forceinline__ void b_half_cell(const G &g, T *fld, T ctxh, T ctyh, int ix, int iy) {
  if (ix > g.nx + 1 || iy > g.ny + 1) return;
  const T *ex = fld + EM2G_EX * g.w, *ey = fld + EM2G_EY * g.w, *ez = fld + EM2G_EZ * g.w;
  T *bx = fld + EM2G_BX * g.w, *by = fld + EM2G_BY * g.w, *bz = fld + EM2G_BZ * g.w;
  const int64_t c = at(g, ix, iy);
  T vbx, vby, vbz;
  b_half_vals(L::ld(bx + c), L::ld(by + c), L::ld(bz + c), L::ld(ez + c), L::ld(ez + c - g.nxg),
              L::ld(ez + c - 1), L::ld(ey + c + 1), L::ld(ey + c), L::ld(ex + c + g.nxg),
              L::ld(ex + c), ctxh, ctyh, vbx, vby, vbz);
  store_with_guards(g, bx, ix, iy, vbx);
  store_with_guards(g, by, ix, iy, vby);
  store_with_guards(g, bz, ix, iy, vbz);
}
template <typename T>
__device__ __forceinline__ void b_half_at(const G &g, T *fld, T ctxh, T ctyh, int tbx, int tby) {
  b_half_cell(g, fld, ctxh, ctyh, 1 + tbx * TX + (int)threadIdx.x, 1 + tby * TY + (int)threadIdx.y);
}
template <typename T>
__global__ void k_b_half(G g, T *fld, T ctxh, T ctyh) {
  b_half_at(g, fld, ctxh, ctyh, (int)blockIdx.x, (int)blockIdx.y);
}

// ---- Yee full step of E (pic/fields.f90:207-224)
template <typename T, typename L = LdPlain>
__device__ __forceinline__ void e_full_cell(const G &g, T *fld, T ctx, T cty, T tem, int ix,
                                            int iy) {
  if (ix > g.nx + 1 || iy > g.ny + 1) return;
  T *ex = fld + EM2G_EX * g.w, *ey = fld + EM2G_EY * g.w, *ez = fld + EM2G_EZ * g.w;
  const T *bx = fld + EM2G_BX * g.w, *by = fld + EM2G_BY * g.w, *bz = fld + EM2G_BZ * g.w;
  const T *jxm = fld + EM2G_JXM * g.w, *jxp = fld + EM2G_JXP * g.w,
          *jym = fld + EM2G_JYM * g.w, *jyp = fld + EM2G_JYP * g.w,
          *jzm = fld + EM2G_JZM * g.w, *jzp = fld + EM2G_JZP * g.w;
  const int64_t c = at(g, ix, iy);
  T vex, vey, vez;
  e_full_vals(L::ld(ex + c), L::ld(ey + c), L::ld(ez + c), L::ld(bz + c), L::ld(bz + c - g.nxg),
              L::ld(bz + c - 1), L::ld(by + c + 1), L::ld(by + c), L::ld(bx + c + g.nxg),
              L::ld(bx + c), L::ld(jxm + c), L::ld(jxp + c), L::ld(jym + c), L::ld(jyp + c),
              L::ld(jzm + c), L::ld(jzp + c), ctx, cty, tem, vex, vey, vez);
  store_with_guards(g, ex, ix, iy, vex);
  store_with_guards(g, ey, ix, iy, vey);
  store_with_guards(g, ez, ix, iy, vez);
}
template <typename T>
__device__ __forceinline__ void e_full_at(const G &g, T *fld, T ctx, T cty, T tem, int tbx,
                                          int tby) {
  e_full_cell(g, fld, ctx, cty, tem, 1 + tbx * TX + (int)threadIdx.x,
              1 + tby * TY + (int)threadIdx.y);
}
template <typename T>
__global__ void k_e_full(G g, T *fld, T ctx, T cty, T tem) {
  e_full_at(g, fld, ctx, cty, tem, (int)blockIdx.x, (int)blockIdx.y);
}

// ---- smooth2 (pic/smooth.f90:143-177): binomial pass into `d`, then the
// compensation pass back into `s`.
template <typename T, typename L = LdPlain>
__device__ __forceinline__ void smooth_binomial_cell(const G &g, const T *__restrict__ s, T *d,
                                                     int ix, int iy) {
  if (ix > g.nx + 1 || iy > g.ny + 1) return;
  const int64_t c = at(g, ix, iy), n = g.nxg;
  const T v = binomial_val(L::ld(s + c), L::ld(s + c - 1), L::ld(s + c + 1), L::ld(s + c - n),
                           L::ld(s + c + n), L::ld(s + c - 1 - n), L::ld(s + c - 1 + n),
                           L::ld(s + c + 1 - n), L::ld(s + c + 1 + n));
  store_with_guards(g, d, ix, iy, v);
}
template <typename T>
__device__ __forceinline__ void smooth_binomial_at(const G &g, const T *__restrict__ s, T *d,
                                                   int tbx, int tby) {
  smooth_binomial_cell(g, s, d, 1 + tbx * TX + (int)threadIdx.x, 1 + tby * TY + (int)threadIdx.y);
}
template <typename T>
__global__ void k_smooth_binomial(G g, const T *__restrict__ s, T *d) {
  smooth_binomial_at(g, s, d, (int)blockIdx.x, (int)blockIdx.y);
}
template <typename T, typename L = LdPlain>
__device__ __forceinline__ void smooth_compensate_cell(const G &g, const T *__restrict__ d, T *s,
                                                       int ix, int iy) {
  if (ix > g.nx + 1 || iy > g.ny + 1) return;
  const int64_t c = at(g, ix, iy), n = g.nxg;
  const T v = compensate_val(L::ld(d + c), L::ld(d + c - 1), L::ld(d + c + 1), L::ld(d + c - n),
                             L::ld(d + c + n), L::ld(d + c - 1 - n), L::ld(d + c - 1 + n),
                             L::ld(d + c + 1 - n), L::ld(d + c + 1 + n));
  store_with_guards(g, s, ix, iy, v);
}
template <typename T>
__device__ __forceinline__ void smooth_compensate_at(const G &g, const T *__restrict__ d, T *s,
                                                     int tbx, int tby) {
  smooth_compensate_cell(g, d, s, 1 + tbx * TX + (int)threadIdx.x,
                         1 + tby * TY + (int)threadIdx.y);
}
template <typename T>
__global__ void k_smooth_compensate(G g, const T *__restrict__ d, T *s) {
  smooth_compensate_at(g, d, s, (int)blockIdx.x, (int)blockIdx.y);
}

// ---- Poisson right-hand side (pic/fields.f90:392-405): f = (div E - rho)
// * dx * dx on the nx*ny periodic grid; written straight into r (u = 0, so
// cgm's first residual r = f - L u is f) and p = r.
template <typename T, typename L = LdPlain>
__device__ __forceinline__ void poisson_rhs_cell(const G &g, const T *__restrict__ fld, T dx,
                                                 T dy, T *r, T *p, int ix, int iy) {
  if (ix > g.nx || iy > g.ny) return;
  const T *ex = fld + EM2G_EX * g.w, *ey = fld + EM2G_EY * g.w, *rho = fld + EM2G_RHO * g.w;
  const int ixm = (ix == 1) ? g.nx : ix - 1;
  const T f = (L::ld(ex + at(g, ix, iy)) - L::ld(ex + at(g, ixm, iy))) / dx +
              (L::ld(ey + at(g, ix, iy)) - L::ld(ey + at(g, ix, iy - 1))) / dy -
              L::ld(rho + at(g, ix, iy));
  const T fs = f * dx * dx;
  const int64_t k = (int64_t)(iy - 1) * g.nx + (ix - 1);
  r[k] = fs;
  p[k] = fs;
}
template <typename T>
__device__ __forceinline__ void poisson_rhs_at(const G &g, const T *__restrict__ fld, T dx, T dy,
                                               T *r, T *p, int tbx, int tby) {
  poisson_rhs_cell(g, fld, dx, dy, r, p, 1 + tbx * TX + (int)threadIdx.x,
                   1 + tby * TY + (int)threadIdx.y);
}
template <typename T>
__global__ void k_poisson_rhs(G g, const T *__restrict__ fld, T dx, T dy, T *r, T *p) {
  poisson_rhs_at(g, fld, dx, dy, r, p, (int)blockIdx.x, (int)blockIdx.y);
}

// ---- E -= grad(phi) with periodic images and guards (pic/fields.f90:410-442)
template <typename T>
__device__ __forceinline__ void store_images(const G &g, T *a, int ix, int iy, T v) {
  // (ix,iy) in 1..nx x 1..ny; its copies in 0..nx+2 x 0..ny+2
  int xs[3], ys[3], nxs = 0, nys = 0;
  xs[nxs++] = ix;
  if (ix == 1) xs[nxs++] = g.nx + 1;
  if (ix == g.nx) xs[nxs++] = 0;
  if (ix == 2) xs[nxs++] = g.nx + 2;
  ys[nys++] = iy;
  if (iy == 1) ys[nys++] = g.ny + 1;
  if (iy == g.ny) ys[nys++] = 0;
  if (iy == 2) ys[nys++] = g.ny + 2;
  for (int a1 = 0; a1 < nys; ++a1)
    for (int a0 = 0; a0 < nxs; ++a0) a[at(g, xs[a0], ys[a1])] = v;
}
template <typename T, typename L = LdPlain>
__device__ __forceinline__ void poisson_correct_cell(const G &g, T *fld, const T *__restrict__ u,
                                                     T dx, T dy, int ix, int iy) {
  if (ix > g.nx || iy > g.ny) return;
  T *ex = fld + EM2G_EX * g.w, *ey = fld + EM2G_EY * g.w;
  const int64_t k = (int64_t)(iy - 1) * g.nx + (ix - 1);
  const int64_t kxp = (int64_t)(iy - 1) * g.nx + (ix == g.nx ? 0 : ix);
  const int64_t kyp = (int64_t)(iy == g.ny ? 0 : iy) * g.nx + (ix - 1);
  const T uc = L::ld(u + k);
  const T vx = L::ld(ex + at(g, ix, iy)) - (L::ld(u + kxp) - uc) / dx;
  const T vy = L::ld(ey + at(g, ix, iy)) - (L::ld(u + kyp) - uc) / dy;
  store_images(g, ex, ix, iy, vx);
  store_images(g, ey, ix, iy, vy);
}
template <typename T>
__device__ __forceinline__ void poisson_correct_at(const G &g, T *fld, const T *__restrict__ u,
                                                   T dx, T dy, int tbx, int tby) {
  poisson_correct_cell(g, fld, u, dx, dy, 1 + tbx * TX + (int)threadIdx.x,
                       1 + tby * TY + (int)threadIdx.y);
}
template <typename T>
__global__ void k_poisson_correct(G g, T *fld, const T *__restrict__ u, T dx, T dy) {
  poisson_correct_at(g, fld, u, dx, dy, (int)blockIdx.x, (int)blockIdx.y);
}

// ---- conjugate gradient, one persistent launch (pic/fields.f90:508-651)
//
// All blocks are co-resident (cooperative launch).  Between phases they
// meet at a software grid barrier whose wait is bounded: after kSpinLimit
// polls a block records a timeout in status[0] and every block leaves.
// Dot products: each block writes a partial; after the barrier every block
// sums all partials in the same fixed order, so all blocks take the same
// decisions on the same values.
constexpr long kSpinLimit = 20000000;  // polls of ~100 ns: about 2 s

__device__ bool grid_barrier(unsigned *bar, unsigned nblocks, int *status) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = bar + 1;
    const unsigned g0 = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long spins = 0;
      while (*gen == g0) {
        if (*(volatile int *)status != 0) break;
        if (++spins > kSpinLimit) {
          atomicExch(status, 1);
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int *)status == 0;
}

// A probe of that bounded wait: one block arrives at a barrier counted for
// two, so nothing releases it; its wait runs out after kSpinLimit polls and
// records the timeout in status[0].  No fault and no trap: the context stays
// usable (em2g_selftest_waits).
__global__ void k_barrier_wait_probe(unsigned *bar, int *status) { grid_barrier(bar, 2u, status); }

// sum of nb partials in a fixed order; result valid in every thread
__device__ double sum_partials(const double *partial, int nb, double *sh) {
  if (threadIdx.x < 32) {
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += 32) v += ((volatile const double *)partial)[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) sh[0] = v;
  }
  __syncthreads();
  const double r = sh[0];
  __syncthreads();
  return r;
}

__device__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (int)(blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

template <typename T>
struct CgArgs {
  int nx, ny;
  T *u, *r, *p, *ap;
  double *partial;  // [2][gridDim.x]
  unsigned *bar;
  int *status;      // [0] timeout, [1] iterations
  double *res;      // [0] mean r^2 before the first iteration, [1] at exit
  int maxits;
  double eps;
};

// The solve on blocks bidx = 0..nb-1 of a launch (all of them for one
// system, or one run's share of an ensemble launch); sh: 33 doubles.
template <typename T>
__device__ __forceinline__ void cg_body(const CgArgs<T> &a, int bidx, unsigned nb, double *sh) {
  const int64_t N = (int64_t)a.nx * a.ny;
  const int64_t tid = (int64_t)bidx * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)nb * blockDim.x;
  double *part0 = a.partial, *part1 = a.partial + nb;
  // rr = sum r^2 for n = 1 (pic/fields.f90:546-556); u starts at 0
  double loc = 0.0;
  for (int64_t k = tid; k < N; k += stride) {
    a.u[k] = T(0);
    loc += (double)a.r[k] * (double)a.r[k];
  }
  loc = block_sum(loc, sh);
  if (threadIdx.x == 0) part0[bidx] = loc;
  if (!grid_barrier(a.bar, nb, a.status)) return;
  double rr = sum_partials(part0, nb, sh);
  if (bidx == 0 && threadIdx.x == 0) a.res[0] = rr / a.nx / a.ny;
  double r_last = rr;
  int n;
  for (n = 1; n <= a.maxits; ++n) {
    // ap = L p and pap = sum p*ap (pic/fields.f90:559-584)
    loc = 0.0;
    for (int64_t k = tid; k < N; k += stride) {
      const int j = (int)(k % a.nx), l = (int)(k / a.nx);
      const int64_t row = (int64_t)l * a.nx;
      const int64_t kxp = row + (j == a.nx - 1 ? 0 : j + 1);
      const int64_t kxm = row + (j == 0 ? a.nx - 1 : j - 1);
      const int64_t kyp = (int64_t)(l == a.ny - 1 ? 0 : l + 1) * a.nx + j;
      const int64_t kym = (int64_t)(l == 0 ? a.ny - 1 : l - 1) * a.nx + j;
      // p was written by other threads before the barrier: read past L1
      const T pc = __ldcg(a.p + k);
      const T v = __ldcg(a.p + kxp) + __ldcg(a.p + kxm) + __ldcg(a.p + kyp) +
                  __ldcg(a.p + kym) - T(4) * pc;
      a.ap[k] = v;
      loc += (double)pc * (double)v;
    }
    loc = block_sum(loc, sh);
    if (threadIdx.x == 0) part1[bidx] = loc;
    if (!grid_barrier(a.bar, nb, a.status)) return;
    const double pap = sum_partials(part1, nb, sh);
    const double ak = rr / pap;
    // u += ak p, r1 = r - ak ap, r_norm = sum r1^2 (pic/fields.f90:586-614)
    loc = 0.0;
    for (int64_t k = tid; k < N; k += stride) {
      a.u[k] = (T)(a.u[k] + ak * a.p[k]);
      const T r1 = (T)(a.r[k] - ak * a.ap[k]);
      a.r[k] = r1;
      loc += (double)r1 * (double)r1;
    }
    loc = block_sum(loc, sh);
    if (threadIdx.x == 0) part0[bidx] = loc;
    if (!grid_barrier(a.bar, nb, a.status)) return;
    const double r_norm = sum_partials(part0, nb, sh);
    r_last = r_norm;
    if (r_norm / a.nx / a.ny < a.eps) break;  // pic/fields.f90:616
    const double bk = r_norm / rr;            // pic/fields.f90:632
    for (int64_t k = tid; k < N; k += stride) a.p[k] = (T)(a.r[k] + bk * a.p[k]);
    rr = r_norm;  // next pass's sum of r^2 over the same r, same order
    if (!grid_barrier(a.bar, nb, a.status)) return;
  }
  if (bidx == 0 && threadIdx.x == 0) {
    a.status[1] = n;
    a.res[1] = r_last / a.nx / a.ny;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_cg(CgArgs<T> a) {
  __shared__ double sh[33];
  cg_body(a, (int)blockIdx.x, gridDim.x, sh);
}

// ---- energies (pic/fields.f90:267-347): per-block partial sums of a^2 over
// rows lo..hi, columns 1..nx of the six E/B arrays.
template <typename T>
__global__ void k_energy_partial(G g, const T *__restrict__ fld, int lo, int hi,
                                 double *partial) {
  __shared__ double sh[32];
  const int k = blockIdx.y;  // field 0..5
  const T *a = fld + k * g.w;
  const int64_t ncols = g.nx, nrows = hi - lo + 1, N = ncols * nrows;
  double loc = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < N;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int ix = 1 + (int)(t % ncols), iy = lo + (int)(t / ncols);
    const double v = (double)a[at(g, ix, iy)];
    loc += v * v;
  }
  loc = block_sum(loc, sh);
  if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = loc;
}
__global__ void k_energy_finish(const double *__restrict__ partial, int nb, double anorml1,
                                int rows_mode, int ny, double *out) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v += partial[k * nb + i];
  v = block_sum(v, sh);
  // pic/fields.f90:341: exe = exes*anorml1*ny/80.d0
  if (threadIdx.x == 0) out[k] = rows_mode ? v * anorml1 * ny / 80.0 : v * anorml1;
}


}  // namespace
}  // namespace grid
}  // namespace em2g

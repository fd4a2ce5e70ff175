// adjoint.cu -- reverse-mode derivative of the FP64 fast step (em2g_step
// with the exact Poisson solve) for periodic states.  em2 has no adjoint;
// the transposes follow the step's structure (pic/move.f90, pic/curnt.f90,
// pic/fields.f90):
//
//   fields, in reverse: the Poisson projection E <- E - grad L^-1 dx^2
//   (div E - rho) is self-adjoint in E and gives rho the adjoint
//   -L^-1 dx^2 div(lambda_E); smooth2 is a symmetric stencil, its own
//   transpose; the Yee half steps transpose into negated transposed curls;
//   J's adjoint is -dt/2 lambda_E.
//   particles, in reverse: the deposits' transpose is a gather of the
//   current and charge adjoints at the particles (with the derivative of
//   the quadratic weights for the positions), the gather's transpose a
//   scatter of the force adjoint onto E and B, and the Boris rotation is
//   reversed stage by stage.
//
// Memory.  The forward sweep keeps a checkpoint every K steps: the
// context's field block and its particles (x, y, vx, vy, vz, gamma, slot
// order).  The reverse sweep takes the segments last to first: it restores
// the segment's checkpoint into the context, recomputes the segment's K
// steps keeping E and B before each (K slots of 6 periodic arrays), and
// sweeps back through them.  So the memory is O(T/K) checkpoints plus K
// field slots, at the price of a second forward pass.  With more slots
// (em2g_adj_field_slots; em2g_adj_keep_all_fields for one per step) the
// forward sweep fills them with E and B of its last steps, which the
// reverse sweep then uses without recomputing; only the steps before them
// are recomputed, a segment at a time, in the slots already gone through.  The particles need no per-step
// store in either mode: the push is invertible, so one kernel per step
// rebuilds the previous particle state from the current one (x -= v dt/dx
// with u's velocity, then the Boris rotation about the same t by the
// opposite angle) and applies the transposed step to it.  Round-off of the
// rebuild grows for at most K steps: at every checkpoint the kept exact
// state replaces it.
//
// Layout.  Field adjoints are periodic (ny, nx) arrays, element [j][i]
// holding em2's node (i+1, j+1).  Particles and their adjoints travel
// together in one working set per species (x, y, ux, uy, uz, and the five
// adjoints), grouped by cell and regrouped every few steps as the rebuilt
// positions drift; a CTA owns a row segment of 32 cells, 4 lanes per cell,
// with the (E, B) pairs, the current and charge adjoints it gathers, and
// the E and B adjoints it scatters, in shared-memory windows.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "em2g_internal.cuh"
#include "sort_common.cuh"

struct em2g_adj {
  em2g_ctx *ctx = nullptr;
  int nx = 0, ny = 0, nsp = 0;
  int64_t N = 0;  // nx*ny
  int max_steps = 0, K = 1;
  int steps = 0, it0 = 0;
  double dx = 0, dy = 0, dt = 0, c = 1;
  double ae[EM2G_MAX_SPECIES] = {}, qd[EM2G_MAX_SPECIES] = {};
  int64_t n[EM2G_MAX_SPECIES] = {}, pb[EM2G_MAX_SPECIES] = {};  // particles, first index
  int64_t ptot = 0;
  double *hist = nullptr;   // nhist x 6 x N: E, B before each step
  int nhist = 0;            // K .. max_steps slots
  int keep_from = 0;        // the forward sweep kept E, B of steps keep_from..steps-1
  double *ckpt = nullptr;   // nck x 6 x ptot (per species 6 x n, slot order)
  double *ckfld = nullptr;  // nck x 13 x w, the context's field block
  int nck = 0;
  double *fin = nullptr;    // 6 x ptot, the particles after the last recorded step
  double *finfld = nullptr; // 13 x w, the field block after it
  double *work = nullptr, *work_alt = nullptr;  // 10 x ptot (per species 10 x n)
  int32_t *slot = nullptr, *slot_alt = nullptr;
  int32_t *off = nullptr;   // per species ncell+1
  int32_t *cnt = nullptr, *cursor = nullptr, *scan_tmp = nullptr;
  double *g = nullptr;      // lE(3N) lB(3N) lJ(3N) lrho(N) w(N) tmp(6N)
  double2 *spec = nullptr, *scaled = nullptr;  // N, nsp x 3 x N
  bool seeded = false, swept = false;
};

namespace em2g {
namespace {

constexpr int TCX = 32, G = 4, WY = 6, WX = TCX + 5;
constexpr int kRegroup = 8;  // reverse steps between regroupings

// periodic wrap of an index within one period of [0, n)
__device__ __forceinline__ int wrapi(int i, int n) {
  return i < 0 ? i + n : (i >= n ? i - n : i);
}
// periodic wrap of any index (the window may be wider than the grid)
__device__ __forceinline__ int wrapm(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

// quadratic weights (pic/move.f90:76-148) with their x-derivatives; `i` is
// em2's index of the middle node
struct W3 {
  int i;
  double m, s, p, dm, ds, dp;
};
__device__ __forceinline__ W3 w_half(double x) {
  const int ix = (int)(x + 1.0);
  const double d = x + 0.5 - ix, e = 1.0 + x - ix, f = ix - x;
  return W3{ix, 0.5 * f * f, 0.75 - d * d, 0.5 * e * e, -f, -2.0 * d, e};
}
__device__ __forceinline__ W3 w_node(double x) {
  const int ix = (int)(x + 1.5);
  const double d = x + 1.0 - ix, e = 1.5 + x - ix, f = -0.5 - x + ix;
  return W3{ix, 0.5 * f * f, 0.75 - d * d, 0.5 * e * e, -f, -2.0 * d, e};
}

// where a 3x3 stencil sits: in the window (column, row of its first node)
// or, outside it, em2's indices of its middle node (periodic wrap applied at
// use).  The weights travel separately.
struct Sten {
  bool win;
  int c0, r0;  // window column and row of em2 node (i-1, j-1)
  int i, j;    // em2 node indices of the middle node
};

struct Seg {
  int x0, y0, nx, ny;
};

// em2 node index i of a particle whose wrapped cell is cx, seen from the
// group cell kx: the same node unwrapped next to the group
__device__ __forceinline__ int unwrap_shift(int cx, int kx, int n) {
  const int d = cx - kx;
  return d > n / 2 ? -n : (d < -n / 2 ? n : 0);
}

__device__ __forceinline__ Sten make_sten(const Seg &s, int i, int j, int shx, int shy) {
  Sten t;
  t.i = i;
  t.j = j;
  t.c0 = i - 1 + shx - (s.x0 - 1);
  t.r0 = j - 1 + shy - (s.y0 - 1);
  t.win = t.c0 >= 0 && t.c0 + 2 < WX && t.r0 >= 0 && t.r0 + 2 < WY;
  return t;
}

// periodic array index of stencil node (a, b), a, b in 0..2 (em2 node
// (i-1+a, j-1+b) is periodic node (i-2+a, j-2+b))
__device__ __forceinline__ int64_t gidx(const Sten &t, int a, int b, int nx, int ny) {
  return (int64_t)wrapi(t.j - 2 + b, ny) * nx + wrapi(t.i - 2 + a, nx);
}

struct Grad {
  double v, gx, gy;
};

// value and x-, y-derivatives of sum F w_x w_y over the stencil
__device__ __forceinline__ Grad gather_g(const double *glob, const double (*win)[WX],
                                         const Sten &t, const W3 &X, const W3 &Y, int nx,
                                         int ny) {
  const double wx[3] = {X.m, X.s, X.p}, dwx[3] = {X.dm, X.ds, X.dp};
  const double wy[3] = {Y.m, Y.s, Y.p}, dwy[3] = {Y.dm, Y.ds, Y.dp};
  double F[3][3];
  if (t.win) {
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q) F[b][q] = win[t.r0 + b][t.c0 + q];
  } else {
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q) F[b][q] = glob[gidx(t, q, b, nx, ny)];
  }
  Grad r{0.0, 0.0, 0.0};
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    double sv = 0.0, sd = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      sv += F[b][q] * wx[q];
      sd += F[b][q] * dwx[q];
    }
    r.v += sv * wy[b];
    r.gx += sd * wy[b];
    r.gy += sv * dwy[b];
  }
  return r;
}

// value of sum (E, B) w_x w_y over the stencil
__device__ __forceinline__ double2 gather_v2(const double2 *glob, const double2 (*win)[WX],
                                             const Sten &t, const W3 &X, const W3 &Y, int nx,
                                             int ny) {
  const double wx[3] = {X.m, X.s, X.p}, wy[3] = {Y.m, Y.s, Y.p};
  double2 F[3][3];
  if (t.win) {
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q) F[b][q] = win[t.r0 + b][t.c0 + q];
  } else {
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q) F[b][q] = glob[gidx(t, q, b, nx, ny)];
  }
  double2 r = make_double2(0.0, 0.0);
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    double2 sv = make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double2 f = F[b][q];
      sv.x += f.x * wx[q];
      sv.y += f.y * wx[q];
    }
    r.x += sv.x * wy[b];
    r.y += sv.y * wy[b];
  }
  return r;
}

// Per-lane accumulators of the E and B adjoints a lane's cell can receive
// from its in-cell particles, every stencil position covered: nodes
// (kx .. kx+3, ky .. ky+3) in em2 indices; x staggering (half, node) 3x4,
// y staggering (node, half) 4x3, z staggering (half, half) 3x3, for E then B.
// Stored entry-major, lane-minor ([kBlk][threads]): no bank conflicts, no
// atomics.
constexpr int kBlk = 66;
// first entry of component c (lEx lEy lEz lBx lBy lBz) and entries per row
__host__ __device__ constexpr int blk_off(int c) {
  return c == 0 ? 0 : c == 1 ? 12 : c == 2 ? 24 : c == 3 ? 33 : c == 4 ? 45 : 57;
}
__host__ __device__ constexpr int blk_w(int c) { return c % 3 == 1 ? 4 : 3; }

// The gather's transpose and its position derivative in one pass over an
// (E, B) stencil of staggering c: add sc (qe, qb) w_x w_y to the E and B
// adjoints -- into this lane's block when the particle is in the lane's
// cell (block row rr, column cc of the stencil's first node), else into the
// arrays with atomics -- and return (qe dE/dx + qb dB/dx, qe dE/dy + qb
// dB/dy) of the gathered pair.
__device__ __forceinline__ double2 scatter_grad2(const double2 *glob, const double2 (*win)[WX],
                                                 double *ge, double *gb, double *blk, int c,
                                                 bool incell, int rr, int cc, const Sten &t,
                                                 const W3 &X, const W3 &Y, int nx, int ny,
                                                 double qe, double qb, double sc) {
  const double wx[3] = {X.m, X.s, X.p}, dwx[3] = {X.dm, X.ds, X.dp};
  const double wy[3] = {Y.m, Y.s, Y.p}, dwy[3] = {Y.dm, Y.ds, Y.dp};
  constexpr int kLanes = TCX * G;
  const int bw = blk_w(c);
  double *be = blk + (int64_t)(blk_off(c) + rr * bw + cc) * kLanes;
  double *bb = blk + (int64_t)(blk_off(c + 3) + rr * bw + cc) * kLanes;
  double gx = 0.0, gy = 0.0;
  const double se = sc * qe, sb = sc * qb;
  double2 F[3][3];
  if (t.win) {
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q) F[b][q] = win[t.r0 + b][t.c0 + q];
  } else {
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q) F[b][q] = glob[gidx(t, q, b, nx, ny)];
  }
#pragma unroll
  for (int b = 0; b < 3; ++b) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double h = qe * F[b][q].x + qb * F[b][q].y;
      gx += h * dwx[q] * wy[b];
      gy += h * wx[q] * dwy[b];
    }
  }
  if (incell) {
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const double w = wx[q] * wy[b];
        be[(b * bw + q) * kLanes] += se * w;
        bb[(b * bw + q) * kLanes] += sb * w;
      }
  } else {
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const double w = wx[q] * wy[b];
        const int64_t k = gidx(t, q, b, nx, ny);
        atomicAdd(ge + k, se * w);
        atomicAdd(gb + k, sb * w);
      }
  }
  return make_double2(gx, gy);
}

__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double dot3(double3 a, double3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
__device__ __forceinline__ double3 add3(double3 a, double3 b) {
  return make_double3(a.x + b.x, a.y + b.y, a.z + b.z);
}
__device__ __forceinline__ double3 sub3(double3 a, double3 b) {
  return make_double3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ double3 mul3(double k, double3 a) {
  return make_double3(k * a.x, k * a.y, k * a.z);
}

struct RevArgs {
  const double2 *ebx, *ebz, *eby;        // (ae E, ae B) pairs, periodic
  const double *ljx, *ljy, *ljz, *lrho;  // current and charge adjoints
  double *lE[3], *lB[3];                 // E and B adjoints (accumulated)
  double *P;                             // working set, 10 x n
  int64_t n;
  const int32_t *off;
  int nx, ny;
  double ae, qd, dtdx, dtdy, c;
};

constexpr int kBlkBytes = kBlk * TCX * G * (int)sizeof(double);

// One reverse step of one species: rebuild each particle's state before the
// step, then the transposed move + curnt.  Staggerings: Ex, Bx, Jx (half, node);
// Ey, By, Jy (node, half); Ez, Bz, Jz (half, half); rho (node, node).
__global__ void __launch_bounds__(TCX *G) k_adj_push(RevArgs a) {
  __shared__ double2 w_eb[3][WY][WX];  // 0: (E,B)x, 1: (E,B)z, 2: (E,B)y
  __shared__ double w_lj[3][WY][WX];   // lJx, lJy, lJz
  __shared__ double w_lr[WY][WX];
  extern __shared__ double blk[];      // kBlk x (TCX*G): per-lane E and B adjoints
  const int nx = a.nx, ny = a.ny;
  const Seg seg{(int)blockIdx.x * TCX, (int)blockIdx.y, nx, ny};
  for (int t = threadIdx.x; t < WY * WX; t += blockDim.x) {
    const int r = t / WX, col = t % WX;
    // window node (em2 index x0-1+col, y0-1+r) -> periodic (index-1)
    const int64_t k = (int64_t)wrapm(seg.y0 - 2 + r, ny) * nx + wrapm(seg.x0 - 2 + col, nx);
    w_eb[0][r][col] = a.ebx[k];
    w_eb[1][r][col] = a.ebz[k];
    w_eb[2][r][col] = a.eby[k];
    w_lj[0][r][col] = a.ljx[k];
    w_lj[1][r][col] = a.ljy[k];
    w_lj[2][r][col] = a.ljz[k];
    w_lr[r][col] = a.lrho[k];
  }
  for (int e = 0; e < kBlk; ++e) blk[e * (TCX * G) + threadIdx.x] = 0.0;
  __syncthreads();

  const int gl = threadIdx.x & (G - 1);
  const int kx = seg.x0 + (int)(threadIdx.x / G), ky = seg.y0;
  const int64_t n = a.n;
  double *P = a.P;
  if (kx < nx) {
    const int64_t cell = (int64_t)ky * nx + kx;
    const int32_t beg = a.off[cell], end = a.off[cell + 1];
    const double q = a.qd;
    // software pipeline: the next particle's state and adjoints are loaded
    // while this one runs
    double nx_[10];
    if (beg + gl < end)
#pragma unroll
      for (int c = 0; c < 10; ++c) nx_[c] = P[c * n + beg + gl];
    for (int32_t i = beg + gl; i < end; i += G) {
      double cur[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) cur[c] = nx_[c];
      if (i + G < end)
#pragma unroll
        for (int c = 0; c < 10; ++c) nx_[c] = P[c * n + i + G];
      // the state after the step
      const double x1 = cur[0], y1 = cur[1];
      const double3 u1 = make_double3(cur[2], cur[3], cur[4]);
      const double g1 = sqrt(1.0 + dot3(u1, u1));
      const double3 v = mul3(1.0 / g1, u1);
      // rebuild the position before the move (pic/curnt.f90:181-194)
      double x0 = x1 - v.x * a.dtdx, y0 = y1 - v.y * a.dtdy;
      if (x0 < 0.0) x0 += nx; else if (x0 >= nx) x0 -= nx;
      if (y0 < 0.0) y0 += ny; else if (y0 >= ny) y0 -= ny;
      const int sx0 = unwrap_shift((int)x0, kx, nx), sy0 = unwrap_shift((int)y0, ky, ny);
      const W3 hx0 = w_half(x0), nx0 = w_node(x0), hy0 = w_half(y0), ny0 = w_node(y0);
      const Sten s_x0 = make_sten(seg, hx0.i, ny0.i, sx0, sy0);  // x staggering (half, node)
      const Sten s_y0 = make_sten(seg, nx0.i, hy0.i, sx0, sy0);  // y staggering (node, half)
      const Sten s_z0 = make_sten(seg, hx0.i, hy0.i, sx0, sy0);  // z staggering (half, half)
      // scaled fields before the step at the old position
      const double2 ebx = gather_v2(a.ebx, w_eb[0], s_x0, hx0, ny0, nx, ny);
      const double2 ebz = gather_v2(a.ebz, w_eb[1], s_z0, hx0, hy0, nx, ny);
      const double2 eby = gather_v2(a.eby, w_eb[2], s_y0, nx0, hy0, nx, ny);
      const double3 aE = make_double3(ebx.x, eby.x, ebz.x);
      const double3 aB = make_double3(ebx.y, eby.y, ebz.y);
      // rebuild u before the Boris rotation (pic/move.f90:176-203): the
      // rotation about t by the opposite angle
      double3 um, t, up, s;
      double gm, f;
      {
        const double3 upl_b = sub3(u1, aE);
        const double3 tb = mul3(1.0 / (a.c * sqrt(1.0 + dot3(upl_b, upl_b))), aB);
        const double3 up_b = sub3(upl_b, cross3(upl_b, tb));
        const double3 sb = mul3(2.0 / (1.0 + dot3(tb, tb)), tb);
        const double3 u0 = sub3(sub3(upl_b, cross3(up_b, sb)), aE);
        // the forward intermediates from the rebuilt state
        um = add3(u0, aE);
        gm = sqrt(1.0 + dot3(um, um));
        t = mul3(1.0 / (a.c * gm), aB);
        up = add3(um, cross3(um, t));
        f = 2.0 / (1.0 + dot3(t, t));
        s = mul3(f, t);
        P[2 * n + i] = u0.x;
        P[3 * n + i] = u0.y;
        P[4 * n + i] = u0.z;
      }
      const double vv[3] = {v.x, v.y, v.z};
      double lv[3] = {0.0, 0.0, 0.0};
      double lx, ly;
      {  // transposed deposits at the new position: rho and jp
        const int sx1 = unwrap_shift((int)x1, kx, nx), sy1 = unwrap_shift((int)y1, ky, ny);
        const W3 hx1 = w_half(x1), nx1 = w_node(x1), hy1 = w_half(y1), ny1 = w_node(y1);
        const Grad gr = gather_g(a.lrho, w_lr, make_sten(seg, nx1.i, ny1.i, sx1, sy1), nx1, ny1,
                                 nx, ny);
        double lxn = cur[5] + q * gr.gx, lyn = cur[6] + q * gr.gy;
        const Grad jx = gather_g(a.ljx, w_lj[0], make_sten(seg, hx1.i, ny1.i, sx1, sy1), hx1,
                                 ny1, nx, ny);
        const Grad jy = gather_g(a.ljy, w_lj[1], make_sten(seg, nx1.i, hy1.i, sx1, sy1), nx1,
                                 hy1, nx, ny);
        const Grad jz = gather_g(a.ljz, w_lj[2], make_sten(seg, hx1.i, hy1.i, sx1, sy1), hx1,
                                 hy1, nx, ny);
        lv[0] = q * jx.v;
        lv[1] = q * jy.v;
        lv[2] = q * jz.v;
        lxn += q * (vv[0] * jx.gx + vv[1] * jy.gx + vv[2] * jz.gx);
        lyn += q * (vv[0] * jx.gy + vv[1] * jy.gy + vv[2] * jz.gy);
        // move: x1 = x0 + v dt/dx
        lx = lxn;
        ly = lyn;
        lv[0] += lxn * a.dtdx;
        lv[1] += lyn * a.dtdy;
      }
      {  // jm at the old position
        const Grad jx = gather_g(a.ljx, w_lj[0], s_x0, hx0, ny0, nx, ny);
        const Grad jy = gather_g(a.ljy, w_lj[1], s_y0, nx0, hy0, nx, ny);
        const Grad jz = gather_g(a.ljz, w_lj[2], s_z0, hx0, hy0, nx, ny);
        lv[0] += q * jx.v;
        lv[1] += q * jy.v;
        lv[2] += q * jz.v;
        lx += q * (vv[0] * jx.gx + vv[1] * jy.gx + vv[2] * jz.gx);
        ly += q * (vv[0] * jx.gy + vv[1] * jy.gy + vv[2] * jz.gy);
      }
      // v = u1 / gamma(u1)
      const double3 lvv = make_double3(lv[0], lv[1], lv[2]);
      const double dt_ = dot3(lvv, u1);
      double3 lun = sub3(mul3(1.0 / g1, lvv), mul3(dt_ / (g1 * g1 * g1), u1));
      lun = add3(lun, make_double3(cur[7], cur[8], cur[9]));
      // Boris, reversed stage by stage
      double3 laE = lun;
      double3 lum = lun;
      const double3 lup = cross3(s, lun);
      const double3 ls = cross3(lun, up);
      double3 lt = mul3(f, ls);
      const double lf = dot3(ls, t);
      lt = sub3(lt, mul3(f * f * lf, t));
      lum = add3(add3(lum, lup), cross3(t, lup));
      lt = add3(lt, cross3(lup, um));
      const double3 laB = mul3(1.0 / (a.c * gm), lt);
      const double lg = -dot3(lt, t) / gm;
      lum = add3(lum, mul3(lg / gm, um));
      laE = add3(laE, lum);
      // transposed gather: the force adjoint onto E and B, and the gathered
      // fields' position derivatives
      const double ae = a.ae;
      // in the lane's cell: half-staggered stencils start at the cell's node,
      // node-staggered ones at it or the next
      const bool incell = (int)x0 == kx && (int)y0 == ky;
      const int ch = hx0.i - 1 - kx, cn = nx0.i - 1 - kx;
      const int rh = hy0.i - 1 - ky, rn = ny0.i - 1 - ky;
      double2 d = scatter_grad2(a.ebx, w_eb[0], a.lE[0], a.lB[0], blk + threadIdx.x, 0, incell,
                                rn, ch, s_x0, hx0, ny0, nx, ny, laE.x, laB.x, ae);
      lx += d.x;
      ly += d.y;
      d = scatter_grad2(a.eby, w_eb[2], a.lE[1], a.lB[1], blk + threadIdx.x, 1, incell, rh, cn,
                        s_y0, nx0, hy0, nx, ny, laE.y, laB.y, ae);
      lx += d.x;
      ly += d.y;
      d = scatter_grad2(a.ebz, w_eb[1], a.lE[2], a.lB[2], blk + threadIdx.x, 2, incell, rh, ch,
                        s_z0, hx0, hy0, nx, ny, laE.z, laB.z, ae);
      lx += d.x;
      ly += d.y;
      // the state before the step and its adjoints, in place
      P[i] = x0;
      P[n + i] = y0;
      P[5 * n + i] = lx;
      P[6 * n + i] = ly;
      P[7 * n + i] = lum.x;
      P[8 * n + i] = lum.y;
      P[9 * n + i] = lum.z;
    }
  }
  __syncthreads();
  // every cell's four lane blocks summed and added to the arrays once
  // (blocks of neighbouring cells and segments overlap: atomics)
  for (int t = threadIdx.x; t < TCX * kBlk; t += blockDim.x) {
    const int cl = t / kBlk, e = t - cl * kBlk;
    const int cx = seg.x0 + cl;
    if (cx >= nx) continue;
    double v = 0.0;
#pragma unroll
    for (int l = 0; l < G; ++l) v += blk[e * (TCX * G) + cl * G + l];
    if (v == 0.0) continue;
    const int comp = e < 12 ? 0 : e < 24 ? 1 : e < 33 ? 2 : e < 45 ? 3 : e < 57 ? 4 : 5;
    const int w = blk_w(comp), f = e - blk_off(comp);
    const int row = f / w, col = f - row * w;
    // em2 node (cx + col, seg.y0 + row) -> periodic (index - 1)
    const int64_t k =
        (int64_t)wrapi(seg.y0 + row - 1, ny) * nx + wrapi(cx + col - 1, nx);
    atomicAdd((comp < 3 ? a.lE[comp] : a.lB[comp - 3]) + k, v);
  }
}

// ---- periodic grid transposes (k = j*nx + i) -------------------------------
struct PG {
  int nx, ny;
};
__device__ __forceinline__ int64_t xm(const PG &p, int64_t k) {
  const int i = (int)(k % p.nx);
  return i == 0 ? k + p.nx - 1 : k - 1;
}
__device__ __forceinline__ int64_t xp(const PG &p, int64_t k) {
  const int i = (int)(k % p.nx);
  return i == p.nx - 1 ? k - (p.nx - 1) : k + 1;
}
__device__ __forceinline__ int64_t ym(const PG &p, int64_t k) {
  return k < p.nx ? k + (int64_t)(p.ny - 1) * p.nx : k - p.nx;
}
__device__ __forceinline__ int64_t yp(const PG &p, int64_t k) {
  return k >= (int64_t)(p.ny - 1) * p.nx ? k - (int64_t)(p.ny - 1) * p.nx : k + p.nx;
}

#define PG_LOOP(N) \
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < (N); k += (int64_t)gridDim.x * blockDim.x)

// rhs = dx^2 div(lE) (backward differences)
__global__ void k_adj_div(PG p, const double *lex, const double *ley, double dx, double dy,
                          double *rhs) {
  PG_LOOP((int64_t)p.nx * p.ny) {
    rhs[k] = ((lex[k] - lex[xm(p, k)]) / dx + (ley[k] - ley[ym(p, k)]) / dy) * dx * dx;
  }
}
// lE -= grad w (forward differences); lrho = -w
__global__ void k_adj_grad(PG p, double *lex, double *ley, const double *w, double dx,
                           double dy, double *lrho) {
  PG_LOOP((int64_t)p.nx * p.ny) {
    const double wc = w[k];
    lex[k] -= (w[xp(p, k)] - wc) / dx;
    ley[k] -= (w[yp(p, k)] - wc) / dy;
    lrho[k] = -wc;
  }
}
// periodic smooth2 (pic/smooth.f90:143-177) of arrays a.p[blockIdx.y], with
// scratch tmp + blockIdx.y * N
struct Ptr6 {
  double *p[6];
};
__global__ void k_adj_smooth_b(PG p, Ptr6 a, double *tmp, int64_t N) {
  const double *s = a.p[blockIdx.y];
  double *d = tmp + blockIdx.y * N;
  PG_LOOP(N) {
    const int64_t l = xm(p, k), r = xp(p, k);
    d[k] = (4 * s[k] + 2 * (s[l] + s[r] + s[ym(p, k)] + s[yp(p, k)]) + s[ym(p, l)] +
            s[yp(p, l)] + s[ym(p, r)] + s[yp(p, r)]) /
           16.0;
  }
}
__global__ void k_adj_smooth_c(PG p, Ptr6 a, const double *tmp, int64_t N) {
  double *s = a.p[blockIdx.y];
  const double *d = tmp + blockIdx.y * N;
  PG_LOOP(N) {
    const int64_t l = xm(p, k), r = xp(p, k);
    s[k] = (20 * d[k] - d[l] - d[r] - d[ym(p, k)] - d[yp(p, k)] - d[ym(p, l)] - d[yp(p, l)] -
            d[ym(p, r)] - d[yp(p, r)]) /
           12.0;
  }
}
// transpose of B += curl E half step: lE += curl^T lB (lB passes through)
__global__ void k_adj_bhalf(PG p, double *lex, double *ley, double *lez, const double *lbx,
                            const double *lby, const double *lbz, double ctxh, double ctyh) {
  PG_LOOP((int64_t)p.nx * p.ny) {
    lez[k] += -ctyh * (lbx[k] - lbx[yp(p, k)]) + ctxh * (lby[k] - lby[xp(p, k)]);
    ley[k] -= ctxh * (lbz[xm(p, k)] - lbz[k]);
    lex[k] += ctyh * (lbz[ym(p, k)] - lbz[k]);
  }
}
// transpose of E += curl B - tem J: lB += curl^T lE, lJ = -tem lE
__global__ void k_adj_efull(PG p, const double *lex, const double *ley, const double *lez,
                            double *lbx, double *lby, double *lbz, double ctx, double cty,
                            double tem, double *ljx, double *ljy, double *ljz) {
  PG_LOOP((int64_t)p.nx * p.ny) {
    lbz[k] += cty * (lex[k] - lex[yp(p, k)]) - ctx * (ley[k] - ley[xp(p, k)]);
    lby[k] += ctx * (lez[xm(p, k)] - lez[k]);
    lbx[k] -= cty * (lez[ym(p, k)] - lez[k]);
    ljx[k] = -tem * lex[k];
    ljy[k] = -tem * ley[k];
    ljz[k] = -tem * lez[k];
  }
}
// (ae E, ae B) pairs of the three staggerings from periodic E, B (6 x N)
__global__ void k_adj_prescale(const double *eb, int64_t N, double ae, double2 *out) {
  PG_LOOP(N) {
    out[k] = make_double2(ae * eb[k], ae * eb[3 * N + k]);               // x
    out[N + k] = make_double2(ae * eb[2 * N + k], ae * eb[5 * N + k]);   // z
    out[2 * N + k] = make_double2(ae * eb[N + k], ae * eb[4 * N + k]);   // y
  }
}
// periodic E, B from the context's guarded FP64 block
__global__ void k_adj_record_fields(const double *fld, int nx, int ny, int64_t w, double *out) {
  const int64_t N = (int64_t)nx * ny;
  PG_LOOP(6 * N) {
    const int c = (int)(k / N);
    const int64_t e = k - c * N;
    const int i = (int)(e % nx), j = (int)(e / nx);
    out[k] = fld[c * w + (int64_t)(j + 1) * (nx + 3) + (i + 1)];
  }
}
// context particles (6 x cap, grouped, with slots) -> x, y, vx, vy, vz,
// gamma (6 x n, slot order): a checkpoint the context can be reset to
__global__ void k_adj_record_parts(const double *part, const int32_t *slot, int64_t n,
                                   int64_t cap, double *out) {
  PG_LOOP(n) {
    const int64_t s = slot[k];
    for (int c = 0; c < 6; ++c) out[c * n + s] = part[c * cap + k];
  }
}
// a checkpoint back into the context's particle arrays, slot order (the
// next push sorts them by cell)
__global__ void k_adj_reset_parts(const double *ck, int64_t n, int64_t cap, double *part,
                                  int32_t *slot) {
  PG_LOOP(n) {
    for (int c = 0; c < 6; ++c) part[c * cap + k] = ck[c * n + k];
    slot[k] = (int32_t)k;
  }
}
// working set from a slot-order checkpoint: x, y, u = v gamma (the
// quantity the Boris push advances, pic/move.f90:176-178), adjoints zero
__global__ void k_adj_load(const double *st, int64_t n, double *P, int32_t *slot) {
  PG_LOOP(n) {
    const double g = st[5 * n + k];
    P[k] = st[k];
    P[n + k] = st[n + k];
    for (int c = 2; c < 5; ++c) P[c * n + k] = st[c * n + k] * g;
    for (int c = 5; c < 10; ++c) P[c * n + k] = 0.0;
    slot[k] = (int32_t)k;
  }
}
// the kept exact state replaces the rebuilt one
__global__ void k_adj_restore(const double *st, int64_t n, double *P, const int32_t *slot) {
  PG_LOOP(n) {
    const int64_t s = slot[k];
    const double g = st[5 * n + s];
    P[k] = st[s];
    P[n + k] = st[n + s];
    for (int c = 2; c < 5; ++c) P[c * n + k] = st[c * n + s] * g;
  }
}
__global__ void k_adj_hist(const double *P, int64_t n, int nx, int ny, int32_t *cnt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = k < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  agg_atomic_add(cnt, cell_key(P[k], P[n + k], nx, ny), am);
}
__global__ void k_adj_scatter(const double *P, const int32_t *slot, int64_t n, int nx, int ny,
                              const int32_t *off, int32_t *cursor, double *Q, int32_t *qslot) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = k < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const int key = cell_key(P[k], P[n + k], nx, ny);
  const int64_t pos = (int64_t)off[key] + agg_atomic_add(cursor, key, am);
  for (int c = 0; c < 10; ++c) Q[c * n + pos] = P[c * n + k];
  qslot[pos] = slot[k];
}
// a checkpoint (x, y, v, gamma) as x, y, u = v gamma
__global__ void k_adj_initial(const double *st, int64_t n, double *x, double *y, double *ux,
                              double *uy, double *uz) {
  PG_LOOP(n) {
    const double g = st[5 * n + k];
    x[k] = st[k];
    y[k] = st[n + k];
    ux[k] = st[2 * n + k] * g;
    uy[k] = st[3 * n + k] * g;
    uz[k] = st[4 * n + k] * g;
  }
}
// adjoints (or the state) of the working set back to slot order
__global__ void k_adj_unsort(const double *P, const int32_t *slot, int64_t n, int first,
                             double *o0, double *o1, double *o2, double *o3, double *o4) {
  PG_LOOP(n) {
    const int64_t s = slot[k];
    o0[s] = P[(first + 0) * n + k];
    o1[s] = P[(first + 1) * n + k];
    o2[s] = P[(first + 2) * n + k];
    o3[s] = P[(first + 3) * n + k];
    o4[s] = P[(first + 4) * n + k];
  }
}

unsigned blocks_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 8192 ? (b < 1 ? 1 : b) : 8192);
}

int check_adj(em2g_adj *a) {
  if (!a || !a->ctx) return fail(EM2G_ERR_INVALID, "null adjoint");
  EM2G_CUDA(cudaSetDevice(a->ctx->device));
  return EM2G_OK;
}

double *lE(em2g_adj *a, int c) { return a->g + c * a->N; }
double *lB(em2g_adj *a, int c) { return a->g + (3 + c) * a->N; }
double *lJ(em2g_adj *a, int c) { return a->g + (6 + c) * a->N; }
double *lrho(em2g_adj *a) { return a->g + 9 * a->N; }
double *wbuf(em2g_adj *a) { return a->g + 10 * a->N; }
double *tmp6(em2g_adj *a) { return a->g + 11 * a->N; }

// sort every species' working set by the cell of its current position
int regroup(em2g_adj *a, cudaStream_t st) {
  const int64_t nc = a->N;
  for (int s = 0; s < a->nsp; ++s) {
    const int64_t n = a->n[s];
    double *P = a->work + 10 * a->pb[s], *Q = a->work_alt + 10 * a->pb[s];
    int32_t *sl = a->slot + a->pb[s], *ql = a->slot_alt + a->pb[s];
    int32_t *off = a->off + s * (nc + 1);
    EM2G_CUDA(cudaMemsetAsync(a->cnt, 0, sizeof(int32_t) * nc, st));
    EM2G_CUDA(cudaMemsetAsync(a->cursor, 0, sizeof(int32_t) * nc, st));
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (n > 0) k_adj_hist<<<nb, 256, 0, st>>>(P, n, a->nx, a->ny, a->cnt);
    int rc = scan_counts(a->cnt, off, nc, 0, a->scan_tmp, st);
    if (rc) return rc;
    if (n > 0) k_adj_scatter<<<nb, 256, 0, st>>>(P, sl, n, a->nx, a->ny, off, a->cursor, Q, ql);
    EM2G_CUDA(cudaGetLastError());
  }
  // every species was regrouped into the other buffers
  std::swap(a->work, a->work_alt);
  std::swap(a->slot, a->slot_alt);
  return EM2G_OK;
}

int smooth_T(em2g_adj *a, const Ptr6 &arr, int count, cudaStream_t st) {
  const PG p{a->nx, a->ny};
  const dim3 grid(blocks_for(a->N), count);
  k_adj_smooth_b<<<grid, 256, 0, st>>>(p, arr, tmp6(a), a->N);
  k_adj_smooth_c<<<grid, 256, 0, st>>>(p, arr, tmp6(a), a->N);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

// transposed fields(it) (pic/fields.f90:2-366 in reverse): lE, lB of the
// state after the step -> of the state before it, plus lJ and lrho
int fields_T(em2g_adj *a, int it, cudaStream_t st) {
  const PG p{a->nx, a->ny};
  const unsigned nb = blocks_for(a->N);
  const em2g_params &P = a->ctx->P;
  // Poisson: the projection is self-adjoint in E; rho's adjoint is -w,
  // w = L^-1 dx^2 div(lE)
  k_adj_div<<<nb, 256, 0, st>>>(p, lE(a, 0), lE(a, 1), a->dx, a->dy, wbuf(a));
  int rc = spectral_solve(wbuf(a), wbuf(a), a->nx, a->ny, a->spec, st);
  if (rc) return rc;
  k_adj_grad<<<nb, 256, 0, st>>>(p, lE(a, 0), lE(a, 1), wbuf(a), a->dx, a->dy, lrho(a));
  // filters (pic/fields.f90:252-260); smooth2 is its own transpose
  if (it % P.isav == 0) {
    Ptr6 eb{{lE(a, 0), lE(a, 1), lE(a, 2), lB(a, 0), lB(a, 1), lB(a, 2)}};
    if ((rc = smooth_T(a, eb, 6, st))) return rc;
  }
  Ptr6 r{{lrho(a), nullptr, nullptr, nullptr, nullptr, nullptr}};
  if ((rc = smooth_T(a, r, 1, st))) return rc;
  // Yee in reverse: B/2, E, B/2 (pic/fields.f90:184-247)
  const double ctx = P.dt * P.c / P.dx, cty = P.dt * P.c / P.dy, tem = 0.5 * P.dt;
  k_adj_bhalf<<<nb, 256, 0, st>>>(p, lE(a, 0), lE(a, 1), lE(a, 2), lB(a, 0), lB(a, 1),
                                  lB(a, 2), 0.5 * ctx, 0.5 * cty);
  k_adj_efull<<<nb, 256, 0, st>>>(p, lE(a, 0), lE(a, 1), lE(a, 2), lB(a, 0), lB(a, 1), lB(a, 2),
                                  ctx, cty, tem, lJ(a, 0), lJ(a, 1), lJ(a, 2));
  k_adj_bhalf<<<nb, 256, 0, st>>>(p, lE(a, 0), lE(a, 1), lE(a, 2), lB(a, 0), lB(a, 1),
                                  lB(a, 2), 0.5 * ctx, 0.5 * cty);
  EM2G_CUDA(cudaGetLastError());
  // the optional current filter after the fold (no em2 counterpart)
  if (P.smooth_current) {
    Ptr6 j{{lJ(a, 0), lJ(a, 1), lJ(a, 2), nullptr, nullptr, nullptr}};
    if ((rc = smooth_T(a, j, 3, st))) return rc;
  }
  return EM2G_OK;
}

}  // namespace
}  // namespace em2g

using namespace em2g;

extern "C" {

int em2g_adj_create(em2g_ctx *ctx, int max_steps, int checkpoint, em2g_adj **out) {
  if (!out) return fail(EM2G_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (!ctx) return fail(EM2G_ERR_INVALID, "null context");
  const em2g_params &P = ctx->P;
  if (P.precision != EM2G_FP64 || P.poisson != 1)
    return fail(EM2G_ERR_INVALID, "the adjoint needs an FP64 context with poisson = 1");
  if (max_steps < 1 || checkpoint < 1) return fail(EM2G_ERR_INVALID, "max_steps, checkpoint >= 1");
  for (int s = 0; s < P.nsp; ++s)
    if (P.tx[s] != 0.0 || P.ty[s] != 0.0)
      return fail(EM2G_ERR_INVALID, "the adjoint assumes tx = ty = 0 (as em2 runs)");
  if (std::fabs(P.dx - P.dy) > 1e-12 * P.dx)
    return fail(EM2G_ERR_INVALID, "the adjoint assumes dx = dy (as cgm does)");
  em2g_adj *a = new (std::nothrow) em2g_adj();
  if (!a) return fail(EM2G_ERR_NOMEM, "host allocation failed");
  auto bail = [&](int code) {
    em2g_adj_destroy(a);
    return code;
  };
  a->ctx = ctx;
  a->nx = P.nx;
  a->ny = P.ny;
  a->nsp = P.nsp;
  a->N = (int64_t)P.nx * P.ny;
  a->max_steps = max_steps;
  a->K = checkpoint;
  a->dx = P.dx;
  a->dy = P.dy;
  a->dt = P.dt;
  a->c = P.c;
  for (int s = 0; s < P.nsp; ++s) {
    a->ae[s] = 0.5 * P.qm[s] * P.dt / P.c;
    a->qd[s] = P.q[s] * P.dn[s] / (P.dx * P.dy);
    a->n[s] = ctx->sp[s].n;
    a->pb[s] = a->ptot;
    a->ptot += a->n[s];
  }
  a->nck = (max_steps + checkpoint - 1) / checkpoint;
  const int64_t N = a->N, pt = a->ptot > 0 ? a->ptot : 1;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaSetDevice"));
#define ALLOC(ptr, bytes)                                                  \
  do {                                                                     \
    e = cudaMalloc((void **)&(ptr), (bytes));                              \
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc " #ptr));   \
  } while (0)
  a->nhist = checkpoint < max_steps ? checkpoint : max_steps;
  ALLOC(a->hist, sizeof(double) * 6 * N * a->nhist);
  ALLOC(a->ckpt, sizeof(double) * 6 * pt * a->nck);
  ALLOC(a->ckfld, sizeof(double) * EM2G_NFIELD * ctx->g.w * a->nck);
  ALLOC(a->fin, sizeof(double) * 6 * pt);
  ALLOC(a->finfld, sizeof(double) * EM2G_NFIELD * ctx->g.w);
  ALLOC(a->work, sizeof(double) * 10 * pt);
  ALLOC(a->work_alt, sizeof(double) * 10 * pt);
  ALLOC(a->slot, sizeof(int32_t) * pt);
  ALLOC(a->slot_alt, sizeof(int32_t) * pt);
  ALLOC(a->off, sizeof(int32_t) * (N + 1) * P.nsp);
  ALLOC(a->cnt, sizeof(int32_t) * N);
  ALLOC(a->cursor, sizeof(int32_t) * N);
  ALLOC(a->scan_tmp, sizeof(int32_t) * scan_tmp_size(N));
  ALLOC(a->g, sizeof(double) * 17 * N);
  ALLOC(a->spec, sizeof(double2) * N);
  ALLOC(a->scaled, sizeof(double2) * 3 * N * P.nsp);
#undef ALLOC
  int rc = spectral_prepare();
  if (rc) return bail(rc);
  e = cudaFuncSetAttribute(k_adj_push, cudaFuncAttributeMaxDynamicSharedMemorySize, kBlkBytes);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaFuncSetAttribute"));
  *out = a;
  return EM2G_OK;
}

int em2g_adj_destroy(em2g_adj *a) {
  if (!a) return EM2G_OK;
  if (a->ctx) cudaSetDevice(a->ctx->device);
  void *bufs[] = {a->hist, a->ckpt,     a->ckfld,    a->fin, a->finfld, a->work, a->work_alt,
                  a->slot, a->slot_alt, a->off,      a->cnt, a->cursor, a->scan_tmp,
                  a->g,    a->spec,     a->scaled};
  for (void *p : bufs) cudaFree(p);
  delete a;
  return EM2G_OK;
}

static int record_parts(em2g_adj *a, double *dst, cudaStream_t st) {
  for (int s = 0; s < a->nsp; ++s) {
    const Species &S = a->ctx->sp[s];
    if (S.n != a->n[s]) return fail(EM2G_ERR_INVALID, "particle count changed since em2g_adj_create");
    if (S.n > 0)
      k_adj_record_parts<<<blocks_for(S.n), 256, 0, st>>>(S.part, S.slot, S.n, S.cap,
                                                          dst + 6 * a->pb[s]);
  }
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

// the context set to a kept state: field block fld, particles ck (6 x ptot,
// slot order; sorted again by the next push), step counter it
static int reset_context(em2g_adj *a, const double *fld, const double *ck, int it,
                         cudaStream_t st) {
  em2g_ctx *c = a->ctx;
  EM2G_CUDA(cudaMemcpyAsync(c->fld, fld, sizeof(double) * EM2G_NFIELD * c->g.w,
                            cudaMemcpyDeviceToDevice, st));
  for (int s = 0; s < a->nsp; ++s) {
    Species &S = c->sp[s];
    if (S.n > 0)
      k_adj_reset_parts<<<blocks_for(S.n), 256, 0, st>>>(ck + 6 * a->pb[s], S.n, S.cap, S.part,
                                                         S.slot);
    S.sorted = false;
  }
  EM2G_CUDA(cudaGetLastError());
  c->jp_live = true;
  c->it = it;
  return EM2G_OK;
}

// checkpoint ck (the state before step ck*K): field block and particles
static int record_checkpoint(em2g_adj *a, int ck, cudaStream_t st) {
  em2g_ctx *c = a->ctx;
  EM2G_CUDA(cudaMemcpyAsync(a->ckfld + (int64_t)EM2G_NFIELD * c->g.w * ck, c->fld,
                            sizeof(double) * EM2G_NFIELD * c->g.w, cudaMemcpyDeviceToDevice,
                            st));
  return record_parts(a, a->ckpt + 6 * a->ptot * ck, st);
}

// the context reset to checkpoint ck
static int reset_to_checkpoint(em2g_adj *a, int ck, cudaStream_t st) {
  return reset_context(a, a->ckfld + (int64_t)EM2G_NFIELD * a->ctx->g.w * ck,
                       a->ckpt + 6 * a->ptot * ck, a->it0 + ck * a->K, st);
}

// E and B before each of the steps k0..k1-1 into hist slots k - k0 (and
// the context advanced to the state before step k1)
static int record_segment(em2g_adj *a, int k0, int k1, cudaStream_t st) {
  em2g_ctx *c = a->ctx;
  for (int k = k0; k < k1; ++k) {
    k_adj_record_fields<<<blocks_for(6 * a->N), 256, 0, st>>>(c->fld, a->nx, a->ny, c->g.w,
                                                             a->hist + 6 * a->N * (k - k0));
    EM2G_CUDA(cudaGetLastError());
    int rc = step_enqueue(c);
    if (rc) return rc;
  }
  return EM2G_OK;
}

int em2g_adj_forward(em2g_adj *a, int nsteps) {
  em2g::NvtxRange nvtx_range("em2g adjoint forward");
  int rc = check_adj(a);
  if (rc) return rc;
  if (nsteps < 1 || nsteps > a->max_steps) return fail(EM2G_ERR_RANGE, "nsteps outside 1..max_steps");
  em2g_ctx *c = a->ctx;
  a->steps = 0;
  a->seeded = a->swept = false;
  a->it0 = c->it;
  // the last nhist steps' E and B go into the slots as the sweep passes
  a->keep_from = nsteps > a->nhist ? nsteps - a->nhist : 0;
  for (int k = 0; k < nsteps; ++k) {
    cudaStream_t st = c->stream;
    if (k >= a->keep_from) {
      k_adj_record_fields<<<blocks_for(6 * a->N), 256, 0, st>>>(
          c->fld, a->nx, a->ny, c->g.w, a->hist + 6 * a->N * (k - a->keep_from));
      EM2G_CUDA(cudaGetLastError());
    }
    if (k % a->K == 0 && (rc = record_checkpoint(a, k / a->K, st))) return rc;
    // em2g_step's pass (the fast path: the stored particles are its own),
    // enqueued without waiting for it
    if ((rc = step_enqueue(c))) return rc;
    a->steps = k + 1;
  }
  if ((rc = record_parts(a, a->fin, c->stream))) return rc;
  EM2G_CUDA(cudaMemcpyAsync(a->finfld, c->fld, sizeof(double) * EM2G_NFIELD * c->g.w,
                            cudaMemcpyDeviceToDevice, c->stream));
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int em2g_adj_seed_fields_device(em2g_adj *a, const double *dev6) {
  int rc = check_adj(a);
  if (rc) return rc;
  if (!dev6) return fail(EM2G_ERR_INVALID, "null pointer");
  cudaStream_t st = a->ctx->stream;
  EM2G_CUDA(cudaMemcpyAsync(a->g, dev6, sizeof(double) * 6 * a->N, cudaMemcpyDeviceToDevice, st));
  EM2G_CUDA(cudaMemsetAsync(a->g + 6 * a->N, 0, sizeof(double) * 11 * a->N, st));
  a->seeded = true;
  return EM2G_OK;
}

int em2g_adj_backward(em2g_adj *a) {
  em2g::NvtxRange nvtx_range("em2g adjoint backward");
  int rc = check_adj(a);
  if (rc) return rc;
  if (a->steps < 1) return fail(EM2G_ERR_INVALID, "run em2g_adj_forward first");
  if (!a->seeded) return fail(EM2G_ERR_INVALID, "seed the final adjoint first");
  cudaStream_t st = a->ctx->stream;
  for (int s = 0; s < a->nsp; ++s)
    if (a->n[s] > 0)
      k_adj_load<<<blocks_for(a->n[s]), 256, 0, st>>>(a->fin + 6 * a->pb[s], a->n[s],
                                                      a->work + 10 * a->pb[s], a->slot + a->pb[s]);
  EM2G_CUDA(cudaGetLastError());
  if ((rc = regroup(a, st))) return rc;
  int since = 0;
  const int keep_from = a->keep_from;
  int seg0 = keep_from;  // first step of the recomputed segment whose E, B are in hist
  for (int k = a->steps - 1; k >= 0; --k) {
    if (k < seg0) {
      // recompute the segment of step k from its checkpoint, into the
      // slots from 0 (the kept steps after it are done with)
      seg0 = (k / a->K) * a->K;
      if ((rc = reset_to_checkpoint(a, k / a->K, st))) return rc;
      if ((rc = record_segment(a, seg0, k + 1, st))) return rc;
    }
    if (since == kRegroup) {
      if ((rc = regroup(a, st))) return rc;
      since = 0;
    }
    if ((rc = fields_T(a, a->it0 + k + 1, st))) return rc;
    const double *eb = a->hist + 6 * a->N * (k >= keep_from ? k - keep_from : k - seg0);
    for (int s = 0; s < a->nsp; ++s) {
      double2 *sc = a->scaled + 3 * a->N * s;
      k_adj_prescale<<<blocks_for(a->N), 256, 0, st>>>(eb, a->N, a->ae[s], sc);
      RevArgs r;
      r.ebx = sc;
      r.ebz = sc + a->N;
      r.eby = sc + 2 * a->N;
      r.ljx = lJ(a, 0);
      r.ljy = lJ(a, 1);
      r.ljz = lJ(a, 2);
      r.lrho = lrho(a);
      for (int q = 0; q < 3; ++q) {
        r.lE[q] = lE(a, q);
        r.lB[q] = lB(a, q);
      }
      r.P = a->work + 10 * a->pb[s];
      r.n = a->n[s];
      r.off = a->off + s * (a->N + 1);
      r.nx = a->nx;
      r.ny = a->ny;
      r.ae = a->ae[s];
      r.qd = a->qd[s];
      r.dtdx = a->dt / a->dx;
      r.dtdy = a->dt / a->dy;
      r.c = a->c;
      if (r.n > 0) {
        const dim3 grid((unsigned)((a->nx + TCX - 1) / TCX), (unsigned)a->ny);
        k_adj_push<<<grid, TCX * G, kBlkBytes, st>>>(r);
      }
      // at a checkpoint the kept exact state replaces the rebuilt one
      if (k % a->K == 0 && r.n > 0)
        k_adj_restore<<<blocks_for(r.n), 256, 0, st>>>(a->ckpt + 6 * a->ptot * (k / a->K) +
                                                           6 * a->pb[s],
                                                       r.n, r.P, a->slot + a->pb[s]);
    }
    EM2G_CUDA(cudaGetLastError());
    ++since;
  }
  // a recomputation moved the context: back to where the forward sweep
  // left it
  if (keep_from > 0 && (rc = reset_context(a, a->finfld, a->fin, a->it0 + a->steps, st)))
    return rc;
  EM2G_CUDA(cudaStreamSynchronize(st));
  a->swept = true;
  return EM2G_OK;
}

int em2g_adj_field_slots(em2g_adj *a, int nslots) {
  int rc = check_adj(a);
  if (rc) return rc;
  const int lo = std::min(a->K, a->max_steps);
  if (nslots < lo || nslots > a->max_steps)
    return fail(EM2G_ERR_RANGE, "field slots outside checkpoint .. max_steps");
  const int n = nslots;
  if (n != a->nhist) {
    EM2G_CUDA(cudaStreamSynchronize(a->ctx->stream));
    cudaFree(a->hist);
    a->hist = nullptr;
    a->nhist = 0;
    EM2G_CUDA(cudaMalloc((void **)&a->hist, sizeof(double) * 6 * a->N * n));
    a->nhist = n;
  }
  a->steps = 0;
  a->seeded = a->swept = false;
  return EM2G_OK;
}

int em2g_adj_keep_all_fields(em2g_adj *a, int on) {
  int rc = check_adj(a);
  if (rc) return rc;
  return em2g_adj_field_slots(a, on ? a->max_steps : std::min(a->K, a->max_steps));
}

int em2g_adj_get_field_slots(em2g_adj *a, int *nslots) {
  int rc = check_adj(a);
  if (rc) return rc;
  if (!nslots) return fail(EM2G_ERR_INVALID, "null pointer");
  *nslots = a->nhist;
  return EM2G_OK;
}

int em2g_adj_get_fields_device(em2g_adj *a, double *dev6) {
  int rc = check_adj(a);
  if (rc) return rc;
  if (!dev6) return fail(EM2G_ERR_INVALID, "null pointer");
  if (!a->swept) return fail(EM2G_ERR_INVALID, "run em2g_adj_backward first");
  EM2G_CUDA(cudaMemcpyAsync(dev6, a->g, sizeof(double) * 6 * a->N, cudaMemcpyDeviceToDevice,
                            a->ctx->stream));
  EM2G_CUDA(cudaStreamSynchronize(a->ctx->stream));
  return EM2G_OK;
}

static int unsort_out(em2g_adj *a, int isp, int first, double *o0, double *o1, double *o2,
                      double *o3, double *o4) {
  if (isp < 0 || isp >= a->nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  if (!o0 || !o1 || !o2 || !o3 || !o4) return fail(EM2G_ERR_INVALID, "null pointer");
  const int64_t n = a->n[isp];
  if (n > 0)
    k_adj_unsort<<<blocks_for(n), 256, 0, a->ctx->stream>>>(
        a->work + 10 * a->pb[isp], a->slot + a->pb[isp], n, first, o0, o1, o2, o3, o4);
  EM2G_CUDA(cudaGetLastError());
  EM2G_CUDA(cudaStreamSynchronize(a->ctx->stream));
  return EM2G_OK;
}

int em2g_adj_get_particles_device(em2g_adj *a, int isp, double *lx, double *ly, double *lux,
                                  double *luy, double *luz) {
  int rc = check_adj(a);
  if (rc) return rc;
  if (!a->swept) return fail(EM2G_ERR_INVALID, "run em2g_adj_backward first");
  return unsort_out(a, isp, 5, lx, ly, lux, luy, luz);
}

int em2g_adj_get_initial_particles_device(em2g_adj *a, int isp, double *x, double *y,
                                          double *ux, double *uy, double *uz) {
  int rc = check_adj(a);
  if (rc) return rc;
  if (a->steps < 1) return fail(EM2G_ERR_INVALID, "run em2g_adj_forward first");
  if (isp < 0 || isp >= a->nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  if (!x || !y || !ux || !uy || !uz) return fail(EM2G_ERR_INVALID, "null pointer");
  const int64_t n = a->n[isp];
  if (n > 0)
    k_adj_initial<<<blocks_for(n), 256, 0, a->ctx->stream>>>(a->ckpt + 6 * a->pb[isp], n, x, y,
                                                             ux, uy, uz);
  EM2G_CUDA(cudaGetLastError());
  EM2G_CUDA(cudaStreamSynchronize(a->ctx->stream));
  return EM2G_OK;
}

}  // extern "C"

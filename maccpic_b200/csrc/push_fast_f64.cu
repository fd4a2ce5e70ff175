// push_fast_f64.cu -- the FP64 fast path: move + curnt for particles that
// are grouped by cell, with the current accumulated in registers.
//
// Layout: each species' particles are ordered by the row-major key of the
// cell they occupied when the previous step began; cell k's particles sit at
// [off[k], off[k+1]) (sort.cu).  A group of G lanes owns one cell k and
// walks its particles G at a time (adjacent lanes read adjacent particles,
// adjacent groups adjacent cells).
//
// Per particle the arithmetic is the reference's (push_common.cuh, compiled
// with -fmad=false): gather + Boris (pic/move.f90), jm at the old position,
// move and wrap, rho and jp at the new one (pic/curnt.f90).  What changes is
// where the deposits go: a particle that is still in cell k adds its rho and
// J into a 49-value register block covering the nodes cell k can touch
// (Jx 4x3, Jy 3x4, Jz 3x3, rho 4x4); one that left cell k (about 1 % per
// step) deposits straight to global memory with atomics.  When the cell is
// done the G blocks are summed across the group with shuffles and added to
// the field arrays once -- about 49 atomics per cell instead of 63 per
// particle.  jm and jp are summed into the jxm/jym/jzm arrays (fields uses
// only jxm+jxp, pic/fields.f90:211-214); jxp/jyp/jzp stay zero on this path.
//
// Each particle is written to the other buffer at off_next[key] + (running
// count of key), key being its cell at the start of this step, and the
// cells of the new positions are counted for the next step's offsets: the
// counting sort rides along with the push.
#include "push_common.cuh"
#include "sort_common.cuh"

namespace em2g {
namespace {

using namespace f64;

constexpr int kThreads = 256;
constexpr int G = 4;  // lanes per cell

struct FastArgs {
  Scaled S;
  double *rho, *jx, *jy, *jz;  // deposit targets (jx = jxm, ...)
  const double *__restrict__ A;
  const int32_t *__restrict__ slotA;
  double *B;
  int32_t *slotB;
  const int32_t *__restrict__ offA;  // ranges of A by cell
  const int32_t *__restrict__ offB;  // ranges of B by cell (scan of cnt_cur)
  int32_t *cursor;                   // running counts into B
  int32_t *cnt_next;                 // counts of the new positions' cells
  int64_t cap;
  int nx, ny, nxg;
  double c, qd, dt, dx, dy, xn, yn;
  double *ake_partial;
};

// 4-entry weight vector of a node-staggered axis relative to the cell:
// offset o = i-1-cell in {0,1}; the three weights land at o, o+1, o+2.
__device__ __forceinline__ void spread4(int o, double m, double s, double p, double w[4]) {
  const bool lo = (o == 0);
  w[0] = lo ? m : 0.0;
  w[1] = lo ? s : m;
  w[2] = lo ? p : s;
  w[3] = lo ? 0.0 : p;
}

struct Block {
  double jx[4][3];  // rows y node (4), cols x half (3)
  double jy[3][4];  // rows y half (3), cols x node (4)
  double jz[3][3];  // rows y half, cols x half
  double rho[4][4];
};

// add one particle's J (at x, y in the group's cell) into the block
__device__ __forceinline__ void block_add_j(Block &b, double x, double y, int cx, int cy,
                                            double qd, double vx, double vy, double vz) {
  int ixh, ixn, iyh, iyn;
  double sxh, sxhp, sxhm, sxn, sxnp, sxnm, syh, syhp, syhm, syn, synp, synm;
  w_half(x, ixh, sxh, sxhp, sxhm);  // ixh = cx + 1
  w_node(x, ixn, sxn, sxnp, sxnm);  // ixn in {cx+1, cx+2}
  w_half(y, iyh, syh, syhp, syhm);
  w_node(y, iyn, syn, synp, synm);
  double wxn[4], wyn[4];
  spread4(ixn - 1 - cx, sxnm, sxn, sxnp, wxn);
  spread4(iyn - 1 - cy, synm, syn, synp, wyn);
  const double wxh[3] = {sxhm, sxh, sxhp}, wyh[3] = {syhm, syh, syhp};
  const double qx = qd * vx, qy = qd * vy, qz = qd * vz;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const double t = wyn[r] * qx;
#pragma unroll
    for (int k = 0; k < 3; ++k) b.jx[r][k] = __fma_rn(wxh[k], t, b.jx[r][k]);
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const double ty = wyh[r] * qy, tz = wyh[r] * qz;
#pragma unroll
    for (int k = 0; k < 4; ++k) b.jy[r][k] = __fma_rn(wxn[k], ty, b.jy[r][k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) b.jz[r][k] = __fma_rn(wxh[k], tz, b.jz[r][k]);
  }
}

__device__ __forceinline__ void block_add_rho(Block &b, double x, double y, int cx, int cy,
                                              double qd) {
  int ixn, iyn;
  double sxn, sxnp, sxnm, syn, synp, synm;
  w_node(x, ixn, sxn, sxnp, sxnm);
  w_node(y, iyn, syn, synp, synm);
  double wxn[4], wyn[4];
  spread4(ixn - 1 - cx, sxnm, sxn, sxnp, wxn);
  spread4(iyn - 1 - cy, synm, syn, synp, wyn);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const double t = wyn[r] * qd;
#pragma unroll
    for (int k = 0; k < 4; ++k) b.rho[r][k] = __fma_rn(wxn[k], t, b.rho[r][k]);
  }
}

__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// flush entry e of the block (all lanes hold the group sum) if it is mine
__device__ __forceinline__ void flush_one(double *A, int nxg, int ix, int iy, double v, int e,
                                          int gl) {
  if ((e % G) == gl && v != 0.0) atomicAdd(A + (int64_t)iy * nxg + ix, v);
}

__global__ void __launch_bounds__(kThreads) k_push_cells_f64(FastArgs a) {
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const int64_t cell = ((int64_t)blockIdx.x * kThreads + threadIdx.x) / G;
  const int64_t ncell = (int64_t)a.nx * a.ny;
  const bool valid = cell < ncell;
  const int cx = valid ? (int)(cell % a.nx) : 0;
  const int cy = valid ? (int)(cell / a.nx) : 0;
  const int32_t beg = valid ? a.offA[cell] : 0;
  const int32_t end = valid ? a.offA[cell + 1] : 0;
  const int64_t cap = a.cap;
  const int nxg = a.nxg;

  Block b;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      b.rho[r][k] = 0.0;
      if (k < 3) b.jx[r][k] = 0.0;
      if (r < 3) b.jy[r][k] = 0.0;
      if (r < 3 && k < 3) b.jz[r][k] = 0.0;
    }
  double akel = 0.0;

  for (int32_t i = beg + gl;; i += G) {
    const bool active = i < end;
    const unsigned am = __ballot_sync(0xffffffffu, active);
    if (am == 0u) break;
    if (active) {
    double x = a.A[i], y = a.A[cap + i];
    double vx = a.A[2 * cap + i], vy = a.A[3 * cap + i], vz = a.A[4 * cap + i];
    double g = a.A[5 * cap + i];
    const int32_t slot = a.slotA[i];
    const int key_cur = cell_key(x, y, a.nx, a.ny);
    const bool in_old = ((int)x == cx) && ((int)y == cy);
    akel += gather_boris(a.S, nxg, a.c, x, y, vx, vy, vz, g) - 1.0;
    // jm at the old position
    if (in_old)
      block_add_j(b, x, y, cx, cy, a.qd, vx, vy, vz);
    else
      deposit_j_atomic(a.jx, a.jy, a.jz, nxg, x, y, a.qd, vx, vy, vz);
    move_wrap(x, y, vx, vy, a.dt, a.dx, a.dy, a.xn, a.yn);
    // rho and jp at the new position
    const bool in_new = ((int)x == cx) && ((int)y == cy);
    if (in_new) {
      block_add_rho(b, x, y, cx, cy, a.qd);
      block_add_j(b, x, y, cx, cy, a.qd, vx, vy, vz);
    } else {
      deposit_rho_atomic(a.rho, nxg, x, y, a.qd);
      deposit_j_atomic(a.jx, a.jy, a.jz, nxg, x, y, a.qd, vx, vy, vz);
    }
    // write back, grouped by the cell of the start of this step
    const int64_t pos = (int64_t)a.offB[key_cur] + agg_atomic_add(a.cursor, key_cur, am);
    a.B[pos] = x;
    a.B[cap + pos] = y;
    a.B[2 * cap + pos] = vx;
    a.B[3 * cap + pos] = vy;
    a.B[4 * cap + pos] = vz;
    a.B[5 * cap + pos] = g;
    a.slotB[pos] = slot;
    // counts of the cells the particles now occupy (next step's offsets)
    agg_atomic_add(a.cnt_next, cell_key(x, y, a.nx, a.ny), am);
    }
  }

  // sum the group's blocks and add them to the arrays once
  if (__any_sync(0xffffffffu, valid && end > beg)) {
    int e = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double v = group_sum(b.rho[r][k]);
        if (valid) flush_one(a.rho, nxg, cx + k, cy + r, v, e, gl);
        ++e;
      }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double v = group_sum(b.jx[r][k]);
        if (valid) flush_one(a.jx, nxg, cx + k, cy + r, v, e, gl);
        ++e;
      }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double v = group_sum(b.jy[r][k]);
        if (valid) flush_one(a.jy, nxg, cx + k, cy + r, v, e, gl);
        ++e;
      }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double v = group_sum(b.jz[r][k]);
        if (valid) flush_one(a.jz, nxg, cx + k, cy + r, v, e, gl);
        ++e;
      }
  }

  // block sum of (gamma - 1) in a fixed order
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) akel += __shfl_down_sync(0xffffffffu, akel, o);
  if (lane == 0) red[threadIdx.x >> 5] = akel;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) a.ake_partial[blockIdx.x] = v;
  }
}

}  // namespace

int launch_push_cells_f64(em2g_ctx *c, int isp) {
  Species &S = c->sp[isp];
  const int64_t w = c->g.w;
  const double *sc = c->scaled + (int64_t)isp * 6 * w;
  FastArgs a;
  a.S = Scaled{sc, sc + w, sc + 2 * w, sc + 3 * w, sc + 4 * w, sc + 5 * w};
  a.rho = c->fld + EM2G_RHO * w;
  a.jx = c->fld + EM2G_JXM * w;
  a.jy = c->fld + EM2G_JYM * w;
  a.jz = c->fld + EM2G_JZM * w;
  a.A = S.part;
  a.slotA = S.slot;
  a.B = S.part_alt;
  a.slotB = S.slot_alt;
  a.offA = S.off;
  a.offB = S.off_alt;
  a.cursor = S.cursor;
  a.cnt_next = S.cnt_alt;
  a.cap = S.cap;
  a.nx = c->g.nx;
  a.ny = c->g.ny;
  a.nxg = c->g.nxg;
  a.c = c->P.c;
  a.qd = c->P.q[isp] * c->P.dn[isp] / (c->P.dx * c->P.dy);  // pic/curnt.f90:41
  a.dt = c->P.dt;
  a.dx = c->P.dx;
  a.dy = c->P.dy;
  a.xn = (double)c->P.nx;
  a.yn = (double)c->P.ny;
  a.ake_partial = c->red;
  const int64_t nb64 = (c->ncell * G + kThreads - 1) / kThreads;
  if (nb64 > c->red_blocks) return fail(EM2G_ERR_RANGE, "grid exceeds reduction scratch");
  const int nb = (int)nb64;
  // offsets of B from the counts of the current cells; fresh counters
  int rc = scan_cells(c, S.cnt, S.off_alt);
  if (rc) return rc;
  EM2G_CUDA(cudaMemsetAsync(S.cursor, 0, sizeof(int32_t) * c->ncell, c->stream));
  EM2G_CUDA(cudaMemsetAsync(S.cnt_alt, 0, sizeof(int32_t) * c->ncell, c->stream));
  if ((rc = timing_begin(c))) return rc;
  k_push_cells_f64<<<nb, kThreads, 0, c->stream>>>(a);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  if ((rc = timing_end(c))) return rc;
  // B is the new A; its ranges and the current-cell counts move along
  std::swap(S.part, S.part_alt);
  std::swap(S.slot, S.slot_alt);
  std::swap(S.off, S.off_alt);
  std::swap(S.cnt, S.cnt_alt);
  return launch_ake_finish(c, isp, nb);
}

}  // namespace em2g

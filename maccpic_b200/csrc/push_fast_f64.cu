// push_fast_f64.cu -- the FP64 fast path: move + curnt for particles that
// are grouped by cell, with the current accumulated in registers.
//
// Layout: each species' particles are ordered by the row-major key of the
// cell they occupied when the previous step began; cell k's particles sit at
// [off[k], off[k+1]) (sort.cu).  A CTA of 128 threads owns a row segment of
// 32 cells; a group of 4 lanes owns one cell and walks its particles 4 at a
// time.  The scaled E and B the segment's particles can touch are staged once
// in shared memory as (E, B) double pairs of the three staggerings.
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

constexpr int G = 4;   // lanes per cell
constexpr int WY = 6;  // window rows: array y0-1 .. y0+4

struct FastArgs {
  const double2 *__restrict__ ebx, *__restrict__ ebz, *__restrict__ eby;
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

// pic/move.f90:95-97 on an (E, B) pair: the nine products summed in the
// reference's order (ix,iy) (ix,iyp) (ix,iym) (ixp,iy) (ixp,iyp) (ixp,iym)
// (ixm,iy) (ixm,iyp) (ixm,iym); `m` points at node (ix-1, iy-1)
__device__ __forceinline__ double2 gather_pair(const double2 *m, int pitch, const W9 &w) {
  const double2 *r0 = m + pitch + 1;  // (ix, iy)
  const double2 a = r0[0], b = r0[pitch], c = r0[-pitch], d = r0[1], e = r0[pitch + 1],
                f = r0[-pitch + 1], g = r0[-1], h = r0[pitch - 1], k = r0[-pitch - 1];
  double2 o;
  o.x = a.x * w.q + b.x * w.qyp + c.x * w.qym + d.x * w.qxp + e.x * w.qxpyp + f.x * w.qxpym +
        g.x * w.qxm + h.x * w.qxmyp + k.x * w.qxmym;
  o.y = a.y * w.q + b.y * w.qyp + c.y * w.qym + d.y * w.qxp + e.y * w.qxpyp + f.y * w.qxpym +
        g.y * w.qxm + h.y * w.qxmyp + k.y * w.qxmym;
  return o;
}

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
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  return v;
}

// flush entry e of the block (all lanes hold the group sum) if it is mine
__device__ __forceinline__ void flush_one(double *A, int nxg, int ix, int iy, double v, int e,
                                          int gl) {
  if ((e & (G - 1)) == gl && v != 0.0) atomicAdd(A + (int64_t)iy * nxg + ix, v);
}

// Asynchronous copies global -> shared (cp.async): a lane's next particle
// is fetched into shared memory while the current one runs (the kernel has
// no registers left to hold it), one commit group per particle.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// TCX cells per CTA (a row segment), MINB: CTAs per SM the register
// allocation must allow (the autotuner's two knobs)
template <int TCX, int MINB>
__global__ void __launch_bounds__(TCX * G, MINB) k_push_cells_f64(FastArgs a) {
  constexpr int kThreads = TCX * G;
  constexpr int WX = TCX + 5;  // window columns: array x0-1 .. x0+TCX+3
  __shared__ double2 win[3][WY][WX];
  // each lane's next particle (x, y, vx, vy, vz, gamma; slot), two buffers
  __shared__ double pf[2][6][kThreads];
  __shared__ int32_t pfs[2][kThreads];
  const int nx = a.nx, ny = a.ny, nxg = a.nxg;
  const int x0 = blockIdx.x * TCX, y0 = blockIdx.y;
  for (int t = threadIdx.x; t < 3 * WY * WX; t += kThreads) {
    const int comp = t / (WY * WX), r = (t / WX) % WY, col = t % WX;
    const int gx = x0 - 1 + col, gy = y0 - 1 + r;
    double2 v = make_double2(0.0, 0.0);
    if (gx >= 0 && gx <= nx + 2 && gy >= 0 && gy <= ny + 2) {
      const double2 *src = comp == 0 ? a.ebx : (comp == 1 ? a.ebz : a.eby);
      v = src[(int64_t)gy * nxg + gx];
    }
    win[comp][r][col] = v;
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, gl = lane & (G - 1);
  const int cx = x0 + (int)(threadIdx.x / G), cy = y0;
  const bool valid = cx < nx;
  const int64_t cell = (int64_t)cy * nx + cx;
  const int32_t beg = valid ? a.offA[cell] : 0;
  const int32_t end = valid ? a.offA[cell + 1] : 0;
  const int64_t cap = a.cap;
  const unsigned gmask = 0xFu << (lane & ~(G - 1));

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
  int stay_new = 0;
  int home_count = 0;  // particles of this group written to the front of cell k

  const int tid = threadIdx.x;
  auto fetch = [&](int buf, int32_t j) {
#pragma unroll
    for (int c = 0; c < 6; ++c) cp_async8(&pf[buf][c][tid], a.A + (int64_t)c * cap + j);
    cp_async4(&pfs[buf][tid], a.slotA + j);
  };
  if (beg + gl < end) fetch(0, beg + gl);
  cp_async_commit();
  int buf = 0;
  for (int32_t i = beg + gl;; i += G) {
    const bool active = i < end;
    const unsigned am = __ballot_sync(0xffffffffu, active);
    if (am == 0u) break;
    if (i + G < end) fetch(buf ^ 1, i + G);
    cp_async_commit();
    cp_async_wait<1>();  // this particle's group (all but the newest) has landed
    if (active) {
      double x = pf[buf][0][tid], y = pf[buf][1][tid];
      double vx = pf[buf][2][tid], vy = pf[buf][3][tid], vz = pf[buf][4][tid];
      double g = pf[buf][5][tid];
      const int32_t slot = pfs[buf][tid];
      const int key_cur = cell_key(x, y, nx, ny);
      const int pcx = (int)x, pcy = (int)y;  // the particle's cell, unwrapped
      const bool in_old = (pcx == cx) && (pcy == cy);
      // gather + Boris (pic/move.f90:76-203), fields from the shared window
      // when the stencil lies inside it, else from global memory
      {
        int ixh, ixn, iyh, iyn;
        double sxh, sxhp, sxhm, sxn, sxnp, sxnm, syh, syhp, syhm, syn, synp, synm;
        w_half(x, ixh, sxh, sxhp, sxhm);
        w_node(y, iyn, syn, synp, synm);
        w_half(y, iyh, syh, syhp, syhm);
        w_node(x, ixn, sxn, sxnp, sxnm);
        const W9 wxn = weights(sxh, sxhp, sxhm, syn, synp, synm);  // Ex, Bx
        const W9 wzz = weights(sxh, sxhp, sxhm, syh, syhp, syhm);  // Ez, Bz
        const W9 wyy = weights(sxn, sxnp, sxnm, syh, syhp, syhm);  // Ey, By
        double2 pex, pez, pey;
        if (pcx >= x0 - 1 && pcx <= x0 + TCX && pcy >= y0 - 1 && pcy <= y0 + 1) {
          pex = gather_pair(&win[0][iyn - y0][ixh - x0], WX, wxn);
          pez = gather_pair(&win[1][iyh - y0][ixh - x0], WX, wzz);
          pey = gather_pair(&win[2][iyh - y0][ixn - x0], WX, wyy);
        } else {
          pex = gather_pair(a.ebx + (int64_t)(iyn - 1) * nxg + ixh - 1, nxg, wxn);
          pez = gather_pair(a.ebz + (int64_t)(iyh - 1) * nxg + ixh - 1, nxg, wzz);
          pey = gather_pair(a.eby + (int64_t)(iyh - 1) * nxg + ixn - 1, nxg, wyy);
        }
        const double aexpt = pex.x, aeypt = pey.x, aezpt = pez.x;
        double abxpt = pex.y, abypt = pey.y, abzpt = pez.y;
        double gvxs = vx * g + aexpt;
        double gvys = vy * g + aeypt;
        double gvzs = vz * g + aezpt;
        double gm = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
        akel += gm - 1.0;
        const double dcg = 1.0 / (a.c * gm);
        abxpt = dcg * abxpt;
        abypt = dcg * abypt;
        abzpt = dcg * abzpt;
        const double vvx = gvxs + gvys * abzpt - gvzs * abypt;
        const double vvy = gvys + gvzs * abxpt - gvxs * abzpt;
        const double vvz = gvzs + gvxs * abypt - gvys * abxpt;
        const double f = 2.0 / (1.0 + abxpt * abxpt + abypt * abypt + abzpt * abzpt);
        abxpt = f * abxpt;
        abypt = f * abypt;
        abzpt = f * abzpt;
        gvxs = gvxs + vvy * abzpt - vvz * abypt + aexpt;
        gvys = gvys + vvz * abxpt - vvx * abzpt + aeypt;
        gvzs = gvzs + vvx * abypt - vvy * abxpt + aezpt;
        gm = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
        g = gm;
        vx = gvxs / gm;
        vy = gvys / gm;
        vz = gvzs / gm;
      }
      // jm at the old position
      if (in_old)
        block_add_j(b, x, y, cx, cy, a.qd, vx, vy, vz);
      else
        deposit_j_atomic(a.jx, a.jy, a.jz, nxg, x, y, a.qd, vx, vy, vz);
      move_wrap(x, y, vx, vy, a.dt, a.dx, a.dy, a.xn, a.yn);
      // rho and jp at the new position
      if (((int)x == cx) && ((int)y == cy)) {
        block_add_rho(b, x, y, cx, cy, a.qd);
        block_add_j(b, x, y, cx, cy, a.qd, vx, vy, vz);
        ++stay_new;
      } else {
        deposit_rho_atomic(a.rho, nxg, x, y, a.qd);
        deposit_j_atomic(a.jx, a.jy, a.jz, nxg, x, y, a.qd, vx, vy, vz);
        atomicAdd(a.cnt_next + cell_key(x, y, nx, ny), 1);
      }
      const bool home = key_cur == (int)cell;
      // write back grouped by the cell of the start of this step: particles
      // that started it in cell k take the next slots from the front of k's
      // segment in processing order (a running count per group, no atomics);
      // the few that came from another cell's range fill it from the back
      const unsigned inm = __ballot_sync(am, home) & gmask;
      int64_t pos;
      if (home)
        pos = (int64_t)a.offB[key_cur] + home_count + __popc(inm & ((1u << lane) - 1u));
      else
        pos = (int64_t)a.offB[key_cur + 1] - 1 - atomicAdd(a.cursor + key_cur, 1);
      home_count += __popc(inm);
      a.B[pos] = x;
      a.B[cap + pos] = y;
      a.B[2 * cap + pos] = vx;
      a.B[3 * cap + pos] = vy;
      a.B[4 * cap + pos] = vz;
      a.B[5 * cap + pos] = g;
      a.slotB[pos] = slot;
    }
    buf ^= 1;
  }
  cp_async_wait<0>();

  // this cell's count of new positions, then the register blocks
  int stay = stay_new;
  stay += __shfl_xor_sync(0xffffffffu, stay, 1);
  stay += __shfl_xor_sync(0xffffffffu, stay, 2);
  if (valid && gl == 0 && stay > 0) atomicAdd(a.cnt_next + cell, stay);
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
  // per-warp partial of sum(gamma - 1); no block barrier at the end
  for (int o = 16; o > 0; o >>= 1) akel += __shfl_down_sync(0xffffffffu, akel, o);
  const int64_t blk = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
  if (lane == 0) a.ake_partial[blk * (kThreads / 32) + (threadIdx.x >> 5)] = akel;
}

struct Variant64 {
  const char *name;
  int tcx;
  void (*kernel)(FastArgs);
};
const Variant64 kVariants64[] = {
    {"f64 tcx32 minb1", 32, k_push_cells_f64<32, 1>},
    {"f64 tcx32 minb2", 32, k_push_cells_f64<32, 2>},
    {"f64 tcx64 minb1", 64, k_push_cells_f64<64, 1>},
};

// pic/move.f90:52-64: E and B times ae = 0.5*qm*dt/c (plus tx/ty), stored
// as (E, B) pairs of the three staggerings
__global__ void k_prescale_pairs(const double *__restrict__ fld, double2 *__restrict__ s,
                                 int64_t w, double ae, double tx, double ty) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= w) return;
  s[k] = make_double2(ae * fld[EM2G_EX * w + k], ae * fld[EM2G_BX * w + k] + tx);
  s[w + k] = make_double2(ae * fld[EM2G_EZ * w + k], ae * fld[EM2G_BZ * w + k]);
  s[2 * w + k] = make_double2(ae * fld[EM2G_EY * w + k], ae * fld[EM2G_BY * w + k] + ty);
}

}  // namespace

int num_variants_f64() { return (int)(sizeof(kVariants64) / sizeof(kVariants64[0])); }
const char *variant_name_f64(int v) { return kVariants64[v].name; }

int launch_push_cells_f64(em2g_ctx *c, int isp) {
  Species &S = c->sp[isp];
  const int64_t w = c->g.w;
  double2 *sc = reinterpret_cast<double2 *>(c->scaled + (int64_t)isp * 6 * w);
  const double ae = 0.5 * c->P.qm[isp] * c->P.dt / c->P.c;  // pic/move.f90:42
  k_prescale_pairs<<<(unsigned)((w + 255) / 256), 256, 0, c->stream>>>(c->fld, sc, w, ae,
                                                                        c->P.tx[isp],
                                                                        c->P.ty[isp]);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  FastArgs a;
  a.ebx = sc;
  a.ebz = sc + w;
  a.eby = sc + 2 * w;
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
  const Variant64 &V = kVariants64[c->variant < num_variants_f64() ? c->variant : 0];
  const int threads = V.tcx * G;
  const dim3 grid((unsigned)((c->g.nx + V.tcx - 1) / V.tcx), (unsigned)c->g.ny);
  const int64_t nparts = (int64_t)grid.x * grid.y * (threads / 32);
  if (nparts > c->red_blocks) return fail(EM2G_ERR_RANGE, "grid exceeds reduction scratch");
  // offsets of B from the counts of the current cells; fresh counters
  int rc = scan_cells(c, S.cnt, S.off_alt);
  if (rc) return rc;
  EM2G_CUDA(cudaMemsetAsync(S.cursor, 0, sizeof(int32_t) * c->ncell, c->stream));
  EM2G_CUDA(cudaMemsetAsync(S.cnt_alt, 0, sizeof(int32_t) * c->ncell, c->stream));
  if ((rc = timing_begin(c))) return rc;
  V.kernel<<<grid, threads, 0, c->stream>>>(a);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  if ((rc = timing_end(c))) return rc;
  // B is the new A; its ranges and the current-cell counts move along
  std::swap(S.part, S.part_alt);
  std::swap(S.slot, S.slot_alt);
  std::swap(S.off, S.off_alt);
  std::swap(S.cnt, S.cnt_alt);
  return launch_ake_finish(c, isp, (int)nparts);
}

}  // namespace em2g

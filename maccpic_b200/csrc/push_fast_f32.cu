// push_fast_f32.cu -- the mixed-precision path: FP32 particles, gather,
// Boris, deposit; FP64 only for the kinetic-energy reduction.
//
// Particle layout (per species, SoA, 24 B per particle): the cell is not
// stored -- particles are grouped by cell (row-major key iy*nx+ix), cell k's
// particles at [off[k], off[k+1]), and each stores its position relative to
// that cell, xr = x - cx, yr = y - cy, as FP32 in (-1, 2) (a particle may
// have crossed into a neighbour since the last regrouping), plus the
// momentum per unit mass u = gamma*v (FP32) and its int32 slot.  Positions
// relative to a cell keep ~1e-7 cells of resolution on any grid size, where
// an absolute FP32 position on a 4096-cell axis would keep only ~5e-4.
//
// The step follows em2's move and curnt (pic/move.f90, pic/curnt.f90) in
// FP32 with the same quadratic weights, written in the cell-relative
// variable f = x - cx:
//   cell-centred nodes (x index cx+1): s = 3/4 - (f-1/2)^2, s+ = f^2/2,
//                                      s- = (1-f)^2/2
//   integer nodes (x index cx+1+[f>=1/2]), h = f - [f>=1/2]:
//                                      s = 3/4 - h^2, s+ = (1/2+h)^2/2,
//                                      s- = (1/2-h)^2/2
// and the relativistic Boris rotation on u.  The cell-group register
// deposit and the fused counting sort are those of push_fast_f64.cu with
// G = 8 lanes per cell (8 FP32 values = one 32-byte sector).
#include "em2g_internal.cuh"
#include "sort_common.cuh"

namespace em2g {
namespace {

constexpr int kThreads = 256;
constexpr int G = 8;

struct Args32 {
  const float *__restrict__ aex, *__restrict__ aey, *__restrict__ aez;
  const float *__restrict__ abx, *__restrict__ aby, *__restrict__ abz;
  float *rho, *jx, *jy, *jz;
  const float *__restrict__ A;  // xr, yr, ux, uy, uz
  const int32_t *__restrict__ slotA;
  float *B;
  int32_t *slotB;
  const int32_t *__restrict__ offA;
  const int32_t *__restrict__ offB;
  int32_t *cursor, *cnt_next;
  int64_t cap;
  int nx, ny, nxg;
  float qd, dtdx, dtdy, c;
  double *ake_partial;
};

struct Wts {
  int i;           // array index of the middle node
  float m, s, p;   // weights of nodes i-1, i, i+1
};

__device__ __forceinline__ Wts half_w(int c, float f) {
  const float d = f - 0.5f;
  const float e = 1.0f - f;
  return Wts{c + 1, 0.5f * e * e, 0.75f - d * d, 0.5f * f * f};
}
__device__ __forceinline__ Wts node_w(int c, float f) {
  const int up = f >= 0.5f ? 1 : 0;
  const float h = f - (float)up;
  const float a = 0.5f - h, b = 0.5f + h;
  return Wts{c + 1 + up, 0.5f * a * a, 0.75f - h * h, 0.5f * b * b};
}

__device__ __forceinline__ float gather9(const float *__restrict__ A, int nxg, const Wts &wx,
                                         const Wts &wy) {
  const float *r0 = A + (int64_t)wy.i * nxg + wx.i;
  const float *rm = r0 - nxg, *rp = r0 + nxg;
  const float row_m = __ldg(rm - 1) * wx.m + __ldg(rm) * wx.s + __ldg(rm + 1) * wx.p;
  const float row_0 = __ldg(r0 - 1) * wx.m + __ldg(r0) * wx.s + __ldg(r0 + 1) * wx.p;
  const float row_p = __ldg(rp - 1) * wx.m + __ldg(rp) * wx.s + __ldg(rp + 1) * wx.p;
  return row_m * wy.m + row_0 * wy.s + row_p * wy.p;
}

__device__ __forceinline__ void scatter9(float *A, int nxg, const Wts &wx, const Wts &wy,
                                         float q) {
  float *r0 = A + (int64_t)wy.i * nxg + wx.i;
  float *rm = r0 - nxg, *rp = r0 + nxg;
  const float qm = wy.m * q, qs = wy.s * q, qp = wy.p * q;
  atomicAdd(rm - 1, wx.m * qm);
  atomicAdd(rm, wx.s * qm);
  atomicAdd(rm + 1, wx.p * qm);
  atomicAdd(r0 - 1, wx.m * qs);
  atomicAdd(r0, wx.s * qs);
  atomicAdd(r0 + 1, wx.p * qs);
  atomicAdd(rp - 1, wx.m * qp);
  atomicAdd(rp, wx.s * qp);
  atomicAdd(rp + 1, wx.p * qp);
}

struct Block32 {
  float jx[4][3], jy[3][4], jz[3][3], rho[4][4];
};

__device__ __forceinline__ void spread4(const Wts &w, int c, float o[4]) {
  const bool lo = (w.i == c + 1);
  o[0] = lo ? w.m : 0.0f;
  o[1] = lo ? w.s : w.m;
  o[2] = lo ? w.p : w.s;
  o[3] = lo ? 0.0f : w.p;
}

// J of one particle at local offsets (fx, fy) of the group's cell (cx, cy)
__device__ __forceinline__ void block_add_j(Block32 &b, int cx, int cy, float fx, float fy,
                                            float qx, float qy, float qz) {
  const Wts hx = half_w(cx, fx), hy = half_w(cy, fy), nxw = node_w(cx, fx), nyw = node_w(cy, fy);
  float wxn[4], wyn[4];
  spread4(nxw, cx, wxn);
  spread4(nyw, cy, wyn);
  const float wxh[3] = {hx.m, hx.s, hx.p}, wyh[3] = {hy.m, hy.s, hy.p};
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const float t = wyn[r] * qx;
#pragma unroll
    for (int k = 0; k < 3; ++k) b.jx[r][k] = fmaf(wxh[k], t, b.jx[r][k]);
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float ty = wyh[r] * qy, tz = wyh[r] * qz;
#pragma unroll
    for (int k = 0; k < 4; ++k) b.jy[r][k] = fmaf(wxn[k], ty, b.jy[r][k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) b.jz[r][k] = fmaf(wxh[k], tz, b.jz[r][k]);
  }
}

__device__ __forceinline__ void block_add_rho(Block32 &b, int cx, int cy, float fx, float fy,
                                              float q) {
  float wxn[4], wyn[4];
  spread4(node_w(cx, fx), cx, wxn);
  spread4(node_w(cy, fy), cy, wyn);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const float t = wyn[r] * q;
#pragma unroll
    for (int k = 0; k < 4; ++k) b.rho[r][k] = fmaf(wxn[k], t, b.rho[r][k]);
  }
}

__device__ __forceinline__ void deposit_j_atomic(const Args32 &a, int cx, int cy, float fx,
                                                 float fy, float qx, float qy, float qz) {
  const Wts hx = half_w(cx, fx), hy = half_w(cy, fy), nxw = node_w(cx, fx), nyw = node_w(cy, fy);
  scatter9(a.jx, a.nxg, hx, nyw, qx);
  scatter9(a.jz, a.nxg, hx, hy, qz);
  scatter9(a.jy, a.nxg, nxw, hy, qy);
}

__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
  for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void flush_one(float *A, int nxg, int ix, int iy, float v, int e,
                                          int gl) {
  if ((e % G) == gl && v != 0.0f) atomicAdd(A + (int64_t)iy * nxg + ix, v);
}

__device__ __forceinline__ int floor_small(float f) { return f < 0.0f ? -1 : (f >= 1.0f ? 1 : 0); }

__global__ void __launch_bounds__(kThreads) k_push_cells_f32(Args32 a) {
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const int64_t cell = ((int64_t)blockIdx.x * kThreads + threadIdx.x) / G;
  const int64_t ncell = (int64_t)a.nx * a.ny;
  const bool valid = cell < ncell;
  const int kx = valid ? (int)(cell % a.nx) : 0;
  const int ky = valid ? (int)(cell / a.nx) : 0;
  const int32_t beg = valid ? a.offA[cell] : 0;
  const int32_t end = valid ? a.offA[cell + 1] : 0;
  const int64_t cap = a.cap;
  const int nxg = a.nxg, nx = a.nx, ny = a.ny;

  Block32 b;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      b.rho[r][k] = 0.0f;
      if (k < 3) b.jx[r][k] = 0.0f;
      if (r < 3) b.jy[r][k] = 0.0f;
      if (r < 3 && k < 3) b.jz[r][k] = 0.0f;
    }
  double akel = 0.0;

  for (int32_t i = beg + gl;; i += G) {
    const bool active = i < end;
    const unsigned am = __ballot_sync(0xffffffffu, active);
    if (am == 0u) break;
    if (active) {
      const float xr = a.A[i], yr = a.A[cap + i];
      float ux = a.A[2 * cap + i], uy = a.A[3 * cap + i], uz = a.A[4 * cap + i];
      const int32_t slot = a.slotA[i];
      // the cell the particle is in now, and its offsets in that cell
      const int ox = floor_small(xr), oy = floor_small(yr);
      int cx = kx + ox, cy = ky + oy;
      cx = cx < 0 ? cx + nx : (cx >= nx ? cx - nx : cx);
      cy = cy < 0 ? cy + ny : (cy >= ny ? cy - ny : cy);
      const float fx = xr - (float)ox, fy = yr - (float)oy;
      const int key_cur = cy * nx + cx;
      // gather (pic/move.f90:76-148) with the scaled fields
      const Wts hx = half_w(cx, fx), hy = half_w(cy, fy), nxw = node_w(cx, fx),
                nyw = node_w(cy, fy);
      const float ex = gather9(a.aex, nxg, hx, nyw), bx = gather9(a.abx, nxg, hx, nyw);
      const float ez = gather9(a.aez, nxg, hx, hy), bz = gather9(a.abz, nxg, hx, hy);
      const float ey = gather9(a.aey, nxg, nxw, hy), by = gather9(a.aby, nxg, nxw, hy);
      // relativistic Boris on u (pic/move.f90:176-203)
      float gx = ux + ex, gy = uy + ey, gz = uz + ez;
      const float gm = sqrtf(1.0f + gx * gx + gy * gy + gz * gz);
      akel += (double)gm - 1.0;
      const float dcg = 1.0f / (a.c * gm);
      float tx = dcg * bx, ty = dcg * by, tz = dcg * bz;
      const float vvx = gx + gy * tz - gz * ty;
      const float vvy = gy + gz * tx - gx * tz;
      const float vvz = gz + gx * ty - gy * tx;
      const float f2 = 2.0f / (1.0f + tx * tx + ty * ty + tz * tz);
      tx *= f2;
      ty *= f2;
      tz *= f2;
      ux = gx + vvy * tz - vvz * ty + ex;
      uy = gy + vvz * tx - vvx * tz + ey;
      uz = gz + vvx * ty - vvy * tx + ez;
      const float ginv = 1.0f / sqrtf(1.0f + ux * ux + uy * uy + uz * uz);
      const float vx = ux * ginv, vy = uy * ginv, vz = uz * ginv;
      const float qx = a.qd * vx, qy = a.qd * vy, qz = a.qd * vz;
      // jm at the old position (pic/curnt.f90:53-132)
      const bool in_old = (cx == kx) && (cy == ky);
      if (in_old)
        block_add_j(b, cx, cy, fx, fy, qx, qy, qz);
      else
        deposit_j_atomic(a, cx, cy, fx, fy, qx, qy, qz);
      // move (pic/curnt.f90:181-194), relative to the start cell
      const float mx = fmaf(vx, a.dtdx, fx), my = fmaf(vy, a.dtdy, fy);
      const int nox = floor_small(mx), noy = floor_small(my);
      int ncx = cx + nox, ncy = cy + noy;
      ncx = ncx < 0 ? ncx + nx : (ncx >= nx ? ncx - nx : ncx);
      ncy = ncy < 0 ? ncy + ny : (ncy >= ny ? ncy - ny : ncy);
      const float nfx = mx - (float)nox, nfy = my - (float)noy;
      // rho and jp at the new position (pic/curnt.f90:197-303)
      const bool in_new = (ncx == kx) && (ncy == ky);
      if (in_new) {
        block_add_rho(b, ncx, ncy, nfx, nfy, a.qd);
        block_add_j(b, ncx, ncy, nfx, nfy, qx, qy, qz);
      } else {
        const Wts nx2 = node_w(ncx, nfx), ny2 = node_w(ncy, nfy);
        scatter9(a.rho, nxg, nx2, ny2, a.qd);
        deposit_j_atomic(a, ncx, ncy, nfx, nfy, qx, qy, qz);
      }
      // write back grouped by the start cell, position relative to it
      const int64_t pos = (int64_t)a.offB[key_cur] + agg_atomic_add(a.cursor, key_cur, am);
      a.B[pos] = mx;
      a.B[cap + pos] = my;
      a.B[2 * cap + pos] = ux;
      a.B[3 * cap + pos] = uy;
      a.B[4 * cap + pos] = uz;
      a.slotB[pos] = slot;
      agg_atomic_add(a.cnt_next, ncy * nx + ncx, am);
    }
  }

  if (__any_sync(0xffffffffu, valid && end > beg)) {
    int e = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float v = group_sum(b.rho[r][k]);
        if (valid) flush_one(a.rho, nxg, kx + k, ky + r, v, e, gl);
        ++e;
      }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float v = group_sum(b.jx[r][k]);
        if (valid) flush_one(a.jx, nxg, kx + k, ky + r, v, e, gl);
        ++e;
      }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float v = group_sum(b.jy[r][k]);
        if (valid) flush_one(a.jy, nxg, kx + k, ky + r, v, e, gl);
        ++e;
      }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float v = group_sum(b.jz[r][k]);
        if (valid) flush_one(a.jz, nxg, kx + k, ky + r, v, e, gl);
        ++e;
      }
  }

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

// E and B times ae = 0.5*qm*dt/c into FP32 copies (pic/move.f90:52-64)
__global__ void k_prescale_f32(const float *__restrict__ fld, float *__restrict__ s, int64_t w,
                               float ae, float tx, float ty) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= w) return;
  s[k] = ae * fld[EM2G_EX * w + k];
  s[w + k] = ae * fld[EM2G_EY * w + k];
  s[2 * w + k] = ae * fld[EM2G_EZ * w + k];
  s[3 * w + k] = ae * fld[EM2G_BX * w + k] + tx;
  s[4 * w + k] = ae * fld[EM2G_BY * w + k] + ty;
  s[5 * w + k] = ae * fld[EM2G_BZ * w + k];
}

// FP64 (x, y, vx, vy, vz, gamma) staging -> histogram of cells
__global__ void k_hist64(const double *__restrict__ st, int64_t n, int nx, int ny,
                         int32_t *cnt) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = j < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  agg_atomic_add(cnt, cell_key(st[j], st[n + j], nx, ny), am);
}

// FP64 staging -> cell-grouped FP32 layout (slot j keeps its slot number)
__global__ void k_scatter_to_f32(const double *__restrict__ st, int64_t n, int nx, int ny,
                                 const int32_t *__restrict__ off, int32_t *cursor, float *P,
                                 int32_t *slot, int64_t cap) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = j < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const double x = st[j], y = st[n + j];
  const int key = cell_key(x, y, nx, ny);
  const int64_t pos = (int64_t)off[key] + agg_atomic_add(cursor, key, am);
  int cx = (int)x, cy = (int)y;
  const double g = st[5 * n + j];
  // offsets relative to the (unwrapped) cell holding x, y
  P[pos] = (float)(x - cx);
  P[cap + pos] = (float)(y - cy);
  P[2 * cap + pos] = (float)(st[2 * n + j] * g);
  P[3 * cap + pos] = (float)(st[3 * n + j] * g);
  P[4 * cap + pos] = (float)(st[4 * n + j] * g);
  slot[pos] = (int32_t)j;
}

// cell-grouped FP32 -> FP64 staging in slot order: x, y, vx, vy, vz, gamma
__global__ void k_gather_from_f32(const float *__restrict__ P, const int32_t *__restrict__ slot,
                                  const int32_t *__restrict__ off, int64_t cap, int nx, int ny,
                                  double *st, int64_t n) {
  const int64_t cell = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int gl = threadIdx.x & (G - 1);
  if (cell >= (int64_t)nx * ny) return;
  const int kx = (int)(cell % nx), ky = (int)(cell / nx);
  for (int32_t i = off[cell] + gl; i < off[cell + 1]; i += G) {
    double x = kx + (double)P[i], y = ky + (double)P[cap + i];
    if (x < 0.0) x += nx;
    if (x >= nx) x -= nx;
    if (y < 0.0) y += ny;
    if (y >= ny) y -= ny;
    const double ux = P[2 * cap + i], uy = P[3 * cap + i], uz = P[4 * cap + i];
    const double g = sqrt(1.0 + ux * ux + uy * uy + uz * uz);
    const int64_t s = slot[i];
    st[s] = x;
    st[n + s] = y;
    st[2 * n + s] = ux / g;
    st[3 * n + s] = uy / g;
    st[4 * n + s] = uz / g;
    st[5 * n + s] = g;
  }
}

}  // namespace

int launch_prescale_f32(em2g_ctx *c, int isp) {
  const double ae = 0.5 * c->P.qm[isp] * c->P.dt / c->P.c;
  const int64_t w = c->g.w;
  k_prescale_f32<<<(unsigned)((w + 255) / 256), 256, 0, c->stream>>>(
      c->fld32, c->scaled32 + (int64_t)isp * 6 * w, w, (float)ae, (float)c->P.tx[isp],
      (float)c->P.ty[isp]);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int launch_push_cells_f32(em2g_ctx *c, int isp) {
  Species &S = c->sp[isp];
  const int64_t w = c->g.w;
  const float *sc = c->scaled32 + (int64_t)isp * 6 * w;
  Args32 a;
  a.aex = sc;
  a.aey = sc + w;
  a.aez = sc + 2 * w;
  a.abx = sc + 3 * w;
  a.aby = sc + 4 * w;
  a.abz = sc + 5 * w;
  a.rho = c->fld32 + EM2G_RHO * w;
  a.jx = c->fld32 + EM2G_JXM * w;
  a.jy = c->fld32 + EM2G_JYM * w;
  a.jz = c->fld32 + EM2G_JZM * w;
  a.A = S.p32;
  a.slotA = S.slot;
  a.B = S.p32_alt;
  a.slotB = S.slot_alt;
  a.offA = S.off;
  a.offB = S.off_alt;
  a.cursor = S.cursor;
  a.cnt_next = S.cnt_alt;
  a.cap = S.cap;
  a.nx = c->g.nx;
  a.ny = c->g.ny;
  a.nxg = c->g.nxg;
  a.qd = (float)(c->P.q[isp] * c->P.dn[isp] / (c->P.dx * c->P.dy));
  a.dtdx = (float)(c->P.dt / c->P.dx);
  a.dtdy = (float)(c->P.dt / c->P.dy);
  a.c = (float)c->P.c;
  a.ake_partial = c->red;
  const int64_t nb64 = (c->ncell * G + kThreads - 1) / kThreads;
  if (nb64 > c->red_blocks) return fail(EM2G_ERR_RANGE, "grid exceeds reduction scratch");
  const int nb = (int)nb64;
  int rc = scan_cells(c, S.cnt, S.off_alt);
  if (rc) return rc;
  EM2G_CUDA(cudaMemsetAsync(S.cursor, 0, sizeof(int32_t) * c->ncell, c->stream));
  EM2G_CUDA(cudaMemsetAsync(S.cnt_alt, 0, sizeof(int32_t) * c->ncell, c->stream));
  if ((rc = timing_begin(c))) return rc;
  k_push_cells_f32<<<nb, kThreads, 0, c->stream>>>(a);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  if ((rc = timing_end(c))) return rc;
  std::swap(S.p32, S.p32_alt);
  std::swap(S.slot, S.slot_alt);
  std::swap(S.off, S.off_alt);
  std::swap(S.cnt, S.cnt_alt);
  return launch_ake_finish(c, isp, nb);
}

// staging (6*n doubles on the device, slot order) -> cell-grouped FP32
int upload_f32(em2g_ctx *c, int isp, const double *staging, int64_t n) {
  Species &S = c->sp[isp];
  EM2G_CUDA(cudaMemsetAsync(S.cnt, 0, sizeof(int32_t) * c->ncell, c->stream));
  EM2G_CUDA(cudaMemsetAsync(S.cursor, 0, sizeof(int32_t) * c->ncell, c->stream));
  const unsigned nb = (unsigned)((n + 255) / 256);
  if (n > 0) {
    k_hist64<<<nb, 256, 0, c->stream>>>(staging, n, c->g.nx, c->g.ny, S.cnt);
    EM2G_CUDA(cudaGetLastError());
  }
  int rc = scan_cells(c, S.cnt, S.off);
  if (rc) return rc;
  if (n > 0) {
    k_scatter_to_f32<<<nb, 256, 0, c->stream>>>(staging, n, c->g.nx, c->g.ny, S.off, S.cursor,
                                                 S.p32, S.slot, S.cap);
    EM2G_CUDA(cudaGetLastError());
  }
  c->launches += 2;
  S.n = n;
  S.sorted = true;
  return EM2G_OK;
}

// cell-grouped FP32 -> staging (6*n doubles, slot order)
int download_f32(em2g_ctx *c, int isp, double *staging) {
  Species &S = c->sp[isp];
  if (S.n == 0) return EM2G_OK;
  const int64_t nb = (c->ncell * G + 255) / 256;
  k_gather_from_f32<<<(unsigned)nb, 256, 0, c->stream>>>(S.p32, S.slot, S.off, S.cap, c->g.nx,
                                                         c->g.ny, staging, S.n);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

}  // namespace em2g

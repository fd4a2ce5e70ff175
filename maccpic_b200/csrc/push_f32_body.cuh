// push_f32_body.cuh -- the device code of the mixed-precision push: the
// particle layout's arguments, the quadratic weights, the gathers, the
// register-block deposits and the row-segment push itself, shared by the
// push kernels of push_fast_f32.cu and the fused ensemble step of
// ens_step.cu.  The algorithm is described at the top of push_fast_f32.cu.
#pragma once
#include "ens_internal.cuh"
#include "sort_common.cuh"

// The compiled variants of the FP32 push, as (TCX, G, NC, MINB): TCX cells
// per CTA pass, G lanes per cell, NC cells per lane group one after the
// other (a segment is TCX*NC cells), MINB CTAs per SM the register
// allocation must allow.  push_fast_f32.cu and ens_step.cu instantiate
// their kernels from this one list, so a variant index means the same
// kernel shape in both.
#define EM2G_F32_VARIANTS(X)                                                   \
  X(32, 4, 1, 4) X(32, 4, 1, 5) X(32, 4, 1, 6) X(64, 4, 1, 2) X(64, 4, 1, 3)  \
  X(32, 8, 1, 2) X(32, 2, 1, 8) X(64, 2, 1, 4) X(32, 4, 2, 4) X(32, 4, 3, 4)

// Bounds-checked build (-DEM2G_BOUNDS_CHECK: libem2g_checked.so, from
// maccpic_b200/build.py): every index the push computes for shared or global
// memory is checked before the access; one out of range is counted in
// Args32::lost (the step then fails with EM2G_ERR_RANGE) and the access is
// skipped -- no trap, no fault.  The ordinary build compiles the checks away.
#ifdef EM2G_BOUNDS_CHECK
#define EM2G_IN(cond, lost) ((cond) ? true : (atomicAdd((lost), 1.0), false))
#else
#define EM2G_IN(cond, lost) true
#endif

namespace em2g {
namespace {

constexpr int kCopyLanes = 4;  // lanes per cell of the download gather
constexpr float kBelowOne = 0.99999994f;  // the largest float below 1
constexpr int WY = 6;  // window rows: y0-1 .. y0+4

struct Args32 {
  const float2 *__restrict__ ebx;  // (a*Ex, a*Bx): x half, y node staggering
  const float2 *__restrict__ ebz;  // (a*Ez, a*Bz): x half, y half
  const float2 *__restrict__ eby;  // (a*Ey, a*By): x node, y half
  float *rho, *jx, *jy, *jz;
  // particles: entry j of 4*cap floats holds (xr, yr, ux, uy) as one float4
  // (one 128-bit load or store), then cap floats hold uz
  const float *__restrict__ A;
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
  double *lost;  // count of particles a regrouping push could not place
};

// the pairs of one ensemble push (a __grid_constant__ kernel parameter)
struct EnsPush32 {
  int npairs, ntiles;
  int *counter;  // next unclaimed segment, zeroed before the launch
  int tile0[kEnsMaxPairs + 1];
  int segs[kEnsMaxPairs];
  Args32 pair[kEnsMaxPairs];
};
static_assert(sizeof(EnsPush32) <= 32764, "kernel parameters are limited to 32764 bytes");

struct Wts {
  int i;          // array index of the middle node
  float m, s, p;  // weights of nodes i-1, i, i+1
  int u;          // integer nodes: the middle node is the cell's upper one (f >= 1/2)
};

// Packed FP32 pairs (sm_100a's f32x2 arithmetic) through the compiler's
// builtins, so that it allocates the register pairs itself: one instruction
// for the two lanes of a pair, each rounded as its scalar FMA / multiply /
// add would be.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }

// The quadratic weights of both axes at once for offsets f = (fx, fy) in
// cell (cx, cy) (the forms of the file header): cell-centred nodes, middle
// index c+1, with d = f - 1/2: (1/2-d)^2/2, 3/4 - d^2, (1/2+d)^2/2; integer
// nodes, middle index c+1+u with u = [f >= 1/2], h = f - u: the same in h.
// The three sum to 1 and differ by d (or h) at the ends, so with s = 3/4 -
// d^2 and t = (1 - s)/2 the ends are t -+ d/2: one packed operation each.
__device__ __forceinline__ void weights2(int cx, int cy, float2 f, Wts &hx, Wts &hy, Wts &nx,
                                         Wts &ny) {
  const float2 d = add2(f, bc2(-0.5f));
  const float2 hs = fma2(make_float2(-d.x, -d.y), d, bc2(0.75f));
  const float2 ht = fma2(bc2(-0.5f), hs, bc2(0.5f));
  const float2 hm = fma2(bc2(-0.5f), d, ht), hp = fma2(bc2(0.5f), d, ht);
  hx = Wts{cx + 1, hm.x, hs.x, hp.x, 0};
  hy = Wts{cy + 1, hm.y, hs.y, hp.y, 0};
  const int ux = f.x >= 0.5f ? 1 : 0, uy = f.y >= 0.5f ? 1 : 0;
  const float2 h = add2(f, make_float2(f.x >= 0.5f ? -1.0f : 0.0f, f.y >= 0.5f ? -1.0f : 0.0f));
  const float2 ns = fma2(make_float2(-h.x, -h.y), h, bc2(0.75f));
  const float2 nt = fma2(bc2(-0.5f), ns, bc2(0.5f));
  const float2 nm = fma2(bc2(-0.5f), h, nt), np = fma2(bc2(0.5f), h, nt);
  nx = Wts{cx + 1 + ux, nm.x, ns.x, np.x, ux};
  ny = Wts{cy + 1 + uy, nm.y, ns.y, np.y, uy};
}

// 9-point gather of an (E, B) pair; base points at node (i-1, j-1) of the
// stencil in an array of row pitch `pitch`.  Both members of the pair go
// through one packed instruction per weight: (a m + b s) + c p per row,
// then the rows combined the same way.
__device__ __forceinline__ float2 gather_pair(const float2 *base, int pitch, const Wts &wx,
                                              const Wts &wy) {
  float2 r[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float2 a = base[k * pitch], b = base[k * pitch + 1], c = base[k * pitch + 2];
    r[k] = fma2(c, bc2(wx.p), fma2(b, bc2(wx.s), mul2(a, bc2(wx.m))));
  }
  return fma2(r[2], bc2(wy.p), fma2(r[1], bc2(wy.s), mul2(r[0], bc2(wy.m))));
}

// The same gather from the shared window, whose entry (row, col) holds the
// pair of node col and the pair of node col+1: two loads per stencil row
// (nodes i-1 and i together, then node i+1) instead of three, the same
// arithmetic.
__device__ __forceinline__ float2 gather_pair_win(const float4 *base, int pitch, const Wts &wx,
                                                  const Wts &wy) {
  float2 r[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float4 ab = base[k * pitch];
    const float2 c = *reinterpret_cast<const float2 *>(base + k * pitch + 2);
    const float2 a = make_float2(ab.x, ab.y), b = make_float2(ab.z, ab.w);
    r[k] = fma2(c, bc2(wx.p), fma2(b, bc2(wx.s), mul2(a, bc2(wx.m))));
  }
  return fma2(r[2], bc2(wy.p), fma2(r[1], bc2(wy.s), mul2(r[0], bc2(wy.m))));
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

// The 49-value register block, kept as pairs so that packed FMAs update two
// values at once.  Jx (4 rows x 3) and Jz (3 x 3) pair rows -- per column k,
// rows (0,1) and (2,3) of Jx, rows (0,1) and the single row 2 of Jz -- so
// that both take the x weight of column k as the broadcast operand; Jy (3 x
// 4) and rho (4 x 4) pair columns (0,1) and (2,3) of each row.
struct Block32 {
  float2 jxr01[3], jxr23[3], jzr01[3], jy01[3], jy23[3], rho01[4], rho23[4];
  float jzr2[3];
};
// element i of a row or column kept as pairs (i a compile-time constant)
__device__ __forceinline__ float pick4(const float2 &lo, const float2 &hi, int i) {
  return i == 0 ? lo.x : i == 1 ? lo.y : i == 2 ? hi.x : hi.y;
}
__device__ __forceinline__ float pick3(const float2 &lo, float last, int i) {
  return i == 0 ? lo.x : i == 1 ? lo.y : last;
}

// The integer-node weights of a particle of cell c as the 4 nodes c .. c+3
// (array indices) the cell's particles can reach.  Only particles in the
// lane's cell deposit into its block (the others with zero charge), so the
// middle node's place is the particle's own u.
__device__ __forceinline__ void spread4(const Wts &w, float o[4]) {
  const bool lo = w.u == 0;
  o[0] = lo ? w.m : 0.0f;
  o[1] = lo ? w.s : w.m;
  o[2] = lo ? w.p : w.s;
  o[3] = lo ? 0.0f : w.p;
}

// J of one particle at local offsets (fx, fy) of the group's cell (cx, cy)
__device__ __forceinline__ void block_add_j(Block32 &b, int cx, int cy, const Wts &hx,
                                            const Wts &hy, const Wts &nxw, const Wts &nyw,
                                            float qx, float qy, float qz) {
  float wxn[4], wyn[4];
  spread4(nxw, wxn);
  spread4(nyw, wyn);
  const float wxh[3] = {hx.m, hx.s, hx.p}, wyh[3] = {hy.m, hy.s, hy.p};
  const float2 n01 = make_float2(wxn[0], wxn[1]), n23 = make_float2(wxn[2], wxn[3]);
  // Jx(r, k) += (wyn[r] qx) wxh[k], Jz(r, k) += (wyh[r] qz) wxh[k]
  const float2 ax01 = mul2(make_float2(wyn[0], wyn[1]), bc2(qx));
  const float2 ax23 = mul2(make_float2(wyn[2], wyn[3]), bc2(qx));
  const float2 az01 = mul2(make_float2(wyh[0], wyh[1]), bc2(qz));
  const float az2 = wyh[2] * qz;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float2 w = bc2(wxh[k]);
    b.jxr01[k] = fma2(ax01, w, b.jxr01[k]);
    b.jxr23[k] = fma2(ax23, w, b.jxr23[k]);
    b.jzr01[k] = fma2(az01, w, b.jzr01[k]);
    b.jzr2[k] = fmaf(az2, wxh[k], b.jzr2[k]);
  }
  // Jy(r, k) += (wyh[r] qy) wxn[k]
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float ty = wyh[r] * qy;
    b.jy01[r] = fma2(n01, bc2(ty), b.jy01[r]);
    b.jy23[r] = fma2(n23, bc2(ty), b.jy23[r]);
  }
}

__device__ __forceinline__ void block_add_rho(Block32 &b, int cx, int cy, const Wts &nxw,
                                              const Wts &nyw, float q) {
  float wxn[4], wyn[4];
  spread4(nxw, wxn);
  spread4(nyw, wyn);
  const float2 n01 = make_float2(wxn[0], wxn[1]), n23 = make_float2(wxn[2], wxn[3]);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const float t = wyn[r] * q;
    b.rho01[r] = fma2(n01, bc2(t), b.rho01[r]);
    b.rho23[r] = fma2(n23, bc2(t), b.rho23[r]);
  }
}

__device__ __forceinline__ void deposit_j_atomic(const Args32 &a, const Wts &hx, const Wts &hy,
                                                 const Wts &nxw, const Wts &nyw, float qx,
                                                 float qy, float qz) {
  scatter9(a.jx, a.nxg, hx, nyw, qx);
  scatter9(a.jz, a.nxg, hx, hy, qz);
  scatter9(a.jy, a.nxg, nxw, hy, qy);
}

// sum over the G lanes of a cell's group (G a power of two)
template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
  for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of a group's G values of one block element, read from the warp's
// scratch row of that element at the group's first lane g0.
template <int G>
__device__ __forceinline__ float group_row_sum(const float *row, int g0) {
  if constexpr (G == 2) {
    const float2 v = *reinterpret_cast<const float2 *>(row + g0);
    return v.x + v.y;
  } else if constexpr (G == 4) {
    const float4 v = *reinterpret_cast<const float4 *>(row + g0);
    return (v.x + v.y) + (v.z + v.w);
  } else {
    static_assert(G == 8, "2, 4 or 8 lanes per cell");
    const float4 v = *reinterpret_cast<const float4 *>(row + g0);
    const float4 w = *reinterpret_cast<const float4 *>(row + g0 + 4);
    return ((v.x + v.y) + (v.z + v.w)) + ((w.x + w.y) + (w.z + w.w));
  }
}

// Add an array's block rows (R rows of C values, elements e0.. of the
// scratch) of a group's cell (kx, ky) to the array: lane gl of the group
// takes rows gl, gl+G, ..
template <int G, int R, int C>
__device__ __forceinline__ void flush_rows(float *A, int nxg, int kx, int ky, const float *red,
                                           int e0, int gl, int g0) {
#pragma unroll
  for (int rr = 0; rr < (R + G - 1) / G; ++rr) {
    const int r = gl + rr * G;
    if (r < R) {
      float *dst = A + (int64_t)(ky + r) * nxg + kx;
      const float *src = red + (e0 + r * C) * 32;
#pragma unroll
      for (int k = 0; k < C; ++k) {
        const float v = group_row_sum<G>(src + k * 32, g0);
        if (v != 0.0f) atomicAdd(dst + k, v);
      }
    }
  }
}

// The whole-cell part of a pair of offsets in (-1, 2) (-1, 0 or 1 each) and
// what is left within that cell: floor as a float is exact, so the rest is
// one packed subtraction.
__device__ __forceinline__ void split_cell(float2 f, int &ox, int &oy, float2 &rest,
                                           float2 &fl) {
  fl = make_float2(floorf(f.x), floorf(f.y));
  ox = (int)fl.x;
  oy = (int)fl.y;
  rest = add2(f, make_float2(-fl.x, -fl.y));
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// 1/gamma of u = gamma v, its sum of squares rounded in one fixed order:
// the push and the deposit stack's drain both take v from u
__device__ __forceinline__ float inv_gamma(float ux, float uy, float uz) {
  return rsqrtf(__fmaf_rn(uz, uz, __fmaf_rn(uy, uy, __fmaf_rn(ux, ux, 1.0f))));
}

// Deposits of particles outside their lane's cell go to global memory with
// atomics.  Done where they arise, they would run with the one or two lanes
// that need them while the rest of the warp waits; instead each warp stacks
// them in shared memory and does 32 at a time, one per lane.  An entry is a
// cell, the offsets in it and the particle's new u; kind 0 deposits J (jm
// at the old position) and, in a regrouping push, writes the particle to
// the back of its start cell's range (it came from another cell's range, so
// its slot comes from an atomic -- one round trip per 32 such particles
// instead of one per warp iteration that has any); kind 1 deposits rho, J
// (jp) and the cell count at the new position.
constexpr int kQCap = 96;  // < 32 left after a drain + at most 2 per lane
struct DepQ {
  int cx[kQCap], cy[kQCap];
  float2 f[kQCap];
  float4 q[kQCap];        // ux, uy, uz, kind
  int32_t slot[kQCap];    // kind 0 of a regrouping push: the particle's slot
};
// A warp's shared scratch: its deposit stack while it pushes, then up to 24
// block values of each of its lanes (value e of lane l at red[e*32 + l])
// for the sums over each cell's lanes.
constexpr int kRedVals = 24;
union WarpScratch {
  DepQ q;
  float red[kRedVals * 32];
};
static_assert(sizeof(DepQ) >= sizeof(float) * kRedVals * 32, "the stack holds 24 rows");

template <bool INPLACE>
__device__ __forceinline__ void drain_entry(const Args32 &a, const DepQ &Q, int e) {
  const int cx = wrap(Q.cx[e], a.nx), cy = wrap(Q.cy[e], a.ny);  // entries are unwrapped
  const float4 uu = Q.q[e];
  // v and q v as the push computed them
  const float ginv = inv_gamma(uu.x, uu.y, uu.z);
  const float vx = uu.x * ginv, vy = uu.y * ginv, vz = uu.z * ginv;
  const float qx = a.qd * vx, qy = a.qd * vy, qz = a.qd * vz;
  const float2 f = Q.f[e];
  Wts hx, hy, nxw, nyw;
  weights2(cx, cy, f, hx, hy, nxw, nyw);
  // every 3 x 3 stencil inside the guarded (nx+3) x (ny+3) arrays
  if (!EM2G_IN(hx.i >= 1 && hx.i + 1 <= a.nx + 2 && nxw.i >= 1 && nxw.i + 1 <= a.nx + 2 &&
                   hy.i >= 1 && hy.i + 1 <= a.ny + 2 && nyw.i >= 1 && nyw.i + 1 <= a.ny + 2,
               a.lost))
    return;
  deposit_j_atomic(a, hx, hy, nxw, nyw, qx, qy, qz);
  if (uu.w != 0.0f) {
    scatter9(a.rho, a.nxg, nxw, nyw, a.qd);
    atomicAdd(a.cnt_next + cy * a.nx + cx, 1);
  } else if constexpr (!INPLACE) {
    // the new position relative to the start cell, as the push moved it
    const float2 mv = fma2(make_float2(vx, vy), make_float2(a.dtdx, a.dtdy), f);
    const int key = cy * a.nx + cx;  // the start cell's key
    const int64_t pos = (int64_t)a.offB[key + 1] - 1 - atomicAdd(a.cursor + key, 1);
    // a guard: the counts of the last push place every particle inside the
    // buffer; a position outside it is counted and not written
    if (pos < 0 || pos >= a.cap) {
      atomicAdd(a.lost, 1.0);
    } else {
      reinterpret_cast<float4 *>(a.B)[pos] = make_float4(mv.x, mv.y, uu.x, uu.y);
      a.B[4 * a.cap + pos] = uu.z;
      a.slotB[pos] = Q.slot[e];
    }
  }
}

// What one particle's push leaves for the write-back and the warp's stack.
// Cells are unwrapped (group cell + offsets, possibly -1 or n..n+1 across
// the periodic boundary); whoever indexes the arrays with them wraps them.
struct PartOut {
  float mx, my, ux, uy, uz;  // new position relative to the start cell, new u
  float oxf, oyf;            // start cell - group cell (-1, 0 or 1 each), as floats
  bool home_x, home_y;       // the new position's cell is the group cell's column / row
  bool in_cell_old;          // the start cell is the group cell
  bool need_old, need_new;   // deposits for the warp's stack
  int cx, cy, ncx, ncy;      // start and end cells, unwrapped
  float fx, fy, nfx, nfy;
};

// Gather, Boris, move and the in-cell deposits of one particle at (xr, yr)
// relative to the group cell (kx, ky) with momentum u; `act` false makes it
// a dry run on harmless input (no deposits, no energy).  cinv = 1/c.
template <int WXW>
__device__ __forceinline__ void push_one(const Args32 &a, float4 (*win)[WY][WXW], int x0,
                                         int y0, int kx, int ky, bool act, float xr, float yr,
                                         float ux, float uy, float uz, float cinv, Block32 &b,
                                         double &akel, int &stay_new, PartOut &o) {
  constexpr int WX = WXW;
  const int nx = a.nx, ny = a.ny, nxg = a.nxg;
  // the cell the particle is in now (it may have left cell k last step)
  int ox, oy;
  float2 fxy;
  float2 oxy;
  split_cell(make_float2(xr, yr), ox, oy, fxy, oxy);
  o.oxf = oxy.x;
  o.oyf = oxy.y;
  const int cx = kx + ox, cy = ky + oy;  // unwrapped
  const float fx = fxy.x, fy = fxy.y;
  o.in_cell_old = (ox == 0) && (oy == 0);
  Wts hx, hy, nxw, nyw;  // array indices of the unwrapped cell
  weights2(cx, cy, make_float2(fx, fy), hx, hy, nxw, nyw);
  // gather from the shared window unless the particle is across the
  // periodic boundary: then its cell is within one of the group cell (kx in
  // x0 .. x0+TCX-1, ky = y0), whose stencils the window holds (window index
  // = array index - (x0-1, y0-1), the stencil starting one node before i);
  // else from global memory at the wrapped cell
  float2 ebx, ebz, eby;
  if ((unsigned)cx < (unsigned)nx && (unsigned)cy < (unsigned)ny) {
#ifdef EM2G_BOUNDS_CHECK
    // three rows and (entries of) three columns from each stencil's corner
    const int r0 = nyw.i - y0, r1 = hy.i - y0, c0 = hx.i - x0, c1 = nxw.i - x0;
    if (!EM2G_IN(r0 >= 0 && r0 + 2 < WY && r1 >= 0 && r1 + 2 < WY && c0 >= 0 &&
                     c0 + 2 < WX && c1 >= 0 && c1 + 2 < WX,
                 a.lost)) {
      ebx = ebz = eby = make_float2(0.0f, 0.0f);
    } else
#endif
    {
      ebx = gather_pair_win(&win[0][nyw.i - y0][hx.i - x0], WX, hx, nyw);
      ebz = gather_pair_win(&win[1][hy.i - y0][hx.i - x0], WX, hx, hy);
      eby = gather_pair_win(&win[2][hy.i - y0][nxw.i - x0], WX, nxw, hy);
    }
  } else {
    const int sx = wrap(cx, nx) - cx, sy = wrap(cy, ny) - cy;
    const int64_t bx0 = (int64_t)(nyw.i + sy - 1) * nxg + hx.i + sx - 1;
    const int64_t bz0 = (int64_t)(hy.i + sy - 1) * nxg + hx.i + sx - 1;
    const int64_t by0 = (int64_t)(hy.i + sy - 1) * nxg + nxw.i + sx - 1;
#ifdef EM2G_BOUNDS_CHECK
    const int64_t w = (int64_t)nxg * (ny + 3), span = 2 * (int64_t)nxg + 2;
    if (!EM2G_IN(bx0 >= 0 && bx0 + span < w && bz0 >= 0 && bz0 + span < w && by0 >= 0 &&
                     by0 + span < w,
                 a.lost)) {
      ebx = ebz = eby = make_float2(0.0f, 0.0f);
    } else
#endif
    {
      ebx = gather_pair(a.ebx + bx0, nxg, hx, nyw);
      ebz = gather_pair(a.ebz + bz0, nxg, hx, hy);
      eby = gather_pair(a.eby + by0, nxg, nxw, hy);
    }
  }
  // relativistic Boris on u (pic/move.f90:176-203).  The reciprocal square
  // roots and divisions are the hardware approximations (rsqrtf, a few ulp),
  // well inside this path's FP32 error; gamma - 1 is taken as
  // g^2 (1/gamma) / (1 + 1/gamma), free of the cancellation of gamma - 1.
  const float gx = ux + ebx.x, gy = uy + eby.x, gz = uz + ebz.x;
  const float g2 = gx * gx + gy * gy + gz * gz;
  const float rg = rsqrtf(1.0f + g2);  // 1 / gamma
  if (act) akel += (double)__fdividef(g2 * rg, 1.0f + rg);
  const float dcg = rg * cinv;
  float tx = dcg * ebx.y, ty = dcg * eby.y, tz = dcg * ebz.y;
  const float vvx = gx + gy * tz - gz * ty;
  const float vvy = gy + gz * tx - gx * tz;
  const float vvz = gz + gx * ty - gy * tx;
  const float f2 = __fdividef(2.0f, 1.0f + tx * tx + ty * ty + tz * tz);
  tx *= f2;
  ty *= f2;
  tz *= f2;
  ux = gx + vvy * tz - vvz * ty + ebx.x;
  uy = gy + vvz * tx - vvx * tz + eby.x;
  uz = gz + vvx * ty - vvy * tx + ebz.x;
  const float ginv = inv_gamma(ux, uy, uz);
  const float vx = ux * ginv, vy = uy * ginv, vz = uz * ginv;
  const float qx = a.qd * vx, qy = a.qd * vy, qz = a.qd * vz;
  o.ux = ux;
  o.uy = uy;
  o.uz = uz;
  // jm at the old position (pic/curnt.f90:53-132)
  o.need_old = act && !o.in_cell_old;
  o.cx = cx;
  o.cy = cy;
  o.fx = fx;
  o.fy = fy;
  // the in-cell deposits run in every lane, with zero charge where the
  // particle is outside the lane's cell or there is none (the weights are
  // finite, so the block is unchanged): no branch around them
  const float mo = (act && o.in_cell_old) ? 1.0f : 0.0f;
  block_add_j(b, kx, ky, hx, hy, nxw, nyw, qx * mo, qy * mo, qz * mo);
  // move (pic/curnt.f90:181-194), relative to the start cell
  const float2 mv = fma2(make_float2(vx, vy), make_float2(a.dtdx, a.dtdy), make_float2(fx, fy));
  o.mx = mv.x;
  o.my = mv.y;
  int nox, noy;
  float2 nf, nfl;
  split_cell(mv, nox, noy, nf, nfl);
  const float nfx = nf.x, nfy = nf.y;
  // rho and jp at the new position (pic/curnt.f90:197-303); with at least 4
  // cells a side, the new cell is the group cell exactly when the offsets
  // cancel
  o.home_x = ox + nox == 0;
  o.home_y = oy + noy == 0;
  const bool stays = o.home_x && o.home_y;
  o.need_new = act && !stays;
  o.ncx = cx + nox;
  o.ncy = cy + noy;
  o.nfx = nfx;
  o.nfy = nfy;
  {
    const float ms = (act && stays) ? 1.0f : 0.0f;
    Wts nhx, nhy, nnx, nny;
    weights2(kx, ky, make_float2(nfx, nfy), nhx, nhy, nnx, nny);
    block_add_rho(b, kx, ky, nnx, nny, a.qd * ms);
    block_add_j(b, kx, ky, nhx, nhy, nnx, nny, qx * ms, qy * ms, qz * ms);
    stay_new += (act && stays) ? 1 : 0;
  }
}

// One row segment: cells x0 .. x0+NC*TCX-1 of row y0, by a CTA of TCX*G
// threads; `blk` numbers the segment for the kinetic-energy partials.  Each
// group of G lanes takes NC cells one after the other (x0 + g, then
// x0 + TCX + g, ..): a warp runs as long as its groups' largest total, and
// totals over several cells vary relatively less than single cells' counts,
// so fewer lanes wait.
// INPLACE: a step between regroupings -- every particle keeps its slot in
// A (B == A) and its position stays relative to its group cell, so the
// offsets drift by at most c*dt/dx per step (the interval is bounded so
// that they stay in (-1, 2)); the counts of the new cells are still taken.
template <int TCX, int G, int NC, bool INPLACE>
__device__ __forceinline__ void push_segment(const Args32 &a, int x0, int y0, int64_t blk,
                                             float4 (*win)[WY][NC * TCX + 5], WarpScratch *ws) {
  constexpr int kThreads = TCX * G;
  constexpr int WX = NC * TCX + 5;  // window columns: x0-1 .. x0+NC*TCX+3
  const int nx = a.nx, ny = a.ny, nxg = a.nxg;
  const int lane = threadIdx.x & 31, gl = lane & (G - 1);
  int kx = x0 + (int)(threadIdx.x / G);  // this group's cell in the current pass
  const int ky = y0;
  bool valid = kx < nx;
  int kxs = valid ? kx : nx - 1;  // the cell lanes past the grid's edge work on
  int64_t cell = (int64_t)ky * nx + kx;
  const int64_t cap = a.cap;
  const unsigned gmask = ((1u << G) - 1u) << (lane & ~(G - 1));  // this lane's group
  // The segment's start has three independent global loads -- the first
  // cell's range, the (E, B) window and the first particle -- issued
  // together before the first wait: the range, then the window into
  // registers, then the particle (once the range is in), then the window
  // into shared memory.
  int32_t beg = valid ? a.offA[cell] : 0;
  int32_t front = (!INPLACE && valid) ? a.offB[cell] : 0;  // cell k's first slot in B
  int32_t end = valid ? a.offA[cell + 1] : 0;
  // the window: array indices x0-1.., y0-1..
  constexpr int kWin = 3 * WY * WX, kWinPer = (kWin + kThreads - 1) / kThreads;
  float4 wv[kWinPer];  // (node col, node col+1)
#pragma unroll
  for (int u = 0; u < kWinPer; ++u) {
    const int t = threadIdx.x + u * kThreads;
    const int comp = t / (WY * WX), r = (t / WX) % WY, col = t % WX;
    const int gx = x0 - 1 + col, gy = y0 - 1 + r;
    wv[u] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t < kWin && gx >= 0 && gx <= nx + 2 && gy >= 0 && gy <= ny + 2) {
      const float2 *src = comp == 0 ? a.ebx : (comp == 1 ? a.ebz : a.eby);
      const float2 v0 = src[(int64_t)gy * nxg + gx];
      const float2 v1 = gx + 1 <= nx + 2 ? src[(int64_t)gy * nxg + gx + 1] : make_float2(0.f, 0.f);
      wv[u] = make_float4(v0.x, v0.y, v1.x, v1.y);
    }
  }
  // software pipeline: the next particle's state is loaded while this one runs
  float pxr = 0.f, pyr = 0.f, pux = 0.f, puy = 0.f, puz = 0.f;
  int32_t pslot = 0;
  const float4 *__restrict__ A4 = reinterpret_cast<const float4 *>(a.A);
  const float *__restrict__ Auz = a.A + 4 * cap;
  float4 *B4 = reinterpret_cast<float4 *>(a.B);
  float *Buz = a.B + 4 * cap;
  if (beg + gl < end && EM2G_IN(beg + gl < cap, a.lost)) {
    const int32_t j = beg + gl;
    const float4 q = A4[j];
    pxr = q.x;
    pyr = q.y;
    pux = q.z;
    puy = q.w;
    puz = Auz[j];
    pslot = a.slotA[j];
  }
#pragma unroll
  for (int u = 0; u < kWinPer; ++u) {
    const int t = threadIdx.x + u * kThreads;
    if (t < kWin) win[t / (WY * WX)][(t / WX) % WY][t % WX] = wv[u];
  }
  __syncthreads();

  double akel = 0.0;  // this lane's sum of gamma - 1
  const float cinv = 1.0f / a.c;
  DepQ &Q = ws[threadIdx.x >> 5].q;
  int qn = 0;  // entries on this warp's stack (the same in every lane)
  const unsigned lt = (1u << lane) - 1u;
  for (int pass = 0; pass < NC; ++pass) {
    if (pass > 0) {  // the group's next cell: its range and first particle
      kx += TCX;
      valid = kx < nx;
      kxs = valid ? kx : nx - 1;
      cell = (int64_t)ky * nx + kx;
      beg = valid ? a.offA[cell] : 0;
      front = (!INPLACE && valid) ? a.offB[cell] : 0;
      end = valid ? a.offA[cell + 1] : 0;
      if (beg + gl < end && EM2G_IN(beg + gl < cap, a.lost)) {
        const int32_t j = beg + gl;
        const float4 q = A4[j];
        pxr = q.x;
        pyr = q.y;
        pux = q.z;
        puy = q.w;
        puz = Auz[j];
        pslot = a.slotA[j];
      }
    }
    Block32 b;
    const float2 z2 = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      b.rho01[r] = b.rho23[r] = z2;
      if (r < 3) {
        b.jxr01[r] = b.jxr23[r] = b.jzr01[r] = b.jy01[r] = b.jy23[r] = z2;
        b.jzr2[r] = 0.0f;
      }
    }
    int stay_new = 0;  // particles of this lane whose new position is in cell k
    int home_count = 0;  // particles of this group written to the front of cell k

    for (int32_t i = beg + gl;; i += G) {
      const bool act = i < end;
      if (__ballot_sync(0xffffffffu, act) == 0u) break;
      const float cxr = pxr, cyr = pyr, cux = pux, cuy = puy, cuz = puz;
      const int32_t cslot = pslot;
      const int32_t j = i + G;
      if (j < end && EM2G_IN(j < cap, a.lost)) {
        const float4 q = A4[j];
        pxr = q.x;
        pyr = q.y;
        pux = q.z;
        puy = q.w;
        puz = Auz[j];
        pslot = a.slotA[j];
      }
      // a lane without a particle runs on a dummy inside a real cell
      PartOut o;
      push_one<WX>(a, win, x0, y0, kxs, ky, act, act ? cxr : 0.25f, act ? cyr : 0.25f, cux, cuy,
                    cuz, cinv, b, akel, stay_new, o);
      if (INPLACE) {
        if (act) {
          // the offset relative to the group cell, kept in the cell the push
          // counted for the next grouping (group cell + o + no): when that is
          // the group cell itself, 1 plus a tiny negative move can round to
          // exactly 1, which would read as the next cell (every other case is
          // exact or rounds within its cell)
          float xn = o.mx + o.oxf, yn = o.my + o.oyf;
          if (o.home_x) xn = fminf(xn, kBelowOne);
          if (o.home_y) yn = fminf(yn, kBelowOne);
          if (EM2G_IN(i < cap, a.lost)) {
            B4[i] = make_float4(xn, yn, o.ux, o.uy);
            Buz[i] = o.uz;
          }
        }
      } else {
        // write back grouped by the cell of the start of this step: particles
        // that started it in cell k take the next slots from the front of k's
        // segment in processing order (a running count per group, no atomics);
        // the few that came from another cell's range fill it from the back,
        // written by the deposit stack's drain with their kind-0 entry
        const unsigned inm = __ballot_sync(0xffffffffu, act && o.in_cell_old) & gmask;
        if (act && o.in_cell_old) {
          const int64_t pos = (int64_t)front + home_count + __popc(inm & lt);
          // a guard: the counts of the last push place every particle inside
          // the buffer; a position outside it is counted and not written
          if (pos < 0 || pos >= cap) {
            atomicAdd(a.lost, 1.0);
          } else {
            B4[pos] = make_float4(o.mx, o.my, o.ux, o.uy);
            Buz[pos] = o.uz;
            a.slotB[pos] = cslot;
          }
        }
        home_count += __popc(inm);
      }
      // the out-of-cell deposits onto the warp's stack; whole warps of them
      // done at once
      const unsigned m_old = __ballot_sync(0xffffffffu, o.need_old);
      const unsigned m_new = __ballot_sync(0xffffffffu, o.need_new);
      if (m_old | m_new) {
        if (o.need_old && EM2G_IN(qn + __popc(m_old & lt) < kQCap, a.lost)) {
          const int q = qn + __popc(m_old & lt);
          Q.cx[q] = o.cx;
          Q.cy[q] = o.cy;
          Q.f[q] = make_float2(o.fx, o.fy);
          Q.q[q] = make_float4(o.ux, o.uy, o.uz, 0.0f);
          if constexpr (!INPLACE) Q.slot[q] = cslot;
        }
        const int qn1 = qn + __popc(m_old);
        if (o.need_new && EM2G_IN(qn1 + __popc(m_new & lt) < kQCap, a.lost)) {
          const int q = qn1 + __popc(m_new & lt);
          Q.cx[q] = o.ncx;
          Q.cy[q] = o.ncy;
          Q.f[q] = make_float2(o.nfx, o.nfy);
          Q.q[q] = make_float4(o.ux, o.uy, o.uz, 1.0f);
        }
        qn = qn1 + __popc(m_new);
        __syncwarp();
        while (qn >= 32) {
          qn -= 32;
          drain_entry<INPLACE>(a, Q, qn + lane);
          __syncwarp();
        }
      }
    }

    if (lane < qn) drain_entry<INPLACE>(a, Q, lane);
    qn = 0;
    // the group's new-position counts for cell k, and its register blocks
    const int stay = group_sum<G>((float)stay_new) + 0.5f;
    if (valid && gl == 0 && stay > 0) atomicAdd(a.cnt_next + cell, stay);
    // the block's rows ky .. ky+3 and columns kx .. kx+3 lie in the arrays
    valid = valid && EM2G_IN(kx + 3 <= nx + 2 && ky + 3 <= ny + 2, a.lost);
    if (__any_sync(0xffffffffu, valid && end > beg)) {
      // the G blocks of each cell summed through the warp's scratch (the
      // stack is empty now), in three passes: rho, Jx and Jy, Jz
      float *red = ws[threadIdx.x >> 5].red;
      const int g0 = lane & ~(G - 1);
      __syncwarp();
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[(r * 4 + k) * 32 + lane] = pick4(b.rho01[r], b.rho23[r], k);
      __syncwarp();
      if (valid) flush_rows<G, 4, 4>(a.rho, nxg, kx, ky, red, 0, gl, g0);
      __syncwarp();
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) red[(r * 3 + k) * 32 + lane] = pick4(b.jxr01[k], b.jxr23[k], r);
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 4; ++k)
          red[(12 + r * 4 + k) * 32 + lane] = pick4(b.jy01[r], b.jy23[r], k);
      __syncwarp();
      if (valid) {
        flush_rows<G, 4, 3>(a.jx, nxg, kx, ky, red, 0, gl, g0);
        flush_rows<G, 3, 4>(a.jy, nxg, kx, ky, red, 12, gl, g0);
      }
      __syncwarp();
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) red[(r * 3 + k) * 32 + lane] = pick3(b.jzr01[k], b.jzr2[k], r);
      __syncwarp();
      if (valid) flush_rows<G, 3, 3>(a.jz, nxg, kx, ky, red, 0, gl, g0);
    }
    __syncwarp();  // the next pass's stack reuses the scratch just read
  }  // pass
  // per-warp partial of sum(gamma - 1); no block barrier at the end
  for (int o = 16; o > 0; o >>= 1) akel += __shfl_down_sync(0xffffffffu, akel, o);
  if (lane == 0) a.ake_partial[blk * (kThreads / 32) + (threadIdx.x >> 5)] = akel;
}

// kinetic energy of every pair of an ensemble: pair p's partials summed in
// a fixed order (pic/move.f90:183, :208)
struct EnsAke {
  const double *partial[kEnsMaxPairs];
  int count[kEnsMaxPairs];
  double scale[kEnsMaxPairs];  // am * dn
  double *out[kEnsMaxPairs];
};

// The push arguments of every (run, species) pair of an ensemble and its
// kinetic-energy table: current buffers and offsets bp, current counts cp
// (0 or 1 each, as em2g_ens's parity and cparity), in place or regrouping,
// for a variant of `cells` cells per segment and `threads` threads per CTA.
inline void ens_push_tables(em2g_ens *e, int bp, int cp, bool inplace, int cells, int threads,
                            EnsPush32 *P, EnsAke *K) {
  float *A = bp ? e->p32_alt : e->p32, *B = bp ? e->p32 : e->p32_alt;
  int32_t *slotA = bp ? e->slot_alt : e->slot, *slotB = bp ? e->slot : e->slot_alt;
  int32_t *offA = bp ? e->off_alt : e->off, *offB = bp ? e->off : e->off_alt;
  int32_t *cntB = cp ? e->cnt : e->cnt_alt;
  if (inplace) {
    B = A;
    slotB = slotA;
    offB = offA;
  }
  int p = 0, t = 0;
  for (size_t r = 0; r < e->runs.size(); ++r) {
    const EnsRun &R = e->runs[r];
    const int64_t w = R.g.w;
    float *fld = e->fld + R.fld_off;
    for (int s = 0; s < R.P.nsp; ++s, ++p) {
      Args32 &a = P->pair[p];
      const float2 *sc =
          reinterpret_cast<const float2 *>(e->scaled + R.sc_off + (int64_t)s * 6 * w);
      a.ebx = sc;
      a.ebz = sc + w;
      a.eby = sc + 2 * w;
      a.rho = fld + EM2G_RHO * w;
      a.jx = fld + EM2G_JXM * w;
      a.jy = fld + EM2G_JYM * w;
      a.jz = fld + EM2G_JZM * w;
      a.A = A;
      a.slotA = slotA;
      a.B = B;
      a.slotB = slotB;
      a.offA = offA + R.cell0[s];
      a.offB = offB + R.cell0[s];
      a.cursor = e->cursor + R.cell0[s];
      a.cnt_next = cntB + R.cell0[s];
      a.cap = e->cap;
      a.nx = R.g.nx;
      a.ny = R.g.ny;
      a.nxg = R.g.nxg;
      a.qd = (float)(R.P.q[s] * R.P.dn[s] / (R.P.dx * R.P.dy));
      a.dtdx = (float)(R.P.dt / R.P.dx);
      a.dtdy = (float)(R.P.dt / R.P.dy);
      a.c = (float)R.P.c;
      a.ake_partial = e->red + R.red_off[s];
      a.lost = e->dev_out + (int64_t)r * kEnsOut + kEnsLost;
      const int segs = (R.g.nx + cells - 1) / cells;
      P->tile0[p] = t;
      P->segs[p] = segs;
      t += segs * R.g.ny;
      K->partial[p] = a.ake_partial;
      K->count[p] = segs * R.g.ny * (threads / 32);
      K->scale[p] = R.P.am[s] * R.P.dn[s];
      K->out[p] = e->dev_out + (int64_t)r * kEnsOut + s;
    }
  }
  P->npairs = p;
  P->ntiles = t;
  P->tile0[p] = t;
  P->counter = e->counter;
}

}  // namespace
}  // namespace em2g

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
// and the relativistic Boris rotation on u.
//
// Work layout.  A CTA owns a row segment of TCX cells (32 or 64); G lanes
// (2, 4 or 8) own one cell and walk its particles G at a time, the next
// particle's state loaded while the current one runs.  The scaled fields the
// segment's particles can touch (x nodes x0-1 .. x0+TCX+3, y nodes y0-1 ..
// y0+4) are staged once in shared memory as (E, B) pairs of the three
// staggerings, each window entry holding the pairs of two neighbouring x
// nodes, so a gather is 9 shared float4 and 9 float2 loads (27 points).
// A particle still in
// the lane's cell adds its rho and J into a 49-value register block (Jx 4x3,
// Jy 3x4, Jz 3x3, rho 4x4) -- every lane runs the update, with zero charge
// where its particle is elsewhere or absent; the deposits of one outside it
// go onto its warp's stack in shared memory and are done with atomics 32 at
// a time, one per lane.  At the end of the cell the lanes write their blocks
// into the warp's (drained) stack and each lane of the cell's group adds
// whole rows over the group before adding them to the arrays once.  Cells
// are handled unwrapped (group cell + offset) and wrapped only where an array
// is indexed.  The gathers, the block updates, the weights and the move use
// sm_100a's packed FP32 pairs (f32x2).  Each particle is written to the other
// buffer grouped by the cell it started the step in, its position relative
// to that cell (front slots by a running count for the common in-cell case,
// back slots by an atomic for the rest), and the cells of the new positions
// are counted for the next step's offsets: the counting sort rides along
// with the push.  The cell a particle is counted in is always the one its
// stored FP32 offset reads back as (uploads and in-place writes keep to
// that), and a regrouping push writes nothing outside the buffer.  Between
// regroupings (the sort interval) the push updates particles in place.
#include <algorithm>
#include <memory>

#include "push_f32_body.cuh"

namespace em2g {
namespace {

// TCX cells per CTA (a row segment), G lanes per cell (the particles a CTA
// has in flight: TCX*G), MINB: CTAs per SM the register allocation must
// allow -- the autotuner's knobs besides the sort interval
template <int TCX, int G, int NC, int MINB, bool INPLACE>
__global__ void __launch_bounds__(TCX * G, MINB) k_push_cells_f32(Args32 a) {
  __shared__ float4 win[3][WY][NC * TCX + 5];
  __shared__ WarpScratch ws[TCX * G / 32];
  push_segment<TCX, G, NC, INPLACE>(a, (int)blockIdx.x * (NC * TCX), (int)blockIdx.y,
                                (int64_t)blockIdx.y * gridDim.x + blockIdx.x, win, ws);
}

// Ensemble: every (run, species) pair of an ensemble in one persistent
// launch.  The pairs' row segments are numbered one after the other
// (tile0[p] .. tile0[p+1]-1 for pair p, row-major within the pair); each
// CTA takes the next unclaimed segment from a counter until none is left,
// so runs of unequal size and density share the SMs without a tail per run.
// INPLACE as for single runs (the ensemble's sort interval).
template <int TCX, int G, int NC, int MINB, bool INPLACE>
__global__ void __launch_bounds__(TCX * G, MINB)
    k_ens_push_f32(const __grid_constant__ EnsPush32 e) {
  __shared__ float4 win[3][WY][NC * TCX + 5];
  __shared__ WarpScratch ws[TCX * G / 32];
  __shared__ int s_tile;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(e.counter, 1);
    __syncthreads();  // also: every thread is done with the last segment's window
    const int t = s_tile;
    if (t >= e.ntiles) break;
    int lo = 0, hi = e.npairs - 1;  // last pair p with tile0[p] <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (e.tile0[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int lt = t - e.tile0[lo];
    const int segs = e.segs[lo];
    const int row = lt / segs;
    push_segment<TCX, G, NC, INPLACE>(e.pair[lo], (lt - row * segs) * (NC * TCX), row, lt, win,
                                      ws);
  }
}

struct Variant32 {
  const char *name;
  int tcx, g;  // lanes per CTA: tcx * g
  int cells;   // cells per CTA (segment width): tcx * cells per group
  void (*kernel)(Args32);
  void (*kernel_inplace)(Args32);
  void (*ens_kernel)(const EnsPush32);
  void (*ens_kernel_inplace)(const EnsPush32);
};
#define EM2G_VARIANT32(T, GG, N, M)                                                        \
  {N == 1 ? "f32 tcx" #T " g" #GG " minb" #M : "f32 tcx" #T "x" #N " g" #GG " minb" #M, T, GG,  \
   T * N, k_push_cells_f32<T, GG, N, M, false>, k_push_cells_f32<T, GG, N, M, true>,           \
   k_ens_push_f32<T, GG, N, M, false>, k_ens_push_f32<T, GG, N, M, true>},
const Variant32 kVariants32[] = {EM2G_F32_VARIANTS(EM2G_VARIANT32)};
#undef EM2G_VARIANT32

// kinetic energy of every pair of an ensemble: block p sums pair p's
// partials in a fixed order (pic/move.f90:183, :208)
__global__ void __launch_bounds__(256) k_ens_ake(const __grid_constant__ EnsAke a) {
  __shared__ double red[8];
  const int p = blockIdx.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < a.count[p]; i += blockDim.x) v += a.partial[p][i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
    for (int o = 4; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) *a.out[p] = v * a.scale[p];
  }
}

// E and B times ae = 0.5*qm*dt/c into (E, B) pairs of the three staggerings
// (pic/move.f90:52-64)
__global__ void k_prescale_f32(const float *__restrict__ fld, float2 *__restrict__ s, int64_t w,
                               float ae, float tx, float ty) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= w) return;
  s[k] = make_float2(ae * fld[EM2G_EX * w + k], ae * fld[EM2G_BX * w + k] + tx);
  s[w + k] = make_float2(ae * fld[EM2G_EZ * w + k], ae * fld[EM2G_BZ * w + k]);
  s[2 * w + k] = make_float2(ae * fld[EM2G_EY * w + k], ae * fld[EM2G_BY * w + k] + ty);
}

// The cell and FP32 offset of an FP64 position x in [0, n + 1/2) of a
// periodic axis of n cells, as the push will read them back: the offset
// x - cell rounded to FP32 can come out as exactly 1, which the push takes
// for the next cell, so such a position is given to the next cell at offset
// 0 (a shift below 2^-25 cells).  The histogram and the scatter of an
// upload both use this, so that the counts match where particles go.
struct CellF32 {
  int c;    // cell, wrapped into 0 .. n-1
  float r;  // offset in [0, 1) relative to the unwrapped cell
};
__device__ __forceinline__ CellF32 cell_f32(double x, int n) {
  int c = (int)x;
  float r = (float)(x - c);
  if (r >= 1.0f) {
    c += 1;
    r = 0.0f;
  }
  if (c >= n) c -= n;
  return CellF32{c, r};
}

// FP64 (x, y, vx, vy, vz, gamma) staging -> histogram of cells
__global__ void k_hist64(const double *__restrict__ st, int64_t n, int nx, int ny,
                         int32_t *cnt) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = j < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const CellF32 cx = cell_f32(st[j], nx), cy = cell_f32(st[n + j], ny);
  agg_atomic_add(cnt, cy.c * nx + cx.c, am);
}

// Transfers between the caller's slot order and the cell-grouped layout
// (of a context, or of one (run, species) pair of an ensemble) go through
// one 32-byte record per particle (a whole
// sector, two 16-byte stores): moving a particle to a random position then
// writes one full sector, where six separate arrays would write six partial
// ones (each a read-modify-write in L2).  rec holds 2*n float4.
//
// FP64 slot-order staging -> records in cell-grouped order:
// (xr, yr, ux, uy), (uz, slot, 0, 0); record pos - base for buffer position
// pos (base: the pair's first position in an ensemble's buffers, else 0)
__global__ void k_scatter_rec(const double *__restrict__ st, int64_t n, int nx, int ny,
                              const int32_t *__restrict__ off, int32_t *cursor, int64_t base,
                              float4 *rec) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = j < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const CellF32 cx = cell_f32(st[j], nx), cy = cell_f32(st[n + j], ny);
  const int key = cy.c * nx + cx.c;
  const int64_t pos = (int64_t)off[key] + agg_atomic_add(cursor, key, am) - base;
  const double g = st[5 * n + j];
  rec[2 * pos] = make_float4(cx.r, cy.r, (float)(st[2 * n + j] * g), (float)(st[3 * n + j] * g));
  rec[2 * pos + 1] = make_float4((float)(st[4 * n + j] * g), __int_as_float((int32_t)j), 0.f, 0.f);
}

// records in cell-grouped order -> entries first.. of the FP32 particle
// arrays ((xr, yr, ux, uy) float4s, then uz) and slots
__global__ void k_rec_to_soa(const float4 *__restrict__ rec, int64_t n, float *P, int32_t *slot,
                             int64_t cap, int64_t first) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 a = rec[2 * i], b = rec[2 * i + 1];
  reinterpret_cast<float4 *>(P)[first + i] = a;
  P[4 * cap + first + i] = b.x;
  slot[first + i] = __float_as_int(b.y);
}

// cell-grouped FP32 -> records in slot order: (x, y) as doubles, wrapped
// into the box, then (ux, uy, uz, 0)
__global__ void k_grouped_to_rec(const float *__restrict__ P, const int32_t *__restrict__ slot,
                                 const int32_t *__restrict__ off, int64_t cap, int nx, int ny,
                                 float4 *rec) {
  const int64_t cell = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kCopyLanes;
  const int gl = threadIdx.x & (kCopyLanes - 1);
  if (cell >= (int64_t)nx * ny) return;
  const int kx = (int)(cell % nx), ky = (int)(cell / nx);
  for (int32_t i = off[cell] + gl; i < off[cell + 1]; i += kCopyLanes) {
    const float4 q = reinterpret_cast<const float4 *>(P)[i];
    double x = kx + (double)q.x, y = ky + (double)q.y;
    if (x < 0.0) x += nx;
    if (x >= nx) x -= nx;
    if (y < 0.0) y += ny;
    if (y >= ny) y -= ny;
    const int64_t s = slot[i];
    reinterpret_cast<double2 *>(rec)[2 * s] = make_double2(x, y);
    rec[2 * s + 1] = make_float4(q.z, q.w, P[4 * cap + i], 0.f);
  }
}

// records in slot order -> FP64 staging: x, y, vx, vy, vz, gamma
__global__ void k_rec_to_fp64(const float4 *__restrict__ rec, int64_t n, double *st) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const double2 xy = reinterpret_cast<const double2 *>(rec)[2 * s];
  const float4 u = rec[2 * s + 1];
  const double ux = u.x, uy = u.y, uz = u.z;
  const double g = sqrt(1.0 + ux * ux + uy * uy + uz * uz);
  st[s] = xy.x;
  st[n + s] = xy.y;
  st[2 * n + s] = ux / g;
  st[3 * n + s] = uy / g;
  st[4 * n + s] = uz / g;
  st[5 * n + s] = g;
}

// ---- a context's particle copies, in slices ------------------------------

struct Src6 {
  const double *a[6];  // x, y, vx, vy, vz, gamma; slot first+i at a[k][i]
};
struct Dst6 {
  double *a[6];
};

// Slots first..first+count of an upload: checked (every value finite,
// 0 <= x < xlim, 0 <= y < ylim), converted to the cell and FP32 offset the
// push reads back (cell_f32) and to u = gamma v, and parked unsorted at
// their slot in the alternate buffer P (offsets, u) with the cell's key in
// key; the cells are counted in cnt.  A rejected particle is counted in
// bad[0] (outside the grid) or bad[1] (non-finite) and parked with key -1.
__global__ void k_stage_f32(Src6 src, int64_t count, int64_t first, int nx, int ny, double xlim,
                            double ylim, float *P, int32_t *key, int64_t cap, int32_t *cnt,
                            unsigned long long *bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < count;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  double v[6];
  bool finite = true;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    v[k] = src.a[k][i];
    finite = finite && isfinite(v[k]);
  }
  const bool ok = finite && v[0] >= 0.0 && v[0] < xlim && v[1] >= 0.0 && v[1] < ylim;
  if (!finite) atomicAdd(bad + 1, 1ull);
  else if (!ok) atomicAdd(bad, 1ull);
  int k = -1;
  float xr = 0.f, yr = 0.f;
  if (ok) {
    const CellF32 cx = cell_f32(v[0], nx), cy = cell_f32(v[1], ny);
    k = cy.c * nx + cx.c;
    xr = cx.r;
    yr = cy.r;
  }
  const unsigned om = __ballot_sync(am, ok);
  if (ok) agg_atomic_add(cnt, k, om);
  const int64_t j = first + i;
  const double g = ok ? v[5] : 0.0;
  reinterpret_cast<float4 *>(P)[j] =
      make_float4(xr, yr, (float)(v[2] * g), (float)(v[3] * g));
  P[4 * cap + j] = (float)(v[4] * g);
  key[j] = k;
}

// parked particle i takes the next position of its cell's range: its key
// is replaced by that position
__global__ void k_place(int32_t *key, int64_t n, const int32_t *__restrict__ off,
                        int32_t *cursor) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const int k = key[i];
  key[i] = off[k] + agg_atomic_add(cursor, k, am);
}

// the parked particles whose position lies in [p0, p0+len): one 32-byte
// record each at rec[pos - p0], (xr, yr, ux, uy), (uz, slot, 0, 0)
__global__ void k_window_rec(const float *__restrict__ P, const int32_t *__restrict__ pos,
                             int64_t n, int64_t cap, int64_t p0, int64_t len, float4 *rec) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t q = (int64_t)pos[i] - p0;
  if (q < 0 || q >= len) return;
  rec[2 * q] = reinterpret_cast<const float4 *>(P)[i];
  rec[2 * q + 1] = make_float4(P[4 * cap + i], __int_as_float((int32_t)i), 0.f, 0.f);
}

// cell-grouped FP32 -> records of the slots in [s0, s0+len), rec[slot - s0]:
// (x, y) as doubles wrapped into the box, then (ux, uy, uz, 0)
__global__ void k_grouped_to_rec_range(const float *__restrict__ P,
                                       const int32_t *__restrict__ slot,
                                       const int32_t *__restrict__ off, int64_t cap, int nx,
                                       int ny, int64_t s0, int64_t len, float4 *rec) {
  const int64_t cell = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kCopyLanes;
  const int gl = threadIdx.x & (kCopyLanes - 1);
  if (cell >= (int64_t)nx * ny) return;
  const int kx = (int)(cell % nx), ky = (int)(cell / nx);
  for (int32_t i = off[cell] + gl; i < off[cell + 1]; i += kCopyLanes) {
    const int64_t q = (int64_t)slot[i] - s0;
    if (q < 0 || q >= len) continue;
    const float4 p = reinterpret_cast<const float4 *>(P)[i];
    double x = kx + (double)p.x, y = ky + (double)p.y;
    if (x < 0.0) x += nx;
    if (x >= nx) x -= nx;
    if (y < 0.0) y += ny;
    if (y >= ny) y -= ny;
    reinterpret_cast<double2 *>(rec)[2 * q] = make_double2(x, y);
    rec[2 * q + 1] = make_float4(p.z, p.w, P[4 * cap + i], 0.f);
  }
}

// records in slot order -> six FP64 arrays: x, y, vx, vy, vz, gamma
__global__ void k_rec_to_dst(const float4 *__restrict__ rec, int64_t len, Dst6 d) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= len) return;
  const double2 xy = reinterpret_cast<const double2 *>(rec)[2 * s];
  const float4 u = rec[2 * s + 1];
  const double ux = u.x, uy = u.y, uz = u.z;
  const double g = sqrt(1.0 + ux * ux + uy * uy + uz * uz);
  d.a[0][s] = xy.x;
  d.a[1][s] = xy.y;
  d.a[2][s] = ux / g;
  d.a[3][s] = uy / g;
  d.a[4][s] = uz / g;
  d.a[5][s] = g;
}

}  // namespace

int num_variants_f32() { return (int)(sizeof(kVariants32) / sizeof(kVariants32[0])); }
const char *variant_name_f32(int v) { return kVariants32[v].name; }

int launch_prescale_f32(em2g_ctx *c, int isp) {
  const double ae = 0.5 * c->P.qm[isp] * c->P.dt / c->P.c;
  const int64_t w = c->g.w;
  k_prescale_f32<<<(unsigned)((w + 255) / 256), 256, 0, c->stream>>>(
      c->fld32, reinterpret_cast<float2 *>(c->scaled32 + (int64_t)isp * 6 * w), w, (float)ae,
      (float)c->P.tx[isp], (float)c->P.ty[isp]);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int launch_push_cells_f32(em2g_ctx *c, int isp) {
  Species &S = c->sp[isp];
  const int64_t w = c->g.w;
  const float2 *sc = reinterpret_cast<const float2 *>(c->scaled32 + (int64_t)isp * 6 * w);
  Args32 a;
  a.ebx = sc;
  a.ebz = sc + w;
  a.eby = sc + 2 * w;
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
  a.lost = c->dev_out + kDevLost;
  const Variant32 &V = kVariants32[c->variant < num_variants_f32() ? c->variant : 0];
  const int threads = V.tcx * V.g;
  const dim3 grid((unsigned)((c->g.nx + V.cells - 1) / V.cells), (unsigned)c->g.ny);
  const int64_t nparts = (int64_t)grid.x * grid.y * (threads / 32);
  if (nparts > c->red_blocks) return fail(EM2G_ERR_RANGE, "grid exceeds reduction scratch");
  const int nb = (int)nparts;
  // regroup on every sort_interval-th push (every push for 0 or 1); the
  // pushes in between update the particles in place
  const bool inplace = c->P.sort_interval > 1 && S.since_sort + 1 < c->P.sort_interval;
  int rc;
  if (inplace) {
    a.B = S.p32;
    ++S.since_sort;
  } else {
    if ((rc = scan_cells(c, S.cnt, S.off_alt))) return rc;
    EM2G_CUDA(cudaMemsetAsync(S.cursor, 0, sizeof(int32_t) * c->ncell, c->stream));
    S.since_sort = 0;
  }
  EM2G_CUDA(cudaMemsetAsync(S.cnt_alt, 0, sizeof(int32_t) * c->ncell, c->stream));
  if ((rc = timing_begin(c))) return rc;
  (inplace ? V.kernel_inplace : V.kernel)<<<grid, threads, 0, c->stream>>>(a);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  if ((rc = timing_end(c))) return rc;
  if (!inplace) {
    std::swap(S.p32, S.p32_alt);
    std::swap(S.slot, S.slot_alt);
    std::swap(S.off, S.off_alt);
  }
  std::swap(S.cnt, S.cnt_alt);
  return launch_ake_finish(c, isp, nb);
}

int stage_f32(em2g_ctx *c, int isp, int64_t first, int64_t count, const double *const *src,
              unsigned long long *bad) {
  Species &S = c->sp[isp];
  if (count <= 0) return EM2G_OK;
  Src6 a;
  for (int k = 0; k < 6; ++k) a.a[k] = src[k];
  k_stage_f32<<<(unsigned)((count + 255) / 256), 256, 0, c->stream>>>(
      a, count, first, c->g.nx, c->g.ny, c->P.nx + 0.5, c->P.ny + 0.5, S.p32_alt, S.slot_alt,
      S.cap, S.cnt_alt, bad);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

// The parked particles become the species' particles, grouped by cell:
// offsets from the counts, a position for every particle, then the records
// of one window of positions at a time, each window moved into the arrays
// by a coalesced pass.
int commit_f32(em2g_ctx *c, int isp, int64_t n, void *rec, int64_t rec_cap) {
  Species &S = c->sp[isp];
  std::swap(S.cnt, S.cnt_alt);  // the counts of the parked positions
  int rc = scan_cells(c, S.cnt, S.off);
  if (rc) return rc;
  EM2G_CUDA(cudaMemsetAsync(S.cursor, 0, sizeof(int32_t) * c->ncell, c->stream));
  if (n > 0) {
    const unsigned nb = (unsigned)((n + 255) / 256);
    k_place<<<nb, 256, 0, c->stream>>>(S.slot_alt, n, S.off, S.cursor);
    EM2G_CUDA(cudaGetLastError());
    c->launches += 1;
    float4 *r = static_cast<float4 *>(rec);
    for (int64_t p0 = 0; p0 < n; p0 += rec_cap) {
      const int64_t len = std::min(rec_cap, n - p0);
      k_window_rec<<<nb, 256, 0, c->stream>>>(S.p32_alt, S.slot_alt, n, S.cap, p0, len, r);
      k_rec_to_soa<<<(unsigned)((len + 255) / 256), 256, 0, c->stream>>>(r, len, S.p32, S.slot,
                                                                          S.cap, p0);
      EM2G_CUDA(cudaGetLastError());
      c->launches += 2;
    }
  }
  S.n = n;
  S.sorted = true;
  S.since_sort = 0;
  return EM2G_OK;
}

int get_range_f32(em2g_ctx *c, int isp, int64_t first, int64_t count, double *const *dst,
                  void *rec) {
  Species &S = c->sp[isp];
  if (count <= 0) return EM2G_OK;
  float4 *r = static_cast<float4 *>(rec);
  const int64_t nb = (c->ncell * kCopyLanes + 255) / 256;
  k_grouped_to_rec_range<<<(unsigned)nb, 256, 0, c->stream>>>(S.p32, S.slot, S.off, S.cap,
                                                               c->g.nx, c->g.ny, first, count, r);
  EM2G_CUDA(cudaGetLastError());
  Dst6 d;
  for (int k = 0; k < 6; ++k) d.a[k] = dst[k];
  k_rec_to_dst<<<(unsigned)((count + 255) / 256), 256, 0, c->stream>>>(r, count, d);
  EM2G_CUDA(cudaGetLastError());
  c->launches += 2;
  return EM2G_OK;
}

// ---- ensembles (ensemble_api.cu) ---------------------------------------

// One push of every pair: for a regrouping push, offsets of the next
// grouping from the current counts (one scan over all pairs); the
// persistent push; the kinetic energies.  bp selects the current particle
// buffers and offsets, cp the current cell counts (which change on every
// push, where the buffers change only on regrouping pushes); an in-place
// push updates the current buffers.
int ens_push(em2g_ens *e, int bp, int cp, bool inplace) {
  int32_t *offB = bp ? e->off : e->off_alt;  // the next grouping's offsets
  int32_t *cntA = cp ? e->cnt_alt : e->cnt, *cntB = cp ? e->cnt : e->cnt_alt;
  const Variant32 &V = kVariants32[e->variant < num_variants_f32() ? e->variant : 0];
  const int threads = V.tcx * V.g;
  cudaStream_t st = e->stream;
  int rc;
  if (!inplace) {
    if ((rc = scan_counts(cntA, offB, e->ncell, 0, e->scan_tmp, st))) return rc;
    EM2G_CUDA(cudaMemsetAsync(e->cursor, 0, sizeof(int32_t) * e->ncell, st));
  }
  EM2G_CUDA(cudaMemsetAsync(cntB, 0, sizeof(int32_t) * e->ncell, st));
  EM2G_CUDA(cudaMemsetAsync(e->counter, 0, sizeof(int), st));
  std::unique_ptr<EnsPush32> P(new EnsPush32());
  std::unique_ptr<EnsAke> K(new EnsAke());
  ens_push_tables(e, bp, cp, inplace, V.cells, threads, P.get(), K.get());
  const int t = P->ntiles, p = P->npairs;
  int per_sm = 0;
  auto kernel = inplace ? V.ens_kernel_inplace : V.ens_kernel;
  EM2G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
  if (per_sm < 1) return fail(EM2G_ERR_CUDA, "ensemble push kernel cannot be resident");
  const int blocks = std::min(per_sm * e->num_sms, t);
  kernel<<<blocks, threads, 0, st>>>(*P);
  k_ens_ake<<<p, 256, 0, st>>>(*K);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

// pair (r, s) from FP64 staging (6*n doubles, slot order, then 32*n bytes
// for the records) into the current buffers: histogram, this pair's
// offsets from its first position, records in cell order, transpose
int ens_upload_pair(em2g_ens *e, int r, int s, double *staging) {
  const EnsRun &R = e->runs[r];
  const int64_t n = R.n[s], nc = (int64_t)R.g.nx * R.g.ny, c0 = R.cell0[s];
  float *P = e->parity ? e->p32_alt : e->p32;
  int32_t *slot = e->parity ? e->slot_alt : e->slot;
  int32_t *off = e->parity ? e->off_alt : e->off;
  int32_t *cnt = e->cparity ? e->cnt_alt : e->cnt;
  cudaStream_t st = e->stream;
  EM2G_CUDA(cudaMemsetAsync(cnt + c0, 0, sizeof(int32_t) * nc, st));
  EM2G_CUDA(cudaMemsetAsync(e->cursor + c0, 0, sizeof(int32_t) * nc, st));
  const unsigned nb = (unsigned)((n + 255) / 256);
  if (n > 0) k_hist64<<<nb, 256, 0, st>>>(staging, n, R.g.nx, R.g.ny, cnt + c0);
  int rc = scan_counts(cnt + c0, off + c0, nc, (int32_t)R.base[s], e->scan_tmp, st);
  if (rc) return rc;
  if (n > 0) {
    float4 *rec = reinterpret_cast<float4 *>(staging + 6 * n);
    k_scatter_rec<<<nb, 256, 0, st>>>(staging, n, R.g.nx, R.g.ny, off + c0, e->cursor + c0,
                                      R.base[s], rec);
    EM2G_CUDA(cudaGetLastError());
    k_rec_to_soa<<<nb, 256, 0, st>>>(rec, n, P, slot, e->cap, R.base[s]);
  }
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

// pair (r, s) from the current buffers to FP64 staging in slot order
// (6*n doubles, then 32*n bytes for the records)
int ens_download_pair(em2g_ens *e, int r, int s, double *staging) {
  const EnsRun &R = e->runs[r];
  const int64_t n = R.n[s];
  if (n == 0) return EM2G_OK;
  const float *P = e->parity ? e->p32_alt : e->p32;
  const int32_t *slot = e->parity ? e->slot_alt : e->slot;
  const int32_t *off = e->parity ? e->off_alt : e->off;
  float4 *rec = reinterpret_cast<float4 *>(staging + 6 * n);
  const int64_t nb = ((int64_t)R.g.nx * R.g.ny * kCopyLanes + 255) / 256;
  k_grouped_to_rec<<<(unsigned)nb, 256, 0, e->stream>>>(P, slot, off + R.cell0[s], e->cap, R.g.nx,
                                                         R.g.ny, rec);
  EM2G_CUDA(cudaGetLastError());
  k_rec_to_fp64<<<(unsigned)((n + 255) / 256), 256, 0, e->stream>>>(rec, n, staging);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

// kernels one ens_push enqueues: scan (3, regrouping pushes only), push,
// kinetic energies
int ens_push_kernels_per_step(const em2g_ens *, bool inplace) { return inplace ? 2 : 5; }

}  // namespace em2g

// tma_stencil.cuh -- em2's Yee updates and smooth2 passes (pic/fields.f90:
// 184-247, pic/smooth.f90:143-177) as TMA-staged tiles: a persistent CTA per
// SM walks the grid's tiles, each tile's input arrays (with a one-cell halo)
// brought into shared memory by tensor copies on an mbarrier while the CTA
// computes the tile before it (two stages).  The arithmetic is grid_kernels'
// value functions, so every cell rounds as the direct-load kernels round it.
//
// The layout at the ABI is em2's: rows of (nx+3) elements, so a row starts on
// any 4- or 8-byte boundary, and a tensor map's row stride must be a multiple
// of 16 bytes.  So a map's rows ("lines") here are M = 16/sizeof(T)
// consecutive field rows: M(nx+3) elements, a stride of 16(nx+3) bytes for
// any nx.  Field row R of a block of arrays (R = k(ny+3) + iy for array k)
// lies in line R/M from column (R%M)(nx+3).  A tile's rows iy0-1 .. iy0+TYO
// come from M boxes: box j holds rows iy0-1+j, iy0-1+j+M, ..; it starts at
// its first row's column ix0-1 rounded down to a multiple of M elements (the
// 16-byte rule of a tiled copy's x coordinate), so its column ix0-1 sits
// shift_j = (r_j(nx+3)) mod M elements in (r_j: the row's residue R mod M).
// Boxes may run past a line's end or the map's last line: those elements are
// zero-filled by the copy and never read.
//
// The map covers the block rounded up to whole lines, so the allocations
// behind it carry a tail of M rows (tail_elems).
#pragma once
#include <cuda.h>

#include "grid_kernels.cuh"

namespace em2g {
namespace tma {
namespace {

template <typename T>
struct Geo {
  static constexpr int M = 16 / (int)sizeof(T);  // field rows per line
  static constexpr int TXO = sizeof(T) == 4 ? 64 : 32;  // output columns per tile
  static constexpr int TYO = 16;                         // output rows per tile
  static constexpr int THREADS = 256;
  static constexpr int RT = THREADS / TXO;  // rows of threads
  static constexpr int HR = TYO + 2;        // staged rows: iy0-1 .. iy0+TYO
  static constexpr int BH = (HR + M - 1) / M;  // box rows (lines)
  // box columns: ix0-1 .. ix0+TXO plus up to M-1 of alignment shift
  static constexpr int BW = (TXO + 2 + M - 1 + M - 1) / M * M;
  static constexpr int BOX_BYTES = BW * BH * (int)sizeof(T);
  static constexpr int SLOT = (BOX_BYTES + 127) / 128 * 128;  // 128-byte aligned boxes
  static constexpr int ARRAY_BYTES = M * SLOT;
  static_assert(BW <= 256 && BH <= 256, "box dimensions are limited to 256");
  static_assert((BW * sizeof(T)) % 16 == 0, "a box row must be a multiple of 16 bytes");
  static_assert(TXO % M == 0, "tile origins ix0-1 must be multiples of M");
  static_assert(TYO % RT == 0, "rows of threads divide the tile");
};

// elements of tail an allocation needs behind a block of arrays for the map
template <typename T>
inline int64_t tail_elems(int nxg) { return (int64_t)Geo<T>::M * nxg; }

enum Stage { kBHalf = 0, kEFull = 1, kBinomial = 2, kCompensate = 3 };
constexpr int kMaxStaged = 12;
// staged arrays per stage: B/2: ex ey ez (halo), bx by bz; E: bx by bz
// (halo), ex ey ez, jxm jxp jym jyp jzm jzp; smooth2 passes: the source
template <int S>
struct Staged {
  static constexpr int N = S == kBHalf ? 6 : (S == kEFull ? 12 : 1);
};

template <typename T>
struct Args {
  grid::G g;
  int ntx, nty, ntiles;
  int row0[kMaxStaged];  // each staged array's row 0 in the map's rows
  T *out[3];             // arrays written (with em2's guard copies)
  T c0, c1, c2;          // B/2: ctxh, ctyh; E: ctx, cty, tem
  int *status;           // bit 1 set when a wait for a tile timed out
};

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// wait for a phase with a bound of about a second; false on timeout
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > 1000000000ull) return false;
  }
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// tile t's origin: output cells ix0 .. ix0+TXO-1, iy0 .. iy0+TYO-1
template <typename T>
__device__ __forceinline__ void tile_origin(const Args<T> &a, int t, int &ix0, int &iy0) {
  ix0 = 1 + (t % a.ntx) * Geo<T>::TXO;
  iy0 = 1 + (t / a.ntx) * Geo<T>::TYO;
}

// Issue the boxes of tile t into stage buffer `buf` (warp 0; lane 0 sets
// the byte count first).  Box b = (staged array, j).
template <typename T, int S>
__device__ __forceinline__ void issue_tile(const Args<T> &a, const CUtensorMap *map, int t,
                                           unsigned char *buf, uint64_t *bar) {
  using Gm = Geo<T>;
  constexpr int NB = Staged<S>::N * Gm::M;
  const int lane = threadIdx.x & 31;
  if (lane == 0) mbar_expect_tx(bar, (unsigned)(NB * Gm::BOX_BYTES));
  __syncwarp();
  int ix0, iy0;
  tile_origin(a, t, ix0, iy0);
  for (int b = lane; b < NB; b += 32) {
    const int arr = b / Gm::M, j = b % Gm::M;
    const int R = a.row0[arr] + iy0 - 1 + j;  // >= 0: iy0 >= 1
    const int line = R / Gm::M, r = R % Gm::M;
    int x = r * a.g.nxg + ix0 - 1;
    x -= x % Gm::M;
    tma_load_2d(buf + (arr * Gm::M + j) * Gm::SLOT, map, x, line, bar);
  }
}

// Row dy (0 = iy0-1) of staged array `arr` of a tile whose first staged row
// has residue rb = (row0 + iy0 - 1) mod M: element dx (0 = ix0-1) is at [dx].
template <typename T>
__device__ __forceinline__ const T *staged_row(const unsigned char *buf, int arr, int dy, int rb,
                                               int nxg) {
  using Gm = Geo<T>;
  const int j = dy % Gm::M, tr = dy / Gm::M;
  const int r = (rb + j) % Gm::M;
  const int sh = (r * nxg) % Gm::M;
  return reinterpret_cast<const T *>(buf + (arr * Gm::M + j) * Gm::SLOT) + tr * Gm::BW + sh;
}

template <typename T, int S>
__device__ __forceinline__ void compute_tile(const Args<T> &a, int t, const unsigned char *buf) {
  using Gm = Geo<T>;
  constexpr int N = Staged<S>::N;
  int ix0, iy0;
  tile_origin(a, t, ix0, iy0);
  const int nxg = a.g.nxg;
  int rb[N];
#pragma unroll
  for (int k = 0; k < N; ++k) rb[k] = (a.row0[k] + iy0 - 1) % Gm::M;
  const int txl = threadIdx.x % Gm::TXO, tyl = threadIdx.x / Gm::TXO;
  const int ix = ix0 + txl, dx = txl + 1;
  if (ix > a.g.nx + 1) return;
#pragma unroll
  for (int q = 0; q < Gm::TYO / Gm::RT; ++q) {
    const int oy = tyl + q * Gm::RT, iy = iy0 + oy, dy = oy + 1;
    if (iy > a.g.ny + 1) break;
    if constexpr (S == kBHalf) {
      // staged: 0 ex, 1 ey, 2 ez, 3 bx, 4 by, 5 bz
      const T *exc = staged_row<T>(buf, 0, dy, rb[0], nxg);
      const T *exn = staged_row<T>(buf, 0, dy + 1, rb[0], nxg);
      const T *eyc = staged_row<T>(buf, 1, dy, rb[1], nxg);
      const T *ezc = staged_row<T>(buf, 2, dy, rb[2], nxg);
      const T *ezs = staged_row<T>(buf, 2, dy - 1, rb[2], nxg);
      const T *bxc = staged_row<T>(buf, 3, dy, rb[3], nxg);
      const T *byc = staged_row<T>(buf, 4, dy, rb[4], nxg);
      const T *bzc = staged_row<T>(buf, 5, dy, rb[5], nxg);
      T vbx, vby, vbz;
      grid::b_half_vals(bxc[dx], byc[dx], bzc[dx], ezc[dx], ezs[dx], ezc[dx - 1], eyc[dx + 1],
                        eyc[dx], exn[dx], exc[dx], a.c0, a.c1, vbx, vby, vbz);
      grid::store_with_guards(a.g, a.out[0], ix, iy, vbx);
      grid::store_with_guards(a.g, a.out[1], ix, iy, vby);
      grid::store_with_guards(a.g, a.out[2], ix, iy, vbz);
    } else if constexpr (S == kEFull) {
      // staged: 0 bx, 1 by, 2 bz, 3 ex, 4 ey, 5 ez, 6 jxm, 7 jxp, 8 jym, 9 jyp,
      // 10 jzm, 11 jzp
      const T *bxc = staged_row<T>(buf, 0, dy, rb[0], nxg);
      const T *bxn = staged_row<T>(buf, 0, dy + 1, rb[0], nxg);
      const T *byc = staged_row<T>(buf, 1, dy, rb[1], nxg);
      const T *bzc = staged_row<T>(buf, 2, dy, rb[2], nxg);
      const T *bzs = staged_row<T>(buf, 2, dy - 1, rb[2], nxg);
      T v[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) v[k] = staged_row<T>(buf, 3 + k, dy, rb[3 + k], nxg)[dx];
      T vex, vey, vez;
      grid::e_full_vals(v[0], v[1], v[2], bzc[dx], bzs[dx], bzc[dx - 1], byc[dx + 1], byc[dx],
                        bxn[dx], bxc[dx], v[3], v[4], v[5], v[6], v[7], v[8], a.c0, a.c1, a.c2,
                        vex, vey, vez);
      grid::store_with_guards(a.g, a.out[0], ix, iy, vex);
      grid::store_with_guards(a.g, a.out[1], ix, iy, vey);
      grid::store_with_guards(a.g, a.out[2], ix, iy, vez);
    } else {
      const T *rs = staged_row<T>(buf, 0, dy - 1, rb[0], nxg);
      const T *rc = staged_row<T>(buf, 0, dy, rb[0], nxg);
      const T *rn = staged_row<T>(buf, 0, dy + 1, rb[0], nxg);
      T v;
      if constexpr (S == kBinomial)
        v = grid::binomial_val(rc[dx], rc[dx - 1], rc[dx + 1], rs[dx], rn[dx], rs[dx - 1],
                               rn[dx - 1], rs[dx + 1], rn[dx + 1]);
      else
        v = grid::compensate_val(rc[dx], rc[dx - 1], rc[dx + 1], rs[dx], rn[dx], rs[dx - 1],
                                 rn[dx - 1], rs[dx + 1], rn[dx + 1]);
      grid::store_with_guards(a.g, a.out[0], ix, iy, v);
    }
  }
}

// smem per CTA: two stage buffers and two mbarriers
template <typename T, int S>
constexpr int smem_bytes() {
  return 2 * Staged<S>::N * Geo<T>::ARRAY_BYTES + 128;
}

// The persistent stage kernel: CTA c takes tiles c, c+grid, ..; tile i+1's
// boxes are in flight while tile i is computed.  One barrier per tile: after
// the wait for tile i (a vote, so that a timeout ends every thread's loop at
// the same point) every thread is done reading tile i-1's buffer, which then
// takes tile i+1's boxes.  A wait that times out sets bit 1 of *status; the
// CTA then waits (bounded) for the copies it issued and stops.
template <typename T, int S>
__global__ void __launch_bounds__(256) k_tma_stage(const __grid_constant__ CUtensorMap map,
                                                   const Args<T> a) {
  using Gm = Geo<T>;
  constexpr int STAGE_BYTES = Staged<S>::N * Gm::ARRAY_BYTES;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * STAGE_BYTES);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int t = blockIdx.x;
  if (t >= a.ntiles) return;
  if (threadIdx.x < 32) issue_tile<T, S>(a, &map, t, smem, &bar[0]);
  for (int i = 0; t < a.ntiles; t += gridDim.x, ++i) {
    const int s = i & 1;
    const unsigned parity = (unsigned)((i >> 1) & 1);
    const bool ok = mbar_wait_bounded(&bar[s], parity);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(a.status, 2);
      mbar_wait_bounded(&bar[s], parity);  // the only copies in flight: tile i's
      return;
    }
    const int tn = t + gridDim.x;
    if (threadIdx.x < 32 && tn < a.ntiles) {
      // order every thread's reads of this buffer (tile i-1) before the copies
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_tile<T, S>(a, &map, tn, smem + (s ^ 1) * STAGE_BYTES, &bar[s ^ 1]);
    }
    compute_tile<T, S>(a, t, smem + s * STAGE_BYTES);
  }
}

}  // namespace
}  // namespace tma
}  // namespace em2g

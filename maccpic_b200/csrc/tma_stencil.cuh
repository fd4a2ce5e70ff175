// tma_stencil.cuh -- em2's Yee updates and smooth2 passes (pic/fields.f90:
// 184-247, pic/smooth.f90:143-177) as TMA-staged tiles: a CTA per tile, the
// arrays a stage reads at neighbouring cells brought into shared memory with
// a one-cell halo by tensor copies on an mbarrier.  The arithmetic is
// grid_kernels' value functions, so every cell rounds as the direct-load
// kernels round it.
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
// behind it carry a tail of M rows (em2g_internal.cuh, tma_tail_elems).
#pragma once
#include <cuda.h>

#include "grid_kernels.cuh"

namespace em2g {
namespace tma {
namespace {

// Tiles of TXO x TYO cells, 256 threads (RT rows of TXO), each thread
// ROWS cells of one column.
template <typename T>
struct Geo {
  static constexpr int M = 16 / (int)sizeof(T);  // field rows per line
  static constexpr int TXO = sizeof(T) == 4 ? 64 : 32;  // output columns per tile
  static constexpr int TYO = 16;                         // output rows per tile
  static constexpr int THREADS = 256;
  static constexpr int RT = THREADS / TXO;  // rows of threads
  static constexpr int ROWS = TYO / RT;      // cells per thread
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

enum Stage { kBHalf = 0, kEFull = 1, kBinomial = 2, kCompensate = 3 };
// Only the arrays a stage reads at neighbouring cells go through shared
// memory: E for B/2 (pic/fields.f90:188-190), B for E (:211-215), the source
// of a smooth2 pass.  The arrays read at the cell itself are loaded directly
// (one coalesced load per cell, no reuse to stage).
constexpr int kStaged = 3;
template <int S>
struct Staged {
  static constexpr int N = (S == kBHalf || S == kEFull) ? 3 : 1;
  static constexpr int NIN = S == kBHalf ? 3 : (S == kEFull ? 9 : 1);  // read at the cell
};

template <typename T>
struct Args {
  grid::G g;
  int ntx, nty, ntiles;
  int row0[kStaged];  // each staged array's row 0 in the map's rows
  const T *in[9];     // arrays read at the cell: B/2: bx by bz; E: ex ey ez jxm jxp jym jyp jzm jzp
  T *out[3];          // arrays written (with em2's guard copies)
  T c0, c1, c2;       // B/2: ctxh, ctyh; E: ctx, cty, tem
  int *status;        // bit 1 set when a wait for a tile timed out
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

// A probe of the bounded tile wait: an mbarrier that no copy and no thread
// completes, so the wait runs out after its bound and bit 1 of *status is
// set, as a stage kernel does on a timeout (em2g_selftest_waits).
__global__ void k_tma_wait_probe(int *status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (!mbar_wait_bounded(&bar, 0) && threadIdx.x == 0) atomicOr(status, 2);
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

// The arrays a stage reads at its cells, loaded before the tile's boxes
// land: cell value q of this thread's column (row tyl + q RT of the tile).
template <typename T, int S>
__device__ __forceinline__ void load_cells(const Args<T> &a, int t,
                                           T (&cv)[Staged<S>::NIN][Geo<T>::ROWS]) {
  using Gm = Geo<T>;
  int ix0, iy0;
  tile_origin(a, t, ix0, iy0);
  const int txl = threadIdx.x % Gm::TXO, tyl = threadIdx.x / Gm::TXO;
  const int ix = ix0 + txl;
#pragma unroll
  for (int q = 0; q < Gm::ROWS; ++q) {
    const int iy = iy0 + tyl + q * Gm::RT;
    const bool in = ix <= a.g.nx + 1 && iy <= a.g.ny + 1;
    const int64_t c = grid::at(a.g, in ? ix : 1, in ? iy : 1);
#pragma unroll
    for (int k = 0; k < Staged<S>::NIN; ++k)
      if constexpr (S == kBHalf || S == kEFull) cv[k][q] = a.in[k][c];
  }
}

template <typename T, int S>
__device__ __forceinline__ void compute_tile(const Args<T> &a, int t, const unsigned char *buf,
                                             const T (&cv)[Staged<S>::NIN][Geo<T>::ROWS]) {
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
  for (int q = 0; q < Gm::ROWS; ++q) {
    const int oy = tyl + q * Gm::RT, iy = iy0 + oy, dy = oy + 1;
    if (iy > a.g.ny + 1) break;
    if constexpr (S == kBHalf) {
      // staged: 0 ex, 1 ey, 2 ez; at the cell: bx, by, bz
      const T *exc = staged_row<T>(buf, 0, dy, rb[0], nxg);
      const T *exn = staged_row<T>(buf, 0, dy + 1, rb[0], nxg);
      const T *eyc = staged_row<T>(buf, 1, dy, rb[1], nxg);
      const T *ezc = staged_row<T>(buf, 2, dy, rb[2], nxg);
      const T *ezs = staged_row<T>(buf, 2, dy - 1, rb[2], nxg);
      T vbx, vby, vbz;
      grid::b_half_vals(cv[0][q], cv[1][q], cv[2][q], ezc[dx], ezs[dx], ezc[dx - 1], eyc[dx + 1],
                        eyc[dx], exn[dx], exc[dx], a.c0, a.c1, vbx, vby, vbz);
      grid::store_with_guards(a.g, a.out[0], ix, iy, vbx);
      grid::store_with_guards(a.g, a.out[1], ix, iy, vby);
      grid::store_with_guards(a.g, a.out[2], ix, iy, vbz);
    } else if constexpr (S == kEFull) {
      // staged: 0 bx, 1 by, 2 bz; at the cell: ex ey ez jxm jxp jym jyp jzm jzp
      const T *bxc = staged_row<T>(buf, 0, dy, rb[0], nxg);
      const T *bxn = staged_row<T>(buf, 0, dy + 1, rb[0], nxg);
      const T *byc = staged_row<T>(buf, 1, dy, rb[1], nxg);
      const T *bzc = staged_row<T>(buf, 2, dy, rb[2], nxg);
      const T *bzs = staged_row<T>(buf, 2, dy - 1, rb[2], nxg);
      T vex, vey, vez;
      grid::e_full_vals(cv[0][q], cv[1][q], cv[2][q], bzc[dx], bzs[dx], bzc[dx - 1], byc[dx + 1],
                        byc[dx], bxn[dx], bxc[dx], cv[3][q], cv[4][q], cv[5][q], cv[6][q],
                        cv[7][q], cv[8][q], a.c0, a.c1, a.c2, vex, vey, vez);
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

// shared memory per CTA: the staged boxes and the mbarrier
template <typename T, int S>
constexpr int smem_bytes() {
  return Staged<S>::N * Geo<T>::ARRAY_BYTES + 128;
}

// One tile per CTA, as many CTAs resident per SM as the shared memory
// allows, so that the tiles' copies overlap one another.  Warp 0 issues the
// tile's boxes; every thread loads the values it reads at its cells while
// they are in flight, waits for the boxes (bounded: a timeout sets bit 1 of
// *status and, after a second bounded wait for the copies, ends the thread)
// and computes its cells.
template <typename T, int S>
__global__ void __launch_bounds__(256) k_tma_stage(const __grid_constant__ CUtensorMap map,
                                                   const Args<T> a) {
  using Gm = Geo<T>;
  constexpr int STAGE_BYTES = Staged<S>::N * Gm::ARRAY_BYTES;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES);
  const int t = blockIdx.x;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x < 32) issue_tile<T, S>(a, &map, t, smem, bar);
  T cv[Staged<S>::NIN][Gm::ROWS];
  load_cells<T, S>(a, t, cv);
  if (!mbar_wait_bounded(bar, 0)) {
    atomicOr(a.status, 2);
    mbar_wait_bounded(bar, 0);
    return;
  }
  compute_tile<T, S>(a, t, smem, cv);
}

}  // namespace
}  // namespace tma
}  // namespace em2g

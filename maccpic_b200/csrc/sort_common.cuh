// sort_common.cuh -- cell keys and warp-aggregated counters shared by the
// cell sort (sort.cu) and the fast push (push_fast_f64.cu).
#pragma once
#include <stdint.h>

namespace em2g {

// Row-major key iy*nx + ix of the cell holding (x, y).  Positions up to n+0.5
// (em2's loader can leave a row there; its guard cells absorb it) are keyed
// to their periodic image.
__device__ __forceinline__ int cell_key(double x, double y, int nx, int ny) {
  int cx = (int)x, cy = (int)y;
  if (cx >= nx) cx -= nx;
  if (cy >= ny) cy -= ny;
  return cy * nx + cx;
}

// atomicAdd(ctr + key, 1) for every active lane, issued once per distinct key
// among the lanes in `active`; returns this lane's old value + its rank among
// the lanes with the same key.  All lanes in `active` must call it.
__device__ __forceinline__ int agg_atomic_add(int32_t *ctr, int key, unsigned active) {
  const unsigned m = __match_any_sync(active, key);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(ctr + key, __popc(m));
  base = __shfl_sync(m, base, leader);
  return base + __popc(m & ((1u << lane) - 1u));
}

}  // namespace em2g

// sort.cu -- counting sort of particles by cell for the fast path.
//
// The fast push (push_fast_f64.cu) reads particles cell by cell and writes
// them back grouped by the cell they were in when the step began, so after
// every step the particle arrays are again ordered by cell up to the few
// particles that crossed a cell edge during that step.  This file holds the
// pieces around it: the exclusive scan of per-cell counts into offsets, and
// the full counting sort used once after particles are uploaded.
#include "em2g_internal.cuh"
#include "sort_common.cuh"

namespace em2g {
namespace {

constexpr int kScanBlock = 1024;

// per-block exclusive scan of in[0..n) into out, block totals into bsum
__global__ void __launch_bounds__(kScanBlock)
    k_scan_local(const int32_t *__restrict__ in, int32_t *out, int64_t n, int32_t *bsum) {
  __shared__ int32_t warp_tot[32];
  const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int32_t v = i < n ? in[i] : 0;
  int32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int32_t w = warp_tot[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    warp_tot[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const int32_t before = wid > 0 ? warp_tot[wid - 1] : 0;
  if (i < n) out[i] = before + incl - v;
  if (threadIdx.x == kScanBlock - 1) bsum[blockIdx.x] = warp_tot[31];
}

// exclusive scan of the nb block totals in place (one block); bsum[nb] = total
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(int32_t *bsum, int nb) {
  __shared__ int32_t warp_tot[32];
  __shared__ int32_t carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += kScanBlock) {
    const int i = base + threadIdx.x;
    const int32_t v = i < nb ? bsum[i] : 0;
    int32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int32_t w = warp_tot[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      warp_tot[lane] = w;
    }
    __syncthreads();
    const int32_t before = (wid > 0 ? warp_tot[wid - 1] : 0) + carry;
    if (i < nb) bsum[i] = before + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_tot[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void k_scan_add(int32_t *out, int64_t n, const int32_t *__restrict__ bsum, int nb,
                           int32_t base) {
  const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += bsum[blockIdx.x] + base;
  if (i == 0) out[n] = bsum[nb] + base;
}

// histogram of the particles' current cells
__global__ void k_hist(const double *__restrict__ part, int64_t n, int64_t cap, int nx, int ny,
                       int32_t *cnt) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = j < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const int key = cell_key(part[j], part[cap + j], nx, ny);
  agg_atomic_add(cnt, key, am);
}

// scatter A -> B at off[key] + (running count of key)
__global__ void k_scatter(const double *__restrict__ A, const int32_t *__restrict__ slotA,
                          int64_t n, int64_t cap, int nx, int ny,
                          const int32_t *__restrict__ off, int32_t *cursor, double *B,
                          int32_t *slotB) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = j < n;
  const unsigned am = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const int key = cell_key(A[j], A[cap + j], nx, ny);
  const int64_t pos = (int64_t)off[key] + agg_atomic_add(cursor, key, am);
  for (int k = 0; k < 6; ++k) B[k * cap + pos] = A[k * cap + j];
  slotB[pos] = slotA[j];
}

}  // namespace

int sort_init(em2g_ctx *c) {
  c->ncell = (int64_t)c->g.nx * c->g.ny;
  const int64_t nc = c->ncell;
  EM2G_CUDA(cudaMalloc(&c->scan_tmp, sizeof(int32_t) * scan_tmp_size(nc)));
  for (int s = 0; s < c->P.nsp; ++s) {
    Species &S = c->sp[s];
    EM2G_CUDA(cudaMalloc(&S.off, sizeof(int32_t) * (nc + 1)));
    EM2G_CUDA(cudaMalloc(&S.off_alt, sizeof(int32_t) * (nc + 1)));
    EM2G_CUDA(cudaMalloc(&S.cnt, sizeof(int32_t) * nc));
    EM2G_CUDA(cudaMalloc(&S.cnt_alt, sizeof(int32_t) * nc));
    EM2G_CUDA(cudaMalloc(&S.cursor, sizeof(int32_t) * nc));
    S.sorted = false;
  }
  return EM2G_OK;
}

void sort_free(em2g_ctx *c) {
  cudaFree(c->scan_tmp);
  c->scan_tmp = nullptr;
  for (auto &S : c->sp) {
    cudaFree(S.off);
    cudaFree(S.off_alt);
    cudaFree(S.cnt);
    cudaFree(S.cnt_alt);
    cudaFree(S.cursor);
    S.off = S.off_alt = S.cnt = S.cnt_alt = S.cursor = nullptr;
  }
}

int64_t scan_tmp_size(int64_t n) { return (n + kScanBlock - 1) / kScanBlock + 1; }

int scan_counts(const int32_t *cnt, int32_t *off, int64_t n, int32_t base, int32_t *tmp,
                cudaStream_t stream) {
  const int nb = (int)((n + kScanBlock - 1) / kScanBlock);
  k_scan_local<<<nb, kScanBlock, 0, stream>>>(cnt, off, n, tmp);
  k_scan_sums<<<1, kScanBlock, 0, stream>>>(tmp, nb);
  k_scan_add<<<nb, kScanBlock, 0, stream>>>(off, n, tmp, nb, base);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int scan_cells(em2g_ctx *c, const int32_t *cnt, int32_t *off) {
  c->launches += 3;
  return scan_counts(cnt, off, c->ncell, 0, c->scan_tmp, c->stream);
}

int sort_full(em2g_ctx *c, int isp) {
  Species &S = c->sp[isp];
  const int64_t nc = c->ncell;
  EM2G_CUDA(cudaMemsetAsync(S.cnt, 0, sizeof(int32_t) * nc, c->stream));
  EM2G_CUDA(cudaMemsetAsync(S.cursor, 0, sizeof(int32_t) * nc, c->stream));
  if (S.n > 0) {
    const unsigned nb = (unsigned)((S.n + 255) / 256);
    k_hist<<<nb, 256, 0, c->stream>>>(S.part, S.n, S.cap, c->g.nx, c->g.ny, S.cnt);
    c->launches += 1;
    EM2G_CUDA(cudaGetLastError());
  }
  int rc = scan_cells(c, S.cnt, S.off);
  if (rc) return rc;
  if (S.n > 0) {
    const unsigned nb = (unsigned)((S.n + 255) / 256);
    k_scatter<<<nb, 256, 0, c->stream>>>(S.part, S.slot, S.n, S.cap, c->g.nx, c->g.ny, S.off,
                                         S.cursor, S.part_alt, S.slot_alt);
    c->launches += 1;
    EM2G_CUDA(cudaGetLastError());
    std::swap(S.part, S.part_alt);
    std::swap(S.slot, S.slot_alt);
  }
  // positions did not move: the counts of the current cells are S.cnt
  S.sorted = true;
  return EM2G_OK;
}

}  // namespace em2g

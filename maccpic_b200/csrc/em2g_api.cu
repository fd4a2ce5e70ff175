// em2g_api.cu -- the C ABI of libem2g.so (declared in include/em2g.h):
// context life cycle, state copies, and the move / curnt / fields /
// smooth2 entry points that stand in for em2's subroutines.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "em2g_internal.cuh"

namespace em2g {

static thread_local std::string g_last_error;

int fail(int status, const std::string &msg) {
  g_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? EM2G_ERR_NOMEM : EM2G_ERR_CUDA;
}

int timing_begin(em2g_ctx *c) {
  if (!c->timing) return EM2G_OK;
  if (c->ev_used + 2 > c->ev.size()) {
    for (int k = 0; k < 2; ++k) {
      cudaEvent_t e;
      EM2G_CUDA(cudaEventCreate(&e));
      c->ev.push_back(e);
    }
  }
  EM2G_CUDA(cudaEventRecord(c->ev[c->ev_used], c->stream));
  return EM2G_OK;
}

int timing_end(em2g_ctx *c) {
  if (!c->timing) return EM2G_OK;
  EM2G_CUDA(cudaEventRecord(c->ev[c->ev_used + 1], c->stream));
  c->ev_used += 2;
  return EM2G_OK;
}

// after a stream synchronisation: fold the recorded pairs into push_ms
static int timing_collect(em2g_ctx *c) {
  for (size_t k = 0; k + 1 < c->ev_used; k += 2) {
    float ms = 0.f;
    EM2G_CUDA(cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]));
    c->push_ms += ms;
    c->push_timed += 1;
  }
  c->ev_used = 0;
  return EM2G_OK;
}

namespace {

// device-side check of uploaded particles: bad[0] counts positions outside
// [0, n+0.5), bad[1] counts non-finite values
__global__ void k_check_particles(const double *__restrict__ part, int64_t n, int64_t cap,
                                  double xlim, double ylim, unsigned long long *bad) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  bool finite = true;
  for (int k = 0; k < 6; ++k) finite = finite && isfinite(part[k * cap + j]);
  if (!finite) {
    atomicAdd(bad + 1, 1ull);
    return;
  }
  const double x = part[j], y = part[cap + j];
  if (!(x >= 0.0 && x < xlim && y >= 0.0 && y < ylim)) atomicAdd(bad, 1ull);
}

// slot-order restore: dst[slot[j]] = src[j] for the 6 arrays
__global__ void k_unsort(const double *__restrict__ src, const int32_t *__restrict__ slot,
                         double *__restrict__ dst, int64_t n, int64_t cap) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t s = slot[j];
  for (int k = 0; k < 6; ++k) dst[k * cap + s] = src[k * cap + j];
}

__global__ void k_iota(int32_t *slot, int64_t n) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) slot[j] = (int32_t)j;
}

__global__ void k_d2f(const double *__restrict__ a, float *b, int64_t n) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) b[k] = (float)a[k];
}
__global__ void k_f2d(const float *__restrict__ a, double *b, int64_t n) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) b[k] = (double)a[k];
}

bool is_fp32(const em2g_ctx *c) { return c->P.precision == EM2G_FP32; }

// The context's FP64 staging buffer on the device (field arrays; slices of
// particles in FP64; the records of a regrouping), grown on demand and kept
// until em2g_destroy so that repeated copies allocate nothing.
int ensure_staging(em2g_ctx *c, int64_t ndoubles) {
  if (ndoubles <= c->staging_n) return EM2G_OK;
  EM2G_CUDA(cudaStreamSynchronize(c->stream));  // the old buffer may still be read
  cudaFree(c->staging);
  c->staging = nullptr;
  c->staging_n = 0;
  EM2G_CUDA(cudaMalloc((void **)&c->staging, sizeof(double) * ndoubles));
  c->staging_n = ndoubles;
  return EM2G_OK;
}

__global__ void k_count_nonfinite(const double *__restrict__ a, int64_t n,
                                  unsigned long long *bad) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool nf = k < n && !isfinite(a[k]);
  const unsigned m = __ballot_sync(0xffffffffu, nf);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(bad, (unsigned long long)__popc(m));
}

// host FP64 arrays [first, first+count) of the field block -> device: copied
// as FP64 to the device, checked there, then converted (FP32) or moved into
// the block; non-finite input leaves the block as it was
int put_fields_host(em2g_ctx *c, int first, int count, const double *host) {
  const int64_t n = (int64_t)count * c->g.w;
  int rc = ensure_staging(c, n);
  if (rc) return rc;
  double *st = c->staging;
  EM2G_CUDA(cudaMemcpyAsync(st, host, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  unsigned long long *bad = (unsigned long long *)c->red;
  EM2G_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), c->stream));
  const unsigned nb = (unsigned)((n + 255) / 256);
  k_count_nonfinite<<<nb, 256, 0, c->stream>>>(st, n, bad);
  EM2G_CUDA(cudaGetLastError());
  unsigned long long hb = 0;
  EM2G_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, c->stream));
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  if (hb) return fail(EM2G_ERR_NONFINITE, std::to_string(hb) + " non-finite field values");
  if (is_fp32(c)) {
    k_d2f<<<nb, 256, 0, c->stream>>>(st, c->fld32 + first * c->g.w, n);
    EM2G_CUDA(cudaGetLastError());
  } else {
    EM2G_CUDA(cudaMemcpyAsync(c->fld + first * c->g.w, st, sizeof(double) * n,
                              cudaMemcpyDeviceToDevice, c->stream));
  }
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  return EM2G_OK;
}

int get_fields_host(em2g_ctx *c, int first, int count, double *host) {
  const int64_t n = (int64_t)count * c->g.w;
  if (is_fp32(c)) {
    int rc = ensure_staging(c, n);
    if (rc) return rc;
    k_f2d<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->fld32 + first * c->g.w,
                                                               c->staging, n);
    EM2G_CUDA(cudaGetLastError());
    EM2G_CUDA(cudaMemcpyAsync(host, c->staging, sizeof(double) * n, cudaMemcpyDeviceToHost,
                              c->stream));
    EM2G_CUDA(cudaStreamSynchronize(c->stream));
  } else {
    EM2G_CUDA(cudaMemcpyAsync(host, c->fld + first * c->g.w, sizeof(double) * n,
                              cudaMemcpyDeviceToHost, c->stream));
    EM2G_CUDA(cudaStreamSynchronize(c->stream));
  }
  return EM2G_OK;
}

int check_ctx(em2g_ctx *c) {
  if (!c) return fail(EM2G_ERR_INVALID, "null context");
  EM2G_CUDA(cudaSetDevice(c->device));
  return EM2G_OK;
}

int validate(const em2g_params *p) {
  if (!p) return fail(EM2G_ERR_INVALID, "null params");
  if (p->struct_size != sizeof(em2g_params))
    return fail(EM2G_ERR_INVALID, "em2g_params.struct_size mismatch (header/library version)");
  if (p->nx < 4 || p->ny < 4) return fail(EM2G_ERR_INVALID, "nx and ny must be >= 4");
  if (p->ny > 65535) return fail(EM2G_ERR_INVALID, "ny must be <= 65535");
  if ((int64_t)(p->nx + 3) * (p->ny + 3) > (int64_t)1 << 31)
    return fail(EM2G_ERR_INVALID, "grid too large");
  if (p->nsp < 1 || p->nsp > EM2G_MAX_SPECIES)
    return fail(EM2G_ERR_INVALID, "nsp must be 1..4");
  if (p->isav < 1) return fail(EM2G_ERR_INVALID, "isav must be >= 1");
  if (p->precision != EM2G_FP64 && p->precision != EM2G_FP32)
    return fail(EM2G_ERR_INVALID, "unknown precision");
  if (!(p->dx > 0) || !(p->dy > 0) || !(p->dt > 0) || !(p->c > 0))
    return fail(EM2G_ERR_INVALID, "dx, dy, dt, c must be > 0");
  if (p->c * p->dt >= p->dx || p->c * p->dt >= p->dy)
    return fail(EM2G_ERR_INVALID, "c*dt must be < dx and dy (one wrap per step)");
  if (p->energy_mode == 1 && p->ny < 170)
    return fail(EM2G_ERR_INVALID, "energy_mode 1 reads rows 88..168 and needs ny >= 170");
  if (p->cg_maxits < 1) return fail(EM2G_ERR_INVALID, "cg_maxits must be >= 1");
  if (p->smooth_current != 0 && p->smooth_current != 1)
    return fail(EM2G_ERR_INVALID, "smooth_current must be 0 or 1");
  if (p->sort_interval < 0) return fail(EM2G_ERR_INVALID, "sort_interval must be >= 0");
  if (p->poisson != 0 && p->poisson != 1) return fail(EM2G_ERR_INVALID, "poisson must be 0 or 1");
  if (p->staging_mib < 0 || p->staging_mib > (1 << 16))
    return fail(EM2G_ERR_INVALID, "staging_mib must be 0..65536");
  if (p->poisson == 1 && (p->precision != EM2G_FP64 || !spectral_size_ok(p->nx, p->ny)))
    return fail(EM2G_ERR_INVALID,
                "poisson 1 (spectral) needs FP64 and power-of-two nx, ny <= 8192");
  if (p->sort_interval > 1) {
    if (p->precision != EM2G_FP32)
      return fail(EM2G_ERR_INVALID, "sort_interval > 1 needs the FP32 path");
    // positions drift from their group cell by < c*dt per step between
    // regroupings and must stay within one cell of it
    if (p->sort_interval * p->c * p->dt >= p->dx || p->sort_interval * p->c * p->dt >= p->dy)
      return fail(EM2G_ERR_INVALID, "sort_interval * c * dt must be < dx and dy");
  }
  for (int s = 0; s < p->nsp; ++s) {
    if (p->np_max[s] < 0 || p->np_max[s] > ((int64_t)1 << 31) - 1)
      return fail(EM2G_ERR_INVALID, "np_max out of range");
    if (!std::isfinite(p->qm[s]) || !std::isfinite(p->q[s]) || !std::isfinite(p->dn[s]) ||
        !std::isfinite(p->am[s]))
      return fail(EM2G_ERR_NONFINITE, "non-finite species constant");
  }
  return EM2G_OK;
}

int finish_outputs(em2g_ctx *c, double *ake_out, double *energies_out, int *cg_iters_out,
                   bool energies_valid) {
  EM2G_CUDA(cudaMemcpyAsync(c->host_out, c->dev_out, sizeof(double) * kDevOut,
                            cudaMemcpyDeviceToHost, c->stream));
  int st[2] = {0, 0};
  EM2G_CUDA(cudaMemcpyAsync(st, c->cg.status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  EM2G_CUDA(cudaGetLastError());
  int rc = timing_collect(c);
  if (rc) return rc;
  if (st[0] & 2)
    return fail(EM2G_ERR_TIMEOUT, "a TMA-staged stencil's wait for its tiles timed out");
  if (st[0] != 0) return fail(EM2G_ERR_TIMEOUT, "cg: a grid barrier wait timed out");
  if (c->host_out[kDevLost] != 0.0) {
    const double lost = c->host_out[kDevLost];
    EM2G_CUDA(cudaMemsetAsync(c->dev_out + kDevLost, 0, sizeof(double), c->stream));
    return fail(EM2G_ERR_RANGE, "regrouping push: " + std::to_string((long long)lost) +
                                    " particles fell outside their cells' ranges");
  }
  if (ake_out)
    for (int s = 0; s < c->P.nsp; ++s) ake_out[s] = c->host_out[s];
  if (energies_out && energies_valid)
    for (int k = 0; k < 6; ++k) energies_out[k] = c->host_out[4 + k];
  if (cg_iters_out) *cg_iters_out = st[1];
  return EM2G_OK;
}

}  // namespace

int validate_params(const em2g_params *p) { return validate(p); }

int check_particles_device(const double *part, int64_t n, int64_t ld, double xlim, double ylim,
                           unsigned long long *bad, cudaStream_t st, bool reset) {
  if (reset) EM2G_CUDA(cudaMemsetAsync(bad, 0, 2 * sizeof(unsigned long long), st));
  if (n > 0)
    k_check_particles<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(part, n, ld, xlim, ylim, bad);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int64_t staging_cap(const em2g_ctx *c) {
  if (c->P.staging_mib > 0) return (int64_t)c->P.staging_mib << 20;
  int64_t n = 1024;
  for (int s = 0; s < c->P.nsp; ++s) n = std::max(n, c->sp[s].cap);
  return 80 * std::min<int64_t>(n, (int64_t)1 << 24);
}

}  // namespace em2g

using namespace em2g;

extern "C" {

int em2g_abi_version(void) { return EM2G_ABI_VERSION; }

const char *em2g_last_error(void) { return g_last_error.c_str(); }

int em2g_params_init(em2g_params *p) {
  if (!p) return fail(EM2G_ERR_INVALID, "null params");
  std::memset(p, 0, sizeof(*p));
  p->struct_size = sizeof(em2g_params);
  p->nsp = 2;
  p->isav = 20;
  p->precision = EM2G_FP64;
  p->c = 1.0;
  p->cg_maxits = 10000;
  p->cg_eps = 1e-9;
  p->qme = -1.0;
  p->wpe = 1.0;
  return EM2G_OK;
}

int em2g_create(const em2g_params *p, em2g_ctx **out) {
  if (!out) return fail(EM2G_ERR_INVALID, "null output pointer");
  *out = nullptr;
  int rc = validate(p);
  if (rc) return rc;
  em2g_ctx *c = new (std::nothrow) em2g_ctx();
  if (!c) return fail(EM2G_ERR_NOMEM, "host allocation failed");
  c->P = *p;
  c->device = p->device;
  c->g.nx = p->nx;
  c->g.ny = p->ny;
  c->g.nxg = p->nx + 3;
  c->g.w = (int64_t)(p->nx + 3) * (p->ny + 3);
  auto bail = [&](int code) {
    em2g_destroy(c);
    return code;
  };
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaSetDevice"));
  e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaDeviceGetAttribute"));
  e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamCreate"));
  c->stream = c->own_stream;
  const int64_t w = c->g.w;
#define ALLOC(ptr, bytes)                                            \
  do {                                                               \
    e = cudaMalloc((void **)&(ptr), (bytes));                        \
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc " #ptr)); \
  } while (0)
  const bool fp32 = p->precision == EM2G_FP32;
  // the field block and the smooth2 scratch carry a tail of a few rows, so
  // that the TMA-staged stages' tensor maps (whole lines of 16 bytes' worth
  // of rows) lie inside the allocations; the tail is zero and never used
  const int64_t tail = tma_tail_elems(c, fp32);
  if (fp32) {
    ALLOC(c->fld32, sizeof(float) * (EM2G_NFIELD * w + tail));
    ALLOC(c->scaled32, sizeof(float) * 6 * w * p->nsp);
    ALLOC(c->smooth_tmp32, sizeof(float) * (w + tail));
  } else {
    ALLOC(c->fld, sizeof(double) * (EM2G_NFIELD * w + tail));
    ALLOC(c->scaled, sizeof(double) * 6 * w * p->nsp);
    ALLOC(c->smooth_tmp, sizeof(double) * (w + tail));
  }
  int64_t maxn = 0;
  for (int s = 0; s < p->nsp; ++s) {
    Species &S = c->sp[s];
    S.cap = p->np_max[s] > 0 ? p->np_max[s] : 1;
    if (S.cap > maxn) maxn = S.cap;
    if (fp32) {
      ALLOC(S.p32, sizeof(float) * 5 * S.cap);
      ALLOC(S.p32_alt, sizeof(float) * 5 * S.cap);
    } else {
      ALLOC(S.part, sizeof(double) * 6 * S.cap);
      ALLOC(S.part_alt, sizeof(double) * 6 * S.cap);
    }
    ALLOC(S.slot, sizeof(int32_t) * S.cap);
    ALLOC(S.slot_alt, sizeof(int32_t) * S.cap);
  }
  c->red_blocks = (int)((maxn + 255) / 256);
  if (c->red_blocks < 6 * kEnergyBlocks) c->red_blocks = 6 * kEnergyBlocks;
  ALLOC(c->red, sizeof(double) * c->red_blocks);
  ALLOC(c->ake_l1, sizeof(double) * kAkeBlocks);
  ALLOC(c->dev_out, sizeof(double) * kDevOut);
  ALLOC(c->up_bad, sizeof(unsigned long long) * 2 * EM2G_MAX_SPECIES);
#undef ALLOC
  e = cudaMallocHost((void **)&c->host_out, sizeof(double) * kDevOut);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMallocHost"));
  if (fp32) {
    e = cudaMemset(c->fld32, 0, sizeof(float) * (EM2G_NFIELD * w + tail));
    if (e == cudaSuccess) e = cudaMemset(c->smooth_tmp32, 0, sizeof(float) * (w + tail));
  } else {
    e = cudaMemset(c->fld, 0, sizeof(double) * (EM2G_NFIELD * w + tail));
    if (e == cudaSuccess) e = cudaMemset(c->smooth_tmp, 0, sizeof(double) * (w + tail));
  }
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMemset"));
  e = cudaMemset(c->dev_out, 0, sizeof(double) * kDevOut);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMemset"));
  rc = fp32 ? cg_init_f32(c) : cg_init(c);
  if (rc) return bail(rc);
  rc = fp32 ? tma_init_f32(c) : tma_init_f64(c);
  if (rc) return bail(rc);
  if (p->poisson == 1) {
    e = cudaMalloc((void **)&c->spec, sizeof(double2) * (int64_t)p->nx * p->ny);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc spec"));
    if ((rc = spectral_prepare())) return bail(rc);
  }
  rc = sort_init(c);
  if (rc) return bail(rc);
  {
    // the fast pushes write one ake partial per block of 64 cells (FP64) or
    // per warp of a row segment (FP32)
    const int64_t fast_blocks = push_partials(c->g.nx, c->g.ny) + 64;
    if (fast_blocks > c->red_blocks) {
      cudaFree(c->red);
      c->red_blocks = (int)fast_blocks;
      e = cudaMalloc((void **)&c->red, sizeof(double) * c->red_blocks);
      if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc red"));
    }
  }
  e = cudaMemset(c->cg.status, 0, sizeof(int) * 2);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMemset"));
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaDeviceSynchronize"));
  *out = c;
  return EM2G_OK;
}

int em2g_destroy(em2g_ctx *c) {
  if (!c) return EM2G_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->fld);
  cudaFree(c->scaled);
  cudaFree(c->smooth_tmp);
  cudaFree(c->fld32);
  cudaFree(c->scaled32);
  cudaFree(c->smooth_tmp32);
  for (auto &S : c->sp) {
    cudaFree(S.part);
    cudaFree(S.part_alt);
    cudaFree(S.p32);
    cudaFree(S.p32_alt);
    cudaFree(S.slot);
    cudaFree(S.slot_alt);
  }
  cudaFree(c->red);
  cudaFree(c->ake_l1);
  cudaFree(c->spec);
  cudaFree(c->staging);
  cudaFree(c->dev_out);
  cudaFree(c->up_bad);
  if (c->host_out) cudaFreeHost(c->host_out);
  cg_free(c);
  sort_free(c);
  for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
  for (int h = 0; h < 2; ++h) {
    if (c->half_copied[h]) cudaEventDestroy(c->half_copied[h]);
    if (c->half_used[h]) cudaEventDestroy(c->half_used[h]);
  }
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
  }
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return EM2G_OK;
}

int em2g_set_stream(em2g_ctx *c, void *stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return EM2G_OK;
}

int em2g_synchronize(em2g_ctx *c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  return EM2G_OK;
}

int em2g_set_field(em2g_ctx *c, int id, const double *host) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (id < 0 || id >= EM2G_NFIELD || !host) return fail(EM2G_ERR_INVALID, "bad field id or pointer");
  c->jp_live = true;
  return put_fields_host(c, id, 1, host);
}

int em2g_get_field(em2g_ctx *c, int id, double *host) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (id < 0 || id >= EM2G_NFIELD || !host) return fail(EM2G_ERR_INVALID, "bad field id or pointer");
  return get_fields_host(c, id, 1, host);
}

int em2g_set_fields(em2g_ctx *c, const double *host13) {
  em2g::NvtxRange nvtx_range("em2g set_fields");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!host13) return fail(EM2G_ERR_INVALID, "null pointer");
  c->jp_live = true;
  return put_fields_host(c, 0, EM2G_NFIELD, host13);
}

int em2g_get_fields(em2g_ctx *c, double *host13) {
  em2g::NvtxRange nvtx_range("em2g get_fields");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!host13) return fail(EM2G_ERR_INVALID, "null pointer");
  return get_fields_host(c, 0, EM2G_NFIELD, host13);
}

int em2g_set_fields_device(em2g_ctx *c, const double *dev13) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!dev13) return fail(EM2G_ERR_INVALID, "null pointer");
  c->jp_live = true;
  const int64_t n = EM2G_NFIELD * c->g.w;
  if (is_fp32(c)) {
    k_d2f<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(dev13, c->fld32, n);
    EM2G_CUDA(cudaGetLastError());
  } else {
    EM2G_CUDA(cudaMemcpyAsync(c->fld, dev13, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                              c->stream));
  }
  return EM2G_OK;
}

int em2g_get_fields_device(em2g_ctx *c, double *dev13) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!dev13) return fail(EM2G_ERR_INVALID, "null pointer");
  const int64_t n = EM2G_NFIELD * c->g.w;
  if (is_fp32(c)) {
    k_f2d<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->fld32, dev13, n);
    EM2G_CUDA(cudaGetLastError());
  } else {
    EM2G_CUDA(cudaMemcpyAsync(dev13, c->fld, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                              c->stream));
  }
  return EM2G_OK;
}

int em2g_field_device_ptr(em2g_ctx *c, int id, void **dptr) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (id < 0 || id >= EM2G_NFIELD || !dptr) return fail(EM2G_ERR_INVALID, "bad field id or pointer");
  c->jp_live = true;  // the caller may write through the pointer
  if (is_fp32(c))
    *dptr = c->fld32 + id * c->g.w;
  else
    *dptr = c->fld + id * c->g.w;
  return EM2G_OK;
}

// ---- particle copies in slices -------------------------------------------
//
// An upload parks its slices in the species' alternate buffers (FP64: the
// sort target; FP32: the regrouping target, with each particle's cell key)
// and counts rejected values on the device; only the end of the upload,
// once every slot is in and none was rejected, makes them the species'
// particles.  Host slices go through the staging buffer, at most
// staging_cap() bytes, so no buffer grows with the particle count.

// the copy stream and the halves' events, made on first use; the copy
// stream then waits for everything already enqueued on the context's stream
// (earlier users of the staging buffer)
static int copy_setup(em2g_ctx *c) {
  if (!c->copy_stream) {
    EM2G_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (int h = 0; h < 2; ++h) {
      EM2G_CUDA(cudaEventCreateWithFlags(&c->half_copied[h], cudaEventDisableTiming));
      EM2G_CUDA(cudaEventCreateWithFlags(&c->half_used[h], cudaEventDisableTiming));
    }
  }
  EM2G_CUDA(cudaEventRecord(c->half_used[0], c->stream));
  EM2G_CUDA(cudaEventRecord(c->half_used[1], c->stream));
  return EM2G_OK;
}

static int particles_begin(em2g_ctx *c, int isp, int64_t n) {
  Species &S = c->sp[isp];
  if (n < 0 || n > S.cap) return fail(EM2G_ERR_RANGE, "particle count exceeds np_max");
  EM2G_CUDA(cudaMemsetAsync(c->up_bad + 2 * isp, 0, 2 * sizeof(unsigned long long), c->stream));
  if (is_fp32(c))
    EM2G_CUDA(cudaMemsetAsync(S.cnt_alt, 0, sizeof(int32_t) * c->ncell, c->stream));
  S.up_n = n;
  S.up_added = 0;
  return EM2G_OK;
}

// slots first..first+count from six arrays in host or device memory
static int particles_add(em2g_ctx *c, int isp, int64_t first, int64_t count,
                         const double *const *src, bool on_device) {
  Species &S = c->sp[isp];
  if (S.up_n < 0) return fail(EM2G_ERR_INVALID, "no particle upload open for this species");
  if (first != S.up_added || count < 0 || first + count > S.up_n)
    return fail(EM2G_ERR_INVALID, "particle slices must be added in slot order, within n");
  if (count == 0) return EM2G_OK;
  for (int k = 0; k < 6; ++k)
    if (!src[k]) return fail(EM2G_ERR_INVALID, "null particle array");
  unsigned long long *bad = c->up_bad + 2 * isp;
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (!is_fp32(c)) {
    // parked at their slots in the sort target, checked there
    for (int k = 0; k < 6; ++k)
      EM2G_CUDA(cudaMemcpyAsync(S.part_alt + k * S.cap + first, src[k], sizeof(double) * count,
                                kind, c->stream));
    int rc = check_particles_device(S.part_alt + first, count, S.cap, c->P.nx + 0.5,
                                    c->P.ny + 0.5, bad, c->stream, false);
    if (rc) return rc;
    S.up_added += count;
    return EM2G_OK;
  }
  if (on_device) {
    int rc = stage_f32(c, isp, first, count, src, bad);
    if (rc) return rc;
    S.up_added += count;
    return EM2G_OK;
  }
  // host slices through the two halves of the staging buffer, 6 doubles per
  // particle: the copy of one half (copy stream) overlaps the check and
  // conversion of the other (the context's stream)
  const int64_t half = staging_cap(c) / 16;  // doubles per half
  const int64_t chunk = half / 6;
  int rc = ensure_staging(c, 2 * half);
  if (rc) return rc;
  if ((rc = copy_setup(c))) return rc;
  for (int64_t a = 0, i = 0; a < count; a += chunk, ++i) {
    const int h = (int)(i & 1);
    const int64_t m = std::min(chunk, count - a);
    EM2G_CUDA(cudaStreamWaitEvent(c->copy_stream, c->half_used[h], 0));
    const double *st[6];
    for (int k = 0; k < 6; ++k) {
      double *d = c->staging + h * half + k * m;
      EM2G_CUDA(cudaMemcpyAsync(d, src[k] + a, sizeof(double) * m, cudaMemcpyHostToDevice,
                                c->copy_stream));
      st[k] = d;
    }
    EM2G_CUDA(cudaEventRecord(c->half_copied[h], c->copy_stream));
    EM2G_CUDA(cudaStreamWaitEvent(c->stream, c->half_copied[h], 0));
    if ((rc = stage_f32(c, isp, first + a, m, st, bad))) {
      // later users of the staging buffer (on the context's stream) wait for
      // the copy this slice started
      cudaStreamSynchronize(c->copy_stream);
      return rc;
    }
    EM2G_CUDA(cudaEventRecord(c->half_used[h], c->stream));
  }
  S.up_added += count;
  return EM2G_OK;
}

static int particles_end(em2g_ctx *c, int isp) {
  Species &S = c->sp[isp];
  if (S.up_n < 0) return fail(EM2G_ERR_INVALID, "no particle upload open for this species");
  if (S.up_added != S.up_n) {
    S.up_n = -1;
    return fail(EM2G_ERR_INVALID, "particle upload ended before every slot was added");
  }
  const int64_t n = S.up_n;
  S.up_n = -1;
  unsigned long long hb[2] = {0, 0};
  EM2G_CUDA(cudaMemcpyAsync(hb, c->up_bad + 2 * isp, sizeof(hb), cudaMemcpyDeviceToHost,
                            c->stream));
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  if (hb[1]) return fail(EM2G_ERR_NONFINITE, std::to_string(hb[1]) + " particles with non-finite values");
  if (hb[0]) return fail(EM2G_ERR_RANGE, std::to_string(hb[0]) + " particles outside the grid");
  int rc;
  if (is_fp32(c)) {
    if ((rc = ensure_staging(c, staging_cap(c) / 8))) return rc;
    if ((rc = commit_f32(c, isp, n, c->staging, staging_cap(c) / 32))) return rc;
  } else {
    std::swap(S.part, S.part_alt);
    if (n > 0) {
      k_iota<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(S.slot, n);
      EM2G_CUDA(cudaGetLastError());
    }
    S.n = n;
    S.sorted = false;
  }
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  return EM2G_OK;
}

// n particles of species isp from six arrays (host or device memory): one
// upload of a single slice
static int load_particles(em2g_ctx *c, int isp, int64_t n, const double *const *src,
                          bool on_device) {
  int rc = particles_begin(c, isp, n);
  if (rc) return rc;
  if ((rc = particles_add(c, isp, 0, n, src, on_device))) {
    c->sp[isp].up_n = -1;
    return rc;
  }
  return particles_end(c, isp);
}

// slots first..first+count of species isp into six arrays in host or
// device memory, in slot order
static int particles_get(em2g_ctx *c, int isp, int64_t first, int64_t count,
                         double *const *dst, bool on_device) {
  Species &S = c->sp[isp];
  if (first < 0 || count < 0 || first + count > S.n)
    return fail(EM2G_ERR_RANGE, "slot range beyond the species' particles");
  if (count == 0) return EM2G_OK;
  for (int k = 0; k < 6; ++k)
    if (!dst[k]) return fail(EM2G_ERR_INVALID, "null particle array");
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (!is_fp32(c)) {
    // restore slot order into the sort target, then copy the range
    k_unsort<<<(unsigned)((S.n + 255) / 256), 256, 0, c->stream>>>(S.part, S.slot, S.part_alt,
                                                                    S.n, S.cap);
    EM2G_CUDA(cudaGetLastError());
    for (int k = 0; k < 6; ++k)
      EM2G_CUDA(cudaMemcpyAsync(dst[k], S.part_alt + k * S.cap + first, sizeof(double) * count,
                                kind, c->stream));
    EM2G_CUDA(cudaStreamSynchronize(c->stream));
    return EM2G_OK;
  }
  // FP32: 32-byte records, then FP64 values (into the caller's device
  // arrays directly, or into the staging buffer and across to the host)
  int rc = ensure_staging(c, staging_cap(c) / 8);
  if (rc) return rc;
  if (on_device) {
    const int64_t chunk = staging_cap(c) / 32;  // records only
    for (int64_t a = 0; a < count; a += chunk) {
      const int64_t m = std::min(chunk, count - a);
      double *d[6];
      for (int k = 0; k < 6; ++k) d[k] = dst[k] + a;
      if ((rc = get_range_f32(c, isp, first + a, m, d, c->staging))) return rc;
    }
    EM2G_CUDA(cudaStreamSynchronize(c->stream));
    return EM2G_OK;
  }
  // to the host through the two halves of the staging buffer: the copy of
  // one half (copy stream) overlaps the gather into the other
  const int64_t half = staging_cap(c) / 16;  // doubles per half
  const int64_t chunk = half / 10;          // 32 B of record, 48 B of values each
  if ((rc = copy_setup(c))) return rc;
  for (int64_t a = 0, i = 0; a < count; a += chunk, ++i) {
    const int h = (int)(i & 1);
    const int64_t m = std::min(chunk, count - a);
    double *base = c->staging + h * half;
    double *d[6];
    for (int k = 0; k < 6; ++k) d[k] = base + 4 * m + k * m;
    // this half's previous contents have crossed to the host
    EM2G_CUDA(cudaStreamWaitEvent(c->stream, c->half_copied[h], 0));
    if ((rc = get_range_f32(c, isp, first + a, m, d, base))) return rc;
    EM2G_CUDA(cudaEventRecord(c->half_used[h], c->stream));
    EM2G_CUDA(cudaStreamWaitEvent(c->copy_stream, c->half_used[h], 0));
    for (int k = 0; k < 6; ++k)
      EM2G_CUDA(cudaMemcpyAsync(dst[k] + a, d[k], sizeof(double) * m, kind, c->copy_stream));
    EM2G_CUDA(cudaEventRecord(c->half_copied[h], c->copy_stream));
  }
  EM2G_CUDA(cudaStreamSynchronize(c->copy_stream));
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  return EM2G_OK;
}

int em2g_set_particles(em2g_ctx *c, int isp, int64_t n, const double *x, const double *y,
                       const double *vx, const double *vy, const double *vz,
                       const double *gamma) {
  em2g::NvtxRange nvtx_range("em2g set_particles");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (isp < 0 || isp >= c->P.nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  const double *src[6] = {x, y, vx, vy, vz, gamma};
  return load_particles(c, isp, n, src, false);
}

int em2g_set_particles_device(em2g_ctx *c, int isp, int64_t n, const double *x,
                              const double *y, const double *vx, const double *vy,
                              const double *vz, const double *gamma) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (isp < 0 || isp >= c->P.nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  const double *src[6] = {x, y, vx, vy, vz, gamma};
  return load_particles(c, isp, n, src, true);
}

int em2g_get_particles(em2g_ctx *c, int isp, int64_t *n, double *x, double *y, double *vx,
                       double *vy, double *vz, double *gamma) {
  em2g::NvtxRange nvtx_range("em2g get_particles");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (isp < 0 || isp >= c->P.nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  Species &S = c->sp[isp];
  if (n) *n = S.n;
  if (S.n == 0) return EM2G_OK;
  if (!x && !y && !vx && !vy && !vz && !gamma) return EM2G_OK;  // count query
  double *dst[6] = {x, y, vx, vy, vz, gamma};
  return particles_get(c, isp, 0, S.n, dst, false);
}

int em2g_particles_begin(em2g_ctx *c, int isp, int64_t n) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (isp < 0 || isp >= c->P.nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  return particles_begin(c, isp, n);
}

int em2g_particles_add(em2g_ctx *c, int isp, int64_t first, int64_t count, const double *x,
                       const double *y, const double *vx, const double *vy, const double *vz,
                       const double *gamma, int on_device) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (isp < 0 || isp >= c->P.nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  const double *src[6] = {x, y, vx, vy, vz, gamma};
  return particles_add(c, isp, first, count, src, on_device != 0);
}

int em2g_particles_end(em2g_ctx *c, int isp) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (isp < 0 || isp >= c->P.nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  return particles_end(c, isp);
}

int em2g_get_particles_range(em2g_ctx *c, int isp, int64_t first, int64_t count, double *x,
                             double *y, double *vx, double *vy, double *vz, double *gamma,
                             int on_device) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (isp < 0 || isp >= c->P.nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  double *dst[6] = {x, y, vx, vy, vz, gamma};
  return particles_get(c, isp, first, count, dst, on_device != 0);
}

int em2g_set_step(em2g_ctx *c, int it) {
  int rc = check_ctx(c);
  if (rc) return rc;
  c->it = it;
  return EM2G_OK;
}

int em2g_get_step(em2g_ctx *c, int *it) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!it) return fail(EM2G_ERR_INVALID, "null pointer");
  *it = c->it;
  return EM2G_OK;
}

int em2g_move(em2g_ctx *c, double *ake_out) {
  em2g::NvtxRange nvtx_range("em2g move");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (is_fp32(c))
    return fail(EM2G_ERR_INVALID,
                "FP32 contexts run move and curnt fused: use em2g_move_curnt or em2g_step");
  for (int s = 0; s < c->P.nsp; ++s) {
    if ((rc = launch_prescale(c, s))) return rc;
    if ((rc = launch_push_f64(c, s, 1))) return rc;
  }
  return finish_outputs(c, ake_out, nullptr, nullptr, false);
}

// one fused move + curnt of every species on the cell-sorted fast path
static int fast_push_all(em2g_ctx *c) {
  int rc;
  for (int s = 0; s < c->P.nsp; ++s) {
    if (is_fp32(c)) {
      if ((rc = launch_prescale_f32(c, s))) return rc;
      if ((rc = launch_push_cells_f32(c, s))) return rc;
      continue;
    }
    if (!c->sp[s].sorted && (rc = sort_full(c, s))) return rc;
    if ((rc = launch_push_cells_f64(c, s))) return rc;  // prescales into pairs itself
  }
  return EM2G_OK;
}

int em2g_move_curnt(em2g_ctx *c, double *ake_out) {
  em2g::NvtxRange nvtx_range("em2g move+curnt");
  int rc = check_ctx(c);
  if (rc) return rc;
  if ((rc = fast_push_all(c))) return rc;
  return finish_outputs(c, ake_out, nullptr, nullptr, false);
}

int em2g_num_variants(em2g_ctx *c, int *n) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!n) return fail(EM2G_ERR_INVALID, "null pointer");
  *n = is_fp32(c) ? num_variants_f32() : num_variants_f64();
  return EM2G_OK;
}

int em2g_set_variant(em2g_ctx *c, int v) {
  int rc = check_ctx(c);
  if (rc) return rc;
  const int n = is_fp32(c) ? num_variants_f32() : num_variants_f64();
  if (v < 0 || v >= n) return fail(EM2G_ERR_INVALID, "variant out of range");
  c->variant = v;
  return EM2G_OK;
}

int em2g_get_variant(em2g_ctx *c, int *v, char *name, int name_len) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (v) *v = c->variant;
  if (name && name_len > 0) {
    const char *s = is_fp32(c) ? variant_name_f32(c->variant) : variant_name_f64(c->variant);
    std::strncpy(name, s, (size_t)name_len - 1);
    name[name_len - 1] = '\0';
  }
  return EM2G_OK;
}

int em2g_set_sort_interval(em2g_ctx *c, int k) {
  int rc = check_ctx(c);
  if (rc) return rc;
  em2g_params p = c->P;
  p.sort_interval = k;
  if ((rc = validate(&p))) return rc;
  c->P.sort_interval = k;
  return EM2G_OK;
}

int em2g_set_timing(em2g_ctx *c, int on) {
  int rc = check_ctx(c);
  if (rc) return rc;
  c->timing = on ? 1 : 0;
  return EM2G_OK;
}

int em2g_get_counters(em2g_ctx *c, int64_t *kernel_launches, int64_t *push_launches_timed,
                      double *push_ms) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (kernel_launches) *kernel_launches = c->launches;
  if (push_launches_timed) *push_launches_timed = c->push_timed;
  if (push_ms) *push_ms = c->push_ms;
  return EM2G_OK;
}

int em2g_reset_counters(em2g_ctx *c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  c->launches = 0;
  c->push_timed = 0;
  c->push_ms = 0.0;
  return EM2G_OK;
}

int em2g_curnt(em2g_ctx *c) {
  em2g::NvtxRange nvtx_range("em2g curnt");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (is_fp32(c))
    return fail(EM2G_ERR_INVALID,
                "FP32 contexts run move and curnt fused: use em2g_move_curnt or em2g_step");
  c->jp_live = true;
  for (int s = 0; s < c->P.nsp; ++s) {
    if ((rc = launch_push_f64(c, s, 2))) return rc;
    c->sp[s].sorted = false;  // positions moved outside the fast path's bookkeeping
  }
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int em2g_fields(em2g_ctx *c, int it, double *energies_out, int *cg_iters_out) {
  em2g::NvtxRange nvtx_range("em2g fields");
  int rc = check_ctx(c);
  if (rc) return rc;
  EM2G_CUDA(cudaMemsetAsync(c->cg.status, 0, sizeof(int) * 2, c->stream));
  c->it = it;
  rc = is_fp32(c) ? fields_f32(c, it, true) : fields_f64(c, it, true, nullptr);
  if (rc) return rc;
  return finish_outputs(c, nullptr, energies_out, cg_iters_out, it % c->P.isav == 0);
}

int em2g_diagnostics(em2g_ctx *c, double *out, int nout) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out || nout < 1) return fail(EM2G_ERR_INVALID, "null or empty output");
  if ((rc = diagnostics(c))) return rc;
  if ((rc = finish_outputs(c, nullptr, nullptr, nullptr, false))) return rc;
  const int n = nout < EM2G_NDIAG ? nout : EM2G_NDIAG;
  for (int k = 0; k < n; ++k) out[k] = c->host_out[10 + k];
  return EM2G_OK;
}

int em2g_smooth2(em2g_ctx *c, int id) {
  em2g::NvtxRange nvtx_range("em2g smooth2");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (id < 0 || id >= EM2G_NFIELD) return fail(EM2G_ERR_INVALID, "bad field id");
  rc = is_fp32(c) ? smooth2_f32(c, c->fld32 + id * c->g.w)
                  : smooth2_f64(c, c->fld + id * c->g.w);
  if (rc) return rc;
  EM2G_CUDA(cudaStreamSynchronize(c->stream));
  if (c->stencils == 1) {  // a TMA-staged pass that timed out marks cg.status
    int st = 0;
    EM2G_CUDA(cudaMemcpy(&st, c->cg.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st & 2) {
      EM2G_CUDA(cudaMemsetAsync(c->cg.status, 0, sizeof(int), c->stream));
      return fail(EM2G_ERR_TIMEOUT, "a TMA-staged stencil's wait for its tiles timed out");
    }
  }
  return EM2G_OK;
}

int em2g_set_stencils(em2g_ctx *c, int mode) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (mode != 0 && mode != 1) return fail(EM2G_ERR_INVALID, "stencils: 0 (direct) or 1 (TMA)");
  if (mode == 1 && !c->tma_ok) return fail(EM2G_ERR_INVALID, "TMA-staged stencils unavailable");
  c->stencils = mode;
  return EM2G_OK;
}

int em2g_selftest_waits(em2g_ctx *c, int *cg_status, int *tma_status) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!cg_status || !tma_status) return fail(EM2G_ERR_INVALID, "null output");
  return selftest_waits(c, cg_status, tma_status);
}

int em2g_get_stencils(em2g_ctx *c, int *mode) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!mode) return fail(EM2G_ERR_INVALID, "null output");
  *mode = c->stencils;
  return EM2G_OK;
}

int em2g_step(em2g_ctx *c, int nsteps, double *ake_out, double *energies_out,
              int *cg_iters_out) {
  em2g::NvtxRange nvtx_range("em2g step");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nsteps < 0) return fail(EM2G_ERR_INVALID, "nsteps < 0");
  EM2G_CUDA(cudaMemsetAsync(c->cg.status, 0, sizeof(int) * 2, c->stream));
  for (int k = 0; k < nsteps; ++k) {
    {
      em2g::NvtxRange r("push (move+curnt)");
      if ((rc = fast_push_all(c))) return rc;
    }
    c->it += 1;
    em2g::NvtxRange r("fields");
    rc = is_fp32(c) ? fields_f32(c, c->it, true) : fields_f64(c, c->it, true, nullptr);
    if (rc) return rc;
  }
  return finish_outputs(c, ake_out, energies_out, cg_iters_out,
                        nsteps > 0 && c->it % c->P.isav == 0);
}

}  // extern "C"

namespace em2g {

// one pass of em2g_step enqueued on the context's stream, without reading
// its outputs back or waiting for it
int step_enqueue(em2g_ctx *c) {
  int rc = fast_push_all(c);
  if (rc) return rc;
  c->it += 1;
  return is_fp32(c) ? fields_f32(c, c->it, true) : fields_f64(c, c->it, true, nullptr);
}

}  // namespace em2g

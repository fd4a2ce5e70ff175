// ensemble_api.cu -- the C ABI of ensembles: many independent FP32 runs of
// em2's step (pic/main.f90:154-169, each run as em2g_step advances it)
// that advance together, one step of all of them per graph launch.
//
// Per step the work is: prescale of every run's fields (one launch), the
// push of every (run, species) pair (one persistent launch that claims row
// segments from a counter, fed by one scan over all pairs' cell counts),
// the kinetic energies (one launch), then em2's fields for every run, one
// launch per stage and one cooperative launch for every run's CG
// (fields_ens.cu).  With a sort interval k > 1 the push regroups the
// particles by cell on every k-th step only and updates them in place in
// between, as single runs do.  Each kind of step (in place or regrouping,
// and which buffers and counts are current) is captured once into a CUDA
// graph and replayed; nothing in it waits on the host.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <vector>

#include "ens_internal.cuh"

using namespace em2g;

namespace {

int check_ens(em2g_ens *e) {
  if (!e) return fail(EM2G_ERR_INVALID, "null ensemble");
  EM2G_CUDA(cudaSetDevice(e->device));
  return EM2G_OK;
}

int check_pair(em2g_ens *e, int run, int isp) {
  int rc = check_ens(e);
  if (rc) return rc;
  if (run < 0 || run >= (int)e->runs.size()) return fail(EM2G_ERR_INVALID, "bad run index");
  if (isp < 0 || isp >= e->runs[run].P.nsp) return fail(EM2G_ERR_INVALID, "bad species index");
  return EM2G_OK;
}

void drop_graphs(em2g_ens *e) {
  for (auto &x : e->exec)
    if (x) {
      cudaGraphExecDestroy(x);
      x = nullptr;
    }
  for (bool &r : e->fused_ready) r = false;  // the fused step's tables follow the variant
}

// the next step's kind: in place between regroupings
bool next_inplace(const em2g_ens *e) {
  return e->sort_interval > 1 && e->since_sort + 1 < e->sort_interval;
}

int graph_key(const em2g_ens *e, bool inplace) {
  return (inplace ? 4 : 0) + 2 * e->parity + e->cparity;
}

int enqueue_step(em2g_ens *e, bool inplace) {
  int rc;
  if (e->fused) return ens_fused_launch(e, graph_key(e, inplace), inplace);
  if ((rc = ens_prescale(e))) return rc;
  if ((rc = ens_push(e, e->parity, e->cparity, inplace))) return rc;
  if ((rc = ens_tick(e))) return rc;
  return ens_fields(e);
}

int capture_step(em2g_ens *e, bool inplace) {
  const int key = graph_key(e, inplace);
  cudaGraph_t g = nullptr;
  int prc;
  if (e->fused && (prc = ens_fused_prepare(e, key, inplace))) return prc;
  EM2G_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue_step(e, inplace);
  const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
  size_t nn = 0;
  cudaError_t ge = cudaGraphGetNodes(g, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  if (ge == cudaSuccess && nn) ge = cudaGraphGetNodes(g, nodes.data(), &nn);
  int64_t kernels = 0;
  for (size_t k = 0; ge == cudaSuccess && k < nn; ++k) {
    cudaGraphNodeType t;
    ge = cudaGraphNodeGetType(nodes[k], &t);
    if (t == cudaGraphNodeTypeKernel) ++kernels;
  }
  if (ge == cudaSuccess) ge = cudaGraphInstantiate(&e->exec[key], g, 0);
  cudaGraphDestroy(g);
  if (ge != cudaSuccess) return cuda_fail(ge, "step graph");
  e->graph_kernels[key] = kernels;
  return EM2G_OK;
}

// staging for n particles: 6*n FP64 values, then 32*n bytes of records
int ensure_staging(em2g_ens *e, int64_t n) {
  if (n <= e->staging_n) return EM2G_OK;
  EM2G_CUDA(cudaStreamSynchronize(e->stream));  // the old buffer may still be read
  cudaFree(e->staging);
  e->staging = nullptr;
  e->staging_n = 0;
  EM2G_CUDA(cudaMalloc(&e->staging, sizeof(double) * 10 * n));
  e->staging_n = n;
  return EM2G_OK;
}

int64_t round64(int64_t v) { return (v + 63) & ~int64_t(63); }

}  // namespace

extern "C" {

int em2g_ens_create(const em2g_params *runs, int nruns, em2g_ens **out) {
  if (!out) return fail(EM2G_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (!runs || nruns < 1 || nruns > kEnsMaxRuns)
    return fail(EM2G_ERR_INVALID, "an ensemble holds 1 to 128 runs");
  int npairs = 0;
  int64_t cap = 0, ncell = 0;
  for (int r = 0; r < nruns; ++r) {
    const em2g_params &P = runs[r];
    int rc = validate_params(&P);
    if (rc) return rc;
    if (P.precision != EM2G_FP32) return fail(EM2G_ERR_INVALID, "ensemble runs are FP32");
    if (P.energy_mode != 0) return fail(EM2G_ERR_INVALID, "ensemble runs use energy_mode 0");
    if (std::max(P.sort_interval, 1) != std::max(runs[0].sort_interval, 1))
      return fail(EM2G_ERR_INVALID, "ensemble runs share one sort_interval");
    if (P.device != runs[0].device) return fail(EM2G_ERR_INVALID, "runs on different devices");
    for (int s = 0; s < P.nsp; ++s) {
      if (P.np_max[s] < 1) return fail(EM2G_ERR_INVALID, "np_max must be the particle count");
      cap += P.np_max[s];
      ncell += (int64_t)P.nx * P.ny;
    }
    npairs += P.nsp;
  }
  if (npairs > kEnsMaxPairs) return fail(EM2G_ERR_INVALID, "more than 160 (run, species) pairs");
  if (cap > std::numeric_limits<int32_t>::max() || ncell >= std::numeric_limits<int32_t>::max())
    return fail(EM2G_ERR_RANGE, "ensemble exceeds 2^31 particles or cells");
  em2g_ens *e = new (std::nothrow) em2g_ens();
  if (!e) return fail(EM2G_ERR_NOMEM, "host allocation failed");
  auto bail = [&](int code) {
    em2g_ens_destroy(e);
    return code;
  };
  e->device = runs[0].device;
  e->sort_interval = std::max(runs[0].sort_interval, 1);
  e->npairs = npairs;
  e->cap = cap;
  e->ncell = ncell;
  e->runs.resize(nruns);
  int64_t fo = 0, so = 0, to = 0, co = 0, ro = 0, c0 = 0, b0 = 0;
  for (int r = 0; r < nruns; ++r) {
    EnsRun &R = e->runs[r];
    R.P = runs[r];
    R.g.nx = R.P.nx;
    R.g.ny = R.P.ny;
    R.g.nxg = R.P.nx + 3;
    R.g.w = (int64_t)(R.P.nx + 3) * (R.P.ny + 3);
    R.fld_off = fo;
    R.sc_off = so;
    R.tmp_off = to;
    R.cg_off = co;
    fo += round64(EM2G_NFIELD * R.g.w);
    so += round64(6 * R.g.w * R.P.nsp);
    to += round64(6 * R.g.w);
    co += round64(4 * (int64_t)R.g.nx * R.g.ny);
    for (int s = 0; s < R.P.nsp; ++s) {
      R.cell0[s] = c0;
      R.base[s] = b0;
      R.n[s] = R.P.np_max[s];
      R.red_off[s] = ro;
      c0 += (int64_t)R.g.nx * R.g.ny;
      b0 += R.n[s];
      ro += push_partials(R.g.nx, R.g.ny) + 8;
    }
    e->any_smooth_current = e->any_smooth_current || R.P.smooth_current;
  }
  e->fld_n = fo;
  e->scaled_n = so;
  e->tmp_n = to;
  e->cgv_n = co;
  e->red_n = std::max<int64_t>(ro, 6 * kEnergyBlocks + 8);
  cudaError_t ce = cudaSetDevice(e->device);
  if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaSetDevice"));
  ce = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, e->device);
  if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaDeviceGetAttribute"));
  ce = cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaStreamCreate"));
  e->stream = e->own_stream;
#define ALLOC(ptr, bytes)                                                 \
  do {                                                                    \
    ce = cudaMalloc((void **)&(ptr), (bytes));                            \
    if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaMalloc " #ptr)); \
  } while (0)
  ALLOC(e->fld, sizeof(float) * e->fld_n);
  ALLOC(e->scaled, sizeof(float) * e->scaled_n);
  ALLOC(e->tmp, sizeof(float) * e->tmp_n);
  ALLOC(e->cgv, sizeof(float) * e->cgv_n);
  ALLOC(e->red, sizeof(double) * e->red_n);
  ALLOC(e->dev_out, sizeof(double) * (kEnsOut * (int64_t)nruns + 16));
  ALLOC(e->p32, sizeof(float) * 5 * cap);
  ALLOC(e->p32_alt, sizeof(float) * 5 * cap);
  ALLOC(e->slot, sizeof(int32_t) * cap);
  ALLOC(e->slot_alt, sizeof(int32_t) * cap);
  ALLOC(e->off, sizeof(int32_t) * (ncell + 1));
  ALLOC(e->off_alt, sizeof(int32_t) * (ncell + 1));
  ALLOC(e->cnt, sizeof(int32_t) * ncell);
  ALLOC(e->cnt_alt, sizeof(int32_t) * ncell);
  ALLOC(e->cursor, sizeof(int32_t) * ncell);
  ALLOC(e->scan_tmp, sizeof(int32_t) * scan_tmp_size(ncell));
  ALLOC(e->counter, sizeof(int));
  ALLOC(e->d_it, sizeof(int));
#undef ALLOC
  ce = cudaMallocHost((void **)&e->host_out, sizeof(double) * (kEnsOut * (int64_t)nruns + 16));
  if (ce == cudaSuccess) ce = cudaMallocHost((void **)&e->host_status, sizeof(int) * 2 * nruns);
  if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaMallocHost"));
  ce = cudaMemset(e->fld, 0, sizeof(float) * e->fld_n);
  if (ce == cudaSuccess) ce = cudaMemset(e->dev_out, 0, sizeof(double) * (kEnsOut * nruns + 16));
  if (ce == cudaSuccess) ce = cudaMemset(e->cnt, 0, sizeof(int32_t) * ncell);
  if (ce == cudaSuccess) ce = cudaMemset(e->d_it, 0, sizeof(int));
  if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaMemset"));
  int rc = ens_cg_setup(e);
  if (rc) return bail(rc);
  ce = cudaDeviceSynchronize();
  if (ce != cudaSuccess) return bail(cuda_fail(ce, "cudaDeviceSynchronize"));
  *out = e;
  return EM2G_OK;
}

int em2g_ens_destroy(em2g_ens *e) {
  if (!e) return EM2G_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop_graphs(e);
  void *bufs[] = {e->fld,   e->scaled,  e->tmp,      e->cgv,        e->red,     e->dev_out,
                  e->p32,   e->p32_alt, e->slot,     e->slot_alt,   e->off,     e->off_alt,
                  e->cnt,   e->cnt_alt, e->cursor,   e->scan_tmp,   e->counter, e->d_it,
                  e->staging, e->cg_partial, e->cg_bar, e->cg_status, e->fused_tab,
                  e->step_sync, e->fused_partial, e->fused_sums, e->fused_marks};
  for (void *p : bufs) cudaFree(p);
  ::operator delete(e->fused_push);
  if (e->host_out) cudaFreeHost(e->host_out);
  if (e->host_status) cudaFreeHost(e->host_status);
  if (e->own_stream) cudaStreamDestroy(e->own_stream);
  delete e;
  return EM2G_OK;
}

int em2g_ens_num_runs(em2g_ens *e, int *nruns) {
  int rc = check_ens(e);
  if (rc) return rc;
  if (!nruns) return fail(EM2G_ERR_INVALID, "null pointer");
  *nruns = (int)e->runs.size();
  return EM2G_OK;
}

int em2g_ens_set_stream(em2g_ens *e, void *stream) {
  int rc = check_ens(e);
  if (rc) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : e->own_stream;
  if (s != e->stream) {
    EM2G_CUDA(cudaStreamSynchronize(e->stream));
    e->stream = s;
  }
  return EM2G_OK;
}

int em2g_ens_set_fused(em2g_ens *e, int on) {
  int rc = check_ens(e);
  if (rc) return rc;
  if ((on != 0) != e->fused) {
    EM2G_CUDA(cudaStreamSynchronize(e->stream));
    drop_graphs(e);
    e->fused = on != 0;
  }
  return EM2G_OK;
}

int em2g_ens_set_graph(em2g_ens *e, int on) {
  int rc = check_ens(e);
  if (rc) return rc;
  e->use_graph = on != 0;
  return EM2G_OK;
}

int em2g_ens_num_variants(em2g_ens *e, int *n) {
  int rc = check_ens(e);
  if (rc) return rc;
  if (!n) return fail(EM2G_ERR_INVALID, "null pointer");
  *n = num_variants_f32();
  return EM2G_OK;
}

int em2g_ens_set_variant(em2g_ens *e, int v) {
  int rc = check_ens(e);
  if (rc) return rc;
  if (v < 0 || v >= num_variants_f32()) return fail(EM2G_ERR_INVALID, "variant out of range");
  if (v != e->variant) {
    EM2G_CUDA(cudaStreamSynchronize(e->stream));
    drop_graphs(e);
    e->variant = v;
  }
  return EM2G_OK;
}

int em2g_ens_set_sort_interval(em2g_ens *e, int k) {
  int rc = check_ens(e);
  if (rc) return rc;
  for (const EnsRun &R : e->runs) {
    em2g_params p = R.P;
    p.sort_interval = k;
    if ((rc = validate_params(&p))) return rc;  // k * c * dt < dx, dy for every run
  }
  k = std::max(k, 1);
  if (k != e->sort_interval) {
    EM2G_CUDA(cudaStreamSynchronize(e->stream));
    drop_graphs(e);
    e->sort_interval = k;
    for (EnsRun &R : e->runs) R.P.sort_interval = k;
  }
  return EM2G_OK;
}

int em2g_ens_set_fields(em2g_ens *e, int run, const double *host13) {
  int rc = check_pair(e, run, 0);
  if (rc) return rc;
  if (!host13) return fail(EM2G_ERR_INVALID, "null pointer");
  const EnsRun &R = e->runs[run];
  const int64_t n = EM2G_NFIELD * R.g.w;
  std::vector<float> tmp((size_t)n);
  for (int64_t k = 0; k < n; ++k) {
    if (!std::isfinite(host13[k])) return fail(EM2G_ERR_NONFINITE, "non-finite field value");
    tmp[k] = (float)host13[k];
  }
  EM2G_CUDA(cudaMemcpyAsync(e->fld + R.fld_off, tmp.data(), sizeof(float) * n,
                            cudaMemcpyHostToDevice, e->stream));
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  return EM2G_OK;
}

int em2g_ens_get_fields(em2g_ens *e, int run, double *host13) {
  int rc = check_pair(e, run, 0);
  if (rc) return rc;
  if (!host13) return fail(EM2G_ERR_INVALID, "null pointer");
  const EnsRun &R = e->runs[run];
  const int64_t n = EM2G_NFIELD * R.g.w;
  std::vector<float> tmp((size_t)n);
  EM2G_CUDA(cudaMemcpyAsync(tmp.data(), e->fld + R.fld_off, sizeof(float) * n,
                            cudaMemcpyDeviceToHost, e->stream));
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  for (int64_t k = 0; k < n; ++k) host13[k] = tmp[k];
  return EM2G_OK;
}

static int set_particles_common(em2g_ens *e, int run, int isp, int64_t n, const double *const *src,
                                cudaMemcpyKind kind) {
  EnsRun &R = e->runs[run];
  if (n != R.n[isp])
    return fail(EM2G_ERR_RANGE, "an ensemble run holds exactly np_max particles per species");
  for (int k = 0; k < 6; ++k)
    if (!src[k]) return fail(EM2G_ERR_INVALID, "null particle array");
  int rc = ensure_staging(e, n);
  if (rc) return rc;
  for (int k = 0; k < 6; ++k)
    EM2G_CUDA(cudaMemcpyAsync(e->staging + k * n, src[k], sizeof(double) * n, kind, e->stream));
  unsigned long long *bad = (unsigned long long *)e->red;
  if ((rc = check_particles_device(e->staging, n, n, R.P.nx + 0.5, R.P.ny + 0.5, bad, e->stream)))
    return rc;
  unsigned long long hb[2] = {0, 0};
  EM2G_CUDA(cudaMemcpyAsync(hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, e->stream));
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  if (hb[1]) return fail(EM2G_ERR_NONFINITE, std::to_string(hb[1]) + " non-finite particles");
  if (hb[0]) return fail(EM2G_ERR_RANGE, std::to_string(hb[0]) + " particles outside the grid");
  if ((rc = ens_upload_pair(e, run, isp, e->staging))) return rc;
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  R.loaded[isp] = true;
  return EM2G_OK;
}

int em2g_ens_set_particles(em2g_ens *e, int run, int isp, int64_t n, const double *x,
                           const double *y, const double *vx, const double *vy, const double *vz,
                           const double *gamma) {
  int rc = check_pair(e, run, isp);
  if (rc) return rc;
  const double *src[6] = {x, y, vx, vy, vz, gamma};
  return set_particles_common(e, run, isp, n, src, cudaMemcpyHostToDevice);
}

int em2g_ens_set_particles_device(em2g_ens *e, int run, int isp, int64_t n, const double *x,
                                  const double *y, const double *vx, const double *vy,
                                  const double *vz, const double *gamma) {
  int rc = check_pair(e, run, isp);
  if (rc) return rc;
  const double *src[6] = {x, y, vx, vy, vz, gamma};
  return set_particles_common(e, run, isp, n, src, cudaMemcpyDeviceToDevice);
}

int em2g_ens_get_particles(em2g_ens *e, int run, int isp, int64_t *n, double *x, double *y,
                           double *vx, double *vy, double *vz, double *gamma) {
  int rc = check_pair(e, run, isp);
  if (rc) return rc;
  const EnsRun &R = e->runs[run];
  const int64_t np = R.n[isp];
  if (n) *n = np;
  if (!x && !y && !vx && !vy && !vz && !gamma) return EM2G_OK;  // count query
  if (!x || !y || !vx || !vy || !vz || !gamma) return fail(EM2G_ERR_INVALID, "null particle array");
  if (!R.loaded[isp]) return fail(EM2G_ERR_INVALID, "particles of this pair were never set");
  if ((rc = ensure_staging(e, np))) return rc;
  if ((rc = ens_download_pair(e, run, isp, e->staging))) return rc;
  double *dst[6] = {x, y, vx, vy, vz, gamma};
  for (int k = 0; k < 6; ++k)
    EM2G_CUDA(cudaMemcpyAsync(dst[k], e->staging + k * np, sizeof(double) * np,
                              cudaMemcpyDeviceToHost, e->stream));
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  return EM2G_OK;
}

int em2g_ens_step(em2g_ens *e, int nsteps, double *ake_out, double *energies_out,
                  int *cg_iters_out) {
  em2g::NvtxRange nvtx_range("em2g ensemble step");
  int rc = check_ens(e);
  if (rc) return rc;
  if (nsteps < 0) return fail(EM2G_ERR_INVALID, "nsteps < 0");
  for (const EnsRun &R : e->runs)
    for (int s = 0; s < R.P.nsp; ++s)
      if (!R.loaded[s]) return fail(EM2G_ERR_INVALID, "set every run's particles before stepping");
  const int nr = (int)e->runs.size();
  EM2G_CUDA(cudaMemsetAsync(e->cg_status, 0, sizeof(int) * 2 * nr, e->stream));
  if (e->step_sync)
    EM2G_CUDA(cudaMemsetAsync(e->step_sync + 2, 0, sizeof(unsigned), e->stream));
  for (int k = 0; k < nsteps; ++k) {
    const bool inplace = next_inplace(e);
    if (e->use_graph) {
      const int key = graph_key(e, inplace);
      if (!e->exec[key] && (rc = capture_step(e, inplace))) return rc;
      EM2G_CUDA(cudaGraphLaunch(e->exec[key], e->stream));
      e->graph_launches += 1;
      e->kernels_per_step = e->graph_kernels[key];
    } else if (e->fused) {
      const int key = graph_key(e, inplace);
      if ((rc = ens_fused_prepare(e, key, inplace))) return rc;
      if ((rc = enqueue_step(e, inplace))) return rc;
      e->kernels_per_step = 1;
    } else {
      if ((rc = enqueue_step(e, inplace))) return rc;
      // prescale, tick, the push's and the fields' kernels
      e->kernels_per_step = 2 + ens_push_kernels_per_step(e, inplace) + ens_fields_kernels(e);
    }
    e->launches += e->kernels_per_step;
    if (inplace) {
      ++e->since_sort;
    } else {
      e->since_sort = 0;
      e->parity ^= 1;
    }
    e->cparity ^= 1;
    e->it += 1;
  }
  EM2G_CUDA(cudaMemcpyAsync(e->host_out, e->dev_out, sizeof(double) * kEnsOut * nr,
                            cudaMemcpyDeviceToHost, e->stream));
  EM2G_CUDA(cudaMemcpyAsync(e->host_status, e->cg_status, sizeof(int) * 2 * nr,
                            cudaMemcpyDeviceToHost, e->stream));
  unsigned step_timeout = 0;
  if (e->step_sync)
    EM2G_CUDA(cudaMemcpyAsync(&step_timeout, e->step_sync + 2, sizeof(unsigned),
                              cudaMemcpyDeviceToHost, e->stream));
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  EM2G_CUDA(cudaGetLastError());
  if (step_timeout) {
    // the barrier's count is left undefined by a wait that gave up
    EM2G_CUDA(cudaMemsetAsync(e->step_sync, 0, sizeof(unsigned) * 3, e->stream));
    EM2G_CUDA(cudaStreamSynchronize(e->stream));
    return fail(EM2G_ERR_TIMEOUT, "fused ensemble step: a grid barrier wait timed out");
  }
  for (int r = 0; r < nr; ++r)
    if (e->host_status[2 * r])
      return fail(EM2G_ERR_TIMEOUT, "cg of run " + std::to_string(r) + ": a barrier wait timed out");
  for (int r = 0; r < nr; ++r) {
    const double lost = e->host_out[(int64_t)r * kEnsOut + kEnsLost];
    if (lost != 0.0) {
      EM2G_CUDA(cudaMemsetAsync(e->dev_out + (int64_t)r * kEnsOut + kEnsLost, 0, sizeof(double),
                                e->stream));
      return fail(EM2G_ERR_RANGE, "regrouping push of run " + std::to_string(r) + ": " +
                                      std::to_string((long long)lost) +
                                      " particles fell outside their cells' ranges");
    }
  }
  for (int r = 0; r < nr; ++r) {
    const EnsRun &R = e->runs[r];
    const double *o = e->host_out + (int64_t)r * kEnsOut;
    if (ake_out)
      for (int s = 0; s < EM2G_MAX_SPECIES; ++s) ake_out[4 * r + s] = s < R.P.nsp ? o[s] : 0.0;
    if (energies_out && nsteps > 0 && e->it % R.P.isav == 0)
      for (int k = 0; k < 6; ++k) energies_out[6 * r + k] = o[4 + k];
    if (cg_iters_out) cg_iters_out[r] = nsteps > 0 ? e->host_status[2 * r + 1] : 0;
  }
  return EM2G_OK;
}

int em2g_ens_get_step(em2g_ens *e, int *it) {
  int rc = check_ens(e);
  if (rc) return rc;
  if (!it) return fail(EM2G_ERR_INVALID, "null pointer");
  *it = e->it;
  return EM2G_OK;
}

int em2g_ens_diagnostics(em2g_ens *e, int run, double *out, int nout) {
  int rc = check_pair(e, run, 0);
  if (rc) return rc;
  if (!out || nout < 1) return fail(EM2G_ERR_INVALID, "null or empty output");
  const EnsRun &R = e->runs[run];
  double *scratch = e->dev_out + kEnsOut * (int64_t)e->runs.size();  // 16 doubles
  if ((rc = diag_fields_f32(e->fld + R.fld_off, R.g, R.P.dx, e->red, scratch, e->stream)))
    return rc;
  double h[EM2G_NDIAG];
  EM2G_CUDA(cudaMemcpyAsync(h, scratch, sizeof(double) * 8, cudaMemcpyDeviceToHost, e->stream));
  EM2G_CUDA(cudaMemcpyAsync(h + 8, e->dev_out + (int64_t)run * kEnsOut + 10, sizeof(double) * 2,
                            cudaMemcpyDeviceToHost, e->stream));
  EM2G_CUDA(cudaStreamSynchronize(e->stream));
  for (int k = 0; k < std::min(nout, EM2G_NDIAG); ++k) out[k] = h[k];
  return EM2G_OK;
}

int em2g_ens_get_phase_ns(em2g_ens *e, int64_t *ns, int n) {
  int rc = check_ens(e);
  if (rc) return rc;
  if (!ns || n < 1 || n > 31) return fail(EM2G_ERR_INVALID, "ns must hold 1..31 values");
  return ens_fused_phase_ns(e, ns, n);
}

int em2g_ens_get_counters(em2g_ens *e, int64_t *kernel_launches, int64_t *graph_launches,
                          int64_t *kernels_per_step) {
  int rc = check_ens(e);
  if (rc) return rc;
  if (kernel_launches) *kernel_launches = e->launches;
  if (graph_launches) *graph_launches = e->graph_launches;
  if (kernels_per_step) *kernels_per_step = e->kernels_per_step;
  return EM2G_OK;
}

}  // extern "C"

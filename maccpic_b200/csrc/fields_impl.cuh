// fields_impl.cuh -- host side of fields (pic/fields.f90:2-367), smooth2
// and the Poisson solve, templated on the storage type of the field block
// (double: fields_f64.cu; float: fields_f32.cu).
#pragma once
#include <mutex>

#include "grid_kernels.cuh"
#include "tma_stencil.cuh"

namespace em2g {
namespace grid {
namespace {

inline G geom(const em2g_ctx *c) { return G{c->g.nx, c->g.ny, c->g.nxg, c->g.w}; }

inline dim3 grid_for(int nxc, int nyc) { return dim3((nxc + TX - 1) / TX, (nyc + TY - 1) / TY); }

template <typename T>
T *field_block(em2g_ctx *c);
template <>
inline float *field_block<float>(em2g_ctx *c) { return c->fld32; }
template <>
inline double *field_block<double>(em2g_ctx *c) { return c->fld; }

// ---- TMA-staged stages (tma_stencil.cuh)

// cuTensorMapEncodeTiled, looked up once through the runtime
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline int encode_tiled_fn(EncodeTiledFn *out) {
  static std::mutex mu;
  static EncodeTiledFn fn = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    EM2G_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000,
                                               cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p)
      return fail(EM2G_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  *out = fn;
  return EM2G_OK;
}

// A map over `rows` field rows of nxg elements from `base` (16-byte
// aligned), M rows to a line; the allocation must reach the last line's end.
template <typename T>
int encode_lines(CUtensorMap *m, T *base, int nxg, int64_t rows) {
  using Gm = tma::Geo<T>;
  EncodeTiledFn fn = nullptr;
  int rc = encode_tiled_fn(&fn);
  if (rc) return rc;
  if (reinterpret_cast<uintptr_t>(base) % 16 != 0)
    return fail(EM2G_ERR_CUDA, "tensor map base not 16-byte aligned");
  const cuuint64_t dim[2] = {(cuuint64_t)Gm::M * nxg, (cuuint64_t)((rows + Gm::M - 1) / Gm::M)};
  const cuuint64_t stride[1] = {(cuuint64_t)Gm::M * nxg * sizeof(T)};
  const cuuint32_t box[2] = {(cuuint32_t)Gm::BW, (cuuint32_t)Gm::BH};
  const cuuint32_t estride[2] = {1, 1};
  const CUresult r =
      fn(m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
         base, dim, stride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(EM2G_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return EM2G_OK;
}

template <typename T, int S>
int tma_prepare_stage(em2g_ctx *c) {
  constexpr int bytes = tma::smem_bytes<T, S>();
  EM2G_CUDA(cudaFuncSetAttribute(tma::k_tma_stage<T, S>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  int per_sm = 0;
  EM2G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tma::k_tma_stage<T, S>,
                                                          tma::Geo<T>::THREADS, bytes));
  if (per_sm < 1) return fail(EM2G_ERR_CUDA, "TMA stage kernel cannot be resident");
  return EM2G_OK;
}

// maps over the field block (13 arrays) and the smooth2 scratch (one), and
// the stage kernels' shared-memory sizes
template <typename T>
int tma_init_t(em2g_ctx *c, T *fld, T *tmp) {
  const G g = geom(c);
  int rc = encode_lines<T>(&c->tmap_fld, fld, g.nxg, (int64_t)EM2G_NFIELD * (g.ny + 3));
  if (!rc) rc = encode_lines<T>(&c->tmap_tmp, tmp, g.nxg, (int64_t)(g.ny + 3));
  if (!rc) rc = tma_prepare_stage<T, tma::kBHalf>(c);
  if (!rc) rc = tma_prepare_stage<T, tma::kEFull>(c);
  if (!rc) rc = tma_prepare_stage<T, tma::kBinomial>(c);
  if (!rc) rc = tma_prepare_stage<T, tma::kCompensate>(c);
  if (rc) return rc;
  c->tma_ok = true;
  return EM2G_OK;
}

template <typename T, int S>
int tma_launch(em2g_ctx *c, const CUtensorMap &map, const int *row0, const T *const *in, int nin,
               T *o0, T *o1, T *o2, T c0, T c1, T c2) {
  using Gm = tma::Geo<T>;
  tma::Args<T> a;
  a.g = geom(c);
  a.ntx = (a.g.nx + 1 + Gm::TXO - 1) / Gm::TXO;
  a.nty = (a.g.ny + 1 + Gm::TYO - 1) / Gm::TYO;
  a.ntiles = a.ntx * a.nty;
  for (int k = 0; k < tma::kStaged; ++k) a.row0[k] = k < tma::Staged<S>::N ? row0[k] : 0;
  for (int k = 0; k < 9; ++k) a.in[k] = k < nin ? in[k] : nullptr;
  a.out[0] = o0;
  a.out[1] = o1;
  a.out[2] = o2;
  a.c0 = c0;
  a.c1 = c1;
  a.c2 = c2;
  a.status = c->cg.status;
  tma::k_tma_stage<T, S><<<a.ntiles, Gm::THREADS, tma::smem_bytes<T, S>(), c->stream>>>(map, a);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

template <typename T>
int smooth2_t(em2g_ctx *c, T *a, T *tmp) {
  const G g = geom(c);
  if (c->stencils == 1) {
    // a is one of the field block's arrays: its row 0 in the block's map
    const int64_t k = (a - field_block<T>(c)) / g.w;
    const int src_row0 = (int)(k * (g.ny + 3)), tmp_row0 = 0;
    int rc = tma_launch<T, tma::kBinomial>(c, c->tmap_fld, &src_row0, nullptr, 0, tmp, nullptr,
                                           nullptr, T(0), T(0), T(0));
    if (!rc)
      rc = tma_launch<T, tma::kCompensate>(c, c->tmap_tmp, &tmp_row0, nullptr, 0, a, nullptr,
                                           nullptr, T(0), T(0), T(0));
    return rc;
  }
  const dim3 grd = grid_for(g.nx + 1, g.ny + 1), blk(TX, TY);
  k_smooth_binomial<T><<<grd, blk, 0, c->stream>>>(g, a, tmp);
  k_smooth_compensate<T><<<grd, blk, 0, c->stream>>>(g, tmp, a);
  c->launches += 2;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

template <typename T>
int cg_init_t(em2g_ctx *c) {
  CgWork &W = c->cg;
  const int64_t N = (int64_t)c->g.nx * c->g.ny;
  int per_sm = 0;
  EM2G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg<T>, W.threads, 0));
  if (per_sm < 1) return fail(EM2G_ERR_CUDA, "cg kernel cannot be resident");
  const int64_t want = (N + W.threads - 1) / W.threads;
  const int64_t maxb = (int64_t)per_sm * c->num_sms;
  W.blocks = (int)(want < maxb ? want : maxb);
  if (W.blocks < 1) W.blocks = 1;
  EM2G_CUDA(cudaMalloc(&W.u, sizeof(T) * N * 4));
  W.elem = sizeof(T);
  EM2G_CUDA(cudaMalloc(&W.partial, sizeof(double) * 2 * W.blocks));
  EM2G_CUDA(cudaMalloc(&W.bar, sizeof(unsigned) * 2));
  EM2G_CUDA(cudaMalloc(&W.status, sizeof(int) * 2));
  EM2G_CUDA(cudaMemset(W.bar, 0, sizeof(unsigned) * 2));
  return EM2G_OK;
}

// pic/fields.f90:384-442 + cgm :508-651.  The CG's exit count and a sticky
// timeout flag land in cg.status; the caller reads them after its last
// launch (no host synchronisation here).
template <typename T>
int poisson_t(em2g_ctx *c, T *fld) {
  const G g = geom(c);
  CgWork &W = c->cg;
  const int64_t N = (int64_t)g.nx * g.ny;
  T *u = (T *)W.u, *r = u + N, *p = u + 2 * N, *ap = u + 3 * N;
  const T dx = (T)c->P.dx, dy = (T)c->P.dy;
  const dim3 blk(TX, TY);
  k_poisson_rhs<T><<<grid_for(g.nx, g.ny), blk, 0, c->stream>>>(g, fld, dx, dy, r, p);
  EM2G_CUDA(cudaGetLastError());
  if constexpr (sizeof(T) == sizeof(double)) {
    if (c->P.poisson == 1) {  // exact solve instead of cgm
      int rc = spectral_solve(r, u, g.nx, g.ny, c->spec, c->stream);
      if (rc) return rc;
      k_poisson_correct<T><<<grid_for(g.nx, g.ny), blk, 0, c->stream>>>(g, fld, u, dx, dy);
      c->launches += 7;
      EM2G_CUDA(cudaGetLastError());
      return EM2G_OK;
    }
  }
  EM2G_CUDA(cudaMemsetAsync(W.bar, 0, sizeof(unsigned) * 2, c->stream));
  CgArgs<T> a;
  a.nx = g.nx;
  a.ny = g.ny;
  a.u = u;
  a.r = r;
  a.p = p;
  a.ap = ap;
  a.partial = W.partial;
  a.bar = W.bar;
  a.status = W.status;
  a.res = c->dev_out + 18;
  a.maxits = c->P.cg_maxits;
  a.eps = c->P.cg_eps;
  void *args[] = {&a};
  EM2G_CUDA(cudaLaunchCooperativeKernel((const void *)k_cg<T>, dim3(W.blocks),
                                        dim3(W.threads), args, 0, c->stream));
  k_poisson_correct<T><<<grid_for(g.nx, g.ny), blk, 0, c->stream>>>(g, fld, u, dx, dy);
  c->launches += 3;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

// pic/fields.f90:267-347 into dev_out[4..9]
template <typename T>
int energies_t(em2g_ctx *c, const T *fld) {
  const G g = geom(c);
  int lo = 1, hi = g.ny;
  const double alx = c->P.dx * g.nx, aly = c->P.dy * g.ny;
  const double t = c->P.qme / c->P.wpe / c->P.c;
  const double rnmec2i = t * t / (alx * aly);  // pic/global.f90:26-27
  const double anorml1 = 0.5 * c->P.dx * c->P.dy * rnmec2i;
  if (c->P.energy_mode == 1) {
    lo = 88;
    hi = 168;
  }
  const int nb = kEnergyBlocks;
  k_energy_partial<T><<<dim3(nb, 6), 256, 0, c->stream>>>(g, fld, lo, hi, c->red);
  k_energy_finish<<<6, 256, 0, c->stream>>>(c->red, nb, anorml1, c->P.energy_mode == 1, g.ny,
                                            c->dev_out + 4);
  c->launches += 2;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

template <typename T>
int fields_t(em2g_ctx *c, T *fld, T *tmp, int it, bool want_energies) {
  const G g = geom(c);
  const dim3 blk(TX, TY);
  // fold (pic/fields.f90:44-137)
  k_fold_x<T><<<dim3((g.ny + 3 + 127) / 128, 7), 128, 0, c->stream>>>(g, fld);
  k_fold_y<T><<<dim3((g.nx + 3 + 127) / 128, 7), 128, 0, c->stream>>>(g, fld);
  c->launches += 2;
  // optional current filter (no em2 counterpart): smooth2 of each J array
  if (c->P.smooth_current)
    for (int k = EM2G_JXM; k <= EM2G_JZP; ++k) {
      const bool is_jp = k == EM2G_JXP || k == EM2G_JYP || k == EM2G_JZP;
      if (is_jp && !c->jp_live) continue;
      const int rc = smooth2_t<T>(c, fld + k * g.w, tmp);
      if (rc) return rc;
    }
  // Yee (pic/fields.f90:184-247)
  const double ctx = c->P.dt * c->P.c / c->P.dx, cty = c->P.dt * c->P.c / c->P.dy;
  const double ctxh = ctx * 0.5, ctyh = cty * 0.5, tem = 0.5 * c->P.dt;
  if (c->stencils == 1) {
    // staged arrays' rows in the block's map (E for B/2, B for E), and the
    // arrays read at the cell, in the stage kernels' order
    const int rows = g.ny + 3;
    const int e_rows[3] = {EM2G_EX * rows, EM2G_EY * rows, EM2G_EZ * rows};
    const int b_rows[3] = {EM2G_BX * rows, EM2G_BY * rows, EM2G_BZ * rows};
    T *bx = fld + EM2G_BX * g.w, *by = fld + EM2G_BY * g.w, *bz = fld + EM2G_BZ * g.w;
    T *ex = fld + EM2G_EX * g.w, *ey = fld + EM2G_EY * g.w, *ez = fld + EM2G_EZ * g.w;
    const T *b_in[3] = {bx, by, bz};
    const T *e_in[9] = {ex, ey, ez, fld + EM2G_JXM * g.w, fld + EM2G_JXP * g.w,
                        fld + EM2G_JYM * g.w, fld + EM2G_JYP * g.w, fld + EM2G_JZM * g.w,
                        fld + EM2G_JZP * g.w};
    int rc = tma_launch<T, tma::kBHalf>(c, c->tmap_fld, e_rows, b_in, 3, bx, by, bz, (T)ctxh,
                                        (T)ctyh, T(0));
    if (!rc)
      rc = tma_launch<T, tma::kEFull>(c, c->tmap_fld, b_rows, e_in, 9, ex, ey, ez, (T)ctx, (T)cty,
                                      (T)tem);
    if (!rc)
      rc = tma_launch<T, tma::kBHalf>(c, c->tmap_fld, e_rows, b_in, 3, bx, by, bz, (T)ctxh,
                                      (T)ctyh, T(0));
    if (rc) return rc;
  } else {
    const dim3 grd = grid_for(g.nx + 1, g.ny + 1);
    k_b_half<T><<<grd, blk, 0, c->stream>>>(g, fld, (T)ctxh, (T)ctyh);
    k_e_full<T><<<grd, blk, 0, c->stream>>>(g, fld, (T)ctx, (T)cty, (T)tem);
    k_b_half<T><<<grd, blk, 0, c->stream>>>(g, fld, (T)ctxh, (T)ctyh);
    c->launches += 3;
    EM2G_CUDA(cudaGetLastError());
  }
  // filters (pic/fields.f90:252-260)
  int rc = smooth2_t<T>(c, fld + EM2G_RHO * g.w, tmp);
  if (rc) return rc;
  if (it % c->P.isav == 0)
    for (int k = EM2G_EX; k <= EM2G_BZ; ++k)
      if ((rc = smooth2_t<T>(c, fld + k * g.w, tmp))) return rc;
  // Poisson (pic/fields.f90:262)
  if ((rc = poisson_t<T>(c, fld))) return rc;
  // energies (pic/fields.f90:267-347)
  if (want_energies && it % c->P.isav == 0)
    if ((rc = energies_t<T>(c, fld))) return rc;
  // reset rho and J (pic/fields.f90:353-365)
  EM2G_CUDA(cudaMemsetAsync(fld + EM2G_RHO * g.w, 0, sizeof(T) * 7 * g.w, c->stream));
  c->jp_live = false;
  return EM2G_OK;
}

}  // namespace
}  // namespace grid
}  // namespace em2g

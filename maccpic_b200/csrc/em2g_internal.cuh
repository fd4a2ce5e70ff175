// em2g_internal.cuh -- context layout and kernel entry points shared by the
// translation units of libem2g.so.  Not part of the public ABI.
#pragma once
#include <cuda.h>  // CUtensorMap (the map is encoded through the runtime's driver entry point)
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>  // header-only; inert unless a profiler is attached
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/em2g.h"

namespace em2g {

constexpr int kEnergyBlocks = 296;
// ensembles (ensemble_api.cu): runs, and (run, species) pairs, per ensemble
constexpr int kEnsMaxRuns = 128;
constexpr int kEnsMaxPairs = 160;  // partial sums per field in the energy reduction
// small device results, mirrored to pinned host memory after each call:
// [0,4) ake per species, [4,10) energies at isav steps, [10,16) energies of
// the current fields, [16,18) reconnected flux of the two sheets, [18,20)
// mean r^2 of the last Poisson solve before and after the CG
constexpr int kDevOut = 32;
// dev_out[kDevLost]: particles a regrouping push found no place for (their
// cell counts disagreed with where they were; the state is then corrupt and
// the step fails -- a guard, never expected to count)
constexpr int kDevLost = kDevOut - 1;

// Sets the per-thread error message and returns the status (api.cu).
int fail(int status, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

// An NVTX range around one ABI call or step phase, so that a timeline
// profiler groups the kernels each one launches under the em2 routine they
// stand for (move, curnt, fields, ...).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

#define EM2G_CUDA(call)                                  \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return cuda_fail(_e, #call);  \
  } while (0)

// Grid geometry of the (0:nx+2, 0:ny+2) arrays.
struct Grid {
  int nx, ny;
  int nxg;      // nx + 3
  int64_t w;    // (nx+3)*(ny+3)
};

// One species' particles on the device, FP64 layout of the reference:
// six arrays of `cap` doubles (x, y, vx, vy, vz, gamma) back to back,
// plus the original slot of each entry (for returning particles in slot
// order after sorting).
struct Species {
  int64_t n = 0, cap = 0;
  double *part = nullptr;      // 6*cap
  int32_t *slot = nullptr;     // cap
  double *part_alt = nullptr;  // 6*cap, sort target
  int32_t *slot_alt = nullptr;
  // Cell-sorted order of the fast path (push_fast_f64.cu, sort.cu): `part`
  // holds the particles grouped by cell (row-major key iy*nx+ix), cell k's
  // particles at [off[k], off[k+1]); cnt[k] counts the particles whose
  // current position lies in cell k.  `sorted` is false until a full sort
  // ran after the last change of positions outside the fast path.
  int32_t *off = nullptr, *off_alt = nullptr;  // ncell+1 each
  int32_t *cnt = nullptr, *cnt_alt = nullptr;  // ncell each
  int32_t *cursor = nullptr;                   // ncell
  bool sorted = false;
  // FP32 contexts: xr, yr (offsets in the cell of the particle's range),
  // ux, uy, uz; 5*cap floats, always grouped by cell (push_fast_f32.cu)
  float *p32 = nullptr, *p32_alt = nullptr;
  int since_sort = 0;  // FP32 pushes in place since the last regrouping
  // an upload in slices (em2g_particles_begin / add / end): the announced
  // count (-1: none open) and the slots added so far, in order.  The slices
  // are parked in the alternate buffers; the species' particles change only
  // at the end, once every slot passed the checks.
  int64_t up_n = -1, up_added = 0;
};

// Device workspace of the Poisson/cgm solve (pic/fields.f90:370-651).
struct CgWork {
  void *u = nullptr;           // u, r, p, Ap: 4 arrays of nx*ny elements
  int elem = 0;                // element size (8 FP64, 4 FP32)
  double *partial = nullptr;   // 2 * max_blocks
  unsigned *bar = nullptr;     // barrier counter + generation
  int *status = nullptr;       // [0] timeout flag, [1] iterations
  int blocks = 0, threads = 256;
};

}  // namespace em2g

struct em2g_ctx {
  em2g_params P;
  em2g::Grid g;
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  int it = 0;
  // 13 field arrays of w doubles back to back (enum em2g_field order)
  double *fld = nullptr;
  // per-species copies of E and B scaled by (q/m)dt/2 (pic/move.f90:52-64)
  double *scaled = nullptr;  // nsp * 6 * w
  double *smooth_tmp = nullptr;  // w, the `dummy` array of smooth2
  // FP32 contexts use these instead of fld / scaled / smooth_tmp
  float *fld32 = nullptr, *scaled32 = nullptr, *smooth_tmp32 = nullptr;
  em2g::Species sp[EM2G_MAX_SPECIES];
  em2g::CgWork cg;
  // reductions: ake partials per species, energy partials
  double *red = nullptr;       // reduction scratch
  int red_blocks = 0;
  double *ake_l1 = nullptr;    // kAkeBlocks first-level sums of the ake partials
  double *dev_out = nullptr;   // small device results (ake[4], e[6])
  double *host_out = nullptr;  // pinned mirror of dev_out
  int num_sms = 0;
  // counters (em2g_get_counters): kernel launches, and when timing is on,
  // CUDA-event time of the particle-push launches
  int64_t launches = 0;
  int32_t *scan_tmp = nullptr;  // block sums of the cell scans
  int variant = 0;              // fast-push kernel variant (em2g_set_variant)
  // false while jxp, jyp, jzp are known to hold zeros (after fields, and
  // the fast path deposits the whole current into jxm, jym, jzm)
  bool jp_live = true;
  double2 *spec = nullptr;  // nx*ny complex work of the spectral Poisson solve
  // FP64 staging of host copies and the regrouping's records, grown on
  // demand up to the field block or staging_cap(): particle copies go
  // through it in slices, so it stays bounded on any particle count
  double *staging = nullptr;
  int64_t staging_n = 0;
  unsigned long long *up_bad = nullptr;  // per species: out of range, non-finite
  // host particle copies overlap their PCIe transfers with the device work on
  // the other half of the staging buffer: a second stream for the copies and,
  // per half, events marking its copy done and its device work done
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t half_copied[2] = {nullptr, nullptr}, half_used[2] = {nullptr, nullptr};
  int64_t ncell = 0;
  // TMA-staged Yee and smooth2 stages (tma_stencil.cuh): tensor maps over the
  // field block and over the smooth2 scratch, and which implementation the
  // field solve runs (0: direct loads, 1: TMA-staged tiles; em2g_set_stencils)
  CUtensorMap tmap_fld, tmap_tmp;
  bool tma_ok = false;
  int stencils = 0;
  int timing = 0;
  std::vector<cudaEvent_t> ev;  // start/stop pairs of the pending push launches
  size_t ev_used = 0;
  double push_ms = 0.0;
  int64_t push_timed = 0;
};

namespace em2g {

// ---- kernels launched from api.cu (defined in push_f64.cu / fields_f64.cu)
int launch_prescale(em2g_ctx *c, int isp);
// mode bit 1: move (gather + Boris); bit 2: curnt (deposit, move, deposit)
int launch_push_f64(em2g_ctx *c, int isp, int mode);
// the kinetic energy of species isp from the push's nblocks_used partials
// in c->red: summed in a fixed order (kAkeBlocks blocks over contiguous
// chunks, then one block), so that it does not change from run to run
constexpr int kAkeBlocks = 256;
int launch_ake_finish(em2g_ctx *c, int isp, int nblocks_used);
int fields_f64(em2g_ctx *c, int it, bool want_energies, int *cg_iters);
int smooth2_f64(em2g_ctx *c, double *a);
int cg_init(em2g_ctx *c);
// cell sort of the fast path (sort.cu)
int sort_init(em2g_ctx *c);
void sort_free(em2g_ctx *c);
int sort_full(em2g_ctx *c, int isp);
int scan_cells(em2g_ctx *c, const int32_t *cnt, int32_t *off);
// one fast-path push of species isp (push_fast_f64.cu)
int launch_push_cells_f64(em2g_ctx *c, int isp);
// fast-push variants (tile width x occupancy) for the autotuner
int num_variants_f64();
const char *variant_name_f64(int v);
int num_variants_f32();
const char *variant_name_f32(int v);
// mixed-precision path (push_fast_f32.cu, fields_f32.cu)
int launch_prescale_f32(em2g_ctx *c, int isp);
int launch_push_cells_f32(em2g_ctx *c, int isp);
// particle transfers of FP32 contexts in slices (push_fast_f32.cu).
// stage_f32: slots first..first+count from six device arrays (src[k][i] for
// slot first+i), checked and parked unsorted in the alternate buffers, their
// cells counted in cnt_alt, rejects counted in bad[0..2).  commit_f32: the
// parked n particles regrouped by cell into the current buffers through
// 32-byte records, rec_cap records at a time (rec: 16-byte aligned).
// get_range_f32: slots first..first+count in FP64 into dst[k][i] (device
// memory) through rec (32 bytes per slot of the range).
int stage_f32(em2g_ctx *c, int isp, int64_t first, int64_t count, const double *const *src,
              unsigned long long *bad);
int commit_f32(em2g_ctx *c, int isp, int64_t n, void *rec, int64_t rec_cap);
int get_range_f32(em2g_ctx *c, int isp, int64_t first, int64_t count, double *const *dst,
                  void *rec);
// bytes of the staging buffer particle copies go through: 80 bytes per
// particle of the largest species, at most 80 * 2^24 (1.3 GB)
int64_t staging_cap(const em2g_ctx *c);
int smooth2_f32(em2g_ctx *c, float *a);
// tensor maps and launch shapes of the TMA-staged stages (fields_f32.cu,
// fields_f64.cu); the field block and the smooth2 scratch must carry
// tma_tail_elems() elements of tail
int tma_init_f32(em2g_ctx *c);
// em2g_selftest_waits (fields_f64.cu)
int selftest_waits(em2g_ctx *c, int *cg_status, int *tma_status);
int tma_init_f64(em2g_ctx *c);
inline int64_t tma_tail_elems(const em2g_ctx *c, bool fp32) {
  return (int64_t)(fp32 ? 4 : 2) * c->g.nxg;  // 16 bytes' worth of rows
}
int cg_init_f32(em2g_ctx *c);
int fields_f32(em2g_ctx *c, int it, bool want_energies);
// em2g_diagnostics into dev_out[10..20) (diag.cu)
int diagnostics(em2g_ctx *c);
// bracket one push launch with events when timing is on (api.cu)
int timing_begin(em2g_ctx *c);
int timing_end(em2g_ctx *c);
void cg_free(em2g_ctx *c);
// kinetic-energy partials one fast push of an nx x ny grid writes, for the
// widest-writing variant: ceil(nx/tcx) * ny segments of tcx*g/32 warps, with
// tcx 32 or 64 cells and g <= 8 lanes per cell -- at most 8 warps per 32
// cells
inline int64_t push_partials(int nx, int ny) { return (int64_t)((nx + 31) / 32) * 8 * ny; }
// exact periodic Poisson solve by FFT (spectral.cu)
bool spectral_size_ok(int nx, int ny);
int spectral_prepare();
int spectral_solve(const double *f, double *u, int nx, int ny, double2 *work, cudaStream_t st);
// one em2g_step pass enqueued without host synchronisation (api.cu)
int step_enqueue(em2g_ctx *c);
// the checks em2g_create applies to a parameter block (api.cu)
int validate_params(const em2g_params *p);
// counts particles of a 6 x ld FP64 block outside [0, xlim) x [0, ylim)
// into bad[0] and those with non-finite values into bad[1], after zeroing
// both unless reset is false (api.cu)
int check_particles_device(const double *part, int64_t n, int64_t ld, double xlim, double ylim,
                           unsigned long long *bad, cudaStream_t st, bool reset = true);
// energies of the current fields and the reconnected flux of both sheets
// of one FP32 field block into out[0..8); red: 6*kEnergyBlocks doubles
// (diag.cu)
int diag_fields_f32(const float *fld, const Grid &g, double dx, double *red, double *out,
                    cudaStream_t st);
// exclusive scan of cnt[0..n) into off[0..n], plus `base`, on `stream`;
// tmp holds scan_tmp_size(n) ints (sort.cu)
int64_t scan_tmp_size(int64_t n);
int scan_counts(const int32_t *cnt, int32_t *off, int64_t n, int32_t base, int32_t *tmp,
                cudaStream_t stream);

}  // namespace em2g

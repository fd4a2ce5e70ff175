// ens_internal.cuh -- layout of an ensemble of independent FP32 runs that
// advance together (ensemble_api.cu), and the launchers its step uses.
// Not part of the public ABI.
//
// Device layout.  Every array kind of all runs lives in one allocation,
// run after run:
//   fld     13 arrays of w_r floats per run (enum em2g_field order)
//   scaled  nsp_r * 6 * w_r floats per run ((E, B) pairs, push_fast_f32.cu)
//   tmp     6 * w_r floats per run (smooth2 scratch of up to six arrays)
//   cgv     4 * nx_r * ny_r floats per run (u, r, p, Ap of the CG)
// Particles of all (run, species) pairs share one cell-grouped buffer pair
// (p32/p32_alt, 5 * cap floats, and their slots): pair (r, s) owns the
// slots base[r][s] .. base[r][s] + n[r][s] - 1, and its cells are the keys
// cell0[r][s] .. cell0[r][s] + nx_r*ny_r - 1 of the shared count and
// offset arrays.  Because every pair holds exactly n[r][s] particles, one
// exclusive scan over all pairs' counts yields every pair's offsets.
#pragma once
#include "em2g_internal.cuh"

namespace em2g {

// per run: [0,4) ake of the last step, [4,10) energies of the last isav
// step, [10,12) mean r^2 before and after the last CG
constexpr int kEnsOut = 16;
constexpr int kEnsLost = kEnsOut - 1;  // per run, as kDevLost of a context

struct EnsRun {
  em2g_params P;
  Grid g;
  int64_t fld_off = 0, sc_off = 0, tmp_off = 0, cg_off = 0;  // elements
  int64_t cell0[EM2G_MAX_SPECIES] = {};
  int64_t base[EM2G_MAX_SPECIES] = {};
  int64_t n[EM2G_MAX_SPECIES] = {};
  int64_t red_off[EM2G_MAX_SPECIES] = {};  // first ake partial of the pair
  bool loaded[EM2G_MAX_SPECIES] = {};
  int cg_block0 = 0, cg_blocks = 0;
};

}  // namespace em2g

struct em2g_ens {
  int device = 0;
  int num_sms = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<em2g::EnsRun> runs;
  int npairs = 0;
  bool any_smooth_current = false;
  // grids
  float *fld = nullptr, *scaled = nullptr, *tmp = nullptr, *cgv = nullptr;
  int64_t fld_n = 0, scaled_n = 0, tmp_n = 0, cgv_n = 0;
  double *cg_partial = nullptr;  // 2 per CG block
  unsigned *cg_bar = nullptr;    // 2 per run
  int *cg_status = nullptr;      // 2 per run: timeout flag, iterations
  int cg_blocks = 0;
  double *red = nullptr;         // ake partials of all pairs
  int64_t red_n = 0;
  double *dev_out = nullptr;     // kEnsOut per run
  double *host_out = nullptr;    // pinned mirror of dev_out
  int *host_status = nullptr;    // pinned mirror of cg_status
  // particles; parity 0: current = p32/slot/off, next = the _alt set;
  // cparity 0: current cell counts = cnt.  A regrouping push flips both,
  // an in-place push (between regroupings, sort_interval > 1) only cparity.
  float *p32 = nullptr, *p32_alt = nullptr;
  int32_t *slot = nullptr, *slot_alt = nullptr;
  int32_t *off = nullptr, *off_alt = nullptr, *cnt = nullptr, *cnt_alt = nullptr;
  int32_t *cursor = nullptr, *scan_tmp = nullptr;
  int64_t cap = 0, ncell = 0;
  int parity = 0, cparity = 0;
  int sort_interval = 1;  // regroup on every sort_interval-th push
  int since_sort = 0;     // in-place pushes since the last regrouping
  double *staging = nullptr;  // 10 * staging_n doubles: 6 per particle of FP64 values,
                              // then a 32-byte record each (uploads, downloads)
  int64_t staging_n = 0;
  int *counter = nullptr;     // the persistent push's segment counter
  int *d_it = nullptr;        // the step counter as the field kernels read it
  int it = 0;
  int variant = 0;
  // one captured graph per (in place, parity, cparity); invalid after a
  // change of variant, sort interval or stream
  bool use_graph = true;
  // 1: each step is one persistent, cooperative launch (ens_step.cu);
  // 0: one launch per stage (push_fast_f32.cu, fields_ens.cu)
  bool fused = false;
  void *fused_tab = nullptr;       // 8 step tables, one per kind of step (device)
  void *fused_push = nullptr;      // 8 push tables, the launch's parameter (host)
  unsigned *step_sync = nullptr;   // [0, 2) the step's grid barrier, [2] its timeout flag
  double *fused_partial = nullptr; // the CG's partial sums, 2 per block of the launch
  int32_t *fused_sums = nullptr;   // the scan's chunk totals
  unsigned long long *fused_marks = nullptr;  // global timer at the fused step's barriers
  int fused_blocks = 0;
  bool fused_ready[8] = {};        // step tables written for the current variant
  cudaGraphExec_t exec[8] = {};
  int64_t graph_kernels[8] = {};
  int64_t kernels_per_step = 0;
  int64_t launches = 0, graph_launches = 0;
};

namespace em2g {

// push_fast_f32.cu
int ens_push(em2g_ens *e, int bp, int cp, bool inplace);
int ens_upload_pair(em2g_ens *e, int r, int s, double *staging);
int ens_download_pair(em2g_ens *e, int r, int s, double *staging);
int ens_push_kernels_per_step(const em2g_ens *e, bool inplace);
// fields_ens.cu
int ens_cg_setup(em2g_ens *e);
int ens_prescale(em2g_ens *e);
int ens_tick(em2g_ens *e);
int ens_fields(em2g_ens *e);
int ens_fields_kernels(const em2g_ens *e);
// ens_step.cu: the table of step kind `key` written to the device (before
// the launch or its capture), and the step as one cooperative launch
int ens_fused_prepare(em2g_ens *e, int key, bool inplace);
int ens_fused_launch(em2g_ens *e, int key, bool inplace);
int ens_fused_phase_ns(em2g_ens *e, int64_t *out, int n);

}  // namespace em2g

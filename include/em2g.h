/*
 * em2g.h -- C ABI of libem2g.so, a B200 (sm_100a) implementation of the
 * time step of em2, the 2D3V relativistic electromagnetic PIC code of
 * fanyumeng666/maccpic (pic/).
 *
 * em2's step is four parameterless Fortran subroutines that act on the
 * module `global` (pic/global.f90:31-45), called from the main loop
 * (pic/main.f90:154-169):
 *     call move; call curnt; [output]; it = it + 1; call fields
 * plus `smooth2(sm)` (pic/smooth.f90:95) which fields calls.  This library
 * keeps the state that `global` holds -- E, B, rho, the six current arrays
 * and the particles -- resident on one GPU and exposes one entry point per
 * subroutine, plus host/device copies of that state, so that a thin
 * iso_c_binding shim can stand in for move.o, curnt.o, fields.o and
 * smooth.o (pic/Makefile:7) without touching main.f90 or output.f90.
 *
 * Conventions
 *  - Every function returns an int status: EM2G_OK (0) or an EM2G_ERR_*
 *    code; em2g_last_error() then gives a message (per host thread).
 *  - Field arrays are the reference's (0:nx+2, 0:ny+2) REAL(8) arrays,
 *    x fastest: element (ix,iy) at iy*(nx+3)+ix, (nx+3)*(ny+3) doubles.
 *  - Particle arrays of species isp (0-based) are the reference's
 *    x(:,isp), y, vx, vy, vz, gamma: x, y in cells in [0,nx) x [0,ny)
 *    (values up to n+0.5, which em2's own loader produces and its guard
 *    cells absorb, are accepted), v in units of c, gamma stored.
 *  - One context per GPU stream; calls on one context must come from one
 *    host thread at a time.  Different contexts are independent.
 *  - The library owns its device memory; host pointers are only read or
 *    written during the call.  Device-pointer variants take pointers in the
 *    context's device memory space and enqueue on the context's stream.
 */
#ifndef EM2G_H
#define EM2G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EM2G_ABI_VERSION 1
#define EM2G_MAX_SPECIES 4

enum em2g_status {
  EM2G_OK = 0,
  EM2G_ERR_INVALID = 1,     /* bad argument or parameter */
  EM2G_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  EM2G_ERR_NOMEM = 3,       /* device allocation failed */
  EM2G_ERR_RANGE = 4,       /* particle outside the grid, count > capacity; from a
                               step: a regrouping push found no place for a particle
                               (the particle state is then inconsistent) */
  EM2G_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  EM2G_ERR_NONFINITE = 6    /* NaN/Inf found in host-provided input */
};

enum em2g_precision {
  EM2G_FP64 = 0,  /* the drop-in path: em2's arithmetic in FP64 */
  EM2G_FP32 = 1   /* mixed: FP32 push/deposit/Yee, FP64 reductions */
};

/* field ids, in the order of the reference's arrays (pic/global.f90:41-43) */
enum em2g_field {
  EM2G_EX = 0, EM2G_EY, EM2G_EZ, EM2G_BX, EM2G_BY, EM2G_BZ, EM2G_RHO,
  EM2G_JXM, EM2G_JXP, EM2G_JYM, EM2G_JYP, EM2G_JZM, EM2G_JZP, EM2G_NFIELD
};

/* Run constants.  They replace the compile-time parameters of
 * pic/input.f90:9-43 and the derived constants of pic/global.f90:18-28;
 * per-species values are those of com_den (pic/input.f90:61-69) and init
 * (pic/init.f90:116-119).  Fill with em2g_params_init() first. */
typedef struct em2g_params {
  uint32_t struct_size;  /* = sizeof(em2g_params) */
  int32_t nx, ny;        /* cells (>= 4 each) */
  int32_t nsp;           /* species, 1..EM2G_MAX_SPECIES */
  int32_t isav;          /* E/B filtering and energy interval (fields) */
  int32_t precision;     /* enum em2g_precision */
  double dx, dy, dt, c;
  double qm[EM2G_MAX_SPECIES];  /* charge/mass */
  double q[EM2G_MAX_SPECIES];   /* macro-particle charge */
  double dn[EM2G_MAX_SPECIES];  /* relative density */
  double am[EM2G_MAX_SPECIES];  /* macro-particle mass (kinetic energy) */
  double tx[EM2G_MAX_SPECIES];  /* background rotation terms of move (0 in em2) */
  double ty[EM2G_MAX_SPECIES];
  int64_t np_max[EM2G_MAX_SPECIES]; /* particle capacity per species */
  int32_t cg_maxits;     /* 10000 in cgm (pic/fields.f90:518) */
  int32_t energy_mode;   /* 0: whole grid; 1: rows 88..168 x ny/80 as em2 */
  double cg_eps;         /* 1e-9 in cgm (pic/fields.f90:519) */
  double qme, wpe;       /* -1, 1 (pic/input.f90:43) */
  int32_t device;        /* CUDA device ordinal */
  int32_t sort_interval; /* FP32 fast path: regroup particles by cell on every
                            k-th push and update them in place in between
                            (0 or 1: every push; k * c * dt < dx, dy) */
  int32_t smooth_current; /* 1: smooth2 each current array after the fold, every
                             step (not in em2, which filters only rho and, every
                             isav steps, E and B); 0 = em2 */
  int32_t poisson;       /* 0: em2's CG (cgm, stops at mean r^2 < cg_eps);
                            1: exact solve by FFT (FP64; nx, ny powers of two
                            <= 8192), a smooth map for the adjoint */
  int32_t staging_mib;   /* device staging for host particle copies and the
                            regrouping, in MiB; 0: 80 bytes x min(largest
                            np_max, 2^24) (particles move through it in slices) */
  int32_t reserved[13];
} em2g_params;

typedef struct em2g_ctx em2g_ctx;

/* version of this header the library was built from */
int em2g_abi_version(void);
/* message for the last failing call on this host thread ("" if none) */
const char *em2g_last_error(void);
/* defaults: em2's constants (c=1, qme=-1, wpe=1, cg 10000 / 1e-9, isav 20) */
int em2g_params_init(em2g_params *p);

int em2g_create(const em2g_params *p, em2g_ctx **out);
int em2g_destroy(em2g_ctx *ctx);
/* enqueue all further work of ctx on this cudaStream_t (NULL = ctx's own) */
int em2g_set_stream(em2g_ctx *ctx, void *cuda_stream);
int em2g_synchronize(em2g_ctx *ctx);

/* ---- state copies (host memory) ------------------------------------ */
/* one field array, (nx+3)*(ny+3) doubles, Fortran layout */
int em2g_set_field(em2g_ctx *ctx, int field_id, const double *host);
int em2g_get_field(em2g_ctx *ctx, int field_id, double *host);
/* all 13 arrays back to back in enum em2g_field order */
int em2g_set_fields(em2g_ctx *ctx, const double *host13);
int em2g_get_fields(em2g_ctx *ctx, double *host13);
/* n particles of species isp (0-based), in slot order j = 0..n-1.  Input
 * is checked on the device (finite values, 0 <= x < nx+0.5, 0 <= y <
 * ny+0.5) before it replaces anything.  Host copies are staged through one
 * device buffer kept until em2g_destroy, as large as the field arrays
 * copied and, for particles, params.staging_mib (by default at most
 * 80 bytes x 2^24): particles go through it in slices, so it does not grow
 * with their count. */
int em2g_set_particles(em2g_ctx *ctx, int isp, int64_t n, const double *x,
                       const double *y, const double *vx, const double *vy,
                       const double *vz, const double *gamma);
/* the same from arrays in device memory (validated on the device) */
int em2g_set_particles_device(em2g_ctx *ctx, int isp, int64_t n, const double *x,
                              const double *y, const double *vx, const double *vy,
                              const double *vz, const double *gamma);
/* returns them in the slot order they were given in, whatever the library
 * did to its internal order; *n receives the count.  With all six array
 * pointers NULL it only reports the count. */
int em2g_get_particles(em2g_ctx *ctx, int isp, int64_t *n, double *x, double *y,
                       double *vx, double *vy, double *vz, double *gamma);
/* The same in slices, for particle sets too large to hold twice on the
 * host or the device (the caller produces and hands over one slice at a
 * time): em2g_particles_begin announces n particles of species isp;
 * em2g_particles_add copies slots first..first+count-1 -- slices in slot
 * order, first = the number added so far -- from host memory (on_device 0)
 * or device memory (1), checking them on the device; em2g_particles_end,
 * once all n are in, makes them the species' particles, or returns
 * EM2G_ERR_RANGE / EM2G_ERR_NONFINITE and keeps the old ones if any slot
 * failed a check.  em2g_set_particles is one begin / add / end. */
int em2g_particles_begin(em2g_ctx *ctx, int isp, int64_t n);
int em2g_particles_add(em2g_ctx *ctx, int isp, int64_t first, int64_t count, const double *x,
                       const double *y, const double *vx, const double *vy, const double *vz,
                       const double *gamma, int on_device);
int em2g_particles_end(em2g_ctx *ctx, int isp);
/* slots first..first+count-1 of species isp into host (on_device 0) or
 * device (1) arrays, in slot order (em2g_get_particles is all slots) */
int em2g_get_particles_range(em2g_ctx *ctx, int isp, int64_t first, int64_t count, double *x,
                             double *y, double *vx, double *vy, double *vz, double *gamma,
                             int on_device);
/* the step counter `it` of pic/global.f90:31 (fields reads it) */
int em2g_set_step(em2g_ctx *ctx, int it);
int em2g_get_step(em2g_ctx *ctx, int *it);

/* ---- state copies (device memory, on the context's stream) --------- */
int em2g_set_fields_device(em2g_ctx *ctx, const double *dev13);
int em2g_get_fields_device(em2g_ctx *ctx, double *dev13);
/* device pointer of one field array owned by the library (FP64 path) */
int em2g_field_device_ptr(em2g_ctx *ctx, int field_id, void **dptr);

/* ---- the subroutines ------------------------------------------------ */
/* move (pic/move.f90:2-217): gather + relativistic Boris for every species.
 * ake_out (nsp doubles, may be NULL) receives ake(isp) = am*dn*sum(gamma-1)
 * as after the MPI_ALLREDUCE of pic/move.f90:214 (one rank: identity). */
int em2g_move(em2g_ctx *ctx, double *ake_out);
/* curnt (pic/curnt.f90:2-379): deposit jm, move and wrap x, y, deposit rho
 * and jp, accumulating into the resident rho/J arrays (not folded). */
int em2g_curnt(em2g_ctx *ctx);
/* fields (pic/fields.f90:2-367) for step `it`: fold, Yee B/2-E-B/2,
 * smooth2(rho), smooth2(E,B) if it%isav==0, Poisson/cgm, energies if
 * it%isav==0 (into energies_out[6] = exe,eye,eze,bxe,bye,bze; may be NULL),
 * zero rho/J.  cg_iters_out (may be NULL) receives cgm's exit count n
 * (cg_maxits+1 when MAXITS was exceeded; em2 carries on then, so does this). */
int em2g_fields(em2g_ctx *ctx, int it, double *energies_out, int *cg_iters_out);
/* smooth2 (pic/smooth.f90:95-179) in place on one resident field array */
int em2g_smooth2(em2g_ctx *ctx, int field_id);
/* move followed by curnt in one fused particle kernel per species, on the
 * cell-sorted fast path: the particles, rho and jm+jp are those of
 * em2g_move then em2g_curnt, but the current is kept as the sum jm+jp in
 * the jxm/jym/jzm arrays with jxp/jyp/jzp zero (fields reads only the sum,
 * pic/fields.f90:211-214).  A shim can map em2's `call move` to nothing and
 * `call curnt` to this (nothing reads v between them, pic/main.f90:154-155). */
int em2g_move_curnt(em2g_ctx *ctx, double *ake_out);

/* ---- fused fast path -------------------------------------------------
 * nsteps iterations of { move; curnt; it = it + 1; fields(it) } with the
 * particle work of move and curnt in one fused kernel per species
 * (as em2g_move_curnt; particles are kept grouped by cell internally).  The
 * outputs refer to the last iteration (energies_out written only when the
 * last `it` is a multiple of isav). */
int em2g_step(em2g_ctx *ctx, int nsteps, double *ake_out, double *energies_out,
              int *cg_iters_out);

/* ---- smooth2 without device allocation -------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (their device memory is managed by someone else, or they are inside a
 * stream capture) and so cannot create a context: filters the caller's
 * (nx+3)*(ny+3) device array in place, as smooth2 does, on cuda_stream.
 * The scratch smooth2 needs is a static device array of
 * EM2G_SMOOTH2_STATIC_MAX_POINTS doubles (4 MiB, held by every GPU that loads
 * the library); larger grids are rejected with EM2G_ERR_RANGE.  The first
 * call on a device looks up that array's device address (make it before any
 * stream capture); calls outside a capture look it up again, calls during
 * one use the address kept from the last.  Calls share the scratch: calls
 * that overlap on the GPU race, so order them.  An error left pending by
 * earlier CUDA work is reported (EM2G_ERR_CUDA) and left pending, not
 * cleared.  No memory is allocated or freed. */
#define EM2G_SMOOTH2_STATIC_MAX_POINTS (1 << 19)
int em2g_smooth2_static(int nx, int ny, double *dev_array, void *cuda_stream);

/* ---- em2's start-up velocity push (pic/setv.f90:36-128) -------------
 * For loaders that draw v at t = 0: one Boris push of -dt/2 with the given
 * E and B gathered with linear weights, as em2's fresh run does before its
 * first step, applied in place to n particles of species isp in device
 * memory (x, y, vx, vy, vz, gamma: 6 arrays of n doubles; v in, v and gamma
 * at t = -dt/2 out; gamma is recomputed from v first).  dev_fields is the
 * FP64 field block in em2's layout (13 arrays of (nx+3)*(ny+3), the order
 * of em2g_field); p supplies nx, ny, dt, c and the species' qm, tx, ty.
 * Each particle's result is bitwise em2's arithmetic.  Every particle must
 * lie in [0,nx) x [0,ny) with |v| < 1, else nothing is changed
 * (EM2G_ERR_RANGE).  No context is needed; the call waits for its check. */
int em2g_setv_device(const em2g_params *p, int isp, const double *dev_fields, double *dev_parts,
                     int64_t n, void *cuda_stream);

/* ---- diagnostics (no counterpart subroutine; FP64 on the GPU) --------
 * out[0..6)  0.5 * mean over the interior of ex^2, ey^2, ez^2, bx^2, by^2,
 *            bz^2 of the current fields (em2's exe..bze over the whole grid,
 *            pic/fields.f90:267-347)
 * out[6..8)  reconnected flux max(psi) - min(psi) along the centre row of
 *            the sheet at ny/4 and at 3ny/4, psi = -integral of By dx
 * out[8..10) mean r^2 of the last Poisson solve before and after the CG
 *            (the charge-conservation residual (div E - rho)^2 dx^4, and the
 *            level cgm stopped at, pic/fields.f90:616)
 * nout values are written (at most EM2G_NDIAG). */
#define EM2G_NDIAG 10
int em2g_diagnostics(em2g_ctx *ctx, double *out, int nout);

/* ---- kernel variants (no counterpart in the reference) ---------------
 * The fast push comes in a few compiled variants -- cells per CTA (tile
 * width) times the CTAs per SM the register allocation allows.  All give the
 * same results; their speed depends on grid, density and GPU.
 * maccpic_b200/autotune.py times them on the live state and keeps the best. */
int em2g_num_variants(em2g_ctx *ctx, int *n);
int em2g_set_variant(em2g_ctx *ctx, int variant);
/* current variant and its name (name may be NULL) */
int em2g_get_variant(em2g_ctx *ctx, int *variant, char *name, int name_len);
/* em2g_params.sort_interval, changed between steps (same rules) */
int em2g_set_sort_interval(em2g_ctx *ctx, int sort_interval);
/* How the Yee updates and the smooth2 passes inside em2g_fields and
 * em2g_smooth2 read their arrays (pic/fields.f90:184-247,
 * pic/smooth.f90:143-177; no reference counterpart for the choice):
 * 0 = direct loads per cell, 1 = tiles staged in shared memory by tensor
 * copies (TMA) in a persistent kernel per stage.  Both round every cell as
 * em2 does (FP64: bitwise the same); only their speed differs. */
int em2g_set_stencils(em2g_ctx *ctx, int mode);
int em2g_get_stencils(em2g_ctx *ctx, int *mode);
/* Self-test of the device waits' bounds (no reference counterpart: em2 has
 * no device waits).  Every wait of a device thread on other threads is
 * bounded: a wait that runs out records a status that the next call returns
 * as EM2G_ERR_TIMEOUT, and the context stays usable.  This runs one wait of
 * each kind that nothing ever releases: the CG's grid barrier (about 2 s)
 * and a TMA-staged tile's mbarrier (about 1 s).  It returns the status each
 * recorded: *cg_status = 1 and *tma_status = 2 when both bounds work.  No
 * fault or trap is involved, and the context's state is left as it was. */
int em2g_selftest_waits(em2g_ctx *ctx, int *cg_status, int *tma_status);

/* ---- instrumentation ------------------------------------------------- */
/* kernel launches since the last reset; with timing on, the number of
 * particle-push launches timed with CUDA events and their summed time */
int em2g_set_timing(em2g_ctx *ctx, int on);
int em2g_get_counters(em2g_ctx *ctx, int64_t *kernel_launches,
                      int64_t *push_launches_timed, double *push_ms);
int em2g_reset_counters(em2g_ctx *ctx);

/* ---- adjoint (no counterpart in the reference) ------------------------
 * Reverse-mode derivative of the FP64 fast step (em2g_step) of a context
 * with the exact Poisson solve (params.poisson = 1), for periodic states
 * (guard cells equal to their periodic images, as em2g_step keeps them).
 * The state it differentiates is the fields E, B and, per particle, the
 * position (x, y) and u = gamma v (the quantity em2's Boris push advances,
 * pic/move.f90:176-203).
 *
 * em2g_adj_forward advances the context nsteps, keeping a checkpoint of
 * the whole state (fields and particles) every `checkpoint` steps.  After
 * seeding the adjoint of the final state, em2g_adj_backward sweeps back to
 * the state em2g_adj_forward started from, one segment of `checkpoint`
 * steps at a time, last first: it restores the segment's checkpoint,
 * recomputes the segment keeping E and B before each of its steps, then
 * goes back through them -- one kernel per step rebuilds the previous
 * particle state by inverting the push (move, then the Boris rotation) and
 * applies the transposed step: gathers of the current and charge adjoints
 * at the particles, the Boris rotation reversed, scatters of the force
 * adjoint onto E and B; the checkpoint resets the rebuilt state at the
 * segment's start.  Device memory: max_steps/checkpoint checkpoints of
 * (13 (nx+3)(ny+3) + 6 x particles) doubles, plus `checkpoint` slots of
 * 6 nx ny doubles.  At its end the context is back at the final state.
 * em2g_adj_field_slots(adj, n), checkpoint <= n <= max_steps, sets the
 * number of slots: the forward sweep fills them with E and B of its last
 * n steps, which the reverse sweep uses as they are, and only the steps
 * before them are recomputed (in the slots already gone through); with n
 * >= the steps run nothing is.  em2g_adj_keep_all_fields(adj, 1) is n =
 * max_steps, 0 is n = checkpoint (the default).  Call either before
 * em2g_adj_forward.  Field adjoints use the periodic (ny, nx) layout
 * (element [j][i] <-> em2 index (i+1, j+1)); particle adjoints are in slot
 * order. */
typedef struct em2g_adj em2g_adj;
int em2g_adj_create(em2g_ctx *ctx, int max_steps, int checkpoint, em2g_adj **out);
int em2g_adj_destroy(em2g_adj *adj);
int em2g_adj_forward(em2g_adj *adj, int nsteps);
int em2g_adj_keep_all_fields(em2g_adj *adj, int on);
int em2g_adj_field_slots(em2g_adj *adj, int nslots);
int em2g_adj_get_field_slots(em2g_adj *adj, int *nslots);
/* adjoint of the final E, B: 6 arrays of ny*nx doubles (ex ey ez bx by bz),
 * device memory; particles' final adjoints are zero */
int em2g_adj_seed_fields_device(em2g_adj *adj, const double *dev6);
int em2g_adj_backward(em2g_adj *adj);
/* adjoints of the initial state (device memory) */
int em2g_adj_get_fields_device(em2g_adj *adj, double *dev6);
int em2g_adj_get_particles_device(em2g_adj *adj, int isp, double *lx, double *ly, double *lux,
                                  double *luy, double *luz);
/* the initial particles as the adjoint sees them: x, y, ux, uy, uz in slot
 * order (device memory) */
int em2g_adj_get_initial_particles_device(em2g_adj *adj, int isp, double *x, double *y,
                                          double *ux, double *uy, double *uz);

/* ---- ensembles (no counterpart in the reference) ----------------------
 * Up to 128 independent runs -- each its own em2 run with its own grid,
 * species constants and particles, as em2g_step would advance it -- that
 * advance together: per step one scan of all runs' cell counts, one
 * persistent push launch whose CTAs claim row segments of all runs from a
 * shared counter, and em2's fields for all runs in one launch per stage
 * (one cooperative launch for all runs' CG, each run stopping at its own
 * tolerance).  The whole step is captured once into a CUDA graph and
 * replayed; nothing in it waits on the host.
 *
 * Every run is FP32 (precision EM2G_FP32) with energy_mode 0, on one device,
 * and all runs share one sort_interval (params.sort_interval, 0 or 1 = 1);
 * at most 160 (run, species) pairs, 2^31 - 1 particles and cells in all.
 * A run holds exactly np_max[s] particles of species s, set (once, or again
 * to replace them) by em2g_ens_set_particles* before the first step.
 * Runs are indexed 0..nruns-1.  Results per run go to arrays of nruns
 * entries: ake_out 4 per run (species 0..3, zero past nsp), energies_out 6
 * per run (written for runs whose isav divides the step count reached),
 * cg_iters_out 1 per run. */
typedef struct em2g_ens em2g_ens;
int em2g_ens_create(const em2g_params *runs, int nruns, em2g_ens **out);
int em2g_ens_destroy(em2g_ens *ens);
int em2g_ens_num_runs(em2g_ens *ens, int *nruns);
int em2g_ens_set_stream(em2g_ens *ens, void *cuda_stream);
/* 1 (default): replay a captured graph per step; 0: launch the kernels */
int em2g_ens_set_graph(em2g_ens *ens, int on);
/* 1: each step is one persistent, cooperative kernel launch whose blocks
 * run every stage above in turn, meeting at bounded grid barriers (a wait
 * that gives up fails the step with EM2G_ERR_TIMEOUT); 0: one launch per
 * stage.  The results are the same up to the order of FP32 sums. */
int em2g_ens_set_fused(em2g_ens *ens, int on);
/* the last fused step's phases: ns[k] = time between consecutive marks
 * (the launch's start, then each grid barrier the step passed), 0 past the
 * last; at most 31 values */
int em2g_ens_get_phase_ns(em2g_ens *ens, int64_t *ns, int n);
/* the FP32 push variants (as em2g_num_variants of an FP32 context) */
int em2g_ens_num_variants(em2g_ens *ens, int *n);
int em2g_ens_set_variant(em2g_ens *ens, int variant);
/* regroup the particles by cell on every k-th step and update them in place
 * in between, as em2g_set_sort_interval does for a context; k * c * dt must
 * be < dx and dy in every run (0 or 1: every step) */
int em2g_ens_set_sort_interval(em2g_ens *ens, int k);
/* one run's 13 arrays, as em2g_set_fields / em2g_get_fields */
int em2g_ens_set_fields(em2g_ens *ens, int run, const double *host13);
int em2g_ens_get_fields(em2g_ens *ens, int run, double *host13);
int em2g_ens_set_particles(em2g_ens *ens, int run, int isp, int64_t n, const double *x,
                           const double *y, const double *vx, const double *vy,
                           const double *vz, const double *gamma);
int em2g_ens_set_particles_device(em2g_ens *ens, int run, int isp, int64_t n,
                                  const double *x, const double *y, const double *vx,
                                  const double *vy, const double *vz, const double *gamma);
int em2g_ens_get_particles(em2g_ens *ens, int run, int isp, int64_t *n, double *x, double *y,
                           double *vx, double *vy, double *vz, double *gamma);
int em2g_ens_step(em2g_ens *ens, int nsteps, double *ake_out, double *energies_out,
                  int *cg_iters_out);
int em2g_ens_get_step(em2g_ens *ens, int *it);
/* em2g_diagnostics of one run */
int em2g_ens_diagnostics(em2g_ens *ens, int run, double *out, int nout);
/* kernels launched (graph replays counted by their kernel nodes), graph
 * launches, and kernels per step */
int em2g_ens_get_counters(em2g_ens *ens, int64_t *kernel_launches, int64_t *graph_launches,
                          int64_t *kernels_per_step);

#ifdef __cplusplus
}
#endif
#endif /* EM2G_H */

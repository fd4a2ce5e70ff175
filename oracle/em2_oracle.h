/*
 * em2_oracle.h -- CPU restatement (FP64, serial) of em2's time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA path: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product (libem2g.so) never links it.
 *
 * It restates, operation for operation and in the same evaluation order,
 * the subroutines of the reference em2 (fanyumeng666/maccpic, pic/):
 *   move     pic/move.f90:35-215
 *   curnt    pic/curnt.f90:35-359
 *   fields   pic/fields.f90:20-366   (fold, Yee, filters, energies, reset)
 *   Poisson  pic/fields.f90:370-444
 *   cgm      pic/fields.f90:508-651
 *   smooth2  pic/smooth.f90:95-179
 * Build with -O2 -ffp-contract=off and without -ffast-math so that every
 * product and sum is rounded exactly as gfortran -O3 rounds it on x86-64
 * (no FMA contraction, left-to-right evaluation).
 *
 * Layout (identical to the reference's module arrays):
 *   field arrays are Fortran (0:nx+2, 0:ny+2), x fastest; element (ix,iy)
 *   sits at iy*(nx+3)+ix.  A field block is 13 such arrays back to back in
 *   the order of enum em2o_field below.
 *   particles of one species are 6 arrays of n doubles back to back:
 *   x, y (cells), vx, vy, vz (v/c), gamma.
 */
#ifndef EM2_ORACLE_H
#define EM2_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum em2o_field {
  EM2O_EX = 0, EM2O_EY, EM2O_EZ, EM2O_BX, EM2O_BY, EM2O_BZ, EM2O_RHO,
  EM2O_JXM, EM2O_JXP, EM2O_JYM, EM2O_JYP, EM2O_JZM, EM2O_JZP, EM2O_NFIELD
};

/* energy_mode: 0 = sum over the whole interior 1..nx x 1..ny;
 *              1 = the reference's rows iy = 88..168 scaled by ny/80
 *                  (pic/fields.f90:278-346; needs ny >= 170). */
typedef struct {
  int32_t nx, ny, nsp, isav;
  double dx, dy, dt, c;
  double qm[4], q[4], dn[4], am[4], tx[4], ty[4];
  int32_t cg_maxits;
  int32_t energy_mode;
  double cg_eps;
  double qme, wpe;
  int32_t smooth_current; /* 1: smooth2 each current array after the fold
                             (an option of the GPU library, not of em2) */
} em2o_params;

/* move for one species (pic/move.f90:37-209): gathers E, B with quadratic
 * weights, Boris-pushes v and gamma in place; returns ake(isp) already
 * multiplied by am*dn (pic/move.f90:208), before any allreduce. */
double em2o_move(const em2o_params *p, const double *fld, int isp, int64_t n,
                 double *part);

/* curnt for one species (pic/curnt.f90:37-358): deposits jm at the old
 * position, moves and wraps x, y, deposits rho and jp at the new position. */
void em2o_curnt(const em2o_params *p, double *fld, int isp, int64_t n,
                double *part);

/* guard-cell fold of rho and the six current arrays (pic/fields.f90:44-137) */
void em2o_fold(const em2o_params *p, double *fld);

/* the three Yee sweeps B/2, E, B/2 with guard copies (pic/fields.f90:184-247) */
void em2o_yee(const em2o_params *p, double *fld);

/* smooth2 on one (0:nx2,0:ny2) array in place (pic/smooth.f90:95-179) */
void em2o_smooth2(const em2o_params *p, double *a);

/* Poisson correction of ex, ey (pic/fields.f90:370-444 + cgm :508-651).
 * Returns the CG iteration count n at exit (cg_maxits+1 if MAXITS was
 * exceeded, matching the loop variable after a completed DO loop). */
int em2o_poisson(const em2o_params *p, double *fld);
/* mean r^2 of the last cgm solve before its first iteration and at exit */
void em2o_last_cg_residuals(double *out);

/* field energies exe,eye,eze,bxe,bye,bze (pic/fields.f90:267-347) */
void em2o_energies(const em2o_params *p, const double *fld, double *e6);

/* the whole of subroutine fields for step `it`: fold, Yee, smooth2(rho),
 * smooth2(E,B) when it%isav==0, Poisson, energies when it%isav==0 (written
 * to e6, else e6 untouched), zero rho and J.  Returns CG iterations. */
int em2o_fields(const em2o_params *p, double *fld, int it, double *e6);

/* one main-loop iteration (pic/main.f90:148-170 without output):
 * move and curnt for every species, then fields(it+1).  part[isp] points
 * at species isp's 6*n block.  ake receives nsp values; e6 as above. */
int em2o_step(const em2o_params *p, double *fld, int it, const int64_t *n,
              double *const *part, double *ake, double *e6);

/* Timing variant used only as the CPU baseline: the particle phase of
 * move+curnt split over `nthreads` POSIX threads, each with private rho/J
 * arrays summed afterwards, which is what em2's particle decomposition over
 * MPI ranks computes (pic/curnt.f90:363-376).  The field phase stays
 * serial as in every em2 rank. */
int em2o_step_mt(const em2o_params *p, double *fld, int it, const int64_t *n,
                  double *const *part, double *ake, double *e6, int nthreads);

#ifdef __cplusplus
}
#endif
#endif

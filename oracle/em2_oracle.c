/*
 * em2_oracle.c -- CPU restatement of em2's step (TEST INFRASTRUCTURE ONLY;
 * see em2_oracle.h).  Every routine names the reference lines it follows.
 * Expressions keep the reference's evaluation order; compile with
 * -ffp-contract=off.
 */
#include "em2_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define NXG(p) ((int64_t)(p)->nx + 3)
#define NYG(p) ((int64_t)(p)->ny + 3)
#define W(p) (NXG(p) * NYG(p))
#define AT(a, ix, iy) (a)[(int64_t)(iy) * nxg + (ix)]

static inline double sq(double t) { return t * t; }

/* ---------------------------------------------------------------------
 * move: pic/move.f90:37-209 (one species)
 * ------------------------------------------------------------------- */
static double move_range(const em2o_params *p, const double *fld, int isp,
                         int64_t n, double *part, int64_t j0, int64_t j1) {
  const int64_t nxg = NXG(p), w = W(p);
  const double *ex = fld + EM2O_EX * w, *ey = fld + EM2O_EY * w,
               *ez = fld + EM2O_EZ * w, *bx = fld + EM2O_BX * w,
               *by = fld + EM2O_BY * w, *bz = fld + EM2O_BZ * w;
  double *x = part, *y = part + n, *vx = part + 2 * n, *vy = part + 3 * n,
         *vz = part + 4 * n, *gm = part + 5 * n;
  /* pic/move.f90:42 ae=0.5d0*qm(isp)*dt/c */
  const double ae = 0.5 * p->qm[isp] * p->dt / p->c;
  /* pic/move.f90:52-64: scaled copies of E and B */
  double *aex = (double *)malloc(sizeof(double) * 6 * w);
  double *aey = aex + w, *aez = aex + 2 * w, *abx = aex + 3 * w,
         *aby = aex + 4 * w, *abz = aex + 5 * w;
  for (int64_t k = 0; k < w; ++k) {
    aex[k] = ae * ex[k];
    aey[k] = ae * ey[k];
    aez[k] = ae * ez[k];
    abx[k] = ae * bx[k] + p->tx[isp];
    aby[k] = ae * by[k] + p->ty[isp];
    abz[k] = ae * bz[k];
  }
  double ake = 0.0;
  const double c = p->c;
  for (int64_t j = j0; j < j1; ++j) {
    const double xj = x[j], yj = y[j];
    /* Ex, Bx: pic/move.f90:76-100 */
    int ix = (int)(xj + 1.0), iy = (int)(yj + 1.5);
    int ixp = ix + 1, iyp = iy + 1, ixm = ix - 1, iym = iy - 1;
    double s2x = 0.75 - sq(xj + 0.5 - ix);
    double s2xp = 0.5 * sq(1.0 + xj - ix);
    double s2xm = 0.5 * sq(-xj + ix);
    double s2y = 0.75 - sq(yj + 1.0 - iy);
    double s2yp = 0.5 * sq(1.5 + yj - iy);
    double s2ym = 0.5 * sq(-0.5 - yj + iy);
    double qxy = s2x * s2y, qxpy = s2xp * s2y, qxmy = s2xm * s2y;
    double qxyp = s2x * s2yp, qxpyp = s2xp * s2yp, qxmyp = s2xm * s2yp;
    double qxym = s2x * s2ym, qxpym = s2xp * s2ym, qxmym = s2xm * s2ym;
#define GATHER(A)                                                          \
  (AT(A, ix, iy) * qxy + AT(A, ix, iyp) * qxyp + AT(A, ix, iym) * qxym +   \
   AT(A, ixp, iy) * qxpy + AT(A, ixp, iyp) * qxpyp + AT(A, ixp, iym) * qxpym + \
   AT(A, ixm, iy) * qxmy + AT(A, ixm, iyp) * qxmyp + AT(A, ixm, iym) * qxmym)
    double aexpt = GATHER(aex);
    double abxpt = GATHER(abx);
    /* Ez, Bz: pic/move.f90:103-124 */
    iy = (int)(yj + 1.0);
    iyp = iy + 1;
    iym = iy - 1;
    s2y = 0.75 - sq(yj + 0.5 - iy);
    s2yp = 0.5 * sq(1.0 + yj - iy);
    s2ym = 0.5 * sq(-yj + iy);
    qxy = s2x * s2y; qxpy = s2xp * s2y; qxmy = s2xm * s2y;
    qxyp = s2x * s2yp; qxpyp = s2xp * s2yp; qxmyp = s2xm * s2yp;
    qxym = s2x * s2ym; qxpym = s2xp * s2ym; qxmym = s2xm * s2ym;
    double aezpt = GATHER(aez);
    double abzpt = GATHER(abz);
    /* Ey, By: pic/move.f90:127-148 */
    ix = (int)(xj + 1.5);
    ixp = ix + 1;
    ixm = ix - 1;
    s2x = 0.75 - sq(xj + 1.0 - ix);
    s2xp = 0.5 * sq(1.5 + xj - ix);
    s2xm = 0.5 * sq(-0.5 - xj + ix);
    qxy = s2x * s2y; qxpy = s2xp * s2y; qxmy = s2xm * s2y;
    qxyp = s2x * s2yp; qxpyp = s2xp * s2yp; qxmyp = s2xm * s2yp;
    qxym = s2x * s2ym; qxpym = s2xp * s2ym; qxmym = s2xm * s2ym;
    double aeypt = GATHER(aey);
    double abypt = GATHER(aby);
#undef GATHER
    /* Boris: pic/move.f90:176-203 */
    double gvxs = vx[j] * gm[j] + aexpt;
    double gvys = vy[j] * gm[j] + aeypt;
    double gvzs = vz[j] * gm[j] + aezpt;
    double g = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
    ake = ake + g - 1.0;
    double dcg = 1.0 / (c * g);
    abxpt = dcg * abxpt;
    abypt = dcg * abypt;
    abzpt = dcg * abzpt;
    double vvx = gvxs + gvys * abzpt - gvzs * abypt;
    double vvy = gvys + gvzs * abxpt - gvxs * abzpt;
    double vvz = gvzs + gvxs * abypt - gvys * abxpt;
    double f = 2.0 / (1.0 + abxpt * abxpt + abypt * abypt + abzpt * abzpt);
    abxpt = f * abxpt;
    abypt = f * abypt;
    abzpt = f * abzpt;
    gvxs = gvxs + vvy * abzpt - vvz * abypt + aexpt;
    gvys = gvys + vvz * abxpt - vvx * abzpt + aeypt;
    gvzs = gvzs + vvx * abypt - vvy * abxpt + aezpt;
    g = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
    gm[j] = g;
    vx[j] = gvxs / g;
    vy[j] = gvys / g;
    vz[j] = gvzs / g;
  }
  free(aex);
  /* pic/move.f90:208 */
  return ake * p->am[isp] * p->dn[isp];
}

double em2o_move(const em2o_params *p, const double *fld, int isp, int64_t n,
                 double *part) {
  return move_range(p, fld, isp, n, part, 0, n);
}

/* ---------------------------------------------------------------------
 * curnt: pic/curnt.f90:37-358 (one species)
 * ------------------------------------------------------------------- */
static void curnt_range(const em2o_params *p, double *fld, int isp,
                        int64_t n, double *part, int64_t j0, int64_t j1) {
  const int64_t nxg = NXG(p), w = W(p);
  double *rho = fld + EM2O_RHO * w, *jxm = fld + EM2O_JXM * w,
         *jxp = fld + EM2O_JXP * w, *jym = fld + EM2O_JYM * w,
         *jyp = fld + EM2O_JYP * w, *jzm = fld + EM2O_JZM * w,
         *jzp = fld + EM2O_JZP * w;
  double *x = part, *y = part + n, *vx = part + 2 * n, *vy = part + 3 * n,
         *vz = part + 4 * n;
  /* pic/curnt.f90:41-42 */
  const double qdxdn = p->q[isp] * p->dn[isp] / (p->dx * p->dy);
  const double qdtdn = qdxdn;
  const double dt = p->dt, dx = p->dx, dy = p->dy;
  const double xn = (double)p->nx, yn = (double)p->ny;
  for (int64_t j = j0; j < j1; ++j) {
    double xj = x[j], yj = y[j];
    const double vxj = vx[j], vyj = vy[j], vzj = vz[j];
    /* jm, Jx staggering: pic/curnt.f90:53-80 */
    int ix = (int)(xj + 1.0), iy = (int)(yj + 1.5);
    int ixp = ix + 1, iyp = iy + 1, ixm = ix - 1, iym = iy - 1;
    double s2x = 0.75 - sq(xj + 0.5 - ix);
    double s2xp = 0.5 * sq(1.0 + xj - ix);
    double s2xm = 0.5 * sq(-xj + ix);
    double s2y = 0.75 - sq(yj + 1.0 - iy);
    double s2yp = 0.5 * sq(1.5 + yj - iy);
    double s2ym = 0.5 * sq(-0.5 - yj + iy);
    double qxy, qxpy, qxmy, qxyp, qxpyp, qxmyp, qxym, qxpym, qxmym;
#define WEIGHTS(Q)                                                        \
  qxy = s2x * s2y * Q; qxpy = s2xp * s2y * Q; qxmy = s2xm * s2y * Q;      \
  qxyp = s2x * s2yp * Q; qxpyp = s2xp * s2yp * Q; qxmyp = s2xm * s2yp * Q; \
  qxym = s2x * s2ym * Q; qxpym = s2xp * s2ym * Q; qxmym = s2xm * s2ym * Q;
#define SCATTER(A, V)                                                     \
  AT(A, ix, iy) += qxy * V; AT(A, ixp, iy) += qxpy * V;                   \
  AT(A, ixm, iy) += qxmy * V; AT(A, ix, iyp) += qxyp * V;                 \
  AT(A, ixp, iyp) += qxpyp * V; AT(A, ixm, iyp) += qxmyp * V;             \
  AT(A, ix, iym) += qxym * V; AT(A, ixp, iym) += qxpym * V;               \
  AT(A, ixm, iym) += qxmym * V;
    WEIGHTS(qdtdn)
    SCATTER(jxm, vxj)
    /* jm, Jz staggering: pic/curnt.f90:82-106 */
    iy = (int)(yj + 1.0);
    iyp = iy + 1;
    iym = iy - 1;
    s2y = 0.75 - sq(yj + 0.5 - iy);
    s2yp = 0.5 * sq(1.0 + yj - iy);
    s2ym = 0.5 * sq(-yj + iy);
    WEIGHTS(qdtdn)
    SCATTER(jzm, vzj)
    /* jm, Jy staggering: pic/curnt.f90:108-132 */
    ix = (int)(xj + 1.5);
    ixp = ix + 1;
    ixm = ix - 1;
    s2x = 0.75 - sq(xj + 1.0 - ix);
    s2xp = 0.5 * sq(1.5 + xj - ix);
    s2xm = 0.5 * sq(-0.5 - xj + ix);
    WEIGHTS(qdtdn)
    SCATTER(jym, vyj)
    /* move and wrap: pic/curnt.f90:181-194 */
    xj = xj + vxj * dt / dx;
    yj = yj + vyj * dt / dy;
    if (xj < 0.0) xj = xj + xn;
    if (xj >= xn) xj = xj - xn;
    if (yj < 0.0) yj = yj + yn;
    if (yj >= yn) yj = yj - yn;
    x[j] = xj;
    y[j] = yj;
    /* rho at the new position: pic/curnt.f90:197-225 */
    ix = (int)(xj + 1.5);
    iy = (int)(yj + 1.5);
    ixp = ix + 1; iyp = iy + 1; ixm = ix - 1; iym = iy - 1;
    s2x = 0.75 - sq(xj + 1.0 - ix);
    s2xp = 0.5 * sq(1.5 + xj - ix);
    s2xm = 0.5 * sq(-0.5 - xj + ix);
    s2y = 0.75 - sq(yj + 1.0 - iy);
    s2yp = 0.5 * sq(1.5 + yj - iy);
    s2ym = 0.5 * sq(-0.5 - yj + iy);
    WEIGHTS(qdxdn)
    AT(rho, ix, iy) += qxy; AT(rho, ixp, iy) += qxpy;
    AT(rho, ixm, iy) += qxmy; AT(rho, ix, iyp) += qxyp;
    AT(rho, ixp, iyp) += qxpyp; AT(rho, ixm, iyp) += qxmyp;
    AT(rho, ix, iym) += qxym; AT(rho, ixp, iym) += qxpym;
    AT(rho, ixm, iym) += qxmym;
    /* jp, Jx staggering: pic/curnt.f90:227-251 */
    ix = (int)(xj + 1.0);
    ixp = ix + 1;
    ixm = ix - 1;
    s2x = 0.75 - sq(xj + 0.5 - ix);
    s2xp = 0.5 * sq(1.0 + xj - ix);
    s2xm = 0.5 * sq(-xj + ix);
    WEIGHTS(qdtdn)
    SCATTER(jxp, vxj)
    /* jp, Jz staggering: pic/curnt.f90:253-277 */
    iy = (int)(yj + 1.0);
    iyp = iy + 1;
    iym = iy - 1;
    s2y = 0.75 - sq(yj + 0.5 - iy);
    s2yp = 0.5 * sq(1.0 + yj - iy);
    s2ym = 0.5 * sq(-yj + iy);
    WEIGHTS(qdtdn)
    SCATTER(jzp, vzj)
    /* jp, Jy staggering: pic/curnt.f90:279-303 */
    ix = (int)(xj + 1.5);
    ixp = ix + 1;
    ixm = ix - 1;
    s2x = 0.75 - sq(xj + 1.0 - ix);
    s2xp = 0.5 * sq(1.5 + xj - ix);
    s2xm = 0.5 * sq(-0.5 - xj + ix);
    WEIGHTS(qdtdn)
    SCATTER(jyp, vyj)
#undef WEIGHTS
#undef SCATTER
  }
}

void em2o_curnt(const em2o_params *p, double *fld, int isp, int64_t n,
                double *part) {
  curnt_range(p, fld, isp, n, part, 0, n);
}

/* ---------------------------------------------------------------------
 * fields pieces
 * ------------------------------------------------------------------- */
void em2o_fold(const em2o_params *p, double *fld) {
  /* pic/fields.f90:44-137: x first over all rows, then y over all columns */
  const int64_t nxg = NXG(p), w = W(p);
  const int nx = p->nx, ny = p->ny, nx1 = nx + 1, nx2 = nx + 2, ny1 = ny + 1,
            ny2 = ny + 2;
  for (int iy = 0; iy <= ny2; ++iy) {
    for (int k = EM2O_RHO; k <= EM2O_JZP; ++k) {
      double *a = fld + k * w;
      AT(a, 1, iy) = AT(a, 1, iy) + AT(a, nx1, iy);
      AT(a, 2, iy) = AT(a, 2, iy) + AT(a, nx2, iy);
      AT(a, nx, iy) = AT(a, nx, iy) + AT(a, 0, iy);
      AT(a, nx1, iy) = AT(a, 1, iy);
      AT(a, nx2, iy) = AT(a, 2, iy);
      AT(a, 0, iy) = AT(a, nx, iy);
    }
  }
  for (int ix = 0; ix <= nx2; ++ix) {
    for (int k = EM2O_RHO; k <= EM2O_JZP; ++k) {
      double *a = fld + k * w;
      AT(a, ix, 1) = AT(a, ix, 1) + AT(a, ix, ny1);
      AT(a, ix, 2) = AT(a, ix, 2) + AT(a, ix, ny2);
      AT(a, ix, ny) = AT(a, ix, ny) + AT(a, ix, 0);
      AT(a, ix, ny1) = AT(a, ix, 1);
      AT(a, ix, ny2) = AT(a, ix, 2);
      AT(a, ix, 0) = AT(a, ix, ny);
    }
  }
}

/* guard copies that close every Yee/filter sweep: columns 0 and nx+2 of
 * rows 1..ny+1, then rows 0 and ny+2 over columns 0..nx+2
 * (e.g. pic/fields.f90:192-200) */
static void guards(const em2o_params *p, double *a) {
  const int64_t nxg = NXG(p);
  const int nx = p->nx, ny = p->ny, nx2 = nx + 2, ny2 = ny + 2;
  for (int iy = 1; iy <= ny + 1; ++iy) {
    AT(a, 0, iy) = AT(a, nx, iy);
    AT(a, nx2, iy) = AT(a, 2, iy);
  }
  for (int ix = 0; ix <= nx2; ++ix) {
    AT(a, ix, 0) = AT(a, ix, ny);
    AT(a, ix, ny2) = AT(a, ix, 2);
  }
}

static void b_half(const em2o_params *p, double *fld) {
  /* pic/fields.f90:184-200 (and :231-247) */
  const int64_t nxg = NXG(p), w = W(p);
  double *ex = fld + EM2O_EX * w, *ey = fld + EM2O_EY * w,
         *ez = fld + EM2O_EZ * w, *bx = fld + EM2O_BX * w,
         *by = fld + EM2O_BY * w, *bz = fld + EM2O_BZ * w;
  const double ctx = p->dt * p->c / p->dx, cty = p->dt * p->c / p->dy;
  const double ctxh = ctx * 0.5, ctyh = cty * 0.5;
  for (int iy = 1; iy <= p->ny + 1; ++iy) {
    const int iyp = iy + 1, iym = iy - 1;
    for (int ix = 1; ix <= p->nx + 1; ++ix) {
      const int ixp = ix + 1, ixm = ix - 1;
      AT(bx, ix, iy) = AT(bx, ix, iy) - ctyh * (AT(ez, ix, iy) - AT(ez, ix, iym));
      AT(by, ix, iy) = AT(by, ix, iy) + ctxh * (AT(ez, ix, iy) - AT(ez, ixm, iy));
      AT(bz, ix, iy) = AT(bz, ix, iy) - ctxh * (AT(ey, ixp, iy) - AT(ey, ix, iy)) +
                       ctyh * (AT(ex, ix, iyp) - AT(ex, ix, iy));
    }
  }
  guards(p, bx);
  guards(p, by);
  guards(p, bz);
}

void em2o_yee(const em2o_params *p, double *fld) {
  const int64_t nxg = NXG(p), w = W(p);
  b_half(p, fld);
  /* E by dt: pic/fields.f90:207-224 */
  double *ex = fld + EM2O_EX * w, *ey = fld + EM2O_EY * w,
         *ez = fld + EM2O_EZ * w, *bx = fld + EM2O_BX * w,
         *by = fld + EM2O_BY * w, *bz = fld + EM2O_BZ * w;
  const double *jxm = fld + EM2O_JXM * w, *jxp = fld + EM2O_JXP * w,
               *jym = fld + EM2O_JYM * w, *jyp = fld + EM2O_JYP * w,
               *jzm = fld + EM2O_JZM * w, *jzp = fld + EM2O_JZP * w;
  const double ctx = p->dt * p->c / p->dx, cty = p->dt * p->c / p->dy;
  const double tem = 0.5 * p->dt;
  for (int iy = 1; iy <= p->ny + 1; ++iy) {
    const int iyp = iy + 1, iym = iy - 1;
    for (int ix = 1; ix <= p->nx + 1; ++ix) {
      const int ixp = ix + 1, ixm = ix - 1;
      AT(ex, ix, iy) = AT(ex, ix, iy) + cty * (AT(bz, ix, iy) - AT(bz, ix, iym)) -
                       tem * (AT(jxm, ix, iy) + AT(jxp, ix, iy));
      AT(ey, ix, iy) = AT(ey, ix, iy) - ctx * (AT(bz, ix, iy) - AT(bz, ixm, iy)) -
                       tem * (AT(jym, ix, iy) + AT(jyp, ix, iy));
      AT(ez, ix, iy) = AT(ez, ix, iy) + ctx * (AT(by, ixp, iy) - AT(by, ix, iy)) -
                       cty * (AT(bx, ix, iyp) - AT(bx, ix, iy)) -
                       tem * (AT(jzm, ix, iy) + AT(jzp, ix, iy));
    }
  }
  guards(p, ex);
  guards(p, ey);
  guards(p, ez);
  b_half(p, fld);
}

void em2o_smooth2(const em2o_params *p, double *sm) {
  /* pic/smooth.f90:143-177 */
  const int64_t nxg = NXG(p), w = W(p);
  double *dm = (double *)calloc((size_t)w, sizeof(double));
  for (int iy = 1; iy <= p->ny + 1; ++iy)
    for (int ix = 1; ix <= p->nx + 1; ++ix)
      AT(dm, ix, iy) =
          (4 * AT(sm, ix, iy) +
           2 * (AT(sm, ix - 1, iy) + AT(sm, ix + 1, iy) + AT(sm, ix, iy - 1) +
                AT(sm, ix, iy + 1)) +
           AT(sm, ix - 1, iy - 1) + AT(sm, ix - 1, iy + 1) +
           AT(sm, ix + 1, iy - 1) + AT(sm, ix + 1, iy + 1)) /
          16.0;
  guards(p, dm);
  for (int iy = 1; iy <= p->ny + 1; ++iy)
    for (int ix = 1; ix <= p->nx + 1; ++ix)
      AT(sm, ix, iy) =
          (20 * AT(dm, ix, iy) - AT(dm, ix - 1, iy) - AT(dm, ix + 1, iy) -
           AT(dm, ix, iy - 1) - AT(dm, ix, iy + 1) - AT(dm, ix - 1, iy - 1) -
           AT(dm, ix - 1, iy + 1) - AT(dm, ix + 1, iy - 1) -
           AT(dm, ix + 1, iy + 1)) /
          12.0;
  guards(p, sm);
  free(dm);
}

/* cgm on (nx1, ny1) arrays stored 1-based in a (nx+2)*(ny+2) buffer;
 * pic/fields.f90:508-651 */
#define CI(j, l) ((int64_t)(l) * (nx + 2) + (j))
/* mean r^2 of the last cgm before its first iteration and at its exit (the
 * quantities em2g_diagnostics reports; test bookkeeping, not part of em2) */
static double g_last_res[2];
void em2o_last_cg_residuals(double *out) {
  out[0] = g_last_res[0];
  out[1] = g_last_res[1];
}
static int cgm(const em2o_params *p, const double *f, double *u) {
  const int nx = p->nx, ny = p->ny, nx1 = nx + 1, ny1 = ny + 1;
  const size_t sz = (size_t)(nx + 2) * (size_t)(ny + 2);
  double *r = (double *)calloc(sz, sizeof(double));
  double *r1 = (double *)calloc(sz, sizeof(double));
  double *pp = (double *)calloc(sz, sizeof(double));
  double *ap = (double *)calloc(sz, sizeof(double));
  for (int j = 1; j <= nx; ++j) {
    const int jm = (j == 1) ? nx : j - 1;
    for (int l = 1; l <= ny; ++l) {
      const int lm = (l == 1) ? ny : l - 1;
      r[CI(j, l)] = f[CI(j, l)] - u[CI(j + 1, l)] - u[CI(jm, l)] -
                    u[CI(j, l + 1)] - u[CI(j, lm)] + 4.0 * u[CI(j, l)];
    }
    r[CI(j, ny1)] = r[CI(j, 1)];
  }
  for (int l = 1; l <= ny1; ++l) r[CI(nx1, l)] = r[CI(1, l)];
  for (int l = 1; l <= ny1; ++l)
    for (int j = 1; j <= nx1; ++j) pp[CI(j, l)] = r[CI(j, l)];
  int n;
  for (n = 1; n <= p->cg_maxits; ++n) {
    double rr = 0.0;
    for (int j = 1; j <= nx; ++j)
      for (int l = 1; l <= ny; ++l) rr = rr + sq(r[CI(j, l)]);
    if (n == 1) g_last_res[0] = rr / nx / ny;
    for (int j = 1; j <= nx; ++j) {
      const int jm = (j == 1) ? nx : j - 1;
      for (int l = 1; l <= ny; ++l) {
        const int lm = (l == 1) ? ny : l - 1;
        ap[CI(j, l)] = pp[CI(j + 1, l)] + pp[CI(jm, l)] + pp[CI(j, l + 1)] +
                       pp[CI(j, lm)] - 4.0 * pp[CI(j, l)];
      }
    }
    double pap = 0.0;
    for (int j = 1; j <= nx; ++j)
      for (int l = 1; l <= ny; ++l) pap = pap + pp[CI(j, l)] * ap[CI(j, l)];
    const double ak = rr / pap;
    for (int j = 1; j <= nx; ++j) {
      for (int l = 1; l <= ny; ++l) {
        u[CI(j, l)] = u[CI(j, l)] + ak * pp[CI(j, l)];
        r1[CI(j, l)] = r[CI(j, l)] - ak * ap[CI(j, l)];
      }
      u[CI(j, ny1)] = u[CI(j, 1)];
      r1[CI(j, ny1)] = r1[CI(j, 1)];
    }
    for (int l = 1; l <= ny1; ++l) {
      u[CI(nx1, l)] = u[CI(1, l)];
      r1[CI(nx1, l)] = r1[CI(1, l)];
    }
    double r_norm = 0.0;
    for (int j = 1; j <= nx; ++j)
      for (int l = 1; l <= ny; ++l) r_norm = r_norm + sq(r1[CI(j, l)]);
    g_last_res[1] = r_norm / nx / ny;
    if (r_norm / nx / ny < p->cg_eps) break;
    const double bk = r_norm / rr;
    for (int j = 1; j <= nx; ++j) {
      for (int l = 1; l <= ny; ++l)
        pp[CI(j, l)] = r1[CI(j, l)] + bk * pp[CI(j, l)];
      pp[CI(j, ny1)] = pp[CI(j, 1)];
    }
    for (int l = 1; l <= ny1; ++l) pp[CI(nx1, l)] = pp[CI(1, l)];
    memcpy(r, r1, sz * sizeof(double));
  }
  free(r); free(r1); free(pp); free(ap);
  return n;
}

int em2o_poisson(const em2o_params *p, double *fld) {
  /* pic/fields.f90:384-442 */
  const int64_t nxg = NXG(p), w = W(p);
  const int nx = p->nx, ny = p->ny, nx1 = nx + 1, ny1 = ny + 1, nx2 = nx + 2,
            ny2 = ny + 2;
  double *ex = fld + EM2O_EX * w, *ey = fld + EM2O_EY * w;
  const double *rho = fld + EM2O_RHO * w;
  const double dx = p->dx, dy = p->dy;
  const size_t sz = (size_t)(nx + 2) * (size_t)(ny + 2);
  double *f = (double *)calloc(sz, sizeof(double));
  double *ph = (double *)calloc(sz, sizeof(double));
  double *php = (double *)calloc(sz, sizeof(double));
  for (int iy = 1; iy <= ny; ++iy) {
    const int iym = iy - 1;
    for (int ix = 2; ix <= nx; ++ix) {
      const int ixm = ix - 1;
      f[CI(ix, iy)] = (AT(ex, ix, iy) - AT(ex, ixm, iy)) / dx +
                      (AT(ey, ix, iy) - AT(ey, ix, iym)) / dy - AT(rho, ix, iy);
    }
    f[CI(1, iy)] = (AT(ex, 1, iy) - AT(ex, nx, iy)) / dx +
                   (AT(ey, 1, iy) - AT(ey, 1, iym)) / dy - AT(rho, 1, iy);
    f[CI(nx1, iy)] = f[CI(1, iy)];
  }
  for (int j = 1; j <= nx1; ++j) f[CI(j, ny1)] = f[CI(j, 1)];
  for (int l = 1; l <= ny1; ++l)
    for (int j = 1; j <= nx1; ++j) f[CI(j, l)] = f[CI(j, l)] * dx * dx;
  /* ph(:,:) = 0.d-4 (calloc) */
  const int iters = cgm(p, f, ph);
  for (int iy = 1; iy <= ny; ++iy) {
    for (int ix = 1; ix <= nx; ++ix)
      php[CI(ix, iy)] = AT(ex, ix, iy) - (ph[CI(ix + 1, iy)] - ph[CI(ix, iy)]) / dx;
    php[CI(nx1, iy)] = php[CI(1, iy)];
  }
  for (int j = 1; j <= nx1; ++j) php[CI(j, ny1)] = php[CI(j, 1)];
  for (int iy = 1; iy <= ny1; ++iy)
    for (int ix = 1; ix <= nx1; ++ix) AT(ex, ix, iy) = php[CI(ix, iy)];
  for (int iy = 1; iy <= ny1; ++iy) {
    AT(ex, 0, iy) = AT(ex, nx, iy);
    AT(ex, nx2, iy) = AT(ex, 2, iy);
  }
  for (int ix = 0; ix <= nx2; ++ix) {
    AT(ex, ix, 0) = AT(ex, ix, ny);
    AT(ex, ix, ny2) = AT(ex, ix, 2);
  }
  for (int ix = 1; ix <= nx; ++ix) {
    for (int iy = 1; iy <= ny; ++iy)
      php[CI(ix, iy)] = AT(ey, ix, iy) - (ph[CI(ix, iy + 1)] - ph[CI(ix, iy)]) / dy;
    php[CI(ix, ny1)] = php[CI(ix, 1)];
  }
  for (int l = 1; l <= ny1; ++l) php[CI(nx1, l)] = php[CI(1, l)];
  for (int iy = 1; iy <= ny1; ++iy)
    for (int ix = 1; ix <= nx1; ++ix) AT(ey, ix, iy) = php[CI(ix, iy)];
  for (int iy = 1; iy <= ny1; ++iy) {
    AT(ey, 0, iy) = AT(ey, nx, iy);
    AT(ey, nx2, iy) = AT(ey, 2, iy);
  }
  for (int ix = 0; ix <= nx2; ++ix) {
    AT(ey, ix, 0) = AT(ey, ix, ny);
    AT(ey, ix, ny2) = AT(ey, ix, 2);
  }
  free(f); free(ph); free(php);
  return iters;
}
#undef CI

void em2o_energies(const em2o_params *p, const double *fld, double *e6) {
  /* pic/fields.f90:267-347.  rnmec2i = (qme/wpe/c)**2/(alx*aly),
   * anorml1 = 0.5*dx*dy*rnmec2i (pic/global.f90:26-27). */
  const int64_t nxg = NXG(p), w = W(p);
  const double alx = p->dx * p->nx, aly = p->dy * p->ny;
  const double t = p->qme / p->wpe / p->c;
  const double rnmec2i = t * t / (alx * aly);
  const double anorml1 = 0.5 * p->dx * p->dy * rnmec2i;
  int lo = 1, hi = p->ny;
  if (p->energy_mode == 1) { lo = 88; hi = 168; }
  for (int k = 0; k < 6; ++k) {
    const double *a = fld + k * w;
    double s = 0.0;
    for (int ix = 1; ix <= p->nx; ++ix)
      for (int iy = lo; iy <= hi; ++iy) s = s + sq(AT(a, ix, iy));
    if (p->energy_mode == 1)
      e6[k] = s * anorml1 * p->ny / 80.0;
    else
      e6[k] = s * anorml1;
  }
}

int em2o_fields(const em2o_params *p, double *fld, int it, double *e6) {
  /* pic/fields.f90:20-366 (bxm copy and the fort.999 debug write omitted:
   * neither feeds the step) */
  const int64_t w = W(p);
  em2o_fold(p, fld);
  if (p->smooth_current)
    for (int k = EM2O_RHO + 1; k < EM2O_NFIELD; ++k) em2o_smooth2(p, fld + k * w);
  em2o_yee(p, fld);
  em2o_smooth2(p, fld + EM2O_RHO * w);
  if (it % p->isav == 0)
    for (int k = EM2O_EX; k <= EM2O_BZ; ++k) em2o_smooth2(p, fld + k * w);
  const int iters = em2o_poisson(p, fld);
  if (it % p->isav == 0 && e6) em2o_energies(p, fld, e6);
  memset(fld + EM2O_RHO * w, 0, sizeof(double) * 7 * (size_t)w);
  return iters;
}

int em2o_step(const em2o_params *p, double *fld, int it, const int64_t *n,
              double *const *part, double *ake, double *e6) {
  for (int isp = 0; isp < p->nsp; ++isp)
    ake[isp] = em2o_move(p, fld, isp, n[isp], part[isp]);
  for (int isp = 0; isp < p->nsp; ++isp)
    em2o_curnt(p, fld, isp, n[isp], part[isp]);
  return em2o_fields(p, fld, it + 1, e6);
}

typedef struct {
  const em2o_params *p;
  const double *fld;
  const int64_t *n;
  double *const *part;
  double *priv; /* this rank's rho/J (7 arrays) */
  double ake[4];
  int tid, nthreads;
} rank_job;

static void *rank_main(void *arg) {
  rank_job *J = (rank_job *)arg;
  const em2o_params *p = J->p;
  const int64_t w = W(p);
  /* this rank's field block: its copy of E and B, its own rho and J */
  double *tmp = (double *)malloc(sizeof(double) * EM2O_NFIELD * (size_t)w);
  memcpy(tmp, J->fld, sizeof(double) * 6 * (size_t)w);
  memset(tmp + 6 * w, 0, sizeof(double) * 7 * (size_t)w);
  for (int isp = 0; isp < p->nsp; ++isp) {
    const int64_t lo = J->n[isp] * J->tid / J->nthreads;
    const int64_t hi = J->n[isp] * (J->tid + 1) / J->nthreads;
    J->ake[isp] = move_range(p, tmp, isp, J->n[isp], J->part[isp], lo, hi);
    curnt_range(p, tmp, isp, J->n[isp], J->part[isp], lo, hi);
  }
  memcpy(J->priv, tmp + 6 * w, sizeof(double) * 7 * (size_t)w);
  free(tmp);
  return NULL;
}

int em2o_step_mt(const em2o_params *p, double *fld, int it, const int64_t *n,
                 double *const *part, double *ake, double *e6, int nthreads) {
  const int64_t w = W(p);
  if (nthreads < 1) nthreads = 1;
  /* each thread plays one em2 rank: its own slice of every species and its
   * own rho/J arrays; the sum below plays MPI_ALLREDUCE. */
  double *priv = (double *)malloc(sizeof(double) * (size_t)nthreads * 7 * (size_t)w);
  rank_job *jobs = (rank_job *)calloc((size_t)nthreads, sizeof(rank_job));
  pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].p = p; jobs[t].fld = fld; jobs[t].n = n; jobs[t].part = part;
    jobs[t].priv = priv + (size_t)t * 7 * (size_t)w;
    jobs[t].tid = t; jobs[t].nthreads = nthreads;
    pthread_create(&th[t], NULL, rank_main, &jobs[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  for (int isp = 0; isp < p->nsp; ++isp) ake[isp] = 0.0;
  for (int t = 0; t < nthreads; ++t) {
    const double *mine = jobs[t].priv;
    for (int64_t k = 0; k < 7 * w; ++k) fld[6 * w + k] += mine[k];
    for (int isp = 0; isp < p->nsp; ++isp) ake[isp] += jobs[t].ake[isp];
  }
  free(priv);
  free(jobs);
  free(th);
  return em2o_fields(p, fld, it + 1, e6);
}

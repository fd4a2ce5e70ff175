/*
 * em2_loader_oracle.c -- CPU restatement of em2's start-up (TEST
 * INFRASTRUCTURE ONLY).  It exists to pin the step oracle against the only
 * known-answer numbers the reference publishes for this path, the
 * initial-state check of pic/RECONNECTION_MODEL.md:454-460 (density 6.0 /
 * 1.0, sheet-1 mean vz -0.0257 c / +0.1070 c, deposited jz 0.663 against
 * 0.669 from the discrete curl of B), which were produced by em2's own
 * loader.  Restated here, in the reference's evaluation order:
 *   init (fields and species constants)  pic/init.f90:2-130
 *   com_den                               pic/input.f90:61-69
 *   maxnp                                 pic/global.f90:15
 *   creator                               pic/creator.f90:24-243
 *   smear                                 pic/smear.f90:2-47
 *   dran2 (ran2 of Numerical Recipes)     pic/dran2.f90:2-42
 *   setv (-dt/2 push, linear weights)     pic/setv.f90:30-133
 * Single-precision literals of the reference (0.1 in init.f90:251-252,
 * 0.001 in creator.f90:120) are kept as float constants.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "em2_oracle.h"

typedef struct {
  int32_t nx, ny, npcel, nsp, nproc;
  double dx, dy, dt, c, wce0, rmass, csw, csden, rtemp;
  double temp[2], aist[2];
} em2o_load_params;

static const double PI = 3.141592653589793;

/* pic/global.f90:15 */
int64_t em2o_maxnp(const em2o_load_params *L) {
  const double gsum = (double)(L->ny / 2) +
                      2 * L->csw / L->dx * L->csden *
                          tanh(L->ny * L->dy / 2 / L->csw);
  const int32_t rows = (int32_t)gsum;
  const int32_t tot = 2 * L->nx * L->npcel * rows;
  return (int64_t)(tot / L->nproc);
}

/* pic/input.f90:61-69 and pic/init.f90:112-119 (nsp = 2) */
void em2o_com_den(const em2o_load_params *L, double *q, double *qm,
                  double *dn, double *am) {
  const double wpe = 1.0, qme = -1.0, qmi = -qme / L->rmass;
  double rm[2] = {1.0, L->rmass};
  dn[0] = 1.0; dn[1] = 1.0;
  qm[0] = -1.0; qm[1] = 1.0 / rm[1];
  for (int s = 0; s < 2; ++s)
    q[s] = L->dx * L->dy * wpe * wpe / (L->npcel * qm[s]) / rm[s];
  am[0] = q[0] / qme;
  am[1] = q[1] / qmi;
}

/* pic/init.f90:46-92: zero fields, double-Harris Bx plus perturbation */
void em2o_init_fields(const em2o_load_params *L, double *fld) {
  const int nx = L->nx, ny = L->ny, nx2 = nx + 2, ny2 = ny + 2;
  const int64_t nxg = nx + 3, w = (int64_t)(nx + 3) * (ny + 3);
  memset(fld, 0, sizeof(double) * EM2O_NFIELD * (size_t)w);
  double *bx = fld + EM2O_BX * w, *by = fld + EM2O_BY * w;
  const double gcsw = L->csw / L->dx;
  const double aw = fabs(L->wce0);
  const double f01 = (double)0.1f;
  const double dbx = f01 * aw / sqrt(L->csden) * sqrt(L->rmass) * 2 * PI / (nx * L->dx);
  const double dby = f01 * aw / sqrt(L->csden) * sqrt(L->rmass) * 2 * PI / (ny * L->dy);
#define B(a, i, j) (a)[(int64_t)(j) * nxg + (i)]
  for (int ix = 0; ix <= nx2; ++ix) {
    for (int iy = 0; iy <= ny / 2; ++iy) {
      const int ku = iy + ny / 2 - 3 * ny / 4;
      B(bx, ix, iy + ny / 2 + 1) =
          aw * tanh(ku / gcsw) +
          dby * cos(2 * PI * (ix - 0.5 - nx * 0.5) / nx + PI) * sin(2 * PI * ku / ny);
      B(bx, ix, iy) =
          -aw * tanh((iy - 1 - ny / 4) / gcsw) -
          dby * cos(2 * PI * (ix - 0.5 - nx * 0.5) / nx) *
              sin(2 * PI * ((iy - 1) - 0.25 * ny) / ny);
      B(by, ix, iy + ny / 2 + 1) =
          -dbx * sin(2 * PI * ((ix - 1) - nx * 0.5) / nx + PI) *
          cos(2 * PI * ((iy + ny / 2) + 0.5 - 3 * ny / 4) / ny);
      B(by, ix, iy) = dbx * sin(2 * PI * ((ix - 1) - nx * 0.5) / nx) *
                      cos(2 * PI * ((iy - 0.5) - 0.25 * ny) / ny);
    }
    B(bx, ix, ny2) = B(bx, ix, 0);
    B(by, ix, ny2) = B(by, ix, 0);
  }
#undef B
}

/* ran2 with Bays-Durham shuffle, state kept as in the SAVE variables of
 * pic/dran2.f90:16-18 */
typedef struct {
  int32_t idum2, iy, iv[32];
} ran2_state;

static double dran2(ran2_state *S, int32_t *idum) {
  const int32_t IM1 = 2147483563, IM2 = 2147483399, IMM1 = IM1 - 1;
  const int32_t IA1 = 40014, IA2 = 40692, IQ1 = 53668, IQ2 = 52774;
  const int32_t IR1 = 12211, IR2 = 3791, NTAB = 32, NDIV = 1 + IMM1 / NTAB;
  const double AM = 1.0 / IM1, EPS = 1.2e-7, RNMX = 1.0 - EPS;
  int32_t j, k;
  if (*idum <= 0) {
    *idum = (-*idum > 1) ? -*idum : 1;
    S->idum2 = *idum;
    for (j = NTAB + 8; j >= 1; --j) {
      k = *idum / IQ1;
      *idum = IA1 * (*idum - k * IQ1) - k * IR1;
      if (*idum < 0) *idum += IM1;
      if (j <= NTAB) S->iv[j - 1] = *idum;
    }
    S->iy = S->iv[0];
  }
  k = *idum / IQ1;
  *idum = IA1 * (*idum - k * IQ1) - k * IR1;
  if (*idum < 0) *idum += IM1;
  k = S->idum2 / IQ2;
  S->idum2 = IA2 * (S->idum2 - k * IQ2) - k * IR2;
  if (S->idum2 < 0) S->idum2 += IM2;
  j = 1 + S->iy / NDIV;
  S->iy = S->iv[j - 1] - S->idum2;
  S->iv[j - 1] = *idum;
  if (S->iy < 1) S->iy += IMM1;
  const double r = AM * S->iy;
  return r < RNMX ? r : RNMX;
}

/* creator + smear for one rank.  part[s] holds 6*maxnp doubles for species
 * s (x, y, vx, vy, vz, gamma), slot j (1-based within the rank) at j-1.
 * Returns 0, or -1 where the reference stops (creator.f90:72, :89). */
int em2o_creator(const em2o_load_params *L, int myrank, int64_t maxnp,
                 double *const *part) {
  const int64_t np = maxnp;
  const double xn = L->nx, yn = L->ny;
  const double gcsw = L->csw / L->dx;
  const int NPROCS = L->nproc;
#define X(s, i) part[s][(i) - 1]
#define Y(s, i) part[s][np + (i) - 1]
#define VX(s, i) part[s][2 * np + (i) - 1]
#define VY(s, i) part[s][3 * np + (i) - 1]
#define VZ(s, i) part[s][4 * np + (i) - 1]
  for (int s = 0; s < L->nsp; ++s) {
    const int64_t npback = (int64_t)((int32_t)lround(xn * yn) * L->npcel / NPROCS);
    const int64_t nph = np / 2;
    const double temp = L->temp[s], aist = L->aist[s];
    const double pxmax = 5.0 * sqrt(temp * (1.0 + aist));
    const double dpx = 2.0 * pxmax / (double)nph;
    const double pymax = 5.0 * sqrt(temp);
    const double dpy = 2.0 * pymax / (double)nph;
    X(s, 1) = 0.0;
    Y(s, 1) = 0.0;
    for (int64_t i = 1; i <= nph; ++i) {
      const double ppx = (i - 1.5) * dpx - pxmax;
      const double fvx = exp(-(sqrt(1.0 + ppx * ppx) - 1.0) / temp / (1.0 + aist));
      const double ppy = (i - 1.5) * dpy - pymax;
      const double fvy = exp(-(sqrt(1.0 + ppy * ppy) - 1.0) / temp);
      X(s, i + 1) = X(s, i) + (fvx > 0.0 ? fvx : 0.0);
      Y(s, i + 1) = Y(s, i) + (fvy > 0.0 ? fvy : 0.0);
    }
    const double dfx = X(s, nph + 1) / (double)nph;
    const double dfy = Y(s, nph + 1) / (double)nph;
    int64_t iq = 1;
    for (int64_t i = 1; i <= nph; ++i) {
      const double fvx = (i - 0.5) * dfx;
      for (int64_t j = 1; j <= nph; ++j) {
        if (fvx >= X(s, iq + 1)) {
          if (++iq > nph) return -1;
        } else
          break;
      }
      VX(s, i) = dpx * ((double)(iq - 1) + (fvx - X(s, iq)) / (X(s, iq + 1) - X(s, iq))) - pxmax;
    }
    iq = 1;
    for (int64_t i = 1; i <= nph; ++i) {
      const double fvy = (i - 0.5) * dfy;
      for (int64_t j = 1; j <= nph; ++j) {
        if (fvy >= Y(s, iq + 1)) {
          if (++iq > nph) return -1;
        } else
          break;
      }
      const double ppy = dpy * ((double)(iq - 1) + (fvy - Y(s, iq)) / (Y(s, iq + 1) - Y(s, iq))) - pymax;
      VY(s, i) = ppy;
      VZ(s, i) = ppy;
    }
    /* configuration space: pic/creator.f90:110-169 */
    const double ddx = 1.0 / sqrt((double)(L->npcel / 2));
    double ddy = ddx;
    const int32_t nnx = (int32_t)(xn / ddx / NPROCS);
    const double strip = xn / NPROCS, x0 = xn * myrank / NPROCS;
    for (int64_t i = 1; i <= npback / 4; ++i) {
      X(s, i) = fmod((i - 0.5) * ddx, strip) + x0;
      Y(s, i) = ddy * ((double)(i / nnx) + 0.5);
    }
    ddy = 0.25 * yn + ddx * (double)0.001f;
    for (int64_t i = npback / 4 + 1; i <= nph / 4 + npback / 8; ++i) {
      X(s, i) = fmod((i - 0.5) * ddx, strip) + x0;
      Y(s, i) = ddy;
      if ((i - npback / 4) % nnx == 0) {
        const double yr = Y(s, i - nnx + 1);
        const double e = exp((yr - 0.25 * yn) / gcsw) + exp((-yr + 0.25 * yn) / gcsw);
        ddy = yr - ddx / L->csden / 4 * (e * e);
      }
      if (Y(s, i) < 0.0) Y(s, i) = Y(s, i) + yn / 2;
    }
    ddy = 0.25 * yn + ddx / L->csden;
    for (int64_t i = nph / 4 + npback / 8 + 1; i <= nph / 2; ++i) {
      X(s, i) = fmod((i - 0.5) * ddx, strip) + x0;
      Y(s, i) = ddy;
      if ((i - nph / 4 - npback / 8) % nnx == 0) {
        const double yr = Y(s, i - nnx + 1);
        const double e = exp((yr - 0.25 * yn) / gcsw) + exp((-yr + 0.25 * yn) / gcsw);
        ddy = yr + ddx / L->csden / 4 * (e * e);
      }
      if (Y(s, i) > yn / 2) Y(s, i) = Y(s, i) - yn / 2;
    }
    for (int64_t i = nph / 2 + 1; i <= nph; ++i) {
      X(s, i) = X(s, i - nph / 2);
      Y(s, i) = Y(s, i - nph / 2) + yn * 0.5;
    }
  }
  /* smear(10): pic/smear.f90:18-46 */
  ran2_state S;
  memset(&S, 0, sizeof S);
  S.idum2 = 123456789;
  for (int rt = 1; rt <= 10; ++rt) {
    for (int s = 0; s < L->nsp; ++s) {
      int32_t idum = -7146 + myrank;
      const int64_t nph = np / 2;
      for (int64_t i = 1; i <= nph; ++i) {
        int64_t ii = (int64_t)(nph * dran2(&S, &idum) + 1);
        double t = VX(s, i); VX(s, i) = VX(s, ii); VX(s, ii) = t;
        ii = (int64_t)(nph * dran2(&S, &idum) + 1);
        t = VY(s, i); VY(s, i) = VY(s, ii); VY(s, ii) = t;
        ii = (int64_t)(nph * dran2(&S, &idum) + 1);
        t = VZ(s, i); VZ(s, i) = VZ(s, ii); VZ(s, ii) = t;
      }
    }
  }
  /* mirror and drift: pic/creator.f90:181-243 */
  for (int s = 0; s < L->nsp; ++s) {
    const int64_t nph = np / 2;
    const int64_t npback = (int64_t)((int32_t)lround(xn * yn) * L->npcel / NPROCS);
    const int isp = s + 1;
    for (int64_t i = 1; i <= nph; ++i) {
      X(s, i + nph) = X(s, i);
      Y(s, i + nph) = Y(s, i);
      VX(s, i + nph) = -VX(s, i);
      VY(s, i + nph) = -VY(s, i);
      VZ(s, i + nph) = -VZ(s, i);
    }
    double va0 = 0.0;
    const double aw = fabs(L->wce0);
    for (int64_t i = 1; i <= np; ++i) {
      if (i <= npback / 4)
        va0 = 0.0;
      else if (i > nph / 2 && i <= nph / 2 + npback / 4)
        va0 = 0.0;
      else if (i > nph && i <= nph + npback / 4)
        va0 = 0.0;
      else if (i > 3 * nph / 2 && i <= 3 * nph / 2 + npback / 4)
        va0 = 0.0;
      else if (Y(s, i) > yn / 2)
        va0 = ((isp + 1) % 2 == 0 ? 1 : -1) * aw / L->csw / L->csden;
      else if (Y(s, i) < yn / 2)
        va0 = ((isp) % 2 == 0 ? 1 : -1) * aw / L->csw / L->csden;
      const double rp = (isp == 1) ? 1.0 : L->rtemp;
      const double vdp = rp / (L->rtemp + 1) * va0;
      const double gamma0a = sqrt(1.0 - vdp * vdp);
      const double gam1 = sqrt(1.0 + VX(s, i) * VX(s, i) + VY(s, i) * VY(s, i) +
                               VZ(s, i) * VZ(s, i));
      const double vvx = VX(s, i) / gam1, vvy = VY(s, i) / gam1, vvz = VZ(s, i) / gam1;
      VZ(s, i) = (vdp + vvz) / (1.0 + vdp * vvz);
      VY(s, i) = vvy * gamma0a / (1.0 + vdp * vvz);
      VX(s, i) = vvx * gamma0a / (1.0 + vdp * vvz);
    }
  }
#undef X
#undef Y
#undef VX
#undef VY
#undef VZ
  return 0;
}

/* setv for one species: pic/setv.f90:36-128 (linear weights, -dt/2) */
void em2o_setv(const em2o_params *p, const double *fld, int isp, int64_t n,
               double *part) {
  const int64_t nxg = p->nx + 3, w = (int64_t)(p->nx + 3) * (p->ny + 3);
  double *x = part, *y = part + n, *vx = part + 2 * n, *vy = part + 3 * n,
         *vz = part + 4 * n, *gm = part + 5 * n;
  const double ae = -0.25 * p->qm[isp] * p->dt / p->c;
  double *sc = (double *)malloc(sizeof(double) * 6 * (size_t)w);
  double *aex = sc, *aey = sc + w, *aez = sc + 2 * w, *abx = sc + 3 * w,
         *aby = sc + 4 * w, *abz = sc + 5 * w;
  for (int64_t k = 0; k < w; ++k) {
    aex[k] = ae * fld[EM2O_EX * w + k];
    aey[k] = ae * fld[EM2O_EY * w + k];
    aez[k] = ae * fld[EM2O_EZ * w + k];
    abx[k] = ae * fld[EM2O_BX * w + k] - 0.5 * p->tx[isp];
    aby[k] = ae * fld[EM2O_BY * w + k] - 0.5 * p->ty[isp];
    abz[k] = ae * fld[EM2O_BZ * w + k];
  }
#define A(a, i, j) (a)[(int64_t)(j) * nxg + (i)]
  const double c = p->c;
  for (int64_t j = 0; j < n; ++j) {
    const int ix1 = (int)(x[j] + 1), iy1 = (int)(y[j] + 1);
    const double drx = x[j] + 1.0 - ix1, duy = y[j] + 1.0 - iy1;
    const double dlx = 1.0 - drx, dly = 1.0 - duy;
    const int ixh = (int)(x[j] + 0.5), iyh = (int)(y[j] + 0.5);
    const double drxh = x[j] + 0.5 - ixh, duyh = y[j] + 0.5 - iyh;
    const double dlxh = 1.0 - drxh, dlyh = 1.0 - duyh;
    const double sh11 = dlxh * dly, sh12 = dlxh * duy, sh21 = drxh * dly, sh22 = drxh * duy;
    const double s1h1 = dlx * dlyh, s1h2 = dlx * duyh, s2h1 = drx * dlyh, s2h2 = drx * duyh;
    const double sh1h1 = dlxh * dlyh, sh1h2 = dlxh * duyh, sh2h1 = drxh * dlyh,
                 sh2h2 = drxh * duyh;
    const int ix1p = ix1 + 1, iy1p = iy1 + 1, ixhp = ixh + 1, iyhp = iyh + 1;
    const double aexpt = A(aex, ixh, iy1) * sh11 + A(aex, ixhp, iy1) * sh21 +
                         A(aex, ixhp, iy1p) * sh22 + A(aex, ixh, iy1p) * sh12;
    const double aeypt = A(aey, ix1, iyh) * s1h1 + A(aey, ix1p, iyh) * s2h1 +
                         A(aey, ix1p, iyhp) * s2h2 + A(aey, ix1, iyhp) * s1h2;
    const double aezpt = A(aez, ixh, iyh) * sh1h1 + A(aez, ixhp, iyh) * sh2h1 +
                         A(aez, ixhp, iyhp) * sh2h2 + A(aez, ixh, iyhp) * sh1h2;
    double abxpt = A(abx, ixh, iy1) * sh11 + A(abx, ixhp, iy1) * sh21 +
                   A(abx, ixhp, iy1p) * sh22 + A(abx, ixh, iy1p) * sh12;
    double abypt = A(aby, ix1, iyh) * s1h1 + A(aby, ix1p, iyh) * s2h1 +
                   A(aby, ix1p, iyhp) * s2h2 + A(aby, ix1, iyhp) * s1h2;
    double abzpt = A(abz, ixh, iyh) * sh1h1 + A(abz, ixhp, iyh) * sh2h1 +
                   A(abz, ixhp, iyhp) * sh2h2 + A(abz, ixh, iyhp) * sh1h2;
    double g = 1.0 / sqrt(1.0 - vx[j] * vx[j] - vy[j] * vy[j] - vz[j] * vz[j]);
    double gvxs = vx[j] * g + aexpt;
    double gvys = vy[j] * g + aeypt;
    double gvzs = vz[j] * g + aezpt;
    g = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
    const double dcg = 1.0 / (c * g);
    abxpt = dcg * abxpt;
    abypt = dcg * abypt;
    abzpt = dcg * abzpt;
    const double vvx = gvxs + gvys * abzpt - gvzs * abypt;
    const double vvy = gvys + gvzs * abxpt - gvxs * abzpt;
    const double vvz = gvzs + gvxs * abypt - gvys * abxpt;
    const double f = 2.0 / (1.0 + abxpt * abxpt + abypt * abypt + abzpt * abzpt);
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
#undef A
  free(sc);
}

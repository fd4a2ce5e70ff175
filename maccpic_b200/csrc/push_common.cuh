// push_common.cuh -- FP64 particle arithmetic shared by the per-particle
// kernels (push_f64.cu) and the cell-sorted fast path (push_fast_f64.cu).
//
// Every expression keeps the evaluation order of the reference's Fortran
// (pic/move.f90, pic/curnt.f90); the including files are compiled with
// -fmad=false so that no product is fused into a sum behind our back.
#pragma once
#include "em2g_internal.cuh"

namespace em2g {
namespace f64 {

__device__ __forceinline__ double sq(double t) { return t * t; }

// Quadratic weights along one axis.
// "half" staggering (cell-centred nodes, index int(x+1)): pic/move.f90:76-81
__device__ __forceinline__ void w_half(double x, int &i, double &s, double &sp, double &sm) {
  i = (int)(x + 1.0);
  s = 0.75 - sq(x + 0.5 - i);
  sp = 0.5 * sq(1.0 + x - i);
  sm = 0.5 * sq(-x + i);
}
// "node" staggering (integer nodes, index int(x+1.5)): pic/move.f90:127-132
__device__ __forceinline__ void w_node(double x, int &i, double &s, double &sp, double &sm) {
  i = (int)(x + 1.5);
  s = 0.75 - sq(x + 1.0 - i);
  sp = 0.5 * sq(1.5 + x - i);
  sm = 0.5 * sq(-0.5 - x + i);
}

// the nine 2D weights of one staggering, named as in pic/move.f90:86-94
struct W9 {
  double q, qxp, qxm, qyp, qxpyp, qxmyp, qym, qxpym, qxmym;
};

__device__ __forceinline__ W9 weights(double s2x, double s2xp, double s2xm, double s2y,
                                      double s2yp, double s2ym) {
  W9 w;
  w.q = s2x * s2y;
  w.qxp = s2xp * s2y;
  w.qxm = s2xm * s2y;
  w.qyp = s2x * s2yp;
  w.qxpyp = s2xp * s2yp;
  w.qxmyp = s2xm * s2yp;
  w.qym = s2x * s2ym;
  w.qxpym = s2xp * s2ym;
  w.qxmym = s2xm * s2ym;
  return w;
}

// pic/move.f90:95-97: 9-point sum in the reference's order
// (ix,iy) (ix,iyp) (ix,iym) (ixp,iy) (ixp,iyp) (ixp,iym) (ixm,iy) (ixm,iyp) (ixm,iym)
__device__ __forceinline__ double gather9(const double *__restrict__ A, int nxg, int ix,
                                          int iy, const W9 &w) {
  const double *r0 = A + (int64_t)iy * nxg;
  const double *rp = r0 + nxg;
  const double *rm = r0 - nxg;
  return __ldg(r0 + ix) * w.q + __ldg(rp + ix) * w.qyp + __ldg(rm + ix) * w.qym +
         __ldg(r0 + ix + 1) * w.qxp + __ldg(rp + ix + 1) * w.qxpyp +
         __ldg(rm + ix + 1) * w.qxpym + __ldg(r0 + ix - 1) * w.qxm +
         __ldg(rp + ix - 1) * w.qxmyp + __ldg(rm + ix - 1) * w.qxmym;
}

// pic/curnt.f90:63-80: A(i,j) += (s2x*s2y*qd) * v at nine points (atomics)
__device__ __forceinline__ void scatter9(double *A, int nxg, int ix, int iy, double s2x,
                                         double s2xp, double s2xm, double s2y, double s2yp,
                                         double s2ym, double qd, double v) {
  double *r0 = A + (int64_t)iy * nxg;
  double *rp = r0 + nxg;
  double *rm = r0 - nxg;
  atomicAdd(r0 + ix, s2x * s2y * qd * v);
  atomicAdd(r0 + ix + 1, s2xp * s2y * qd * v);
  atomicAdd(r0 + ix - 1, s2xm * s2y * qd * v);
  atomicAdd(rp + ix, s2x * s2yp * qd * v);
  atomicAdd(rp + ix + 1, s2xp * s2yp * qd * v);
  atomicAdd(rp + ix - 1, s2xm * s2yp * qd * v);
  atomicAdd(rm + ix, s2x * s2ym * qd * v);
  atomicAdd(rm + ix + 1, s2xp * s2ym * qd * v);
  atomicAdd(rm + ix - 1, s2xm * s2ym * qd * v);
}

// rho (pic/curnt.f90:208-225): the same pattern without a velocity factor
__device__ __forceinline__ void scatter9_rho(double *A, int nxg, int ix, int iy, double s2x,
                                             double s2xp, double s2xm, double s2y,
                                             double s2yp, double s2ym, double qd) {
  double *r0 = A + (int64_t)iy * nxg;
  double *rp = r0 + nxg;
  double *rm = r0 - nxg;
  atomicAdd(r0 + ix, s2x * s2y * qd);
  atomicAdd(r0 + ix + 1, s2xp * s2y * qd);
  atomicAdd(r0 + ix - 1, s2xm * s2y * qd);
  atomicAdd(rp + ix, s2x * s2yp * qd);
  atomicAdd(rp + ix + 1, s2xp * s2yp * qd);
  atomicAdd(rp + ix - 1, s2xm * s2yp * qd);
  atomicAdd(rm + ix, s2x * s2ym * qd);
  atomicAdd(rm + ix + 1, s2xp * s2ym * qd);
  atomicAdd(rm + ix - 1, s2xm * s2ym * qd);
}

// Pointers to the six scaled field arrays of one species (pic/move.f90:52-64).
struct Scaled {
  const double *aex, *aey, *aez, *abx, *aby, *abz;
};

// Field gather and relativistic Boris push of one particle
// (pic/move.f90:76-203).  Updates vx, vy, vz, g in place; returns the
// gamma used for ake (the one after the first half acceleration).
__device__ __forceinline__ double gather_boris(const Scaled &S, int nxg, double c, double xj,
                                               double yj, double &vx, double &vy, double &vz,
                                               double &g) {
  int ixh, ixn, iyh, iyn;
  double sxh, sxhp, sxhm, sxn, sxnp, sxnm, syh, syhp, syhm, syn, synp, synm;
  w_half(xj, ixh, sxh, sxhp, sxhm);
  w_node(yj, iyn, syn, synp, synm);
  // Ex, Bx: x half, y node (pic/move.f90:76-100)
  W9 w = weights(sxh, sxhp, sxhm, syn, synp, synm);
  const double aexpt = gather9(S.aex, nxg, ixh, iyn, w);
  double abxpt = gather9(S.abx, nxg, ixh, iyn, w);
  // Ez, Bz: half, half (pic/move.f90:103-124)
  w_half(yj, iyh, syh, syhp, syhm);
  w = weights(sxh, sxhp, sxhm, syh, syhp, syhm);
  const double aezpt = gather9(S.aez, nxg, ixh, iyh, w);
  double abzpt = gather9(S.abz, nxg, ixh, iyh, w);
  // Ey, By: node, half (pic/move.f90:127-148)
  w_node(xj, ixn, sxn, sxnp, sxnm);
  w = weights(sxn, sxnp, sxnm, syh, syhp, syhm);
  const double aeypt = gather9(S.aey, nxg, ixn, iyh, w);
  double abypt = gather9(S.aby, nxg, ixn, iyh, w);
  // relativistic Boris (pic/move.f90:176-203)
  double gvxs = vx * g + aexpt;
  double gvys = vy * g + aeypt;
  double gvzs = vz * g + aezpt;
  double gm = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
  const double g_ake = gm;
  const double dcg = 1.0 / (c * gm);
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
  gm = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
  g = gm;
  vx = gvxs / gm;
  vy = gvys / gm;
  vz = gvzs / gm;
  return g_ake;
}

// pic/curnt.f90:181-194: x += vx*dt/dx, one periodic wrap
__device__ __forceinline__ void move_wrap(double &x, double &y, double vx, double vy,
                                          double dt, double dx, double dy, double xn,
                                          double yn) {
  x = x + vx * dt / dx;
  y = y + vy * dt / dy;
  if (x < 0.0) x = x + xn;
  if (x >= xn) x = x - xn;
  if (y < 0.0) y = y + yn;
  if (y >= yn) y = y - yn;
}

// jm (or jp) of one particle with atomics, pic/curnt.f90:53-132
__device__ __forceinline__ void deposit_j_atomic(double *jx, double *jy, double *jz, int nxg,
                                                 double x, double y, double qd, double vx,
                                                 double vy, double vz) {
  int ixh, ixn, iyh, iyn;
  double sxh, sxhp, sxhm, sxn, sxnp, sxnm, syh, syhp, syhm, syn, synp, synm;
  w_half(x, ixh, sxh, sxhp, sxhm);
  w_node(y, iyn, syn, synp, synm);
  scatter9(jx, nxg, ixh, iyn, sxh, sxhp, sxhm, syn, synp, synm, qd, vx);
  w_half(y, iyh, syh, syhp, syhm);
  scatter9(jz, nxg, ixh, iyh, sxh, sxhp, sxhm, syh, syhp, syhm, qd, vz);
  w_node(x, ixn, sxn, sxnp, sxnm);
  scatter9(jy, nxg, ixn, iyh, sxn, sxnp, sxnm, syh, syhp, syhm, qd, vy);
}

// rho of one particle with atomics, pic/curnt.f90:197-225
__device__ __forceinline__ void deposit_rho_atomic(double *rho, int nxg, double x, double y,
                                                   double qd) {
  int ixn, iyn;
  double sxn, sxnp, sxnm, syn, synp, synm;
  w_node(x, ixn, sxn, sxnp, sxnm);
  w_node(y, iyn, syn, synp, synm);
  scatter9_rho(rho, nxg, ixn, iyn, sxn, sxnp, sxnm, syn, synp, synm, qd);
}

}  // namespace f64
}  // namespace em2g

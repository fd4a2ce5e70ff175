// push_f64.cu -- particle kernels of the FP64 drop-in path.
//
// This file is compiled with -fmad=false: every product and sum is rounded
// on its own, in the order of the reference's Fortran, so for given fields a
// particle's new v, gamma, x, y and its deposit contributions are bitwise
// those of em2 (pic/move.f90, pic/curnt.f90).  Only the order in which the
// contributions of different particles are summed into rho/J (atomics) and
// into ake differs from the reference's serial loop.
#include "em2g_internal.cuh"

namespace em2g {
namespace {

constexpr int kThreads = 256;

struct PushArgs {
  const double *__restrict__ s;  // aex, aey, aez, abx, aby, abz (6*w)
  double *fld;                   // field block (deposit targets)
  double *part;                  // 6*cap
  int64_t n, cap, w;
  int nxg;
  double c, qd, dt, dx, dy, xn, yn;
  double *ake_partial;
};

__device__ __forceinline__ double sq(double t) { return t * t; }

// 9-point quadratic-spline weights of one staggering, in the reference's
// naming: s2x/s2xp/s2xm along x, s2y/s2yp/s2ym along y.
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

// pic/move.f90:95-97: sum in the reference's order
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

// pic/curnt.f90:72-80: A(i,j) += (s2x*s2y*qd) * v, nine points
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

// rho (pic/curnt.f90:208-225): same pattern without the velocity factor
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

// Quadratic weights of the two staggerings along one axis.
// "half" (cell-centred node, index int(x+1)): pic/move.f90:76-81
__device__ __forceinline__ void w_half(double x, int &i, double &s, double &sp, double &sm) {
  i = (int)(x + 1.0);
  s = 0.75 - sq(x + 0.5 - i);
  sp = 0.5 * sq(1.0 + x - i);
  sm = 0.5 * sq(-x + i);
}
// "node" (integer node, index int(x+1.5)): pic/move.f90:127-132
__device__ __forceinline__ void w_node(double x, int &i, double &s, double &sp, double &sm) {
  i = (int)(x + 1.5);
  s = 0.75 - sq(x + 1.0 - i);
  sp = 0.5 * sq(1.5 + x - i);
  sm = 0.5 * sq(-0.5 - x + i);
}

template <int MODE>
__global__ void __launch_bounds__(kThreads) k_push_f64(PushArgs a) {
  const int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  double akel = 0.0;
  if (j < a.n) {
    double *x = a.part, *y = a.part + a.cap, *vx = a.part + 2 * a.cap,
           *vy = a.part + 3 * a.cap, *vz = a.part + 4 * a.cap, *gm = a.part + 5 * a.cap;
    double xj = x[j], yj = y[j];
    double vxj = vx[j], vyj = vy[j], vzj = vz[j];
    const int nxg = a.nxg;
    if (MODE & 1) {
      const double gj = gm[j];
      const double *aex = a.s, *aey = a.s + a.w, *aez = a.s + 2 * a.w, *abx = a.s + 3 * a.w,
                   *aby = a.s + 4 * a.w, *abz = a.s + 5 * a.w;
      int ixh, ixn, iyh, iyn;
      double sxh, sxhp, sxhm, sxn, sxnp, sxnm, syh, syhp, syhm, syn, synp, synm;
      w_half(xj, ixh, sxh, sxhp, sxhm);
      w_node(yj, iyn, syn, synp, synm);
      // Ex, Bx: x half, y node (pic/move.f90:76-100)
      W9 w = weights(sxh, sxhp, sxhm, syn, synp, synm);
      const double aexpt = gather9(aex, nxg, ixh, iyn, w);
      double abxpt = gather9(abx, nxg, ixh, iyn, w);
      // Ez, Bz: half, half (pic/move.f90:103-124)
      w_half(yj, iyh, syh, syhp, syhm);
      w = weights(sxh, sxhp, sxhm, syh, syhp, syhm);
      const double aezpt = gather9(aez, nxg, ixh, iyh, w);
      double abzpt = gather9(abz, nxg, ixh, iyh, w);
      // Ey, By: node, half (pic/move.f90:127-148)
      w_node(xj, ixn, sxn, sxnp, sxnm);
      w = weights(sxn, sxnp, sxnm, syh, syhp, syhm);
      const double aeypt = gather9(aey, nxg, ixn, iyh, w);
      double abypt = gather9(aby, nxg, ixn, iyh, w);
      // relativistic Boris (pic/move.f90:176-203)
      double gvxs = vxj * gj + aexpt;
      double gvys = vyj * gj + aeypt;
      double gvzs = vzj * gj + aezpt;
      double g = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
      akel = g - 1.0;
      const double dcg = 1.0 / (a.c * g);
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
      vxj = gvxs / g;
      vyj = gvys / g;
      vzj = gvzs / g;
      gm[j] = g;
      vx[j] = vxj;
      vy[j] = vyj;
      vz[j] = vzj;
    }
    if (MODE & 2) {
      double *rho = a.fld + EM2G_RHO * a.w, *jxm = a.fld + EM2G_JXM * a.w,
             *jxp = a.fld + EM2G_JXP * a.w, *jym = a.fld + EM2G_JYM * a.w,
             *jyp = a.fld + EM2G_JYP * a.w, *jzm = a.fld + EM2G_JZM * a.w,
             *jzp = a.fld + EM2G_JZP * a.w;
      const double qd = a.qd;
      int ixh, ixn, iyh, iyn;
      double sxh, sxhp, sxhm, sxn, sxnp, sxnm, syh, syhp, syhm, syn, synp, synm;
      // jm at the old position (pic/curnt.f90:53-132)
      w_half(xj, ixh, sxh, sxhp, sxhm);
      w_node(yj, iyn, syn, synp, synm);
      scatter9(jxm, nxg, ixh, iyn, sxh, sxhp, sxhm, syn, synp, synm, qd, vxj);
      w_half(yj, iyh, syh, syhp, syhm);
      scatter9(jzm, nxg, ixh, iyh, sxh, sxhp, sxhm, syh, syhp, syhm, qd, vzj);
      w_node(xj, ixn, sxn, sxnp, sxnm);
      scatter9(jym, nxg, ixn, iyh, sxn, sxnp, sxnm, syh, syhp, syhm, qd, vyj);
      // move and wrap (pic/curnt.f90:181-194)
      xj = xj + vxj * a.dt / a.dx;
      yj = yj + vyj * a.dt / a.dy;
      if (xj < 0.0) xj = xj + a.xn;
      if (xj >= a.xn) xj = xj - a.xn;
      if (yj < 0.0) yj = yj + a.yn;
      if (yj >= a.yn) yj = yj - a.yn;
      x[j] = xj;
      y[j] = yj;
      // rho at the new position (pic/curnt.f90:197-225)
      w_node(xj, ixn, sxn, sxnp, sxnm);
      w_node(yj, iyn, syn, synp, synm);
      scatter9_rho(rho, nxg, ixn, iyn, sxn, sxnp, sxnm, syn, synp, synm, qd);
      // jp at the new position (pic/curnt.f90:227-303)
      w_half(xj, ixh, sxh, sxhp, sxhm);
      scatter9(jxp, nxg, ixh, iyn, sxh, sxhp, sxhm, syn, synp, synm, qd, vxj);
      w_half(yj, iyh, syh, syhp, syhm);
      scatter9(jzp, nxg, ixh, iyh, sxh, sxhp, sxhm, syh, syhp, syhm, qd, vzj);
      scatter9(jyp, nxg, ixn, iyh, sxn, sxnp, sxnm, syh, syhp, syhm, qd, vyj);
    }
  }
  if (MODE & 1) {
    // block sum of (gamma - 1) in a fixed order
    __shared__ double red[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) akel += __shfl_down_sync(0xffffffffu, akel, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = akel;
    __syncthreads();
    if (threadIdx.x < 32) {
      double v = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (threadIdx.x == 0) a.ake_partial[blockIdx.x] = v;
    }
  }
}

// pic/move.f90:52-64: E and B times ae = 0.5*qm*dt/c, plus tx/ty on Bx/By
__global__ void k_prescale(const double *__restrict__ fld, double *__restrict__ s, int64_t w,
                           double ae, double tx, double ty) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= w) return;
  s[k] = ae * fld[EM2G_EX * w + k];
  s[w + k] = ae * fld[EM2G_EY * w + k];
  s[2 * w + k] = ae * fld[EM2G_EZ * w + k];
  s[3 * w + k] = ae * fld[EM2G_BX * w + k] + tx;
  s[4 * w + k] = ae * fld[EM2G_BY * w + k] + ty;
  s[5 * w + k] = ae * fld[EM2G_BZ * w + k];
}

// one block: sum the per-block partials in a fixed order, times am*dn
__global__ void k_ake_finish(const double *__restrict__ partial, int nb, double amdn_am,
                             double amdn_dn, double *out) {
  __shared__ double red[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v += partial[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) *out = v * amdn_am * amdn_dn;
  }
}

}  // namespace

int launch_prescale(em2g_ctx *c, int isp) {
  const double ae = 0.5 * c->P.qm[isp] * c->P.dt / c->P.c;
  const int64_t w = c->g.w;
  const int blocks = (int)((w + 255) / 256);
  k_prescale<<<blocks, 256, 0, c->stream>>>(c->fld, c->scaled + (int64_t)isp * 6 * w, w, ae,
                                            c->P.tx[isp], c->P.ty[isp]);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

int launch_push_f64(em2g_ctx *c, int isp, int mode) {
  Species &S = c->sp[isp];
  PushArgs a;
  a.s = c->scaled + (int64_t)isp * 6 * c->g.w;
  a.fld = c->fld;
  a.part = S.part;
  a.n = S.n;
  a.cap = S.cap;
  a.w = c->g.w;
  a.nxg = c->g.nxg;
  a.c = c->P.c;
  a.qd = c->P.q[isp] * c->P.dn[isp] / (c->P.dx * c->P.dy);  // pic/curnt.f90:41
  a.dt = c->P.dt;
  a.dx = c->P.dx;
  a.dy = c->P.dy;
  a.xn = (double)c->P.nx;
  a.yn = (double)c->P.ny;
  a.ake_partial = c->red;
  const int64_t nb64 = (S.n + kThreads - 1) / kThreads;
  if (nb64 > c->red_blocks) return fail(EM2G_ERR_RANGE, "particle count exceeds reduction scratch");
  const int nb = (int)(nb64 > 0 ? nb64 : 1);
  if (mode < 1 || mode > 3) return fail(EM2G_ERR_INVALID, "bad push mode");
  int rc = timing_begin(c);
  if (rc) return rc;
  switch (mode) {
    case 1: k_push_f64<1><<<nb, kThreads, 0, c->stream>>>(a); break;
    case 2: k_push_f64<2><<<nb, kThreads, 0, c->stream>>>(a); break;
    default: k_push_f64<3><<<nb, kThreads, 0, c->stream>>>(a); break;
  }
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  if ((rc = timing_end(c))) return rc;
  if (mode & 1) {
    k_ake_finish<<<1, 256, 0, c->stream>>>(c->red, nb, c->P.am[isp], c->P.dn[isp],
                                           c->dev_out + isp);
    c->launches += 1;
    EM2G_CUDA(cudaGetLastError());
  }
  return EM2G_OK;
}

}  // namespace em2g

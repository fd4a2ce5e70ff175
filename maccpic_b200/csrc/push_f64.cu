// push_f64.cu -- particle kernels of the FP64 drop-in path.
//
// This file is compiled with -fmad=false: every product and sum is rounded
// on its own, in the order of the reference's Fortran, so for given fields a
// particle's new v, gamma, x, y and its deposit contributions are bitwise
// those of em2 (pic/move.f90, pic/curnt.f90).  Only the order in which the
// contributions of different particles are summed into rho/J (atomics) and
// into ake differs from the reference's serial loop.
#include "push_common.cuh"

namespace em2g {
namespace {

using namespace f64;

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
      const Scaled S{a.s, a.s + a.w, a.s + 2 * a.w, a.s + 3 * a.w, a.s + 4 * a.w,
                     a.s + 5 * a.w};
      double gj = gm[j];
      akel = gather_boris(S, nxg, a.c, xj, yj, vxj, vyj, vzj, gj) - 1.0;
      gm[j] = gj;
      vx[j] = vxj;
      vy[j] = vyj;
      vz[j] = vzj;
    }
    if (MODE & 2) {
      double *rho = a.fld + EM2G_RHO * a.w;
      // jm at the old position, move and wrap, rho and jp at the new one
      // (pic/curnt.f90:53-303)
      deposit_j_atomic(a.fld + EM2G_JXM * a.w, a.fld + EM2G_JYM * a.w, a.fld + EM2G_JZM * a.w,
                       nxg, xj, yj, a.qd, vxj, vyj, vzj);
      move_wrap(xj, yj, vxj, vyj, a.dt, a.dx, a.dy, a.xn, a.yn);
      x[j] = xj;
      y[j] = yj;
      deposit_rho_atomic(rho, nxg, xj, yj, a.qd);
      deposit_j_atomic(a.fld + EM2G_JXP * a.w, a.fld + EM2G_JYP * a.w, a.fld + EM2G_JZP * a.w,
                       nxg, xj, yj, a.qd, vxj, vyj, vzj);
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

// first level of the ake sum: block b adds the partials of its contiguous
// chunk, in a fixed order, into l1[b]
__global__ void k_ake_level1(const double *__restrict__ partial, int nb, double *l1) {
  __shared__ double red[32];
  const int chunk = (nb + (int)gridDim.x - 1) / (int)gridDim.x;
  const int lo = (int)blockIdx.x * chunk, hi = min(nb, lo + chunk);
  double v = 0.0;
  for (int i = lo + (int)threadIdx.x; i < hi; i += blockDim.x) v += partial[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) l1[blockIdx.x] = v;
  }
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
  if (mode & 1) return launch_ake_finish(c, isp, nb);
  return EM2G_OK;
}

int launch_ake_finish(em2g_ctx *c, int isp, int nblocks_used) {
  const double *src = c->red;
  int n = nblocks_used;
  // many partials (the fast pushes write one per warp of a row segment):
  // first spread the reading over kAkeBlocks blocks
  if (n > 16 * kAkeBlocks) {
    k_ake_level1<<<kAkeBlocks, 256, 0, c->stream>>>(c->red, n, c->ake_l1);
    c->launches += 1;
    src = c->ake_l1;
    n = kAkeBlocks;
  }
  k_ake_finish<<<1, 1024, 0, c->stream>>>(src, n, c->P.am[isp], c->P.dn[isp], c->dev_out + isp);
  c->launches += 1;
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

}  // namespace em2g

// setv.cu -- em2's start-up push of the velocities from t = 0 back to
// t = -dt/2 (pic/setv.f90:36-128) on a block of particles in device memory:
// one Boris push of half a step with the initial E and B gathered with
// LINEAR weights (the only place em2 uses them), so that a loader that
// draws v at t = 0 starts a run exactly as em2's fresh run does.
//
// Compiled with -fmad=false and written in setv's evaluation order, so each
// particle's result is bitwise that of em2's arithmetic (the C restatement
// in oracle/em2_loader_oracle.c, em2o_setv).  Context-free, like
// em2g_smooth2_static: the parameters come from an em2g_params, the fields
// from the caller's FP64 block in em2's layout.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "em2g_internal.cuh"

namespace {

struct SetvArgs {
  const double *fld;  // 13 x (ny+3) x (nx+3), em2's (0:nx+2, 0:ny+2) order
  double *part;       // x, y, vx, vy, vz, gamma, n each
  int64_t n;
  int nx, ny;
  double ae, c, htx, hty;  // ae = -qm dt / (4c); 0.5 tx, 0.5 ty
};

// a particle setv can take: position inside [0, nx) x [0, ny) (its
// stencils then stay inside the guarded arrays), finite speed below c
__device__ __forceinline__ bool setv_ok(const SetvArgs &a, int64_t j) {
  const int64_t n = a.n;
  const double x = a.part[j], y = a.part[n + j];
  const double vx = a.part[2 * n + j], vy = a.part[3 * n + j], vz = a.part[4 * n + j];
  const double v2 = vx * vx + vy * vy + vz * vz;
  return x >= 0.0 && x < (double)a.nx && y >= 0.0 && y < (double)a.ny && v2 < 1.0;
}

__global__ void k_setv_check(SetvArgs a, unsigned long long *bad) {
  unsigned long long cnt = 0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < a.n;
       j += (int64_t)gridDim.x * blockDim.x)
    cnt += setv_ok(a, j) ? 0 : 1;
  if (cnt) atomicAdd(bad, cnt);
}

__global__ void k_setv(SetvArgs a) {
  const int64_t n = a.n, w = (int64_t)(a.nx + 3) * (a.ny + 3), nxg = a.nx + 3;
  const double *ex = a.fld + EM2G_EX * w, *ey = a.fld + EM2G_EY * w, *ez = a.fld + EM2G_EZ * w;
  const double *bx = a.fld + EM2G_BX * w, *by = a.fld + EM2G_BY * w, *bz = a.fld + EM2G_BZ * w;
  double *x = a.part, *y = a.part + n, *vx = a.part + 2 * n, *vy = a.part + 3 * n,
         *vz = a.part + 4 * n, *gm = a.part + 5 * n;
  const double ae = a.ae, c = a.c;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    // the scaled fields of setv's arrays aex..abz, point by point
    auto sE = [&](const double *f, int i, int k) { return ae * f[(int64_t)k * nxg + i]; };
    auto sB = [&](const double *f, int i, int k, double h) {
      return ae * f[(int64_t)k * nxg + i] - h;
    };
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
    const double aexpt = sE(ex, ixh, iy1) * sh11 + sE(ex, ixhp, iy1) * sh21 +
                         sE(ex, ixhp, iy1p) * sh22 + sE(ex, ixh, iy1p) * sh12;
    const double aeypt = sE(ey, ix1, iyh) * s1h1 + sE(ey, ix1p, iyh) * s2h1 +
                         sE(ey, ix1p, iyhp) * s2h2 + sE(ey, ix1, iyhp) * s1h2;
    const double aezpt = sE(ez, ixh, iyh) * sh1h1 + sE(ez, ixhp, iyh) * sh2h1 +
                         sE(ez, ixhp, iyhp) * sh2h2 + sE(ez, ixh, iyhp) * sh1h2;
    double abxpt = sB(bx, ixh, iy1, a.htx) * sh11 + sB(bx, ixhp, iy1, a.htx) * sh21 +
                   sB(bx, ixhp, iy1p, a.htx) * sh22 + sB(bx, ixh, iy1p, a.htx) * sh12;
    double abypt = sB(by, ix1, iyh, a.hty) * s1h1 + sB(by, ix1p, iyh, a.hty) * s2h1 +
                   sB(by, ix1p, iyhp, a.hty) * s2h2 + sB(by, ix1, iyhp, a.hty) * s1h2;
    double abzpt = sB(bz, ixh, iyh, 0.0) * sh1h1 + sB(bz, ixhp, iyh, 0.0) * sh2h1 +
                   sB(bz, ixhp, iyhp, 0.0) * sh2h2 + sB(bz, ixh, iyhp, 0.0) * sh1h2;
    double g = 1.0 / sqrt(1.0 - vx[j] * vx[j] - vy[j] * vy[j] - vz[j] * vz[j]);
    // half acceleration along E, the rotation about B / gamma, the second
    // half acceleration (pic/setv.f90:99-121)
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
    // v = u / gamma (pic/setv.f90:125-128)
    g = sqrt(1.0 + gvxs * gvxs + gvys * gvys + gvzs * gvzs);
    gm[j] = g;
    vx[j] = gvxs / g;
    vy[j] = gvys / g;
    vz[j] = gvzs / g;
  }
}

}  // namespace

using namespace em2g;

extern "C" {

int em2g_setv_device(const em2g_params *p, int isp, const double *dev_fields, double *dev_parts,
                     int64_t n, void *cuda_stream) {
  if (!p || !dev_fields || (!dev_parts && n > 0))
    return fail(EM2G_ERR_INVALID, "setv: null pointer");
  if (p->nx < 4 || p->ny < 4) return fail(EM2G_ERR_INVALID, "setv: nx and ny must be >= 4");
  if (p->nsp < 1 || p->nsp > EM2G_MAX_SPECIES || isp < 0 || isp >= p->nsp)
    return fail(EM2G_ERR_INVALID, "setv: species index outside 0..nsp-1");
  if (!(p->c > 0.0) || !std::isfinite(p->dt) || !std::isfinite(p->qm[isp]) ||
      !std::isfinite(p->tx[isp]) || !std::isfinite(p->ty[isp]))
    return fail(EM2G_ERR_INVALID, "setv: c must be > 0 and dt, qm, tx, ty finite");
  if (n < 0) return fail(EM2G_ERR_INVALID, "setv: negative particle count");
  if (n == 0) return EM2G_OK;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(EM2G_ERR_CUDA, std::string("setv: an earlier CUDA error is pending (") +
                                   cudaGetErrorString(e) + "); nothing was launched");
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  SetvArgs a;
  a.fld = dev_fields;
  a.part = dev_parts;
  a.n = n;
  a.nx = p->nx;
  a.ny = p->ny;
  a.ae = -0.25 * p->qm[isp] * p->dt / p->c;
  a.c = p->c;
  a.htx = 0.5 * p->tx[isp];
  a.hty = 0.5 * p->ty[isp];
  int dev = 0, sms = 1;
  EM2G_CUDA(cudaGetDevice(&dev));
  EM2G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t want = (n + 255) / 256, cap = (int64_t)sms * 8;
  const int blocks = (int)(want < cap ? want : cap);
  // every particle checked before any is changed: a rejected block is left
  // as it was
  unsigned long long *bad = nullptr, nbad = 0;
  EM2G_CUDA(cudaMallocAsync((void **)&bad, sizeof(unsigned long long), st));
  e = cudaMemsetAsync(bad, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    k_setv_check<<<blocks, 256, 0, st>>>(a, bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFreeAsync(bad, st);
  if (e != cudaSuccess) return cuda_fail(e, "setv check");
  if (nbad)
    return fail(EM2G_ERR_RANGE, "setv: " + std::to_string(nbad) +
                                    " particles outside [0,nx) x [0,ny) or not slower than c");
  k_setv<<<blocks, 256, 0, st>>>(a);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

}  // extern "C"

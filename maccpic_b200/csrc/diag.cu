// diag.cu -- run diagnostics computed on the GPU in FP64, for both field
// precisions: the field energies of the current state (the quantity of
// pic/fields.f90:267-347 over the whole grid), the reconnected flux of both
// current sheets, and the Poisson residuals of the last cleaning.
//
// Reconnected flux.  With Bx = d(psi)/dy and By = -d(psi)/dx, psi along the
// row through a sheet's centre is psi(x) = -integral of By dx; the flux
// between the X point and the O point is max(psi) - min(psi) along that row.
// By(ix, iy) sits at x = (ix-1) dx, y = (iy-1/2) dy; the sheet centre
// y = ny/4 (ny/4 + ny/2 for the second sheet) lies half-way between rows
// iy = ny/4 and ny/4 + 1, whose By values are averaged.
#include "em2g_internal.cuh"

namespace em2g {
namespace {

template <typename T>
__global__ void k_sheet_flux(const T *__restrict__ by, int nx, int nxg, int row_lo,
                             double dx, double *out) {
  // one block: serial prefix sum by warp 0 in fixed order (nx values)
  __shared__ double smin[32], smax[32];
  if (threadIdx.x >= 32) return;
  const T *r0 = by + (int64_t)row_lo * nxg, *r1 = r0 + nxg;
  // each lane sums a contiguous chunk, then an exclusive scan of the chunks
  const int chunk = (nx + 31) / 32;
  const int lo = threadIdx.x * chunk, hi = min(nx, lo + chunk);
  double s = 0.0;
  for (int i = lo; i < hi; ++i) s += 0.5 * ((double)r0[1 + i] + (double)r1[1 + i]);
  double incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const double t = __shfl_up_sync(0xffffffffu, incl, o);
    if ((int)threadIdx.x >= o) incl += t;
  }
  double run = incl - s;  // sum before this chunk
  double mn = 1e300, mx = -1e300;
  for (int i = lo; i < hi; ++i) {
    run += 0.5 * ((double)r0[1 + i] + (double)r1[1 + i]);
    const double psi = -run * dx;
    mn = fmin(mn, psi);
    mx = fmax(mx, psi);
  }
  smin[threadIdx.x] = mn;
  smax[threadIdx.x] = mx;
  __syncwarp();
  if (threadIdx.x == 0) {
    double a = smin[0], b = smax[0];
    for (int k = 1; k < 32; ++k) {
      a = fmin(a, smin[k]);
      b = fmax(b, smax[k]);
    }
    *out = b - a;
  }
}

template <typename T>
__global__ void k_energy_now(const T *__restrict__ fld, int nx, int ny, int nxg, int64_t w,
                             double *partial) {
  __shared__ double sh[32];
  const int k = blockIdx.y;
  const T *a = fld + k * w;
  const int64_t N = (int64_t)nx * ny;
  double loc = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < N;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int ix = 1 + (int)(t % nx), iy = 1 + (int)(t / nx);
    const double v = (double)a[(int64_t)iy * nxg + ix];
    loc += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) loc += __shfl_down_sync(0xffffffffu, loc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = loc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = v;
  }
}

__global__ void k_energy_now_finish(const double *__restrict__ partial, int nb, double scale,
                                    double *out) {
  const int k = threadIdx.x;
  if (k >= 6) return;
  double v = 0.0;
  for (int i = 0; i < nb; ++i) v += partial[k * nb + i];
  out[k] = v * scale;
}

// out[0..6) energies, out[6..8) flux of the sheets at ny/4 and 3ny/4
template <typename T>
int diag_t(const T *fld, const Grid &g, double dx, double *red, double *out, cudaStream_t st) {
  const int nx = g.nx, ny = g.ny, nxg = g.nxg;
  const int64_t w = g.w;
  const int nb = kEnergyBlocks;
  // 0.5 * mean of E^2 + B^2 per component over the interior (pic/fields.f90:341
  // with the whole grid): anorml1 = 0.5*dx*dy/(Lx*Ly) = 0.5/(nx*ny)
  const double scale = 0.5 / ((double)nx * ny);
  k_energy_now<T><<<dim3(nb, 6), 256, 0, st>>>(fld, nx, ny, nxg, w, red);
  k_energy_now_finish<<<1, 32, 0, st>>>(red, nb, scale, out);
  const T *by = fld + EM2G_BY * w;
  k_sheet_flux<T><<<1, 32, 0, st>>>(by, nx, nxg, ny / 4, dx, out + 6);
  k_sheet_flux<T><<<1, 32, 0, st>>>(by, nx, nxg, ny / 4 + ny / 2, dx, out + 7);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

}  // namespace

int diagnostics(em2g_ctx *c) {
  c->launches += 4;
  if (c->P.precision == EM2G_FP32)
    return diag_t<float>(c->fld32, c->g, c->P.dx, c->red, c->dev_out + 10, c->stream);
  return diag_t<double>(c->fld, c->g, c->P.dx, c->red, c->dev_out + 10, c->stream);
}

int diag_fields_f32(const float *fld, const Grid &g, double dx, double *red, double *out,
                    cudaStream_t st) {
  return diag_t<float>(fld, g, dx, red, out, st);
}

}  // namespace em2g

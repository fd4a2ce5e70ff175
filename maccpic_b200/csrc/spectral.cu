// spectral.cu -- exact solve of em2's periodic Poisson problem by FFT, an
// option next to the CG of cgm (pic/fields.f90:508-651).
//
// cgm solves L u = f on the nx*ny periodic grid with the unit 5-point
// Laplacian L u = u(i+1) + u(i-1) + u(j+1) + u(j-1) - 4 u and stops at mean
// r^2 < 1e-9.  Fourier modes diagonalise L with eigenvalues
// 2 cos(2 pi kx/nx) + 2 cos(2 pi ky/ny) - 4, so the exact mean-free solution
// is u = F^-1 [ F f / eig ] with the (0, 0) mode set to zero.  The exact
// solve makes the step a smooth function of its input (the CG's stopping
// test is not), which the adjoint needs; it is not em2's arithmetic and is
// never the default.
//
// FFTs are radix-2 Cooley-Tukey, decimation in time, one CTA per row (then
// per column) with the whole line in shared memory: bit-reversed load,
// log2(n) butterfly stages with a block barrier between them.  Grids must
// have power-of-two sides up to 8192.
#include "em2g_internal.cuh"

namespace em2g {
namespace {

constexpr int kFftThreads = 256;

__device__ __forceinline__ void fft_shared(double2 *x, int m, double sign) {
  const int n = 1 << m;
  for (int s = 1; s <= m; ++s) {
    const int half = 1 << (s - 1);
    for (int b = threadIdx.x; b < n / 2; b += blockDim.x) {
      const int k = b & (half - 1);
      const int i0 = ((b >> (s - 1)) << s) + k;
      const int i1 = i0 + half;
      double sn, cs;
      sincospi(sign * (double)k / (double)half, &sn, &cs);
      const double2 a = x[i0], c = x[i1];
      const double tr = c.x * cs - c.y * sn, ti = c.x * sn + c.y * cs;
      x[i0] = make_double2(a.x + tr, a.y + ti);
      x[i1] = make_double2(a.x - tr, a.y - ti);
    }
    __syncthreads();
  }
}

// one row of n = 2^m values: real input fin or complex z; complex output z
// or the real part, times scale, to fout
__global__ void __launch_bounds__(kFftThreads)
    k_fft_rows(const double *fin, double2 *z, double *fout, int n, int m, double sign,
               double scale) {
  extern __shared__ double2 x[];
  const int64_t row = (int64_t)blockIdx.x * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    x[__brev((unsigned)i) >> (32 - m)] = fin ? make_double2(fin[row + i], 0.0) : z[row + i];
  __syncthreads();
  fft_shared(x, m, sign);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (fout)
      fout[row + i] = x[i].x * scale;
    else
      z[row + i] = x[i];
  }
}

// one column of ny = 2^m values (row pitch nx), in place
__global__ void __launch_bounds__(kFftThreads)
    k_fft_cols(double2 *z, int nx, int ny, int m, double sign) {
  extern __shared__ double2 x[];
  const int col = blockIdx.x;
  for (int j = threadIdx.x; j < ny; j += blockDim.x)
    x[__brev((unsigned)j) >> (32 - m)] = z[(int64_t)j * nx + col];
  __syncthreads();
  fft_shared(x, m, sign);
  for (int j = threadIdx.x; j < ny; j += blockDim.x) z[(int64_t)j * nx + col] = x[j];
}

__global__ void k_divide_eig(double2 *z, int nx, int ny) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)nx * ny) return;
  const int i = (int)(k % nx), j = (int)(k / nx);
  if (i == 0 && j == 0) {
    z[k] = make_double2(0.0, 0.0);
    return;
  }
  const double e = 2.0 * cospi(2.0 * i / nx) + 2.0 * cospi(2.0 * j / ny) - 4.0;
  z[k] = make_double2(z[k].x / e, z[k].y / e);
}

int log2_exact(int n) {
  int m = 0;
  while ((1 << m) < n) ++m;
  return (1 << m) == n ? m : -1;
}

}  // namespace

bool spectral_size_ok(int nx, int ny) {
  return log2_exact(nx) >= 2 && log2_exact(ny) >= 2 && nx <= 8192 && ny <= 8192;
}

int spectral_prepare() {
  const int bytes = (int)sizeof(double2) * 8192;  // the longest line allowed
  EM2G_CUDA(cudaFuncSetAttribute(k_fft_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EM2G_CUDA(cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return EM2G_OK;
}

// u = L^-1 f (mean-free), f and u nx*ny row-major; work: nx*ny double2.
// f and u may be the same array.  5 launches.
int spectral_solve(const double *f, double *u, int nx, int ny, double2 *work, cudaStream_t st) {
  const int mx = log2_exact(nx), my = log2_exact(ny);
  if (mx < 2 || my < 2) return fail(EM2G_ERR_INVALID, "spectral solve needs power-of-two sides");
  const size_t sx = sizeof(double2) * nx, sy = sizeof(double2) * ny;
  const int64_t N = (int64_t)nx * ny;
  k_fft_rows<<<ny, kFftThreads, sx, st>>>(f, work, nullptr, nx, mx, -1.0, 1.0);
  k_fft_cols<<<nx, kFftThreads, sy, st>>>(work, nx, ny, my, -1.0);
  k_divide_eig<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(work, nx, ny);
  k_fft_cols<<<nx, kFftThreads, sy, st>>>(work, nx, ny, my, 1.0);
  k_fft_rows<<<ny, kFftThreads, sx, st>>>(nullptr, work, u, nx, mx, 1.0, 1.0 / (double)N);
  EM2G_CUDA(cudaGetLastError());
  return EM2G_OK;
}

}  // namespace em2g

// smooth2_static.cu -- em2g_smooth2_static: smooth2 (pic/smooth.f90:95-179)
// on a caller's device array, with no device allocation at all.
//
// Who needs it: callers that cannot call cudaMalloc and so cannot create an
// em2g context -- host code that hands over device arrays it manages itself
// under a fixed memory budget, code running while a stream is being
// captured, or a process whose GPU memory is already reserved by another
// allocator.  They pass the array in and get it back filtered in place.
//
// smooth2 needs one scratch array the size of its input (the reference's
// local `dummy`).  Here that scratch is the file-scope device array below, of
// EM2G_SMOOTH2_STATIC_MAX_POINTS doubles (4 MiB); every GPU that loads the
// library holds it until the process exits.  All calls on a device share it:
// two calls whose kernels overlap on the GPU race on it, so callers order
// their calls (one stream, or events).  Each call overwrites every scratch
// element it reads before reading it, so no clearing is needed and the
// previous call's leftovers never leak into a result.
//
// In host code `g_smooth2_scratch` names a host-side stand-in, not a device
// address.  The device address comes from cudaGetSymbolAddress, looked up
// again on every call made outside a stream capture (the module, and so the
// array, can move when the caller makes another context current or resets
// the device) and kept per device for calls made during a capture, where
// only the kept address is used.  The first call on a device must therefore
// come before any stream capture begins.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "em2g_internal.cuh"
#include "grid_kernels.cuh"

static __device__ __align__(256) double g_smooth2_scratch[EM2G_SMOOTH2_STATIC_MAX_POINTS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_addr[kMaxDevices] = {nullptr};

// the two passes are the library's own stencils (grid_kernels.cuh), on the
// guarded (nx+3) x (ny+3) array: binomial sm -> scratch, then compensation
// scratch -> sm (pic/smooth.f90:143-146, :163-166)
__global__ void k_binomial_static(em2g::grid::G g, const double *__restrict__ s, double *d) {
  em2g::grid::smooth_binomial_at(g, s, d, (int)blockIdx.x, (int)blockIdx.y);
}
__global__ void k_compensate_static(em2g::grid::G g, const double *__restrict__ d, double *s) {
  em2g::grid::smooth_compensate_at(g, d, s, (int)blockIdx.x, (int)blockIdx.y);
}

}  // namespace

extern "C" int em2g_smooth2_static(int nx, int ny, double *dev_array, void *cuda_stream) {
  using em2g::fail;
  if (nx < 4 || ny < 4) return fail(EM2G_ERR_INVALID, "smooth2_static: nx and ny must be >= 4");
  if (!dev_array) return fail(EM2G_ERR_INVALID, "smooth2_static: null array");
  const int64_t points = (int64_t)(nx + 3) * (ny + 3);
  if (points > EM2G_SMOOTH2_STATIC_MAX_POINTS)
    return fail(EM2G_ERR_RANGE,
                "smooth2_static: (nx+3)*(ny+3) = " + std::to_string(points) +
                    " exceeds the static scratch of " +
                    std::to_string((long long)EM2G_SMOOTH2_STATIC_MAX_POINTS) +
                    " points; use an em2g context and em2g_smooth2");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return em2g::cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(EM2G_ERR_INVALID, "smooth2_static: device ordinal");
  // an error left pending by earlier work of another component is not this
  // call's: report it as such and leave it pending for its owner
  e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(EM2G_ERR_CUDA, std::string("smooth2_static: an earlier CUDA error is pending "
                                           "(not from this call): ") + cudaGetErrorString(e));
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return em2g::cuda_fail(e, "cudaStreamIsCapturing");
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_smooth2_scratch);
      if (e != cudaSuccess) return em2g::cuda_fail(e, "cudaGetSymbolAddress(g_smooth2_scratch)");
      g_scratch_addr[dev] = static_cast<double *>(p);
    } else if (!g_scratch_addr[dev]) {
      return fail(EM2G_ERR_INVALID,
                  "smooth2_static: the first call on a device must come before a stream capture");
    }
    scratch = g_scratch_addr[dev];
  }
  using em2g::grid::TX;
  using em2g::grid::TY;
  const em2g::grid::G g{nx, ny, nx + 3, (int64_t)(nx + 3) * (ny + 3)};
  const dim3 blk(TX, TY), grd((nx + 1 + TX - 1) / TX, (ny + 1 + TY - 1) / TY);
  k_binomial_static<<<grd, blk, 0, st>>>(g, dev_array, scratch);
  k_compensate_static<<<grd, blk, 0, st>>>(g, scratch, dev_array);
  e = cudaGetLastError();
  if (e != cudaSuccess) return em2g::cuda_fail(e, "smooth2_static launch");
  return EM2G_OK;
}

// lgv_noalloc.cu -- measurement entry point that allocates no device memory.
//
// lgv_measure_aos_noalloc() runs the same measurement as lgv_measure_device()
// but for a lattice the caller already holds in device memory (host-order AoS
// layout), without a handle and without any allocation: its scratch space is
// the file-scope array below.  It exists for callers that cannot make device
// allocations of their own while they run: a host whose device memory is owned
// by another allocator (a framework's caching pool that has reserved most of
// the GPU, where an extra cudaMalloc can fail although the pool has room), or
// a process held to a fixed device-memory budget.
//
// Limits and sharing rules:
//  - N <= LGV_NOALLOC_MAX_N (128).  The scratch holds two 25 x N x N partial
//    sum tables: 2 * 25 * 128 * 128 doubles = 6.55 MB, resident on every GPU
//    that loads this library until the process exits.
//  - Every call on a device uses the same array and leaves its partial sums
//    there.  Each call overwrites every element it later reads, so nothing
//    needs clearing between calls; but two calls whose kernels overlap on the
//    GPU (different streams without ordering, or several host threads) race
//    on the array and corrupt each other's results.
//  - Host code cannot use g_scratch's name as a device address: every call
//    made outside stream capture looks the address up with
//    cudaGetSymbolAddress for the current device (so a context made anew,
//    e.g. after cudaDeviceReset, is followed) and records it; a call made
//    while `stream` is being captured uses the address recorded for its
//    device.  So make the first call on each device before any capture
//    begins.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/lgv.h"
#include "lgv_internal.h"

void lgv_internal_set_error(const char *msg);

namespace {

constexpr int kMaxN = LGV_NOALLOC_MAX_N;
constexpr size_t kScratchDoubles = 2ull * 25 * kMaxN * kMaxN;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_scratch[kScratchDoubles];

std::mutex g_mu;
double *g_scratch_addr[kMaxDevices] = {nullptr};

int fail(int code, const char *msg) {
  lgv_internal_set_error(msg);
  return code;
}

}  // namespace

extern "C" int lgv_measure_aos_noalloc(const double *dev_aos, int N, double *dev_out, void *stream) {
  if (!dev_aos || !dev_out) return fail(LGV_ERR_INVALID, "lgv_measure_aos_noalloc: NULL device pointer");
  if (N < 4 || (N & 1)) return fail(LGV_ERR_INVALID, "lgv_measure_aos_noalloc: N must be even and >= 4");
  if (N > kMaxN)
    return fail(LGV_ERR_INVALID,
                "lgv_measure_aos_noalloc: N exceeds LGV_NOALLOC_MAX_N = 128 (static scratch is sized for 128^2 walls)");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(LGV_ERR_CUDA, "lgv_measure_aos_noalloc: no usable current CUDA device");
  cudaStream_t st = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess)
    return fail(LGV_ERR_CUDA, "lgv_measure_aos_noalloc: cudaStreamIsCapturing failed");
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (cap == cudaStreamCaptureStatusNone) {
      // host code may not use g_scratch directly: resolve its address in the current context
      double *p = nullptr;
      if (cudaGetSymbolAddress((void **)&p, g_scratch) != cudaSuccess || !p)
        return fail(LGV_ERR_CUDA, "lgv_measure_aos_noalloc: cudaGetSymbolAddress of the static scratch failed");
      g_scratch_addr[dev] = p;
    } else if (!g_scratch_addr[dev]) {
      return fail(LGV_ERR_STATE,
                  "lgv_measure_aos_noalloc: first call on this device made during stream capture; call it once "
                  "before capturing");
    }
    scratch = g_scratch_addr[dev];
  }
  const size_t table = 25ull * N * N;
  if (lgv::launch_measure_sums_aos(dev_aos, N, scratch, scratch + table, st) != cudaSuccess ||
      lgv::launch_measure_finish(scratch, scratch + table, N, dev_out, st) != cudaSuccess)
    return fail(LGV_ERR_CUDA, "lgv_measure_aos_noalloc: kernel launch failed");
  return LGV_OK;
}

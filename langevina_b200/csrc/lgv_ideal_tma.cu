// lgv_ideal_tma.cu -- the fused ideal step (IdealPV2::step_no_reject,
// Stepper.cxx:68-176) with its tiles staged by the Tensor Memory Accelerator.
//
// A CTA of 256 threads owns a 32 x 8 column of sites and marches up a
// z-chunk, as ideal_kernel does.  What changes is how a plane reaches shared
// memory: the tile's own 256 sites of each of the 10 components are one TMA
// box {16 m, 8 rows, 1 plane, 2 parity halves} of the red-black layout
// (cp.async.bulk.tensor, completion on an mbarrier, issued by one thread),
// and only the 84-site ring around the tile (periodic wrap) still comes by
// per-thread cp.async.  Shared memory keeps the red-black order, and each
// half warp owns the sites of one x-parity, so every shared-memory access of
// a half warp is 16 consecutive doubles.
//
// Used for N divisible by 32 (whole tiles; TMA strides need N/2 even), for a
// single lattice and for those replicas of an ensemble; other sizes use
// ideal_kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>
#include <utility>

#include "lgv_ideal_tma_cta.cuh"
#include "lgv_internal.h"

namespace lgv {

namespace {

using namespace tma;

__global__ void __launch_bounds__(NT, 2)
    ideal_tma_kernel(const __grid_constant__ TmaMaps maps, Fields in, Fields out, Geo g, int zchunk, IdealArgs a) {
  ideal_tma_cta(maps.m, in, out, g, zchunk, a, blockIdx.x, blockIdx.y,
                g.zrev ? (int)(gridDim.z - 1 - blockIdx.z) : (int)blockIdx.z);
}

// Ensembles: the CTAs of every replica with N divisible by 32 in one launch.
__global__ void __launch_bounds__(NT, 2)
    batch_ideal_tma_kernel(const RepDesc *__restrict__ d, const CUtensorMap *__restrict__ gmaps,
                           const int *__restrict__ rep, const int *__restrict__ first, int pphi, int pq, double dt,
                           unsigned long long *waits, int wait_limit) {
  batch_tma_item(d, gmaps, rep, first, blockIdx.x, pphi, pq, dt, waits, wait_limit);
}

// ---------------------------------------------------------------------------
// Tensor maps: one per component plane, 4-D view (m, j, k, half) of the
// red-black layout; cached by (plane address, N).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

bool plane_map(const double *plane, int N, int Nz, CUtensorMap *out) {
  static std::mutex mu;
  static std::map<std::tuple<const double *, int, int>, CUtensorMap> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find({plane, N, Nz});
  if (it != cache.end()) {
    *out = it->second;
    return true;
  }
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t H = (cuuint64_t)(N / 2);
  const cuuint64_t dims[4] = {H, (cuuint64_t)N, (cuuint64_t)Nz, 2};
  const cuuint64_t strides[3] = {H * 8, (cuuint64_t)N * H * 8, (cuuint64_t)N * Nz * H * 8};
  const cuuint32_t box[4] = {HM, TY, 1, 2};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMap m;
  if (fn(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double *>(plane), dims, strides, box, estr,
         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  if (cache.size() > 4096) cache.clear();
  cache.emplace(std::make_tuple(plane, N, Nz), m);
  *out = m;
  return true;
}

}  // namespace

bool ideal_tma_supported(int N) {
  return N >= 32 && N % 32 == 0 && encode_fn() != nullptr;
}

cudaError_t launch_ideal_tma(Fields in, Fields out, const Geo &g, int zchunk, const IdealArgs &a, cudaStream_t st) {
  const int N = g.N;
  if (!ideal_tma_supported(N)) return cudaErrorInvalidValue;
  for (int c = 0; c < 10; ++c)
    if (((uintptr_t)in.c[c] & 15) != 0) return cudaErrorMisalignedAddress;
  TmaMaps maps;
  for (int c = 0; c < 10; ++c)
    if (!plane_map(in.c[c], N, g.Nz, &maps.m[c])) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(ideal_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  if (e != cudaSuccess) return e;
  dim3 grid(N / TX, N / TY, (unsigned)((g.Nz + zchunk - 1) / zchunk));
  ideal_tma_kernel<<<grid, NT, kSmemBytes, st>>>(maps, in, out, g, zchunk, a);
  return cudaGetLastError();
}

int batch_tma_blocks(int N, int zchunk) { return (N / TX) * (N / TY) * ((N + zchunk - 1) / zchunk); }

bool tma_plane_map(const double *plane, int N, void *out128) {
  if (((uintptr_t)plane & 15) != 0) return false;
  return plane_map(plane, N, N, reinterpret_cast<CUtensorMap *>(out128));
}

cudaError_t launch_batch_ideal_tma(const RepDesc *d, const void *gmaps, const int *rep, const int *first, int nblocks,
                                   int phase_phi, int phase_q, double dt, unsigned long long *waits, int wait_limit,
                                   cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(batch_ideal_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmemBytes);
  if (e != cudaSuccess) return e;
  batch_ideal_tma_kernel<<<nblocks, NT, kSmemBytes, st>>>(d, reinterpret_cast<const CUtensorMap *>(gmaps), rep, first,
                                                          phase_phi, phase_q, dt, waits, wait_limit);
  return cudaGetLastError();
}

}  // namespace lgv

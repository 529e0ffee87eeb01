// lgv_ideal_tma_cta.cuh -- the CTA body of the TMA-staged ideal step, shared
// by the ideal kernels of lgv_ideal_tma.cu and the persistent ensemble step of
// lgv_kernels.cu.
//
// A CTA of 256 threads owns a 32 x 8 column of sites and marches up a
// z-chunk.  The tile's own 256 sites of each of the 10 components arrive as
// one TMA box {16 m, 8 rows, 1 plane, 2 parity halves} of the red-black
// layout (cp.async.bulk.tensor, completion on an mbarrier, issued by one
// thread), and only the 84-site ring around the tile (periodic wrap) comes by
// per-thread cp.async.  Shared memory keeps the red-black order, and each
// half warp owns the sites of one x-parity, so every shared-memory access of a
// half warp is 16 consecutive doubles.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "lgv_internal.h"

namespace lgv {
namespace tma {

constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int HM = TX / 2;                    // m per half row of the tile
constexpr int CORE = 2 * TY * HM;             // doubles per component per plane (both halves)
constexpr int NHALO = 2 * (TX + 2) + 2 * TY;  // ring sites
constexpr int PM = HM + 2;                    // m slots per padded phi' half row
constexpr int PR = TY + 2;                    // padded rows
constexpr int PH = 2 * PR * PM;               // doubles per padded phi' component plane
constexpr unsigned kBoxBytes = CORE * 8;
constexpr unsigned kPlaneBytes = 10 * kBoxBytes;
// Two pipeline stages: plane p is consumed while plane p+1 loads.  (A third
// stage, prefetching p+2, measured slower on B200: 0.88 against 0.67 ms per
// 256^3 launch, with more barrier and MIO stalls.)
constexpr int NS = 2;
// dynamic shared memory (doubles): core [NS][10][CORE], ring [NS][10][NHALO], phi' [2][4][PH];
// offsets rounded to 16 doubles (128-byte shared-memory wavefronts)
constexpr size_t round16(size_t n) { return (n + 15) / 16 * 16; }
constexpr size_t kCoreOff = 0, kHaloOff = NS * 10 * CORE, kPhiOff = round16(kHaloOff + NS * 10 * NHALO);
constexpr size_t kSmemBytes = (kPhiOff + 2 * 4 * PH) * sizeof(double) + 128;  // + alignment slack
static_assert(NHALO <= NT, "ring larger than the CTA");
static_assert((kBoxBytes % 128) == 0, "TMA boxes stay 128-byte aligned");

struct TmaMaps {
  CUtensorMap m[10];
};

__device__ __forceinline__ int wrapn(int a, int n) {
  a %= n;
  return a < 0 ? a + n : a;
}

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the phase `parity` of an mbarrier: false (and a count in
// *waits) when it gives up after `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int limit, unsigned long long *waits) {
  for (int i = 0; i < limit; ++i)
    if (mbar_try(bar, parity)) return true;
  if (waits) atomicAdd(waits, 1ull);
  return false;
}

// One thread: the 10 component boxes of plane k into core stage `dst`.
__device__ __forceinline__ void issue_plane(const CUtensorMap *maps, double *dst, unsigned bar, int m0, int j0, int k) {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(kPlaneBytes) : "memory");
#pragma unroll
  for (int c = 0; c < 10; ++c) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(smem_addr(dst + c * CORE)),
        "l"(maps + c), "r"(m0), "r"(j0), "r"(k), "r"(0), "r"(bar)
        : "memory");
  }
}

// One CTA: tile (bx, by) of the xy plane, z-chunk bz.  maps: the tensor maps
// of the 10 component planes of `in` (kernel parameters or global memory).
__device__ __forceinline__ void ideal_tma_cta(const CUtensorMap *maps, const Fields &in, const Fields &out, const Geo &g,
                                              int zchunk, const IdealArgs &a, int bx, int by, int bz) {
  extern __shared__ __align__(128) double smem_raw[];
  __shared__ __align__(8) unsigned long long mbar[NS];
  __shared__ int s_abort;
  // TMA destinations must be 128-byte aligned: align the base explicitly
  double *smem = smem_raw + ((128 - (smem_addr(smem_raw) & 127)) & 127) / sizeof(double);
  double *core = smem + kCoreOff;
  double *halo = smem + kHaloOff;
  double *phs = smem + kPhiOff;
  const int N = g.N;
  const int tid = threadIdx.x;
  const int ty = tid >> 5, hw = (tid >> 4) & 1, t = tid & 15;
  const int lx = 2 * t + hw;  // each half warp owns one x-parity of the row
  const int x0 = bx * TX, y0 = by * TY;
  const int z0 = bz * zchunk;
  const int z1 = min(z0 + zchunk, g.Nz);
  const int nit = (z1 - z0) + 2;
  const int xi = x0 + lx, yj = y0 + ty;
  const unsigned bar0 = smem_addr(&mbar[0]);  // stage s uses bar0 + 8 s

  // ring site of this thread: padded coordinates (hx, hy), global (hxg, hyg)
  int hx = 0, hy = 0, hxg = 0, hyg = 0;
  const bool ring = tid < NHALO;
  if (ring) {
    const int h = tid;
    if (h < TX + 2) { hx = h; hy = 0; }
    else if (h < 2 * (TX + 2)) { hx = h - (TX + 2); hy = PR - 1; }
    else if (h < 2 * (TX + 2) + TY) { hx = 0; hy = 1 + (h - 2 * (TX + 2)); }
    else { hx = TX + 1; hy = 1 + (h - 2 * (TX + 2) - TY); }
    hxg = wrapn(x0 - 1 + hx, N);
    hyg = wrapn(y0 - 1 + hy, N);
  }

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar0 + 8 * s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();
  // Plane q of the march (q = 0 is z0-1, which feeds only the own column's
  // z-1 neighbour and needs no ring) goes to stage q % NS; one cp.async group
  // per plane, possibly empty, so waiting for all groups covers plane q.
  // Planes are tracked incrementally (q covers z0-1 .. z1, within one wrap of
  // the buffer), so the march does no integer division.
  const int zfirst = z0 == 0 ? g.Nz - 1 : z0 - 1;  // plane of q = 0
  const long long NH = (long long)N * g.H;
  const int ring_xy = hyg * g.H + (hxg >> 1);  // in-plane parts of the ring and own sites' offsets
  const int own_xy = yj * g.H + (xi >> 1);
  auto plane_of = [&](int q) {  // zfirst + q wrapped; q < nit <= Nz + 2, so at most two wraps
    int pl = zfirst + q;
    if (pl >= g.Nz) pl -= g.Nz;
    if (pl >= g.Nz) pl -= g.Nz;
    return pl;
  };
  auto issue = [&](int q) {
    const int pl = plane_of(q), sn = q % NS;
    if (tid == 0) issue_plane(maps, core + sn * 10 * CORE, bar0 + 8 * sn, x0 / 2, y0, pl);
    if (ring && q >= 1) {
      const long long oh = (long long)((hxg + hyg + pl) & 1) * g.V2 + (long long)pl * NH + ring_xy;
#pragma unroll
      for (int c = 0; c < 10; ++c) cp_async8(&halo[(sn * 10 + c) * NHALO + tid], in.c[c] + oh);
    }
  };
  for (int q = 0; q < NS - 1; ++q) {  // nit >= 3 >= NS - 1
    issue(q);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }

  double pm[4], pc[4], pn[4], qc[6], qn[6];
  unsigned wbar = bar0, wpar = 0;  // the barrier phase waited on last
  int kk = zfirst;  // plane p - 1 (used from it >= 2)
  for (int it = 0; it < nit; ++it) {
    const int p = plane_of(it);
    const int st = it % NS;
    wbar = bar0 + 8 * st;
    wpar = (unsigned)((it / NS) & 1);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (!mbar_wait(wbar, wpar, a.wait_limit, a.waits)) s_abort = 1;
    __syncthreads();
    if (s_abort) break;
    if (it + NS - 1 < nit) issue(it + NS - 1);  // its stage was last read in iteration it - 1
    asm volatile("cp.async.commit_group;\n" ::: "memory");

    const double *cr = core + st * 10 * CORE;
    double *ph = phs + (it & 1) * 4 * PH;
    // own site of plane p: half, core and padded phi' positions
    const int hp = (hw + y0 + ty + p) & 1;
    const int co = (hp * TY + ty) * HM + t;
    const int po = (hp * PR + ty + 1) * PM + t + 1;
#pragma unroll
    for (int l = 0; l < 4; ++l) pn[l] = cr[l * CORE + co];
#pragma unroll
    for (int s = 0; s < 6; ++s) qn[s] = cr[(4 + s) * CORE + co];
    rotate_site(pn, qn, a.dto2chi);
#pragma unroll
    for (int l = 0; l < 4; ++l) ph[l * PH + po] = pn[l];
    if (ring && it >= 1) {
      const double *hr = halo + st * 10 * NHALO;
      double phh[4], qh[6];
#pragma unroll
      for (int l = 0; l < 4; ++l) phh[l] = hr[l * NHALO + tid];
#pragma unroll
      for (int s = 0; s < 6; ++s) qh[s] = hr[(4 + s) * NHALO + tid];
      rotate_site(phh, qh, a.dto2chi);
      const int lxh = hx - 1, lyh = hy - 1;
      const int hh = (lxh + y0 + lyh + p) & 1;
      const int pho = (hh * PR + hy) * PM + ((lxh + 2) >> 1);
#pragma unroll
      for (int l = 0; l < 4; ++l) ph[l * PH + pho] = phh[l];
    }

    if (it >= 2) {
      // phi' of plane p-1, written last iteration; the barrier at the top of
      // this iteration also ends last iteration's reads of the buffer written now
      const double *pp = phs + ((it + 1) & 1) * 4 * PH;
      const int nh = ((hw + y0 + ty + kk) & 1) ^ 1;  // the neighbours' half
      const int rx = (nh * PR + ty + 1) * PM;
      const int oxp = rx + t + 1 + hw, oxm = rx + t + hw;
      const int oyp = (nh * PR + ty + 2) * PM + t + 1, oym = (nh * PR + ty) * PM + t + 1;
      double xp[4], xm[4], yp[4], ym[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        xp[l] = pp[l * PH + oxp];
        xm[l] = pp[l * PH + oxm];
        yp[l] = pp[l * PH + oyp];
        ym[l] = pp[l * PH + oym];
      }
      const double *c = pc, *zp = pn, *zm = pm;
      double S[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) S[l] = ((xp[l] + xm[l]) + (yp[l] + ym[l])) + (zp[l] + zm[l]);
      charge_currents(c, S, a.dt, a.a2, a.H, qc);
      // second half rotation on a copy: pc (phi') stays the z-1 neighbour of the next plane
      double pf[4] = {pc[0], pc[1], pc[2], pc[3]};
      rotate_site(pf, qc, a.dto2chi);
      const long long o = (long long)((xi + yj + kk) & 1) * g.V2 + (long long)kk * NH + own_xy;
#pragma unroll
      for (int l = 0; l < 4; ++l) out.c[l][o] = pf[l];
#pragma unroll
      for (int s = 0; s < 6; ++s) out.c[4 + s][o] = qc[s];
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      pm[l] = pc[l];
      pc[l] = pn[l];
    }
#pragma unroll
    for (int s = 0; s < 6; ++s) qc[s] = qn[s];
    kk = p;
  }
  if (s_abort) {
    // the plane that timed out may still be in flight: one more bounded wait
    // (the full limit, whatever the first one had) before the CTA retires
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (tid == 0) mbar_wait(wbar, wpar, kWaitLimit, a.waits);
    __syncthreads();
  }
}

// Ensembles: CTA blk of the flat grid of every replica with N divisible by 32,
// through the same CTA body.  Replica r's maps for phi buffer pphi and charge
// buffer pq are gmaps[((r * 2 + pphi) * 2 + pq) * 10 + c]; the host wrote them
// before any launch, and the acquire fence orders those writes before the
// tensor-map proxy reads them.
__device__ __forceinline__ void batch_tma_item(const RepDesc *__restrict__ d, const CUtensorMap *__restrict__ gmaps,
                                               const int *__restrict__ rep, const int *__restrict__ first, int blk,
                                               int pphi, int pq, double dt, unsigned long long *waits,
                                               int wait_limit) {
  const int r = rep[blk];
  const RepDesc &R = d[r];
  const int l = blk - first[r];
  const int ntx = R.g.N / TX, nty = R.g.N / TY;
  const int bx = l % ntx, by = (l / ntx) % nty, bz = l / (ntx * nty);
  const CUtensorMap *maps = gmaps + ((size_t)(r * 2 + pphi) * 2 + pq) * 10;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < 10; ++c)
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(maps + c) : "memory");
  }
  Fields in, out;
#pragma unroll
  for (int L = 0; L < 10; ++L) {
    in.c[L] = R.base[L < 4 ? pphi : pq] + (long long)L * R.pstride;
    out.c[L] = R.base[L < 4 ? (pphi ^ 1) : (pq ^ 1)] + (long long)L * R.pstride;
  }
  IdealArgs a;
  a.dto2chi = (dt / 2.0) / R.chi;
  a.dt = dt;
  a.a2 = R.a2;
  a.H = R.H;
  a.waits = waits;
  a.wait_limit = wait_limit;
  ideal_tma_cta(maps, in, out, R.g, R.izc, a, bx, by, bz);
}

}  // namespace tma
}  // namespace lgv

// lgv_kernels.cu -- sm_100a kernels of the Model A / Model G stepper and
// measurer.  FP64 throughout; HBM-bound stencils, no tensor-core work.
//
// Kernel map (reference loop each one replaces):
//   hb_pass_kernel      EulerLangevinHB::step, one checkerboard parity per
//                       launch (Stepper.cxx:287-389)
//   hb_sweep_kernel     the same, both parities in one z-marching launch (opt-in)
//   charge_pass_kernel  ModelGChargeHB::step, one (direction, parity) face
//                       (Stepper.cxx:471-518, modelg_update_charge_pair :419-441)
//   charge_slab_kernel, both faces of one direction per launch (opt-in):
//   charge_x_kernel,    shared-memory slabs for N divisible by 32, otherwise x
//   charge_line_kernel  rows per CTA and y, z streamed lines with two-site halos
//   ideal_kernel        IdealPV2::step_no_reject fused: half rotation, charge
//                       advection stencil, half rotation (Stepper.cxx:68-202);
//                       the TMA-staged ideal_tma_kernel (lgv_ideal_tma.cu)
//                       replaces it for N divisible by 32
//   em_kernel           Euler-Maruyama Model A step (action of Stepper.cxx:354-355)
//   energy_*            IdealPV2::computeEnergy (Stepper.cxx:204-268)
//   meas_*              Measurer::computeSliceAverage / ...Phase /
//                       computeDerivedObs (measurer.cxx:10-317)
//   batch_*             the same steps for every replica of an ensemble in one
//                       launch (no counterpart: the reference runs one lattice)
//   em_adjoint_kernel, rot_phi_kernel, ideal_adj_a/b_kernel, batch_em_*
//                       adjoints of the Euler-Maruyama and ideal steps for the
//                       differentiable runs (no counterpart)
#include "lgv_ideal_tma_cta.cuh"
#include "lgv_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace lgv {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void warp_sum(double &v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
}
__device__ __forceinline__ void warp_sum(unsigned long long &v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
}

// Sums v[0..3] over the CTA into partial[blockIdx.x][0..3]; the last CTA of
// the grid to finish then adds the CTA partials in block order (fixed, so the
// result does not depend on which CTA ends last), scaled, into out[0..3]
// (accumulating when add) and re-arms the counter.  `done` is zero on entry.
template <int NT>
__device__ __forceinline__ void grid_sum4(double (&v)[4], double *partial, unsigned *done, double *out, double scale,
                                          bool add) {
  static_assert(NT % 32 == 0 && NT >= 128, "grid_sum4: NT");
  constexpr int NW = NT / 32;
  __shared__ double sm[4][NW];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    warp_sum(v[q]);
    if (lane == 0) sm[q][warp] = v[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double t = 0;
#pragma unroll
      for (int w = 0; w < NW; ++w) t += sm[q][w];
      partial[(size_t)blockIdx.x * 4 + q] = t;
    }
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (warp < 4) {
    double t = 0;
    for (unsigned b = lane; b < gridDim.x; b += 32) t += __ldcg(partial + (size_t)b * 4 + warp);
    warp_sum(t);
    if (lane == 0) out[warp] = add ? out[warp] + t * scale : t * scale;
  }
  if (threadIdx.x == 0) *done = 0u;
}

// Flat site-pair index -> (m, j, k) of the red-black half rows: idx = (k N + j) H + m.
// 32-bit unsigned divisions (64-bit ones are emulated); idx < V/2 <= 2^32 for N <= 2048.
__device__ __forceinline__ void pair_coords(long long idx, const Geo &g, int &m, int &j, int &k) {
  const unsigned u = (unsigned)idx, H = (unsigned)g.H, N = (unsigned)g.N;
  const unsigned row = u / H;
  m = (int)(u - row * H);
  k = (int)(row / N);
  j = (int)(row - (unsigned)k * N);
}

// Per-thread monitor tally, reduced per block and added once per block.
struct MonLocal {
  unsigned long long dc = 0, uc = 0, uy = 0, un = 0;
  double dd = 0, ud = 0;
  __device__ __forceinline__ void down(double dS) { dc++; dd += dS; }
  __device__ __forceinline__ void up_yes(double dS) { uc++; uy++; ud += dS; }
  __device__ __forceinline__ void up_no() { uc++; un++; }
};

__device__ void mon_flush(MonLocal &m, MonAcc *acc) {
  __shared__ unsigned long long s_c[4][kThreads / 32];
  __shared__ double s_d[2][kThreads / 32];
  warp_sum(m.dc);
  warp_sum(m.uc);
  warp_sum(m.uy);
  warp_sum(m.un);
  warp_sum(m.dd);
  warp_sum(m.ud);
  // linear thread index: CTAs may be two-dimensional (charge_x_kernel)
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
  const int w = tid >> 5, l = tid & 31;
  if (l == 0) {
    s_c[0][w] = m.dc;
    s_c[1][w] = m.uc;
    s_c[2][w] = m.uy;
    s_c[3][w] = m.un;
    s_d[0][w] = m.dd;
    s_d[1][w] = m.ud;
  }
  __syncthreads();
  if (tid == 0) {
    MonLocal t;
    for (int i = 0; i < nwarps; ++i) {
      t.dc += s_c[0][i];
      t.uc += s_c[1][i];
      t.uy += s_c[2][i];
      t.un += s_c[3][i];
      t.dd += s_d[0][i];
      t.ud += s_d[1][i];
    }
    atomicAdd(&acc->down_counts, t.dc);
    atomicAdd(&acc->up_counts, t.uc);
    atomicAdd(&acc->up_yes, t.uy);
    atomicAdd(&acc->up_no, t.un);
    atomicAdd(&acc->down_dS, t.dd);
    atomicAdd(&acc->up_dS, t.ud);
  }
}

// ----------------------------------------------------------------------------
// Layout conversion: host-order AoS u[k][j][i][10] <-> red-black SoA.
__global__ void aos_to_rb_kernel(const double *__restrict__ aos, Fields f, Geo g) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long V = 2 * g.V2;
  if (n >= V) return;
  const int i = (int)(n % g.N);
  const long long r = n / g.N;
  const int j = (int)(r % g.N), k = (int)(r / g.N);
  const long long o = rb_off(g, i, j, k);
#pragma unroll
  for (int L = 0; L < 10; ++L) f.c[L][o] = aos[n * 10 + L];
}

__global__ void rb_to_aos_kernel(Fields f, double *__restrict__ aos, Geo g) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long V = 2 * g.V2;
  if (n >= V) return;
  const int i = (int)(n % g.N);
  const long long r = n / g.N;
  const int j = (int)(r % g.N), k = (int)(r / g.N);
  const long long o = rb_off(g, i, j, k);
#pragma unroll
  for (int L = 0; L < 10; ++L) aos[n * 10 + L] = f.c[L][o];
}

// ----------------------------------------------------------------------------
// Initial conditions from the counter streams (stream index = natural index).
__global__ void init_phi_kernel(Fields f, Geo g, uint64_t sk, double scale) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= 2 * g.V2) return;
  const int i = (int)(n % g.N);
  const long long r = n / g.N;
  const int j = (int)(r % g.N), k = (int)(r / g.N);
  Xoro x = stream_at(sk, (uint64_t)n);
  double z[4];
  const uint64_t r1 = x.next(), r2 = x.next(), r3 = x.next(), r4 = x.next();
  box_muller(r1, r2, z[0], z[1]);
  box_muller(r3, r4, z[2], z[3]);
  const long long o = rb_off(g, i, j, k);
#pragma unroll
  for (int l = 0; l < 4; ++l) f.c[l][o] = scale * z[l];
}

// ModelA::initialize_gaussian_charges (ModelA.h:463-525): n = sqrt(chi) N(0,1)
// then the zero mode is removed.  Pass 1 draws and writes per-block partial
// sums; pass 2 sums the partials in a fixed order and subtracts the mean.
__global__ void init_charge_kernel(Fields f, Geo g, uint64_t sk, double sqrtchi, double *partial) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double z[6] = {0, 0, 0, 0, 0, 0};
  if (n < 2 * g.V2) {
    const int i = (int)(n % g.N);
    const long long r = n / g.N;
    const int j = (int)(r % g.N), k = (int)(r / g.N);
    Xoro x = stream_at(sk, (uint64_t)n);
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      const uint64_t ra = x.next(), rb = x.next();
      box_muller(ra, rb, z[2 * p], z[2 * p + 1]);
    }
    const long long o = rb_off(g, i, j, k);
#pragma unroll
    for (int L = 0; L < 6; ++L) {
      z[L] *= sqrtchi;
      f.c[4 + L][o] = z[L];
    }
  }
  __shared__ double s[6][kThreads / 32];
#pragma unroll
  for (int L = 0; L < 6; ++L) {
    warp_sum(z[L]);
    if ((threadIdx.x & 31) == 0) s[L][threadIdx.x >> 5] = z[L];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double t = 0;
    for (int w = 0; w < kThreads / 32; ++w) t += s[threadIdx.x][w];
    partial[(long long)blockIdx.x * 6 + threadIdx.x] = t;
  }
}

__global__ void charge_mean_kernel(const double *partial, int nblk, double invV, double *mean) {
  // one warp per component, fixed-order strided sums then a fixed shuffle tree
  const int L = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (L >= 6) return;
  double t = 0;
  for (int b = l; b < nblk; b += 32) t += partial[(long long)b * 6 + L];
  warp_sum(t);
  if (l == 0) mean[L] = t * invV;
}

__global__ void charge_sub_kernel(Fields f, long long V, const double *mean) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= V) return;
#pragma unroll
  for (int L = 0; L < 6; ++L) f.c[4 + L][n] -= mean[L];
}

// ----------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async, one double per copy).
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(double *smem, const double *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ int wrapn(int a, int n) {
  a %= n;
  return a < 0 ? a + n : a;
}

// One heat-bath decision (Stepper.cxx:332-378): proposal phi_n = phi_o +
// sqrt(2 dt Gamma) * variance1, action change dS, Metropolis accept.
struct HbDecision {
  double pn[4];
  double dS;
  bool accept;
  uint8_t flag;
};

// GAUSS (counter noise): the proposals are the four normals of two
// Box-Muller pairs from the site's first four draws (as Euler-Maruyama's
// noise) instead of the reference's U(-sqrt3, sqrt3), Stepper.cxx:343; both
// are symmetric with variance one, so detailed balance and the proposal scale
// are the same.  The accept uniform is the next draw either way.
template <bool INJECTED, bool GAUSS = false>
__device__ __forceinline__ void hb_decide(const double po[4], const double heff[4], const HbArgs &a, long long nat,
                                          long long V, HbDecision &r) {
  Xoro rng;
  if (!INJECTED) rng = stream_at(a.sk, (uint64_t)nat);
  double z[4] = {0., 0., 0., 0.};
  if (!INJECTED && GAUSS) {
    const uint64_t r1 = rng.next(), r2 = rng.next(), r3 = rng.next(), r4 = rng.next();
    box_muller(r1, r2, z[0], z[1]);
    box_muller(r3, r4, z[2], z[3]);
  }
  double hphi_o = 0., hphi_n = 0., s_o = 0., s_n = 0.;
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const double v = INJECTED ? a.prop[(long long)l * V + nat] : (GAUSS ? z[l] : var1(rng.next()));
    r.pn[l] = po[l] + a.rdtg * v;
    s_o += po[l] * po[l];
    s_n += r.pn[l] * r.pn[l];
    hphi_o += heff[l] * po[l];
    hphi_n += heff[l] * r.pn[l];
  }
  hphi_o += a.H * po[0];
  hphi_n += a.H * r.pn[0];
  r.dS = -(hphi_n - hphi_o) + a.Lambda2 * (s_n - s_o) + a.lam4 * (s_n * s_n - s_o * s_o);
  if (r.dS < 0) {
    r.accept = true;
    r.flag = 1;
  } else {
    const double u = INJECTED ? a.acc[nat] : u53(rng.next());
    r.accept = u < exp(-r.dS);
    r.flag = r.accept ? 2 : 0;
  }
}

__device__ __forceinline__ void mon_count(MonLocal &m, const HbDecision &d) {
  if (d.flag == 1) m.down(d.dS);
  else if (d.flag == 2) m.up_yes(d.dS);
  else m.up_no();
}

// ----------------------------------------------------------------------------
// Phi heat bath, one checkerboard parity (EulerLangevinHB::step,
// Stepper.cxx:325-381).  One thread per site of `parity`: element m of the
// parity half-row (j, k); its six neighbours are elements of the other
// parity's half-rows.
// CG: phi is read at L2 (ld.global.cg), never from a possibly stale L1 line;
// the ordered sweep (hb_ordered_kernel) reads sites other CTAs of the same
// launch have just written.
template <bool CG>
__device__ __forceinline__ double ld_phi(const double *p) {
  if (CG) return __ldcg(p);
  return *p;
}

// I: the type of element offsets -- int when the buffer (2 V2 elements) and
// the lattice's global site count fit in 31 bits (idx32), so that every load
// address is one wide multiply-add of a component base; long long otherwise.
__host__ __forceinline__ bool idx32(const Geo &g) {
  return 2 * g.V2 <= 0x7fffffffLL && (long long)g.N * g.N * g.Ng <= 0x7fffffffLL;
}

template <typename I>
__device__ __forceinline__ I nat_index_t(const Geo &g, int i, int j, int k) {
  int kk = k + g.kg;
  if (kk < 0) kk += g.Ng;
  else if (kk >= g.Ng) kk -= g.Ng;
  return ((I)kk * g.N + j) * g.N + i;
}

template <bool INJECTED, bool MON, bool CG = false, typename I = long long, bool GAUSS = false>
__device__ __forceinline__ void hb_site(const Fields &f, const Geo &g, int parity, const HbArgs &a, int m, int j,
                                        int k, MonLocal &mon) {
  const int H = g.H, N = g.N;
  const int s = (parity + j + k) & 1;
  int xm = m - 1 + s, xp = m + s;
  if (xm < 0) xm += H;
  if (xp == H) xp = 0;
  const I ob = (I)(parity ^ 1) * (I)g.V2;
  const I row = ((I)k * N + j) * H;
  const I orow = ob + row;
  const I ojp = ob + ((I)k * N + wrap_inc(j, N)) * H + m;
  const I ojm = ob + ((I)k * N + wrap_dec(j, N)) * H + m;
  const I okp = ob + ((I)wrap_inc(k, g.Nz) * N + j) * H + m;
  const I okm = ob + ((I)wrap_dec(k, g.Nz) * N + j) * H + m;
  const I own = (I)parity * (I)g.V2 + row + m;
  double po[4], heff[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const double *P = f.c[l];
    heff[l] = (ld_phi<CG>(P + (orow + xp)) + ld_phi<CG>(P + (orow + xm))) +
              (ld_phi<CG>(P + ojp) + ld_phi<CG>(P + ojm)) +
              (ld_phi<CG>(P + okp) + ld_phi<CG>(P + okm));
    po[l] = ld_phi<CG>(P + own);
  }
  const long long nat = (long long)nat_index_t<I>(g, 2 * m + s, j, k);
  HbDecision d;
  hb_decide<INJECTED, GAUSS>(po, heff, a, nat, global_sites(g), d);
  if (d.accept) {
#pragma unroll
    for (int l = 0; l < 4; ++l) f.c[l][own] = d.pn[l];
  }
  if (MON) mon_count(mon, d);
  if (a.flags) a.flags[nat] = d.flag;
}

// Site of this thread in a one-parity pass.  ROWS (half rows a multiple of
// 128 long): grid (H/128, N, N), no index arithmetic.  Otherwise grid
// (N*H/128 rounded up, N): the sites of plane k are flat over the x blocks,
// so no lanes idle when a half row is shorter than the block (N < 256).
template <bool ROWS>
__device__ __forceinline__ bool pass_site(const Geo &g, int &m, int &j, int &k) {
  if (ROWS) {
    m = blockIdx.x * 128 + threadIdx.x;
    j = blockIdx.y;
    k = g.zrev ? (int)(gridDim.z - 1 - blockIdx.z) : (int)blockIdx.z;
    return true;
  }
  const unsigned t = blockIdx.x * 128 + threadIdx.x, H = (unsigned)g.H;
  if (t >= (unsigned)g.N * H) return false;
  const unsigned jj = t / H;
  m = (int)(t - jj * H);
  j = (int)jj;
  k = g.zrev ? (int)(gridDim.y - 1 - blockIdx.y) : (int)blockIdx.y;
  return true;
}

__host__ __forceinline__ dim3 pass_grid(const Geo &g, bool rows) {
  return rows ? dim3(g.H / 128, g.N, g.Nz) : dim3((unsigned)(((long long)g.N * g.H + 127) / 128), g.Nz);
}

template <bool INJECTED, bool MON, bool ROWS, typename I, bool GAUSS = false>
__global__ void __launch_bounds__(128) hb_pass_kernel(Fields f, Geo g, int parity, HbArgs a) {
  int m, j, k;
  MonLocal mon;
  if (pass_site<ROWS>(g, m, j, k)) hb_site<INJECTED, MON, false, I, GAUSS>(f, g, parity, a, m, j, k, mon);
  if (MON) mon_flush(mon, a.mon);
}

// ----------------------------------------------------------------------------
// Phi heat bath, one checkerboard parity per launch, z-marching
// (EulerLangevinHB::step, Stepper.cxx:325-381).  A CTA of 32 x ZP_TY threads
// owns elements m0 .. m0+31 of half rows j0 .. j0+ZP_TY-1 and marches up a
// z-chunk.  The other parity's values of each plane are loaded once: the
// thread's own element stays in registers for three planes (its z-1, z and
// z+1 neighbours), and the plane's tile with a one-element ring goes to
// shared memory for the x and y neighbours.  A site therefore costs 8 global
// loads (its own 4 components and the other parity's 4 of the plane above)
// plus the ring's share, against 28 for hb_pass_kernel, and every value of
// the other parity crosses L2 about once.  Decisions, streams and results are
// those of hb_site.
constexpr int ZP_TM = 32, ZP_TY = 8, ZP_NT = ZP_TM * ZP_TY;
constexpr int ZP_W = ZP_TM + 2, ZP_R = ZP_TY + 2, ZP_PL = ZP_W * ZP_R;  // padded tile of one component
constexpr int ZP_RING = 2 * ZP_TM + 2 * ZP_TY;

template <bool INJECTED, bool MON>
__global__ void __launch_bounds__(ZP_NT) hb_zpass_kernel(Fields f, Geo g, int parity, int zchunk, HbArgs a) {
  __shared__ double tile[2][4][ZP_PL];
  const int N = g.N, H = g.H;
  const int tm = threadIdx.x, ty = threadIdx.y, tid = ty * ZP_TM + tm;
  const int m0 = blockIdx.x * ZP_TM, j0 = blockIdx.y * ZP_TY;
  const int k0 = blockIdx.z * zchunk, k1 = min(k0 + zchunk, N);
  const int tme = min(ZP_TM, H - m0), tye = min(ZP_TY, N - j0);  // valid extent of this tile
  const bool own = tm < tme && ty < tye;
  const int m = m0 + tm, j = j0 + ty;
  const long long ob = (long long)(parity ^ 1) * g.V2, pb = (long long)parity * g.V2;
  // ring element of this thread (tid < ZP_RING): padded position (rx, ry) and half-row element (rm, rj)
  // rows above and below the tile (tme elements each), then the columns left
  // and right of it (tye rows each); corners are not needed
  int rx = 0, ry = 0, rm = 0, rj = 0;
  bool ring_live = false;
  if (tid < ZP_TM) {
    rx = 1 + tid, ry = 0, ring_live = tid < tme;
  } else if (tid < 2 * ZP_TM) {
    rx = 1 + tid - ZP_TM, ry = tye + 1, ring_live = tid - ZP_TM < tme;
  } else if (tid < 2 * ZP_TM + ZP_TY) {
    rx = 0, ry = 1 + tid - 2 * ZP_TM, ring_live = tid - 2 * ZP_TM < tye;
  } else if (tid < ZP_RING) {
    rx = tme + 1, ry = 1 + tid - 2 * ZP_TM - ZP_TY, ring_live = tid - 2 * ZP_TM - ZP_TY < tye;
  }
  if (ring_live) {
    rm = m0 + rx - 1;
    rj = j0 + ry - 1;
    rm = rm < 0 ? rm + H : (rm >= H ? rm - H : rm);
    rj = rj < 0 ? rj + N : (rj >= N ? rj - N : rj);
  }
  // the other parity's values of plane kk: own element -> o[], ring element -> smem
  auto load_other = [&](int kk, double (&o)[4], int buf) {
    const int kw = kk < 0 ? kk + N : (kk >= N ? kk - N : kk);
    if (own) {
      const long long off = ob + ((long long)kw * N + j) * H + m;
#pragma unroll
      for (int l = 0; l < 4; ++l) o[l] = f.c[l][off];
    }
    if (ring_live) {
      const long long off = ob + ((long long)kw * N + rj) * H + rm;
#pragma unroll
      for (int l = 0; l < 4; ++l) tile[buf][l][ry * ZP_W + rx] = f.c[l][off];
    }
  };
  double oz[4] = {0, 0, 0, 0}, oc[4] = {0, 0, 0, 0}, on[4] = {0, 0, 0, 0};
  load_other(k0 - 1, oz, 0);  // only the own element is used (z-1 neighbour); the ring is overwritten below
  load_other(k0, oc, 0);
  if (own) {
#pragma unroll
    for (int l = 0; l < 4; ++l) tile[0][l][(ty + 1) * ZP_W + tm + 1] = oc[l];
  }
  __syncthreads();
  MonLocal mon;
  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    load_other(k + 1, on, b ^ 1);
    if (own) {
      const int s = (parity + j + k) & 1;
      const double *T = &tile[b][0][0];
      const int c = (ty + 1) * ZP_W + tm + 1;
      const long long offp = pb + ((long long)k * N + j) * H + m;
      double po[4], heff[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const double *Tl = T + l * ZP_PL;
        // x neighbours: elements m-1+s and m+s of the other parity's row
        heff[l] = (Tl[c + s] + Tl[c - 1 + s]) + (Tl[c + ZP_W] + Tl[c - ZP_W]) + (on[l] + oz[l]);
        po[l] = f.c[l][offp];
      }
      const long long nat = ((long long)k * N + j) * N + 2 * m + s;
      HbDecision d;
      hb_decide<INJECTED>(po, heff, a, nat, 2 * g.V2, d);
      if (d.accept) {
#pragma unroll
        for (int l = 0; l < 4; ++l) f.c[l][offp] = d.pn[l];
      }
      if (MON) mon_count(mon, d);
      if (a.flags) a.flags[nat] = d.flag;
#pragma unroll
      for (int l = 0; l < 4; ++l) tile[b ^ 1][l][c] = on[l];
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      oz[l] = oc[l];
      oc[l] = on[l];
    }
    __syncthreads();
  }
  if (MON) mon_flush(mon, a.mon);
}

// ----------------------------------------------------------------------------
// Phi heat bath, one or more whole sweeps (EulerLangevinHB::step,
// Stepper.cxx:287-389) in one persistent launch, ordered through the lattice
// by z-slabs so that the odd pass of a slab runs while its phi is still in
// L2.
//
// The lattice is cut into nslab slabs of S planes.  An item is one parity
// pass (phase p: sweep p/2, parity p&1) over one slab; it is split into cpi
// chunks of `spc` sites (sites of that parity in slab-local (k, j, m) order).
// A host-built schedule lists every chunk of every item in an order in which
// item (p, s) comes after the three items (p-1, s-1), (p-1, s), (p-1, s+1)
// (periodic in s) it depends on: the pass of phase p reads the sites of the
// other parity in planes sS-1 .. (s+1)S, which those items write, and writes
// sites those items read.  CTAs draw chunks in schedule order from an atomic
// ticket; a chunk of phase p >= 1 first waits until its three items have
// completed all their chunks.  Chunks are only ever handed to running CTAs
// and a chunk waits only on chunks with lower tickets, so the waits always
// end; each is still bounded, and a wait that gives up counts in
// sync[kSyncTimeouts], skips its sites and lets the host report
// LGV_ERR_TIMEOUT.  The result is that of the sequential passes bit for bit:
// every site sees exactly the neighbour values it sees there.
//
// phi moves 32 B/site in and 32 B/site out per sweep when the odd pass of a
// slab re-reads it from L2 (the two one-parity launches move 48 B/site each).
constexpr int kSyncTicket = 0, kSyncExit = 1, kSyncTimeouts = 2, kSyncDone = 3;
constexpr int kHbOrderedThreads = 128;

struct HbSched {
  const int *sched;            // ticket -> item * cpi + chunk, item = phase * nslab + slab
  unsigned long long *sync;    // [ticket, exits, timeouts, done[nphase * nslab]]
  int total;                   // tickets
  int cpi;                     // chunks per item
  int spc;                     // sites per chunk (a multiple of kHbOrderedThreads)
  int nslab, S, nphase;
  int limit;                   // polls before a dependency wait gives up
  uint64_t sk[4];              // counter keys of the sweeps (phase / 2)
};

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Thread 0 waits until the three items item (p, s) depends on have completed
// all their chunks; false (and a count in sync[kSyncTimeouts]) if a wait gives
// up.  `seen` caches the last two items already found ready.
__device__ __forceinline__ bool hb_deps_ready(const HbSched &s, int item, int (&seen)[2]) {
  const int phase = item / s.nslab, slab = item - phase * s.nslab;
  if (phase == 0 || item == seen[0] || item == seen[1]) return true;
  for (int d = -1; d <= 1; ++d) {
    const int dep = (phase - 1) * s.nslab + (slab + d + s.nslab) % s.nslab;
    const unsigned long long *p = &s.sync[kSyncDone + dep];
    int it = 0;
    while (ld_acquire(p) < (unsigned long long)s.cpi) {
      if (++it > s.limit) {
        atomicAdd(&s.sync[kSyncTimeouts], 1ull);
        return false;
      }
      __nanosleep(64);
    }
  }
  seen[1] = seen[0];
  seen[0] = item;
  return true;
}

template <bool INJECTED, bool MON>
__global__ void __launch_bounds__(kHbOrderedThreads) hb_ordered_kernel(Fields f, Geo g, HbArgs a, HbSched s) {
  __shared__ int s_work, s_ok;
  MonLocal mon;
  const long long item_sites = (long long)s.S * g.N * g.H;
  // Thread 0 draws the next ticket while the CTA works on the current chunk.
  // A CTA then holds at most two tickets, and each waits only on lower ones,
  // so the lowest unfinished chunk can always proceed.
  unsigned long long next = 0;
  int seen[2] = {-1, -1};
  if (threadIdx.x == 0) next = atomicAdd(&s.sync[kSyncTicket], 1ull);
  for (;;) {
    if (threadIdx.x == 0) {
      const int w = next < (unsigned long long)s.total ? __ldg(s.sched + next) : -1;
      s_ok = w >= 0 ? (int)hb_deps_ready(s, w / s.cpi, seen) : 1;
      s_work = w;
    }
    __syncthreads();
    const int w = s_work, ok = s_ok;
    if (w < 0) break;
    if (threadIdx.x == 0) next = atomicAdd(&s.sync[kSyncTicket], 1ull);
    const int item = w / s.cpi, chunk = w - item * s.cpi;
    const int phase = item / s.nslab, slab = item - phase * s.nslab;
    if (ok) {
      HbArgs aa = a;
      if (!INJECTED) {
        const int q = phase >> 1;  // constant indices: the key array stays in kernel parameters
        aa.sk = q == 0 ? s.sk[0] : q == 1 ? s.sk[1] : q == 2 ? s.sk[2] : s.sk[3];
      }
      const int parity = phase & 1;
      for (int r = threadIdx.x; r < s.spc; r += kHbOrderedThreads) {
        const long long q = (long long)chunk * s.spc + r;
        if (q >= item_sites) break;
        const unsigned u = (unsigned)q, H = (unsigned)g.H, N = (unsigned)g.N;
        const unsigned row = u / H;
        const int m = (int)(u - row * H);
        const unsigned kk = row / N;
        const int j = (int)(row - kk * N);
        hb_site<INJECTED, MON, true>(f, g, parity, aa, m, j, slab * s.S + (int)kk, mon);
      }
    }
    // The barrier orders every thread's stores before thread 0's fence, and
    // the fence (cumulative) before the completion count.
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&s.sync[kSyncDone + item], 1ull);
    }
  }
  if (MON) mon_flush(mon, a.mon);
  // The last CTA out clears the ticket, exit and completion counters for the
  // next launch (the timeout count stays for the host to read).
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&s.sync[kSyncExit], 1ull) == gridDim.x - 1) {
      s.sync[kSyncTicket] = 0;
      s.sync[kSyncExit] = 0;
      for (int i = 0; i < s.nphase * s.nslab; ++i) s.sync[kSyncDone + i] = 0;
    }
  }
}

// ----------------------------------------------------------------------------
// Phi heat bath, one full checkerboard sweep (EulerLangevinHB::step,
// Stepper.cxx:287-389) in a single launch.  A CTA owns HB_TM x HB_TY
// pair-columns -- element m of both parity half-rows of row j, i.e. natural
// x = 2m and 2m+1 -- and marches up a z-chunk.  At plane p it
//   (1) runs the even pass on plane p over its tile plus a one-element ring,
//       from the old odd values of planes p-1, p, p+1 kept in shared memory
//       over a two-element ring;
//   (2) runs the odd pass on plane p-1 over its tile from the new even values
//       of planes p-2, p-1, p, and writes both parities of plane p-1.
// The ring's even updates are recomputed by the neighbouring CTAs bit for bit
// (same inputs, same counter stream), so no CTA waits for another.  phi is
// read once and written once (to `out`): 64 B per site per sweep.  cp.async
// brings plane p+2 (odd) and p+1 (even) in while plane p computes.
constexpr int HB_TM = 32, HB_TY = 8;
constexpr int HB_OW = HB_TM + 4, HB_OH = HB_TY + 4, HB_OP = HB_OW * HB_OH;  // old odd: two-element ring
constexpr int HB_EW = HB_TM + 2, HB_EH = HB_TY + 2, HB_EP = HB_EW * HB_EH;  // even: one-element ring
constexpr size_t HB_SMEM = (size_t)(4 * 4 * HB_OP + 2 * 4 * HB_EP + 3 * 4 * HB_EP) * sizeof(double);

template <bool INJECTED, bool MON>
__global__ void __launch_bounds__(HB_TM *HB_TY, 2) hb_sweep_kernel(Fields in, Fields out, Geo g, int zchunk, HbArgs a) {
  extern __shared__ double smem[];
  double *oo = smem;                     // [4 stages][4][HB_OP] old odd
  double *oe = oo + 4 * 4 * HB_OP;       // [2 stages][4][HB_EP] old even
  double *ne = oe + 2 * 4 * HB_EP;       // [3 stages][4][HB_EP] new even
  const int N = g.N, H = g.H;
  const long long V2 = g.V2, V = 2 * V2;
  const int tid = threadIdx.x;
  const int tm = tid % HB_TM, tj = tid / HB_TM;
  const int m0 = blockIdx.x * HB_TM, j0 = blockIdx.y * HB_TY;
  const int z0 = blockIdx.z * zchunk;
  const int z1 = min(z0 + zchunk, N);
  const int nit = (z1 - z0) + 2;
  MonLocal mon;

  auto issue_odd = [&](int plane, int stage) {
    for (int idx = tid; idx < HB_OP; idx += HB_TM * HB_TY) {
      const int qm = idx % HB_OW, qj = idx / HB_OW;
      const int m = wrapn(m0 - 2 + qm, H), j = wrapn(j0 - 2 + qj, N);
      const long long off = V2 + ((long long)plane * N + j) * H + m;
#pragma unroll
      for (int l = 0; l < 4; ++l) cp_async8(&oo[(stage * 4 + l) * HB_OP + idx], in.c[l] + off);
    }
  };
  auto issue_even = [&](int plane, int stage) {
    for (int idx = tid; idx < HB_EP; idx += HB_TM * HB_TY) {
      const int qm = idx % HB_EW, qj = idx / HB_EW;
      const int m = wrapn(m0 - 1 + qm, H), j = wrapn(j0 - 1 + qj, N);
      const long long off = ((long long)plane * N + j) * H + m;
#pragma unroll
      for (int l = 0; l < 4; ++l) cp_async8(&oe[(stage * 4 + l) * HB_EP + idx], in.c[l] + off);
    }
  };

  issue_odd(wrapn(z0 - 2, N), 0);
  issue_odd(wrapn(z0 - 1, N), 1);
  issue_odd(z0, 2);
  issue_even(wrapn(z0 - 1, N), 0);
  cp_async_commit();

  for (int it = 0; it < nit; ++it) {
    const int p = wrapn(z0 - 1 + it, N);
    cp_async_wait_all();
    __syncthreads();
    if (it + 1 < nit) {
      issue_odd(wrapn(p + 2, N), (it + 3) & 3);
      issue_even(wrapn(p + 1, N), (it + 1) & 1);
    }
    cp_async_commit();

    // (1) even pass on plane p over the tile and its one-element ring
    const double *oom = oo + ((it & 3) * 4) * HB_OP;        // plane p-1
    const double *ooc = oo + (((it + 1) & 3) * 4) * HB_OP;  // plane p
    const double *oop = oo + (((it + 2) & 3) * 4) * HB_OP;  // plane p+1
    const double *oec = oe + ((it & 1) * 4) * HB_EP;
    double *nec = ne + ((it % 3) * 4) * HB_EP;
    const bool in_chunk_e = (it >= 1) && (it <= nit - 2);
    for (int e = tid; e < HB_EP; e += HB_TM * HB_TY) {
      const int qm = e % HB_EW, qj = e / HB_EW;
      const int mr = m0 - 1 + qm, jr = j0 - 1 + qj;
      const int m = wrapn(mr, H), j = wrapn(jr, N);
      const int s0 = (j + p) & 1;
      const int oc = (qj + 1) * HB_OW + (qm + 1);
      double po[4], heff[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const double *C = ooc + l * HB_OP;
        heff[l] = (C[oc + s0] + C[oc - 1 + s0]) + (C[oc + HB_OW] + C[oc - HB_OW]) +
                  (oop[l * HB_OP + oc] + oom[l * HB_OP + oc]);
        po[l] = oec[l * HB_EP + e];
      }
      const long long nat = ((long long)p * N + j) * N + 2 * m + s0;
      HbDecision d;
      hb_decide<INJECTED>(po, heff, a, nat, V, d);
#pragma unroll
      for (int l = 0; l < 4; ++l) nec[l * HB_EP + e] = d.accept ? d.pn[l] : po[l];
      const bool own = in_chunk_e && qm >= 1 && qm <= HB_TM && qj >= 1 && qj <= HB_TY && mr < H && jr < N;
      if (own) {
        if (MON) mon_count(mon, d);
        if (a.flags) a.flags[nat] = d.flag;
      }
    }
    __syncthreads();

    // (2) odd pass on plane q = p-1 over the tile; write both parities of q
    if (it >= 2) {
      const int q = wrapn(p - 1, N);
      const int mr = m0 + tm, jr = j0 + tj;
      const bool act = mr < H && jr < N;
      const int m = wrapn(mr, H), j = wrapn(jr, N);
      const int s1 = (1 + j + q) & 1;
      const int ec = (tj + 1) * HB_EW + (tm + 1);
      const double *nem = ne + (((it + 1) % 3) * 4) * HB_EP;  // plane p-2
      const double *neq = ne + (((it + 2) % 3) * 4) * HB_EP;  // plane p-1
      const double *oq = oom;                                  // old odd of plane p-1
      const int oc = (tj + 2) * HB_OW + (tm + 2);
      double po[4], heff[4], ev[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const double *C = neq + l * HB_EP;
        heff[l] = (C[ec + s1] + C[ec - 1 + s1]) + (C[ec + HB_EW] + C[ec - HB_EW]) +
                  (nec[l * HB_EP + ec] + nem[l * HB_EP + ec]);
        po[l] = oq[l * HB_OP + oc];
        ev[l] = C[ec];
      }
      const long long nat = ((long long)q * N + j) * N + 2 * m + s1;
      HbDecision d;
      hb_decide<INJECTED>(po, heff, a, nat, V, d);
      if (act) {
        const long long row = ((long long)q * N + j) * H + m;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          out.c[l][row] = ev[l];
          out.c[l][V2 + row] = d.accept ? d.pn[l] : po[l];
        }
        if (MON) mon_count(mon, d);
        if (a.flags) a.flags[nat] = d.flag;
      }
    }
  }
  if (MON) mon_flush(mon, a.mon);
}

// ----------------------------------------------------------------------------
// Charge heat bath, one face (direction `dir`, A-site parity eoA).  One thread
// per link (A, B = A + e_dir); the links of a face are disjoint, so the update
// is race free and conserves each charge exactly (Stepper.cxx:493-517).
template <bool INJECTED, bool MON, typename I = long long>
__device__ __forceinline__ void charge_link_site(const Fields &f, const Geo &g, int dir, int eoA, const ChargeArgs &a,
                                                 int m, int j, int k, MonLocal &mon) {
  const int H = g.H, N = g.N;
  const int s = (eoA + j + k) & 1;
  const int i = 2 * m + s;
  const I offA = (I)eoA * (I)g.V2 + ((I)k * N + j) * H + m;
  I offB;
  const I ob = (I)(eoA ^ 1) * (I)g.V2;
  if (dir == 0) {
    int mb = m + s;
    if (mb == H) mb = 0;
    offB = ob + ((I)k * N + j) * H + mb;
  } else if (dir == 1) {
    offB = ob + ((I)k * N + wrap_inc(j, N)) * H + m;
  } else {
    offB = ob + ((I)wrap_inc(k, g.Nz) * N + j) * H + m;
  }
  const long long nat = (long long)nat_index_t<I>(g, i, j, k);
  const long long V = global_sites(g);
  WordStream ws{};
  if (!INJECTED) ws = words_at(a.sk, 6 * (uint64_t)nat);
#pragma unroll
  for (int L = 0; L < 6; ++L) {
    double *P = f.c[4 + L];
    const double nA = P[offA], nB = P[offB];
    const long long ii = (long long)(a.pass * 6 + L) * V + nat;
    uint64_t ra = 0;
    double v;
    if (INJECTED) {
      v = a.q[ii];
    } else {
      ra = ws.next();
      v = v32(lo32(ra));
    }
    const double q = a.rms * v;
    const double dA = nA - q, dB = nB + q;
    const double dS = (dA * dA + dB * dB - nA * nA - nB * nB) * a.inv2chi;
    bool accept;
    uint8_t fl;
    if (dS < 0) {
      accept = true;
      fl = 1;
      if (MON) mon.down(dS);
    } else {
      const double r = INJECTED ? a.acc[ii] : u32(hi32(ra));
      accept = r < exp(-dS);
      fl = accept ? 2 : 0;
      if (MON) {
        if (accept) mon.up_yes(dS);
        else mon.up_no();
      }
    }
    if (accept) {
      P[offA] = nA + (-q);
      P[offB] = nB + q;
    }
    if (a.flags) a.flags[ii] = fl;
  }
}

// Grid as hb_pass_kernel (pass_site).
// 16 blocks of 128 threads per SM (32 registers): the link updates are long
// integer / FP64 chains, and full occupancy hides them best
template <bool INJECTED, bool MON, bool ROWS, typename I>
__global__ void __launch_bounds__(128, 16) charge_pass_kernel(Fields f, Geo g, int dir, int eoA, ChargeArgs a) {
  int m, j, k;
  MonLocal mon;
  if (pass_site<ROWS>(g, m, j, k)) charge_link_site<INJECTED, MON, I>(f, g, dir, eoA, a, m, j, k, mon);
  if (MON) mon_flush(mon, a.mon);
}

// ----------------------------------------------------------------------------
// Charge heat bath, both parity passes of one direction in one launch
// (ModelGChargeHB::step, Stepper.cxx:471-518): the two faces (dir, eo[0]) and
// (dir, eo[1]) are applied in that order.  Every link update is
// modelg_update_charge_pair (:419-441) for the six charges at once, drawing
// from the counter stream of its pass keyed by the link's A site.
struct ChargeDirArgs {
  double rms, inv2chi;
  uint64_t sk[2];
  int pass[2];  // positions of the two faces in the step (injected indexing / flags)
  int eo[2];
  const double *q, *acc;
  uint8_t *flags;
  MonAcc *mon;
};

template <bool INJECTED, bool MON>
__device__ __forceinline__ void charge_link(double nA[6], double nB[6], const ChargeDirArgs &a, int pi,
                                            long long natA, long long V, bool own, MonLocal &mon) {
  WordStream ws{};
  if (!INJECTED) ws = words_at(a.sk[pi], 6 * (uint64_t)natA);
#pragma unroll
  for (int L = 0; L < 6; ++L) {
    const long long ii = (long long)(a.pass[pi] * 6 + L) * V + natA;
    uint64_t ra = 0;
    double v;
    if (INJECTED) {
      v = a.q[ii];
    } else {
      ra = ws.next();
      v = v32(lo32(ra));
    }
    const double q = a.rms * v;
    const double dA = nA[L] - q, dB = nB[L] + q;
    const double dS = (dA * dA + dB * dB - nA[L] * nA[L] - nB[L] * nB[L]) * a.inv2chi;
    bool accept;
    uint8_t fl;
    if (dS < 0) {
      accept = true;
      fl = 1;
    } else {
      const double r = INJECTED ? a.acc[ii] : u32(hi32(ra));
      accept = r < exp(-dS);
      fl = accept ? 2 : 0;
    }
    if (own) {
      if (MON) {
        if (fl == 1) mon.down(dS);
        else if (fl == 2) mon.up_yes(dS);
        else mon.up_no();
      }
      if (a.flags) a.flags[ii] = fl;
    }
    if (accept) {
      nA[L] = nA[L] + (-q);
      nB[L] = nB[L] + q;
    }
  }
}

// x direction.  A CTA owns whole rows (blockDim.x = N/2, blockDim.y rows);
// thread m holds natural sites 2m and 2m+1 of its row (element m of both
// parity half-rows).  Of the two x faces one pairs (2m, 2m+1) inside the
// thread, the other pairs (2m+1, 2m+2) across threads: its A-site owner
// computes it and hands the B site's new charges over through shared memory.
template <bool INJECTED, bool MON>
__global__ void __launch_bounds__(256) charge_x_kernel(Fields f, Geo g, ChargeDirArgs a) {
  extern __shared__ double xs[];  // [6][blockDim.y][H]
  const int H = g.H, N = g.N;
  const int m = threadIdx.x, ty = threadIdx.y;
  const long long R = (long long)blockIdx.x * blockDim.y + ty;
  const bool valid = R < (long long)N * N;
  const int j = valid ? (int)(R % N) : 0, k = valid ? (int)(R / N) : 0;
  const int r = (j + k) & 1;  // parity of site 2m
  const long long row = ((long long)k * N + j) * H;
  const long long V = 2 * g.V2;
  const long long offa = (long long)r * g.V2 + row + m, offb = (long long)(r ^ 1) * g.V2 + row + m;
  double va[6], vb[6];
  MonLocal mon;
  if (valid) {
#pragma unroll
    for (int L = 0; L < 6; ++L) {
      va[L] = f.c[4 + L][offa];
      vb[L] = f.c[4 + L][offb];
    }
  }
  double *sh = xs + (size_t)ty * H;
  const size_t lstride = (size_t)blockDim.y * H;
  const long long nat0 = ((long long)k * N + j) * N + 2 * m;
  // Rows of a CTA differ in parity, so some take the in-thread face while
  // others take the cross face: every thread runs the exchange barriers of
  // both faces, and only the work between them is conditional.
  const int mr = (m + 1 == H) ? 0 : m + 1;
#pragma unroll
  for (int pi = 0; pi < 2; ++pi) {
    const bool cross = a.eo[pi] != r;
    if (valid && !cross) charge_link<INJECTED, MON>(va, vb, a, pi, nat0, V, true, mon);
    // cross link (2m+1, 2m+2): B is thread m+1's site 2m+2
    if (valid && cross) {
#pragma unroll
      for (int L = 0; L < 6; ++L) sh[L * lstride + m] = va[L];
    }
    __syncthreads();
    double nb[6];
    if (valid && cross) {
#pragma unroll
      for (int L = 0; L < 6; ++L) nb[L] = sh[L * lstride + mr];
      charge_link<INJECTED, MON>(vb, nb, a, pi, nat0 + 1, V, true, mon);
    }
    __syncthreads();
    if (valid && cross) {
#pragma unroll
      for (int L = 0; L < 6; ++L) sh[L * lstride + mr] = nb[L];
    }
    __syncthreads();
    if (valid && cross) {
#pragma unroll
      for (int L = 0; L < 6; ++L) va[L] = sh[L * lstride + m];
    }
    __syncthreads();
  }
  if (valid) {
#pragma unroll
    for (int L = 0; L < 6; ++L) {
      f.c[4 + L][offa] = va[L];
      f.c[4 + L][offb] = vb[L];
    }
  }
  if (MON) mon_flush(mon, a.mon);
}

// y (DIR = 1) and z (DIR = 2) directions.  A thread owns element m of the
// parity half-rows along one line (natural columns x = 2m and 2m+1) and
// streams through a segment [s0, s1) of the line plus two sites either side.
// Along a column the two faces alternate link by link, so as site t arrives
// the first face's link (t-1, t) and then the second face's link (t-2, t-1)
// are applied (three-site register window); a site is final after its second
// face link.  Links in the halo are recomputed bit for bit by the thread that
// owns them, so segments are independent; because halos are read while
// neighbours write, the kernel reads `in` and writes `out`.
template <int DIR, bool INJECTED, bool MON>
__global__ void __launch_bounds__(128) charge_line_kernel(Fields in, Fields out, Geo g, ChargeDirArgs a, int seglen) {
  const int H = g.H, N = g.N;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int c2 = blockIdx.y;  // k for DIR = 1, j for DIR = 2
  const int s0 = blockIdx.z * seglen;
  const int s1 = min(s0 + seglen, N);
  const long long V = 2 * g.V2;
  MonLocal mon;
  if (m < H) {
    double w0[2][6], w1[2][6], w2[2][6];  // sites t-2, t-1, t; [column a (x=2m) / b (x=2m+1)][charge]
    const int e1 = a.eo[0], e2 = a.eo[1];
    const int n = (s1 - s0) + 4;
    int tm1 = 0, jm1 = 0, km1 = 0, tm2 = 0, jm2 = 0, km2 = 0;
    for (int u = 0; u < n; ++u) {
      const int t = s0 - 2 + u;  // line position (unwrapped)
      const int tw = wrapn(t, N);
      const int j = DIR == 1 ? tw : c2, k = DIR == 1 ? c2 : tw;
      const int ra = (j + k) & 1;  // parity of column a's site at t
      const long long row = ((long long)k * N + j) * H + m;
#pragma unroll
      for (int L = 0; L < 6; ++L) {
        w2[0][L] = in.c[4 + L][(long long)ra * g.V2 + row];
        w2[1][L] = in.c[4 + L][(long long)(ra ^ 1) * g.V2 + row];
      }
      if (u >= 1) {
        const int rpa = (jm1 + km1) & 1;  // parity of column a at t-1
#pragma unroll
        for (int col = 0; col < 2; ++col) {
          const int par = rpa ^ col;  // parity of this column's site at t-1
          if (par == e1) {  // first face: link (t-1, t), A = t-1
            const long long natA = ((long long)km1 * N + jm1) * N + 2 * m + col;
            charge_link<INJECTED, MON>(w1[col], w2[col], a, 0, natA, V, (t - 1) >= s0 && (t - 1) < s1, mon);
          }
          if (u >= 3 && (par ^ 1) == e2) {  // second face: link (t-2, t-1), A = t-2
            const long long natA = ((long long)km2 * N + jm2) * N + 2 * m + col;
            charge_link<INJECTED, MON>(w0[col], w1[col], a, 1, natA, V, (t - 2) >= s0 && (t - 2) < s1, mon);
            // sites t-2 and t-1 of this column are final
            if ((t - 2) >= s0 && (t - 2) < s1) {
              const long long o2 = (long long)(((jm2 + km2) & 1) ^ col) * g.V2 + ((long long)km2 * N + jm2) * H + m;
#pragma unroll
              for (int L = 0; L < 6; ++L) out.c[4 + L][o2] = w0[col][L];
            }
            if ((t - 1) >= s0 && (t - 1) < s1) {
              const long long o1 = (long long)(rpa ^ col) * g.V2 + ((long long)km1 * N + jm1) * H + m;
#pragma unroll
              for (int L = 0; L < 6; ++L) out.c[4 + L][o1] = w1[col][L];
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int L = 0; L < 6; ++L) {
          w0[c][L] = w1[c][L];
          w1[c][L] = w2[c][L];
        }
      tm2 = tm1; jm2 = jm1; km2 = km1;
      tm1 = tw; jm1 = j; km1 = k;
    }
    (void)tm2;
  }
  if (MON) mon_flush(mon, a.mon);
}

// ----------------------------------------------------------------------------
// Both faces of one charge direction per launch, staged in shared memory.
// The CTA copies its slab of the six charge planes to shared memory with
// coalesced half-row loads, applies every link of the first face, then every
// link of the second, and writes the slab back: the two faces cost one read
// and one write of the charges instead of two of each.
//   x (DIR 0): the slab is `nrows` whole rows (no halo: x links stay in a row).
//   y, z (DIR 1, 2): 32 natural columns (16 elements of each parity half-row)
//   along a segment [s0, s1) of the line at fixed k (y) or j (z), plus two
//   sites either side; halo links are recomputed bit for bit, only links whose
//   A site lies in the segment count in monitors and flags, and only segment
//   sites are written, so the kernel reads `in` and writes `out`.
// Links are the same charge_link updates, streams and order as the per-face
// kernels (Stepper.cxx:471-518).
constexpr int kSlabThreads = 256;

template <int DIR, bool INJECTED, bool MON>
__global__ void __launch_bounds__(kSlabThreads) charge_slab_kernel(Fields in, Fields out, Geo g, ChargeDirArgs a,
                                                                   int seglen, int nrows) {
  extern __shared__ double S[];
  const int N = g.N, H = g.H;
  const long long V2 = g.V2, V = 2 * V2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  MonLocal mon;
  if (DIR == 0) {
    const long long R0 = (long long)blockIdx.x * nrows;
    const int nr = (int)min((long long)nrows, (long long)N * N - R0);
    // S[L][r][h][m]
    // 16-byte cp.async: every load of the slab in flight at once
    const int HC = H / 2;  // 16-byte chunks per half row
#pragma unroll
    for (int L = 0; L < 6; ++L)  // static component index: Fields stays in the parameter space
      for (int e = tid; e < nr * H; e += kSlabThreads) {
        const int r = e / H, cc = e - r * H;
        const int h = cc >= HC ? 1 : 0, m = 2 * (cc - h * HC);
        cp_async16(&S[((L * nrows + r) * 2 + h) * H + m], in.c[4 + L] + h * V2 + (R0 + r) * H + m);
      }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
#pragma unroll
    for (int pi = 0; pi < 2; ++pi) {  // static face index: the arguments stay in the parameter space
      const int eo = a.eo[pi];
      for (int e = tid; e < nr * H; e += kSlabThreads) {
        const int r = e / H, u = e - r * H;
        const long long R = R0 + r;
        const int j = (int)(R % N), k = (int)(R / N);
        const int sA = (eo + j + k) & 1;  // A sites at i = 2u + sA
        {
          const int iA = 2 * u + sA;
          const int iB = (iA + 1 == N) ? 0 : iA + 1;
          double *pa = S + ((size_t)r * 2 + eo) * H + u;
          double *pb = S + ((size_t)r * 2 + (eo ^ 1)) * H + (iB >> 1);
          const size_t ls = (size_t)nrows * 2 * H;
          double nA[6], nB[6];
#pragma unroll
          for (int L = 0; L < 6; ++L) {
            nA[L] = pa[L * ls];
            nB[L] = pb[L * ls];
          }
          charge_link<INJECTED, MON>(nA, nB, a, pi, R * N + iA, V, true, mon);
#pragma unroll
          for (int L = 0; L < 6; ++L) {
            pa[L * ls] = nA[L];
            pb[L * ls] = nB[L];
          }
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int L = 0; L < 6; ++L)
      for (int r = 0; r < nr; ++r)
        for (int e = tid; e < 2 * H; e += kSlabThreads) {
          const int h = e >= H ? 1 : 0, m = e - h * H;
          out.c[4 + L][h * V2 + (R0 + r) * H + m] = S[((L * nrows + r) * 2 + h) * H + m];
        }
  } else {
    const int x0 = blockIdx.x * 32, m0 = x0 >> 1;
    const int c2 = blockIdx.y;  // k for y lines, j for z lines
    const int s0 = blockIdx.z * seglen, s1 = min(s0 + seglen, N);
    const int W = (s1 - s0) + 4;  // window positions t = s0 - 2 + w
    // S[L][w][h][mm]: 32 doubles per (L, w)
    const int h = lane >> 4, mm = lane & 15;
    // 16-byte cp.async: every load of the slab in flight at once
#pragma unroll
    for (int L = 0; L < 6; ++L)
      for (int e = tid; e < W * 16; e += kSlabThreads) {
        const int w = e >> 4, cc = e & 15;
        const int hc = cc >> 3, mc = 2 * (cc & 7);
        const int t = wrapn(s0 - 2 + w, N);
        const int j = DIR == 1 ? t : c2, k = DIR == 1 ? c2 : t;
        cp_async16(&S[((L * W + w) * 2 + hc) * 16 + mc], in.c[4 + L] + hc * V2 + ((long long)k * N + j) * H + m0 + mc);
      }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    const size_t ls = (size_t)W * 32;
    const int lx = lane;  // natural column x0 + lx
#pragma unroll
    for (int pi = 0; pi < 2; ++pi) {
      const int eo = a.eo[pi];
      const int w0 = (eo + lx + c2 + s0) & 1;  // A sites of this column at w = w0 + 2u
      // first face: every link inside the window; second face: links with both ends in [1, W-2]
      const int wlo = pi == 0 ? 0 : 1, whi = pi == 0 ? W - 1 : W - 2;
      for (int w = w0 + 2 * warp; w + 1 <= whi; w += 2 * (kSlabThreads / 32)) {
        if (w < wlo) continue;
        const int tA = wrapn(s0 - 2 + w, N);
        const int j = DIR == 1 ? tA : c2, k = DIR == 1 ? c2 : tA;
        double *pa = S + ((size_t)w * 2 + eo) * 16 + (lx >> 1);
        double *pb = S + ((size_t)(w + 1) * 2 + (eo ^ 1)) * 16 + (lx >> 1);
        double nA[6], nB[6];
#pragma unroll
        for (int L = 0; L < 6; ++L) {
          nA[L] = pa[L * ls];
          nB[L] = pb[L * ls];
        }
        const bool own = (w - 2) >= 0 && (w - 2) < (s1 - s0);
        charge_link<INJECTED, MON>(nA, nB, a, pi, ((long long)k * N + j) * N + x0 + lx, V, own, mon);
#pragma unroll
        for (int L = 0; L < 6; ++L) {
          pa[L * ls] = nA[L];
          pb[L * ls] = nB[L];
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int L = 0; L < 6; ++L)
      for (int w = 2 + warp; w < W - 2; w += kSlabThreads / 32) {
        const int t = s0 - 2 + w;
        const int j = DIR == 1 ? t : c2, k = DIR == 1 ? c2 : t;
        out.c[4 + L][h * V2 + ((long long)k * N + j) * H + m0 + mm] = S[(L * W + w) * 32 + lane];
      }
  }
  if (MON) mon_flush(mon, a.mon);
}

// ----------------------------------------------------------------------------
// Euler-Maruyama Model A step (Jacobi: reads `in`, writes phi of `out`).
// One thread per element m of both parity half-rows of row (j, k).  I: the
// element offset type (int when idx32 holds, as the heat-bath pass).
template <bool INJECTED, typename I = long long>
__device__ __forceinline__ void em_pair(const Fields &in, const Fields &out, const Geo &g, const EmArgs &a, int m,
                                        int j, int k, double (&acc)[4]) {
  const int H = g.H, N = g.N;
  const I row = ((I)k * N + j) * H;
  const I rjp = ((I)k * N + wrap_inc(j, N)) * H + m;
  const I rjm = ((I)k * N + wrap_dec(j, N)) * H + m;
  const I rkp = ((I)wrap_inc(k, g.Nz) * N + j) * H + m;
  const I rkm = ((I)wrap_dec(k, g.Nz) * N + j) * H + m;
#pragma unroll
  for (int parity = 0; parity < 2; ++parity) {
    const int s = (parity + j + k) & 1;
    const int i = 2 * m + s;
    int xm = m - 1 + s, xp = m + s;
    if (xm < 0) xm += H;
    if (xp == H) xp = 0;
    const I own = (I)parity * (I)g.V2 + row + m;
    const I ob = (I)(parity ^ 1) * (I)g.V2;
    const I orow = ob + row;
    const long long nat = (long long)nat_index_t<I>(g, i, j, k);
    double xi[4];
    if (INJECTED) {
#pragma unroll
      for (int l = 0; l < 4; ++l) xi[l] = a.xi[(long long)l * global_sites(g) + nat];
    } else {
      Xoro rng = stream_at(a.sk, (uint64_t)nat);
      const uint64_t r1 = rng.next(), r2 = rng.next(), r3 = rng.next(), r4 = rng.next();
      box_muller(r1, r2, xi[0], xi[1]);
      box_muller(r3, r4, xi[2], xi[3]);
    }
    double c[4];
#pragma unroll
    for (int l = 0; l < 4; ++l) c[l] = in.c[l][own];
    const double p2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const double *P = in.c[l];
      const double heff = (P[orow + xp] + P[orow + xm]) + (P[ob + rjp] + P[ob + rjm]) + (P[ob + rkp] + P[ob + rkm]);
      double fo = -heff + a.c6 * c[l] + a.lambda * p2 * c[l];
      if (l == 0) fo -= a.H;
      const double v = c[l] - a.dtg * fo + a.sq * xi[l];
      out.c[l][own] = v;
      acc[l] += v;
    }
  }
}

// One thread per site pair (element m of both parity half rows of row (j, k)),
// flat over the V/2 pairs.  AVG: also the volume averages of the new phi into
// avg_out[0..3] (grid_sum4).  Six 256-thread CTAs per SM (40 registers): the
// step is bound by issue and its loads' latency, and measured fastest there
// (0.399 ms per 256^3 step against 0.404 at five, 0.420 at four, 0.399 at
// seven or eight with more spill).
template <bool INJECTED, bool AVG, typename I>
__global__ void __launch_bounds__(kThreads, 6) em_kernel(Fields in, Fields out, Geo g, EmArgs a, double *partial,
                                                      unsigned *done, double *avg_out) {
  const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
  double acc[4] = {0, 0, 0, 0};
  if (idx < g.V2) {
    int m, j, k;
    pair_coords(idx, g, m, j, k);
    em_pair<INJECTED, I>(in, out, g, a, m, j, k, acc);
  }
  if (AVG) grid_sum4<kThreads>(acc, partial, done, avg_out, 1.0 / (2.0 * (double)g.V2), false);
}

// Adjoint of the Euler-Maruyama step for one site pair (see em_adjoint_kernel).
// Both parities of site pair (m, j, k); adds the parameter sums into v[0..3].
template <typename I = long long>
__device__ __forceinline__ void em_adjoint_pair(const Fields &phi, const Fields &lin, const Fields &lout, const Geo &g,
                                                const EmAdjArgs &a, int m, int j, int k, double (&v)[4]) {
  const int H = g.H, N = g.N;
  const I row = ((I)k * N + j) * H;
  const I rjp = ((I)k * N + wrap_inc(j, N)) * H + m;
  const I rjm = ((I)k * N + wrap_dec(j, N)) * H + m;
  const I rkp = ((I)wrap_inc(k, N) * N + j) * H + m;
  const I rkm = ((I)wrap_dec(k, N) * N + j) * H + m;
  double gm = 0, gla = 0, gh = 0, gg = 0;
#pragma unroll
  for (int parity = 0; parity < 2; ++parity) {
    const int s = (parity + j + k) & 1;
    int xm = m - 1 + s, xp = m + s;
    if (xm < 0) xm += H;
    if (xp == H) xp = 0;
    const I own = (I)parity * (I)g.V2 + row + m;
    const I ob = (I)(parity ^ 1) * (I)g.V2;
    const I orow = ob + row;
    const long long nat = (long long)(((I)k * N + j) * N + 2 * m + s);
    double c[4], l[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      c[b] = phi.c[b][own];
      l[b] = lin.c[b][own];
    }
    Xoro rng = stream_at(a.sk, (uint64_t)nat);
    double xi[4];
    const uint64_t r1 = rng.next(), r2 = rng.next(), r3 = rng.next(), r4 = rng.next();
    box_muller(r1, r2, xi[0], xi[1]);
    box_muller(r3, r4, xi[2], xi[3]);
    const double p2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
    const double dot = c[0] * l[0] + c[1] * l[1] + c[2] * l[2] + c[3] * l[3];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const double *P = phi.c[b], *Lm = lin.c[b];
      const double hf = (P[orow + xp] + P[orow + xm]) + (P[ob + rjp] + P[ob + rjm]) + (P[ob + rkp] + P[ob + rkm]);
      const double nl = (Lm[orow + xp] + Lm[orow + xm]) + (Lm[ob + rjp] + Lm[ob + rjm]) + (Lm[ob + rkp] + Lm[ob + rkm]);
      const double jl = a.c6 * l[b] + a.lambda * (p2 * l[b] + 2.0 * c[b] * dot) - nl;
      lout.c[b][own] = l[b] - a.dtg * jl + a.gl[b];
      double F = -hf + a.c6 * c[b] + a.lambda * p2 * c[b];
      if (b == 0) F -= a.H;
      gg += l[b] * (-a.dt * F + a.cxi * xi[b]);
    }
    gm += -a.dtg * dot;
    gla += -a.dtg * p2 * dot;
    gh += a.dtg * l[0];
  }
  v[0] += gm;
  v[1] += gla;
  v[2] += gh;
  v[3] += gg;
}

// ----------------------------------------------------------------------------
// Fused ideal step (IdealPV2::step_no_reject, Stepper.cxx:68-176).
// A CTA owns a TX x TY column of sites and marches up a z-chunk.  At plane p
// it rotates phi by the half step (phi') for its sites and a one-site ring
// into shared memory (3 rotating plane buffers); for plane p-1 it advects the
// charges with the 7-point stencil on phi', applies the second half rotation
// with the updated charges and writes the site to `out`.  The 10 components
// of plane p+1 arrive by cp.async while plane p computes.  Each site is read
// once (80 B) and written once (80 B).
template <int TX, int TY>
struct IdealTile {
  static constexpr int SX = TX + 2, SY = TY + 2, SP = SX * SY;
  static constexpr int NHALO = 2 * SX + 2 * TY;
  static constexpr size_t SMEM = (size_t)(2 * 10 * SP + 3 * 4 * SP) * sizeof(double);
};

template <int TX, int TY>
__device__ __forceinline__ void ideal_tile(const Fields &in, const Fields &out, const Geo &g, int zchunk,
                                           const IdealArgs &a, int bx, int by, int bz) {
  using T = IdealTile<TX, TY>;
  constexpr int SX = T::SX, SY = T::SY, SP = T::SP, NHALO = T::NHALO;
  static_assert(NHALO <= TX * TY, "halo ring larger than the CTA");
  extern __shared__ double smem[];
  double *raw = smem;               // [2 stages][10][SP]
  double *phs = raw + 2 * 10 * SP;  // [3][4][SP]
  const int N = g.N;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int x0 = bx * TX, y0 = by * TY;
  const int z0 = bz * zchunk;
  const int z1 = min(z0 + zchunk, g.Nz);
  const int nit = (z1 - z0) + 2;
  const bool act = (x0 + tx < N) && (y0 + ty < N);
  const int xi = (x0 + tx) % N, yj = (y0 + ty) % N;
  const int sc = (ty + 1) * SX + tx + 1;

  int hs = -1, hxg = 0, hyg = 0;
  if (threadIdx.x < NHALO) {
    const int h = threadIdx.x;
    int hx, hy;
    if (h < SX) { hx = h; hy = 0; }
    else if (h < 2 * SX) { hx = h - SX; hy = SY - 1; }
    else if (h < 2 * SX + TY) { hx = 0; hy = 1 + (h - 2 * SX); }
    else { hx = SX - 1; hy = 1 + (h - 2 * SX - TY); }
    hs = hy * SX + hx;
    hxg = wrapn(x0 - 1 + hx, N);
    hyg = wrapn(y0 - 1 + hy, N);
  }

  // Planes z0-1 .. z1 of the march, tracked incrementally (within two wraps
  // of the buffer: nit <= Nz + 2), and rb_off split into its in-plane part
  // and plane part, so the march does no integer division.
  const int zfirst = z0 == 0 ? g.Nz - 1 : z0 - 1;
  auto plane_of = [&](int q) {
    int pl = zfirst + q;
    if (pl >= g.Nz) pl -= g.Nz;
    if (pl >= g.Nz) pl -= g.Nz;
    return pl;
  };
  const long long NH = (long long)N * g.H;
  const int own_xy = yj * g.H + (xi >> 1), own_par = (xi + yj) & 1;
  const int ring_xy = hyg * g.H + (hxg >> 1), ring_par = (hxg + hyg) & 1;
  auto issue = [&](int plane, int stage, bool halo) {
    const long long o = (long long)((own_par + plane) & 1) * g.V2 + (long long)plane * NH + own_xy;
#pragma unroll
    for (int c = 0; c < 10; ++c) cp_async8(&raw[(stage * 10 + c) * SP + sc], in.c[c] + o);
    if (halo && hs >= 0) {
      const long long oh = (long long)((ring_par + plane) & 1) * g.V2 + (long long)plane * NH + ring_xy;
#pragma unroll
      for (int c = 0; c < 10; ++c) cp_async8(&raw[(stage * 10 + c) * SP + hs], in.c[c] + oh);
    }
  };

  issue(zfirst, 0, false);
  cp_async_commit();

  double pm[4], pc[4], pn[4], qc[6], qn[6];
  int pprev = zfirst;  // plane p - 1 (used from it >= 2)
  for (int it = 0; it < nit; ++it) {
    const int p = plane_of(it);
    cp_async_wait_all();
    __syncthreads();
    if (it + 1 < nit) issue(plane_of(it + 1), (it + 1) & 1, true);
    cp_async_commit();

    const double *rw = raw + (it & 1) * 10 * SP;
    double *ph = phs + (it % 3) * 4 * SP;
#pragma unroll
    for (int l = 0; l < 4; ++l) pn[l] = rw[l * SP + sc];
#pragma unroll
    for (int s = 0; s < 6; ++s) qn[s] = rw[(4 + s) * SP + sc];
    rotate_site(pn, qn, a.dto2chi);
#pragma unroll
    for (int l = 0; l < 4; ++l) ph[l * SP + sc] = pn[l];
    if (hs >= 0 && it >= 1) {
      double phh[4], qh[6];
#pragma unroll
      for (int l = 0; l < 4; ++l) phh[l] = rw[l * SP + hs];
#pragma unroll
      for (int s = 0; s < 6; ++s) qh[s] = rw[(4 + s) * SP + hs];
      rotate_site(phh, qh, a.dto2chi);
#pragma unroll
      for (int l = 0; l < 4; ++l) ph[l * SP + hs] = phh[l];
    }

    if (it >= 2 && act) {
      const double *pp = phs + ((it + 2) % 3) * 4 * SP;  // phi' of plane p-1 (written last iteration)
      double xp[4], xm[4], yp[4], ym[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        xp[l] = pp[l * SP + sc + 1];
        xm[l] = pp[l * SP + sc - 1];
        yp[l] = pp[l * SP + sc + SX];
        ym[l] = pp[l * SP + sc - SX];
      }
      const double *c = pc, *zp = pn, *zm = pm;
      double S[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) S[l] = ((xp[l] + xm[l]) + (yp[l] + ym[l])) + (zp[l] + zm[l]);
      charge_currents(c, S, a.dt, a.a2, a.H, qc);
      // second half rotation on a copy: pc (phi') stays the z-1 neighbour of the next plane
      double pf[4] = {pc[0], pc[1], pc[2], pc[3]};
      rotate_site(pf, qc, a.dto2chi);
      const long long o = (long long)((own_par + pprev) & 1) * g.V2 + (long long)pprev * NH + own_xy;
#pragma unroll
      for (int l = 0; l < 4; ++l) out.c[l][o] = pf[l];
#pragma unroll
      for (int s = 0; s < 6; ++s) out.c[4 + s][o] = qc[s];
    }
    pprev = p;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      pm[l] = pc[l];
      pc[l] = pn[l];
    }
#pragma unroll
    for (int s = 0; s < 6; ++s) qc[s] = qn[s];
  }
}

template <int TX, int TY>
__global__ void __launch_bounds__(TX *TY, 2) ideal_kernel(Fields in, Fields out, Geo g, int zchunk, IdealArgs a) {
  ideal_tile<TX, TY>(in, out, g, zchunk, a, blockIdx.x, blockIdx.y,
                    g.zrev ? (int)(gridDim.z - 1 - blockIdx.z) : (int)blockIdx.z);
}

// ----------------------------------------------------------------------------
// Energy (IdealPV2::computeEnergy, Stepper.cxx:204-268): forward differences.
__global__ void energy_kernel(Fields f, Geo g, double *partial) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double grad2 = 0, nab2 = 0, hphi = 0;
  if (t < 2 * g.V2) {
    const int N = g.N;
    const long long n = t;
    const int i = (int)(n % N);
    const long long r = n / N;
    const int j = (int)(r % N), k = (int)(r / N);
    const long long o = rb_off(g, i, j, k);
    const long long ox = rb_off(g, wrap_inc(i, N), j, k);
    const long long oy = rb_off(g, i, wrap_inc(j, N), k);
    const long long oz = rb_off(g, i, j, wrap_inc(k, N));
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const double pm = f.c[s][o];
      const double a = f.c[s][oz] - pm, b = f.c[s][oy] - pm, c = f.c[s][ox] - pm;
      grad2 += a * a + b * b + c * c;
    }
    hphi = f.c[0][o];
#pragma unroll
    for (int s = 0; s < 6; ++s) nab2 += f.c[4 + s][o] * f.c[4 + s][o];
  }
  __shared__ double s3[3][kThreads / 32];
  warp_sum(grad2);
  warp_sum(nab2);
  warp_sum(hphi);
  if ((threadIdx.x & 31) == 0) {
    s3[0][threadIdx.x >> 5] = grad2;
    s3[1][threadIdx.x >> 5] = nab2;
    s3[2][threadIdx.x >> 5] = hphi;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t2 = 0;
    for (int w = 0; w < kThreads / 32; ++w) t2 += s3[threadIdx.x][w];
    partial[(long long)blockIdx.x * 3 + threadIdx.x] = t2;
  }
}

__global__ void energy_final_kernel(const double *partial, int nblk, double H, double half_over_chi,
                                    double *out) {
  __shared__ double s[3];
  const int c = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (c < 3) {
    double t = 0;
    for (int b = l; b < nblk; b += 32) t += partial[(long long)b * 3 + c];
    warp_sum(t);
    if (l == 0) s[c] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) out[0] = half_over_chi * s[1] + 0.5 * s[0] - H * s[2];
}

// ----------------------------------------------------------------------------
// Measurer.  The 25 per-site observables: 11 of computeSliceAverage
// (phi_a, A, V, phi^2; measurer.cxx:46-69) then 14 of computeSliceAveragePhase
// (sigma, n_a, A_a, V_a, sigma^2; measurer.cxx:152-192).
constexpr int kNObs = 25;

__device__ __forceinline__ void site_obs(const double f[10], double o[kNObs]) {
  double phi2 = 0.0;
#pragma unroll
  for (int l = 0; l < 10; ++l) o[l] = f[l];
#pragma unroll
  for (int l = 0; l < 4; ++l) phi2 += f[l] * f[l];
  o[10] = phi2;
  const double sigma = sqrt(phi2);
  double n[4];
  if (phi2 > 100. * 2.2250738585072014e-308) {
    // one division instead of four (equal to phi_a / sigma up to an ulp)
    const double inv = 1.0 / sigma;
#pragma unroll
    for (int l = 0; l < 4; ++l) n[l] = f[l] * inv;
  } else {
    n[0] = 1;
    n[1] = n[2] = n[3] = 0;
  }
  const double *rho = f + 4;  // (A1..3, V1..3)
  // contract_rho(n, rho) and contract_rho(n, dual rho) (measurer.cxx:101-114)
  const double A0 = -(n[1] * rho[0]) - n[2] * rho[1] - n[3] * rho[2];
  const double A1 = n[0] * rho[0] + n[3] * rho[4] - n[2] * rho[5];
  const double A2 = n[0] * rho[1] - n[3] * rho[3] + n[1] * rho[5];
  const double A3 = n[0] * rho[2] + n[2] * rho[3] - n[1] * rho[4];
  const double V0 = -(n[1] * rho[3]) - n[2] * rho[4] - n[3] * rho[5];
  const double V1 = n[0] * rho[3] + n[3] * rho[1] - n[2] * rho[2];
  const double V2 = n[0] * rho[4] - n[3] * rho[0] + n[1] * rho[2];
  const double V3 = n[0] * rho[5] + n[2] * rho[0] - n[1] * rho[1];
  o[11] = sigma;
#pragma unroll
  for (int l = 0; l < 4; ++l) o[12 + l] = n[l];
  o[16] = A0; o[17] = A1; o[18] = A2; o[19] = A3;
  o[20] = V0; o[21] = V1; o[22] = V2; o[23] = V3;
  o[24] = sigma * sigma;
}

__device__ __forceinline__ void load_site(const Fields &f, const Geo &g, int i, int j, int k, double s[10]) {
  const long long o = rb_off(g, i, j, k);
#pragma unroll
  for (int L = 0; L < 10; ++L) s[L] = f.c[L][o];
}

// T[o][kout + k - klo][i] = sum_j obs(i, j, k) for local planes k in [klo, klo + nk);
// T is [25][Ng][N]
__global__ void meas_sum_j_kernel(Fields f, Geo g, double *T, int klo, int nk, int kout) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = g.N;
  if (t >= (long long)N * nk) return;
  const int i = (int)(t % N), kl = (int)(t / N), k = klo + kl;
  double acc[kNObs];
#pragma unroll
  for (int o = 0; o < kNObs; ++o) acc[o] = 0;
  for (int j = 0; j < N; ++j) {
    double s[10], ob[kNObs];
    load_site(f, g, i, j, k, s);
    site_obs(s, ob);
#pragma unroll
    for (int o = 0; o < kNObs; ++o) acc[o] += ob[o];
  }
  const long long NT = (long long)g.Ng * N;
#pragma unroll
  for (int o = 0; o < kNObs; ++o) T[o * NT + (long long)(kout + kl) * N + i] = acc[o];
}

// U[o][j][i] = sum_k obs(i, j, k) over local planes [klo, klo + nk)
__global__ void meas_sum_k_kernel(Fields f, Geo g, double *U, int klo, int nk) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = g.N;
  if (t >= (long long)N * N) return;
  const int i = (int)(t % N), j = (int)(t / N);
  double acc[kNObs];
#pragma unroll
  for (int o = 0; o < kNObs; ++o) acc[o] = 0;
  for (int k = klo; k < klo + nk; ++k) {
    double s[10], ob[kNObs];
    load_site(f, g, i, j, k, s);
    site_obs(s, ob);
#pragma unroll
    for (int o = 0; o < kNObs; ++o) acc[o] += ob[o];
  }
  const long long NN = (long long)N * N;
#pragma unroll
  for (int o = 0; o < kNObs; ++o) U[o * NN + (long long)j * N + i] = acc[o];
}

struct MeasOut {
  double *oavg;
  double *wall[3], *wk[3], *wkr[3], *ph[3], *phk[3];
};

__host__ __device__ inline MeasOut meas_layout(double *base, int N) {
  const int NK = N / 2 + 1;
  MeasOut m;
  double *p = base;
  m.oavg = p;
  p += 11;
  for (int a = 0; a < 3; ++a) { m.wall[a] = p; p += 11 * N; }
  for (int a = 0; a < 3; ++a) { m.wk[a] = p; p += 11 * NK * 2; }
  for (int a = 0; a < 3; ++a) { m.wkr[a] = p; p += 14 * NK * 2; }
  for (int a = 0; a < 3; ++a) { m.ph[a] = p; p += 14 * N; }
  for (int a = 0; a < 3; ++a) { m.phk[a] = p; p += 14 * NK * 2; }
  return m;
}

// walls: axis 0 (X): sum_k T[o][k][i]; axis 2 (Z): sum_i T[o][k][i];
// axis 1 (Y): sum_i U[o][j][i]; divided by N^2 (measurer.cxx:78-80).
__global__ void meas_walls_kernel(const double *T, const double *U, int N, MeasOut mo) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * kNObs * N) return;
  const int pos = t % N;
  const int o = (t / N) % kNObs;
  const int axis = t / (N * kNObs);
  const long long NN = (long long)N * N;
  double s = 0;
  if (axis == 0) {
    for (int k = 0; k < N; ++k) s += T[o * NN + (long long)k * N + pos];
  } else if (axis == 2) {
    for (int i = 0; i < N; ++i) s += T[o * NN + (long long)pos * N + i];
  } else {
    for (int i = 0; i < N; ++i) s += U[o * NN + (long long)pos * N + i];
  }
  s /= (double)(N * N);
  if (o < 11) mo.wall[axis][o * N + pos] = s;
  else mo.ph[axis][(o - 11) * N + pos] = s;
}

// OAverage[l] = mean_x wallX(l, x) (measurer.cxx:292-300) and the r2c DFT of
// every wall row, W(k) = (1/N) sum_x W(x) e^{-2 pi i k x / N}, k = 0..N/2.
__global__ void meas_dft_kernel(int N, MeasOut mo) {
  const int NK = N / 2 + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 11) {
    double s = 0;
    for (int i = 0; i < N; ++i) s += mo.wall[0][t * N + i];
    mo.oavg[t] = s / (double)N;
  }
  if (t >= 3 * kNObs * NK) return;
  const int kk = t % NK;
  const int o = (t / NK) % kNObs;
  const int axis = t / (NK * kNObs);
  const double *row = (o < 11) ? mo.wall[axis] + o * N : mo.ph[axis] + (o - 11) * N;
  double re = 0, im = 0;
  for (int x = 0; x < N; ++x) {
    const int m = (int)(((long long)kk * x) % N);
    double sn, cs;
    sincospi(2.0 * (double)m / (double)N, &sn, &cs);
    re += row[x] * cs;
    im -= row[x] * sn;
  }
  double *dst = (o < 11) ? mo.wk[axis] + (o * NK + kk) * 2 : mo.phk[axis] + ((o - 11) * NK + kk) * 2;
  dst[0] = re / (double)N;
  dst[1] = im / (double)N;
}

// rotate_to_vev (measurer.cxx:231-286), complex arithmetic as the reference.
__global__ void meas_rotate_kernel(int N, MeasOut mo) {
  const int NK = N / 2 + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * NK) return;
  const int kk = t % NK, axis = t / NK;
  const double *w = mo.wk[axis];
  auto re = [&](int a, int k) { return w[(a * NK + k) * 2]; };
  auto im = [&](int a, int k) { return w[(a * NK + k) * 2 + 1]; };
  double nr[4], ni[4];
  double nrm = 0;
  for (int a = 0; a < 4; ++a) {
    nr[a] = re(a, 0);
    ni[a] = im(a, 0);
    nrm += nr[a] * nr[a] + ni[a] * ni[a];
  }
  nrm = sqrt(nrm);
  if (nrm < 2.2250738585072014e-308) {
    nr[0] = 1; ni[0] = 0;
    for (int a = 1; a < 4; ++a) nr[a] = ni[a] = 0;
  } else {
    for (int a = 0; a < 4; ++a) { nr[a] /= nrm; ni[a] /= nrm; }
  }
  double pr[4], pi[4], rr[6], ri[6];
  for (int a = 0; a < 4; ++a) { pr[a] = re(a, kk); pi[a] = im(a, kk); }
  for (int b = 0; b < 6; ++b) { rr[b] = re(4 + b, kk); ri[b] = im(4 + b, kk); }
  // phis = sum_a n_a phi_a (complex, no conjugation)
  double sr = 0, si = 0;
  for (int a = 0; a < 4; ++a) {
    sr += nr[a] * pr[a] - ni[a] * pi[a];
    si += nr[a] * pi[a] + ni[a] * pr[a];
  }
  double *o = mo.wkr[axis];
  auto put = [&](int a, double x, double y) { o[(a * NK + kk) * 2] = x; o[(a * NK + kk) * 2 + 1] = y; };
  put(0, sr, si);
  for (int a = 0; a < 4; ++a) {
    // phir = phi - n * phis
    put(1 + a, pr[a] - (nr[a] * sr - ni[a] * si), pi[a] - (nr[a] * si + ni[a] * sr));
  }
  // complex products c = n_a * rho_b
#define CMR(a, b) (nr[a] * rr[b] - ni[a] * ri[b])
#define CMI(a, b) (nr[a] * ri[b] + ni[a] * rr[b])
  // contract_rho(n, rho)
  put(5, -CMR(1, 0) - CMR(2, 1) - CMR(3, 2), -CMI(1, 0) - CMI(2, 1) - CMI(3, 2));
  put(6, CMR(0, 0) + CMR(3, 4) - CMR(2, 5), CMI(0, 0) + CMI(3, 4) - CMI(2, 5));
  put(7, CMR(0, 1) - CMR(3, 3) + CMR(1, 5), CMI(0, 1) - CMI(3, 3) + CMI(1, 5));
  put(8, CMR(0, 2) + CMR(2, 3) - CMR(1, 4), CMI(0, 2) + CMI(2, 3) - CMI(1, 4));
  // contract_rho(n, dualize_rho(rho)), dual = (rho3..5, rho0..2)
  put(9, -CMR(1, 3) - CMR(2, 4) - CMR(3, 5), -CMI(1, 3) - CMI(2, 4) - CMI(3, 5));
  put(10, CMR(0, 3) + CMR(3, 1) - CMR(2, 2), CMI(0, 3) + CMI(3, 1) - CMI(2, 2));
  put(11, CMR(0, 4) - CMR(3, 0) + CMR(1, 2), CMI(0, 4) - CMI(3, 0) + CMI(1, 2));
  put(12, CMR(0, 5) + CMR(2, 0) - CMR(1, 1), CMI(0, 5) + CMI(2, 0) - CMI(1, 1));
#undef CMR
#undef CMI
  put(13, re(10, kk), im(10, kk));
}

// Sums of the 25 observables over a lattice given in the host-order AoS layout
// u[k][j][i][10] (used by the allocation-free measurement entry point).
// T[o][k][i] = sum_j obs(i, j, k)
__global__ void meas_sum_j_aos_kernel(const double *__restrict__ aos, int N, double *T) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * N) return;
  const int i = (int)(t % N), k = (int)(t / N);
  double acc[kNObs];
#pragma unroll
  for (int o = 0; o < kNObs; ++o) acc[o] = 0;
  for (int j = 0; j < N; ++j) {
    const double *src = aos + (((long long)k * N + j) * N + i) * 10;
    double s[10], ob[kNObs];
#pragma unroll
    for (int L = 0; L < 10; ++L) s[L] = src[L];
    site_obs(s, ob);
#pragma unroll
    for (int o = 0; o < kNObs; ++o) acc[o] += ob[o];
  }
  const long long NN = (long long)N * N;
#pragma unroll
  for (int o = 0; o < kNObs; ++o) T[o * NN + (long long)k * N + i] = acc[o];
}

// U[o][j][i] = sum_k obs(i, j, k)
__global__ void meas_sum_k_aos_kernel(const double *__restrict__ aos, int N, double *U) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * N) return;
  const int i = (int)(t % N), j = (int)(t / N);
  double acc[kNObs];
#pragma unroll
  for (int o = 0; o < kNObs; ++o) acc[o] = 0;
  for (int k = 0; k < N; ++k) {
    const double *src = aos + (((long long)k * N + j) * N + i) * 10;
    double s[10], ob[kNObs];
#pragma unroll
    for (int L = 0; L < 10; ++L) s[L] = src[L];
    site_obs(s, ob);
#pragma unroll
    for (int o = 0; o < kNObs; ++o) acc[o] += ob[o];
  }
  const long long NN = (long long)N * N;
#pragma unroll
  for (int o = 0; o < kNObs; ++o) U[o * NN + (long long)j * N + i] = acc[o];
}

// ----------------------------------------------------------------------------
// Batched kernels: one launch advances every replica of an ensemble.  The
// flat grid is partitioned into per-replica block ranges (rep[b] is the
// replica of block b, first[r] its first block; the order of the ranges is
// the packing order chosen by the autotuner).  Each block rebuilds its
// replica's arguments exactly as the single-lattice host code does (same
// expressions, no FMA contraction), so a replica evolves bit for bit like a
// lattice of its own; sub-step keys come from the device-resident counter.
// the replica's planes: phi from buffer pphi, charges from buffer pq
__device__ __forceinline__ Fields rep_fields(const RepDesc &r, int pphi, int pq) {
  Fields f;
#pragma unroll
  for (int L = 0; L < 10; ++L) f.c[L] = r.base[L < 4 ? pphi : pq] + (long long)L * r.pstride;
  return f;
}

__device__ __forceinline__ double rep_mass(const RepDesc &r, const EnsDyn &dyn) {
  return __dadd_rn(r.mass0, __dmul_rn(r.dmassdt, dyn.t));
}

// plane kernels: 128 threads cover 128 consecutive (j, m) elements of a plane
__device__ __forceinline__ bool plane_coords(const RepDesc &r, int local, int &m, int &j, int &k) {
  const int chunk = local % r.nchunk;
  k = local / r.nchunk;
  const int t = chunk * 128 + (int)threadIdx.x;
  j = t / r.g.H;
  m = t - j * r.g.H;
  return j < r.g.N;
}

// slab kernels: a block covers 128 consecutive (j, m) elements of kBatchPlanes
// consecutive planes of one replica, so the block-map and descriptor loads
// (two dependent round trips before the first site load) are paid once per
// kBatchPlanes planes
__device__ __forceinline__ bool slab_coords(const RepDesc &r, int local, int lane, int &m, int &j, int &k0) {
  const int chunk = local % r.nchunk;
  k0 = (local / r.nchunk) * kBatchPlanes;
  const int t = chunk * 128 + lane;
  j = t / r.g.H;
  m = t - j * r.g.H;
  return j < r.g.N;
}

// Items of the batched heat-bath and charge sub-steps: block blk of the slab
// map, lane 0..127 of its 128 threads (a kernel of their own, or half of a
// CTA of the persistent step).
template <typename I>
__device__ __forceinline__ void batch_hb_item(const RepDesc *__restrict__ d, const EnsDyn *__restrict__ dyn,
                                              const int *__restrict__ rep, const int *__restrict__ first, int blk,
                                              int lane, int phase, int parity, double dt, int ctr_off) {
  const int r = rep[blk];
  const RepDesc &R = d[r];
  const EnsDyn y = *dyn;
  int m, j, k0;
  if (!slab_coords(R, blk - first[r], lane, m, j, k0)) return;
  HbArgs a{};
  a.rdtg = sqrt(2. * dt * R.gamma);
  a.Lambda2 = 0.5 * (2. * 3. + rep_mass(R, y));
  a.lam4 = R.lambda / 4.;
  a.H = R.H;
  a.sk = sub_key(R.key, y.ctr + (unsigned long long)ctr_off);
  const Fields f = rep_fields(R, phase, phase);
  MonLocal mon;
  // one plane after the other: unrolled (the planes' loads interleaved) the
  // ensemble step measured 4 % slower, at 62 registers against 64 here
#pragma unroll 1
  for (int q = 0; q < kBatchPlanes; ++q)
    if (k0 + q < R.g.N) hb_site<false, false, false, I>(f, R.g, parity, a, m, j, k0 + q, mon);
}

template <typename I>
__global__ void __launch_bounds__(128) batch_hb_kernel(const RepDesc *__restrict__ d, const EnsDyn *__restrict__ dyn,
                                                       const int *__restrict__ rep, const int *__restrict__ first,
                                                       int phase, int parity, double dt, int ctr_off) {
  batch_hb_item<I>(d, dyn, rep, first, blockIdx.x, threadIdx.x, phase, parity, dt, ctr_off);
}

template <typename I>
__device__ __forceinline__ void batch_charge_item(const RepDesc *__restrict__ d, const EnsDyn *__restrict__ dyn,
                                                  const int *__restrict__ rep, const int *__restrict__ first, int blk,
                                                  int lane, int phase, int pass, double dt, int ctr_off_order) {
  const int r = rep[blk];
  const RepDesc &R = d[r];
  const EnsDyn y = *dyn;
  int m, j, k0;
  if (!slab_coords(R, blk - first[r], lane, m, j, k0)) return;
  // the replica's pass order (counter mode of ModelGChargeHB::step)
  const unsigned long long c0 = y.ctr + (unsigned long long)ctr_off_order;
  const uint64_t w = split_word(sub_key(R.key, c0), 0);
  const int pi = (int)((w & 0xffffffffull) % 6ull);
  // lexicographic permutation pi of (0, 1, 2): first element pi / 2, then the
  // remaining two in order (pi even) or swapped (pi odd)
  const int p0 = pi / 2;
  const int lo = (p0 == 0) ? 1 : 0, hi = (p0 == 2) ? 1 : 2;
  const int ixyz = pass / 2;
  const int dir = ixyz == 0 ? p0 : (ixyz == 1 ? ((pi & 1) ? hi : lo) : ((pi & 1) ? lo : hi));
  const int e0 = (int)(w >> 63);
  const int eoA = (pass & 1) ? (e0 ^ 1) : e0;
  ChargeArgs a{};
  a.rms = sqrt(2. * dt * (R.diffusion * R.chi));
  a.inv2chi = 1.0 / (2. * R.chi);
  a.sk = sub_key(R.key, c0 + 1 + pass);
  a.pass = pass;
  const Fields f = rep_fields(R, phase, phase);
  MonLocal mon;
#pragma unroll 1
  for (int q = 0; q < kBatchPlanes; ++q)
    if (k0 + q < R.g.N) charge_link_site<false, false, I>(f, R.g, dir, eoA, a, m, j, k0 + q, mon);
}

// 32 registers, full occupancy (as charge_pass_kernel)
template <typename I>
__global__ void __launch_bounds__(128, 16) batch_charge_kernel(const RepDesc *__restrict__ d,
                                                           const EnsDyn *__restrict__ dyn, const int *__restrict__ rep,
                                                           const int *__restrict__ first, int phase, int pass,
                                                           double dt, int ctr_off_order) {
  batch_charge_item<I>(d, dyn, rep, first, blockIdx.x, threadIdx.x, phase, pass, dt, ctr_off_order);
}

// ---- differentiable Euler-Maruyama runs of an ensemble ---------------------
// Per-replica sums of v[0..3] over the replica's blocks first[r] ..
// first[r] + count[r] - 1 (contiguous in the grid): the replica's last block to
// finish adds the block partials in block order into out[0..3] (accumulating
// when add).  done[r] is zero on entry and re-armed.
__device__ __forceinline__ void rep_sum4(double (&v)[4], int r, int local, int nloc, double *partial, unsigned *done,
                                         double *out, double scale, bool add) {
  constexpr int NW = 4;  // 128 threads
  __shared__ double sm[4][NW];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    warp_sum(v[q]);
    if (lane == 0) sm[q][warp] = v[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) partial[(size_t)blockIdx.x * 4 + q] = ((sm[q][0] + sm[q][1]) + sm[q][2]) + sm[q][3];
    __threadfence();
    last = atomicAdd(done + r, 1u) == (unsigned)(nloc - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const size_t b0 = (size_t)(blockIdx.x - local);
  if (warp < 4) {
    double t = 0;
    for (int b = lane; b < nloc; b += 32) t += __ldcg(partial + (b0 + b) * 4 + warp);
    warp_sum(t);
    if (lane == 0) out[warp] = add ? out[warp] + t * scale : t * scale;
  }
  if (threadIdx.x == 0) done[r] = 0u;
}

__device__ __forceinline__ Fields diff_planes(double *base, long long V, long long first) {
  Fields f{};
#pragma unroll
  for (int l = 0; l < 4; ++l) f.c[l] = base + (first + l) * V;
  return f;
}

__device__ __forceinline__ EmArgs rep_em_args(const RepDesc &R, unsigned long long ctr, double t, double dt) {
  EmArgs a{};
  a.c6 = 6.0 + __dadd_rn(R.mass0, __dmul_rn(R.dmassdt, t));
  a.dtg = dt * R.gamma;
  a.sq = sqrt(2.0 * R.gamma * dt);
  a.lambda = R.lambda;
  a.H = R.H;
  a.sk = sub_key(R.key, ctr);
  return a;
}

__global__ void __launch_bounds__(128) batch_em_fwd_kernel(const RepDesc *__restrict__ d, const DiffDesc *__restrict__ dd,
                                                           const int *__restrict__ rep, const int *__restrict__ first,
                                                           const int *__restrict__ count, int phase,
                                                           unsigned long long ctr, double t, double dt, int n,
                                                           double *partial, unsigned *done) {
  const int r = rep[blockIdx.x];
  const RepDesc &R = d[r];
  const DiffDesc &D = dd[r];
  const int local = blockIdx.x - first[r];
  int m, j, k;
  double acc[4] = {0, 0, 0, 0};
  if (plane_coords(R, local, m, j, k))
    em_pair<false>(rep_fields(R, phase, phase), rep_fields(R, phase ^ 1, phase ^ 1), R.g, rep_em_args(R, ctr, t, dt), m,
                   j, k, acc);
  rep_sum4(acc, r, local, count[r], partial, done, D.avg + (size_t)(n + 1) * 4, 1.0 / (double)D.V, false);
}

__global__ void __launch_bounds__(128) batch_em_seg_kernel(const RepDesc *__restrict__ d, const DiffDesc *__restrict__ dd,
                                                           const int *__restrict__ rep, const int *__restrict__ first,
                                                           int slot, unsigned long long ctr, double t, double dt) {
  const int r = rep[blockIdx.x];
  const RepDesc &R = d[r];
  const DiffDesc &D = dd[r];
  int m, j, k;
  if (!plane_coords(R, blockIdx.x - first[r], m, j, k)) return;
  double acc[4] = {0, 0, 0, 0};
  em_pair<false>(diff_planes(D.seg, D.V, 4LL * slot), diff_planes(D.seg, D.V, 4LL * (slot + 1)), R.g,
                 rep_em_args(R, ctr, t, dt), m, j, k, acc);
}

// dJ/dphi_a(n) of J = w0 obs0 + w1 obs1 (the per-replica averages of the run)
__device__ __forceinline__ void rep_gl(const DiffDesc &D, int n, int b, int S, double gl[4]) {
  gl[0] = gl[1] = gl[2] = gl[3] = 0.0;
  if (n <= b) return;
  const double M = (double)(S - b);
  gl[0] = D.w[0] / ((double)D.V * M);
#pragma unroll
  for (int a = 1; a < 4; ++a) gl[a] = D.w[1] * 2.0 * D.avg[(size_t)n * 4 + a] / M;
}

__global__ void __launch_bounds__(128, 4) batch_em_adj_kernel(const RepDesc *__restrict__ d,
                                                              const DiffDesc *__restrict__ dd,
                                                              const int *__restrict__ rep,
                                                              const int *__restrict__ first,
                                                              const int *__restrict__ count, int slot, int cur, int n,
                                                              int b, int S, unsigned long long ctr, double t, double dt,
                                                              double *partial, unsigned *done) {
  const int r = rep[blockIdx.x];
  const RepDesc &R = d[r];
  const DiffDesc &D = dd[r];
  const int local = blockIdx.x - first[r];
  EmAdjArgs a{};
  a.c6 = 6.0 + __dadd_rn(R.mass0, __dmul_rn(R.dmassdt, t));
  a.dtg = dt * R.gamma;
  a.dt = dt;
  a.lambda = R.lambda;
  a.H = R.H;
  a.cxi = sqrt(2.0 * dt) / (2.0 * sqrt(R.gamma));
  rep_gl(D, n, b, S, a.gl);
  a.sk = sub_key(R.key, ctr);
  double v[4] = {0, 0, 0, 0};
  int m, j, k;
  if (plane_coords(R, local, m, j, k))
    em_adjoint_pair(diff_planes(D.seg, D.V, 4LL * slot), diff_planes(D.lam, D.V, 4LL * cur),
                    diff_planes(D.lam, D.V, 4LL * (cur ^ 1)), R.g, a, m, j, k, v);
  rep_sum4(v, r, local, count[r], partial, done, D.grad, 1.0, true);
}

__global__ void __launch_bounds__(128) batch_diff_copy_kernel(const RepDesc *__restrict__ d,
                                                              const DiffDesc *__restrict__ dd,
                                                              const int *__restrict__ rep,
                                                              const int *__restrict__ first, int dir, int phase, int s,
                                                              int b, int S) {
  const int r = rep[blockIdx.x];
  const RepDesc &R = d[r];
  const DiffDesc &D = dd[r];
  int m, j, k;
  if (!plane_coords(R, blockIdx.x - first[r], m, j, k)) return;
  const long long row = ((long long)k * R.g.N + j) * R.g.H + m;
  double gl[4];
  if (dir == 2) rep_gl(D, S, b, S, gl);
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int par = 0; par < 2; ++par) {
      const long long o = par * R.g.V2 + row;
      if (dir == 0) D.ckpt[((long long)s * 4 + l) * D.V + o] = R.base[phase][l * R.pstride + o];
      else if (dir == 1) D.seg[(long long)l * D.V + o] = D.ckpt[((long long)s * 4 + l) * D.V + o];
      else D.lam[(long long)l * D.V + o] = gl[l];
    }
}

__global__ void __launch_bounds__(128) batch_em_kernel(const RepDesc *__restrict__ d, const EnsDyn *__restrict__ dyn,
                                                       const int *__restrict__ rep, const int *__restrict__ first,
                                                       int phase_in, double dt, int ctr_off) {
  const int r = rep[blockIdx.x];
  const RepDesc &R = d[r];
  const EnsDyn y = *dyn;
  int m, j, k;
  if (!plane_coords(R, blockIdx.x - first[r], m, j, k)) return;
  EmArgs a{};
  a.c6 = 6.0 + rep_mass(R, y);
  a.dtg = dt * R.gamma;
  a.sq = sqrt(2.0 * R.gamma * dt);
  a.lambda = R.lambda;
  a.H = R.H;
  a.sk = sub_key(R.key, y.ctr + (unsigned long long)ctr_off);
  double acc[4] = {0, 0, 0, 0};
  em_pair<false>(rep_fields(R, phase_in, phase_in), rep_fields(R, phase_in ^ 1, phase_in ^ 1), R.g, a, m, j, k, acc);
}

template <int TX, int TY>
__device__ __forceinline__ void batch_ideal_item(const RepDesc *__restrict__ d, const int *__restrict__ rep,
                                                 const int *__restrict__ first, int blk, int pphi, int pq, double dt) {
  const int r = rep[blk];
  const RepDesc &R = d[r];
  const int l = blk - first[r];
  const int bx = l % R.igx, by = (l / R.igx) % R.igy, bz = l / (R.igx * R.igy);
  IdealArgs a;
  a.dto2chi = (dt / 2.0) / R.chi;
  a.dt = dt;
  a.a2 = R.a2;
  a.H = R.H;
  ideal_tile<TX, TY>(rep_fields(R, pphi, pq), rep_fields(R, pphi ^ 1, pq ^ 1), R.g, R.izc, a, bx, by, bz);
}

template <int TX, int TY>
__global__ void __launch_bounds__(TX *TY, 2) batch_ideal_kernel(const RepDesc *__restrict__ d,
                                                                const int *__restrict__ rep,
                                                                const int *__restrict__ first, int pphi, int pq,
                                                                double dt) {
  batch_ideal_item<TX, TY>(d, rep, first, blockIdx.x, pphi, pq, dt);
}

// ---- persistent ensemble step -------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier over the co-resident CTAs of a cooperative launch.  bar[0]
// counts the arrivals of the current generation, bar[1] is the generation and
// bar[2] an error flag.  One thread per CTA reads the generation, publishes
// the CTA's writes (fence) and arrives; the last to arrive resets the count
// and advances the generation, the others poll it -- at most `limit` times,
// after which the CTA raises the error flag, counts a timed-out wait and
// gives up.  A CTA that sees the error flag gives up too, so every CTA leaves
// the launch after a bounded number of polls whatever happened to the
// others.  Returns false when the launch should stop.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned nblocks, int limit, unsigned long long *waits) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned gen = ld_acquire_u32(bar + 1);
    __threadfence();
    if (atomicAdd(bar, 1u) == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      for (int i = 0;; ++i) {
        if (ld_acquire_u32(bar + 1) != gen) break;
        if (ld_acquire_u32(bar + 2) != 0u) {
          ok = 0;
          break;
        }
        if (i >= limit) {
          ok = 0;
          atomicExch(bar + 2, 1u);
          if (waits) atomicAdd(waits, 1ull);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

constexpr size_t kPersistSmem = (tma::kSmemBytes > IdealTile<32, 8>::SMEM)
                                    ? (tma::kSmemBytes > IdealTile<16, 16>::SMEM ? tma::kSmemBytes
                                                                                 : IdealTile<16, 16>::SMEM)
                                    : (IdealTile<32, 8>::SMEM > IdealTile<16, 16>::SMEM ? IdealTile<32, 8>::SMEM
                                                                                        : IdealTile<16, 16>::SMEM);

// The persistent step's bodies as calls, so that each keeps the register
// allocation of its own kernel instead of the union of all of them.
__device__ __noinline__ void persist_tma_tile(const PersistPtrs &q, int w, const PersistPhase &ph, int limit) {
  tma::batch_tma_item(q.d, reinterpret_cast<const CUtensorMap *>(q.gmaps), q.tma_rep, q.tma_first, w, ph.pphi, ph.pq,
                      ph.dt, q.waits, limit);
}
template <int TX, int TY>
__device__ __noinline__ void persist_cp_tile(const PersistPtrs &q, int w, const PersistPhase &ph) {
  batch_ideal_item<TX, TY>(q.d, q.cp_rep, q.cp_first, w, ph.pphi, ph.pq, ph.dt);
}
template <typename I>
__device__ __noinline__ void persist_phi_item(const PersistPtrs &q, int blk, int lane, const PersistPhase &ph) {
  batch_hb_item<I>(q.d, q.dyn, q.slab_rep, q.slab_first, blk, lane, ph.pphi, ph.arg, ph.dt, ph.ctr_off);
}
template <typename I>
__device__ __noinline__ void persist_charge_item(const PersistPtrs &q, int blk, int lane, const PersistPhase &ph) {
  batch_charge_item<I>(q.d, q.dyn, q.slab_rep, q.slab_first, blk, lane, ph.pq, ph.arg, ph.dt, ph.ctr_off);
}

// One step of an ensemble in one launch of 256-thread CTAs, two per SM (the
// ideal step's CTA bodies set the shape).  Each phase hands its items out
// round robin over the grid: ideal tiles (TMA replicas first, through the
// same CTA bodies as batch_ideal_tma_kernel and batch_ideal_kernel), or pairs
// of 128-lane slab items of the heat-bath and charge sub-steps (each half of
// the CTA one item, as batch_hb_kernel / batch_charge_kernel).  Phases are
// separated by grid_barrier; after the last one block 0 advances the
// ensemble's counter and clock, as launch_ens_advance does after the
// one-launch-per-sub-step sequence.  Results equal that sequence's bit for
// bit (same device functions, same noise indexing).
template <typename I>
__global__ void __launch_bounds__(256, 2) ens_persistent_kernel(const __grid_constant__ PersistPlan P,
                                                                const PersistPtrs q) {
  const int lane = threadIdx.x & 127, half = threadIdx.x >> 7;
  for (int f = 0; f < P.nphase; ++f) {
    const PersistPhase &ph = P.ph[f];
    if (ph.kind == kPersistIdeal) {
      const int n = P.nb_tma + P.nb_cp;
      for (int w = blockIdx.x; w < n; w += gridDim.x) {
        if (w < P.nb_tma) {
          // the TMA loads (async proxy) read what the previous phase stored
          if (threadIdx.x == 0) asm volatile("fence.proxy.async.global;\n" ::: "memory");
          persist_tma_tile(q, w, ph, P.wait_limit);
        } else if (P.tile == LGV_TILE_16x16) {
          persist_cp_tile<16, 16>(q, w - P.nb_tma, ph);
        } else {
          persist_cp_tile<32, 8>(q, w - P.nb_tma, ph);
        }
        __syncthreads();  // the tile's shared memory and barriers are reused by the next one
      }
    } else {
      const int n = (P.nb_slab + 1) / 2;
      for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const int blk = 2 * w + half;
        if (blk < P.nb_slab) {
          if (ph.kind == kPersistPhi) persist_phi_item<I>(q, blk, lane, ph);
          else persist_charge_item<I>(q, blk, lane, ph);
        }
      }
    }
    if (!grid_barrier(q.bar, gridDim.x, P.wait_limit, q.waits)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    q.dyn->ctr += P.dctr;
    q.dyn->t += P.dt_step;
  }
}

__global__ void ens_set_kernel(EnsDyn *dyn, unsigned long long ctr, double t) {
  dyn->ctr = ctr;
  dyn->t = t;
}
__global__ void ens_advance_kernel(EnsDyn *dyn, unsigned long long dctr, double dt) {
  dyn->ctr += dctr;
  dyn->t += dt;
}

// Volume averages of the 11 OAverage observables per replica.
__global__ void __launch_bounds__(128) batch_oavg_kernel(const RepDesc *__restrict__ d, const int *__restrict__ rep,
                                                         const int *__restrict__ first, int pphi, int pq,
                                                         double *partial) {
  const int r = rep[blockIdx.x];
  const RepDesc &R = d[r];
  int m, j, k;
  double acc[11];
#pragma unroll
  for (int o = 0; o < 11; ++o) acc[o] = 0;
  if (plane_coords(R, blockIdx.x - first[r], m, j, k)) {
    const long long row = ((long long)k * R.g.N + j) * R.g.H + m;
#pragma unroll
    for (int par = 0; par < 2; ++par) {
      const long long o = par * R.g.V2 + row;
      double p2 = 0;
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const double v = R.base[pphi][(long long)l * R.pstride + o];
        acc[l] += v;
        p2 += v * v;
      }
#pragma unroll
      for (int l = 4; l < 10; ++l) acc[l] += R.base[pq][(long long)l * R.pstride + o];
      acc[10] += p2;
    }
  }
  __shared__ double sm[11][4];
#pragma unroll
  for (int o = 0; o < 11; ++o) {
    warp_sum(acc[o]);
    if ((threadIdx.x & 31) == 0) sm[o][threadIdx.x >> 5] = acc[o];
  }
  __syncthreads();
  if (threadIdx.x < 11) {
    const int o = threadIdx.x;
    partial[(long long)blockIdx.x * 11 + o] = ((sm[o][0] + sm[o][1]) + sm[o][2]) + sm[o][3];
  }
}

__global__ void batch_oavg_final_kernel(const RepDesc *__restrict__ d, const int *__restrict__ first, int nrep,
                                        const int *__restrict__ count, const double *partial, double *out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrep * 11) return;
  const int r = t / 11, o = t % 11;
  double s = 0;
  for (int b = 0; b < count[r]; ++b) s += partial[(long long)(first[r] + b) * 11 + o];
  out[t] = s / (2.0 * (double)d[r].g.V2);
}

// ----------------------------------------------------------------------------
// Adjoint of the Euler-Maruyama step (noise fixed).  The step is
//   phi'_a = phi_a - dt G F_a(phi) + sqrt(2 G dt) xi_a,
//   F_a = -sum_nbr phi_a + (6 + m^2) phi_a + lambda phi^2 phi_a - H delta_a0,
// so with lam = dL/dphi' (lam_in) the adjoint of the state is
//   lam_b - dt G [(6 + m^2) lam_b + lambda (phi^2 lam_b + 2 phi_b (phi . lam))
//                 - sum_nbr lam_b] + gl_b
// (the lattice Laplacian is symmetric), and the parameter sensitivities are
//   dL/dm^2 += -dtG (phi . lam),  dL/dlambda += -dtG phi^2 (phi . lam),
//   dL/dH += dtG lam_0,  dL/dG += lam . (-dt F + sqrt(2dt)/(2 sqrt G) xi).
// One thread per site pair, flat over the V/2 pairs; the parameter sums are
// accumulated into g4[0..3] (grid_sum4).
// One thread per site pair, flat over the V/2 pairs; the parameter sums are
// accumulated into g4[0..3] (grid_sum4).
constexpr int kAdjThreads = 128;
template <typename I>
__global__ void __launch_bounds__(kAdjThreads, 4) em_adjoint_kernel(Fields phi, Fields lin, Fields lout, Geo g,
                                                                    EmAdjArgs a, double *partial, unsigned *done,
                                                                    double *g4) {
  const long long idx = (long long)blockIdx.x * kAdjThreads + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (idx < g.V2) {
    int m, j, k;
    pair_coords(idx, g, m, j, k);
    em_adjoint_pair<I>(phi, lin, lout, g, a, m, j, k, v);
  }
  grid_sum4<kAdjThreads>(v, partial, done, g4, 1.0, true);
}

// ----------------------------------------------------------------------------
// Adjoint of the ideal step (IdealPV2::step_no_reject, Stepper.cxx:68-176):
//   phi1 = rot(phi, n), n' = n + dt J(phi1), phi2 = rot(phi1, n'),
// with the currents J, summed over directions,
//   J_A,l = a2 (phi1_0 S_l - phi1_l S_0) - H phi1_l,
//   J_V,s = a2 (phi1_s1 S_s2 - phi1_s2 S_s1),   S_a = sum_nbr phi1_a.
// Three passes: rot_phi_kernel writes phi1; ideal_adj_a_kernel recomputes n'
// exactly as the forward does and back-propagates through the second
// rotation (phi1_bar partial -> PB, n'_bar -> QB, dL/dH); ideal_adj_b_kernel
// adds the currents' adjoint (a stencil over QB * phi1), back-propagates
// through the first rotation and writes lam_out = (phi_bar + gl, n_bar).
// Pair (a, b, c): charge c gets a2 (phi1_a S_b - phi1_b S_a).
__host__ __device__ constexpr int pair_a(int c) { return c < 3 ? 0 : (c == 3 ? 2 : (c == 4 ? 3 : 1)); }
__host__ __device__ constexpr int pair_b(int c) { return c < 3 ? c + 1 : (c == 3 ? 3 : (c == 4 ? 1 : 2)); }

struct SiteNbrs {
  long long own, o[6];  // x+, x-, y+, y-, z+, z-
};

__device__ __forceinline__ SiteNbrs site_nbrs(const Geo &g, int m, int j, int k, int parity) {
  const int H = g.H, N = g.N;
  const long long row = ((long long)k * N + j) * H;
  const int s = (parity + j + k) & 1;
  int xm = m - 1 + s, xp = m + s;
  if (xm < 0) xm += H;
  if (xp == H) xp = 0;
  const long long ob = (long long)(parity ^ 1) * g.V2;
  SiteNbrs r;
  r.own = (long long)parity * g.V2 + row + m;
  r.o[0] = ob + row + xp;
  r.o[1] = ob + row + xm;
  r.o[2] = ob + ((long long)k * N + wrap_inc(j, N)) * H + m;
  r.o[3] = ob + ((long long)k * N + wrap_dec(j, N)) * H + m;
  r.o[4] = ob + ((long long)wrap_inc(k, N) * N + j) * H + m;
  r.o[5] = ob + ((long long)wrap_dec(k, N) * N + j) * H + m;
  return r;
}

__global__ void __launch_bounds__(kThreads) rot_phi_kernel(Fields u, Fields P1, long long V, double k) {
  const long long n = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (n >= V) return;
  double ph[4], q[6];
#pragma unroll
  for (int l = 0; l < 4; ++l) ph[l] = u.c[l][n];
#pragma unroll
  for (int s = 0; s < 6; ++s) q[s] = u.c[4 + s][n];
  rotate_site(ph, q, k);
#pragma unroll
  for (int l = 0; l < 4; ++l) P1.c[l][n] = ph[l];
}

__global__ void __launch_bounds__(128) ideal_adj_a_kernel(Fields u, Fields lin, Fields P1, Fields PB, Fields QB, Geo g,
                                                          IdealAdjArgs a, double *partial, unsigned *done,
                                                          double *g4) {
  const long long idx = (long long)blockIdx.x * 128 + threadIdx.x;
  double hb = 0;
  if (idx < g.V2) {
    int m, j, k;
    pair_coords(idx, g, m, j, k);
#pragma unroll 1
    for (int parity = 0; parity < 2; ++parity) {
      const SiteNbrs sn = site_nbrs(g, m, j, k, parity);
      double c[4], xp[4], xm[4], yp[4], ym[4], zp[4], zm[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const double *P = P1.c[l];
        c[l] = P[sn.own];
        xp[l] = P[sn.o[0]];
        xm[l] = P[sn.o[1]];
        yp[l] = P[sn.o[2]];
        ym[l] = P[sn.o[3]];
        zp[l] = P[sn.o[4]];
        zm[l] = P[sn.o[5]];
      }
      // n' exactly as the forward computes it (ideal_tile, ideal_tma_kernel)
      double q2[6], S[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) S[l] = ((xp[l] + xm[l]) + (yp[l] + ym[l])) + (zp[l] + zm[l]);
#pragma unroll
      for (int s = 0; s < 6; ++s) q2[s] = u.c[4 + s][sn.own];
      charge_currents(c, S, a.dt, a.a2, a.H, q2);
      double ob[4], pb[4], qb[6];
#pragma unroll
      for (int l = 0; l < 4; ++l) ob[l] = lin.c[l][sn.own];
      rotate_site_adj(c, q2, a.k, ob, pb, qb);
#pragma unroll
      for (int l = 0; l < 4; ++l) PB.c[l][sn.own] = pb[l];
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        const double Q = lin.c[4 + s][sn.own] + qb[s];
        QB.c[s][sn.own] = Q;
        if (s < 3) hb += -a.dt * Q * c[s + 1];
      }
    }
  }
  double v[4] = {0.0, 0.0, hb, 0.0};
  grid_sum4<128>(v, partial, done, g4, 1.0, true);
}

__global__ void __launch_bounds__(128) ideal_adj_b_kernel(Fields u, Fields lout, Fields P1, Fields PB, Fields QB, Geo g,
                                                          IdealAdjArgs a) {
  const long long idx = (long long)blockIdx.x * 128 + threadIdx.x;
  if (idx >= g.V2) return;
  int m, j, k;
  pair_coords(idx, g, m, j, k);
#pragma unroll 1
  for (int parity = 0; parity < 2; ++parity) {
    const SiteNbrs sn = site_nbrs(g, m, j, k, parity);
    double S[4] = {0, 0, 0, 0}, Na[6] = {0, 0, 0, 0, 0, 0}, Nb[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      double P[4], Q[6];
#pragma unroll
      for (int l = 0; l < 4; ++l) P[l] = P1.c[l][sn.o[d]];
#pragma unroll
      for (int s = 0; s < 6; ++s) Q[s] = QB.c[s][sn.o[d]];
#pragma unroll
      for (int l = 0; l < 4; ++l) S[l] += P[l];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        Na[c] += Q[c] * P[pair_b(c)];
        Nb[c] += Q[c] * P[pair_a(c)];
      }
    }
    double pb[4], Qc[6];
#pragma unroll
    for (int l = 0; l < 4; ++l) pb[l] = PB.c[l][sn.own];
#pragma unroll
    for (int s = 0; s < 6; ++s) Qc[s] = QB.c[s][sn.own];
    const double da = a.dt * a.a2;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const int ia = pair_a(c), ib = pair_b(c);
      pb[ia] += da * (Qc[c] * S[ib] - Na[c]);
      pb[ib] += da * (Nb[c] - Qc[c] * S[ia]);
    }
#pragma unroll
    for (int l = 0; l < 3; ++l) pb[l + 1] += -a.dt * a.H * Qc[l];
    double ph[4], q[6], phb[4], qb[6];
#pragma unroll
    for (int l = 0; l < 4; ++l) ph[l] = u.c[l][sn.own];
#pragma unroll
    for (int s = 0; s < 6; ++s) q[s] = u.c[4 + s][sn.own];
    rotate_site_adj(ph, q, a.k, pb, phb, qb);
#pragma unroll
    for (int l = 0; l < 4; ++l) lout.c[l][sn.own] = phb[l] + a.gl[l];
#pragma unroll
    for (int s = 0; s < 6; ++s) lout.c[4 + s][sn.own] = Qc[s] + qb[s];
  }
}

// volume averages of phi_0..3 into out[0..3]
__global__ void __launch_bounds__(kThreads) phi_avg_kernel(Fields f, Geo g, double *partial, unsigned *done,
                                                           double *out) {
  const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (idx < g.V2) {
#pragma unroll
    for (int b = 0; b < 4; ++b) v[b] = f.c[b][idx] + f.c[b][g.V2 + idx];
  }
  grid_sum4<kThreads>(v, partial, done, out, 1.0 / (2.0 * (double)g.V2), false);
}

__global__ void fill_phi_kernel(Fields f, long long V, double v0, double v1, double v2, double v3) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= V) return;
  f.c[0][n] = v0;
  f.c[1][n] = v1;
  f.c[2][n] = v2;
  f.c[3][n] = v3;
}

inline unsigned nblocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// ============================================================================
// Launchers.
cudaError_t launch_aos_to_rb(const double *aos, Fields f, const Geo &g, cudaStream_t st) {
  aos_to_rb_kernel<<<nblocks(2 * g.V2, kThreads), kThreads, 0, st>>>(aos, f, g);
  return cudaGetLastError();
}
cudaError_t launch_aos_to_rb(const double *aos, Fields f, int N, cudaStream_t st) {
  return launch_aos_to_rb(aos, f, make_geo(N), st);
}

cudaError_t launch_rb_to_aos(Fields f, double *aos, const Geo &g, cudaStream_t st) {
  rb_to_aos_kernel<<<nblocks(2 * g.V2, kThreads), kThreads, 0, st>>>(f, aos, g);
  return cudaGetLastError();
}
cudaError_t launch_rb_to_aos(Fields f, double *aos, int N, cudaStream_t st) {
  return launch_rb_to_aos(f, aos, make_geo(N), st);
}

cudaError_t launch_init_phi(Fields f, int N, uint64_t sk, double scale, cudaStream_t st) {
  const Geo g = make_geo(N);
  init_phi_kernel<<<nblocks(2 * g.V2, kThreads), kThreads, 0, st>>>(f, g, sk, scale);
  return cudaGetLastError();
}

cudaError_t launch_init_charges(Fields f, int N, uint64_t sk, double sqrtchi, double *scratch,
                                cudaStream_t st) {
  const Geo g = make_geo(N);
  const long long V = 2 * g.V2;
  const unsigned nb = nblocks(V, kThreads);
  double *partial = scratch;
  double *mean = scratch + (size_t)nb * 6;
  init_charge_kernel<<<nb, kThreads, 0, st>>>(f, g, sk, sqrtchi, partial);
  charge_mean_kernel<<<1, 6 * 32, 0, st>>>(partial, (int)nb, 1.0 / (double)V, mean);
  // the red-black planes are contiguous in V, so subtract on the flat planes
  charge_sub_kernel<<<nb, kThreads, 0, st>>>(f, V, mean);
  return cudaGetLastError();
}

template <typename K>
static cudaError_t allow_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// The z-marching pass is opt-in (LGV_HB_ZPASS=1 in the environment, for half
// rows of at least one tile): on B200 at 256^3 it measured 0.22 ms per pass
// against 0.19 ms for hb_pass_kernel -- at 80 registers three CTAs of 8 warps
// per SM wait out the load of the plane above on every plane.
static bool hb_zpass_default(int N) {
  static const bool on = [] {
    const char *v = std::getenv("LGV_HB_ZPASS");
    return v && v[0] == '1';
  }();
  return on && N / 2 >= ZP_TM;
}

cudaError_t launch_hb_zpass(Fields f, int N, int parity, const HbArgs &a, cudaStream_t st) {
  const Geo g = make_geo(N);
  const long long bxy = (long long)((g.H + ZP_TM - 1) / ZP_TM) * ((N + ZP_TY - 1) / ZP_TY);
  long long zc = (long long)N * bxy / (148 * 4 * 3);  // about three waves of 4 CTAs per SM
  zc = std::max(4LL, std::min(32LL, zc));
  zc = std::min<long long>(zc, N);
  const dim3 grid((g.H + ZP_TM - 1) / ZP_TM, (N + ZP_TY - 1) / ZP_TY, (unsigned)((N + zc - 1) / zc));
  const dim3 block(ZP_TM, ZP_TY);
  const bool inj = a.prop != nullptr, mon = a.mon != nullptr;
  if (inj) {
    if (mon) hb_zpass_kernel<true, true><<<grid, block, 0, st>>>(f, g, parity, (int)zc, a);
    else hb_zpass_kernel<true, false><<<grid, block, 0, st>>>(f, g, parity, (int)zc, a);
  } else {
    if (mon) hb_zpass_kernel<false, true><<<grid, block, 0, st>>>(f, g, parity, (int)zc, a);
    else hb_zpass_kernel<false, false><<<grid, block, 0, st>>>(f, g, parity, (int)zc, a);
  }
  return cudaGetLastError();
}

cudaError_t launch_hb_pass(Fields f, int N, int parity, const HbArgs &a, cudaStream_t st) {
  if (hb_zpass_default(N)) return launch_hb_zpass(f, N, parity, a, st);
  return launch_hb_pass(f, make_geo(N), parity, a, st);
}

cudaError_t launch_hb_pass(Fields f, const Geo &g, int parity, const HbArgs &a, cudaStream_t st) {
  const bool inj = a.prop != nullptr, mon = a.mon != nullptr;
  const bool gauss = a.gauss && !inj;  // injected proposals are used as given
  if (!gauss && g.Nz == g.Ng && g.kg == 0 && hb_zpass_default(g.N)) return launch_hb_zpass(f, g.N, parity, a, st);
  const bool rows = g.H % 128 == 0;
  const dim3 grid = pass_grid(g, rows);
  const bool i32 = idx32(g);
#define LGV_HBP1(I, M, T, G)                                                                                 \
  if (rows) hb_pass_kernel<I, M, true, T, G><<<grid, 128, 0, st>>>(f, g, parity, a);                        \
  else hb_pass_kernel<I, M, false, T, G><<<grid, 128, 0, st>>>(f, g, parity, a)
#define LGV_HBP(I, M, G)                                                                                     \
  if (i32) { LGV_HBP1(I, M, int, G); } else { LGV_HBP1(I, M, long long, G); }
  if (inj) { if (mon) { LGV_HBP(true, true, false); } else { LGV_HBP(true, false, false); } }
  else if (gauss) { if (mon) { LGV_HBP(false, true, true); } else { LGV_HBP(false, false, true); } }
  else { if (mon) { LGV_HBP(false, true, false); } else { LGV_HBP(false, false, false); } }
#undef LGV_HBP
#undef LGV_HBP1
  return cudaGetLastError();
}

// ---- ordered sweeps ---------------------------------------------------------
// Slab thickness: the largest divisor of N not above `target` that leaves at
// least three slabs (an item depends on three distinct neighbours).
static int hb_slab_planes(int N, int target) {
  for (int S = std::min(target, N / 3); S >= 1; --S)
    if (N % S == 0) return S;
  return 0;
}

cudaError_t hb_plan_build(HbPlan &pl, int N, int slab_target, int spc, int lag) {
  hb_plan_free(pl);
  const int S = hb_slab_planes(N, slab_target);
  if (S < 1 || spc < kHbOrderedThreads || spc % kHbOrderedThreads || lag < 1) return cudaErrorInvalidValue;
  pl.N = N;
  pl.S = S;
  pl.nslab = N / S;
  pl.spc = spc;
  const long long item_sites = (long long)S * N * (N / 2);
  pl.cpi = (int)((item_sites + spc - 1) / spc);
  const int n = pl.nslab;
  cudaError_t e;
  for (int ns = 1; ns <= kHbMaxSweeps; ++ns) {
    // T(0, s) = s; T(p, s) = lag + max T(p-1, s-1 .. s+1); items grouped by T,
    // chunks of one group interleaved item by item.
    const int P = 2 * ns;
    std::vector<int> T((size_t)P * n);
    for (int sl = 0; sl < n; ++sl) T[sl] = sl;
    for (int ph = 1; ph < P; ++ph)
      for (int sl = 0; sl < n; ++sl) {
        int t = 0;
        for (int d = -1; d <= 1; ++d) t = std::max(t, T[(size_t)(ph - 1) * n + (sl + d + n) % n]);
        T[(size_t)ph * n + sl] = t + lag;
      }
    std::vector<int> items((size_t)P * n);
    for (int i = 0; i < P * n; ++i) items[i] = i;
    std::stable_sort(items.begin(), items.end(), [&](int x, int y) { return T[x] < T[y]; });
    std::vector<int> sched;
    sched.reserve((size_t)P * n * pl.cpi);
    for (size_t a = 0; a < items.size();) {
      size_t b = a;
      while (b < items.size() && T[items[b]] == T[items[a]]) ++b;
      for (int c = 0; c < pl.cpi; ++c)
        for (size_t q = a; q < b; ++q) sched.push_back(items[q] * pl.cpi + c);
      a = b;
    }
    pl.total[ns - 1] = (int)sched.size();
    if ((e = cudaMalloc((void **)&pl.sched[ns - 1], sched.size() * sizeof(int))) != cudaSuccess) return e;
    if ((e = cudaMemcpy(pl.sched[ns - 1], sched.data(), sched.size() * sizeof(int), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
      return e;
  }
  const size_t nsync = kSyncDone + (size_t)2 * kHbMaxSweeps * n;
  if ((e = cudaMalloc((void **)&pl.sync, nsync * sizeof(unsigned long long))) != cudaSuccess) return e;
  if ((e = cudaMemset(pl.sync, 0, nsync * sizeof(unsigned long long))) != cudaSuccess) return e;
  int dev = 0, sms = 0, occ = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, hb_ordered_kernel<false, false>, kHbOrderedThreads,
                                                          0)) != cudaSuccess)
    return e;
  pl.grid = std::max(1, sms * std::max(1, occ));
  return cudaSuccess;
}

void hb_plan_free(HbPlan &pl) {
  for (int i = 0; i < kHbMaxSweeps; ++i) {
    if (pl.sched[i]) cudaFree(pl.sched[i]);
    pl.sched[i] = nullptr;
    pl.total[i] = 0;
  }
  if (pl.sync) cudaFree(pl.sync);
  pl.sync = nullptr;
  pl.N = 0;
}

cudaError_t launch_hb_ordered(Fields f, int N, const HbArgs &a, const HbPlan &pl, int nsweeps, const uint64_t *sk,
                              cudaStream_t st) {
  if (pl.N != N || nsweeps < 1 || nsweeps > kHbMaxSweeps) return cudaErrorInvalidValue;
  const bool inj = a.prop != nullptr, mon = a.mon != nullptr;
  if ((inj || a.flags) && nsweeps != 1) return cudaErrorInvalidValue;
  HbSched s{};
  s.sched = pl.sched[nsweeps - 1];
  s.sync = pl.sync;
  s.total = pl.total[nsweeps - 1];
  s.cpi = pl.cpi;
  s.spc = pl.spc;
  s.nslab = pl.nslab;
  s.S = pl.S;
  s.nphase = 2 * nsweeps;
  s.limit = pl.wait_limit;
  for (int q = 0; q < nsweeps; ++q) s.sk[q] = sk ? sk[q] : a.sk;
  const Geo g = make_geo(N);
  const int grid = std::min(pl.grid, s.total);
  if (inj) {
    if (mon) hb_ordered_kernel<true, true><<<grid, kHbOrderedThreads, 0, st>>>(f, g, a, s);
    else hb_ordered_kernel<true, false><<<grid, kHbOrderedThreads, 0, st>>>(f, g, a, s);
  } else {
    if (mon) hb_ordered_kernel<false, true><<<grid, kHbOrderedThreads, 0, st>>>(f, g, a, s);
    else hb_ordered_kernel<false, false><<<grid, kHbOrderedThreads, 0, st>>>(f, g, a, s);
  }
  return cudaGetLastError();
}

cudaError_t hb_plan_timeouts(const HbPlan &pl, cudaStream_t st, unsigned long long *out, bool clear) {
  *out = 0;
  if (!pl.sync) return cudaSuccess;
  cudaError_t e = cudaMemcpyAsync(out, pl.sync + kSyncTimeouts, sizeof(*out), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && clear && *out) e = cudaMemsetAsync(pl.sync + kSyncTimeouts, 0, sizeof(*out), st);
  return e;
}

static int hb_zchunk(int N) {
  const int H = N / 2;
  const long long bxy = (long long)((H + HB_TM - 1) / HB_TM) * ((N + HB_TY - 1) / HB_TY);
  long long z = (long long)N * bxy / 1184;  // aim at >= 4 CTAs per SM slot
  if (z > 32) z = 32;
  if (z < 4) z = 4;
  if (z > N) z = N;
  return (int)z;
}

cudaError_t launch_hb_sweep(Fields in, Fields out, int N, const HbArgs &a, cudaStream_t st) {
  const Geo g = make_geo(N);
  const int zc = hb_zchunk(N);
  dim3 grid((g.H + HB_TM - 1) / HB_TM, (N + HB_TY - 1) / HB_TY, (N + zc - 1) / zc);
  const bool inj = a.prop != nullptr, mon = a.mon != nullptr;
  cudaError_t e;
  if (inj) {
    if (mon) {
      if ((e = allow_smem(hb_sweep_kernel<true, true>, HB_SMEM)) != cudaSuccess) return e;
      hb_sweep_kernel<true, true><<<grid, HB_TM * HB_TY, HB_SMEM, st>>>(in, out, g, zc, a);
    } else {
      if ((e = allow_smem(hb_sweep_kernel<true, false>, HB_SMEM)) != cudaSuccess) return e;
      hb_sweep_kernel<true, false><<<grid, HB_TM * HB_TY, HB_SMEM, st>>>(in, out, g, zc, a);
    }
  } else {
    if (mon) {
      if ((e = allow_smem(hb_sweep_kernel<false, true>, HB_SMEM)) != cudaSuccess) return e;
      hb_sweep_kernel<false, true><<<grid, HB_TM * HB_TY, HB_SMEM, st>>>(in, out, g, zc, a);
    } else {
      if ((e = allow_smem(hb_sweep_kernel<false, false>, HB_SMEM)) != cudaSuccess) return e;
      hb_sweep_kernel<false, false><<<grid, HB_TM * HB_TY, HB_SMEM, st>>>(in, out, g, zc, a);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_charge_pass(Fields f, int N, int dir, int eoA, const ChargeArgs &a, cudaStream_t st) {
  return launch_charge_pass(f, make_geo(N), dir, eoA, a, st);
}

cudaError_t launch_charge_pass(Fields f, const Geo &g, int dir, int eoA, const ChargeArgs &a, cudaStream_t st) {
  const bool rows = g.H % 128 == 0;
  const dim3 grid = pass_grid(g, rows);
  const bool inj = a.q != nullptr, mon = a.mon != nullptr;
  const bool i32 = idx32(g);
#define LGV_CHP1(I, M, T)                                                                                    \
  if (rows) charge_pass_kernel<I, M, true, T><<<grid, 128, 0, st>>>(f, g, dir, eoA, a);                     \
  else charge_pass_kernel<I, M, false, T><<<grid, 128, 0, st>>>(f, g, dir, eoA, a)
#define LGV_CHP(I, M)                                                                                        \
  if (i32) { LGV_CHP1(I, M, int); } else { LGV_CHP1(I, M, long long); }
  if (inj) { if (mon) { LGV_CHP(true, true); } else { LGV_CHP(true, false); } }
  else { if (mon) { LGV_CHP(false, true); } else { LGV_CHP(false, false); } }
#undef LGV_CHP
#undef LGV_CHP1
  return cudaGetLastError();
}

static int charge_seglen(int N) { return N >= 64 ? 32 : N; }

bool charge_slab_supported(int N) { return N >= 32 && N % 32 == 0 && N <= 2048; }

cudaError_t launch_charge_dir(Fields in, Fields out, int N, int dir, const ChargeDirPair &p, cudaStream_t st,
                              bool *swapped) {
  const Geo g = make_geo(N);
  ChargeDirArgs a;
  a.rms = p.rms;
  a.inv2chi = p.inv2chi;
  for (int i = 0; i < 2; ++i) {
    a.sk[i] = p.sk[i];
    a.pass[i] = p.pass[i];
    a.eo[i] = p.eo[i];
  }
  a.q = p.q;
  a.acc = p.acc;
  a.flags = p.flags;
  a.mon = p.mon;
  const bool inj = a.q != nullptr, mon = a.mon != nullptr;
  if (charge_slab_supported(N)) {
    *swapped = true;
    int sl = 0, nr = 0;
    size_t sm = 0;
    dim3 grid;
    if (dir == 0) {
      nr = (int)std::max(1, std::min(4, 512 / g.H));
      sm = (size_t)6 * nr * 2 * g.H * sizeof(double);
      grid = dim3((unsigned)(((long long)N * N + nr - 1) / nr));
    } else {
      sl = std::min(N, 32);
      sm = (size_t)6 * (sl + 4) * 32 * sizeof(double);
      grid = dim3(N / 32, N, (N + sl - 1) / sl);
    }
#define LGV_SLAB(D, I, M)                                                                   \
  do {                                                                                      \
    cudaError_t e_ = allow_smem(charge_slab_kernel<D, I, M>, sm);                           \
    if (e_ != cudaSuccess) return e_;                                                       \
    charge_slab_kernel<D, I, M><<<grid, kSlabThreads, sm, st>>>(in, out, g, a, sl, nr);     \
  } while (0)
#define LGV_SLAB_DIR(D) \
  if (inj) { if (mon) LGV_SLAB(D, true, true); else LGV_SLAB(D, true, false); } \
  else { if (mon) LGV_SLAB(D, false, true); else LGV_SLAB(D, false, false); }
    if (dir == 0) { LGV_SLAB_DIR(0) }
    else if (dir == 1) { LGV_SLAB_DIR(1) }
    else { LGV_SLAB_DIR(2) }
#undef LGV_SLAB_DIR
#undef LGV_SLAB
    return cudaGetLastError();
  }
  if (dir == 0 && g.H > 256) {
    // rows longer than one 256-thread CTA: the two faces as separate launches
    *swapped = false;
    for (int i = 0; i < 2; ++i) {
      ChargeArgs c{};
      c.rms = p.rms;
      c.inv2chi = p.inv2chi;
      c.sk = p.sk[i];
      c.pass = p.pass[i];
      c.q = p.q;
      c.acc = p.acc;
      c.flags = p.flags;
      c.mon = p.mon;
      cudaError_t e = launch_charge_pass(in, N, 0, p.eo[i], c, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  if (dir == 0) {
    *swapped = false;
    const int H = g.H;
    const int by = H >= 256 ? 1 : 256 / H;
    const long long rows = (long long)N * N;
    dim3 block(H, by), grid((unsigned)((rows + by - 1) / by));
    const size_t sm = (size_t)6 * by * H * sizeof(double);
    if (inj) {
      if (mon) charge_x_kernel<true, true><<<grid, block, sm, st>>>(in, g, a);
      else charge_x_kernel<true, false><<<grid, block, sm, st>>>(in, g, a);
    } else {
      if (mon) charge_x_kernel<false, true><<<grid, block, sm, st>>>(in, g, a);
      else charge_x_kernel<false, false><<<grid, block, sm, st>>>(in, g, a);
    }
    return cudaGetLastError();
  }
  *swapped = true;
  const int sl = charge_seglen(N);
  dim3 grid((g.H + 127) / 128, N, (N + sl - 1) / sl);
#define LGV_LINE(D, I, M) charge_line_kernel<D, I, M><<<grid, 128, 0, st>>>(in, out, g, a, sl)
  if (dir == 1) {
    if (inj) { if (mon) LGV_LINE(1, true, true); else LGV_LINE(1, true, false); }
    else { if (mon) LGV_LINE(1, false, true); else LGV_LINE(1, false, false); }
  } else {
    if (inj) { if (mon) LGV_LINE(2, true, true); else LGV_LINE(2, true, false); }
    else { if (mon) LGV_LINE(2, false, true); else LGV_LINE(2, false, false); }
  }
#undef LGV_LINE
  return cudaGetLastError();
}

cudaError_t launch_em(Fields in, Fields out, int N, const EmArgs &a, cudaStream_t st) {
  return launch_em(in, out, make_geo(N), a, st);
}

cudaError_t launch_em(Fields in, Fields out, const Geo &g, const EmArgs &a, cudaStream_t st) {
  const unsigned nb = nblocks(g.V2, kThreads);
  const bool i32 = idx32(g);
  if (a.xi) {
    if (i32) em_kernel<true, false, int><<<nb, kThreads, 0, st>>>(in, out, g, a, nullptr, nullptr, nullptr);
    else em_kernel<true, false, long long><<<nb, kThreads, 0, st>>>(in, out, g, a, nullptr, nullptr, nullptr);
  } else {
    if (i32) em_kernel<false, false, int><<<nb, kThreads, 0, st>>>(in, out, g, a, nullptr, nullptr, nullptr);
    else em_kernel<false, false, long long><<<nb, kThreads, 0, st>>>(in, out, g, a, nullptr, nullptr, nullptr);
  }
  return cudaGetLastError();
}

cudaError_t launch_em_avg(Fields in, Fields out, int N, const EmArgs &a, double *partial, unsigned *done,
                          double *avg_out, cudaStream_t st) {
  const Geo g = make_geo(N);
  const unsigned nb = nblocks(g.V2, kThreads);
  if (idx32(g)) {
    if (a.xi) em_kernel<true, true, int><<<nb, kThreads, 0, st>>>(in, out, g, a, partial, done, avg_out);
    else em_kernel<false, true, int><<<nb, kThreads, 0, st>>>(in, out, g, a, partial, done, avg_out);
  } else {
    if (a.xi) em_kernel<true, true, long long><<<nb, kThreads, 0, st>>>(in, out, g, a, partial, done, avg_out);
    else em_kernel<false, true, long long><<<nb, kThreads, 0, st>>>(in, out, g, a, partial, done, avg_out);
  }
  return cudaGetLastError();
}

cudaError_t launch_ideal(Fields in, Fields out, int N, const IdealArgs &a, cudaStream_t st) {
  return launch_ideal(in, out, make_geo(N), a, st);
}

cudaError_t launch_ideal(Fields in, Fields out, const Geo &g, const IdealArgs &a, cudaStream_t st) {
  const int N = g.N;
  constexpr int TX = 32, TY = 8;
  using T = IdealTile<TX, TY>;
  const long long bxy = (long long)((N + TX - 1) / TX) * ((N + TY - 1) / TY);
  long long zc = (long long)g.Nz * bxy / 1184;
  if (zc > 32) zc = 32;
  if (zc < 4) zc = 4;
  if (zc > g.Nz) zc = g.Nz;
  static const bool tma_off = [] {
    const char *v = std::getenv("LGV_IDEAL_TMA");
    return v && v[0] == '0';
  }();
  if (!tma_off && ideal_tma_supported(N)) return launch_ideal_tma(in, out, g, (int)zc, a, st);
  dim3 grid((N + TX - 1) / TX, (N + TY - 1) / TY, (unsigned)((g.Nz + zc - 1) / zc));
  cudaError_t e = allow_smem(ideal_kernel<TX, TY>, T::SMEM);
  if (e != cudaSuccess) return e;
  ideal_kernel<TX, TY><<<grid, TX * TY, T::SMEM, st>>>(in, out, g, (int)zc, a);
  return cudaGetLastError();
}

size_t energy_scratch_doubles(int N) {
  const long long V = (long long)N * N * N;
  return (size_t)nblocks(V, kThreads) * 3 + 8;
}

cudaError_t launch_energy(Fields f, int N, double H, double half_over_chi, double *scratch, double *dev_out,
                          cudaStream_t st) {
  const Geo g = make_geo(N);
  const unsigned nb = nblocks(2 * g.V2, kThreads);
  energy_kernel<<<nb, kThreads, 0, st>>>(f, g, scratch);
  energy_final_kernel<<<1, 96, 0, st>>>(scratch, (int)nb, H, half_over_chi, dev_out);
  return cudaGetLastError();
}

size_t measure_size(int N) {
  const size_t NK = N / 2 + 1;
  return 11 + 75 * (size_t)N + 234 * NK;
}

size_t measure_scratch_doubles(int N) { return 2 * (size_t)kNObs * N * N; }

cudaError_t launch_measure(Fields f, int N, double *scratch, double *dev_out, cudaStream_t st) {
  const Geo g = make_geo(N);
  const long long NN = (long long)N * N;
  double *T = scratch, *U = scratch + (size_t)kNObs * NN;
  meas_sum_j_kernel<<<nblocks(NN, 128), 128, 0, st>>>(f, g, T, 0, N, 0);
  meas_sum_k_kernel<<<nblocks(NN, 128), 128, 0, st>>>(f, g, U, 0, N);
  const MeasOut mo = meas_layout(dev_out, N);
  meas_walls_kernel<<<nblocks(3LL * kNObs * N, 128), 128, 0, st>>>(T, U, N, mo);
  const int NK = N / 2 + 1;
  meas_dft_kernel<<<nblocks(3LL * kNObs * NK, 128), 128, 0, st>>>(N, mo);
  meas_rotate_kernel<<<nblocks(3LL * NK, 128), 128, 0, st>>>(N, mo);
  return cudaGetLastError();
}


cudaError_t launch_measure_partials(Fields f, const Geo &g, int klo, int nk, int kout, double *T, double *U,
                                    cudaStream_t st) {
  const long long NN = (long long)g.N * g.N;
  meas_sum_j_kernel<<<nblocks((long long)g.N * nk, 128), 128, 0, st>>>(f, g, T, klo, nk, kout);
  meas_sum_k_kernel<<<nblocks(NN, 128), 128, 0, st>>>(f, g, U, klo, nk);
  return cudaGetLastError();
}

cudaError_t launch_measure_sums_aos(const double *aos, int N, double *T, double *U, cudaStream_t st) {
  const long long NN = (long long)N * N;
  meas_sum_j_aos_kernel<<<nblocks(NN, 128), 128, 0, st>>>(aos, N, T);
  meas_sum_k_aos_kernel<<<nblocks(NN, 128), 128, 0, st>>>(aos, N, U);
  return cudaGetLastError();
}

cudaError_t launch_measure_finish(const double *T, const double *U, int N, double *dev_out, cudaStream_t st) {
  const MeasOut mo = meas_layout(dev_out, N);
  meas_walls_kernel<<<nblocks(3LL * kNObs * N, 128), 128, 0, st>>>(T, U, N, mo);
  const int NK = N / 2 + 1;
  meas_dft_kernel<<<nblocks(3LL * kNObs * NK, 128), 128, 0, st>>>(N, mo);
  meas_rotate_kernel<<<nblocks(3LL * NK, 128), 128, 0, st>>>(N, mo);
  return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Batched launchers.
int ideal_tile_dims(int tile, int *tx, int *ty) {
  if (tile == LGV_TILE_16x16) {
    *tx = 16;
    *ty = 16;
  } else {
    *tx = 32;
    *ty = 8;
  }
  return 0;
}

cudaError_t launch_batch_ideal(const RepDesc *d, const int *rep, const int *first, int nblocks, int tile,
                               int phase_phi, int phase_q, double dt, cudaStream_t st) {
  cudaError_t e;
  if (tile == LGV_TILE_16x16) {
    using T = IdealTile<16, 16>;
    if ((e = allow_smem(batch_ideal_kernel<16, 16>, T::SMEM)) != cudaSuccess) return e;
    batch_ideal_kernel<16, 16><<<nblocks, 256, T::SMEM, st>>>(d, rep, first, phase_phi, phase_q, dt);
  } else {
    using T = IdealTile<32, 8>;
    if ((e = allow_smem(batch_ideal_kernel<32, 8>, T::SMEM)) != cudaSuccess) return e;
    batch_ideal_kernel<32, 8><<<nblocks, 256, T::SMEM, st>>>(d, rep, first, phase_phi, phase_q, dt);
  }
  return cudaGetLastError();
}

bool batch_idx32(const RepDesc *hd, int nrep) {
  for (int r = 0; r < nrep; ++r)
    if (!idx32(hd[r].g)) return false;
  return true;
}

cudaError_t launch_batch_hb(const RepDesc *d, const EnsDyn *dyn, const int *rep, const int *first, int nblocks,
                            int phase, int parity, double dt, int ctr_off, bool i32, cudaStream_t st) {
  if (i32) batch_hb_kernel<int><<<nblocks, 128, 0, st>>>(d, dyn, rep, first, phase, parity, dt, ctr_off);
  else batch_hb_kernel<long long><<<nblocks, 128, 0, st>>>(d, dyn, rep, first, phase, parity, dt, ctr_off);
  return cudaGetLastError();
}

cudaError_t launch_batch_charge(const RepDesc *d, const EnsDyn *dyn, const int *rep, const int *first, int nblocks,
                                int phase, int pass, double dt, int ctr_off_order, bool i32, cudaStream_t st) {
  if (i32) batch_charge_kernel<int><<<nblocks, 128, 0, st>>>(d, dyn, rep, first, phase, pass, dt, ctr_off_order);
  else batch_charge_kernel<long long><<<nblocks, 128, 0, st>>>(d, dyn, rep, first, phase, pass, dt, ctr_off_order);
  return cudaGetLastError();
}

int persist_grid(bool i32) {
  // per device (the shared-memory attribute is set on the current device)
  constexpr int kMaxDevices = 64;
  static int cached[kMaxDevices][2];
  static std::once_flag once;
  std::call_once(once, [] {
    for (auto &d : cached) d[0] = d[1] = -1;
  });
  int dev = 0, coop = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  int &c = cached[dev][i32 ? 1 : 0];
  if (c >= 0) return c;
  c = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  const void *kern = i32 ? (const void *)ens_persistent_kernel<int> : (const void *)ens_persistent_kernel<long long>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPersistSmem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, kPersistSmem) != cudaSuccess) return 0;
  c = per * sms;
  return c;
}

cudaError_t launch_ens_persistent(const PersistPlan &plan, const PersistPtrs &q, bool i32, cudaStream_t st) {
  const int grid = persist_grid(i32);
  if (grid <= 0) return cudaErrorCooperativeLaunchTooLarge;
  const void *kern = i32 ? (const void *)ens_persistent_kernel<int> : (const void *)ens_persistent_kernel<long long>;
  void *args[] = {const_cast<PersistPlan *>(&plan), const_cast<PersistPtrs *>(&q)};
  return cudaLaunchCooperativeKernel(kern, grid, 256, args, kPersistSmem, st);
}

cudaError_t launch_batch_em(const RepDesc *d, const EnsDyn *dyn, const int *rep, const int *first, int nblocks,
                            int phase_in, double dt, int ctr_off, cudaStream_t st) {
  batch_em_kernel<<<nblocks, 128, 0, st>>>(d, dyn, rep, first, phase_in, dt, ctr_off);
  return cudaGetLastError();
}

cudaError_t launch_batch_em_fwd(const RepDesc *d, const DiffDesc *dd, const int *rep, const int *first,
                                const int *count, int nblocks, int phase, unsigned long long ctr, double t, double dt,
                                int n, double *partial, unsigned *done, cudaStream_t st) {
  batch_em_fwd_kernel<<<nblocks, 128, 0, st>>>(d, dd, rep, first, count, phase, ctr, t, dt, n, partial, done);
  return cudaGetLastError();
}

cudaError_t launch_batch_em_seg(const RepDesc *d, const DiffDesc *dd, const int *rep, const int *first, int nblocks,
                                int m, unsigned long long ctr, double t, double dt, cudaStream_t st) {
  batch_em_seg_kernel<<<nblocks, 128, 0, st>>>(d, dd, rep, first, m, ctr, t, dt);
  return cudaGetLastError();
}

cudaError_t launch_batch_em_adj(const RepDesc *d, const DiffDesc *dd, const int *rep, const int *first,
                                const int *count, int nblocks, int m, int cur, int n, int b, int S,
                                unsigned long long ctr, double t, double dt, double *partial, unsigned *done,
                                cudaStream_t st) {
  batch_em_adj_kernel<<<nblocks, 128, 0, st>>>(d, dd, rep, first, count, m, cur, n, b, S, ctr, t, dt, partial, done);
  return cudaGetLastError();
}

cudaError_t launch_batch_diff_copy(const RepDesc *d, const DiffDesc *dd, const int *rep, const int *first,
                                   int nblocks, int dir, int phase, int s, int b, int S, cudaStream_t st) {
  batch_diff_copy_kernel<<<nblocks, 128, 0, st>>>(d, dd, rep, first, dir, phase, s, b, S);
  return cudaGetLastError();
}

cudaError_t launch_ens_set(EnsDyn *dyn, unsigned long long ctr, double t, cudaStream_t st) {
  ens_set_kernel<<<1, 1, 0, st>>>(dyn, ctr, t);
  return cudaGetLastError();
}

cudaError_t launch_ens_advance(EnsDyn *dyn, unsigned long long dctr, double dt, cudaStream_t st) {
  ens_advance_kernel<<<1, 1, 0, st>>>(dyn, dctr, dt);
  return cudaGetLastError();
}

cudaError_t launch_batch_oavg(const RepDesc *d, const int *rep, const int *first, int nblocks, int phase_phi,
                              int phase_q, double *partial, int nrep, double *out, cudaStream_t st) {
  // per-replica block counts sit after the partial sums: count[r] = first[r+1] - first[r] in map order
  batch_oavg_kernel<<<nblocks, 128, 0, st>>>(d, rep, first, phase_phi, phase_q, partial);
  return cudaGetLastError();
}

cudaError_t launch_batch_oavg_final(const RepDesc *d, const int *first, const int *count, int nrep,
                                    const double *partial, double *out, cudaStream_t st) {
  batch_oavg_final_kernel<<<nblocks((long long)nrep * 11, 128), 128, 0, st>>>(d, first, nrep, count, partial, out);
  return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Euler-Maruyama adjoint launchers.
size_t em_reduce_blocks(int N) {
  const Geo g = make_geo(N);
  return std::max<size_t>(nblocks(g.V2, kThreads), nblocks(g.V2, std::min(kAdjThreads, 128)));
}

cudaError_t launch_em_adjoint(Fields phi, Fields lam_in, Fields lam_out, int N, const EmAdjArgs &a, double *partial,
                              unsigned *done, double *g4, cudaStream_t st) {
  const Geo g = make_geo(N);
  if (idx32(g))
    em_adjoint_kernel<int><<<nblocks(g.V2, kAdjThreads), kAdjThreads, 0, st>>>(phi, lam_in, lam_out, g, a, partial,
                                                                              done, g4);
  else
    em_adjoint_kernel<long long><<<nblocks(g.V2, kAdjThreads), kAdjThreads, 0, st>>>(phi, lam_in, lam_out, g, a,
                                                                                    partial, done, g4);
  return cudaGetLastError();
}

cudaError_t launch_ideal_adjoint(Fields u, Fields lam_in, Fields lam_out, Fields P1, Fields PB, Fields QB, int N,
                                 const IdealAdjArgs &a, double *partial, unsigned *done, double *g4,
                                 cudaStream_t st) {
  const Geo g = make_geo(N);
  const long long V = 2 * g.V2;
  rot_phi_kernel<<<nblocks(V, kThreads), kThreads, 0, st>>>(u, P1, V, a.k);
  ideal_adj_a_kernel<<<nblocks(g.V2, 128), 128, 0, st>>>(u, lam_in, P1, PB, QB, g, a, partial, done, g4);
  ideal_adj_b_kernel<<<nblocks(g.V2, 128), 128, 0, st>>>(u, lam_out, P1, PB, QB, g, a);
  return cudaGetLastError();
}

cudaError_t launch_phi_avg(Fields f, int N, double *partial, unsigned *done, double *out, cudaStream_t st) {
  const Geo g = make_geo(N);
  phi_avg_kernel<<<nblocks(g.V2, kThreads), kThreads, 0, st>>>(f, g, partial, done, out);
  return cudaGetLastError();
}

cudaError_t launch_fill_phi(Fields f, int N, const double v[4], cudaStream_t st) {
  const Geo g = make_geo(N);
  const long long V = 2 * g.V2;
  fill_phi_kernel<<<nblocks(V, 256), 256, 0, st>>>(f, V, v[0], v[1], v[2], v[3]);
  return cudaGetLastError();
}

}  // namespace lgv

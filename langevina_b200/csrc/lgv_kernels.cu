// lgv_kernels.cu -- sm_100a kernels of the Model A / Model G stepper and
// measurer.  FP64 throughout; HBM-bound stencils, no tensor-core work.
//
// Kernel map (reference loop each one replaces):
//   hb_pass_kernel      EulerLangevinHB::step, one checkerboard parity
//                       (Stepper.cxx:309-386)
//   charge_pass_kernel  ModelGChargeHB::step, one (direction, parity) face
//                       (Stepper.cxx:471-518, modelg_update_charge_pair :419-441)
//   ideal_kernel        IdealPV2::step_no_reject fused: half rotation, charge
//                       advection stencil, half rotation (Stepper.cxx:68-202)
//   em_kernel           Euler-Maruyama Model A step (action of Stepper.cxx:354-355)
//   energy_*            IdealPV2::computeEnergy (Stepper.cxx:204-268)
//   meas_*              Measurer::computeSliceAverage / ...Phase /
//                       computeDerivedObs (measurer.cxx:10-317)
#include "lgv_internal.h"

#include <cstdio>

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
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    s_c[0][w] = m.dc;
    s_c[1][w] = m.uc;
    s_c[2][w] = m.uy;
    s_c[3][w] = m.un;
    s_d[0][w] = m.dd;
    s_d[1][w] = m.ud;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    MonLocal t;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
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
// Phi heat bath, one checkerboard parity (EulerLangevinHB::step,
// Stepper.cxx:325-381).  One thread per site of `parity`; the six neighbours
// are sites of the other parity, read from its half-plane.
template <bool INJECTED, bool MON>
__global__ void __launch_bounds__(kThreads) hb_pass_kernel(Fields f, Geo g, int parity, HbArgs a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  MonLocal mon;
  if (t < g.V2) {
    const int H = g.H, N = g.N;
    const int m = (int)(t % H);
    const long long rr = t / H;
    const int j = (int)(rr % N), k = (int)(rr / N);
    const int s = (parity + j + k) & 1;
    const int i = 2 * m + s;
    int xm = m - 1 + s, xp = m + s;
    if (xm < 0) xm += H;
    if (xp == H) xp = 0;
    const long long row = ((long long)k * N + j) * H;
    const long long rjp = ((long long)k * N + wrap_inc(j, N)) * H;
    const long long rjm = ((long long)k * N + wrap_dec(j, N)) * H;
    const long long rkp = ((long long)wrap_inc(k, N) * N + j) * H;
    const long long rkm = ((long long)wrap_dec(k, N) * N + j) * H;
    const long long own = (long long)parity * g.V2 + row + m;
    const long long ob = (long long)(parity ^ 1) * g.V2;
    const long long nat = ((long long)k * N + j) * N + i;

    Xoro rng;
    if (!INJECTED) rng = stream_at(a.sk, (uint64_t)nat);
    double po[4], pn[4];
    double hphi_o = 0., hphi_n = 0., s_o = 0., s_n = 0.;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const double *P = f.c[l];
      const double heff = (P[ob + row + xp] + P[ob + row + xm]) + (P[ob + rjp + m] + P[ob + rjm + m]) +
                          (P[ob + rkp + m] + P[ob + rkm + m]);
      po[l] = P[own];
      const double v = INJECTED ? a.prop[(long long)l * 2 * g.V2 + nat] : var1(rng.next());
      pn[l] = po[l] + a.rdtg * v;
      s_o += po[l] * po[l];
      s_n += pn[l] * pn[l];
      hphi_o += heff * po[l];
      hphi_n += heff * pn[l];
    }
    hphi_o += a.H * po[0];
    hphi_n += a.H * pn[0];
    const double dS = -(hphi_n - hphi_o) + a.Lambda2 * (s_n - s_o) + a.lam4 * (s_n * s_n - s_o * s_o);
    bool accept;
    uint8_t fl;
    if (dS < 0) {
      accept = true;
      fl = 1;
      if (MON) mon.down(dS);
    } else {
      const double r = INJECTED ? a.acc[nat] : u53(rng.next());
      accept = r < exp(-dS);
      fl = accept ? 2 : 0;
      if (MON) {
        if (accept) mon.up_yes(dS);
        else mon.up_no();
      }
    }
    if (accept) {
#pragma unroll
      for (int l = 0; l < 4; ++l) f.c[l][own] = pn[l];
    }
    if (a.flags) a.flags[nat] = fl;
  }
  if (MON) mon_flush(mon, a.mon);
}

// ----------------------------------------------------------------------------
// Charge heat bath, one face (direction `dir`, A-site parity eoA).  One thread
// per link (A, B = A + e_dir); the links of a face are disjoint, so the update
// is race free and conserves each charge exactly (Stepper.cxx:493-517).
template <bool INJECTED, bool MON>
__global__ void __launch_bounds__(kThreads) charge_pass_kernel(Fields f, Geo g, int dir, int eoA, ChargeArgs a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  MonLocal mon;
  if (t < g.V2) {
    const int H = g.H, N = g.N;
    const int m = (int)(t % H);
    const long long rr = t / H;
    const int j = (int)(rr % N), k = (int)(rr / N);
    const int s = (eoA + j + k) & 1;
    const int i = 2 * m + s;
    const long long offA = (long long)eoA * g.V2 + ((long long)k * N + j) * H + m;
    long long offB;
    const long long ob = (long long)(eoA ^ 1) * g.V2;
    if (dir == 0) {
      int mb = m + s;
      if (mb == H) mb = 0;
      offB = ob + ((long long)k * N + j) * H + mb;
    } else if (dir == 1) {
      offB = ob + ((long long)k * N + wrap_inc(j, N)) * H + m;
    } else {
      offB = ob + ((long long)wrap_inc(k, N) * N + j) * H + m;
    }
    const long long nat = ((long long)k * N + j) * N + i;
    const long long V = 2 * g.V2;
    Xoro rng;
    if (!INJECTED) rng = stream_at(a.sk, (uint64_t)nat);
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
        v = var1(rng.next());
        ra = rng.next();
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
        const double r = INJECTED ? a.acc[ii] : u53(ra);
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
  if (MON) mon_flush(mon, a.mon);
}

// ----------------------------------------------------------------------------
// Euler-Maruyama Model A step (Jacobi: reads `in`, writes phi of `out`).
template <bool INJECTED>
__global__ void __launch_bounds__(kThreads) em_kernel(Fields in, Fields out, Geo g, EmArgs a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * g.V2) return;
  const int H = g.H, N = g.N;
  const int parity = (int)(t / g.V2);
  const long long u = t - (long long)parity * g.V2;
  const int m = (int)(u % H);
  const long long rr = u / H;
  const int j = (int)(rr % N), k = (int)(rr / N);
  const int s = (parity + j + k) & 1;
  const int i = 2 * m + s;
  int xm = m - 1 + s, xp = m + s;
  if (xm < 0) xm += H;
  if (xp == H) xp = 0;
  const long long row = ((long long)k * N + j) * H;
  const long long rjp = ((long long)k * N + wrap_inc(j, N)) * H;
  const long long rjm = ((long long)k * N + wrap_dec(j, N)) * H;
  const long long rkp = ((long long)wrap_inc(k, N) * N + j) * H;
  const long long rkm = ((long long)wrap_dec(k, N) * N + j) * H;
  const long long own = (long long)parity * g.V2 + row + m;
  const long long ob = (long long)(parity ^ 1) * g.V2;
  const long long nat = ((long long)k * N + j) * N + i;
  double xi[4];
  if (INJECTED) {
#pragma unroll
    for (int l = 0; l < 4; ++l) xi[l] = a.xi[(long long)l * 2 * g.V2 + nat];
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
    const double heff = (P[ob + row + xp] + P[ob + row + xm]) + (P[ob + rjp + m] + P[ob + rjm + m]) +
                        (P[ob + rkp + m] + P[ob + rkm + m]);
    double fo = -heff + a.c6 * c[l] + a.lambda * p2 * c[l];
    if (l == 0) fo -= a.H;
    out.c[l][own] = c[l] - a.dtg * fo + a.sq * xi[l];
  }
}

// ----------------------------------------------------------------------------
// Fused ideal step (IdealPV2::step_no_reject, Stepper.cxx:68-176).
// A CTA owns a TX x TY column of sites and marches up a z-chunk.  For every
// plane it rotates phi by the half step (phi') for its sites and a one-site
// ring around them into shared memory (3 rotating plane buffers), then for the
// plane below: advects the charges with the 7-point stencil on phi', applies
// the second half rotation with the updated charges and writes the site.
// Reads each site once (80 B), writes it once (80 B) to the other buffer.
template <int TX, int TY>
__global__ void __launch_bounds__(TX *TY, 2) ideal_kernel(Fields in, Fields out, Geo g, int zchunk, IdealArgs a) {
  constexpr int SX = TX + 2, SY = TY + 2, SP = SX * SY;
  constexpr int NHALO = 2 * SX + 2 * TY;
  static_assert(NHALO <= TX * TY, "halo ring larger than the CTA");
  __shared__ double sp[3][4][SP];
  const int N = g.N;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int z0 = blockIdx.z * zchunk;
  const int z1 = min(z0 + zchunk, N);
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
    hxg = ((x0 - 1 + hx) % N + N) % N;
    hyg = ((y0 - 1 + hy) % N + N) % N;
  }

  auto load = [&](int ii, int jj, int kk, double phi[4], double q[6]) {
    const long long o = rb_off(g, ii, jj, kk);
#pragma unroll
    for (int l = 0; l < 4; ++l) phi[l] = in.c[l][o];
#pragma unroll
    for (int s = 0; s < 6; ++s) q[s] = in.c[4 + s][o];
  };

  double pm[4], pc[4], pn[4], qc[6], qn[6];
  {
    const int km = z0 == 0 ? N - 1 : z0 - 1;
    double q[6];
    load(xi, yj, km, pm, q);
    rotate_site(pm, q, a.dto2chi);
  }
  load(xi, yj, z0, pc, qc);
  rotate_site(pc, qc, a.dto2chi);
#pragma unroll
  for (int l = 0; l < 4; ++l) sp[0][l][sc] = pc[l];
  if (hs >= 0) {
    double ph[4], qh[6];
    load(hxg, hyg, z0, ph, qh);
    rotate_site(ph, qh, a.dto2chi);
#pragma unroll
    for (int l = 0; l < 4; ++l) sp[0][l][hs] = ph[l];
  }

  int bc = 0;
  for (int kc = z0; kc < z1; ++kc) {
    const int kn = (kc + 1 == N) ? 0 : kc + 1;
    const int bn = (bc == 2) ? 0 : bc + 1;
    load(xi, yj, kn, pn, qn);
    rotate_site(pn, qn, a.dto2chi);
#pragma unroll
    for (int l = 0; l < 4; ++l) sp[bn][l][sc] = pn[l];
    if (hs >= 0) {
      double ph[4], qh[6];
      load(hxg, hyg, kn, ph, qh);
      rotate_site(ph, qh, a.dto2chi);
#pragma unroll
      for (int l = 0; l < 4; ++l) sp[bn][l][hs] = ph[l];
    }
    __syncthreads();
    if (act) {
      double xp[4], xm[4], yp[4], ym[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        xp[l] = sp[bc][l][sc + 1];
        xm[l] = sp[bc][l][sc - 1];
        yp[l] = sp[bc][l][sc + SX];
        ym[l] = sp[bc][l][sc - SX];
      }
      const double *c = pc, *zp = pn, *zm = pm;
      // axial charges (Stepper.cxx:112-133)
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        const double bx = -xp[0] * c[l + 1] + c[0] * xp[l + 1] + c[0] * xm[l + 1] - xm[0] * c[l + 1];
        const double by = -yp[0] * c[l + 1] + c[0] * yp[l + 1] + c[0] * ym[l + 1] - ym[0] * c[l + 1];
        const double bz = -zp[0] * c[l + 1] + c[0] * zp[l + 1] + c[0] * zm[l + 1] - zm[0] * c[l + 1];
        qc[l] += a.dt * (bx * a.a2 + by * a.a2 + bz * a.a2 - a.H * c[l + 1]);
      }
      // vector charges, epsilon = +1 for the cyclic (s, s+1, s+2) (Stepper.cxx:135-163)
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const int s1 = 1 + (s + 1) % 3, s2 = 1 + (s + 2) % 3;
        const double bx = xp[s2] * c[s1] - c[s2] * xm[s1] - xp[s1] * c[s2] + c[s1] * xm[s2];
        const double by = yp[s2] * c[s1] - c[s2] * ym[s1] - yp[s1] * c[s2] + c[s1] * ym[s2];
        const double bz = zp[s2] * c[s1] - c[s2] * zm[s1] - zp[s1] * c[s2] + c[s1] * zm[s2];
        qc[3 + s] += a.dt * (bx * a.a2 + by * a.a2 + bz * a.a2);
      }
      // second half rotation on a copy: pc (phi') is still the z-1 neighbour of the next plane
      double pf[4] = {pc[0], pc[1], pc[2], pc[3]};
      rotate_site(pf, qc, a.dto2chi);
      const long long o = rb_off(g, xi, yj, kc);
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
    bc = bn;
  }
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
#pragma unroll
    for (int l = 0; l < 4; ++l) n[l] = f[l] / sigma;
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

// T[o][k][i] = sum_j obs(i, j, k)
__global__ void meas_sum_j_kernel(Fields f, Geo g, double *T) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = g.N;
  if (t >= (long long)N * N) return;
  const int i = (int)(t % N), k = (int)(t / N);
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
  const long long NN = (long long)N * N;
#pragma unroll
  for (int o = 0; o < kNObs; ++o) T[o * NN + (long long)k * N + i] = acc[o];
}

// U[o][j][i] = sum_k obs(i, j, k)
__global__ void meas_sum_k_kernel(Fields f, Geo g, double *U) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = g.N;
  if (t >= (long long)N * N) return;
  const int i = (int)(t % N), j = (int)(t / N);
  double acc[kNObs];
#pragma unroll
  for (int o = 0; o < kNObs; ++o) acc[o] = 0;
  for (int k = 0; k < N; ++k) {
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

inline unsigned nblocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// ============================================================================
// Launchers.
cudaError_t launch_aos_to_rb(const double *aos, Fields f, int N, cudaStream_t st) {
  const Geo g = make_geo(N);
  aos_to_rb_kernel<<<nblocks(2 * g.V2, kThreads), kThreads, 0, st>>>(aos, f, g);
  return cudaGetLastError();
}

cudaError_t launch_rb_to_aos(Fields f, double *aos, int N, cudaStream_t st) {
  const Geo g = make_geo(N);
  rb_to_aos_kernel<<<nblocks(2 * g.V2, kThreads), kThreads, 0, st>>>(f, aos, g);
  return cudaGetLastError();
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

cudaError_t launch_hb_pass(Fields f, int N, int parity, const HbArgs &a, cudaStream_t st) {
  const Geo g = make_geo(N);
  const unsigned nb = nblocks(g.V2, kThreads);
  const bool inj = a.prop != nullptr;
  const bool mon = a.mon != nullptr;
  if (inj) {
    if (mon) hb_pass_kernel<true, true><<<nb, kThreads, 0, st>>>(f, g, parity, a);
    else hb_pass_kernel<true, false><<<nb, kThreads, 0, st>>>(f, g, parity, a);
  } else {
    if (mon) hb_pass_kernel<false, true><<<nb, kThreads, 0, st>>>(f, g, parity, a);
    else hb_pass_kernel<false, false><<<nb, kThreads, 0, st>>>(f, g, parity, a);
  }
  return cudaGetLastError();
}

cudaError_t launch_charge_pass(Fields f, int N, int dir, int eoA, const ChargeArgs &a, cudaStream_t st) {
  const Geo g = make_geo(N);
  const unsigned nb = nblocks(g.V2, kThreads);
  const bool inj = a.q != nullptr;
  const bool mon = a.mon != nullptr;
  if (inj) {
    if (mon) charge_pass_kernel<true, true><<<nb, kThreads, 0, st>>>(f, g, dir, eoA, a);
    else charge_pass_kernel<true, false><<<nb, kThreads, 0, st>>>(f, g, dir, eoA, a);
  } else {
    if (mon) charge_pass_kernel<false, true><<<nb, kThreads, 0, st>>>(f, g, dir, eoA, a);
    else charge_pass_kernel<false, false><<<nb, kThreads, 0, st>>>(f, g, dir, eoA, a);
  }
  return cudaGetLastError();
}

cudaError_t launch_em(Fields in, Fields out, int N, const EmArgs &a, cudaStream_t st) {
  const Geo g = make_geo(N);
  const unsigned nb = nblocks(2 * g.V2, kThreads);
  if (a.xi) em_kernel<true><<<nb, kThreads, 0, st>>>(in, out, g, a);
  else em_kernel<false><<<nb, kThreads, 0, st>>>(in, out, g, a);
  return cudaGetLastError();
}

cudaError_t launch_ideal(Fields in, Fields out, int N, const IdealArgs &a, cudaStream_t st) {
  const Geo g = make_geo(N);
  constexpr int TX = 32, TY = 8;
  const int zchunk = N >= 128 ? 32 : (N >= 32 ? 16 : N);
  dim3 grid((N + TX - 1) / TX, (N + TY - 1) / TY, (N + zchunk - 1) / zchunk);
  ideal_kernel<TX, TY><<<grid, TX * TY, 0, st>>>(in, out, g, zchunk, a);
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
  meas_sum_j_kernel<<<nblocks(NN, 128), 128, 0, st>>>(f, g, T);
  meas_sum_k_kernel<<<nblocks(NN, 128), 128, 0, st>>>(f, g, U);
  const MeasOut mo = meas_layout(dev_out, N);
  meas_walls_kernel<<<nblocks(3LL * kNObs * N, 128), 128, 0, st>>>(T, U, N, mo);
  const int NK = N / 2 + 1;
  meas_dft_kernel<<<nblocks(3LL * kNObs * NK, 128), 128, 0, st>>>(N, mo);
  meas_rotate_kernel<<<nblocks(3LL * NK, 128), 128, 0, st>>>(N, mo);
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

}  // namespace lgv

// lgv_post.cu -- post-processing of measurement histories on the device: the
// reference's x2k.exe and x2k_rotated.exe transforms and the time correlators
// of its analysis library, for data that already sits in device memory.
//
//   lgv_x2k              x2k.cxx:94-113         r2c DFT / N of every wall row
//   lgv_x2k_rotated      x2k_rotated.cxx:92-143 k walls into the vev frame
//   lgv_time_correlator  python/Loader.py:229-254 computeOtOtp (mean statistic)
//
// All three are stateless, take device pointers and run asynchronously on the
// caller's stream.  Results are deterministic: every sum runs in a fixed order.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/lgv.h"

void lgv_internal_set_error(const char *msg);

namespace {

int fail(int code, const char *msg) {
  lgv_internal_set_error(msg);
  return code;
}

int launched(const char *where) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    lgv_internal_set_error(where);
    return LGV_ERR_CUDA;
  }
  return LGV_OK;
}

// ----------------------------------------------------------------------------
// x2k: W(k) = (1/N) sum_x W(x) e^{-2 pi i k x / N}, k = 0..N/2 (FFTW's r2c sign
// and the 1/N of x2k.cxx:107-108).  One thread per (row, k); the block first
// tabulates cos and sin of 2 pi m / N with the same sincospi call and argument
// as the measurer's DFT, and the sum runs over x in order, so the transform of
// a measured wall reproduces the measurer's k wall bit for bit.
__global__ void __launch_bounds__(256) x2k_kernel(const double *__restrict__ w, long long rows, int N,
                                                  double *__restrict__ out) {
  extern __shared__ double tw[];  // tw[m] = sin, tw[N + m] = cos of 2 pi m / N
  for (int m = threadIdx.x; m < N; m += blockDim.x) sincospi(2.0 * (double)m / (double)N, &tw[m], &tw[N + m]);
  __syncthreads();
  const int NK = N / 2 + 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= rows * NK) return;
  const long long r = t / NK;
  const int k = (int)(t - r * NK);
  const double *row = w + r * N;
  double re = 0, im = 0;
  int m = 0;  // (k x) mod N
  for (int x = 0; x < N; ++x) {
    const double v = row[x];
    re += v * tw[N + m];
    im -= v * tw[m];
    m += k;
    if (m >= N) m -= N;
  }
  out[t * 2] = re / (double)N;
  out[t * 2 + 1] = im / (double)N;
}

// Same transform for N <= kX2kTileMaxN with 32 rows per block staged in shared
// memory (row stride N + 1, odd, so the 32 lanes -- one row each -- read
// distinct banks) and the lanes of a warp sharing one k, so every twiddle read
// is a broadcast.  Warp w of the block takes k = w, w + 8, ...; the sum over x
// runs in the same order with the same table, so results equal x2k_kernel's.
constexpr int kX2kTileRows = 32, kX2kTileMaxN = 512;

__global__ void __launch_bounds__(256) x2k_tile_kernel(const double *__restrict__ w, long long rows, int N,
                                                       double *__restrict__ out) {
  extern __shared__ double sm[];
  double *tw = sm;            // 2N: sin, cos
  double *tile = sm + 2 * N;  // [32][N + 1]
  const int S = N + 1, NK = N / 2 + 1;
  for (int m = threadIdx.x; m < N; m += blockDim.x) sincospi(2.0 * (double)m / (double)N, &tw[m], &tw[N + m]);
  const long long r0 = (long long)blockIdx.x * kX2kTileRows;
  const int nr = (int)min((long long)kX2kTileRows, rows - r0);
  for (int e = threadIdx.x; e < nr * N; e += blockDim.x) {
    const int rr = e / N, x = e - rr * N;
    tile[rr * S + x] = w[(r0 + rr) * N + x];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane >= nr) return;
  const double *row = tile + lane * S;
  double *o = out + (r0 + lane) * NK * 2;
  // four k per pass over the row (k, k + 8, k + 16, k + 24): each row value
  // read from shared memory serves eight multiply-adds
  for (int k0 = warp; k0 < NK; k0 += 32) {
    double re[4] = {0, 0, 0, 0}, im[4] = {0, 0, 0, 0};
    int m[4] = {0, 0, 0, 0}, dk[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) dk[q] = (k0 + 8 * q) % N;  // k itself for every k < NK; keeps m < N beyond
    for (int x = 0; x < N; ++x) {
      const double v = row[x];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        re[q] += v * tw[N + m[q]];
        im[q] -= v * tw[m[q]];
        m[q] += dk[q];
        if (m[q] >= N) m[q] -= N;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = k0 + 8 * q;
      if (k < NK) {
        o[k * 2] = re[q] / (double)N;
        o[k * 2 + 1] = im[q] / (double)N;
      }
    }
  }
}

// ----------------------------------------------------------------------------
// x2k_rotated (x2k_rotated.cxx:92-143).  Per row, n = (Re W_a(k=0)) / |.| for
// the four phi rows a = 0..3 (the identity direction (1,0,0,0) when the norm is
// below DBL_MIN); per k: phis = n.phi(k), phir_a = phi_a - n_a phis,
// A = contract_rho(n, rho(k)), V = contract_rho(n, dual(rho(k))) with rho the
// six charge rows 4..9 and dual(rho) = (rho3..5, rho0..2).  Output rows:
// 0 phis, 1-4 phir, 5-8 A, 9-12 V.
__global__ void __launch_bounds__(128) x2k_rotated_kernel(const double *__restrict__ in, long long rows, int nf,
                                                          int NK, double *__restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= rows * NK) return;
  const long long r = t / NK;
  const int k = (int)(t - r * NK);
  const double *w = in + r * nf * NK * 2;
  auto re = [&](int a, int kk) { return w[((long long)a * NK + kk) * 2]; };
  auto im = [&](int a, int kk) { return w[((long long)a * NK + kk) * 2 + 1]; };
  double n[4], nrm = 0;
  for (int a = 0; a < 4; ++a) {
    n[a] = re(a, 0);
    nrm += n[a] * n[a];
  }
  nrm = sqrt(nrm);
  if (nrm < 2.2250738585072014e-308) {
    n[0] = 1;
    n[1] = n[2] = n[3] = 0;
  } else {
    for (int a = 0; a < 4; ++a) n[a] /= nrm;
  }
  double pr[4], pi[4], rr[6], ri[6];
  for (int a = 0; a < 4; ++a) {
    pr[a] = re(a, k);
    pi[a] = im(a, k);
  }
  for (int b = 0; b < 6; ++b) {
    rr[b] = re(4 + b, k);
    ri[b] = im(4 + b, k);
  }
  double sr = 0, si = 0;
  for (int a = 0; a < 4; ++a) {
    sr += n[a] * pr[a];
    si += n[a] * pi[a];
  }
  double *o = out + r * 13 * NK * 2;
  auto put = [&](int a, double x, double y) {
    o[((long long)a * NK + k) * 2] = x;
    o[((long long)a * NK + k) * 2 + 1] = y;
  };
  put(0, sr, si);
  for (int a = 0; a < 4; ++a) put(1 + a, pr[a] - n[a] * sr, pi[a] - n[a] * si);
  // contract_rho(n, rho) (x2k_rotated.cxx:16-26) on real and imaginary parts
  auto contract = [&](const double *q, double *c) {
    c[0] = -(n[1] * q[0]) - n[2] * q[1] - n[3] * q[2];
    c[1] = n[0] * q[0] + n[3] * q[4] - n[2] * q[5];
    c[2] = n[0] * q[1] - n[3] * q[3] + n[1] * q[5];
    c[3] = n[0] * q[2] + n[2] * q[3] - n[1] * q[4];
  };
  double cr[4], ci[4];
  contract(rr, cr);
  contract(ri, ci);
  for (int a = 0; a < 4; ++a) put(5 + a, cr[a], ci[a]);
  const double dr[6] = {rr[3], rr[4], rr[5], rr[0], rr[1], rr[2]};
  const double di[6] = {ri[3], ri[4], ri[5], ri[0], ri[1], ri[2]};
  contract(dr, cr);
  contract(di, ci);
  for (int a = 0; a < 4; ++a) put(9 + a, cr[a], ci[a]);
}

// ----------------------------------------------------------------------------
// Time correlator (computeOtOtp, Loader.py:229-254): for every series s and
// lag tau < ntmax,
//   C_s(tau) = mean over t = 0, decim, 2 decim, ... < T - tau of a_s(t) b_s(t + tau)
// (complex product, no conjugation: the caller conjugates b, as the reference's
// computeOtOtp(d, np.conj(d))), minus mean(a_s) mean(b_s) over all T when
// `conn`.  Series are columns of time-major arrays: element t of series s at
// a[t * ld + s] (real) or a[t * ld + 2 s], +1 (complex).  Output time-major too:
// out[tau * ns + s] (complex: pairs).
//
// Block: 32 series (lanes) x 4 lag groups (warps); a thread owns G consecutive
// lags and keeps their sums in registers.  For decim = 1 time runs in chunks of
// G steps: the 2G-1 values of b the chunk needs are loaded once into registers,
// so G^2 multiply-adds cost G + 2G - 1 loads (the same b value serves G lags).
// Each lag's sum still runs over t in increasing order.
template <bool CPLX>
struct Val {
  double re, im;
};

// VEC: complex pairs are 16-byte aligned (both arrays and ld even), so one
// 16-byte load brings a pair.
template <bool CPLX, bool VEC>
__device__ __forceinline__ Val<CPLX> ld_val(const double *p) {
  Val<CPLX> v;
  if (CPLX && VEC) {
    const double2 q = *reinterpret_cast<const double2 *>(p);
    v.re = q.x;
    v.im = q.y;
  } else {
    v.re = p[0];
    v.im = CPLX ? p[1] : 0.0;
  }
  return v;
}

template <bool CPLX>
__device__ __forceinline__ void mac(Val<CPLX> &acc, const Val<CPLX> &x, const Val<CPLX> &y) {
  if (CPLX) {
    acc.re += x.re * y.re - x.im * y.im;
    acc.im += x.re * y.im + x.im * y.re;
  } else {
    acc.re += x.re * y.re;
  }
}

constexpr int kCorrLagWarps = 4;

template <bool CPLX, bool VEC, int G>
__global__ void __launch_bounds__(32 * kCorrLagWarps) otot_kernel(const double *__restrict__ a,
                                                                 const double *__restrict__ b, long long T,
                                                                 long long ns, long long ld, int ntmax, int decim,
                                                                 int conn, double *__restrict__ out) {
  constexpr int W = CPLX ? 2 : 1;
  const long long s = (long long)blockIdx.x * 32 + threadIdx.x;
  const long long tau0 = ((long long)blockIdx.y * kCorrLagWarps + threadIdx.y) * G;
  if (s >= ns || tau0 >= ntmax) return;
  const double *pa = a + s * W;
  const double *pb = b + s * W;
  Val<CPLX> acc[G];
#pragma unroll
  for (int g = 0; g < G; ++g) acc[g].re = acc[g].im = 0.0;
  if (decim == 1) {
    long long t0 = 0;
    // every (t, lag) of a chunk is in range when t0 + G - 1 + tau0 + G - 1 < T
    for (; t0 + tau0 + 2 * G - 2 < T; t0 += G) {
      Val<CPLX> wb[2 * G - 1];
#pragma unroll
      for (int i = 0; i < 2 * G - 1; ++i) wb[i] = ld_val<CPLX, VEC>(pb + (t0 + tau0 + i) * ld);
#pragma unroll
      for (int u = 0; u < G; ++u) {
        const Val<CPLX> x = ld_val<CPLX, VEC>(pa + (t0 + u) * ld);
#pragma unroll
        for (int g = 0; g < G; ++g) mac<CPLX>(acc[g], x, wb[u + g]);
      }
    }
#pragma unroll
    for (int g = 0; g < G; ++g)
      for (long long t = t0; t < T - tau0 - g; ++t)
        mac<CPLX>(acc[g], ld_val<CPLX, VEC>(pa + t * ld), ld_val<CPLX, VEC>(pb + (t + tau0 + g) * ld));
  } else {
#pragma unroll
    for (int g = 0; g < G; ++g)
      for (long long t = 0; t < T - tau0 - g; t += decim)
        mac<CPLX>(acc[g], ld_val<CPLX, VEC>(pa + t * ld), ld_val<CPLX, VEC>(pb + (t + tau0 + g) * ld));
  }
  Val<CPLX> cc;
  cc.re = cc.im = 0.0;
  if (conn) {
    Val<CPLX> sa, sb;
    sa.re = sa.im = sb.re = sb.im = 0.0;
    for (long long t = 0; t < T; ++t) {
      const Val<CPLX> x = ld_val<CPLX, VEC>(pa + t * ld), y = ld_val<CPLX, VEC>(pb + t * ld);
      sa.re += x.re;
      sa.im += x.im;
      sb.re += y.re;
      sb.im += y.im;
    }
    sa.re /= (double)T;
    sa.im /= (double)T;
    sb.re /= (double)T;
    sb.im /= (double)T;
    mac<CPLX>(cc, sa, sb);
  }
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const long long tau = tau0 + g;
    if (tau >= ntmax) break;
    const double cnt = (double)((T - tau + decim - 1) / decim);
    double *o = out + (tau * ns + s) * W;
    o[0] = acc[g].re / cnt - cc.re;
    if (CPLX) o[1] = acc[g].im / cnt - cc.im;
  }
}

constexpr int kGReal = 16, kGCplx = 8;

}  // namespace

extern "C" {

int lgv_x2k(const double *walls, int64_t rows, int N, double *out, void *stream) {
  if (!walls || !out) return fail(LGV_ERR_INVALID, "lgv_x2k: NULL device pointer");
  if (rows < 0 || N < 2 || (N & 1) || N > 8192)
    return fail(LGV_ERR_INVALID, "lgv_x2k: rows >= 0, N even in [2, 8192]");
  if (rows == 0) return LGV_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (N <= kX2kTileMaxN) {
    const long long blocks = (rows + kX2kTileRows - 1) / kX2kTileRows;
    if (blocks > 0x7fffffffLL) return fail(LGV_ERR_INVALID, "lgv_x2k: too many rows for one launch");
    const size_t smem = (2 * (size_t)N + (size_t)kX2kTileRows * (N + 1)) * sizeof(double);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(x2k_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return fail(LGV_ERR_CUDA, "lgv_x2k: shared memory for the row tile");
    x2k_tile_kernel<<<(unsigned)blocks, 256, smem, st>>>(walls, rows, N, out);
    return launched("lgv_x2k: launch failed");
  }
  const long long NK = N / 2 + 1, total = rows * NK;
  const int threads = 256;
  const long long blocks = (total + threads - 1) / threads;
  if (blocks > 0x7fffffffLL) return fail(LGV_ERR_INVALID, "lgv_x2k: too many rows for one launch");
  const size_t smem = 2 * (size_t)N * sizeof(double);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(x2k_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return fail(LGV_ERR_CUDA, "lgv_x2k: shared memory for the twiddle table");
  x2k_kernel<<<(unsigned)blocks, threads, smem, st>>>(walls, rows, N, out);
  return launched("lgv_x2k: launch failed");
}

int lgv_x2k_rotated(const double *walls_k, int64_t rows, int nfields, int NK, double *out, void *stream) {
  if (!walls_k || !out) return fail(LGV_ERR_INVALID, "lgv_x2k_rotated: NULL device pointer");
  if (rows < 0 || nfields < 10 || NK < 1)
    return fail(LGV_ERR_INVALID, "lgv_x2k_rotated: rows >= 0, nfields >= 10, NK >= 1");
  if (rows == 0) return LGV_OK;
  const long long total = rows * (long long)NK;
  const long long blocks = (total + 127) / 128;
  if (blocks > 0x7fffffffLL) return fail(LGV_ERR_INVALID, "lgv_x2k_rotated: too many rows for one launch");
  x2k_rotated_kernel<<<(unsigned)blocks, 128, 0, (cudaStream_t)stream>>>(walls_k, rows, nfields, NK, out);
  return launched("lgv_x2k_rotated: launch failed");
}

int lgv_time_correlator(const double *a, const double *b, int64_t T, int64_t nseries, int64_t ld, int is_complex,
                        int ntmax, int decim, int conn, double *out, void *stream) {
  if (!a || !b || !out) return fail(LGV_ERR_INVALID, "lgv_time_correlator: NULL device pointer");
  if (T < 1 || nseries < 1 || decim < 1) return fail(LGV_ERR_INVALID, "lgv_time_correlator: T, nseries, decim >= 1");
  if (ntmax < 1 || ntmax > T) return fail(LGV_ERR_INVALID, "lgv_time_correlator: 1 <= ntmax <= T");
  if (ld < nseries * (is_complex ? 2 : 1)) return fail(LGV_ERR_INVALID, "lgv_time_correlator: ld below the row width");
  const int G = is_complex ? kGCplx : kGReal;
  const long long gs = (nseries + 31) / 32;
  const long long gl = ((long long)ntmax + G * kCorrLagWarps - 1) / (G * kCorrLagWarps);
  if (gs > 0x7fffffffLL || gl > 65535) return fail(LGV_ERR_INVALID, "lgv_time_correlator: grid too large");
  const dim3 grid((unsigned)gs, (unsigned)gl), block(32, kCorrLagWarps);
  const bool vec = ((uintptr_t)a % 16 == 0) && ((uintptr_t)b % 16 == 0) && ld % 2 == 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (is_complex && vec)
    otot_kernel<true, true, kGCplx><<<grid, block, 0, st>>>(a, b, T, nseries, ld, ntmax, decim, conn, out);
  else if (is_complex)
    otot_kernel<true, false, kGCplx><<<grid, block, 0, st>>>(a, b, T, nseries, ld, ntmax, decim, conn, out);
  else
    otot_kernel<false, false, kGReal><<<grid, block, 0, st>>>(a, b, T, nseries, ld, ntmax, decim, conn, out);
  return launched("lgv_time_correlator: launch failed");
}

}  // extern "C"

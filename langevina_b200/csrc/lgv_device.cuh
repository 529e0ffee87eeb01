// lgv_device.cuh -- device-side building blocks of the B200 stepper.
//
// Lattice layout in HBM ("red-black SoA"):
//   Fields holds one pointer per site component L = 0..9 (phi_0..3, A_1..3,
//   V_1..3, the order of data_node::x, ModelA.h:283-286).  Each component
//   plane holds V = N^3 doubles split by checkerboard parity p = (i+j+k)&1:
//     plane[p * V/2 + (k*N + j) * N/2 + (i >> 1)].
//   In a row (j, k) the sites of parity p sit at i = 2m + ((p + j + k) & 1).
//   A parity pass of the heat baths therefore reads and writes whole
//   contiguous half-rows: every load and store is coalesced and nothing of
//   the other parity is rewritten.
#pragma once

#include <cstdint>

namespace lgv {

struct Fields {
  double *c[10];
};

// Geometry helpers -----------------------------------------------------------
// A buffer holds Nz planes of N x N sites.  For a whole lattice Nz = N; a
// z-slab of a lattice split over ranks holds its own planes plus ghost planes,
// local plane 0 being global plane kg (even, so the checkerboard parity of a
// local site is that of its global site) of the Ng-plane lattice.
struct Geo {
  int N;         // lattice extent in x and y
  int H;         // N / 2
  long long V2;  // sites of one parity in the buffer: N * N * Nz / 2
  int Nz;        // planes in the buffer
  int kg;        // global plane of local plane 0 (0 for a whole lattice)
  int Ng;        // planes of the whole lattice (N)
  // 1: the blocks of a pass take the planes (or z-chunks) from the top down.
  // Every pass is independent of the order its sites are visited in, so
  // consecutive passes alternate the order and each starts on the planes the
  // previous one left in L2.
  int zrev;
};

__host__ __device__ __forceinline__ Geo make_geo(int N) {
  Geo g;
  g.N = N;
  g.H = N >> 1;
  g.V2 = (long long)N * N * (N >> 1);
  g.Nz = N;
  g.kg = 0;
  g.Ng = N;
  g.zrev = 0;
  return g;
}

__host__ __device__ __forceinline__ Geo make_slab_geo(int N, int Nz, int kg) {
  Geo g = make_geo(N);
  g.V2 = (long long)N * N * Nz / 2;
  g.Nz = Nz;
  g.kg = kg;
  return g;
}

// Natural index of the global site of local site (i, j, k): the noise streams,
// injected arrays and per-site flags are indexed by it.
__host__ __device__ __forceinline__ long long nat_index(const Geo &g, int i, int j, int k) {
  int kk = k + g.kg;
  if (kk < 0) kk += g.Ng;
  else if (kk >= g.Ng) kk -= g.Ng;
  return ((long long)kk * g.N + j) * g.N + i;
}
__host__ __device__ __forceinline__ long long global_sites(const Geo &g) { return (long long)g.N * g.N * g.Ng; }

// red-black offset of natural site (i, j, k) inside a component plane
__host__ __device__ __forceinline__ long long rb_off(const Geo &g, int i, int j, int k) {
  return (long long)((i + j + k) & 1) * g.V2 + ((long long)k * g.N + j) * g.H + (i >> 1);
}

__device__ __forceinline__ int wrap_inc(int a, int n) { return (a + 1 == n) ? 0 : a + 1; }
__device__ __forceinline__ int wrap_dec(int a, int n) { return (a == 0) ? n - 1 : a - 1; }

// Counter-indexed noise ------------------------------------------------------
// Every sub-step has a key sk; word w of it is splitmix64 output w of the
// sequence seeded with sk (split_word).  Stream n is a xoroshiro128+
// generator -- the reference's engine, rotations 55/14/36,
// xoroshiro128plus.h:86-107 -- whose 128-bit state is words 2n and 2n+1: the
// heat-bath site n draws its four proposals and then, only when dS >= 0, its
// accept uniform from it (53-bit uniforms), and the Gaussian draws
// (Euler-Maruyama, initial states) come from it.  The charge link of A-site n
// takes 32-bit uniforms straight from words 6n .. 6n+5 instead (component L:
// the proposal from the low half of word 6n+L, the accept uniform from its
// high half): six splitmix64 outputs per link cost fewer instructions than a
// stream's two seeding outputs and twelve steps, and measured faster, while
// for the heat bath the stream measured faster (0.180 against 0.196 ms per
// 256^3 pass on one B200).
static constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t make_key(uint64_t seed) { return mix64(seed + kGolden); }
__host__ __device__ __forceinline__ uint64_t sub_key(uint64_t key, uint64_t ctr) {
  return mix64(key + (ctr + 1) * kGolden);
}
__host__ __device__ __forceinline__ uint64_t split_word(uint64_t sk, uint64_t w) {
  return mix64(sk + (w + 1) * kGolden);
}

struct Xoro {
  uint64_t s0, s1;
  __device__ __forceinline__ uint64_t next() {
    const uint64_t a = s0;
    uint64_t b = s1;
    const uint64_t r = a + b;
    b ^= a;
    s0 = ((a << 55) | (a >> 9)) ^ b ^ (b << 14);
    s1 = (b << 36) | (b >> 28);
    return r;
  }
};

__device__ __forceinline__ Xoro stream_at(uint64_t sk, uint64_t n) {
  Xoro x;
  x.s0 = split_word(sk, 2 * n);
  x.s1 = split_word(sk, 2 * n + 1);
  return x;
}

// Consecutive words w0, w0 + 1, ... of the sequence of sub-step key sk.
struct WordStream {
  uint64_t z;  // sk + (w + 1) * kGolden for the next word w
  __device__ __forceinline__ uint64_t next() {
    const uint64_t r = mix64(z);
    z += kGolden;
    return r;
  }
};
__device__ __forceinline__ WordStream words_at(uint64_t sk, uint64_t w0) { return WordStream{sk + (w0 + 1) * kGolden}; }
__device__ __forceinline__ uint32_t lo32(uint64_t r) { return (uint32_t)r; }
__device__ __forceinline__ uint32_t hi32(uint64_t r) { return (uint32_t)(r >> 32); }
// uniform in (0,1) from 32 bits: (k + 1/2) 2^-32, exact and symmetric about 1/2
__device__ __forceinline__ double u32(uint32_t k) { return fma((double)k, 0x1p-32, 0x1p-33); }
// variance-1 uniform in (-sqrt3, sqrt3) from 32 bits: ((k + 1/2) 2^-31 - 1) sqrt3;
// the bracket is exact, the product rounds once
__device__ __forceinline__ double v32(uint32_t k) {
  return __dmul_rn(fma((double)k, 0x1p-31, 0x1p-32 - 1.0), 1.7320508075688772);
}

// uniform in [0,1) from the top 53 bits (exact conversion)
__device__ __forceinline__ double u53(uint64_t r) { return (double)(r >> 11) * 0x1p-53; }
// variance-1 uniform in [-sqrt3, sqrt3): (2u - 1) is exact, one rounding in the product
__device__ __forceinline__ double var1(uint64_t r) {
  const double t = 2.0 * u53(r) - 1.0;
  return __dmul_rn(t, 1.7320508075688772);
}
// Box-Muller pair, u1 = 1 - u53(ra) in (0,1], angle 2*pi*u53(rb)
__device__ __forceinline__ void box_muller(uint64_t ra, uint64_t rb, double &z0, double &z1) {
  const double u1 = 1.0 - u53(ra);
  const double u2 = u53(rb);
  const double rho = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  z0 = rho * c;
  z1 = rho * s;
}

// O(4) algebra (O4AlgebraHelper.h:17-97) ------------------------------------
// expmul(v) = (cos|v|, -sin|v|/|v| * v).  The cosine and sin(x)/x come from
// their Maclaurin series in x^2: through x^6 for |v|^2 <= 1e-4 (the first
// omitted terms, x^8/8! and x^8/9!, stay below 3e-21) and through x^12 for
// |v|^2 <= 1/16 (below 1e-17 relative); larger angles use sincos().  Below
// |v| = 1e-20 the identity is returned, as in the reference.
__device__ __forceinline__ void cos_sinc(double x2, double &c, double &sc) {
  if (x2 <= 1e-4) {
    c = fma(fma(fma(-1.0 / 720.0, x2, 1.0 / 24.0), x2, -0.5), x2, 1.0);
    sc = fma(fma(fma(-1.0 / 5040.0, x2, 1.0 / 120.0), x2, -1.0 / 6.0), x2, 1.0);
  } else if (x2 <= 0.0625) {
    // cos x = sum (-1)^n x^2n/(2n)!,  sin x / x = sum (-1)^n x^2n/(2n+1)!
    c = 1.0 / 479001600.0;                 // 1/12!
    c = fma(c, -x2, 1.0 / 3628800.0);      // 1/10!
    c = fma(c, -x2, 1.0 / 40320.0);        // 1/8!
    c = fma(c, -x2, 1.0 / 720.0);          // 1/6!
    c = fma(c, -x2, 1.0 / 24.0);           // 1/4!
    c = fma(c, -x2, 1.0 / 2.0);            // 1/2!
    c = fma(c, -x2, 1.0);
    sc = 1.0 / 6227020800.0;               // 1/13!
    sc = fma(sc, -x2, 1.0 / 39916800.0);   // 1/11!
    sc = fma(sc, -x2, 1.0 / 362880.0);     // 1/9!
    sc = fma(sc, -x2, 1.0 / 5040.0);       // 1/7!
    sc = fma(sc, -x2, 1.0 / 120.0);        // 1/5!
    sc = fma(sc, -x2, 1.0 / 6.0);          // 1/3!
    sc = fma(sc, -x2, 1.0);
  } else {
    const double a = sqrt(x2);
    double s;
    sincos(a, &s, &c);
    sc = s / a;
  }
}

__device__ __forceinline__ void expmul(const double v0, const double v1, const double v2, double w[4]) {
  const double x2 = v0 * v0 + v1 * v1 + v2 * v2;
  if (x2 > 1e-40) {
    double c, sc;
    cos_sinc(x2, c, sc);
    w[0] = c;
    w[1] = -sc * v0;
    w[2] = -sc * v1;
    w[3] = -sc * v2;
  } else {
    w[0] = 1.0;
    w[1] = w[2] = w[3] = 0.0;
  }
}

// w = v1 * v2 as quaternions (scalar, vector): (a0 b0 - a.b, a x b + b0 a + a0 b)
__device__ __forceinline__ void quatmul(const double a[4], const double b[4], double w[4]) {
  w[0] = a[0] * b[0] - (a[1] * b[1] + a[2] * b[2] + a[3] * b[3]);
  w[1] = (a[2] * b[3] - b[2] * a[3]) + b[0] * a[1] + a[0] * b[1];
  w[2] = (a[3] * b[1] - a[1] * b[3]) + b[0] * a[2] + a[0] * b[2];
  w[3] = (a[1] * b[2] - b[1] * a[2]) + b[0] * a[3] + a[0] * b[3];
}

// Charge advection of the ideal step at one site (Stepper.cxx:99-166).  The
// reference's forward and backward difference terms, summed over the three
// directions with equal spacing, reduce to
//   n_A,l += dt [a2 (c_0 S_l - c_l S_0) - H c_l]            l = 1..3
//   n_V,s += dt a2 (c_s1 S_s2 - c_s2 S_s1)                 (s, s1, s2) cyclic
// with c = phi' at the site and S the sum of phi' over its six neighbours.
// (dt a2 and dt H are multiplied out once per call site: equal up to rounding.)
__device__ __forceinline__ void charge_currents(const double c[4], const double S[4], double dt, double a2,
                                                double H, double q[6]) {
  const double da2 = dt * a2, dH = dt * H;
#pragma unroll
  for (int l = 0; l < 3; ++l) q[l] += fma(da2, fma(c[0], S[l + 1], -(c[l + 1] * S[0])), -(dH * c[l + 1]));
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int s1 = 1 + (s + 1) % 3, s2 = 1 + (s + 2) % 3;
    q[3 + s] = fma(da2, fma(c[s1], S[s2], -(c[s2] * S[s1])), q[3 + s]);
  }
}

// rotatePhi for one site (Stepper.cxx:178-202): mu = -n k with k = dt / chi,
// and the O(4) rotation phi <- L phi R with R = exp(-(muV - muA)/2),
// L = exp((muV + muA)/2) (O4Rotation, O4AlgebraHelper.h:78-97).  The
// exponents are formed directly from the charges, vR = h (nV - nA) and
// vL = -h (nV + nA) with h = k / 2: two operations per component instead of
// the four through mu (equal up to rounding).
__device__ __forceinline__ void rotation_args(const double q[6], double k, double vR[3], double vL[3]) {
  const double h = 0.5 * k;
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    vR[s] = h * (q[3 + s] - q[s]);
    vL[s] = -h * (q[3 + s] + q[s]);
  }
}

__device__ __forceinline__ void rotate_site(double phi[4], const double q[6], double dt_over_chi) {
  double vR[3], vL[3], R[4], L[4], t[4];
  rotation_args(q, dt_over_chi, vR, vL);
  expmul(vR[0], vR[1], vR[2], R);
  expmul(vL[0], vL[1], vL[2], L);
  quatmul(phi, R, t);
  quatmul(L, t, phi);
}

// ---------------------------------------------------------------------------
// Adjoint of the O(4) rotation (no counterpart in the reference).
//
// expmul_d: w = expmul(v) and, for its adjoint, sc = sin|v|/|v| and
// ds = d sc / d|v|^2, the latter from the Maclaurin series
// sum_{n>=1} (-1)^n n x^(2n-2) / (2n+1)! for |v|^2 <= 1/16 (8 terms; the next
// is below 1e-22 relative) and (cos|v| - sc) / (2|v|^2) beyond.
__device__ __forceinline__ void expmul_d(const double v[3], double w[4], double &sc, double &ds) {
  const double x2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  double c;
  cos_sinc(x2, c, sc);
  if (x2 <= 0.0625) {
    ds = 1.0 / 44460928512000.0;        //  8 / 17!
    ds = fma(ds, x2, -1.0 / 186810624000.0);  // -7 / 15!
    ds = fma(ds, x2, 1.0 / 1037836800.0);     //  6 / 13!
    ds = fma(ds, x2, -1.0 / 7983360.0);       // -5 / 11!
    ds = fma(ds, x2, 1.0 / 90720.0);          //  4 / 9!
    ds = fma(ds, x2, -1.0 / 1680.0);          // -3 / 7!
    ds = fma(ds, x2, 1.0 / 60.0);             //  2 / 5!
    ds = fma(ds, x2, -1.0 / 6.0);             // -1 / 3!
  } else {
    ds = (c - sc) / (2.0 * x2);
  }
  if (x2 > 1e-40) {  // the forward's identity below |v| = 1e-20
    w[0] = c;
    w[1] = -sc * v[0];
    w[2] = -sc * v[1];
    w[3] = -sc * v[2];
  } else {
    w[0] = 1.0;
    w[1] = w[2] = w[3] = 0.0;
  }
}

// v_bar of w = expmul(v) given w_bar: dw0/dv = -sc v, dw_j/dv_i = -sc d_ij - 2 ds v_i v_j.
__device__ __forceinline__ void expmul_adj(const double v[3], double sc, double ds, const double wb[4], double vb[3]) {
  const double vd = wb[1] * v[0] + wb[2] * v[1] + wb[3] * v[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) vb[i] = -sc * (wb[0] * v[i] + wb[1 + i]) - 2.0 * ds * v[i] * vd;
}

__device__ __forceinline__ void qconj(const double a[4], double w[4]) {
  w[0] = a[0];
  w[1] = -a[1];
  w[2] = -a[2];
  w[3] = -a[3];
}

// Adjoint of out = rotate_site(phi, q, k): given ob = d/d out, returns
// pb = d/d phi and qb = d/d q.  Quaternion products are bilinear with
// transposes given by the conjugate: for w = a b, a_bar = w_bar conj(b) and
// b_bar = conj(a) w_bar.
__device__ __forceinline__ void rotate_site_adj(const double phi[4], const double q[6], double k, const double ob[4],
                                                double pb[4], double qb[6]) {
  double vR[3], vL[3];
  rotation_args(q, k, vR, vL);
  double R[4], L[4], scR, dsR, scL, dsL;
  expmul_d(vR, R, scR, dsR);
  expmul_d(vL, L, scL, dsL);
  double t[4], cj[4], tb[4], Lb[4], Rb[4];
  quatmul(phi, R, t);
  qconj(L, cj);
  quatmul(cj, ob, tb);
  qconj(t, cj);
  quatmul(ob, cj, Lb);
  qconj(R, cj);
  quatmul(tb, cj, pb);
  qconj(phi, cj);
  quatmul(cj, tb, Rb);
  double vLb[3], vRb[3];
  expmul_adj(vL, scL, dsL, Lb, vLb);
  expmul_adj(vR, scR, dsR, Rb, vRb);
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    qb[s] = -k * (0.5 * vLb[s] + 0.5 * vRb[s]);      // via mu_A
    qb[3 + s] = -k * (0.5 * vLb[s] - 0.5 * vRb[s]);  // via mu_V
  }
}

}  // namespace lgv

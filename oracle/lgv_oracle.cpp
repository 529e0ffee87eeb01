// lgv_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the langevinA (derek-teaney/langevinA) Model A / Model G
// time stepper and measurer, used as the checker of the CUDA library and as the
// timed CPU baseline.  Nothing in the product path may load this library: only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
//
// Each routine cites the reference file:line it restates.  Three noise sources:
//   SEQUENTIAL : the reference's own serial stream -- xoroshiro128+ seeded per
//                rank from std::seed_seq (NoiseGenerator.h:68-81), libstdc++
//                uniform_real_distribution / normal_distribution / std::shuffle,
//                drawn in the reference's loop order (k, j, i; conditional
//                accept draws).  This reproduces a single-rank reference run
//                draw for draw (same g++/libstdc++).
//   COUNTER    : the counter-indexed streams of the CUDA library (restated
//                independently here: splitmix64-seeded xoroshiro128+ per site).
//   INJECTED   : caller-supplied arrays, the same ones the CUDA library consumes.
// "Ranks" emulate the reference's MPI z-slab decomposition with one thread per
// rank, each with its own serial stream, so the CPU baseline uses all cores the
// way `mpiexec -n R SuperPions.exe` would.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off, no FMA contraction so the
// reference's rounding order is kept).

#include "../include/lgv.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <barrier>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <random>
#include <string>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// xoroshiro128+ with the reference's seeding (xoroshiro128plus.h:86-107).
struct Xoro {
  using result_type = uint64_t;
  uint64_t s[2] = {0, 0};
  static constexpr uint64_t min() { return 0; }
  static constexpr uint64_t max() { return std::numeric_limits<uint64_t>::max(); }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  void seed(uint64_t v) {
    s[0] = 0x01d353e5f3993bb0ull + v;
    s[1] = 0x7b9c0df6cb193b20ull * (v + 1);
  }
  uint64_t operator()() {
    const uint64_t s0 = s[0];
    uint64_t s1 = s[1];
    const uint64_t r = s0 + s1;
    s1 ^= s0;
    s[0] = rotl(s0, 55) ^ s1 ^ (s1 << 14);
    s[1] = rotl(s1, 36);
    return r;
  }
};

// NoiseGenerator (NoiseGenerator.h:62-157): per-rank seed from seed_seq, the
// three libstdc++ distributions.
struct NoiseGen {
  Xoro rng;
  std::normal_distribution<double> nd;
  std::uniform_real_distribution<double> rt3{-std::sqrt(3.), std::sqrt(3.)};
  std::uniform_real_distribution<double> u01;
  void init(int base_seed, int rank, int size) {
    std::seed_seq seq = {base_seed};
    std::vector<unsigned int> seeds(size, 0);
    seq.generate(seeds.begin(), seeds.end());
    rng.seed(seeds[rank]);
    nd.reset();
  }
  double normal() { return nd(rng); }
  double uniform() { return u01(rng); }
  double variance1() { return rt3(rng); }
};

// ---------------------------------------------------------------------------
// Counter streams (the CUDA library's production noise), restated.
//   key        = mix(seed + G)
//   subkey(c)  = mix(key + (c + 1) G)            one value per sub-step
//   word(sk,w) = mix(sk + (w + 1) G)             splitmix64 output w
//   stream n   : xoroshiro128+ state (word(sk, 2n), word(sk, 2n + 1))
//   uniform    : (r >> 11) * 2^-53 in [0, 1)
//   variance1  : (2u - 1) * sqrt(3)
//   phi heat bath, site n: stream n -> 4 proposals, then the accept uniform
//     only if dS >= 0;  Gaussian draws: stream n
//   charge link, A-site n, component L: 32-bit uniforms from word 6n+L,
//     u32(k) = (k + 1/2) 2^-32, v32(k) = ((k + 1/2) 2^-31 - 1) sqrt(3):
//     the proposal from the low half, the accept uniform from the high half
static constexpr uint64_t G = 0x9E3779B97F4A7C15ull;
static inline uint64_t mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline uint64_t make_key(uint64_t seed) { return mix(seed + G); }
static inline uint64_t subkey(uint64_t key, uint64_t ctr) { return mix(key + (ctr + 1) * G); }
static inline uint64_t word(uint64_t sk, uint64_t w) { return mix(sk + (w + 1) * G); }
static const double SQRT3 = std::sqrt(3.0);
static inline double u53(uint64_t r) { return (double)(r >> 11) * 0x1p-53; }
static inline double v1_of(uint64_t r) { return (2.0 * u53(r) - 1.0) * SQRT3; }
static inline double u32_of(uint32_t k) { return ((double)k + 0.5) * 0x1p-32; }
static inline double v32_of(uint32_t k) { return (((double)k + 0.5) * 0x1p-31 - 1.0) * SQRT3; }
static inline uint32_t lo32(uint64_t r) { return (uint32_t)r; }
static inline uint32_t hi32(uint64_t r) { return (uint32_t)(r >> 32); }
struct CtrStream {
  Xoro x;
  CtrStream(uint64_t sk, uint64_t n) {
    x.s[0] = word(sk, 2 * n);
    x.s[1] = word(sk, 2 * n + 1);
  }
  uint64_t next() { return x(); }
};
// Box-Muller pair from two draws: u1 = 1 - u53(ra) in (0,1], angle 2 pi u53(rb).
static inline void box_muller(uint64_t ra, uint64_t rb, double &z0, double &z1) {
  const double u1 = 1.0 - u53(ra);
  const double u2 = u53(rb);
  const double rho = std::sqrt(-2.0 * std::log(u1));
  const long double ang = 2.0L * 3.141592653589793238462643383279502884L * (long double)u2;
  z0 = rho * (double)cosl(ang);
  z1 = rho * (double)sinl(ang);
}

// ---------------------------------------------------------------------------
// O4AlgebraHelper (O4AlgebraHelper.h:17-97), same operation order.
static inline double norm3(const double *v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static inline double dot3(const double *a, const double *b) {
  double r = 0;
  for (int i = 0; i < 3; ++i) r += a[i] * b[i];
  return r;
}
static inline void cross3(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - b[1] * a[2];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - b[0] * a[1];
}
static inline void quatmul(const double *v1, const double *v2, double *w) {
  w[0] = v1[0] * v2[0] - dot3(v1 + 1, v2 + 1);
  cross3(v1 + 1, v2 + 1, w + 1);
  for (int i = 0; i < 3; ++i) w[1 + i] += v2[0] * v1[1 + i];
  for (int i = 0; i < 3; ++i) w[1 + i] += v1[0] * v2[1 + i];
}
static inline void expmul(const double *v, double *w) {
  const double a = norm3(v);
  if (a > 1e-20) {
    w[0] = std::cos(a);
    const double s = -(std::sin(a) / a);
    for (int i = 0; i < 3; ++i) w[1 + i] = s * v[i];
  } else {
    w[0] = 1;
    w[1] = w[2] = w[3] = 0.0;
  }
}
static inline void o4_rotation(const double *V, const double *A, double *phi) {
  double t1[4], t2[4], t3[4];
  for (int i = 0; i < 3; ++i) {
    t1[i] = -0.5 * (V[i] - A[i]);
    t2[i] = 0.5 * (V[i] + A[i]);
  }
  expmul(t1, t3);  // R
  expmul(t2, t1);  // L
  quatmul(phi, t3, t2);
  quatmul(t1, t2, phi);
}

// ---------------------------------------------------------------------------
// Handle.
enum { SEQ = 0, CTR = 1, INJ = 2 };

struct Handle {
  lgv_params p{};
  int N = 0;
  size_t V = 0;
  std::vector<double> u, snap;  // AoS natural [k][j][i][10]
  int mode = SEQ;
  int R = 1;
  std::vector<NoiseGen> gens;
  std::vector<int> k0, k1;
  uint64_t key = 0, ctr = 0;
  // injected
  std::vector<double> hb_prop, hb_acc, ch_q, ch_acc, em_xi;
  std::array<int, 5> ch_order{0, 1, 2, 0, 1};
  bool have_hb = false, have_ch = false, have_em = false;
  // monitors [ideal, phi hb, charge hb]; per rank accumulators for thread safety
  std::vector<std::array<lgv_monitor, 3>> mon;
  bool flags_on = false;
  std::vector<uint8_t> flags;
  // counter noise only: Gaussian phi heat-bath proposals (the four normals of
  // two Box-Muller pairs from the site's first four draws) instead of the
  // reference's U(-sqrt3, sqrt3); lgv_set_hb_proposal of the CUDA library
  bool hb_gauss = false;
  double last_E[2] = {0, 0};
  std::vector<double> part;  // per-rank scratch for reductions

  inline size_t idx(int i, int j, int k) const {
    i = (i % N + N) % N;
    j = (j % N + N) % N;
    k = (k % N + N) % N;
    return ((size_t)k * N + j) * N + i;
  }
};

static void mon_down(lgv_monitor &m, double dS) { m.down_counts++; m.down_dS += dS; }
static void mon_up_yes(lgv_monitor &m, double dS) { m.up_counts++; m.up_yes++; m.up_dS += dS; }
static void mon_up_no(lgv_monitor &m) { m.up_counts++; m.up_no++; }

static void run_ranks(Handle &h, const std::function<void(int)> &fn) {
  if (h.R == 1) {
    fn(0);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(h.R);
  for (int r = 0; r < h.R; ++r) th.emplace_back(fn, r);
  for (auto &t : th) t.join();
}

static void take_snapshot(Handle &h) {
  // DMGlobalToLocal: full copy of the 10 dof (Stepper.cxx:81-82, 312-315, 477-480).
  run_ranks(h, [&](int r) {
    const size_t a = (size_t)h.k0[r] * h.N * h.N * LGV_NDOF;
    const size_t b = (size_t)h.k1[r] * h.N * h.N * LGV_NDOF;
    std::memcpy(h.snap.data() + a, h.u.data() + a, (b - a) * sizeof(double));
  });
}

// ---------------------------------------------------------------------------
// IdealPV2 (Stepper.cxx:23-268).
static void rotate_phi(Handle &h, int r, double dt) {  // Stepper.cxx:178-202
  const double chi = h.p.chi;
  for (int k = h.k0[r]; k < h.k1[r]; ++k)
    for (int j = 0; j < h.N; ++j)
      for (int i = 0; i < h.N; ++i) {
        double *s = &h.u[h.idx(i, j, k) * LGV_NDOF];
        double amu[3], vmu[3];
        for (int c = 0; c < 3; ++c) vmu[c] = -s[7 + c] / chi * dt;
        for (int c = 0; c < 3; ++c) amu[c] = -s[4 + c] / chi * dt;
        o4_rotation(vmu, amu, s);
      }
}

static void advect(Handle &h, int r, double dt) {  // Stepper.cxx:89-166
  const double Hh = h.p.H;
  const double hx = h.p.LX / h.N;
  const double a2 = std::pow(1. / hx, 2);
  const double *S = h.snap.data();
  for (int k = h.k0[r]; k < h.k1[r]; ++k)
    for (int j = 0; j < h.N; ++j)
      for (int i = 0; i < h.N; ++i) {
        const double *c = S + h.idx(i, j, k) * LGV_NDOF;
        const double *xp = S + h.idx(i + 1, j, k) * LGV_NDOF;
        const double *xm = S + h.idx(i - 1, j, k) * LGV_NDOF;
        const double *yp = S + h.idx(i, j + 1, k) * LGV_NDOF;
        const double *ym = S + h.idx(i, j - 1, k) * LGV_NDOF;
        const double *zp = S + h.idx(i, j, k + 1) * LGV_NDOF;
        const double *zm = S + h.idx(i, j, k - 1) * LGV_NDOF;
        double *o = &h.u[h.idx(i, j, k) * LGV_NDOF];
        for (int l = 0; l < 3; ++l) {
          const double ax = (-xp[0] * c[l + 1] + c[0] * xp[l + 1] + c[0] * xm[l + 1] - xm[0] * c[l + 1]) * a2;
          const double ay = (-yp[0] * c[l + 1] + c[0] * yp[l + 1] + c[0] * ym[l + 1] - ym[0] * c[l + 1]) * a2;
          const double az = (-zp[0] * c[l + 1] + c[0] * zp[l + 1] + c[0] * zm[l + 1] - zm[0] * c[l + 1]) * a2;
          o[4 + l] += dt * (ax + ay + az - Hh * c[l + 1]);
        }
        for (int s = 0; s < 3; ++s) {
          const int s1 = (s + 1) % 3, s2 = (s + 2) % 3;
          const double eps = ((double)(s - s1) * (s1 - s2) * (s2 - s)) / 2.;
          const double ax = eps * (xp[1 + s2] * c[1 + s1] - c[1 + s2] * xm[1 + s1] - xp[1 + s1] * c[1 + s2] + c[1 + s1] * xm[1 + s2]) * a2;
          const double ay = eps * (yp[1 + s2] * c[1 + s1] - c[1 + s2] * ym[1 + s1] - yp[1 + s1] * c[1 + s2] + c[1 + s1] * ym[1 + s2]) * a2;
          const double az = eps * (zp[1 + s2] * c[1 + s1] - c[1 + s2] * zm[1 + s1] - zp[1 + s1] * c[1 + s2] + c[1 + s1] * zm[1 + s2]) * a2;
          o[7 + s] += dt * (ax + ay + az);
        }
      }
}

static double energy(Handle &h) {  // Stepper.cxx:204-268
  const double Hv[4] = {h.p.H, 0., 0., 0.};
  std::vector<double> g(h.R), he(h.R), nb(h.R);
  run_ranks(h, [&](int r) {
    double grad2 = 0, nab2 = 0, hEn = 0;
    for (int k = h.k0[r]; k < h.k1[r]; ++k)
      for (int j = 0; j < h.N; ++j)
        for (int i = 0; i < h.N; ++i) {
          const double *c = &h.u[h.idx(i, j, k) * LGV_NDOF];
          const double *zp = &h.u[h.idx(i, j, k + 1) * LGV_NDOF];
          const double *yp = &h.u[h.idx(i, j + 1, k) * LGV_NDOF];
          const double *xp = &h.u[h.idx(i + 1, j, k) * LGV_NDOF];
          for (int s = 0; s < 4; ++s) {
            const double pm = c[s];
            grad2 += std::pow(zp[s] - pm, 2);
            grad2 += std::pow(yp[s] - pm, 2);
            grad2 += std::pow(xp[s] - pm, 2);
            hEn += pm * Hv[s];
          }
          for (int s = 0; s < 3; ++s) nab2 += std::pow(c[7 + s], 2);
          for (int s = 0; s < 3; ++s) nab2 += std::pow(c[4 + s], 2);
        }
    g[r] = grad2;
    he[r] = hEn;
    nb[r] = nab2;
  });
  double E = 0;
  for (int r = 0; r < h.R; ++r) {
    double le = 0;
    le += 0.5 / h.p.chi * nb[r];
    le += 0.5 * g[r];
    le -= he[r];
    E += le;
  }
  return E;
}

static void ideal_step(Handle &h, double dt) {  // Stepper.cxx:23-66, 68-176
  const double Eold = energy(h);
  run_ranks(h, [&](int r) { rotate_phi(h, r, dt / 2.0); });
  take_snapshot(h);
  run_ranks(h, [&](int r) { advect(h, r, dt); });
  run_ranks(h, [&](int r) { rotate_phi(h, r, dt / 2.0); });
  const double Enew = energy(h);
  h.last_E[0] = Eold;
  h.last_E[1] = Enew;
  const double dE = Enew - Eold;
  lgv_monitor &m = h.mon[0][0];
  if (dE > 0) {
    if (h.mode == SEQ) {
      // rank 0 draws a uniform for the statistics even without accept/reject (:43-55)
      const double prob = h.gens[0].uniform();
      if (prob > std::exp(-dE)) mon_up_no(m);
      else mon_up_yes(m, dE);
    } else {
      mon_up_yes(m, dE);
    }
  } else {
    mon_down(m, dE);
  }
}

// ---------------------------------------------------------------------------
// EulerLangevinHB (Stepper.cxx:287-389).
static inline bool is_tie(double dS, double r, bool up) {
  if (std::fabs(dS) < 1e-14) return true;
  return up && std::fabs(r - std::exp(-dS)) < 1e-12;
}

static void hb_sweep(Handle &h, double dt, double mass) {
  const double Lambda2 = 0.5 * (2. * 3. + mass);
  const double lambda = h.p.lambda, Hh = h.p.H;
  const double rdtg = std::sqrt(2. * dt * h.p.gamma);
  const uint64_t sk = (h.mode == CTR) ? subkey(h.key, h.ctr) : 0;
  if (h.mode == INJ && !h.have_hb) throw std::string("hb: injected noise missing");
  for (int ieo = 0; ieo < 2; ++ieo) {
    take_snapshot(h);
    run_ranks(h, [&](int r) {
      const double *S = h.snap.data();
      lgv_monitor &m = h.mon[r][1];
      NoiseGen &g = h.gens[r];
      for (int k = h.k0[r]; k < h.k1[r]; ++k)
        for (int j = 0; j < h.N; ++j)
          for (int i = 0; i < h.N; ++i) {
            if ((k + j + i) % 2 != ieo) continue;
            const size_t n = h.idx(i, j, k);
            const double *c = S + n * LGV_NDOF;
            const double *xp = S + h.idx(i + 1, j, k) * LGV_NDOF, *xm = S + h.idx(i - 1, j, k) * LGV_NDOF;
            const double *yp = S + h.idx(i, j + 1, k) * LGV_NDOF, *ym = S + h.idx(i, j - 1, k) * LGV_NDOF;
            const double *zp = S + h.idx(i, j, k + 1) * LGV_NDOF, *zm = S + h.idx(i, j, k - 1) * LGV_NDOF;
            CtrStream cs(sk, h.mode == CTR ? n : 0);
            double hphi_o = 0., hphi_n = 0., s_o = 0., s_n = 0.;
            double pn[4], z[4] = {0, 0, 0, 0};
            if (h.mode == CTR && h.hb_gauss) {
              const uint64_t r1 = cs.next(), r2 = cs.next(), r3 = cs.next(), r4 = cs.next();
              box_muller(r1, r2, z[0], z[1]);
              box_muller(r3, r4, z[2], z[3]);
            }
            for (int l = 0; l < 4; ++l) {
              const double heff = (xp[l] + xm[l]) + (yp[l] + ym[l]) + (zp[l] + zm[l]);
              const double po = c[l];
              double v;
              if (h.mode == SEQ) v = g.variance1();
              else if (h.mode == CTR) v = h.hb_gauss ? z[l] : v1_of(cs.next());
              else v = h.hb_prop[(size_t)l * h.V + n];
              pn[l] = po + rdtg * v;
              s_o += std::pow(po, 2);
              s_n += std::pow(pn[l], 2);
              hphi_o += heff * po;
              hphi_n += heff * pn[l];
            }
            hphi_o += (Hh * c[0]);
            hphi_n += (Hh * pn[0]);
            const double dS = -(hphi_n - hphi_o) + Lambda2 * (s_n - s_o) + lambda / 4. * (s_n * s_n - s_o * s_o);
            double *o = &h.u[n * LGV_NDOF];
            uint8_t fl;
            if (dS < 0) {
              for (int l = 0; l < 4; ++l) o[l] = pn[l];
              mon_down(m, dS);
              fl = 1;
              if (h.flags_on && is_tie(dS, 0, false)) fl |= 4;
            } else {
              double rr;
              if (h.mode == SEQ) rr = g.uniform();
              else if (h.mode == CTR) rr = u53(cs.next());
              else rr = h.hb_acc[n];
              if (rr < std::exp(-dS)) {
                for (int l = 0; l < 4; ++l) o[l] = pn[l];
                mon_up_yes(m, dS);
                fl = 2;
              } else {
                mon_up_no(m);
                fl = 0;
              }
              if (h.flags_on && is_tie(dS, rr, true)) fl |= 4;
            }
            if (h.flags_on) h.flags[n] = fl;
          }
    });
  }
  if (h.mode == CTR) h.ctr += 1;
  if (h.mode == INJ) h.have_hb = false;
}

// ---------------------------------------------------------------------------
// ModelGChargeHB (Stepper.cxx:402-522).
static const int kPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

static void charge_order(Handle &h, std::array<int, 3> &xyz, std::array<int, 2> &eo) {
  xyz = {0, 1, 2};
  eo = {0, 1};
  if (h.mode == SEQ) {  // rank 0 shuffles with its engine (:461-466)
    std::shuffle(xyz.begin(), xyz.end(), h.gens[0].rng);
    std::shuffle(eo.begin(), eo.end(), h.gens[0].rng);
  } else if (h.mode == CTR) {
    const uint64_t w = word(subkey(h.key, h.ctr), 0);
    const int pi = (int)((w & 0xffffffffull) % 6ull);
    for (int a = 0; a < 3; ++a) xyz[a] = kPerm[pi][a];
    if (w >> 63) eo = {1, 0};
  } else {
    for (int a = 0; a < 3; ++a) xyz[a] = h.ch_order[a];
    eo = {h.ch_order[3], h.ch_order[4]};
  }
}

static void charge_hb(Handle &h, double dt) {
  const double rms = std::sqrt(2. * dt * (h.p.diffusion * h.p.chi));
  const double chi = h.p.chi;
  if (h.mode == INJ && !h.have_ch) throw std::string("charge: injected noise missing");
  std::array<int, 3> xyz;
  std::array<int, 2> eo;
  charge_order(h, xyz, eo);
  const uint64_t ctr0 = h.ctr;
  for (int ixyz = 0; ixyz < 3; ++ixyz)
    for (int ieo = 0; ieo < 2; ++ieo) {
      const int pass = ixyz * 2 + ieo;
      const int dir = xyz[ixyz], eoA = eo[ieo];
      const int di = dir == 0, dj = dir == 1, dk = dir == 2;
      const uint64_t sk = (h.mode == CTR) ? subkey(h.key, ctr0 + 1 + pass) : 0;
      take_snapshot(h);
      run_ranks(h, [&](int r) {
        const double *S = h.snap.data();
        lgv_monitor &m = h.mon[r][2];
        NoiseGen &g = h.gens[r];
        for (int k = h.k0[r]; k < h.k1[r]; ++k)
          for (int j = 0; j < h.N; ++j)
            for (int i = 0; i < h.N; ++i) {
              if ((k + j + i) % 2 != eoA) continue;
              const size_t nA = h.idx(i, j, k), nB = h.idx(i + di, j + dj, k + dk);
              for (int L = 4; L < 10; ++L) {
                const double a = S[nA * LGV_NDOF + L], b = S[nB * LGV_NDOF + L];
                const size_t ii = ((size_t)(pass * 6 + (L - 4))) * h.V + nA;
                uint64_t ra = 0;
                double v;
                if (h.mode == SEQ) v = g.variance1();
                else if (h.mode == CTR) { ra = word(sk, 6 * (uint64_t)nA + (L - 4)); v = v32_of(lo32(ra)); }
                else v = h.ch_q[ii];
                // modelg_update_charge_pair (:419-441)
                double q = rms * v;
                const double dS = (std::pow(a - q, 2) + std::pow(b + q, 2) - std::pow(a, 2) - std::pow(b, 2)) / (2. * chi);
                uint8_t fl;
                if (dS < 0) {
                  mon_down(m, dS);
                  fl = 1;
                  if (h.flags_on && is_tie(dS, 0, false)) fl |= 4;
                } else {
                  double rr;
                  if (h.mode == SEQ) rr = g.uniform();
                  else if (h.mode == CTR) rr = u32_of(hi32(ra));
                  else rr = h.ch_acc[ii];
                  if (rr < std::exp(-dS)) {
                    mon_up_yes(m, dS);
                    fl = 2;
                  } else {
                    mon_up_no(m);
                    q = 0.;
                    fl = 0;
                  }
                  if (h.flags_on && is_tie(dS, rr, true)) fl |= 4;
                }
                if (h.flags_on) h.flags[ii] = fl;
                // dn[A] = -q, dn[B] = q, then LocalToGlobal(ADD_VALUES) (:508-517)
                h.u[nA * LGV_NDOF + L] = a + (-q);
                h.u[nB * LGV_NDOF + L] = b + q;
              }
            }
      });
    }
  if (h.mode == CTR) h.ctr = ctr0 + 7;
  if (h.mode == INJ) h.have_ch = false;
}

// ---------------------------------------------------------------------------
// Euler-Maruyama Model A step.  Not in the reference tree: derived from the
// action whose local change EulerLangevinHB uses (Stepper.cxx:298, 332-355),
//   dS/dphi_a = -sum_nbr phi_a + (6 + m^2) phi_a + lambda phi^2 phi_a - H delta_a0,
//   phi_a <- phi_a - dt Gamma dS/dphi_a + sqrt(2 Gamma dt) xi_a.
static void em_step(Handle &h, double dt, double mass) {
  const double c6 = 6.0 + mass;
  const double dtg = dt * h.p.gamma;
  const double sq = std::sqrt(2.0 * h.p.gamma * dt);
  const uint64_t sk = (h.mode == CTR) ? subkey(h.key, h.ctr) : 0;
  if (h.mode == SEQ) throw std::string("em: no sequential stream in the reference");
  if (h.mode == INJ && !h.have_em) throw std::string("em: injected noise missing");
  take_snapshot(h);
  run_ranks(h, [&](int r) {
    const double *S = h.snap.data();
    for (int k = h.k0[r]; k < h.k1[r]; ++k)
      for (int j = 0; j < h.N; ++j)
        for (int i = 0; i < h.N; ++i) {
          const size_t n = h.idx(i, j, k);
          const double *c = S + n * LGV_NDOF;
          const double *xp = S + h.idx(i + 1, j, k) * LGV_NDOF, *xm = S + h.idx(i - 1, j, k) * LGV_NDOF;
          const double *yp = S + h.idx(i, j + 1, k) * LGV_NDOF, *ym = S + h.idx(i, j - 1, k) * LGV_NDOF;
          const double *zp = S + h.idx(i, j, k + 1) * LGV_NDOF, *zm = S + h.idx(i, j, k - 1) * LGV_NDOF;
          double xi[4];
          if (h.mode == CTR) {
            CtrStream cs(sk, n);
            const uint64_t r1 = cs.next(), r2 = cs.next(), r3 = cs.next(), r4 = cs.next();
            box_muller(r1, r2, xi[0], xi[1]);
            box_muller(r3, r4, xi[2], xi[3]);
          } else {
            for (int l = 0; l < 4; ++l) xi[l] = h.em_xi[(size_t)l * h.V + n];
          }
          const double p2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
          double *o = &h.u[n * LGV_NDOF];
          for (int l = 0; l < 4; ++l) {
            const double heff = (xp[l] + xm[l]) + (yp[l] + ym[l]) + (zp[l] + zm[l]);
            double f = -heff + c6 * c[l] + h.p.lambda * p2 * c[l];
            if (l == 0) f -= h.p.H;
            o[l] = c[l] - dtg * f + sq * xi[l];
          }
        }
  });
  if (h.mode == CTR) h.ctr += 1;
  if (h.mode == INJ) h.have_em = false;
}

// ---------------------------------------------------------------------------
// Measurer (measurer.cxx:10-317).
template <typename T>
static inline std::array<T, 4> contract_rho(const std::array<T, 4> &n, const std::array<T, 6> &rho) {
  return {-(n[1] * rho[0]) - n[2] * rho[1] - n[3] * rho[2], n[0] * rho[0] + n[3] * rho[4] - n[2] * rho[5],
          n[0] * rho[1] - n[3] * rho[3] + n[1] * rho[5], n[0] * rho[2] + n[2] * rho[3] - n[1] * rho[4]};
}
template <typename T>
static inline std::array<T, 6> dualize_rho(const std::array<T, 6> &rho) {
  return {rho[3], rho[4], rho[5], rho[0], rho[1], rho[2]};
}

static void dft_rows(const std::vector<double> &in, int rows, int N, std::vector<double> &out) {
  // W(k) = (1/N) sum_x W(x) e^{-2 pi i k x / N}, k = 0..N/2 (FFTW r2c sign, measurer.h:33-41)
  const int NK = N / 2 + 1;
  out.assign((size_t)rows * NK * 2, 0.0);
  for (int r = 0; r < rows; ++r)
    for (int k = 0; k < NK; ++k) {
      long double re = 0, im = 0;
      for (int x = 0; x < N; ++x) {
        const long long m = ((long long)k * x) % N;
        const long double ang = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)N;
        re += (long double)in[(size_t)r * N + x] * cosl(ang);
        im -= (long double)in[(size_t)r * N + x] * sinl(ang);
      }
      out[((size_t)r * NK + k) * 2 + 0] = (double)(re / N);
      out[((size_t)r * NK + k) * 2 + 1] = (double)(im / N);
    }
}

static void rotate_to_vev(const std::vector<double> &wk, int NK, std::vector<double> &out) {  // :231-286
  typedef std::complex<double> C;
  auto at = [&](int a, int k) { return C(wk[((size_t)a * NK + k) * 2], wk[((size_t)a * NK + k) * 2 + 1]); };
  out.assign((size_t)LGV_NOBS_PHASE * NK * 2, 0.0);
  std::array<C, 4> n{}, phi{}, phir{};
  std::array<C, 6> rho{};
  double nrm = 0.;
  for (int a = 0; a < 4; ++a) {
    n[a] = at(a, 0);
    nrm += std::norm(n[a]);
  }
  nrm = std::sqrt(nrm);
  if (nrm < std::numeric_limits<double>::min()) n = {C(1), C(0), C(0), C(0)};
  else for (int a = 0; a < 4; ++a) n[a] /= nrm;
  auto put = [&](int a, int k, C v) {
    out[((size_t)a * NK + k) * 2] = v.real();
    out[((size_t)a * NK + k) * 2 + 1] = v.imag();
  };
  for (int k = 0; k < NK; ++k) {
    for (int a = 0; a < 4; ++a) phi[a] = at(a, k);
    for (int ab = 0; ab < 6; ++ab) rho[ab] = at(4 + ab, k);
    C phi2k = at(10, k);
    C phis(0.);
    for (int a = 0; a < 4; ++a) phis += n[a] * phi[a];
    for (int a = 0; a < 4; ++a) phir[a] = phi[a] - n[a] * phis;
    auto A = contract_rho(n, rho);
    auto Vv = contract_rho(n, dualize_rho(rho));
    put(0, k, phis);
    for (int a = 0; a < 4; ++a) {
      put(1 + a, k, phir[a]);
      put(5 + a, k, A[a]);
      put(9 + a, k, Vv[a]);
    }
    put(13, k, phi2k);
  }
}

static void measure(Handle &h, lgv_measurement *out) {
  const int N = h.N, NK = N / 2 + 1;
  const int NO = LGV_NOBS, NP = LGV_NOBS_PHASE;
  std::vector<std::vector<double>> W(3 * h.R, std::vector<double>((size_t)NO * N, 0.0));
  std::vector<std::vector<double>> P(3 * h.R, std::vector<double>((size_t)NP * N, 0.0));
  run_ranks(h, [&](int r) {
    auto &wx = W[3 * r], &wy = W[3 * r + 1], &wz = W[3 * r + 2];
    auto &px = P[3 * r], &py = P[3 * r + 1], &pz = P[3 * r + 2];
    for (int k = h.k0[r]; k < h.k1[r]; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          const double *f = &h.u[h.idx(i, j, k) * LGV_NDOF];
          // computeSliceAverage (:46-76)
          double phi2 = 0.0;
          for (int l = 0; l < 4; ++l) {
            wx[l * N + i] += f[l];
            wy[l * N + j] += f[l];
            wz[l * N + k] += f[l];
            phi2 += std::pow(f[l], 2);
          }
          for (int l = 4; l < 10; ++l) {
            wx[l * N + i] += f[l];
            wy[l * N + j] += f[l];
            wz[l * N + k] += f[l];
          }
          wx[10 * N + i] += phi2;
          wy[10 * N + j] += phi2;
          wz[10 * N + k] += phi2;
          // computeSliceAveragePhase (:152-199)
          std::array<double, 4> n{}, ph{};
          std::array<double, 6> rho{};
          double p2 = 0.0;
          for (int l = 0; l < 4; ++l) {
            ph[l] = f[l];
            p2 += std::pow(ph[l], 2);
          }
          const double sigma = std::sqrt(p2);
          if (p2 > 100. * std::numeric_limits<double>::min()) {
            for (int l = 0; l < 4; ++l) n[l] = ph[l] / sigma;
          } else {
            n = {1, 0, 0, 0};
          }
          for (int l = 0; l < 3; ++l) {
            rho[l] = f[4 + l];
            rho[l + 3] = f[7 + l];
          }
          auto A = contract_rho(n, rho);
          auto Vv = contract_rho(n, dualize_rho(rho));
          px[0 * N + i] += sigma;
          py[0 * N + j] += sigma;
          pz[0 * N + k] += sigma;
          for (int l = 0; l < 4; ++l) {
            px[(1 + l) * N + i] += n[l];
            py[(1 + l) * N + j] += n[l];
            pz[(1 + l) * N + k] += n[l];
            px[(5 + l) * N + i] += A[l];
            py[(5 + l) * N + j] += A[l];
            pz[(5 + l) * N + k] += A[l];
            px[(9 + l) * N + i] += Vv[l];
            py[(9 + l) * N + j] += Vv[l];
            pz[(9 + l) * N + k] += Vv[l];
          }
          px[13 * N + i] += sigma * sigma;
          py[13 * N + j] += sigma * sigma;
          pz[13 * N + k] += sigma * sigma;
        }
    const double nn = (double)(N * N);
    for (int a = 0; a < 3; ++a) {
      for (auto &x : W[3 * r + a]) x /= nn;
      for (auto &x : P[3 * r + a]) x /= nn;
    }
  });
  // MPI_Reduce(SUM) to rank 0 in rank order
  std::vector<double> w[3], pw[3];
  for (int a = 0; a < 3; ++a) {
    w[a] = W[a];
    pw[a] = P[a];
    for (int r = 1; r < h.R; ++r) {
      for (size_t q = 0; q < w[a].size(); ++q) w[a][q] += W[3 * r + a][q];
      for (size_t q = 0; q < pw[a].size(); ++q) pw[a][q] += P[3 * r + a][q];
    }
  }
  // computeDerivedObs (:288-317)
  if (out->OAverage) {
    for (int l = 0; l < NO; ++l) {
      double s = 0.;
      for (int i = 0; i < N; ++i) s += w[0][l * N + i];
      out->OAverage[l] = s / (double)N;
    }
  }
  for (int a = 0; a < 3; ++a) {
    if (out->wall[a]) std::memcpy(out->wall[a], w[a].data(), w[a].size() * sizeof(double));
    if (out->wall_phase[a]) std::memcpy(out->wall_phase[a], pw[a].data(), pw[a].size() * sizeof(double));
    std::vector<double> wk, wkr, pk;
    dft_rows(w[a], NO, N, wk);
    if (out->wall_k[a]) std::memcpy(out->wall_k[a], wk.data(), wk.size() * sizeof(double));
    rotate_to_vev(wk, NK, wkr);
    if (out->wall_k_rotated[a]) std::memcpy(out->wall_k_rotated[a], wkr.data(), wkr.size() * sizeof(double));
    dft_rows(pw[a], NP, N, pk);
    if (out->wall_phase_k[a]) std::memcpy(out->wall_phase_k[a], pk.data(), pk.size() * sizeof(double));
  }
}

// ---------------------------------------------------------------------------
// Initial conditions.
static void initialize(Handle &h, int kind, double scale) {
  const size_t V = h.V;
  if (kind == LGV_INIT_ZERO) {  // ModelA.h:443-458 without a function
    std::fill(h.u.begin(), h.u.end(), 0.0);
    return;
  }
  if (kind == LGV_INIT_PHI_GAUSSIAN) {
    if (h.mode == SEQ) {
      for (int r = 0; r < h.R; ++r)
        for (int k = h.k0[r]; k < h.k1[r]; ++k)
          for (int j = 0; j < h.N; ++j)
            for (int i = 0; i < h.N; ++i)
              for (int l = 0; l < 4; ++l) h.u[h.idx(i, j, k) * LGV_NDOF + l] = scale * h.gens[r].normal();
    } else {
      const uint64_t sk = subkey(h.key, h.ctr);
      for (size_t n = 0; n < V; ++n) {
        CtrStream cs(sk, n);
        double z[4];
        const uint64_t r1 = cs.next(), r2 = cs.next(), r3 = cs.next(), r4 = cs.next();
        box_muller(r1, r2, z[0], z[1]);
        box_muller(r3, r4, z[2], z[3]);
        for (int l = 0; l < 4; ++l) h.u[n * LGV_NDOF + l] = scale * z[l];
      }
      h.ctr += 1;
    }
    return;
  }
  if (kind == LGV_INIT_CHARGES_GAUSSIAN) {  // ModelA.h:463-525
    const double sc = std::sqrt(h.p.chi);
    std::vector<double> sum(LGV_NDOF, 0.);
    if (h.mode == SEQ) {
      for (int r = 0; r < h.R; ++r) {
        std::vector<double> loc(LGV_NDOF, 0.);
        for (int k = h.k0[r]; k < h.k1[r]; ++k)
          for (int j = 0; j < h.N; ++j)
            for (int i = 0; i < h.N; ++i)
              for (int L = 4; L < 10; ++L) {
                double &x = h.u[h.idx(i, j, k) * LGV_NDOF + L];
                x = sc * h.gens[r].normal();
                loc[L] += x;
              }
        for (int L = 0; L < LGV_NDOF; ++L) sum[L] += loc[L];
      }
    } else {
      const uint64_t sk = subkey(h.key, h.ctr);
      for (size_t n = 0; n < V; ++n) {
        CtrStream cs(sk, n);
        double z[6];
        for (int pr = 0; pr < 3; ++pr) {
          const uint64_t ra = cs.next(), rb = cs.next();
          box_muller(ra, rb, z[2 * pr], z[2 * pr + 1]);
        }
        for (int L = 4; L < 10; ++L) {
          double &x = h.u[n * LGV_NDOF + L];
          x = sc * z[L - 4];
          sum[L] += x;
        }
      }
      h.ctr += 1;
    }
    const double Vd = (double)h.N * h.N * h.N;
    for (size_t n = 0; n < V; ++n)
      for (int L = 4; L < 10; ++L) h.u[n * LGV_NDOF + L] -= sum[L] / Vd;
    return;
  }
  throw std::string("initialize: unknown kind");
}

// ---------------------------------------------------------------------------
// PV2HBSplit and the evolver switch (Stepper.cxx:542-580, SuperPions.cxx:209-225).
static void step_once(Handle &h, int ev, int inner, int outer, double dt, double t) {
  const double mass = h.p.mass0 + h.p.dmassdt * t;
  switch (ev) {
    case LGV_PV2HBSPLIT:
    case LGV_PV2HBSPLIT_NODIFFUSE:
    case LGV_PV2HBSPLIT_ONLYDIFFUSE: {
      if (ev != LGV_PV2HBSPLIT_ONLYDIFFUSE) {
        for (int i1 = 0; i1 < outer; ++i1) {
          ideal_step(h, dt / (unsigned)outer);
          for (int i0 = 0; i0 < inner; ++i0) hb_sweep(h, dt / ((unsigned)inner * (unsigned)outer), mass);
        }
      }
      if (ev != LGV_PV2HBSPLIT_NODIFFUSE) charge_hb(h, dt);
      break;
    }
    case LGV_IDEAL_PV2: ideal_step(h, dt); break;
    case LGV_EULER_LANGEVIN_HB: hb_sweep(h, dt, mass); break;
    case LGV_CHARGE_HB: charge_hb(h, dt); break;
    case LGV_MODELA_EM: em_step(h, dt, mass); break;
    case LGV_IDEAL_EM:  // no counterpart in the reference: the ideal step, then Euler-Maruyama
      ideal_step(h, dt);
      em_step(h, dt, mass);
      break;
    default: throw std::string("step: unknown evolver");
  }
}

}  // namespace orc

// ===========================================================================
// C ABI of the oracle (loaded by tests through ctypes).
using orc::Handle;

extern "C" {

static thread_local std::string g_err;

const char *orc_last_error(void) { return g_err.c_str(); }

void *orc_create(const lgv_params *p, int mode, int nranks) {
  if (!p || p->N < 4 || (p->N % 2) || nranks < 1 || nranks > p->N) return nullptr;
  Handle *h = new Handle();
  h->p = *p;
  h->N = p->N;
  h->V = (size_t)p->N * p->N * p->N;
  h->u.assign(h->V * LGV_NDOF, 0.0);
  h->snap.assign(h->V * LGV_NDOF, 0.0);
  h->mode = mode;
  h->R = nranks;
  h->gens.resize(nranks);
  for (int r = 0; r < nranks; ++r) h->gens[r].init((int)p->seed, r, nranks);
  // PETSc-like slab sizes: the first N % R ranks own one extra plane.
  int k = 0;
  for (int r = 0; r < nranks; ++r) {
    const int sz = p->N / nranks + (r < p->N % nranks ? 1 : 0);
    h->k0.push_back(k);
    h->k1.push_back(k + sz);
    k += sz;
  }
  h->key = orc::make_key(p->seed);
  h->mon.assign(nranks, std::array<lgv_monitor, 3>{});
  return h;
}

void orc_destroy(void *hh) { delete (Handle *)hh; }

void orc_set_params(void *hh, const lgv_params *p) {
  Handle *h = (Handle *)hh;
  h->p = *p;
}

void orc_set_state(void *hh, const double *aos) {
  Handle *h = (Handle *)hh;
  std::memcpy(h->u.data(), aos, h->u.size() * sizeof(double));
}
void orc_get_state(void *hh, double *aos) {
  Handle *h = (Handle *)hh;
  std::memcpy(aos, h->u.data(), h->u.size() * sizeof(double));
}
void orc_set_counter(void *hh, uint64_t c) { ((Handle *)hh)->ctr = c; }
uint64_t orc_get_counter(void *hh) { return ((Handle *)hh)->ctr; }

void orc_inject_hb(void *hh, const double *prop, const double *acc) {
  Handle *h = (Handle *)hh;
  h->hb_prop.assign(prop, prop + 4 * h->V);
  h->hb_acc.assign(acc, acc + h->V);
  h->have_hb = true;
}
void orc_inject_charge(void *hh, const int32_t *order, const double *q, const double *acc) {
  Handle *h = (Handle *)hh;
  for (int a = 0; a < 5; ++a) h->ch_order[a] = order[a];
  h->ch_q.assign(q, q + 36 * h->V);
  h->ch_acc.assign(acc, acc + 36 * h->V);
  h->have_ch = true;
}
void orc_inject_em(void *hh, const double *xi) {
  Handle *h = (Handle *)hh;
  h->em_xi.assign(xi, xi + 4 * h->V);
  h->have_em = true;
}

int orc_step(void *hh, int ev, int inner, int outer, double dt, double t, int nsteps) {
  Handle *h = (Handle *)hh;
  try {
    for (int s = 0; s < nsteps; ++s) {
      orc::step_once(*h, ev, inner, outer, dt, t);
      t += dt;
    }
  } catch (const std::string &e) {
    g_err = e;
    return LGV_ERR_STATE;
  }
  return LGV_OK;
}

int orc_initialize(void *hh, int kind, double scale) {
  try {
    orc::initialize(*(Handle *)hh, kind, scale);
  } catch (const std::string &e) {
    g_err = e;
    return LGV_ERR_INVALID;
  }
  return LGV_OK;
}

void orc_measure(void *hh, lgv_measurement *out) { orc::measure(*(Handle *)hh, out); }

double orc_energy(void *hh) { return orc::energy(*(Handle *)hh); }
void orc_last_energies(void *hh, double *e2) {
  Handle *h = (Handle *)hh;
  e2[0] = h->last_E[0];
  e2[1] = h->last_E[1];
}

void orc_get_monitor(void *hh, int which, lgv_monitor *out) {
  Handle *h = (Handle *)hh;
  lgv_monitor m{};
  for (int r = 0; r < h->R; ++r) {
    const lgv_monitor &a = h->mon[r][which];
    m.down_counts += a.down_counts;
    m.up_counts += a.up_counts;
    m.up_yes += a.up_yes;
    m.up_no += a.up_no;
    m.down_dS += a.down_dS;
    m.up_dS += a.up_dS;
  }
  *out = m;
}

void orc_set_hb_proposal(void *hh, int kind) { ((Handle *)hh)->hb_gauss = kind == 1; }

void orc_debug_flags(void *hh, int on) {
  Handle *h = (Handle *)hh;
  h->flags_on = on != 0;
  if (on) h->flags.assign(36 * h->V, 0);
}
void orc_get_flags(void *hh, uint8_t *out) {
  Handle *h = (Handle *)hh;
  std::memcpy(out, h->flags.data(), h->flags.size());
}

// --- building blocks, exposed for the known-answer tests -------------------
void orc_o4_rotation(const double *V, const double *A, double *phi) { orc::o4_rotation(V, A, phi); }

// Sequential (reference) stream of rank `rank` of `size`: kind 0 raw u64 (as
// double bits), 1 uniform, 2 variance1, 3 normal.
void orc_seq_draws(int base_seed, int rank, int size, int kind, int n, double *out) {
  orc::NoiseGen g;
  g.init(base_seed, rank, size);
  for (int i = 0; i < n; ++i) {
    if (kind == 0) {
      uint64_t r = g.rng();
      std::memcpy(&out[i], &r, 8);
    } else if (kind == 1) out[i] = g.uniform();
    else if (kind == 2) out[i] = g.variance1();
    else out[i] = g.normal();
  }
}
// xoroshiro128+ raw outputs from an explicit state.
void orc_xoro_raw(uint64_t s0, uint64_t s1, int n, uint64_t *out) {
  orc::Xoro x;
  x.s[0] = s0;
  x.s[1] = s1;
  for (int i = 0; i < n; ++i) out[i] = x();
}
// seed_seq-derived 32-bit seeds for all ranks (NoiseGenerator.h:76-80).
void orc_seed_seq(int base_seed, int size, uint32_t *out) {
  std::seed_seq seq = {base_seed};
  std::vector<unsigned int> seeds(size, 0);
  seq.generate(seeds.begin(), seeds.end());
  for (int i = 0; i < size; ++i) out[i] = seeds[i];
}
// Counter streams: raw draws of stream n at counter ctr.
void orc_ctr_draws(uint64_t seed, uint64_t ctr, uint64_t n, int ndraw, uint64_t *out) {
  orc::CtrStream cs(orc::subkey(orc::make_key(seed), ctr), n);
  for (int i = 0; i < ndraw; ++i) out[i] = cs.next();
}
// Counter-mode Euler-Maruyama normals of step counter ctr: xi[l * N^3 + n] for
// natural site n = (k N + j) N + i, the draws em_step takes in counter mode.
void orc_em_noise(uint64_t seed, uint64_t ctr, int N, double *xi) {
  const uint64_t sk = orc::subkey(orc::make_key(seed), ctr);
  const size_t V = (size_t)N * N * N;
  for (size_t n = 0; n < V; ++n) {
    orc::CtrStream cs(sk, n);
    const uint64_t r1 = cs.next(), r2 = cs.next(), r3 = cs.next(), r4 = cs.next();
    orc::box_muller(r1, r2, xi[n], xi[V + n]);
    orc::box_muller(r3, r4, xi[2 * V + n], xi[3 * V + n]);
  }
}
// Charge pass order of a counter-mode charge step at counter ctr.
void orc_ctr_order(uint64_t seed, uint64_t ctr, int32_t *order5) {
  const uint64_t w = orc::word(orc::subkey(orc::make_key(seed), ctr), 0);
  const int pi = (int)((w & 0xffffffffull) % 6ull);
  for (int a = 0; a < 3; ++a) order5[a] = orc::kPerm[pi][a];
  order5[3] = (w >> 63) ? 1 : 0;
  order5[4] = (w >> 63) ? 0 : 1;
}
// The single-link chain of q_heatbathtest.cxx:121-137 (t1): n steps of
// modelg_update_charge_pair on one pair with the reference's serial stream.
void orc_charge_pair_chain(double chi, double rms, double nA, double nB, int base_seed, int n, double *out_nA,
                           double *out_nB) {
  orc::NoiseGen g;
  g.init(base_seed, 0, 1);
  for (int i = 0; i < n; ++i) {
    double q = rms * g.variance1();
    const double dS = (std::pow(nA - q, 2) + std::pow(nB + q, 2) - std::pow(nA, 2) - std::pow(nB, 2)) / (2. * chi);
    if (!(dS < 0)) {
      const double r = g.uniform();
      if (!(r < std::exp(-dS))) q = 0.;
    }
    nA -= q;
    nB += q;
    out_nA[i] = nA;
    out_nB[i] = nB;
  }
}

}  // extern "C"

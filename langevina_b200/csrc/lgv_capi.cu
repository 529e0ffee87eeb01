// lgv_capi.cu -- the C ABI of include/lgv.h.
//
// The handle owns two red-black SoA lattices (current and alternate, for the
// stencils that cannot update in place), a staging buffer for the host
// boundary, and small scratch areas.  It sequences the sub-steps of each
// reference stepper (Stepper.cxx:542-580) and keeps the 64-bit counter that
// indexes the noise streams.  No computation happens on the host: a missing
// or failed kernel surfaces as LGV_ERR_CUDA.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/lgv.h"
#include "lgv_internal.h"

using lgv::Fields;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  // A failed runtime call (an allocation above all) leaves its error as the
  // runtime's last error, which the next launch's cudaGetLastError would
  // report as its own: clear it now that it is reported here.  (Sticky
  // errors of a lost context are not cleared by this and stay visible.)
  if (code == LGV_ERR_CUDA || code == LGV_ERR_NOMEM) (void)cudaGetLastError();
  return code;
}

#define LGV_CK(call)                                                                          \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(LGV_ERR_CUDA, "%s: %s (%s:%d)", #call,                 \
                                       cudaGetErrorString(e_), __FILE__, __LINE__);           \
  } while (0)

#define LGV_TRY(expr)       \
  do {                      \
    int r_ = (expr);        \
    if (r_ != LGV_OK) return r_; \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// pass orderings of the counter-mode charge step (lexicographic permutations)
const int kPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

}  // namespace

struct lgv_handle {
  lgv_params p{};
  int N = 0;
  size_t V = 0;
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  double *bufA = nullptr, *bufB = nullptr;
  Fields cur{}, alt{};
  double *staging = nullptr;
  double *scratch = nullptr;
  size_t scratch_len = 0;
  double *meas_dev = nullptr;
  double *small_dev = nullptr;  // 8 doubles
  uint64_t key = 0, ctr = 0;
  int noise_mode = LGV_NOISE_COUNTER;
  double *inj_hb_prop = nullptr, *inj_hb_acc = nullptr, *inj_ch_q = nullptr, *inj_ch_acc = nullptr,
         *inj_em_xi = nullptr;
  int32_t inj_order[5] = {0, 1, 2, 0, 1};
  bool have_hb = false, have_ch = false, have_em = false;
  bool mon_on = false;
  // phi heat bath as one z-marching sweep kernel instead of two parity
  // passes (LGV_HB_FUSED=1 in the environment at lgv_create)
  bool hb_fused = false;
  // phi sweeps as ordered persistent launches (hb_ordered_kernel), opt-in:
  // LGV_HB_ORDERED=1 (=1,S,spc,lag,fuse also sets planes per slab, sites per
  // chunk, schedule lag and how many consecutive sweeps share a launch).  On
  // B200 at 256^3 the two one-parity launches are faster: the pass is near
  // its instruction-issue limit, and at ~1300 resident CTAs the odd pass of a
  // slab re-reads it from DRAM anyway (57.5 of 64 B/site per sweep measured)
  bool hb_ordered = false;
  int hb_fuse = 2;
  lgv::HbPlan hb_plan;
  // this handle's count of bounded device waits that gave up (TMA copies of
  // the ideal step), and the polls before one gives up (LGV_WAIT_LIMIT at
  // lgv_create; the default is lgv::kWaitLimit)
  unsigned long long *waits_dev = nullptr;
  int wait_limit = lgv::kWaitLimit;
  // Plane order of the next ideal, phi-pass or charge-face launch: it flips
  // after every such launch, so each pass starts on the planes the previous
  // one touched last (still in L2).  LGV_ZALT=0 at creation keeps every pass
  // bottom-up.
  bool zalt = true;
  int zrev = 0;
  // Gaussian phi heat-bath proposals with counter noise (lgv_set_hb_proposal)
  bool hb_gauss = false;
  // Geometry of the buffers: the whole lattice, or for a slab handle
  // (lgv_slab_create) its planes k0 .. k0+nz-1 with two ghost planes on each
  // side, filled by the caller's halo exchange before every sub-pass that
  // reads across planes.
  lgv::Geo geo{};
  bool slab = false;
  int k0 = 0, nz = 0;
  lgv_halo_fn halo_fn = nullptr;
  void *halo_ctx = nullptr;
  // charge heat bath as three two-face launches (one per direction) instead
  // of six single-face launches (LGV_CHARGE_FUSED=1 at lgv_create)
  bool charge_per_face = true;
  lgv::MonAcc *mon_dev = nullptr;  // [3]
  lgv_monitor mon_ideal{};
  uint8_t *flags_dev = nullptr;
  // live per-kernel timing (lgv_timing_enable): event pairs around launches
  bool timing_on = false;
  std::vector<cudaEvent_t> ev_pool;
  struct TimedLaunch {
    int cls, units;  // units: faces / passes the launch covers
    cudaEvent_t a, b;
  };
  std::vector<TimedLaunch> ev_used;
  double t_ms[LGV_NKCLASS] = {0};
  int64_t t_n[LGV_NKCLASS] = {0};
  // differentiable Euler-Maruyama run (lgv_em_forward / lgv_em_backward)
  // differentiable run (lgv_diff_forward / lgv_diff_backward)
  struct {
    bool ready = false;
    int ev = 0, ncomp = 4;  // evolver; planes per stored state (phi only, or phi and charges)
    lgv_params p{};         // parameters and key of the forward run, used by the backward
    uint64_t key = 0;
    double dt = 0;
    int S = 0, b = 0, K = 1;
    uint64_t ctr0 = 0;
    std::vector<double> tn, avg;
    double *ckpt = nullptr, *seg = nullptr, *lam = nullptr, *work = nullptr, *avg_dev = nullptr, *partial = nullptr,
           *g4 = nullptr;
    unsigned *done = nullptr;  // grid_sum4 counter, zero between launches
    size_t ckpt_len = 0, seg_len = 0, avg_len = 0, lam_len = 0, work_len = 0;
  } adj;
};

namespace {

int ensure(double **p, size_t n) {
  if (*p) return LGV_OK;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(double));
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(LGV_ERR_NOMEM, "cudaMalloc(%zu doubles): %s", n, cudaGetErrorString(e));
  }
  return LGV_OK;
}

// A bounded device wait that gave up -- a TMA copy of the ideal step, or an
// ordered sweep's wait for the slabs it depends on -- leaves a count in this
// handle's counters: report it once, as LGV_ERR_TIMEOUT.  Synchronises the
// handle's stream.
int check_waits(lgv_handle *h) {
  unsigned long long n = 0, m = 0;
  if (h->waits_dev) {
    LGV_CK(cudaMemcpyAsync(&n, h->waits_dev, sizeof(n), cudaMemcpyDeviceToHost, h->stream));
    LGV_CK(cudaStreamSynchronize(h->stream));
    if (n) LGV_CK(cudaMemsetAsync(h->waits_dev, 0, sizeof(n), h->stream));
  }
  LGV_CK(lgv::hb_plan_timeouts(h->hb_plan, h->stream, &m, true));
  if (n || m)
    return fail(LGV_ERR_TIMEOUT,
                "bounded device waits timed out: %llu TMA copy waits, %llu ordered-sweep dependency waits; the state "
                "is not valid",
                n, m);
  return LGV_OK;
}

// Slab handles: ask the caller's exchange to fill the ghost planes of the
// current buffer for the component groups `comps` (LGV_HALO_*).
int halo(lgv_handle *h, int comps) {
  if (!h->slab) return LGV_OK;
  if (!h->halo_fn) return fail(LGV_ERR_STATE, "slab handle has no halo exchange (lgv_slab_set_halo)");
  const int r = h->halo_fn(h->halo_ctx, h, comps);
  if (r != 0) return fail(LGV_ERR_STATE, "halo exchange failed (%d)", r);
  return LGV_OK;
}

int no_slab(lgv_handle *h, const char *what) {
  return h->slab ? fail(LGV_ERR_UNSUPPORTED, "%s: not available on a slab handle", what) : LGV_OK;
}

int ensure_scratch(lgv_handle *h, size_t n) {
  if (h->scratch && h->scratch_len >= n) return LGV_OK;
  if (h->scratch) cudaFree(h->scratch);
  h->scratch = nullptr;
  LGV_TRY(ensure(&h->scratch, n));
  h->scratch_len = n;
  return LGV_OK;
}

int check_params(const lgv_params *p) {
  if (!p) return fail(LGV_ERR_INVALID, "params is NULL");
  if (p->N < 4 || (p->N & 1)) return fail(LGV_ERR_INVALID, "N=%d: must be even and >= 4", p->N);
  if (p->N > 2048) return fail(LGV_ERR_INVALID, "N=%d exceeds the supported 2048", p->N);
  if (p->reserved0 != 0) return fail(LGV_ERR_INVALID, "reserved0 must be 0");
  if (!(p->chi > 0)) return fail(LGV_ERR_INVALID, "chi must be > 0");
  if (!(p->LX > 0)) return fail(LGV_ERR_INVALID, "LX must be > 0");
  if (!(p->gamma >= 0) || !(p->diffusion >= 0)) return fail(LGV_ERR_INVALID, "gamma, diffusion must be >= 0");
  return LGV_OK;
}

// Component planes are V doubles each; consecutive planes start kPlaneSkew
// doubles apart beyond V so that the ten concurrently streamed planes do not
// share a power-of-two stride (at N = 256 a plane is exactly 128 MiB), which
// maps them onto the same DRAM channels at the same time.
constexpr size_t kPlaneSkew = 4352;  // 34 KiB: an odd multiple of 256 B

size_t lattice_doubles(size_t V) { return 10 * (V + kPlaneSkew); }

Fields fields_of(double *base, size_t V) {
  Fields f;
  for (int L = 0; L < 10; ++L) f.c[L] = base + (size_t)L * (V + kPlaneSkew);
  return f;
}

cudaEvent_t pool_event(lgv_handle *h) {
  if (!h->ev_pool.empty()) {
    cudaEvent_t e = h->ev_pool.back();
    h->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records a CUDA event pair around the launches of one kernel class when
// timing is enabled; the events are resolved in lgv_timing_read.
struct KTimer {
  lgv_handle *h;
  int cls, units;
  cudaEvent_t a = nullptr, b = nullptr;
  KTimer(lgv_handle *hh, int c, int u = 1) : h(hh), cls(c), units(u) {
    if (!h->timing_on) return;
    a = pool_event(h);
    b = pool_event(h);
    cudaEventRecord(a, h->stream);
  }
  ~KTimer() {
    if (!a) return;
    cudaEventRecord(b, h->stream);
    h->ev_used.push_back({cls, units, a, b});
  }
};

lgv::MonAcc *mon_ptr(lgv_handle *h, int which) { return h->mon_on ? h->mon_dev + which : nullptr; }

int energy_now(lgv_handle *h, double *E) {
  LGV_TRY(ensure_scratch(h, lgv::energy_scratch_doubles(h->N)));
  LGV_TRY(ensure(&h->small_dev, 8));
  LGV_CK(lgv::launch_energy(h->cur, h->N, h->p.H, 0.5 / h->p.chi, h->scratch, h->small_dev, h->stream));
  LGV_CK(cudaMemcpyAsync(E, h->small_dev, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  return LGV_OK;
}

// --- sub-steps -------------------------------------------------------------
// Geometry for the next pass launch, in the plane order its turn gives.
lgv::Geo pass_geo(lgv_handle *h) {
  lgv::Geo g = h->geo;
  if (h->zalt) {
    g.zrev = h->zrev;
    h->zrev ^= 1;
  }
  return g;
}

int sub_ideal(lgv_handle *h, double dt) {  // IdealPV2::step (Stepper.cxx:23-66)
  double Eold = 0, Enew = 0;
  if (h->mon_on) LGV_TRY(energy_now(h, &Eold));
  lgv::IdealArgs a{};
  a.dto2chi = (dt / 2.0) / h->p.chi;
  a.dt = dt;
  const double hx = h->p.LX / h->N;
  a.a2 = std::pow(1.0 / hx, 2);
  a.H = h->p.H;
  a.waits = h->waits_dev;
  a.wait_limit = h->wait_limit;
  LGV_TRY(halo(h, LGV_HALO_ALL));
  {
    KTimer tm(h, LGV_KCLASS_IDEAL);
    LGV_CK(lgv::launch_ideal(h->cur, h->alt, pass_geo(h), a, h->stream));
  }
  std::swap(h->cur, h->alt);
  if (h->mon_on) {
    LGV_TRY(energy_now(h, &Enew));
    const double dE = Enew - Eold;
    if (dE > 0) {
      h->mon_ideal.up_counts++;
      h->mon_ideal.up_yes++;
      h->mon_ideal.up_dS += dE;
    } else {
      h->mon_ideal.down_counts++;
      h->mon_ideal.down_dS += dE;
    }
  }
  return LGV_OK;
}

int sub_hb(lgv_handle *h, double dt, double mass) {  // EulerLangevinHB::step (Stepper.cxx:287-389)
  lgv::HbArgs a{};
  a.rdtg = std::sqrt(2. * dt * h->p.gamma);
  a.Lambda2 = 0.5 * (2. * 3. + mass);
  a.lam4 = h->p.lambda / 4.;
  a.H = h->p.H;
  a.mon = mon_ptr(h, LGV_MONITOR_PHI_HB);
  a.flags = h->flags_dev;
  if (h->noise_mode == LGV_NOISE_INJECTED) {
    if (!h->have_hb) return fail(LGV_ERR_STATE, "phi heat bath: injected noise not supplied");
    a.prop = h->inj_hb_prop;
    a.acc = h->inj_hb_acc;
  } else {
    a.sk = lgv::sub_key(h->key, h->ctr);
    a.gauss = h->hb_gauss ? 1 : 0;
  }
  if (h->hb_ordered) {
    KTimer tm(h, LGV_KCLASS_PHI_HB, 2);  // one launch, both parity passes
    LGV_CK(lgv::launch_hb_ordered(h->cur, h->N, a, h->hb_plan, 1, nullptr, h->stream));
  } else if (h->hb_fused) {
    KTimer tm(h, LGV_KCLASS_PHI_HB, 2);  // one launch, both parity passes
    LGV_CK(lgv::launch_hb_sweep(h->cur, h->alt, h->N, a, h->stream));
    for (int l = 0; l < 4; ++l) std::swap(h->cur.c[l], h->alt.c[l]);
  } else {
    for (int parity = 0; parity < 2; ++parity) {
      LGV_TRY(halo(h, LGV_HALO_PHI));
      KTimer tm(h, LGV_KCLASS_PHI_HB);
      LGV_CK(lgv::launch_hb_pass(h->cur, pass_geo(h), parity, a, h->stream));
    }
  }
  if (h->noise_mode == LGV_NOISE_INJECTED) h->have_hb = false;
  else h->ctr += 1;
  return LGV_OK;
}

// n consecutive heat-bath sweeps (the inner loop of PV2HBSplit::step,
// Stepper.cxx:562-564).  With counter noise and no per-site flags, up to
// hb_fuse of them share one ordered launch: sweep q draws with counter
// ctr + q, exactly as n separate sweeps do.
int sub_hb_n(lgv_handle *h, double dt, double mass, int n) {
  if (!h->hb_ordered || h->noise_mode != LGV_NOISE_COUNTER || h->flags_dev || h->hb_fuse < 2 || n < 2) {
    for (int i = 0; i < n; ++i) LGV_TRY(sub_hb(h, dt, mass));
    return LGV_OK;
  }
  lgv::HbArgs a{};
  a.rdtg = std::sqrt(2. * dt * h->p.gamma);
  a.Lambda2 = 0.5 * (2. * 3. + mass);
  a.lam4 = h->p.lambda / 4.;
  a.H = h->p.H;
  a.mon = mon_ptr(h, LGV_MONITOR_PHI_HB);
  for (int done = 0; done < n;) {
    const int k = std::min(n - done, std::min(h->hb_fuse, lgv::kHbMaxSweeps));
    uint64_t sk[lgv::kHbMaxSweeps];
    for (int q = 0; q < k; ++q) sk[q] = lgv::sub_key(h->key, h->ctr + q);
    a.sk = sk[0];
    {
      KTimer tm(h, LGV_KCLASS_PHI_HB, 2 * k);
      LGV_CK(lgv::launch_hb_ordered(h->cur, h->N, a, h->hb_plan, k, sk, h->stream));
    }
    h->ctr += k;
    done += k;
  }
  return LGV_OK;
}

int sub_charge(lgv_handle *h, double dt) {  // ModelGChargeHB::step (Stepper.cxx:449-522)
  int xyz[3] = {0, 1, 2}, eo[2] = {0, 1};
  if (h->noise_mode == LGV_NOISE_INJECTED) {
    if (!h->have_ch) return fail(LGV_ERR_STATE, "charge heat bath: injected noise not supplied");
    for (int a = 0; a < 3; ++a) xyz[a] = h->inj_order[a];
    eo[0] = h->inj_order[3];
    eo[1] = h->inj_order[4];
  } else {
    const uint64_t w = lgv::split_word(lgv::sub_key(h->key, h->ctr), 0);
    const int pi = (int)((w & 0xffffffffull) % 6ull);
    for (int a = 0; a < 3; ++a) xyz[a] = kPerm[pi][a];
    if (w >> 63) {
      eo[0] = 1;
      eo[1] = 0;
    }
  }
  lgv::ChargeArgs a{};
  a.rms = std::sqrt(2. * dt * (h->p.diffusion * h->p.chi));
  a.inv2chi = 1.0 / (2. * h->p.chi);
  a.mon = mon_ptr(h, LGV_MONITOR_CHARGE_HB);
  a.flags = h->flags_dev;
  if (h->noise_mode == LGV_NOISE_INJECTED) {
    a.q = h->inj_ch_q;
    a.acc = h->inj_ch_acc;
  }
  if (h->charge_per_face) {
    for (int p = 0; p < 6; ++p) {
      a.pass = p;
      if (h->noise_mode != LGV_NOISE_INJECTED) a.sk = lgv::sub_key(h->key, h->ctr + 1 + p);
      if (xyz[p / 2] == 2) LGV_TRY(halo(h, LGV_HALO_CHARGES));  // links across planes
      KTimer tm(h, LGV_KCLASS_CHARGE);
      LGV_CK(lgv::launch_charge_pass(h->cur, pass_geo(h), xyz[p / 2], eo[p % 2], a, h->stream));
    }
  } else {
    // both faces of a direction per launch (same streams and order as per face)
    lgv::ChargeDirPair d{};
    d.rms = a.rms;
    d.inv2chi = a.inv2chi;
    d.q = a.q;
    d.acc = a.acc;
    d.flags = a.flags;
    d.mon = a.mon;
    for (int ixyz = 0; ixyz < 3; ++ixyz) {
      for (int i = 0; i < 2; ++i) {
        d.pass[i] = 2 * ixyz + i;
        d.eo[i] = eo[i];
        d.sk[i] = (h->noise_mode != LGV_NOISE_INJECTED) ? lgv::sub_key(h->key, h->ctr + 1 + 2 * ixyz + i) : 0;
      }
      bool swapped = false;
      KTimer tm(h, LGV_KCLASS_CHARGE, 2);
      LGV_CK(lgv::launch_charge_dir(h->cur, h->alt, h->N, xyz[ixyz], d, h->stream, &swapped));
      if (swapped)
        for (int L = 4; L < 10; ++L) std::swap(h->cur.c[L], h->alt.c[L]);
    }
  }
  if (h->noise_mode == LGV_NOISE_INJECTED) h->have_ch = false;
  else h->ctr += 7;
  return LGV_OK;
}

int sub_em(lgv_handle *h, double dt, double mass) {
  lgv::EmArgs a{};
  a.c6 = 6.0 + mass;
  a.dtg = dt * h->p.gamma;
  a.sq = std::sqrt(2.0 * h->p.gamma * dt);
  a.lambda = h->p.lambda;
  a.H = h->p.H;
  if (h->noise_mode == LGV_NOISE_INJECTED) {
    if (!h->have_em) return fail(LGV_ERR_STATE, "Euler-Maruyama: injected noise not supplied");
    a.xi = h->inj_em_xi;
  } else {
    a.sk = lgv::sub_key(h->key, h->ctr);
  }
  LGV_TRY(halo(h, LGV_HALO_PHI));
  {
    KTimer tm(h, LGV_KCLASS_EM);
    LGV_CK(lgv::launch_em(h->cur, h->alt, h->geo, a, h->stream));
  }
  for (int l = 0; l < 4; ++l) std::swap(h->cur.c[l], h->alt.c[l]);
  if (h->noise_mode == LGV_NOISE_INJECTED) h->have_em = false;
  else h->ctr += 1;
  return LGV_OK;
}

int step_once(lgv_handle *h, int ev, int inner, int outer, double dt, double t) {
  const double mass = h->p.mass0 + h->p.dmassdt * t;  // ModelACoefficients::mass (ModelA.h:84)
  switch (ev) {
    case LGV_PV2HBSPLIT:
    case LGV_PV2HBSPLIT_NODIFFUSE:
    case LGV_PV2HBSPLIT_ONLYDIFFUSE:
      if (ev != LGV_PV2HBSPLIT_ONLYDIFFUSE) {
        for (int i1 = 0; i1 < outer; ++i1) {
          LGV_TRY(sub_ideal(h, dt / (unsigned)outer));
          LGV_TRY(sub_hb_n(h, dt / ((unsigned)inner * (unsigned)outer), mass, inner));
        }
      }
      if (ev != LGV_PV2HBSPLIT_NODIFFUSE) LGV_TRY(sub_charge(h, dt));
      return LGV_OK;
    case LGV_IDEAL_PV2: return sub_ideal(h, dt);
    case LGV_EULER_LANGEVIN_HB: return sub_hb(h, dt, mass);
    case LGV_CHARGE_HB: return sub_charge(h, dt);
    case LGV_MODELA_EM: return sub_em(h, dt, mass);
    case LGV_IDEAL_EM:
      LGV_TRY(sub_ideal(h, dt));
      return sub_em(h, dt, mass);
    default: return fail(LGV_ERR_INVALID, "unknown evolver %d", ev);
  }
}

int copy_injected(double **dst, const double *src, size_t n) {
  LGV_TRY(ensure(dst, n));
  LGV_CK(cudaMemcpy(*dst, src, n * sizeof(double), cudaMemcpyHostToDevice));
  return LGV_OK;
}

}  // namespace

// Lets other translation units of the library report through lgv_last_error().
void lgv_internal_set_error(const char *msg) { g_last_error = msg ? msg : ""; }

// ============================================================================
extern "C" {

int lgv_version(void) { return 10000; }

const char *lgv_status_string(int s) {
  switch (s) {
    case LGV_OK: return "ok";
    case LGV_ERR_INVALID: return "invalid argument";
    case LGV_ERR_CUDA: return "CUDA error";
    case LGV_ERR_NOMEM: return "out of memory";
    case LGV_ERR_TIMEOUT: return "device wait timed out";
    case LGV_ERR_STATE: return "invalid state";
    case LGV_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

const char *lgv_last_error(void) { return g_last_error.c_str(); }

namespace {
// Shared by lgv_create and lgv_slab_create: buffers for geometry g.
int create_handle(const lgv_params *params, const lgv::Geo &g, bool slab, int k0, int nz, lgv_handle **out) {
  int dev = 0;
  LGV_CK(cudaGetDevice(&dev));
  lgv_handle *h = new lgv_handle();
  h->p = *params;
  h->N = params->N;
  h->geo = g;
  h->V = (size_t)(2 * g.V2);
  h->slab = slab;
  h->k0 = k0;
  h->nz = nz;
  h->device = dev;
  h->key = lgv::make_key(params->seed);
  if (!slab) {
    const char *f = std::getenv("LGV_HB_FUSED");
    h->hb_fused = f && f[0] == '1';
    // one face per launch (the faster path on B200); LGV_CHARGE_FUSED=1 selects
    // both faces of a direction per launch
    const char *c = std::getenv("LGV_CHARGE_FUSED");
    h->charge_per_face = !(c && c[0] == '1');
  }
  int hb_slab = 4, hb_spc = 1024, hb_lag = 2;
  {
    const char *o = std::getenv("LGV_HB_ORDERED");
    h->hb_ordered = false;
    if (o && o[0]) {
      int on = 1, fuse = h->hb_fuse;
      std::sscanf(o, "%d,%d,%d,%d,%d", &on, &hb_slab, &hb_spc, &hb_lag, &fuse);
      h->hb_ordered = on != 0;
      h->hb_fuse = fuse;
    }
    if (h->hb_fused) h->hb_ordered = false;
  }
  {
    const char *wl = std::getenv("LGV_WAIT_LIMIT");
    if (wl && wl[0]) h->wait_limit = std::max(0, std::atoi(wl));
    const char *za = std::getenv("LGV_ZALT");
    h->zalt = !(za && za[0] == '0');
  }
  int rc = LGV_OK;
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    rc = fail(LGV_ERR_CUDA, "cudaStreamCreate failed");
  }
  h->stream = h->own_stream;
  if (rc == LGV_OK) rc = ensure(&h->bufA, lattice_doubles(h->V));
  if (rc == LGV_OK) rc = ensure(&h->bufB, lattice_doubles(h->V));
  if (rc == LGV_OK) rc = ensure(&h->small_dev, 8);
  if (rc == LGV_OK) {
    cudaError_t e = cudaMalloc((void **)&h->mon_dev, 3 * sizeof(lgv::MonAcc));
    if (e != cudaSuccess) rc = fail(LGV_ERR_NOMEM, "monitor alloc: %s", cudaGetErrorString(e));
  }
  if (rc == LGV_OK) {
    h->cur = fields_of(h->bufA, h->V);
    h->alt = fields_of(h->bufB, h->V);
    if (cudaMemsetAsync(h->bufA, 0, lattice_doubles(h->V) * sizeof(double), h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->mon_dev, 0, 3 * sizeof(lgv::MonAcc), h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      rc = fail(LGV_ERR_CUDA, "initial memset failed");
  }
  if (rc == LGV_OK) {
    if (cudaMalloc((void **)&h->waits_dev, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemset(h->waits_dev, 0, sizeof(unsigned long long)) != cudaSuccess)
      rc = fail(LGV_ERR_NOMEM, "wait counter alloc failed");
  }
  if (rc == LGV_OK && h->hb_ordered) {
    h->hb_plan.wait_limit = h->wait_limit;
    const cudaError_t e = lgv::hb_plan_build(h->hb_plan, h->N, hb_slab, hb_spc, hb_lag);
    if (e != cudaSuccess) rc = fail(LGV_ERR_CUDA, "ordered sweep plan: %s", cudaGetErrorString(e));
  }
  if (rc != LGV_OK) {
    lgv_destroy(h);
    return rc;
  }
  *out = h;
  return LGV_OK;
}
}  // namespace

int lgv_create(const lgv_params *params, lgv_handle **out) {
  if (!out) return fail(LGV_ERR_INVALID, "out is NULL");
  *out = nullptr;
  LGV_TRY(check_params(params));
  return create_handle(params, lgv::make_geo(params->N), false, 0, 0, out);
}

int lgv_slab_create(const lgv_params *params, int k0, int nz, lgv_handle **out) {
  if (!out) return fail(LGV_ERR_INVALID, "out is NULL");
  *out = nullptr;
  LGV_TRY(check_params(params));
  const int N = params->N;
  if (nz < 2 || (nz & 1) || k0 < 0 || (k0 & 1) || k0 + nz > N)
    return fail(LGV_ERR_INVALID, "slab planes [%d, %d): need k0 even, nz even >= 2, k0 + nz <= N = %d", k0, k0 + nz, N);
  return create_handle(params, lgv::make_slab_geo(N, nz + 4, k0 - 2), true, k0, nz, out);
}

int lgv_slab_set_halo(lgv_handle *h, lgv_halo_fn fn, void *ctx) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  if (!h->slab) return fail(LGV_ERR_INVALID, "not a slab handle");
  h->halo_fn = fn;
  h->halo_ctx = ctx;
  return LGV_OK;
}

size_t lgv_slab_halo_doubles(lgv_handle *h, int comps) {
  if (!h || !h->slab) return 0;
  const int nc = ((comps & LGV_HALO_PHI) ? 4 : 0) + ((comps & LGV_HALO_CHARGES) ? 6 : 0);
  return (size_t)nc * 2 * 2 * h->N * (h->N / 2);
}

namespace {
// The two planes of side `side` (0 below, 1 above) of the current buffer:
// interior planes to send (ghost = false) or ghost planes to fill (true), as
// per (component, parity half) runs of 2 N^2/2 contiguous doubles.
int slab_copy(lgv_handle *h, int side, int comps, double *buf, bool unpack) {
  if (!h || !buf) return fail(LGV_ERR_INVALID, "NULL argument");
  if (!h->slab) return fail(LGV_ERR_INVALID, "not a slab handle");
  if ((side != 0 && side != 1) || comps < 1 || comps > LGV_HALO_ALL) return fail(LGV_ERR_INVALID, "side/comps");
  DeviceGuard g(h->device);
  const size_t run = (size_t)2 * h->N * (h->N / 2);  // two planes of one parity half
  int plane;
  if (unpack) plane = side == 0 ? 0 : h->nz + 2;
  else plane = side == 0 ? 2 : h->nz;
  const size_t off = (size_t)plane * h->N * (h->N / 2);
  size_t q = 0;
  for (int c = 0; c < 10; ++c) {
    if (!((c < 4 && (comps & LGV_HALO_PHI)) || (c >= 4 && (comps & LGV_HALO_CHARGES)))) continue;
    for (int par = 0; par < 2; ++par) {
      double *field = h->cur.c[c] + (size_t)par * h->geo.V2 + off;
      if (unpack)
        LGV_CK(cudaMemcpyAsync(field, buf + q, run * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      else
        LGV_CK(cudaMemcpyAsync(buf + q, field, run * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      q += run;
    }
  }
  return LGV_OK;
}
}  // namespace

int lgv_slab_pack(lgv_handle *h, int side, int comps, double *dev_buf) { return slab_copy(h, side, comps, dev_buf, false); }
int lgv_slab_unpack(lgv_handle *h, int side, int comps, const double *dev_buf) {
  return slab_copy(h, side, comps, const_cast<double *>(dev_buf), true);
}

int lgv_slab_measure_partials(lgv_handle *h, double *dev_T, double *dev_U) {
  if (!h || !dev_T || !dev_U) return fail(LGV_ERR_INVALID, "NULL argument");
  if (!h->slab) return fail(LGV_ERR_INVALID, "not a slab handle");
  DeviceGuard g(h->device);
  LGV_CK(lgv::launch_measure_partials(h->cur, h->geo, 2, h->nz, h->k0, dev_T, dev_U, h->stream));
  return LGV_OK;
}

int lgv_measure_from_partials(const double *dev_T, const double *dev_U, int N, double *dev_out, void *stream) {
  if (!dev_T || !dev_U || !dev_out) return fail(LGV_ERR_INVALID, "NULL argument");
  if (N < 4 || (N & 1)) return fail(LGV_ERR_INVALID, "N must be even and >= 4");
  LGV_CK(lgv::launch_measure_finish(dev_T, dev_U, N, dev_out, (cudaStream_t)stream));
  return LGV_OK;
}

int lgv_destroy(lgv_handle *h) {
  if (!h) return LGV_OK;
  DeviceGuard g(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  double *bufs[] = {h->bufA, h->bufB, h->staging, h->scratch, h->meas_dev, h->small_dev, h->inj_hb_prop,
                    h->inj_hb_acc, h->inj_ch_q, h->inj_ch_acc, h->inj_em_xi};
  for (double *b : bufs)
    if (b) cudaFree(b);
  if (h->mon_dev) cudaFree(h->mon_dev);
  if (h->flags_dev) cudaFree(h->flags_dev);
  for (double *b : {h->adj.ckpt, h->adj.seg, h->adj.lam, h->adj.work, h->adj.avg_dev, h->adj.partial, h->adj.g4})
    if (b) cudaFree(b);
  if (h->adj.done) cudaFree(h->adj.done);
  lgv::hb_plan_free(h->hb_plan);
  if (h->waits_dev) cudaFree(h->waits_dev);
  for (auto &u : h->ev_used) {
    cudaEventDestroy(u.a);
    cudaEventDestroy(u.b);
  }
  for (auto e : h->ev_pool) cudaEventDestroy(e);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return LGV_OK;
}

int lgv_set_params(lgv_handle *h, const lgv_params *params) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  LGV_TRY(check_params(params));
  if (params->N != h->N) return fail(LGV_ERR_INVALID, "N cannot change (%d -> %d)", h->N, params->N);
  if (params->seed != h->p.seed) h->key = lgv::make_key(params->seed);
  h->p = *params;
  return LGV_OK;
}

int lgv_set_state(lgv_handle *h, const double *host_aos) {
  if (!h || !host_aos) return fail(LGV_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  LGV_TRY(ensure(&h->staging, 10 * h->V));
  LGV_CK(cudaMemcpyAsync(h->staging, host_aos, 10 * h->V * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  LGV_CK(lgv::launch_aos_to_rb(h->staging, h->cur, h->geo, h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  return LGV_OK;
}

int lgv_get_state(lgv_handle *h, double *host_aos) {
  if (!h || !host_aos) return fail(LGV_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  LGV_TRY(ensure(&h->staging, 10 * h->V));
  LGV_CK(lgv::launch_rb_to_aos(h->cur, h->staging, h->geo, h->stream));
  LGV_CK(cudaMemcpyAsync(host_aos, h->staging, 10 * h->V * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  return check_waits(h);
}

int lgv_set_state_device(lgv_handle *h, const double *dev_aos) {
  if (!h || !dev_aos) return fail(LGV_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  LGV_CK(lgv::launch_aos_to_rb(dev_aos, h->cur, h->geo, h->stream));
  return LGV_OK;
}

int lgv_get_state_device(lgv_handle *h, double *dev_aos) {
  if (!h || !dev_aos) return fail(LGV_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  LGV_CK(lgv::launch_rb_to_aos(h->cur, dev_aos, h->geo, h->stream));
  return LGV_OK;
}

int lgv_initialize(lgv_handle *h, int kind, double scale) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  LGV_TRY(no_slab(h, "lgv_initialize"));
  DeviceGuard g(h->device);
  switch (kind) {
    case LGV_INIT_ZERO:
      for (int L = 0; L < 10; ++L) LGV_CK(cudaMemsetAsync(h->cur.c[L], 0, h->V * sizeof(double), h->stream));
      return LGV_OK;
    case LGV_INIT_PHI_GAUSSIAN:
      LGV_CK(lgv::launch_init_phi(h->cur, h->N, lgv::sub_key(h->key, h->ctr), scale, h->stream));
      h->ctr += 1;
      return LGV_OK;
    case LGV_INIT_CHARGES_GAUSSIAN: {
      const size_t nb = (h->V + 255) / 256;
      LGV_TRY(ensure_scratch(h, nb * 6 + 16));
      LGV_CK(lgv::launch_init_charges(h->cur, h->N, lgv::sub_key(h->key, h->ctr), std::sqrt(h->p.chi), h->scratch,
                                      h->stream));
      h->ctr += 1;
      return LGV_OK;
    }
    default: return fail(LGV_ERR_INVALID, "unknown init kind %d", kind);
  }
}

int lgv_set_noise_mode(lgv_handle *h, int mode) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  if (mode != LGV_NOISE_COUNTER && mode != LGV_NOISE_INJECTED) return fail(LGV_ERR_INVALID, "noise mode %d", mode);
  if (mode == LGV_NOISE_INJECTED) LGV_TRY(no_slab(h, "injected noise"));
  h->noise_mode = mode;
  return LGV_OK;
}

int lgv_set_hb_proposal(lgv_handle *h, int kind) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  if (kind != LGV_HB_PROPOSAL_UNIFORM && kind != LGV_HB_PROPOSAL_GAUSSIAN)
    return fail(LGV_ERR_INVALID, "heat-bath proposal kind %d", kind);
  if (kind == LGV_HB_PROPOSAL_GAUSSIAN && (h->hb_fused || h->hb_ordered))
    return fail(LGV_ERR_UNSUPPORTED, "Gaussian proposals run on the one-parity pass only (LGV_HB_FUSED / LGV_HB_ORDERED set)");
  h->hb_gauss = kind == LGV_HB_PROPOSAL_GAUSSIAN;
  return LGV_OK;
}

int lgv_set_counter(lgv_handle *h, uint64_t c) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  h->ctr = c;
  return LGV_OK;
}

int lgv_get_counter(lgv_handle *h, uint64_t *c) {
  if (!h || !c) return fail(LGV_ERR_INVALID, "NULL argument");
  *c = h->ctr;
  return LGV_OK;
}

int lgv_inject_hb(lgv_handle *h, const double *prop, const double *acc) {
  if (!h || !prop || !acc) return fail(LGV_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  LGV_TRY(copy_injected(&h->inj_hb_prop, prop, 4 * h->V));
  LGV_TRY(copy_injected(&h->inj_hb_acc, acc, h->V));
  h->have_hb = true;
  return LGV_OK;
}

int lgv_inject_charge(lgv_handle *h, const int32_t *order, const double *q, const double *acc) {
  if (!h || !order || !q || !acc) return fail(LGV_ERR_INVALID, "NULL argument");
  bool seen[3] = {false, false, false};
  for (int a = 0; a < 3; ++a) {
    if (order[a] < 0 || order[a] > 2 || seen[order[a]]) return fail(LGV_ERR_INVALID, "order[0:3] not a permutation");
    seen[order[a]] = true;
  }
  if (!((order[3] == 0 && order[4] == 1) || (order[3] == 1 && order[4] == 0)))
    return fail(LGV_ERR_INVALID, "order[3:5] not a permutation of (0,1)");
  DeviceGuard g(h->device);
  LGV_TRY(copy_injected(&h->inj_ch_q, q, 36 * h->V));
  LGV_TRY(copy_injected(&h->inj_ch_acc, acc, 36 * h->V));
  for (int a = 0; a < 5; ++a) h->inj_order[a] = order[a];
  h->have_ch = true;
  return LGV_OK;
}

int lgv_inject_em(lgv_handle *h, const double *xi) {
  if (!h || !xi) return fail(LGV_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  LGV_TRY(copy_injected(&h->inj_em_xi, xi, 4 * h->V));
  h->have_em = true;
  return LGV_OK;
}

int lgv_step(lgv_handle *h, int evolver, int inner, int outer, double dt, double t, int nsteps) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  if (nsteps < 0) return fail(LGV_ERR_INVALID, "nsteps < 0");
  if (evolver <= LGV_PV2HBSPLIT_ONLYDIFFUSE && (inner < 1 || outer < 1))
    return fail(LGV_ERR_INVALID, "PV2HBSplit scounts must be >= 1 (got {%d, %d})", inner, outer);
  if (!std::isfinite(dt) || !std::isfinite(t)) return fail(LGV_ERR_INVALID, "dt/t not finite");
  DeviceGuard g(h->device);
  for (int s = 0; s < nsteps; ++s) {
    LGV_TRY(step_once(h, evolver, inner, outer, dt, t));
    t += dt;
  }
  return LGV_OK;
}

size_t lgv_measure_size(int N) { return lgv::measure_size(N); }

int lgv_measure_device(lgv_handle *h, double *dev_out) {
  if (!h || !dev_out) return fail(LGV_ERR_INVALID, "NULL argument");
  LGV_TRY(no_slab(h, "lgv_measure_device (use lgv_slab_measure_partials)"));
  DeviceGuard g(h->device);
  LGV_TRY(ensure_scratch(h, lgv::measure_scratch_doubles(h->N)));
  KTimer tm(h, LGV_KCLASS_MEASURE);
  LGV_CK(lgv::launch_measure(h->cur, h->N, h->scratch, dev_out, h->stream));
  return LGV_OK;
}

int lgv_measure(lgv_handle *h, lgv_measurement *out) {
  if (!h || !out) return fail(LGV_ERR_INVALID, "NULL argument");
  DeviceGuard g(h->device);
  const size_t n = lgv::measure_size(h->N);
  LGV_TRY(ensure(&h->meas_dev, n));
  LGV_TRY(lgv_measure_device(h, h->meas_dev));
  std::vector<double> host(n);
  LGV_CK(cudaMemcpyAsync(host.data(), h->meas_dev, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  const int N = h->N, NK = N / 2 + 1;
  const double *p = host.data();
  auto take = [&](double *dst, size_t cnt) {
    if (dst) std::memcpy(dst, p, cnt * sizeof(double));
    p += cnt;
  };
  take(out->OAverage, 11);
  for (int a = 0; a < 3; ++a) take(out->wall[a], 11 * (size_t)N);
  for (int a = 0; a < 3; ++a) take(out->wall_k[a], 11 * (size_t)NK * 2);
  for (int a = 0; a < 3; ++a) take(out->wall_k_rotated[a], 14 * (size_t)NK * 2);
  for (int a = 0; a < 3; ++a) take(out->wall_phase[a], 14 * (size_t)N);
  for (int a = 0; a < 3; ++a) take(out->wall_phase_k[a], 14 * (size_t)NK * 2);
  return LGV_OK;
}

int lgv_energy(lgv_handle *h, double *energy) {
  if (!h || !energy) return fail(LGV_ERR_INVALID, "NULL argument");
  LGV_TRY(no_slab(h, "lgv_energy"));
  DeviceGuard g(h->device);
  return energy_now(h, energy);
}

int lgv_enable_monitors(lgv_handle *h, int enable) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  if (enable) LGV_TRY(no_slab(h, "accept statistics"));
  DeviceGuard g(h->device);
  h->mon_on = enable != 0;
  h->mon_ideal = lgv_monitor{};
  LGV_CK(cudaMemsetAsync(h->mon_dev, 0, 3 * sizeof(lgv::MonAcc), h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  return LGV_OK;
}

int lgv_get_monitor(lgv_handle *h, int which, lgv_monitor *out) {
  if (!h || !out) return fail(LGV_ERR_INVALID, "NULL argument");
  if (which < 0 || which > 2) return fail(LGV_ERR_INVALID, "monitor %d", which);
  if (which == LGV_MONITOR_IDEAL) {
    *out = h->mon_ideal;
    return LGV_OK;
  }
  DeviceGuard g(h->device);
  lgv::MonAcc m;
  LGV_CK(cudaMemcpyAsync(&m, h->mon_dev + which, sizeof(m), cudaMemcpyDeviceToHost, h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  out->down_counts = (int64_t)m.down_counts;
  out->up_counts = (int64_t)m.up_counts;
  out->up_yes = (int64_t)m.up_yes;
  out->up_no = (int64_t)m.up_no;
  out->down_dS = m.down_dS;
  out->up_dS = m.up_dS;
  return LGV_OK;
}

int lgv_set_stream(lgv_handle *h, void *s) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  // NULL selects the legacy default stream, as documented in lgv.h
  cudaStream_t next = s ? (cudaStream_t)s : (cudaStream_t)0;
  if (next == h->stream) return LGV_OK;
  // work already queued on the old stream must finish before the new
  // stream touches the lattice
  DeviceGuard g(h->device);
  cudaEvent_t ev = pool_event(h);
  LGV_CK(cudaEventRecord(ev, h->stream));
  LGV_CK(cudaStreamWaitEvent(next, ev, 0));
  h->ev_pool.push_back(ev);
  h->stream = next;
  return LGV_OK;
}

int lgv_synchronize(lgv_handle *h) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  DeviceGuard g(h->device);
  LGV_CK(cudaStreamSynchronize(h->stream));
  return check_waits(h);
}

int lgv_timing_enable(lgv_handle *h, int enable) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  DeviceGuard g(h->device);
  LGV_CK(cudaStreamSynchronize(h->stream));
  for (auto &u : h->ev_used) {
    h->ev_pool.push_back(u.a);
    h->ev_pool.push_back(u.b);
  }
  h->ev_used.clear();
  for (int c = 0; c < LGV_NKCLASS; ++c) {
    h->t_ms[c] = 0;
    h->t_n[c] = 0;
  }
  h->timing_on = enable != 0;
  return LGV_OK;
}

int lgv_timing_read(lgv_handle *h, int kclass, double *total_ms, int64_t *launches) {
  if (!h || !total_ms || !launches) return fail(LGV_ERR_INVALID, "NULL argument");
  if (kclass < 0 || kclass >= LGV_NKCLASS) return fail(LGV_ERR_INVALID, "kernel class %d", kclass);
  DeviceGuard g(h->device);
  LGV_CK(cudaStreamSynchronize(h->stream));
  for (auto &u : h->ev_used) {
    float ms = 0;
    LGV_CK(cudaEventElapsedTime(&ms, u.a, u.b));
    h->t_ms[u.cls] += ms;
    h->t_n[u.cls] += u.units;
    h->ev_pool.push_back(u.a);
    h->ev_pool.push_back(u.b);
  }
  h->ev_used.clear();
  *total_ms = h->t_ms[kclass];
  *launches = h->t_n[kclass];
  return LGV_OK;
}

// ---------------------------------------------------------------------------
// Differentiable runs: Euler-Maruyama Model A, the ideal step, or the two in
// sequence, with the noise fixed by seed and counter.
namespace {

int adj_realloc(double **p, size_t *len, size_t n) {
  if (*p && *len >= n) return LGV_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *len = 0;
  LGV_TRY(ensure(p, n));
  *len = n;
  return LGV_OK;
}

// planes first .. first+n-1 of a buffer of V-double planes as Fields c[0..n-1]
Fields planes(double *base, size_t V, size_t first, int n) {
  Fields f{};
  for (int l = 0; l < n; ++l) f.c[l] = base + (first + l) * V;
  return f;
}

// the reduction buffers of the differentiable run: CTA partials, the
// grid_sum4 counter (zeroed once, re-armed by the kernels) and g4
int adj_counters(lgv_handle *h) {
  auto &A = h->adj;
  if (!A.partial) LGV_TRY(ensure(&A.partial, lgv::em_reduce_blocks(h->N) * 4));
  if (!A.g4) LGV_TRY(ensure(&A.g4, 4));
  if (!A.done) {
    LGV_CK(cudaMalloc((void **)&A.done, sizeof(unsigned)));
    LGV_CK(cudaMemsetAsync(A.done, 0, sizeof(unsigned), h->stream));
  }
  return LGV_OK;
}

// arguments of Euler-Maruyama step number ctr at time t (counter noise), as sub_em builds them
lgv::EmArgs em_args(const lgv_params &p, uint64_t key, uint64_t ctr, double dt, double t) {
  lgv::EmArgs e{};
  e.c6 = 6.0 + (p.mass0 + p.dmassdt * t);
  e.dtg = dt * p.gamma;
  e.sq = std::sqrt(2.0 * p.gamma * dt);
  e.lambda = p.lambda;
  e.H = p.H;
  e.sk = lgv::sub_key(key, ctr);
  return e;
}

// arguments of an ideal step of size dt, as sub_ideal builds them
lgv::IdealArgs ideal_args(const lgv_params &p, int N, double dt, const lgv_handle *h) {
  lgv::IdealArgs a{};
  a.dto2chi = (dt / 2.0) / p.chi;
  a.dt = dt;
  const double hx = p.LX / N;
  a.a2 = std::pow(1.0 / hx, 2);
  a.H = p.H;
  a.waits = h->waits_dev;
  a.wait_limit = h->wait_limit;
  return a;
}

bool has_ideal(int ev) { return ev == LGV_IDEAL_PV2 || ev == LGV_IDEAL_EM; }
bool has_em(int ev) { return ev == LGV_MODELA_EM || ev == LGV_IDEAL_EM; }

}  // namespace

int lgv_diff_forward(lgv_handle *h, int evolver, double dt, double t, int nsteps, int avg_begin, int ckpt_every,
                     double *obs) {
  if (!h || !obs) return fail(LGV_ERR_INVALID, "NULL argument");
  LGV_TRY(no_slab(h, "lgv_diff_forward"));
  if (!has_ideal(evolver) && !has_em(evolver))
    return fail(LGV_ERR_INVALID, "lgv_diff_forward: evolver %d has no adjoint (LGV_MODELA_EM, LGV_IDEAL_PV2, LGV_IDEAL_EM)",
                evolver);
  if (nsteps < 1 || avg_begin < 0 || avg_begin >= nsteps || ckpt_every < 1)
    return fail(LGV_ERR_INVALID, "lgv_diff_forward: need nsteps >= 1, 0 <= avg_begin < nsteps, ckpt_every >= 1");
  if (has_em(evolver) && h->noise_mode != LGV_NOISE_COUNTER)
    return fail(LGV_ERR_STATE, "lgv_diff_forward needs counter noise");
  DeviceGuard g(h->device);
  auto &A = h->adj;
  A.ready = false;
  const size_t V = h->V;
  const int S = nsteps, K = ckpt_every;
  A.ev = evolver;
  A.ncomp = has_ideal(evolver) ? 10 : 4;
  const size_t nck = (size_t)(S - 1) / K + 1;
  LGV_TRY(adj_realloc(&A.ckpt, &A.ckpt_len, nck * A.ncomp * V));
  LGV_TRY(adj_realloc(&A.avg_dev, &A.avg_len, (size_t)(S + 1) * 4));
  LGV_TRY(adj_counters(h));
  A.dt = dt;
  A.S = S;
  A.b = avg_begin;
  A.K = K;
  A.ctr0 = h->ctr;
  A.p = h->p;
  A.key = h->key;
  A.tn.assign(S + 1, 0.0);
  A.tn[0] = t;
  for (int n = 0; n < S; ++n) A.tn[n + 1] = A.tn[n] + dt;
  const lgv::IdealArgs ia = ideal_args(A.p, h->N, dt, h);
  LGV_CK(lgv::launch_phi_avg(h->cur, h->N, A.partial, A.done, A.avg_dev, h->stream));
  for (int n = 0; n < S; ++n) {
    if (n % K == 0)
      for (int l = 0; l < A.ncomp; ++l)
        LGV_CK(cudaMemcpyAsync(A.ckpt + ((size_t)(n / K) * A.ncomp + l) * V, h->cur.c[l], V * sizeof(double),
                               cudaMemcpyDeviceToDevice, h->stream));
    double *avg_n = A.avg_dev + (size_t)(n + 1) * 4;
    if (has_ideal(evolver)) {
      KTimer tm(h, LGV_KCLASS_IDEAL);
      LGV_CK(lgv::launch_ideal(h->cur, h->alt, h->N, ia, h->stream));
      std::swap(h->cur, h->alt);
    }
    if (has_em(evolver)) {
      KTimer tm(h, LGV_KCLASS_EM);
      const lgv::EmArgs e = em_args(A.p, A.key, A.ctr0 + (uint64_t)n, dt, A.tn[n]);
      LGV_CK(lgv::launch_em_avg(h->cur, h->alt, h->N, e, A.partial, A.done, avg_n, h->stream));
      for (int l = 0; l < 4; ++l) std::swap(h->cur.c[l], h->alt.c[l]);
    } else {
      LGV_CK(lgv::launch_phi_avg(h->cur, h->N, A.partial, A.done, avg_n, h->stream));
    }
  }
  if (has_em(evolver)) h->ctr += (uint64_t)S;
  A.avg.assign((size_t)(S + 1) * 4, 0.0);
  LGV_CK(cudaMemcpyAsync(A.avg.data(), A.avg_dev, A.avg.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  // obs[0] = (1/M) sum_{n=b+1}^{S} sigma(n),  obs[1] = (1/M) sum_{n=b+1}^{S} V sum_{a=1..3} pibar_a(n)^2,
  // M = S - b, sigma and pibar_a the volume averages of phi_0 and phi_a after step n
  const double Vd = (double)V;
  double o0 = 0, o1 = 0;
  for (int n = avg_begin + 1; n <= S; ++n) {
    const double *a = &A.avg[(size_t)n * 4];
    o0 += a[0];
    o1 += Vd * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
  }
  obs[0] = o0 / (double)(S - avg_begin);
  obs[1] = o1 / (double)(S - avg_begin);
  A.ready = true;
  return LGV_OK;
}

int lgv_diff_averages(lgv_handle *h, double *out, int nsteps) {
  if (!h || !out) return fail(LGV_ERR_INVALID, "NULL argument");
  if (!h->adj.ready) return fail(LGV_ERR_STATE, "lgv_diff_averages: no forward run");
  if (nsteps != h->adj.S)
    return fail(LGV_ERR_INVALID, "lgv_diff_averages: nsteps %d != forward's %d", nsteps, h->adj.S);
  std::copy(h->adj.avg.begin(), h->adj.avg.end(), out);
  return LGV_OK;
}

int lgv_diff_backward(lgv_handle *h, const double *w, double *grad) {
  if (!h || !w || !grad) return fail(LGV_ERR_INVALID, "NULL argument");
  auto &A = h->adj;
  if (!A.ready) return fail(LGV_ERR_STATE, "lgv_diff_backward: no forward run to differentiate");
  DeviceGuard g(h->device);
  const size_t V = h->V;
  const int S = A.S, K = A.K, M = S - A.b, nc = A.ncomp, N = h->N;
  const int ev = A.ev;
  LGV_TRY(adj_realloc(&A.seg, &A.seg_len, (size_t)K * nc * V));
  LGV_TRY(adj_realloc(&A.lam, &A.lam_len, 2 * 10 * V));
  if (has_ideal(ev)) LGV_TRY(adj_realloc(&A.work, &A.work_len, 28 * V));
  LGV_TRY(adj_counters(h));
  LGV_CK(cudaMemsetAsync(A.g4, 0, 4 * sizeof(double), h->stream));
  const double Vd = (double)V;
  // dJ/dphi_a(x, n) of J = w0 obs0 + w1 obs1: w0 / (M V) for a = 0, w1 2 pibar_a(n) / M for a >= 1
  auto gl = [&](int n, double out[4]) {
    for (int a = 0; a < 4; ++a) out[a] = 0;
    if (n <= A.b) return;
    const double *av = &A.avg[(size_t)n * 4];
    out[0] = w[0] / (Vd * M);
    for (int a = 1; a < 4; ++a) out[a] = w[1] * 2.0 * av[a] / M;
  };
  const lgv::IdealArgs ia = ideal_args(A.p, N, A.dt, h);
  lgv::IdealAdjArgs iadj{};
  iadj.k = ia.dto2chi;
  iadj.dt = ia.dt;
  iadj.a2 = ia.a2;
  iadj.H = ia.H;
  // work planes: tmp state (0..9), phi adjoint after the EM step (10..13), P1 (14..17), PB (18..21), QB (22..27)
  const Fields tmp = planes(A.work, V, 0, 10), lamx = planes(A.work, V, 10, 4), P1 = planes(A.work, V, 14, 4),
               PB = planes(A.work, V, 18, 4), QB = planes(A.work, V, 22, 6);
  auto lam = [&](int which) { return planes(A.lam, V, (size_t)which * 10, 10); };
  auto slot = [&](int m) { return planes(A.seg, V, (size_t)m * nc, nc); };
  int cur = 0;
  {
    double v[4];
    gl(S, v);
    LGV_CK(cudaMemsetAsync(A.lam, 0, 10 * V * sizeof(double), h->stream));
    LGV_CK(lgv::launch_fill_phi(lam(0), N, v, h->stream));
  }
  int loaded = -1;
  for (int n = S - 1; n >= 0; --n) {
    const int s = n / K;
    if (s != loaded) {
      // states u_{sK} .. u_{min(sK+K, S)-1} again from the checkpoint, with the forward's noise
      for (int l = 0; l < nc; ++l)
        LGV_CK(cudaMemcpyAsync(A.seg + (size_t)l * V, A.ckpt + ((size_t)s * nc + l) * V, V * sizeof(double),
                               cudaMemcpyDeviceToDevice, h->stream));
      const int last = std::min(s * K + K - 1, S - 1);
      for (int m = s * K; m < last; ++m) {
        const Fields a = slot(m - s * K), b = slot(m - s * K + 1);
        const lgv::EmArgs e = em_args(A.p, A.key, A.ctr0 + (uint64_t)m, A.dt, A.tn[m]);
        if (ev == LGV_MODELA_EM) {
          LGV_CK(lgv::launch_em(a, b, N, e, h->stream));
        } else if (ev == LGV_IDEAL_PV2) {
          LGV_CK(lgv::launch_ideal(a, b, N, ia, h->stream));
        } else {
          Fields mid = b;  // phi to tmp, charges straight into the next slot
          for (int l = 0; l < 4; ++l) mid.c[l] = tmp.c[l];
          LGV_CK(lgv::launch_ideal(a, mid, N, ia, h->stream));
          LGV_CK(lgv::launch_em(mid, b, N, e, h->stream));
        }
      }
      loaded = s;
    }
    const Fields u = slot(n - s * K);
    double gln[4];
    gl(n, gln);
    if (has_em(ev)) {
      lgv::EmAdjArgs a{};
      a.c6 = 6.0 + (A.p.mass0 + A.p.dmassdt * A.tn[n]);
      a.dtg = A.dt * A.p.gamma;
      a.dt = A.dt;
      a.lambda = A.p.lambda;
      a.H = A.p.H;
      a.cxi = std::sqrt(2.0 * A.dt) / (2.0 * std::sqrt(A.p.gamma));
      a.sk = lgv::sub_key(A.key, A.ctr0 + (uint64_t)n);
      if (ev == LGV_MODELA_EM) {
        for (int q = 0; q < 4; ++q) a.gl[q] = gln[q];
        LGV_CK(lgv::launch_em_adjoint(u, lam(cur), lam(cur ^ 1), N, a, A.partial, A.done, A.g4, h->stream));
      } else {
        LGV_CK(lgv::launch_ideal(u, tmp, N, ia, h->stream));
        LGV_CK(lgv::launch_em_adjoint(tmp, lam(cur), lamx, N, a, A.partial, A.done, A.g4, h->stream));
        Fields lmid = lam(cur);  // charges' adjoint passes the EM step unchanged
        for (int l = 0; l < 4; ++l) lmid.c[l] = lamx.c[l];
        for (int q = 0; q < 4; ++q) iadj.gl[q] = gln[q];
        LGV_CK(lgv::launch_ideal_adjoint(u, lmid, lam(cur ^ 1), P1, PB, QB, N, iadj, A.partial, A.done, A.g4,
                                         h->stream));
      }
    } else {
      for (int q = 0; q < 4; ++q) iadj.gl[q] = gln[q];
      LGV_CK(lgv::launch_ideal_adjoint(u, lam(cur), lam(cur ^ 1), P1, PB, QB, N, iadj, A.partial, A.done, A.g4,
                                       h->stream));
    }
    cur ^= 1;
  }
  LGV_CK(cudaMemcpyAsync(grad, A.g4, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  return LGV_OK;
}

int lgv_debug_flags(lgv_handle *h, int enable) {
  if (!h) return fail(LGV_ERR_INVALID, "handle is NULL");
  if (enable) LGV_TRY(no_slab(h, "per-site flags"));
  DeviceGuard g(h->device);
  if (enable) {
    if (!h->flags_dev) {
      cudaError_t e = cudaMalloc((void **)&h->flags_dev, 36 * h->V);
      if (e != cudaSuccess) return fail(LGV_ERR_NOMEM, "flags alloc: %s", cudaGetErrorString(e));
    }
    LGV_CK(cudaMemsetAsync(h->flags_dev, 0, 36 * h->V, h->stream));
  } else if (h->flags_dev) {
    LGV_CK(cudaStreamSynchronize(h->stream));
    cudaFree(h->flags_dev);
    h->flags_dev = nullptr;
  }
  return LGV_OK;
}

int lgv_get_flags(lgv_handle *h, uint8_t *host_out) {
  if (!h || !host_out) return fail(LGV_ERR_INVALID, "NULL argument");
  if (!h->flags_dev) return fail(LGV_ERR_STATE, "debug flags not enabled");
  DeviceGuard g(h->device);
  LGV_CK(cudaMemcpyAsync(host_out, h->flags_dev, 36 * h->V, cudaMemcpyDeviceToHost, h->stream));
  LGV_CK(cudaStreamSynchronize(h->stream));
  return LGV_OK;
}

}  // extern "C"

// lgv_ensemble.cu -- batched ensembles of independent lattices.
//
// The reference runs an ensemble as separate processes or events, one lattice
// at a time (eventmode loop SuperPions.cxx:228-235; SLURM job arrays,
// grunner.py:153-241).  Here R replicas of any mix of sizes, seeds and
// coefficients advance together: each sub-step is one launch over all of them
// (per-replica block ranges of a flat grid), a captured CUDA graph replays two
// steps at a time, and a small autotuner picks the ideal-kernel tile shape,
// its z-chunk and the order in which replicas are packed into the grid.
// Replica r evolves exactly as a single lgv handle created with params[r]
// and stepped with the same counter (same kernels, same streams).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/lgv.h"
#include "lgv_internal.h"

void lgv_internal_set_error(const char *msg);

using lgv::EnsDyn;
using lgv::Fields;
using lgv::RepDesc;

namespace {

int efail(int code, const std::string &msg) {
  lgv_internal_set_error(msg.c_str());
  // as fail() in lgv_capi.cu: the reported runtime error must not surface
  // again at the next launch
  if (code == LGV_ERR_CUDA || code == LGV_ERR_NOMEM) (void)cudaGetLastError();
  return code;
}

#define ECK(call)                                                                                    \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) return efail(LGV_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define ETRY(x)                 \
  do {                          \
    int r_ = (x);               \
    if (r_ != LGV_OK) return r_; \
  } while (0)

constexpr size_t kSkew = 4352;  // same plane skew as single lattices

struct BlockMap {
  int *rep = nullptr, *first = nullptr, *count = nullptr;
  int nblocks = 0;
};

}  // namespace

struct lgv_ensemble {
  int R = 0;
  int device = 0;
  std::vector<lgv_params> p;
  std::vector<RepDesc> hd;
  std::vector<double *> bufs;
  RepDesc *dd = nullptr;
  EnsDyn *dyn = nullptr;
  BlockMap ideal_map, plane_map, slab_map, tma_map;  // tma_map: ideal step of the TMA replicas
  std::vector<char> tma_ok;                          // replica r takes the TMA ideal kernel
  void *gmaps = nullptr;                             // their tensor maps, [R][2][2][10] x 128 B
  double *partial = nullptr, *oavg = nullptr;
  cudaStream_t own = nullptr, stream = nullptr;
  int phase_phi = 0, phase_q = 0;
  unsigned long long ctr = 0;
  int tile = LGV_TILE_32x8, zchunk = 16, order = LGV_PACK_GIVEN;
  bool graphs = true;
  std::map<std::tuple<int, int, int, double, int, int>, cudaGraphExec_t> cache;
  // bounded device waits of this ensemble's TMA ideal launches that gave up,
  // and the polls before one gives up (LGV_WAIT_LIMIT at creation)
  unsigned long long *waits = nullptr;
  int wait_limit = lgv::kWaitLimit;
  // The ideal step's two launches (TMA replicas, cp.async replicas) write
  // disjoint replicas: the cp.async one runs on `side`, forked from and joined
  // back into `stream` by events (also inside graph capture), so the two
  // overlap.  LGV_ENS_CONCURRENT=0 at creation keeps them in sequence.
  bool concurrent = true;
  cudaStream_t side = nullptr;
  // every replica's element offsets fit 31 bits (set at creation)
  bool idx32 = false;
  // one cooperative launch per step instead of one launch per sub-step
  // (lgv_ensemble_use_persistent; LGV_ENS_PERSISTENT=1 at creation), and its
  // grid barrier (arrivals, generation, error flag)
  bool persistent = false;
  unsigned *bar = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // differentiable Euler-Maruyama run (lgv_ensemble_diff_forward / _backward)
  struct {
    bool ready = false;
    double dt = 0;
    int S = 0, b = 0, K = 1;
    unsigned long long ctr0 = 0;
    std::vector<double> tn;
    std::vector<lgv::DiffDesc> hd;
    std::vector<double *> bufs;
    std::vector<size_t> lens;
    lgv::DiffDesc *dd = nullptr;
    double *wg = nullptr;  // [R][2] weights then [R][4] gradients
    double *partial = nullptr;
    unsigned *done = nullptr;  // one counter per replica
    size_t partial_len = 0;
  } diff;
};

namespace {

// After a stream synchronisation: a bounded wait that gave up in this
// ensemble's launches is reported once, as LGV_ERR_TIMEOUT (the states of the
// replicas it touched are not valid).
int ens_check_waits(lgv_ensemble *e) {
  unsigned long long n = 0;
  if (!e->waits) return LGV_OK;
  ECK(cudaMemcpyAsync(&n, e->waits, sizeof(n), cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  if (n) {
    ECK(cudaMemsetAsync(e->waits, 0, sizeof(n), e->stream));
    if (e->bar) ECK(cudaMemsetAsync(e->bar, 0, 3 * sizeof(unsigned), e->stream));  // a barrier that gave up
    return efail(LGV_ERR_TIMEOUT, "bounded device waits timed out: " + std::to_string(n) +
                                      " TMA copy waits of the ideal step; the ensemble state is not valid");
  }
  return LGV_OK;
}

void free_map(BlockMap &m) {
  if (m.rep) cudaFree(m.rep);
  if (m.first) cudaFree(m.first);
  if (m.count) cudaFree(m.count);
  m = BlockMap{};
}

void clear_graphs(lgv_ensemble *e) {
  for (auto &kv : e->cache) cudaGraphExecDestroy(kv.second);
  e->cache.clear();
}

std::vector<int> pack_order(const lgv_ensemble *e) {
  std::vector<int> o(e->R);
  std::iota(o.begin(), o.end(), 0);
  if (e->order == LGV_PACK_LARGEST_FIRST) {
    std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return e->p[a].N > e->p[b].N; });
  } else if (e->order == LGV_PACK_INTERLEAVED) {
    // round robin over the size classes, largest class first
    std::map<int, std::vector<int>, std::greater<int>> cls;
    for (int r = 0; r < e->R; ++r) cls[e->p[r].N].push_back(r);
    o.clear();
    size_t depth = 0;
    bool any = true;
    while (any) {
      any = false;
      for (auto &c : cls)
        if (depth < c.second.size()) {
          o.push_back(c.second[depth]);
          any = true;
        }
      ++depth;
    }
  }
  return o;
}

int build_map(lgv_ensemble *e, BlockMap &m, const std::vector<int> &blocks_per_rep) {
  free_map(m);
  const std::vector<int> o = pack_order(e);
  std::vector<int> rep, first(e->R), count(e->R);
  for (int r : o) {
    first[r] = (int)rep.size();
    count[r] = blocks_per_rep[r];
    rep.insert(rep.end(), blocks_per_rep[r], r);
  }
  m.nblocks = (int)rep.size();
  ECK(cudaMalloc((void **)&m.rep, std::max<size_t>(rep.size(), 1) * sizeof(int)));
  ECK(cudaMalloc((void **)&m.first, e->R * sizeof(int)));
  ECK(cudaMalloc((void **)&m.count, e->R * sizeof(int)));
  ECK(cudaMemcpy(m.rep, rep.data(), rep.size() * sizeof(int), cudaMemcpyHostToDevice));
  ECK(cudaMemcpy(m.first, first.data(), e->R * sizeof(int), cudaMemcpyHostToDevice));
  ECK(cudaMemcpy(m.count, count.data(), e->R * sizeof(int), cudaMemcpyHostToDevice));
  return LGV_OK;
}

// Replicas with N divisible by 32 take the TMA ideal kernel: encode the
// tensor maps of their component planes for every (phi buffer, charge
// buffer) pairing once, since the buffers never move.  LGV_IDEAL_TMA=0 keeps
// every replica on the cp.async kernel, as for single lattices.
int tensor_maps(lgv_ensemble *e) {
  const char *env = std::getenv("LGV_IDEAL_TMA");
  const bool off = env && env[0] == '0';
  e->tma_ok.assign(e->R, 0);
  std::vector<unsigned char> host((size_t)e->R * 40 * 128, 0);
  bool any = false;
  for (int r = 0; r < e->R; ++r) {
    const RepDesc &d = e->hd[r];
    if (off || !lgv::ideal_tma_supported(d.g.N)) continue;
    bool ok = true;
    for (int pphi = 0; pphi < 2 && ok; ++pphi)
      for (int pq = 0; pq < 2 && ok; ++pq)
        for (int c = 0; c < 10 && ok; ++c) {
          const double *plane = d.base[c < 4 ? pphi : pq] + (size_t)c * d.pstride;
          ok = lgv::tma_plane_map(plane, d.g.N, &host[(((size_t)r * 2 + pphi) * 2 + pq) * 10 * 128 + (size_t)c * 128]);
        }
    e->tma_ok[r] = ok ? 1 : 0;
    any = any || ok;
  }
  if (!any) return LGV_OK;
  ECK(cudaMalloc(&e->gmaps, host.size()));
  ECK(cudaMemcpy(e->gmaps, host.data(), host.size(), cudaMemcpyHostToDevice));
  return LGV_OK;
}

// (Re)derive the per-replica launch geometry for the current tuning and
// upload the descriptors and block maps.
int configure(lgv_ensemble *e) {
  int tx = 32, ty = 8;
  lgv::ideal_tile_dims(e->tile, &tx, &ty);
  std::vector<int> ib(e->R), pb(e->R), sb(e->R), tb(e->R);
  for (int r = 0; r < e->R; ++r) {
    RepDesc &d = e->hd[r];
    const int N = d.g.N;
    d.nchunk = (int)(((long long)N * d.g.H + 127) / 128);
    d.igx = (N + tx - 1) / tx;
    d.igy = (N + ty - 1) / ty;
    d.izc = std::min(e->zchunk, N);
    d.igz = (N + d.izc - 1) / d.izc;
    ib[r] = e->tma_ok[r] ? 0 : d.igx * d.igy * d.igz;
    tb[r] = e->tma_ok[r] ? lgv::batch_tma_blocks(N, d.izc) : 0;
    pb[r] = d.nchunk * N;
    sb[r] = d.nchunk * ((N + lgv::kBatchPlanes - 1) / lgv::kBatchPlanes);
  }
  ECK(cudaMemcpy(e->dd, e->hd.data(), e->R * sizeof(RepDesc), cudaMemcpyHostToDevice));
  ETRY(build_map(e, e->ideal_map, ib));
  ETRY(build_map(e, e->tma_map, tb));
  ETRY(build_map(e, e->plane_map, pb));
  ETRY(build_map(e, e->slab_map, sb));
  if (e->partial) cudaFree(e->partial);
  e->partial = nullptr;
  ECK(cudaMalloc((void **)&e->partial, (size_t)e->plane_map.nblocks * 11 * sizeof(double)));
  clear_graphs(e);
  return LGV_OK;
}

// Counter use per step, identical to the single-lattice sequencing
// (lgv_capi.cu step_once): one per phi sweep, 7 per charge step, 1 per EM step.
int step_ctr(int ev, int inner, int outer) {
  switch (ev) {
    case LGV_PV2HBSPLIT: return inner * outer + 7;
    case LGV_PV2HBSPLIT_NODIFFUSE: return inner * outer;
    case LGV_PV2HBSPLIT_ONLYDIFFUSE: return 7;
    case LGV_IDEAL_PV2: return 0;
    case LGV_EULER_LANGEVIN_HB: return 1;
    case LGV_CHARGE_HB: return 7;
    case LGV_MODELA_EM: return 1;
    default: return -1;
  }
}

// Sub-step phases of one step (the persistent launch's plan), or -1 for an
// evolver it does not run (Euler-Maruyama keeps its own kernel).
int persist_phases(int ev, int inner, int outer) {
  switch (ev) {
    case LGV_PV2HBSPLIT: return outer * (1 + 2 * inner) + 6;
    case LGV_PV2HBSPLIT_NODIFFUSE: return outer * (1 + 2 * inner);
    case LGV_PV2HBSPLIT_ONLYDIFFUSE: return 6;
    case LGV_IDEAL_PV2: return 1;
    case LGV_EULER_LANGEVIN_HB: return 2;
    case LGV_CHARGE_HB: return 6;
    default: return -1;
  }
}

// One step as one cooperative launch (lgv::launch_ens_persistent): the same
// sub-steps, buffer phases and counter offsets as enqueue_step below, as the
// phases of a plan.
int enqueue_step_persistent(lgv_ensemble *e, int ev, int inner, int outer, double dt) {
  lgv::PersistPlan P{};
  P.nb_tma = e->tma_map.nblocks;
  P.nb_cp = e->ideal_map.nblocks;
  P.nb_slab = e->slab_map.nblocks;
  P.tile = e->tile;
  P.wait_limit = e->wait_limit;
  int off = 0;
  auto add = [&](int kind, int arg, double d) {
    lgv::PersistPhase &ph = P.ph[P.nphase++];
    ph.kind = kind;
    ph.arg = arg;
    ph.pphi = e->phase_phi;
    ph.pq = e->phase_q;
    ph.ctr_off = off;
    ph.dt = d;
  };
  auto ideal = [&](double d) {
    add(lgv::kPersistIdeal, 0, d);
    e->phase_phi ^= 1;
    e->phase_q ^= 1;
  };
  auto hb = [&](double d) {
    for (int parity = 0; parity < 2; ++parity) add(lgv::kPersistPhi, parity, d);
    off += 1;
  };
  auto charge = [&](double d) {
    for (int pass = 0; pass < 6; ++pass) add(lgv::kPersistCharge, pass, d);
    off += 7;
  };
  switch (ev) {
    case LGV_PV2HBSPLIT:
    case LGV_PV2HBSPLIT_NODIFFUSE:
    case LGV_PV2HBSPLIT_ONLYDIFFUSE:
      if (ev != LGV_PV2HBSPLIT_ONLYDIFFUSE)
        for (int i1 = 0; i1 < outer; ++i1) {
          ideal(dt / (unsigned)outer);
          for (int i0 = 0; i0 < inner; ++i0) hb(dt / ((unsigned)inner * (unsigned)outer));
        }
      if (ev != LGV_PV2HBSPLIT_NODIFFUSE) charge(dt);
      break;
    case LGV_IDEAL_PV2: ideal(dt); break;
    case LGV_EULER_LANGEVIN_HB: hb(dt); break;
    case LGV_CHARGE_HB: charge(dt); break;
    default: return efail(LGV_ERR_INVALID, "ensemble: evolver without a persistent plan");
  }
  P.dctr = (unsigned long long)off;
  P.dt_step = dt;
  lgv::PersistPtrs q{};
  q.d = e->dd;
  q.dyn = e->dyn;
  q.gmaps = e->gmaps;
  q.tma_rep = e->tma_map.rep;
  q.tma_first = e->tma_map.first;
  q.cp_rep = e->ideal_map.rep;
  q.cp_first = e->ideal_map.first;
  q.slab_rep = e->slab_map.rep;
  q.slab_first = e->slab_map.first;
  q.waits = e->waits;
  q.bar = e->bar;
  ECK(lgv::launch_ens_persistent(P, q, e->idx32, e->stream));
  e->ctr += (unsigned long long)off;
  return LGV_OK;
}

// Enqueue one step on e->stream (also used inside graph capture).
int enqueue_step(lgv_ensemble *e, int ev, int inner, int outer, double dt) {
  if (e->persistent) {
    const int np = persist_phases(ev, inner, outer);
    if (np > 0 && np <= lgv::kMaxPersistPhases) return enqueue_step_persistent(e, ev, inner, outer, dt);
  }
  const int nb_i = e->ideal_map.nblocks, nb_p = e->plane_map.nblocks, nb_s = e->slab_map.nblocks;
  int off = 0;
  auto ideal = [&](double d) -> int {
    const bool both = e->concurrent && e->side && e->tma_map.nblocks > 0 && nb_i > 0;
    if (both) {
      ECK(cudaEventRecord(e->fork, e->stream));
      ECK(cudaStreamWaitEvent(e->side, e->fork, 0));
    }
    if (e->tma_map.nblocks > 0)
      ECK(lgv::launch_batch_ideal_tma(e->dd, e->gmaps, e->tma_map.rep, e->tma_map.first, e->tma_map.nblocks,
                                      e->phase_phi, e->phase_q, d, e->waits, e->wait_limit, e->stream));
    if (nb_i > 0)
      ECK(lgv::launch_batch_ideal(e->dd, e->ideal_map.rep, e->ideal_map.first, nb_i, e->tile, e->phase_phi,
                                  e->phase_q, d, both ? e->side : e->stream));
    if (both) {
      ECK(cudaEventRecord(e->join, e->side));
      ECK(cudaStreamWaitEvent(e->stream, e->join, 0));
    }
    // the ideal step writes all ten components to the other buffer
    e->phase_phi ^= 1;
    e->phase_q ^= 1;
    return LGV_OK;
  };
  auto hb = [&](double d) -> int {
    for (int parity = 0; parity < 2; ++parity)
      ECK(lgv::launch_batch_hb(e->dd, e->dyn, e->slab_map.rep, e->slab_map.first, nb_s, e->phase_phi, parity, d, off,
                               e->idx32, e->stream));
    off += 1;
    return LGV_OK;
  };
  auto charge = [&](double d) -> int {
    for (int pass = 0; pass < 6; ++pass)
      ECK(lgv::launch_batch_charge(e->dd, e->dyn, e->slab_map.rep, e->slab_map.first, nb_s, e->phase_q, pass, d,
                                   off, e->idx32, e->stream));
    off += 7;
    return LGV_OK;
  };
  switch (ev) {
    case LGV_PV2HBSPLIT:
    case LGV_PV2HBSPLIT_NODIFFUSE:
    case LGV_PV2HBSPLIT_ONLYDIFFUSE:
      if (ev != LGV_PV2HBSPLIT_ONLYDIFFUSE)
        for (int i1 = 0; i1 < outer; ++i1) {
          ETRY(ideal(dt / (unsigned)outer));
          for (int i0 = 0; i0 < inner; ++i0) ETRY(hb(dt / ((unsigned)inner * (unsigned)outer)));
        }
      if (ev != LGV_PV2HBSPLIT_NODIFFUSE) ETRY(charge(dt));
      break;
    case LGV_IDEAL_PV2: ETRY(ideal(dt)); break;
    case LGV_EULER_LANGEVIN_HB: ETRY(hb(dt)); break;
    case LGV_CHARGE_HB: ETRY(charge(dt)); break;
    case LGV_MODELA_EM:
      ECK(lgv::launch_batch_em(e->dd, e->dyn, e->plane_map.rep, e->plane_map.first, nb_p, e->phase_phi, dt, off,
                               e->stream));
      e->phase_phi ^= 1;
      off += 1;
      break;
    default: return efail(LGV_ERR_INVALID, "ensemble: unknown evolver");
  }
  ECK(lgv::launch_ens_advance(e->dyn, (unsigned long long)off, dt, e->stream));
  e->ctr += (unsigned long long)off;
  return LGV_OK;
}

Fields cur_fields(const lgv_ensemble *e, int r) {
  Fields f;
  const RepDesc &d = e->hd[r];
  for (int L = 0; L < 10; ++L) f.c[L] = d.base[L < 4 ? e->phase_phi : e->phase_q] + (size_t)L * d.pstride;
  return f;
}

int check_rep(const lgv_ensemble *e, int r) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  if (r < 0 || r >= e->R) return efail(LGV_ERR_INVALID, "replica index out of range");
  return LGV_OK;
}

}  // namespace

extern "C" {

int lgv_ensemble_create(int nrep, const lgv_params *params, lgv_ensemble **out) {
  if (!out || !params || nrep < 1) return efail(LGV_ERR_INVALID, "lgv_ensemble_create: bad arguments");
  *out = nullptr;
  for (int r = 0; r < nrep; ++r) {
    const lgv_params &q = params[r];
    if (q.N < 4 || (q.N & 1) || q.N > 2048 || q.reserved0 != 0 || !(q.chi > 0) || !(q.LX > 0))
      return efail(LGV_ERR_INVALID, "lgv_ensemble_create: replica " + std::to_string(r) + " has invalid params");
  }
  lgv_ensemble *e = new lgv_ensemble();
  e->R = nrep;
  e->p.assign(params, params + nrep);
  cudaGetDevice(&e->device);
  int rc = LGV_OK;
  auto bail = [&](int code) {
    lgv_ensemble_destroy(e);
    return code;
  };
  if (cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking) != cudaSuccess)
    return bail(efail(LGV_ERR_CUDA, "stream"));
  e->stream = e->own;
  {
    const char *wl = std::getenv("LGV_WAIT_LIMIT");
    if (wl && wl[0]) e->wait_limit = std::max(0, std::atoi(wl));
  }
  if (cudaMalloc((void **)&e->waits, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemset(e->waits, 0, sizeof(unsigned long long)) != cudaSuccess)
    return bail(efail(LGV_ERR_NOMEM, "wait counter"));
  {
    const char *cv = std::getenv("LGV_ENS_CONCURRENT");
    e->concurrent = !(cv && cv[0] == '0');
  }
  if (cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->join, cudaEventDisableTiming) != cudaSuccess)
    return bail(efail(LGV_ERR_CUDA, "side stream"));
  e->hd.resize(nrep);
  for (int r = 0; r < nrep; ++r) {
    const lgv_params &q = params[r];
    RepDesc &d = e->hd[r];
    d.g = lgv::make_geo(q.N);
    d.key = lgv::make_key(q.seed);
    d.mass0 = q.mass0;
    d.dmassdt = q.dmassdt;
    d.lambda = q.lambda;
    d.H = q.H;
    d.chi = q.chi;
    d.gamma = q.gamma;
    d.diffusion = q.diffusion;
    d.a2 = std::pow(1.0 / (q.LX / q.N), 2);
    const size_t V = (size_t)q.N * q.N * q.N;
    d.pstride = (long long)(V + kSkew);
    for (int b = 0; b < 2; ++b) {
      double *buf = nullptr;
      if (cudaMalloc((void **)&buf, 10 * (V + kSkew) * sizeof(double)) != cudaSuccess)
        return bail(efail(LGV_ERR_NOMEM, "ensemble lattice allocation failed"));
      e->bufs.push_back(buf);
      if (cudaMemset(buf, 0, 10 * (V + kSkew) * sizeof(double)) != cudaSuccess) return bail(efail(LGV_ERR_CUDA, "memset"));
      d.base[b] = buf;
    }
  }
  e->idx32 = lgv::batch_idx32(e->hd.data(), nrep);
  if (cudaMalloc((void **)&e->bar, 3 * sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(e->bar, 0, 3 * sizeof(unsigned)) != cudaSuccess)
    return bail(efail(LGV_ERR_NOMEM, "grid barrier"));
  {
    const char *pv = std::getenv("LGV_ENS_PERSISTENT");
    e->persistent = pv && pv[0] == '1' && lgv::persist_grid(e->idx32) > 0;
  }
  if (cudaMalloc((void **)&e->dd, nrep * sizeof(RepDesc)) != cudaSuccess ||
      cudaMalloc((void **)&e->dyn, sizeof(EnsDyn)) != cudaSuccess ||
      cudaMalloc((void **)&e->oavg, (size_t)nrep * 11 * sizeof(double)) != cudaSuccess)
    return bail(efail(LGV_ERR_NOMEM, "ensemble tables"));
  if ((rc = tensor_maps(e)) != LGV_OK) return bail(rc);
  if ((rc = configure(e)) != LGV_OK) return bail(rc);
  if (lgv::launch_ens_set(e->dyn, 0, 0.0, e->stream) != cudaSuccess || cudaStreamSynchronize(e->stream) != cudaSuccess)
    return bail(efail(LGV_ERR_CUDA, "ensemble init"));
  *out = e;
  return LGV_OK;
}

int lgv_ensemble_destroy(lgv_ensemble *e) {
  if (!e) return LGV_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  clear_graphs(e);
  for (double *b : e->bufs) cudaFree(b);
  free_map(e->ideal_map);
  free_map(e->plane_map);
  free_map(e->slab_map);
  free_map(e->tma_map);
  if (e->gmaps) cudaFree(e->gmaps);
  if (e->dd) cudaFree(e->dd);
  if (e->dyn) cudaFree(e->dyn);
  if (e->partial) cudaFree(e->partial);
  if (e->oavg) cudaFree(e->oavg);
  for (double *b : e->diff.bufs)
    if (b) cudaFree(b);
  if (e->diff.dd) cudaFree(e->diff.dd);
  if (e->diff.wg) cudaFree(e->diff.wg);
  if (e->diff.partial) cudaFree(e->diff.partial);
  if (e->diff.done) cudaFree(e->diff.done);
  if (e->waits) cudaFree(e->waits);
  if (e->bar) cudaFree(e->bar);
  if (e->side) {
    cudaStreamSynchronize(e->side);
    cudaStreamDestroy(e->side);
  }
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->join) cudaEventDestroy(e->join);
  if (e->own) cudaStreamDestroy(e->own);
  delete e;
  return LGV_OK;
}

int lgv_ensemble_size(lgv_ensemble *e, int *nrep) {
  if (!e || !nrep) return efail(LGV_ERR_INVALID, "NULL argument");
  *nrep = e->R;
  return LGV_OK;
}

int lgv_ensemble_set_state(lgv_ensemble *e, int r, const double *host_aos) {
  ETRY(check_rep(e, r));
  if (!host_aos) return efail(LGV_ERR_INVALID, "NULL state");
  const size_t V = (size_t)e->p[r].N * e->p[r].N * e->p[r].N;
  double *stage = nullptr;
  ECK(cudaMalloc((void **)&stage, 10 * V * sizeof(double)));
  cudaError_t c1 = cudaMemcpyAsync(stage, host_aos, 10 * V * sizeof(double), cudaMemcpyHostToDevice, e->stream);
  cudaError_t c2 = lgv::launch_aos_to_rb(stage, cur_fields(e, r), e->p[r].N, e->stream);
  cudaError_t c3 = cudaStreamSynchronize(e->stream);
  cudaFree(stage);
  ECK(c1);
  ECK(c2);
  ECK(c3);
  return LGV_OK;
}

int lgv_ensemble_get_state(lgv_ensemble *e, int r, double *host_aos) {
  ETRY(check_rep(e, r));
  if (!host_aos) return efail(LGV_ERR_INVALID, "NULL state");
  const size_t V = (size_t)e->p[r].N * e->p[r].N * e->p[r].N;
  double *stage = nullptr;
  ECK(cudaMalloc((void **)&stage, 10 * V * sizeof(double)));
  cudaError_t c1 = lgv::launch_rb_to_aos(cur_fields(e, r), stage, e->p[r].N, e->stream);
  cudaError_t c2 = cudaMemcpyAsync(host_aos, stage, 10 * V * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
  cudaError_t c3 = cudaStreamSynchronize(e->stream);
  cudaFree(stage);
  ECK(c1);
  ECK(c2);
  ECK(c3);
  return ens_check_waits(e);
}

int lgv_ensemble_initialize(lgv_ensemble *e, int kind, double scale) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  double *scratch = nullptr;
  size_t need = 16;
  for (int r = 0; r < e->R; ++r) {
    const size_t V = (size_t)e->p[r].N * e->p[r].N * e->p[r].N;
    need = std::max(need, ((V + 255) / 256) * 6 + 16);
  }
  if (kind == LGV_INIT_CHARGES_GAUSSIAN) ECK(cudaMalloc((void **)&scratch, need * sizeof(double)));
  int rc = LGV_OK;
  for (int r = 0; r < e->R && rc == LGV_OK; ++r) {
    const Fields f = cur_fields(e, r);
    const uint64_t sk = lgv::sub_key(e->hd[r].key, e->ctr);
    const size_t V = (size_t)e->p[r].N * e->p[r].N * e->p[r].N;
    cudaError_t c = cudaSuccess;
    if (kind == LGV_INIT_ZERO) {
      for (int L = 0; L < 10 && c == cudaSuccess; ++L) c = cudaMemsetAsync(f.c[L], 0, V * sizeof(double), e->stream);
    } else if (kind == LGV_INIT_PHI_GAUSSIAN) {
      c = lgv::launch_init_phi(f, e->p[r].N, sk, scale, e->stream);
    } else if (kind == LGV_INIT_CHARGES_GAUSSIAN) {
      c = lgv::launch_init_charges(f, e->p[r].N, sk, std::sqrt(e->p[r].chi), scratch, e->stream);
    } else {
      rc = efail(LGV_ERR_INVALID, "unknown init kind");
    }
    if (c != cudaSuccess) rc = efail(LGV_ERR_CUDA, cudaGetErrorString(c));
  }
  if (scratch) {
    cudaStreamSynchronize(e->stream);
    cudaFree(scratch);
  }
  if (rc != LGV_OK) return rc;
  if (kind != LGV_INIT_ZERO) {
    e->ctr += 1;
    ECK(lgv::launch_ens_set(e->dyn, e->ctr, 0.0, e->stream));
  }
  return LGV_OK;
}

int lgv_ensemble_set_counter(lgv_ensemble *e, uint64_t c) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  e->ctr = c;
  return LGV_OK;
}

int lgv_ensemble_get_counter(lgv_ensemble *e, uint64_t *c) {
  if (!e || !c) return efail(LGV_ERR_INVALID, "NULL argument");
  *c = e->ctr;
  return LGV_OK;
}

int lgv_ensemble_step(lgv_ensemble *e, int evolver, int inner, int outer, double dt, double t, int nsteps) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  if (nsteps < 0 || step_ctr(evolver, inner, outer) < 0) return efail(LGV_ERR_INVALID, "bad evolver or nsteps");
  if (evolver <= LGV_PV2HBSPLIT_ONLYDIFFUSE && (inner < 1 || outer < 1)) return efail(LGV_ERR_INVALID, "scounts");
  ECK(lgv::launch_ens_set(e->dyn, e->ctr, t, e->stream));
  int done = 0;
  if (e->graphs && nsteps >= 2) {
    // two steps return both buffer phases to where they started, so a
    // two-step graph can be replayed back to back
    const auto key = std::make_tuple(evolver, inner, outer, dt, e->phase_phi, e->phase_q);
    auto it = e->cache.find(key);
    if (it == e->cache.end()) {
      const int pp = e->phase_phi, pq = e->phase_q;
      const unsigned long long c0 = e->ctr;
      cudaGraph_t g = nullptr;
      // Capture on the ensemble's own stream: the caller's stream may be the
      // legacy default stream, which cannot be captured.  The graph is then
      // launched on the caller's stream.
      cudaStream_t user = e->stream;
      ECK(cudaStreamBeginCapture(e->own, cudaStreamCaptureModeThreadLocal));
      e->stream = e->own;
      int rc = enqueue_step(e, evolver, inner, outer, dt);
      if (rc == LGV_OK) rc = enqueue_step(e, evolver, inner, outer, dt);
      cudaError_t ce = cudaStreamEndCapture(e->own, &g);
      e->stream = user;
      e->phase_phi = pp;  // capture issued nothing: restore the host mirrors
      e->phase_q = pq;
      e->ctr = c0;
      if (rc != LGV_OK) return rc;
      ECK(ce);
      cudaGraphExec_t ex = nullptr;
      cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      ECK(ie);
      it = e->cache.emplace(key, ex).first;
    }
    const int per = step_ctr(evolver, inner, outer);
    while (nsteps - done >= 2) {
      ECK(cudaGraphLaunch(it->second, e->stream));
      e->ctr += 2ull * (unsigned long long)per;
      done += 2;
    }
  }
  for (; done < nsteps; ++done) ETRY(enqueue_step(e, evolver, inner, outer, dt));
  return LGV_OK;
}

int lgv_ensemble_diff_forward(lgv_ensemble *e, double dt, double t, int nsteps, int avg_begin, int ckpt_every,
                              double *obs) {
  if (!e || !obs) return efail(LGV_ERR_INVALID, "NULL argument");
  if (nsteps < 1 || avg_begin < 0 || avg_begin >= nsteps || ckpt_every < 1)
    return efail(LGV_ERR_INVALID, "lgv_ensemble_diff_forward: need nsteps >= 1, 0 <= avg_begin < nsteps, ckpt_every >= 1");
  auto &D = e->diff;
  D.ready = false;
  const int R = e->R, S = nsteps, K = ckpt_every;
  const size_t nck = (size_t)(S - 1) / K + 1;
  if (D.bufs.empty()) {
    D.bufs.assign(R, nullptr);
    D.lens.assign(R, 0);
    D.hd.assign(R, lgv::DiffDesc{});
    ECK(cudaMalloc((void **)&D.dd, R * sizeof(lgv::DiffDesc)));
    ECK(cudaMalloc((void **)&D.wg, (size_t)R * 6 * sizeof(double)));
    ECK(cudaMalloc((void **)&D.done, R * sizeof(unsigned)));
    ECK(cudaMemsetAsync(D.done, 0, R * sizeof(unsigned), e->stream));
  }
  const size_t need_partial = (size_t)e->plane_map.nblocks * 4 + 16;
  if (D.partial_len < need_partial) {
    if (D.partial) cudaFree(D.partial);
    D.partial = nullptr;
    D.partial_len = 0;
    ECK(cudaMalloc((void **)&D.partial, need_partial * sizeof(double)));
    D.partial_len = need_partial;
  }
  for (int r = 0; r < R; ++r) {
    const size_t V = (size_t)e->p[r].N * e->p[r].N * e->p[r].N;
    // checkpoints, segment states, two adjoint states, averages
    const size_t need = (nck + (size_t)K + 2) * 4 * V + (size_t)(S + 1) * 4;
    if (D.lens[r] < need) {
      if (D.bufs[r]) cudaFree(D.bufs[r]);
      D.bufs[r] = nullptr;
      D.lens[r] = 0;
      ECK(cudaMalloc((void **)&D.bufs[r], need * sizeof(double)));
      D.lens[r] = need;
    }
    lgv::DiffDesc &d = D.hd[r];
    d.V = (long long)V;
    d.ckpt = D.bufs[r];
    d.seg = d.ckpt + nck * 4 * V;
    d.lam = d.seg + (size_t)K * 4 * V;
    d.avg = d.lam + 8 * V;
    d.w = D.wg + 2 * r;
    d.grad = D.wg + 2 * R + 4 * r;
  }
  ECK(cudaMemcpyAsync(D.dd, D.hd.data(), R * sizeof(lgv::DiffDesc), cudaMemcpyHostToDevice, e->stream));
  D.dt = dt;
  D.S = S;
  D.b = avg_begin;
  D.K = K;
  D.ctr0 = e->ctr;
  D.tn.assign(S + 1, 0.0);
  D.tn[0] = t;
  for (int n = 0; n < S; ++n) D.tn[n + 1] = D.tn[n] + dt;
  const BlockMap &pm = e->plane_map;
  for (int r = 0; r < R; ++r)
    ECK(lgv::launch_phi_avg(cur_fields(e, r), e->p[r].N, D.partial, D.done, D.hd[r].avg, e->stream));
  for (int n = 0; n < S; ++n) {
    if (n % K == 0)
      ECK(lgv::launch_batch_diff_copy(e->dd, D.dd, pm.rep, pm.first, pm.nblocks, 0, e->phase_phi, n / K, avg_begin, S,
                                      e->stream));
    ECK(lgv::launch_batch_em_fwd(e->dd, D.dd, pm.rep, pm.first, pm.count, pm.nblocks, e->phase_phi, D.ctr0 + n,
                                 D.tn[n], dt, n, D.partial, D.done, e->stream));
    e->phase_phi ^= 1;
  }
  e->ctr += (unsigned long long)S;
  std::vector<double> avg((size_t)(S + 1) * 4);
  for (int r = 0; r < R; ++r) {
    ECK(cudaMemcpyAsync(avg.data(), D.hd[r].avg, avg.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ECK(cudaStreamSynchronize(e->stream));
    const double Vd = (double)D.hd[r].V;
    double o0 = 0, o1 = 0;
    for (int n = avg_begin + 1; n <= S; ++n) {
      const double *a = &avg[(size_t)n * 4];
      o0 += a[0];
      o1 += Vd * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
    }
    obs[2 * r] = o0 / (double)(S - avg_begin);
    obs[2 * r + 1] = o1 / (double)(S - avg_begin);
  }
  D.ready = true;
  return ens_check_waits(e);
}

int lgv_ensemble_diff_backward(lgv_ensemble *e, const double *w, double *grad) {
  if (!e || !w || !grad) return efail(LGV_ERR_INVALID, "NULL argument");
  auto &D = e->diff;
  if (!D.ready) return efail(LGV_ERR_STATE, "lgv_ensemble_diff_backward: no forward run to differentiate");
  const int R = e->R, S = D.S, K = D.K;
  const BlockMap &pm = e->plane_map;
  ECK(cudaMemcpyAsync(D.wg, w, (size_t)R * 2 * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  ECK(cudaMemsetAsync(D.wg + 2 * R, 0, (size_t)R * 4 * sizeof(double), e->stream));
  ECK(lgv::launch_batch_diff_copy(e->dd, D.dd, pm.rep, pm.first, pm.nblocks, 2, 0, 0, D.b, S, e->stream));
  int cur = 0, loaded = -1;
  for (int n = S - 1; n >= 0; --n) {
    const int s = n / K;
    if (s != loaded) {
      ECK(lgv::launch_batch_diff_copy(e->dd, D.dd, pm.rep, pm.first, pm.nblocks, 1, 0, s, D.b, S, e->stream));
      const int last = std::min(s * K + K - 1, S - 1);
      for (int m = s * K; m < last; ++m)
        ECK(lgv::launch_batch_em_seg(e->dd, D.dd, pm.rep, pm.first, pm.nblocks, m - s * K, D.ctr0 + m, D.tn[m], D.dt,
                                     e->stream));
      loaded = s;
    }
    ECK(lgv::launch_batch_em_adj(e->dd, D.dd, pm.rep, pm.first, pm.count, pm.nblocks, n - s * K, cur, n, D.b, S,
                                 D.ctr0 + n, D.tn[n], D.dt, D.partial, D.done, e->stream));
    cur ^= 1;
  }
  ECK(cudaMemcpyAsync(grad, D.wg + 2 * R, (size_t)R * 4 * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return ens_check_waits(e);
}

int lgv_ensemble_oaverage_device(lgv_ensemble *e, double *dev_out) {
  if (!e || !dev_out) return efail(LGV_ERR_INVALID, "NULL argument");
  ECK(lgv::launch_batch_oavg(e->dd, e->plane_map.rep, e->plane_map.first, e->plane_map.nblocks, e->phase_phi,
                             e->phase_q, e->partial, e->R, dev_out, e->stream));
  ECK(lgv::launch_batch_oavg_final(e->dd, e->plane_map.first, e->plane_map.count, e->R, e->partial, dev_out,
                                   e->stream));
  return LGV_OK;
}

int lgv_ensemble_oaverage(lgv_ensemble *e, double *host_out) {
  if (!e || !host_out) return efail(LGV_ERR_INVALID, "NULL argument");
  ETRY(lgv_ensemble_oaverage_device(e, e->oavg));
  ECK(cudaMemcpyAsync(host_out, e->oavg, (size_t)e->R * 11 * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return ens_check_waits(e);
}

int lgv_ensemble_tune(lgv_ensemble *e, int tile, int zchunk, int order) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  if ((tile != LGV_TILE_32x8 && tile != LGV_TILE_16x16) || zchunk < 1 || order < 0 || order > 2)
    return efail(LGV_ERR_INVALID, "lgv_ensemble_tune: bad choice");
  ECK(cudaStreamSynchronize(e->stream));
  e->tile = tile;
  e->zchunk = zchunk;
  e->order = order;
  return configure(e);
}

int lgv_ensemble_use_graphs(lgv_ensemble *e, int enable) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  e->graphs = enable != 0;
  return LGV_OK;
}

int lgv_ensemble_use_persistent(lgv_ensemble *e, int enable) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  if (enable && lgv::persist_grid(e->idx32) <= 0)
    return efail(LGV_ERR_UNSUPPORTED, "persistent ensemble step: no cooperative launch on this device");
  if ((enable != 0) != e->persistent) {
    ECK(cudaStreamSynchronize(e->stream));
    clear_graphs(e);
  }
  e->persistent = enable != 0;
  return LGV_OK;
}

// Times every (tile, z-chunk, packing order) candidate on a copy of the
// current state (the state and the counter are restored afterwards) and
// keeps the fastest.  choice[3] receives (tile, zchunk, order); ms_per_step
// the candidate's time per step.
int lgv_ensemble_autotune(lgv_ensemble *e, int evolver, int inner, int outer, double dt, int steps, int *choice,
                          double *ms_per_step) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  if (steps < 2) steps = 2;
  ECK(cudaStreamSynchronize(e->stream));
  // save every replica's current buffers
  std::vector<double *> saved;
  const int pp0 = e->phase_phi, pq0 = e->phase_q;
  const unsigned long long c0 = e->ctr;
  for (int r = 0; r < e->R; ++r) {
    const size_t V = (size_t)e->p[r].N * e->p[r].N * e->p[r].N;
    double *s = nullptr;
    if (cudaMalloc((void **)&s, 10 * V * sizeof(double)) != cudaSuccess) {
      for (double *q : saved) cudaFree(q);
      return efail(LGV_ERR_NOMEM, "autotune: no room for the state copy");
    }
    const Fields f = cur_fields(e, r);
    for (int L = 0; L < 10; ++L) cudaMemcpyAsync(s + L * V, f.c[L], V * sizeof(double), cudaMemcpyDeviceToDevice, e->stream);
    saved.push_back(s);
  }
  auto restore = [&]() {
    e->phase_phi = pp0;
    e->phase_q = pq0;
    e->ctr = c0;
    for (int r = 0; r < e->R; ++r) {
      const size_t V = (size_t)e->p[r].N * e->p[r].N * e->p[r].N;
      const Fields f = cur_fields(e, r);
      for (int L = 0; L < 10; ++L)
        cudaMemcpyAsync(f.c[L], saved[r] + L * V, V * sizeof(double), cudaMemcpyDeviceToDevice, e->stream);
    }
    cudaStreamSynchronize(e->stream);
  };
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 1e300;
  int bt = e->tile, bz = e->zchunk, bo = e->order;
  const int tiles[2] = {LGV_TILE_32x8, LGV_TILE_16x16};
  const int zcs[3] = {8, 16, 32};
  int rc = LGV_OK;
  for (int ti = 0; ti < 2 && rc == LGV_OK; ++ti)
    for (int zi = 0; zi < 3 && rc == LGV_OK; ++zi)
      for (int oi = 0; oi < 3 && rc == LGV_OK; ++oi) {
        e->tile = tiles[ti];
        e->zchunk = zcs[zi];
        e->order = oi;
        if ((rc = configure(e)) != LGV_OK) break;
        if ((rc = lgv_ensemble_step(e, evolver, inner, outer, dt, 0.0, 2)) != LGV_OK) break;  // warm / capture
        cudaEventRecord(a, e->stream);
        if ((rc = lgv_ensemble_step(e, evolver, inner, outer, dt, 0.0, steps)) != LGV_OK) break;
        cudaEventRecord(b, e->stream);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms / steps < best) {
          best = ms / steps;
          bt = e->tile;
          bz = e->zchunk;
          bo = e->order;
        }
        restore();
      }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  e->tile = bt;
  e->zchunk = bz;
  e->order = bo;
  int rc2 = configure(e);
  restore();
  for (double *q : saved) cudaFree(q);
  ETRY(rc);
  ETRY(rc2);
  if (choice) {
    choice[0] = bt;
    choice[1] = bz;
    choice[2] = bo;
  }
  if (ms_per_step) *ms_per_step = best;
  return LGV_OK;
}

int lgv_ensemble_set_stream(lgv_ensemble *e, void *s) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  cudaStream_t next = s ? (cudaStream_t)s : (cudaStream_t)0;
  if (next == e->stream) return LGV_OK;
  cudaEvent_t ev;
  ECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  ECK(cudaEventRecord(ev, e->stream));
  ECK(cudaStreamWaitEvent(next, ev, 0));
  cudaEventDestroy(ev);
  e->stream = next;
  return LGV_OK;
}

int lgv_ensemble_synchronize(lgv_ensemble *e) {
  if (!e) return efail(LGV_ERR_INVALID, "ensemble is NULL");
  ECK(cudaStreamSynchronize(e->stream));
  return ens_check_waits(e);
}

}  // extern "C"

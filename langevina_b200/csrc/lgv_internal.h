// lgv_internal.h -- host-side declarations shared by the kernel and C-ABI
// translation units of liblgv.so (not installed, not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/lgv.h"
#include "lgv_device.cuh"

namespace lgv {

// Device monitor accumulator (o4_stepper_monitor, Stepper.h:17-49).
struct MonAcc {
  unsigned long long down_counts, up_counts, up_yes, up_no;
  double down_dS, up_dS;
};

struct HbArgs {
  double rdtg;     // sqrt(2 dt gamma)
  double Lambda2;  // (6 + m^2) / 2
  double lam4;     // lambda / 4
  double H;
  uint64_t sk;          // sub-step key (counter mode)
  const double *prop;   // injected [4][V] or null
  const double *acc;    // injected [V] or null
  uint8_t *flags;       // [V] or null
  MonAcc *mon;          // or null
  int gauss;            // counter noise: Gaussian proposals (lgv_set_hb_proposal); the one-parity pass only
};

struct ChargeArgs {
  double rms;       // sqrt(2 dt sigma)
  double inv2chi;   // 1 / (2 chi)
  uint64_t sk;
  int pass;         // position 0..5 in the step (injected indexing / flags)
  const double *q;    // injected [6][6][V] or null
  const double *acc;  // injected [6][6][V] or null
  uint8_t *flags;     // [36 V] or null
  MonAcc *mon;
};

// Both faces of one direction of the charge heat bath.
struct ChargeDirPair {
  double rms, inv2chi;
  uint64_t sk[2];     // sub-step keys of the two faces
  int pass[2];        // positions of the faces in the step (0..5)
  int eo[2];          // A-site parities, in application order
  const double *q, *acc;  // injected [6][6][V] or null
  uint8_t *flags;
  MonAcc *mon;
};

struct EmArgs {
  double c6;    // 6 + m^2
  double dtg;   // dt * gamma
  double sq;    // sqrt(2 gamma dt)
  double lambda;
  double H;
  uint64_t sk;
  const double *xi;  // injected [4][V] or null
};

struct IdealArgs {
  double dto2chi;  // (dt / 2) / chi  : half-step rotation angle per unit charge
  double dt;
  double a2;       // (1 / h)^2
  double H;
  // Bounded device waits (TMA completion): a wait gives up after wait_limit
  // polls and counts itself in *waits, the owning handle's or ensemble's
  // counter, which the host reads at its next synchronising call.
  unsigned long long *waits;
  int wait_limit;
};

// Polls before a bounded device wait gives up (a few seconds at most).
constexpr int kWaitLimit = 1 << 22;

// ---------------------------------------------------------------------------
// Batched ensembles: many independent lattices advanced by one launch per
// sub-step.  Per-replica data lives in a device table; the sub-step counter
// and the clock live in device memory so that captured CUDA graphs replay
// with advancing noise.
struct RepDesc {
  double *base[2];     // the two lattice buffers; which is current is a launch argument
  long long pstride;   // doubles from one component plane to the next (V + skew)
  Geo g;
  uint64_t key;  // make_key(seed)
  double mass0, dmassdt, lambda, H, chi, gamma, diffusion, a2;
  int nchunk;    // plane kernels: ceil(N * N/2 / 128) blocks per plane
  int igx, igy, igz, izc;  // ideal kernel: tiles in x, y, z and the z-chunk
};
struct EnsDyn {
  unsigned long long ctr;  // counter at the start of the current step
  double t;                // clock at the start of the current step
};


// Differentiable Euler-Maruyama runs of an ensemble: per-replica buffers of
// V-double planes.  ckpt: checkpoint slots of 4 planes; seg: the K states of
// the segment being differentiated; lam: two 4-plane adjoint states; avg:
// (S+1) x 4 volume averages; w: the replica's observable weights.
struct DiffDesc {
  double *ckpt, *seg, *lam, *avg, *w, *grad;
  long long V;
};

// forward step n: phi of the lattice buffer `phase` -> phase ^ 1, averages into avg[n+1]
cudaError_t launch_batch_em_fwd(const RepDesc *d, const DiffDesc *dd, const int *rep, const int *first,
                                const int *count, int nblocks, int phase, unsigned long long ctr, double t, double dt,
                                int n, double *partial, unsigned *done, cudaStream_t st);
// recompute: seg slot m -> m + 1
cudaError_t launch_batch_em_seg(const RepDesc *d, const DiffDesc *dd, const int *rep, const int *first, int nblocks,
                                int m, unsigned long long ctr, double t, double dt, cudaStream_t st);
// adjoint of step n at seg slot m: lam[cur] -> lam[cur ^ 1], gradients into grad
cudaError_t launch_batch_em_adj(const RepDesc *d, const DiffDesc *dd, const int *rep, const int *first,
                                const int *count, int nblocks, int m, int cur, int n, int b, int S,
                                unsigned long long ctr, double t, double dt, double *partial, unsigned *done,
                                cudaStream_t st);
// phi planes: lattice buffer `phase` -> ckpt slot s (dir 0); ckpt slot s -> seg slot 0 (dir 1);
// lam[0] = dJ/dphi(S) from avg and w (dir 2)
cudaError_t launch_batch_diff_copy(const RepDesc *d, const DiffDesc *dd, const int *rep, const int *first,
                                   int nblocks, int dir, int phase, int s, int b, int S, cudaStream_t st);

// planes per block of the batched heat-bath and charge kernels: their block
// map holds nchunk * ceil(N / kBatchPlanes) blocks per replica
constexpr int kBatchPlanes = 4;

// phase_phi / phase_q: which buffer holds the current phi / charges
cudaError_t launch_batch_ideal(const RepDesc *d, const int *rep, const int *first, int nblocks, int tile,
                               int phase_phi, int phase_q, double dt, cudaStream_t st);
// rep / first / nblocks of launch_batch_hb and launch_batch_charge: the slab map (kBatchPlanes planes per block)
// true when every replica's element offsets fit 31 bits (the batched heat-bath
// and charge kernels then index with int; i32 of their launchers)
bool batch_idx32(const RepDesc *hd, int nrep);
cudaError_t launch_batch_hb(const RepDesc *d, const EnsDyn *dyn, const int *rep, const int *first, int nblocks,
                            int phase_phi, int parity, double dt, int ctr_off, bool i32, cudaStream_t st);
cudaError_t launch_batch_charge(const RepDesc *d, const EnsDyn *dyn, const int *rep, const int *first, int nblocks,
                                int phase_q, int pass, double dt, int ctr_off_order, bool i32, cudaStream_t st);
cudaError_t launch_batch_em(const RepDesc *d, const EnsDyn *dyn, const int *rep, const int *first, int nblocks,
                            int phase_phi, double dt, int ctr_off, cudaStream_t st);
cudaError_t launch_ens_set(EnsDyn *dyn, unsigned long long ctr, double t, cudaStream_t st);
cudaError_t launch_ens_advance(EnsDyn *dyn, unsigned long long dctr, double dt, cudaStream_t st);
// volume averages (the 11 OAverage observables) of every replica: partial[nblocks][11], out[nrep][11]
cudaError_t launch_batch_oavg(const RepDesc *d, const int *rep, const int *first, int nblocks, int phase_phi,
                              int phase_q, double *partial, int nrep, double *out, cudaStream_t st);
cudaError_t launch_batch_oavg_final(const RepDesc *d, const int *first, const int *count, int nrep,
                                    const double *partial, double *out, cudaStream_t st);
int ideal_tile_dims(int tile, int *tx, int *ty);

// ---- persistent ensemble step ----------------------------------------------
// One cooperative launch runs every sub-step of a step over all replicas, as
// phases separated by a grid barrier: the ideal step (TMA replicas' tiles,
// then cp.async replicas' tiles), a phi parity pass or a charge face, each
// over the same block maps as the one-launch-per-sub-step path.
enum PersistKind { kPersistIdeal = 0, kPersistPhi = 1, kPersistCharge = 2 };
struct PersistPhase {
  int kind;       // PersistKind
  int arg;        // parity (phi pass) or pass 0..5 (charge face)
  int pphi, pq;   // buffers holding the current phi / charges
  int ctr_off;    // counter offset of the sub-step within the step
  double dt;      // the sub-step's dt
};
constexpr int kMaxPersistPhases = 64;
struct PersistPlan {
  int nphase;
  int nb_tma, nb_cp, nb_slab;  // blocks of the TMA ideal, cp.async ideal and slab maps
  int tile;                    // cp.async ideal tile (LGV_TILE_*)
  int wait_limit;              // polls before a device wait gives up
  unsigned long long dctr;     // counter advance of the step
  double dt_step;              // clock advance of the step
  PersistPhase ph[kMaxPersistPhases];
};
struct PersistPtrs {
  const RepDesc *d;
  EnsDyn *dyn;
  const void *gmaps;
  const int *tma_rep, *tma_first, *cp_rep, *cp_first, *slab_rep, *slab_first;
  unsigned long long *waits;  // bounded waits that gave up (barrier or TMA)
  unsigned *bar;              // grid barrier: arrivals, generation, error (zeroed)
};
// CTAs of the launch (resident at once): 0 when a cooperative launch is not possible
int persist_grid(bool i32);
cudaError_t launch_ens_persistent(const PersistPlan &plan, const PersistPtrs &q, bool i32, cudaStream_t st);

// ---------------------------------------------------------------------------
// Adjoint of the Euler-Maruyama Model A step (noise held fixed).
struct EmAdjArgs {
  double c6;      // 6 + m^2
  double dtg;     // dt * gamma
  double dt;
  double lambda;
  double H;
  double cxi;     // d sqrt(2 gamma dt) / d gamma = sqrt(2 dt) / (2 sqrt(gamma))
  double gl[4];   // uniform loss gradient dL/dphi_a added to the adjoint of this state
  uint64_t sk;    // the step's noise key (regenerates xi)
};
// lam_out = J^T lam_in + gl at state phi; per-block parameter-gradient partial
// sums (dm2, dlambda, dH, dgamma) into partial[nblocks][4]
struct IdealAdjArgs {
  double k;   // (dt / 2) / chi
  double dt;
  double a2;  // (1 / h)^2
  double H;
  double gl[4];  // added to the phi adjoint at every site
};

// Adjoint of one ideal step at state u (10 planes): lam_in (10 planes) ->
// lam_out (10 planes); adds dL/dH into g4[2].  P1, PB: 4 planes, QB: 6 planes
// of scratch; partial / done as for launch_em_avg.
cudaError_t launch_ideal_adjoint(Fields u, Fields lam_in, Fields lam_out, Fields P1, Fields PB, Fields QB, int N,
                                 const IdealAdjArgs &a, double *partial, unsigned *done, double *g4,
                                 cudaStream_t st);

// Euler-Maruyama step that also writes the volume averages of the new phi
// to avg_out[0..3]; partial holds em_reduce_blocks(N) * 4 doubles and *done
// is a zeroed counter (left zeroed).
cudaError_t launch_em_avg(Fields in, Fields out, int N, const EmArgs &a, double *partial, unsigned *done,
                          double *avg_out, cudaStream_t st);
size_t em_reduce_blocks(int N);
// adjoint of one Euler-Maruyama step; adds dL/d(m^2, lambda, H, Gamma) of the step into g4[0..3]
cudaError_t launch_em_adjoint(Fields phi, Fields lam_in, Fields lam_out, int N, const EmAdjArgs &a, double *partial,
                              unsigned *done, double *g4, cudaStream_t st);
// volume averages of phi_0..3 -> out[4]
cudaError_t launch_phi_avg(Fields f, int N, double *partial, unsigned *done, double *out, cudaStream_t st);
// phi planes of f set to the constants v[4]
cudaError_t launch_fill_phi(Fields f, int N, const double v[4], cudaStream_t st);

// Launchers (lgv_kernels.cu).  All asynchronous on `st`; return cudaError_t.
cudaError_t launch_aos_to_rb(const double *aos, Fields f, int N, cudaStream_t st);
cudaError_t launch_rb_to_aos(Fields f, double *aos, int N, cudaStream_t st);
// The same for a buffer of any geometry (a z-slab with ghost planes).
cudaError_t launch_aos_to_rb(const double *aos, Fields f, const Geo &g, cudaStream_t st);
cudaError_t launch_rb_to_aos(Fields f, double *aos, const Geo &g, cudaStream_t st);
cudaError_t launch_init_phi(Fields f, int N, uint64_t sk, double scale, cudaStream_t st);
cudaError_t launch_init_charges(Fields f, int N, uint64_t sk, double sqrtchi, double *scratch,
                                cudaStream_t st);
// one phi heat-bath parity pass, in place
cudaError_t launch_hb_pass(Fields f, int N, int parity, const HbArgs &a, cudaStream_t st);
cudaError_t launch_hb_pass(Fields f, const Geo &g, int parity, const HbArgs &a, cudaStream_t st);
// Ordered phi sweeps (hb_ordered_kernel): one persistent launch runs 1 ..
// kHbMaxSweeps whole sweeps in place, z-slab by z-slab.  A plan holds the
// chunk schedule for each sweep count and the launch's counters; it is built
// once per lattice size (device allocations) and used by one stream at a time.
constexpr int kHbMaxSweeps = 4;
struct HbPlan {
  int N = 0, S = 0, nslab = 0, spc = 0, cpi = 0, grid = 0;
  int *sched[kHbMaxSweeps] = {};
  int total[kHbMaxSweeps] = {};
  unsigned long long *sync = nullptr;
  int wait_limit = kWaitLimit;  // polls before a dependency wait gives up
};
// slab_target: planes per slab at most; spc: sites per chunk (multiple of
// 128); lag: schedule rounds between an item and its dependants
cudaError_t hb_plan_build(HbPlan &plan, int N, int slab_target, int spc, int lag);
void hb_plan_free(HbPlan &plan);
// nsweeps sweeps with counter keys sk[0..nsweeps) (null: a.sk, one sweep);
// injected noise and per-site flags allow one sweep per launch
cudaError_t launch_hb_ordered(Fields f, int N, const HbArgs &a, const HbPlan &plan, int nsweeps, const uint64_t *sk,
                              cudaStream_t st);
// bounded waits of the plan's launches that gave up (synchronises `st`)
cudaError_t hb_plan_timeouts(const HbPlan &plan, cudaStream_t st, unsigned long long *out, bool clear);
// one full phi heat-bath sweep (both parities, z-marching): reads phi of `in`, writes phi of `out`
cudaError_t launch_hb_sweep(Fields in, Fields out, int N, const HbArgs &a, cudaStream_t st);
cudaError_t launch_charge_pass(Fields f, int N, int dir, int eoA, const ChargeArgs &a, cudaStream_t st);
cudaError_t launch_charge_pass(Fields f, const Geo &g, int dir, int eoA, const ChargeArgs &a, cudaStream_t st);
// Both faces of direction dir.  x runs in place on `in`; y and z read `in`
// and write the charges of `out` (*swapped = true: the caller swaps the
// charge planes).
// shared-memory slab kernel for both faces of a direction (N divisible by 32)
bool charge_slab_supported(int N);
cudaError_t launch_charge_dir(Fields in, Fields out, int N, int dir, const ChargeDirPair &p, cudaStream_t st,
                              bool *swapped);
cudaError_t launch_em(Fields in, Fields out, int N, const EmArgs &a, cudaStream_t st);
cudaError_t launch_ideal(Fields in, Fields out, int N, const IdealArgs &a, cudaStream_t st);
cudaError_t launch_em(Fields in, Fields out, const Geo &g, const EmArgs &a, cudaStream_t st);
cudaError_t launch_ideal(Fields in, Fields out, const Geo &g, const IdealArgs &a, cudaStream_t st);
// TMA-staged ideal step (lgv_ideal_tma.cu): N divisible by 32
bool ideal_tma_supported(int N);
cudaError_t launch_ideal_tma(Fields in, Fields out, const Geo &g, int zchunk, const IdealArgs &a, cudaStream_t st);
// Ensembles: the TMA ideal step for replicas with N divisible by 32.
// tma_plane_map encodes the 128-byte tensor map of one component plane; gmaps
// holds, per replica r, buffer phases (pphi, pq) and component c, the map at
// ((r * 2 + pphi) * 2 + pq) * 10 + c; a replica takes batch_tma_blocks(N, izc) blocks.
bool tma_plane_map(const double *plane, int N, void *out128);
int batch_tma_blocks(int N, int zchunk);
cudaError_t launch_batch_ideal_tma(const RepDesc *d, const void *gmaps, const int *rep, const int *first, int nblocks,
                                   int phase_phi, int phase_q, double dt, unsigned long long *waits, int wait_limit,
                                   cudaStream_t st);
// energy: writes E into dev_out[0]; scratch >= energy_scratch_doubles(N)
size_t energy_scratch_doubles(int N);
cudaError_t launch_energy(Fields f, int N, double H, double inv2chi_half, double *scratch, double *dev_out,
                          cudaStream_t st);
// measurement: dev_out receives measure_size(N) doubles (lgv.h packing);
// scratch >= measure_scratch_doubles(N)
size_t measure_size(int N);
size_t measure_scratch_doubles(int N);
cudaError_t launch_measure(Fields f, int N, double *scratch, double *dev_out, cudaStream_t st);
// Pieces of the measurement for a lattice in host-order AoS layout (device
// memory): the observable sums into T[25][N][N] and U[25][N][N], then walls,
// OAverage, DFT and vev rotation into dev_out (lgv.h packing).
cudaError_t launch_measure_sums_aos(const double *aos, int N, double *T, double *U, cudaStream_t st);
cudaError_t launch_measure_finish(const double *T, const double *U, int N, double *dev_out, cudaStream_t st);
// A slab's share of those sums: T rows of its planes (local planes klo ..
// klo+nk-1 = global rows kout .. kout+nk-1 of T[25][Ng][N], other rows left as
// they are) and U summed over those planes only.
cudaError_t launch_measure_partials(Fields f, const Geo &g, int klo, int nk, int kout, double *T, double *U,
                                    cudaStream_t st);

}  // namespace lgv

/*
 * lgv.h -- C ABI of the B200 (sm_100a) Model A / Model G stepper and measurer.
 *
 * This is the drop-in boundary for the time stepper of langevinA
 * (derek-teaney/langevinA, directory ModelG/).  Every entry point below names the
 * reference interface it replaces.  Signatures use plain C types only: no CUDA,
 * PETSc or torch types cross this boundary, so the library can be bound from C,
 * C++ (see langevina.hpp), Python ctypes or any other FFI.
 *
 * Conventions
 *  - Every function returns an int status: LGV_OK (0) or a negative LGV_ERR_*.
 *    lgv_status_string() turns it into text; lgv_last_error() gives the detail
 *    of the last failure on the calling thread.
 *  - A handle owns one periodic N^3 lattice on the current CUDA device.  It is
 *    not thread safe: use one handle per host thread.
 *  - Host state arrays use the reference's site layout (G_node / data_node,
 *    ModelA.h:274-286) in DMDA natural ordering u[k][j][i][L], L = 0..9 =
 *    (phi_0..phi_3, A_1..A_3, V_1..V_3), FP64, 80 bytes per site.
 *  - All arithmetic is FP64.
 */
#ifndef LGV_H
#define LGV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LGV_NPHI 4
#define LGV_NA 3
#define LGV_NV 3
#define LGV_NDOF 10
#define LGV_NOBS 11       /* Measurer::NObs, measurer.h:91-92 */
#define LGV_NOBS_PHASE 14 /* Measurer::NObsPhase = NObsRotated, measurer.h:111,119 */

/* Status codes. */
#define LGV_OK 0
#define LGV_ERR_INVALID (-1)     /* bad argument (size, pointer, enum) */
#define LGV_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define LGV_ERR_NOMEM (-3)       /* device or host allocation failed */
#define LGV_ERR_TIMEOUT (-4)     /* a bounded device wait gave up */
#define LGV_ERR_STATE (-5)       /* call not valid now (e.g. injected noise not supplied) */
#define LGV_ERR_UNSUPPORTED (-6) /* valid request this build does not implement */

/* Model parameters.  Replaces ModelAData / ModelACoefficients (ModelA.h:71-111,
 * 185-248); the JSON keys of the same names are read by langevina.hpp. */
typedef struct lgv_params {
  int32_t N;         /* NX = NY = NZ; even and >= 4 (checkerboard) */
  int32_t reserved0; /* must be 0 */
  double LX;         /* box length, lattice spacing hX = LX / N (ModelA.h:199) */
  double mass0;      /* m^2(t) = mass0 + dmassdt * t (ModelA.h:84) */
  double dmassdt;
  double lambda;
  double H;
  double chi;
  double gamma;
  double diffusion; /* sigma = diffusion * chi (ModelA.h:86) */
  uint64_t seed;    /* base seed of the counter-based noise */
} lgv_params;

/* Steppers.  PV2HBSplit is the composer of Stepper.cxx:537-580; with
 * (inner, outer) = (2, 3) it is the reference's "PV2HBSplit23". */
#define LGV_PV2HBSPLIT 0             /* (A B^inner)^outer C */
#define LGV_PV2HBSPLIT_NODIFFUSE 1   /* (A B^inner)^outer       */
#define LGV_PV2HBSPLIT_ONLYDIFFUSE 2 /*                      C  */
#define LGV_IDEAL_PV2 3              /* A : IdealPV2 (no accept/reject) */
#define LGV_EULER_LANGEVIN_HB 4      /* B : phi checkerboard heat bath */
#define LGV_CHARGE_HB 5              /* C : link charge heat bath */
#define LGV_MODELA_EM 6              /* Euler-Maruyama Model A relaxation */
#define LGV_IDEAL_EM 7               /* ideal step then Euler-Maruyama relaxation (no counterpart) */

/* Noise sources. */
#define LGV_NOISE_COUNTER 0  /* counter-indexed xoroshiro128+ streams (production) */
#define LGV_NOISE_INJECTED 1 /* caller-supplied uniforms / normals (parity tests) */

/* lgv_initialize() kinds. */
#define LGV_INIT_ZERO 0             /* ModelA::initialize() without a function */
#define LGV_INIT_PHI_GAUSSIAN 1     /* phi_a ~ scale * N(0,1), charges untouched */
#define LGV_INIT_CHARGES_GAUSSIAN 2 /* n ~ sqrt(chi) N(0,1), zero mode removed */

/* Monitors (o4_stepper_monitor, Stepper.h:17-49). */
#define LGV_MONITOR_IDEAL 0
#define LGV_MONITOR_PHI_HB 1
#define LGV_MONITOR_CHARGE_HB 2

typedef struct lgv_monitor {
  int64_t down_counts; /* dS < 0 */
  int64_t up_counts;   /* dS >= 0 */
  int64_t up_yes;      /* accepted with dS >= 0 */
  int64_t up_no;       /* rejected */
  double down_dS;      /* sum of dS over dS < 0 */
  double up_dS;        /* sum of dS over accepted dS >= 0 */
} lgv_monitor;

/* Measurement output, caller-owned.  Any pointer may be NULL to skip that
 * output.  Layouts follow Measurer (measurer.h:88-128) row-major:
 *   OAverage            [11]
 *   wall[a]             [11][N]            a = 0,1,2 for X,Y,Z
 *   wall_k[a]           [11][N/2+1][2]     (re, im)
 *   wall_k_rotated[a]   [14][N/2+1][2]
 *   wall_phase[a]       [14][N]
 *   wall_phase_k[a]     [14][N/2+1][2]                                      */
typedef struct lgv_measurement {
  double *OAverage;
  double *wall[3];
  double *wall_k[3];
  double *wall_k_rotated[3];
  double *wall_phase[3];
  double *wall_phase_k[3];
} lgv_measurement;

typedef struct lgv_handle lgv_handle;

/* Library identification. */
int lgv_version(void);
const char *lgv_status_string(int status);
const char *lgv_last_error(void);

/* Replaces: ModelA::ModelA (ModelA.h:311-336) -- DMDACreate3d + Vec + seeding.
 * Allocates the device lattice on the current CUDA device. */
int lgv_create(const lgv_params *params, lgv_handle **out);
/* Replaces: ModelA::finalize / Stepper::finalize resource release
 * (ModelA.h:338-352, Stepper.cxx:270-279,390-398,524-533). */
int lgv_destroy(lgv_handle *h);
/* Update coefficients (mass0, lambda, H, chi, gamma, diffusion, dmassdt, LX,
 * seed) without reallocating; N must match. */
int lgv_set_params(lgv_handle *h, const lgv_params *params);

/* Replaces: VecLoad / direct writes into model->solution (ModelA.h:356-380,
 * 443-458).  host_aos holds N^3 * 10 doubles in u[k][j][i][L] order. */
int lgv_set_state(lgv_handle *h, const double *host_aos);
/* Replaces: reads of model->solution (DMDAVecGetArray, VecView ModelA.h:384-402). */
int lgv_get_state(lgv_handle *h, double *host_aos);
/* Same two calls with a device pointer to an AoS array on the handle's device. */
int lgv_set_state_device(lgv_handle *h, const double *dev_aos);
int lgv_get_state_device(lgv_handle *h, double *dev_aos);

/* Replaces: ModelA::initialize (ModelA.h:408-461, zero start) and
 * ModelA::initialize_gaussian_charges (ModelA.h:463-525).  Noise comes from
 * the counter streams (one counter value per call). */
int lgv_initialize(lgv_handle *h, int kind, double scale);

/* Noise control.  Replaces the global ModelARndm (NoiseGenerator.h:62-160) for
 * the device-side draws.  The counter is the 64-bit sub-step index of the
 * counter streams; saving (seed, counter) replaces the <tag>_<rank>.rng file
 * (NoiseGenerator.h:112-146). */
int lgv_set_noise_mode(lgv_handle *h, int mode);
/* Proposal of the phi heat bath with counter noise: LGV_HB_PROPOSAL_UNIFORM
 * (the default: U(-sqrt3, sqrt3) per component, as EulerLangevinHB::step,
 * Stepper.cxx:343) or LGV_HB_PROPOSAL_GAUSSIAN (four normals per site, two
 * Box-Muller pairs from the site's first four draws; variance one as well, so
 * the same proposal scale and detailed balance).  Injected proposals are used
 * as given either way.  Gaussian proposals run on the one-parity pass kernel:
 * LGV_ERR_UNSUPPORTED when LGV_HB_FUSED or LGV_HB_ORDERED was set at
 * creation; ensembles propose uniformly. */
#define LGV_HB_PROPOSAL_UNIFORM 0
#define LGV_HB_PROPOSAL_GAUSSIAN 1
int lgv_set_hb_proposal(lgv_handle *h, int kind);
int lgv_set_counter(lgv_handle *h, uint64_t counter);
int lgv_get_counter(lgv_handle *h, uint64_t *counter);
/* Injected noise for the next sub-step of each kind (host pointers, copied).
 *  hb:     prop[4][V] proposals in (-sqrt3, sqrt3) (variance1()), acc[V] in [0,1)
 *          indexed by natural site index n = (k*N + j)*N + i.
 *  charge: order[5] = (orderxyz[3], ordereo[2]) as after std::shuffle
 *          (Stepper.cxx:461-466); q[6][6][V], acc[6][6][V] indexed by
 *          (pass, L-4, natural index of the A site).
 *  em:     xi[4][V] standard normals. */
int lgv_inject_hb(lgv_handle *h, const double *prop, const double *acc);
int lgv_inject_charge(lgv_handle *h, const int32_t *order, const double *q, const double *acc);
int lgv_inject_em(lgv_handle *h, const double *xi);

/* Replaces: Stepper::step(dt) (Stepper.h:6-11) for every stepper of
 * Stepper.cxx (IdealPV2::step :23-66, EulerLangevinHB::step :287-389,
 * ModelGChargeHB::step :449-522, PV2HBSplit::step :542-580) plus the
 * Euler-Maruyama Model A step.  Runs nsteps steps of size dt starting at time
 * t (t advances by dt per step; it sets m^2(t)).  inner/outer are the
 * PV2HBSplit scounts {inner, outer} (ignored by the other evolvers).
 * Asynchronous on the handle's stream. */
int lgv_step(lgv_handle *h, int evolver, int inner, int outer, double dt, double t, int nsteps);

/* Replaces: Measurer::measure(Vec*) (measurer.h:169-179, measurer.cxx:10-317):
 * wall sums, phase walls, OAverage, x->k modes (FFTW r2c / N) and rotate_to_vev.
 * Synchronous: the outputs are filled when it returns. */
int lgv_measure(lgv_handle *h, lgv_measurement *out);
/* Same measurement, left in device memory: dev_out receives
 * lgv_measure_size(N) doubles packed in the order of lgv_measurement's fields
 * (OAverage, wall[0..2], wall_k[0..2], wall_k_rotated[0..2], wall_phase[0..2],
 * wall_phase_k[0..2]).  Asynchronous. */
int lgv_measure_device(lgv_handle *h, double *dev_out);
size_t lgv_measure_size(int N);

/* Replaces: IdealPV2::computeEnergy (Stepper.cxx:204-268).  Synchronous. */
int lgv_energy(lgv_handle *h, double *energy);

/* Replaces: o4_stepper_monitor counters (Stepper.h:17-83).  Counting is off
 * by default (it costs one block reduction per launch); lgv_enable_monitors
 * turns it on and zeroes the counters. */
int lgv_enable_monitors(lgv_handle *h, int enable);
int lgv_get_monitor(lgv_handle *h, int which, lgv_monitor *out);

/* Stream control: all work of the handle is issued on this cudaStream_t
 * (NULL = the legacy default stream).  A new handle uses a non-blocking stream
 * of its own.  Work already queued on the previous stream is ordered before
 * any work issued on the new one. */
int lgv_set_stream(lgv_handle *h, void *cuda_stream);
int lgv_synchronize(lgv_handle *h);

/* Live kernel timing.  When enabled, every kernel launch of the classes below
 * is bracketed by a CUDA event pair on the handle's stream; lgv_timing_read
 * synchronizes, adds the elapsed times of all pairs recorded so far and
 * returns the running total and launch count of one class.  Enabling (or
 * re-enabling) resets the totals.  A "launch" of LGV_KCLASS_PHI_HB is one
 * checkerboard parity pass; of LGV_KCLASS_CHARGE one (direction, parity) face;
 * of LGV_KCLASS_MEASURE one full measurement (five small kernels). */
#define LGV_KCLASS_IDEAL 0
#define LGV_KCLASS_PHI_HB 1
#define LGV_KCLASS_CHARGE 2
#define LGV_KCLASS_EM 3
#define LGV_KCLASS_MEASURE 4
#define LGV_NKCLASS 5
int lgv_timing_enable(lgv_handle *h, int enable);
int lgv_timing_read(lgv_handle *h, int kclass, double *total_ms, int64_t *launches);

/* Parity-test aid: when enabled, the next noisy sub-steps record per-decision
 * flags (0 rejected, 1 accepted with dS < 0, 2 accepted with dS >= 0).
 * Phi heat bath: flags[n] for site n.  Charge heat bath: flags[(p*6+L-4)*V+nA].
 * lgv_get_flags copies 36*V bytes. */
int lgv_debug_flags(lgv_handle *h, int enable);
int lgv_get_flags(lgv_handle *h, uint8_t *host_out);

/* ---------------------------------------------------------------------------
 * Differentiable runs.  No counterpart in the reference (it has no gradients
 * and no Euler-Maruyama stepper); built on the same steps as lgv_step with
 * evolver LGV_MODELA_EM (Euler-Maruyama Model A), LGV_IDEAL_PV2 (the ideal
 * O(4) rotation step) or LGV_IDEAL_EM (both in sequence).  The Metropolis
 * heat baths have no adjoint.
 *
 * lgv_diff_forward runs S = nsteps steps of size dt from time t, the
 * Euler-Maruyama noise fixed by seed and counter, keeps a copy of the state
 * every ckpt_every steps and returns two time averages over the steps
 * n = b+1 .. S (b = avg_begin, M = S - b):
 *   obs[0] = 1/M sum_n sigma(n)                          sigma = <phi_0>
 *   obs[1] = 1/M sum_n V sum_{a=1..3} pibar_a(n)^2      pibar_a = <phi_a>
 * (<.> the volume average, obs[1] the zero-momentum pi equal-time correlator).
 * The lattice is left at the final state and the counter advanced by S when
 * the run has Euler-Maruyama steps (counter noise mode only).
 * lgv_diff_backward returns in grad[4] the derivative of w[0]*obs[0] +
 * w[1]*obs[1] with respect to (mass0, lambda, H, gamma), the noise held
 * fixed, by the hand-written adjoint kernels of the steps; each checkpoint
 * segment is recomputed with the forward's noise.  It may be called any
 * number of times after one forward.
 * lgv_diff_averages copies the volume averages <phi_a>(n), n = 0..nsteps,
 * a = 0..3, of the last forward into out ((nsteps+1)*4 doubles; nsteps must
 * be the forward's). */
int lgv_diff_forward(lgv_handle *h, int evolver, double dt, double t, int nsteps, int avg_begin, int ckpt_every,
                     double *obs);
int lgv_diff_backward(lgv_handle *h, const double *w, double *grad);
int lgv_diff_averages(lgv_handle *h, double *out, int nsteps);

/* ---------------------------------------------------------------------------
 * Batched ensembles.  Replaces running an ensemble as separate processes or
 * events, one lattice at a time (eventmode loop SuperPions.cxx:228-235, SLURM
 * job arrays grunner.py:153-241): nrep independent replicas, each with its own
 * lgv_params (any mix of N, seed and coefficients), advance together -- one
 * launch per sub-step over all replicas, two steps per replayed CUDA graph.
 * Replica r evolves exactly as an lgv handle created with params[r] and
 * stepped with the same counter.  The packing order is the order in which
 * replicas' blocks fill the grid. */
typedef struct lgv_ensemble lgv_ensemble;
#define LGV_PACK_GIVEN 0
#define LGV_PACK_LARGEST_FIRST 1
#define LGV_PACK_INTERLEAVED 2
/* ideal-kernel tile shapes */
#define LGV_TILE_32x8 0
#define LGV_TILE_16x16 1
int lgv_ensemble_create(int nrep, const lgv_params *params, lgv_ensemble **out);
int lgv_ensemble_destroy(lgv_ensemble *e);
int lgv_ensemble_size(lgv_ensemble *e, int *nrep);
int lgv_ensemble_set_state(lgv_ensemble *e, int replica, const double *host_aos);
int lgv_ensemble_get_state(lgv_ensemble *e, int replica, double *host_aos);
/* as lgv_initialize, for every replica (one counter value for the ensemble) */
int lgv_ensemble_initialize(lgv_ensemble *e, int kind, double scale);
int lgv_ensemble_set_counter(lgv_ensemble *e, uint64_t counter);
int lgv_ensemble_get_counter(lgv_ensemble *e, uint64_t *counter);
/* as lgv_step, for every replica; asynchronous */
int lgv_ensemble_step(lgv_ensemble *e, int evolver, int inner, int outer, double dt, double t, int nsteps);
/* volume averages of the 11 OAverage observables, [nrep][11] */
int lgv_ensemble_oaverage(lgv_ensemble *e, double *host_out);
int lgv_ensemble_oaverage_device(lgv_ensemble *e, double *dev_out);
/* explicit tuning: ideal tile (LGV_TILE_*), its z-chunk, packing (LGV_PACK_*) */
int lgv_ensemble_tune(lgv_ensemble *e, int tile, int zchunk, int order);
/* time every (tile, z-chunk in {8,16,32}, packing) candidate over `steps`
 * steps on a copy of the state (state and counter restored), keep the
 * fastest; choice[3] = (tile, zchunk, order), *ms_per_step its time */
int lgv_ensemble_autotune(lgv_ensemble *e, int evolver, int inner, int outer, double dt, int steps, int *choice,
                          double *ms_per_step);
/* CUDA-graph replay of lgv_ensemble_step (on by default): two steps are
 * captured once per (evolver, inner, outer, dt, buffer phases) on the
 * ensemble's own stream and replayed on its current stream, which may be any
 * stream the caller set, the legacy default stream included. */
int lgv_ensemble_use_graphs(lgv_ensemble *e, int enable);
/* One persistent launch per step (off by default; LGV_ENS_PERSISTENT=1 in the
 * environment at lgv_ensemble_create turns it on): a cooperative launch of
 * two 256-thread CTAs per SM runs every sub-step of the step over all
 * replicas, the sub-steps separated by a grid barrier whose waits are bounded
 * (a wait that gives up is reported as LGV_ERR_TIMEOUT by the next
 * synchronising call), and is captured in the CUDA graphs as any other launch.
 * Same results as the default one launch per sub-step, bit for bit.  The
 * Euler-Maruyama evolver keeps its own launch.  LGV_ERR_UNSUPPORTED when the
 * device has no cooperative launch. */
int lgv_ensemble_use_persistent(lgv_ensemble *e, int enable);
/* Differentiable Euler-Maruyama Model A runs of all replicas at once (no
 * counterpart in the reference): one launch per step over all replicas.
 * Replica r gets what lgv_diff_forward / lgv_diff_backward with evolver
 * LGV_MODELA_EM return for a single lattice with params[r] and the
 * ensemble's counter: obs holds [R][2], w [R][2] and grad [R][4]. */
int lgv_ensemble_diff_forward(lgv_ensemble *e, double dt, double t, int nsteps, int avg_begin, int ckpt_every,
                              double *obs);
int lgv_ensemble_diff_backward(lgv_ensemble *e, const double *w, double *grad);
int lgv_ensemble_set_stream(lgv_ensemble *e, void *cuda_stream);
int lgv_ensemble_synchronize(lgv_ensemble *e);

/* Allocation-free measurement.  No counterpart in the reference: it is the
 * measurement of lgv_measure_device() for callers that cannot allocate device
 * memory while they run -- a host whose GPU memory belongs to another
 * allocator (a framework's caching pool that has reserved most of the device,
 * where an extra cudaMalloc can fail even though the pool has room) or a
 * process held to a fixed device-memory budget.  The caller passes the lattice
 * (dev_aos: N^3 * 10 doubles in device memory, the host-order AoS layout of
 * lgv_set_state) and the output (dev_out: lgv_measure_size(N) doubles in device
 * memory, packed as for lgv_measure_device) and needs no handle.  Scratch space
 * is a static device array inside the library sized for N <= 128 (6.55 MB,
 * held on every GPU that loads the library until exit); larger N is rejected
 * with LGV_ERR_INVALID.  The array is shared by all calls on a device, so calls
 * whose kernels overlap on the GPU race with each other.  A call made outside
 * stream capture looks the array's address up (cudaGetSymbolAddress) in the
 * current device's context; a call made while `stream` is being captured uses
 * the address its device's last uncaptured call found, and fails with
 * LGV_ERR_STATE if there was none -- so make the first call on each device
 * before any stream capture.  Asynchronous on `stream` (NULL = legacy default
 * stream); calls no allocator. */
#define LGV_NOALLOC_MAX_N 128
int lgv_measure_aos_noalloc(const double *dev_aos, int N, double *dev_out, void *stream);

/* ---- Lattices split into z-slabs over ranks, for lattices larger than one
 * GPU (no single counterpart: it replaces the z-decomposition of DMDACreate3d,
 * ModelA.h:315-318, with its ghost exchanges DMGlobalToLocal before every
 * pass, Stepper.cxx:81-82, 312-315, 477-480).
 *
 * lgv_slab_create makes a handle for global planes k0 .. k0+nz-1 of the N^3
 * lattice of `params` (k0 and nz even, nz >= 2), held with two ghost planes on
 * each side: its buffers are N x N x (nz + 4) sites, local plane 0 being global
 * plane k0 - 2 (mod N).  lgv_step then advances the slab exactly as a whole
 * lattice would advance those planes -- the same counter streams, indexed by
 * the global site -- provided that before every sub-pass that reads across
 * planes (each ideal step, each phi parity pass, each z-face of the charge
 * heat bath, each Euler-Maruyama step) the ghost planes hold the neighbours'
 * current values.  lgv_step calls the halo function set by lgv_slab_set_halo
 * at those points, from the calling thread, with the component groups to
 * refresh (LGV_HALO_PHI, LGV_HALO_CHARGES or both); it returns 0 on success.
 * The function packs this slab's two lowest and two highest planes
 * (lgv_slab_pack, side 0 / 1), sends them to the rank below / above (global
 * planes wrap), and unpacks what it receives from the rank below into side 0
 * and from the rank above into side 1 (lgv_slab_unpack).  Pack and unpack are
 * asynchronous on the handle's stream; the halo function synchronises it
 * before handing buffers to another stream or process.  A buffer holds
 * lgv_slab_halo_doubles(h, comps) doubles.
 *
 * lgv_set_state / lgv_get_state (and the _device forms) move the whole
 * buffer, ghosts included: N x N x (nz + 4) x 10 doubles, u[k][j][i][L] with k
 * the local plane.  Counter noise only; initialisation, injected noise,
 * per-site flags, accept statistics, energies and the differentiable runs are
 * refused (LGV_ERR_UNSUPPORTED).
 *
 * Measurement: lgv_slab_measure_partials writes this slab's rows of
 * T[25][N][N] (T[o][k][i] = sum_j obs, rows k0 .. k0+nz-1; other rows are not
 * touched) and U[25][N][N] (U[o][j][i] = sum over this slab's planes of obs),
 * device memory, asynchronous.  Summing every rank's T (zero elsewhere) and U
 * and calling lgv_measure_from_partials gives lgv_measure_device's output for
 * the whole lattice. */
#define LGV_HALO_PHI 1
#define LGV_HALO_CHARGES 2
#define LGV_HALO_ALL 3
typedef int (*lgv_halo_fn)(void *ctx, lgv_handle *h, int comps);
int lgv_slab_create(const lgv_params *params, int k0, int nz, lgv_handle **out);
int lgv_slab_set_halo(lgv_handle *h, lgv_halo_fn fn, void *ctx);
size_t lgv_slab_halo_doubles(lgv_handle *h, int comps);
int lgv_slab_pack(lgv_handle *h, int side, int comps, double *dev_buf);
int lgv_slab_unpack(lgv_handle *h, int side, int comps, const double *dev_buf);
int lgv_slab_measure_partials(lgv_handle *h, double *dev_T, double *dev_U);
int lgv_measure_from_partials(const double *dev_T, const double *dev_U, int N, double *dev_out, void *stream);

/* Post-processing of measurement histories held in device memory.  Stateless,
 * asynchronous on `stream` (NULL = legacy default stream), no allocation,
 * deterministic (every sum in a fixed order).
 *
 * lgv_x2k replaces the x2k.exe transform (ModelG/x2k.cxx:94-113): for every row
 * of walls ([rows][N], N even, <= 8192), out[row][k] = (1/N) sum_x walls[row][x]
 * e^{-2 pi i k x / N} for k = 0..N/2, stored as (re, im) pairs: out is
 * [rows][N/2+1][2].  On a wall of lgv_measure it reproduces the measurer's k
 * wall bit for bit. */
int lgv_x2k(const double *walls, int64_t rows, int N, double *out, void *stream);
/* lgv_x2k_rotated replaces x2k_rotated.exe (ModelG/x2k_rotated.cxx:92-143):
 * walls_k is [rows][nfields >= 10][NK][2] (fields phi_0..3, A_1..3, V_1..3, ...
 * as lgv_x2k writes them); per row the direction n is the real part of the four
 * phi modes at k = 0, normalised ((1,0,0,0) below DBL_MIN), and out is
 * [rows][13][NK][2]: phi along n, phi minus that (4), contract_rho(n, rho) (4),
 * contract_rho(n, dual rho) (4). */
int lgv_x2k_rotated(const double *walls_k, int64_t rows, int nfields, int NK, double *out, void *stream);
/* lgv_time_correlator replaces computeOtOtp with its default mean statistic
 * (python/Loader.py:229-254) for many series at once.  a and b are time-major:
 * element t of series s is a[t*ld + s] (real) or the pair a[t*ld + 2s], +1
 * (is_complex); T samples, nseries series, ld >= nseries (x2 if complex).  For
 * tau = 0..ntmax-1: out[tau][s] = mean over t = 0, decim, 2 decim, ... < T - tau
 * of a_s(t) * b_s(t + tau) (complex product, no conjugation), minus
 * mean(a_s) * mean(b_s) over all T samples when conn != 0.  out is
 * [ntmax][nseries] (x2 if complex).  1 <= ntmax <= T (the reference's slices
 * past T - 1 are empty or wrap; they are rejected here). */
int lgv_time_correlator(const double *a, const double *b, int64_t T, int64_t nseries, int64_t ld, int is_complex,
                        int ntmax, int decim, int conn, double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LGV_H */

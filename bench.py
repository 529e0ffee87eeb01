#!/usr/bin/env python
"""Model G stepper throughput on B200: site-updates/s and % of the HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--N 256]

Workload: the full Model G step "PV2HBSplit23" (3 x [ideal PV2(dt/3) + 2 x phi
heat bath(dt/6)] + charge heat bath(dt), Stepper.cxx:542-580) on a 256^3
periodic FP64 lattice with the heat-bath coefficients at H = 0.003 (m^2 = -4.813,
lambda = 10, Gamma = 1, chi = 5, D = 1/3, dt = 0.04), measuring every 10 steps
(saveFrequency, SuperPions.cxx:127-140).  Seeded synthetic state: phi ~
0.1 N(0,1), charges ~ sqrt(chi) N(0,1) with the zero mode removed.  The state
(1.34 GB) is larger than L2, so no flush is needed between steps.

One process per GPU; for N > 1 each rank advances its own replica (distinct
seed): the stepper does not shard, so scaling is weak, with no data-path
collective.  Rank 0 prints one JSON line.

--impl reference times the reference's own implementation on the host cores:
Stepper.cxx, NoiseGenerator.cxx and measurer.cxx compiled unmodified against
single-node PETSc/MPI/FFTW stand-ins (oracle/_ref/ref_stepper, built with the
oracle), one process per MPI rank, on the same 256^3 workload (K timed steps
after W warm-up, measuring every 10).  Without that build it falls back to the
oracle's restatement on a 128^3 sample.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

ALG_BYTES = {  # algorithmic bytes per site, per launch (each input read once, each output written once)
    "ideal": 160.0,    # 10 doubles in, 10 out
    "phi_hb": 32.0,    # one parity pass: 64 B/site per full sweep, half the sites per launch
    "charge": 96.0,    # one (direction, parity) face: 6 charges in and out for every site
    "em": 64.0,
}
STEP_BYTES = {"PV2HBSplit23": 1440.0, "PV2HBSplit11": 800.0}
NOMINAL_HBM_GBS = 7700.0  # B200 HBM3e, HGX figure
KCLASS = {"ideal": 0, "phi_hb": 1, "charge": 2, "em": 3, "measure": 4}
COEF = dict(mass0=-4.813, lam=10.0, H=0.003, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0)
DT = 0.04
MEASURE_EVERY = 10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--scounts", default="2,3")
    ap.add_argument("--seed", type=int, default=122335456)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-postprocess", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the 64^3 Model G run and the z-slab emulation")
    return ap.parse_args()


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_table():
    p = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}", "--format=csv,noheader",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                mhz.append(float(r[1].split()[0]))
                mx = float(r[2].split()[0])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if "Active" in v and "Not" not in v:
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(mhz)}


def reference_build_run(N, scounts, warmup, steps, ranks, seed=122335456):
    """The reference's own stepper and measurer (oracle/_ref/ref_stepper: Stepper.cxx,
    NoiseGenerator.cxx, measurer.cxx compiled unmodified against single-node
    PETSc/MPI/FFTW stand-ins), one process per MPI rank (z-slabs), the
    workload of run_ours: phi ~ 0.1 N(0,1) and Gaussian charges from the
    reference's own stream, `warmup` untimed steps, then `steps` timed steps
    with Measurer::measure every MEASURE_EVERY steps, as run_event does
    (SuperPions.cxx:127-158).  Returns (site-updates/s, ms per step, seconds)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import refbuild

    name = "PV2HBSplit%d%d" % scounts
    P = refbuild.params_json(N, mass0=COEF["mass0"], lam=COEF["lam"], H=COEF["H"], chi=COEF["chi"],
                             gamma=COEF["gamma"], diffusion=COEF["diffusion"], seed=seed, dt=DT)
    ops = ["phi=0.1", "charges"]
    if warmup:
        ops.append(f"step={name},{warmup}")
    timed = []
    s = 0
    while s < steps:
        n = min(MEASURE_EVERY, steps - s)
        timed += ["measure", f"step={name},{n}"]
        s += n
    res = refbuild.run(P, ops + timed, ranks=ranks, timeout=3600)
    el = sum(t for _, t in res.times[len(ops):])
    return N ** 3 * steps / el, el / steps * 1e3, el


def reference_available():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import refbuild

    return refbuild.available()


def cpu_port_rate(N, scounts, steps, warmup=1):
    """Fallback when the reference build is absent: the oracle's restatement
    with the reference's serial RNG, one thread per emulated MPI rank."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle

    cores = os.cpu_count() or 1
    R = max(1, min(cores, N))
    o = oracle.Oracle(N, mode=oracle.SEQUENTIAL, nranks=R, seed=122335456, **COEF)
    o.initialize(1, 0.1)
    o.initialize(2)
    for _ in range(warmup):
        o.step(0, DT, inner=scounts[0], outer=scounts[1])
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(0, DT, inner=scounts[0], outer=scounts[1])
    el = time.perf_counter() - t0
    return N ** 3 * steps / el, el / steps * 1e3, el, R


def cpu_baseline_sample(N, scounts):
    """cpu_baseline of the GPU arm: a bounded sample (2 timed steps after 1
    warm-up) of the same workload on all host cores."""
    name = "PV2HBSplit%d%d" % scounts
    cores = os.cpu_count() or 1
    if reference_available():
        R = max(1, min(cores, N // 2))
        rate, ms, el = reference_build_run(N, scounts, 1, 2, R)
        return {"value": rate, "unit": "site-updates/s", "cores": R, "kind": "reference",
                "sample": f"2 timed {name} steps (after 1 warm-up, measurement every {MEASURE_EVERY}) of the {N}^3 "
                          f"lattice, {el:.1f} s: the reference's Stepper.cxx/measurer.cxx built against single-node "
                          f"PETSc/MPI stand-ins, {R} MPI ranks (processes, z-slabs)"}
    Ns = min(N, 128)
    rate, ms, el, R = cpu_port_rate(Ns, scounts, 2)
    return {"value": rate, "unit": "site-updates/s", "cores": R, "kind": "port",
            "sample": f"2 {name} steps of a {Ns}^3 sample lattice ({el:.1f} s), oracle port with the reference "
                      f"serial RNG, one thread per emulated MPI rank"}


def run_reference(a):
    _, rank, _ = rank_env()
    if rank != 0:
        return 0
    scounts = tuple(int(x) for x in a.scounts.split(","))
    name = "PV2HBSplit%d%d" % scounts
    cores = os.cpu_count() or 1
    config = {"workload": f"Model G {name}, {a.N}^3 periodic lattice, FP64, measure every {MEASURE_EVERY} steps",
              "N": a.N, "evolver": name, "dt": DT, **COEF}
    if reference_available():
        R = max(1, min(cores, a.N // 2))
        # a reference step of the 256^3 lattice takes ~3 s on 16 cores: at most
        # REF_MAX_STEPS timed steps (and 3 warm-up) keep the run within minutes
        nst, nw = min(a.steps, REF_MAX_STEPS), min(a.warmup, 3)
        rate, ms, el = reference_build_run(a.N, scounts, nw, nst, R)
        cpu = {"kind": "reference", "cores": R,
               "sample": f"the whole workload, {nst} timed steps after {nw} warm-up on the {a.N}^3 lattice "
                         f"({el:.1f} s; at most {REF_MAX_STEPS} timed steps whatever --steps asks), the reference's "
                         f"Stepper.cxx/NoiseGenerator.cxx/measurer.cxx built unmodified against single-node "
                         f"PETSc/MPI/FFTW stand-ins, {R} MPI ranks (processes)"}
        config["implementation"] = "reference stepper and measurer (oracle/_ref/ref_stepper)"
    else:
        Ns = min(a.N, 128)
        nst, nw = a.steps, a.warmup
        rate, ms, el, R = cpu_port_rate(Ns, scounts, a.steps, a.warmup)
        cpu = {"kind": "port", "cores": R,
               "sample": f"{a.steps} timed steps of a {Ns}^3 sample lattice ({el:.1f} s), oracle port with the "
                         f"reference serial RNG; the reference build is absent"}
        config["sample_N"] = Ns
    cpu.update(value=rate, unit="site-updates/s")
    line = {
        "impl": "reference", "metric": "Model G site-updates/s", "value": rate, "unit": "site-updates/s",
        "n_gpus": a.gpus, "steps": nst, "warmup": nw, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config, "cpu_baseline": cpu,
        "e2e": {"value": rate, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


REF_MAX_STEPS = 30  # timed steps of the reference arm at most (bench.py --impl reference)
ENSEMBLE = [(32, 256), (48, 64), (64, 16)]  # (N, replicas)
ENS_H = (0.003, 0.006, 0.012)


def run_ensemble(steps=20, plain_steps=2):
    """Batched ensemble (one launch per sub-step over all replicas, autotuned,
    two-step CUDA graphs) vs looping the single-lattice path one replica per
    launch, and the same ensemble as one persistent launch per step.  Returns
    replica-steps/s of the batched and plain forms and the persistent step time."""
    import ctypes as C

    import torch
    from langevina_b200 import _lib as L

    lib = L.load()
    specs = []
    for N, n in ENSEMBLE:
        for _ in range(n):
            specs.append((N, 1000 + len(specs), ENS_H[len(specs) % 3]))
    R = len(specs)
    sites = sum(N ** 3 for N, _, _ in specs)
    arr = (L.lgv_params * R)()
    for i, (N, seed, H) in enumerate(specs):
        arr[i] = L.make_params(N, seed=seed, **dict(COEF, H=H))
    e = C.c_void_p()
    L.check(lib.lgv_ensemble_create(R, arr, C.byref(e)), "ensemble_create")
    stream = torch.cuda.Stream()
    L.check(lib.lgv_ensemble_set_stream(e, C.c_void_p(stream.cuda_stream)), "ens stream")
    L.check(lib.lgv_ensemble_initialize(e, L.INIT_PHI_GAUSSIAN, 0.1), "init")
    L.check(lib.lgv_ensemble_initialize(e, L.INIT_CHARGES_GAUSSIAN, 0.0), "init")
    choice = (C.c_int * 3)()
    tms = C.c_double()
    L.check(lib.lgv_ensemble_autotune(e, L.PV2HBSPLIT, 2, 3, DT, 4, choice, C.byref(tms)), "autotune")
    L.check(lib.lgv_ensemble_step(e, L.PV2HBSPLIT, 2, 3, DT, 0.0, 4), "warm")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    L.check(lib.lgv_ensemble_step(e, L.PV2HBSPLIT, 2, 3, DT, 0.0, steps), "ens step")
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    # the same steps as one persistent (cooperative) launch per step
    persistent_ms = None
    if lib.lgv_ensemble_use_persistent(e, 1) == L.LGV_OK:
        L.check(lib.lgv_ensemble_step(e, L.PV2HBSPLIT, 2, 3, DT, 0.0, 4), "warm persistent")
        torch.cuda.synchronize()
        e0.record(stream)
        L.check(lib.lgv_ensemble_step(e, L.PV2HBSPLIT, 2, 3, DT, 0.0, steps), "persistent step")
        e1.record(stream)
        torch.cuda.synchronize()
        L.check(lib.lgv_ensemble_synchronize(e), "persistent sync")
        persistent_ms = e0.elapsed_time(e1) / steps
    lib.lgv_ensemble_destroy(e)

    plain = {}
    for mode in ("one_stream", "own_streams"):
        hs = []
        s1 = torch.cuda.Stream()
        for N, seed, H in specs:
            p = L.make_params(N, seed=seed, **dict(COEF, H=H))
            h = C.c_void_p()
            L.check(lib.lgv_create(C.byref(p), C.byref(h)), "create")
            if mode == "one_stream":
                L.check(lib.lgv_set_stream(h, C.c_void_p(s1.cuda_stream)), "stream")
            L.check(lib.lgv_initialize(h, L.INIT_PHI_GAUSSIAN, 0.1), "init")
            L.check(lib.lgv_initialize(h, L.INIT_CHARGES_GAUSSIAN, 0.0), "init")
            hs.append(h)
        for h in hs:
            L.check(lib.lgv_step(h, L.PV2HBSPLIT, 2, 3, DT, 0.0, 1), "warm")
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(3):  # best of three rounds: the loop's host timing is noisy
            t0 = time.perf_counter()
            for _ in range(plain_steps):
                for h in hs:
                    L.check(lib.lgv_step(h, L.PV2HBSPLIT, 2, 3, DT, 0.0, 1), "step")
            torch.cuda.synchronize()
            best = min(best, (time.perf_counter() - t0) / plain_steps * 1e3)
        plain[mode] = best
        for h in hs:
            lib.lgv_destroy(h)
    best_plain = min(plain.values())
    return {
        "workload": "PV2HBSplit23, 256 x 32^3 + 64 x 48^3 + 16 x 64^3 replicas, distinct seeds, "
                    "H in (0.003, 0.006, 0.012) round robin, m^2=-4.813, lambda=10, Gamma=1, chi=5, D=1/3",
        "replicas": R, "sites": sites,
        "batched_ms_per_step": ms, "batched_replica_steps_per_s": R / (ms / 1e3),
        "batched_site_updates_per_s": sites / (ms / 1e3),
        "autotune_choice": {"tile": ["32x8", "16x16"][choice[0]], "zchunk": choice[1],
                            "packing": ["given", "largest_first", "interleaved"][choice[2]]},
        "plain_ms_per_step": plain, "plain_replica_steps_per_s": R / (best_plain / 1e3),
        "speedup_vs_plain": best_plain / ms,
        "persistent_ms_per_step": persistent_ms,
        "persistent_over_batched": (persistent_ms / ms) if persistent_ms else None,
        "timing": "batched: CUDA events over graph replays; persistent: the same with one cooperative launch per "
                  "step (lgv_ensemble_use_persistent); plain: host wall clock around a loop of lgv_step, "
                  "one replica per call (one shared stream / each handle on its own stream), best of three rounds",
    }


MODEL_G_64 = dict(N=64, steps=10000, measure_every=10, mass0=-4.813, lam=10.0, H=0.006, chi=5.0, gamma=1.0,
                  diffusion=1.0 / 3.0, dt=0.04)


def run_slab_emulated(N=256, R=2, steps=5):
    """The z-slab decomposition on one GPU: R slabs of the N^3 lattice, each
    stepping in its own host thread, ghost planes refreshed by device copies
    at host barriers before every cross-plane sub-pass (ThreadHalo).  Reports
    the PV2HBSplit23 step time of the split lattice (wall clock around the
    threads; all slabs share the GPU) against one whole-lattice handle, and the
    exchanges per step.  On one GPU this measures the cost of the exchanges
    and their host synchronisation, not multi-GPU scaling."""
    import ctypes as C

    import numpy as np
    import torch

    from langevina_b200 import _lib as L
    from langevina_b200 import slab as S

    rng = np.random.default_rng(5)
    u = np.zeros((N, N, N, 10))
    u[..., :4] = 0.1 * rng.normal(size=(N, N, N, 4))
    u[..., 4:] = np.sqrt(COEF["chi"]) * rng.normal(size=(N, N, N, 6))
    halo = S.ThreadHalo(R)
    calls = [0]
    inner_exchange = halo.exchange

    def counted(slab, comps):
        if slab.rank == 0:
            calls[0] += 1
        inner_exchange(slab, comps)

    halo.exchange = counted
    slabs = [S.SlabLattice(N, k0, nz, halo, rank=r, seed=99, **COEF) for r, (k0, nz) in enumerate(S.slab_planes(N, R))]
    try:
        for s_ in slabs:
            halo.attach(s_)
            s_.set_global_state(u)
        S.run_threads(slabs, lambda s_: s_.step(L.PV2HBSPLIT, DT, inner=2, outer=3, nsteps=1))
        calls[0] = 0
        t0 = time.perf_counter()
        S.run_threads(slabs, lambda s_: s_.step(L.PV2HBSPLIT, DT, inner=2, outer=3, nsteps=steps))
        for s_ in slabs:
            s_.sync()
        ms_split = (time.perf_counter() - t0) / steps * 1e3
        exchanges = calls[0] / steps
    finally:
        for s_ in slabs:
            s_.close()
    lib = L.load()
    p = L.make_params(N, seed=99, **COEF)
    h = C.c_void_p()
    L.check(lib.lgv_create(C.byref(p), C.byref(h)), "create")
    try:
        u = np.ascontiguousarray(u)  # held while the call reads it
        L.check(lib.lgv_set_state(h, L.ptr(u)), "set_state")
        L.check(lib.lgv_step(h, L.PV2HBSPLIT, 2, 3, DT, 0.0, 1), "warm")
        L.check(lib.lgv_synchronize(h), "sync")
        t0 = time.perf_counter()
        L.check(lib.lgv_step(h, L.PV2HBSPLIT, 2, 3, DT, 0.0, steps), "step")
        L.check(lib.lgv_synchronize(h), "sync")
        ms_whole = (time.perf_counter() - t0) / steps * 1e3
    finally:
        lib.lgv_destroy(h)
    torch.cuda.synchronize()
    return {"workload": f"PV2HBSplit23 on {N}^3 split into {R} z-slabs emulated on one GPU (host threads, "
                        f"device copies of the ghost planes at host barriers)",
            "ranks": R, "split_ms_per_step": ms_split, "whole_ms_per_step": ms_whole,
            "split_over_whole": ms_split / ms_whole, "exchanges_per_step": exchanges,
            "timing": "host wall clock around the steps (both arms), after one warm-up step"}


def run_model_g_64():
    """Full Model G on 64^3 with the (1, 1) composer (one ideal step, one phi
    heat-bath sweep, one charge heat bath per step), charges starting at 0, phi
    from N(0, 0.1^2), 10^4 steps with the full measurement (walls, phase walls,
    z-axis and x/y k modes) into device memory every 10 steps; CUDA events
    around the whole run.  The 21 MB state fits in L2, so this is a rate, not
    an HBM-roofline figure.  Total vector charge is conserved by both the
    advection and the link heat bath; the axial charge is sourced by H."""
    import ctypes as C

    import numpy as np
    import torch
    from langevina_b200 import _lib as L

    lib = L.load()
    c = MODEL_G_64
    N, S, E = c["N"], c["steps"], c["measure_every"]
    V = N ** 3
    p = L.make_params(N, seed=2024, mass0=c["mass0"], lam=c["lam"], H=c["H"], chi=c["chi"], gamma=c["gamma"],
                      diffusion=c["diffusion"])
    h = C.c_void_p()
    L.check(lib.lgv_create(C.byref(p), C.byref(h)), "lgv_create")
    stream = torch.cuda.Stream()
    L.check(lib.lgv_set_stream(h, C.c_void_p(stream.cuda_stream)), "lgv_set_stream")
    L.check(lib.lgv_initialize(h, L.INIT_ZERO, 0.0), "init zero")
    L.check(lib.lgv_initialize(h, L.INIT_PHI_GAUSSIAN, 0.1), "init phi")
    msize = lib.lgv_measure_size(N)
    nmeas = S // E
    meas = torch.empty((nmeas + 1, msize), dtype=torch.float64, device="cuda")
    L.check(lib.lgv_measure_device(h, C.c_void_p(meas[0].data_ptr())), "measure")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t = 0.0
    for n in range(S):
        L.check(lib.lgv_step(h, L.PV2HBSPLIT, 1, 1, c["dt"], t, 1), "step")
        t += c["dt"]
        if (n + 1) % E == 0:
            L.check(lib.lgv_measure_device(h, C.c_void_p(meas[(n + 1) // E].data_ptr())), "measure")
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    oavg = meas[:, :L.NOBS].cpu().numpy()  # OAverage: <phi_a>, <n_A>, <n_V>, <phi^2>
    lib.lgv_destroy(h)
    qv = np.abs(oavg[:, 7:10] * V).max()
    qa = np.abs(oavg[-1, 4:7] * V).max()
    half = oavg[nmeas // 2:]
    return {
        "workload": f"Model G PV2HBSplit11 (ideal + phi heat bath + charge heat bath), {N}^3 periodic, FP64, "
                    f"{S} steps, measurement every {E} steps, charges from 0, phi from N(0, 0.1^2), m^2={c['mass0']}, "
                    f"lambda={c['lam']}, H={c['H']}, chi={c['chi']}, D=1/3, dt={c['dt']}",
        "ms_total": ms, "ms_per_step": ms / S, "site_updates_per_s": V * S / (ms / 1e3),
        "measurements": nmeas, "l2": "state (21 MB) fits in L2: a rate, not an HBM-roofline figure",
        "sigma_second_half": float(half[:, 0].mean()), "pi_sq_second_half": float((half[:, 1:4] ** 2).sum(1).mean()),
        "max_abs_total_vector_charge": float(qv), "final_abs_total_axial_charge": float(qa),
        "timing": "CUDA events on the handle's stream around all steps and measurements",
    }


ADJ = dict(N=48, steps=2000, avg_begin=1000, ckpt=50, dt=0.02, mass0=-4.813, lam=10.0, H=0.01, gamma=1.0)


def run_adjoint(reps=3):
    """Differentiable Euler-Maruyama Model A at 48^3: 2000 steps, loss averaged
    over steps 1001..2000, checkpoints every 50 steps.  Times the plain
    forward (2000 x lgv_step), the differentiable forward (lgv_diff_forward:
    steps + checkpoints + per-step volume averages) and the adjoint
    (lgv_diff_backward: segment recomputation + adjoint kernel) with CUDA events
    on the handle's stream; best of `reps`."""
    import ctypes as C

    import numpy as np
    import torch
    from langevina_b200 import _lib as L

    lib = L.load()
    c = ADJ
    N, S = c["N"], c["steps"]
    p = L.make_params(N, seed=4242, mass0=c["mass0"], lam=c["lam"], H=c["H"], gamma=c["gamma"])
    h = C.c_void_p()
    L.check(lib.lgv_create(C.byref(p), C.byref(h)), "lgv_create")
    stream = torch.cuda.Stream()
    L.check(lib.lgv_set_stream(h, C.c_void_p(stream.cuda_stream)), "lgv_set_stream")
    L.check(lib.lgv_initialize(h, L.INIT_PHI_GAUSSIAN, 0.1), "init phi")
    obs = np.zeros(2)
    w = np.ones(2)
    g = np.zeros(4)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def plain():
        L.check(lib.lgv_step(h, L.MODELA_EM, 1, 1, c["dt"], 0.0, S), "em step")

    def fwd():
        L.check(lib.lgv_diff_forward(h, L.MODELA_EM, c["dt"], 0.0, S, c["avg_begin"], c["ckpt"], L.ptr(obs)),
                "diff_forward")

    def bwd():
        L.check(lib.lgv_diff_backward(h, L.ptr(w), L.ptr(g)), "diff_backward")

    fwd(), bwd(), plain()  # warm-up (allocations, first launches)
    t_plain, t_fwd, t_bwd = [], [], []
    for _ in range(reps):
        t_plain.append(timed(plain))
        t_fwd.append(timed(fwd))
        t_bwd.append(timed(bwd))
    lib.lgv_destroy(h)
    tp, tf, tb = min(t_plain), min(t_fwd), min(t_bwd)
    return {
        "workload": f"Euler-Maruyama Model A {N}^3 FP64, {S} steps, dt={c['dt']}, loss = time average over steps "
                    f"{c['avg_begin'] + 1}..{S} of sigma + V sum_a pibar_a^2, checkpoints every {c['ckpt']} steps, "
                    f"m^2={c['mass0']}, lambda={c['lam']}, H={c['H']}, Gamma={c['gamma']}",
        "plain_forward_ms": tp, "diff_forward_ms": tf, "adjoint_ms": tb,
        "adjoint_over_forward": tb / tp, "forward_plus_adjoint_over_forward": (tf + tb) / tp,
        "gradients_per_s": 1e3 / (tf + tb), "grad": g.tolist(), "obs": obs.tolist(),
        "timing": "CUDA events on the handle's stream, best of %d" % reps,
    }


ADJ_BATCH = dict(R=32, N=32, steps=1000, avg_begin=500, ckpt=50, dt=0.02, mass0=-4.813, lam=10.0, H=0.003, gamma=1.0)


def run_adjoint_batch(reps=3):
    """Batched adjoint: 32 Euler-Maruyama Model A replicas at 32^3 (distinct
    seeds), 1000 steps, loss averaged over steps 501..1000, checkpoints every
    50 steps, all replicas in one launch per step.  Times the plain batched
    forward (lgv_ensemble_step), the differentiable batched forward and the
    batched adjoint with CUDA events, and the same 32 gradients taken one
    replica at a time through lgv_diff_forward / lgv_diff_backward."""
    import ctypes as C

    import numpy as np
    import torch
    from langevina_b200 import _lib as L

    lib = L.load()
    c = ADJ_BATCH
    R, N, S = c["R"], c["N"], c["steps"]
    kw = dict(mass0=c["mass0"], lam=c["lam"], H=c["H"], gamma=c["gamma"])
    arr = (L.lgv_params * R)()
    for r in range(R):
        arr[r] = L.make_params(N, seed=7000 + r, **kw)
    e = C.c_void_p()
    L.check(lib.lgv_ensemble_create(R, arr, C.byref(e)), "ensemble_create")
    stream = torch.cuda.Stream()
    L.check(lib.lgv_ensemble_set_stream(e, C.c_void_p(stream.cuda_stream)), "ens stream")
    L.check(lib.lgv_ensemble_initialize(e, L.INIT_PHI_GAUSSIAN, 0.1), "init")
    obs = np.zeros((R, 2))
    w = np.ones((R, 2))
    g = np.zeros((R, 4))

    def timed(fn, st):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def plain():
        L.check(lib.lgv_ensemble_step(e, L.MODELA_EM, 1, 1, c["dt"], 0.0, S), "ens step")

    def fwd():
        L.check(lib.lgv_ensemble_diff_forward(e, c["dt"], 0.0, S, c["avg_begin"], c["ckpt"], L.ptr(obs)), "fwd")

    def bwd():
        L.check(lib.lgv_ensemble_diff_backward(e, L.ptr(w), L.ptr(g)), "bwd")

    fwd(), bwd(), plain()
    tp, tf, tb = [], [], []
    for _ in range(reps):
        tp.append(timed(plain, stream))
        tf.append(timed(fwd, stream))
        tb.append(timed(bwd, stream))
    lib.lgv_ensemble_destroy(e)

    # one replica at a time through the single-lattice differentiable path
    h = C.c_void_p()
    p0 = L.make_params(N, seed=7000, **kw)
    L.check(lib.lgv_create(C.byref(p0), C.byref(h)), "create")
    s1 = torch.cuda.Stream()
    L.check(lib.lgv_set_stream(h, C.c_void_p(s1.cuda_stream)), "stream")
    o1, g1 = np.zeros(2), np.zeros(4)

    def loop():
        for r in range(R):
            pr = L.make_params(N, seed=7000 + r, **kw)
            L.check(lib.lgv_set_params(h, C.byref(pr)), "params")
            L.check(lib.lgv_initialize(h, L.INIT_PHI_GAUSSIAN, 0.1), "init")
            L.check(lib.lgv_diff_forward(h, L.MODELA_EM, c["dt"], 0.0, S, c["avg_begin"], c["ckpt"], L.ptr(o1)), "f")
            L.check(lib.lgv_diff_backward(h, L.ptr(w[0]), L.ptr(g1)), "b")

    loop()
    tl = timed(loop, s1)
    lib.lgv_destroy(h)
    tp, tf, tb = min(tp), min(tf), min(tb)
    return {
        "workload": f"{R} Euler-Maruyama Model A replicas at {N}^3 FP64, distinct seeds, {S} steps, dt={c['dt']}, "
                    f"loss over steps {c['avg_begin'] + 1}..{S}, checkpoints every {c['ckpt']}, "
                    f"m^2={c['mass0']}, lambda={c['lam']}, H={c['H']}, Gamma={c['gamma']}",
        "plain_batched_forward_ms": tp, "diff_batched_forward_ms": tf, "batched_adjoint_ms": tb,
        "adjoint_over_forward": tb / tp, "forward_plus_adjoint_over_forward": (tf + tb) / tp,
        "gradients_per_s": R * 1e3 / (tf + tb),
        "one_replica_at_a_time_ms": tl, "one_replica_at_a_time_gradients_per_s": R * 1e3 / tl,
        "speedup_vs_one_at_a_time": tl / (tf + tb),
        "timing": "CUDA events, best of %d (batched); one pass (one replica at a time, incl. init)" % reps,
    }


NOMINAL_FP64_TFLOPS = 37.0  # B200 dense FP64 (HGX B200 datasheet); no measured FP64 peak on this pool
POST = dict(T=4096, N=256, ntmax=512, cpu_series=64)


def run_postprocess(reps=5):
    """Post-processing of a 256^3 run's measurement history on the device: the
    k walls of the 11 observables on the 3 axes (3 x 11 x 129 complex series)
    over T = 4096 measurements, their time correlators <O(t) O*(t + tau)>,
    tau < 512 (computeOtOtp, Loader.py:229-254), and the x2k transform of the
    T x 3 x 11 walls of 256 sites (x2k.cxx:94-113).  CUDA events, best of
    `reps`; the CPU leg runs the numpy restatement of the same correlator on
    64 of the series and scales by the series count."""
    import torch

    from langevina_b200 import postprocess as G

    T, N, ntmax = POST["T"], POST["N"], POST["ntmax"]
    NK = N // 2 + 1
    ns = 3 * 11 * NK
    gen = torch.Generator(device="cuda").manual_seed(11)
    d = torch.randn((T, 3, 11, NK), dtype=torch.complex128, device="cuda", generator=gen)
    dc = torch.conj(d).resolve_conj()
    walls = torch.randn((T, 3, 11, N), dtype=torch.float64, device="cuda", generator=gen)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.current_stream()
        torch.cuda.synchronize()
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    corr = lambda: G.computeOtOtp(d, dc, nTMax=ntmax)  # noqa: E731
    xk = lambda: G.x2k(walls)  # noqa: E731
    corr(), xk()
    tc = min(timed(corr) for _ in range(reps))
    tx = min(timed(xk) for _ in range(reps))
    macs = ns * sum(T - tau for tau in range(ntmax))
    flops_c = 8.0 * macs
    flops_x = 4.0 * (T * 3 * 11) * NK * N
    out = {
        "workload": f"measurement history of a {N}^3 run: T={T} samples of the k walls of 11 observables x 3 axes "
                    f"({ns} complex series), correlators for tau < {ntmax}; x2k of T x 3 x 11 walls of {N} sites",
        "correlator_ms": tc, "correlator_fp64_tflops": flops_c / (tc / 1e3) / 1e12,
        "correlator_frac_of_nominal_fp64": flops_c / (tc / 1e3) / 1e12 / NOMINAL_FP64_TFLOPS,
        "x2k_ms": tx, "x2k_fp64_tflops": flops_x / (tx / 1e3) / 1e12,
        "nominal_fp64_tflops": NOMINAL_FP64_TFLOPS,
        "flop_count": "8 per complex multiply-add of the correlator; 4 per real x complex twiddle term of x2k",
        "timing": f"CUDA events, best of {reps}",
    }
    try:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import postprocess as P  # the numpy restatement (CPU leg only)

        k = POST["cpu_series"]
        a = d.reshape(T, -1)[:, :k].cpu().numpy()
        b = dc.reshape(T, -1)[:, :k].cpu().numpy()
        t0 = time.perf_counter()
        P.computeOtOtp(a, b, nTMax=ntmax)
        el = time.perf_counter() - t0
        cpu_ms = el * 1e3 * ns / k
        out["cpu_baseline"] = {"correlator_ms": cpu_ms, "kind": "port", "cores": 1,
                               "sample": f"numpy restatement of computeOtOtp on {k} of the {ns} series "
                                         f"({el:.2f} s), scaled by the series count"}
        out["speedup_vs_cpu"] = cpu_ms / tc
    except Exception as exc:  # the CPU leg is a reported baseline only
        out["cpu_baseline"] = {"unavailable": str(exc)}
    return out


def rank_env():
    """(world, rank, local rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base, rank):
    """Each rank advances its own replica: the lattice does not shard."""
    return base + rank


def max_over_ranks(x, dist, device):
    """The slowest rank's time (every rank calls this at the same point)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, seconds):
    """Units processed by all ranks per second of the slowest rank."""
    return units_per_rank * world / seconds


def run_ours(a):
    import ctypes as C

    import numpy as np
    import torch

    world, rank, local = rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from langevina_b200 import _lib as L

    lib = L.load()
    scounts = tuple(int(x) for x in a.scounts.split(","))
    name = "PV2HBSplit%d%d" % scounts
    N = a.N
    V = N ** 3
    p = L.make_params(N, seed=replica_seed(a.seed, rank), **COEF)
    h = C.c_void_p()
    L.check(lib.lgv_create(C.byref(p), C.byref(h)), "lgv_create")
    stream = torch.cuda.Stream()
    L.check(lib.lgv_set_stream(h, C.c_void_p(stream.cuda_stream)), "lgv_set_stream")
    L.check(lib.lgv_initialize(h, L.INIT_PHI_GAUSSIAN, 0.1), "init phi")
    L.check(lib.lgv_initialize(h, L.INIT_CHARGES_GAUSSIAN, 0.0), "init charges")
    msize = lib.lgv_measure_size(N)
    meas = torch.empty(msize, dtype=torch.float64, device="cuda")

    t_sim = 0.0

    def one_step(s):
        nonlocal t_sim
        if s % MEASURE_EVERY == 0:
            L.check(lib.lgv_measure_device(h, C.c_void_p(meas.data_ptr())), "measure")
        L.check(lib.lgv_step(h, L.PV2HBSPLIT, scounts[0], scounts[1], DT, t_sim, 1), "step")
        t_sim += DT

    for s in range(a.warmup):
        one_step(s)
    torch.cuda.synchronize()

    # ---- timed region: device-resident state, no per-launch instrumentation ---
    clocks = ClockSampler(local)
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in range(a.steps):
        one_step(s)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ck = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    n_meas = len(range(0, a.steps, MEASURE_EVERY))

    # ---- per-kernel split: the same steps again with an event pair around every launch
    split_steps = min(a.steps, 20)
    L.check(lib.lgv_timing_enable(h, 1), "timing")
    for s in range(split_steps):
        one_step(s)
    torch.cuda.synchronize()
    kern = {}
    for k, c in KCLASS.items():
        tot, n = C.c_double(), C.c_int64()
        L.check(lib.lgv_timing_read(h, c, C.byref(tot), C.byref(n)), "timing_read")
        kern[k] = (tot.value, n.value)
    L.check(lib.lgv_timing_enable(h, 0), "timing off")
    # launches of the timed region: the split pass's count per step (the
    # measurement every MEASURE_EVERY steps is 5 launches)
    per_step = sum(n for k, (tot, n) in kern.items() if k != "measure") / split_steps
    launches = int(round(per_step * a.steps)) + 5 * n_meas

    value = whole_job_rate(V * a.steps, world, ms / 1e3)
    peak, peak_kind = peaks()
    dom = max((k for k in ALG_BYTES if kern[k][1] > 0), key=lambda k: kern[k][0])
    tot, n = kern[dom]
    avg_ms = tot / n
    alg = ALG_BYTES[dom] * V
    achieved = alg / (avg_ms / 1e3) / 1e9
    ttab = traffic_table()
    trow = ttab.get(dom)
    traffic = None
    if trow:
        # measured per site at 256^3 (profiles/traffic.json), per launch of this lattice
        traffic = trow["bytes_per_site"] * V
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6.65 TB/s",
                "traffic": traffic, "alg_bytes_per_launch": alg, "avg_launch_ms": avg_ms,
                "traffic_over_alg": (traffic / alg) if traffic else None,
                "frac_of_nominal": achieved / NOMINAL_HBM_GBS, "nominal_GBps": NOMINAL_HBM_GBS}
    kernels = {k: {"launches": kern[k][1], "total_ms": kern[k][0],
                   "avg_ms": (kern[k][0] / kern[k][1]) if kern[k][1] else None,
                   "alg_GBps": (ALG_BYTES[k] * V / (kern[k][0] / kern[k][1] / 1e3) / 1e9)
                   if (k in ALG_BYTES and kern[k][1]) else None,
                   "traffic_over_alg": (ttab[k]["bytes_per_site"] / ttab[k]["alg_bytes_per_site"])
                   if k in ttab else None}
               for k in kern}
    step_frac = STEP_BYTES.get(name, float("nan")) * V * a.steps * 1.0 / (ms / 1e3) / 1e9 / peak

    # ---- e2e: through the C ABI with host buffers -----------------------------
    e2e = None
    if not a.no_e2e:
        u_host = torch.empty(V * 10, dtype=torch.float64).pin_memory()
        meas_host = L.Measurement(N)
        ms_struct = meas_host.struct()
        L.check(lib.lgv_get_state(h, C.c_void_p(u_host.data_ptr())), "get_state")
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        L.check(lib.lgv_set_state(h, C.c_void_p(u_host.data_ptr())), "set_state")
        ts = 0.0
        for s in range(a.steps):
            if s % MEASURE_EVERY == 0:
                L.check(lib.lgv_measure(h, C.byref(ms_struct)), "measure")
            L.check(lib.lgv_step(h, L.PV2HBSPLIT, scounts[0], scounts[1], DT, ts, 1), "step")
            ts += DT
        L.check(lib.lgv_get_state(h, C.c_void_p(u_host.data_ptr())), "get_state")
        el = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        mbytes = msize * 8
        e2e = {"value": whole_job_rate(V * a.steps, world, el), "unit": "site-updates/s",
               "h2d_bytes_per_step": 80 * V / a.steps,
               "d2h_bytes_per_step": (80 * V + n_meas * mbytes) / a.steps,
               "what": "lgv_set_state from pinned host AoS, K x lgv_step with lgv_measure to host every 10 steps, "
                       "lgv_get_state back to pinned host AoS; host wall clock"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline_sample(N, scounts)

    # ---- the other steppers on the same 256^3 lattice ---------------------------
    variants = None
    if rank == 0 and world == 1 and not a.no_variants:
        variants = {}
        for vname, ev, inner, outer, dt, bytes_site in (
                ("PV2HBSplit11", L.PV2HBSPLIT, 1, 1, DT, 800.0),
                ("EulerLangevinHB (Model A heat-bath sweep)", L.EULER_LANGEVIN_HB, 1, 1, DT / 6, 64.0),
                ("ModelAEulerMaruyama", L.MODELA_EM, 1, 1, 0.02, 64.0)):
            nst = 20
            L.check(lib.lgv_step(h, ev, inner, outer, dt, 0.0, 3), "variant warm-up")
            torch.cuda.synchronize()
            v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            v0.record(stream)
            L.check(lib.lgv_step(h, ev, inner, outer, dt, 0.0, nst), "variant")
            v1.record(stream)
            torch.cuda.synchronize()
            vms = v0.elapsed_time(v1) / nst
            variants[vname] = {"ms_per_step": vms, "site_updates_per_s": V / (vms / 1e3),
                               "alg_bytes_per_site": bytes_site,
                               "hbm_frac": bytes_site * V / (vms / 1e3) / 1e9 / peak,
                               "steps": nst, "dt": dt}

    lgv_destroy = lib.lgv_destroy
    lgv_destroy(h)
    ensemble = None
    if world == 1 and not a.no_ensemble:
        ensemble = run_ensemble()
    adjoint = None
    if world == 1 and not a.no_adjoint:
        adjoint = run_adjoint()
        adjoint["batched"] = run_adjoint_batch()
    model_g_64 = None
    slab = None
    if world == 1 and not a.no_variants and not a.no_extras:
        model_g_64 = run_model_g_64()
        slab = run_slab_emulated()
    postprocess = None
    if world == 1 and not a.no_postprocess:
        postprocess = run_postprocess()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": "Model G site-updates/s", "value": value, "unit": "site-updates/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"Model G {name}, {N}^3 periodic lattice, FP64, measure every {MEASURE_EVERY} steps",
                   "N": N, "evolver": name, "dt": DT, **COEF, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (state 1.34 GB at 256^3), no flush"},
        "roofline": roofline,
        "step_hbm_frac": step_frac,
        "step_alg_bytes_per_site": STEP_BYTES.get(name),
        "kernels": kernels,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "ensemble": ensemble,
        "adjoint": adjoint,
        "variants": variants,
        "model_g_64cubed": model_g_64,
        "slab_emulated": slab,
        "postprocess": postprocess,
        "gpu_launches": launches,
        "clocks": ck,
    }
    # The targets in a few compact keys at the end of the line (a truncated
    # log tail still shows them).
    summary = {"step_hbm_frac": step_frac, "ms_per_step": ms / a.steps,
               "dominant_kernel": dom, "dominant_kernel_frac": roofline["frac"]}
    if ensemble:
        summary["ensemble_speedup_vs_plain"] = ensemble["speedup_vs_plain"]
    if adjoint:
        summary["adjoint_over_forward"] = adjoint.get("adjoint_over_forward")
        if adjoint.get("batched"):
            summary["batched_adjoint_over_forward"] = adjoint["batched"].get("adjoint_over_forward")
    if cpu:
        summary["gpu_over_cpu_baseline"] = value / cpu["value"]
    line["summary"] = summary
    print(json.dumps(line))
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())

"""Statistical checks of the GPU stepper against the reference's own physics
goldens and known answers (run on the device, seconds each).

- Equilibrium of the phi heat bath at N=32, m^2=-4.813, H=0.01: <phi_0> and
  <phi^2> against ModelG/hcrit1_N032_m-04813_h010000_l10000_averages_ave.out:1
  (columns 1-2 and 13-14).  The two columns are reproduced at lambda = 4, the
  coupling of the reference's heatbathtest.json that produced the file.
  The same point with two 64-replica ensembles (batched launches): the
  equilibrium does not depend on the proposal width (dt = 0.05 vs 0.2), and
  the pooled averages sit within 5 sigma of the golden (measured pulls -3.3
  for <phi_0> and -2.8 for <phi^2>; the golden's error bar implies a run
  of ~45000 measurements, longer than heatbathtest.json's, so its settings
  are not fully known).
- Free field (lambda = 0, H = 0): the stationary equal-time wall correlator of
  the Euler-Maruyama step equals free2ptFE of ModelG/freeCase.ipynb (cell 7).
- Charge heat bath: the equilibrium of exp(-n^2 / 2 chi) at fixed total charge
  gives <n^2> = chi (1 - 1/V) per component and a flat equal-time spectrum
  <|n_k|^2> = chi / V.
- Ideal PV2 step: second order, the energy error over a fixed time scales as
  dt^2 (plotidealtest.ipynb cells 8-10).
- Counter-stream normals: mean 0, variance 1, kurtosis 3 (test_random.cxx:45-89).
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

from lgvtest import GpuLattice, rand_state

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PV2, NODIFF, ONLYDIFF, IDEAL, HB, CHARGE, EM = 0, 1, 2, 3, 4, 5, 6


class History:
    """Device-side record of measurements: packed lgv_measure_device output,
    one slice kept per sample, all on the lattice's stream."""

    def __init__(self, g, nsamp, lo, hi):
        import torch

        self.torch = torch
        self.g = g
        self.stream = torch.cuda.current_stream()
        g.L.check(g.lib.lgv_set_stream(g.h, C.c_void_p(self.stream.cuda_stream)), "set_stream")
        self.buf = torch.empty(int(g.lib.lgv_measure_size(g.N)), dtype=torch.float64, device="cuda")
        self.hist = torch.empty((nsamp, hi - lo), dtype=torch.float64, device="cuda")
        self.lo, self.hi, self.i = lo, hi, 0

    def take(self):
        g = self.g
        g.L.check(g.lib.lgv_measure_device(g.h, C.c_void_p(self.buf.data_ptr())), "measure_device")
        self.hist[self.i].copy_(self.buf[self.lo:self.hi])
        self.i += 1

    def numpy(self):
        self.torch.cuda.synchronize()
        return self.hist[: self.i].cpu().numpy()


def blocked_err(x, nblock=20):
    n = len(x) // nblock * nblock
    b = x[:n].reshape(nblock, -1).mean(axis=1)
    return b.std(ddof=1) / math.sqrt(nblock)


def test_equilibrium_matches_hcrit1_golden(lgv):
    with open(os.path.join(GOLD, "hcrit1.json")) as f:
        gold = json.load(f)
    N = 32
    g = GpuLattice(lgv, N, mass0=-4.813, lam=4.0, H=0.01, gamma=1.0, seed=31337)
    g.initialize(1, 0.3)
    g.step(HB, 0.1, nsteps=4000)
    nsamp, every = 8000, 25
    h = History(g, nsamp, 0, 11)
    for _ in range(nsamp):
        g.step(HB, 0.1, nsteps=every)
        h.take()
    o = h.numpy()
    phi0, phi2 = o[:, 0], o[:, 10]
    m0, e0 = phi0.mean(), blocked_err(phi0)
    m2, e2 = phi2.mean(), blocked_err(phi2)
    s0 = math.hypot(e0, gold["phi0_err"])
    s2 = math.hypot(e2, 4.8322472767e-05)
    print(f"<phi0> = {m0:.5f} +- {e0:.5f} (golden {gold['phi0_mean']:.5f} +- {gold['phi0_err']:.5f}); "
          f"<phi^2> = {m2:.5f} +- {e2:.5f} (golden 0.99771)")
    assert e0 < 0.002, "run too short for a meaningful check"
    assert abs(m0 - gold["phi0_mean"]) < 4 * s0
    assert abs(m2 - 0.99771450882) < 4 * s2


def ensemble_hb_equilibrium(lgv, R, seed0, dt, therm=4000, nsamp=4000, every=25, N=32):
    """<phi_0> and <phi^2> of R independent 32^3 replicas of the phi heat
    bath at the hcrit1 point (lambda = 4), one batched launch per half sweep;
    the error is the spread of the replica means (independent runs)."""
    import torch
    from langevina_b200 import _lib as L

    lib = L.load()
    arr = (L.lgv_params * R)()
    for r in range(R):
        arr[r] = L.make_params(N, mass0=-4.813, lam=4.0, H=0.01, gamma=1.0, seed=seed0 + r)
    e = C.c_void_p()
    L.check(lib.lgv_ensemble_create(R, arr, C.byref(e)), "ensemble_create")
    try:
        L.check(lib.lgv_ensemble_set_stream(e, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
        L.check(lib.lgv_ensemble_initialize(e, 1, 0.3), "init")
        L.check(lib.lgv_ensemble_step(e, HB, 1, 1, dt, 0.0, therm), "thermalise")
        hist = torch.empty((nsamp, R, 11), dtype=torch.float64, device="cuda")
        for i in range(nsamp):
            L.check(lib.lgv_ensemble_step(e, HB, 1, 1, dt, 0.0, every), "sweeps")
            L.check(lib.lgv_ensemble_oaverage_device(e, C.c_void_p(hist[i].data_ptr())), "oaverage")
        torch.cuda.synchronize()
    finally:
        lib.lgv_ensemble_destroy(e)
    h = hist.cpu().numpy()
    out = {}
    for name, col in (("phi0", 0), ("phi2", 10)):
        m = h[:, :, col].mean(axis=0)
        out[name] = (m.mean(), m.std(ddof=1) / math.sqrt(R))
    return out


def test_heat_bath_equilibrium_is_dt_independent_and_near_hcrit1(lgv):
    """Metropolis with a symmetric proposal of width sqrt(2 dt Gamma) samples
    exp(-S) whatever dt is: two 64-replica ensembles at dt = 0.05 and 0.2
    must agree.  Their pooled <phi_0>, <phi^2> are then set against the
    equilibrium of the reference's own EulerLangevinHB at the same point
    (tests/golden/hcrit1_refbuild.json: seven runs of the reference build,
    tests/golden/make_hcrit_refbuild.py) within 4 sigma, and against the
    hcrit1 file golden (columns 1-2 and 13-14) within 5 sigma -- the file sits
    4.0 and 3.3 sigma above the reference's own heat bath too."""
    with open(os.path.join(GOLD, "hcrit1.json")) as f:
        gold = json.load(f)
    with open(os.path.join(GOLD, "hcrit1_refbuild.json")) as f:
        ref = json.load(f)
    a = ensemble_hb_equilibrium(lgv, 64, 7000, 0.05)
    b = ensemble_hb_equilibrium(lgv, 64, 9000, 0.2)
    golden = {"phi0": (gold["phi0_mean"], gold["phi0_err"]), "phi2": (0.99771450882, 4.8322472767e-05)}
    for k in ("phi0", "phi2"):
        (ma, ea), (mb, eb) = a[k], b[k]
        assert ea < 5e-4 and eb < 5e-4
        assert abs(ma - mb) < 4 * math.hypot(ea, eb), f"{k}: dt 0.05 {ma:.6f}+-{ea:.6f} vs dt 0.2 {mb:.6f}+-{eb:.6f}"
        w = np.array([1 / ea ** 2, 1 / eb ** 2])
        m = (w[0] * ma + w[1] * mb) / w.sum()
        e = 1 / math.sqrt(w.sum())
        g, ge = golden[k]
        pull = (m - g) / math.hypot(e, ge)
        rm, re = ref[k]["mean"], ref[k]["err"]
        rpull = (m - rm) / math.hypot(e, re)
        print(f"{k}: dt 0.05 {ma:.6f}+-{ea:.6f}, dt 0.2 {mb:.6f}+-{eb:.6f}, pooled {m:.6f}+-{e:.6f}, "
              f"reference build {rm:.6f}+-{re:.6f} (pull {rpull:+.2f}), file golden {g:.6f}+-{ge:.6f} "
              f"(pull {pull:+.2f})")
        assert abs(rpull) < 4
        assert abs(pull) < 5


def free2pt_fe(n, m2, dt, N, gamma=1.0):
    """free2ptFE of freeCase.ipynb (cell 7), S -> infinity."""
    kn2 = -2.0 * (np.cos(2.0 * np.pi * n / N) - 1.0)
    w2 = m2 + kn2
    return 2.0 / w2 / (2.0 - dt * gamma * w2) / N ** 3


def test_free_field_euler_maruyama_propagator(lgv):
    # the Jacobi Euler step is stable for dt * (m^2 + 12) < 2 (12 = largest
    # eigenvalue of the 3-D lattice Laplacian)
    N, m2, dt = 8, 0.25, 0.1
    g = GpuLattice(lgv, N, mass0=m2, lam=0.0, H=0.0, gamma=1.0, seed=2024)
    g.initialize(0)
    g.step(EM, dt, nsteps=500)
    NK = N // 2 + 1
    lo = 11 + 33 * N  # wall_k[0..2] start in the packed measurement
    hi = lo + 3 * 11 * NK * 2
    nsamp, every = 20000, 20
    h = History(g, nsamp, lo, hi)
    for _ in range(nsamp):
        g.step(EM, dt, nsteps=every)
        h.take()
    w = h.numpy().reshape(nsamp, 3, 11, NK, 2)[:, :, :4]  # phi components only
    p = (w ** 2).sum(axis=-1)  # |W(k)|^2
    per = p.reshape(nsamp, -1, NK)
    mean = per.mean(axis=(0, 1))
    err = np.array([blocked_err(per[:, :, k].mean(axis=1)) for k in range(NK)])
    want = free2pt_fe(np.arange(NK), m2, dt, N)
    print("ratio to free2ptFE:", mean / want, "rel err", err / want)
    assert np.all(np.abs(mean - want) < 5 * err + 1e-3 * want)
    # distinguishes the Euler scheme from the continuum propagator 1/(w^2 N^3)
    cont = 1.0 / (m2 + 2 * (1 - np.cos(2 * np.pi * np.arange(NK) / N))) / N ** 3
    assert abs(mean[-1] / cont[-1] - 1) > 0.2


def test_charge_susceptibility_and_white_spectrum(lgv):
    N, chi = 16, 5.0
    V = N ** 3
    g = GpuLattice(lgv, N, chi=chi, diffusion=1.0 / 3.0, seed=77)
    g.initialize(0)  # zero charges: conserved total 0
    g.step(CHARGE, 0.5, nsteps=3000)
    s = []
    NK = N // 2 + 1
    lo = 11 + 33 * N
    hi = lo + 3 * 11 * NK * 2
    nsamp = 300
    h = History(g, nsamp, lo, hi)
    for _ in range(nsamp):
        g.step(CHARGE, 0.5, nsteps=20)
        h.take()
    u = g.get_state()
    n2 = (u[..., 4:] ** 2).mean()
    assert abs(n2 - chi * (1 - 1.0 / V)) < 0.02 * chi, n2
    assert np.max(np.abs(u[..., 4:].reshape(-1, 6).sum(axis=0))) < 1e-9  # conserved
    w = h.numpy().reshape(nsamp, 3, 11, NK, 2)[:, :, 4:10, 1:]  # charges, k != 0
    pk = (w ** 2).sum(axis=-1).mean()
    assert abs(pk / (chi / V) - 1) < 0.05, pk / (chi / V)


def test_ideal_step_energy_error_is_second_order(lgv):
    N = 16
    u = rand_state(N, 5, phi_scale=0.5, chi=5.0)
    errs = []
    for dt in (0.04, 0.02):
        g = GpuLattice(lgv, N, mass0=-4.813, lam=4.0, H=0.0, chi=5.0, seed=1)
        g.set_state(u)
        e0 = g.energy()
        g.step(IDEAL, dt, nsteps=int(round(0.8 / dt)))
        errs.append(abs(g.energy() - e0))
    ratio = errs[0] / errs[1]
    assert 3.0 < ratio < 5.0, (errs, ratio)


def test_counter_normals_moments(lgv):
    N = 64
    g = GpuLattice(lgv, N, seed=99)
    g.initialize(1, 1.0)
    x = g.get_state()[..., :4].ravel()
    assert abs(x.mean()) < 5 / math.sqrt(x.size)
    assert abs(x.var() - 1) < 5 * math.sqrt(2 / x.size)
    k = ((x - x.mean()) ** 4).mean() / x.var() ** 2
    assert abs(k - 3) < 5 * math.sqrt(24 / x.size)

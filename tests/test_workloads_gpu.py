"""End-to-end GPU parity on the workloads of the first two benchmark
configurations, against the CPU oracle.

- Plain Model A on 32^3: 1000 phi heat-bath sweeps from phi ~ 0.1 N(0,1)
  (m^2 = -4.813, lambda = 10, H = 0.01, dt = 0.04) with injected identical
  noise on both sides, measuring every 10 sweeps (volume averages and the
  z-axis k modes k = 0..16, the x2k output).  Accept decisions must agree at
  every sweep; states and measurements within 1e-11.
- Full Model G on 64^3 with the (1, 1) composer (ideal step, phi heat bath,
  charge heat bath), charges from 0, phi ~ N(0, 0.1^2), H = 0.006, chi = 5,
  D = 1/3, dt = 0.04, counter noise (restated independently in the oracle):
  20 steps, measuring every 10, with the total vector charge conserved.
"""
import numpy as np
import pytest

from lgvtest import GpuLattice, assert_state_close, compare_flags, hb_noise, rand_state

pytestmark = pytest.mark.gpu

HB, PV2 = 4, 0
INJECTED = 1


def _meas_close(gm, om, rtol, what):
    ga, oa = gm.arrays(), om.arrays()
    for k in ga:
        d = np.max(np.abs(ga[k] - oa[k]))
        scale = max(1.0, np.max(np.abs(oa[k])))
        assert d <= rtol * scale, f"{what} {k}: {d:.3e}"


def test_model_a_32cubed_1000_sweeps_injected(lgv, oracle_mod):
    from langevina_b200 import _lib as L

    N, seed = 32, 20240101
    c = dict(mass0=-4.813, lam=10.0, H=0.01, gamma=1.0, seed=seed)
    g = GpuLattice(lgv, N, **c)
    o = oracle_mod.Oracle(N, mode=oracle_mod.INJECTED, nranks=4, **c)
    u = np.zeros((N, N, N, 10))
    u[..., :4] = 0.1 * np.random.default_rng(seed).normal(size=(N, N, N, 4))
    g.set_state(u)
    o.set_state(u)
    g.mode(INJECTED)
    g.flags(True)
    o.debug_flags(True)
    for sweep in range(1000):
        prop, acc = hb_noise(N, seed + sweep)
        g.inject_hb(prop, acc)
        o.inject_hb(prop, acc)
        g.step(HB, 0.04, t=0.0)
        o.step(HB, 0.04, t=0.0)
        assert compare_flags(g.get_flags(), o.get_flags(), N ** 3) == 0, f"sweep {sweep}"
        if (sweep + 1) % 10 == 0:
            gm, om = g.measure(), o.measure(L.Measurement(N))
            _meas_close(gm, om, 1e-11, f"sweep {sweep + 1}")
            kz = gm.wall_k[2][:, :17]  # z-axis modes k = 0..16 of the 11 observables
            assert kz.shape == (11, 17, 2) and np.all(np.isfinite(kz))
    assert_state_close(g.get_state(), o.get_state(), rtol=1e-11, what="32^3 Model A after 1000 sweeps")


def test_model_g_64cubed_counter(lgv, oracle_mod):
    from langevina_b200 import _lib as L

    N, seed = 64, 2024
    c = dict(mass0=-4.813, lam=10.0, H=0.006, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=seed)
    g = GpuLattice(lgv, N, **c)
    o = oracle_mod.Oracle(N, mode=oracle_mod.COUNTER, nranks=8, **c)
    u = rand_state(N, seed, phi_scale=0.1, charges=False)
    g.set_state(u)
    o.set_state(u)
    V = N ** 3
    t = 0.0
    for step in range(20):
        g.step(PV2, 0.04, t=t, inner=1, outer=1)
        o.step(PV2, 0.04, t=t, inner=1, outer=1)
        t += 0.04
        if (step + 1) % 10 == 0:
            gm, om = g.measure(), o.measure(L.Measurement(N))
            _meas_close(gm, om, 1e-11, f"step {step + 1}")
            assert np.abs(gm.OAverage[7:10] * V).max() < 1e-10  # total vector charge stays 0
    assert g.counter() == o.get_counter()
    gs = g.get_state()
    assert_state_close(gs, o.get_state(), rtol=1e-11, what="64^3 Model G after 20 steps")
    assert np.abs(gs[..., 7:10].sum(axis=(0, 1, 2))).max() < 1e-10

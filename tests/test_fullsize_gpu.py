"""Parity at the bench's full size, 256^3 (16.8 M sites, 1.34 GB of state).

At this size the phi and charge passes run on their row grid (half rows of
128 sites, one block per row) and the ideal step on the TMA kernel with a
full z-march, none of which the smaller parity lattices reach.  Against the
oracle in counter noise, from one seeded state:
- one Model G step PV2HBSplit23 (3 x [ideal + 2 phi sweeps] + charge heat
  bath), then one Euler-Maruyama step: per-site relative error <= 1e-12;
- the full measurement (walls, phase walls, k modes) within 1e-11;
- the noise counter.
Size-independent properties on the device alone: a rerun from the same state
and counter is bit-identical (no atomics on the state path), two single steps
equal one two-step call, and the total vector charge is conserved.
"""
import os

import numpy as np
import pytest

from lgvtest import GpuLattice, assert_state_close, rand_state

pytestmark = pytest.mark.gpu

N = 256
PV2, HB, EM = 0, 4, 6
COEF = dict(mass0=-4.813, lam=10.0, H=0.003, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=2718)


@pytest.fixture(scope="module")
def start():
    return rand_state(N, 256, phi_scale=0.3)


def _meas_close(gm, om, rtol, what):
    ga, oa = gm.arrays(), om.arrays()
    for k in ga:
        d = np.max(np.abs(ga[k] - oa[k]))
        scale = max(1.0, np.max(np.abs(oa[k])))
        assert d <= rtol * scale, f"{what} {k}: {d:.3e}"


def test_model_g_step_matches_oracle_at_256(lgv, oracle_mod, start):
    from langevina_b200 import _lib as L

    g = GpuLattice(lgv, N, **COEF)
    o = oracle_mod.Oracle(N, mode=oracle_mod.COUNTER, nranks=min(16, os.cpu_count() or 1), **COEF)
    g.set_state(start)
    o.set_state(start)
    g.step(PV2, 0.04, t=0.0, inner=2, outer=3)
    o.step(PV2, 0.04, t=0.0, inner=2, outer=3)
    assert g.counter() == o.get_counter() == 3 * 2 + 7
    assert_state_close(g.get_state(), o.get_state(), what="PV2HBSplit23 at 256^3")
    _meas_close(g.measure(), o.measure(L.Measurement(N)), 1e-11, "measurement at 256^3")
    g.step(EM, 0.02, t=0.04)
    o.step(EM, 0.02, t=0.04)
    assert_state_close(g.get_state(), o.get_state(), what="Euler-Maruyama at 256^3")
    g.close()


def test_rerun_is_bit_identical_and_steps_compose(lgv, start):
    runs = []
    for split in (False, True, False):
        g = GpuLattice(lgv, N, **COEF)
        g.set_state(start)
        if split:
            g.step(PV2, 0.04, t=0.0, inner=2, outer=3)
            g.step(PV2, 0.04, t=0.04, inner=2, outer=3)
        else:
            g.step(PV2, 0.04, t=0.0, nsteps=2, inner=2, outer=3)
        runs.append((g.counter(), g.get_state(), g.measure().OAverage.copy()))
        g.close()
    (c0, u0, m0), (c1, u1, m1), (c2, u2, m2) = runs
    assert c0 == c1 == c2 == 2 * 13
    assert np.array_equal(u0, u2) and np.array_equal(m0, m2), "rerun differs"
    assert np.array_equal(u0, u1), "two single steps differ from one two-step call"
    # the initial total vector charge is sum(start[..., 7:10]); the ideal
    # step moves it between sites and the charge heat bath exchanges it on links
    dv = (u0[..., 7:10] - start[..., 7:10]).sum(axis=(0, 1, 2))
    assert np.abs(dv).max() < 1e-9, f"vector charge drift {dv}"

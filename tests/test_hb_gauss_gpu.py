"""Gaussian proposals for the phi heat bath (lgv_set_hb_proposal), an option
beside the reference's U(-sqrt3, sqrt3) proposals (Stepper.cxx:343).

- With counter noise the GPU equals the oracle's restatement (the four
  normals of two Box-Muller pairs from the site's first four draws, then the
  accept uniform): states to the parity tolerance and the same accept
  decisions except flagged ties, for heat-bath sweeps and PV2HBSplit23 steps.
- A slab split of the lattice equals the whole lattice bit for bit with the
  option on.
- The option is refused where it is not implemented, and the default stays
  the uniform proposal (bit-identical to a handle that never set it).
- Both proposals sample the same equilibrium: <phi_0> and <phi^2> at the
  hcrit1 point (N = 16) agree within their batch errors.
"""
import ctypes as C

import numpy as np
import pytest

from lgvtest import GpuLattice, assert_state_close, compare_flags, rand_state

pytestmark = pytest.mark.gpu

PV2, HB = 0, 4
COEF = dict(mass0=-4.813, lam=10.0, H=0.01, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=8675309)


def gauss_on(g):
    from langevina_b200 import _lib as L

    L.check(g.lib.lgv_set_hb_proposal(g.h, L.HB_PROPOSAL_GAUSSIAN), "set_hb_proposal")


@pytest.mark.parametrize("N,ev,n", [(8, HB, 3), (16, HB, 2), (34, HB, 2), (16, PV2, 2)])
def test_gaussian_proposals_match_the_oracle(lgv, oracle_mod, N, ev, n):
    g = GpuLattice(lgv, N, **COEF)
    o = oracle_mod.Oracle(N, mode=oracle_mod.COUNTER, **COEF)
    gauss_on(g)
    o.set_hb_proposal(1)
    u = rand_state(N, 900 + N)
    g.set_state(u)
    o.set_state(u)
    if ev == HB:
        g.flags(True)
        o.debug_flags(True)
    g.step(ev, 0.05, nsteps=n, inner=2, outer=3)
    o.step(ev, 0.05, nsteps=n, inner=2, outer=3)
    if ev == HB:
        assert compare_flags(g.get_flags(), o.get_flags(), N ** 3) == 0
    assert g.counter() == o.get_counter()
    assert_state_close(g.get_state(), o.get_state(), rtol=1e-11, what="Gaussian-proposal heat bath")
    # and the proposals are not the uniform ones: the same steps without the option differ
    g2 = GpuLattice(lgv, N, **COEF)
    g2.set_state(u)
    g2.step(ev, 0.05, nsteps=n, inner=2, outer=3)
    assert not np.array_equal(g2.get_state(), g.get_state())
    for x in (g, g2):
        x.close()


def test_gaussian_proposals_on_slabs_equal_the_whole_lattice(lgv):
    from langevina_b200 import _lib as L
    from langevina_b200 import slab as S

    N, R = 32, 2
    u = rand_state(N, 4040)
    halo = S.ThreadHalo(R)
    slabs = [S.SlabLattice(N, k0, nz, halo, rank=r, **COEF) for r, (k0, nz) in enumerate(S.slab_planes(N, R))]
    for s in slabs:
        halo.attach(s)
        s.set_global_state(u)
        L.check(s.lib.lgv_set_hb_proposal(s.h, L.HB_PROPOSAL_GAUSSIAN), "slab proposal")
    S.run_threads(slabs, lambda s: s.step(PV2, 0.04, nsteps=2, inner=2, outer=3))
    got = np.concatenate([s.get_interior() for s in slabs], axis=0)
    g = GpuLattice(lgv, N, **COEF)
    gauss_on(g)
    g.set_state(u)
    g.step(PV2, 0.04, nsteps=2, inner=2, outer=3)
    assert np.array_equal(got, g.get_state())
    for s in slabs:
        s.close()
    g.close()


def test_proposal_argument_checks_and_default(lgv, monkeypatch):
    from langevina_b200 import _lib as L

    g = GpuLattice(lgv, 8, **COEF)
    assert g.lib.lgv_set_hb_proposal(g.h, 2) == L.LGV_ERR_INVALID
    assert g.lib.lgv_set_hb_proposal(None, 0) == L.LGV_ERR_INVALID
    u = rand_state(8, 12)
    g.set_state(u)
    L.check(g.lib.lgv_set_hb_proposal(g.h, L.HB_PROPOSAL_UNIFORM), "uniform")
    g.step(HB, 0.05, nsteps=2)
    g0 = GpuLattice(lgv, 8, **COEF)  # never set: the uniform default
    g0.set_state(u)
    g0.step(HB, 0.05, nsteps=2)
    assert np.array_equal(g.get_state(), g0.get_state())
    monkeypatch.setenv("LGV_HB_FUSED", "1")
    gf = GpuLattice(lgv, 8, **COEF)
    monkeypatch.delenv("LGV_HB_FUSED")
    assert gf.lib.lgv_set_hb_proposal(gf.h, L.HB_PROPOSAL_GAUSSIAN) == L.LGV_ERR_UNSUPPORTED
    for x in (g, g0, gf):
        x.close()


def _equilibrium(lgv, gaussian, N=16, therm=2000, sweeps=20000, every=10, nbatch=20):
    from langevina_b200 import _lib as L

    g = GpuLattice(lgv, N, **dict(COEF, seed=31337 if gaussian else 27182))
    if gaussian:
        gauss_on(g)
    L.check(g.lib.lgv_initialize(g.h, L.INIT_PHI_GAUSSIAN, 0.1), "init")
    g.step(HB, 0.1, nsteps=therm)
    phi0, phi2 = [], []
    for _ in range(sweeps // every):
        g.step(HB, 0.1, nsteps=every)
        m = g.measure()
        phi0.append(m.OAverage[0])
        phi2.append(m.OAverage[10])
    g.close()
    out = []
    for x in (np.array(phi0), np.array(phi2)):
        b = x.reshape(nbatch, -1).mean(axis=1)
        out.append((b.mean(), b.std(ddof=1) / np.sqrt(nbatch)))
    return out


def test_both_proposals_sample_the_same_equilibrium(lgv):
    gu = _equilibrium(lgv, False)
    gg = _equilibrium(lgv, True)
    for (mu, eu), (mg, eg), name in zip(gu, gg, ("<phi_0>", "<phi^2>")):
        z = abs(mu - mg) / np.hypot(eu, eg)
        assert z < 5.0, f"{name}: uniform {mu:.5f}+-{eu:.5f}, Gaussian {mg:.5f}+-{eg:.5f} ({z:.1f} sigma)"

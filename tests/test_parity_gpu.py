"""GPU parity: the sm_100a kernels (through the C ABI) against the CPU oracle.

Each stepper of ModelG/Stepper.cxx is run on the same seeded state with the
same noise -- injected arrays, or the counter streams, which the oracle
restates independently -- and compared per site at 1e-12 relative (FP64 with
FMA contraction on the device), with identical accept decisions except where
the oracle flags a tie (|dS| < 1e-14 or |r - exp(-dS)| < 1e-12).
"""
import math

import numpy as np
import pytest

from lgvtest import (RTOL, GpuLattice, assert_state_close, charge_noise, compare_flags, em_noise, hb_noise,
                     rand_state)

pytestmark = pytest.mark.gpu

PV2, NODIFF, ONLYDIFF, IDEAL, HB, CHARGE, EM = 0, 1, 2, 3, 4, 5, 6
COUNTER, INJECTED = 0, 1

COEF = dict(mass0=-4.813, lam=10.0, H=0.01, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=122335456)


def pair(lgv, oracle_mod, N, mode_orc, **kw):
    c = dict(COEF)
    c.update(kw)
    g = GpuLattice(lgv, N, **c)
    o = oracle_mod.Oracle(N, mode=mode_orc, **c)
    return g, o


@pytest.mark.parametrize("N", [4, 6, 8, 34])
def test_state_roundtrip_is_exact(lgv, N):
    g = GpuLattice(lgv, N)
    u = rand_state(N, 1)
    g.set_state(u)
    assert np.array_equal(g.get_state(), u)


@pytest.mark.parametrize("N,seed", [(4, 1), (6, 2), (8, 3), (16, 4), (34, 5)])
def test_phi_heatbath_injected(lgv, oracle_mod, N, seed):
    g, o = pair(lgv, oracle_mod, N, oracle_mod.INJECTED)
    u = rand_state(N, seed)
    g.set_state(u)
    o.set_state(u)
    g.mode(INJECTED)
    g.flags(True)
    o.debug_flags(True)
    for sweep in range(2):
        prop, acc = hb_noise(N, 100 * seed + sweep)
        g.inject_hb(prop, acc)
        o.inject_hb(prop, acc)
        g.step(HB, 0.04 / 6, t=0.0)
        o.step(HB, 0.04 / 6, t=0.0)
        ties = compare_flags(g.get_flags(), o.get_flags(), N ** 3)
        assert ties == 0
    assert_state_close(g.get_state(), o.get_state(), what="phi HB injected")


@pytest.mark.parametrize("N", [4, 8, 12])
def test_phi_heatbath_counter(lgv, oracle_mod, N):
    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER, dmassdt=0.1)
    u = rand_state(N, 7)
    g.set_state(u)
    o.set_state(u)
    g.counter(5)
    o.set_counter(5)
    g.step(HB, 0.1, t=0.5, nsteps=4)
    o.step(HB, 0.1, t=0.5, nsteps=4)
    assert g.counter() == o.get_counter() == 9
    assert_state_close(g.get_state(), o.get_state(), what="phi HB counter")


@pytest.mark.parametrize("N,seed", [(4, 11), (6, 12), (8, 13), (16, 14)])
def test_charge_heatbath_injected(lgv, oracle_mod, N, seed):
    g, o = pair(lgv, oracle_mod, N, oracle_mod.INJECTED)
    u = rand_state(N, seed)
    g.set_state(u)
    o.set_state(u)
    g.mode(INJECTED)
    g.flags(True)
    o.debug_flags(True)
    order, q, acc = charge_noise(N, seed)
    g.inject_charge(order, q, acc)
    o.inject_charge(order, q, acc)
    g.step(CHARGE, 0.04)
    o.step(CHARGE, 0.04)
    ties = compare_flags(g.get_flags(), o.get_flags(), 36 * N ** 3)
    assert ties == 0
    gs, os_ = g.get_state(), o.get_state()
    assert_state_close(gs, os_, what="charge HB injected")
    assert np.array_equal(gs[..., :4], u[..., :4])  # phi untouched


@pytest.mark.parametrize("N", [4, 8, 10])
def test_charge_heatbath_counter(lgv, oracle_mod, N):
    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER)
    u = rand_state(N, 21)
    g.set_state(u)
    o.set_state(u)
    g.step(CHARGE, 0.2, nsteps=3)
    o.step(CHARGE, 0.2, nsteps=3)
    assert g.counter() == o.get_counter() == 21
    assert_state_close(g.get_state(), o.get_state(), what="charge HB counter")


@pytest.mark.parametrize("N,dt,chi", [(4, 0.04, 5.0), (6, 0.04, 5.0), (8, 0.2, 5.0), (16, 0.04, 5.0),
                                      (34, 0.04, 5.0), (48, 0.01, 5.0), (8, 0.5, 0.2), (32, 0.04, 5.0),
                                      (64, 0.04, 5.0), (32, 0.5, 0.2), (96, 0.02, 5.0)])
def test_ideal_step(lgv, oracle_mod, N, dt, chi):
    """dt=0.5, chi=0.2 drives half-step angles past 1/4: the sincos branch.
    N divisible by 32 runs the TMA-staged kernel, other N the cp.async one."""
    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER, chi=chi)
    u = rand_state(N, 31, chi=chi)
    g.set_state(u)
    o.set_state(u)
    g.step(IDEAL, dt, nsteps=2)
    o.step(IDEAL, dt, nsteps=2)
    assert_state_close(g.get_state(), o.get_state(), rtol=RTOL, what="ideal")


@pytest.mark.parametrize("N", [4, 8, 12])
def test_em_injected_and_counter(lgv, oracle_mod, N):
    g, o = pair(lgv, oracle_mod, N, oracle_mod.INJECTED, dmassdt=-0.2)
    u = rand_state(N, 41)
    g.set_state(u)
    o.set_state(u)
    g.mode(INJECTED)
    xi = em_noise(N, 42)
    g.inject_em(xi)
    o.inject_em(xi)
    g.step(EM, 0.02, t=0.3)
    o.step(EM, 0.02, t=0.3)
    assert_state_close(g.get_state(), o.get_state(), what="EM injected")

    g2, o2 = pair(lgv, oracle_mod, N, oracle_mod.COUNTER)
    g2.set_state(u)
    o2.set_state(u)
    g2.step(EM, 0.02, nsteps=5)
    o2.step(EM, 0.02, nsteps=5)
    assert_state_close(g2.get_state(), o2.get_state(), what="EM counter")
    assert np.array_equal(g2.get_state()[..., 4:], u[..., 4:])


@pytest.mark.parametrize("ev,inner,outer,N", [(PV2, 2, 3, 8), (PV2, 1, 1, 8), (PV2, 2, 3, 16), (NODIFF, 2, 3, 6),
                                              (ONLYDIFF, 2, 3, 6), (PV2, 3, 1, 4), (PV2, 2, 3, 32)])
def test_pv2hbsplit_counter(lgv, oracle_mod, ev, inner, outer, N):
    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER)
    u = rand_state(N, 51)
    g.set_state(u)
    o.set_state(u)
    g.step(ev, 0.04, t=0.0, nsteps=2, inner=inner, outer=outer)
    o.step(ev, 0.04, t=0.0, nsteps=2, inner=inner, outer=outer)
    assert g.counter() == o.get_counter()
    assert_state_close(g.get_state(), o.get_state(), rtol=1e-11, what="PV2HBSplit")


def _cmp_meas(gm, om, atol):
    ga, oa = gm.arrays(), om.arrays()
    for k in ga:
        d = np.max(np.abs(ga[k] - oa[k]))
        scale = max(1.0, np.max(np.abs(oa[k])))
        assert d <= atol * scale, f"{k}: {d:.3e}"


@pytest.mark.parametrize("N", [4, 8, 16, 32])
def test_measurer(lgv, oracle_mod, N):
    from langevina_b200 import _lib as L

    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER)
    u = rand_state(N, 61)
    u[..., 0] += 0.3  # a vev, so rotate_to_vev picks a direction
    g.set_state(u)
    o.set_state(u)
    gm = g.measure()
    om = o.measure(L.Measurement(N))
    _cmp_meas(gm, om, 1e-13)


def test_measurer_zero_field(lgv, oracle_mod):
    """phi = 0: sigma^2 below 100*DBL_MIN takes n = (1,0,0,0) (measurer.cxx:159-165)."""
    from langevina_b200 import _lib as L

    N = 6
    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER)
    u = rand_state(N, 62)
    u[..., :4] = 0.0
    g.set_state(u)
    o.set_state(u)
    _cmp_meas(g.measure(), o.measure(L.Measurement(N)), 1e-13)


@pytest.mark.parametrize("N", [4, 8, 20])
def test_energy(lgv, oracle_mod, N):
    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER)
    u = rand_state(N, 71)
    g.set_state(u)
    o.set_state(u)
    e1, e2 = g.energy(), o.energy()
    assert abs(e1 - e2) <= 1e-12 * abs(e2)


@pytest.mark.parametrize("N", [4, 10])
def test_counter_initial_conditions(lgv, oracle_mod, N):
    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER)
    g.counter(3)
    o.set_counter(3)
    g.initialize(0)
    o.initialize(0)
    g.initialize(1, 0.1)  # phi ~ 0.1 N(0,1)
    o.initialize(1, 0.1)
    g.initialize(2)       # charges ~ sqrt(chi) N(0,1), zero mode removed
    o.initialize(2)
    gs, os_ = g.get_state(), o.get_state()
    assert g.counter() == o.get_counter() == 5
    assert np.max(np.abs(gs - os_)) < 1e-13
    assert np.max(np.abs(gs[..., 4:].reshape(-1, 6).sum(axis=0))) < 1e-11


def _totals(u):
    return np.array([math.fsum(u[..., L].ravel()) for L in range(4, 10)])


@pytest.mark.parametrize("ev,H,conserved", [(ONLYDIFF, 0.01, range(6)), (PV2, 0.0, range(6)),
                                            (PV2, 0.01, range(3, 6))])
def test_charge_conservation_long_run(lgv, ev, H, conserved):
    """The link heat bath conserves all six charges exactly (Stepper.cxx:508-517);
    the ideal step's advection is a lattice divergence, but its -H phi_l term
    (Stepper.cxx:131-132) sources the axial charges, so with H != 0 only the
    vector charges are conserved by the full step."""
    N = 16
    c = dict(COEF)
    c["H"] = H
    g = GpuLattice(lgv, N, **c)
    u = rand_state(N, 81)
    g.set_state(u)
    g.step(ev, 0.04, nsteps=50, inner=2, outer=3)
    d = _totals(g.get_state()) - _totals(u)
    assert np.max(np.abs(d[list(conserved)])) < 1e-10, d


def test_counter_continuity_and_determinism(lgv):
    N = 8
    u = rand_state(N, 91)
    a = GpuLattice(lgv, N, **COEF)
    a.set_state(u)
    a.step(PV2, 0.04, nsteps=4, inner=2, outer=3)
    b = GpuLattice(lgv, N, **COEF)
    b.set_state(u)
    b.step(PV2, 0.04, nsteps=2, inner=2, outer=3)
    b.step(PV2, 0.04, t=0.08, nsteps=2, inner=2, outer=3)
    assert a.counter() == b.counter()
    assert np.array_equal(a.get_state(), b.get_state())


def test_monitors_match_oracle_counts(lgv, oracle_mod):
    N = 8
    g, o = pair(lgv, oracle_mod, N, oracle_mod.INJECTED)
    u = rand_state(N, 101)
    g.set_state(u)
    o.set_state(u)
    g.mode(INJECTED)
    g.monitors(True)
    prop, acc = hb_noise(N, 102)
    g.inject_hb(prop, acc)
    o.inject_hb(prop, acc)
    g.step(HB, 0.01)
    o.step(HB, 0.01)
    order, q, acc2 = charge_noise(N, 103)
    g.inject_charge(order, q, acc2)
    o.inject_charge(order, q, acc2)
    g.step(CHARGE, 0.04)
    o.step(CHARGE, 0.04)
    gm = g.monitors()
    for w in (1, 2):
        om = o.monitor(w)
        for k in ("down_counts", "up_counts", "up_yes", "up_no"):
            assert gm[w][k] == om[k], (w, k)
        assert abs(gm[w]["down_dS"] - om["down_dS"]) < 1e-9 * max(1, abs(om["down_dS"]))
    assert gm[1]["down_counts"] + gm[1]["up_counts"] == N ** 3
    assert gm[2]["down_counts"] + gm[2]["up_counts"] == 6 * 6 * N ** 3 // 2


def test_injected_noise_required(lgv):
    from langevina_b200 import _lib as L

    g = GpuLattice(lgv, 4)
    g.mode(INJECTED)
    with pytest.raises(L.LgvError):
        g.step(HB, 0.01)


@pytest.mark.parametrize("N,mode", [(4, COUNTER), (8, INJECTED), (16, COUNTER), (34, COUNTER), (66, INJECTED)])
def test_phi_heatbath_fused_sweep_variant(lgv, oracle_mod, N, mode, monkeypatch):
    """The z-marching single-launch sweep (LGV_HB_FUSED=1) gives the oracle's
    result too: the same decisions from the same streams."""
    monkeypatch.setenv("LGV_HB_FUSED", "1")
    g, o = pair(lgv, oracle_mod, N, oracle_mod.INJECTED if mode else oracle_mod.COUNTER)
    monkeypatch.delenv("LGV_HB_FUSED")
    u = rand_state(N, 111 + N)
    g.set_state(u)
    o.set_state(u)
    g.flags(True)
    o.debug_flags(True)
    if mode == INJECTED:
        g.mode(INJECTED)
        prop, acc = hb_noise(N, 112)
        g.inject_hb(prop, acc)
        o.inject_hb(prop, acc)
        g.step(HB, 0.02)
        o.step(HB, 0.02)
    else:
        g.step(HB, 0.02, nsteps=3)
        o.step(HB, 0.02, nsteps=3)
    assert compare_flags(g.get_flags(), o.get_flags(), N ** 3) == 0
    assert_state_close(g.get_state(), o.get_state(), what="fused HB sweep")


@pytest.mark.parametrize("N,seed,fused", [(64, 15, True), (66, 16, True), (8, 17, True), (66, 18, False),
                                          (32, 20, True), (64, 23, False), (96, 24, True)])
def test_charge_heatbath_injected_segments_and_fused(lgv, oracle_mod, N, seed, fused, monkeypatch):
    """LGV_CHARGE_FUSED=1 runs both faces of a direction per launch and
    reproduces the oracle decision for decision: for N divisible by 32 the
    shared-memory slab kernel (x: whole rows; y, z: 32-site segments with
    two-site halos), otherwise x rows per CTA and y, z streamed in 32-site
    segments (66 leaves a ragged last segment).  The default single-face
    launches (fused=False) do too."""
    if fused:
        monkeypatch.setenv("LGV_CHARGE_FUSED", "1")
    g, o = pair(lgv, oracle_mod, N, oracle_mod.INJECTED)
    monkeypatch.delenv("LGV_CHARGE_FUSED", raising=False)
    u = rand_state(N, seed)
    g.set_state(u)
    o.set_state(u)
    g.mode(INJECTED)
    g.flags(True)
    o.debug_flags(True)
    g.monitors(True)
    order, q, acc = charge_noise(N, seed)
    g.inject_charge(order, q, acc)
    o.inject_charge(order, q, acc)
    g.step(CHARGE, 0.04)
    o.step(CHARGE, 0.04)
    assert compare_flags(g.get_flags(), o.get_flags(), 36 * N ** 3) == 0
    assert_state_close(g.get_state(), o.get_state(), what="charge HB segments")
    gm, om = g.monitors()[2], o.monitor(2)
    for k in ("down_counts", "up_counts", "up_yes", "up_no"):
        assert gm[k] == om[k], k


@pytest.mark.parametrize("N", [64, 70, 96, 160])
def test_charge_heatbath_counter_segments(lgv, oracle_mod, N, monkeypatch):
    """64, 96, 160: the slab kernel; 70: streamed lines with a ragged last segment."""
    monkeypatch.setenv("LGV_CHARGE_FUSED", "1")
    g, o = pair(lgv, oracle_mod, N, oracle_mod.COUNTER)
    monkeypatch.delenv("LGV_CHARGE_FUSED")
    u = rand_state(N, 19)
    g.set_state(u)
    o.set_state(u)
    g.step(CHARGE, 0.2, nsteps=2)
    o.step(CHARGE, 0.2, nsteps=2)
    assert_state_close(g.get_state(), o.get_state(), what="charge HB counter segments")


def test_stream_switch_keeps_order(lgv):
    """Work queued on the handle's stream finishes before a newly set stream
    touches the lattice (lgv_set_stream orders the two streams)."""
    import ctypes as C

    import torch

    N = 48
    u = rand_state(N, 131)
    a = GpuLattice(lgv, N, **COEF)
    a.set_state(u)
    a.step(PV2, 0.04, nsteps=30, inner=2, outer=3)
    want = a.get_state()
    b = GpuLattice(lgv, N, **COEF)
    b.set_state(u)
    b.step(PV2, 0.04, nsteps=30, inner=2, outer=3)  # queued on b's own stream, not synchronized
    s = torch.cuda.Stream()
    b.L.check(b.lib.lgv_set_stream(b.h, C.c_void_p(s.cuda_stream)), "set_stream")
    assert np.array_equal(b.get_state(), want)

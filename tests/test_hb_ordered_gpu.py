"""The ordered phi sweep (hb_ordered_kernel): one persistent launch runs whole
heat-bath sweeps (EulerLangevinHB::step, Stepper.cxx:287-389) slab by slab,
each odd-parity slab pass waiting on device counters for the three even-parity
slab passes it depends on.  It must give the oracle's result decision for
decision -- counter and injected noise, any slab thickness, chunk size and
schedule lag, one sweep or the two consecutive sweeps of PV2HBSplit23 fused
into one launch -- and bit for bit what the two one-parity launches give.

LGV_HB_ORDERED (read at lgv_create) selects it: "1,S,spc,lag,fuse" = on,
at most S planes per slab, spc sites per chunk, lag schedule rounds, fuse
sweeps per launch.  A bounded dependency wait that gives up is reported as
LGV_ERR_TIMEOUT by the handle's next synchronising call (LGV_WAIT_LIMIT=0
makes every wait give up at once; no wait can hang).
"""
import numpy as np
import pytest

from lgvtest import GpuLattice, assert_state_close, compare_flags, hb_noise, rand_state

pytestmark = pytest.mark.gpu

PV2, HB = 0, 4
COUNTER, INJECTED = 0, 1
COEF = dict(mass0=-4.813, lam=10.0, H=0.01, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=9182)

CONFIGS = ["1,1,128,1,2", "1,2,256,2,2", "1,4,1024,2,2", "1,8,512,3,3", "1,3,384,1,4"]


def make(lgv, oracle_mod, N, cfg, monkeypatch, mode_orc, **kw):
    c = dict(COEF)
    c.update(kw)
    monkeypatch.setenv("LGV_HB_ORDERED", cfg)
    g = GpuLattice(lgv, N, **c)
    monkeypatch.delenv("LGV_HB_ORDERED")
    o = oracle_mod.Oracle(N, mode=mode_orc, **c)
    return g, o


@pytest.mark.parametrize("N,cfg", [(4, CONFIGS[0]), (8, CONFIGS[1]), (16, CONFIGS[2]), (34, CONFIGS[3]),
                                   (48, CONFIGS[2]), (66, CONFIGS[4]), (24, CONFIGS[0])])
def test_ordered_sweep_counter(lgv, oracle_mod, N, cfg, monkeypatch):
    g, o = make(lgv, oracle_mod, N, cfg, monkeypatch, oracle_mod.COUNTER)
    u = rand_state(N, 7 + N)
    g.set_state(u)
    o.set_state(u)
    g.flags(True)
    o.debug_flags(True)
    g.step(HB, 0.02, nsteps=3)
    o.step(HB, 0.02, nsteps=3)
    assert compare_flags(g.get_flags(), o.get_flags(), N ** 3) == 0
    assert_state_close(g.get_state(), o.get_state(), what="ordered sweep")
    assert g.counter() == o.get_counter()


@pytest.mark.parametrize("N,cfg", [(8, CONFIGS[0]), (18, CONFIGS[1]), (40, CONFIGS[3])])
def test_ordered_sweep_injected(lgv, oracle_mod, N, cfg, monkeypatch):
    g, o = make(lgv, oracle_mod, N, cfg, monkeypatch, oracle_mod.INJECTED)
    u = rand_state(N, 70 + N)
    g.set_state(u)
    o.set_state(u)
    g.mode(INJECTED)
    g.flags(True)
    o.debug_flags(True)
    for sweep in range(2):
        prop, acc = hb_noise(N, 900 + sweep)
        g.inject_hb(prop, acc)
        o.inject_hb(prop, acc)
        g.step(HB, 0.03)
        o.step(HB, 0.03)
        assert compare_flags(g.get_flags(), o.get_flags(), N ** 3) == 0
    assert_state_close(g.get_state(), o.get_state(), what="ordered sweep injected")


@pytest.mark.parametrize("N,cfg,inner,outer", [(16, CONFIGS[1], 2, 3), (32, CONFIGS[2], 2, 3), (34, CONFIGS[4], 3, 1),
                                               (64, CONFIGS[3], 2, 3), (12, CONFIGS[0], 4, 2)])
def test_fused_sweeps_in_pv2hbsplit(lgv, oracle_mod, N, cfg, inner, outer, monkeypatch):
    """Consecutive sweeps of PV2HBSplit's inner loop share one launch; the
    accept statistics (o4_stepper_monitor) count every decision once."""
    g, o = make(lgv, oracle_mod, N, cfg, monkeypatch, oracle_mod.COUNTER)
    u = rand_state(N, 300 + N)
    g.set_state(u)
    o.set_state(u)
    g.monitors(True)
    g.step(PV2, 0.04, nsteps=2, inner=inner, outer=outer)
    o.step(PV2, 0.04, nsteps=2, inner=inner, outer=outer)
    assert_state_close(g.get_state(), o.get_state(), what="PV2HBSplit with fused sweeps")
    assert g.counter() == o.get_counter()
    mg = g.monitors()[1]
    mo = o.monitor(1)
    for k in ("down_counts", "up_counts", "up_yes", "up_no"):
        assert mg[k] == mo[k], k


@pytest.mark.parametrize("N,cfg", [(128, "1,4,512,3,2"), (130, "1,8,1024,2,1")])
def test_ordered_equals_two_passes(lgv, N, cfg, monkeypatch):
    """On the device alone: ordered sweeps (two per launch, or one) and the
    default two one-parity launches agree bit for bit."""
    u = rand_state(N, 5150)
    a = GpuLattice(lgv, N, **COEF)
    monkeypatch.setenv("LGV_HB_ORDERED", cfg)
    b = GpuLattice(lgv, N, **COEF)
    monkeypatch.delenv("LGV_HB_ORDERED")
    for g in (a, b):
        g.set_state(u)
        g.step(PV2, 0.04, nsteps=2, inner=2, outer=3)
    x, y = a.get_state(), b.get_state()
    a.close()
    b.close()
    assert np.array_equal(x, y)


def test_dependency_wait_gives_up_with_an_error(lgv, monkeypatch):
    """LGV_WAIT_LIMIT=0: every dependency wait and every TMA completion wait
    gives up at its first poll.  The step returns, the next synchronising call
    reports LGV_ERR_TIMEOUT, and the context stays usable."""
    from langevina_b200 import _lib as L

    N = 32
    monkeypatch.setenv("LGV_HB_ORDERED", "1,2,128,1,2")
    monkeypatch.setenv("LGV_WAIT_LIMIT", "0")
    g = GpuLattice(lgv, N, **COEF)
    monkeypatch.delenv("LGV_WAIT_LIMIT")
    g.set_state(rand_state(N, 1))
    g.step(PV2, 0.04, inner=2, outer=3)
    with pytest.raises(L.LgvError) as ei:
        g.get_state()
    assert ei.value.status == L.LGV_ERR_TIMEOUT
    assert "timed out" in str(ei.value)
    g.close()
    # a fresh handle with the default limit works on the same context
    h = GpuLattice(lgv, N, **COEF)
    monkeypatch.delenv("LGV_HB_ORDERED")
    u = rand_state(N, 2)
    h.set_state(u)
    h.step(PV2, 0.04, inner=2, outer=3)
    assert np.isfinite(h.get_state()).all()
    h.close()


def test_ensemble_wait_gives_up_with_an_error(lgv, monkeypatch):
    """An ensemble counts its own bounded waits: with LGV_WAIT_LIMIT=0 the TMA
    ideal step of its 32^3 replica gives up, and lgv_ensemble_synchronize and
    lgv_ensemble_get_state report LGV_ERR_TIMEOUT; a lattice handle created
    beside it with the default limit is not charged with the ensemble's
    timeouts."""
    import ctypes as C

    from langevina_b200 import _lib as L

    lib = L.load()
    arr = (L.lgv_params * 2)()
    for i, N in enumerate((32, 8)):
        arr[i] = L.make_params(N, mass0=-4.813, lam=10.0, H=0.003, chi=5.0, gamma=1.0, diffusion=1 / 3, seed=40 + i)
    e = C.c_void_p()
    monkeypatch.setenv("LGV_WAIT_LIMIT", "0")
    L.check(lib.lgv_ensemble_create(2, arr, C.byref(e)), "ensemble_create")
    monkeypatch.delenv("LGV_WAIT_LIMIT")
    g = GpuLattice(lgv, 32, **COEF)
    try:
        u = rand_state(32, 3)
        L.check(lib.lgv_ensemble_set_state(e, 0, L.ptr(u)), "set_state")
        L.check(lib.lgv_ensemble_step(e, IDEAL_PV2, 1, 1, 0.04, 0.0, 1), "step")
        assert lib.lgv_ensemble_synchronize(e) == L.LGV_ERR_TIMEOUT
        g.set_state(u)
        g.step(IDEAL_PV2, 0.04)
        assert np.isfinite(g.get_state()).all()
        L.check(lib.lgv_ensemble_step(e, IDEAL_PV2, 1, 1, 0.04, 0.0, 1), "step")
        out = np.empty_like(u)
        assert lib.lgv_ensemble_get_state(e, 0, L.ptr(out)) == L.LGV_ERR_TIMEOUT
    finally:
        g.close()
        lib.lgv_ensemble_destroy(e)


IDEAL_PV2 = 3

"""Batched ensembles (lgv_ensemble_*): every replica of a mixed ensemble
evolves like a lattice of its own (an lgv handle with the same params and
counter), for every packing order, ideal tile shape and z-chunk, with and
without CUDA-graph replay -- bit for bit through heat-bath, charge and
Euler-Maruyama steps, and to 1-2 ulp through the ideal step (the same device
code compiled into a second kernel; replicas with N divisible by 32 go
through the TMA kernel's CTA body, the others through the cp.async one); volume averages match the single-lattice
measurer; the autotuner restores state and counter."""
import ctypes as C

import numpy as np
import pytest

from lgvtest import GpuLattice, rand_state, site_rel_err

pytestmark = pytest.mark.gpu

PV2, HB, CHARGE, EM, IDEAL = 0, 4, 5, 6, 3


def make(lgv, specs):
    from langevina_b200 import _lib as L

    lib = L.load()
    arr = (L.lgv_params * len(specs))()
    for i, (N, seed, H) in enumerate(specs):
        arr[i] = L.make_params(N, mass0=-4.813, lam=10.0, H=H, chi=5.0, gamma=1.0, diffusion=1 / 3, seed=seed)
    e = C.c_void_p()
    L.check(lib.lgv_ensemble_create(len(specs), arr, C.byref(e)), "ensemble_create")
    return L, lib, e


# 32 takes the TMA ideal kernel, the other sizes the cp.async one, in the same step
SPECS = [(8, 11, 0.003), (6, 12, 0.006), (16, 13, 0.012), (8, 14, 0.003), (34, 15, 0.006), (4, 16, 0.012),
         (32, 17, 0.003)]


def singles(lgv, specs, states, plan):
    out = []
    for (N, seed, H), u in zip(specs, states):
        g = GpuLattice(lgv, N, mass0=-4.813, lam=10.0, H=H, chi=5.0, gamma=1.0, diffusion=1 / 3, seed=seed)
        g.set_state(u)
        for ev, dt, t, n in plan:
            g.step(ev, dt, t=t, nsteps=n, inner=2, outer=3)
        out.append(g.get_state())
    return out


@pytest.mark.parametrize("tile,zchunk,order,graphs", [(0, 16, 0, 1), (1, 8, 1, 1), (0, 32, 2, 0), (1, 16, 2, 1)])
def test_replicas_match_single_lattices(lgv, tile, zchunk, order, graphs):
    L, lib, e = make(lgv, SPECS)
    try:
        L.check(lib.lgv_ensemble_tune(e, tile, zchunk, order), "tune")
        L.check(lib.lgv_ensemble_use_graphs(e, graphs), "graphs")
        states = [rand_state(N, 100 + i) for i, (N, _, _) in enumerate(SPECS)]
        for r, u in enumerate(states):
            L.check(lib.lgv_ensemble_set_state(e, r, L.ptr(u)), "set_state")
        plan = [(PV2, 0.04, 0.0, 5), (EM, 0.01, 0.2, 3), (PV2, 0.04, 0.3, 2), (CHARGE, 0.1, 0.0, 1), (HB, 0.02, 0.0, 2)]
        for ev, dt, t, n in plan:
            L.check(lib.lgv_ensemble_step(e, ev, 2, 3, dt, t, n), "ensemble_step")
        want = singles(lgv, SPECS, states, plan)
        for r, w in enumerate(want):
            got = np.empty_like(w)
            L.check(lib.lgv_ensemble_get_state(e, r, L.ptr(got)), "get_state")
            assert site_rel_err(got, w) <= 1e-13, f"replica {r}: max diff {np.max(np.abs(got - w)):.3e}"
        c = C.c_uint64()
        L.check(lib.lgv_ensemble_get_counter(e, C.byref(c)), "counter")
        assert c.value == 5 * 13 + 3 + 2 * 13 + 7 + 2
    finally:
        lib.lgv_ensemble_destroy(e)


def test_initialize_and_oaverage_match_single_lattices(lgv):
    L, lib, e = make(lgv, SPECS)
    try:
        L.check(lib.lgv_ensemble_initialize(e, 1, 0.1), "init phi")
        L.check(lib.lgv_ensemble_initialize(e, 2, 0.0), "init charges")
        L.check(lib.lgv_ensemble_step(e, PV2, 2, 3, 0.04, 0.0, 4), "step")
        oav = np.zeros((len(SPECS), 11))
        L.check(lib.lgv_ensemble_oaverage(e, L.ptr(oav)), "oaverage")
        for r, (N, seed, H) in enumerate(SPECS):
            g = GpuLattice(lgv, N, mass0=-4.813, lam=10.0, H=H, chi=5.0, gamma=1.0, diffusion=1 / 3, seed=seed)
            g.initialize(1, 0.1)
            g.initialize(2)
            g.step(PV2, 0.04, nsteps=4, inner=2, outer=3)
            got = np.empty((N, N, N, 10))
            L.check(lib.lgv_ensemble_get_state(e, r, L.ptr(got)), "get_state")
            assert site_rel_err(got, g.get_state()) <= 1e-13
            m = g.measure().OAverage
            assert np.allclose(oav[r], m, rtol=1e-12, atol=1e-14)
    finally:
        lib.lgv_ensemble_destroy(e)


def test_autotune_restores_state_and_counter(lgv):
    L, lib, e = make(lgv, SPECS[:4])
    try:
        states = [rand_state(N, 200 + i) for i, (N, _, _) in enumerate(SPECS[:4])]
        for r, u in enumerate(states):
            L.check(lib.lgv_ensemble_set_state(e, r, L.ptr(u)), "set_state")
        L.check(lib.lgv_ensemble_set_counter(e, 17), "set_counter")
        choice = (C.c_int * 3)()
        ms = C.c_double()
        L.check(lib.lgv_ensemble_autotune(e, PV2, 2, 3, 0.04, 2, choice, C.byref(ms)), "autotune")
        assert choice[0] in (0, 1) and choice[1] in (8, 16, 32) and choice[2] in (0, 1, 2) and ms.value > 0
        c = C.c_uint64()
        L.check(lib.lgv_ensemble_get_counter(e, C.byref(c)), "counter")
        assert c.value == 17
        for r, u in enumerate(states):
            got = np.empty_like(u)
            L.check(lib.lgv_ensemble_get_state(e, r, L.ptr(got)), "get_state")
            assert np.array_equal(got, u)
    finally:
        lib.lgv_ensemble_destroy(e)


@pytest.mark.parametrize("ev,dt", [(HB, 0.02), (CHARGE, 0.1), (EM, 0.01)])
def test_noisy_substeps_are_bit_exact(lgv, ev, dt):
    L, lib, e = make(lgv, SPECS)
    try:
        states = [rand_state(N, 300 + i) for i, (N, _, _) in enumerate(SPECS)]
        for r, u in enumerate(states):
            L.check(lib.lgv_ensemble_set_state(e, r, L.ptr(u)), "set_state")
        L.check(lib.lgv_ensemble_step(e, ev, 1, 1, dt, 0.0, 3), "step")
        want = singles(lgv, SPECS, states, [(ev, dt, 0.0, 3)])
        for r, w in enumerate(want):
            got = np.empty_like(w)
            L.check(lib.lgv_ensemble_get_state(e, r, L.ptr(got)), "get_state")
            assert np.array_equal(got, w)
    finally:
        lib.lgv_ensemble_destroy(e)


def test_graphs_replay_on_the_legacy_default_stream(lgv):
    """A caller's stream that cannot be captured (the legacy default stream,
    passed as NULL) still gets graph replay: the ensemble captures on its own
    stream and launches the graph on the caller's."""
    specs = SPECS[:4]
    states = [rand_state(N, 400 + i) for i, (N, _, _) in enumerate(specs)]
    got = []
    for stream in (None, 0):
        L, lib, e = make(lgv, specs)
        try:
            L.check(lib.lgv_ensemble_use_graphs(e, 1), "graphs")
            if stream is not None:
                L.check(lib.lgv_ensemble_set_stream(e, C.c_void_p(stream)), "set_stream")
            for r, u in enumerate(states):
                L.check(lib.lgv_ensemble_set_state(e, r, L.ptr(u)), "set_state")
            L.check(lib.lgv_ensemble_step(e, PV2, 2, 3, 0.04, 0.0, 4), "step")
            L.check(lib.lgv_ensemble_step(e, HB, 1, 1, 0.02, 0.0, 3), "step")
            L.check(lib.lgv_ensemble_synchronize(e), "sync")
            out = []
            for r, u in enumerate(states):
                g = np.empty_like(u)
                L.check(lib.lgv_ensemble_get_state(e, r, L.ptr(g)), "get_state")
                out.append(g)
            got.append(out)
        finally:
            lib.lgv_ensemble_destroy(e)
    for a, b in zip(*got):
        assert np.array_equal(a, b)

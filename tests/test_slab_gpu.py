"""Lattices split into z-slabs (lgv_slab_*, langevina_b200.slab).

R ranks, emulated as host threads of one process on one GPU (ThreadHalo: the
boundary planes move between the slabs' buffers by device copies at host
barriers, so no kernel waits on another), each hold planes k0 .. k0+nz-1 and
two ghost planes per side.  Because the counter noise is indexed by the global
site and every sub-pass that reads across planes first refreshes the ghosts
(as the reference's DMGlobalToLocal does before every pass,
Stepper.cxx:81-82, 312-315, 477-480), the gathered slabs must equal one
handle holding the whole lattice bit for bit -- PV2HBSplit23 and {1,1}, the
sub-steppers alone and Euler-Maruyama, for the TMA (N divisible by 32) and
cp.async ideal kernels, one to four ranks -- and the per-rank measurement
partials must combine into the whole lattice's measurement.
"""
import ctypes as C

import numpy as np
import pytest

from lgvtest import GpuLattice, rand_state

pytestmark = pytest.mark.gpu

PV2, IDEAL, HB, CHARGE, EM = 0, 3, 4, 5, 6
COEF = dict(mass0=-4.813, lam=10.0, H=0.01, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=51515)


def run_slabs(N, R, u, plan, coef=COEF):
    from langevina_b200 import slab as S

    halo = S.ThreadHalo(R)
    slabs = [S.SlabLattice(N, k0, nz, halo, rank=r, **coef) for r, (k0, nz) in enumerate(S.slab_planes(N, R))]
    for s in slabs:
        halo.attach(s)
        s.set_global_state(u)

    def go(s):
        for ev, dt, n, inner, outer in plan:
            s.step(ev, dt, nsteps=n, inner=inner, outer=outer)

    S.run_threads(slabs, go)
    out = np.concatenate([s.get_interior() for s in slabs], axis=0)
    return slabs, out


def run_whole(N, u, plan, coef=COEF):
    g = GpuLattice(None, N, **coef)
    g.set_state(u)
    for ev, dt, n, inner, outer in plan:
        g.step(ev, dt, nsteps=n, inner=inner, outer=outer)
    return g


@pytest.mark.parametrize("N,R", [(32, 1), (32, 2), (32, 4), (48, 3), (64, 2), (20, 2), (34, 4)])
def test_slabs_equal_whole_lattice_pv2hbsplit23(lgv, N, R):
    u = rand_state(N, 600 + N + R)
    plan = [(PV2, 0.04, 2, 2, 3)]
    slabs, got = run_slabs(N, R, u, plan)
    g = run_whole(N, u, plan)
    want = g.get_state()
    assert np.array_equal(got, want)
    assert all(int(_counter(s)) == g.counter() for s in slabs)
    for s in slabs:
        s.close()
    g.close()


@pytest.mark.parametrize("plan", [
    [(PV2, 0.04, 2, 1, 1)],
    [(IDEAL, 0.05, 2, 1, 1), (HB, 0.02, 2, 1, 1), (CHARGE, 0.04, 2, 1, 1)],
    [(EM, 0.02, 3, 1, 1)],
])
def test_slabs_equal_whole_lattice_substeps(lgv, plan):
    N, R = 32, 2
    u = rand_state(N, 777)
    slabs, got = run_slabs(N, R, u, plan)
    g = run_whole(N, u, plan)
    assert np.array_equal(got, g.get_state())
    for s in slabs:
        s.close()
    g.close()


class DownHalo:
    def exchange(self, slab, comps):
        raise OSError("neighbour unreachable")


def _counter(s):
    v = C.c_uint64()
    s.lib.lgv_get_counter(s.h, C.byref(v))
    return v.value


def test_measurement_from_slab_partials(lgv):
    import torch

    from langevina_b200 import _lib as L
    from langevina_b200 import slab as S

    N, R = 32, 4
    u = rand_state(N, 4242)
    slabs, _ = run_slabs(N, R, u, [(PV2, 0.04, 1, 2, 3)])
    T = torch.zeros(S.NOBS * N * N, dtype=torch.float64, device="cuda")
    U = torch.zeros(S.NOBS * N * N, dtype=torch.float64, device="cuda")
    for s in slabs:
        Ur = torch.zeros_like(U)
        s.measure_partials(T, Ur)
        U += Ur
    out = torch.empty(int(L.load().lgv_measure_size(N)), dtype=torch.float64, device="cuda")
    S.measure_from_partials(T, U, N, out)
    torch.cuda.synchronize()
    g = run_whole(N, u, [(PV2, 0.04, 1, 2, 3)])
    want = torch.empty_like(out)
    L.check(g.lib.lgv_measure_device(g.h, C.c_void_p(want.data_ptr())), "measure")
    L.check(g.lib.lgv_synchronize(g.h), "sync")
    d = (out - want).abs().max().item()
    assert d <= 1e-12 * max(1.0, want.abs().max().item()), d
    for s in slabs:
        s.close()
    g.close()


def test_slab_refuses_what_it_cannot_do(lgv):
    from langevina_b200 import _lib as L
    from langevina_b200 import slab as S

    lib = L.load()
    p = L.make_params(16, **COEF)
    h = C.c_void_p()
    assert lib.lgv_slab_create(C.byref(p), 1, 4, C.byref(h)) == L.LGV_ERR_INVALID   # odd k0
    assert lib.lgv_slab_create(C.byref(p), 0, 3, C.byref(h)) == L.LGV_ERR_INVALID   # odd nz
    assert lib.lgv_slab_create(C.byref(p), 14, 4, C.byref(h)) == L.LGV_ERR_INVALID  # past N
    s = S.SlabLattice(16, 0, 8, halo=None, **COEF)
    try:
        assert lib.lgv_initialize(s.h, 1, 0.1) == L.LGV_ERR_UNSUPPORTED
        assert lib.lgv_set_noise_mode(s.h, 1) == L.LGV_ERR_UNSUPPORTED
        assert lib.lgv_enable_monitors(s.h, 1) == L.LGV_ERR_UNSUPPORTED
        out = np.empty(16)
        assert lib.lgv_measure_device(s.h, C.c_void_p(out.ctypes.data)) == L.LGV_ERR_UNSUPPORTED
        # an exchange that fails: the step stops at its first cross-plane pass, before any launch
        s.halo = DownHalo()
        with pytest.raises(RuntimeError):
            s.step(PV2, 0.04, inner=2, outer=3)
    finally:
        s.close()

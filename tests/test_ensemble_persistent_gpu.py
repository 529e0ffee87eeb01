"""The persistent ensemble step (lgv_ensemble_use_persistent): one cooperative
launch per step runs every sub-step over all replicas, phases separated by a
grid barrier.  It must leave every replica bit for bit where the default one
launch per sub-step leaves it -- PV2HBSplit with (2, 3) and (1, 1), the
NoDiffuse / OnlyDiffuse variants and the sub-steppers alone, with and without
CUDA-graph replay, for both cp.async tile shapes and every packing, on a mix
of TMA (N divisible by 32) and cp.async replicas -- with the same counter; an
Euler-Maruyama step falls back to its own launch; and a grid barrier whose
waits are cut to nothing reports LGV_ERR_TIMEOUT and leaves the context
usable."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from lgvtest import rand_state

pytestmark = pytest.mark.gpu

PV2, PV2_NODIFF, PV2_ONLYDIFF, IDEAL, HB, CHARGE, EM = 0, 1, 2, 3, 4, 5, 6

SPECS = [(8, 11, 0.003), (6, 12, 0.006), (16, 13, 0.012), (32, 17, 0.003), (34, 15, 0.006), (4, 16, 0.012),
         (64, 18, 0.006), (32, 19, 0.012)]


def make(specs):
    from langevina_b200 import _lib as L

    lib = L.load()
    arr = (L.lgv_params * len(specs))()
    for i, (N, seed, H) in enumerate(specs):
        arr[i] = L.make_params(N, mass0=-4.813, lam=10.0, H=H, chi=5.0, gamma=1.0, diffusion=1 / 3, seed=seed)
    e = C.c_void_p()
    L.check(lib.lgv_ensemble_create(len(specs), arr, C.byref(e)), "ensemble_create")
    return L, lib, e


def run(persistent, plan, tile=0, zchunk=16, order=0, graphs=1, inner=2, outer=3):
    L, lib, e = make(SPECS)
    try:
        L.check(lib.lgv_ensemble_tune(e, tile, zchunk, order), "tune")
        L.check(lib.lgv_ensemble_use_graphs(e, graphs), "graphs")
        L.check(lib.lgv_ensemble_use_persistent(e, persistent), "persistent")
        states = [rand_state(N, 300 + r) for r, (N, _, _) in enumerate(SPECS)]  # alive through the copies
        for r, u in enumerate(states):
            L.check(lib.lgv_ensemble_set_state(e, r, L.ptr(u)), "set_state")
        for ev, dt, t, n in plan:
            L.check(lib.lgv_ensemble_step(e, ev, inner, outer, dt, t, n), "ensemble_step")
        out = []
        for r, (N, _, _) in enumerate(SPECS):
            u = np.empty((N, N, N, 10))
            L.check(lib.lgv_ensemble_get_state(e, r, L.ptr(u)), "get_state")
            out.append(u)
        c = C.c_uint64()
        L.check(lib.lgv_ensemble_get_counter(e, C.byref(c)), "counter")
        return out, c.value
    finally:
        lib.lgv_ensemble_destroy(e)


@pytest.mark.parametrize("tile,zchunk,order,graphs", [(0, 16, 0, 1), (1, 8, 1, 1), (0, 32, 2, 0), (1, 16, 2, 0)])
def test_persistent_equals_one_launch_per_substep(lgv, tile, zchunk, order, graphs):
    plan = [(PV2, 0.04, 0.0, 5), (PV2, 0.04, 0.3, 2), (EM, 0.01, 0.2, 3), (CHARGE, 0.1, 0.0, 1), (HB, 0.02, 0.0, 2),
            (IDEAL, 0.05, 0.0, 3), (PV2_NODIFF, 0.04, 0.0, 2), (PV2_ONLYDIFF, 0.04, 0.0, 3)]
    want, cw = run(0, plan, tile, zchunk, order, graphs)
    got, cg = run(1, plan, tile, zchunk, order, graphs)
    assert cg == cw
    for r, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"replica {r} (N={SPECS[r][0]}): max diff {np.max(np.abs(a - b)):.3e}"


def test_persistent_scounts_11(lgv):
    plan = [(PV2, 0.04, 0.0, 4)]
    want, cw = run(0, plan, inner=1, outer=1)
    got, cg = run(1, plan, inner=1, outer=1)
    assert cg == cw
    assert all(np.array_equal(a, b) for a, b in zip(got, want))


_TIMEOUT_CHILD = r"""
import ctypes as C, sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import numpy as np
from lgvtest import rand_state
from langevina_b200 import _lib as L
lib = L.load()
specs = [(32, 1), (16, 2)]
arr = (L.lgv_params * 2)()
for i, (N, seed) in enumerate(specs):
    arr[i] = L.make_params(N, seed=seed)
e = C.c_void_p()
L.check(lib.lgv_ensemble_create(2, arr, C.byref(e)), "create")
L.check(lib.lgv_ensemble_use_persistent(e, 1), "persistent")
L.check(lib.lgv_ensemble_use_graphs(e, 0), "graphs")
states = [rand_state(N, 5 + r) for r, (N, _) in enumerate(specs)]
for r, u in enumerate(states):
    L.check(lib.lgv_ensemble_set_state(e, r, L.ptr(u)), "set")
rc1 = lib.lgv_ensemble_step(e, 0, 2, 3, 0.04, 0.0, 1)
rc2 = lib.lgv_ensemble_synchronize(e)
# the context is still usable: a single lattice steps and syncs
p = L.make_params(16, seed=3)
h = C.c_void_p()
L.check(lib.lgv_create(C.byref(p), C.byref(h)), "create single")
L.check(lib.lgv_initialize(h, 1, 0.1), "init")
L.check(lib.lgv_step(h, 0, 1, 1, 0.04, 0.0, 1), "single step")
rc3 = lib.lgv_synchronize(h)
print("RC", rc1, rc2, rc3, L.LGV_ERR_TIMEOUT)
"""


def test_barrier_wait_limit_reports_timeout(lgv):
    """LGV_WAIT_LIMIT=0: every grid-barrier wait (and TMA wait) gives up at once;
    the step's launch ends, the next synchronising call reports the timeout,
    and the context keeps working.  Run in a child so the limit stays local."""
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, LGV_WAIT_LIMIT="0")
    r = subprocess.run([sys.executable, "-c", _TIMEOUT_CHILD, repo], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("RC")][-1].split()
    rc1, rc2, rc3, tmo = map(int, line[1:])
    assert rc1 == 0
    assert rc2 == tmo
    assert rc3 == 0

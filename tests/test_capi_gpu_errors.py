"""Allocation failures through the C ABI: a lattice larger than the device's
memory (N = 2048, 1.4 TB for the two buffers) is refused with
LGV_ERR_NOMEM and no handle, and the failure does not leak into later calls
-- a lattice created next initialises, steps, measures and synchronises with
LGV_OK.  The same for an ensemble with one oversized replica."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_oversized_lattice_is_refused_and_the_next_one_works(lgv):
    from langevina_b200 import _lib as L

    lib = L.load()
    big = L.make_params(2048)
    h = C.c_void_p()
    assert lib.lgv_create(C.byref(big), C.byref(h)) == L.LGV_ERR_NOMEM
    assert not h.value
    assert b"cudaMalloc" in lib.lgv_last_error()

    p = L.make_params(16, seed=5)
    g = C.c_void_p()
    L.check(lib.lgv_create(C.byref(p), C.byref(g)), "create after a refused one")
    try:
        L.check(lib.lgv_initialize(g, L.INIT_PHI_GAUSSIAN, 0.1), "init")
        L.check(lib.lgv_step(g, L.PV2HBSPLIT, 2, 3, 0.04, 0.0, 2), "step")
        import torch

        m = torch.empty(int(lib.lgv_measure_size(16)), dtype=torch.float64, device="cuda")
        L.check(lib.lgv_measure_device(g, C.c_void_p(m.data_ptr())), "measure")
        assert lib.lgv_synchronize(g) == L.LGV_OK
        assert np.isfinite(m.cpu().numpy()).all()
    finally:
        lib.lgv_destroy(g)


def test_oversized_replica_refuses_the_ensemble(lgv):
    from langevina_b200 import _lib as L

    lib = L.load()
    arr = (L.lgv_params * 2)()
    arr[0] = L.make_params(16, seed=1)
    arr[1] = L.make_params(2048, seed=2)
    e = C.c_void_p()
    assert lib.lgv_ensemble_create(2, arr, C.byref(e)) == L.LGV_ERR_NOMEM
    arr[1] = L.make_params(8, seed=2)
    L.check(lib.lgv_ensemble_create(2, arr, C.byref(e)), "ensemble after a refused one")
    try:
        L.check(lib.lgv_ensemble_initialize(e, L.INIT_PHI_GAUSSIAN, 0.1), "init")
        L.check(lib.lgv_ensemble_step(e, L.PV2HBSPLIT, 2, 3, 0.04, 0.0, 2), "step")
        assert lib.lgv_ensemble_synchronize(e) == L.LGV_OK
    finally:
        lib.lgv_ensemble_destroy(e)

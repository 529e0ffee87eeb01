"""The C-ABI library loads and exports every entry point include/lgv.h declares.

No call here touches a GPU: only pure host helpers and argument validation
(which runs before any CUDA call) are exercised.
"""
import ctypes as C
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in sorted(os.listdir(os.path.join(REPO, "include"))):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(REPO, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(lgv_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    d = declared()
    assert "lgv_step" in d and "lgv_measure" in d and len(d) >= 25


def test_library_exports_every_declared_symbol():
    from langevina_b200 import _lib

    lib = _lib.load()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(declared()) <= bound, set(declared()) - bound


def test_host_only_helpers():
    from langevina_b200 import _lib

    lib = _lib.load()
    assert lib.lgv_version() >= 10000
    assert lib.lgv_status_string(0) == b"ok"
    assert lib.lgv_status_string(-1) == b"invalid argument"
    N = 32
    assert lib.lgv_measure_size(N) == 11 + 75 * N + 234 * (N // 2 + 1)


@pytest.mark.parametrize("N", [3, 5, 2, 0, -4])
def test_create_rejects_bad_lattice_before_touching_the_device(N):
    from langevina_b200 import _lib

    lib = _lib.load()
    p = _lib.make_params(8)
    p.N = N
    h = C.c_void_p()
    assert lib.lgv_create(C.byref(p), C.byref(h)) == -1
    assert b"N=" in lib.lgv_last_error()
    assert not h.value


def test_create_rejects_bad_coefficients():
    from langevina_b200 import _lib

    lib = _lib.load()
    for field, bad in (("chi", 0.0), ("LX", -1.0), ("reserved0", 1)):
        p = _lib.make_params(8)
        setattr(p, field, bad)
        h = C.c_void_p()
        assert lib.lgv_create(C.byref(p), C.byref(h)) == -1


def test_postprocess_argument_checks_need_no_gpu():
    """Argument validation of the post-processing entry points runs before any
    CUDA call (the dummy pointers are never dereferenced)."""
    from langevina_b200 import _lib

    lib = _lib.load()
    d = C.c_void_p(16)
    inv = _lib.LGV_ERR_INVALID
    assert lib.lgv_x2k(None, 1, 8, d, None) == inv
    assert lib.lgv_x2k(d, 1, 7, d, None) == inv  # odd N
    assert lib.lgv_x2k(d, 0, 8, d, None) == _lib.LGV_OK  # nothing to do
    assert lib.lgv_x2k_rotated(d, 1, 9, 5, d, None) == inv  # fewer than 10 fields
    assert lib.lgv_time_correlator(d, d, 10, 2, 2, 0, 11, 1, 0, d, None) == inv  # ntmax > T
    assert lib.lgv_time_correlator(d, d, 10, 2, 3, 1, 5, 1, 0, d, None) == inv  # ld below 2 * nseries
    assert lib.lgv_time_correlator(d, d, 10, 2, 2, 0, 5, 0, 0, d, None) == inv  # decim 0

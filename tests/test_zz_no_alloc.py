"""The allocation-free measurement entry point, lgv_measure_aos_noalloc.

Some hosts cannot allocate device memory of their own once they are running:
their GPU memory belongs to another allocator (a framework's caching pool that
has reserved most of the device, so a stray cudaMalloc can fail even though the
pool has room), or they run under a fixed device-memory budget.  For them the
library measures a lattice they hold in device memory using only a static
scratch array compiled into liblgv.so.  This test calls that entry point
through the C ABI twice in a row -- on two different lattices, so stale scratch
contents from the first call would show up in the second -- and compares each
result with the handle-based lgv_measure at the tolerance of the other
measurement tests.  It also checks the size limit is enforced.
"""
import ctypes as C

import numpy as np
import pytest

from lgvtest import GpuLattice, rand_state

pytestmark = pytest.mark.gpu

COEF = dict(mass0=-4.813, lam=10.0, H=0.01, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=7)


def unpack(buf, N):
    """Split a packed lgv_measure_device/noalloc buffer into named arrays."""
    NK = N // 2 + 1
    out, p = {}, 0

    def take(name, shape):
        nonlocal p
        n = int(np.prod(shape))
        out[name] = buf[p:p + n].reshape(shape)
        p += n

    take("OAverage", (11,))
    for ax in "XYZ":
        take(f"wall{ax}", (11, N))
    for ax in "XYZ":
        take(f"wall{ax}_k", (11, NK, 2))
    for ax in "XYZ":
        take(f"wall{ax}_k_rotated", (14, NK, 2))
    for ax in "XYZ":
        take(f"wall{ax}Phase", (14, N))
    for ax in "XYZ":
        take(f"wall{ax}Phase_k", (14, NK, 2))
    assert p == buf.size
    return out


@pytest.mark.parametrize("N", [32, 128])
def test_measure_noalloc_matches_measure_on_two_calls(lgv, N):
    """N = 32, and N = LGV_NOALLOC_MAX_N = 128, where the two partial-sum
    tables fill the static array to its last element."""
    import torch

    from langevina_b200 import _lib as L

    lib = L.load()
    assert N <= L.NOALLOC_MAX_N
    torch.cuda.set_device(0)
    out = torch.empty(int(lib.lgv_measure_size(N)), dtype=torch.float64, device="cuda")
    for call, seed in enumerate((401, 402)):
        u = rand_state(N, seed)
        u[..., 0] += 0.2 * (call + 1)
        g = GpuLattice(lgv, N, **COEF)
        g.set_state(u)
        want = g.measure().arrays()
        g.close()
        dev_aos = torch.from_numpy(np.ascontiguousarray(u).reshape(-1)).to("cuda")
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = lib.lgv_measure_aos_noalloc(C.c_void_p(dev_aos.data_ptr()), N, C.c_void_p(out.data_ptr()), None)
        assert rc == 0, lib.lgv_last_error()
        torch.cuda.synchronize()
        got = unpack(out.cpu().numpy(), N)
        for k, w in want.items():
            d = np.max(np.abs(got[k] - w))
            assert d <= 1e-13 * max(1.0, np.max(np.abs(w))), f"call {call}: {k} differs by {d:.3e}"


def test_measure_noalloc_rejects_sizes_beyond_its_scratch(lgv):
    import torch

    from langevina_b200 import _lib as L

    lib = L.load()
    big = L.NOALLOC_MAX_N + 2
    dummy = torch.empty(16, dtype=torch.float64, device="cuda")
    rc = lib.lgv_measure_aos_noalloc(C.c_void_p(dummy.data_ptr()), big, C.c_void_p(dummy.data_ptr()), None)
    assert rc == -1
    assert b"LGV_NOALLOC_MAX_N" in lib.lgv_last_error()
    rc = lib.lgv_measure_aos_noalloc(C.c_void_p(dummy.data_ptr()), 7, C.c_void_p(dummy.data_ptr()), None)
    assert rc == -1

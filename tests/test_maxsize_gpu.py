"""A 512^3 lattice (134 M sites, 10.7 GB per state; about 64 GB of device
memory for the two handles below), eight times the bench's size.  The oracle
is too slow here, so two independent implementations of the same step are set
against each other on the device:

- the default kernels (phi heat bath as two parity passes on the row grid,
  charge heat bath one face per launch);
- LGV_HB_FUSED=1 and LGV_CHARGE_FUSED=1 (one z-marching launch per phi sweep
  with its ring recomputed, and the shared-memory slab kernel doing both faces
  of a direction per launch).

Both draw the same counter streams, so after a PV2HBSplit23 step from the same
initial state the lattices agree per site to 1e-12, and the total vector
charge is conserved.  Comparisons run on the device (no 10 GB host copies).
"""
import ctypes as C

import pytest

from lgvtest import GpuLattice

pytestmark = pytest.mark.gpu

N = 512
PV2 = 0
COEF = dict(mass0=-4.813, lam=10.0, H=0.003, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=512)


def device_state(g, torch):
    u = torch.empty((N, N, N, 10), dtype=torch.float64, device="cuda")
    # the handle writes on its own stream: let torch's pending work on memory
    # the allocator may hand out again finish first
    torch.cuda.synchronize()
    g.L.check(g.lib.lgv_get_state_device(g.h, C.c_void_p(u.data_ptr())), "get_state_device")
    g.L.check(g.lib.lgv_synchronize(g.h), "synchronize")
    return u


def test_two_implementations_agree_at_512(lgv, monkeypatch):
    import torch

    lattices = []
    for fused in (False, True):
        if fused:
            monkeypatch.setenv("LGV_HB_FUSED", "1")
            monkeypatch.setenv("LGV_CHARGE_FUSED", "1")
        g = GpuLattice(lgv, N, **COEF)
        monkeypatch.delenv("LGV_HB_FUSED", raising=False)
        monkeypatch.delenv("LGV_CHARGE_FUSED", raising=False)
        g.initialize(1, 0.3)
        g.initialize(2)
        lattices.append(g)
    u0 = device_state(lattices[0], torch)
    v0 = u0[..., 7:10].sum(dim=(0, 1, 2))
    for g in lattices:
        g.step(PV2, 0.04, t=0.0, inner=2, outer=3)
    assert lattices[0].counter() == lattices[1].counter() == 13 + 2
    a = device_state(lattices[0], torch)
    lattices[0].close()
    dv = (a[..., 7:10] - u0[..., 7:10]).sum(dim=(0, 1, 2)).tolist()
    v0 = v0.tolist()
    del u0
    b = device_state(lattices[1], torch)
    lattices[1].close()
    worst = 0.0
    for lo, hi in ((0, 4), (4, 7), (7, 10)):
        d = (a[..., lo:hi] - b[..., lo:hi]).abs().amax(dim=-1)
        s = b[..., lo:hi].abs().amax(dim=-1).clamp_min(1e-6)
        worst = max(worst, float((d / s).max()))
        del d, s
    assert worst <= 1e-12, f"per-site relative difference {worst:.3e}"
    assert max(abs(x) for x in dv) < 1e-8, f"vector charge moved by {dv} (total {v0})"

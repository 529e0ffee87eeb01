"""The z-slab halo exchange over torch.distributed (langevina_b200.slab.DistHalo)
on CPU: two and three gloo ranks, each with a stand-in slab whose planes are
numpy arrays (the exchange treats the packed buffers as opaque), must end with
the two ghost planes below holding the global planes k0-2, k0-1 of the rank
below and the two above holding k0+nz, k0+nz+1 of the rank above (periodic),
only for the component groups asked for; and the plane split must give every
rank an even number of planes >= 2.  The lgv slab kernels themselves are
checked on the GPU against one whole-lattice handle (tests/test_slab_gpu.py).
"""
import os
import socket
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

N = 12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def global_lattice():
    # value = 1000 * global plane + 10 * component + a site pattern
    k = np.arange(N)[:, None, None, None]
    c = np.arange(10)[None, None, None, :]
    site = (np.arange(N)[None, :, None, None] * N + np.arange(N)[None, None, :, None]) / 1e4
    return 1000.0 * k + 10.0 * c + site


class HostSlab:
    """A slab whose box (nz + 4 planes, ghosts included) is a numpy array."""

    def __init__(self, k0, nz, u):
        self.k0, self.nz = k0, nz
        self.box = np.full((nz + 4, N, N, 10), np.nan)
        self.box[2:2 + nz] = u[k0:k0 + nz]

    @staticmethod
    def _cols(comps):
        return ([0, 1, 2, 3] if comps & 1 else []) + ([4, 5, 6, 7, 8, 9] if comps & 2 else [])

    def halo_doubles(self, comps):
        return 2 * N * N * len(self._cols(comps))

    def pack(self, side, comps, buf):
        import torch

        planes = self.box[2:4] if side == 0 else self.box[self.nz:self.nz + 2]
        buf.copy_(torch.from_numpy(np.ascontiguousarray(planes[..., self._cols(comps)]).ravel()))

    def unpack(self, side, comps, buf):
        cols = self._cols(comps)
        vals = buf.numpy().reshape(2, N, N, len(cols))
        target = slice(0, 2) if side == 0 else slice(self.nz + 2, self.nz + 4)
        self.box[target][..., cols] = vals

    def sync(self):
        pass


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from langevina_b200 import slab as S

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        u = global_lattice()
        k0, nz = S.slab_planes(N, world)[rank]
        s = HostSlab(k0, nz, u)
        halo = S.DistHalo(dist, staging="device", device="cpu")
        halo.exchange(s, 1)  # phi only
        phi_ok = (np.array_equal(s.box[0:2, ..., :4], u[[(k0 - 2) % N, (k0 - 1) % N]][..., :4])
                  and np.array_equal(s.box[nz + 2:, ..., :4], u[[(k0 + nz) % N, (k0 + nz + 1) % N]][..., :4])
                  and np.isnan(s.box[0:2, ..., 4:]).all() and np.isnan(s.box[nz + 2:, ..., 4:]).all())
        halo.exchange(s, 3)  # everything
        all_ok = (np.array_equal(s.box[0:2], u[[(k0 - 2) % N, (k0 - 1) % N]])
                  and np.array_equal(s.box[nz + 2:], u[[(k0 + nz) % N, (k0 + nz + 1) % N]])
                  and np.array_equal(s.box[2:2 + nz], u[k0:k0 + nz]))
        dist.barrier()
        out.put((rank, bool(phi_ok), bool(all_ok)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchange_ghost_planes(world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in res] == list(range(world))
    assert all(phi for _, phi, _ in res), res
    assert all(a for _, _, a in res), res


def test_slab_plane_split():
    from langevina_b200 import slab as S

    for n, r in [(256, 8), (48, 3), (34, 4), (12, 6), (4, 1)]:
        parts = S.slab_planes(n, r)
        assert sum(nz for _, nz in parts) == n
        assert all(nz >= 2 and nz % 2 == 0 and k0 % 2 == 0 for k0, nz in parts)
        assert [k0 for k0, _ in parts] == list(np.cumsum([0] + [nz for _, nz in parts[:-1]]))
    with pytest.raises(ValueError):
        S.slab_planes(12, 7)

"""Lattices split into z-slabs over ranks (the lgv_slab_* entry points).

The reference decomposes its lattice with DMDACreate3d (ModelA.h:315-318) and
refreshes the ghost layer with DMGlobalToLocal before every pass
(Stepper.cxx:81-82, 312-315, 477-480).  Here each rank holds global planes
k0 .. k0+nz-1 of the N^3 lattice (nz even) plus two ghost planes on each side
in one lgv slab handle, and lgv_step calls back into this module whenever a
sub-pass is about to read across planes; the callback refreshes the ghost
planes from the neighbouring ranks (periodic in z).  Because the counter
noise is indexed by the global site, every rank advances its planes exactly as
one handle holding the whole lattice would.

Two exchanges are provided:

- ThreadHalo: ranks as threads of one process on one GPU (each slab steps in
  its own host thread; the boundary planes move by device-to-device copies
  between the slabs' buffers).  It checks the decomposition on a single GPU.
- DistHalo: one slab per process with torch.distributed point-to-point
  operations -- device buffers over NCCL between GPUs, or buffers staged in
  host memory for gloo.

Measurements combine per-rank partial sums (lgv_slab_measure_partials), summed
over ranks, into the whole lattice's measurement (lgv_measure_from_partials).
"""
import ctypes as C
import threading

import numpy as np

from . import _lib as L

NOBS = 25  # observables of the measurement's partial sums


def slab_planes(N, R):
    """(k0, nz) of each of R ranks: nz even, planes split as evenly as possible
    (the first ranks take the remaining pairs)."""
    if N % 2 or R < 1 or N < 2 * R:
        raise ValueError(f"cannot split {N} planes into {R} slabs of an even number of planes >= 2")
    base, extra = divmod(N // 2, R)
    out, k = [], 0
    for r in range(R):
        nz = 2 * (base + (1 if r < extra else 0))
        out.append((k, nz))
        k += nz
    return out


class SlabLattice:
    """One rank's slab: an lgv slab handle and its halo exchange."""

    def __init__(self, N, k0, nz, halo, rank=0, **coef):
        self.lib = L.load()
        self.N, self.k0, self.nz, self.Nz, self.rank = N, k0, nz, nz + 4, rank
        self.halo = halo
        self.halo_error = None
        p = L.make_params(N, **coef)
        h = C.c_void_p()
        L.check(self.lib.lgv_slab_create(C.byref(p), k0, nz, C.byref(h)), "lgv_slab_create")
        self.h = h
        self._cb = L.HALO_FN(self._on_halo)  # kept alive as long as the handle
        L.check(self.lib.lgv_slab_set_halo(h, C.cast(self._cb, C.c_void_p), None), "lgv_slab_set_halo")

    def close(self):
        if self.h:
            self.lib.lgv_destroy(self.h)
            self.h = None

    def _on_halo(self, ctx, h, comps):
        try:
            self.halo.exchange(self, comps)
            return 0
        except Exception as e:  # reported by lgv_step as LGV_ERR_STATE; the cause is kept here
            self.halo_error = e
            return 1

    # ---- geometry and state -------------------------------------------------
    def box_planes(self):
        """Global planes of the buffer's local planes 0 .. nz+3."""
        return [(self.k0 - 2 + q) % self.N for q in range(self.Nz)]

    def set_global_state(self, u):
        """Load this slab's planes (ghosts included) from a whole lattice u[k][j][i][10]."""
        box = np.ascontiguousarray(np.asarray(u, dtype=np.float64)[self.box_planes()])
        L.check(self.lib.lgv_set_state(self.h, L.ptr(box)), "lgv_set_state")

    def get_interior(self):
        """This slab's own planes k0 .. k0+nz-1 as u[k][j][i][10]."""
        box = np.empty((self.Nz, self.N, self.N, 10))
        L.check(self.lib.lgv_get_state(self.h, L.ptr(box)), "lgv_get_state")
        return box[2:2 + self.nz]

    def set_counter(self, c):
        L.check(self.lib.lgv_set_counter(self.h, int(c)), "lgv_set_counter")

    def step(self, ev, dt, t=0.0, nsteps=1, inner=1, outer=1):
        rc = self.lib.lgv_step(self.h, ev, inner, outer, float(dt), float(t), int(nsteps))
        if rc != L.LGV_OK and self.halo_error is not None:
            raise RuntimeError(f"rank {self.rank}: halo exchange failed") from self.halo_error
        L.check(rc, "lgv_step")

    # ---- halo buffers ---------------------------------------------------------
    def halo_doubles(self, comps):
        return int(self.lib.lgv_slab_halo_doubles(self.h, comps))

    def pack(self, side, comps, buf):
        """Copy the two lowest (side 0) or highest (side 1) own planes of the
        component groups `comps` into the device tensor `buf` (asynchronous)."""
        L.check(self.lib.lgv_slab_pack(self.h, side, comps, C.c_void_p(buf.data_ptr())), "lgv_slab_pack")

    def unpack(self, side, comps, buf):
        """Fill the two ghost planes below (side 0) or above (side 1) from `buf`."""
        L.check(self.lib.lgv_slab_unpack(self.h, side, comps, C.c_void_p(buf.data_ptr())), "lgv_slab_unpack")

    def sync(self):
        L.check(self.lib.lgv_synchronize(self.h), "lgv_synchronize")

    # ---- measurement ----------------------------------------------------------
    def measure_partials(self, T, U):
        """Write this slab's rows of T[25][N][N] and its partial sums U[25][N][N]
        (device tensors; T's other rows are left as they are); synchronises."""
        L.check(self.lib.lgv_slab_measure_partials(self.h, C.c_void_p(T.data_ptr()), C.c_void_p(U.data_ptr())),
                "lgv_slab_measure_partials")
        self.sync()


def measure_from_partials(T, U, N, out):
    """The whole lattice's measurement (lgv_measure_device packing) from the
    summed partials; device tensors, synchronous on the default stream."""
    lib = L.load()
    L.check(lib.lgv_measure_from_partials(C.c_void_p(T.data_ptr()), C.c_void_p(U.data_ptr()), N,
                                          C.c_void_p(out.data_ptr()), None), "lgv_measure_from_partials")


class ThreadHalo:
    """Ranks as host threads of one process on one GPU.

    At an exchange every rank packs its two lowest and two highest planes into
    its own device buffers and synchronises its stream; all ranks meet at a
    barrier; each unpacks the buffers of the rank below into its lower ghost
    planes and those of the rank above into its upper ghost planes; all meet
    again before a buffer is packed anew.  Kernels of different ranks never
    wait on each other on the device: every wait is a host barrier between
    launches."""

    def __init__(self, R, device="cuda"):
        import torch

        self.R = R
        self.torch = torch
        self.device = device
        self.barrier = threading.Barrier(R)
        self.bufs = {}

    def attach(self, slab):
        n = slab.halo_doubles(L.HALO_ALL)
        t = self.torch
        self.bufs[slab.rank] = (t.empty(n, dtype=t.float64, device=self.device),
                                t.empty(n, dtype=t.float64, device=self.device))

    def exchange(self, slab, comps):
        r, R = slab.rank, self.R
        n = slab.halo_doubles(comps)
        lo, hi = self.bufs[r]
        slab.pack(0, comps, lo[:n])
        slab.pack(1, comps, hi[:n])
        slab.sync()
        self.barrier.wait(timeout=120)
        slab.unpack(0, comps, self.bufs[(r - 1) % R][1][:n])
        slab.unpack(1, comps, self.bufs[(r + 1) % R][0][:n])
        slab.sync()
        self.barrier.wait(timeout=120)


def run_threads(slabs, fn):
    """Run fn(slab) for every slab in its own thread; re-raise the first error."""
    errs = [None] * len(slabs)

    def body(i):
        try:
            fn(slabs[i])
        except BaseException as e:  # noqa: BLE001  (re-raised below)
            errs[i] = e

    th = [threading.Thread(target=body, args=(i,)) for i in range(len(slabs))]
    for x in th:
        x.start()
    for x in th:
        x.join()
    for e in errs:
        if e is not None:
            raise e


class DistHalo:
    """One slab per process over torch.distributed.

    Two shifts per exchange, so that every message has one sender and one
    receiver whatever the number of ranks: each rank sends its two highest
    planes to the rank above and receives the lower ghosts from the rank below;
    then sends its two lowest planes below and receives the upper ghosts from
    above.  `staging` "device" hands the device buffers to the process group
    (NCCL); "host" copies them through pinned host memory (gloo)."""

    def __init__(self, dist, staging="device", device="cuda"):
        import torch

        self.dist = dist
        self.torch = torch
        self.staging = staging
        self.device = device
        self.rank = dist.get_rank()
        self.R = dist.get_world_size()
        self._bufs = None

    def _buffers(self, n):
        t = self.torch
        if self._bufs is None or self._bufs[0].numel() < n:
            mk = (lambda: t.empty(n, dtype=t.float64, device=self.device))
            self._bufs = [mk() for _ in range(4)]  # send lo, send hi, recv lo, recv hi
            if self.staging == "host":
                pin = self.device != "cpu"
                self._host = [t.empty(n, dtype=t.float64, pin_memory=pin) for _ in range(4)]
        return [b[:n] for b in self._bufs]

    def _shift(self, send, dst, recv, src):
        d = self.dist
        if self.staging == "host" and self.device != "cpu":
            hs, hr = self._host[0][:send.numel()], self._host[1][:recv.numel()]
            hs.copy_(send)
            ops = [d.P2POp(d.isend, hs, dst), d.P2POp(d.irecv, hr, src)]
            for w in d.batch_isend_irecv(ops):
                w.wait()
            recv.copy_(hr)
        else:
            ops = [d.P2POp(d.isend, send, dst), d.P2POp(d.irecv, recv, src)]
            for w in d.batch_isend_irecv(ops):
                w.wait()

    def exchange(self, slab, comps):
        n = slab.halo_doubles(comps)
        s_lo, s_hi, r_lo, r_hi = self._buffers(n)
        slab.pack(0, comps, s_lo)
        slab.pack(1, comps, s_hi)
        slab.sync()
        below, above = (self.rank - 1) % self.R, (self.rank + 1) % self.R
        if self.R == 1:
            r_lo.copy_(s_hi)
            r_hi.copy_(s_lo)
        else:
            self._shift(s_hi, above, r_lo, below)
            self._shift(s_lo, below, r_hi, above)
        if self.device != "cpu":
            self.torch.cuda.current_stream().synchronize()
        slab.unpack(0, comps, r_lo)
        slab.unpack(1, comps, r_hi)
        slab.sync()

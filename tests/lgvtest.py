"""Shared helpers of the parity tests: seeded inputs and comparisons."""
import ctypes as C
import math

import numpy as np

SQRT3 = math.sqrt(3.0)
RTOL = 1e-12  # per-site relative tolerance of the FP64 parity bar


def rand_state(N, seed, phi_scale=0.5, chi=5.0, charges=True):
    rng = np.random.default_rng(seed)
    u = np.zeros((N, N, N, 10))
    u[..., :4] = phi_scale * rng.normal(size=(N, N, N, 4))
    if charges:
        u[..., 4:] = math.sqrt(chi) * rng.normal(size=(N, N, N, 6))
    return u


def hb_noise(N, seed):
    rng = np.random.default_rng(seed)
    V = N ** 3
    prop = rng.uniform(-SQRT3, SQRT3, size=(4, V))
    acc = rng.uniform(0.0, 1.0, size=V)
    return prop, acc


def charge_noise(N, seed):
    rng = np.random.default_rng(seed)
    V = N ** 3
    xyz = rng.permutation(3)
    eo = rng.permutation(2)
    order = np.array(list(xyz) + list(eo), dtype=np.int32)
    q = rng.uniform(-SQRT3, SQRT3, size=(36, V))
    acc = rng.uniform(0.0, 1.0, size=(36, V))
    return order, q, acc


def em_noise(N, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(4, N ** 3))


def site_rel_err(a, b, floor=1e-6):
    """Largest per-site relative error, per field group (phi, A, V)."""
    a = a.reshape(-1, 10)
    b = b.reshape(-1, 10)
    worst = 0.0
    for lo, hi in ((0, 4), (4, 7), (7, 10)):
        d = np.abs(a[:, lo:hi] - b[:, lo:hi]).max(axis=1)
        s = np.maximum(np.abs(b[:, lo:hi]).max(axis=1), floor)
        worst = max(worst, float((d / s).max()))
    return worst


def assert_state_close(gpu, cpu, rtol=RTOL, skip_sites=None, what=""):
    g = gpu.reshape(-1, 10).copy()
    c = cpu.reshape(-1, 10).copy()
    if skip_sites is not None and len(skip_sites):
        g = np.delete(g, skip_sites, axis=0)
        c = np.delete(c, skip_sites, axis=0)
    err = site_rel_err(g, c)
    assert err <= rtol, f"{what}: per-site relative error {err:.3e} > {rtol:.0e}"
    return err


def compare_flags(gpu_flags, orc_flags, n):
    """Accept decisions must agree except where the oracle flagged a tie (bit 4)."""
    g = gpu_flags[:n]
    o = orc_flags[:n]
    tie = (o & 4) != 0
    bad = np.nonzero((g != (o & 3)) & ~tie)[0]
    assert bad.size == 0, f"{bad.size} accept decisions differ, first at {bad[:5]}"
    return int(tie.sum())


class GpuLattice:
    """Thin owner of an lgv handle for the tests (calls go through the C ABI)."""

    def __init__(self, lgv, N, **kw):
        from langevina_b200 import _lib as L

        self.L = L
        self.lib = L.load()
        self.N, self.V = N, N ** 3
        self.p = L.make_params(N, **kw)
        h = C.c_void_p()
        L.check(self.lib.lgv_create(C.byref(self.p), C.byref(h)), "lgv_create")
        self.h = h

    def close(self):
        if self.h:
            self.lib.lgv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.L.check(self.lib.lgv_set_state(self.h, self.L.ptr(u)), "set_state")

    def get_state(self):
        u = np.empty((self.N, self.N, self.N, 10))
        self.L.check(self.lib.lgv_get_state(self.h, self.L.ptr(u)), "get_state")
        return u

    def mode(self, m):
        self.L.check(self.lib.lgv_set_noise_mode(self.h, m), "noise_mode")

    def counter(self, c=None):
        if c is not None:
            self.L.check(self.lib.lgv_set_counter(self.h, int(c)), "set_counter")
        v = C.c_uint64()
        self.L.check(self.lib.lgv_get_counter(self.h, C.byref(v)), "get_counter")
        return v.value

    def inject_hb(self, prop, acc):
        self.L.check(self.lib.lgv_inject_hb(self.h, self.L.ptr(prop), self.L.ptr(acc)), "inject_hb")

    def inject_charge(self, order, q, acc):
        o = np.ascontiguousarray(order, dtype=np.int32)
        self.L.check(self.lib.lgv_inject_charge(self.h, self.L.ptr(o), self.L.ptr(q), self.L.ptr(acc)),
                     "inject_charge")

    def inject_em(self, xi):
        xi = np.ascontiguousarray(xi)  # held while the call reads it
        self.L.check(self.lib.lgv_inject_em(self.h, self.L.ptr(xi)), "inject_em")

    def step(self, ev, dt, t=0.0, nsteps=1, inner=1, outer=1):
        self.L.check(self.lib.lgv_step(self.h, ev, inner, outer, float(dt), float(t), int(nsteps)), "step")

    def initialize(self, kind, scale=0.0):
        self.L.check(self.lib.lgv_initialize(self.h, kind, float(scale)), "initialize")

    def flags(self, on=True):
        self.L.check(self.lib.lgv_debug_flags(self.h, 1 if on else 0), "debug_flags")

    def get_flags(self):
        f = np.zeros(36 * self.V, dtype=np.uint8)
        self.L.check(self.lib.lgv_get_flags(self.h, self.L.ptr(f)), "get_flags")
        return f

    def energy(self):
        e = C.c_double()
        self.L.check(self.lib.lgv_energy(self.h, C.byref(e)), "energy")
        return e.value

    def measure(self):
        m = self.L.Measurement(self.N)
        s = m.struct()
        self.L.check(self.lib.lgv_measure(self.h, C.byref(s)), "measure")
        return m

    def monitors(self, on=None):
        if on is not None:
            self.L.check(self.lib.lgv_enable_monitors(self.h, 1 if on else 0), "enable_monitors")
            return None
        out = []
        for w in range(3):
            m = self.L.lgv_monitor()
            self.L.check(self.lib.lgv_get_monitor(self.h, w, C.byref(m)), "get_monitor")
            out.append(m.as_dict())
        return out

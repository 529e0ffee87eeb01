"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (lgv_oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this module.  It restates the reference algorithm on the CPU; the product path
never calls it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblgv_oracle.so")

SEQUENTIAL, COUNTER, INJECTED = 0, 1, 2


class _params(C.Structure):
    _fields_ = [("N", C.c_int32), ("reserved0", C.c_int32), ("LX", C.c_double), ("mass0", C.c_double),
                ("dmassdt", C.c_double), ("lambda_", C.c_double), ("H", C.c_double), ("chi", C.c_double),
                ("gamma", C.c_double), ("diffusion", C.c_double), ("seed", C.c_uint64)]


class _monitor(C.Structure):
    _fields_ = [("down_counts", C.c_int64), ("up_counts", C.c_int64), ("up_yes", C.c_int64),
                ("up_no", C.c_int64), ("down_dS", C.c_double), ("up_dS", C.c_double)]


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "liblgv_oracle.so"])


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    V = C.c_void_p
    sig = {
        "orc_create": (V, [C.c_void_p, C.c_int, C.c_int]),
        "orc_destroy": (None, [V]),
        "orc_set_params": (None, [V, C.c_void_p]),
        "orc_set_state": (None, [V, C.c_void_p]),
        "orc_get_state": (None, [V, C.c_void_p]),
        "orc_set_counter": (None, [V, C.c_uint64]),
        "orc_get_counter": (C.c_uint64, [V]),
        "orc_inject_hb": (None, [V, C.c_void_p, C.c_void_p]),
        "orc_inject_charge": (None, [V, C.c_void_p, C.c_void_p, C.c_void_p]),
        "orc_inject_em": (None, [V, C.c_void_p]),
        "orc_step": (C.c_int, [V, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]),
        "orc_initialize": (C.c_int, [V, C.c_int, C.c_double]),
        "orc_measure": (None, [V, C.c_void_p]),
        "orc_energy": (C.c_double, [V]),
        "orc_last_energies": (None, [V, C.c_void_p]),
        "orc_get_monitor": (None, [V, C.c_int, C.c_void_p]),
        "orc_debug_flags": (None, [V, C.c_int]),
        "orc_set_hb_proposal": (None, [V, C.c_int]),
        "orc_get_flags": (None, [V, C.c_void_p]),
        "orc_o4_rotation": (None, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "orc_seq_draws": (None, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
        "orc_xoro_raw": (None, [C.c_uint64, C.c_uint64, C.c_int, C.c_void_p]),
        "orc_seed_seq": (None, [C.c_int, C.c_int, C.c_void_p]),
        "orc_ctr_draws": (None, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, C.c_void_p]),
        "orc_ctr_order": (None, [C.c_uint64, C.c_uint64, C.c_void_p]),
        "orc_em_noise": (None, [C.c_uint64, C.c_uint64, C.c_int, C.c_void_p]),
        "orc_charge_pair_chain": (None, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p]),
        "orc_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _ptr(a):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def params(N, LX=None, mass0=-4.70052, dmassdt=0.0, lam=4.0, H=0.003, chi=5.0, gamma=1.0, diffusion=None,
           seed=10):
    p = _params()
    p.N, p.reserved0 = int(N), 0
    p.LX = float(N if LX is None else LX)
    p.mass0, p.dmassdt, p.lambda_, p.H, p.chi, p.gamma = map(float, (mass0, dmassdt, lam, H, chi, gamma))
    p.diffusion = float(1.0 / 3.0 * gamma if diffusion is None else diffusion)
    p.seed = int(seed) & ((1 << 64) - 1)
    return p


class Oracle:
    """One lattice of the CPU restatement.  mode: SEQUENTIAL / COUNTER / INJECTED."""

    def __init__(self, N, mode=COUNTER, nranks=1, **kw):
        self.lib = load()
        self.N, self.V = N, N ** 3
        self._p = params(N, **kw)
        self.h = self.lib.orc_create(C.byref(self._p), mode, nranks)
        if not self.h:
            raise ValueError("orc_create failed (N even >= 4, 1 <= nranks <= N)")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.size == 10 * self.V
        self.lib.orc_set_state(self.h, _ptr(u))

    def get_state(self):
        u = np.empty((self.N, self.N, self.N, 10))
        self.lib.orc_get_state(self.h, _ptr(u))
        return u

    def set_counter(self, c):
        self.lib.orc_set_counter(self.h, int(c))

    def get_counter(self):
        return int(self.lib.orc_get_counter(self.h))

    # (the contiguous copies are held in locals while the library reads them)
    def inject_hb(self, prop, acc):
        prop, acc = np.ascontiguousarray(prop), np.ascontiguousarray(acc)
        self.lib.orc_inject_hb(self.h, _ptr(prop), _ptr(acc))

    def inject_charge(self, order, q, acc):
        o = np.ascontiguousarray(order, dtype=np.int32)
        q, acc = np.ascontiguousarray(q), np.ascontiguousarray(acc)
        self.lib.orc_inject_charge(self.h, _ptr(o), _ptr(q), _ptr(acc))

    def inject_em(self, xi):
        xi = np.ascontiguousarray(xi)
        self.lib.orc_inject_em(self.h, _ptr(xi))

    def set_hb_proposal(self, kind):
        """0: uniform U(-sqrt3, sqrt3) proposals (the reference's); 1: Gaussian
        (counter noise only, as the CUDA library's lgv_set_hb_proposal)."""
        self.lib.orc_set_hb_proposal(self.h, int(kind))

    def step(self, evolver, dt, t=0.0, nsteps=1, inner=1, outer=1):
        rc = self.lib.orc_step(self.h, evolver, inner, outer, float(dt), float(t), int(nsteps))
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())

    def initialize(self, kind, scale=0.0):
        rc = self.lib.orc_initialize(self.h, kind, float(scale))
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())

    def energy(self):
        return float(self.lib.orc_energy(self.h))

    def last_energies(self):
        e = np.zeros(2)
        self.lib.orc_last_energies(self.h, _ptr(e))
        return e

    def monitor(self, which):
        m = _monitor()
        self.lib.orc_get_monitor(self.h, which, C.byref(m))
        return {k: getattr(m, k) for k, _ in m._fields_}

    def debug_flags(self, on=True):
        self.lib.orc_debug_flags(self.h, 1 if on else 0)

    def get_flags(self):
        f = np.zeros(36 * self.V, dtype=np.uint8)
        self.lib.orc_get_flags(self.h, _ptr(f))
        return f

    def measure(self, meas):
        """meas: langevina_b200._lib.Measurement-like object with .struct()."""
        s = meas.struct()
        self.lib.orc_measure(self.h, C.byref(s))
        return meas


def o4_rotation(V, A, phi):
    lib = load()
    V = np.ascontiguousarray(V, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64)
    p = np.array(phi, dtype=np.float64)
    lib.orc_o4_rotation(_ptr(V), _ptr(A), _ptr(p))
    return p


def seq_draws(base_seed, rank, size, kind, n):
    """kind: 'raw' (uint64), 'unif', 'var1', 'norm' of the reference serial stream."""
    lib = load()
    k = {"raw": 0, "unif": 1, "var1": 2, "norm": 3}[kind]
    out = np.zeros(n)
    lib.orc_seq_draws(int(base_seed), int(rank), int(size), k, int(n), _ptr(out))
    return out.view(np.uint64) if kind == "raw" else out


def seed_seq(base_seed, size):
    lib = load()
    out = np.zeros(size, dtype=np.uint32)
    lib.orc_seed_seq(int(base_seed), int(size), _ptr(out))
    return out


def xoro_raw(s0, s1, n):
    lib = load()
    out = np.zeros(n, dtype=np.uint64)
    lib.orc_xoro_raw(int(s0), int(s1), int(n), _ptr(out))
    return out


def ctr_draws(seed, ctr, n, ndraw):
    lib = load()
    out = np.zeros(ndraw, dtype=np.uint64)
    lib.orc_ctr_draws(int(seed), int(ctr), int(n), int(ndraw), _ptr(out))
    return out


def ctr_order(seed, ctr):
    lib = load()
    out = np.zeros(5, dtype=np.int32)
    lib.orc_ctr_order(int(seed), int(ctr), _ptr(out))
    return out


def em_noise(seed, ctr, N):
    """Counter-mode Euler-Maruyama normals of step counter ctr, shape (4, N, N, N) = [l, k, j, i]."""
    lib = load()
    out = np.zeros((4, N, N, N))
    lib.orc_em_noise(int(seed), int(ctr), int(N), _ptr(out))
    return out


def charge_pair_chain(chi, rms, nA, nB, base_seed, n):
    lib = load()
    a = np.zeros(n)
    b = np.zeros(n)
    lib.orc_charge_pair_chain(float(chi), float(rms), float(nA), float(nB), int(base_seed), int(n), _ptr(a), _ptr(b))
    return a, b

"""ctypes binding of liblgv.so (include/lgv.h).

The library is built in-tree by ``langevina_b200.build``.  Loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblgv.so")

LGV_OK = 0
LGV_ERR_INVALID, LGV_ERR_CUDA, LGV_ERR_NOMEM, LGV_ERR_TIMEOUT, LGV_ERR_STATE, LGV_ERR_UNSUPPORTED = -1, -2, -3, -4, -5, -6
HALO_PHI, HALO_CHARGES, HALO_ALL = 1, 2, 3
# int (*lgv_halo_fn)(void *ctx, lgv_handle *h, int comps)
HALO_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int)
NPHI, NA, NV, NDOF = 4, 3, 3, 10
NOBS, NOBS_PHASE = 11, 14
NOALLOC_MAX_N = 128

PV2HBSPLIT, PV2HBSPLIT_NODIFFUSE, PV2HBSPLIT_ONLYDIFFUSE = 0, 1, 2
IDEAL_PV2, EULER_LANGEVIN_HB, CHARGE_HB, MODELA_EM, IDEAL_EM = 3, 4, 5, 6, 7
NOISE_COUNTER, NOISE_INJECTED = 0, 1
INIT_ZERO, INIT_PHI_GAUSSIAN, INIT_CHARGES_GAUSSIAN = 0, 1, 2
HB_PROPOSAL_UNIFORM, HB_PROPOSAL_GAUSSIAN = 0, 1
MONITOR_IDEAL, MONITOR_PHI_HB, MONITOR_CHARGE_HB = 0, 1, 2
KCLASS_IDEAL, KCLASS_PHI_HB, KCLASS_CHARGE, KCLASS_EM, KCLASS_MEASURE = 0, 1, 2, 3, 4
PACK_GIVEN, PACK_LARGEST_FIRST, PACK_INTERLEAVED = 0, 1, 2
TILE_32x8, TILE_16x16 = 0, 1


class lgv_params(C.Structure):
    _fields_ = [("N", C.c_int32), ("reserved0", C.c_int32), ("LX", C.c_double), ("mass0", C.c_double),
                ("dmassdt", C.c_double), ("lambda_", C.c_double), ("H", C.c_double), ("chi", C.c_double),
                ("gamma", C.c_double), ("diffusion", C.c_double), ("seed", C.c_uint64)]


class lgv_monitor(C.Structure):
    _fields_ = [("down_counts", C.c_int64), ("up_counts", C.c_int64), ("up_yes", C.c_int64),
                ("up_no", C.c_int64), ("down_dS", C.c_double), ("up_dS", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_DP = C.POINTER(C.c_double)


class lgv_measurement(C.Structure):
    _fields_ = [("OAverage", _DP), ("wall", _DP * 3), ("wall_k", _DP * 3), ("wall_k_rotated", _DP * 3),
                ("wall_phase", _DP * 3), ("wall_phase_k", _DP * 3)]


# (name, restype, argtypes) of every entry point declared in include/lgv.h
_H = C.c_void_p
SIGNATURES = [
    ("lgv_version", C.c_int, []),
    ("lgv_status_string", C.c_char_p, [C.c_int]),
    ("lgv_last_error", C.c_char_p, []),
    ("lgv_create", C.c_int, [C.POINTER(lgv_params), C.POINTER(_H)]),
    ("lgv_destroy", C.c_int, [_H]),
    ("lgv_set_params", C.c_int, [_H, C.POINTER(lgv_params)]),
    ("lgv_set_state", C.c_int, [_H, C.c_void_p]),
    ("lgv_get_state", C.c_int, [_H, C.c_void_p]),
    ("lgv_set_state_device", C.c_int, [_H, C.c_void_p]),
    ("lgv_get_state_device", C.c_int, [_H, C.c_void_p]),
    ("lgv_initialize", C.c_int, [_H, C.c_int, C.c_double]),
    ("lgv_set_noise_mode", C.c_int, [_H, C.c_int]),
    ("lgv_set_hb_proposal", C.c_int, [_H, C.c_int]),
    ("lgv_set_counter", C.c_int, [_H, C.c_uint64]),
    ("lgv_get_counter", C.c_int, [_H, C.POINTER(C.c_uint64)]),
    ("lgv_inject_hb", C.c_int, [_H, C.c_void_p, C.c_void_p]),
    ("lgv_inject_charge", C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("lgv_inject_em", C.c_int, [_H, C.c_void_p]),
    ("lgv_step", C.c_int, [_H, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]),
    ("lgv_measure", C.c_int, [_H, C.POINTER(lgv_measurement)]),
    ("lgv_measure_device", C.c_int, [_H, C.c_void_p]),
    ("lgv_measure_size", C.c_size_t, [C.c_int]),
    ("lgv_energy", C.c_int, [_H, C.POINTER(C.c_double)]),
    ("lgv_enable_monitors", C.c_int, [_H, C.c_int]),
    ("lgv_get_monitor", C.c_int, [_H, C.c_int, C.POINTER(lgv_monitor)]),
    ("lgv_set_stream", C.c_int, [_H, C.c_void_p]),
    ("lgv_synchronize", C.c_int, [_H]),
    ("lgv_timing_enable", C.c_int, [_H, C.c_int]),
    ("lgv_timing_read", C.c_int, [_H, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("lgv_debug_flags", C.c_int, [_H, C.c_int]),
    ("lgv_get_flags", C.c_int, [_H, C.c_void_p]),
    ("lgv_measure_aos_noalloc", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("lgv_diff_forward", C.c_int, [_H, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    ("lgv_diff_backward", C.c_int, [_H, C.c_void_p, C.c_void_p]),
    ("lgv_diff_averages", C.c_int, [_H, C.c_void_p, C.c_int]),
    ("lgv_ensemble_create", C.c_int, [C.c_int, C.c_void_p, C.POINTER(_H)]),
    ("lgv_ensemble_destroy", C.c_int, [_H]),
    ("lgv_ensemble_size", C.c_int, [_H, C.POINTER(C.c_int)]),
    ("lgv_ensemble_set_state", C.c_int, [_H, C.c_int, C.c_void_p]),
    ("lgv_ensemble_get_state", C.c_int, [_H, C.c_int, C.c_void_p]),
    ("lgv_ensemble_initialize", C.c_int, [_H, C.c_int, C.c_double]),
    ("lgv_ensemble_set_counter", C.c_int, [_H, C.c_uint64]),
    ("lgv_ensemble_get_counter", C.c_int, [_H, C.POINTER(C.c_uint64)]),
    ("lgv_ensemble_step", C.c_int, [_H, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]),
    ("lgv_ensemble_oaverage", C.c_int, [_H, C.c_void_p]),
    ("lgv_ensemble_oaverage_device", C.c_int, [_H, C.c_void_p]),
    ("lgv_ensemble_tune", C.c_int, [_H, C.c_int, C.c_int, C.c_int]),
    ("lgv_ensemble_autotune", C.c_int, [_H, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p,
                                        C.POINTER(C.c_double)]),
    ("lgv_ensemble_use_graphs", C.c_int, [_H, C.c_int]),
    ("lgv_ensemble_diff_forward", C.c_int, [_H, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    ("lgv_ensemble_diff_backward", C.c_int, [_H, C.c_void_p, C.c_void_p]),
    ("lgv_ensemble_use_persistent", C.c_int, [_H, C.c_int]),
    ("lgv_ensemble_set_stream", C.c_int, [_H, C.c_void_p]),
    ("lgv_ensemble_synchronize", C.c_int, [_H]),
    ("lgv_slab_create", C.c_int, [C.POINTER(lgv_params), C.c_int, C.c_int, C.POINTER(_H)]),
    ("lgv_slab_set_halo", C.c_int, [_H, C.c_void_p, C.c_void_p]),
    ("lgv_slab_halo_doubles", C.c_size_t, [_H, C.c_int]),
    ("lgv_slab_pack", C.c_int, [_H, C.c_int, C.c_int, C.c_void_p]),
    ("lgv_slab_unpack", C.c_int, [_H, C.c_int, C.c_int, C.c_void_p]),
    ("lgv_slab_measure_partials", C.c_int, [_H, C.c_void_p, C.c_void_p]),
    ("lgv_measure_from_partials", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("lgv_x2k", C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_void_p]),
    ("lgv_x2k_rotated", C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    ("lgv_time_correlator", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
]

_lib = None


class LgvError(RuntimeError):
    def __init__(self, status, where, detail):
        super().__init__(f"{where}: {detail} (status {status})")
        self.status = status


def load(path=LIB_PATH):
    """Load liblgv.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"liblgv.so not found at {path}: build it with `python langevina_b200/build.py`")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status, where):
    if status != LGV_OK:
        lib = load()
        raise LgvError(status, where, (lib.lgv_last_error() or b"").decode() or
                       lib.lgv_status_string(status).decode())
    return status


def ptr(a):
    """Address of a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C contiguous"
    return a.ctypes.data


def make_params(N, LX=None, mass0=-4.70052, dmassdt=0.0, lam=4.0, H=0.003, chi=5.0, gamma=1.0,
                diffusion=None, seed=10):
    """lgv_params with the reference's defaults (ModelA.h:71-111, 185-248)."""
    p = lgv_params()
    p.N = int(N)
    p.reserved0 = 0
    p.LX = float(N if LX is None else LX)
    p.mass0 = float(mass0)
    p.dmassdt = float(dmassdt)
    p.lambda_ = float(lam)
    p.H = float(H)
    p.chi = float(chi)
    p.gamma = float(gamma)
    p.diffusion = float(1.0 / 3.0 * gamma if diffusion is None else diffusion)
    p.seed = int(seed) & ((1 << 64) - 1)
    return p


class Measurement:
    """Host arrays of one Measurer::measure() call (measurer.h:96-127)."""

    def __init__(self, N):
        NK = N // 2 + 1
        self.N = N
        self.OAverage = np.zeros(NOBS)
        self.wall = [np.zeros((NOBS, N)) for _ in range(3)]
        self.wall_k = [np.zeros((NOBS, NK, 2)) for _ in range(3)]
        self.wall_k_rotated = [np.zeros((NOBS_PHASE, NK, 2)) for _ in range(3)]
        self.wall_phase = [np.zeros((NOBS_PHASE, N)) for _ in range(3)]
        self.wall_phase_k = [np.zeros((NOBS_PHASE, NK, 2)) for _ in range(3)]

    def struct(self):
        m = lgv_measurement()
        dp = lambda a: a.ctypes.data_as(_DP)
        m.OAverage = dp(self.OAverage)
        for a in range(3):
            m.wall[a] = dp(self.wall[a])
            m.wall_k[a] = dp(self.wall_k[a])
            m.wall_k_rotated[a] = dp(self.wall_k_rotated[a])
            m.wall_phase[a] = dp(self.wall_phase[a])
            m.wall_phase_k[a] = dp(self.wall_phase_k[a])
        return m

    # reference-style names
    @property
    def wallX(self): return self.wall[0]
    @property
    def wallY(self): return self.wall[1]
    @property
    def wallZ(self): return self.wall[2]
    @property
    def wallX_k(self): return self.wall_k[0][..., 0] + 1j * self.wall_k[0][..., 1]
    @property
    def wallY_k(self): return self.wall_k[1][..., 0] + 1j * self.wall_k[1][..., 1]
    @property
    def wallZ_k(self): return self.wall_k[2][..., 0] + 1j * self.wall_k[2][..., 1]

    def arrays(self):
        out = {"OAverage": self.OAverage}
        for a, ax in enumerate("XYZ"):
            out[f"wall{ax}"] = self.wall[a]
            out[f"wall{ax}_k"] = self.wall_k[a]
            out[f"wall{ax}_k_rotated"] = self.wall_k_rotated[a]
            out[f"wall{ax}Phase"] = self.wall_phase[a]
            out[f"wall{ax}Phase_k"] = self.wall_phase_k[a]
        return out

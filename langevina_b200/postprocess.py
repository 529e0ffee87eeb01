"""Post-processing of measurement histories on the GPU.

Mirrors the reference's downstream tools for data a run produces:

- ``x2k(walls)``: the x2k.exe transform (ModelG/x2k.cxx:94-113), the r2c DFT
  divided by N of every wall row, k = 0..N/2, as (re, im) pairs;
- ``x2k_rotated(walls_k)``: x2k_rotated.exe (ModelG/x2k_rotated.cxx:92-143),
  k walls rotated into the frame of the k = 0 phi direction (13 rows);
- ``computeOtOtp``, ``computeBlockedOtOtp``, ``blockedOtOtp``: the time
  correlators of python/Loader.py:229-300 with the same names, arguments and
  results, computed for every trailing column of the input at once.

Inputs may be numpy arrays (copied to the device; results come back as numpy)
or CUDA torch tensors (results stay on the device, ordered on the current
stream).  Every routine calls a CUDA kernel of liblgv.so; there is no host
fallback.
"""
import ctypes as C

import numpy as np

from . import _lib as L

__all__ = ["x2k", "x2k_rotated", "computeOtOtp", "computeBlockedOtOtp", "blockedOtOtp"]


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("langevina_b200.postprocess needs a CUDA device")
    return torch


def _to_device(x):
    """(tensor on the device, was_numpy)."""
    torch = _torch()
    if isinstance(x, torch.Tensor):
        if not x.is_cuda:
            return x.cuda(), False
        return x, False
    a = np.asarray(x)
    if np.iscomplexobj(a):
        a = a.astype(np.complex128, copy=False)
    else:
        a = a.astype(np.float64, copy=False)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda(), True


def _back(t, was_numpy):
    if was_numpy:
        _torch().cuda.current_stream().synchronize()
        return t.cpu().numpy()
    return t


def _stream():
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


def x2k(walls):
    """W(k) = (1/N) sum_x W(x) e^{-2 pi i k x/N}, k = 0..N/2, over the last axis:
    [..., N] -> [..., N/2+1, 2] (x2k.cxx:94-113)."""
    torch = _torch()
    complex_in = walls.is_complex() if isinstance(walls, torch.Tensor) else np.iscomplexobj(walls)
    if complex_in:
        raise ValueError("x2k transforms real walls (x2k.cxx reads real rows)")
    w, was_np = _to_device(walls)
    w = w.to(torch.float64).contiguous()
    N = w.shape[-1]
    rows = w.numel() // N if N else 0
    out = torch.empty(tuple(w.shape[:-1]) + (N // 2 + 1, 2), dtype=torch.float64, device=w.device)
    lib = L.load()
    L.check(lib.lgv_x2k(C.c_void_p(w.data_ptr()), rows, N, C.c_void_p(out.data_ptr()), _stream()), "lgv_x2k")
    return _back(out, was_np)


def x2k_rotated(walls_k):
    """[..., nfields >= 10, NK, 2] k walls -> [..., 13, NK, 2] in the frame of
    the k = 0 phi direction (x2k_rotated.cxx:92-143)."""
    torch = _torch()
    w, was_np = _to_device(walls_k)
    w = w.to(torch.float64).contiguous()
    if w.dim() < 3 or w.shape[-1] != 2:
        raise ValueError("x2k_rotated expects [..., nfields, NK, 2]")
    nf, NK = w.shape[-3], w.shape[-2]
    rows = w.numel() // (nf * NK * 2)
    out = torch.empty(tuple(w.shape[:-3]) + (13, NK, 2), dtype=torch.float64, device=w.device)
    lib = L.load()
    L.check(lib.lgv_x2k_rotated(C.c_void_p(w.data_ptr()), rows, nf, NK, C.c_void_p(out.data_ptr()), _stream()),
            "lgv_x2k_rotated")
    return _back(out, was_np)


def _correlate(a, b, nTMax, decim, conn):
    """Device tensors a, b of shape [T, ...] (same shape and dtype) ->
    [nTMax, ...] on the device."""
    torch = _torch()
    cplx = a.is_complex() or b.is_complex()
    dt = torch.complex128 if cplx else torch.float64
    a = a.to(dt).contiguous()
    b = b.to(dt).contiguous()
    if a.shape != b.shape:
        raise ValueError(f"arrays of different shapes {tuple(a.shape)} and {tuple(b.shape)}")
    T = a.shape[0]
    ns = a.numel() // T if T else 0
    if T < 1 or ns < 1:
        raise ValueError("empty time series")
    if not (1 <= nTMax <= T):
        raise ValueError(f"nTMax must lie in [1, {T}] (got {nTMax})")
    if decim < 1:
        raise ValueError("decim must be >= 1")
    out = torch.empty((nTMax,) + tuple(a.shape[1:]), dtype=dt, device=a.device)
    ar = torch.view_as_real(a) if cplx else a
    br = torch.view_as_real(b) if cplx else b
    orr = torch.view_as_real(out) if cplx else out
    lib = L.load()
    L.check(lib.lgv_time_correlator(C.c_void_p(ar.data_ptr()), C.c_void_p(br.data_ptr()), T, ns,
                                    ns * (2 if cplx else 1), 1 if cplx else 0, int(nTMax), int(decim),
                                    1 if conn else 0, C.c_void_p(orr.data_ptr()), _stream()),
            "lgv_time_correlator")
    return out


def _mean_only(statFunc):
    if statFunc is not None:
        raise NotImplementedError("only the default mean statistic (Loader.py:229) runs on the GPU")


def computeOtOtp(arr1, arr2, statFunc=None, conn=False, nTMax=-1, decim=1):
    """Cttp[tt] = mean of arr1[t] * arr2[t + tt] over t = 0, decim, ... <
    len - tt, minus mean(arr1) mean(arr2) if conn (Loader.py:229-254), for
    every trailing column of [T, ...] inputs.  Returns (Cttp, CttpErr) with
    CttpErr zero, as the reference's default statistic."""
    _mean_only(statFunc)
    a, was_np = _to_device(arr1)
    b, _ = _to_device(arr2)
    if nTMax == -1:
        nTMax = a.shape[0]
    out = _correlate(a, b, nTMax, decim, conn)
    return _back(out, was_np), _back(_torch().zeros_like(out), was_np)


def computeBlockedOtOtp(arr1, arr2, nTMax, steps, decim=1, conn=False):
    """computeOtOtp over consecutive blocks of `steps` samples starting at 0,
    steps, ... < len - steps (Loader.py:269-281); [nblocks, nTMax, ...]."""
    torch = _torch()
    a, was_np = _to_device(arr1)
    b, _ = _to_device(arr2)
    res = [_correlate(a[s:s + steps], b[s:s + steps], nTMax, decim, conn) for s in range(0, a.shape[0] - steps, steps)]
    if not res:  # the reference returns an empty array
        return _back(torch.empty(0, dtype=torch.float64, device=a.device), was_np)
    return _back(torch.stack(res), was_np)


def blockedOtOtp(arr1, arr2, nTMax, nblocks, decim=1):
    """Blocks of steps = (len - nTMax) // nblocks samples (Loader.py:284-300).
    The reference hands each block arr2[s:s + steps + nTMax] but keeps only
    t < steps - tt, so only arr2[s:s + steps] enters; nTMax <= steps."""
    torch = _torch()
    a, was_np = _to_device(arr1)
    b, _ = _to_device(arr2)
    sMax = a.shape[0] - nTMax
    steps = int(sMax / nblocks)
    sMax = steps * nblocks
    if steps < 1:  # the reference's range() is empty (or its step zero, which raises)
        raise ValueError("blocks are empty: len(arr1) - nTMax < nblocks")
    res = [_correlate(a[s:s + steps], b[s:s + steps], nTMax, decim, False) for s in range(0, sMax, steps)]
    return _back(torch.stack(res), was_np)

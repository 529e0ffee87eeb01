"""TEST INFRASTRUCTURE ONLY: numpy restatement of the reference's
post-processing, the checker of langevina_b200.postprocess.

Only tests/ and bench.py's CPU-baseline leg may import this module; the
product path never calls it.

- x2k:          ModelG/x2k.cxx:94-113 (FFTW r2c, then / N), written as a direct
                DFT, W(k) = (1/N) sum_x W(x) e^{-2 pi i k x / N}, k = 0..N/2;
- x2k_rotated:  ModelG/x2k_rotated.cxx:16-26 (contract_rho, dualize_rho) and
                :92-143 (the per-row rotation), in complex arithmetic as there;
- computeOtOtp, computeBlockedOtOtp, blockedOtOtp: python/Loader.py:229-300
                with the default mean statistic, applied to every column of
                [T, ...] inputs (the reference takes one series at a time).
"""
import numpy as np


def x2k(walls):
    """[..., N] real walls -> [..., N/2+1, 2] (x2k.cxx:94-113)."""
    w = np.asarray(walls, dtype=np.float64)
    N = w.shape[-1]
    x = np.arange(N)
    k = np.arange(N // 2 + 1)
    phase = np.exp(-2j * np.pi * ((np.outer(k, x) % N) / N))
    W = (w @ phase.T) / N
    return np.stack([W.real, W.imag], axis=-1)


def _contract_rho(n, rho):
    """x2k_rotated.cxx:16-20."""
    return np.array([-(n[1] * rho[0]) - n[2] * rho[1] - n[3] * rho[2],
                     n[0] * rho[0] + n[3] * rho[4] - n[2] * rho[5],
                     n[0] * rho[1] - n[3] * rho[3] + n[1] * rho[5],
                     n[0] * rho[2] + n[2] * rho[3] - n[1] * rho[4]])


def _dualize_rho(rho):
    """x2k_rotated.cxx:22-26."""
    return np.array([rho[3], rho[4], rho[5], rho[0], rho[1], rho[2]])


def x2k_rotated(walls_k):
    """[..., nfields, NK, 2] -> [..., 13, NK, 2] (x2k_rotated.cxx:92-143)."""
    w = np.asarray(walls_k, dtype=np.float64)
    lead = w.shape[:-3]
    nf, NK = w.shape[-3], w.shape[-2]
    rows = w.reshape(-1, nf, NK, 2)
    out = np.zeros((rows.shape[0], 13, NK, 2))
    for r in range(rows.shape[0]):
        c = rows[r, :, :, 0] + 1j * rows[r, :, :, 1]
        n = rows[r, 0:4, 0, 0].astype(np.complex128)
        norm = np.sqrt(np.sum(np.abs(n) ** 2))
        if norm < np.finfo(np.float64).tiny:
            n = np.array([1, 0, 0, 0], dtype=np.complex128)
        else:
            n = n / norm
        for k in range(NK):
            phi = c[0:4, k]
            rho = c[4:10, k]
            phis = np.sum(n * phi)
            phir = phi - n * phis
            A = _contract_rho(n, rho)
            V = _contract_rho(n, _dualize_rho(rho))
            vals = [phis, *phir, *A, *V]
            for a, v in enumerate(vals):
                out[r, a, k, 0] = v.real
                out[r, a, k, 1] = v.imag
    return out.reshape(lead + (13, NK, 2))


def computeOtOtp(arr1, arr2, conn=False, nTMax=-1, decim=1):
    """Loader.py:229-254 with statFunc = mean, per column of [T, ...] arrays."""
    arr1 = np.asarray(arr1)
    arr2 = np.asarray(arr2)
    Npoints = len(arr1)
    if nTMax == -1:
        nTMax = Npoints
    dtype = np.result_type(arr1.dtype, arr2.dtype)
    Cttp = np.zeros((nTMax,) + arr1.shape[1:], dtype=dtype)
    if conn:
        av1 = np.mean(arr1, axis=0)
        av2 = np.mean(arr2, axis=0)
    for tt in range(nTMax):
        tmp = arr1 * np.roll(arr2, -tt, axis=0)[0:len(arr1)]
        if conn:
            tmp = tmp - av1 * av2
        Cttp[tt] = np.mean(tmp[0:Npoints - tt:decim], axis=0)
    return Cttp, np.zeros_like(Cttp)


def computeBlockedOtOtp(arr1, arr2, nTMax, steps, decim=1, conn=False):
    """Loader.py:269-281."""
    res = []
    sMax = len(arr1) - steps
    for s in range(0, sMax, steps):
        r, _ = computeOtOtp(arr1[s:s + steps], arr2[s:s + steps], conn=conn, nTMax=nTMax, decim=decim)
        res.append(r)
    return np.asarray(res)


def blockedOtOtp(arr1, arr2, nTMax, nblocks, decim=1):
    """Loader.py:284-300."""
    res = []
    sMax = len(arr1) - nTMax
    steps = int(sMax / nblocks)
    sMax = steps * nblocks
    for s in range(0, sMax, steps):
        r, _ = computeOtOtp(arr1[s:s + steps], arr2[s:s + steps + nTMax], conn=False, nTMax=nTMax, decim=decim)
        res.append(r)
    return np.asarray(res)

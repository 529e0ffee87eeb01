"""Regenerate tests/golden/otot.json: outputs of the reference's own time
correlators (python/Loader.py:229-300, computeOtOtp, computeBlockedOtOtp,
blockedOtOtp), imported from the reference tree and run on seeded synthetic
series.  Run in a container that has the reference sources mounted.

Loader.py imports h5py at module level for its file loaders; the correlators do
not use it, and h5py is not installed here, so an empty stand-in module is put
in sys.modules before the import.

The inputs are not stored: tests rebuild them from the recorded seeds with
series(seed, T, ncol, complex).

Usage:  python tests/golden/make_postprocess_golden.py --ref <reference python directory>
"""
import argparse
import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def series(seed, T, ncol, cplx):
    """AR(1) series with a nonzero mean, [T, ncol] (complex if cplx)."""
    rng = np.random.default_rng(seed)
    x = np.zeros((T, ncol), dtype=np.complex128 if cplx else np.float64)
    e = rng.normal(size=(T, ncol)) + (1j * rng.normal(size=(T, ncol)) if cplx else 0)
    x[0] = e[0]
    for t in range(1, T):
        x[t] = 0.8 * x[t - 1] + e[t]
    return x + 0.3


def enc(a):
    a = np.asarray(a)
    if np.iscomplexobj(a):
        return {"re": a.real.tolist(), "im": a.imag.tolist()}
    return {"re": a.tolist()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's python directory")
    a = ap.parse_args()
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    spec = importlib.util.spec_from_file_location("reference_loader", os.path.join(a.ref, "Loader.py"))
    Loader = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(Loader)

    cases = []
    for seed, T, cplx, conn, nTMax, decim in [(1, 97, False, False, -1, 1), (2, 97, False, True, 40, 1),
                                             (3, 120, True, False, 33, 1), (4, 120, True, True, 50, 3),
                                             (5, 64, False, False, 64, 2), (6, 5, True, False, -1, 1)]:
        x = series(seed, T, 1, cplx)[:, 0]
        y = series(seed + 100, T, 1, cplx)[:, 0]
        arr2 = np.conj(y) if cplx else y
        C, E = Loader.computeOtOtp(x, arr2, conn=conn, nTMax=nTMax, decim=decim)
        cases.append({"fn": "computeOtOtp", "seed": seed, "T": T, "complex": cplx, "conn": conn, "nTMax": nTMax,
                      "decim": decim, "conj_b": cplx, "out": enc(C)})
    for seed, T, cplx, nTMax, steps, decim, conn in [(7, 130, True, 10, 25, 1, False), (8, 100, False, 8, 30, 2, True)]:
        x = series(seed, T, 1, cplx)[:, 0]
        y = series(seed + 100, T, 1, cplx)[:, 0]
        R = Loader.computeBlockedOtOtp(x, y, nTMax, steps, decim=decim, conn=conn)
        cases.append({"fn": "computeBlockedOtOtp", "seed": seed, "T": T, "complex": cplx, "nTMax": nTMax,
                      "steps": steps, "decim": decim, "conn": conn, "out": enc(R)})
    for seed, T, cplx, nTMax, nblocks, decim in [(9, 150, False, 12, 4, 1), (10, 140, True, 9, 3, 2)]:
        x = series(seed, T, 1, cplx)[:, 0]
        y = series(seed + 100, T, 1, cplx)[:, 0]
        R = Loader.blockedOtOtp(x, y, nTMax, nblocks, decim=decim)
        cases.append({"fn": "blockedOtOtp", "seed": seed, "T": T, "complex": cplx, "nTMax": nTMax,
                      "nblocks": nblocks, "decim": decim, "out": enc(R)})
    doc = {"source": "python/Loader.py:229-300 (computeOtOtp, computeBlockedOtOtp, blockedOtOtp), run as is",
           "series": "tests/golden/make_postprocess_golden.py:series(seed, T, 1, complex)[:, 0] for a, "
                     "seed + 100 for b (conjugated for computeOtOtp on complex cases)",
           "cases": cases}
    with open(os.path.join(HERE, "otot.json"), "w") as f:
        json.dump(doc, f)


if __name__ == "__main__":
    main()

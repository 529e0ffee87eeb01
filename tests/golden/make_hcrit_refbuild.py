"""Equilibrium of the reference's own heat bath at the hcrit1 point -> hcrit1_refbuild.json.

Runs oracle/_ref/ref_stepper -- the reference's unmodified Stepper.cxx,
NoiseGenerator.cxx and measurer.cxx built against the PETSc/MPI/FFTW stand-ins
of oracle/shim/ (make -C oracle ref REF=<reference ModelG directory>) -- as
independent single-rank runs: N = 32, m^2 = -4.813, lambda = 4, H = 0.01,
Gamma = 1, dt = 0.1 (the heat bath's equilibrium does not depend on dt), phi
from 0.3 N(0,1) of the reference's stream, 4000 thermalisation sweeps of
EulerLangevinHB, then Measurer::measure every 25 sweeps, 8000 times.  Each
run takes about 20 minutes on one core.

    python tests/golden/make_hcrit_refbuild.py [--seeds 101 ... 107] [--samples DIR]

The per-run OAverage samples go to DIR (default: a temporary directory); with
--analyse-only the samples already in DIR are analysed without running.
"""
import argparse
import concurrent.futures as cf
import glob
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))

PARAMS = dict(N=32, mass0=-4.813, lam=4.0, H=0.01, gamma=1.0, dt=0.1)
THERM, SAMPLES, EVERY = 4000, 8000, 25


def run_one(seed, outdir):
    import refbuild

    P = refbuild.params_json(PARAMS["N"], mass0=PARAMS["mass0"], lam=PARAMS["lam"], H=PARAMS["H"],
                             gamma=PARAMS["gamma"], seed=seed, dt=PARAMS["dt"])
    r = refbuild.run(P, ["phi=0.3", f"step=EulerLangevinHB,{THERM}", f"sample=EulerLangevinHB,{SAMPLES},{EVERY}"],
                     timeout=20000)
    np.save(os.path.join(outdir, f"ref_{seed}.npy"), r.averages)
    return seed


def blocked_err(x, nb=40):
    n = len(x) // nb * nb
    b = x[:n].reshape(nb, -1).mean(axis=1)
    return float(b.std(ddof=1) / np.sqrt(nb))


def analyse(outdir):
    files = sorted(glob.glob(os.path.join(outdir, "ref_*.npy")))
    runs = [np.load(f) for f in files]
    out = {"source": "oracle/_ref/ref_stepper (the reference's EulerLangevinHB and Measurer, unmodified)",
           "params": PARAMS, "thermalisation_sweeps": THERM, "samples_per_run": SAMPLES, "sweeps_per_sample": EVERY,
           "seeds": [int(os.path.basename(f)[4:-4]) for f in files]}
    for col, name in ((0, "phi0"), (10, "phi2")):
        means = np.array([r[:, col].mean() for r in runs])
        err_spread = float(means.std(ddof=1) / np.sqrt(len(means)))
        err_blocked = float(np.sqrt(sum(blocked_err(r[:, col]) ** 2 for r in runs)) / len(runs))
        out[name] = {"mean": float(means.mean()), "err": max(err_spread, err_blocked), "err_spread": err_spread,
                     "err_blocked": err_blocked, "run_means": [float(m) for m in means]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, nargs="+", default=[101, 102, 103, 104, 105, 106, 107])
    ap.add_argument("--samples", default=None)
    ap.add_argument("--analyse-only", action="store_true")
    a = ap.parse_args()
    outdir = a.samples or tempfile.mkdtemp(prefix="hcrit_ref_")
    if not a.analyse_only:
        with cf.ProcessPoolExecutor(max_workers=len(a.seeds)) as ex:
            list(ex.map(run_one, a.seeds, [outdir] * len(a.seeds)))
    res = analyse(outdir)
    with open(os.path.join(HERE, "hcrit1_refbuild.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({k: res[k] for k in ("phi0", "phi2")}))


if __name__ == "__main__":
    main()

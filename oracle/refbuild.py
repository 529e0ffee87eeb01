"""TEST INFRASTRUCTURE ONLY: runs the oracle's reference build.

`_ref/ref_stepper` is the reference's own Stepper.cxx, NoiseGenerator.cxx and
measurer.cxx compiled unmodified against the PETSc/MPI/FFTW stand-ins of
oracle/shim/ (`make -C oracle ref REF=<reference ModelG directory>`).  This
module writes its input file (the reference's JSON keys, ModelA.h:55-159,
185-248), runs it, and parses what it returns: states, measurements in the
packing of lgv_measure_device, energies, the per-operation wall times, the
PetscLogEvent timers and the accept statistics the reference prints from its
steppers' finalize() (Stepper.h:51-82).

Only tests/ and bench.py's reference arm use it.
"""
import json
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BINARY = os.path.join(HERE, "_ref", "ref_stepper")

NOBS, NOBS_PHASE = 11, 14


def available():
    return os.path.exists(BINARY)


def params_json(N, mass0=-4.813, lam=10.0, H=0.01, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=10, dt=0.04,
                dmassdt=0.0, t0=0.0):
    """The reference's input keys (ModelA.h:55-159, 222-248)."""
    return {"NX": int(N), "mass0": mass0, "dmassdt": dmassdt, "lambda": lam, "H": H, "chi": chi, "gamma": gamma,
            "diffusion": diffusion, "seed": int(seed), "deltat": dt, "initialtime": t0,
            "finaltime": t0 + 1000 * dt, "saveFrequency": 1, "evolverType": "PV2HBSplit23",
            "outputfiletag": "ref_stepper"}


def unpack_measurement(N, v):
    """Split one packed measurement (the field order of lgv_measurement)."""
    NK = N // 2 + 1
    sizes = ([("OAverage", (NOBS,))]
             + [(f"wall{a}", (NOBS, N)) for a in "XYZ"]
             + [(f"wall{a}_k", (NOBS, NK, 2)) for a in "XYZ"]
             + [(f"wall{a}_k_rotated", (NOBS_PHASE, NK, 2)) for a in "XYZ"]
             + [(f"wall{a}Phase", (NOBS_PHASE, N)) for a in "XYZ"]
             + [(f"wall{a}Phase_k", (NOBS_PHASE, NK, 2)) for a in "XYZ"])
    out, o = {}, 0
    for name, shp in sizes:
        n = int(np.prod(shp))
        out[name] = v[o:o + n].reshape(shp)
        o += n
    assert o == v.size, (o, v.size)
    return out


_STAT = re.compile(r"==== Statistics for (.+?) ====")


def parse_stats(text):
    """Integer accept counts of o4_stepper_monitor::print (Stepper.h:51-82)."""
    stats, cur = {}, None
    for line in text.splitlines():
        m = _STAT.search(line)
        if m:
            cur = stats.setdefault(m.group(1), {})
            continue
        if cur is None:
            continue
        m = re.match(r"dS >0: accepts = (\d+);", line)
        if m:
            cur["up_yes"] = int(m.group(1))
        m = re.match(r"dS =0: rejects = (\d+);", line)
        if m:
            cur["up_no"] = int(m.group(1))
        m = re.match(r"dS>=0: counts  = (\d+);", line)
        if m:
            cur["up_counts"] = int(m.group(1))
        m = re.match(r"dS <0: counts  = (\d+);", line)
        if m:
            cur["down_counts"] = int(m.group(1))
    return stats


class Result:
    def __init__(self, N, records, stdout):
        self.N = N
        self.states = [v.reshape(N, N, N, 10) for t, v in records if t == 1]
        self.measurements = [unpack_measurement(N, v) for t, v in records if t == 2]
        self.energies = [float(v[0]) for t, v in records if t == 3]
        self.averages = np.array([v for t, v in records if t == 4]).reshape(-1, NOBS)
        self.stdout = stdout
        self.times = [(m.group(1), float(m.group(2))) for m in re.finditer(r"^REFTIME (\S+) (\S+)$", stdout, re.M)]
        self.events = {m.group(1): (float(m.group(2)), int(m.group(3)))
                       for m in re.finditer(r"^REFEVENT (.+) (\S+) (\d+)$", stdout, re.M)}
        self.stats = parse_stats(stdout)


def run(params, ops, state=None, ranks=1, timeout=3600, workdir=None):
    """Run the reference build: `ops` as documented in ref_stepper_main.cpp.

    `state` (N^3 x 10 doubles, u[k][j][i][L]) is loaded first when given.
    """
    if not available():
        raise RuntimeError("oracle/_ref/ref_stepper is not built (make -C oracle ref REF=...)")
    N = int(params["NX"])
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        pj = os.path.join(d, "params.json")
        with open(pj, "w") as f:
            json.dump(params, f)
        ob = os.path.join(d, "out.bin")
        pre = []
        if state is not None:
            sp = os.path.join(d, "state.bin")
            np.ascontiguousarray(state, dtype=np.float64).tofile(sp)
            pre = ["load=" + sp]
        cmd = [BINARY, "--ranks", str(int(ranks)), pj, ob] + pre + list(ops)
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=d)
        if r.returncode != 0:
            raise RuntimeError(f"ref_stepper failed ({r.returncode}): {r.stderr[-2000:]}")
        records = []
        with open(ob, "rb") as f:
            buf = f.read()
        o = 0
        while o < len(buf):
            tag = int(np.frombuffer(buf, np.uint32, 1, o)[0])
            n = int(np.frombuffer(buf, np.uint64, 1, o + 4)[0])
            records.append((tag, np.frombuffer(buf, np.float64, n, o + 12).copy()))
            o += 12 + 8 * n
    return Result(N, records, r.stdout)

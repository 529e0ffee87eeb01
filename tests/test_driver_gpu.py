"""The superpions driver end to end on the GPU.

- Its measurement series equals the same run made through the Python API
  (same library, same counter streams): the driver adds no arithmetic.
- Restart: N steps, then a restart run of N more steps (state from
  <tag>_save.npy, noise counter from <tag>_0.rng) ends in exactly the state
  of one run of 2N steps (the reference's restart semantics,
  SuperPions.cxx:84-86, 107-110, ModelA.h:330-332)."""
import json
import math
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def driver():
    import importlib.util

    spec = importlib.util.spec_from_file_location("b", os.path.join(REPO, "langevina_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b.build_driver()


def run(cfg, cwd):
    (cwd / "in.json").write_text(json.dumps(cfg))
    r = subprocess.run([driver(), "-input", "in.json"], cwd=cwd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


BASE = {"NX": 8, "deltat": 0.04, "mass0": -4.813, "lambda": 10, "H": 0.006, "chi": 5.0, "diffusion": 1 / 3,
        "evolverType": "PV2HBSplit23", "seed": 11, "saveFrequency": 2, "thermalization_time": 0.08,
        "outputfiletag": "run"}


def test_driver_matches_python_api(lgv, tmp_path):
    cfg = dict(BASE, finaltime=0.4)
    run(cfg, tmp_path)
    phi = np.fromfile(tmp_path / "run.phi.f64").reshape(-1, 11)
    tout = np.fromfile(tmp_path / "run.timeout.f64").reshape(-1, 2)
    idx = json.loads((tmp_path / "run.datasets.json").read_text())
    assert idx["wallx_k"] == [11, 5, 2] and idx["phi"] == [11]

    from langevina_b200 import _lib as L

    data = lgv.ModelAData(dict(cfg))
    model = lgv.ModelA(data)
    model.initialize()
    model.initialize_gaussian_charges()
    dt = data.atime.dt()
    for _ in range(int(data.ahandler.thermalization_time / dt) * 6):
        L.check(model.lib.lgv_step(model.handle, L.EULER_LANGEVIN_HB, 1, 1, dt / 6, data.atime.t(), 1), "thermalize")
    step = lgv.make_stepper(model, "PV2HBSplit23")
    meas = lgv.Measurer(model)
    rows, steps = [], 0
    while data.atime.t() < data.atime.tfinal() - 1e-10:
        if steps % data.ahandler.saveFrequency == 0:
            rows.append(meas.measure().OAverage.copy())
        step.step(dt)
        steps += 1
        data.atime += dt
    assert phi.shape == (len(rows), 11) and len(rows) == 5
    assert np.array_equal(phi, np.array(rows))
    assert np.allclose(tout[:, 0], np.arange(5) * 2 * dt) and np.all(tout[:, 1] == -4.813)


def test_restart_continues_the_run(lgv, tmp_path):
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    run(dict(BASE, finaltime=0.8), a)
    run(dict(BASE, finaltime=0.4), b)
    run(dict(BASE, finaltime=0.4, restart=True), b)
    ua = np.load(a / "run_save.npy")
    ub = np.load(b / "run_save.npy")
    assert ua.shape == (8, 8, 8, 10)
    assert np.array_equal(ua, ub)
    ca = (a / "run_0.rng").read_text().split()
    cb = (b / "run_0.rng").read_text().split()
    assert ca[2] == cb[2]  # device counter
    pa = np.fromfile(a / "run.phi.f64").reshape(-1, 11)
    pb = np.fromfile(b / "run.phi.f64").reshape(-1, 11)
    assert pa.shape == pb.shape == (10, 11)
    assert np.array_equal(pa, pb)


def test_driver_event_mode_and_quench(lgv, tmp_path):
    cfg = dict(BASE, finaltime=0.16, eventmode=True, nevents=2, quench_mode=True, quench_mode_mass0=-3.0)
    out = run(cfg, tmp_path)
    assert "Settinng up a quench initial condition with initial mass -3.000000e+00" in out
    for e in range(2):
        phi = np.fromfile(tmp_path / f"run_{e:04d}.phi.f64").reshape(-1, 11)
        assert phi.shape == (2, 11) and np.all(np.isfinite(phi))
    assert not (tmp_path / "run_save.npy").exists()  # event mode writes no restart state

"""The C++ host layer (include/langevina.hpp) and the superpions driver, on
the CPU: a compiled check program (JSON input keys and defaults, host noise
stream against the reference engine's golden draws, .npy files) and the
driver's -quit path, which parses the input and exits before any GPU call."""
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_host_api_program(tmp_path):
    exe = tmp_path / "host_api_test"
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", os.path.join(REPO, "include"),
                           os.path.join(REPO, "tests", "cpp", "host_api_test.cpp"), "-o", str(exe)])
    r = subprocess.run([str(exe), os.path.join(REPO, "tests", "golden", "ref_xoro.txt")], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"
    a = np.load(tmp_path / "host_api_test.npy")
    assert a.shape == (2, 3) and a[0, 1] == -2.0


def test_driver_quit_parses_reference_style_input(tmp_path):
    import importlib.util

    spec = importlib.util.spec_from_file_location("b", os.path.join(REPO, "langevina_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    drv = b.build_driver()
    cfg = tmp_path / "in.json"
    cfg.write_text('{\n "NX": 16,\n "finaltime": 3.0,\n "deltat": 0.6,\n "saveFrequency": 3,\n'
                   ' "evolverType": "PV2HBSplit23",\n "seed": 7,\n}\n')
    r = subprocess.run([drv, "-input", str(cfg), "-quit"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "finaltime = 1.800000e+00" in r.stdout
    assert "evolverType = PV2HBSplit23" in r.stdout
    r = subprocess.run([drv, "-input", str(tmp_path / "missing.json")], capture_output=True, text=True)
    assert r.returncode != 0 and "Unable to open input file" in r.stderr

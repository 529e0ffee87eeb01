"""The post-processing restatement (oracle/postprocess.py) pinned on the CPU:

- the time correlators against the reference's own Loader.py outputs
  (tests/golden/otot.json, made by tests/golden/make_postprocess_golden.py);
- x2k on the test signal of ModelG/x2ktest.py (cos and sin of 2 pi k x / 8,
  k = 0, 1, 2): single modes of weight 1 (k = 0) or 1/2;
- x2k_rotated known answers: for n = (1, 0, 0, 0) the rotated A and V rows are
  (0, A_1..3) and (0, V_1..3), phi splits into its n part and the rest;
- both transforms reproduce the C++ oracle's measurer (its k walls and
  rotated k walls) on a random lattice.
"""
import importlib.util
import json
import os

import numpy as np
import pytest

import postprocess as P  # oracle/postprocess.py (test infrastructure)

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def golden_series():
    spec = importlib.util.spec_from_file_location("make_pp_golden", os.path.join(GOLD, "make_postprocess_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.series


def dec(o):
    re = np.array(o["re"])
    return re + 1j * np.array(o["im"]) if "im" in o else re


def golden_cases():
    with open(os.path.join(GOLD, "otot.json")) as f:
        return json.load(f)["cases"]


def case_inputs(c, series):
    x = series(c["seed"], c["T"], 1, c["complex"])[:, 0]
    y = series(c["seed"] + 100, c["T"], 1, c["complex"])[:, 0]
    if c["fn"] == "computeOtOtp" and c["conj_b"]:
        y = np.conj(y)
    return x, y


def run_case(mod, c, x, y):
    if c["fn"] == "computeOtOtp":
        return mod.computeOtOtp(x, y, conn=c["conn"], nTMax=c["nTMax"], decim=c["decim"])[0]
    if c["fn"] == "computeBlockedOtOtp":
        return mod.computeBlockedOtOtp(x, y, c["nTMax"], c["steps"], decim=c["decim"], conn=c["conn"])
    return mod.blockedOtOtp(x, y, c["nTMax"], c["nblocks"], decim=c["decim"])


@pytest.mark.parametrize("i", range(10))
def test_correlators_match_reference_loader(i):
    series = golden_series()
    c = golden_cases()[i]
    x, y = case_inputs(c, series)
    got = run_case(P, c, x, y)
    want = dec(c["out"])
    assert got.shape == want.shape
    assert np.allclose(got, want, rtol=1e-13, atol=1e-13)


def x2ktest_signal(size=8):
    x = np.arange(size, dtype=np.float64)
    d = np.zeros((2, 3, size))
    for k in range(3):
        d[0, k] = np.cos(2 * np.pi * k * x / size)
        d[1, k] = np.sin(2 * np.pi * k * x / size)
    return d


def test_x2k_single_modes():
    w = P.x2k(x2ktest_signal())  # [2, 3, 5, 2]
    want = np.zeros_like(w)
    want[0, 0, 0, 0] = 1.0
    for k in (1, 2):
        want[0, k, k, 0] = 0.5
        want[1, k, k, 1] = -0.5
    assert np.allclose(w, want, atol=1e-15)


def test_x2k_rotated_known_answers():
    rng = np.random.default_rng(3)
    NK = 5
    wk = rng.normal(size=(2, 10, NK, 2))
    wk[0, 0:4, 0, :] = [[2.0, 0.0], [0, 0], [0, 0], [0, 0]]  # n = (1, 0, 0, 0)
    wk[1, 0:4, 0, :] = 0.0  # below DBL_MIN: the identity direction
    out = P.x2k_rotated(wk)
    for r in range(2):
        c = wk[r, :, :, 0] + 1j * wk[r, :, :, 1]
        o = out[r, :, :, 0] + 1j * out[r, :, :, 1]
        assert np.allclose(o[0], c[0])  # phi along n
        assert np.allclose(o[1], 0) and np.allclose(o[2:5], c[1:4])  # the rest
        assert np.allclose(o[5], 0) and np.allclose(o[6:9], c[4:7])  # A
        assert np.allclose(o[9], 0) and np.allclose(o[10:13], c[7:10])  # V


def test_x2k_rotated_is_a_rotation_of_phi():
    rng = np.random.default_rng(4)
    wk = rng.normal(size=(3, 11, 4, 2))
    out = P.x2k_rotated(wk)
    c = wk[..., 0] + 1j * wk[..., 1]
    o = out[..., 0] + 1j * out[..., 1]
    n = wk[:, 0:4, 0, 0] / np.linalg.norm(wk[:, 0:4, 0, 0], axis=1, keepdims=True)
    # phi = n phis + phir with phir orthogonal to n
    assert np.allclose(n[:, :, None] * o[:, None, 0] + o[:, 1:5], c[:, 0:4])
    assert np.allclose(np.einsum("ra,rak->rk", n, o[:, 1:5]), 0)


def test_restatements_agree_with_the_measurer_restatement(oracle_mod):
    """x2k and x2k_rotated restated here reproduce the C++ oracle's measurer
    (measurer.cxx: r2c walls / N and rotate_to_vev) on a random lattice."""
    from langevina_b200 import _lib as L

    N = 8
    o = oracle_mod.Oracle(N, mode=oracle_mod.COUNTER, seed=5)
    rng = np.random.default_rng(12)
    u = np.zeros((N, N, N, 10))
    u[..., :4] = 0.4 * rng.normal(size=(N, N, N, 4)) + np.array([0.5, 0.1, -0.2, 0.05])
    u[..., 4:] = rng.normal(size=(N, N, N, 6))
    o.set_state(u)
    m = o.measure(L.Measurement(N))
    for a in range(3):
        assert np.allclose(P.x2k(m.wall[a]), m.wall_k[a], rtol=1e-12, atol=1e-14)
        assert np.allclose(P.x2k(m.wall_phase[a]), m.wall_phase_k[a], rtol=1e-12, atol=1e-14)
        assert np.allclose(P.x2k_rotated(m.wall_k[a][None])[0], m.wall_k_rotated[a][:13], rtol=1e-12, atol=1e-14)

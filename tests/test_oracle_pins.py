"""Pins of the CPU oracle against the reference's own golden data.

- The serial noise stream (seed_seq -> xoroshiro128+ -> libstdc++ distributions)
  against the output of the reference engine ModelG/xoroshiro128plus.h compiled
  from source (tests/golden/ref_xoro.txt, made by tests/golden/make_golden.py).
- O(4) rotation sign conventions: known answers of ModelG/O4AlgebraSignTest.cxx:20-39.
- Single-link charge heat bath chain of ModelG/q_heatbathtest.cxx:121-137 (t1):
  n_A is Gaussian about (nA+nB)/2 with variance chi/2; nA + nB is conserved.
"""
import json
import math
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _records():
    recs = []
    with open(os.path.join(GOLD, "ref_xoro.txt")) as f:
        for line in f:
            recs.append(line.split())
    return recs


def test_seed_seq_matches_reference(oracle_mod):
    n = 0
    for r in _records():
        if r[0] != "seeds":
            continue
        base, size = int(r[1]), int(r[2])
        want = np.array([int(x) for x in r[3:]], dtype=np.uint32)
        assert np.array_equal(oracle_mod.seed_seq(base, size), want)
        n += 1
    assert n >= 6


@pytest.mark.parametrize("kind", ["raw", "unif", "var1", "norm"])
def test_serial_stream_matches_reference(oracle_mod, kind):
    n = 0
    for r in _records():
        if r[0] != kind:
            continue
        base, rank, size, cnt = map(int, r[1:5])
        got = oracle_mod.seq_draws(base, rank, size, kind, cnt)
        if kind == "raw":
            want = np.array([int(x) for x in r[5:]], dtype=np.uint64)
            assert np.array_equal(got, want), (base, rank, size)
        else:
            want = np.array([float(x) for x in r[5:]])
            assert np.array_equal(got, want), (kind, base, rank, size)  # bit-exact
        n += 1
    assert n >= 15


def test_engine_state_and_restart_format(oracle_mod):
    """xoroshiro128plus::seed(uint64) state and stream (.rng text format 's0 s1')."""
    for r in _records():
        if r[0] != "state":
            continue
        s0, s1, cnt = int(r[2]), int(r[3]), int(r[4])
        want = np.array([int(x) for x in r[5:]], dtype=np.uint64)
        assert np.array_equal(oracle_mod.xoro_raw(s0, s1, cnt), want)


def test_o4_sign_conventions(oracle_mod):
    with open(os.path.join(GOLD, "o4_known.json")) as f:
        known = json.load(f)
    for c in known["cases"]:
        got = oracle_mod.o4_rotation(c["V"], c["A"], c["phi"])
        assert np.allclose(got, c["expect"], atol=1e-15, rtol=0), (c, got)


def test_o4_rotation_preserves_norm(oracle_mod):
    rng = np.random.default_rng(3)
    for _ in range(200):
        V, A, phi = rng.normal(size=3), rng.normal(size=3), rng.normal(size=4)
        got = oracle_mod.o4_rotation(V, A, phi)
        assert abs(np.linalg.norm(got) - np.linalg.norm(phi)) < 1e-13 * np.linalg.norm(phi)
    # identity below |v| = 1e-20 (O4AlgebraHelper.h:66-75)
    got = oracle_mod.o4_rotation([0, 0, 0], [0, 0, 0], [0.3, -0.2, 0.1, 0.7])
    assert np.array_equal(got, [0.3, -0.2, 0.1, 0.7])


def test_charge_pair_chain_distribution(oracle_mod):
    chi = 0.9  # q_heatbathtest.json
    dt, sigma = 0.5, 1.66666666 * chi
    rms = math.sqrt(2.0 * dt * sigma)
    nA, nB = oracle_mod.charge_pair_chain(chi, rms, 2.0, 1.0, 122335456, 500000)
    tot = nA + nB
    assert np.max(np.abs(tot - 3.0)) < 1e-10
    x = nA[1000:]
    mean, var = x.mean(), x.var()
    # equilibrium of exp(-(nA^2 + nB^2)/(2 chi)) at fixed nA + nB = 3
    assert abs(mean - 1.5) < 0.02
    assert abs(var - chi / 2) < 0.03 * chi / 2


def test_counter_stream_moments(oracle_mod):
    seed = 2021
    draws = np.concatenate([oracle_mod.ctr_draws(seed, c, n, 8) for c in range(4) for n in range(2000)])
    u = (draws >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    assert abs(u.mean() - 0.5) < 0.01
    v = (2 * u - 1) * math.sqrt(3)
    assert abs(v.var() - 1.0) < 0.02
    # streams of neighbouring sites are uncorrelated
    a = np.array([oracle_mod.ctr_draws(seed, 0, n, 1)[0] for n in range(4000)])
    b = np.array([oracle_mod.ctr_draws(seed, 0, n + 1, 1)[0] for n in range(4000)])
    ua = (a >> np.uint64(11)).astype(np.float64)
    ub = (b >> np.uint64(11)).astype(np.float64)
    assert abs(np.corrcoef(ua, ub)[0, 1]) < 0.05


def test_counter_order_covers_all_faces(oracle_mod):
    seen = set()
    for c in range(200):
        o = oracle_mod.ctr_order(77, c)
        assert sorted(o[:3]) == [0, 1, 2] and sorted(o[3:]) == [0, 1]
        seen.add(tuple(o))
    assert len(seen) == 12

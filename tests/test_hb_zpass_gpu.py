"""The z-marching one-parity heat-bath pass (hb_zpass_kernel, opt-in with
LGV_HB_ZPASS=1 for half rows of at least 32 elements, N >= 64): the oracle's
decisions and states for counter and injected noise, with per-site flags and
accept statistics, on lattices whose half rows fill the 32-element tile
exactly (64, 128), leave a ragged last tile in x (66, 70, 98) or in y and z
(N not a multiple of the 8-row tile: 66, 70, 98, 130).

The library reads LGV_HB_ZPASS once per process, so the cases run in a fresh
child process with it set.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HB = 4
INJECTED = 1
COEF = dict(mass0=-4.813, lam=10.0, H=0.01, chi=5.0, gamma=1.0, diffusion=1.0 / 3.0, seed=4417)


def case_counter(N):
    import oracle
    from lgvtest import GpuLattice, assert_state_close, compare_flags, rand_state

    g = GpuLattice(None, N, **COEF)
    o = oracle.Oracle(N, mode=oracle.COUNTER, **COEF)
    u = rand_state(N, 50 + N)
    g.set_state(u)
    o.set_state(u)
    g.flags(True)
    o.debug_flags(True)
    g.monitors(True)
    g.step(HB, 0.02, nsteps=2)
    o.step(HB, 0.02, nsteps=2)
    assert compare_flags(g.get_flags(), o.get_flags(), N ** 3) == 0
    assert_state_close(g.get_state(), o.get_state(), what="z-marching pass")
    mg, mo = g.monitors()[1], o.monitor(1)
    for k in ("down_counts", "up_counts", "up_yes", "up_no"):
        assert mg[k] == mo[k], k


def case_injected(N):
    import oracle
    from lgvtest import GpuLattice, assert_state_close, compare_flags, hb_noise, rand_state

    g = GpuLattice(None, N, **COEF)
    o = oracle.Oracle(N, mode=oracle.INJECTED, **COEF)
    u = rand_state(N, 90 + N)
    g.set_state(u)
    o.set_state(u)
    g.mode(INJECTED)
    g.flags(True)
    o.debug_flags(True)
    prop, acc = hb_noise(N, 5)
    g.inject_hb(prop, acc)
    o.inject_hb(prop, acc)
    g.step(HB, 0.05)
    o.step(HB, 0.05)
    assert compare_flags(g.get_flags(), o.get_flags(), N ** 3) == 0
    assert_state_close(g.get_state(), o.get_state(), what="z-marching pass injected")


@pytest.mark.gpu
def test_zpass_matches_oracle_in_child_process(lgv):
    env = dict(os.environ, LGV_HB_ZPASS="1")
    r = subprocess.run([sys.executable, os.path.abspath(__file__)], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "zpass cases ok" in r.stdout


if __name__ == "__main__":
    repo = os.path.dirname(HERE)
    for p in (HERE, repo, os.path.join(repo, "oracle")):
        sys.path.insert(0, p)
    import torch

    assert torch.cuda.is_available()
    for N in (64, 66, 70, 98, 128, 130):
        case_counter(N)
    for N in (64, 70):
        case_injected(N)
    print("zpass cases ok")

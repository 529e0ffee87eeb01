"""CPU checks of the numpy restatement of the Euler-Maruyama adjoint
(oracle/em_adjoint.py): its forward against the oracle's em_step, and its
gradient against central finite differences with common random numbers."""
import numpy as np
import pytest

from lgvtest import rand_state

SEED = 977
THETA = np.array([-4.813, 10.0, 0.01, 1.0])  # (m^2, lambda, H, Gamma)


@pytest.fixture(scope="module")
def ema(oracle_mod):
    import em_adjoint
    return em_adjoint


def test_numpy_forward_matches_oracle_em_step(oracle_mod, ema):
    N, S = 4, 6
    u = rand_state(N, 5)
    o = oracle_mod.Oracle(N, mode=oracle_mod.COUNTER, mass0=THETA[0], lam=THETA[1], H=THETA[2], gamma=THETA[3],
                          dmassdt=-0.3, seed=SEED)
    o.set_state(u)
    o.set_counter(11)
    o.step(6, 0.02, t=0.5, nsteps=S)
    phis = ema.em_run(u[..., :4], THETA, 0.02, S, SEED, 11, t0=0.5, dmassdt=-0.3)
    np.testing.assert_allclose(phis[-1], o.get_state()[..., :4], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("w", [(1.0, 1.0), (1.0, 0.0), (0.0, 1.0)])
def test_numpy_adjoint_matches_central_fd(ema, w):
    N, S, b, dt, h = 4, 30, 10, 0.02, 1e-5
    phi0 = rand_state(N, 7)[..., :4]
    g = ema.em_gradient(ema.em_run(phi0, THETA, dt, S, SEED, 3), THETA, dt, b, SEED, 3, w=w)
    fd = np.zeros(4)
    for i in range(4):
        e = np.zeros(4)
        e[i] = h
        jp = np.dot(w, ema.observables(ema.em_run(phi0, THETA + e, dt, S, SEED, 3), b))
        jm = np.dot(w, ema.observables(ema.em_run(phi0, THETA - e, dt, S, SEED, 3), b))
        fd[i] = (jp - jm) / (2 * h)
    scale = np.max(np.abs(fd))
    assert scale > 0
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-6 * scale)

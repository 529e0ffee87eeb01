"""CPU checks of the numpy restatement of the differentiable runs and their
adjoints (oracle/diff_adjoint.py): the forward steps against the oracle's
em_step and ideal_step, the rotation adjoint against directional finite
differences, and the run gradients against central finite differences with
common random numbers."""
import numpy as np
import pytest

from lgvtest import rand_state

SEED = 977
THETA = np.array([-4.813, 10.0, 0.01, 1.0])  # (m^2, lambda, H, Gamma)
EM, IDEAL = 6, 3


@pytest.fixture(scope="module")
def da(oracle_mod):
    import diff_adjoint
    return diff_adjoint


def test_numpy_em_matches_oracle_em_step(oracle_mod, da):
    N, S = 4, 6
    u = rand_state(N, 5)
    o = oracle_mod.Oracle(N, mode=oracle_mod.COUNTER, mass0=THETA[0], lam=THETA[1], H=THETA[2], gamma=THETA[3],
                          dmassdt=-0.3, seed=SEED)
    o.set_state(u)
    o.set_counter(11)
    o.step(EM, 0.02, t=0.5, nsteps=S)
    us = da.Run("em", THETA, 0.02, SEED, 11, t0=0.5, dmassdt=-0.3).forward(u, S)
    np.testing.assert_allclose(us[-1], o.get_state(), rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("N,H", [(4, 0.01), (6, 0.3)])
def test_numpy_ideal_matches_oracle_ideal_step(oracle_mod, da, N, H):
    u = rand_state(N, 8)
    o = oracle_mod.Oracle(N, mode=oracle_mod.COUNTER, H=H, chi=5.0, seed=SEED)
    o.set_state(u)
    o.step(IDEAL, 0.04, nsteps=3)
    v = u
    for _ in range(3):
        v = da.ideal(v, 0.04, 5.0, H, 1.0)
    np.testing.assert_allclose(v, o.get_state(), rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("scale", [1e-3, 0.2, 3.0])
def test_rotation_adjoint_directional_fd(da, scale):
    rng = np.random.default_rng(4)
    phi = rng.normal(size=(50, 4))
    q = scale * rng.normal(size=(50, 6))
    k = 0.37
    ob = rng.normal(size=(50, 4))
    dphi, dq = rng.normal(size=(50, 4)), rng.normal(size=(50, 6))
    pb, qb = da.rot_adj(phi, q, k, ob)
    h = 1e-6
    f = lambda t: np.sum(ob * da.rot(phi + t * dphi, q + t * dq, k))
    fd = (f(h) - f(-h)) / (2 * h)
    an = np.sum(pb * dphi) + np.sum(qb * dq)
    assert abs(an - fd) <= 1e-8 * max(1.0, abs(fd))


@pytest.mark.parametrize("scheme", ["em", "ideal", "ideal_em"])
@pytest.mark.parametrize("w", [(1.0, 1.0), (1.0, 0.0), (0.0, 1.0)])
def test_numpy_adjoint_matches_central_fd(da, scheme, w):
    N, S, b, dt, h = 4, 20, 6, 0.02, 1e-5
    u0 = rand_state(N, 7)
    theta = THETA.copy()
    theta[2] = 0.3  # a larger H so the ideal step's -H phi source is visible
    run = lambda th: da.Run(scheme, th, dt, SEED, 3)
    r = run(theta)
    g = r.gradient(r.forward(u0, S), b, w=w)
    fd = np.zeros(4)
    for i in range(4):
        e = np.zeros(4)
        e[i] = h
        jp = np.dot(w, da.Run.observables(run(theta + e).forward(u0, S), b))
        jm = np.dot(w, da.Run.observables(run(theta - e).forward(u0, S), b))
        fd[i] = (jp - jm) / (2 * h)
    scale = np.max(np.abs(fd))
    assert scale > 0
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-7 * scale)
    if scheme == "ideal":
        assert g[0] == 0 and g[1] == 0 and g[3] == 0

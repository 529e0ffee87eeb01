"""GPU checks of the differentiable runs (lgv_diff_forward / lgv_diff_backward
and the torch.autograd.Function over them): Euler-Maruyama Model A ("em"),
the ideal O(4) rotation step ("ideal") and the two in sequence ("ideal_em").

- the time averages and the adjoint gradient against the numpy restatement of
  the runs and their adjoints (oracle/diff_adjoint.py), on the same counter
  noise;
- the gradient with respect to (m^2, lambda, H, Gamma) against central finite
  differences, h = 1e-5, with common random numbers (same state, same seed and
  counter), within 1e-6 relative: on small lattices and on the 48^3, 2000-step
  run with checkpoints every 50 steps;
- at equilibrium, d<sigma>/dH against the fluctuation-dissipation
  susceptibility V (<sigma^2> - <sigma>^2) of the same trajectories.
"""
import ctypes as C

import numpy as np
import pytest

from lgvtest import GpuLattice, rand_state

pytestmark = pytest.mark.gpu

SEED = 977
CFG4 = dict(mass0=-4.813, lam=10.0, H=0.01, gamma=1.0)  # (m^2, lambda, H, Gamma) of the 48^3 run
EVOLVER = {"em": 6, "ideal": 3, "ideal_em": 7}


def theta_of(c):
    return np.array([c["mass0"], c["lam"], c["H"], c["gamma"]])


def kw_of(theta):
    return dict(mass0=float(theta[0]), lam=float(theta[1]), H=float(theta[2]), gamma=float(theta[3]))


class EmLattice(GpuLattice):
    scheme = "em"

    def forward(self, dt, S, b, K, t=0.0):
        obs = np.zeros(2)
        self.L.check(self.lib.lgv_diff_forward(self.h, EVOLVER[self.scheme], float(dt), float(t), int(S), int(b),
                                               int(K), self.L.ptr(obs)), "diff_forward")
        return obs

    def backward(self, w=(1.0, 1.0)):
        w = np.ascontiguousarray(w, dtype=np.float64)
        g = np.zeros(4)
        self.L.check(self.lib.lgv_diff_backward(self.h, self.L.ptr(w), self.L.ptr(g)), "diff_backward")
        return g

    def averages(self, S):
        out = np.zeros((S + 1, 4))
        self.L.check(self.lib.lgv_diff_averages(self.h, self.L.ptr(out), int(S)), "diff_averages")
        return out

    def set_theta(self, theta, **extra):
        self.p = self.L.make_params(self.N, seed=SEED, **kw_of(theta), **extra)
        self.L.check(self.lib.lgv_set_params(self.h, C.byref(self.p)), "set_params")


def central_fd(lat, u, ctr, theta, run, w=(1.0, 1.0), h=1e-5, **extra):
    fd = np.zeros(4)
    for i in range(4):
        vals = []
        for sgn in (1.0, -1.0):
            th = np.array(theta, dtype=np.float64)
            th[i] += sgn * h
            lat.set_theta(th, **extra)
            lat.set_state(u)
            lat.counter(ctr)
            vals.append(np.dot(w, lat.forward(*run)))
        fd[i] = (vals[0] - vals[1]) / (2 * h)
    lat.set_theta(theta, **extra)
    return fd


def assert_grad_close(g, ref, rtol, what):
    scale = np.max(np.abs(ref))
    err = np.abs(g - ref) / np.maximum(np.abs(ref), 1e-3 * scale)
    assert np.all(err <= rtol), f"{what}: relative errors {err} > {rtol:.0e} (grad {g}, reference {ref})"
    return err


@pytest.mark.parametrize("scheme,N,S,b,K", [("em", 8, 40, 15, 7), ("em", 6, 25, 0, 25), ("em", 10, 33, 32, 4),
                                             ("ideal", 8, 30, 10, 7), ("ideal", 6, 12, 0, 12),
                                             ("ideal_em", 8, 40, 15, 7), ("ideal_em", 10, 21, 3, 5)])
def test_adjoint_matches_numpy_restatement(lgv, oracle_mod, scheme, N, S, b, K):
    import diff_adjoint as da

    theta = theta_of(CFG4)
    theta[2] = 0.3  # a larger H so the ideal step's -H phi source is visible
    lat = EmLattice(lgv, N, seed=SEED, dmassdt=-0.3, **kw_of(theta))
    lat.scheme = scheme
    u = rand_state(N, 3 + N)
    lat.set_state(u)
    lat.counter(5)
    dt, t0 = 0.02, 0.5
    obs = lat.forward(dt, S, b, K, t=t0)
    assert lat.counter() == 5 + (S if scheme != "ideal" else 0)
    run = da.Run(scheme, theta, dt, SEED, 5, t0=t0, dmassdt=-0.3)
    us = run.forward(u, S)
    np.testing.assert_allclose(lat.get_state(), us[-1], rtol=1e-11, atol=1e-11)
    if scheme == "em":
        np.testing.assert_array_equal(lat.get_state()[..., 4:], u[..., 4:])
    np.testing.assert_allclose(obs, da.Run.observables(us, b), rtol=1e-11, atol=1e-13)
    avg = lat.averages(S)
    np.testing.assert_allclose(avg, np.array([x[..., :4].mean(axis=(0, 1, 2)) for x in us]), rtol=1e-11, atol=1e-13)
    for w in [(1.0, 1.0), (0.5, -2.0), (0.0, 1.0)]:
        g = lat.backward(w)
        ref = run.gradient(us, b, w=w)
        assert_grad_close(g, ref, 1e-9, f"{scheme} adjoint vs numpy restatement N={N} w={w}")
        if scheme == "ideal":
            assert g[0] == 0 and g[1] == 0 and g[3] == 0


@pytest.mark.parametrize("scheme,N,S,b,K", [("em", 16, 400, 200, 50), ("em", 12, 300, 100, 64),
                                             ("ideal_em", 16, 300, 100, 50), ("ideal", 12, 200, 50, 40)])
def test_adjoint_matches_central_fd_small(lgv, scheme, N, S, b, K):
    theta = theta_of(CFG4)
    if scheme == "ideal":
        theta[2] = 0.3
    lat = EmLattice(lgv, N, seed=SEED, **kw_of(theta))
    lat.scheme = scheme
    u = rand_state(N, 21, charges=(scheme != "em"))
    run = (0.02, S, b, K)
    lat.set_state(u)
    lat.counter(0)
    lat.forward(*run)
    g = lat.backward((1.0, 1.0))
    fd = central_fd(lat, u, 0, theta, run)
    assert_grad_close(g, fd, 1e-6, f"{scheme} adjoint vs central FD N={N}")


def test_ideal_em_step_matches_oracle(lgv, oracle_mod):
    """lgv_step with LGV_IDEAL_EM against the oracle's ideal step then Euler-Maruyama step."""
    N = 8
    c = dict(CFG4, chi=5.0, seed=SEED)
    g = GpuLattice(lgv, N, **c)
    o = oracle_mod.Oracle(N, mode=oracle_mod.COUNTER, **c)
    u = rand_state(N, 77)
    g.set_state(u)
    o.set_state(u)
    g.step(7, 0.02, t=0.1, nsteps=4)
    o.step(7, 0.02, t=0.1, nsteps=4)
    from lgvtest import assert_state_close
    assert_state_close(g.get_state(), o.get_state(), what="ideal + EM")
    assert g.counter() == 4


def test_adjoint_matches_central_fd_48cubed_2000_steps(lgv):
    """The 48^3 Euler-Maruyama run: 2000 steps, dt = 0.02, loss averaged over
    steps 1001..2000, checkpoints every 50 steps."""
    N = 48
    theta = theta_of(CFG4)
    lat = EmLattice(lgv, N, seed=SEED, **kw_of(theta))
    u = rand_state(N, 48, phi_scale=0.1, charges=False)
    run = (0.02, 2000, 1000, 50)
    lat.set_state(u)
    lat.counter(0)
    lat.forward(*run)
    g = lat.backward((1.0, 1.0))
    fd = central_fd(lat, u, 0, theta, run)
    assert_grad_close(g, fd, 1e-6, "adjoint vs central FD at 48^3")


def test_backward_is_repeatable_and_leaves_state(lgv):
    N = 8
    lat = EmLattice(lgv, N, seed=SEED, **CFG4)
    lat.set_state(rand_state(N, 2))
    lat.forward(0.02, 60, 20, 16)
    after = lat.get_state()
    c = lat.counter()
    g1 = lat.backward((1.0, 1.0))
    g2 = lat.backward((1.0, 1.0))
    assert np.array_equal(g1, g2)
    assert np.array_equal(lat.get_state(), after)
    assert lat.counter() == c
    # the gradient is linear in the weights
    np.testing.assert_allclose(lat.backward((2.0, 0.0)) + lat.backward((0.0, 3.0)),
                               2 * lat.backward((1.0, 0.0)) + 3 * lat.backward((0.0, 1.0)), rtol=1e-13, atol=1e-15)


def test_adjoint_errors(lgv):
    N = 4
    lat = EmLattice(lgv, N, seed=SEED, **CFG4)
    w, g = np.ones(2), np.zeros(4)
    assert lat.lib.lgv_diff_backward(lat.h, lat.L.ptr(w), lat.L.ptr(g)) != 0  # no forward yet
    obs = np.zeros(2)
    assert lat.lib.lgv_diff_forward(lat.h, 6, 0.02, 0.0, 10, 10, 5, lat.L.ptr(obs)) != 0  # avg_begin == nsteps
    assert lat.lib.lgv_diff_forward(lat.h, 6, 0.02, 0.0, 10, 0, 0, lat.L.ptr(obs)) != 0  # ckpt_every 0
    assert lat.lib.lgv_diff_forward(lat.h, 4, 0.02, 0.0, 10, 0, 5, lat.L.ptr(obs)) != 0  # Metropolis: no adjoint
    lat.mode(1)
    assert lat.lib.lgv_diff_forward(lat.h, 6, 0.02, 0.0, 10, 0, 5, lat.L.ptr(obs)) != 0  # injected noise
    assert lat.lib.lgv_diff_forward(lat.h, 3, 0.02, 0.0, 10, 0, 5, lat.L.ptr(obs)) == 0  # ideal: no noise needed


def _model(lgv, N, theta, seed=SEED):
    data = lgv.ModelAData(dict(NX=N, mass0=theta[0], **{"lambda": theta[1]}, H=theta[2], gamma=theta[3],
                               seed=seed, deltat=0.02, finaltime=1.0))
    return lgv.ModelA(data)


def test_autograd_function_gradcheck(lgv):
    import torch

    from langevina_b200.adjoint import diff_observables, em_observables

    N = 8
    model = _model(lgv, N, theta_of(CFG4))
    u = rand_state(N, 9)
    model.set_state(u)

    def f(theta):
        model.set_state(u)
        model.set_counter(4)
        return em_observables(model, theta, 0.02, 50, 20, ckpt_every=16)

    theta = torch.tensor(theta_of(CFG4), dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(f, (theta,), eps=1e-5, atol=1e-9, rtol=1e-6)

    obs = f(theta)
    (obs[0] + obs[1]).backward()
    lat_g = model.diff_backward((1.0, 1.0))
    assert np.array_equal(theta.grad.numpy(), lat_g)


def test_autograd_backward_after_another_forward(lgv):
    import torch

    from langevina_b200.adjoint import diff_observables, em_observables

    N = 8
    model = _model(lgv, N, theta_of(CFG4))
    u = rand_state(N, 10)
    model.set_state(u)
    model.set_counter(0)
    th1 = torch.tensor(theta_of(CFG4), dtype=torch.float64, requires_grad=True)
    o1 = em_observables(model, th1, 0.02, 40, 10, ckpt_every=8)
    expect = model.diff_backward((1.0, 1.0))
    th2 = torch.tensor(theta_of(CFG4) * 1.01, dtype=torch.float64, requires_grad=True)
    o2 = em_observables(model, th2, 0.02, 30, 5, ckpt_every=8)
    state2, ctr2 = model.get_state(), model.get_counter()
    o1.sum().backward()
    assert np.array_equal(th1.grad.numpy(), expect)
    assert np.array_equal(model.get_state(), state2) and model.get_counter() == ctr2
    o2.sum().backward()
    assert th2.grad is not None and np.all(np.isfinite(th2.grad.numpy()))


def test_autograd_ideal_em_gradcheck(lgv):
    import torch

    from langevina_b200.adjoint import diff_observables

    N = 8
    th0 = theta_of(CFG4)
    model = _model(lgv, N, th0)
    u = rand_state(N, 12)

    def f(theta):
        model.set_state(u)
        model.set_counter(0)
        return diff_observables(model, theta, 0.02, 40, 10, ckpt_every=9, evolver="ideal_em")

    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(f, (theta,), eps=1e-5, atol=1e-9, rtol=1e-6)


def test_fluctuation_dissipation_susceptibility(lgv):
    """At equilibrium d<sigma>/dH = V (<sigma^2> - <sigma>^2) (the stationary
    weight is exp(-S) with S linear in -H sum phi_0).  Symmetric phase,
    m^2 = 1, lambda = 1, H = 0.2, dt = 0.005; 8 seeds of 60000 steps on 8^3,
    the first 10000 dropped.  The Euler-Maruyama chain's own stationary
    variance is larger by about dt m_eff^2 / 2 (< 1%); the check allows that
    plus 4 standard errors over the seeds."""
    N, S, b, K, dt = 8, 60000, 10000, 500, 0.005
    theta = np.array([1.0, 1.0, 0.2, 1.0])
    V = N ** 3
    adj, fdt = [], []
    for s in range(8):
        lat = EmLattice(lgv, N, seed=1000 + s, **kw_of(theta))
        lat.set_state(np.zeros((N, N, N, 10)))
        lat.counter(0)
        lat.forward(dt, S, b, K)
        adj.append(lat.backward((1.0, 0.0))[2])
        sig = lat.averages(S)[b + 1:, 0]
        fdt.append(V * sig.var())
        lat.close()
    adj, fdt = np.array(adj), np.array(fdt)
    ma, mf = adj.mean(), fdt.mean()
    se = np.sqrt(adj.var(ddof=1) / len(adj) + fdt.var(ddof=1) / len(fdt))
    assert abs(ma - mf) <= 4 * se + 0.01 * mf, f"d<sigma>/dH {ma:.4f} vs V var(sigma) {mf:.4f} (se {se:.4f})"


def test_ensemble_adjoint_matches_single_lattices(lgv):
    """lgv_ensemble_diff_forward/backward over uneven replicas (sizes, seeds,
    H) against lgv_diff_forward/backward of each replica alone."""
    from langevina_b200 import _lib as L

    lib = L.load()
    sizes = [8, 12, 8, 16, 6]
    specs = [dict(N=N, seed=500 + r, H=(0.003, 0.006, 0.012)[r % 3], mass0=-4.813 + 0.1 * r, lam=10.0, gamma=1.0)
             for r, N in enumerate(sizes)]
    R = len(specs)
    arr = (L.lgv_params * R)()
    for r, sp in enumerate(specs):
        arr[r] = L.make_params(sp["N"], seed=sp["seed"], mass0=sp["mass0"], lam=sp["lam"], H=sp["H"],
                               gamma=sp["gamma"], dmassdt=-0.2)
    e = C.c_void_p()
    L.check(lib.lgv_ensemble_create(R, arr, C.byref(e)), "ensemble_create")
    try:
        states = [rand_state(sp["N"], 60 + r) for r, sp in enumerate(specs)]
        for r in range(R):
            L.check(lib.lgv_ensemble_set_state(e, r, L.ptr(states[r])), "set_state")
        L.check(lib.lgv_ensemble_set_counter(e, 9), "set_counter")
        S, b, K, dt, t0 = 50, 20, 16, 0.02, 0.25
        obs = np.zeros((R, 2))
        L.check(lib.lgv_ensemble_diff_forward(e, dt, t0, S, b, K, L.ptr(obs)), "ensemble_diff_forward")
        w = np.array([[1.0, 1.0], [0.5, -1.0], [0.0, 2.0], [1.0, 0.0], [-1.0, 0.25]])
        grad = np.zeros((R, 4))
        L.check(lib.lgv_ensemble_diff_backward(e, L.ptr(w), L.ptr(grad)), "ensemble_diff_backward")
        c = C.c_uint64()
        L.check(lib.lgv_ensemble_get_counter(e, C.byref(c)), "get_counter")
        assert c.value == 9 + S
        for r, sp in enumerate(specs):
            lat = EmLattice(lgv, sp["N"], seed=sp["seed"], mass0=sp["mass0"], lam=sp["lam"], H=sp["H"],
                            gamma=sp["gamma"], dmassdt=-0.2)
            lat.set_state(states[r])
            lat.counter(9)
            o1 = lat.forward(dt, S, b, K, t=t0)
            g1 = lat.backward(w[r])
            fin = np.empty((sp["N"],) * 3 + (10,))
            L.check(lib.lgv_ensemble_get_state(e, r, L.ptr(fin)), "get_state")
            assert np.array_equal(fin, lat.get_state()), f"replica {r}: final state differs"
            np.testing.assert_allclose(obs[r], o1, rtol=1e-13, atol=1e-15)
            assert_grad_close(grad[r], g1, 1e-12, f"ensemble replica {r}")
            lat.close()
    finally:
        lib.lgv_ensemble_destroy(e)

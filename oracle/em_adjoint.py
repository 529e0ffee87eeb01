"""TEST INFRASTRUCTURE ONLY: numpy restatement of the differentiable
Euler-Maruyama Model A run and of its adjoint.

Only tests/ may import this module; the product path (liblgv.so,
lgv_em_forward / lgv_em_backward) never calls it.

The step is the one of oracle/lgv_oracle.cpp em_step, derived from the action
whose local change the reference's heat bath uses (ModelG/Stepper.cxx:298,
332-355):
    F_a   = -sum_nbr phi_a + (6 + m^2(t)) phi_a + lambda phi^2 phi_a - H delta_a0
    phi' = phi - dt G F + sqrt(2 G dt) xi,        m^2(t) = mass0 + dmassdt t
with xi the counter-mode normals of step counter ctr0 + n (orc_em_noise).  The
observables are the time averages over steps n = b+1 .. S
    obs0 = 1/M sum_n <phi_0>(n),   obs1 = 1/M sum_n V sum_{a>=1} <phi_a>(n)^2.
The adjoint runs lam_S = dJ/dphi_S, lam_n = (d phi_{n+1}/d phi_n)^T lam_{n+1}
+ dJ/dphi_n, and accumulates lam_{n+1} . d phi_{n+1}/d theta.  The reference
has no counterpart (no Euler-Maruyama stepper, no gradients).
"""
import numpy as np

import oracle as _orc  # oracle/oracle.py, on the path of the tests


def _nbr(f):
    """sum over the 6 periodic neighbours; f has shape (N, N, N, ...) = [k, j, i, ...]."""
    return sum(np.roll(f, s, axis=a) for a in (0, 1, 2) for s in (1, -1))


def force(phi, c6, lam, H):
    p2 = np.sum(phi * phi, axis=-1, keepdims=True)
    F = -_nbr(phi) + c6 * phi + lam * p2 * phi
    F[..., 0] -= H
    return F


def em_run(phi0, theta, dt, S, seed, ctr0, t0=0.0, dmassdt=0.0):
    """Forward: returns the list of states phi_0..phi_S, shape (N, N, N, 4) each."""
    mass0, lam, H, gamma = theta
    N = phi0.shape[0]
    phis = [np.array(phi0, dtype=np.float64)]
    t = t0
    for n in range(S):
        xi = np.moveaxis(_orc.em_noise(seed, ctr0 + n, N), 0, -1)
        phi = phis[-1]
        c6 = 6.0 + (mass0 + dmassdt * t)
        phis.append(phi - dt * gamma * force(phi, c6, lam, H) + np.sqrt(2.0 * gamma * dt) * xi)
        t = t + dt
    return phis


def observables(phis, b):
    S = len(phis) - 1
    V = phis[0][..., 0].size
    o0 = sum(p[..., 0].mean() for p in phis[b + 1:]) / (S - b)
    o1 = sum(V * np.sum(p[..., 1:].mean(axis=(0, 1, 2)) ** 2) for p in phis[b + 1:]) / (S - b)
    return np.array([o0, o1])


def em_gradient(phis, theta, dt, b, seed, ctr0, w=(1.0, 1.0), t0=0.0, dmassdt=0.0):
    """d(w0 obs0 + w1 obs1)/d(mass0, lambda, H, gamma) by the adjoint recursion."""
    mass0, lam, H, gamma = theta
    S = len(phis) - 1
    N = phis[0].shape[0]
    V = N ** 3
    M = S - b
    ts = [t0]
    for _ in range(S):
        ts.append(ts[-1] + dt)

    def gl(n):
        g = np.zeros(4)
        if n > b:
            av = phis[n].mean(axis=(0, 1, 2))
            g[0] = w[0] / (V * M)
            g[1:] = w[1] * 2.0 * av[1:] / M
        return g

    dtg = dt * gamma
    cxi = np.sqrt(2.0 * dt) / (2.0 * np.sqrt(gamma))
    L = np.broadcast_to(gl(S), phis[0].shape).copy()
    grad = np.zeros(4)
    for n in range(S - 1, -1, -1):
        phi = phis[n]
        xi = np.moveaxis(_orc.em_noise(seed, ctr0 + n, N), 0, -1)
        c6 = 6.0 + (mass0 + dmassdt * ts[n])
        p2 = np.sum(phi * phi, axis=-1, keepdims=True)
        dot = np.sum(phi * L, axis=-1, keepdims=True)
        F = force(phi, c6, lam, H)
        grad[0] += -dtg * np.sum(dot)
        grad[1] += -dtg * np.sum(p2 * dot)
        grad[2] += dtg * np.sum(L[..., 0])
        grad[3] += np.sum(L * (-dt * F + cxi * xi))
        L = L - dtg * (c6 * L + lam * (p2 * L + 2.0 * phi * dot) - _nbr(L)) + gl(n)
    return grad

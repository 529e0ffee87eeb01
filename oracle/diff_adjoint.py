"""TEST INFRASTRUCTURE ONLY: numpy restatement of the differentiable runs
(Euler-Maruyama Model A, the ideal O(4) rotation step, and the two in
sequence) and of their adjoints.

Only tests/ may import this module; the product path (liblgv.so,
lgv_diff_forward / lgv_diff_backward) never calls it.

State: u of shape (N, N, N, 10) = [k, j, i, c], c = phi_0..3, n_A 1..3,
n_V 1..3 (the layout of the reference's restart files).

Euler-Maruyama (oracle/lgv_oracle.cpp em_step; the action is the one whose
local change the reference's heat bath uses, ModelG/Stepper.cxx:298, 332-355):
    F_a  = -sum_nbr phi_a + (6 + m^2(t)) phi_a + lambda phi^2 phi_a - H delta_a0
    phi' = phi - dt G F + sqrt(2 G dt) xi,         m^2(t) = mass0 + dmassdt t
with xi the counter-mode normals of step counter ctr0 + n (orc_em_noise).

Ideal step (IdealPV2::step_no_reject, ModelG/Stepper.cxx:68-176):
    phi1 = R(phi, n; dt/2)        O(4) rotation with mu = -n dt / (2 chi)
    nA_l += dt [a2 (phi1_0 S_l - phi1_l S_0) - H phi1_l]
    nV_s += dt a2 (phi1_s1 S_s2 - phi1_s2 S_s1),   (s, s1, s2) cyclic
    phi2 = R(phi1, n'; dt/2)
with S_a the sum of phi1_a over the 6 neighbours (the reference's forward
and backward differences summed over directions reduce to these currents)
and R(phi, n) = L phi R as quaternions, R = exp(-(muV - muA)/2),
L = exp((muV + muA)/2) (O4AlgebraHelper.h:17-97).

Observables: time averages over steps n = b+1 .. S of sigma = <phi_0> and of
V sum_{a>=1} <phi_a>^2 (the zero-momentum pi equal-time correlator).

Adjoint: lam_S = dJ/du_S, lam_n = (du_{n+1}/du_n)^T lam_{n+1} + dJ/du_n,
accumulating lam_{n+1} . du_{n+1}/dtheta for theta = (mass0, lambda, H,
Gamma).  Quaternion products are bilinear, so their transposes are products
with the conjugate: for w = a b, a_bar = w_bar conj(b), b_bar = conj(a) w_bar.
The reference has no counterpart (no Euler-Maruyama stepper, no gradients).
"""
import math

import numpy as np

import oracle as _orc  # oracle/oracle.py, on the path of the tests

SCHEMES = ("em", "ideal", "ideal_em")
# q_c += dt a2 (phi_a S_b - phi_b S_a): axial l (a = 0, b = l + 1), vector s (a = s1, b = s2)
PAIRS = [(0, 1, 0), (0, 2, 1), (0, 3, 2)] + [(1 + (s + 1) % 3, 1 + (s + 2) % 3, 3 + s) for s in range(3)]


def _nbr(f):
    """sum over the 6 periodic neighbours; f has shape (N, N, N, ...) = [k, j, i, ...]."""
    return sum(np.roll(f, s, axis=a) for a in (0, 1, 2) for s in (1, -1))


# ---- O(4) algebra -----------------------------------------------------------
def qmul(a, b):
    a0, a1, a2, a3 = (a[..., i] for i in range(4))
    b0, b1, b2, b3 = (b[..., i] for i in range(4))
    return np.stack([a0 * b0 - (a1 * b1 + a2 * b2 + a3 * b3),
                     (a2 * b3 - b2 * a3) + b0 * a1 + a0 * b1,
                     (a3 * b1 - a1 * b3) + b0 * a2 + a0 * b2,
                     (a1 * b2 - b1 * a2) + b0 * a3 + a0 * b3], axis=-1)


def conj(a):
    return a * np.array([1.0, -1.0, -1.0, -1.0])


def _sinc(x2):
    a = np.sqrt(x2)
    return np.where(x2 > 0, np.sin(a) / np.where(a > 0, a, 1.0), 1.0)


def _dsinc(x2):
    """d/dx2 of sin(sqrt x2)/sqrt x2: the series sum_n (-1)^n n x2^(n-1)/(2n+1)! for x2 <= 1/16."""
    ser = sum((-1) ** n * n * x2 ** (n - 1) / math.factorial(2 * n + 1) for n in range(1, 9))
    a = np.sqrt(np.maximum(x2, 1e-300))
    big = (np.cos(a) - np.sin(a) / a) / (2.0 * np.maximum(x2, 1e-300))
    return np.where(x2 <= 0.0625, ser, big)


def expmul(v):
    """(cos|v|, -sin|v|/|v| v)."""
    x2 = np.sum(v * v, axis=-1, keepdims=True)
    return np.concatenate([np.cos(np.sqrt(x2)), -_sinc(x2) * v], axis=-1)


def expmul_adj(v, wb):
    x2 = np.sum(v * v, axis=-1, keepdims=True)
    vdot = np.sum(wb[..., 1:] * v, axis=-1, keepdims=True)
    return -_sinc(x2) * (wb[..., 0:1] * v + wb[..., 1:]) - 2.0 * _dsinc(x2) * v * vdot


def _rot_parts(phi, q, k):
    muA, muV = -q[..., 0:3] * k, -q[..., 3:6] * k
    vR, vL = -0.5 * (muV - muA), 0.5 * (muV + muA)
    return vR, vL, expmul(vR), expmul(vL)


def rot(phi, q, k):
    _, _, R, L = _rot_parts(phi, q, k)
    return qmul(L, qmul(phi, R))


def rot_adj(phi, q, k, ob):
    """(phi_bar, q_bar) of out = rot(phi, q, k) given out_bar."""
    vR, vL, R, L = _rot_parts(phi, q, k)
    t = qmul(phi, R)
    tb, Lb = qmul(conj(L), ob), qmul(ob, conj(t))
    pb, Rb = qmul(tb, conj(R)), qmul(conj(phi), tb)
    vLb, vRb = expmul_adj(vL, Lb), expmul_adj(vR, Rb)
    muVb, muAb = 0.5 * vLb - 0.5 * vRb, 0.5 * vLb + 0.5 * vRb
    return pb, np.concatenate([-k * muAb, -k * muVb], axis=-1)


# ---- steps ----------------------------------------------------------------------
def _ideal_parts(u, dt, chi, H, a2):
    k = dt / (2.0 * chi)
    phi, q = u[..., :4], u[..., 4:]
    p1 = rot(phi, q, k)
    S = _nbr(p1)
    q2 = q.copy()
    for a, b, c in PAIRS:
        q2[..., c] += dt * a2 * (p1[..., a] * S[..., b] - p1[..., b] * S[..., a])
    for l in range(3):
        q2[..., l] -= dt * H * p1[..., l + 1]
    return k, p1, S, q2


def ideal(u, dt, chi, H, a2):
    k, p1, _, q2 = _ideal_parts(u, dt, chi, H, a2)
    return np.concatenate([rot(p1, q2, k), q2], axis=-1)


def ideal_adj(u, dt, chi, H, a2, ub):
    """(u_bar, H_bar) of the ideal step at state u given the adjoint ub of its output."""
    k, p1, S, q2 = _ideal_parts(u, dt, chi, H, a2)
    p1b, q2b = rot_adj(p1, q2, k, ub[..., :4])
    Q = ub[..., 4:] + q2b
    for a, b, c in PAIRS:
        g = dt * a2 * Q[..., c]
        p1b[..., a] += g * S[..., b] - _nbr(g * p1[..., b])
        p1b[..., b] += _nbr(g * p1[..., a]) - g * S[..., a]
    Hb = 0.0
    for l in range(3):
        p1b[..., l + 1] += -dt * H * Q[..., l]
        Hb += -dt * np.sum(Q[..., l] * p1[..., l + 1])
    phib, qb = rot_adj(u[..., :4], u[..., 4:], k, p1b)
    return np.concatenate([phib, Q + qb], axis=-1), Hb


def force(phi, c6, lam, H):
    p2 = np.sum(phi * phi, axis=-1, keepdims=True)
    F = -_nbr(phi) + c6 * phi + lam * p2 * phi
    F[..., 0] -= H
    return F


class Run:
    """A differentiable run: scheme in SCHEMES, theta = (mass0, lambda, H, Gamma)."""

    def __init__(self, scheme, theta, dt, seed, ctr0, t0=0.0, dmassdt=0.0, chi=5.0, a2=1.0):
        assert scheme in SCHEMES
        self.scheme, self.theta, self.dt = scheme, np.asarray(theta, dtype=np.float64), dt
        self.seed, self.ctr0, self.t0, self.dmassdt, self.chi, self.a2 = seed, ctr0, t0, dmassdt, chi, a2

    def _xi(self, n, N):
        return np.moveaxis(_orc.em_noise(self.seed, self.ctr0 + n, N), 0, -1)

    def _t(self, n):
        t = self.t0
        for _ in range(n):
            t = t + self.dt
        return t

    def _mid(self, u):
        if self.scheme == "em":
            return u
        return ideal(u, self.dt, self.chi, self.theta[2], self.a2)

    def forward(self, u0, S):
        """States u_0..u_S."""
        mass0, lam, H, gamma = self.theta
        dt = self.dt
        us = [np.array(u0, dtype=np.float64)]
        t = self.t0
        for n in range(S):
            u = self._mid(us[-1])
            if self.scheme != "ideal":
                u = u.copy()
                c6 = 6.0 + (mass0 + self.dmassdt * t)
                phi = u[..., :4]
                u[..., :4] = phi - dt * gamma * force(phi, c6, lam, H) + np.sqrt(2.0 * gamma * dt) * self._xi(n, phi.shape[0])
            us.append(u)
            t = t + dt
        return us

    @staticmethod
    def observables(us, b):
        S = len(us) - 1
        V = us[0][..., 0].size
        o0 = sum(u[..., 0].mean() for u in us[b + 1:]) / (S - b)
        o1 = sum(V * np.sum(u[..., 1:4].mean(axis=(0, 1, 2)) ** 2) for u in us[b + 1:]) / (S - b)
        return np.array([o0, o1])

    def gradient(self, us, b, w=(1.0, 1.0)):
        """d(w0 obs0 + w1 obs1)/d(mass0, lambda, H, Gamma) by the adjoint recursion."""
        mass0, lam, H, gamma = self.theta
        dt = self.dt
        S = len(us) - 1
        N = us[0].shape[0]
        V, M = N ** 3, S - b

        def gl(n):
            g = np.zeros(10)
            if n > b:
                av = us[n][..., :4].mean(axis=(0, 1, 2))
                g[0] = w[0] / (V * M)
                g[1:4] = w[1] * 2.0 * av[1:4] / M
            return g

        dtg = dt * gamma
        cxi = np.sqrt(2.0 * dt) / (2.0 * np.sqrt(gamma))
        L = np.broadcast_to(gl(S), us[0].shape).copy()
        grad = np.zeros(4)
        for n in range(S - 1, -1, -1):
            if self.scheme != "ideal":
                mid = self._mid(us[n])
                phi = mid[..., :4]
                Lp = L[..., :4]
                xi = self._xi(n, N)
                c6 = 6.0 + (mass0 + self.dmassdt * self._t(n))
                p2 = np.sum(phi * phi, axis=-1, keepdims=True)
                dot = np.sum(phi * Lp, axis=-1, keepdims=True)
                F = force(phi, c6, lam, H)
                grad[0] += -dtg * np.sum(dot)
                grad[1] += -dtg * np.sum(p2 * dot)
                grad[2] += dtg * np.sum(Lp[..., 0])
                grad[3] += np.sum(Lp * (-dt * F + cxi * xi))
                L = L.copy()
                L[..., :4] = Lp - dtg * (c6 * Lp + lam * (p2 * Lp + 2.0 * phi * dot) - _nbr(Lp))
            if self.scheme != "em":
                L, Hb = ideal_adj(us[n], dt, self.chi, H, self.a2, L)
                grad[2] += Hb
            L = L + gl(n)
        return grad

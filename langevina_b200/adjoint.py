"""Differentiable Model A (Euler-Maruyama) behind torch.autograd.

``em_observables(model, theta, ...)`` runs the Euler-Maruyama relaxation
phi <- phi - dt G dS/dphi + sqrt(2 G dt) xi on the device lattice of ``model``
with theta = (m^2, lambda, H, Gamma) and returns the time averages

    obs[0] = 1/M sum_n sigma(n),          sigma = <phi_0>
    obs[1] = 1/M sum_n V sum_a pibar_a(n)^2,   pibar_a = <phi_a>, a = 1..3

over the last M steps.  The noise xi is fixed by the model's seed and counter
(counter-indexed xoroshiro streams), so two calls from the same state and
counter use common random numbers.  The backward is the hand-written adjoint
kernel of the step (liblgv.so, lgv_em_backward), with phi checkpointed every
``ckpt_every`` steps and recomputed in between; it returns d obs / d theta
contracted with the incoming gradient.  The Metropolis heat baths of the
reference have no adjoint and are not part of this path.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib as L

PARAM_NAMES = ("mass0", "lambda", "H", "gamma")


def _apply_theta(model, theta):
    c = model.data.acoefficients
    c.mass0, c.lambda_, c.H, c.gamma = (float(v) for v in theta)
    model.sync_params()


def _snapshot(model):
    """Device copy of the lattice (AoS) and the noise counter."""
    buf = torch.empty(model.V * L.NDOF, dtype=torch.float64, device="cuda")
    L.check(model.lib.lgv_get_state_device(model.handle, C.c_void_p(buf.data_ptr())), "lgv_get_state_device")
    model.synchronize()
    return buf, model.get_counter()


def _restore(model, snap):
    buf, ctr = snap
    L.check(model.lib.lgv_set_state_device(model.handle, C.c_void_p(buf.data_ptr())), "lgv_set_state_device")
    model.synchronize()
    model.set_counter(ctr)


class EMObservables(torch.autograd.Function):
    """autograd.Function over lgv_em_forward / lgv_em_backward.

    The handle keeps the checkpoints of its latest forward only.  When the
    model ran another differentiable forward before this backward, the
    backward restores this forward's initial lattice, counter and theta,
    runs it again, differentiates it and puts the model back as it was.
    """

    @staticmethod
    def forward(ctx, theta, model, dt, nsteps, avg_begin, ckpt_every, t0):
        th = theta.detach().to("cpu", torch.float64).numpy().copy()
        ctx.snap = _snapshot(model)
        _apply_theta(model, th)
        obs = model.em_forward(dt, nsteps, avg_begin, ckpt_every, t=t0)
        model._em_generation = getattr(model, "_em_generation", 0) + 1
        ctx.model, ctx.generation, ctx.theta = model, model._em_generation, th
        ctx.run = (dt, nsteps, avg_begin, ckpt_every, t0)
        ctx.theta_device, ctx.theta_dtype = theta.device, theta.dtype
        return torch.from_numpy(obs).to(theta.device, theta.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        model = ctx.model
        w = grad_out.detach().to("cpu", torch.float64).numpy()
        if getattr(model, "_em_generation", None) == ctx.generation:
            g = model.em_backward(w)
        else:
            c = model.data.acoefficients
            saved_theta = (c.mass0, c.lambda_, c.H, c.gamma)
            now = _snapshot(model)
            _restore(model, ctx.snap)
            _apply_theta(model, ctx.theta)
            dt, nsteps, avg_begin, ckpt_every, t0 = ctx.run
            model.em_forward(dt, nsteps, avg_begin, ckpt_every, t=t0)
            g = model.em_backward(w)
            _restore(model, now)
            _apply_theta(model, saved_theta)
            model._em_generation = getattr(model, "_em_generation", 0) + 1
        return (torch.from_numpy(g).to(ctx.theta_device, ctx.theta_dtype), None, None, None, None, None, None)


def em_observables(model, theta, dt, nsteps, avg_begin, ckpt_every=50, t0=0.0):
    """Differentiable time averages (sigma, zero-mode pi correlator) of an Euler-Maruyama run.

    theta: tensor (m^2, lambda, H, Gamma); the lattice of ``model`` is the
    initial state and is left at the final state, its noise counter advanced
    by ``nsteps``.
    """
    if not isinstance(theta, torch.Tensor):
        theta = torch.as_tensor(np.asarray(theta, dtype=np.float64))
    if theta.shape != (4,):
        raise ValueError("theta must hold (m^2, lambda, H, Gamma)")
    if not (0 <= avg_begin < nsteps):
        raise ValueError("need 0 <= avg_begin < nsteps")
    return EMObservables.apply(theta, model, float(dt), int(nsteps), int(avg_begin), int(ckpt_every), float(t0))

"""Differentiable runs behind torch.autograd.

``diff_observables(model, theta, ..., evolver)`` runs, on the device lattice
of ``model`` with theta = (m^2, lambda, H, Gamma), the Euler-Maruyama
relaxation phi <- phi - dt G dS/dphi + sqrt(2 G dt) xi ("em"), the ideal
O(4) rotation step of phi by the charges ("ideal"), or the two in sequence
("ideal_em"), and returns the time averages

    obs[0] = 1/M sum_n sigma(n),          sigma = <phi_0>
    obs[1] = 1/M sum_n V sum_a pibar_a(n)^2,   pibar_a = <phi_a>, a = 1..3

over the last M steps.  The noise xi is fixed by the model's seed and counter
(counter-indexed xoroshiro streams), so two calls from the same state and
counter use common random numbers.  The backward is the hand-written adjoint
kernels of the steps (liblgv.so, lgv_diff_backward), with the state
checkpointed every ``ckpt_every`` steps and recomputed in between; it returns d obs / d theta
contracted with the incoming gradient.  The Metropolis heat baths of the
reference have no adjoint and are not part of this path.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib as L

PARAM_NAMES = ("mass0", "lambda", "H", "gamma")
EVOLVERS = {"em": L.MODELA_EM, "ideal": L.IDEAL_PV2, "ideal_em": L.IDEAL_EM}


def _apply_theta(model, theta):
    c = model.data.acoefficients
    c.mass0, c.lambda_, c.H, c.gamma = (float(v) for v in theta)
    model.sync_params()


def _snapshot(model):
    """Device copy of the lattice (AoS) and the noise counter."""
    buf = torch.empty(model.V * L.NDOF, dtype=torch.float64, device="cuda")
    # the handle writes on its own stream: torch's pending work on memory its
    # allocator may have handed out again must finish first
    torch.cuda.current_stream().synchronize()
    L.check(model.lib.lgv_get_state_device(model.handle, C.c_void_p(buf.data_ptr())), "lgv_get_state_device")
    model.synchronize()
    return buf, model.get_counter()


def _restore(model, snap):
    buf, ctr = snap
    L.check(model.lib.lgv_set_state_device(model.handle, C.c_void_p(buf.data_ptr())), "lgv_set_state_device")
    model.synchronize()
    model.set_counter(ctr)


class DiffObservables(torch.autograd.Function):
    """autograd.Function over lgv_diff_forward / lgv_diff_backward.

    The handle keeps the checkpoints of its latest forward only.  When the
    model ran another differentiable forward before this backward, the
    backward restores this forward's initial lattice, counter and theta,
    runs it again, differentiates it and puts the model back as it was.
    """

    @staticmethod
    def forward(ctx, theta, model, dt, nsteps, avg_begin, ckpt_every, t0, evolver):
        th = theta.detach().to("cpu", torch.float64).numpy().copy()
        ctx.snap = _snapshot(model)
        _apply_theta(model, th)
        obs = model.diff_forward(dt, nsteps, avg_begin, ckpt_every, t=t0, evolver=evolver)
        model._diff_generation = getattr(model, "_diff_generation", 0) + 1
        ctx.model, ctx.generation, ctx.theta = model, model._diff_generation, th
        ctx.run = (dt, nsteps, avg_begin, ckpt_every, t0, evolver)
        ctx.theta_device, ctx.theta_dtype = theta.device, theta.dtype
        return torch.from_numpy(obs).to(theta.device, theta.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        model = ctx.model
        w = grad_out.detach().to("cpu", torch.float64).numpy()
        if getattr(model, "_diff_generation", None) == ctx.generation:
            g = model.diff_backward(w)
        else:
            c = model.data.acoefficients
            saved_theta = (c.mass0, c.lambda_, c.H, c.gamma)
            now = _snapshot(model)
            _restore(model, ctx.snap)
            _apply_theta(model, ctx.theta)
            dt, nsteps, avg_begin, ckpt_every, t0, evolver = ctx.run
            model.diff_forward(dt, nsteps, avg_begin, ckpt_every, t=t0, evolver=evolver)
            g = model.diff_backward(w)
            _restore(model, now)
            _apply_theta(model, saved_theta)
            model._diff_generation = getattr(model, "_diff_generation", 0) + 1
        return (torch.from_numpy(g).to(ctx.theta_device, ctx.theta_dtype),) + (None,) * 7


def diff_observables(model, theta, dt, nsteps, avg_begin, ckpt_every=50, t0=0.0, evolver="em"):
    """Differentiable time averages (sigma, zero-mode pi correlator) of a run.

    theta: tensor (m^2, lambda, H, Gamma); evolver: "em", "ideal" or
    "ideal_em".  The lattice of ``model`` is the initial state and is left at
    the final state, its noise counter advanced by ``nsteps`` when the run has
    Euler-Maruyama steps.
    """
    if evolver not in EVOLVERS:
        raise ValueError(f"evolver must be one of {sorted(EVOLVERS)}")
    if not isinstance(theta, torch.Tensor):
        theta = torch.as_tensor(np.asarray(theta, dtype=np.float64))
    if theta.shape != (4,):
        raise ValueError("theta must hold (m^2, lambda, H, Gamma)")
    if not (0 <= avg_begin < nsteps):
        raise ValueError("need 0 <= avg_begin < nsteps")
    return DiffObservables.apply(theta, model, float(dt), int(nsteps), int(avg_begin), int(ckpt_every), float(t0),
                                 EVOLVERS[evolver])


def em_observables(model, theta, dt, nsteps, avg_begin, ckpt_every=50, t0=0.0):
    """diff_observables of an Euler-Maruyama Model A run."""
    return diff_observables(model, theta, dt, nsteps, avg_begin, ckpt_every, t0, evolver="em")

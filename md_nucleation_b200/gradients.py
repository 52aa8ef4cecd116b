"""The gradient harness: parameters of the ion-vapor interaction as a torch
tensor, the window objective of mdn_adjoint as a differentiable function.

    theta0, rows = parameters(spec)                 # the spec's own values
    theta = theta0.clone().requires_grad_()
    J = window_objective(theta, spec, n_steps=2000)  # runs the engine forward
    J.backward()                                     # theta.grad from the adjoint

theta holds, in mdn_adjoint_params order, (eps, sigma) of every gas-ion and
vapor-ion type pair, then the ion charge scale s.  Evaluating at theta builds
the replica with those pair parameters (ReplicaSpec.pair_eps / pair_sigma)
and its ion charges times s, runs n_steps on the GPU and returns the window
average of the objective; the backward pass returns dJ/dtheta from the
discrete adjoint (FP64) computed in the same call.
"""
from __future__ import annotations

import copy

import numpy as np
import torch

from . import engine


def parameters(spec):
    """(theta0 as a float64 tensor, rows) of a spec: its pair eps / sigma and s = 1."""
    with engine.Engine([spec]) as e:
        rows, n = e.adjoint_params()
    eps, sig = spec.pair_parameters()
    theta = np.zeros(n)
    for k, (kind, a, b) in enumerate(rows[:-1]):
        theta[2 * k] = eps[a, b]
        theta[2 * k + 1] = sig[a, b]
    theta[-1] = 1.0
    return torch.tensor(theta, dtype=torch.float64), rows


def apply(spec, theta: np.ndarray, rows):
    """A copy of spec with the parameters theta."""
    s = copy.deepcopy(spec)
    eps, sig = spec.pair_parameters()
    eps, sig = eps.copy(), sig.copy()
    for k, (kind, a, b) in enumerate(rows[:-1]):
        eps[a, b] = eps[b, a] = theta[2 * k]
        sig[a, b] = sig[b, a] = theta[2 * k + 1]
    s.pair_eps, s.pair_sigma = eps, sig
    s.ion.charge = np.ascontiguousarray(spec.ion.charge * theta[-1])
    return s


class _Window(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, spec, rows, kw):
        th = theta.detach().cpu().numpy()
        s = apply(spec, th, rows)
        with engine.Engine([s], **kw.pop("engine_options", {})) as e:
            J, g, ms = e.adjoint(**kw)
        g = g.copy()
        g[-1] /= th[-1]  # mdn_adjoint differentiates a scale of the charges it was given
        ctx.save_for_backward(torch.tensor(g, dtype=torch.float64))
        ctx.timing = ms
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        (g,) = ctx.saved_tensors
        return gJ * g, None, None, None


def window_objective(theta: torch.Tensor, spec, rows=None, engine_options=None, **adjoint_kw) -> torch.Tensor:
    """J(theta) over a window of the replica `spec` (mdn_adjoint's objective);
    adjoint_kw: n_steps, checkpoint_every, count_radius, count_width,
    w_energy, w_count."""
    if rows is None:
        _, rows = parameters(spec)
    kw = dict(adjoint_kw)
    kw["engine_options"] = engine_options or {}
    return _Window.apply(theta, spec, rows, kw)

"""Thin torch.autograd binding of the device derivatives (test binding).

The differentiable input is an algebra field omega of shape (n_links, 3) acting on fixed
start links U0 as U = exp(omega) U0 (exp of exp_gauge.cc, per link).  ``WilsonAction``
returns S(U) = get_S_G_hmc and ``FlowEnergy`` returns t^2 E_p(t) after the Wilson flow; their
backward passes call su2b_action_backward / su2b_flow_adjoint for the left derivative at U
and map it to omega with the transposed left-trivialised differential of exp.
"""
from __future__ import annotations

import numpy as np
import torch


def _exp_links(U0: np.ndarray, omega: np.ndarray) -> np.ndarray:
    """exp(omega) U0 per link in the reference layout (4 reals per link)."""
    a, b, c = omega[:, 0], omega[:, 1], omega[:, 2]
    al = np.sqrt(a * a + b * b + c * c)
    f = np.where(al > 0, np.sin(al) / np.where(al > 0, al, 1.0), 1.0)
    E = np.stack([np.cos(al), f * c, f * b, f * a], axis=1)
    Q = U0.reshape(-1, 4)
    ar = E[:, 0] * Q[:, 0] - E[:, 1] * Q[:, 1] - (E[:, 2] * Q[:, 2] + E[:, 3] * Q[:, 3])
    ai = E[:, 0] * Q[:, 1] + E[:, 1] * Q[:, 0] - (E[:, 3] * Q[:, 2] - E[:, 2] * Q[:, 3])
    br = E[:, 0] * Q[:, 2] - E[:, 1] * Q[:, 3] + (E[:, 2] * Q[:, 0] + E[:, 3] * Q[:, 1])
    bi = E[:, 0] * Q[:, 3] + E[:, 1] * Q[:, 2] + (E[:, 3] * Q[:, 0] - E[:, 2] * Q[:, 1])
    return np.ascontiguousarray(np.stack([ar, ai, br, bi], axis=1).reshape(-1))


def _dexp_T(omega: np.ndarray, lam: np.ndarray) -> np.ndarray:
    """J(omega)^T lam with J the left-trivialised differential of exp on su(2)."""
    x = omega
    th = 2.0 * np.linalg.norm(x, axis=1)
    small = th < 1e-4
    ths = np.where(small, 1.0, th)
    c1 = np.where(small, 0.5 - th ** 2 / 24, (1 - np.cos(ths)) / ths ** 2)
    c2 = np.where(small, 1 / 6 - th ** 2 / 120, (ths - np.sin(ths)) / ths ** 3)
    ad = -2.0 * np.cross(x, lam)
    ad2 = -2.0 * np.cross(x, ad)
    return lam - c1[:, None] * ad + c2[:, None] * ad2


class WilsonAction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, omega, cfg, U0):
        om = omega.detach().cpu().numpy().astype(np.float64).reshape(-1, 3)
        cfg.upload(_exp_links(U0, om))
        S, dS = cfg.action_backward(1.0)
        ctx.save_for_backward(omega)
        ctx.dS = dS.reshape(-1, 3)
        return omega.new_tensor(S)

    @staticmethod
    def backward(ctx, grad):
        (omega,) = ctx.saved_tensors
        om = omega.detach().cpu().numpy().astype(np.float64).reshape(-1, 3)
        g = _dexp_T(om, ctx.dS) * float(grad)
        return torch.from_numpy(g).to(omega).reshape(omega.shape), None, None


class FlowEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, omega, cfg, U0, eps, n_steps, checkpoint_every=0):
        om = omega.detach().cpu().numpy().astype(np.float64).reshape(-1, 3)
        cfg.upload(_exp_links(U0, om))
        O, g = cfg.flow_objective(eps, n_steps, grad=True, checkpoint_every=checkpoint_every)
        ctx.save_for_backward(omega)
        ctx.g = g.reshape(-1, 3)
        return omega.new_tensor(O)

    @staticmethod
    def backward(ctx, grad):
        (omega,) = ctx.saved_tensors
        om = omega.detach().cpu().numpy().astype(np.float64).reshape(-1, 3)
        g = _dexp_T(om, ctx.g) * float(grad)
        return torch.from_numpy(g).to(omega).reshape(omega.shape), None, None, None, None, None

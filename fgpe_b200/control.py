"""Optimal control of the real-time evolution through the library's adjoint.

`ControlLoss` wraps gpe_control_gradient (forward RK4 with the control
potential W_n = V + sum_k u[n, k] G_k, final-state infidelity
1 - |<target|psi(T)>|^2, gradient by the hand-written adjoint with
checkpoints) as a torch.autograd.Function, so that a torch optimiser can
drive the controls; `optimise` is that driver.  Both run entirely through
libgpe: torch only holds the control array and applies the update.
"""
from __future__ import annotations

import numpy as np


def _torch():
    import torch
    return torch


class _ControlLossFn:
    """Built lazily so that importing this module does not import torch."""
    fn = None

    @classmethod
    def get(cls):
        if cls.fn is None:
            torch = _torch()

            class ControlLoss(torch.autograd.Function):
                @staticmethod
                def forward(ctx, u, solver, target, checkpoint_every):
                    un = u.detach().cpu().numpy().astype(np.float64)
                    loss, grad = solver.control_gradient(un, target, checkpoint_every, want_grad=True)
                    ctx.save_for_backward(torch.from_numpy(grad).to(u.dtype))
                    return u.new_tensor(loss)

                @staticmethod
                def backward(ctx, g):
                    (grad,) = ctx.saved_tensors
                    return g * grad.to(g.device), None, None, None

            cls.fn = ControlLoss
        return cls.fn


def control_loss(u, solver, target, checkpoint_every=50):
    """Infidelity as a differentiable function of the (nsteps, nctrl) tensor u."""
    return _ControlLossFn.get().apply(u, solver, target, checkpoint_every)


def optimise(solver, u0, target, iters=10, lr=0.5, checkpoint_every=50):
    """Gradient descent (torch.optim.Adam) on the controls; returns (u, losses)."""
    torch = _torch()
    u = torch.tensor(np.asarray(u0, dtype=np.float64), requires_grad=True)
    opt = torch.optim.Adam([u], lr=lr)
    losses = []
    for _ in range(iters):
        opt.zero_grad()
        loss = control_loss(u, solver, target, checkpoint_every)
        loss.backward()
        opt.step()
        losses.append(float(loss))
    return u.detach().numpy(), losses

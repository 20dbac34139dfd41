"""Differentiating react(): the discrete adjoint and its checking wrapper.

``Reactor.adjoint`` / ``Reactor.tangent`` (reactor.py) call the engine's
discrete adjoint and tangent-linear model of the BDF integration
(``ppb_adjoint_flat_device`` / ``ppb_tangent_flat_device``).  This module adds

* ``ReactFunction`` -- a thin ``torch.autograd.Function`` around them, used
  only to check the adjoint against torch-side compositions (the product path
  is the C ABI);
* ``rhs_exact`` -- pointwise exact derivatives of the reactor RHS;
* ``loss_T_OH`` -- the loss sum_cells(w_T T + w_OH Y_OH) of the adjoint
  workload and its seed dL/dy.

Parameters are [ln A | beta | Ea/R] per reaction (A as the mechanism tables
hold it, SI units; for fall-off reactions the high-pressure limit).
"""

from __future__ import annotations

import numpy as np

from ._lib import check, lib, mechanism_info
from .reactor import Reactor, _ptr


def params_of(reactor: Reactor):
    """The reactor's current parameter vector [ln A | beta | Ea/R] (numpy)."""
    A, b, e = reactor.get_arrhenius()
    return np.concatenate([np.log(A), b, e])


def set_params(reactor: Reactor, p):
    """Set [ln A | beta | Ea/R] on the reactor (a private copy of its tables)."""
    p = np.asarray(p, dtype=np.float64)
    R = reactor.nrxn
    reactor.set_arrhenius(np.exp(p[:R]), p[R:2 * R], p[2 * R:])


class ReactFunction:
    """y(dt) = react(y0, rhoe; p) with the discrete adjoint as its backward.

    For checking only.  ``apply(rY0, rX, params, reactor, rYsrc, rX_src, dt)``
    with torch CUDA float64 tensors: rY0 [ncells, N+1], rX [ncells], params
    [3R] (set on the reactor when they differ from its current values).
    """

    @staticmethod
    def apply(rY0, rX, params, reactor, rYsrc, rX_src, dt):
        return _function().apply(rY0, rX, params, reactor, rYsrc, rX_src, dt)


_fn = None


def _function():
    global _fn
    if _fn is not None:
        return _fn
    import torch

    class _ReactFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, rY0, rX, params, reactor, rYsrc, rX_src, dt):
            p = params.detach().cpu().numpy()
            if not np.array_equal(p, params_of(reactor)):
                set_params(reactor, p)
            y = rY0.detach().clone().contiguous()
            x = rX.detach().clone().contiguous()
            reactor.react(y, rYsrc, x, rX_src, dt)
            ctx.reactor = reactor
            ctx.dt = dt
            ctx.save_for_backward(rY0.detach(), rX.detach(), rYsrc, rX_src)
            return y

        @staticmethod
        def backward(ctx, gy):
            rY0, rX, rYsrc, rX_src = ctx.saved_tensors
            _, lam_y0, lam_e, grad = ctx.reactor.adjoint(rY0, rYsrc, rX, rX_src, ctx.dt, gy.contiguous())
            return lam_y0, lam_e, grad, None, None, None, None

    _fn = _ReactFn
    return _fn


def rhs_exact(mechanism, reactor_type, t, y, rhoe, rhoesrc=None, src=None, v=None):
    """f, df/dy ([c][j][i] = d f_i / d y_j), df/drhoe and, with weights v,
    v^T df/dy, v^T df/drhoe and v^T df/dp per cell (torch CUDA tensors)."""
    import torch

    nsp, nrxn = mechanism_info(mechanism)
    n = nsp + 1
    nc = y.shape[0]
    dev = y.device
    f = torch.empty((nc, n), dtype=torch.float64, device=dev)
    J = torch.empty((nc, n, n), dtype=torch.float64, device=dev)
    fE = torch.empty((nc, n), dtype=torch.float64, device=dev)
    vy = vE = vp = None
    if v is not None:
        vy = torch.empty((nc, n), dtype=torch.float64, device=dev)
        vE = torch.empty(nc, dtype=torch.float64, device=dev)
        vp = torch.empty((nc, 3 * nrxn), dtype=torch.float64, device=dev)
    check(lib().ppb_rhs_exact(mechanism.encode(), int(reactor_type), float(t), _ptr(y), _ptr(rhoe), _ptr(rhoesrc),
                              _ptr(src), _ptr(v), _ptr(f), _ptr(J), _ptr(fE), _ptr(vy), _ptr(vE), _ptr(vp), int(nc),
                              None))
    return f, J, fE, vy, vE, vp


def loss_T_OH(y, mw_index_oh, w_T, w_OH):
    """L = sum_c w_T[c] T[c] + w_OH[c] Y_OH[c] over y [ncells, N+1] (rhoY_k,
    T) and its seed dL/dy (numpy or torch, same kind as y)."""
    N = y.shape[1] - 1
    rho = y[:, :N].sum(1)
    Yoh = y[:, mw_index_oh] / rho
    L = (w_T * y[:, N] + w_OH * Yoh).sum()
    lam = y * 0.0
    lam[:, :N] = (-w_OH * Yoh / rho)[:, None]
    lam[:, mw_index_oh] += w_OH / rho
    lam[:, N] = w_T
    return L, lam

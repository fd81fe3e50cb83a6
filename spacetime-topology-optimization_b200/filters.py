"""Drop-in for ``sttopt.filters``' density path: the cone density filter and the
Heaviside projection (sttopt/filters.py:38-133), on the device.

``density_filter`` returns a :class:`ConeFilter` (the stencil behind the reference's
sparse ``H``) with the row sums ``Hs``; ``apply_density_filter`` applies it through
``stt_cone_filter`` and differentiates through ``stt_cone_filter_adjoint`` (``H`` is
symmetric, so its transpose is the same stencil).  ``filter_and_project`` fuses the
filter with the projection, forward and backward, in one kernel each.  The continuity
filter of the time field (``continuity_filter``) is not on this path.
"""

from __future__ import annotations

import math

import numpy as np
import torch
from torch import Tensor

from . import _lib


class ConeFilter:
    """``H[e1, e2] = max(0, rmin - dist(e1, e2))`` on an ``nelx x nely`` element grid,
    offsets ``|d| <= ceil(rmin) - 1`` (sttopt/filters.py:38-64), kept as its radius;
    ``tocsr()`` builds the explicit matrix on the host for callers that want it."""

    def __init__(self, nelx: int, nely: int, rmin: float):
        if not (0.0 < rmin <= 8.0):
            raise ValueError("rmin must be in (0, 8]")
        self.nelx, self.nely, self.rmin = int(nelx), int(nely), float(rmin)
        self.shape = (self.nelx * self.nely, self.nelx * self.nely)

    def _weights(self):
        r = int(math.ceil(self.rmin)) - 1
        return [(di, dj, max(0.0, self.rmin - math.hypot(di, dj)))
                for di in range(-r, r + 1) for dj in range(-r, r + 1)]

    def row_sums(self) -> np.ndarray:
        """``Hs``: per element, the sum of the weights that stay in the grid."""
        nelx, nely = self.nelx, self.nely
        i = np.arange(nelx * nely) % nelx
        j = np.arange(nelx * nely) // nelx
        hs = np.zeros(nelx * nely)
        for di, dj, w in self._weights():
            if w == 0.0:
                continue
            hs += w * ((i + di >= 0) & (i + di < nelx) & (j + dj >= 0) & (j + dj < nely))
        return hs

    def tocsr(self):
        import scipy.sparse as sp

        nelx, nely = self.nelx, self.nely
        e = np.arange(nelx * nely)
        i, j = e % nelx, e // nelx
        rows, cols, vals = [], [], []
        for di, dj, w in self._weights():
            if w == 0.0:
                continue
            ok = (i + di >= 0) & (i + di < nelx) & (j + dj >= 0) & (j + dj < nely)
            rows.append(e[ok])
            cols.append(((j + dj) * nelx + (i + di))[ok])
            vals.append(np.full(ok.sum(), w))
        return sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=self.shape).tocsr()


def density_filter(nelx: int, nely: int, rmin: float) -> tuple[ConeFilter, np.ndarray]:
    """The filter and its row sums ``Hs`` (sttopt/filters.py:38-64)."""
    H = ConeFilter(nelx, nely, rmin)
    return H, H.row_sums()


def _rows(field: Tensor, H: ConeFilter) -> tuple[Tensor, tuple]:
    nel = H.nelx * H.nely
    if field.shape[-2:] == (H.nely, H.nelx):
        batch = field.shape[:-2]
    elif field.shape[-1] == nel:
        batch = field.shape[:-1]
    else:
        raise ValueError(f"field of shape {tuple(field.shape)} is not on the {H.nelx}x{H.nely} grid")
    return field.detach().to(torch.float64).reshape(-1, nel).contiguous(), batch


def _filter(x: Tensor, H: ConeFilter, beta: float, eta: float) -> tuple[Tensor, Tensor | None]:
    _lib.require_cuda(x)
    X, batch = _rows(x, H)
    nel = X.shape[1]
    xt = torch.empty_like(X)
    xp = torch.empty_like(X) if beta > 0 else None
    _lib.check(_lib.lib().stt_cone_filter(H.nelx, H.nely, X.shape[0], H.rmin, _lib.ptr(X), nel, _lib.ptr(xt),
                                          _lib.ptr(xp), nel, float(beta), float(eta), _lib.stream()))
    shape = x.shape
    return xt.reshape(shape), (None if xp is None else xp.reshape(shape))


def _adjoint(g: Tensor, H: ConeFilter, xt: Tensor | None, beta: float, eta: float) -> Tensor:
    G, _ = _rows(g, H)
    nel = G.shape[1]
    T = None if xt is None else _rows(xt, H)[0]
    out = torch.empty_like(G)
    _lib.check(_lib.lib().stt_cone_filter_adjoint(H.nelx, H.nely, G.shape[0], H.rmin, _lib.ptr(G), nel,
                                                  _lib.ptr(T), nel, float(beta), float(eta), _lib.ptr(out),
                                                  nel, _lib.stream()))
    return out.reshape(g.shape)


class _Filter(torch.autograd.Function):
    @staticmethod
    def forward(ctx, field, H):
        ctx.H = H
        return _filter(field, H, 0.0, 0.5)[0].to(field.dtype)

    @staticmethod
    def backward(ctx, g):
        return _adjoint(g, ctx.H, None, 0.0, 0.5).to(g.dtype), None


class _FilterProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, field, H, beta, eta):
        xt, xp = _filter(field, H, beta, eta)
        ctx.H, ctx.beta, ctx.eta = H, beta, eta
        ctx.save_for_backward(xt)
        ctx.mark_non_differentiable(xt)
        return xp.to(field.dtype), xt.to(field.dtype)

    @staticmethod
    def backward(ctx, gp, gt):
        (xt,) = ctx.saved_tensors
        g = _adjoint(gp, ctx.H, xt, ctx.beta, ctx.eta)
        return g.to(gp.dtype), None, None, None


def apply_density_filter(field: Tensor, H: ConeFilter, Hs: Tensor | np.ndarray | None = None) -> Tensor:
    """``H @ field / Hs``, shape-preserving and differentiable (sttopt/filters.py:67-78).
    ``Hs`` is accepted for the reference's signature; the kernel forms the row sums."""
    if not isinstance(H, ConeFilter):
        raise TypeError("apply_density_filter takes the ConeFilter from this module's density_filter")
    return _Filter.apply(field, H)


def heaviside_projection(xTilde: Tensor, beta: float, eta: float) -> Tensor:
    """Smoothed threshold at ``eta`` (sttopt/filters.py:109-127)."""
    if math.isinf(beta):
        return torch.heaviside(xTilde - eta, xTilde.new_tensor(0.5))
    denom = math.tanh(beta * eta) + math.tanh(beta * (1 - eta))
    return (math.tanh(beta * eta) + torch.tanh(beta * (xTilde - eta))) / denom


def heaviside_projection_derivative(xTilde: Tensor, beta: float, eta: float) -> Tensor:
    """``d heaviside_projection / d xTilde`` (sttopt/filters.py:128-133)."""
    denom = math.tanh(beta * eta) + math.tanh(beta * (1 - eta))
    return beta * (1 - torch.tanh(beta * (xTilde - eta)) ** 2) / denom


def filter_and_project(x: Tensor, H: ConeFilter, beta: float, eta: float) -> tuple[Tensor, Tensor]:
    """``(xPhys, xTilde)`` with ``xTilde = H x / Hs`` and ``xPhys = P(xTilde)`` in one kernel;
    the backward pass is ``H (g * P'(xTilde) / Hs)`` in one kernel (the physical density
    of sttopt/stto_heat.py:180-189)."""
    if not isinstance(H, ConeFilter):
        raise TypeError("filter_and_project takes the ConeFilter from this module's density_filter")
    if not beta > 0:
        raise ValueError("beta must be positive (use apply_density_filter for the filter alone)")
    return _FilterProject.apply(x, H, float(beta), float(eta))


__all__ = ["ConeFilter", "density_filter", "apply_density_filter", "heaviside_projection",
           "heaviside_projection_derivative", "filter_and_project"]

"""Drop-in for ``sttopt.gravity``: the self-weight load matrix as a stencil on the device
(sttopt/gravity.py:15-36).

``C`` maps a per-element density field to the nodal self-weight (``fe / 4`` of each
element to each of its corners, ``fe = 1 / (nelx nely)``).  ``gravity_load_matrix``
returns a :class:`GravityLoad`, whose ``@`` runs ``stt_gravity_load`` (a node-centric
gather, no sparse matrix) and differentiates through its transpose; ``tocsr()`` builds
the reference's explicit matrix on the host for callers that want it.
"""

from __future__ import annotations

import numpy as np
import torch
from torch import Tensor

from . import _lib, fem


def _rows(x: Tensor, n: int) -> Tensor:
    if x.shape[-1] != n:
        raise ValueError(f"expected a trailing dimension of {n}, got {tuple(x.shape)}")
    return x.detach().to(torch.float64).reshape(-1, n).contiguous()


def _gather(x: Tensor, nelx: int, nely: int, transpose: bool) -> Tensor:
    _lib.require_cuda(x)
    nel, nnode = nelx * nely, (nelx + 1) * (nely + 1)
    n_in, n_out = (nnode, nel) if transpose else (nel, nnode)
    X = _rows(x, n_in)
    out = torch.empty(X.shape[0], n_out, dtype=torch.float64, device=X.device)
    _lib.check(_lib.lib().stt_gravity_load(nelx, nely, X.shape[0], _lib.ptr(X), n_in, _lib.ptr(out), n_out,
                                           int(transpose), _lib.stream()))
    return out.reshape(*x.shape[:-1], n_out)


class _Apply(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, nelx, nely, transpose):
        ctx.grid = (nelx, nely, transpose)
        return _gather(x, nelx, nely, transpose).to(x.dtype)

    @staticmethod
    def backward(ctx, g):
        nelx, nely, transpose = ctx.grid
        return _gather(g, nelx, nely, not transpose).to(g.dtype), None, None, None


class GravityLoad:
    """``C``, shape ``((nelx+1)(nely+1), nelx nely)``: ``C @ x`` for an element field
    ``x`` (trailing dimension ``nel``), ``C.T @ g`` for a nodal one."""

    def __init__(self, nelx: int, nely: int, transpose: bool = False):
        self.nelx, self.nely, self.transpose = int(nelx), int(nely), bool(transpose)
        nnode, nel = (self.nelx + 1) * (self.nely + 1), self.nelx * self.nely
        self.shape = (nel, nnode) if self.transpose else (nnode, nel)

    @property
    def T(self) -> "GravityLoad":
        return GravityLoad(self.nelx, self.nely, not self.transpose)

    def to(self, *args, **kwargs) -> "GravityLoad":
        return self  # a stencil: nothing to move

    def __matmul__(self, x: Tensor) -> Tensor:
        return _Apply.apply(x, self.nelx, self.nely, self.transpose)

    def tocsr(self):
        import scipy.sparse as sp

        nelx, nely = self.nelx, self.nely
        nodes = fem.node_grid(nelx, nely)
        rows = np.concatenate([nodes[:-1, :-1].ravel(), nodes[1:, :-1].ravel(),
                               nodes[:-1, 1:].ravel(), nodes[1:, 1:].ravel()])
        cols = np.tile(np.arange(nelx * nely), 4)
        vals = np.full(rows.size, 0.25 / (nelx * nely))
        C = sp.coo_matrix((vals, (rows, cols)), shape=((nelx + 1) * (nely + 1), nelx * nely)).tocsr()
        return C.T.tocsr() if self.transpose else C


def gravity_load_matrix(nelx: int, nely: int) -> GravityLoad:
    """The self-weight load matrix ``C`` (sttopt/gravity.py:15-36), as a device stencil."""
    return GravityLoad(nelx, nely)


__all__ = ["GravityLoad", "gravity_load_matrix"]

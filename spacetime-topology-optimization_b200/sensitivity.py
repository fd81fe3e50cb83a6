"""Drop-in for ``sttopt.sensitivity``: per-output Jacobian rows (sttopt/sensitivity.py:15-52).

One ``torch.autograd.grad`` per output; with this package's modules in the graph each
row runs the hand-written adjoint kernels of ``FemSolve.backward``.
"""

from __future__ import annotations

from typing import Sequence

import torch
from torch import Tensor


def jacobian_rows(outputs: Tensor, leaves: Sequence[Tensor]) -> tuple[Tensor, ...]:
    """One ``(k, leaf.numel())`` block per leaf; an unused leaf's block is zero."""
    rows = [torch.autograd.grad(o, tuple(leaves), retain_graph=True, allow_unused=True) for o in outputs]
    return tuple(
        torch.stack([
            torch.zeros(leaf.numel(), dtype=leaf.dtype, device=leaf.device) if g is None else g.reshape(-1)
            for g in grads
        ])
        for leaf, grads in zip(leaves, zip(*rows))
    )

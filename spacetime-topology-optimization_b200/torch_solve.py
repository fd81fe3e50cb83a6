"""Drop-in for ``sttopt.torch_solve``: the MG-PCG solve as an autograd ``Function``.

Forward builds the device hierarchy through ``torch_mg.build_hierarchy`` (looked up on
the module at call time, as the reference does, so it stays a patch point) and runs
the device PCG.  Backward reuses that hierarchy, warm-starts the adjoint from
``alpha U`` with ``alpha = (U . g) / (U . F)`` (exact for compliance, which therefore
returns at iteration 0) and forms the element terms in one kernel:
``grad_density = -lam_e^T KE U_e``, ``grad_reaction = -lam_e . U_e / 4``, ``grad_F = lam``
(sttopt/torch_solve.py:52-173).
"""

from __future__ import annotations

import torch
from torch import Tensor

from . import torch_fem, torch_mg

DEFAULT_CG_RTOL = 1e-8  # sttopt/torch_solve.py:49


class FemSolve(torch.autograd.Function):
    """``K @ U = F`` as a differentiable op (sttopt/torch_solve.py:52-173).

    With ``recompute`` the forward pass keeps the hierarchy but not ``U``: the backward
    pass solves for ``U`` again (the same kernels on the same inputs, so the same ``U``)
    before the adjoint, trading one forward solve for the memory of ``U``."""

    @staticmethod
    def forward(ctx, density, F, reaction, edofMat, KE, mask, nelx, nely, rtol, max_iter, x0,
                omega, n_smooth, gamma, max_coarse_elements, info, precision=None, recompute=False):
        levels = torch_mg.build_hierarchy(density, edofMat, KE, mask, nelx, nely, reaction=reaction,
                                          max_coarse_elements=max_coarse_elements, precision=precision)
        precond = torch_mg.VCycle(levels, omega=omega, n_smooth=n_smooth, gamma=gamma)
        b = torch_fem.project(F, mask)
        U, n_iter = torch_fem.pcg(levels[0], b, precond, rtol=rtol, max_iter=max_iter, x0=x0)
        U = torch_fem.project(U, mask)
        ctx.recompute = bool(recompute)
        if ctx.recompute:
            ctx.x0 = None if x0 is None else x0.detach()
            ctx.save_for_backward(density, F)
        else:
            ctx.save_for_backward(U, density, F)
        ctx.levels = levels
        ctx.edofMat, ctx.KE, ctx.mask = edofMat, KE, mask
        ctx.rtol, ctx.max_iter = rtol, max_iter
        ctx.omega, ctx.n_smooth, ctx.gamma = omega, n_smooth, gamma
        ctx.info = info
        if info is not None:
            info["forward_n_iter"] = n_iter
        return U

    @staticmethod
    def backward(ctx, grad_output):
        if ctx.recompute:
            density, F = ctx.saved_tensors
            precond = torch_mg.VCycle(ctx.levels, omega=ctx.omega, n_smooth=ctx.n_smooth, gamma=ctx.gamma)
            U, _ = torch_fem.pcg(ctx.levels[0], torch_fem.project(F, ctx.mask), precond, rtol=ctx.rtol,
                                 max_iter=ctx.max_iter, x0=ctx.x0)
            U = torch_fem.project(U, ctx.mask)
        else:
            U, density, F = ctx.saved_tensors
        Fb = F.expand_as(U)
        UF = torch_fem._dots(U.contiguous(), Fb.contiguous())
        Ug = torch_fem._dots(U.contiguous(), grad_output.expand_as(U).contiguous())
        alpha = torch_fem.safe_div(Ug, UF)
        x0 = alpha[..., None] * U
        precond = torch_mg.VCycle(ctx.levels, omega=ctx.omega, n_smooth=ctx.n_smooth, gamma=ctx.gamma)
        b = torch_fem.project(grad_output, ctx.mask)
        lam, n_iter = torch_fem.pcg(ctx.levels[0], b, precond, rtol=ctx.rtol, max_iter=ctx.max_iter, x0=x0)
        lam = torch_fem.project(lam, ctx.mask)
        if ctx.info is not None:
            ctx.info["backward_n_iter"] = n_iter
        grad_density = grad_reaction = None
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[2]:
            terms = torch_fem.element_terms(U, ctx.edofMat, ctx.KE, lam=lam)
            grad_density = terms["gdens"] if ctx.needs_input_grad[0] else None
            grad_reaction = terms["greac"] if ctx.needs_input_grad[2] else None
        grad_F = lam if ctx.needs_input_grad[1] else None
        return (grad_density, grad_F, grad_reaction) + (None,) * 15


def femsolve(density: Tensor, F: Tensor, edofMat: Tensor, KE: Tensor, mask: Tensor, nelx: int,
             nely: int, *, rtol: float = DEFAULT_CG_RTOL, max_iter: int = 500,
             x0: Tensor | None = None, omega: float = 0.6, n_smooth: int = 2, gamma: int = 1,
             max_coarse_elements: int = torch_mg.MAX_COARSE_ELEMENTS, info: dict | None = None,
             reaction: Tensor | None = None, precision: str | None = None, recompute: bool = False) -> Tensor:
    """``FemSolve.apply`` with the reference's keyword defaults (sttopt/torch_solve.py:176-243).

    ``precision`` ("fp64" default, or "mixed") selects the V-cycle precision; the outer
    PCG is FP64 either way.  ``recompute`` keeps ``U`` out of the autograd graph and solves
    for it again in the backward pass (memory for one more solve).
    """
    assert x0 is None or not x0.requires_grad, (
        "femsolve: the warm start x0 requires grad, but the solve has no gradient for it; "
        "pass x0.detach()"
    )
    return FemSolve.apply(density, F, reaction, edofMat, KE, mask, nelx, nely, rtol, max_iter, x0,
                          omega, n_smooth, gamma, max_coarse_elements, info, precision, recompute)


def lifted_femsolve(density: Tensor, F: Tensor, g: Tensor, edofMat: Tensor, KE: Tensor,
                    mask: Tensor, nelx: int, nely: int, *, reaction: Tensor | None = None,
                    **solve_kwargs) -> Tensor:
    """``femsolve`` with Dirichlet data ``g`` on the fixed dofs by lifting
    (sttopt/torch_solve.py:246-287)."""
    lift = g * ~mask
    K_lift = torch_fem.matvec(lift, density, edofMat, KE, mask.shape[-1])
    if reaction is not None:
        K_lift = K_lift + torch_fem.lumped_reaction(reaction, edofMat, mask.shape[-1]) * lift
    free = femsolve(density, F - K_lift, edofMat, KE, mask, nelx, nely, reaction=reaction, **solve_kwargs)
    return free + lift

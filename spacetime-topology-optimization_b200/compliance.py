"""Drop-in for the solve-facing part of ``sttopt.compliance``: stage masks, strain
energy, gravity load and the batched whole + stage compliance call
(sttopt/compliance.py:33-253).

``_solve_fe`` / ``_solve_fe_batched`` stay module attributes (the reference's patch
points).  ``time_mask`` is the reference's smooth indicator; ``hard_time_mask`` is
the hard threshold ``tPhys <= ti`` the space-time configurations use.
"""

from __future__ import annotations

import math

import torch
from torch import Tensor

from . import torch_fem, torch_solve


def time_mask(tPhys: Tensor, ti: float, beta: float) -> Tensor:
    """Smooth stage indicator (sttopt/compliance.py:33-46)."""
    num = math.tanh(beta * ti) + torch.tanh(beta * (tPhys - ti))
    den = math.tanh(beta * ti) + math.tanh(beta * (1 - ti))
    return torch.clamp(1 - num / den, min=0)


def hard_time_mask(tPhys: Tensor, ti: float, beta: float | None = None) -> Tensor:
    """Hard stage membership ``tPhys <= ti`` as 0/1 (not differentiable in ``tPhys``)."""
    return (tPhys <= ti).to(tPhys.dtype)


class _StrainEnergy(torch.autograd.Function):
    """``ce_e = U_e^T KE U_e`` in one kernel; backward ``dU = 2 K(g) U`` (the element
    weights ``g`` act as a density field)."""

    @staticmethod
    def forward(ctx, U, edofMat, KE):
        ctx.save_for_backward(U)
        ctx.edofMat, ctx.KE = edofMat, KE
        return torch_fem.element_terms(U, edofMat, KE)["ce"]

    @staticmethod
    def backward(ctx, g):
        (U,) = ctx.saved_tensors
        return 2 * torch_fem._apply(U.to(torch.float64), g.contiguous().to(torch.float64), ctx.edofMat,
                                    ctx.KE, U.shape[-1], None, None, 0), None, None


def _element_strain_energy(U: Tensor, edofMat: Tensor, KE: Tensor, nely: int, nelx: int) -> Tensor:
    """``U_e^T KE U_e`` on the ``(nely, nelx)`` grid (sttopt/compliance.py:49-59)."""
    return _StrainEnergy.apply(U, edofMat, KE).reshape(nely, nelx)


def _solve_fe(KE, xPhys, Emin, Emax, penal, edofMat, freedofs, F, ndof, *, x0=None):
    """One solve through ``femsolve`` (sttopt/compliance.py:62-87)."""
    nely, nelx = xPhys.shape
    density = torch_fem.simp_density(xPhys, Emin, Emax, penal)
    mask = torch_fem.free_mask(ndof, freedofs, device=xPhys.device)
    return torch_solve.femsolve(density.flatten(), F, edofMat, KE, mask, nelx, nely, x0=x0)


def _solve_fe_batched(KE, density, edofMat, mask, nelx, nely, F, *, x0=None):
    """Batched solve patch point (sttopt/compliance.py:90-108)."""
    return torch_solve.femsolve(density, F, edofMat, KE, mask, nelx, nely, x0=x0)


def whole_compliance(xPhys, KE, edofMat, Emin, Emax, penal, freedofs, F, ndof, *, x0=None):
    """SIMP compliance under a fixed load (sttopt/compliance.py:111-134)."""
    U = _solve_fe(KE, xPhys, Emin, Emax, penal, edofMat, freedofs, F, ndof, x0=x0)
    nely, nelx = xPhys.shape
    ce = _element_strain_energy(U, edofMat, KE, nely, nelx)
    simp = Emin + xPhys**penal * (Emax - Emin)
    return torch.sum(simp * ce), U


def _gravity_load(xPhys, tPhys, ti, C, beta_t, ndof, mask_fn=None):
    """Stage mask, ``xtJoint`` and self-weight load ``F[1::2] = -C xt``
    (sttopt/compliance.py:137-161)."""
    t_mask = (time_mask if mask_fn is None else mask_fn)(tPhys, ti, beta_t)
    xtJoint = xPhys * t_mask
    f = -(C @ xtJoint.flatten())
    F = torch.zeros(ndof, dtype=xPhys.dtype, device=xPhys.device)
    F[1::2] = f
    return t_mask, xtJoint, F


def gravity_compliance(xPhys, tPhys, KE, edofMat, Emin, Emax, penal, ti, C, beta_t, freedofs, ndof,
                       *, x0=None):
    """Self-weight compliance of one stage (sttopt/compliance.py:164-195)."""
    _, xtJoint, F = _gravity_load(xPhys, tPhys, ti, C, beta_t, ndof)
    U = _solve_fe(KE, xtJoint, Emin, Emax, penal, edofMat, freedofs, F, ndof, x0=x0)
    nely, nelx = xPhys.shape
    ce = _element_strain_energy(U, edofMat, KE, nely, nelx)
    simp = Emin + xtJoint**penal * (Emax - Emin)
    return torch.sum(simp * ce), U


def batched_whole_and_gravity_compliance(xPhys, tPhys, KE, edofMat, Emin, Emax, penal, freedofs, F,
                                         ndof, C, beta_t, stage_times, *, x0=None, mask_fn=None):
    """Whole compliance + every stage's gravity compliance in one batched ``femsolve``
    (sttopt/compliance.py:198-253).  ``mask_fn`` replaces ``time_mask`` (e.g.
    ``hard_time_mask``)."""
    nely, nelx = xPhys.shape
    mask = torch_fem.free_mask(ndof, freedofs, device=xPhys.device)
    density_rows = [torch_fem.simp_density(xPhys, Emin, Emax, penal).flatten()]
    F_rows = [F]
    xtJoints = []
    for ti in stage_times:
        _, xtJoint, F_g = _gravity_load(xPhys, tPhys, ti, C, beta_t, ndof, mask_fn)
        density_rows.append(torch_fem.simp_density(xtJoint, Emin, Emax, penal).flatten())
        F_rows.append(F_g)
        xtJoints.append(xtJoint)
    density = torch.stack(density_rows)
    F_stack = torch.stack(F_rows)
    U = _solve_fe_batched(KE, density, edofMat, mask, nelx, nely, F_stack, x0=x0)
    ce_whole = _element_strain_energy(U[0], edofMat, KE, nely, nelx)
    c = torch.sum((Emin + xPhys**penal * (Emax - Emin)) * ce_whole)
    stages = []
    for i, xtJoint in enumerate(xtJoints):
        ce = _element_strain_energy(U[1 + i], edofMat, KE, nely, nelx)
        stages.append(torch.sum((Emin + xtJoint**penal * (Emax - Emin)) * ce))
    return c, stages, U

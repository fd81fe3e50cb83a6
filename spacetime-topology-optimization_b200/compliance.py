"""Drop-in for the solve-facing part of ``sttopt.compliance``: stage masks, strain
energy, the self-weight load and the batched whole + stage compliance call
(sttopt/compliance.py:33-253), on this package's kernels.

Every compliance here has the form ``c_r = sum_e rho_r[e] (U_r,e^T KE U_r,e)`` for a
row ``r`` of one batched solve ``K(rho_r) U_r = F_r``, where ``rho_r`` is the SIMP
density of the row's material: ``x`` for the whole structure, ``xt_s = x * m_s`` for
stage ``s``.  So the module is three autograd nodes around the solve:

1. ``_StageRows``: every stage mask (the smooth ``time_mask`` evaluated in the kernel, or
   the caller's mask rows), the stage materials, the density rows and the load rows (the
   self-weight ``F[1::2] = -C xt`` as a node-centric gather when ``C`` is this package's
   ``GravityLoad``) in one device pass, ``stt_stage_glue_rows``.  Its backward folds the
   density, load and material gradients of all rows into ``d/dx`` and ``d/dt`` (or
   ``d/dmask``) in one pass, ``stt_stage_glue_adjoint``.
2. The solve, through the reference's patch points ``_solve_fe`` / ``_solve_fe_batched``
   (module attributes, so a substitute solver still sees every call).
3. ``_RowCompliance``: ``c_r`` of every row (``stt_element_sens`` for the element
   energies, ``stt_vec_dots`` for the weighted sums); backward ``dc_r/dU_r =
   2 K(rho_r) U_r`` in one batched apply and ``dc_r/drho_r = ce_r``.

``hard_time_mask`` is the hard threshold ``tPhys <= ti`` the space-time configurations
use, passed as ``mask_fn``.
"""

from __future__ import annotations

import math

import torch
from torch import Tensor

from . import _lib, gravity, torch_fem, torch_solve


def time_mask(tPhys: Tensor, ti: float, beta: float) -> Tensor:
    """Smooth stage indicator (sttopt/compliance.py:33-46), for callers that want the
    mask itself; the batched path evaluates the same formula inside its row kernel."""
    num = math.tanh(beta * ti) + torch.tanh(beta * (tPhys - ti))
    den = math.tanh(beta * ti) + math.tanh(beta * (1 - ti))
    return torch.clamp(1 - num / den, min=0)


def hard_time_mask(tPhys: Tensor, ti: float, beta: float | None = None) -> Tensor:
    """Hard stage membership ``tPhys <= ti`` as 0/1 (not differentiable in ``tPhys``)."""
    return (tPhys <= ti).to(tPhys.dtype)


def _f64(v: Tensor | None) -> Tensor | None:
    return None if v is None else v.detach().to(torch.float64).contiguous()


class _StageRows(torch.autograd.Function):
    """Stage materials ``xt (S, nel)``, density rows ``rho (R, nel)`` and load rows
    ``F (R, ndof)`` (``R = S + whole``; row 0 the whole structure when ``whole``).  The
    masks are the smooth indicator of ``t`` at ``times`` when ``M`` is None, else ``M``.
    ``F`` is computed only with ``loads`` (the gravity stencil), else left empty."""

    @staticmethod
    def forward(ctx, x, t, M, F0, times, beta, Emin, Emax, penal, nelx, nely, whole, loads):
        S = len(times)
        nel, ndof = nelx * nely, 2 * (nelx + 1) * (nely + 1)
        dev = x.device
        xd, td, Md, F0d = _f64(x), _f64(t) if M is None else None, _f64(M), _f64(F0) if whole else None
        xt = torch.empty(S, nel, dtype=torch.float64, device=dev)
        rho = torch.empty(S + whole, nel, dtype=torch.float64, device=dev)
        F = torch.empty(S + whole if loads else 0, ndof, dtype=torch.float64, device=dev)
        ts = _lib.dbl_array([float(v) for v in times]) if S else None
        _lib.check(_lib.lib().stt_stage_glue_rows(
            nelx, nely, S, int(whole), _lib.ptr(xd), _lib.ptr(td), ts, float(beta), _lib.ptr(Md), None,
            _lib.ptr(F0d), Emin, Emax, penal, _lib.ptr(xt), _lib.ptr(rho), _lib.ptr(F) if loads else None,
            _lib.stream()))
        ctx.save_for_backward(xd, td, Md)
        ctx.args = (tuple(float(v) for v in times), float(beta), Emin, Emax, penal, nelx, nely, int(whole), loads)
        if not loads:
            ctx.mark_non_differentiable(F)
        return xt, rho, F

    @staticmethod
    def backward(ctx, g_xt, g_rho, g_F):
        xd, td, Md = ctx.saved_tensors
        times, beta, Emin, Emax, penal, nelx, nely, whole, loads = ctx.args
        S = len(times)
        need_x, need_t, need_M, need_F0 = ctx.needs_input_grad[:4]
        gx = torch.empty_like(xd)
        gt = torch.empty_like(xd) if (need_t and td is not None) else None
        gM = torch.empty(S, xd.numel(), dtype=torch.float64, device=xd.device) if (need_M and Md is not None) else None
        gF = _f64(g_F) if (loads and g_F is not None) else None
        ts = _lib.dbl_array(list(times)) if S else None
        _lib.check(_lib.lib().stt_stage_glue_adjoint(
            nelx, nely, S, whole, _lib.ptr(xd), _lib.ptr(td), ts, beta, _lib.ptr(Md), _lib.ptr(_f64(g_xt)),
            _lib.ptr(_f64(g_rho)), _lib.ptr(gF), Emin, Emax, penal, _lib.ptr(gx), _lib.ptr(gt), _lib.ptr(gM),
            _lib.stream()))
        gF0 = gF[0] if (need_F0 and whole and gF is not None) else None
        return (gx if need_x else None, gt, gM, gF0) + (None,) * 9


def _stage_rows(xPhys: Tensor, tPhys: Tensor | None, times, beta: float, masks: Tensor | None, C, F0,
                Emin: float, Emax: float, penal: float, whole: bool):
    """``(xt, rho, F)`` rows of one batched solve (see ``_StageRows``); a ``C`` other than
    this grid's ``GravityLoad`` (e.g. the reference's torch CSR matrix) gives the stage
    loads through ``C @ xt`` instead."""
    nely, nelx = xPhys.shape
    ndof = 2 * (nelx + 1) * (nely + 1)
    loads = isinstance(C, gravity.GravityLoad) and (C.nelx, C.nely, C.transpose) == (nelx, nely, False)
    t = None if tPhys is None else tPhys.reshape(-1)
    xt, rho, F = _StageRows.apply(xPhys.reshape(-1), t, masks, F0, tuple(times), beta, Emin, Emax, penal,
                                  nelx, nely, whole, loads)
    if not loads and (len(times) or F0 is not None):
        rows = []
        if whole and F0 is not None:
            rows.append(F0.reshape(1, ndof).to(torch.float64))
        if len(times):
            f = torch.stack([-(C @ xt[s]) for s in range(len(times))])
            rows.append(torch.stack((torch.zeros_like(f), f), dim=-1).reshape(len(times), ndof))
        F = torch.cat(rows)
    return xt, rho, F


class _RowCompliance(torch.autograd.Function):
    """``c_r = sum_e rho_r[e] ce_r[e]`` for every row of ``U (R, ndof)``."""

    @staticmethod
    def forward(ctx, U, rho, edofMat, KE):
        Ud, rd = _f64(U), _f64(rho)
        ce = torch_fem.element_terms(Ud, edofMat, KE)["ce"]
        c = torch_fem._dots(rd, ce)
        ctx.save_for_backward(Ud, rd, ce)
        ctx.edofMat, ctx.KE = edofMat, KE
        return c

    @staticmethod
    def backward(ctx, gc):
        Ud, rd, ce = ctx.saved_tensors
        gc = gc.to(torch.float64).reshape(-1, 1)
        gU = grho = None
        if ctx.needs_input_grad[0]:
            # d c_r / d U_r = 2 K(rho_r) U_r, the row weight folded into the density (K is linear in it)
            gU = torch_fem._apply(Ud, (2 * gc) * rd, ctx.edofMat, ctx.KE, Ud.shape[-1], None, None, 0)
        if ctx.needs_input_grad[1]:
            grho = gc * ce
        return gU, grho, None, None


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
    """The single-solve patch point (sttopt/compliance.py:62-87): SIMP density of
    ``xPhys``, then ``femsolve``."""
    nely, nelx = xPhys.shape
    density = torch_fem.simp_density(xPhys, Emin, Emax, penal)
    mask = torch_fem.free_mask(ndof, freedofs, device=xPhys.device)
    return torch_solve.femsolve(density.flatten(), F, edofMat, KE, mask, nelx, nely, x0=x0)


def _solve_fe_batched(KE, density, edofMat, mask, nelx, nely, F, *, x0=None):
    """The batched patch point (sttopt/compliance.py:90-108): density and load rows
    already formed."""
    return torch_solve.femsolve(density, F, edofMat, KE, mask, nelx, nely, x0=x0)


def _compliance(U: Tensor, rho: Tensor, edofMat: Tensor, KE: Tensor) -> Tensor:
    return _RowCompliance.apply(U.reshape(-1, U.shape[-1]), rho, edofMat, KE)


def whole_compliance(xPhys, KE, edofMat, Emin, Emax, penal, freedofs, F, ndof, *, x0=None):
    """SIMP compliance under the fixed load ``F`` (sttopt/compliance.py:111-134):
    ``(c, U)``."""
    U = _solve_fe(KE, xPhys, Emin, Emax, penal, edofMat, freedofs, F, ndof, x0=x0)
    _, rho, _ = _stage_rows(xPhys, None, (), 0.0, None, None, None, Emin, Emax, penal, whole=True)
    return _compliance(U, rho, edofMat, KE)[0], U


def _gravity_load(xPhys, tPhys, ti, C, beta_t, ndof, mask_fn=None):
    """One stage's ``(t_mask, xtJoint, F)`` with ``F[1::2] = -C xtJoint``
    (sttopt/compliance.py:137-161)."""
    t_mask = (time_mask if mask_fn is None else mask_fn)(tPhys, ti, beta_t)
    xt, _, F = _stage_rows(xPhys, tPhys, (ti,), beta_t, t_mask.reshape(1, -1), C, None, 0.0, 1.0, 1.0,
                           whole=False)
    return t_mask, xt[0].reshape(xPhys.shape), F[0]


def gravity_compliance(xPhys, tPhys, KE, edofMat, Emin, Emax, penal, ti, C, beta_t, freedofs, ndof,
                       *, x0=None):
    """Self-weight compliance of the material built by stage time ``ti``
    (sttopt/compliance.py:164-195): ``(cg, U)``."""
    xt, rho, F = _stage_rows(xPhys, tPhys, (ti,), beta_t, None, C, None, Emin, Emax, penal, whole=False)
    U = _solve_fe(KE, xt[0].reshape(xPhys.shape), Emin, Emax, penal, edofMat, freedofs, F[0], ndof, x0=x0)
    return _compliance(U, rho, edofMat, KE)[0], U


def batched_whole_and_gravity_compliance(xPhys, tPhys, KE, edofMat, Emin, Emax, penal, freedofs, F,
                                         ndof, C, beta_t, stage_times, *, x0=None, mask_fn=None):
    """The whole structure under ``F`` plus one self-weight row per stage time, as ONE
    batched solve (sttopt/compliance.py:198-253): ``(c, [c_s, ...], U)`` with ``U`` of
    shape ``(1 + len(stage_times), ndof)``.  ``mask_fn`` replaces ``time_mask`` (e.g.
    ``hard_time_mask``)."""
    nely, nelx = xPhys.shape
    masks = None
    if mask_fn is not None and mask_fn is not time_mask and len(stage_times):
        masks = torch.stack([mask_fn(tPhys, ti, beta_t).reshape(-1) for ti in stage_times])
    _, rho, F_rows = _stage_rows(xPhys, tPhys, stage_times, beta_t, masks, C, F, Emin, Emax, penal, whole=True)
    free = torch_fem.free_mask(ndof, freedofs, device=xPhys.device)
    U = _solve_fe_batched(KE, rho, edofMat, free, nelx, nely, F_rows, x0=x0)
    c = _compliance(U, rho, edofMat, KE)
    return c[0], list(c[1:].unbind(0)), U

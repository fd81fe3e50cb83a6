"""The space-time objective and its gradient in one batched device pass.

For a density field ``xPhys`` on an ``nelx x nely`` grid (bottom node row clamped and
the build plate, self-weight loading, SIMP ``Emin + x^p (E0 - Emin)``):

1. virtual-heat time field: ``-div(chi grad T) + alpha T = 0``, ``T = 1`` on the plate,
   ``chi = max(x^q, 1e-6)`` (``q`` the conduction penalty, ``mu = 1/2``),
   ``alpha = drain_beta / (nelx nely)``; ``t = 1 - T``, element means, normalised over
   the part (sttopt/virtual_heat.py:404-462);
2. stage membership ``m_s = [tPhys <= s / n_stage]`` (bit-exact FP64 compare);
3. all stage solves ``K(x m_s) U_s = F_s`` with ``F_s[y] = -C (x m_s)`` as ONE batched
   device PCG (sttopt/compliance.py:137-161,198-253 with the hard threshold);
4. objective ``sum_s c_s + sum(w tPhys)``;
5. gradient: the stage adjoints (warm-started at ``alpha U``, exact for compliance), the
   element terms and the load-dependence term in one kernel, plus the true adjoint of
   the heat solve on the heat hierarchy.

``precision="mixed"`` runs both V-cycles in FP32 inside the FP64 PCG; ``"fp64"`` runs
everything in FP64.  ``batched=False`` solves the stages one at a time (the plain
form the batched one is compared against).
"""

from __future__ import annotations

import torch
from torch import Tensor

from . import _geom, _lib, fem, torch_fem, torch_mg

EMIN, EMAX, PENAL, NU = 1e-9, 1.0, 3.0, 0.3


class SpaceTimeProblem:
    """Grid-level constants of the space-time objective, built once per shape."""

    def __init__(self, nelx: int, nely: int, device, *, nu: float = NU):
        self.nelx, self.nely = nelx, nely
        self.nel = nelx * nely
        self.nnode = (nelx + 1) * (nely + 1)
        self.device = device
        self.KE = torch.tensor(fem.plane_stress_KE(nu), dtype=torch.float64, device=device)
        self.KEh = torch.tensor(fem.diffusion_KE(), dtype=torch.float64, device=device)
        self.edof = torch_mg.element_dof_map_tensor(nelx, nely, device, 2)
        self.edof1 = torch_mg.element_dof_map_tensor(nelx, nely, device, 1)
        nodes = torch.arange(self.nnode, device=device).reshape(nely + 1, nelx + 1)
        plate = torch.zeros(self.nnode, dtype=torch.bool, device=device)
        plate[nodes[-1, :].reshape(-1)] = True
        self.plate = plate
        self.heat_mask = ~plate
        self.mask = (~plate)[:, None].expand(self.nnode, 2).reshape(-1).contiguous()
        self.fixed2 = _geom.fixed_flags(self.mask, self.nnode, 2)
        self.fixed1 = _geom.fixed_flags(self.heat_mask, self.nnode, 1)
        self.lift = plate.to(torch.float64)
        self.ke = _lib.dbl_array(_geom.host_KE(self.KE))
        self.keh = _lib.dbl_array(_geom.host_KE(self.KEh))


def _pcg(levels, b, x0, rtol, max_iter, info_key, info):
    M = torch_mg.VCycle(levels)
    sub = {}
    x, n = torch_fem.pcg(levels[0], b, M, rtol=rtol, max_iter=max_iter, x0=x0, info=sub)
    if info is not None:
        info[info_key] = n
    return x


def objective_and_gradient(xPhys: Tensor, w: Tensor, *, n_stage: int = 16, precision: str = "mixed",
                           rtol: float = 1e-8, max_iter: int = 500, drain_beta: float = 25.0,
                           conduction_penal: float = 3.0, Emin: float = EMIN, Emax: float = EMAX,
                           penal: float = PENAL, max_coarse_elements: int = torch_mg.MAX_COARSE_ELEMENTS,
                           gradient: bool = True, batched: bool = True,
                           problem: SpaceTimeProblem | None = None, info: dict | None = None) -> dict:
    """Objective, stage compliances, ``tPhys`` and (optionally) ``d objective / d xPhys``."""
    _lib.require_cuda(xPhys, w)
    nely, nelx = xPhys.shape
    dev = xPhys.device
    P = problem if problem is not None and (problem.nelx, problem.nely) == (nelx, nely) else \
        SpaceTimeProblem(nelx, nely, dev)
    L = _lib.lib()
    st = _lib.stream()
    x = xPhys.detach().to(torch.float64).reshape(-1).contiguous()
    nel, nnode = P.nel, P.nnode

    # 1. heat time field
    chi = torch.clamp(x ** conduction_penal, min=1e-6).contiguous()
    alpha = drain_beta / (nelx * nely)
    reac = torch.full_like(chi, alpha)
    hl = torch_mg.build_hierarchy(chi, P.edof1, P.KEh, P.heat_mask, nelx, nely, reaction=reac,
                                  max_coarse_elements=max_coarse_elements, precision=precision)
    rdiag = hl[0].reaction_diag
    Klift = torch.empty(nnode, dtype=torch.float64, device=dev)
    _lib.check(L.stt_q4_apply(_lib.STT_FP64, 1, nelx, nely, 1, _lib.ptr(P.lift), nnode, _lib.ptr(Klift),
                              nnode, _lib.ptr(chi), nel, _lib.ptr(rdiag), nnode, _lib.ptr(P.fixed1),
                              _lib.STT_PROJECT_OUT, P.keh, st))
    heat_rhs = (-Klift).contiguous()  # F - K_lift, projected (F = 0)
    T_free = _pcg(hl, heat_rhs, None, rtol, max_iter, "heat_n_iter", info)
    T = T_free + P.lift
    t_e = torch.empty(nel, dtype=torch.float64, device=dev)
    _lib.check(L.stt_heat_element_means(nelx, nely, _lib.ptr(T), _lib.ptr(t_e), st))
    part = x >= x.max() / 2
    scale = torch.where(part, t_e, torch.full_like(t_e, -torch.inf)).max()
    tPhys = (t_e / scale).contiguous()

    # 2.-3. stage rows and the batched stage solves
    member = torch.empty(n_stage, nel, dtype=torch.uint8, device=dev)
    _lib.check(L.stt_stage_membership(nel, n_stage, _lib.ptr(tPhys), _lib.ptr(member), st))
    rho = torch.empty(n_stage, nel, dtype=torch.float64, device=dev)
    F = torch.empty(n_stage, 2 * nnode, dtype=torch.float64, device=dev)
    _lib.check(L.stt_stage_rows(nelx, nely, n_stage, _lib.ptr(x), _lib.ptr(member), Emin, Emax, penal,
                                _lib.ptr(P.fixed2), _lib.ptr(rho), _lib.ptr(F), st))
    if batched:
        sl = torch_mg.build_hierarchy(rho, P.edof, P.KE, P.mask, nelx, nely,
                                      max_coarse_elements=max_coarse_elements, precision=precision)
        U = _pcg(sl, F, None, rtol, max_iter, "stage_n_iter", info)
        stage_levels = [sl]
    else:
        Us, stage_levels = [], []
        for s in range(n_stage):
            sl = torch_mg.build_hierarchy(rho[s], P.edof, P.KE, P.mask, nelx, nely,
                                          max_coarse_elements=max_coarse_elements, precision=precision)
            Us.append(_pcg(sl, F[s], None, rtol, max_iter, f"stage{s}_n_iter", info))
            stage_levels.append(sl)
        U = torch.stack(Us)
    terms = torch_fem.element_terms(U, P.edof, P.KE)
    ce = terms["ce"]
    c_s = (rho * ce).sum(-1)
    J_t = (w.reshape(-1).to(torch.float64) * tPhys).sum()
    out = dict(objective=c_s.sum() + J_t, c_s=c_s, J_t=J_t, tPhys=tPhys.reshape(nely, nelx), U=U,
               T=T, member=member)
    if not gradient:
        return out

    # 5a. stage adjoints: dL/dU = 2 K U; warm start alpha U (exact for compliance)
    g = torch.empty_like(U)
    _lib.check(L.stt_q4_apply(_lib.STT_FP64, 2, nelx, nely, n_stage, _lib.ptr(U), 2 * nnode, _lib.ptr(g),
                              2 * nnode, _lib.ptr(rho), nel, None, 0, _lib.ptr(P.fixed2),
                              _lib.STT_PROJECT_OUT, P.ke, st))
    g = 2 * g
    a = torch_fem.safe_div(torch_fem._dots(U, g), torch_fem._dots(U, F))
    x0 = (a[:, None] * U).contiguous()
    if batched:
        lam = _pcg(stage_levels[0], g, x0, rtol, max_iter, "adjoint_n_iter", info)
    else:
        lam = torch.stack([_pcg(stage_levels[s], g[s], x0[s], rtol, max_iter, f"adjoint{s}_n_iter", info)
                           for s in range(n_stage)])
    gd = torch_fem.element_terms(U, P.edof, P.KE, lam=lam)["gdens"]
    grad = torch.zeros(nel, dtype=torch.float64, device=dev)
    _lib.check(L.stt_stage_gradient(nelx, nely, n_stage, _lib.ptr(x), _lib.ptr(member), _lib.ptr(ce),
                                    _lib.ptr(gd), _lib.ptr(lam.contiguous()), Emin, Emax, penal,
                                    _lib.ptr(grad), st))

    # 5b. heat adjoint: d(sum w tPhys)/dT = -(w / scale) / 4 per corner
    ws = (w.reshape(-1).to(torch.float64) / scale).contiguous()
    gT = torch.empty(nnode, dtype=torch.float64, device=dev)
    _lib.check(L.stt_heat_adjoint_load(nelx, nely, _lib.ptr(ws), 1.0, _lib.ptr(gT), st))
    gT = torch_fem.project(gT, P.heat_mask).contiguous()
    ah = torch_fem.safe_div(torch_fem._dots(T_free, gT), torch_fem._dots(T_free, heat_rhs))
    lam_h = _pcg(hl, gT, (ah * T_free).contiguous(), rtol, max_iter, "heat_adjoint_n_iter", info)
    # -lam_e^T KE_h T_e covers both femsolve's density term and the lift term
    g_chi = torch_fem.element_terms(T, P.edof1, P.KEh, lam=lam_h)["gdens"]
    q = conduction_penal
    dpen = torch.where(x ** q >= 1e-6, q * x ** (q - 1), torch.zeros_like(x))
    grad = grad + g_chi * dpen
    out["gradient"] = grad.reshape(nely, nelx)
    out["lam"] = lam
    return out


class SpaceTimeObjective(torch.autograd.Function):
    """``objective(xPhys)`` as an autograd node: the forward pass runs the batched solves
    and the hand-written adjoints at once (``objective_and_gradient``); the backward
    pass scales the stored gradient, so ``torch.autograd.grad`` and
    ``sensitivity.jacobian_rows`` see the space-time objective like any torch function
    (the reference reaches it through autograd over compliance.py and
    virtual_heat.py)."""

    @staticmethod
    def forward(ctx, xPhys, w, kw):
        out = objective_and_gradient(xPhys, w, gradient=ctx.needs_input_grad[0], **kw)
        ctx.save_for_backward(out.get("gradient", torch.zeros_like(xPhys)))
        return out["objective"].clone()

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return g * grad.to(g.dtype), None, None


def objective(xPhys: Tensor, w: Tensor, **kw) -> Tensor:
    """Differentiable space-time objective ``sum_s c_s + sum(w tPhys)`` (a 0-d tensor);
    keyword arguments as ``objective_and_gradient``."""
    return SpaceTimeObjective.apply(xPhys, w, kw)

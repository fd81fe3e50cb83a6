"""Drop-in for ``sttopt.torch_fem``: the matrix-free Q4 operator and batched PCG.

Same names, signatures, broadcasting and errors as the reference module
(sttopt/torch_fem.py); the arithmetic runs in the sm_100a kernels of
``libsttb200.so``.  Tensors must be on a CUDA device (there is no CPU path).

* ``matvec`` / ``operator`` / ``matvec_diagonal`` / ``lumped_reaction`` /
  ``jacobi_preconditioner_diag``: one fused kernel each (SIMP-scaled element matrix
  gathered per node, projection and reaction folded in); ``matvec`` is differentiable
  in ``U`` and ``density`` like the reference's torch composition.
* ``pcg``: when ``apply_A`` is a level of a ``torch_mg`` hierarchy and ``apply_M`` its
  ``VCycle``, the whole solve runs on the device (``stt_pcg_mg``); any other pair of
  callables runs the reference's loop, row retirement through ``select`` included,
  with the vector updates in fused kernels.
"""

from __future__ import annotations

import torch
from torch import Tensor

from . import _geom, _lib

#: Compact the CG batch once the active rows fall to this fraction (torch_fem.py:30).
COMPACTION_RATIO = 0.75


class CGConvergenceError(RuntimeError):
    """PCG did not reach ``rtol`` within ``max_iter`` (sttopt/torch_fem.py:33-52)."""

    def __init__(self, residuals: Tensor, n_iter: int, rtol: float) -> None:
        self.residuals = residuals
        self.n_iter = n_iter
        self.rtol = rtol
        worst = residuals.max().item()
        failed = torch.nonzero(residuals > rtol).flatten().tolist()
        super().__init__(
            f"CG did not converge to rtol={rtol:g} within {n_iter} iterations "
            f"(worst relative residual {worst:g}); failed batch indices {failed}"
        )


def simp_density(xPhys: Tensor, Emin: float, Emax: float, penal: float) -> Tensor:
    """``Emin + xPhys**penal * (Emax - Emin)`` (sttopt/torch_fem.py:55-59)."""
    return Emin + xPhys**penal * (Emax - Emin)


def _dims(KE: Tensor) -> int:
    return KE.shape[-1] // 4


def _apply(U: Tensor, density: Tensor, edofMat: Tensor, KE: Tensor, ndof: int,
           mask: Tensor | None, reaction_diag: Tensor | None, flags: int) -> Tensor:
    """The fused level-0 kernel over broadcast batch rows."""
    _lib.require_cuda(U, density, mask, reaction_diag)
    d = _dims(KE)
    nelx, nely = _geom.grid_shape(edofMat, ndof, d)
    nel = nelx * nely
    prec = _lib.precision_of(U.dtype)
    if density.dtype != U.dtype:
        raise TypeError("U and density must share a dtype")
    batch = torch.broadcast_shapes(U.shape[:-1], density.shape[:-1],
                                   () if reaction_diag is None else reaction_diag.shape[:-1])
    nrows = 1
    for b in batch:
        nrows *= b
    Ub, u_rs = _geom.rows2d(U.expand(*batch, ndof), ndof)
    Db, d_rs = _geom.rows2d(density.expand(*batch, nel), nel)
    if Ub.shape[0] == 1:
        u_rs = 0
    if Db.shape[0] == 1:
        d_rs = 0
    rd, rd_rs = None, 0
    if reaction_diag is not None:
        rd, rd_rs = _geom.rows2d(reaction_diag.to(U.dtype).expand(*batch, ndof), ndof)
        if rd.shape[0] == 1:
            rd_rs = 0
    out = torch.empty(*batch, ndof, dtype=U.dtype, device=U.device)
    fixed = _geom.fixed_flags(mask, ndof // d, d)
    ke = _lib.dbl_array(_geom.host_KE(KE))
    _lib.check(_lib.lib().stt_q4_apply(
        prec, d, nelx, nely, max(nrows, 1), _lib.ptr(Ub), u_rs, _lib.ptr(out), ndof,
        _lib.ptr(Db), d_rs, _lib.ptr(rd), rd_rs, _lib.ptr(fixed), flags, ke, _lib.stream()))
    return out


class _Matvec(torch.autograd.Function):
    """``K(density) U``; backward: ``K g`` for ``U`` (K symmetric) and
    ``g_e^T KE U_e`` for ``density`` (the reference's gather/bmm/index_add chain)."""

    @staticmethod
    def forward(ctx, U, density, edofMat, KE, ndof):
        ctx.save_for_backward(U, density)
        ctx.edofMat, ctx.KE, ctx.ndof = edofMat, KE, ndof
        return _apply(U, density, edofMat, KE, ndof, None, None, 0)

    @staticmethod
    def backward(ctx, g):
        U, density = ctx.saved_tensors
        gU = gd = None
        if ctx.needs_input_grad[0]:
            gU = _apply(g, density, ctx.edofMat, ctx.KE, ctx.ndof, None, None, 0)
        if ctx.needs_input_grad[1]:
            batch = torch.broadcast_shapes(U.shape[:-1], density.shape[:-1], g.shape[:-1])
            gd = -element_terms(U.expand(*batch, ctx.ndof), ctx.edofMat, ctx.KE,
                                lam=g.expand(*batch, ctx.ndof))["gdens"]
        return gU, gd, None, None, None


def matvec(U: Tensor, density: Tensor, edofMat: Tensor, KE: Tensor, ndof: int) -> Tensor:
    """Matrix-free ``K @ U`` (sttopt/torch_fem.py:62-83); batch dims broadcast."""
    if torch.is_grad_enabled() and (U.requires_grad or density.requires_grad):
        return _Matvec.apply(U, density, edofMat, KE, ndof)
    return _apply(U, density, edofMat, KE, ndof, None, None, 0)


def matvec_diagonal(density: Tensor, edofMat: Tensor, KE: Tensor, ndof: int) -> Tensor:
    """``diag(K)`` (sttopt/torch_fem.py:86-98)."""
    return _diag(density, edofMat, KE, ndof, None, None)


def _diag(density, edofMat, KE, ndof, mask, reaction_diag):
    _lib.require_cuda(density, mask, reaction_diag)
    if density.dtype != torch.float64:
        raise TypeError("the diagonal is computed in float64")
    d = _dims(KE)
    nelx, nely = _geom.grid_shape(edofMat, ndof, d)
    batch = density.shape[:-1] if reaction_diag is None else torch.broadcast_shapes(
        density.shape[:-1], reaction_diag.shape[:-1])
    Db, d_rs = _geom.rows2d(density.detach().expand(*batch, nelx * nely), nelx * nely)
    if Db.shape[0] == 1:
        d_rs = 0
    rd, rd_rs = None, 0
    if reaction_diag is not None:
        rd, rd_rs = _geom.rows2d(reaction_diag.detach().expand(*batch, ndof), ndof)
        if rd.shape[0] == 1:
            rd_rs = 0
    nrows = max(Db.shape[0], 1 if rd is None else rd.shape[0])
    out = torch.empty(*batch, ndof, dtype=torch.float64, device=density.device)
    fixed = _geom.fixed_flags(mask, ndof // d, d)
    _lib.check(_lib.lib().stt_q4_diag(
        d, nelx, nely, nrows, _lib.ptr(Db), d_rs, _lib.ptr(rd), rd_rs, _lib.ptr(fixed),
        _lib.ptr(out), ndof, _lib.dbl_array(_geom.host_KE(KE)), _lib.stream()))
    return out


def free_mask(ndof: int, freedofs: Tensor, device=None) -> Tensor:
    """Bool mask, True at free dofs (sttopt/torch_fem.py:101-107)."""
    mask = torch.zeros(ndof, dtype=torch.bool, device=device)
    mask[freedofs] = True
    return mask


def project(v: Tensor, mask: Tensor) -> Tensor:
    """Zero the fixed dofs (sttopt/torch_fem.py:110-114)."""
    return v * mask


class _LumpedReaction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, reaction, edofMat, ndof, d, nelx, nely):
        ctx.grid = (ndof, d, nelx, nely)
        Rb, r_rs = _geom.rows2d(reaction, nelx * nely)
        out = torch.empty(*reaction.shape[:-1], ndof, dtype=torch.float64, device=reaction.device)
        _lib.check(_lib.lib().stt_lumped_reaction(d, nelx, nely, Rb.shape[0], _lib.ptr(Rb), r_rs,
                                                  _lib.ptr(out), ndof, _lib.stream()))
        return out

    @staticmethod
    def backward(ctx, g):
        # each element's value reaches its 4 * d dofs with weight 1/4: the element-centric
        # gather of stt_lumped_reaction_adjoint
        ndof, d, nelx, nely = ctx.grid
        Gb, g_rs = _geom.rows2d(g.to(torch.float64), ndof)
        out = torch.empty(*g.shape[:-1], nelx * nely, dtype=torch.float64, device=g.device)
        _lib.check(_lib.lib().stt_lumped_reaction_adjoint(d, nelx, nely, Gb.shape[0], _lib.ptr(Gb), g_rs,
                                                          _lib.ptr(out), nelx * nely, _lib.stream()))
        return out.to(g.dtype), None, None, None, None, None


def lumped_reaction(reaction: Tensor, edofMat: Tensor, ndof: int) -> Tensor:
    """Lumped reaction diagonal, a quarter per corner (sttopt/torch_fem.py:117-132)."""
    _lib.require_cuda(reaction)
    d = edofMat.shape[-1] // 4
    nelx, nely = _geom.grid_shape(edofMat, ndof, d)
    return _LumpedReaction.apply(reaction.to(torch.float64), edofMat, ndof, d, nelx, nely)


def operator(v: Tensor, density: Tensor, edofMat: Tensor, KE: Tensor, ndof: int, mask: Tensor,
             reaction_diag: Tensor | None = None) -> Tensor:
    """``P(K P v)`` (+ reaction diagonal), one fused kernel (sttopt/torch_fem.py:135-159)."""
    if torch.is_grad_enabled() and any(
            t is not None and t.requires_grad for t in (v, density, reaction_diag)):
        pv = project(v, mask)
        Kv = matvec(pv, density, edofMat, KE, ndof)
        if reaction_diag is not None:
            Kv = Kv + reaction_diag * pv
        return project(Kv, mask)
    return _apply(v, density, edofMat, KE, ndof, mask, reaction_diag,
                  _lib.STT_PROJECT_IN | _lib.STT_PROJECT_OUT)


def jacobi_preconditioner_diag(density: Tensor, edofMat: Tensor, KE: Tensor, ndof: int,
                               mask: Tensor, reaction_diag: Tensor | None = None) -> Tensor:
    """Diagonal of the projected operator, 1 at fixed dofs (sttopt/torch_fem.py:162-181)."""
    return _diag(density, edofMat, KE, ndof, mask, reaction_diag)


def safe_div(num: Tensor, den: Tensor) -> Tensor:
    """``num / den``, 0 where ``den == 0`` (sttopt/torch_fem.py:184-192)."""
    safe_den = torch.where(den != 0, den, torch.ones_like(den))
    return torch.where(den != 0, num / safe_den, torch.zeros_like(den))


def element_terms(U: Tensor, edofMat: Tensor, KE: Tensor, lam: Tensor | None = None) -> dict:
    """Per element and row: ``ce = U_e^T KE U_e``; with ``lam``, ``gdens = -lam_e^T KE U_e``
    and ``greac = -lam_e . U_e / 4`` (torch_solve.py:146-152, compliance.py:49-59)."""
    _lib.require_cuda(U, lam)
    d = _dims(KE)
    ndof = U.shape[-1]
    nelx, nely = _geom.grid_shape(edofMat, ndof, d)
    nel = nelx * nely
    Ub, u_rs = _geom.rows2d(U.detach().to(torch.float64), ndof)
    lb, l_rs = (None, 0) if lam is None else _geom.rows2d(
        lam.detach().to(torch.float64).expand_as(U), ndof)
    rows = Ub.shape[0]
    ce = torch.empty(*U.shape[:-1], nel, dtype=torch.float64, device=U.device)
    gd = torch.empty_like(ce) if lam is not None else None
    gr = torch.empty_like(ce) if lam is not None else None
    _lib.check(_lib.lib().stt_element_sens(
        d, nelx, nely, rows, _lib.ptr(Ub), u_rs, _lib.ptr(lb), l_rs,
        _lib.dbl_array(_geom.host_KE(KE)), _lib.ptr(ce), _lib.ptr(gd), _lib.ptr(gr), nel,
        _lib.stream()))
    return {"ce": ce, "gdens": gd, "greac": gr}


def _report(info: dict | None, row_iters: int) -> None:
    if info is not None:
        info["row_iters"] = row_iters


def row_iters_from_schedule(conv_iter: list[int], n_rows: int, max_iter: int) -> int:
    """``info['row_iters']`` of the reference's compaction schedule (torch_fem.py:270-331)
    from each row's convergence iteration (0 = converged before the first iteration,
    negative = never converged)."""
    never = max_iter + 1
    c = [never if v < 0 else v for v in conv_iter]

    def remaining(n):
        return sum(1 for v in c if v > n)

    if remaining(0) == 0:
        return 0
    last = rows = n_rows
    if n_rows > 1 and remaining(0) <= COMPACTION_RATIO * last:
        rows = last = remaining(0)
    total = 0
    for n in range(1, max_iter + 1):
        total += rows
        rem = remaining(n)
        if rem == 0:
            break
        if n_rows > 1 and rem <= COMPACTION_RATIO * last:
            rows = last = rem
    return total


def pcg(apply_A, b: Tensor, apply_M, *, rtol: float = 1e-8, max_iter: int = 10000,
        x0: Tensor | None = None, info: dict | None = None) -> tuple[Tensor, int]:
    """Preconditioned CG on ``apply_A(x) = b`` (sttopt/torch_fem.py:201-343).

    Raises ``CGConvergenceError`` rather than return an unconverged row.
    """
    native = getattr(apply_A, "_native_pcg", None)
    if native is not None and getattr(apply_M, "_is_vcycle_of", None) is not None:
        out = native(b, apply_M, rtol=rtol, max_iter=max_iter, x0=x0, info=info)
        if out is not None:
            return out
    return _pcg_generic(apply_A, b, apply_M, rtol=rtol, max_iter=max_iter, x0=x0, info=info)


def _dots(a: Tensor, b: Tensor) -> Tensor:
    n = a.shape[-1]
    A, rs = _geom.rows2d(a, n)
    B, rs2 = _geom.rows2d(b, n)
    if rs != rs2 or A.shape[0] != B.shape[0]:
        A, B = A.contiguous(), B.contiguous()
        rs = n
    out = torch.empty(A.shape[0], dtype=torch.float64, device=a.device)
    _lib.check(_lib.lib().stt_vec_dots(A.shape[0], n, _lib.ptr(A), _lib.ptr(B), None, None, None,
                                       None, rs, _lib.ptr(out), _lib.stream()))
    return out.reshape(a.shape[:-1])


def _pcg_generic(apply_A, b, apply_M, *, rtol, max_iter, x0, info):
    _lib.require_cuda(b)
    b = b.to(torch.float64)
    b_norm = _dots(b, b).sqrt()
    b_norm_safe = torch.where(b_norm > 0, b_norm, torch.ones_like(b_norm))
    x = torch.zeros_like(b) if x0 is None else x0.detach().to(torch.float64).clone()
    r = (b - apply_A(x)).contiguous()
    rel_resid = _dots(r, r).sqrt() / b_norm_safe
    converged = rel_resid <= rtol
    n_remaining = int(torch.count_nonzero(~converged))
    n_rows = b.shape[0] if b.ndim == 2 else 1
    row_iters = 0
    if n_remaining == 0:
        _report(info, row_iters)
        return x, 0
    can_retire = b.ndim == 2 and r.ndim == 2 and hasattr(apply_A, "select") and hasattr(apply_M, "select")
    st = {}
    if can_retire:
        st = dict(x_out=torch.zeros_like(b), resid_out=torch.zeros_like(rel_resid),
                  active=torch.arange(b.shape[0], device=b.device), last=b.shape[0])

    def worth():
        return can_retire and n_remaining <= COMPACTION_RATIO * st["last"]

    def retire():
        nonlocal apply_A, apply_M, b_norm_safe, rel_resid, n_rows
        done, keep = (torch.nonzero(m).flatten() for m in (converged, ~converged))
        st["x_out"][st["active"][done]] = x[done]
        st["resid_out"][st["active"][done]] = rel_resid[done]
        st["active"] = st["active"][keep]
        st["last"] = keep.numel()
        apply_A, apply_M = apply_A.select(keep), apply_M.select(keep)
        b_norm_safe, rel_resid = b_norm_safe[keep], rel_resid[keep]
        n_rows = keep.numel()
        return keep

    if worth():
        keep = retire()
        x, r = x[keep].contiguous(), r[keep].contiguous()
    z = apply_M(r).to(torch.float64)
    p = z.clone().contiguous()
    rz_old = _dots(r, z)
    for n_iter in range(1, max_iter + 1):
        row_iters += n_rows
        Ap = apply_A(p).contiguous()
        alpha = safe_div(rz_old, _dots(p, Ap)).reshape(-1).contiguous()
        n = b.shape[-1]
        R = x.numel() // n
        rr = torch.empty(R, dtype=torch.float64, device=b.device)
        _lib.check(_lib.lib().stt_vec_cg_update(R, n, _lib.ptr(alpha), _lib.ptr(x),
                                                _lib.ptr(r), _lib.ptr(p), _lib.ptr(Ap), n,
                                                _lib.ptr(rr), _lib.stream()))
        rel_resid = rr.reshape(b_norm_safe.shape).sqrt() / b_norm_safe
        converged = rel_resid <= rtol
        n_remaining = int(torch.count_nonzero(~converged))
        if n_remaining == 0:
            break
        z = apply_M(r).to(torch.float64).contiguous()
        rz_new = _dots(r, z)
        beta = safe_div(rz_new, rz_old).reshape(-1).contiguous()
        _lib.check(_lib.lib().stt_vec_xpay(R, n, _lib.ptr(z), _lib.ptr(beta),
                                           _lib.ptr(p), n, _lib.stream()))
        rz_old = rz_new
        if worth():
            keep = retire()
            x, r, p, rz_old = (x[keep].contiguous(), r[keep].contiguous(), p[keep].contiguous(),
                               rz_old[keep])
    else:
        if can_retire:
            st["resid_out"][st["active"]] = rel_resid
            rel_resid = st["resid_out"]
        _report(info, row_iters)
        raise CGConvergenceError(rel_resid, max_iter, rtol)
    _report(info, row_iters)
    if can_retire:
        st["x_out"][st["active"]] = x
        return st["x_out"], n_iter
    return x, n_iter


def solve(F: Tensor, xPhys: Tensor, edofMat: Tensor, KE: Tensor, Emin: float, Emax: float,
          penal: float, mask: Tensor, *, rtol: float = 1e-8, max_iter: int = 10000,
          x0: Tensor | None = None) -> tuple[Tensor, int]:
    """SIMP + Jacobi-preconditioned CG (sttopt/torch_fem.py:346-383)."""
    ndof = mask.shape[-1]
    density = simp_density(xPhys, Emin, Emax, penal)

    def apply_A(v):
        return operator(v, density, edofMat, KE, ndof, mask)

    diag = jacobi_preconditioner_diag(density, edofMat, KE, ndof, mask)
    b = project(F, mask)
    U, n_iter = pcg(apply_A, b, lambda r: r / diag, rtol=rtol, max_iter=max_iter, x0=x0)
    return project(U, mask), n_iter

"""Drop-in for ``sttopt.torch_mg``: the Galerkin geometric-multigrid V-cycle.

``build_hierarchy`` builds every level on the device in one call (``stt_hier_create``):
exact Galerkin element products ``sum_m S_m^T K_child S_m`` (sttopt/torch_mg.py:355-370),
stored as symmetric 9-point block stencils, coarse masks sampled at collocated nodes
(:376), and the coarsest level factorised by a block-banded FP64 Cholesky (:269-290).
The hierarchy policy is the reference's: factors 2 or 3 per dimension
(``coarsening_factors``), stop at ``max_coarse_elements``.

``precision="mixed"`` keeps FP32 copies of the level operators and runs the V-cycle's
smoothing, transfers and stencil applies in FP32 (the coarse Cholesky stays FP64);
``"fp64"`` (the default) runs everything in FP64.
"""

from __future__ import annotations

import ctypes
import functools

import numpy as np
import torch
from torch import Tensor

from . import _geom, _lib, autotune, fem, torch_fem

MAX_COARSE_ELEMENTS = 700  # sttopt/torch_mg.py:50
#: "fp64" or "mixed"; the precision ``build_hierarchy`` uses when none is given.
DEFAULT_PRECISION = "fp64"


def coarsening_factors(nelx: int, nely: int) -> tuple[int, int]:
    """Smallest of 2, 3 dividing each dimension, else 1 (sttopt/torch_mg.py:53-72)."""

    def factor(n: int) -> int:
        return next((k for k in (2, 3) if n % k == 0), 1)

    return factor(nelx), factor(nely)


@functools.lru_cache(maxsize=None)
def element_dof_map_tensor(nelx: int, nely: int, device, dofs_per_node: int = 2) -> Tensor:
    """``fem.element_dof_map`` as a device tensor, memoised (sttopt/torch_mg.py:112-127)."""
    return torch.tensor(fem.element_dof_map(nelx, nely, dofs_per_node), dtype=torch.int64,
                        device=device)


def _precision_code(precision: str | None) -> int:
    p = DEFAULT_PRECISION if precision is None else precision
    if p == "fp64":
        return _lib.STT_FP64
    if p in ("mixed", "fp32"):
        return _lib.STT_FP32
    raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")


class _Hierarchy:
    """Owner of one device hierarchy (C handle + workspace), or a row-selected view."""

    def __init__(self, handle, ws, d, hrows, batch_shape, device, KE_host, parent=None,
                 row_map: Tensor | None = None, nrows: int | None = None):
        self.handle = handle
        self.ws = ws
        self.d = d
        self.hrows = hrows
        self.batch_shape = batch_shape  # leading batch shape of the density rows
        self.device = device
        self.KE_host = KE_host
        self.parent = parent
        self.row_map = row_map
        # rows the view represents (hrows for the base, len(row_map) for views)
        self.nrows = hrows if nrows is None else nrows
        n = ctypes.c_int()
        dims = (ctypes.c_int * 96)()
        _lib.check(_lib.lib().stt_hier_info(handle, ctypes.byref(n), dims, 24))
        self.nlevels = n.value
        self.dims = [tuple(dims[4 * i: 4 * i + 4]) for i in range(self.nlevels)]
        self.precision = None

    @classmethod
    def build(cls, density: Tensor, mask: Tensor, KE: Tensor, nelx: int, nely: int,
              reaction: Tensor | None, max_coarse_elements: int, precision: str | None,
              check: bool = True):
        _lib.require_cuda(density, mask, reaction)
        d = KE.shape[-1] // 4
        nel = nelx * nely
        prec = _precision_code(precision)
        batch_shape = density.shape[:-1]
        rho = density.detach().to(torch.float64).reshape(-1, nel).contiguous()
        hrows = rho.shape[0]
        reac = None
        if reaction is not None:
            reac = reaction.detach().to(torch.float64).expand(*batch_shape, nel).reshape(-1, nel).contiguous()
        fixed = _geom.fixed_flags(mask, (nelx + 1) * (nely + 1), d)
        nbytes = _lib.lib().stt_hier_workspace_bytes(d, nelx, nely, hrows, max_coarse_elements, prec)
        if nbytes < 0:
            raise ValueError("bad hierarchy shape")
        ws = _lib.workspace(nbytes, density.device)
        ke_host = _geom.host_KE(KE)
        handle = ctypes.c_void_p()
        _lib.check(_lib.lib().stt_hier_create(
            ctypes.byref(handle), _lib.ptr(ws), ws.numel(), d, nelx, nely, hrows, _lib.ptr(rho),
            nel, _lib.ptr(reac), nel, _lib.ptr(fixed), _lib.dbl_array(ke_host),
            max_coarse_elements, prec, _lib.stream()))
        h = cls(handle, ws, d, hrows, batch_shape, density.device, ke_host)
        h.precision = "fp64" if prec == _lib.STT_FP64 else "mixed"
        if check:  # the reference raises at build time on a failed coarse factorisation
            _lib.check(_lib.lib().stt_hier_status(handle, _lib.stream()))
        return h

    def select(self, rows: Tensor) -> "_Hierarchy":
        """The same operators restricted to batch rows ``rows``."""
        if self.hrows == 1 and self.row_map is None:
            return self  # one shared density field: nothing to select
        rows = rows.to(device=self.device, dtype=torch.int64)
        base = self.row_map if self.row_map is not None else torch.arange(
            self.hrows, device=self.device, dtype=torch.int32)
        rm = base[rows].to(torch.int32).contiguous()
        handle = ctypes.c_void_p()
        _lib.check(_lib.lib().stt_hier_select(self.handle, _lib.ptr(rm), ctypes.byref(handle)))
        v = _Hierarchy(handle, None, self.d, self.hrows, self.batch_shape, self.device,
                       self.KE_host, parent=self, row_map=rm, nrows=rm.numel())
        v.precision = self.precision
        return v

    def __del__(self):
        try:
            if self.handle:
                _lib.lib().stt_hier_destroy(self.handle)
                self.handle = None
        except Exception:  # interpreter shutdown
            pass


def _rows_for(h: _Hierarchy, v: Tensor) -> tuple[Tensor, int, tuple]:
    """``v`` as ``(rows, n)``: one row per view row (broadcast against a shared field)."""
    n = v.shape[-1]
    if h.hrows == 1 and h.row_map is None:
        flat = v.reshape(-1, n)
        return flat.contiguous(), flat.shape[0], v.shape[:-1]
    batch = torch.broadcast_shapes(v.shape[:-1], (h.nrows,) if h.row_map is not None else h.batch_shape)
    flat = v.expand(*batch, n).reshape(-1, n).contiguous()
    if flat.shape[0] != h.nrows:
        raise ValueError(f"{flat.shape[0]} vector rows for a hierarchy of {h.nrows} rows")
    return flat, flat.shape[0], batch


class _Level:
    """One grid of the hierarchy; calling it applies ``P(K P v)`` at this level
    (sttopt/torch_mg.py:211-266).  ``diag`` and ``mask`` are read back from the
    device on first access."""

    def __init__(self, hier: _Hierarchy, index: int, *, edofMat=None, KE=None, density=None,
                 reaction_diag=None):
        self._hier = hier
        self._index = index
        nelx, nely, kx, ky = hier.dims[index]
        self.nelx, self.nely, self.kx, self.ky = nelx, nely, kx, ky
        self.ndof = hier.d * (nelx + 1) * (nely + 1)
        self.KE = KE
        self.density = density
        self.reaction_diag = reaction_diag
        self.keff = None  # coarse operators live on the device as stencils
        self.chol = None  # the coarse factor lives on the device in band blocks
        self._edofMat = edofMat
        self._diag = None
        self._mask = None

    @property
    def edofMat(self) -> Tensor:
        if self._edofMat is None:
            self._edofMat = element_dof_map_tensor(self.nelx, self.nely, self._hier.device, self._hier.d)
        return self._edofMat

    @property
    def mask(self) -> Tensor:
        if self._mask is None:
            h = self._hier
            nnode = (self.nelx + 1) * (self.nely + 1)
            flags = torch.empty(nnode, dtype=torch.uint8, device=h.device)
            _lib.check(_lib.lib().stt_hier_level_fixed(h.handle, self._index, _lib.ptr(flags), _lib.stream()))
            bits = torch.stack([(flags >> i) & 1 for i in range(h.d)], dim=-1).reshape(-1)
            self._mask = bits == 0
        return self._mask

    @property
    def diag(self) -> Tensor:
        if self._diag is None:
            h = self._hier
            full = torch.empty(h.hrows, self.ndof, dtype=torch.float64, device=h.device)
            _lib.check(_lib.lib().stt_hier_level_diag(h.handle, self._index, _lib.ptr(full), _lib.stream()))
            if h.row_map is not None:
                full = full[h.row_map.to(torch.int64)]
            elif h.hrows == 1 and len(h.batch_shape) == 0:
                full = full[0]
            else:
                full = full.reshape(*h.batch_shape, self.ndof)
            self._diag = full
        return self._diag

    def __call__(self, v: Tensor) -> Tensor:
        _lib.require_cuda(v)
        h = self._hier
        flat, rows, batch = _rows_for(h, v.to(torch.float64))
        out = torch.empty_like(flat)
        _lib.check(_lib.lib().stt_level_apply(h.handle, self._index, rows, _lib.ptr(flat), self.ndof,
                                              _lib.ptr(out), self.ndof, _lib.stream()))
        return out.reshape(*batch, self.ndof)

    def select(self, rows: Tensor) -> "_Level":
        lv = _Level(self._hier.select(rows), self._index, edofMat=self._edofMat, KE=self.KE,
                    density=None if self.density is None or self.density.ndim == 1 else self.density[rows],
                    reaction_diag=self.reaction_diag)
        lv._mask = self._mask
        return lv

    def _native_pcg(self, b: Tensor, M: "VCycle", *, rtol, max_iter, x0, info, x0_inplace: bool = False):
        """The whole MG-PCG solve on the device when ``M`` cycles this hierarchy.
        ``x0_inplace``: ``x0`` (contiguous FP64 rows of this solve's shape) becomes the
        solution buffer instead of being copied (for the package's own warm starts)."""
        h = self._hier
        if self._index != 0 or M._is_vcycle_of is not h or b.ndim > 2:
            return None
        _lib.require_cuda(b, x0)
        flat, rows, batch = _rows_for(h, b.detach().to(torch.float64))
        n = self.ndof
        if (x0_inplace and x0 is not None and x0.dtype == torch.float64 and x0.is_contiguous()
                and x0.numel() == flat.numel() and x0.device == flat.device):
            x = x0.detach().view(-1, n)
        else:
            x = torch.empty_like(flat)
            if x0 is not None:
                x.copy_(x0.detach().to(torch.float64).expand(*batch, n).reshape(-1, n))
        autotune.apply(h, flat, rows, n, M.gamma, M.omega, M.n_smooth)
        nbytes = _lib.lib().stt_solve_workspace_bytes(h.handle, rows, M.gamma)
        ws = _lib.workspace(nbytes, flat.device)
        rel = (ctypes.c_double * rows)()
        conv = (ctypes.c_int * rows)()
        n_iter = ctypes.c_int()
        mixed = h.precision == "mixed"
        # FP64 follows the reference's row retirement (a converged row iterates on until the
        # compaction), so every row's x is the reference's; the mixed form stops a row when
        # it converges (less work; its FP32 cycle makes the iterates differ anyway)
        retire = 0 if mixed else 1
        rc = _lib.lib().stt_pcg_mg(
            h.handle, rows, _lib.ptr(flat), n, _lib.ptr(x), n, 1 if x0 is not None else 0, rtol, max_iter,
            M.omega, M.n_smooth, M.gamma, 1 if M.flexible else 0, M.replace_every, retire, rel, conv,
            ctypes.byref(n_iter),
            _lib.ptr(ws), ws.numel(), _lib.stream())
        conv_list = list(conv)
        n_rows_ref = b.shape[0] if b.ndim == 2 else 1
        if info is not None:
            if b.ndim != 2:
                info["row_iters"] = max(conv_list) if min(conv_list) >= 0 else max_iter
            elif retire:  # each row iterated until the iteration it stopped at
                info["row_iters"] = sum(v if v >= 0 else max_iter for v in conv_list)
            else:
                info["row_iters"] = torch_fem.row_iters_from_schedule(conv_list, n_rows_ref, max_iter)
        if rc == _lib.STT_ERR_NOT_CONVERGED:
            resid = torch.tensor(list(rel), dtype=torch.float64, device=b.device)
            raise torch_fem.CGConvergenceError(resid.reshape(batch) if b.ndim == 2 else resid[0], max_iter, rtol)
        _lib.check(rc)
        return x.reshape(*batch, n), n_iter.value


def build_hierarchy(density: Tensor, edofMat: Tensor, KE: Tensor, mask: Tensor, nelx: int,
                    nely: int, *, reaction: Tensor | None = None,
                    max_coarse_elements: int = MAX_COARSE_ELEMENTS,
                    precision: str | None = None, check: bool = True) -> list[_Level]:
    """Levels from finest to coarsest (sttopt/torch_mg.py:293-400), built on the device.
    ``check=False`` skips the build-time synchronisation of the coarse factorisation's
    checks; a failure then surfaces at the first solve on the hierarchy."""
    ndof = mask.shape[-1]
    d = KE.shape[-1] // 4
    if d * (nelx + 1) * (nely + 1) != ndof:
        raise ValueError("mask does not match the grid")
    h = _Hierarchy.build(density, mask, KE, nelx, nely, reaction, max_coarse_elements, precision, check)
    reaction_diag = None
    if reaction is not None:
        reaction_diag = torch_fem.lumped_reaction(reaction.detach(), edofMat, ndof)
    levels = [_Level(h, 0, edofMat=edofMat, KE=KE, density=density, reaction_diag=reaction_diag)]
    for i in range(1, h.nlevels):
        levels.append(_Level(h, i))
    levels[0]._mask = mask.to(torch.bool)
    return levels


class VCycle:
    """Damped-Jacobi V-cycle with an exact coarse solve, as an SPD preconditioner
    (sttopt/torch_mg.py:403-476); one ``stt_vcycle`` call per application.

    ``flexible``: a PCG preconditioned by this cycle on the device takes the flexible
    (Polak-Ribiere) beta, r_new . (z_new - z_old) / (r . z), instead of the reference's
    r_new . z_new / (r . z).  The cycle is symmetric, in FP32 up to its rounding, so the
    two agree to that rounding (~1e-7 relative in the mixed form); the flexible form costs
    the extra dot r_new . z_old an iteration.

    ``replace_every``: that PCG recomputes the true residual b - A x in FP64 every k
    iterations (0: never; each costs an operator apply and an x flush)."""

    def __init__(self, levels: list[_Level], *, omega: float = 0.6, n_smooth: int = 2,
                 gamma: int = 1, flexible: bool = False, replace_every: int = 0) -> None:
        if not levels or not isinstance(levels[0], _Level):
            raise TypeError("VCycle needs levels from sttopt_b200.torch_mg.build_hierarchy")
        self.levels = levels
        self.omega = omega
        self.n_smooth = n_smooth
        self.gamma = gamma
        self.flexible = flexible
        self.replace_every = int(replace_every)
        self._is_vcycle_of = levels[0]._hier

    def select(self, rows: Tensor) -> "VCycle":
        return VCycle([lv.select(rows) for lv in self.levels], omega=self.omega,
                      n_smooth=self.n_smooth, gamma=self.gamma, flexible=self.flexible,
                      replace_every=self.replace_every)

    def __call__(self, r: Tensor) -> Tensor:
        _lib.require_cuda(r)
        h = self._is_vcycle_of
        n = self.levels[0].ndof
        flat, rows, batch = _rows_for(h, r.to(torch.float64))
        z = torch.empty_like(flat)
        nbytes = _lib.lib().stt_vcycle_workspace_bytes(h.handle, rows, self.gamma)
        ws = _lib.workspace(nbytes, flat.device)
        _lib.check(_lib.lib().stt_vcycle(h.handle, rows, _lib.ptr(flat), n, _lib.ptr(z), n, self.omega,
                                         self.n_smooth, self.gamma, _lib.ptr(ws), ws.numel(), _lib.stream()))
        return z.reshape(*batch, n)


def solve(F: Tensor, xPhys: Tensor, edofMat: Tensor, KE: Tensor, Emin: float, Emax: float,
          penal: float, mask: Tensor, nelx: int, nely: int, *, rtol: float = 1e-8,
          max_iter: int = 500, x0: Tensor | None = None, omega: float = 0.6, n_smooth: int = 2,
          gamma: int = 1, max_coarse_elements: int = MAX_COARSE_ELEMENTS,
          info: dict | None = None, precision: str | None = None) -> tuple[Tensor, int]:
    """MG-preconditioned CG for ``K U = F`` (sttopt/torch_mg.py:479-535)."""
    density = torch_fem.simp_density(xPhys, Emin, Emax, penal)
    levels = build_hierarchy(density, edofMat, KE, mask, nelx, nely,
                             max_coarse_elements=max_coarse_elements, precision=precision)
    precond = VCycle(levels, omega=omega, n_smooth=n_smooth, gamma=gamma)
    U, n_iter = torch_fem.pcg(levels[0], torch_fem.project(F, mask), precond, rtol=rtol,
                              max_iter=max_iter, x0=x0, info=info)
    return torch_fem.project(U, mask), n_iter


# ---- host-side transfer utilities (API parity; the cycle uses device kernels) ------


def child_interpolation_matrices(kx: int, ky: int, device=None, dtype=torch.float64,
                                 dofs_per_node: int = 2) -> Tensor:
    """``S[m]``: coarse element dofs -> child ``m``'s dofs (sttopt/torch_mg.py:140-165)."""
    d = dofs_per_node
    nk = 4 * d
    S = np.zeros((kx * ky, nk, nk))
    corner = [(1, 0), (1, 1), (0, 1), (0, 0)]  # BL, BR, TR, TL (row, col)

    def interp1(a, b, j, k):
        if j == k:
            return b
        w = j / k
        return a * (1 - w) + b * w

    for qc, (cr, cc) in enumerate(corner):
        for my in range(ky):
            for mx in range(kx):
                for qf, (fr0, fc0) in enumerate(corner):
                    fr, fc = my + fr0, mx + fc0
                    g = [interp1(1.0 if (R == cr and cc == 0) else 0.0,
                                 1.0 if (R == cr and cc == 1) else 0.0, fc, kx) for R in (0, 1)]
                    v = interp1(g[0], g[1], fr, ky)
                    for i in range(d):
                        S[my * kx + mx, qf * d + i, qc * d + i] = v
    return torch.tensor(S, dtype=dtype, device=device)


# ---- grid transfers and explicit element matrices (the reference's helpers) ---------


def _transfer(v: Tensor, cnnx: int, cnny: int, kx: int, ky: int, d: int, restrict: bool) -> Tensor:
    _lib.require_cuda(v)
    fnnx, fnny = kx * (cnnx - 1) + 1, ky * (cnny - 1) + 1
    n_in, n_out = (d * fnnx * fnny, d * cnnx * cnny) if restrict else (d * cnnx * cnny, d * fnnx * fnny)
    if v.shape[-1] != n_in:
        raise ValueError(f"expected a trailing dimension of {n_in}, got {tuple(v.shape)}")
    V = v.detach().to(torch.float64).reshape(-1, n_in).contiguous()
    out = torch.empty(V.shape[0], n_out, dtype=torch.float64, device=V.device)
    _lib.check(_lib.lib().stt_grid_transfer(d, kx, ky, cnnx, cnny, V.shape[0], int(restrict), _lib.ptr(V), n_in,
                                            _lib.ptr(out), n_out, _lib.stream()))
    return out.reshape(*v.shape[:-1], n_out).to(v.dtype)


class _Transfer(torch.autograd.Function):
    """P (restrict = False) or R = P^T (True); the backward pass is the other one."""

    @staticmethod
    def forward(ctx, v, cnnx, cnny, kx, ky, d, restrict):
        ctx.args = (cnnx, cnny, kx, ky, d, restrict)
        return _transfer(v, cnnx, cnny, kx, ky, d, restrict)

    @staticmethod
    def backward(ctx, g):
        cnnx, cnny, kx, ky, d, restrict = ctx.args
        return _transfer(g, cnnx, cnny, kx, ky, d, not restrict), None, None, None, None, None, None


def _interp_axis(c: Tensor, k: int) -> Tensor:
    """Piecewise-linear interpolation by ``k`` along the last axis, ``nc + 1 -> k nc + 1``
    (sttopt/torch_mg.py:75-81), on the device (``stt_grid_transfer``, x pass only)."""
    if k == 1:
        return c
    lead = c.shape[:-1]
    rows = int(np.prod(lead)) if lead else 1
    out = _Transfer.apply(c.reshape(1, rows * c.shape[-1]), c.shape[-1], rows, k, 1, 1, False)
    return out.reshape(*lead, k * (c.shape[-1] - 1) + 1)


def _restrict_axis(f: Tensor, k: int) -> Tensor:
    """The exact transpose of ``_interp_axis`` along the last axis (sttopt/torch_mg.py:84-93)."""
    if k == 1:
        return f
    if (f.shape[-1] - 1) % k:
        raise ValueError(f"{f.shape[-1]} nodes do not coarsen by {k}")
    lead = f.shape[:-1]
    rows = int(np.prod(lead)) if lead else 1
    nc = (f.shape[-1] - 1) // k + 1
    out = _Transfer.apply(f.reshape(1, rows * f.shape[-1]), nc, rows, k, 1, 1, True)
    return out.reshape(*lead, nc)


def _on_node_grid(v: Tensor, nnx: int, nny: int, kx: int, ky: int, axis_op) -> Tensor:
    """``axis_op`` along the node grid's x then y axes of a dof vector (sttopt/torch_mg.py:96-109).
    ``_interp_axis`` / ``_restrict_axis`` with 1 or 2 dofs per node run as one device pass
    (``stt_grid_transfer``); any other operator runs through its own calls."""
    d = v.shape[-1] // (nny * nnx)
    if d in (1, 2) and axis_op in (_interp_axis, _restrict_axis):
        if axis_op is _interp_axis:
            return _Transfer.apply(v, nnx, nny, kx, ky, d, False)
        if (nnx - 1) % kx or (nny - 1) % ky:
            raise ValueError("the node grid does not coarsen by these factors")
        return _Transfer.apply(v, (nnx - 1) // kx + 1, (nny - 1) // ky + 1, kx, ky, d, True)
    g = v.reshape(*v.shape[:-1], nny, nnx, d)
    g = axis_op(g.movedim(-2, -1), kx).movedim(-1, -2)
    g = axis_op(g.movedim(-3, -1), ky).movedim(-1, -3)
    return g.reshape(*v.shape[:-1], -1)


@functools.lru_cache(maxsize=None)
def _child_elements(nelx: int, nely: int, kx: int, ky: int, device) -> Tensor:
    """Fine element indices under each coarse element, in the child order of
    ``fem.element_dof_map(kx, ky)`` (sttopt/torch_mg.py:130-137)."""
    e = torch.arange(nelx * nely, device=device).reshape(nely, nelx)
    return e.reshape(nely // ky, ky, nelx // kx, kx).permute(0, 2, 1, 3).reshape(-1, ky * kx)


def _scatter(per_element: Tensor, edofMat: Tensor, ndof: int) -> Tensor:
    """Scatter-add of per-element dof values into a dof vector (sttopt/torch_mg.py:168-176)."""
    batch = per_element.shape[:-2]
    flat = per_element.reshape(*batch, -1)
    return flat.new_zeros(*batch, ndof).index_add_(-1, edofMat.reshape(-1), flat)


def keff_matvec(U: Tensor, keff: Tensor, edofMat: Tensor, ndof: int) -> Tensor:
    """``sum_e scatter(keff_e U_e)`` for explicit per-element matrices (sttopt/torch_mg.py:179-193),
    batch dims broadcasting as in the reference, by ``stt_keff_apply`` (FP64)."""
    _lib.require_cuda(U, keff)
    k = keff.shape[-1]
    d = k // 4
    nelx, nely = _geom.grid_shape(edofMat, ndof, d)
    nel = nelx * nely
    if keff.shape[-3:] != (nel, k, k):
        raise ValueError(f"keff of shape {tuple(keff.shape)} does not match {nel} elements of {k} dofs")
    batch = torch.broadcast_shapes(U.shape[:-1], keff.shape[:-3])
    Ub = U.detach().to(torch.float64).expand(*batch, ndof).reshape(-1, ndof).contiguous()
    if keff.dim() == 3:
        Kb, k_rs = keff.detach().to(torch.float64).contiguous(), 0
    else:
        Kb, k_rs = keff.detach().to(torch.float64).expand(*batch, nel, k, k).reshape(-1, nel, k, k).contiguous(), nel * k * k
    out = torch.empty_like(Ub)
    _lib.check(_lib.lib().stt_keff_apply(d, nelx, nely, Ub.shape[0], _lib.ptr(Ub), ndof, _lib.ptr(Kb), k_rs,
                                         _lib.ptr(out), ndof, _lib.stream()))
    return out.reshape(*batch, ndof).to(U.dtype)


def _select_rows(t: Tensor | None, rows: Tensor, core_ndim: int):
    """``t[rows]`` along its batch dim; an unbatched tensor passes through (sttopt/torch_mg.py:196-209)."""
    if t is None or t.ndim == core_ndim:
        return t
    if t.ndim != core_ndim + 1:
        raise ValueError(f"row selection needs a single batch dim, got shape {tuple(t.shape)}")
    return t[rows]


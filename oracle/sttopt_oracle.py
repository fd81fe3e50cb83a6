"""CPU oracle for the matrix-free FEM solve path of ``sttopt`` -- TEST INFRASTRUCTURE ONLY.

A NumPy/SciPy restatement, in FP64, of the reference algorithms this repository
accelerates.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline legs may import it, and only as the checker or as the timed CPU baseline:
the product path (the CUDA extension behind ``include/sttb200.h``) never calls into it.

Parity pin: every function below is checked against golden vectors produced by running
the reference's own torch implementation in FP64 (``tests/golden/make_golden.py``,
committed fixtures ``tests/golden/*.npz``), by ``tests/test_oracle_golden.py``.

Each function cites the reference file:line it restates (paths inside the ``sttopt``
project).  Array conventions follow the reference: nodes in C order
``row * (nelx + 1) + col`` with row 0 at the top, dofs interleaved ``d * node + i``,
elements ``row * nelx + col``, local element node order bottom-left, bottom-right,
top-right, top-left.
"""

from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np
import scipy.linalg

# ---------------------------------------------------------------------------------
# Optional C/OpenMP loops (oracle_kernels.c, built by oracle/build_oracle.py into
# oracle/_build/): the element products, the Jacobi update and the PCG's row operations,
# with the arithmetic of the NumPy forms below (only the summation order differs).
# Without the library the NumPy forms run.
# ---------------------------------------------------------------------------------

_C_PATH = Path(__file__).resolve().parent / "_build" / "liboracle_kernels.so"
_C_LIB = None


def c_kernels():
    """The C loops, or None when ``liboracle_kernels.so`` was not built."""
    global _C_LIB
    if _C_LIB is None:
        if not _C_PATH.exists():
            _C_LIB = False
        else:
            lib = ctypes.CDLL(str(_C_PATH))
            P, I, LL, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double
            lib.orc_element_apply.argtypes = [I, I, I, I, P, LL, P, LL, LL, P, LL, P, LL]
            lib.orc_jacobi_update.argtypes = [I, LL, P, LL, P, LL, P, LL, P, LL, D]
            lib.orc_row_dots.argtypes = [I, LL, P, LL, P, LL, P]
            lib.orc_row_axpy.argtypes = [I, LL, P, P, LL, P, LL]
            lib.orc_row_xpay.argtypes = [I, LL, P, LL, P, P, LL]
            for f in (lib.orc_element_apply, lib.orc_jacobi_update, lib.orc_row_dots, lib.orc_row_axpy,
                      lib.orc_row_xpay):
                f.restype = None
            _C_LIB = lib
    return _C_LIB or None


def _rows(a, n):
    """``(array, row stride, rows)`` of a 1-D (one broadcast row, stride 0) or C-ordered
    2-D float64 array."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim == 1:
        return a, 0, 1
    return a, n, a.shape[0]


def _ptr(a):
    return None if a is None else a.ctypes.data


def _grid_of(edof, d):
    """``(nelx, nely)`` of the reference's structured element dof map."""
    nelx = int(edof[0, 0]) // d - 1
    nely = edof.shape[0] // nelx
    return nelx, nely


def _row_axpy(alpha, x, y):
    """``y += alpha * x`` per row, in place (``alpha`` one value per row)."""
    lib = c_kernels()
    if lib is None or x.ndim > 2 or not y.flags.c_contiguous:
        y += np.reshape(alpha, (-1, 1) if y.ndim == 2 else ()) * x
        return y
    n = y.shape[-1]
    X, x_rs, _ = _rows(x, n)
    a = np.ascontiguousarray(np.reshape(alpha, -1), dtype=np.float64)
    lib.orc_row_axpy(a.size, n, _ptr(a), _ptr(X), x_rs, _ptr(y), n if y.ndim == 2 else 0)
    return y


def _row_xpay(z, beta, p):
    """``p = p * beta + z`` per row, in place."""
    lib = c_kernels()
    if lib is None or z.ndim > 2 or not p.flags.c_contiguous:
        p *= np.reshape(beta, (-1, 1) if p.ndim == 2 else ())
        p += z
        return p
    n = p.shape[-1]
    Z, z_rs, _ = _rows(z, n)
    bt = np.ascontiguousarray(np.reshape(beta, -1), dtype=np.float64)
    lib.orc_row_xpay(bt.size, n, _ptr(Z), z_rs, _ptr(bt), _ptr(p), n if p.ndim == 2 else 0)
    return p


def _row_dots(a, b):
    lib = c_kernels()
    if lib is None or a.ndim > 2 or b.ndim > 2:
        return (a * b).sum(axis=-1)
    n = a.shape[-1]
    A, a_rs, ra = _rows(a, n)
    B, b_rs, rb = _rows(b, n)
    rows = max(ra, rb)
    out = np.empty(rows)
    lib.orc_row_dots(rows, n, _ptr(A), a_rs, _ptr(B), b_rs, _ptr(out))
    return out if (a.ndim == 2 or b.ndim == 2) else out[0]

# ---------------------------------------------------------------------------------
# Mesh set-up (sttopt/fem.py)
# ---------------------------------------------------------------------------------


def plane_stress_KE(nu: float) -> np.ndarray:
    """Q4 plane-stress element matrix ``(A + nu B) / (1 - nu^2) / 24`` (fem.py:17-30)."""
    A11 = np.array([[12, 3, -6, -3], [3, 12, 3, 0], [-6, 3, 12, -3], [-3, 0, -3, 12]])
    A12 = np.array([[-6, -3, 0, 3], [-3, -6, -3, -6], [0, -3, -6, 3], [3, -6, 3, -6]])
    B11 = np.array([[-4, 3, -2, 9], [3, -4, -9, 4], [-2, -9, -4, -3], [9, 4, -3, -4]])
    B12 = np.array([[2, -3, 4, -9], [-3, 2, 9, -2], [4, 9, 2, 3], [-9, -2, 3, 2]])
    A = np.block([[A11, A12], [A12.T, A11]])
    B = np.block([[B11, B12], [B12.T, B11]])
    return (A + nu * B) / (1 - nu**2) / 24


def diffusion_KE() -> np.ndarray:
    """Scalar Q4 element matrix of ``-div grad`` (fem.py:98-111)."""
    return np.array(
        [[4, -1, -2, -1], [-1, 4, -1, -2], [-2, -1, 4, -1], [-1, -2, -1, 4]], dtype=np.float64
    ) / 6


def node_grid(nelx: int, nely: int) -> np.ndarray:
    """C-order node numbers on the ``(nely+1, nelx+1)`` grid (fem.py:60-69)."""
    return np.arange((nely + 1) * (nelx + 1)).reshape(nely + 1, nelx + 1)


def element_dof_map(nelx: int, nely: int, dofs_per_node: int = 2) -> np.ndarray:
    """Element dof map, corners BL, BR, TR, TL, dofs interleaved (fem.py:72-95)."""
    nodes = node_grid(nelx, nely)
    corners = np.stack(
        [nodes[1:, :-1], nodes[1:, 1:], nodes[:-1, 1:], nodes[:-1, :-1]], axis=-1
    ).reshape(-1, 4)
    d = dofs_per_node
    return np.stack([d * corners + i for i in range(d)], axis=-1).reshape(-1, 4 * d)


def cantilever_point_load(nelx: int, nely: int):
    """Bottom-right unit downward point load, left edge clamped.

    ``load_cases.load_case(CANTILEVER, nelx, nely, 0, 0, 1)`` (load_cases.py:96-98):
    ``edge_load_shares(n, 0)`` is a point load on the first node of ``right_up``, i.e.
    the bottom-right node.  Returns ``(F, mask)`` with ``mask`` True at free dofs.
    """
    nodes = node_grid(nelx, nely)
    ndof = 2 * nodes.size
    F = np.zeros(ndof)
    F[2 * nodes[-1, -1] + 1] = -1.0
    mask = np.ones(ndof, bool)
    left = nodes[:, 0]
    mask[2 * left] = False
    mask[2 * left + 1] = False
    return F, mask


def mbb_point_load(nelx: int, nely: int):
    """MBB half-beam: x-roller on the left edge, y-fixed bottom-right corner, unit
    downward load at the top-left node.

    ``load_case(MBB, nelx, nely, 0, 0, 1)`` (load_cases.py:116-120): the support patch
    of length 0 centred at distance 0 along the reversed bottom row holds exactly the
    bottom-right node; a load span of 0 is a point load on the top-left node.
    """
    nodes = node_grid(nelx, nely)
    ndof = 2 * nodes.size
    F = np.zeros(ndof)
    F[2 * nodes[0, 0] + 1] = -1.0
    mask = np.ones(ndof, bool)
    mask[2 * nodes[:, 0]] = False
    mask[2 * nodes[-1, -1] + 1] = False
    return F, mask


def mid_right_cantilever(nelx: int, nely: int):
    """Left edge clamped, unit ``-y`` load at ``nodes[nely // 2, -1]`` (a 1024x512-style
    cantilever built directly as ``F``/``mask``; no reference load case has it)."""
    nodes = node_grid(nelx, nely)
    ndof = 2 * nodes.size
    F = np.zeros(ndof)
    F[2 * nodes[nely // 2, -1] + 1] = -1.0
    mask = np.ones(ndof, bool)
    mask[2 * nodes[:, 0]] = False
    mask[2 * nodes[:, 0] + 1] = False
    return F, mask


def bottom_clamped_mask(nelx: int, nely: int) -> np.ndarray:
    """Free-dof mask with both dofs of the bottom node row fixed (the build plate)."""
    nodes = node_grid(nelx, nely)
    mask = np.ones(2 * nodes.size, bool)
    mask[2 * nodes[-1, :]] = False
    mask[2 * nodes[-1, :] + 1] = False
    return mask


# ---------------------------------------------------------------------------------
# Operator (sttopt/torch_fem.py)
# ---------------------------------------------------------------------------------


def simp_density(x, Emin: float, Emax: float, penal: float):
    """``Emin + x**penal * (Emax - Emin)`` (torch_fem.py:55-59)."""
    return Emin + x**penal * (Emax - Emin)


def _scatter(per_element: np.ndarray, edof: np.ndarray, ndof: int) -> np.ndarray:
    """Scatter-add ``(*batch, nel, k)`` element contributions to ``(*batch, ndof)``.

    The ``index_add_`` of torch_fem.py:80-82, as one ``bincount`` per batch row.
    """
    batch = per_element.shape[:-2]
    flat = per_element.reshape(-1, per_element.shape[-2] * per_element.shape[-1])
    idx = edof.reshape(-1)
    out = np.stack([np.bincount(idx, weights=row, minlength=ndof) for row in flat])
    return out.reshape(*batch, ndof)


def matvec(U, density, edof, KE, ndof):
    """``K(density) U`` element by element: gather, ``@ KE``, scale, scatter
    (torch_fem.py:62-83).  Leading batch dims of ``U`` and ``density`` broadcast."""
    lib = c_kernels()
    if lib is not None and U.ndim <= 2 and np.ndim(density) <= 2:
        d = KE.shape[-1] // 4
        nelx, nely = _grid_of(edof, d)
        Ub, u_rs, ru = _rows(U, ndof)
        Db, d_rs, rd = _rows(density, edof.shape[0])
        rows = max(ru, rd)
        out = np.empty((rows, ndof))
        K = np.ascontiguousarray(KE, dtype=np.float64)
        lib.orc_element_apply(rows, nelx, nely, d, _ptr(Ub), u_rs, _ptr(K), 0, 0, _ptr(Db), d_rs, _ptr(out), ndof)
        return out if (U.ndim == 2 or np.ndim(density) == 2) else out[0]
    Ue = U[..., edof]
    scaled = (Ue @ KE) * density[..., :, None]
    return _scatter(scaled, edof, ndof)


def matvec_diagonal(density, edof, KE, ndof):
    """``diag(K)`` (torch_fem.py:86-98)."""
    contrib = density[..., :, None] * np.diagonal(KE)
    return _scatter(contrib, edof, ndof)


def project(v, mask):
    """Zero the fixed dofs (torch_fem.py:110-114)."""
    return v * mask


def lumped_reaction(reaction, edof, ndof):
    """Lumped reaction diagonal, a quarter of each element's value per corner dof
    (torch_fem.py:117-132)."""
    contrib = np.broadcast_to(reaction[..., :, None], (*reaction.shape, edof.shape[-1])) / 4
    return _scatter(np.ascontiguousarray(contrib), edof, ndof)


def operator(v, density, edof, KE, ndof, mask, reaction_diag=None):
    """``P(K P v)`` (+ the reaction diagonal) (torch_fem.py:135-159)."""
    v = project(v, mask)
    Kv = matvec(v, density, edof, KE, ndof)
    if reaction_diag is not None:
        Kv = Kv + reaction_diag * v
    return project(Kv, mask)


def jacobi_preconditioner_diag(density, edof, KE, ndof, mask, reaction_diag=None):
    """Diagonal of the projected operator with fixed dofs set to 1 (torch_fem.py:162-181)."""
    diag = matvec_diagonal(density, edof, KE, ndof)
    if reaction_diag is not None:
        diag = diag + reaction_diag
    return np.where(mask, diag, 1.0)


def safe_div(num, den):
    """``num / den``, 0 where ``den == 0`` (torch_fem.py:184-192)."""
    num = np.asarray(num, dtype=np.float64)
    den = np.asarray(den, dtype=np.float64)
    safe = np.where(den != 0, den, 1.0)
    return np.where(den != 0, num / safe, 0.0)


class CGConvergenceError(RuntimeError):
    """Non-convergence with the per-row residuals (torch_fem.py:33-52)."""

    def __init__(self, residuals, n_iter, rtol):
        self.residuals = np.asarray(residuals)
        self.n_iter = n_iter
        self.rtol = rtol
        failed = np.flatnonzero(self.residuals > rtol).tolist()
        super().__init__(
            f"CG did not converge to rtol={rtol:g} within {n_iter} iterations "
            f"(worst relative residual {float(self.residuals.max()):g}); "
            f"failed batch indices {failed}"
        )


COMPACTION_RATIO = 0.75  # torch_fem.py:30


def pcg(apply_A, b, apply_M, *, rtol=1e-8, max_iter=10000, x0=None, info=None):
    """Batched PCG with per-row convergence and row retirement (torch_fem.py:201-343).

    Rows are independent, so retirement changes no row's arithmetic; it is restated
    here (compaction at ``COMPACTION_RATIO``) so ``info['row_iters']`` matches.
    """
    b = np.asarray(b, dtype=np.float64)
    b_norm = np.linalg.norm(b, axis=-1)
    b_norm_safe = np.where(b_norm > 0, b_norm, 1.0)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    r = b - apply_A(x)
    rel = np.linalg.norm(r, axis=-1) / b_norm_safe
    converged = rel <= rtol
    n_remaining = int(np.count_nonzero(~converged))
    n_rows = b.shape[0] if b.ndim == 2 else 1
    row_iters = 0
    if n_remaining == 0:
        if info is not None:
            info["row_iters"] = 0
        return x, 0
    can_retire = b.ndim == 2 and hasattr(apply_A, "select") and hasattr(apply_M, "select")
    state = {}
    if can_retire:
        state.update(
            x_out=np.zeros_like(b),
            resid_out=np.zeros_like(rel),
            active=np.arange(b.shape[0]),
            last=b.shape[0],
        )

    def worth():
        return can_retire and n_remaining <= COMPACTION_RATIO * state["last"]

    def retire():
        nonlocal apply_A, apply_M, b_norm_safe, rel, n_rows
        done = np.flatnonzero(converged)
        keep = np.flatnonzero(~converged)
        state["x_out"][state["active"][done]] = x[done]
        state["resid_out"][state["active"][done]] = rel[done]
        state["active"] = state["active"][keep]
        state["last"] = keep.size
        apply_A, apply_M = apply_A.select(keep), apply_M.select(keep)
        b_norm_safe, rel = b_norm_safe[keep], rel[keep]
        n_rows = keep.size
        return keep

    if worth():
        keep = retire()
        x, r = x[keep], r[keep]
    z = apply_M(r)
    p = np.array(z, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    rz_old = _row_dots(r, z)
    n_iter = 0
    for n_iter in range(1, max_iter + 1):
        row_iters += n_rows
        Ap = apply_A(p)
        alpha = safe_div(rz_old, _row_dots(p, Ap))
        _row_axpy(alpha, p, x)
        _row_axpy(-alpha, Ap, r)
        rel = np.sqrt(_row_dots(r, r)) / b_norm_safe
        converged = rel <= rtol
        n_remaining = int(np.count_nonzero(~converged))
        if n_remaining == 0:
            break
        z = apply_M(r)
        rz_new = _row_dots(r, z)
        _row_xpay(z, safe_div(rz_new, rz_old), p)
        rz_old = rz_new
        if worth():
            keep = retire()
            x, r, p, rz_old = x[keep], r[keep], p[keep], rz_old[keep]
    else:
        if can_retire:
            state["resid_out"][state["active"]] = rel
            rel = state["resid_out"]
        if info is not None:
            info["row_iters"] = row_iters
        raise CGConvergenceError(rel, max_iter, rtol)
    if info is not None:
        info["row_iters"] = row_iters
    if can_retire:
        state["x_out"][state["active"]] = x
        return state["x_out"], n_iter
    return x, n_iter


# ---------------------------------------------------------------------------------
# Geometric multigrid (sttopt/torch_mg.py)
# ---------------------------------------------------------------------------------

MAX_COARSE_ELEMENTS = 700  # torch_mg.py:50


def coarsening_factors(nelx: int, nely: int):
    """Smallest of 2, 3 dividing each dimension, else 1 (torch_mg.py:53-72)."""

    def factor(n):
        return next((k for k in (2, 3) if n % k == 0), 1)

    return factor(nelx), factor(nely)


def interp_axis(c, k):
    """Piecewise-linear interpolation by ``k`` along the last axis (torch_mg.py:75-81)."""
    if k == 1:
        return c
    w = np.arange(k) / k
    body = c[..., :-1, None] * (1 - w) + c[..., 1:, None] * w
    return np.concatenate([body.reshape(*c.shape[:-1], -1), c[..., -1:]], axis=-1)


def restrict_axis(f, k):
    """Full weighting, the exact transpose of ``interp_axis`` (torch_mg.py:84-93)."""
    if k == 1:
        return f
    w = np.arange(k) / k
    body = f[..., :-1].reshape(*f.shape[:-1], -1, k)
    lo = (body * (1 - w)).sum(-1)
    hi = (body * w).sum(-1)
    out = np.zeros((*f.shape[:-1], lo.shape[-1] + 1))
    out[..., :-1] += lo
    out[..., 1:] += hi
    out[..., -1] += f[..., -1]
    return out


def on_node_grid(v, nnx, nny, kx, ky, axis_op):
    """Apply ``axis_op`` along x then y of a dof vector (torch_mg.py:96-109)."""
    g = v.reshape(*v.shape[:-1], nny, nnx, v.shape[-1] // (nny * nnx))
    g = np.moveaxis(axis_op(np.moveaxis(g, -2, -1), kx), -1, -2)
    g = np.moveaxis(axis_op(np.moveaxis(g, -3, -1), ky), -1, -3)
    return g.reshape(*v.shape[:-1], -1)


def child_elements(nelx, nely, kx, ky):
    """Fine elements under each coarse element (torch_mg.py:130-137)."""
    e = np.arange(nelx * nely).reshape(nely, nelx)
    blocks = e.reshape(nely // ky, ky, nelx // kx, kx)
    return blocks.transpose(0, 2, 1, 3).reshape(-1, ky * kx)


def child_interpolation_matrices(kx, ky, dofs_per_node=2):
    """``S[m]``: coarse element dofs -> child ``m``'s dofs (torch_mg.py:140-165)."""
    d = dofs_per_node
    edof_c = element_dof_map(1, 1, d)[0]
    edof_f = element_dof_map(kx, ky, d)
    basis = np.zeros((4 * d, 4 * d))
    basis[np.arange(4 * d), edof_c] = 1.0
    fine = on_node_grid(basis, 2, 2, kx, ky, interp_axis)
    return np.ascontiguousarray(fine[:, edof_f].transpose(1, 2, 0))


def _select_rows(t, rows, core_ndim):
    if t is None or t.ndim == core_ndim:
        return t
    return t[rows]


class Level:
    """One multigrid level; calling it applies ``P(K P v)`` (torch_mg.py:211-266)."""

    def __init__(self, nelx, nely, ndof, mask, diag, edof, KE=None, density=None,
                 keff=None, reaction_diag=None, kx=1, ky=1, chol=None):
        self.nelx, self.nely, self.ndof = nelx, nely, ndof
        self.mask, self.diag, self.edof = mask, diag, edof
        self.KE, self.density, self.keff = KE, density, keff
        self.reaction_diag = reaction_diag
        self.kx, self.ky, self.chol = kx, ky, chol

    def __call__(self, v):
        if self.keff is None:
            return operator(v, self.density, self.edof, self.KE, self.ndof, self.mask,
                            self.reaction_diag)
        return project(keff_matvec(project(v, self.mask), self.keff, self.edof, self.ndof),
                       self.mask)

    def select(self, rows):
        out = Level(**self.__dict__)
        out.diag = _select_rows(self.diag, rows, 1)
        out.density = _select_rows(self.density, rows, 1)
        out.reaction_diag = _select_rows(self.reaction_diag, rows, 1)
        out.keff = _select_rows(self.keff, rows, 3)
        out.chol = _select_rows(self.chol, rows, 2)
        return out


def keff_matvec(U, keff, edof, ndof):
    """Coarse apply with one explicit matrix per element (torch_mg.py:179-193)."""
    lib = c_kernels()
    if lib is not None and U.ndim <= 2 and keff.ndim in (3, 4):
        k = edof.shape[1]
        d = k // 4
        nelx, nely = _grid_of(edof, d)
        nel = edof.shape[0]
        Ub, u_rs, ru = _rows(U, ndof)
        Kb = np.ascontiguousarray(keff, dtype=np.float64)
        rk = Kb.shape[0] if Kb.ndim == 4 else 1
        rows = max(ru, rk)
        out = np.empty((rows, ndof))
        lib.orc_element_apply(rows, nelx, nely, d, _ptr(Ub), u_rs, _ptr(Kb), k * k,
                              nel * k * k if Kb.ndim == 4 else 0, None, 0, _ptr(out), ndof)
        return out if (U.ndim == 2 or Kb.ndim == 4) else out[0]
    return _scatter(np.einsum("...ei,...eij->...ej", U[..., edof], keff), edof, ndof)


def dense_cholesky(keff, edof, ndof, mask):
    """Dense assembly + symmetrisation + identity on fixed dofs + Cholesky
    (torch_mg.py:269-290)."""
    idx = (edof[:, :, None] * ndof + edof[:, None, :]).reshape(-1)
    batch = keff.shape[:-3]
    flat = keff.reshape(-1, keff.shape[-3] * keff.shape[-2] * keff.shape[-1])
    dense = np.stack([np.bincount(idx, weights=row, minlength=ndof * ndof) for row in flat])
    dense = dense.reshape(*batch, ndof, ndof)
    dense = (dense + np.swapaxes(dense, -1, -2)) / 2
    free = mask[:, None] & mask[None, :]
    dense = np.where(free, dense, 0.0)
    dense = dense + np.diag((~mask).astype(np.float64))
    # one LAPACK thread per factorisation: a multi-threaded potrf of this size stalls when
    # its threads oversubscribe the cores (0.8 s against 24 ms measured on 8 cores)
    from threadpoolctl import threadpool_limits

    with threadpool_limits(limits=1, user_api="blas"):
        if dense.ndim == 2:
            return scipy.linalg.cholesky(dense, lower=True)
        return np.stack([scipy.linalg.cholesky(m, lower=True) for m in dense.reshape(-1, ndof, ndof)]).reshape(
            dense.shape)


def build_hierarchy(density, edof, KE, mask, nelx, nely, *, reaction=None,
                    max_coarse_elements=MAX_COARSE_ELEMENTS):
    """Galerkin hierarchy, finest first, coarsest factorised (torch_mg.py:293-400)."""
    ndof = mask.shape[-1]
    d = KE.shape[-1] // 4
    reaction_diag = None
    ME = None
    if reaction is not None:
        reaction_diag = lumped_reaction(reaction, edof, ndof)
        ME = np.eye(KE.shape[-1]) / 4
    diag = jacobi_preconditioner_diag(density, edof, KE, ndof, mask, reaction_diag)
    levels = [Level(nelx, nely, ndof, mask, diag, edof, KE=KE, density=density,
                    reaction_diag=reaction_diag)]
    keff = None
    while True:
        top = levels[-1]
        if top.nelx * top.nely <= max_coarse_elements:
            break
        kx, ky = coarsening_factors(top.nelx, top.nely)
        if (kx, ky) == (1, 1):
            break
        S = child_interpolation_matrices(kx, ky, d)
        children = child_elements(top.nelx, top.nely, kx, ky)
        if keff is None:
            G = np.einsum("mpi,pq,mqj->mij", S, KE, S, optimize=True)
            keff = np.einsum("...em,mij->...eij", density[..., children], G, optimize=True)
            if reaction is not None:
                GM = np.einsum("mpi,pq,mqj->mij", S, ME, S, optimize=True)
                keff = keff + np.einsum("...em,mij->...eij", reaction[..., children], GM, optimize=True)
        else:
            keff = np.einsum("mpi,...empq,mqj->...eij", S, keff[..., children, :, :], S, optimize=True)
        keff = np.ascontiguousarray(keff)
        top.kx, top.ky = kx, ky
        cnelx, cnely = top.nelx // kx, top.nely // ky
        cedof = element_dof_map(cnelx, cnely, d)
        cndof = d * (cnelx + 1) * (cnely + 1)
        cmask = top.mask.reshape(top.nely + 1, top.nelx + 1, d)[::ky, ::kx].reshape(-1)
        cdiag = _scatter(np.ascontiguousarray(np.diagonal(keff, axis1=-2, axis2=-1)), cedof, cndof)
        cdiag = np.where(cmask, cdiag, 1.0)
        levels.append(Level(cnelx, cnely, cndof, cmask, cdiag, cedof, keff=keff))
    coarsest = levels[-1]
    if keff is None:
        keff = density[..., :, None, None] * KE
        if reaction is not None:
            keff = keff + reaction[..., :, None, None] * ME
    coarsest.chol = dense_cholesky(keff, coarsest.edof, coarsest.ndof, coarsest.mask)
    return levels


class VCycle:
    """Damped-Jacobi V-cycle, exact coarse Cholesky solve (torch_mg.py:403-476)."""

    def __init__(self, levels, *, omega=0.6, n_smooth=2, gamma=1):
        self.levels, self.omega, self.n_smooth, self.gamma = levels, omega, n_smooth, gamma

    def select(self, rows):
        return VCycle([lv.select(rows) for lv in self.levels], omega=self.omega,
                      n_smooth=self.n_smooth, gamma=self.gamma)

    def _smooth(self, level, x, b):
        lib = c_kernels()
        if lib is not None and b.ndim <= 2:
            n = b.shape[-1]
            x = np.array(np.broadcast_to(x, b.shape), dtype=np.float64)
            X, x_rs, rows = _rows(x, n)
            B, b_rs, _ = _rows(b, n)
            G, g_rs, _ = _rows(level.diag, n)
            for _ in range(self.n_smooth):
                Ax, a_rs, _ = _rows(level(X), n)
                lib.orc_jacobi_update(rows, n, _ptr(X), x_rs, _ptr(B), b_rs, _ptr(Ax), a_rs, _ptr(G), g_rs,
                                      self.omega)
            return project(X, level.mask)
        for _ in range(self.n_smooth):
            x = x + self.omega * (b - level(x)) / level.diag
        return project(x, level.mask)

    def _cycle(self, i, b):
        level = self.levels[i]
        if i == len(self.levels) - 1:
            L = level.chol
            if L.ndim == 2:
                y = scipy.linalg.solve_triangular(L, b.T, lower=True)
                x = scipy.linalg.solve_triangular(L.T, y, lower=False).T
            else:
                x = np.stack([
                    scipy.linalg.solve_triangular(
                        L[s].T, scipy.linalg.solve_triangular(L[s], b[s], lower=True),
                        lower=False)
                    for s in range(L.shape[0])
                ]) if b.ndim == 2 else None
            return project(x, level.mask)
        x = self._smooth(level, np.zeros_like(b), b)
        r = b - level(x)
        coarse = self.levels[i + 1]
        rc = on_node_grid(r, level.nelx + 1, level.nely + 1, level.kx, level.ky, restrict_axis)
        rc = project(rc, coarse.mask)
        ec = self._cycle(i + 1, rc)
        for _ in range(self.gamma - 1):
            ec = ec + self._cycle(i + 1, rc - coarse(ec))
        ef = on_node_grid(project(ec, coarse.mask), coarse.nelx + 1, coarse.nely + 1,
                          level.kx, level.ky, interp_axis)
        x = x + project(ef, level.mask)
        return self._smooth(level, x, b)

    def __call__(self, r):
        return self._cycle(0, project(r, self.levels[0].mask))


def mg_solve(F, xPhys, edof, KE, Emin, Emax, penal, mask, nelx, nely, *, rtol=1e-8,
             max_iter=500, x0=None, omega=0.6, n_smooth=2, gamma=1,
             max_coarse_elements=MAX_COARSE_ELEMENTS, info=None):
    """SIMP + hierarchy + MG-PCG (torch_mg.py:479-535)."""
    density = simp_density(xPhys, Emin, Emax, penal)
    levels = build_hierarchy(density, edof, KE, mask, nelx, nely,
                             max_coarse_elements=max_coarse_elements)
    M = VCycle(levels, omega=omega, n_smooth=n_smooth, gamma=gamma)
    U, n = pcg(levels[0], project(F, mask), M, rtol=rtol, max_iter=max_iter, x0=x0, info=info)
    return project(U, mask), n


# ---------------------------------------------------------------------------------
# Differentiable solve (sttopt/torch_solve.py), written as explicit forward/adjoint
# ---------------------------------------------------------------------------------


class FemSolveOracle:
    """Forward solve and the adjoint of ``FemSolve`` (torch_solve.py:52-173)."""

    def __init__(self, density, F, edof, KE, mask, nelx, nely, *, reaction=None, rtol=1e-8,
                 max_iter=500, x0=None, omega=0.6, n_smooth=2, gamma=1,
                 max_coarse_elements=MAX_COARSE_ELEMENTS):
        self.density, self.F, self.edof, self.KE, self.mask = density, F, edof, KE, mask
        self.reaction = reaction
        self.rtol, self.max_iter = rtol, max_iter
        self.levels = build_hierarchy(density, edof, KE, mask, nelx, nely, reaction=reaction,
                                      max_coarse_elements=max_coarse_elements)
        self.M = VCycle(self.levels, omega=omega, n_smooth=n_smooth, gamma=gamma)
        info = {}
        U, self.forward_n_iter = pcg(self.levels[0], project(F, mask), self.M, rtol=rtol,
                                     max_iter=max_iter, x0=x0, info=info)
        self.U = project(U, mask)

    def adjoint(self, g):
        """``(grad_density, grad_F, grad_reaction, n_iter)`` for ``dL/dU = g``
        (torch_solve.py:118-154): warm start ``alpha U``, ``alpha = (U.g)/(U.F)``."""
        U, F = self.U, np.broadcast_to(self.F, self.U.shape)
        alpha = safe_div((U * g).sum(-1), (U * F).sum(-1))
        x0 = alpha[..., None] * U
        lam, n = pcg(self.levels[0], project(g, self.mask), self.M, rtol=self.rtol,
                     max_iter=self.max_iter, x0=x0)
        lam = project(lam, self.mask)
        Ue = U[..., self.edof]
        le = lam[..., self.edof]
        grad_density = -np.sum((le @ self.KE) * Ue, axis=-1)
        grad_reaction = -np.sum(le * Ue, axis=-1) / 4
        return grad_density, lam, grad_reaction, n


# ---------------------------------------------------------------------------------
# Virtual-heat time field (sttopt/virtual_heat.py), one_minus map
# ---------------------------------------------------------------------------------

DENSITY_FLOOR = 1e-6  # virtual_heat.py:44


def plate_nodes(nelx, nely, print_base="bottom_edge"):
    """Build-plate node mask on the whole mesh (virtual_heat.py:82-108)."""
    plate = np.zeros((nely + 1, nelx + 1), bool)
    if print_base == "left_edge":
        plate[:, 0] = True
    elif print_base == "bottom_edge":
        plate[-1, :] = True
    elif print_base == "right_edge":
        plate[:, -1] = True
    else:
        raise ValueError(print_base)
    return plate.ravel()


def element_means(u, edof):
    """Mean of the four nodal values (virtual_heat.py:162-166)."""
    return u[..., edof].mean(axis=-1)


def part_mask(xPhys):
    """``xPhys >= max(xPhys) / 2`` (virtual_heat.py:180-186)."""
    return xPhys >= xPhys.max() / 2


def heat_time_field(xPhys, mu, *, drain_beta=25.0, chi_contrast=1000.0, rtol=1e-8,
                    conduction_penal=1.0, print_base="bottom_edge",
                    max_coarse_elements=MAX_COARSE_ELEMENTS, want_adjoint=None):
    """``one_minus`` virtual-heat time field (virtual_heat.py:404-462 with
    ScalarMesh.solve virtual_heat.py:253-288 and lifted_femsolve torch_solve.py:246-287).

    Returns a dict with ``tPhys`` (nely, nelx), ``T`` (nodal), ``t_e``, ``scale``,
    ``chi`` and the solver object.  If ``want_adjoint`` is a ``(nely, nelx)`` weight
    ``w``, also returns ``grad_x``/``grad_mu`` of ``sum(w * tPhys)`` with the
    normalisation scale held constant (its gradient is discarded in the reference).
    """
    nely, nelx = xPhys.shape
    edof = element_dof_map(nelx, nely, 1)
    KE = diffusion_KE()
    x = xPhys.ravel()
    penalized = np.maximum(x**conduction_penal, DENSITY_FLOOR)
    chi_mu = chi_contrast ** (mu.ravel() - 0.5)
    chi = penalized * chi_mu
    alpha = drain_beta / (nelx * nely)
    plate = plate_nodes(nelx, nely, print_base)
    mask = ~plate
    lift = plate.astype(np.float64)
    reaction = np.full_like(chi, alpha)
    ndof = (nelx + 1) * (nely + 1)
    K_lift = matvec(lift, chi, edof, KE, ndof) + lumped_reaction(reaction, edof, ndof) * lift
    rhs = -K_lift
    solver = FemSolveOracle(chi, rhs, edof, KE, mask, nelx, nely, reaction=reaction, rtol=rtol,
                            max_coarse_elements=max_coarse_elements)
    T = solver.U + lift
    t = 1 - T
    t_e = element_means(t, edof).reshape(nely, nelx)
    scale = t_e[part_mask(xPhys)].max()
    out = dict(tPhys=t_e / scale, T=T, t_e=t_e, scale=scale, chi=chi, solver=solver,
               forward_n_iter=solver.forward_n_iter,
               _adj=(x, lift, edof, KE, ndof, chi_mu, penalized, conduction_penal, chi_contrast))
    if want_adjoint is not None:
        out.update(heat_adjoint(out, want_adjoint))
    return out


def heat_adjoint(heat, w):
    """``grad_x``, ``grad_mu`` and ``backward_n_iter`` of ``sum(w * tPhys)`` for a
    ``heat_time_field`` result, the normalisation scale held constant."""
    x, lift, edof, KE, ndof, chi_mu, penalized, conduction_penal, chi_contrast = heat["_adj"]
    nely, nelx = heat["t_e"].shape
    scale, solver = heat["scale"], heat["solver"]
    w = np.asarray(w).ravel()
    # d/dT of sum(w * (1 - mean(T)) / scale): -w_e/(4 scale) to each corner node
    gT = _scatter(np.broadcast_to((-w / (4 * scale))[:, None], edof.shape).copy(), edof, ndof)
    gd, gF, gr, n = solver.adjoint(gT)
    # rhs = -K(chi) lift - rdiag lift, so d rhs / d chi_e contributes
    # grad_F . (-KE lift_e); combined with grad_density this is -lam_e KE T_e.
    lift_e = lift[edof]
    g_chi = gd - np.sum((gF[edof] @ KE) * lift_e, axis=-1)
    dpen = np.where(x**conduction_penal >= DENSITY_FLOOR, conduction_penal * x ** (conduction_penal - 1), 0.0)
    return dict(grad_x=(g_chi * chi_mu * dpen).reshape(nely, nelx),
                grad_mu=(g_chi * penalized * chi_mu * math.log(chi_contrast)).reshape(nely, nelx),
                backward_n_iter=n)


# ---------------------------------------------------------------------------------
# Space-time stage compliances (sttopt/compliance.py, sttopt/gravity.py)
# ---------------------------------------------------------------------------------


def time_mask_smooth(tPhys, ti, beta):
    """The reference's smooth stage indicator (compliance.py:33-46)."""
    num = math.tanh(beta * ti) + np.tanh(beta * (tPhys - ti))
    den = math.tanh(beta * ti) + math.tanh(beta * (1 - ti))
    return np.maximum(1 - num / den, 0.0)


def stage_membership(tPhys, n_stage):
    """Hard stage membership ``t <= s / n_stage`` for ``s = 1..n_stage`` as uint8
    ``(n_stage, nel)``; the threshold ``s / n_stage`` is the FP64 quotient."""
    t = tPhys.ravel()
    return np.stack([(t <= s / n_stage) for s in range(1, n_stage + 1)]).astype(np.uint8)


def gravity_load(xt, nelx, nely):
    """``F[1::2] = -C xt`` with ``fe / 4`` per corner, ``fe = 1/(nelx nely)``
    (gravity.py:15-36, compliance.py:158-160).  ``xt`` is ``(*batch, nel)``."""
    fe = 1 / (nelx * nely)
    edof1 = element_dof_map(nelx, nely, 1)
    nnode = (nelx + 1) * (nely + 1)
    per = np.broadcast_to((xt * (fe / 4))[..., :, None], (*xt.shape, 4)).copy()
    f = -_scatter(per, edof1, nnode)
    F = np.zeros((*xt.shape[:-1], 2 * nnode))
    F[..., 1::2] = f
    return F


def element_strain_energy(U, edof, KE):
    """``U_e^T KE U_e`` (compliance.py:49-59)."""
    Ue = U[..., edof]
    return np.sum((Ue @ KE) * Ue, axis=-1)


def _stage_row_task(args):
    """One stage of the space-time objective, alone: its self-weight solve, compliance,
    adjoint and gradient contribution (a worker's share of ``spacetime_objective`` with a
    process pool)."""
    x, m, nelx, nely, Emin, Emax, penal, nu, rtol, mce = args
    KE = plane_stress_KE(nu)
    edof = element_dof_map(nelx, nely, 2)
    xt = x * m
    density = simp_density(xt, Emin, Emax, penal)
    F = gravity_load(xt[None], nelx, nely)[0]
    mask = bottom_clamped_mask(nelx, nely)
    solver = FemSolveOracle(density, F, edof, KE, mask, nelx, nely, rtol=rtol, max_coarse_elements=mce)
    U = solver.U
    ce = element_strain_energy(U, edof, KE)
    c = float(np.sum(density * ce))
    g = 2 * matvec(U, density, edof, KE, U.shape[-1])
    gd, gF, _, n_adj = solver.adjoint(g)
    dxt = (ce + gd) * penal * xt ** (penal - 1) * (Emax - Emin)
    edof1 = element_dof_map(nelx, nely, 1)
    dxt = dxt - (1 / (4 * nelx * nely)) * gF[1::2][edof1].sum(-1)
    return c, dxt * m, solver.forward_n_iter, n_adj


def _single_thread_worker():
    """Pool initializer: one thread per worker process (the pool supplies the parallelism)."""
    import os

    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"


def stage_pool(workers):
    """A spawn-started process pool for ``spacetime_objective(..., pool=...)`` (spawn: a
    forked child of a process that has used a GPU can hang)."""
    import multiprocessing

    return multiprocessing.get_context("spawn").Pool(workers, initializer=_single_thread_worker)


def spacetime_objective(xPhys, w, *, n_stage=16, Emin=1e-9, Emax=1.0, penal=3.0, nu=0.3,
                        drain_beta=25.0, conduction_penal=3.0, rtol=1e-8,
                        max_coarse_elements=MAX_COARSE_ELEMENTS, gradient=True, pool=None):
    """The space-time objective ``sum_s c_s + sum(w * tPhys)`` and its gradient in xPhys.

    Heat time field with a bottom-edge plate (``one_minus`` map, mu = 1/2), stage
    membership ``tPhys <= s / n_stage``, per-stage self-weight load on the stage's
    elements with the bottom node row clamped, SIMP stiffness of ``xPhys * m_s``.  The
    gradient is the autograd chain of the reference (compliance.py:137-161,198-253,
    torch_solve.py:118-154) written out: per stage
    ``m (-p (E0-Emin) xt^(p-1) ce - 2 C^T U_y)`` plus the heat adjoint term.

    With ``pool`` (``stage_pool``) the stages are solved one per task in the pool's worker
    processes while this process runs the heat adjoint; each stage is then its own PCG
    (stopping when it converges) instead of a row of one batched PCG.
    """
    nely, nelx = xPhys.shape
    nel = nelx * nely
    if pool is not None:
        return _spacetime_objective_pool(xPhys, w, pool, n_stage=n_stage, Emin=Emin, Emax=Emax, penal=penal, nu=nu,
                                         drain_beta=drain_beta, conduction_penal=conduction_penal, rtol=rtol,
                                         max_coarse_elements=max_coarse_elements, gradient=gradient)
    KE = plane_stress_KE(nu)
    edof = element_dof_map(nelx, nely, 2)
    mu = np.full_like(xPhys, 0.5)
    heat = heat_time_field(xPhys, mu, drain_beta=drain_beta, rtol=rtol,
                           conduction_penal=conduction_penal,
                           max_coarse_elements=max_coarse_elements,
                           want_adjoint=w if gradient else None)
    tPhys = heat["tPhys"]
    m = stage_membership(tPhys, n_stage).astype(np.float64)
    xt = xPhys.ravel()[None, :] * m
    density = simp_density(xt, Emin, Emax, penal)
    F = gravity_load(xt, nelx, nely)
    mask = bottom_clamped_mask(nelx, nely)
    solver = FemSolveOracle(density, F, edof, KE, mask, nelx, nely, rtol=rtol,
                            max_coarse_elements=max_coarse_elements)
    U = solver.U
    ce = element_strain_energy(U, edof, KE)
    c_s = np.sum(density * ce, axis=-1)
    J_t = float(np.sum(w * tPhys))
    out = dict(objective=float(c_s.sum()) + J_t, c_s=c_s, J_t=J_t, tPhys=tPhys,
               membership=m.astype(np.uint8), U=U, T=heat["T"],
               forward_n_iter=solver.forward_n_iter, heat_n_iter=heat["forward_n_iter"])
    if gradient:
        # dL/dU = 2 K(density) U per stage row; adjoint warm start makes it exact.
        g = 2 * matvec(U, density, edof, KE, U.shape[-1])
        gd, gF, _, n_adj = solver.adjoint(g)
        # dL/d density = ce (direct) + grad_density; d density/d xt = p xt^(p-1)(E0-Emin)
        dxt = (ce + gd) * penal * xt ** (penal - 1) * (Emax - Emin)
        # F_y = -C xt -> d/dxt_e = -(fe/4) sum of gF_y over its corners
        edof1 = element_dof_map(nelx, nely, 1)
        fe = 1 / nel
        gFy = gF[..., 1::2]
        dxt = dxt - (fe / 4) * gFy[..., edof1].sum(-1)
        grad = (dxt * m).sum(0).reshape(nely, nelx) + heat["grad_x"]
        out.update(gradient=grad, adjoint_n_iter=n_adj, heat_adjoint_n_iter=heat["backward_n_iter"])
    return out


def _spacetime_objective_pool(xPhys, w, pool, *, n_stage, Emin, Emax, penal, nu, drain_beta, conduction_penal,
                              rtol, max_coarse_elements, gradient):
    nely, nelx = xPhys.shape
    mu = np.full_like(xPhys, 0.5)
    heat = heat_time_field(xPhys, mu, drain_beta=drain_beta, rtol=rtol, conduction_penal=conduction_penal,
                           max_coarse_elements=max_coarse_elements)
    tPhys = heat["tPhys"]
    m = stage_membership(tPhys, n_stage).astype(np.float64)
    x = xPhys.ravel()
    tasks = [(x, m[s], nelx, nely, Emin, Emax, penal, nu, rtol, max_coarse_elements) for s in range(n_stage)]
    pending = pool.map_async(_stage_row_task, tasks)
    heat_grad = heat_adjoint(heat, w) if gradient else None  # overlaps the stage tasks
    rows = pending.get()
    c_s = np.array([r[0] for r in rows])
    J_t = float(np.sum(w * tPhys))
    out = dict(objective=float(c_s.sum()) + J_t, c_s=c_s, J_t=J_t, tPhys=tPhys, membership=m.astype(np.uint8),
               T=heat["T"], forward_n_iter=max(r[2] for r in rows), heat_n_iter=heat["forward_n_iter"])
    if gradient:
        grad = np.sum([r[1] for r in rows], axis=0).reshape(nely, nelx) + heat_grad["grad_x"]
        out.update(gradient=grad, adjoint_n_iter=max(r[3] for r in rows),
                   heat_adjoint_n_iter=heat_grad["backward_n_iter"])
    return out


# ---------------------------------------------------------------------------------
# Density filter (sttopt/filters.py) -- used to make the smoothed synthetic densities
# ---------------------------------------------------------------------------------


def cone_filter(field, rmin):
    """``H x / Hs`` with ``H[e1,e2] = max(0, rmin - dist)`` over the square of offsets
    ``|d| <= ceil(rmin) - 1`` (filters.py:22-64,67-76), as a zero-padded correlation."""
    nely, nelx = field.shape
    r = int(np.ceil(rmin)) - 1
    num = np.zeros_like(field)
    den = np.zeros_like(field)
    ones = np.ones_like(field)
    pad_f = np.pad(field, r)
    pad_o = np.pad(ones, r)
    for di in range(-r, r + 1):
        for dj in range(-r, r + 1):
            wgt = max(0.0, rmin - math.hypot(di, dj))
            if wgt == 0.0:
                continue
            num += wgt * pad_f[r + dj: r + dj + nely, r + di: r + di + nelx]
            den += wgt * pad_o[r + dj: r + dj + nely, r + di: r + di + nelx]
    return num / den


def smoothed_density(nelx, nely, seed, rmin=4.0, lo=1e-3, hi=1.0):
    """Seeded N(0,1) noise -> cone filter (rmin) -> min-max map to ``[lo, hi]``."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((nely, nelx))
    sm = cone_filter(noise, rmin)
    sm = (sm - sm.min()) / (sm.max() - sm.min())
    return lo + (hi - lo) * sm


# ---- density filter and projection (sttopt/filters.py) ----------------------------------

def density_filter(nelx, nely, rmin):
    """``H[e1, e2] = max(0, rmin - dist)`` over offsets ``|d| <= ceil(rmin) - 1`` and its row
    sums ``Hs`` (filters.py:38-64), as a SciPy CSR matrix."""
    import math

    import scipy.sparse as sp

    r = int(math.ceil(rmin)) - 1
    e = np.arange(nelx * nely)
    i, j = e % nelx, e // nelx
    rows, cols, vals = [], [], []
    for di in range(-r, r + 1):
        for dj in range(-r, r + 1):
            w = max(0.0, rmin - math.hypot(di, dj))
            if w == 0.0:
                continue
            ok = (i + di >= 0) & (i + di < nelx) & (j + dj >= 0) & (j + dj < nely)
            rows.append(e[ok])
            cols.append(((j + dj) * nelx + (i + di))[ok])
            vals.append(np.full(ok.sum(), w))
    H = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nelx * nely, nelx * nely)).tocsr()
    return H, np.asarray(H.sum(axis=1)).ravel()


def apply_density_filter(field, H, Hs):
    """``H @ field / Hs``, shape-preserving (filters.py:67-78)."""
    return (H @ np.asarray(field).ravel() / Hs).reshape(np.shape(field))


def heaviside_projection(xt, beta, eta):
    """Smoothed threshold (filters.py:109-127); ``beta = inf`` is the step, 1/2 at eta."""
    import math

    if math.isinf(beta):
        return np.where(xt > eta, 1.0, np.where(xt < eta, 0.0, 0.5))
    den = math.tanh(beta * eta) + math.tanh(beta * (1 - eta))
    return (math.tanh(beta * eta) + np.tanh(beta * (xt - eta))) / den


def heaviside_projection_derivative(xt, beta, eta):
    """(filters.py:128-133)"""
    import math

    den = math.tanh(beta * eta) + math.tanh(beta * (1 - eta))
    return beta * (1 - np.tanh(beta * (xt - eta)) ** 2) / den

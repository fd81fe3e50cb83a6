"""Drop-in for ``sttopt.mma``: Svanberg's method of moving asymptotes on the device
(sttopt/mma.py:22-557).

``mmasub`` and ``subsolv`` keep the reference's signatures and return values.  Every
n-sized and m x n-sized quantity stays on the GPU and is handled by fused FP64 passes in
``libsttb200.so`` (``stt_mma_sub``, ``stt_mma_subsolv``): the asymptotes and move limits,
and for each Newton step of the primal-dual interior-point solve one pass that forms the
residual, the Newton right-hand side and the m x m matrix ``GG diag(1/diagx) GG^T``, one
pass for ``dx`` with its step limits and one pass per line-search halving.  ``mmasub``
never stores the approximation ``P, Q``: the passes rebuild it from ``dfdx``.  The
m-sized algebra (y, z, lam, mu, zet, s and the bordered Newton system) runs on the host,
where the reference also solves that system.  With ``m >= n`` the whole subproblem has
at most m variables and is solved in the library's host code.  Up to 64 constraints
when ``m < n``.

``trust_region_params``, ``History``, ``unit_box_step`` and ``floor_share`` are the
reference's small wrappers around ``mmasub`` (sttopt/mma.py:22-147).
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass

import numpy as np
import torch
from torch import Tensor

from . import _lib

EPSIMIN = 1e-7  # sttopt/mma.py:218
MAX_CONSTRAINTS = 64  # the device path's limit on m when m < n


def trust_region_params(move_limit: Tensor, xrange: Tensor, *, asyclamp_min_ratio: float = 0.02,
                        asyclamp_max_ratio: float = 20.0) -> dict[str, Tensor]:
    """``mmasub`` keywords for a trust region of half-width ``move_limit``: the asymptotes
    start at ``move_limit / xrange`` and are clamped to ``[asyclamp_min_ratio,
    asyclamp_max_ratio]`` times that (sttopt/mma.py:22-56)."""
    asyinit = move_limit / xrange
    return {"asyinit": asyinit, "asyclamp_min": asyclamp_min_ratio * asyinit,
            "asyclamp_max": asyclamp_max_ratio * asyinit, "move": asyinit}


@dataclass(frozen=True)
class History:
    """What ``mmasub`` carries between iterations: the last two points and the
    asymptotes (sttopt/mma.py:59-75)."""

    xold1: Tensor
    xold2: Tensor
    low: Tensor
    upp: Tensor

    @classmethod
    def initial(cls, xold: Tensor) -> "History":
        zeros = torch.zeros_like(xold)
        return cls(xold1=xold, xold2=xold.clone(), low=zeros, upp=zeros.clone())


def unit_box_step(history: History, iteration: int, xval: Tensor, move_limit: Tensor, f0val: float,
                  df0dx: Tensor, fval: Tensor, dfdx: Tensor, *, a0: float, c: float, raa0: float,
                  stats: dict | None = None) -> tuple[Tensor, Tensor, History]:
    """One MMA iteration on variables in [0, 1] with a trust region of half-width
    ``move_limit`` and every constraint relaxed at cost ``c`` (sttopt/mma.py:78-128).
    Returns ``(xmma, lam, history)``."""
    m = len(fval)
    xmin = torch.zeros_like(xval)
    xmax = torch.ones_like(xval)
    zeros = torch.zeros(m, device=xval.device, dtype=xval.dtype)
    xmma, _, _, lam, *_, low, upp = mmasub(
        m, len(xval), iteration, xval, xmin, xmax, history.xold1, history.xold2, f0val, df0dx, fval, dfdx,
        history.low, history.upp, a0, zeros, torch.full_like(zeros, c), zeros.clone(), raa0=raa0, stats=stats,
        **trust_region_params(move_limit, xmax - xmin))
    return xmma, lam, History(xold1=xval, xold2=history.xold1, low=low, upp=upp)


def floor_share(history: History, move_limit: Tensor, mask: Tensor) -> float:
    """Share of the variables in ``mask`` whose asymptotes sit at their floor
    (sttopt/mma.py:131-147); 0 for an empty mask."""
    floor = trust_region_params(move_limit, torch.ones_like(move_limit))["asyclamp_min"]
    at_floor = (history.upp - history.low) / 2 <= floor * (1 + 1e-6)
    return float(at_floor[mask].double().mean()) if bool(mask.any()) else 0.0


def _dev(t: Tensor, n: int, name: str) -> Tensor:
    if not isinstance(t, Tensor) or t.dtype != torch.float64 or t.numel() != n:
        raise TypeError(f"{name}: expected a float64 tensor of {n} entries")
    _lib.require_cuda(t)
    return t.reshape(n).contiguous()


def _rows(t: Tensor, m: int, n: int, name: str) -> Tensor:
    if not isinstance(t, Tensor) or t.dtype != torch.float64 or tuple(t.shape) != (m, n):
        raise TypeError(f"{name}: expected a float64 tensor of shape ({m}, {n})")
    _lib.require_cuda(t)
    return t if t.stride(1) == 1 and t.stride(0) >= n else t.contiguous()


def _host(v, m: int, name: str) -> np.ndarray:
    arr = v.detach().to("cpu", torch.float64).numpy() if isinstance(v, Tensor) else np.asarray(v, np.float64)
    arr = np.ascontiguousarray(arr.reshape(-1), dtype=np.float64)
    if arr.size != m:
        raise ValueError(f"{name}: expected {m} entries, got {arr.size}")
    return arr


def _param(v, n: int, name: str, keep: list) -> tuple[int | None, float]:
    """A per-variable keyword: a device n-vector (pointer) or a scalar (value)."""
    if isinstance(v, Tensor) and v.numel() != 1:
        t = _dev(v, n, name)
        keep.append(t)
        return t.data_ptr(), 0.0
    return None, float(v)


class _Out:
    """The m-sized results (host) of one subproblem solve."""

    def __init__(self, m: int):
        self.y, self.lam, self.mu, self.s = (np.zeros(m) for _ in range(4))
        self.z, self.zet, self.eps = (np.zeros(1) for _ in range(3))
        self.counts = np.zeros(3, np.int32)  # levels at the Newton cap, Newton steps, line-search tries

    def ptrs(self) -> list[int]:
        return [a.ctypes.data for a in (self.y, self.z, self.lam, self.mu, self.zet, self.s, self.counts, self.eps)]

    def tensors(self, device) -> tuple[Tensor, ...]:
        def dev(a):
            return torch.from_numpy(a.copy()).to(device)

        return dev(self.y), dev(self.z).reshape(()), dev(self.lam), dev(self.mu), dev(self.zet).reshape(()), dev(self.s)

    def report(self, stats: dict | None) -> None:
        hits, steps, tries = (int(v) for v in self.counts)
        if stats is not None:
            stats["subsolv_newton_steps"] = stats.get("subsolv_newton_steps", 0) + steps
            stats["subsolv_line_search_tries"] = stats.get("subsolv_line_search_tries", 0) + tries
        if hits:
            if stats is not None:
                stats["subsolv_cap_hits"] = stats.get("subsolv_cap_hits", 0) + hits
            warnings.warn(
                f"subsolv: inner Newton loop hit the iteration cap (ittt=200) at {hits} barrier level(s), the last "
                f"at epsi={float(self.eps[0])}, without reaching the 0.9*epsi residual target",
                RuntimeWarning, stacklevel=3)


def _check_m(m: int, n: int) -> None:
    if m < 1 or n < 1:
        raise ValueError(f"mma: m and n must be positive (got m={m}, n={n})")
    if m < n and m > MAX_CONSTRAINTS:
        raise ValueError(f"mma: the device subproblem takes at most {MAX_CONSTRAINTS} constraints when m < n "
                         f"(got m={m})")


def mmasub(m: int, n: int, iteration: int, xval: Tensor, xmin: Tensor, xmax: Tensor, xold1: Tensor,
           xold2: Tensor, f0val: float, df0dx: Tensor, fval: Tensor, dfdx: Tensor, low: Tensor, upp: Tensor,
           a0: float, a: Tensor, c: Tensor, d: Tensor, asyinit=0.5, asyclamp_min=0.01, asyclamp_max=10.0,
           move=0.5, raa0: float = 1e-5, albefa: float = 0.1, asyincr: float = 1.2, asydecr: float = 0.7,
           stats: dict | None = None):
    """One MMA iteration (sttopt/mma.py:150-285): the moving asymptotes, the separable
    approximation and its solution by ``subsolv``.  Returns ``(xmma, ymma, zmma, lam, xsi,
    eta, mu, zet, s, low, upp)``; ``f0val`` is unused, as in the reference.  ``stats``
    gathers ``subsolv_cap_hits`` as the reference's does, and the solve's Newton steps
    and line-search tries (``subsolv_newton_steps``, ``subsolv_line_search_tries``)."""
    del f0val
    _check_m(m, n)
    xs = [_dev(t, n, nm) for t, nm in ((xval, "xval"), (xmin, "xmin"), (xmax, "xmax"), (xold1, "xold1"),
                                        (xold2, "xold2"), (df0dx, "df0dx"))]
    G = _rows(dfdx, m, n, "dfdx")
    device = xs[0].device
    low_o = _dev(low, n, "low").clone()
    upp_o = _dev(upp, n, "upp").clone()
    keep: list = []
    params = [_param(v, n, nm, keep) for v, nm in ((asyinit, "asyinit"), (asyclamp_min, "asyclamp_min"),
                                                   (asyclamp_max, "asyclamp_max"), (move, "move"))]
    hf, ha, hc, hd = (_host(v, m, nm) for v, nm in ((fval, "fval"), (a, "a"), (c, "c"), (d, "d")))
    xmma, xsi, eta = (torch.empty(n, dtype=torch.float64, device=device) for _ in range(3))
    out = _Out(m)
    with torch.cuda.device(device):
        nbytes = _lib.lib().stt_mma_workspace_bytes(m, n)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=device)
        flat = [p for pv in params for p in pv]
        _lib.check(_lib.lib().stt_mma_sub(
            m, n, int(iteration), *(t.data_ptr() for t in xs[:5]), xs[5].data_ptr(), hf.ctypes.data, G.data_ptr(),
            G.stride(0), low_o.data_ptr(), upp_o.data_ptr(), float(a0), ha.ctypes.data, hc.ctypes.data,
            hd.ctypes.data, *flat, float(raa0), float(albefa), float(asyincr), float(asydecr), xmma.data_ptr(),
            xsi.data_ptr(), eta.data_ptr(), *out.ptrs(), ws.data_ptr(), nbytes, _lib.stream()))
    out.report(stats)
    y, z, lam, mu, zet, s = out.tensors(device)
    return xmma, y, z, lam, xsi, eta, mu, zet, s, low_o, upp_o


def subsolv(m: int, n: int, epsimin: float, low: Tensor, upp: Tensor, alfa: Tensor, beta: Tensor, p0: Tensor,
            q0: Tensor, P: Tensor, Q: Tensor, a0: float, a: Tensor, b: Tensor, c: Tensor, d: Tensor,
            stats: dict | None = None):
    """The MMA subproblem's primal-dual Newton solve along the barrier path
    (sttopt/mma.py:346-557).  Returns ``(x, y, z, lam, xsi, eta, mu, zet, s)``."""
    _check_m(m, n)
    vs = [_dev(t, n, nm) for t, nm in ((low, "low"), (upp, "upp"), (alfa, "alfa"), (beta, "beta"), (p0, "p0"),
                                        (q0, "q0"))]
    Pm, Qm = _rows(P, m, n, "P"), _rows(Q, m, n, "Q")
    if Pm.stride(0) != Qm.stride(0):
        Pm, Qm = Pm.contiguous(), Qm.contiguous()
    device = vs[0].device
    ha, hb, hc, hd = (_host(v, m, nm) for v, nm in ((a, "a"), (b, "b"), (c, "c"), (d, "d")))
    x, xsi, eta = (torch.empty(n, dtype=torch.float64, device=device) for _ in range(3))
    out = _Out(m)
    with torch.cuda.device(device):
        nbytes = _lib.lib().stt_mma_workspace_bytes(m, n)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=device)
        _lib.check(_lib.lib().stt_mma_subsolv(
            m, n, float(epsimin), *(t.data_ptr() for t in vs), Pm.data_ptr(), Qm.data_ptr(), Pm.stride(0), float(a0),
            ha.ctypes.data, hb.ctypes.data, hc.ctypes.data, hd.ctypes.data, x.data_ptr(), xsi.data_ptr(),
            eta.data_ptr(), *out.ptrs(), ws.data_ptr(), nbytes, _lib.stream()))
    out.report(stats)
    y, z, lam, mu, zet, s = out.tensors(device)
    return x, y, z, lam, xsi, eta, mu, zet, s

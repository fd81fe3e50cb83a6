"""Drop-in for the solve path of ``sttopt.virtual_heat``: the scalar Q4 mesh and the
virtual-heat time field (sttopt/virtual_heat.py:82-108,162-201,205-288,404-462).

``heat_time_field`` solves ``-div(chi grad T) + alpha T = 0`` with ``T = 1`` on the
build plate through ``lifted_femsolve`` (device hierarchy with the lumped drain,
device PCG, adjoint kernels), then maps ``T`` to ``t`` (``one_minus`` or ``neg_log``),
or ``poisson``: a second scalar solve fitted to the direction of ``-grad T``), takes
element means and normalises over the part.  ``laplace_time_field`` (Variant 2,
sttopt/virtual_heat.py:546-607) solves ``div(chi grad t) = 0`` with the wall data on the
domain's boundary arc, with the ``identity`` or ``poisson`` map.  The Poisson fit's load
(``divergence_load(w, direction_field(s))``), the element means and their adjoints are
device kernels (``stt_poisson_load``, ``stt_element_means``).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import NamedTuple

import numpy as np
import torch
from torch import Tensor

from . import _geom, _lib, fem, torch_solve

DENSITY_FLOOR = 1e-6  # sttopt/virtual_heat.py:44
NEG_LOG_FLOOR = 1e-3  # sttopt/virtual_heat.py:48


def domain_nodes(active: np.ndarray) -> np.ndarray:
    """Nodes of at least one active element (sttopt/virtual_heat.py:74-79)."""
    padded = np.pad(active, 1)
    return padded[1:, 1:] | padded[1:, :-1] | padded[:-1, 1:] | padded[:-1, :-1]


def plate_nodes(nelx: int, nely: int, print_base: str, active: np.ndarray | None = None) -> np.ndarray:
    """The build plate's nodes on the design domain (sttopt/virtual_heat.py:82-108)."""
    plate = np.zeros((nely + 1, nelx + 1), bool)
    base = print_base.lower()
    if base == "left_edge":
        plate[:, 0] = True
    elif base == "bottom_edge":
        plate[-1, :] = True
    elif base == "right_edge":
        plate[:, -1] = True
    else:
        raise ValueError(
            "a virtual-heat time field needs a plate print base (left_edge, bottom_edge or "
            f"right_edge), got {print_base!r}")
    active = np.ones((nely, nelx), bool) if active is None else active
    return (plate & domain_nodes(active)).ravel()


# 2 x 2 Gauss points of the unit square, (xi, eta) with xi fastest
_G = (0.5 - 0.5 / np.sqrt(3.0), 0.5 + 0.5 / np.sqrt(3.0))
_GAUSS = [(xi, eta) for eta in _G for xi in _G]


def shape_gradients() -> np.ndarray:
    """``(4, 2, 4)``: grad of the bilinear shape functions at the Gauss points, x right
    and y up, local order BL, BR, TR, TL (sttopt/virtual_heat.py:55-67)."""
    return np.array([[[eta - 1.0, 1.0 - eta, eta, -eta], [xi - 1.0, -xi, xi, 1.0 - xi]]
                     for xi, eta in _GAUSS])


_shape_gradients = shape_gradients


def _whole(nelx: int, nely: int) -> np.ndarray:
    """The whole mesh as the design domain."""
    return np.ones((nely, nelx), bool)


def _boundary_loop(active: np.ndarray) -> np.ndarray:
    """The domain's boundary nodes, once each, clockwise from its top-left node
    (sttopt/virtual_heat.py:111-140); raises unless the boundary is one simple loop."""
    nely, nelx = active.shape
    inside = np.pad(active, 1)
    links: dict[tuple[int, int], list[tuple[int, int]]] = {}

    def link(a, b):
        links.setdefault(a, []).append(b)
        links.setdefault(b, []).append(a)

    # horizontal edge (r, c)-(r, c+1) lies between element rows r-1 and r
    for r, c in zip(*np.nonzero(inside[1:, 1:-1] != inside[:-1, 1:-1])):
        link((int(r), int(c)), (int(r), int(c) + 1))
    # vertical edge (r, c)-(r+1, c) lies between element columns c-1 and c
    for r, c in zip(*np.nonzero(inside[1:-1, 1:] != inside[1:-1, :-1])):
        link((int(r), int(c)), (int(r) + 1, int(c)))
    if any(len(v) != 2 for v in links.values()):
        raise ValueError("the design domain's boundary must be one simple loop")
    start = min(links)
    order, prev, cur = [start], start, (start[0], start[1] + 1)
    while cur != start:
        order.append(cur)
        a, b = links[cur]
        prev, cur = cur, (b if a == prev else a)
    if len(order) != len(links):
        raise ValueError("the design domain's boundary must be one simple loop")
    return np.array([r * (nelx + 1) + c for r, c in order], dtype=np.int64)


def wall_arc(nelx: int, nely: int, print_base: str, active: np.ndarray | None = None) -> np.ndarray:
    """The boundary nodes off the plate, along the boundary from one end of the plate to
    the other (sttopt/virtual_heat.py:143-159)."""
    active = np.ones((nely, nelx), bool) if active is None else active
    loop = _boundary_loop(active)
    on_plate = plate_nodes(nelx, nely, print_base, active)
    last = int(np.flatnonzero(on_plate[loop])[-1])
    rolled = np.concatenate([loop[last + 1:], loop[:last + 1]])
    return rolled[~on_plate[rolled]]


def _means(u: Tensor, nelx: int, nely: int, transpose: bool) -> Tensor:
    nel, nnode = nelx * nely, (nelx + 1) * (nely + 1)
    n_in, n_out = (nel, nnode) if transpose else (nnode, nel)
    U = u.detach().to(torch.float64).reshape(-1, n_in).contiguous()
    out = torch.empty(U.shape[0], n_out, dtype=torch.float64, device=U.device)
    _lib.check(_lib.lib().stt_element_means(nelx, nely, U.shape[0], _lib.ptr(U), n_in, _lib.ptr(out), n_out,
                                            int(transpose), _lib.stream()))
    return out.reshape(*u.shape[:-1], n_out).to(u.dtype)


class _ElementMeans(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, nelx, nely):
        ctx.grid = (nelx, nely)
        return _means(u, nelx, nely, False)

    @staticmethod
    def backward(ctx, g):
        return _means(g, *ctx.grid, True), None, None


def element_means(u: Tensor, edof: Tensor) -> Tensor:
    """Mean of each element's four nodal values (sttopt/virtual_heat.py:162-166), by the
    ``stt_element_means`` gather; differentiable."""
    _lib.require_cuda(u)
    nelx, nely = _geom.grid_shape(edof, u.shape[-1], 1)
    return _ElementMeans.apply(u, nelx, nely)


class _PoissonLoad(torch.autograd.Function):
    """``divergence_load(w, direction_field(s))`` in one kernel, forward and adjoint."""

    @staticmethod
    def forward(ctx, s, w, nelx, nely):
        S = s.detach().to(torch.float64).contiguous()
        W = w.detach().to(torch.float64).contiguous()
        F = torch.empty_like(S)
        _lib.check(_lib.lib().stt_poisson_load(nelx, nely, 1, _lib.ptr(S), S.numel(), _lib.ptr(W), W.numel(),
                                               _lib.ptr(F), F.numel(), _lib.stream()))
        ctx.save_for_backward(S, W)
        ctx.grid = (nelx, nely)
        return F.to(s.dtype)

    @staticmethod
    def backward(ctx, gF):
        S, W = ctx.saved_tensors
        nelx, nely = ctx.grid
        G = gF.detach().to(torch.float64).contiguous()
        gs = torch.empty_like(S) if ctx.needs_input_grad[0] else None
        gw = torch.empty_like(W) if ctx.needs_input_grad[1] else None
        if gs is None and gw is None:
            return None, None, None, None
        _lib.check(_lib.lib().stt_poisson_load_adjoint(
            nelx, nely, 1, _lib.ptr(S), S.numel(), _lib.ptr(W), W.numel(), _lib.ptr(G), G.numel(),
            _lib.ptr(gs), S.numel(), _lib.ptr(gw), W.numel(), _lib.stream()))
        return gs, gw, None, None


def diffusivity(mu: Tensor, contrast: float) -> Tensor:
    """``contrast**(mu - 1/2)`` (sttopt/virtual_heat.py:169-177)."""
    return contrast ** (mu - 0.5)


def part_mask(xPhys: Tensor) -> Tensor:
    """``xPhys >= max(xPhys) / 2`` (sttopt/virtual_heat.py:180-186)."""
    return xPhys >= xPhys.max() / 2


def normalize(t: Tensor, xPhys: Tensor) -> Tensor:
    """``t`` over its maximum on the part, the scale held constant (:189-201)."""
    return t / t[part_mask(xPhys)].max().detach()


@dataclass(frozen=True)
class ScalarMesh:
    """The scalar Q4 mesh of the time field (sttopt/virtual_heat.py:204-288)."""

    nelx: int
    nely: int
    edof: Tensor
    KE: Tensor
    B: Tensor  # (4, 2, 4) shape-function gradients at the Gauss points
    plate: Tensor
    arc: Tensor  # the domain's walls off the plate, in boundary order
    active: Tensor

    @classmethod
    def build(cls, nelx: int, nely: int, print_base: str, device, dtype,
              active: np.ndarray | None = None) -> "ScalarMesh":
        active = np.ones((nely, nelx), bool) if active is None else active
        return cls(
            nelx=nelx, nely=nely,
            edof=torch.as_tensor(fem.element_dof_map(nelx, nely, 1), device=device, dtype=torch.int64),
            KE=torch.as_tensor(fem.diffusion_KE(), device=device, dtype=dtype),
            B=torch.as_tensor(shape_gradients(), device=device, dtype=dtype),
            plate=torch.as_tensor(plate_nodes(nelx, nely, print_base, active), device=device),
            arc=torch.as_tensor(wall_arc(nelx, nely, print_base, active), device=device, dtype=torch.int64),
            active=torch.as_tensor(active.ravel(), device=device),
        )

    @property
    def ndof(self) -> int:
        return (self.nelx + 1) * (self.nely + 1)

    @property
    def unit_length(self) -> float:
        return (self.nelx * self.nely) ** 0.5

    def solve(self, chi: Tensor, g: Tensor, fixed: Tensor, rtol: float, *, F: Tensor | None = None,
              reaction: Tensor | None = None, x0: Tensor | None = None,
              precision: str | None = None) -> Tensor:
        """``-div(chi grad u) + reaction u = F`` with ``u = g`` on ``fixed`` (:253-288)."""
        mask = ~fixed
        return torch_solve.lifted_femsolve(
            chi, torch.zeros_like(g) if F is None else F, g, self.edof, self.KE, mask, self.nelx,
            self.nely, reaction=reaction, rtol=rtol, x0=None if x0 is None else (x0 * mask).detach(),
            precision=precision)

    def gauss_gradients(self, u: Tensor) -> Tensor:
        """``(nel, 4, 2)``: grad u at each element's Gauss points (:290-293)."""
        return torch.einsum("gdi,ei->egd", self.B, u[self.edof])

    def direction_field(self, s: Tensor) -> Tensor:
        """``grad s / |grad s|`` at the Gauss points (:295-309)."""
        grad = self.gauss_gradients(s)
        return grad / torch.sqrt((grad**2).sum(dim=-1) + torch.finfo(grad.dtype).tiny)[..., None]

    def divergence_load(self, w: Tensor, X: Tensor) -> Tensor:
        """``F_i = sum_e w_e / 4 sum_g X_eg . grad N_i(g)`` for a given direction field
        (:311-318)."""
        per_node = torch.einsum("e,egd,gdi->ei", w, X, self.B) / 4
        return per_node.new_zeros(self.ndof).index_add(0, self.edof.reshape(-1), per_node.reshape(-1))

    def poisson_load(self, s: Tensor, w: Tensor) -> Tensor:
        """``divergence_load(w, direction_field(s))`` in one device kernel; differentiable
        in ``s`` and ``w``."""
        _lib.require_cuda(s, w)
        return _PoissonLoad.apply(s, w, self.nelx, self.nely)

    def poisson_distance(self, s: Tensor, w: Tensor, rtol: float, x0: Tensor | None = None,
                         precision: str | None = None) -> Tensor:
        """``div(w grad phi) = div(w X)``, ``phi = 0`` on the plate, zero flux elsewhere, X
        the direction in which ``s`` increases (:320-343)."""
        return self.solve(w, torch.zeros_like(s), self.plate, rtol, F=self.poisson_load(s, w), x0=x0,
                          precision=precision)


class TimeFieldSolution(NamedTuple):
    tPhys: Tensor
    primary: Tensor
    poisson: Tensor | None
    t: Tensor


def heat_time_field(config, mesh: ScalarMesh, xPhys: Tensor, mu: Tensor,
                    previous: TimeFieldSolution | None = None, conduction_penal: float = 1.0,
                    density_weighted: bool = True, precision: str | None = None) -> TimeFieldSolution:
    """Variant 1 time field (sttopt/virtual_heat.py:404-462).  ``config`` needs
    ``chi_contrast``, ``drain_beta``, ``heat_cg_rtol`` and ``time_map``."""
    shape = xPhys.shape
    if density_weighted:
        density = torch.clamp(xPhys.flatten(), min=DENSITY_FLOOR)
        penalized = torch.clamp(xPhys.flatten() ** conduction_penal, min=DENSITY_FLOOR)
    else:
        density = penalized = torch.ones_like(xPhys.flatten())
    chi = penalized * diffusivity(mu.flatten(), config.chi_contrast)
    alpha = config.drain_beta / mesh.unit_length**2
    T = mesh.solve(chi, mesh.plate.to(chi.dtype), mesh.plate, config.heat_cg_rtol,
                   reaction=torch.full_like(chi, alpha),
                   x0=None if previous is None else previous.primary, precision=precision)
    phi = None
    time_map = str(getattr(config.time_map, "value", config.time_map))
    if time_map == "one_minus":
        t = 1 - T
    elif time_map == "neg_log":
        with torch.no_grad():
            part = part_mask(xPhys).flatten()
            floor = NEG_LOG_FLOOR * element_means(T, mesh.edof)[part].min()
        t = -torch.log(torch.clamp(T, min=0) + floor)
    elif time_map == "poisson":
        # time runs along -grad T (T falls away from the plate)
        phi = mesh.poisson_distance(-T, density, config.poisson_cg_rtol,
                                    x0=None if previous is None else previous.poisson, precision=precision)
        t = phi
    else:
        raise ValueError(f"time_map {time_map!r} is not one of one_minus, neg_log, poisson")
    t_e = element_means(t, mesh.edof).reshape(shape)
    return TimeFieldSolution(normalize(t_e, xPhys), T, phi, t)


def laplace_time_field(config, mesh: ScalarMesh, xPhys: Tensor, mu: Tensor, b: Tensor,
                       previous: TimeFieldSolution | None = None, density_exponent: float = 0.0,
                       precision: str | None = None) -> TimeFieldSolution:
    """Variant 2 time field, ``div(chi grad t) = 0`` with ``t = 0`` on the plate and
    ``t = b`` on the wall arc (sttopt/virtual_heat.py:546-607).  ``config`` needs
    ``chi_contrast``, ``chi_density_floor``, ``chi_density_sensitivity``,
    ``laplace_cg_rtol``, ``time_map`` (``identity`` or ``poisson``) and, for ``poisson``,
    ``poisson_cg_rtol``."""
    shape = xPhys.shape
    chi = diffusivity(mu.flatten(), config.chi_contrast)
    if density_exponent != 0:
        rho = xPhys if config.chi_density_sensitivity else xPhys.detach()
        chi = chi * torch.clamp(rho.flatten() ** density_exponent, min=config.chi_density_floor)
    chi = torch.where(mesh.active, chi, 1.0)
    g = torch.zeros(mesh.ndof, device=chi.device, dtype=chi.dtype).index_put((mesh.arc,), b)
    fixed = mesh.plate.clone()
    fixed[mesh.arc] = True
    u = mesh.solve(chi, g, fixed, config.laplace_cg_rtol,
                   x0=None if previous is None else previous.primary, precision=precision)
    phi = None
    time_map = str(getattr(config.time_map, "value", config.time_map))
    if time_map == "identity":
        t = u
    elif time_map == "poisson":
        # the walls act only through the direction of grad u
        phi = mesh.poisson_distance(u, torch.ones_like(chi), config.poisson_cg_rtol,
                                    x0=None if previous is None else previous.poisson, precision=precision)
        t = phi
    else:
        raise ValueError(f"time_map {time_map!r} is not one of identity, poisson")
    t_e = element_means(t, mesh.edof).reshape(shape)
    return TimeFieldSolution(normalize(t_e, xPhys), u, phi, t)


# ---- host helpers of the Laplace time field's wall design and the start check -------


def _node_edges(active: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The 8-connected node adjacencies through the design domain, both directions, with
    their Euclidean lengths (sttopt/virtual_heat.py:465-489): an axis step along an edge of
    a domain element, a diagonal across one."""
    nely, nelx = active.shape
    inside = np.pad(active, 1)  # element (r, c) at inside[r + 1, c + 1]
    node = np.arange((nely + 1) * (nelx + 1)).reshape(nely + 1, nelx + 1)
    src, dst, length = [], [], []
    for dr, dc in ((0, 1), (1, 0), (1, 1), (1, -1)):
        r, c = np.mgrid[0:nely + 1 - dr, max(0, -dc):nelx + 1 - max(0, dc)]
        cl = np.minimum(c, c + dc)  # the element column the step runs beside or across
        if dr == 0:
            ok = inside[r, cl + 1] | inside[r + 1, cl + 1]
        elif dc == 0:
            ok = inside[r + 1, cl] | inside[r + 1, cl + 1]
        else:
            ok = inside[r + 1, cl + 1]
        a, b = node[r, c][ok], node[r + dr, c + dc][ok]
        src += [a, b]
        dst += [b, a]
        length.append(np.full(2 * a.size, float(np.hypot(dr, dc))))
    return np.concatenate(src), np.concatenate(dst), np.concatenate(length)


def _plate_distance(mesh: "ScalarMesh") -> Tensor:
    """The wall arc's grid-graph distance to the plate through the domain, in
    ``unit_length`` (sttopt/virtual_heat.py:492-507)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import dijkstra

    active = mesh.active.cpu().numpy().reshape(mesh.nely, mesh.nelx)
    src, dst, length = _node_edges(active)
    graph = csr_matrix((length, (src, dst)), shape=(mesh.ndof, mesh.ndof))
    plate = np.flatnonzero(mesh.plate.cpu().numpy())
    dist = dijkstra(graph, indices=plate, min_only=True)[mesh.arc.cpu().numpy()]
    return torch.as_tensor(dist / mesh.unit_length, device=mesh.arc.device, dtype=mesh.KE.dtype)


def distance_wall(mesh: "ScalarMesh") -> Tensor:
    """The wall data of the distance to the plate, scaled to a largest value of 1/2
    (sttopt/virtual_heat.py:510-520)."""
    d = _plate_distance(mesh)
    return d / (2 * d.max())


def wall_filter(n_arc: int, rmin: float) -> np.ndarray:
    """Cone weights ``max(0, rmin - distance)`` along the wall arc, reflected with the sign
    flipped past either end (into the plate, where t = 0), normalised by the full cone's
    sum (sttopt/virtual_heat.py:523-543)."""
    k = np.arange(n_arc)
    cone = lambda dist: np.maximum(0.0, rmin - np.abs(dist))  # noqa: E731
    H = cone(k[:, None] - k[None, :])
    H[k, k] = max(rmin, 1.0)
    # the plate corners sit at -1 and n_arc: node j reflects to -2 - j and 2 n_arc - j
    H -= cone(k[:, None] + 2 + k[None, :])
    H -= cone(2 * n_arc - k[None, :] - k[:, None])
    full = max(rmin, 1.0) + 2 * cone(np.arange(1, int(np.ceil(rmin)))).sum()
    return H / full


def start_report(mesh: "ScalarMesh", solution: TimeFieldSolution, solid: np.ndarray, base: np.ndarray) -> dict:
    """The print-start check (sttopt/virtual_heat.py:356-390): the part touches the plate,
    and every node of a solid element off the plate has ``t > 0``."""
    t = solution.t.detach().cpu().numpy()
    tPhys = solution.tPhys.detach().cpu().numpy().ravel()
    edof = mesh.edof.cpu().numpy()
    solid = np.asarray(solid).ravel()
    on_base = np.zeros(solid.size, bool)
    on_base[np.asarray(base)] = True
    nodes = np.unique(edof[solid])
    nodes = nodes[~mesh.plate.cpu().numpy()[nodes]]
    earliest = float(t[nodes].min()) if nodes.size else None
    base_t = tPhys[solid & on_base]
    off_t = tPhys[solid & ~on_base]
    return dict(
        passed=bool(base_t.size) and (earliest is None or earliest > 0),
        solid_base_elements=int(base_t.size),
        earliest_node_t=earliest,
        max_base_t=float(base_t.max()) if base_t.size else None,
        earliest_off_base_t=float(off_t.min()) if off_t.size else None,
    )


def warn_start(start: dict) -> None:
    """Warns that a ``start_report`` failed (sttopt/virtual_heat.py:393-398)."""
    import warnings

    warnings.warn(f"print start: {start['solid_base_elements']} solid base element(s), and the earliest node of "
                  f"the part off the plate at t = {start['earliest_node_t']} (must be > 0)")


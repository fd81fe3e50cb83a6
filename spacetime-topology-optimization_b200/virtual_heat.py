"""Drop-in for the solve path of ``sttopt.virtual_heat``: the scalar Q4 mesh and the
virtual-heat time field (sttopt/virtual_heat.py:82-108,162-201,205-288,404-462).

``heat_time_field`` solves ``-div(chi grad T) + alpha T = 0`` with ``T = 1`` on the
build plate through ``lifted_femsolve`` (device hierarchy with the lumped drain,
device PCG, adjoint kernels), then maps ``T`` to ``t`` (``one_minus`` or ``neg_log``),
takes element means and normalises over the part.  The ``poisson`` map and the
Laplace variant are not part of this package.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import NamedTuple

import numpy as np
import torch
from torch import Tensor

from . import fem, torch_solve

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


def element_means(u: Tensor, edof: Tensor) -> Tensor:
    """Mean of each element's four nodal values (sttopt/virtual_heat.py:162-166)."""
    return u[..., edof].mean(dim=-1)


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
    plate: Tensor
    active: Tensor

    @classmethod
    def build(cls, nelx: int, nely: int, print_base: str, device, dtype,
              active: np.ndarray | None = None) -> "ScalarMesh":
        active = np.ones((nely, nelx), bool) if active is None else active
        return cls(
            nelx=nelx, nely=nely,
            edof=torch.as_tensor(fem.element_dof_map(nelx, nely, 1), device=device, dtype=torch.int64),
            KE=torch.as_tensor(fem.diffusion_KE(), device=device, dtype=dtype),
            plate=torch.as_tensor(plate_nodes(nelx, nely, print_base, active), device=device),
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
        penalized = torch.clamp(xPhys.flatten() ** conduction_penal, min=DENSITY_FLOOR)
    else:
        penalized = torch.ones_like(xPhys.flatten())
    chi = penalized * diffusivity(mu.flatten(), config.chi_contrast)
    alpha = config.drain_beta / mesh.unit_length**2
    T = mesh.solve(chi, mesh.plate.to(chi.dtype), mesh.plate, config.heat_cg_rtol,
                   reaction=torch.full_like(chi, alpha),
                   x0=None if previous is None else previous.primary, precision=precision)
    time_map = str(getattr(config.time_map, "value", config.time_map))
    if time_map == "one_minus":
        t = 1 - T
    elif time_map == "neg_log":
        with torch.no_grad():
            part = part_mask(xPhys).flatten()
            floor = NEG_LOG_FLOOR * element_means(T, mesh.edof)[part].min()
        t = -torch.log(torch.clamp(T, min=0) + floor)
    else:
        raise ValueError(f"time_map {time_map!r} is not supported here (one_minus, neg_log)")
    t_e = element_means(t, mesh.edof).reshape(shape)
    return TimeFieldSolution(normalize(t_e, xPhys), T, None, t)

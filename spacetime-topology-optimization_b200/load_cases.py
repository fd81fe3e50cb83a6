"""Drop-in for ``sttopt.load_cases``: the nodal force vector and free dofs of each
structural load case (sttopt/load_cases.py:18-149), plus the two boundary conditions of
the benchmark configurations that the reference forms by hand (config 2's mid-right
cantilever load, the clamped build plate of the space-time stages).

Host NumPy set-up code, run once per problem; the outputs feed ``torch_fem.free_mask``
and the solves.  Lengths are in metres and converted to elements through
``in_elements``; loads are spread over their span by ``fem.edge_load_shares``.
Positions follow the mesh convention of ``fem.node_grid`` (row 0 at the top).
"""

from __future__ import annotations

import math
import sys
from enum import StrEnum

import numpy as np

from . import fem

# a quotient of decimal lengths that is meant as a whole number of elements lands within
# a few ulps of it (sttopt/units.py:12-15)
LENGTH_RTOL = 4 * sys.float_info.epsilon


def in_elements(length_m: float, element_size_m: float) -> float:
    """``length_m / element_size_m``, snapped to the whole number it is within a few ulps
    of (sttopt/units.py:18-33)."""
    n = length_m / element_size_m
    k = round(n)
    return float(k) if math.isclose(n, k, rel_tol=LENGTH_RTOL) else n


class LoadCase(StrEnum):
    """The reference's named cases (sttopt/load_cases.py:18-42)."""

    CANTILEVER = "cantilever"
    CORNER_LOADS = "corner_loads"
    EDGE_TRACTION = "edge_traction"
    MBB = "mbb"
    L_BRACKET_CORNER = "l_bracket_corner"
    L_BRACKET_MIDDLE = "l_bracket_middle"


def _both_dofs(nodes: np.ndarray) -> np.ndarray:
    nodes = np.asarray(nodes)
    return np.column_stack([2 * nodes, 2 * nodes + 1]).reshape(-1)


def _span_nodes(edge: np.ndarray, centre: float, length: float) -> np.ndarray:
    """Nodes of ``edge`` (ordered) within ``[centre - length/2, centre + length/2]``
    elements of its first node, a node on either end kept against round-off
    (sttopt/load_cases.py:47-68)."""
    lo, hi = centre - 0.5 * length, centre + 0.5 * length
    last = edge.size - 1
    if lo < 0 or hi > last:
        raise ValueError(f"a support patch over [{lo}, {hi}] elements does not fit on an edge of {last} elements")
    at = np.arange(edge.size)
    keep = (at >= lo - 1e-9) & (at <= hi + 1e-9)
    if not keep.any():
        raise ValueError(f"a support patch over [{lo}, {hi}] elements holds no node; lengthen support_length_m")
    return edge[keep]


def _require_even(nelx: int, nely: int) -> None:
    if nelx % 2 or nely % 2:
        raise ValueError(f"an L bracket needs even nelx and nely to split into quarters, got {nelx} x {nely}")


def load_case(case: LoadCase, nelx: int, nely: int, load_length_m: float, support_length_m: float,
              element_size_m: float) -> tuple[np.ndarray, np.ndarray]:
    """``(F, freedofs)`` of ``case`` on an ``nelx x nely`` mesh (sttopt/load_cases.py:74-130):
    ``F`` the nodal forces (``ndof``,), ``freedofs`` the sorted free dof indices."""
    case = LoadCase(case)
    grid = fem.node_grid(nelx, nely)
    F = np.zeros(2 * grid.size)
    span = in_elements(load_length_m, element_size_m)
    right_top_down = grid[:, -1]
    right_bottom_up = right_top_down[::-1]
    left_bottom_up = grid[::-1, 0]
    if case is LoadCase.CANTILEVER:
        F[2 * right_bottom_up + 1] = -fem.edge_load_shares(nely + 1, span)
        fixed = _both_dofs(left_bottom_up)
    elif case is LoadCase.CORNER_LOADS:
        w = fem.edge_load_shares(nely + 1, span) / math.sqrt(2.0)
        np.add.at(F, 2 * right_top_down, w)
        np.add.at(F, 2 * right_top_down + 1, -w)
        np.add.at(F, 2 * right_bottom_up, -w)
        np.add.at(F, 2 * right_bottom_up + 1, -w)
        fixed = _both_dofs(left_bottom_up)
    elif case is LoadCase.EDGE_TRACTION:
        F[2 * right_bottom_up] = fem.edge_load_shares(nely + 1, nely)
        sup = in_elements(support_length_m, element_size_m)
        fixed = _both_dofs(np.concatenate([_span_nodes(left_bottom_up, 0.25 * nely, sup),
                                           _span_nodes(left_bottom_up, 0.80 * nely, sup),
                                           _span_nodes(grid[-1, :], 0.30 * nelx, sup)]))
    elif case is LoadCase.MBB:
        F[2 * grid[0, :] + 1] = -fem.edge_load_shares(nelx + 1, span)
        sup = in_elements(support_length_m, element_size_m)
        roller = _span_nodes(grid[-1, ::-1], sup / 2, sup)
        fixed = np.concatenate([2 * left_bottom_up, 2 * roller + 1])
    else:  # the two L brackets
        _require_even(nelx, nely)
        col = 0 if case is LoadCase.L_BRACKET_CORNER else nelx // 2
        F[2 * grid[:nely // 2 + 1, col]] = fem.edge_load_shares(nely // 2 + 1, span)
        fixed = _both_dofs(grid[nely // 2:, -1])
    return F, np.setdiff1d(np.arange(F.size), fixed)


def active_mask(case: LoadCase, nelx: int, nely: int) -> np.ndarray:
    """Elements that may hold material (sttopt/load_cases.py:141-149): all of them, but
    the top-right quarter of an L bracket."""
    case = LoadCase(case)
    act = np.ones((nely, nelx), dtype=bool)
    if case in (LoadCase.L_BRACKET_CORNER, LoadCase.L_BRACKET_MIDDLE):
        _require_even(nelx, nely)
        act[:nely // 2, nelx // 2:] = False
    return act


def mid_right_cantilever(nelx: int, nely: int) -> tuple[np.ndarray, np.ndarray]:
    """Config 2's case: the left edge clamped, a unit downward point load at the
    right-edge node ``node_grid[nely // 2, -1]``.  ``(F, freedofs)``."""
    grid = fem.node_grid(nelx, nely)
    F = np.zeros(2 * grid.size)
    F[2 * grid[nely // 2, -1] + 1] = -1.0
    return F, np.setdiff1d(np.arange(F.size), _both_dofs(grid[:, 0]))


def build_plate_clamp(nelx: int, nely: int) -> tuple[np.ndarray, np.ndarray]:
    """The space-time stages' support: both dofs of the bottom node row (the build
    plate) fixed, no point load.  ``(F, freedofs)``."""
    grid = fem.node_grid(nelx, nely)
    F = np.zeros(2 * grid.size)
    return F, np.setdiff1d(np.arange(F.size), _both_dofs(grid[-1, :]))


__all__ = ["LoadCase", "load_case", "active_mask", "in_elements", "mid_right_cantilever", "build_plate_clamp"]

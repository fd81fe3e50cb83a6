"""Mesh set-up of the structured Q4 grid (the reference's ``sttopt.fem`` conventions).

Nodes in C order ``row * (nelx + 1) + col`` with row 0 at the top; element dofs in
local corner order bottom-left, bottom-right, top-right, top-left, ``d`` interleaved
dofs per node (sttopt/fem.py:60-95).  The element matrices are the closed forms of
sttopt/fem.py:17-30 (plane stress) and :98-111 (scalar diffusion).
"""

from __future__ import annotations

import numpy as np


def plane_stress_KE(nu: float) -> np.ndarray:
    """Unit-square bilinear plane-stress element matrix ``(A + nu B) / (1 - nu^2) / 24``."""
    a11 = np.array([[12, 3, -6, -3], [3, 12, 3, 0], [-6, 3, 12, -3], [-3, 0, -3, 12]])
    a12 = np.array([[-6, -3, 0, 3], [-3, -6, -3, -6], [0, -3, -6, 3], [3, -6, 3, -6]])
    b11 = np.array([[-4, 3, -2, 9], [3, -4, -9, 4], [-2, -9, -4, -3], [9, 4, -3, -4]])
    b12 = np.array([[2, -3, 4, -9], [-3, 2, 9, -2], [4, 9, 2, 3], [-9, -2, 3, 2]])
    A = np.block([[a11, a12], [a12.T, a11]])
    B = np.block([[b11, b12], [b12.T, b11]])
    return (A + nu * B) / (1 - nu**2) / 24


def diffusion_KE() -> np.ndarray:
    """Element matrix of ``-div grad`` on a unit-square bilinear quad."""
    return np.array(
        [[4, -1, -2, -1], [-1, 4, -1, -2], [-2, -1, 4, -1], [-1, -2, -1, 4]], dtype=np.float64
    ) / 6


def edge_load_shares(n_nodes: int, length: float) -> np.ndarray:
    """Each edge node's share of a unit force spread uniformly over ``[0, length]``
    elements from the edge's first node (sttopt/fem.py:33-57): the exact integral of the
    node's hat function over the span, divided by the span, so the shares sum to 1;
    ``length == 0`` is a point load on the first node."""
    if not 0 <= length <= n_nodes - 1:
        raise ValueError(f"a traction over {length} elements does not fit on an edge of {n_nodes - 1} elements")
    if length == 0:
        shares = np.zeros(n_nodes)
        shares[0] = 1.0
        return shares

    def cumulative_hat(u):
        # integral of the unit hat (support [-1, 1]) from -inf to u
        u = np.clip(u, -1.0, 1.0)
        return np.where(u < 0, 0.5 * (1.0 + u) ** 2, 1.0 - 0.5 * (1.0 - u) ** 2)

    at = np.arange(n_nodes, dtype=np.float64)
    return (cumulative_hat(length - at) - cumulative_hat(-at)) / length


def node_grid(nelx: int, nely: int) -> np.ndarray:
    return np.arange((nely + 1) * (nelx + 1)).reshape(nely + 1, nelx + 1)


def element_dof_map(nelx: int, nely: int, dofs_per_node: int = 2) -> np.ndarray:
    nodes = node_grid(nelx, nely)
    corners = np.stack(
        [nodes[1:, :-1], nodes[1:, 1:], nodes[:-1, 1:], nodes[:-1, :-1]], axis=-1
    ).reshape(-1, 4)
    d = dofs_per_node
    return np.stack([d * corners + i for i in range(d)], axis=-1).reshape(-1, 4 * d)

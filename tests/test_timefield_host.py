"""Host logic of the time fields and the stage glue against the reference's outputs
(golden fixtures): the wall arc of the Laplace variant (boundary order, bit-exact), the
plate nodes, the Gauss-point shape gradients and the gravity load matrix's explicit
form.  No GPU."""

import numpy as np

from conftest import golden


def test_wall_arcs_and_plates_bit_exact(pkg):
    from sttopt_b200 import virtual_heat as vh

    g = golden("time_maps")
    for base in ("bottom_edge", "left_edge", "right_edge"):
        np.testing.assert_array_equal(vh.wall_arc(13, 7, base), g[f"arc_rect_{base}"])
        np.testing.assert_array_equal(vh.wall_arc(12, 8, base, g["lshape"]), g[f"arc_L_{base}"])
        np.testing.assert_array_equal(vh.plate_nodes(12, 8, base, g["lshape"]), g[f"plate_L_{base}"])
    for k in g:
        if k.startswith("lap_") and k.endswith("_arc"):
            nelx, nely = (int(v) for v in k.split("_")[1].split("x"))
            base = "left_edge" if "left_edge" in k else "bottom_edge"
            np.testing.assert_array_equal(vh.wall_arc(nelx, nely, base), g[k])


def test_boundary_loop_rejects_two_pieces(pkg):
    import pytest

    from sttopt_b200 import virtual_heat as vh

    active = np.ones((4, 6), bool)
    active[:, 3] = False
    with pytest.raises(ValueError):
        vh.wall_arc(6, 4, "bottom_edge", active)


def test_shape_gradients_sum_to_zero_and_reproduce_linears(pkg):
    from sttopt_b200 import virtual_heat as vh

    B = vh.shape_gradients()
    assert B.shape == (4, 2, 4)
    np.testing.assert_allclose(B.sum(axis=-1), 0.0, atol=1e-15)
    # u = x + 2y at the corners BL (0,0), BR (1,0), TR (1,1), TL (0,1): grad = (1, 2)
    u = np.array([0.0, 1.0, 3.0, 2.0])
    np.testing.assert_allclose(B @ u, np.tile([1.0, 2.0], (4, 1)), atol=1e-15)


def test_gravity_matrix_explicit_form(pkg):
    from sttopt_b200 import gravity

    g = golden("compliance_smooth")
    C = gravity.gravity_load_matrix(7, 4)
    assert C.shape == (40, 28)
    np.testing.assert_array_equal(C.tocsr().toarray(), g["C_7x4"])
    np.testing.assert_array_equal(C.T.tocsr().toarray(), g["C_7x4"].T)


def test_wall_filter_distance_wall_and_start_report(pkg):
    import torch

    from sttopt_b200 import virtual_heat as vh

    g = golden("time_maps")
    for n_arc, rmin in [(30, 1.0), (30, 3.5), (45, 6.0), (5, 8.0)]:
        np.testing.assert_allclose(vh.wall_filter(n_arc, rmin), g[f"wf_{n_arc}_{rmin}"], rtol=0, atol=1e-15)
    for key, (nx, ny, base, act) in {"rect": (13, 7, "bottom_edge", None), "L": (12, 8, "left_edge", g["lshape"]),
                                     "Lb": (12, 8, "bottom_edge", g["lshape"])}.items():
        mesh = vh.ScalarMesh.build(nx, ny, base, torch.device("cpu"), torch.float64, act)
        np.testing.assert_allclose(vh.distance_wall(mesh).numpy(), g[f"dw_{key}"], rtol=1e-14, atol=0)
    mesh = vh.ScalarMesh.build(10, 6, "bottom_edge", torch.device("cpu"), torch.float64)
    t_nodes = torch.as_tensor(g["sr_t"])
    sol = vh.TimeFieldSolution(torch.as_tensor(g["sr_tPhys"]), t_nodes, None, t_nodes)
    rep = vh.start_report(mesh, sol, g["sr_solid"], g["sr_base"])
    assert repr(sorted(rep.items())) == str(g["sr_report"])
    import warnings

    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        vh.warn_start(rep)
    assert len(w) == 1 and "print start" in str(w[0].message)

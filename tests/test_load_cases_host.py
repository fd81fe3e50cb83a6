"""The package's load cases against the reference's (golden fixture made by running
``sttopt.load_cases`` and ``sttopt.fem.edge_load_shares``): every case on three meshes
and span pairs, bit-exact free dofs and active masks, forces to 1e-15 (host NumPy, no
GPU)."""

import numpy as np
import pytest

from conftest import golden

CASES = ["cantilever", "corner_loads", "edge_traction", "mbb", "l_bracket_corner", "l_bracket_middle"]
MESHES = [(12, 8, 0.0, 0.5, 0.25), (20, 10, 0.4, 0.3, 0.1), (16, 12, 0.27, 0.13, 0.05)]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("mesh", MESHES)
def test_load_case_matches_reference(pkg, case, mesh):
    from sttopt_b200 import load_cases

    g = golden("load_cases")
    nelx, nely, load_m, sup_m, h = mesh
    k = f"{case}_{nelx}x{nely}_{load_m}_{sup_m}_{h}"
    F, free = load_cases.load_case(load_cases.LoadCase(case), nelx, nely, load_m, sup_m, h)
    np.testing.assert_array_equal(free, g[f"{k}_free"])
    np.testing.assert_allclose(F, g[f"{k}_F"], rtol=0, atol=1e-15)
    np.testing.assert_array_equal(load_cases.active_mask(case, nelx, nely), g[f"{k}_active"])


def test_edge_load_shares_and_lengths(pkg):
    from sttopt_b200 import fem, load_cases

    g = golden("load_cases")
    for n, length in [(5, 0.0), (5, 1.0), (9, 2.5), (9, 8.0), (33, 7.3)]:
        s = fem.edge_load_shares(n, length)
        np.testing.assert_allclose(s, g[f"shares_{n}_{length}"], rtol=0, atol=1e-15)
        assert abs(s.sum() - 1.0) < 1e-14
    got = [load_cases.in_elements(a, b) for a, b in [(0.3, 0.1), (1.0, 0.25), (0.35, 0.1), (0.7, 0.1), (1.0, 0.3)]]
    np.testing.assert_array_equal(np.array(got), g["in_elements"])
    with pytest.raises(ValueError):
        fem.edge_load_shares(4, 3.5)
    with pytest.raises(ValueError):
        load_cases.load_case("l_bracket_corner", 11, 8, 0.0, 0.0, 1.0)


def test_config_boundary_conditions(pkg):
    """Config 1 is the reference's MBB case with zero spans; config 2's mid-right load and
    the build-plate clamp are the hand-formed cases of the benchmark configurations."""
    from oracle import sttopt_oracle as O
    from sttopt_b200 import load_cases

    F, free = load_cases.load_case("mbb", 120, 40, 0.0, 0.0, 1.0)
    F_o, mask_o = O.mbb_point_load(120, 40)
    np.testing.assert_array_equal(F, F_o)
    np.testing.assert_array_equal(free, np.flatnonzero(mask_o))
    F, free = load_cases.mid_right_cantilever(64, 32)
    F_o, mask_o = O.mid_right_cantilever(64, 32)
    np.testing.assert_array_equal(F, F_o)
    np.testing.assert_array_equal(free, np.flatnonzero(mask_o))
    F, free = load_cases.build_plate_clamp(24, 12)
    assert not F.any()
    np.testing.assert_array_equal(free, np.flatnonzero(O.bottom_clamped_mask(24, 12)))

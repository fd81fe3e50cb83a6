"""The CPU oracle against the reference's own outputs (golden fixtures).

These pin the oracle: every later GPU parity test compares the CUDA path with the
oracle, so the oracle itself is first shown to reproduce the reference.
"""

import numpy as np
import pytest

from conftest import golden, rel_err
from oracle import sttopt_oracle as O

EMIN, EMAX, PENAL = 1e-9, 1.0, 3.0


def test_mesh_setup_bit_exact():
    g = golden("fem_basic")
    np.testing.assert_array_equal(O.plane_stress_KE(0.3), g["KE"])
    np.testing.assert_array_equal(O.plane_stress_KE(0.0), g["KE_nu0"])
    np.testing.assert_array_equal(O.diffusion_KE(), g["KEh"])
    np.testing.assert_array_equal(O.element_dof_map(5, 3, 2), g["edof_5x3_d2"])
    np.testing.assert_array_equal(O.element_dof_map(5, 3, 1), g["edof_5x3_d1"])
    np.testing.assert_array_equal(O.element_dof_map(7, 4, 2), g["edof_7x4_d2"])
    F, mask = O.mbb_point_load(12, 4)
    np.testing.assert_array_equal(F, g["mbb_F"])
    np.testing.assert_array_equal(np.flatnonzero(mask), g["mbb_free"])
    F, mask = O.cantilever_point_load(12, 4)
    np.testing.assert_array_equal(F, g["cant_F"])
    np.testing.assert_array_equal(np.flatnonzero(mask), g["cant_free"])
    np.testing.assert_array_equal(O.plate_nodes(6, 4, "bottom_edge"), g["plate_bottom_6x4"])
    np.testing.assert_array_equal(O.plate_nodes(6, 4, "left_edge"), g["plate_left_6x4"])
    sizes = [(180, 60), (45, 15), (15, 5), (5, 5), (2048, 1024), (120, 40), (30, 10), (7, 9),
             (6, 9), (768, 384)]
    np.testing.assert_array_equal(np.array([O.coarsening_factors(a, b) for a, b in sizes]),
                                  g["coarsen"])


def test_gravity_load_matches_reference_matrix():
    g = golden("fem_basic")
    C = g["gravity_C"]
    rng = np.random.default_rng(0)
    xt = rng.uniform(0, 1, 24)
    F = O.gravity_load(xt[None], 6, 4)[0]
    np.testing.assert_allclose(F[1::2], -(C @ xt), rtol=1e-14, atol=1e-16)
    assert np.all(F[0::2] == 0)


def test_operator_applies():
    g = golden("operator")
    nelx, nely = 12, 8
    ndof = 2 * 13 * 9
    edof = O.element_dof_map(nelx, nely)
    KE = O.plane_stress_KE(0.3)
    dens = O.simp_density(g["x"], EMIN, EMAX, PENAL)
    np.testing.assert_allclose(dens, g["dens"], rtol=1e-15)
    np.testing.assert_allclose(O.matvec(g["U"], dens, edof, KE, ndof), g["matvec"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(O.matvec(g["U"], dens[0], edof, KE, ndof), g["matvec_bcast"],
                               rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(O.matvec_diagonal(dens, edof, KE, ndof), g["diag"], rtol=1e-13)
    np.testing.assert_allclose(O.operator(g["U"], dens, edof, KE, ndof, g["mask"]), g["op"],
                               rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(O.jacobi_preconditioner_diag(dens, edof, KE, ndof, g["mask"]),
                               g["jdiag"], rtol=1e-13)
    hedof = O.element_dof_map(9, 7, 1)
    KEh = O.diffusion_KE()
    rd = O.lumped_reaction(g["h_reac"], hedof, 80)
    np.testing.assert_allclose(rd, g["h_rdiag"], rtol=1e-14)
    np.testing.assert_allclose(O.operator(g["h_U"], g["h_chi"], hedof, KEh, 80, g["h_mask"], rd),
                               g["h_op"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(
        O.jacobi_preconditioner_diag(g["h_chi"], hedof, KEh, 80, g["h_mask"], rd), g["h_jdiag"],
        rtol=1e-13)


@pytest.mark.parametrize("kx,ky", [(2, 2), (3, 3), (3, 1), (2, 3), (1, 2)])
@pytest.mark.parametrize("d", [1, 2])
def test_transfers(kx, ky, d):
    g = golden("transfers")
    key = f"k{kx}{ky}_d{d}"
    P = O.on_node_grid(g[f"c_{key}"], 4, 3, kx, ky, O.interp_axis)
    R = O.on_node_grid(g[f"f_{key}"], 3 * kx + 1, 2 * ky + 1, kx, ky, O.restrict_axis)
    np.testing.assert_allclose(P, g[f"P_{key}"], rtol=1e-15, atol=1e-15)
    np.testing.assert_allclose(R, g[f"R_{key}"], rtol=1e-14, atol=1e-15)
    np.testing.assert_array_equal(O.child_interpolation_matrices(kx, ky, d), g[f"S_{key}"])
    np.testing.assert_array_equal(O.child_elements(6 * kx, 2 * ky, kx, ky), g[f"children_{kx}{ky}"])


def test_hierarchy_and_vcycle_vector():
    g = golden("hierarchy")
    nelx, nely = 24, 18
    x = g["v_x"]
    dens = O.simp_density(x, EMIN, EMAX, PENAL)
    edof = O.element_dof_map(nelx, nely)
    KE = O.plane_stress_KE(0.3)
    levels = O.build_hierarchy(dens, edof, KE, g["v_mask"], nelx, nely, max_coarse_elements=10)
    assert len(levels) == int(g["v_nlevels"])
    for i, lv in enumerate(levels):
        np.testing.assert_array_equal([lv.nelx, lv.nely, lv.kx, lv.ky], g[f"v_L{i}_shape"])
        np.testing.assert_array_equal(lv.mask, g[f"v_L{i}_mask"])
        np.testing.assert_allclose(lv.diag, g[f"v_L{i}_diag"], rtol=1e-12)
        if lv.keff is not None:
            assert rel_err(lv.keff, g[f"v_L{i}_keff"]) < 1e-13
    assert rel_err(levels[-1].chol, g["v_chol"]) < 1e-12
    M = O.VCycle(levels)
    assert rel_err(levels[0](g["v_r"]), g["v_Ar"]) < 1e-13
    assert rel_err(M(g["v_r"]), g["v_Mr"]) < 1e-10


def test_hierarchy_and_vcycle_scalar_with_reaction():
    g = golden("hierarchy")
    hx, hy = 18, 12
    edof = O.element_dof_map(hx, hy, 1)
    mask = ~O.plate_nodes(hx, hy, "bottom_edge")
    reac = np.full(hx * hy, 25.0 / (hx * hy))
    levels = O.build_hierarchy(g["h_chi"], edof, O.diffusion_KE(), mask, hx, hy, reaction=reac,
                               max_coarse_elements=10)
    assert len(levels) == int(g["h_nlevels"])
    for i, lv in enumerate(levels):
        np.testing.assert_array_equal([lv.nelx, lv.nely, lv.kx, lv.ky], g[f"h_L{i}_shape"])
        np.testing.assert_array_equal(lv.mask, g[f"h_L{i}_mask"])
        np.testing.assert_allclose(lv.diag, g[f"h_L{i}_diag"], rtol=1e-12)
        if lv.keff is not None:
            assert rel_err(lv.keff, g[f"h_L{i}_keff"]) < 1e-13
    assert rel_err(levels[-1].chol, g["h_chol"]) < 1e-12
    assert rel_err(O.VCycle(levels)(g["h_r"]), g["h_Mr"]) < 1e-10


def test_pcg_retirement_zero_row_and_nonconvergence():
    g = golden("pcg_cases")
    nelx, nely = 18, 12
    edof = O.element_dof_map(nelx, nely)
    KE = O.plane_stress_KE(0.3)
    info = {}
    U, n = O.mg_solve(g["F"], g["x"], edof, KE, EMIN, EMAX, PENAL, g["mask"], nelx, nely,
                      rtol=1e-11, max_coarse_elements=24, info=info)
    assert n == int(g["n_iter"])
    assert info["row_iters"] == int(g["row_iters"])
    assert np.all(U[1] == 0.0)
    for s in (0, 2):
        assert rel_err(U[s], g["U"][s]) < 1e-9
    with pytest.raises(O.CGConvergenceError) as e:
        O.mg_solve(g["F"], g["x"], edof, KE, EMIN, EMAX, PENAL, g["mask"], nelx, nely,
                   rtol=1e-14, max_iter=2, max_coarse_elements=24)
    assert str(e.value) == str(g["fail_msg"])
    np.testing.assert_allclose(e.value.residuals, g["fail_resid"], rtol=1e-6)


def test_mbb_120x40_config():
    g = golden("mbb120x40")
    nelx, nely = 120, 40
    F, mask = O.mbb_point_load(nelx, nely)
    np.testing.assert_array_equal(F, g["F"])
    np.testing.assert_array_equal(mask, g["mask"])
    KE = O.plane_stress_KE(0.3)
    edof = O.element_dof_map(nelx, nely)
    x = np.full(nelx * nely, 0.5)
    dens = O.simp_density(x, EMIN, EMAX, PENAL)
    solver = O.FemSolveOracle(dens, F, edof, KE, mask, nelx, nely)
    assert solver.forward_n_iter == int(g["forward_n_iter"])
    assert [[lv.nelx, lv.nely] for lv in solver.levels] == g["level_shapes"].tolist()
    assert solver.levels[-1].ndof == int(g["coarse_ndof"])
    assert rel_err(solver.U, g["U"]) < 1e-9
    ce = O.element_strain_energy(solver.U, edof, KE)
    c = float(np.sum(dens * ce))
    assert abs(c - float(g["c"])) / abs(float(g["c"])) < 1e-9
    gU = 2 * O.matvec(solver.U, dens, edof, KE, len(F))
    gd, _, _, n = solver.adjoint(gU)
    assert n == int(g["backward_n_iter"])
    dc = ((ce + gd) * PENAL * x ** (PENAL - 1) * (EMAX - EMIN)).reshape(nely, nelx)
    assert rel_err(dc, g["dc"]) < 1e-9


def test_cantilever_config_shape():
    g = golden("cantilever")
    for nelx, nely in [(64, 32), (96, 48)]:
        k = f"{nelx}x{nely}"
        x = O.smoothed_density(nelx, nely, 2 if nelx == 64 else 3)
        np.testing.assert_array_equal(x, g[f"{k}_x"])
        F, mask = O.mid_right_cantilever(nelx, nely)
        np.testing.assert_array_equal(F, g[f"{k}_F"])
        np.testing.assert_array_equal(mask, g[f"{k}_mask"])
        KE = O.plane_stress_KE(0.3)
        edof = O.element_dof_map(nelx, nely)
        dens = O.simp_density(x.ravel(), EMIN, EMAX, PENAL)
        solver = O.FemSolveOracle(dens, F, edof, KE, mask, nelx, nely,
                                  max_coarse_elements=int(g[f"{k}_mce"]))
        assert solver.forward_n_iter == int(g[f"{k}_fwd_iter"])
        assert rel_err(solver.U, g[f"{k}_U"]) < 1e-9
        ce = O.element_strain_energy(solver.U, edof, KE)
        c = float(np.sum(dens * ce))
        assert abs(c - float(g[f"{k}_c"])) / abs(float(g[f"{k}_c"])) < 1e-9
        gd, _, _, n = solver.adjoint(2 * O.matvec(solver.U, dens, edof, KE, len(F)))
        assert n == int(g[f"{k}_bwd_iter"])
        dc = ((ce + gd) * PENAL * x.ravel() ** (PENAL - 1)).reshape(nely, nelx)
        # sensitivities carry the (U.KU)/(U.F) factor of the adjoint warm start, which
        # two FP64 runs converged to rtol 1e-8 reproduce to about 1e-9
        assert rel_err(dc, g[f"{k}_dc"]) < 5e-9


@pytest.mark.parametrize("nelx,nely,seed", [(40, 20, 4), (60, 30, 5)])
def test_heat_time_field_and_adjoint(nelx, nely, seed):
    g = golden("heat")
    k = f"{nelx}x{nely}"
    out = O.heat_time_field(g[f"{k}_x"], g[f"{k}_mu"], conduction_penal=3.0, want_adjoint=g[f"{k}_w"])
    assert rel_err(out["T"], g[f"{k}_T"]) < 1e-9
    assert rel_err(out["tPhys"], g[f"{k}_tPhys"]) < 1e-9
    J = float(np.sum(g[f"{k}_w"] * out["tPhys"]))
    assert abs(J - float(g[f"{k}_J"])) <= 1e-9 * abs(float(g[f"{k}_J"]))
    assert rel_err(out["grad_x"], g[f"{k}_gx"]) < 1e-8
    assert rel_err(out["grad_mu"], g[f"{k}_gmu"]) < 1e-8


@pytest.mark.parametrize("nelx,nely,n_stage", [(48, 24, 4), (64, 32, 16)])
def test_spacetime_objective_and_gradient(nelx, nely, n_stage):
    g = golden("spacetime")
    k = f"{nelx}x{nely}s{n_stage}"
    out = O.spacetime_objective(g[f"{k}_x"], g[f"{k}_w"], n_stage=n_stage)
    np.testing.assert_array_equal(out["membership"], g[f"{k}_member"])
    assert rel_err(out["tPhys"], g[f"{k}_tPhys"]) < 1e-9
    assert rel_err(out["c_s"], g[f"{k}_c_s"]) < 1e-9
    assert abs(out["objective"] - float(g[f"{k}_L"])) <= 1e-9 * abs(float(g[f"{k}_L"]))
    assert rel_err(out["U"], g[f"{k}_U"]) < 1e-9
    assert rel_err(out["gradient"], g[f"{k}_grad"]) < 1e-8


def test_stage_membership_is_bit_exact_on_identical_tphys():
    g = golden("spacetime")
    for k, n_stage in [("48x24s4", 4), ("64x32s16", 16)]:
        np.testing.assert_array_equal(O.stage_membership(g[f"{k}_tPhys"], n_stage), g[f"{k}_member"])


@pytest.mark.parametrize("key", ["37x23r1.5", "37x23r2.5", "64x40r4.0", "20x11r8.0"])
def test_density_filter_and_projection_against_the_reference(key, pkg):
    """The oracle's cone filter / projection and the package's host-side filter (row
    sums, explicit matrix) against the reference's outputs."""
    from sttopt_b200 import filters

    g = golden("filters")
    nelx, nely = (int(v) for v in key.split("r")[0].split("x"))
    rmin = float(key.split("r")[1])
    H, Hs = O.density_filter(nelx, nely, rmin)
    np.testing.assert_allclose(Hs, g[f"{key}_Hs"], rtol=1e-15)
    xt = O.apply_density_filter(g[f"{key}_x"], H, Hs)
    np.testing.assert_allclose(xt, g[f"{key}_xTilde"], rtol=1e-14, atol=1e-15)
    for beta in (1.0, 8.0, float("inf")):
        np.testing.assert_allclose(O.heaviside_projection(xt, beta, 0.5), g[f"{key}_b{beta}_xPhys"],
                                   rtol=1e-13, atol=1e-14)
    Hb, Hsb = filters.density_filter(nelx, nely, rmin)
    np.testing.assert_allclose(Hsb, g[f"{key}_Hs"], rtol=1e-14)  # summation order differs
    assert (Hb.tocsr() != H).nnz == 0

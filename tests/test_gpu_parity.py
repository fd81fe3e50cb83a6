"""GPU parity: the CUDA path (through the C ABI and the drop-in modules) against the
CPU oracle and the reference's golden fixtures, on the same seeded inputs.

Tolerances: FP64 operator applies 1e-13 relative; hierarchy diagonals 1e-12; one V-cycle
1e-10; converged FP64 solves (rtol 1e-8) 1e-9 on U and compliance, 5e-9 on sensitivity
fields (two FP64 runs of the same algorithm converged to rtol 1e-8 agree to about 1e-9
there); mixed precision 1e-6 against the FP64 oracle.  Integer work (masks, coarsening,
stage membership) is compared bit-exactly.
"""

import numpy as np
import pytest
import torch

from conftest import golden, rel_err
from oracle import sttopt_oracle as O

pytestmark = pytest.mark.gpu
EMIN, EMAX, PENAL = 1e-9, 1.0, 3.0
DEV = "cuda"


def T(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=DEV)


@pytest.fixture(scope="module")
def m(pkg):
    from sttopt_b200 import compliance, spacetime, torch_fem, torch_mg, torch_solve, virtual_heat

    class M:
        pass

    mm = M()
    mm.fem, mm.mg, mm.solve, mm.vh, mm.comp, mm.st = torch_fem, torch_mg, torch_solve, virtual_heat, compliance, spacetime
    return mm


def test_operator_applies_fp64(m):
    g = golden("operator")
    nelx, nely, ndof = 12, 8, 2 * 13 * 9
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    dens, U, mask = T(g["dens"]), T(g["U"]), T(g["mask"], torch.bool)
    assert rel_err(m.fem.matvec(U, dens, edof, KE, ndof).cpu(), g["matvec"]) < 1e-13
    assert rel_err(m.fem.matvec(U, dens[0], edof, KE, ndof).cpu(), g["matvec_bcast"]) < 1e-13
    assert rel_err(m.fem.matvec_diagonal(dens, edof, KE, ndof).cpu(), g["diag"]) < 1e-14
    assert rel_err(m.fem.operator(U, dens, edof, KE, ndof, mask).cpu(), g["op"]) < 1e-13
    assert rel_err(m.fem.jacobi_preconditioner_diag(dens, edof, KE, ndof, mask).cpu(), g["jdiag"]) < 1e-14
    hedof, KEh = T(O.element_dof_map(9, 7, 1), torch.int64), T(O.diffusion_KE())
    rd = m.fem.lumped_reaction(T(g["h_reac"]), hedof, 80)
    assert rel_err(rd.cpu(), g["h_rdiag"]) < 1e-15
    hm = T(g["h_mask"], torch.bool)
    assert rel_err(m.fem.operator(T(g["h_U"]), T(g["h_chi"]), hedof, KEh, 80, hm, rd).cpu(), g["h_op"]) < 1e-13
    assert rel_err(m.fem.jacobi_preconditioner_diag(T(g["h_chi"]), hedof, KEh, 80, hm, rd).cpu(),
                   g["h_jdiag"]) < 1e-14
    # fixed dofs come back exactly zero (torch_fem.py:135-159)
    out = m.fem.operator(U, dens, edof, KE, ndof, mask).cpu().numpy()
    assert np.all(out[:, ~g["mask"]] == 0.0)


def test_operator_fp32_and_large_grid(m):
    rng = np.random.default_rng(3)
    nelx, nely = 257, 130  # ragged against the 32 x 8 tiles
    ndof = 2 * (nelx + 1) * (nely + 1)
    KE_np, edof_np = O.plane_stress_KE(0.3), O.element_dof_map(nelx, nely)
    x = rng.uniform(1e-3, 1, nelx * nely)
    dens = O.simp_density(x, EMIN, EMAX, PENAL)
    U = rng.standard_normal((2, ndof))
    ref = O.matvec(U, dens, edof_np, KE_np, ndof)
    KE, edof = T(KE_np), T(edof_np, torch.int64)
    got64 = m.fem.matvec(T(U), T(dens), edof, KE, ndof).cpu().numpy()
    assert rel_err(got64, ref) < 1e-13
    got32 = m.fem.matvec(T(U, torch.float32), T(dens, torch.float32), edof, KE, ndof).cpu().numpy()
    assert rel_err(got32, ref) < 1e-5


def _generic_KE():
    """A symmetric positive semi-definite element matrix outside the modal form (the
    library's generic path): plane stress plus a small seeded rank-one term."""
    v = np.random.default_rng(21).standard_normal(8)
    return O.plane_stress_KE(0.3) + 1e-3 * np.outer(v, v)


def test_generic_element_matrix_path(m, pkg):
    """A KE that stt_ke_modal rejects runs the generic 8 x 8 product: applies and a
    V-cycle still match the oracle at the plane-stress tolerances."""
    import ctypes

    from sttopt_b200 import _lib

    KE_np = _generic_KE()
    mm = (ctypes.c_double * 8)()
    assert _lib.lib().stt_ke_modal(2, _lib.dbl_array(KE_np.ravel().tolist()), mm) == 0
    rng = np.random.default_rng(11)
    nelx, nely = 67, 45
    ndof = 2 * (nelx + 1) * (nely + 1)
    edof_np = O.element_dof_map(nelx, nely)
    dens = O.simp_density(rng.uniform(1e-3, 1, nelx * nely), EMIN, EMAX, PENAL)
    U = rng.standard_normal((3, ndof))
    ref = O.matvec(U, dens, edof_np, KE_np, ndof)
    KE, edof = T(KE_np), T(edof_np, torch.int64)
    assert rel_err(m.fem.matvec(T(U), T(dens), edof, KE, ndof).cpu(), ref) < 1e-13
    got32 = m.fem.matvec(T(U, torch.float32), T(dens, torch.float32), edof, KE, ndof).cpu().numpy()
    assert rel_err(got32, ref) < 1e-5
    nelx, nely = 48, 36
    x = rng.uniform(1e-3, 1.0, nelx * nely)
    F, mask = O.cantilever_point_load(nelx, nely)
    dens = O.simp_density(x, EMIN, EMAX, PENAL)
    levels = m.mg.build_hierarchy(T(dens), T(O.element_dof_map(nelx, nely), torch.int64), KE,
                                  T(mask, torch.bool), nelx, nely, max_coarse_elements=20)
    ol = O.build_hierarchy(dens, O.element_dof_map(nelx, nely), KE_np, mask, nelx, nely,
                           max_coarse_elements=20)
    u = O.project(rng.standard_normal(len(F)), mask)
    assert rel_err(levels[0](T(u)).cpu(), ol[0](u)) < 1e-13
    assert rel_err(m.mg.VCycle(levels)(T(u)).cpu(), O.VCycle(ol)(u)) < 1e-10


def _levels(m, nelx, nely, x, mask, mce, precision="fp64"):
    dens = O.simp_density(x, EMIN, EMAX, PENAL)
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    return m.mg.build_hierarchy(T(dens), edof, KE, T(mask, torch.bool), nelx, nely,
                                max_coarse_elements=mce, precision=precision)


def test_hierarchy_matches_golden_levels(m):
    g = golden("hierarchy")
    nelx, nely = 24, 18
    levels = _levels(m, nelx, nely, g["v_x"], g["v_mask"], 10)
    assert len(levels) == int(g["v_nlevels"])
    for i, lv in enumerate(levels):
        assert [lv.nelx, lv.nely, lv.kx, lv.ky] == g[f"v_L{i}_shape"].tolist()
        np.testing.assert_array_equal(lv.mask.cpu().numpy(), g[f"v_L{i}_mask"])
        assert rel_err(lv.diag.cpu(), g[f"v_L{i}_diag"]) < 1e-12
    r = T(g["v_r"])
    assert rel_err(levels[0](r).cpu(), g["v_Ar"]) < 1e-13
    assert rel_err(m.mg.VCycle(levels)(r).cpu(), g["v_Mr"]) < 1e-10


def test_coarse_levels_are_exact_galerkin(m):
    """Every coarse apply equals R A P of the level above (torch_mg.py:355-370)."""
    g = golden("hierarchy")
    nelx, nely = 24, 18
    levels = _levels(m, nelx, nely, g["v_x"], g["v_mask"], 4)
    ol = O.build_hierarchy(O.simp_density(g["v_x"], EMIN, EMAX, PENAL), O.element_dof_map(nelx, nely),
                           O.plane_stress_KE(0.3), g["v_mask"], nelx, nely, max_coarse_elements=4)
    rng = np.random.default_rng(1)
    for i, (lv, olv) in enumerate(zip(levels, ol)):
        v = O.project(rng.standard_normal((2, lv.ndof)), olv.mask)
        assert rel_err(lv(T(v)).cpu(), olv(v)) < 1e-12, i


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_by_two_hierarchy_is_exact_galerkin(m, precision):
    """2 x 2 coarsening on every level (64x32 -> 4x2, five levels: level 1 from the
    densities, level 2 from its grandchildren, levels 3-4 by Galerkin products): every
    level's FP64 apply equals the oracle's R A P of the level above to 1e-12, and the
    mixed hierarchy's FP32 cycle the FP64 one to FP32 rounding."""
    rng = np.random.default_rng(17)
    nelx, nely = 64, 32
    x = rng.uniform(1e-3, 1.0, nelx * nely)
    F, mask = O.cantilever_point_load(nelx, nely)
    levels = _levels(m, nelx, nely, x, mask, 8, precision=precision)
    assert [(lv.nelx, lv.nely) for lv in levels] == [(64, 32), (32, 16), (16, 8), (8, 4), (4, 2)]
    ol = O.build_hierarchy(O.simp_density(x, EMIN, EMAX, PENAL), O.element_dof_map(nelx, nely),
                           O.plane_stress_KE(0.3), mask, nelx, nely, max_coarse_elements=8)
    for i, (lv, olv) in enumerate(zip(levels, ol)):
        v = O.project(rng.standard_normal((2, lv.ndof)), olv.mask)
        assert rel_err(lv(T(v)).cpu(), olv(v)) < 1e-12, i
    if precision == "mixed":
        M64 = m.mg.VCycle(_levels(m, nelx, nely, x, mask, 8))
        u = O.project(rng.standard_normal((2, len(F))), mask)
        assert rel_err(m.mg.VCycle(levels)(T(u)).cpu().numpy(), M64(T(u)).cpu().numpy()) < 1e-4


def test_scalar_hierarchy_with_reaction(m):
    g = golden("hierarchy")
    hx, hy = 18, 12
    mask = ~O.plate_nodes(hx, hy, "bottom_edge")
    reac = np.full(hx * hy, 25.0 / (hx * hy))
    levels = m.mg.build_hierarchy(T(g["h_chi"]), T(O.element_dof_map(hx, hy, 1), torch.int64),
                                  T(O.diffusion_KE()), T(mask, torch.bool), hx, hy, reaction=T(reac),
                                  max_coarse_elements=10)
    assert len(levels) == int(g["h_nlevels"])
    for i, lv in enumerate(levels):
        np.testing.assert_array_equal(lv.mask.cpu().numpy(), g[f"h_L{i}_mask"])
        assert rel_err(lv.diag.cpu(), g[f"h_L{i}_diag"]) < 1e-12
    assert rel_err(m.mg.VCycle(levels)(T(g["h_r"])).cpu(), g["h_Mr"]) < 1e-10


@pytest.mark.parametrize("gamma", [1, 2])
def test_vcycle_matches_oracle_and_is_spd(m, gamma):
    nelx, nely = 48, 36  # 2, 2, then 3 in each dimension
    rng = np.random.default_rng(5)
    x = rng.uniform(1e-3, 1.0, nelx * nely)
    F, mask = O.cantilever_point_load(nelx, nely)
    levels = _levels(m, nelx, nely, x, mask, 20)
    ol = O.build_hierarchy(O.simp_density(x, EMIN, EMAX, PENAL), O.element_dof_map(nelx, nely),
                           O.plane_stress_KE(0.3), mask, nelx, nely, max_coarse_elements=20)
    M, OM = m.mg.VCycle(levels, gamma=gamma), O.VCycle(ol, gamma=gamma)
    u = O.project(rng.standard_normal(len(F)), mask)
    v = O.project(rng.standard_normal(len(F)), mask)
    Mu, Mv = M(T(u)).cpu().numpy(), M(T(v)).cpu().numpy()
    assert rel_err(Mu, OM(u)) < 1e-10
    assert abs(Mu @ v - u @ Mv) <= 1e-10 * abs(Mu @ v)
    assert u @ Mu > 0
    assert np.all(Mu[~mask] == 0.0)


@pytest.mark.parametrize("nelx,nely,mce", [(64, 32, 700), (96, 48, 700), (48, 36, 20)])
def test_vcycle_fp32_matches_fp64(m, nelx, nely, mce):
    """The mixed-precision cycle (FP32 smoothing and transfers, the coarsest level solved
    by its explicit FP64 inverse) against the FP64 cycle (block Cholesky solves), on
    coarse matrices of band widths 32 and 64: agreement to FP32 rounding."""
    rng = np.random.default_rng(7)
    x = rng.uniform(1e-3, 1.0, nelx * nely)
    F, mask = O.cantilever_point_load(nelx, nely)
    M64 = m.mg.VCycle(_levels(m, nelx, nely, x, mask, mce))
    M32 = m.mg.VCycle(_levels(m, nelx, nely, x, mask, mce, precision="mixed"))
    u = O.project(rng.standard_normal((3, len(F))), mask)
    z64, z32 = M64(T(u)).cpu().numpy(), M32(T(u)).cpu().numpy()
    assert rel_err(z32, z64) < 1e-4
    # and the inverse is symmetric: M is symmetric to FP32 rounding
    v = O.project(rng.standard_normal(len(F)), mask)
    a, b = M32(T(u[0])).cpu().numpy() @ v, u[0] @ M32(T(v)).cpu().numpy()
    assert abs(a - b) <= 1e-4 * abs(a)


@pytest.mark.parametrize("n_smooth,gamma", [(1, 1), (3, 1), (2, 2)])
def test_vcycle_fp32_unchained_paths_match_fp64(m, n_smooth, gamma):
    """Sweep counts and W-cycles that the chained level-0 / level-1 passes do not take:
    the FP32 cycle runs the separate first sweep, sweeps and residuals, on a level 1 that
    keeps only its centre diagonal (swept from the level-0 densities); against the FP64
    cycle with the same n_smooth and gamma, to FP32 rounding."""
    rng = np.random.default_rng(11)
    nelx, nely = 128, 64
    x = rng.uniform(1e-3, 1.0, nelx * nely)
    F, mask = O.cantilever_point_load(nelx, nely)
    M64 = m.mg.VCycle(_levels(m, nelx, nely, x, mask, 700), n_smooth=n_smooth, gamma=gamma)
    M32 = m.mg.VCycle(_levels(m, nelx, nely, x, mask, 700, precision="mixed"), n_smooth=n_smooth, gamma=gamma)
    u = O.project(rng.standard_normal((3, len(F))), mask)
    z64, z32 = M64(T(u)).cpu().numpy(), M32(T(u)).cpu().numpy()
    assert rel_err(z32, z64) < 1e-4


def test_mixed_level1_fp64_stencil_assembled_on_first_use(m):
    """An FP32 hierarchy swept from the level-0 densities builds only level 1's FP32
    diagonal; its FP64 stencil is assembled by the first entry point that reads it (a
    view's apply first, then the parent's diagonal) and equals the FP64 hierarchy's."""
    rng = np.random.default_rng(13)
    nelx, nely, rows = 96, 48, 3
    x = rng.uniform(1e-3, 1.0, (rows, nelx * nely))
    F, mask = O.cantilever_point_load(nelx, nely)
    lv64, lv32 = (_levels(m, nelx, nely, x, mask, 300, precision=p) for p in ("fp64", "mixed"))
    assert len(lv32) > 2
    u = T(O.project(rng.standard_normal((rows, lv32[1].ndof)), lv32[1].mask.cpu().numpy()))
    sel = torch.tensor([2, 0], device=DEV)
    got = lv32[1].select(sel)(u[sel])
    assert rel_err(got.cpu().numpy(), lv64[1](u)[sel].cpu().numpy()) < 1e-13
    assert rel_err(lv32[1].diag.cpu().numpy(), lv64[1].diag.cpu().numpy()) < 1e-14
    assert rel_err(lv32[1](u).cpu().numpy(), lv64[1](u).cpu().numpy()) < 1e-13


@pytest.mark.parametrize("kx,ky,d", [(2, 2, 2), (3, 2, 2), (2, 3, 1), (3, 3, 1), (1, 2, 2)])
def test_grid_transfer_helpers_match_oracle_and_are_adjoint(m, kx, ky, d):
    """torch_mg._on_node_grid with _interp_axis / _restrict_axis (stt_grid_transfer) against
    the oracle's restatement, the 1-D helpers alone, and R = P^T (the reference's test)."""
    rng = np.random.default_rng(kx * 10 + ky + d)
    ncx, ncy = 5, 4
    cnnx, cnny, fnnx, fnny = ncx + 1, ncy + 1, ncx * kx + 1, ncy * ky + 1
    c = rng.standard_normal((3, d * cnnx * cnny))
    f = rng.standard_normal((3, d * fnnx * fnny))
    Pc = m.mg._on_node_grid(T(c), cnnx, cnny, kx, ky, m.mg._interp_axis).cpu().numpy()
    Rf = m.mg._on_node_grid(T(f), fnnx, fnny, kx, ky, m.mg._restrict_axis).cpu().numpy()
    assert rel_err(Pc, O.on_node_grid(c, cnnx, cnny, kx, ky, O.interp_axis)) < 1e-15
    assert rel_err(Rf, O.on_node_grid(f, fnnx, fnny, kx, ky, O.restrict_axis)) < 1e-15
    assert abs((Pc * f).sum() - (c * Rf).sum()) <= 1e-12 * abs((Pc * f).sum())
    a = rng.standard_normal((2, 3, 7))
    assert rel_err(m.mg._interp_axis(T(a), kx).cpu().numpy(), O.interp_axis(a, kx)) < 1e-15
    b = rng.standard_normal((2, 3, 6 * ky + 1))
    assert rel_err(m.mg._restrict_axis(T(b), ky).cpu().numpy(), O.restrict_axis(b, ky)) < 1e-15


@pytest.mark.parametrize("d", [2, 1])
def test_keff_matvec_matches_oracle(m, d):
    """torch_mg.keff_matvec (stt_keff_apply) with per-row and shared element matrices."""
    rng = np.random.default_rng(4 + d)
    nelx, nely = 9, 7
    nel, k = nelx * nely, 4 * d
    ndof = d * (nelx + 1) * (nely + 1)
    edof = O.element_dof_map(nelx, nely, d)
    keff = rng.standard_normal((2, nel, k, k))
    U = rng.standard_normal((2, ndof))
    got = m.mg.keff_matvec(T(U), T(keff), T(edof, torch.int64), ndof).cpu().numpy()
    assert rel_err(got, O.keff_matvec(U, keff, edof, ndof)) < 1e-14
    got1 = m.mg.keff_matvec(T(U), T(keff[0]), T(edof, torch.int64), ndof).cpu().numpy()
    assert rel_err(got1, O.keff_matvec(U, keff[0], edof, ndof)) < 1e-14


def test_vcycle_fp32_many_rows_uses_block_solves(m):
    """With more hierarchy rows than the coarse inverse is kept for, the FP32 cycle solves
    the coarsest level by the block-banded Cholesky solves: same agreement with FP64."""
    rng = np.random.default_rng(9)
    nelx, nely, rows = 64, 32, 50
    x = rng.uniform(1e-3, 1.0, (rows, nelx * nely))
    F, mask = O.cantilever_point_load(nelx, nely)
    dens = O.simp_density(x, EMIN, EMAX, PENAL)
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    lv = [m.mg.build_hierarchy(T(dens), edof, KE, T(mask, torch.bool), nelx, nely, precision=p)
          for p in ("fp64", "mixed")]
    u = O.project(rng.standard_normal((rows, len(F))), mask)
    z64, z32 = (m.mg.VCycle(levels)(T(u)).cpu().numpy() for levels in lv)
    assert rel_err(z32, z64) < 1e-4


def test_coarse_factorisation_failure_is_reported(m, pkg):
    """A coarse operator that is not positive definite (a negated KE): the default build
    raises at once; the unsynchronised build (check=False) raises at the first solve, also
    when the solve ends before its first V-cycle (a zero load)."""
    from sttopt_b200 import _lib

    nelx, nely = 24, 12
    F, mask = O.cantilever_point_load(nelx, nely)
    KE, edof = T(-O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    dens = T(np.full(nelx * nely, 0.5))
    with pytest.raises(_lib.SttError, match="positive definite"):
        m.mg.build_hierarchy(dens, edof, KE, T(mask, torch.bool), nelx, nely, max_coarse_elements=50)
    levels = m.mg.build_hierarchy(dens, edof, KE, T(mask, torch.bool), nelx, nely, max_coarse_elements=50,
                                  check=False)
    with pytest.raises(_lib.SttError, match="positive definite"):
        m.fem.pcg(levels[0], T(F), m.mg.VCycle(levels), rtol=1e-8, max_iter=5)
    levels = m.mg.build_hierarchy(dens, edof, KE, T(mask, torch.bool), nelx, nely, max_coarse_elements=50,
                                  check=False)
    with pytest.raises(_lib.SttError, match="positive definite"):
        m.fem.pcg(levels[0], T(np.zeros_like(F)), m.mg.VCycle(levels), rtol=1e-8, max_iter=5)


def test_mbb_config_solve_compliance_and_sensitivities(m):
    """120 x 40 MBB, rho = 0.5: U, iterations, compliance, dc/dx vs the reference."""
    g = golden("mbb120x40")
    nelx, nely = 120, 40
    F, mask = O.mbb_point_load(nelx, nely)
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    xPhys = torch.full((nely, nelx), 0.5, dtype=torch.float64, device=DEV, requires_grad=True)
    info = {}
    density = m.fem.simp_density(xPhys, EMIN, EMAX, PENAL).flatten()
    U = m.solve.femsolve(density, T(F), edof, KE, T(mask, torch.bool), nelx, nely, info=info)
    ce = m.comp._element_strain_energy(U, edof, KE, nely, nelx)
    c = torch.sum(m.fem.simp_density(xPhys, EMIN, EMAX, PENAL) * ce)
    (dc,) = torch.autograd.grad(c, [xPhys])
    assert info["forward_n_iter"] == int(g["forward_n_iter"])
    assert info["backward_n_iter"] == int(g["backward_n_iter"]) == 0
    assert rel_err(U.detach().cpu(), g["U"]) < 1e-9
    assert abs(float(c.detach()) - float(g["c"])) <= 1e-9 * abs(float(g["c"]))
    assert rel_err(dc.cpu(), g["dc"]) < 5e-9
    assert torch.all(U.detach()[~T(mask, torch.bool)] == 0.0)


def test_cantilever_config_shapes(m):
    g = golden("cantilever")
    for nelx, nely in [(64, 32), (96, 48)]:
        k = f"{nelx}x{nely}"
        KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
        xPhys = T(g[f"{k}_x"]).requires_grad_(True)
        info = {}
        density = m.fem.simp_density(xPhys, EMIN, EMAX, PENAL).flatten()
        U = m.solve.femsolve(density, T(g[f"{k}_F"]), edof, KE, T(g[f"{k}_mask"], torch.bool), nelx, nely,
                             info=info, max_coarse_elements=int(g[f"{k}_mce"]))
        ce = m.comp._element_strain_energy(U, edof, KE, nely, nelx)
        c = torch.sum(m.fem.simp_density(xPhys, EMIN, EMAX, PENAL) * ce)
        (dc,) = torch.autograd.grad(c, [xPhys])
        assert info["forward_n_iter"] == int(g[f"{k}_fwd_iter"])
        assert rel_err(U.detach().cpu(), g[f"{k}_U"]) < 1e-9
        assert abs(float(c.detach()) - float(g[f"{k}_c"])) <= 1e-9 * abs(float(g[f"{k}_c"]))
        assert rel_err(dc.cpu(), g[f"{k}_dc"]) < 5e-9


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_flexible_and_standard_beta_agree(m, precision):
    """The device PCG with the reference's beta (default), with the flexible beta
    (VCycle(flexible=True)) and with the true residual recomputed every 5 iterations
    (replace_every=5): all reach rtol on the true residual and take the same iterations
    as the default to within one; the mixed solves agree with an FP64 rtol-1e-12 solve to
    1e-6, and the FP64 ones with each other to 1e-10 (the cycle is symmetric up to its
    rounding, so the betas differ only there, and the FP64 recursive residual does not
    drift)."""
    rng = np.random.default_rng(21)
    nelx, nely, rows = 256, 128, 6
    F, mask = O.cantilever_point_load(nelx, nely)
    x = np.stack([O.smoothed_density(nelx, nely, 40 + k) for k in range(rows)]).reshape(rows, -1)
    dens = O.simp_density(x, EMIN, EMAX, PENAL)
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    Fr = T(np.tile(F, (rows, 1)) * rng.uniform(0.5, 2.0, (rows, 1)))
    ref_lv = m.mg.build_hierarchy(T(dens), edof, KE, T(mask, torch.bool), nelx, nely, precision="fp64")
    ref, _ = m.fem.pcg(ref_lv[0], Fr, m.mg.VCycle(ref_lv), rtol=1e-12, max_iter=400)
    lv = m.mg.build_hierarchy(T(dens), edof, KE, T(mask, torch.bool), nelx, nely, precision=precision)
    iters, sol = {}, {}
    for key in ("standard", "flexible", "replace"):
        M = m.mg.VCycle(lv, flexible=key == "flexible", replace_every=5 if key == "replace" else 0)
        U, n = m.fem.pcg(lv[0], Fr, M, rtol=1e-8, max_iter=400)
        res = (Fr - ref_lv[0](U)).norm(dim=1) / Fr.norm(dim=1)
        assert float(res.max()) <= 1.5e-8, (key, res)
        if precision == "mixed":
            err = float(((U - ref).norm(dim=1) / ref.norm(dim=1)).max())
            assert err < 1e-6, (key, err)
        iters[key], sol[key] = n, U
    assert abs(iters["flexible"] - iters["standard"]) <= 1 and abs(iters["replace"] - iters["standard"]) <= 1, iters
    if precision == "fp64":
        for key in ("flexible", "replace"):
            assert float(((sol[key] - sol["standard"]).norm(dim=1) / sol["standard"].norm(dim=1)).max()) < 1e-10


def test_retirement_zero_rows_and_nonconvergence(m):
    g = golden("pcg_cases")
    nelx, nely = 18, 12
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    info = {}
    U, n = m.mg.solve(T(g["F"]), T(g["x"]), edof, KE, EMIN, EMAX, PENAL, T(g["mask"], torch.bool), nelx,
                      nely, rtol=1e-11, max_coarse_elements=24, info=info)
    assert n == int(g["n_iter"])
    assert info["row_iters"] == int(g["row_iters"])
    assert torch.all(U[1] == 0.0)
    for s in (0, 2):
        assert rel_err(U[s].cpu(), g["U"][s]) < 1e-9
    with pytest.raises(m.fem.CGConvergenceError) as e:
        m.mg.solve(T(g["F"]), T(g["x"]), edof, KE, EMIN, EMAX, PENAL, T(g["mask"], torch.bool), nelx, nely,
                   rtol=1e-14, max_iter=2, max_coarse_elements=24)
    assert str(e.value) == str(g["fail_msg"])
    assert e.value.n_iter == 2


def test_warm_start_exact_solution_returns_unchanged(m):
    nelx, nely = 30, 10
    F, mask = O.cantilever_point_load(nelx, nely)
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    x = T(np.full(nelx * nely, 0.4))
    U, _ = m.mg.solve(T(F), x, edof, KE, EMIN, EMAX, PENAL, T(mask, torch.bool), nelx, nely, rtol=1e-10,
                      max_coarse_elements=24)
    U2, n = m.mg.solve(T(F), x, edof, KE, EMIN, EMAX, PENAL, T(mask, torch.bool), nelx, nely, rtol=1e-10,
                       x0=U, max_coarse_elements=24)
    assert n == 0 and torch.equal(U, U2)


def test_generic_pcg_with_selectable_wrappers(m):
    """Plain callables and counting wrappers go through the reference's loop."""
    nelx, nely = 18, 12
    g = golden("pcg_cases")
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    mask = T(g["mask"], torch.bool)
    dens = m.fem.simp_density(T(g["x"]), EMIN, EMAX, PENAL)
    levels = m.mg.build_hierarchy(dens, edof, KE, mask, nelx, nely, max_coarse_elements=24)
    log = []

    class Count:
        def __init__(self, op):
            self.op = op

        def __call__(self, v):
            log.append(v.shape[0])
            return self.op(v)

        def select(self, rows):
            return Count(self.op.select(rows))

    U, n = m.fem.pcg(Count(levels[0]), m.fem.project(T(g["F"]), mask), Count(m.mg.VCycle(levels)),
                     rtol=1e-11)
    assert n == int(g["n_iter"])
    assert log[0] == 3 and log[1] == 2  # the zero row retires before the first iteration
    assert rel_err(U[0].cpu(), g["U"][0]) < 1e-9


@pytest.mark.parametrize("nelx,nely", [(40, 20), (60, 30)])
def test_heat_time_field_and_gradient(m, nelx, nely):
    g = golden("heat")
    k = f"{nelx}x{nely}"
    mesh = m.vh.ScalarMesh.build(nelx, nely, "bottom_edge", torch.device(DEV), torch.float64)

    class Cfg:
        chi_contrast, drain_beta, time_map, heat_cg_rtol = 1000.0, 25.0, "one_minus", 1e-8

    x = T(g[f"{k}_x"]).requires_grad_(True)
    mu = T(g[f"{k}_mu"]).requires_grad_(True)
    sol = m.vh.heat_time_field(Cfg, mesh, x, mu, conduction_penal=3.0)
    J = torch.sum(T(g[f"{k}_w"]) * sol.tPhys)
    gx, gmu = torch.autograd.grad(J, [x, mu])
    assert rel_err(sol.primary.detach().cpu(), g[f"{k}_T"]) < 1e-9
    assert rel_err(sol.tPhys.detach().cpu(), g[f"{k}_tPhys"]) < 1e-9
    assert abs(float(J.detach()) - float(g[f"{k}_J"])) <= 1e-9 * abs(float(g[f"{k}_J"]))
    assert rel_err(gx.cpu(), g[f"{k}_gx"]) < 5e-9
    assert rel_err(gmu.cpu(), g[f"{k}_gmu"]) < 5e-9


@pytest.mark.parametrize("nelx,nely,n_stage", [(48, 24, 4), (64, 32, 16)])
def test_spacetime_objective_fp64_and_mixed(m, nelx, nely, n_stage):
    g = golden("spacetime")
    k = f"{nelx}x{nely}s{n_stage}"
    x, w = T(g[f"{k}_x"]), T(g[f"{k}_w"])
    for precision, tol_c, tol_g in [("fp64", 1e-9, 5e-9), ("mixed", 1e-6, 1e-6)]:
        out = m.st.objective_and_gradient(x, w, n_stage=n_stage, precision=precision)
        np.testing.assert_array_equal(out["member"].cpu().numpy(), g[f"{k}_member"])
        assert rel_err(out["tPhys"].cpu(), g[f"{k}_tPhys"]) < tol_c
        assert rel_err(out["c_s"].cpu(), g[f"{k}_c_s"]) < tol_c, precision
        L = float(out["objective"])
        assert abs(L - float(g[f"{k}_L"])) <= tol_c * abs(float(g[f"{k}_L"])), precision
        assert rel_err(out["gradient"].cpu(), g[f"{k}_grad"]) < tol_g, precision


def test_spacetime_unbatched_matches_batched(m):
    g = golden("spacetime")
    k = "48x24s4"
    x, w = T(g[f"{k}_x"]), T(g[f"{k}_w"])
    a = m.st.objective_and_gradient(x, w, n_stage=4, precision="fp64")
    b = m.st.objective_and_gradient(x, w, n_stage=4, precision="fp64", batched=False)
    assert rel_err(b["c_s"].cpu(), a["c_s"].cpu()) < 1e-12
    assert rel_err(b["gradient"].cpu(), a["gradient"].cpu()) < 1e-10


def test_stage_membership_bit_exact(pkg):
    from sttopt_b200 import _lib

    g = golden("spacetime")
    for k, n_stage in [("48x24s4", 4), ("64x32s16", 16)]:
        t = T(g[f"{k}_tPhys"]).reshape(-1).contiguous()
        member = torch.empty(n_stage, t.numel(), dtype=torch.uint8, device=DEV)
        _lib.check(_lib.lib().stt_stage_membership(t.numel(), n_stage, _lib.ptr(t), _lib.ptr(member),
                                                   _lib.stream()))
        np.testing.assert_array_equal(member.cpu().numpy(), g[f"{k}_member"])


def test_femsolve_recompute_gives_the_same_gradient(m):
    """``femsolve(..., recompute=True)`` drops U after the forward solve and solves for it
    again in the backward pass: the same U (same kernels, same inputs), so the same
    gradients, bit for bit."""
    nelx, nely = 64, 32
    F, mask = O.cantilever_point_load(nelx, nely)
    KE, edof = T(O.plane_stress_KE(0.3)), T(O.element_dof_map(nelx, nely), torch.int64)
    x = T(O.smoothed_density(nelx, nely, 3))
    grads = []
    for recompute in (False, True):
        xPhys = x.clone().requires_grad_(True)
        density = m.fem.simp_density(xPhys, EMIN, EMAX, PENAL).flatten()
        U = m.solve.femsolve(density, T(F), edof, KE, T(mask, torch.bool), nelx, nely, recompute=recompute)
        ce = m.comp._element_strain_energy(U, edof, KE, nely, nelx)
        c = torch.sum(m.fem.simp_density(xPhys, EMIN, EMAX, PENAL) * ce)
        grads.append(torch.autograd.grad(c, [xPhys])[0])
    assert torch.equal(grads[0], grads[1])

"""Parity at the benchmark sizes, against the reference run at those sizes (fixtures
made by ``tests/golden/make_golden.py --full-size``, which runs the reference's FP64
torch path on the CPU; inputs are regenerated here from the seeds).

Two element forms (``sttopt_b200.element_form``): the default modal form applies each
element through its edge modes and annihilates rigid translations exactly; the product
form is the reference's 8 x 8 product of the corner values.  A float64 KE gives a rigid
translation a stiffness of ~1e-16 per element, so on a large-displacement problem the two
FP64 discretisations differ by ~1e-9 relative in compliance (measured: 7.5e-10 on the
1024x512 cantilever, whose tip moves ~400 units; the oracle, a third FP64 code with the
product form, agrees with the reference to 3e-12).  The product form therefore carries
the 1e-9 FP64 parity bound; the modal form is held to the bounds measured for it.

* Config 2, the 1024x512 cantilever in FP64 (6 levels, 1122-dof coarse Cholesky): product
  form at the config's rtol 1e-8 (iteration counts equal to the reference's) and at rtol
  1e-12: U, c and dc to 1e-9; modal form: c to 1e-9, U and dc to 2e-9; the mixed form
  (FP32 V-cycle) at rtol 1e-8 to 1e-6 against the reference's rtol-1e-12 run.
* The space-time objective at 1024x512 and at 2048x1024 (the benchmark's grid, seed and
  16 stages): the mixed form at rtol 1e-8 (the benchmark's form) against the reference's
  rtol-1e-12 run to 1e-6 on the stage compliances, the objective, tPhys and the gradient;
  FP64 modal at rtol 1e-12 to 1e-9; FP64 at the config's rtol 1e-8 with the reference's
  stage and adjoint iteration counts and its stage membership (three exact integers a
  stage), to 1e-9 (product form; U of the modal form to the solve tolerance 1e-8, its
  iterates rounding differently).

Large fields are compared through ``summary_error`` (seeded projections and a strided
subsample; relative L2).  Measured errors are printed and, with ``STT_PARITY_LOG`` set,
appended to that file as JSON lines.
"""

import json
import os
import sys

import numpy as np
import pytest
import torch

from conftest import GOLDEN, golden

sys.path.insert(0, str(GOLDEN))
from summary import summary_error  # noqa: E402

from oracle import sttopt_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu
EMIN, EMAX, PENAL = 1e-9, 1.0, 3.0
DEV = "cuda"


def T(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=DEV)


def record(case: str, **errs) -> None:
    line = {"case": case, **{k: (float(v) if isinstance(v, (float, np.floating)) else v) for k, v in errs.items()}}
    print(json.dumps(line))
    path = os.environ.get("STT_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(line) + "\n")


def rel(a, b) -> float:
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def member_hash(member: np.ndarray) -> np.ndarray:
    m = member.astype(bool)
    idx = np.arange(m.shape[-1], dtype=np.int64)
    return np.stack([m.sum(-1), (m * idx).sum(-1), (m * (idx * idx % 1000003)).sum(-1)], axis=1)


# ---- config 2: the 1024x512 cantilever, FP64 ------------------------------------------

@pytest.fixture(scope="module")
def cantilever(pkg):
    g = golden("cantilever1024")
    nelx, nely, seed = int(g["nelx"]), int(g["nely"]), int(g["seed"])
    x = O.smoothed_density(nelx, nely, seed)
    assert abs(x.sum() - float(g["x_sum"])) <= 1e-12 * abs(float(g["x_sum"]))
    nodes = O.node_grid(nelx, nely)
    ndof = 2 * nodes.size
    F = np.zeros(ndof)
    F[2 * nodes[nely // 2, -1] + 1] = -1.0
    mask = np.ones(ndof, bool)
    mask[2 * nodes[:, 0]] = False
    mask[2 * nodes[:, 0] + 1] = False
    return g, x, F, mask


def _cantilever_solve(x, F, mask, rtol, precision):
    from sttopt_b200 import compliance, fem, torch_fem, torch_solve

    nely, nelx = x.shape
    KE = T(fem.plane_stress_KE(0.3))
    edof = T(fem.element_dof_map(nelx, nely), torch.int64)
    xPhys = T(x).requires_grad_(True)
    info = {}
    density = torch_fem.simp_density(xPhys, EMIN, EMAX, PENAL).flatten()
    U = torch_solve.femsolve(density, T(F), edof, KE, T(mask, torch.bool), nelx, nely, info=info, rtol=rtol,
                             precision=precision)
    ce = compliance._element_strain_energy(U, edof, KE, nely, nelx)
    c = torch.sum(torch_fem.simp_density(xPhys, EMIN, EMAX, PENAL) * ce)
    (dc,) = torch.autograd.grad(c, [xPhys])
    return U.detach().cpu().numpy(), float(c.detach()), dc.cpu().numpy(), info


def test_cantilever1024_hierarchy_shapes(cantilever, pkg):
    from sttopt_b200 import fem, torch_fem, torch_mg

    g, x, F, mask = cantilever
    nely, nelx = x.shape
    levels = torch_mg.build_hierarchy(torch_fem.simp_density(T(x), EMIN, EMAX, PENAL).flatten(),
                                      T(fem.element_dof_map(nelx, nely), torch.int64),
                                      T(fem.plane_stress_KE(0.3)), T(mask, torch.bool), nelx, nely)
    np.testing.assert_array_equal(np.array([[lv.nelx, lv.nely] for lv in levels]), g["level_shapes"])
    assert levels[-1].ndof == int(g["coarse_ndof"])


@pytest.mark.parametrize("precision,rtol,tag,form,tol_c,tol_u,tol_dc", [
    ("fp64", 1e-8, "r8", "product", 1e-9, 1e-9, 1e-9),
    ("fp64", 1e-12, "r12", "product", 1e-9, 1e-9, 1e-9),
    ("fp64", 1e-8, "r8", "modal", 1e-9, 2e-9, 2e-9),
    ("fp64", 1e-12, "r12", "modal", 1e-9, 2e-9, 2e-9),
    ("mixed", 1e-8, "r12", "modal", 1e-6, 1e-6, 1e-6),
])
def test_cantilever1024(cantilever, precision, rtol, tag, form, tol_c, tol_u, tol_dc):
    from sttopt_b200 import element_form

    g, x, F, mask = cantilever
    with element_form(form):
        U, c, dc, info = _cantilever_solve(x, F, mask, rtol, precision)
    eu, edc = summary_error(f"{tag}_U", g, U), summary_error(f"{tag}_dc", g, dc)
    ec = abs(c - float(g[f"{tag}_c"])) / abs(float(g[f"{tag}_c"]))
    record(f"cantilever1024 {precision} {form} rtol {rtol:g} vs reference rtol {'1e-8' if tag == 'r8' else '1e-12'}",
           c=ec, U=max(eu["proj"], eu["sub"]), dc=max(edc["proj"], edc["sub"]), fwd_iter=info["forward_n_iter"],
           bwd_iter=info["backward_n_iter"], ref_fwd_iter=int(g[f"{tag}_fwd_iter"]),
           ref_bwd_iter=int(g[f"{tag}_bwd_iter"]))
    if precision == "fp64" and tag == "r8":
        assert info["forward_n_iter"] == int(g["r8_fwd_iter"])
        assert info["backward_n_iter"] == int(g["r8_bwd_iter"]) == 0
    assert ec <= tol_c
    assert eu["proj"] < tol_u and eu["sub"] < tol_u
    assert edc["proj"] < tol_dc and edc["sub"] < tol_dc
    # fixed dofs exactly zero
    assert np.all(U[~mask] == 0.0)


# ---- the space-time objective at benchmark sizes -----------------------------------------

def _spacetime_case(name):
    g = golden(name)
    nelx, nely, seed = int(g["nelx"]), int(g["nely"]), int(g["seed"])
    x = O.smoothed_density(nelx, nely, seed)
    w = np.random.default_rng(seed).uniform(-1, 1, (nely, nelx))
    assert abs(x.sum() - float(g["x_sum"])) <= 1e-12 * abs(float(g["x_sum"]))
    assert abs(w.sum() - float(g["w_sum"])) <= 1e-9
    return g, x, w


@pytest.mark.parametrize("name", ["spacetime1024", "spacetime2048"])
@pytest.mark.parametrize("precision,rtol,tag,form,tol,tol_u", [
    ("mixed", 1e-8, "r12", "modal", 1e-6, 1e-6),
    ("fp64", 1e-12, "r12", "modal", 1e-9, 1e-9),
    ("fp64", 1e-8, "r8", "product", 1e-9, 1e-9),
    ("fp64", 1e-8, "r8", "modal", 1e-9, 1e-8),
])
def test_spacetime_fullsize(pkg, name, precision, rtol, tag, form, tol, tol_u):
    from sttopt_b200 import element_form, spacetime

    g, x, w = _spacetime_case(name)
    n_stage = int(g["n_stage"])
    info = {}
    with element_form(form):
        out = spacetime.objective_and_gradient(T(x), T(w), n_stage=n_stage, precision=precision, rtol=rtol,
                                               info=info)
        torch.cuda.synchronize()
    c_s = out["c_s"].cpu().numpy()
    e_c = rel(c_s, g[f"{tag}_c_s"])
    e_cmax = float(np.max(np.abs(c_s - g[f"{tag}_c_s"]) / np.abs(g[f"{tag}_c_s"])))
    e_L = abs(float(out["objective"]) - float(g[f"{tag}_L"])) / abs(float(g[f"{tag}_L"]))
    e_g = summary_error(f"{tag}_grad", g, out["gradient"].cpu().numpy())
    e_t = summary_error(f"{tag}_tPhys", g, out["tPhys"].cpu().numpy())
    U = out["U"].cpu().numpy()
    e_u = summary_error(f"{tag}_U", g, U)
    mh = member_hash(out["member"].cpu().numpy())
    member_equal = bool(np.array_equal(mh, g[f"{tag}_member"]))
    count_diff = int(np.abs(mh[:, 0] - g[f"{tag}_member"][:, 0]).max())
    record(f"{name} {precision} {form} rtol {rtol:g} vs reference rtol {'1e-8' if tag == 'r8' else '1e-12'}",
           c_s=e_c, c_s_max=e_cmax, objective=e_L, gradient=max(e_g["proj"], e_g["sub"]),
           tPhys=max(e_t["proj"], e_t["sub"]), U=max(e_u["proj"], e_u["sub"]), member_equal=member_equal,
           member_count_diff=count_diff, iters={k: v for k, v in info.items()},
           ref_fwd_iter=int(g[f"{tag}_fwd_iter"]), ref_bwd_iter=int(g[f"{tag}_bwd_iter"]))
    if precision == "fp64":
        assert member_equal
    else:
        # FP32-cycle rounding moves tPhys by ~1e-9 relative; an element lying that close to
        # a stage threshold may change stage (none did in the measured runs)
        assert count_diff <= 2
    if precision == "fp64" and tag == "r8":
        assert info["stage_n_iter"] == int(g["r8_fwd_iter"])
        assert info["adjoint_n_iter"] == int(g["r8_bwd_iter"])
    assert e_cmax < tol and e_L < tol
    assert e_t["proj"] < tol and e_t["sub"] < tol
    assert e_u["proj"] < tol_u and e_u["sub"] < tol_u
    assert e_g["proj"] < tol and e_g["sub"] < tol

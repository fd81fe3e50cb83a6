"""The differentiation configuration at 512x256 (16 stages): the space-time objective
through its autograd node, against the reference's full sensitivity field (golden
fixture made by running the reference) and against central finite differences (step
1e-6) on 64 seeded elements, in FP64 and in mixed precision.

Tolerances: FP64 gradient 5e-9 relative (two FP64 solves stopped at rtol 1e-8 agree to
about 1e-9 there), mixed 1e-6; stage membership bit-exact.  Finite differences run the
FP64 objective at rtol 1e-12 and skip an element whose perturbation moves any element
across a stage threshold (the hard threshold is not differentiable there); their noise
floor is the objective's solve noise over 2h, about 1e-6 absolute."""

import numpy as np
import pytest
import torch

from conftest import golden, rel_err
from oracle import sttopt_oracle as O

pytestmark = pytest.mark.gpu
NELX, NELY, NSTAGE, SEED = 512, 256, 16, 4


@pytest.fixture(scope="module")
def case(pkg):
    g = golden("spacetime512")
    x = O.smoothed_density(NELX, NELY, SEED)
    w = np.random.default_rng(SEED).uniform(-1, 1, (NELY, NELX))
    assert abs(x.sum() - float(g["x_sum"])) <= 1e-12 * abs(float(g["x_sum"]))
    assert abs(w.sum() - float(g["w_sum"])) <= 1e-9
    member = np.unpackbits(g["member_bits"], axis=-1)[:, :NELX * NELY]
    return g, x, w, member


@pytest.mark.parametrize("precision,tol", [("fp64", 5e-9), ("mixed", 1e-6)])
def test_objective_autograd_matches_reference_sensitivity_field(case, precision, tol):
    from sttopt_b200 import sensitivity, spacetime

    g, x, w, member = case
    xt = torch.tensor(x, device="cuda").requires_grad_(True)
    wt = torch.tensor(w, device="cuda")
    L = spacetime.objective(xt, wt, n_stage=NSTAGE, precision=precision)
    assert abs(float(L.detach()) - float(g["L"])) <= tol * abs(float(g["L"]))
    (jac,) = sensitivity.jacobian_rows(L[None], [xt])
    assert rel_err(jac.reshape(NELY, NELX).cpu(), g["grad"]) < tol
    out = spacetime.objective_and_gradient(xt.detach(), wt, n_stage=NSTAGE, precision=precision)
    np.testing.assert_array_equal(out["member"].cpu().numpy(), member)
    assert rel_err(out["c_s"].cpu(), g["c_s"]) < tol
    assert rel_err(out["tPhys"].cpu(), g["tPhys"]) < tol


def test_gradient_matches_central_differences(case):
    from sttopt_b200 import spacetime

    g, x, w, _ = case
    dev = torch.device("cuda")
    wt = torch.tensor(w, device=dev)
    problem = spacetime.SpaceTimeProblem(NELX, NELY, dev)
    kw = dict(n_stage=NSTAGE, precision="fp64", rtol=1e-12, problem=problem)
    base = spacetime.objective_and_gradient(torch.tensor(x, device=dev), wt, **kw)
    grad = base["gradient"].reshape(-1).cpu().numpy()
    # the reference's field comes from rtol-1e-8 solves: agreement to its solve accuracy
    assert rel_err(grad, g["grad"].ravel()) < 1e-7
    idx = np.random.default_rng(SEED).choice(NELX * NELY, 64, replace=False)
    h = 1e-6
    fd, an = [], []
    for e in idx:
        vals = []
        for sgn in (1.0, -1.0):
            xp = x.copy().ravel()
            xp[e] += sgn * h
            o = spacetime.objective_and_gradient(torch.tensor(xp.reshape(NELY, NELX), device=dev), wt,
                                                 gradient=False, **kw)
            vals.append((float(o["objective"]), torch.equal(o["member"], base["member"])))
        if not (vals[0][1] and vals[1][1]):
            continue  # a stage threshold was crossed
        fd.append((vals[0][0] - vals[1][0]) / (2 * h))
        an.append(grad[e])
    fd, an = np.array(fd), np.array(an)
    assert len(fd) >= 56, len(fd)
    # central differences at h = 1e-6 carry the objective's solve noise (~1e-12 of it at
    # rtol 1e-12) divided by 2h: about 1e-6 absolute here, against |grad| up to ~0.4
    scale = np.abs(grad).max()
    err = np.abs(fd - an)
    assert np.all(err <= 2e-3 * np.abs(an) + 5e-5 * scale), (err.max(), scale)
    big = np.abs(an) > 1e-2 * scale
    assert big.sum() >= 8 and np.median(err[big] / np.abs(an[big])) < 1e-3


@pytest.mark.parametrize("precision,tol", [("fp64", 5e-9), ("mixed", 1e-6)])
def test_dropin_chain_matches_the_reference_and_the_fused_path(case, precision, tol):
    """The objective composed only of the reference-signature functions
    (heat_time_field -> batched_whole_and_gravity_compliance(mask_fn=hard_time_mask) ->
    jacobian_rows, ``spacetime.DropInChain``) against the reference's field and the fused
    ``objective_and_gradient``: the two device paths to 1e-10 in FP64."""
    from sttopt_b200 import spacetime

    g, x, w, member = case
    dev = torch.device("cuda")
    chain = spacetime.DropInChain(NELX, NELY, dev, n_stage=NSTAGE)
    xt, wt = torch.tensor(x, device=dev), torch.tensor(w, device=dev)
    out = chain(xt, wt, precision=precision)
    assert abs(float(out["objective"]) - float(g["L"])) <= tol * abs(float(g["L"]))
    assert rel_err(out["c_s"].cpu(), g["c_s"]) < tol
    assert rel_err(out["gradient"].cpu(), g["grad"]) < tol
    assert rel_err(out["tPhys"].cpu(), g["tPhys"]) < tol
    if precision == "fp64":
        fused = spacetime.objective_and_gradient(xt, wt, n_stage=NSTAGE, precision="fp64")
        assert rel_err(out["c_s"].cpu(), fused["c_s"].cpu()) < 1e-10
        assert rel_err(out["gradient"].cpu(), fused["gradient"].cpu()) < 1e-10

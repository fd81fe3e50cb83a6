"""GPU parity of the cone density filter and the Heaviside projection (the density's
upstream step) against the reference's outputs (golden fixtures) and the oracle.

Tolerances: filter and projection 1e-13 relative (FP64, same arithmetic to rounding);
gradients through the adjoint kernel 1e-12."""

import numpy as np
import pytest
import torch

from conftest import golden, rel_err
from oracle import sttopt_oracle as O

pytestmark = pytest.mark.gpu
KEYS = ["37x23r1.5", "37x23r2.5", "64x40r4.0", "20x11r8.0"]


def _dims(key):
    nelx, nely = (int(v) for v in key.split("r")[0].split("x"))
    return nelx, nely, float(key.split("r")[1])


@pytest.mark.parametrize("key", KEYS)
def test_filter_projection_and_gradients(pkg, key):
    from sttopt_b200 import filters

    g = golden("filters")
    nelx, nely, rmin = _dims(key)
    H, Hs = filters.density_filter(nelx, nely, rmin)
    x = torch.tensor(g[f"{key}_x"], device="cuda").requires_grad_(True)
    w = torch.tensor(g[f"{key}_w"], device="cuda")
    xt = filters.apply_density_filter(x, H, Hs)
    assert rel_err(xt.detach().cpu(), g[f"{key}_xTilde"]) < 1e-13
    (gx,) = torch.autograd.grad(torch.sum(w * xt), [x])
    assert rel_err(gx.cpu(), g[f"{key}_grad_filter"]) < 1e-12
    for beta in (1.0, 8.0, float("inf")):
        xp, xt2 = filters.filter_and_project(x, H, beta, 0.5)
        assert rel_err(xp.detach().cpu(), g[f"{key}_b{beta}_xPhys"]) < 1e-13
        assert torch.equal(xt2, xt.detach())
        if not np.isinf(beta):
            (gp,) = torch.autograd.grad(torch.sum(w * xp), [x])
            assert rel_err(gp.cpu(), g[f"{key}_b{beta}_grad"]) < 1e-12
            d = filters.heaviside_projection_derivative(xt.detach(), beta, 0.5)
            assert rel_err(d.cpu(), g[f"{key}_b{beta}_dP"]) < 1e-13


def test_batched_rows_and_a_large_grid(pkg):
    from sttopt_b200 import filters

    nelx, nely, rmin = 512, 256, 4.0
    rng = np.random.default_rng(5)
    xs = rng.uniform(0, 1, (3, nely, nelx))
    Ho, Hso = O.density_filter(nelx, nely, rmin)
    H, _ = filters.density_filter(nelx, nely, rmin)
    got = filters.apply_density_filter(torch.tensor(xs, device="cuda"), H).cpu().numpy()
    for k in range(3):
        assert rel_err(got[k], O.apply_density_filter(xs[k], Ho, Hso)) < 1e-13
    # adjoint: <H v / Hs, u> == <v, H (u / Hs)>
    u = torch.tensor(rng.standard_normal((nely, nelx)), device="cuda").requires_grad_(True)
    v = torch.tensor(rng.standard_normal((nely, nelx)), device="cuda")
    lhs = torch.sum(filters.apply_density_filter(u, H) * v)
    (gu,) = torch.autograd.grad(lhs, [u])
    lhs = lhs.detach()
    assert abs(float(torch.sum(gu * u.detach()) - lhs)) <= 1e-12 * abs(float(lhs))


@pytest.mark.parametrize("beta", [None, 4.0])
def test_filtered_objective_gradient_through_the_filter(pkg, beta):
    """``objective_and_gradient`` with the density filter (and projection) inside: the
    objective of ``P(H x / Hs)`` and its gradient in the design variable x equal the
    autograd composition of ``filters.filter_and_project`` (or ``apply_density_filter``)
    with the objective node, and central differences of the FP64 objective on seeded
    elements."""
    import numpy as np

    from sttopt_b200 import filters, spacetime, synthetic

    nelx, nely, n_stage = 96, 48, 8
    dev = torch.device("cuda")
    x = synthetic.smoothed_density(nelx, nely, 31, device=dev)
    w = synthetic.time_weights(nelx, nely, 31, device=dev)
    H, Hs = filters.density_filter(nelx, nely, 2.5)
    kw = dict(n_stage=n_stage, precision="fp64", rtol=1e-12)
    fused = spacetime.objective_and_gradient(x, w, filter=H, beta=beta, **kw)
    xv = x.clone().requires_grad_(True)
    xp = filters.apply_density_filter(xv, H) if beta is None else filters.filter_and_project(xv, H, beta, 0.5)[0]
    L = spacetime.objective(xp, w, **kw)
    (g,) = torch.autograd.grad(L, [xv])
    L = L.detach()
    assert abs(float(fused["objective"]) - float(L)) <= 1e-12 * abs(float(L))
    assert float((fused["gradient"] - g).norm() / g.norm()) < 1e-12
    assert torch.equal(fused["xPhys"], xp.detach())
    # central differences (h = 1e-6) on elements whose perturbation moves no stage
    # membership; their noise floor is the objective's solve noise over 2h, as in the
    # differentiation configuration's check
    rng = np.random.default_rng(5)
    h = 1e-6
    grad = fused["gradient"].reshape(-1)
    scale = float(grad.abs().max())
    fd, an = [], []
    for e in rng.choice(nelx * nely, 24, replace=False):
        xs = []
        for sgn in (1, -1):
            xe = x.clone().reshape(-1)
            xe[e] += sgn * h
            xs.append(spacetime.objective_and_gradient(xe.reshape(nely, nelx), w, filter=H, beta=beta, gradient=False,
                                                       **kw))
        if not torch.equal(xs[0]["member"], fused["member"]) or not torch.equal(xs[1]["member"], fused["member"]):
            continue
        fd.append((float(xs[0]["objective"]) - float(xs[1]["objective"])) / (2 * h))
        an.append(float(grad[e]))
    fd, an = np.array(fd), np.array(an)
    assert len(fd) >= 16
    assert np.all(np.abs(fd - an) <= 2e-3 * np.abs(an) + 5e-5 * scale), (np.abs(fd - an).max(), scale)

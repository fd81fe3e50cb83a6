"""Many space-time problems of uneven sizes and stage counts in one call (the batched
uneven configuration): grouped by grid size into batched device solves on concurrent
streams.  Each problem's result must equal the one-problem call on the same inputs, and
the oracle's, in FP64 and in mixed precision.

Tolerances: grouped against one-problem calls 1e-12 (same arithmetic per row, only the
batching differs); against the oracle 1e-9 on the objective and 5e-9 on the gradient
(two FP64 solves at rtol 1e-8); mixed precision 1e-6 against the oracle."""

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import sttopt_oracle as O

pytestmark = pytest.mark.gpu

SIZES = [(48, 24), (32, 16), (48, 24), (64, 32), (32, 16), (40, 20)]
STAGES = [3, 5, 4, 2, 6, 1]


def _inputs():
    xs, ws = [], []
    for k, (nx, ny) in enumerate(SIZES):
        xs.append(O.smoothed_density(nx, ny, 100 + k))
        ws.append(np.random.default_rng(100 + k).uniform(-1, 1, (ny, nx)))
    return xs, ws


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_many_equals_one_at_a_time_and_the_oracle(pkg, precision):
    from sttopt_b200 import spacetime

    xs, ws = _inputs()
    X = [torch.tensor(x, device="cuda") for x in xs]
    W = [torch.tensor(w, device="cuda") for w in ws]
    info = {}
    many = spacetime.objective_and_gradient_many(X, W, STAGES, precision=precision, info=info)
    assert set(info) == {(nx, ny) for nx, ny in SIZES}
    for k, (x, w, n) in enumerate(zip(X, W, STAGES)):
        one = spacetime.objective_and_gradient(x, w, n_stage=n, precision=precision)
        got = many[k]
        assert got["c_s"].shape == (n,)
        assert got["gradient"].shape == x.shape
        assert torch.equal(got["member"], one["member"])
        assert rel_err(got["c_s"].cpu(), one["c_s"].cpu()) < 1e-12
        assert rel_err(got["gradient"].cpu(), one["gradient"].cpu()) < 1e-12
        assert abs(float(got["objective"] - one["objective"])) <= 1e-12 * abs(float(one["objective"]))
    tol_c, tol_g = (1e-9, 5e-9) if precision == "fp64" else (1e-6, 1e-6)
    for k in (0, 3, 5):
        ref = O.spacetime_objective(xs[k], ws[k], n_stage=STAGES[k])
        got = many[k]
        assert abs(float(got["objective"]) - ref["objective"]) <= tol_c * abs(ref["objective"])
        assert rel_err(got["gradient"].cpu(), ref["gradient"]) < tol_g


def test_many_sequential_matches_concurrent(pkg):
    from sttopt_b200 import spacetime

    xs, ws = _inputs()
    X = [torch.tensor(x, device="cuda") for x in xs]
    W = [torch.tensor(w, device="cuda") for w in ws]
    a = spacetime.objective_and_gradient_many(X, W, STAGES, precision="mixed", concurrent=True)
    b = spacetime.objective_and_gradient_many(X, W, STAGES, precision="mixed", concurrent=False)
    for p, q in zip(a, b):
        assert torch.equal(p["gradient"], q["gradient"])
        assert torch.equal(p["c_s"], q["c_s"])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_split_objective_shares_add_up_to_the_whole(pkg, precision, tol):
    """The shares of a split objective (``objective_and_gradient_part``), computed one
    after another on one GPU as three ranks would: rank 0 solves the heat field (handing
    tPhys to the others through ``publish``), every share solves its stages, and the sum
    of the gradient terms and the stage compliances equals the whole objective."""
    from sttopt_b200 import sharding, spacetime, synthetic

    nelx, nely, n_stage = 128, 64, 16
    x = synthetic.smoothed_density(nelx, nely, 21)
    w = synthetic.time_weights(nelx, nely, 21)
    whole = spacetime.objective_and_gradient(x, w, n_stage=n_stage, precision=precision)
    parts = sharding.stage_partition(n_stage, 3)
    got = {}
    p0 = spacetime.objective_and_gradient_part(x, w, n_stage=n_stage, stages=parts[0], precision=precision,
                                               publish=lambda t: got.setdefault("tPhys", t.clone()))
    shares = [p0] + [spacetime.objective_and_gradient_part(x, w, n_stage=n_stage, stages=p, precision=precision,
                                                           tphys=got["tPhys"].reshape(nely, nelx))
                     for p in parts[1:]]
    grad = sum(s["gradient"] for s in shares)
    c_s = torch.zeros(n_stage, dtype=torch.float64, device=x.device)
    for p, s in zip(parts, shares):
        c_s[torch.tensor(p, device=x.device)] = s["c_s"]
    assert torch.equal(got["tPhys"].reshape(nely, nelx), whole["tPhys"])
    assert rel_err(c_s.cpu(), whole["c_s"].cpu()) < tol
    assert rel_err(grad.cpu(), whole["gradient"].cpu()) < tol


def test_memory_budget_waves_give_the_same_results(pkg):
    """A memory budget below the whole batch's estimate runs the groups in waves (a group
    cut into slices where it alone exceeds the budget): every problem's result equals the
    unbounded call's, and the waves' estimates fit the budget."""
    from sttopt_b200 import spacetime, synthetic

    dev = torch.device("cuda")
    shapes = [(96, 48), (64, 32), (96, 48), (128, 64), (64, 32), (128, 64)]
    xs = [synthetic.smoothed_density(nx, ny, 40 + k, device=dev) for k, (nx, ny) in enumerate(shapes)]
    ws = [synthetic.time_weights(nx, ny, 40 + k, device=dev) for k, (nx, ny) in enumerate(shapes)]
    ns = [4, 6, 5, 8, 7, 4]
    full = spacetime.objective_and_gradient_many(xs, ws, ns, precision="fp64")
    groups: dict = {}
    for k, x in enumerate(xs):
        groups.setdefault(tuple(x.shape), []).append(k)
    biggest = max(spacetime.group_bytes(s[1], s[0], len(i), sum(ns[k] for k in i), "fp64") for s, i in groups.items())
    budget = int(0.7 * biggest)
    waves = spacetime.budget_waves(groups, ns, budget, "fp64", 700)
    assert len(waves) > 1
    assert sorted(k for w in waves for _, idx in w for k in idx) == list(range(len(xs)))
    for w in waves:
        assert len({shape for shape, _ in w}) == len(w)
    got = spacetime.objective_and_gradient_many(xs, ws, ns, precision="fp64", memory_budget=budget)
    for a, b in zip(full, got):
        assert rel_err(b["c_s"].cpu(), a["c_s"].cpu()) < 1e-12
        assert rel_err(b["gradient"].cpu(), a["gradient"].cpu()) < 1e-12

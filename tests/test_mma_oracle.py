"""The CPU oracle of the MMA subproblem against the reference's own outputs.

``tests/golden/mma.npz`` holds ``mma.mmasub`` run on seeded subproblems (the script is
``tests/golden/make_golden.py``, generator ``mma``): the first-iteration asymptotes
(m = 1), the adaptive asymptotes with per-variable trust regions (m = 3), more
constraints (m = 12) and the m >= n elimination (m = 6, n = 4).  The oracle reproduces
them to rounding; the device path is then checked against both.
"""

import numpy as np
import pytest

from conftest import golden
from oracle import mma_oracle as M

NAMES = ("xmma", "ymma", "zmma", "lam", "xsi", "eta", "mu", "zet", "s", "low", "upp")
TAGS = ("first", "adapt", "wide", "mgen")


def mma_case(g, tag):
    """The inputs of one golden case, as ``mmasub``'s positional and keyword arguments."""
    p = {k[len(tag) + 4:]: g[k] for k in g if k.startswith(f"{tag}_in_")}
    args = (int(p["m"]), int(p["n"]), int(p["iteration"]), p["xval"], p["xmin"], p["xmax"], p["xold1"],
            p["xold2"], float(p["f0val"]), p["df0dx"], p["fval"], p["dfdx"], p["low"], p["upp"],
            float(p["a0"]), p["a"], p["c"], p["d"])
    kw = {k: g[f"{tag}_{k}"] for k in ("asyinit", "asyclamp_min", "asyclamp_max", "move") if f"{tag}_{k}" in g}
    return args, kw


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_mmasub_matches_reference(tag):
    g = golden("mma")
    args, kw = mma_case(g, tag)
    got = M.mmasub(*args, **kw)
    for name, v in zip(NAMES, got):
        want = g[f"{tag}_{name}"]
        scale = max(float(np.abs(want).max()), 1e-300)
        assert float(np.abs(np.asarray(v) - want).max()) / scale < 1e-12, name


def _kkt_residual(sol, epsi, args):
    return M._residual(sol, epsi, *args)


@pytest.mark.parametrize("m,n", [(3, 8), (3, 2)])
def test_oracle_subsolv_meets_barrier_target(m, n):
    """Both eliminations end at a point whose barrier residual is below 0.9 epsi at the
    last barrier level (the Newton loop's own exit test)."""
    rng = np.random.default_rng(7)
    low, upp = np.full(n, -1.0), np.full(n, 1.0)
    alfa, beta = np.full(n, -0.9), np.full(n, 0.9)
    p0, q0 = rng.uniform(0.5, 2.0, n), rng.uniform(0.5, 2.0, n)
    P, Q = rng.uniform(0.1, 1.0, (m, n)), rng.uniform(0.1, 1.0, (m, n))
    a0, a = 1.0, rng.uniform(0.1, 0.3, m)
    b = 0.8 * (P + Q).sum(1)
    c, d = np.full(m, 10.0), rng.uniform(0.25, 1.0, m)
    args = (low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d)
    sol = M.subsolv(m, n, M.EPSIMIN, *args)
    epsi_last = 1e-7  # 0.1 ** 7, the last level above epsimin
    assert np.abs(_kkt_residual(sol, epsi_last, args)).max() <= 0.9 * epsi_last * 1.0001
    assert np.all(sol[0] > alfa) and np.all(sol[0] < beta)


def test_trust_region_and_floor_share_host_logic(pkg):
    """The drop-in's small torch wrappers (sttopt/mma.py:22-147) on CPU tensors."""
    import torch
    from sttopt_b200 import mma

    move = torch.tensor([0.01, 0.05, 0.1, 0.2], dtype=torch.float64)
    tr = mma.trust_region_params(move, torch.full_like(move, 2.0))
    assert torch.equal(tr["asyinit"], move / 2.0) and torch.equal(tr["move"], move / 2.0)
    assert torch.equal(tr["asyclamp_min"], 0.02 * (move / 2.0))
    assert torch.equal(tr["asyclamp_max"], 20.0 * (move / 2.0))
    h = mma.History.initial(torch.full((4,), 0.5, dtype=torch.float64))
    assert torch.equal(h.xold1, h.xold2) and h.xold1 is not h.xold2 and float(h.low.abs().sum()) == 0.0
    floor = 0.02 * move
    half = torch.tensor([1.0, 1.0, 1.0, 1.0], dtype=torch.float64) * floor
    half[2] *= 3.0
    hist = mma.History(xold1=h.xold1, xold2=h.xold2, low=0.5 - half, upp=0.5 + half)
    assert mma.floor_share(hist, move, torch.tensor([True, True, True, False])) == pytest.approx(2 / 3)
    assert mma.floor_share(hist, move, torch.zeros(4, dtype=torch.bool)) == 0.0

"""The device MMA subproblem (``sttopt_b200.mma``) against the reference's own outputs
(``tests/golden/mma.npz``) and the CPU oracle (``oracle/mma_oracle.py``).

Bound: every output within 1e-9 of the reference's, relative to the output's largest
magnitude.  The device sums in another order than the reference (block partials, fused
P/Q rebuilt from dfdx), so agreement is to rounding along the same Newton path, not bit
for bit.  At sizes the oracle finishes in seconds the same bound holds against the
oracle; at the production size (2 x 2048 x 1024 variables, 17 constraints) the check is
the solve's own exit test: the barrier residual at the returned point below 0.9 epsi at
the last barrier level.
"""

import numpy as np
import pytest
import torch

from conftest import golden
from oracle import mma_oracle as M
from test_mma_oracle import NAMES, TAGS, mma_case

pytestmark = pytest.mark.gpu
TOL = 1e-9


@pytest.fixture(scope="module")
def mma(pkg):
    from sttopt_b200 import mma as mod

    return mod


def dev(v):
    return torch.as_tensor(np.asarray(v, np.float64)).cuda()


def rel_max(got, want):
    got = got.detach().cpu().numpy() if torch.is_tensor(got) else np.asarray(got)
    want = np.asarray(want)
    return float(np.abs(got - want).max()) / max(float(np.abs(want).max()), 1e-300)


def run_device(mma, args, kw, stats=None):
    m, n, it, *vecs = args
    xval, xmin, xmax, xold1, xold2, f0val, df0dx, fval, dfdx, low, upp, a0, a, c, d = vecs
    t = [dev(v) for v in (xval, xmin, xmax, xold1, xold2)]
    kwd = {k: dev(v) for k, v in kw.items()}
    return mma.mmasub(m, n, it, *t, f0val, dev(df0dx), dev(fval), dev(dfdx), dev(low), dev(upp), a0, dev(a),
                      dev(c), dev(d), stats=stats, **kwd)


@pytest.mark.parametrize("tag", TAGS)
def test_mmasub_matches_reference_outputs(mma, tag):
    """The outputs, and the same Newton path as the oracle: as many Newton steps and
    line-search candidates."""
    g = golden("mma")
    args, kw = mma_case(g, tag)
    got_stats, want_stats = {}, {}
    got = run_device(mma, args, kw, got_stats)
    oracle = M.mmasub(*args, **kw, stats=want_stats)
    for name, v, o in zip(NAMES, got, oracle):
        assert rel_max(v, g[f"{tag}_{name}"]) < TOL, (name, rel_max(v, g[f"{tag}_{name}"]))
        assert rel_max(v, o) < TOL, name
    for key in ("subsolv_newton_steps", "subsolv_line_search_tries"):
        assert got_stats[key] == want_stats[key], (key, got_stats, want_stats)
    assert got_stats.get("subsolv_cap_hits", 0) == want_stats["subsolv_cap_hits"] == 0


def _subproblem(rng, m, n):
    low, upp = np.full(n, -1.0), np.full(n, 1.0)
    alfa, beta = np.full(n, -0.9), np.full(n, 0.9)
    p0, q0 = rng.uniform(0.5, 2.0, n), rng.uniform(0.5, 2.0, n)
    P, Q = rng.uniform(0.1, 1.0, (m, n)), rng.uniform(0.1, 1.0, (m, n))
    a = rng.uniform(0.1, 0.3, m)
    b = 0.8 * (P + Q).sum(1)
    c, d = np.full(m, 10.0), rng.uniform(0.25, 1.0, m)
    return (low, upp, alfa, beta, p0, q0, P, Q, 1.0, a, b, c, d)


@pytest.mark.parametrize("m,n", [(3, 8), (5, 1000), (17, 4096), (40, 3000), (64, 5000), (3, 2), (6, 6)])
def test_subsolv_matches_oracle(mma, m, n):
    """Both eliminations (m < n on the device, m >= n in host code) and every template
    bucket of m (4, 8, 16, 32, 64) against the oracle's subsolv."""
    rng = np.random.default_rng(m * 1000 + n)
    args = _subproblem(rng, m, n)
    want = M.subsolv(m, n, M.EPSIMIN, *args)
    low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d = args
    got = mma.subsolv(m, n, M.EPSIMIN, *(dev(v) for v in (low, upp, alfa, beta, p0, q0, P, Q)), a0,
                      *(dev(v) for v in (a, b, c, d)))
    for k, (gv, wv) in enumerate(zip(got, want)):
        assert rel_max(gv, wv) < TOL, (k, rel_max(gv, wv))


def test_subsolv_on_a_side_stream(mma):
    """The call runs on the caller's current stream, here not the default one."""
    rng = np.random.default_rng(17)
    m, n = 5, 3000
    args = _subproblem(rng, m, n)
    low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d = args
    dargs = [dev(v) for v in (low, upp, alfa, beta, p0, q0, P, Q)]
    rest = [dev(v) for v in (a, b, c, d)]
    want = mma.subsolv(m, n, M.EPSIMIN, *dargs, a0, *rest)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        got = mma.subsolv(m, n, M.EPSIMIN, *dargs, a0, *rest)
    torch.cuda.current_stream().wait_stream(side)
    for gv, wv in zip(got, want):
        assert torch.equal(gv, wv)


def test_subsolv_strided_rows(mma):
    """P and Q as row views with a row stride larger than n."""
    rng = np.random.default_rng(5)
    m, n = 4, 777
    args = _subproblem(rng, m, n)
    want = M.subsolv(m, n, M.EPSIMIN, *args)
    low, upp, alfa, beta, p0, q0, P, Q, a0, a, b, c, d = args
    big = torch.zeros(2 * m, n + 13, dtype=torch.float64, device="cuda")
    big[:m, :n] = dev(P)
    big[m:, :n] = dev(Q)
    got = mma.subsolv(m, n, M.EPSIMIN, *(dev(v) for v in (low, upp, alfa, beta, p0, q0)), big[:m, :n],
                      big[m:, :n], a0, *(dev(v) for v in (a, b, c, d)))
    for gv, wv in zip(got, want):
        assert rel_max(gv, wv) < TOL


def _production_case(n, m, seed):
    rng = np.random.default_rng(seed)
    xval = rng.uniform(0.05, 0.95, n)
    xold1 = np.clip(xval + rng.normal(0, 0.02, n), 0, 1)
    xold2 = np.clip(xold1 + rng.normal(0, 0.02, n), 0, 1)
    return dict(xval=xval, xold1=xold1, xold2=xold2, df0dx=rng.normal(0, 1e-6, n), fval=rng.normal(0, 0.1, m),
                dfdx=rng.normal(0, 1e-6, (m, n)), move=rng.uniform(0.02, 0.1, n))


def test_mmasub_oracle_at_a_quarter_million_variables(mma):
    """The unit-box step the optimisation loop takes (trust-region asymptotes, a = d = 0,
    c = 1000, raa0 scaled by n) on 2^18 variables and 17 constraints, against the oracle."""
    n, m = 1 << 18, 17
    p = _production_case(n, m, 3)
    tr = M_trust(p["move"], np.ones(n))
    args = (m, n, 4, p["xval"], np.zeros(n), np.ones(n), p["xold1"], p["xold2"], 0.0, p["df0dx"], p["fval"],
            p["dfdx"], p["xval"] - 0.2, p["xval"] + 0.2, 1.0, np.zeros(m), np.full(m, 1000.0), np.zeros(m))
    want_stats, got_stats = {}, {}
    want = M.mmasub(*args, raa0=1e-5 / n, stats=want_stats, **tr)
    t = [dev(v) for v in args[3:8]]
    got = mma.mmasub(m, n, 4, *t, 0.0, dev(p["df0dx"]), dev(p["fval"]), dev(p["dfdx"]), dev(args[12]),
                     dev(args[13]), 1.0, dev(np.zeros(m)), dev(np.full(m, 1000.0)), dev(np.zeros(m)),
                     raa0=1e-5 / n, stats=got_stats, **{k: dev(v) for k, v in tr.items()})
    for name, gv, wv in zip(NAMES, got, want):
        assert rel_max(gv, wv) < TOL, (name, rel_max(gv, wv))
    assert got_stats["subsolv_newton_steps"] == want_stats["subsolv_newton_steps"]
    assert got_stats["subsolv_line_search_tries"] == want_stats["subsolv_line_search_tries"]


def M_trust(move, xrange):
    asyinit = move / xrange
    return {"asyinit": asyinit, "asyclamp_min": 0.02 * asyinit, "asyclamp_max": 20.0 * asyinit, "move": asyinit}


def test_mmasub_production_size_meets_barrier_target(mma):
    """2 x 2048 x 1024 variables (density and time field) and 17 constraints, the
    adaptive-asymptote branch: the returned point passes the Newton loop's exit test at
    the last barrier level (the oracle's residual of the subproblem the returned
    asymptotes define, below 0.9 epsi), within the move limits."""
    n, m = 2 * 2048 * 1024, 17
    p = _production_case(n, m, 9)
    tr = M_trust(p["move"], np.ones(n))
    low, upp = p["xval"] - 0.2, p["xval"] + 0.2
    zeros, cc = np.zeros(m), np.full(m, 1000.0)
    stats = {}
    got = mma.mmasub(m, n, 2, *(dev(v) for v in (p["xval"], np.zeros(n), np.ones(n), p["xold1"], p["xold2"])), 0.0,
                     dev(p["df0dx"]), dev(p["fval"]), dev(p["dfdx"]), dev(low), dev(upp), 1.0, dev(zeros), dev(cc),
                     dev(zeros), raa0=1e-5 / n, stats=stats, **{k: dev(v) for k, v in tr.items()})
    assert stats.get("subsolv_cap_hits", 0) == 0
    sol = [v.cpu().numpy() if v.dim() else float(v) for v in got[:9]]
    low_d, upp_d = got[9].cpu().numpy(), got[10].cpu().numpy()
    want_low, want_upp = M.asymptotes(2, p["xval"], np.zeros(n), np.ones(n), p["xold1"], p["xold2"], low, upp,
                                      tr["asyinit"], tr["asyclamp_min"], tr["asyclamp_max"], 1.2, 0.7)
    assert rel_max(low_d, want_low) < 1e-15 and rel_max(upp_d, want_upp) < 1e-15
    approx = M.approximation(p["xval"], np.zeros(n), np.ones(n), low_d, upp_d, p["df0dx"], p["fval"], p["dfdx"],
                             tr["move"], 1e-5 / n, 0.1)
    alfa, beta, p0, q0, P, Q, b = approx
    epsi_last = 0.1 ** 7
    r = M._residual(sol, epsi_last, low_d, upp_d, alfa, beta, p0, q0, P, Q, 1.0, zeros, b, cc, zeros)
    assert np.abs(r).max() <= 0.9 * epsi_last * (1 + 1e-6)
    x = sol[0]
    assert np.all(x >= alfa) and np.all(x <= beta)
    assert np.all(np.abs(x - p["xval"]) <= p["move"] * (1 + 1e-12))


def test_subsolv_counts_barrier_levels_at_the_cap(mma):
    """A barrier target below float precision cannot be met, so levels stop at the
    200-iteration cap and are counted and warned about; a reachable one counts none
    (sttopt/mma.py:540-555)."""
    torch.manual_seed(0)
    n, m = 6, 1
    f64 = dict(dtype=torch.float64, device="cuda")
    x = torch.full((n,), 0.5, **f64)
    args = (x - 0.1, x + 0.1, x - 0.05, x + 0.05, torch.rand(n, **f64), torch.rand(n, **f64),
            torch.rand(m, n, **f64), torch.rand(m, n, **f64), 1.0, torch.zeros(m, **f64), torch.ones(m, **f64),
            torch.full((m,), 1000.0, **f64), torch.zeros(m, **f64))
    reachable, unreachable = {}, {}
    mma.subsolv(m, n, 1e-7, *args, reachable)
    with pytest.warns(RuntimeWarning, match="iteration cap"):
        mma.subsolv(m, n, 1e-30, *args, unreachable)
    assert reachable.get("subsolv_cap_hits", 0) == 0
    assert unreachable["subsolv_cap_hits"] > 0


def test_mma_rejects_bad_inputs(mma):
    n, m = 100, 65
    f64 = dict(dtype=torch.float64, device="cuda")
    z = torch.zeros(n, **f64)
    with pytest.raises(ValueError, match="at most 64"):
        mma.subsolv(m, n, 1e-7, z, z, z, z, z, z, torch.zeros(m, n, **f64), torch.zeros(m, n, **f64), 1.0,
                    *(torch.zeros(m, **f64) for _ in range(4)))
    with pytest.raises(ValueError, match="CUDA"):
        mma.subsolv(1, 4, 1e-7, *(torch.zeros(4, dtype=torch.float64) for _ in range(6)),
                    torch.zeros(1, 4, dtype=torch.float64), torch.zeros(1, 4, dtype=torch.float64), 1.0,
                    *(torch.zeros(1, dtype=torch.float64) for _ in range(4)))
    with pytest.raises(TypeError, match="float64"):
        mma.subsolv(1, 4, 1e-7, *(torch.zeros(4, device="cuda") for _ in range(6)),
                    torch.zeros(1, 4, device="cuda"), torch.zeros(1, 4, device="cuda"), 1.0,
                    *(torch.zeros(1, device="cuda") for _ in range(4)))

"""The coarse factorisation's side stream.

A hierarchy's coarse Cholesky (and, for FP32 cycles, its explicit inverse) runs on a
pooled stream of the library, ordered after the build on the caller's stream; the coarse
solves, the status read and the last destroy of the hierarchy wait for it.  These checks
create the orderings a caller can: a row-selected view used after its parent's handle is
destroyed, several hierarchies built back to back before any solve (the pool's streams
reused after a destroy), and V-cycles on another stream than the build's.  Each V-cycle
is compared with the same V-cycle on a hierarchy whose build was checked (synchronised)
first, at 1e-12 relative: the same kernels on the same inputs.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import sttopt_oracle as O

pytestmark = pytest.mark.gpu
EMIN, EMAX, PENAL = 1e-9, 1.0, 3.0
NELX, NELY = 48, 36


def _rel(a, b):
    return float((a - b).norm() / b.norm())


def _build(torch_mg, x, mask, precision, check):
    dev = torch.device("cuda")
    return torch_mg.build_hierarchy(
        torch.tensor(O.simp_density(x, EMIN, EMAX, PENAL), device=dev),
        torch.tensor(O.element_dof_map(NELX, NELY), device=dev),
        torch.tensor(O.plane_stress_KE(0.3), device=dev),
        torch.tensor(mask, device=dev), NELX, NELY, max_coarse_elements=20, precision=precision, check=check)


def _inputs(seed, rows):
    rng = np.random.default_rng(seed)
    x = rng.uniform(1e-3, 1.0, (rows, NELX * NELY))
    _, mask = O.cantilever_point_load(NELX, NELY)
    n = 2 * (NELX + 1) * (NELY + 1)
    r = O.project(rng.standard_normal((rows, n)), mask)
    return x, mask, torch.tensor(r, device="cuda").contiguous()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_view_outlives_its_parent_handle(pkg, precision):
    from sttopt_b200 import _lib, torch_mg

    lib = _lib.lib()
    x, mask, r = _inputs(21, 3)
    ref = torch_mg.VCycle(_build(torch_mg, x, mask, precision, True))(r)
    levels = _build(torch_mg, x, mask, precision, False)
    h = levels[0]._hier
    ws = h.ws  # the view's arrays live in the parent's workspace
    rm = torch.tensor([2, 0], dtype=torch.int32, device="cuda")
    view = ctypes.c_void_p()
    _lib.check(lib.stt_hier_select(h.handle, _lib.ptr(rm), ctypes.byref(view)))
    _lib.check(lib.stt_hier_destroy(h.handle))  # the parent's handle goes first
    h.handle = None
    n = r.shape[1]
    rv = r[[2, 0]].contiguous()
    zv = torch.full_like(rv, float("nan"))
    sws = _lib.workspace(lib.stt_solve_workspace_bytes(view, 2, 1), r.device)
    _lib.check(lib.stt_vcycle(view, 2, _lib.ptr(rv), n, _lib.ptr(zv), n, 0.6, 2, 1, _lib.ptr(sws), sws.numel(),
                              _lib.stream()))
    _lib.check(lib.stt_hier_status(view, _lib.stream()))
    _lib.check(lib.stt_hier_destroy(view))  # the last reference: waits for the factorisation
    torch.cuda.synchronize()
    del ws
    assert torch.isfinite(zv).all()
    assert _rel(zv, ref[[2, 0]]) <= 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_back_to_back_builds_reuse_the_pool(pkg, precision):
    from sttopt_b200 import torch_mg

    cases = [_inputs(30 + k, 2) for k in range(5)]
    built = [_build(torch_mg, x, mask, precision, False) for x, mask, _ in cases[:3]]
    del built[0]  # returns its stream and events to the pool before the next builds
    built = [None] + built + [_build(torch_mg, x, mask, precision, False) for x, mask, _ in cases[3:]]
    for k in range(1, 5):
        x, mask, r = cases[k]
        z = torch_mg.VCycle(built[k])(r)
        ref = torch_mg.VCycle(_build(torch_mg, x, mask, precision, True))(r)
        assert torch.isfinite(z).all()
        assert _rel(z, ref) <= 1e-12, k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cycles_on_another_stream_than_the_build(pkg, precision):
    from sttopt_b200 import torch_mg

    x, mask, r = _inputs(44, 3)
    ref = torch_mg.VCycle(_build(torch_mg, x, mask, precision, True))(r)
    levels = _build(torch_mg, x, mask, precision, False)
    other = torch.cuda.Stream()
    other.wait_stream(torch.cuda.current_stream())  # the levels and r (the caller's ordering)
    with torch.cuda.stream(other):
        z = torch_mg.VCycle(levels)(r)
    torch.cuda.current_stream().wait_stream(other)
    torch.cuda.synchronize()
    assert torch.isfinite(z).all()
    assert _rel(z, ref) <= 1e-12

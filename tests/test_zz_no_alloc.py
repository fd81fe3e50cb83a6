"""The V-cycle entry point that allocates nothing (``stt_vcycle_noalloc``).

Callers that cannot allocate device memory -- plugins in a host application that owns
the device memory pool, pipelines that cannot take cudaMalloc's implicit device
synchronisation mid-run, bindings that can hand over only inputs and outputs -- call
this variant; its scratch is a fixed 32 MiB array inside the library.
These checks call it through the C ABI and compare it with ``stt_vcycle`` (which runs
the same kernels in a caller workspace) on two calls in a row, at the V-cycle tolerance
of the parity tests (1e-10 relative).  The file is named to be collected last.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import sttopt_oracle as O

pytestmark = pytest.mark.gpu
EMIN, EMAX, PENAL = 1e-9, 1.0, 3.0


def _rel(a, b):
    return float((a - b).norm() / b.norm())


def test_vcycle_noalloc_matches_the_workspace_entry_point(pkg):
    from sttopt_b200 import _lib, torch_mg

    lib = _lib.lib()
    nelx, nely = 48, 36
    rng = np.random.default_rng(5)
    x = rng.uniform(1e-3, 1.0, (3, nelx * nely))
    F, mask = O.cantilever_point_load(nelx, nely)
    dev = torch.device("cuda")
    for precision in ("fp64", "mixed"):
        levels = torch_mg.build_hierarchy(
            torch.tensor(O.simp_density(x, EMIN, EMAX, PENAL), device=dev),
            torch.tensor(O.element_dof_map(nelx, nely), device=dev),
            torch.tensor(O.plane_stress_KE(0.3), device=dev),
            torch.tensor(mask, device=dev), nelx, nely, max_coarse_elements=20, precision=precision)
        h = levels[0]._hier
        n = levels[0].ndof
        r = torch.tensor(O.project(rng.standard_normal((3, n)), mask), device=dev).contiguous()
        ws = _lib.workspace(lib.stt_solve_workspace_bytes(h.handle, 3, 1), dev)
        z_ref = torch.empty_like(r)
        _lib.check(lib.stt_vcycle(h.handle, 3, _lib.ptr(r), n, _lib.ptr(z_ref), n, 0.6, 2, 1,
                                  _lib.ptr(ws), ws.numel(), _lib.stream()))
        for _ in range(2):  # two calls in a row share the library's scratch
            z = torch.full_like(r, float("nan"))
            _lib.check(lib.stt_vcycle_noalloc(h.handle, 3, _lib.ptr(r), n, _lib.ptr(z), n, 0.6, 2, 1,
                                              _lib.stream()))
            torch.cuda.synchronize()
            assert torch.isfinite(z).all()
            assert _rel(z, z_ref) <= 1e-10, precision


def test_vcycle_noalloc_rejects_sizes_beyond_its_scratch(pkg):
    from sttopt_b200 import _lib, torch_mg

    lib = _lib.lib()
    nelx, nely = 512, 256
    dev = torch.device("cuda")
    F, mask = O.cantilever_point_load(nelx, nely)
    levels = torch_mg.build_hierarchy(
        torch.full((nelx * nely,), 0.5, dtype=torch.float64, device=dev),
        torch.tensor(O.element_dof_map(nelx, nely), device=dev),
        torch.tensor(O.plane_stress_KE(0.3), device=dev), torch.tensor(mask, device=dev), nelx, nely)
    h = levels[0]._hier
    rows = 16
    assert lib.stt_solve_workspace_bytes(h.handle, rows, 1) > 32 << 20
    r = torch.zeros(rows, levels[0].ndof, dtype=torch.float64, device=dev)
    z = torch.empty_like(r)
    rc = lib.stt_vcycle_noalloc(h.handle, rows, _lib.ptr(r), r.shape[1], _lib.ptr(z), r.shape[1], 0.6, 2,
                                1, _lib.stream())
    assert rc == _lib.STT_ERR_WORKSPACE
    assert b"32 MiB" in lib.stt_last_error()

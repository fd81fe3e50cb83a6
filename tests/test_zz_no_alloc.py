"""The V-cycle entry point that allocates nothing (``stt_vcycle_noalloc``).

Callers that cannot allocate device memory -- plugins in a host application that owns
the device memory pool, pipelines that cannot take cudaMalloc's implicit device
synchronisation mid-run, bindings that can hand over only inputs and outputs -- call
this variant; its scratch is a fixed 32 MiB array inside the library.
These checks call it through the C ABI and compare it with ``stt_vcycle`` (which runs
the same kernels in a caller workspace) on two calls in a row, at the V-cycle tolerance
of the parity tests (1e-10 relative).  The shared array keeps the previous call's
contents, so a call on a larger hierarchy with a NaN residual first leaves NaN under
the next calls' buffers: any scratch word read before it is written would show.  The
workspace entry point is also run on a workspace filled with NaN bytes.  The file is
named to be collected last.
"""

import numpy as np
import pytest
import torch

from oracle import sttopt_oracle as O

pytestmark = pytest.mark.gpu
EMIN, EMAX, PENAL = 1e-9, 1.0, 3.0


def _rel(a, b):
    return float((a - b).norm() / b.norm())


def _hierarchy(nelx, nely, rows, precision, seed, mce=20):
    from sttopt_b200 import torch_mg

    dev = torch.device("cuda")
    rng = np.random.default_rng(seed)
    x = rng.uniform(1e-3, 1.0, (rows, nelx * nely))
    _, mask = O.cantilever_point_load(nelx, nely)
    levels = torch_mg.build_hierarchy(
        torch.tensor(O.simp_density(x, EMIN, EMAX, PENAL), device=dev),
        torch.tensor(O.element_dof_map(nelx, nely), device=dev),
        torch.tensor(O.plane_stress_KE(0.3), device=dev),
        torch.tensor(mask, device=dev), nelx, nely, max_coarse_elements=mce, precision=precision)
    r = torch.tensor(O.project(rng.standard_normal((rows, levels[0].ndof)), mask), device=dev).contiguous()
    return levels, r


def test_vcycle_noalloc_matches_the_workspace_entry_point(pkg):
    from sttopt_b200 import _lib

    lib = _lib.lib()
    for precision in ("fp64", "mixed"):
        # the workspace entry point on a workspace of NaN bytes against one of zeros, on two
        # identical hierarchies: no word is read unwritten.  Two cycles each, as an FP32
        # hierarchy's first coarse solve takes the block solves and later ones its inverse.
        (levels, r), (twin, _) = _hierarchy(48, 36, 3, precision, 5), _hierarchy(48, 36, 3, precision, 5)
        h, n = levels[0]._hier, levels[0].ndof
        outs = {}
        for key, hh, fill in (("nan", h, 255), ("zero", twin[0]._hier, 0)):
            ws = _lib.workspace(lib.stt_vcycle_workspace_bytes(hh.handle, 3, 1), r.device)
            ws.fill_(fill)
            zs = []
            for _ in range(2):
                z = torch.empty_like(r)
                _lib.check(lib.stt_vcycle(hh.handle, 3, _lib.ptr(r), n, _lib.ptr(z), n, 0.6, 2, 1,
                                          _lib.ptr(ws), ws.numel(), _lib.stream()))
                zs.append(z)
            outs[key] = zs
        torch.cuda.synchronize()
        for k in range(2):
            assert torch.isfinite(outs["nan"][k]).all()
            assert torch.equal(outs["nan"][k], outs["zero"][k])
        z_ref = outs["nan"][1]
        # a larger hierarchy with a NaN residual fills the shared scratch with NaN first
        big, rb = _hierarchy(160, 96, 4, precision, 6)
        hb, nb = big[0]._hier, big[0].ndof
        assert lib.stt_vcycle_workspace_bytes(hb.handle, 4, 1) > lib.stt_vcycle_workspace_bytes(h.handle, 3, 1)
        rb.fill_(float("nan"))
        zb = torch.empty_like(rb)
        _lib.check(lib.stt_vcycle_noalloc(hb.handle, 4, _lib.ptr(rb), nb, _lib.ptr(zb), nb, 0.6, 2, 1,
                                          _lib.stream()))
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
    assert lib.stt_vcycle_workspace_bytes(h.handle, rows, 1) > 32 << 20
    r = torch.zeros(rows, levels[0].ndof, dtype=torch.float64, device=dev)
    z = torch.empty_like(r)
    rc = lib.stt_vcycle_noalloc(h.handle, rows, _lib.ptr(r), r.shape[1], _lib.ptr(z), r.shape[1], 0.6, 2,
                                1, _lib.stream())
    assert rc == _lib.STT_ERR_WORKSPACE
    assert b"32 MiB" in lib.stt_last_error()
    # the V-cycle's own plan is smaller than the PCG's, which the fixed array need not hold
    assert lib.stt_vcycle_workspace_bytes(h.handle, 2, 1) < lib.stt_solve_workspace_bytes(h.handle, 2, 1)

"""CPU-only checks of the boundary: the C-ABI library loads and exports every entry
point ``include/sttb200.h`` declares, the Python binding covers them all, and the host
logic (hierarchy planning, row accounting) matches the reference's policies.  No
compute is launched here."""

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from oracle import sttopt_oracle as O

HEADER = ROOT / "include" / "sttb200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(stt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(pkg):
    from sttopt_b200 import _lib

    lib = _lib.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(_lib.exported_symbols()) == declared_symbols()


def declared_arity():
    """Parameter count of every prototype in the header."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(stt_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        params = params.strip()
        out[name] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_argument_counts_match_the_header(pkg):
    """Every ctypes signature has as many arguments as its C prototype (an argument past
    the declared ones would be passed as a 32-bit int)."""
    from sttopt_b200 import _lib

    arity = declared_arity()
    assert set(arity) == set(declared_symbols())
    wrong = {n: (len(args), arity[n]) for n, (_, args) in _lib._SIGS.items() if len(args) != arity[n]}
    assert not wrong, wrong


def test_workspace_planning_follows_the_reference_policy(pkg):
    from sttopt_b200 import _lib

    lib = _lib.lib()
    # sizes are positive and grow with rows; invalid shapes are rejected
    a = lib.stt_hier_workspace_bytes(2, 120, 40, 1, 700, 0)
    b = lib.stt_hier_workspace_bytes(2, 120, 40, 4, 700, 0)
    c = lib.stt_hier_workspace_bytes(2, 120, 40, 4, 700, 1)
    assert 0 < a < b < c
    assert lib.stt_hier_workspace_bytes(3, 120, 40, 1, 700, 0) < 0
    assert lib.stt_hier_workspace_bytes(2, 0, 40, 1, 700, 0) < 0


def test_invalid_arguments_fail_without_a_device(pkg):
    from sttopt_b200 import _lib

    lib = _lib.lib()
    rc = lib.stt_q4_apply(0, 3, 4, 4, 1, None, 0, None, 0, None, 0, None, 0, None, 0, None, None)
    assert rc == _lib.STT_ERR_INVALID
    assert b"stt_q4_apply" in lib.stt_last_error()
    out = ctypes.c_void_p()
    rc = lib.stt_hier_create(ctypes.byref(out), None, 0, 2, 4, 4, 1, None, 0, None, 0, None, None,
                             700, 0, None)
    assert rc == _lib.STT_ERR_INVALID


@pytest.mark.parametrize("sizes", [(2048, 1024), (1024, 512), (512, 256), (120, 40), (768, 384),
                                   (1536, 768), (256, 128), (30, 10), (97, 89)])
def test_coarsening_policy_matches_oracle(pkg, sizes):
    from sttopt_b200 import torch_mg

    nelx, nely = sizes
    assert torch_mg.coarsening_factors(nelx, nely) == O.coarsening_factors(nelx, nely)


def test_child_interpolation_matches_golden_bitwise(pkg):
    from sttopt_b200 import torch_mg

    g = golden("transfers")
    for kx, ky in [(2, 2), (3, 3), (3, 1), (2, 3), (1, 2)]:
        for d in (1, 2):
            S = torch_mg.child_interpolation_matrices(kx, ky, dofs_per_node=d).numpy()
            np.testing.assert_array_equal(S, g[f"S_k{kx}{ky}_d{d}"])


def test_row_iters_schedule_matches_reference(pkg):
    from sttopt_b200 import torch_fem

    g = golden("pcg_cases")
    # per-row convergence iterations of the oracle run that the reference recorded
    nelx, nely = 18, 12
    edof = O.element_dof_map(nelx, nely)
    KE = O.plane_stress_KE(0.3)
    conv = []
    for s in range(3):
        if not np.any(g["F"][s]):
            conv.append(0)
            continue
        _, n = O.mg_solve(g["F"][s], g["x"][s], edof, KE, 1e-9, 1.0, 3.0, g["mask"], nelx, nely,
                          rtol=1e-11, max_coarse_elements=24)
        conv.append(n)
    assert torch_fem.row_iters_from_schedule(conv, 3, 500) == int(g["row_iters"])
    assert torch_fem.row_iters_from_schedule([0, 0], 2, 500) == 0
    assert torch_fem.row_iters_from_schedule([5], 1, 500) == 5


def test_package_refuses_cpu_tensors(pkg):
    import torch

    from sttopt_b200 import torch_fem

    KE = torch.tensor(O.plane_stress_KE(0.3))
    edof = torch.tensor(O.element_dof_map(4, 3))
    with pytest.raises(ValueError, match="CUDA"):
        torch_fem.matvec(torch.zeros(40, dtype=torch.float64), torch.ones(12, dtype=torch.float64),
                         edof, KE, 40)


def test_modal_form_recognises_the_reference_element_matrices(pkg):
    """stt_ke_modal accepts the plane-stress KE for any nu and the diffusion KE, and
    rebuilds them exactly from the modal constants; a general SPD KE is rejected."""
    from sttopt_b200 import _lib

    lib = _lib.lib()
    pat = np.array([[-1, 1, 1, -1], [-1, -1, 1, 1], [1, -1, 1, -1]], dtype=np.float64)

    def modal(d, KE):
        m = (ctypes.c_double * 8)()
        ok = lib.stt_ke_modal(d, _lib.dbl_array(np.ascontiguousarray(KE).ravel().tolist()), m)
        return ok, np.array(m[:])

    for nu in (0.0, 0.25, 0.3, 0.45):
        KE = O.plane_stress_KE(nu)
        ok, m = modal(2, KE)
        assert ok == 1, nu
        T = np.zeros((6, 8))
        T[0, 0::2], T[1, 1::2], T[2, 0::2], T[3, 1::2], T[4, 0::2], T[5, 1::2] = pat[0], pat[1], pat[1], pat[0], pat[2], pat[2]
        M = np.zeros((6, 6))
        M[0, 0], M[0, 1], M[1, 0], M[1, 1] = m[0], m[1], m[1], m[2]
        M[2:4, 2:4] = m[3]
        M[4, 4], M[5, 5] = m[4], m[5]
        assert np.abs(T.T @ M @ T - KE).max() < 1e-15
        assert m[6] == m[7] == KE[0, 0]
    ok, m = modal(1, O.diffusion_KE())
    assert ok == 1
    assert np.abs(pat.T @ np.diag([m[0], m[2], m[3]]) @ pat - O.diffusion_KE()).max() < 1e-15
    rng = np.random.default_rng(0)
    A = rng.standard_normal((8, 8))
    assert modal(2, A @ A.T)[0] == 0
    KE = O.plane_stress_KE(0.3).copy()
    KE[0, 3] += 1e-9
    KE[3, 0] += 1e-9
    assert modal(2, KE)[0] == 0


def test_host_conversions_are_memoised_per_tensor_object(pkg):
    """Element-matrix and grid conversions are cached on the tensor object and follow
    in-place edits; a new tensor never inherits another tensor's cached result (torch's
    allocator reuses freed addresses, so an address-keyed cache would)."""
    import torch

    from sttopt_b200 import _geom

    a = torch.tensor(O.plane_stress_KE(0.3))
    va = _geom.host_KE(a)
    assert va == tuple(O.plane_stress_KE(0.3).ravel())
    a.mul_(2.0)
    assert _geom.host_KE(a) == tuple((2.0 * O.plane_stress_KE(0.3)).ravel())
    for nu in (0.1, 0.2, 0.3):
        b = torch.tensor(O.plane_stress_KE(nu))
        assert _geom.host_KE(b) == tuple(O.plane_stress_KE(nu).ravel())
        del b
    e1 = torch.as_tensor(O.element_dof_map(6, 4))
    assert _geom.grid_shape(e1, 2 * 7 * 5, 2) == (6, 4)
    e2 = torch.as_tensor(O.element_dof_map(4, 6))
    assert _geom.grid_shape(e2, 2 * 5 * 7, 2) == (4, 6)


def test_mma_entry_points_size_and_validate_without_a_device(pkg):
    """``stt_mma_*``: the workspace grows with the variables and the constraints, and bad
    sizes, null pointers or a short workspace are refused before any CUDA call."""
    from sttopt_b200 import _lib

    lib = _lib.lib()
    a, b, c = (lib.stt_mma_workspace_bytes(m, n) for m, n in ((17, 1 << 20), (17, 1 << 22), (40, 1 << 22)))
    assert 0 < a < b < c
    assert b >= 4 * 8 * (1 << 22)  # alfa, beta, raa0 / range and dx
    assert lib.stt_mma_workspace_bytes(0, 100) == 0 and lib.stt_mma_workspace_bytes(3, 0) == 0
    need = lib.stt_mma_workspace_bytes(3, 1000)

    def subsolv(m, ws_bytes):
        # m, n, epsimin, low upp alfa beta p0 q0 P Q, ld, a0, a b c d, x xsi eta y z lam mu zet s,
        # counts, cap_epsi, ws, ws_bytes, stream
        return lib.stt_mma_subsolv(m, 1000, 1e-7, *[None] * 8, 1000, 1.0, *[None] * 4, *[None] * 9, None, None,
                                   None, ws_bytes, None)

    def sub(m, ws_bytes):
        # m, n, iteration, xval xmin xmax xold1 xold2 df0dx fval dfdx, ld, low upp, a0, a c d,
        # four (pointer, value) keywords, raa0 albefa asyincr asydecr, 9 outputs, counts,
        # cap_epsi, ws, ws_bytes, stream
        return lib.stt_mma_sub(m, 1000, 0, *[None] * 8, 1000, None, None, 1.0, None, None, None, None, 0.5, None,
                               0.01, None, 10.0, None, 0.5, 1e-5, 0.1, 1.2, 0.7, *[None] * 9, None, None, None,
                               ws_bytes, None)

    assert subsolv(65, 1 << 30) == _lib.STT_ERR_INVALID  # m < n beyond 64 constraints
    assert b"64" in lib.stt_last_error()
    assert subsolv(3, need - 1) == _lib.STT_ERR_WORKSPACE
    assert subsolv(3, need) == _lib.STT_ERR_INVALID  # null pointers
    assert b"null pointer" in lib.stt_last_error()
    assert sub(3, need - 1) == _lib.STT_ERR_WORKSPACE
    assert sub(3, need) == _lib.STT_ERR_INVALID
    assert sub(0, need) == _lib.STT_ERR_INVALID

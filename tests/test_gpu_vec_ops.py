"""The PCG vector steps for arbitrary operators (``stt_vec_dots``, ``stt_vec_cg_update``,
``stt_vec_xpay``) against torch FP64 on the same inputs: dots to 1e-13 relative (the
kernels sum in another, fixed order), updates to three units in the last place of the
terms' magnitude (the kernels may fuse the multiply-add into one rounding).  The dot
cases cover one to three pairs, the shared-first-operand pass (two pairs with the same
first vector, 128-bit loads) at even and odd lengths, a single row with an odd stride,
and padded row strides."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _rows(g, rows, n, rs):
    buf = torch.randn(rows, rs, generator=g, dtype=torch.float64).cuda()
    return buf, buf[:, :n]


@pytest.mark.parametrize("rows,n,rs", [(1, 2_100_225, 2_100_225), (3, 4_200_450, 4_200_450),
                                       (4, 1001, 1002), (2, 999, 999), (5, 64, 70)])
def test_vec_dots_match_torch(pkg, rows, n, rs):
    from sttopt_b200 import _lib

    lib = _lib.lib()
    g = torch.Generator().manual_seed(rows * 7 + n)
    (A, a), (B0, b0), (B1, b1), (B2, b2) = (_rows(g, rows, n, rs) for _ in range(4))
    ref = [(a * b0).sum(1), (a * b1).sum(1), (a * b2).sum(1), (b0 * b1).sum(1)]
    scale = [(a.abs() * b.abs()).sum(1) for b in (b0, b1, b2)] + [(b0.abs() * b1.abs()).sum(1)]

    def dots(pairs):
        out = torch.full((rows, len(pairs)), float("nan"), dtype=torch.float64, device="cuda")
        ptrs = [_lib.ptr(p) for pair in pairs for p in pair] + [None] * (6 - 2 * len(pairs))
        _lib.check(lib.stt_vec_dots(rows, n, *ptrs, rs, _lib.ptr(out), _lib.stream()))
        torch.cuda.synchronize()
        return out

    cases = [([(A, B0)], [0]), ([(A, B0), (A, B1)], [0, 1]), ([(A, B0), (B0, B1)], [0, 3]),
             ([(A, B0), (A, B1), (A, B2)], [0, 1, 2])]
    for pairs, idx in cases:
        out = dots(pairs)
        for j, k in enumerate(idx):
            err = (out[:, j] - ref[k]).abs() / scale[k]
            assert float(err.max()) <= 1e-13, (len(pairs), k)


def _close(out, ref, mag):
    return bool(((out - ref).abs() <= 6.7e-16 * mag).all())


def test_vec_cg_update_and_xpay_match_torch(pkg):
    from sttopt_b200 import _lib

    lib = _lib.lib()
    g = torch.Generator().manual_seed(3)
    rows, n = 3, 100_003
    x, r, p, Ap = (torch.randn(rows, n, generator=g, dtype=torch.float64).cuda() for _ in range(4))
    alpha = torch.tensor([0.5, -1.25, 3.0], dtype=torch.float64, device="cuda")
    x_ref, r_ref = x + alpha[:, None] * p, r - alpha[:, None] * Ap
    rr = torch.empty(rows, dtype=torch.float64, device="cuda")
    _lib.check(lib.stt_vec_cg_update(rows, n, _lib.ptr(alpha), _lib.ptr(x), _lib.ptr(r), _lib.ptr(p), _lib.ptr(Ap),
                                     n, _lib.ptr(rr), _lib.stream()))
    torch.cuda.synchronize()
    assert _close(x, x_ref, x_ref.abs() + (alpha[:, None] * p).abs())
    assert _close(r, r_ref, r_ref.abs() + (alpha[:, None] * Ap).abs())
    assert float(((rr - (r_ref * r_ref).sum(1)).abs() / (r_ref * r_ref).sum(1)).max()) <= 1e-13
    z = torch.randn(rows, n, generator=g, dtype=torch.float64).cuda()
    beta = torch.tensor([0.0, 2.0, -0.5], dtype=torch.float64, device="cuda")
    p_ref = p * beta[:, None] + z
    _lib.check(lib.stt_vec_xpay(rows, n, _lib.ptr(z), _lib.ptr(beta), _lib.ptr(p), n, _lib.stream()))
    torch.cuda.synchronize()
    assert _close(p, p_ref, p_ref.abs() + z.abs())


@pytest.mark.parametrize("d,form", [(2, "modal"), (2, "product"), (1, "modal")])
def test_apply_dots_and_warm_start(pkg, d, form):
    """``stt_q4_apply_dots`` (the stage adjoint's load 2 K U with U . gK and U . F in one
    pass) against ``stt_q4_apply`` (projected output) bit for bit and the dots against
    torch to 1e-13; ``stt_adjoint_warm_start`` against alpha U with alpha the reference's
    safe_div, including a row whose U . F is zero (alpha 0)."""
    import numpy as np

    from oracle import sttopt_oracle as O
    from sttopt_b200 import _lib, element_form, fem

    lib = _lib.lib()
    nelx, nely, rows = 300, 170, 3
    nnode = (nelx + 1) * (nely + 1)
    n = d * nnode
    g = torch.Generator().manual_seed(d * 11)
    rho = torch.rand(rows, nelx * nely, generator=g, dtype=torch.float64).cuda() + 1e-3
    KE = fem.plane_stress_KE(0.3) if d == 2 else fem.diffusion_KE()
    ke2 = _lib.dbl_array([2.0 * v for v in np.asarray(KE).ravel()])
    fixed = torch.zeros(nnode, dtype=torch.uint8)
    fixed[-(nelx + 1):] = (1 << d) - 1  # the bottom row clamped
    fixed = fixed.cuda()
    mask = torch.ones(rows, nnode, d, dtype=torch.float64)
    mask[:, -(nelx + 1):, :] = 0.0
    mask = mask.reshape(rows, n).cuda()
    U = torch.randn(rows, n, generator=g, dtype=torch.float64).cuda() * mask
    F = torch.randn(rows, n, generator=g, dtype=torch.float64).cuda() * mask
    F[2] = 0.0
    st = _lib.stream()
    with element_form(form):
        ref = torch.empty_like(U)
        _lib.check(lib.stt_q4_apply(_lib.STT_FP64, d, nelx, nely, rows, _lib.ptr(U), n, _lib.ptr(ref), n,
                                    _lib.ptr(rho), nelx * nely, None, 0, _lib.ptr(fixed), _lib.STT_PROJECT_OUT,
                                    ke2, st))
        out = torch.full_like(U, float("nan"))
        dots = torch.full((rows, 2), float("nan"), dtype=torch.float64, device="cuda")
        ws = _lib.workspace(lib.stt_q4_apply_dots_workspace_bytes(nelx, nely, rows), U.device)
        ws.fill_(255)  # the counters are reset by the call
        for _ in range(2):  # a second call reuses the workspace
            _lib.check(lib.stt_q4_apply_dots(d, nelx, nely, rows, _lib.ptr(U), n, _lib.ptr(out), n, _lib.ptr(rho),
                                             nelx * nely, _lib.ptr(fixed), ke2, _lib.ptr(F), n, _lib.ptr(dots),
                                             _lib.ptr(ws), ws.numel(), st))
        torch.cuda.synchronize()
    assert torch.equal(out, ref)
    want = torch.stack([(U * ref).sum(1), (U * F).sum(1)], dim=1)
    scale = torch.stack([(U * ref).abs().sum(1), (U * F).abs().sum(1)], dim=1)
    assert float(((dots - want).abs() / scale.clamp_min(1e-300)).max()) < 1e-13
    x0 = torch.full_like(U, float("nan"))
    _lib.check(lib.stt_adjoint_warm_start(rows, n, _lib.ptr(dots), _lib.ptr(U), n, _lib.ptr(x0), n, st))
    torch.cuda.synchronize()
    alpha = torch.where(dots[:, 1] != 0, dots[:, 0] / torch.where(dots[:, 1] != 0, dots[:, 1], 1.0), 0.0)
    assert torch.equal(x0, alpha[:, None] * U)
    assert torch.all(x0[2] == 0.0)

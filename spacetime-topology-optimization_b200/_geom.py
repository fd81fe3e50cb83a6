"""Host-side helpers shared by the drop-in modules: grid shape from an element dof map,
host copies of element matrices, and per-node "fixed" flags from a free-dof mask.

The reference's functions take ``edofMat``/``KE``/``mask`` tensors; the kernels need
the grid shape, the element matrix as a small host array and a byte of flags per
node.  Each conversion is memoised on the tensor object itself (keyed on its version
counter), so a solve loop pays the device-to-host read once, and a new tensor that
reuses a freed tensor's memory never sees the old tensor's result.
"""

from __future__ import annotations

import numpy as np
import torch

from . import fem

_MEMO = "_sttb200_memo"


def _memo_get(t: torch.Tensor, key):
    store = getattr(t, _MEMO, None)
    return None if store is None else store.get((t._version,) + key)


def _memo_put(t: torch.Tensor, key, value):
    store = getattr(t, _MEMO, None)
    if store is None:
        store = {}
        try:
            setattr(t, _MEMO, store)
        except (AttributeError, TypeError):  # a tensor subclass without a __dict__: no memo
            return value
    if len(store) > 8:
        store.clear()
    store[(t._version,) + key] = value
    return value


def grid_shape(edofMat: torch.Tensor, ndof: int, dofs_per_node: int) -> tuple[int, int]:
    """``(nelx, nely)`` of the structured grid ``edofMat`` maps; checks it is the
    reference's map (sttopt/fem.py:72-95) -- the kernels handle no other."""
    key = ("grid", ndof, dofs_per_node)
    hit = _memo_get(edofMat, key)
    if hit is not None:
        return hit
    d = dofs_per_node
    nel = edofMat.shape[0]
    nelx = int(edofMat[0, 0].item()) // d - 1
    if nelx <= 0 or nel % nelx:
        raise ValueError("edofMat is not a structured Q4 grid dof map")
    nely = nel // nelx
    if d * (nelx + 1) * (nely + 1) != ndof:
        raise ValueError(f"edofMat ({nelx}x{nely}) does not match ndof={ndof}")
    expect = torch.as_tensor(fem.element_dof_map(nelx, nely, d), device=edofMat.device)
    if not torch.equal(edofMat.to(expect.dtype), expect):
        raise ValueError("edofMat is not the reference's element dof map of a structured grid")
    return _memo_put(edofMat, key, (nelx, nely))


def host_KE(KE: torch.Tensor) -> tuple[float, ...]:
    """Element matrix as a flat tuple of doubles (row-major); must be symmetric."""
    key = ("KE",)
    hit = _memo_get(KE, key)
    if hit is not None:
        return hit
    k = KE.detach().to("cpu", torch.float64).numpy()
    if k.ndim != 2 or k.shape[0] != k.shape[1] or k.shape[0] not in (4, 8):
        raise ValueError("KE must be 4x4 (scalar) or 8x8 (plane stress)")
    if not np.array_equal(k, k.T):
        raise ValueError("KE must be exactly symmetric")
    return _memo_put(KE, key, tuple(float(v) for v in k.ravel()))


def fixed_flags(mask: torch.Tensor | None, nnode: int, d: int) -> torch.Tensor | None:
    """One byte per node, bit ``i`` set when dof ``i`` is fixed (``mask`` False)."""
    if mask is None:
        return None
    key = ("flags", nnode, d)
    hit = _memo_get(mask, key)
    if hit is not None:
        return hit
    fixed = (~mask.to(torch.bool)).reshape(nnode, d).to(torch.uint8)
    flags = fixed[:, 0].clone()
    for i in range(1, d):
        flags |= fixed[:, i] << i
    return _memo_put(mask, key, flags.contiguous())


def rows2d(t: torch.Tensor, n: int) -> tuple[torch.Tensor, int]:
    """``t`` viewed as ``(rows, n)`` with unit inner stride; returns the row stride
    (0 for a broadcast row)."""
    if t.shape[-1] != n:
        raise ValueError(f"last dim {t.shape[-1]} != {n}")
    flat = t.reshape(-1, n)
    if flat.stride(-1) != 1 or flat.data_ptr() % 16 or (flat.shape[0] > 1 and flat.stride(0) % 2):
        flat = flat.contiguous()
    rs = flat.stride(0) if flat.shape[0] > 1 else n
    return flat, rs

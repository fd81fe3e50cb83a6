"""Compact pins of large fields for the benchmark-size fixtures.

A field of millions of values is stored as its sum, its L2 norm, ``N_PROJ`` seeded
Gaussian projections ``V @ a`` and a strided subsample.  For a computed field ``b`` the
projections give ``V @ (b - a)``, whose entries are each about ``||b - a||`` in size, so
``max_k |V_k @ b - V_k @ a| / ||a||`` estimates the relative L2 error of the whole field
(and a single wrong value of size ``e`` shows up as ~``e``) without storing the field.
The generator (``make_golden.py``) and the tests share these two functions.
"""

from __future__ import annotations

import numpy as np

N_PROJ = 4


def _vectors(n: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).standard_normal((N_PROJ, n))


def field_summary(prefix: str, a, seed: int, stride: int) -> dict:
    """``{prefix_sum, prefix_norm, prefix_proj, prefix_sub, prefix_stride, prefix_seed}``
    of the flattened field ``a``."""
    a = np.asarray(a, dtype=np.float64).ravel()
    return {f"{prefix}_sum": a.sum(), f"{prefix}_norm": np.linalg.norm(a),
            f"{prefix}_proj": _vectors(a.size, seed) @ a, f"{prefix}_sub": a[::stride].copy(),
            f"{prefix}_stride": stride, f"{prefix}_seed": seed, f"{prefix}_n": a.size}


def summary_error(prefix: str, g: dict, b) -> dict:
    """Errors of the computed field ``b`` against the stored summary ``prefix`` of ``g``:
    ``proj`` (relative L2 estimate from the projections), ``sub`` (relative L2 error of the
    subsample) and ``sub_max`` (largest elementwise error of the subsample relative to the
    field's largest subsampled magnitude)."""
    b = np.asarray(b, dtype=np.float64).ravel()
    n = int(g[f"{prefix}_n"])
    if b.size != n:
        raise ValueError(f"{prefix}: field of {b.size} values, fixture has {n}")
    norm = float(g[f"{prefix}_norm"])
    proj = _vectors(n, int(g[f"{prefix}_seed"])) @ b
    sub_ref = g[f"{prefix}_sub"]
    sub = b[::int(g[f"{prefix}_stride"])]
    scale = float(np.abs(sub_ref).max()) or 1.0
    return {"proj": float(np.abs(proj - g[f"{prefix}_proj"]).max() / norm),
            "sub": float(np.linalg.norm(sub - sub_ref) / (np.linalg.norm(sub_ref) or 1.0)),
            "sub_max": float(np.abs(sub - sub_ref).max() / scale),
            "norm": abs(float(np.linalg.norm(b)) - norm) / norm}

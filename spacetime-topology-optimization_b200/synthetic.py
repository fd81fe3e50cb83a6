"""Seeded synthetic inputs of the benchmark configurations.

Density: ``numpy.random.default_rng(seed)`` N(0, 1) noise on the ``(nely, nelx)`` element
grid, smoothed by the radius-``rmin`` cone filter ``H x / Hs`` with
``H[e1, e2] = max(0, rmin - dist)`` over offsets ``|d| <= ceil(rmin) - 1``
(sttopt/filters.py:38-76, a zero-padded correlation), then min-max mapped to
``[lo, hi]``.  The filter runs on the device as a 2-D correlation.
"""

from __future__ import annotations

import math

import numpy as np
import torch


def cone_weights(rmin: float) -> np.ndarray:
    r = int(math.ceil(rmin)) - 1
    k = np.zeros((2 * r + 1, 2 * r + 1))
    for di in range(-r, r + 1):
        for dj in range(-r, r + 1):
            k[dj + r, di + r] = max(0.0, rmin - math.hypot(di, dj))
    return k


def smoothed_density(nelx: int, nely: int, seed: int, *, rmin: float = 4.0, lo: float = 1e-3,
                     hi: float = 1.0, device="cuda") -> torch.Tensor:
    noise = np.random.default_rng(seed).standard_normal((nely, nelx))
    k = torch.tensor(cone_weights(rmin), dtype=torch.float64, device=device)[None, None]
    r = k.shape[-1] // 2
    x = torch.tensor(noise, dtype=torch.float64, device=device)[None, None]
    num = torch.nn.functional.conv2d(x, k, padding=r)
    den = torch.nn.functional.conv2d(torch.ones_like(x), k, padding=r)
    sm = (num / den)[0, 0]
    sm = (sm - sm.min()) / (sm.max() - sm.min())
    return lo + (hi - lo) * sm


def time_weights(nelx: int, nely: int, seed: int, device="cuda") -> torch.Tensor:
    """Seeded ``w ~ U(-1, 1)`` of the time-field term ``sum(w * tPhys)``."""
    w = np.random.default_rng(seed).uniform(-1, 1, (nely, nelx))
    return torch.tensor(w, dtype=torch.float64, device=device)

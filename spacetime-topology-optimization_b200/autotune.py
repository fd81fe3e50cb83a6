"""Launch-shape autotuner of the device solves.

Two launch shapes of a solve are runtime choices (``stt_hier_tune``): the grid rows a
block of the PCG's level-0 passes marches (8, 16 or 32), and how many waves of blocks the
stencil levels' kernels aim at (their band heights follow from it).  The library's
built-in heuristics pick them from the grid and the batch rows; this module picks them by
measurement: for a hierarchy it times a few PCG iterations of each candidate on the
hierarchy itself (CUDA events on the current stream, the heuristic always among the
candidates, best of two sweeps) and caches the fastest per key
``(dofs per node, nelx, nely, precision, batch rows, gamma)``.  Launch shapes change no
result beyond the order of the blocks' partial sums.

Modes: off (default; the heuristics), ``enable()`` (tune every key the solves meet the
first time, then reuse it), ``freeze()`` (apply cached choices, tune nothing new).  The
environment variable ``STT_AUTOTUNE=1`` starts enabled.  ``cache()`` returns the choices,
``save``/``load`` keep them as JSON.
"""

from __future__ import annotations

import ctypes
import json
import os
import threading

import torch

from . import _lib

PCG_BANDS = (0, 8, 16, 32)
LEVEL_WAVES = (0, 2, 8)
ITERS = 3

_CACHE: dict = {}
_LOCK = threading.Lock()
_MODE = "enabled" if os.environ.get("STT_AUTOTUNE") == "1" else "off"


def enable() -> None:
    global _MODE
    _MODE = "enabled"


def freeze() -> None:
    global _MODE
    _MODE = "frozen"


def disable() -> None:
    global _MODE
    _MODE = "off"


def mode() -> str:
    return _MODE


def cache() -> dict:
    """``{key: {"pcg_band": .., "level_waves": .., "ms": {candidate: ms}}}`` as strings."""
    with _LOCK:
        return {repr(k): dict(v) for k, v in _CACHE.items()}


def save(path: str) -> None:
    with _LOCK:
        data = [[list(k), v["pcg_band"], v["level_waves"]] for k, v in _CACHE.items()]
    with open(path, "w") as f:
        json.dump(data, f)


def load(path: str) -> None:
    with open(path) as f:
        data = json.load(f)
    with _LOCK:
        for k, band, waves in data:
            _CACHE[tuple(k)] = {"pcg_band": int(band), "level_waves": int(waves), "ms": {}}


def _key(h, rows: int, gamma: int) -> tuple:
    nelx, nely = h.dims[0][0], h.dims[0][1]
    return (h.d, nelx, nely, h.precision or "fp64", int(rows), int(gamma))


def _time_candidate(h, rows, flat, n, gamma, omega, n_smooth, band, waves, ws, x) -> float:
    L = _lib.lib()
    _lib.check(L.stt_hier_tune(h.handle, band, waves))
    rel = (ctypes.c_double * rows)()
    conv = (ctypes.c_int * rows)()
    n_iter = ctypes.c_int()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    # rtol 0: every row with a nonzero right-hand side iterates ITERS times
    rc = L.stt_pcg_mg(h.handle, rows, _lib.ptr(flat), n, _lib.ptr(x), n, 0, 0.0, ITERS, omega, n_smooth, gamma,
                      0, 0, 0, rel, conv, ctypes.byref(n_iter), _lib.ptr(ws), ws.numel(),
                      _lib.stream())
    b.record()
    if rc not in (_lib.STT_OK, _lib.STT_ERR_NOT_CONVERGED):
        _lib.check(rc)
    b.synchronize()
    return a.elapsed_time(b)


def tune(h, flat: torch.Tensor, rows: int, n: int, gamma: int, omega: float, n_smooth: int) -> dict:
    """Times the candidates on hierarchy ``h`` with right-hand side rows ``flat`` and
    applies the fastest; returns the cache entry."""
    L = _lib.lib()
    ws = _lib.workspace(L.stt_solve_workspace_bytes(h.handle, rows, gamma), flat.device)
    x = torch.empty_like(flat)
    cands = [(b, w) for b in PCG_BANDS for w in LEVEL_WAVES]
    _time_candidate(h, rows, flat, n, gamma, omega, n_smooth, 0, 0, ws, x)  # warm-up
    times = {c: float("inf") for c in cands}
    for _ in range(2):
        for band, waves in cands:
            t = _time_candidate(h, rows, flat, n, gamma, omega, n_smooth, band, waves, ws, x)
            times[(band, waves)] = min(times[(band, waves)], t)
    best = min(cands, key=lambda c: (times[c], c != (0, 0)))
    _lib.check(L.stt_hier_tune(h.handle, best[0], best[1]))
    return {"pcg_band": best[0], "level_waves": best[1], "ms": {f"{b}/{w}": round(t, 4) for (b, w), t in times.items()}}


def apply(h, flat: torch.Tensor, rows: int, n: int, gamma: int, omega: float, n_smooth: int) -> None:
    """Before a device solve on ``h``: the cached launch shapes of its key, tuned first
    when the key is new and tuning is enabled."""
    if _MODE == "off":
        return
    key = _key(h, rows, gamma)
    with _LOCK:
        entry = _CACHE.get(key)
    if entry is None:
        if _MODE != "enabled":
            return
        entry = tune(h, flat, rows, n, gamma, omega, n_smooth)
        with _LOCK:
            _CACHE[key] = entry
        return
    _lib.check(_lib.lib().stt_hier_tune(h.handle, entry["pcg_band"], entry["level_waves"]))


__all__ = ["enable", "freeze", "disable", "mode", "cache", "save", "load", "tune", "apply", "PCG_BANDS",
           "LEVEL_WAVES"]

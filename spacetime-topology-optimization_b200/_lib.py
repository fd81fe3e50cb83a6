"""ctypes binding of ``libsttb200.so`` (the C ABI in ``include/sttb200.h``).

There is no fallback: if the library is missing or a tensor is not on a CUDA device,
the call raises.  Every entry point runs on the caller's current CUDA stream.
"""

from __future__ import annotations

import ctypes
import functools
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libsttb200.so"

STT_OK = 0
STT_ERR_INVALID = 1
STT_ERR_NOT_CONVERGED = 2
STT_ERR_BREAKDOWN = 3
STT_ERR_TIMEOUT = 4
STT_ERR_CUDA = 5
STT_ERR_WORKSPACE = 6
STT_FP64 = 0
STT_FP32 = 1
STT_PROJECT_IN = 1
STT_PROJECT_OUT = 2
STT_FORM_MODAL = 0
STT_FORM_PRODUCT = 1
_FORMS = {"modal": STT_FORM_MODAL, "product": STT_FORM_PRODUCT}

_c_int, _c_ll, _c_double = ctypes.c_int, ctypes.c_longlong, ctypes.c_double
_p = ctypes.c_void_p
_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)

# name -> (restype, argtypes)
_SIGS = {
    "stt_last_error": (ctypes.c_char_p, []),
    "stt_q4_apply": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p, _c_ll,
                              _p, _c_ll, _p, _c_int, _pd, _p]),
    "stt_q4_diag": (_c_int, [_c_int, _c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p, _p, _c_ll, _pd, _p]),
    "stt_lumped_reaction": (_c_int, [_c_int, _c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p]),
    "stt_lumped_reaction_adjoint": (_c_int, [_c_int, _c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p]),
    "stt_q4_apply_dots_workspace_bytes": (_c_ll, [_c_int, _c_int, _c_int]),
    "stt_q4_apply_dots": (_c_int, [_c_int, _c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p, _c_ll, _p, _pd, _p,
                                   _c_ll, _p, _p, _c_ll, _p]),
    "stt_adjoint_warm_start": (_c_int, [_c_int, _c_ll, _p, _p, _c_ll, _p, _c_ll, _p]),
    "stt_mma_workspace_bytes": (ctypes.c_size_t, [_c_int, _c_ll]),
    "stt_mma_sub": (_c_int, [_c_int, _c_ll, _c_int, _p, _p, _p, _p, _p, _p, _p, _p, _c_ll, _p, _p, _c_double, _p, _p,
                             _p, _p, _c_double, _p, _c_double, _p, _c_double, _p, _c_double, _c_double, _c_double,
                             _c_double, _c_double, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, ctypes.c_size_t,
                             _p]),
    "stt_mma_subsolv": (_c_int, [_c_int, _c_ll, _c_double, _p, _p, _p, _p, _p, _p, _p, _p, _c_ll, _c_double, _p, _p,
                                 _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, ctypes.c_size_t, _p]),
    "stt_stage_glue_rows": (_c_int, [_c_int, _c_int, _c_int, _c_int, _p, _p, _pd, _c_double, _p, _p, _p,
                                     _c_double, _c_double, _c_double, _p, _p, _p, _p]),
    "stt_stage_glue_adjoint": (_c_int, [_c_int, _c_int, _c_int, _c_int, _p, _p, _pd, _c_double, _p, _p, _p, _p,
                                        _c_double, _c_double, _c_double, _p, _p, _p, _p]),
    "stt_ke_modal": (_c_int, [_c_int, _pd, _pd]),
    "stt_set_element_form": (_c_int, [_c_int]),
    "stt_cone_filter": (_c_int, [_c_int, _c_int, _c_int, _c_double, _p, _c_ll, _p, _p, _c_ll, _c_double,
                                 _c_double, _p]),
    "stt_cone_filter_adjoint": (_c_int, [_c_int, _c_int, _c_int, _c_double, _p, _c_ll, _p, _c_ll, _c_double,
                                         _c_double, _p, _c_ll, _p]),
    "stt_hier_workspace_bytes": (_c_ll, [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int]),
    "stt_hier_create": (_c_int, [ctypes.POINTER(_p), _p, _c_ll, _c_int, _c_int, _c_int, _c_int, _p, _c_ll,
                                 _p, _c_ll, _p, _pd, _c_int, _c_int, _p]),
    "stt_hier_select": (_c_int, [_p, _p, ctypes.POINTER(_p)]),
    "stt_hier_status": (_c_int, [_p, _p]),
    "stt_pap_timing": (_c_int, [_c_int]),
    "stt_pap_timing_read": (_c_int, [_pd, ctypes.POINTER(_c_ll), ctypes.POINTER(_c_ll)]),
    "stt_hier_destroy": (_c_int, [_p]),
    "stt_hier_tune": (_c_int, [_p, _c_int, _c_int]),
    "stt_hier_info": (_c_int, [_p, _pi, _pi, _c_int]),
    "stt_hier_level_diag": (_c_int, [_p, _c_int, _p, _p]),
    "stt_hier_level_fixed": (_c_int, [_p, _c_int, _p, _p]),
    "stt_level_apply": (_c_int, [_p, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p]),
    "stt_solve_workspace_bytes": (_c_ll, [_p, _c_int, _c_int]),
    "stt_vcycle_workspace_bytes": (_c_ll, [_p, _c_int, _c_int]),
    "stt_vcycle": (_c_int, [_p, _c_int, _p, _c_ll, _p, _c_ll, _c_double, _c_int, _c_int, _p, _c_ll, _p]),
    "stt_vcycle_noalloc": (_c_int, [_p, _c_int, _p, _c_ll, _p, _c_ll, _c_double, _c_int, _c_int, _p]),
    "stt_pcg_mg": (_c_int, [_p, _c_int, _p, _c_ll, _p, _c_ll, _c_int, _c_double, _c_int, _c_double, _c_int,
                            _c_int, _c_int, _c_int, _c_int, _pd, _pi, _pi, _p, _c_ll, _p]),
    "stt_vec_dots": (_c_int, [_c_int, _c_ll, _p, _p, _p, _p, _p, _p, _c_ll, _p, _p]),
    "stt_vec_cg_update": (_c_int, [_c_int, _c_ll, _p, _p, _p, _p, _p, _c_ll, _p, _p]),
    "stt_vec_xpay": (_c_int, [_c_int, _c_ll, _p, _p, _p, _c_ll, _p]),
    "stt_element_sens": (_c_int, [_c_int, _c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _pd, _p, _p, _p,
                                  _c_ll, _p]),
    "stt_stage_membership": (_c_int, [_c_int, _c_int, _p, _p, _p]),
    "stt_stage_rows": (_c_int, [_c_int, _c_int, _c_int, _p, _p, _c_double, _c_double, _c_double, _p, _p,
                                _p, _p]),
    "stt_stage_gradient": (_c_int, [_c_int, _c_int, _c_int, _p, _p, _p, _p, _p, _c_double, _c_double,
                                    _c_double, _p, _p]),
    "stt_heat_element_means": (_c_int, [_c_int, _c_int, _p, _p, _p]),
    "stt_heat_adjoint_load": (_c_int, [_c_int, _c_int, _p, _c_double, _p, _p]),
    "stt_gravity_load": (_c_int, [_c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _c_int, _p]),
    "stt_grid_transfer": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p]),
    "stt_keff_apply": (_c_int, [_c_int, _c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p, _c_ll, _p]),
    "stt_element_means": (_c_int, [_c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _c_int, _p]),
    "stt_poisson_load": (_c_int, [_c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p, _c_ll, _p]),
    "stt_poisson_load_adjoint": (_c_int, [_c_int, _c_int, _c_int, _p, _c_ll, _p, _c_ll, _p, _c_ll, _p, _c_ll,
                                          _p, _c_ll, _p]),
}


class SttError(RuntimeError):
    """A C-ABI call returned an error status."""

    def __init__(self, code: int, message: str):
        self.code = code
        super().__init__(f"sttb200 error {code}: {message}")


@functools.lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    """Load the shared library once; raise if it was not built."""
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA extension first "
            "(python __graft_entry__.py, or build_ext.py in the package folder)"
        )
    handle = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    return handle


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(rc: int) -> None:
    if rc != STT_OK:
        raise SttError(rc, lib().stt_last_error().decode(errors="replace"))


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def require_cuda(*tensors: torch.Tensor | None) -> None:
    for t in tensors:
        if t is not None and not t.is_cuda:
            raise ValueError(
                "sttopt_b200 runs on CUDA tensors only (no CPU fallback); got a tensor on "
                f"{t.device}"
            )


def set_element_form(form: str) -> str:
    """How the library applies element matrices from now on (hierarchies built and
    applies launched after the call): ``"modal"`` (default; the element's edge modes,
    faster and exact on rigid translations) or ``"product"`` (the 8 x 8 product of the
    corner values, as the reference computes it, reproducing its FP64 rounding).
    Returns the previous form."""
    if form not in _FORMS:
        raise ValueError(f"element form must be one of {sorted(_FORMS)}, got {form!r}")
    prev = lib().stt_set_element_form(_FORMS[form])
    return {v: k for k, v in _FORMS.items()}[prev]


class element_form:
    """``with element_form("product"): ...`` -- ``set_element_form`` for a block."""

    def __init__(self, form: str):
        self.form = form

    def __enter__(self):
        self.prev = set_element_form(self.form)
        return self

    def __exit__(self, *exc):
        set_element_form(self.prev)


def precision_of(dtype: torch.dtype) -> int:
    if dtype == torch.float64:
        return STT_FP64
    if dtype == torch.float32:
        return STT_FP32
    raise TypeError(f"unsupported dtype {dtype}; use float64 or float32")


def dbl_array(values) -> ctypes.Array:
    arr = (ctypes.c_double * len(values))(*values)
    return arr


def workspace(nbytes: int, device) -> torch.Tensor:
    """A 256-byte aligned device byte buffer (torch's allocator aligns to 512)."""
    t = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
    assert t.data_ptr() % 256 == 0
    return t

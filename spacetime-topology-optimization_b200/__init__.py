"""B200-native (sm_100a) matrix-free FEM solve path of ``sttopt``.

Drop-in modules with the reference's names and call signatures:
``torch_fem``, ``torch_mg``, ``torch_solve``, ``sensitivity``, ``virtual_heat``,
``compliance``, ``gravity``, ``filters``, ``load_cases``, ``mma``; plus ``spacetime``, the batched
space-time objective + gradient.
All compute runs in ``libsttb200.so`` (C ABI: ``include/sttb200.h``) on the caller's
CUDA stream; there is no CPU path.
"""

from . import _lib  # noqa: F401
from ._lib import element_form, set_element_form  # noqa: F401

__all__ = ["torch_fem", "torch_mg", "torch_solve", "sensitivity", "virtual_heat", "compliance",
           "spacetime", "fem", "gravity", "filters", "load_cases", "sharding", "autotune", "mma"]


def __getattr__(name):
    if name in __all__:
        import importlib

        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(name)

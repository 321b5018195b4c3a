"""smaxkernels_b200 -- the SmaxKernels sparse hot path on B200 (sm_100a).

The kernels and the C ABI live in ``libsmax_b200.so`` (built from ``csrc/``
by ``python smaxkernels_b200/build.py``); this package is the Python side of
that boundary: a mirror of the reference's ``SMAX::Interface`` API
(:mod:`smaxkernels_b200.interface`) and the synthetic matrix generators used
by the tests and the benchmark (:mod:`smaxkernels_b200.matrices`).

The library is loaded on first use of an Interface name (``Interface``,
``KernelType``, ``lib`` ...), not at package import: a process that only needs
the numpy generators (``smaxkernels_b200.matrices``), such as the benchmark's
reference arm that times the reference's own CPU kernels, never maps it.  The
first such access raises ImportError if the library is missing; there is no
fallback.
"""
from __future__ import annotations

import importlib

_FROM_LIB = ("SmaxError", "lib")
_FROM_INTERFACE = ("FloatType", "Interface", "IntType", "Kernel", "KernelType", "PlatformType", "SpMVType")

__all__ = ["Interface", "Kernel", "KernelType", "PlatformType", "IntType", "FloatType", "SpMVType", "SmaxError"]


def __getattr__(name):
    if name in _FROM_LIB:
        mod = importlib.import_module("._lib", __name__)
    elif name in _FROM_INTERFACE:
        mod = importlib.import_module(".interface", __name__)
    else:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
    value = getattr(mod, name)
    globals()[name] = value
    return value

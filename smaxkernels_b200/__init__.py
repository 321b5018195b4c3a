"""smaxkernels_b200 -- the SmaxKernels sparse hot path on B200 (sm_100a).

The kernels and the C ABI live in ``libsmax_b200.so`` (built from ``csrc/``
by ``python smaxkernels_b200/build.py``); this package is the Python side of
that boundary: a mirror of the reference's ``SMAX::Interface`` API
(:mod:`smaxkernels_b200.interface`) and the synthetic matrix generators used
by the tests and the benchmark (:mod:`smaxkernels_b200.matrices`).
"""
from ._lib import SmaxError, lib  # noqa: F401  (raises if the library is missing)
from .interface import FloatType, Interface, IntType, Kernel, KernelType, PlatformType, SpMVType  # noqa: F401

__all__ = ["Interface", "Kernel", "KernelType", "PlatformType", "IntType", "FloatType", "SpMVType", "SmaxError"]

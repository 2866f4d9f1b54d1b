"""B200 (sm_100a) implementation of the ASOHF particle hot path.

The kernels and the C ABI live in libasohf_gpu.so (asohf_b200/csrc, declared
in include/asohf_gpu.h); asohf_b200.api binds them, asohf_b200.driver runs
the hot-path sequence, asohf_b200.autograd wraps the deposit+Poisson layer.
"""
from .api import Asohf, AsohfError, GpuBackend, load  # noqa: F401

__all__ = ["Asohf", "AsohfError", "GpuBackend", "load"]

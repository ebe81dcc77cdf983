"""UltraPrecise exact-decimal execution path for NVIDIA B200 (sm_100a).

Host-side Python mirror of the reference's operator interface over the C ABI
of libultraprecise.so (include/ultraprecise.h).  The compute path is the
library's CUDA kernels; there is no CPU fallback: every entry point fails
loudly when the library (or a GPU, for launches) is missing.
"""
from . import abi, codec, expr  # noqa: F401
from .expr import col, dec, lit, rescale, ColType  # noqa: F401

__all__ = ["abi", "codec", "expr", "col", "dec", "lit", "rescale", "ColType"]

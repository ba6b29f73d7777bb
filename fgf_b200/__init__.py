"""fgf_b200 -- sm_100a implementation of fgf's packed-vector ops hot path.

`fgf_b200.ops` mirrors `fgf::ops` over device buffers through the C ABI of
libfgfcuda.so (include/fgf_cuda.h); `fgf_b200.fields` carries the field
markers and host scalar arithmetic.
"""
from . import fields  # noqa: F401
from .fields import Gf8B, Gf8D, Gf16, Gf32  # noqa: F401

__version__ = "0.1.0"

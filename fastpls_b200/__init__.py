"""fastpls_b200: B200-native (sm_100a) fit/predict hot path of fastPLS.

The numerical work runs in libfastpls_b200.so (hand-written CUDA behind a C
ABI, include/fastpls_b200.h).  This package is the host-side mirror of the R
API of fastPLS (``pls``, ``predict``, ``fastsvd``, cross-validation helpers)
and a ctypes binding of the C ABI; it has no CPU fallback.
"""
from . import _lib  # noqa: F401
from ._lib import FastPLSError, has_cuda, reset_workspace, version  # noqa: F401

__all__ = ["FastPLSError", "has_cuda", "reset_workspace", "version"]

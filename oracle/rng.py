"""libstdc++ Gaussian sketch for the oracle (test infrastructure only).

Mirrors ``gaussian_matrix`` (reference src/svd_cpu_rsvd.cpp:10-22) and
``gaussian_matrix_local`` (src/fastPLS.cpp:99-115): ``std::mt19937(seed)`` +
``std::normal_distribution<double>(0,1)`` filled in column-major order.  The
draws come from oracle/rng.cpp compiled by g++ (see oracle/build.py).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_rng.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            from .build import build_oracle
            build_oracle()
        lib = ctypes.CDLL(_LIB_PATH)
        lib.oracle_gaussian_matrix.argtypes = [
            ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint]
        lib.oracle_gaussian_matrix.restype = None
        lib.oracle_mt19937_raw.argtypes = [
            ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint]
        lib.oracle_mt19937_raw.restype = None
        _lib = lib
    return _lib


def gaussian_matrix(n_rows, n_cols, seed):
    """n_rows x n_cols column-major N(0,1) matrix from mt19937(seed)."""
    lib = _load()
    out = np.empty((int(n_rows), int(n_cols)), dtype=np.float64, order="F")
    if out.size:
        lib.oracle_gaussian_matrix(out.ctypes.data, out.size,
                                   ctypes.c_uint(int(seed) & 0xFFFFFFFF))
    return out


def mt19937_raw(n, seed=5489):
    lib = _load()
    out = np.empty(int(n), dtype=np.uint32)
    lib.oracle_mt19937_raw(out.ctypes.data, out.size,
                           ctypes.c_uint(int(seed) & 0xFFFFFFFF))
    return out

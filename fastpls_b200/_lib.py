"""ctypes binding of libfastpls_b200.so (C ABI in include/fastpls_b200.h).

Each wrapper mirrors one `.Call` routine of the R package fastPLS used with
backend = "cuda" and returns the same fields as the reference's R list.  There
is no fallback: if the library or a B200 device is missing, calls raise.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfastpls_b200.so")

_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_int_p = ctypes.POINTER(ctypes.c_int)
_lib = None

FPLS_ERRORS = {1: "argument", 2: "cuda", 3: "numerical", 4: "no_device", 5: "internal"}


class FastPLSError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fastpls_b200 [{FPLS_ERRORS.get(code, code)}]: {msg}")
        self.code = code


# name -> argtypes (restype int unless noted)
_D, _I, _DP, _IP, _S, _C = (ctypes.c_double, ctypes.c_int, _c_double_p, _c_int_p,
                            ctypes.c_size_t, ctypes.c_char_p)
# int (*fpls_allreduce_fn)(double* buf, long long count, void* stream, void* user)
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p,
                                ctypes.c_void_p)
_VP = ctypes.c_void_p
SIGNATURES = {
    "fpls_pls_model1_rows": ([_DP, _I, _I, _DP, _I, _IP, _I, _I, _I, _I, _I, _I, _D, _I, ALLREDUCE_FN, _VP,
                              _IP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _IP, _C, _S],
                             ctypes.c_int),
    "fpls_pls_model2_fast_rows": ([_DP, _I, _I, _DP, _I, _IP, _I, _I, _I, _I, ALLREDUCE_FN, _VP, _DP, _DP,
                                   _DP, _DP, _DP, _DP, _DP, _DP, _IP, _C, _S], ctypes.c_int),
    "fpls_has_cuda": ([], ctypes.c_int),
    "fpls_version": ([], ctypes.c_char_p),
    "fpls_reset_workspace": ([_C, _S], ctypes.c_int),
    "fpls_matrix_multiply": ([_DP, _I, _I, _DP, _I, _DP, _C, _S], ctypes.c_int),
    "fpls_truncated_svd": ([_DP, _I, _I, _I, _I, _I, _I, _D, _I, _I, _DP, _DP, _DP, _IP, _C, _S],
                           ctypes.c_int),
    "fpls_pls_model1": ([_DP, _I, _I, _DP, _I, _IP, _I, _I, _I, _I, _I, _I, _D, _I, _IP, _DP,
                         _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _IP, _C, _S],
                        ctypes.c_int),
    "fpls_pls_model2_fast": ([_DP, _I, _I, _DP, _I, _IP, _I, _I, _I, _I, _DP, _DP, _DP, _DP, _DP,
                              _DP, _DP, _DP, _IP, _C, _S], ctypes.c_int),
    "fpls_pls_model1_xprod": ([_DP, _I, _I, _DP, _I, _IP, _I, _I, _I, _I, _I, _D, _I, _I, _IP, _DP,
                               _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _IP, _C, _S],
                              ctypes.c_int),
    "fpls_pls_model2_fast_xprod": ([_DP, _I, _I, _DP, _I, _IP, _I, _I, _I, _I, _I, _DP, _DP, _DP,
                                    _DP, _DP, _DP, _DP, _DP, _IP, _C, _S], ctypes.c_int),
    "fpls_pls_model2": ([_DP, _I, _I, _DP, _I, _IP, _I, _I, _I, _I, _I, _I, _D, _I, _DP, _DP,
                         _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _IP, _C, _S], ctypes.c_int),
    "fpls_predict_lowrank": ([_DP, _I, _I, _DP, _DP, _DP, _I, _DP, _I, _DP, _IP, _I, _DP, _DP,
                              _C, _S], ctypes.c_int),
    "fpls_predict_classes": ([_DP, _I, _I, _DP, _DP, _DP, _I, _DP, _I, _DP, _IP, _I, _DP, _I,
                              _IP, _DP, _C, _S], ctypes.c_int),
    "fpls_lda_train_prefix": ([_DP, _I, _I, _IP, _I, _IP, _I, _D, _DP, _DP, _DP, _DP, _DP, _C,
                               _S], ctypes.c_int),
    "fpls_lda_project_train_prefix": ([_DP, _I, _I, _DP, _I, _DP, _IP, _I, _IP, _I, _D, _DP, _DP,
                                       _DP, _DP, _DP, _C, _S], ctypes.c_int),
    "fpls_lda_predict": ([_DP, _I, _I, _DP, _DP, _I, _IP, _DP, _C, _S], ctypes.c_int),
    "fpls_lda_project_predict": ([_DP, _I, _I, _DP, _I, _DP, _DP, _DP, _I, _IP, _DP, _C, _S],
                                 ctypes.c_int),
    "fpls_bf16x3_gemm": ([_DP, _I, _I, _DP, _I, _DP, _C, _S], ctypes.c_int),
    "fpls_int8_emulated_gemm": ([_DP, _I, _I, _DP, _I, _I, _DP, _C, _S], ctypes.c_int),
    "fpls_kernel_matrix": ([_DP, _I, _DP, _I, _I, _I, _D, _I, _D, _DP, _C, _S], ctypes.c_int),
    "fpls_center_kernel_train": ([_DP, _I, _DP, _DP, _DP, _C, _S], ctypes.c_int),
    "fpls_center_kernel_test": ([_DP, _I, _I, _DP, _D, _DP, _C, _S], ctypes.c_int),
    "fpls_kernel_pls_model2_fast": ([_DP, _I, _I, _DP, _I, _IP, _I, _I, _I, _D, _I, _D, _I, _I, _DP, _DP, _DP,
                                     _DP, _DP, _DP, _DP, _DP, _IP, _DP, _DP, _DP, _DP, _DP, _C, _S],
                                    ctypes.c_int),
    "fpls_cv_predict": ([ctypes.c_void_p, _I, _I, _I, _IP, _I, _IP, _I, _IP, _I, _I, _I, _I, _I,
                         _I, _IP, _IP, _C, _S], ctypes.c_int),
    "fpls_double_cv": ([ctypes.c_void_p, _I, _I, _I, _IP, _I, _IP, _I, _IP, _I, _IP, _I, _I, _I,
                        _I, _I, _I, _IP, _DP, _IP, _IP, _IP, _C, _S], ctypes.c_int),
    "fpls_cv_predict_scores": ([ctypes.c_void_p, _I, _I, _I, _IP, _I, _IP, _I, _IP, _I, _I, _I, _I, _I,
                                _I, _IP, _IP, _DP, _C, _S], ctypes.c_int),
    "fpls_double_cv_scores": ([ctypes.c_void_p, _I, _I, _I, _IP, _I, _IP, _I, _IP, _I, _IP, _I, _I, _I,
                               _I, _I, _I, _IP, _DP, _IP, _IP, _IP, _DP, _DP, _C, _S], ctypes.c_int),
    "fpls_pls_lda": ([ctypes.c_void_p, _I, _I, _I, _DP, _I, _IP, ctypes.c_void_p, _I, _IP, _I, _I, _I, _I, _I, _I,
                      _I, _I, _D, _I, _D, _IP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _IP, _IP, _DP, _DP, _DP,
                      _DP, _DP, _DP, _DP, _IP, _C, _S], ctypes.c_int),
    "fpls_set_autotune": ([_I, _C, _S], ctypes.c_int),
    "fpls_autotune_report": ([ctypes.c_char_p, _S, ctypes.POINTER(ctypes.c_size_t), _C, _S], ctypes.c_int),
    "fpls_int8_gram": ([ctypes.c_void_p, _I, _I, _I, _DP, _I, _DP, _C, _S], ctypes.c_int),
    "fpls_x_alloc": ([_I, _I, _I, _IP, _C, _S], ctypes.c_int),
    "fpls_x_device_pointer": ([_I, ctypes.POINTER(ctypes.c_void_p), _C, _S], ctypes.c_int),
    "fpls_x_download": ([_I, ctypes.c_void_p, _C, _S], ctypes.c_int),
    "fpls_bf16x3_gemm_noalloc": ([ctypes.c_void_p, _I, _I, ctypes.c_void_p, _I, ctypes.c_void_p,
                                  _C, _S], ctypes.c_int),
    "fpls_gaussian_y_encode": ([_DP, _I, _I, _DP, _I, _DP, _DP, _DP, _C, _S], ctypes.c_int),
    "fpls_gaussian_y_decode": ([_DP, _I, _I, _DP, _DP, _I, _DP, _C, _S], ctypes.c_int),
    "fpls_nearest_code_classes": ([_DP, _I, _I, _DP, _I, _IP, _C, _S], ctypes.c_int),
    "fpls_opls_filter": ([_DP, _I, _I, _DP, _I, _I, _I, _DP, _DP, _DP, _DP, _DP, _IP, _C, _S],
                         ctypes.c_int),
    "fpls_plssvd_label_aware": ([ctypes.c_void_p, _I, _I, _I, _IP, _I, _IP, _I, _I, _I, _I, _I, _I,
                                 _IP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _IP, _C, _S],
                                ctypes.c_int),
    "fpls_label_aware_cknn": ([ctypes.c_void_p, _I, _I, _I, _IP, _I, ctypes.c_void_p, _I, _I, _I, _I,
                               _I, _I, _I, _I, _D, _D, _I, _I, _IP, _DP, _C, _S], ctypes.c_int),
    "fpls_label_aware_cknn_resident": ([_I, _IP, _I, _I, _I, _I, _I, _I, _I, _I, _I, _D, _D, _I, _I,
                                        _IP, _DP, _C, _S], ctypes.c_int),
    "fpls_profile_class": ([_I, ctypes.c_char_p, _S, _DP, ctypes.POINTER(ctypes.c_longlong), _DP, _DP,
                            _C, _S], ctypes.c_int),
    "fpls_set_precision": ([_I, _C, _S], ctypes.c_int),
    "fpls_get_precision": ([], ctypes.c_int),
    "fpls_host_register": ([ctypes.c_void_p, _S, _C, _S], ctypes.c_int),
    "fpls_host_unregister": ([ctypes.c_void_p, _C, _S], ctypes.c_int),
    "fpls_gaussian_sketch": ([_I, _I, ctypes.c_uint, _DP, _C, _S], ctypes.c_int),
    "fpls_candidate_scores": ([_DP, _I, _I, _DP, _DP, _C, _S], ctypes.c_int),
    "fpls_candidate_centroids": ([_DP, _I, _I, _IP, _I, _DP, _C, _S], ctypes.c_int),
    "fpls_candidate_knn_predict": ([_DP, _I, _DP, _I, _I, _IP, _DP, _I, _DP, _I, _I, _I, _D, _D,
                                    _IP, _DP, _C, _S], ctypes.c_int),
    "fpls_opls_apply_filter": ([_DP, _I, _I, _DP, _DP, _DP, _DP, _I, _DP, _C, _S], ctypes.c_int),
    "fpls_x_upload": ([ctypes.c_void_p, _I, _I, _I, _IP, _C, _S], ctypes.c_int),
    "fpls_x_free": ([_I, _C, _S], ctypes.c_int),
    "fpls_double_cv_resident": ([_I, _IP, _I, _IP, _I, _IP, _I, _IP, _I, _I, _I, _I, _I, _I,
                                 _IP, _DP, _IP, _IP, _IP, _C, _S], ctypes.c_int),
    "fpls_double_cv_outer_subset": ([ctypes.c_void_p, _I, _I, _I, _IP, _I, _IP, _I, _IP, _I, _IP, _I,
                                     _IP, _I, _I, _I, _I, _I, _I, _IP, _DP, _IP, _IP, _IP, _C, _S],
                                    ctypes.c_int),
    "fpls_double_cv_resident_outer_subset": ([_I, _IP, _I, _IP, _I, _IP, _I, _IP, _I, _IP, _I, _I, _I, _I,
                                              _I, _I, _IP, _DP, _IP, _IP, _IP, _C, _S], ctypes.c_int),
    "fpls_launch_count": ([], ctypes.c_longlong),
    "fpls_last_call_ms": ([], ctypes.c_double),
    "fpls_profile": ([_I, _DP, ctypes.POINTER(ctypes.c_longlong), _DP, _C, _S], ctypes.c_int),
}


def load():
    """Loads the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m fastpls_b200.build` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (argtypes, restype) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = restype
        _lib = lib
    return _lib


def exported_symbols():
    return sorted(SIGNATURES)


def has_cuda():
    return bool(load().fpls_has_cuda())


def version():
    return load().fpls_version().decode()


# ---------------------------------------------------------------- helpers ---
class DeviceMatrix:
    """A column-major FP64 matrix already in device memory, taken from any
    object exposing __cuda_array_interface__ (for instance the transpose of a
    contiguous torch CUDA tensor).  The matrix entry points accept it for X, Y,
    Xtest, the response and the filtered-X output: the library then copies
    within HBM instead of across PCIe (the C ABI tells host and device
    pointers apart by unified addressing)."""

    def __init__(self, obj, allow_f32=False):
        cai = obj.__cuda_array_interface__
        shape = tuple(int(v) for v in cai["shape"])
        ok_types = ("<f8", "<f4") if allow_f32 else ("<f8",)
        if cai["typestr"] not in ok_types or len(shape) not in (1, 2):
            raise ValueError("device matrices must be float64 vectors or matrices")
        esz = 4 if cai["typestr"] == "<f4" else 8
        if len(shape) == 1:
            shape = (shape[0], 1)
        rows, cols = shape
        strides = cai.get("strides")  # None: C-contiguous
        if len(cai["shape"]) == 2 and rows > 1 and cols > 1 and \
                (strides is None or tuple(strides) != (esz, esz * rows)):
            raise ValueError("device matrices must be column-major and contiguous")
        self.ptr = int(cai["data"][0])
        self.shape = shape
        self.dtype = np.dtype(np.float32 if esz == 4 else np.float64)
        self.owner = obj


def _is_device(a):
    return isinstance(a, DeviceMatrix) or hasattr(a, "__cuda_array_interface__")


def _f64(a, shape=None):
    if _is_device(a):
        return a if isinstance(a, DeviceMatrix) else DeviceMatrix(a)
    a = np.asarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return np.asfortranarray(a)


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def _p(a):
    if a is None:
        return None
    if isinstance(a, DeviceMatrix):
        return ctypes.cast(ctypes.c_void_p(a.ptr), _c_double_p)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_c_int_p)
    return a.ctypes.data_as(_c_double_p)


def _out(*shape):
    return np.zeros(shape, dtype=np.float64, order="F")


def _call(name, *args):
    err = ctypes.create_string_buffer(1024)
    rc = getattr(load(), name)(*args, err, ctypes.sizeof(err))
    if rc != 0:
        raise FastPLSError(rc, err.value.decode(errors="replace"))


def reset_workspace():
    _call("fpls_reset_workspace")


# -------------------------------------------------------------- wrappers ---
def matrix_multiply(A, B):
    A = _f64(A)
    B = _f64(B)
    C = _out(A.shape[0], B.shape[1])
    _call("fpls_matrix_multiply", _p(A), A.shape[0], A.shape[1], _p(B), B.shape[1], _p(C))
    return C


def truncated_svd(A, k, svd_method=4, oversample=10, power_iters=1, svds_tol=0.0, seed=1,
                  left_only=False):
    A = _f64(A)
    rows, cols = A.shape
    kcap = min(rows, cols, max(int(k), 1))
    U = _out(rows, kcap)
    s = np.zeros(kcap)
    Vt = None if left_only else _out(kcap, cols)
    rank = ctypes.c_int(0)
    _call("fpls_truncated_svd", _p(A), rows, cols, int(k), int(svd_method), int(oversample),
          int(power_iters), float(svds_tol), int(seed), int(bool(left_only)), _p(U), _p(s),
          _p(Vt), ctypes.byref(rank))
    r = rank.value
    return dict(u=U[:, :r], d=s[:r], vt=None if Vt is None else Vt[:r, :])


def allreduce_callback(fn):
    """Wraps fn(buf_ptr, count, stream_ptr) -- a sum of `count` doubles of
    device memory over the ranks, ordered on the library's stream -- as the
    fpls_allreduce_fn of the row-sharded fits.  Returns (callback, errors): an
    exception raised by fn is kept in errors and the library sees status 1."""
    errors = []

    def cb(buf, count, stream, user):
        try:
            fn(int(buf or 0), int(count), int(stream or 0))
            return 0
        except BaseException as e:   # never let an exception cross the C frames
            errors.append(e)
            return 1
    return ALLREDUCE_FN(cb), errors


def _call_sharded(errors, name, *args):
    try:
        _call(name, *args)
    except FastPLSError as e:
        if errors:
            raise errors[0] from e
        raise


def pls_model1(X, Y, ncomp, scaling=1, fit=False, svd_method=4, oversample=10, power_iters=1,
               svds_tol=0.0, seed=1, store_B=True, xprod=False, allreduce=None, n_total=None):
    """PLSSVD (fpls_pls_model1), or its matrix-free form with xprod=True.

    Row-sharded (fpls_pls_model1_rows) when allreduce = fn(buf, count, stream)
    is given: X and Y are this rank's rows, n_total the rows over all ranks
    (see fastpls_b200.row_shards)."""
    X = _f64(X)
    Y = _f64(Y)
    n, p = X.shape
    m = Y.shape[1]
    nc = _i32(np.atleast_1d(ncomp))
    L = nc.size
    if allreduce is not None and (xprod or n_total is None):
        raise ValueError("a row-sharded PLSSVD forms S (xprod=False) and needs n_total")
    max_rank = min(n if allreduce is None else int(n_total), p, m)
    K0 = min(int(np.clip(nc, 1, max_rank).max()), max_rank)
    out = dict(C_latent=_out(K0, K0, L), W_latent=_out(K0, m, L), Q=_out(m, K0), Ttrain=_out(n, K0),
               R=_out(p, K0), mX=_out(1, p), vX=_out(1, p), mY=_out(1, m),
               B=_out(p, m, L) if store_B else None, Yfit=_out(n, m, L) if fit else None,
               R2Y=np.zeros(L), singular_values=np.zeros(K0))
    nco = np.zeros(L, dtype=np.int32)
    keff = ctypes.c_int(0)
    errors = []
    if xprod:
        head = ("fpls_pls_model1_xprod", _p(X), n, p, _p(Y), m, _p(nc), L, int(scaling),
                int(bool(fit)), int(oversample), int(power_iters), float(svds_tol), int(seed), 3)
    elif allreduce is not None:
        cb, errors = allreduce_callback(allreduce)
        head = ("fpls_pls_model1_rows", _p(X), n, p, _p(Y), m, _p(nc), L, int(scaling), int(bool(fit)),
                int(svd_method), int(oversample), int(power_iters), float(svds_tol), int(seed), cb, None)
    else:
        head = ("fpls_pls_model1", _p(X), n, p, _p(Y), m, _p(nc), L, int(scaling), int(bool(fit)),
                int(svd_method), int(oversample), int(power_iters), float(svds_tol), int(seed))
    _call_sharded(errors, *head, _p(nco),
          _p(out["C_latent"]), _p(out["W_latent"]), _p(out["Q"]), _p(out["Ttrain"]), _p(out["R"]),
          _p(out["mX"]), _p(out["vX"]), _p(out["mY"]), _p(out["B"]), _p(out["Yfit"]),
          _p(out["R2Y"]), _p(out["singular_values"]), ctypes.byref(keff))
    k = keff.value
    out["R"] = out["R"][:, :k]
    out["Q"] = out["Q"][:, :k]
    out["Ttrain"] = out["Ttrain"][:, :k]
    out["singular_values"] = out["singular_values"][:k]
    out.update(ncomp=nco, p=p, m=m, pls_method="plssvd", B_stored=bool(store_B),
               compact_prediction=not store_B)
    if not store_B:
        out.pop("B")
    return out


def pls_model2_fast(X, Y, ncomp, scaling=1, fit=False, seed=1, store_B=True, xprod=False, allreduce=None):
    """Fast SIMPLS (fpls_pls_model2_fast), or its matrix-free form with xprod=True.

    Row-sharded (fpls_pls_model2_fast_rows) when allreduce = fn(buf, count,
    stream) is given: X and Y are this rank's rows (see fastpls_b200.row_shards)."""
    if allreduce is not None and xprod:
        raise ValueError("a row-sharded fast SIMPLS forms S (xprod=False)")
    X = _f64(X)
    Y = _f64(Y)
    n, p = X.shape
    m = Y.shape[1]
    nc = _i32(np.maximum(np.atleast_1d(ncomp), 1))
    L = nc.size
    K = int(nc.max())
    out = dict(R=_out(p, K), Q=_out(m, K), mX=_out(1, p), vX=_out(1, p), mY=_out(1, m),
               B=_out(p, m, L) if store_B else None, Yfit=_out(n, m, L) if fit else None,
               R2Y=np.zeros(L))
    ncmp = ctypes.c_int(0)
    errors = []
    if allreduce is not None:
        cb, errors = allreduce_callback(allreduce)
        head = ("fpls_pls_model2_fast_rows", _p(X), n, p, _p(Y), m, _p(nc), L, int(scaling),
                int(bool(fit)), int(seed), cb, None)
    else:
        head = (("fpls_pls_model2_fast_xprod", _p(X), n, p, _p(Y), m, _p(nc), L, int(scaling),
                 int(bool(fit)), int(seed), 3) if xprod else
                ("fpls_pls_model2_fast", _p(X), n, p, _p(Y), m, _p(nc), L, int(scaling), int(bool(fit)),
                 int(seed)))
    _call_sharded(errors, *head, _p(out["R"]), _p(out["Q"]), _p(out["mX"]), _p(out["vX"]), _p(out["mY"]),
          _p(out["B"]), _p(out["Yfit"]), _p(out["R2Y"]), ctypes.byref(ncmp))
    out.update(ncomp=nc, p=p, m=m, pls_method="simpls", n_components=ncmp.value,
               B_stored=bool(store_B), compact_prediction=not store_B)
    if not store_B:
        out.pop("B")
    return out


def pls_model2(X, Y, ncomp, scaling=1, fit=False, svd_method=3, oversample=10, power_iters=1,
               svds_tol=0.0, seed=1, store_B=True):
    X = _f64(X)
    Y = _f64(Y)
    n, p = X.shape
    m = Y.shape[1]
    nc = _i32(np.atleast_1d(ncomp))
    L = nc.size
    K = int(nc.max())
    out = dict(R=_out(p, K), Q=_out(m, K), P=_out(p, K), Ttrain=_out(n, K), mX=_out(1, p),
               vX=_out(1, p), mY=_out(1, m), B=_out(p, m, L) if store_B else None,
               Yfit=_out(n, m, L) if fit else None, R2Y=np.zeros(L))
    ncmp = ctypes.c_int(0)
    _call("fpls_pls_model2", _p(X), n, p, _p(Y), m, _p(nc), L, int(scaling), int(bool(fit)),
          int(svd_method), int(oversample), int(power_iters), float(svds_tol), int(seed),
          _p(out["R"]), _p(out["Q"]), _p(out["P"]), _p(out["Ttrain"]), _p(out["mX"]),
          _p(out["vX"]), _p(out["mY"]), _p(out["B"]), _p(out["Yfit"]), _p(out["R2Y"]),
          ctypes.byref(ncmp))
    out.update(ncomp=nc, p=p, m=m, pls_method="simpls", n_components=ncmp.value,
               B_stored=bool(store_B), compact_prediction=not store_B)
    if not store_B:
        out.pop("B")
    return out


def compact_weights(model):
    """Per-slice latent weights (kmax x m x L) as compact_prediction_weights
    (src/fastPLS.cpp:3737-3836)."""
    R = model["R"]
    kmax = R.shape[1]
    m = int(model["m"])
    nc = np.atleast_1d(model["ncomp"])
    L = nc.size
    W = np.zeros((kmax, m, L), order="F")
    if model["pls_method"] in ("simpls", "simpls_fast"):
        Q = model["Q"]
        for a in range(L):
            mc = int(nc[a])
            W[:mc, :, a] = Q[:, :mc].T
    elif "W_latent" in model:
        Wl = model["W_latent"]
        W[:, :, :] = Wl[:kmax, :, :L]
    else:
        C = model["C_latent"]
        Q = model["Q"]
        for a in range(L):
            mc = int(nc[a])
            W[:mc, :, a] = C[:mc, :mc, a] @ Q[:, :mc].T
    return W


def predict_lowrank(model, Xtest, proj=False):
    Xt = _f64(Xtest)
    w, p = Xt.shape
    R = _f64(model["R"])
    kmax = R.shape[1]
    W = _f64(compact_weights(model))
    m = int(model["m"])
    nc = _i32(np.minimum(np.atleast_1d(model["ncomp"]), kmax))
    L = nc.size
    Yp = _out(w, m, L)
    T = _out(w, kmax) if proj else None
    _call("fpls_predict_lowrank", _p(Xt), w, p, _p(_f64(model["mX"]).ravel()),
          _p(_f64(model["vX"]).ravel()), _p(_f64(model["mY"]).ravel()), m, _p(R), kmax, _p(W),
          _p(nc), L, _p(Yp), _p(T))
    out = dict(Ypred=Yp)
    if proj:
        out["Ttest"] = T
    return out


def predict_classes(model, Xtest, class_bias=None, top_k=1, return_scores=False):
    Xt = _f64(Xtest)
    w, p = Xt.shape
    R = _f64(model["R"])
    kmax = R.shape[1]
    W = _f64(compact_weights(model))
    m = int(model["m"])
    nc = _i32(np.minimum(np.atleast_1d(model["ncomp"]), kmax))
    L = nc.size
    idx = np.zeros((w, top_k, L), dtype=np.int32, order="F")
    sc = _out(w, top_k, L) if return_scores else None
    bias = None if class_bias is None else np.ascontiguousarray(class_bias, dtype=np.float64)
    _call("fpls_predict_classes", _p(Xt), w, p, _p(_f64(model["mX"]).ravel()),
          _p(_f64(model["vX"]).ravel()), _p(_f64(model["mY"]).ravel()), m, _p(R), kmax, _p(W),
          _p(nc), L, _p(bias), int(top_k), idx.ctypes.data_as(_c_int_p), _p(sc))
    return dict(top_index=idx, top_score=sc)


def _lda_unpack(means, linear, constants, priors, lam, ncomp):
    models = {}
    for a, kk in enumerate(ncomp):
        kk = int(kk)
        models[str(kk)] = dict(means=means[:, :kk, a].copy(), linear=linear[:, :kk, a].copy(),
                               constants=constants[:, a].copy(), priors=priors.copy(),
                               ridge=float(lam[a]))
    return models


def lda_train_prefix(T, y, n_classes, ncomp, ridge=1e-8):
    T = _f64(T)
    n, kmax = T.shape
    yy = _i32(y)
    nc = _i32(np.atleast_1d(ncomp))
    L = nc.size
    km = int(nc.max())
    C = int(n_classes)
    means, linear = _out(C, km, L), _out(C, km, L)
    constants, priors, lam = _out(C, L), np.zeros(C), np.zeros(L)
    _call("fpls_lda_train_prefix", _p(T), n, kmax, _p(yy), C, _p(nc), L, float(ridge), _p(means),
          _p(linear), _p(constants), _p(priors), _p(lam))
    return _lda_unpack(means, linear, constants, priors, lam, nc)


def lda_project_train_prefix(X, R, offset, y, n_classes, ncomp, ridge=1e-8):
    X = _f64(X)
    R = _f64(R)
    n, p = X.shape
    k = R.shape[1]
    off = None if offset is None else np.ascontiguousarray(offset, dtype=np.float64).ravel()
    yy = _i32(y)
    nc = _i32(np.atleast_1d(ncomp))
    L = nc.size
    km = int(nc.max())
    C = int(n_classes)
    means, linear = _out(C, km, L), _out(C, km, L)
    constants, priors, lam = _out(C, L), np.zeros(C), np.zeros(L)
    _call("fpls_lda_project_train_prefix", _p(X), n, p, _p(R), k, _p(off), _p(yy), C, _p(nc), L,
          float(ridge), _p(means), _p(linear), _p(constants), _p(priors), _p(lam))
    return _lda_unpack(means, linear, constants, priors, lam, nc)


def lda_predict(T, lda, return_scores=False):
    T = _f64(T)
    w, k = T.shape
    lin = _f64(lda["linear"])
    C = lin.shape[0]
    const = np.ascontiguousarray(lda["constants"], dtype=np.float64).ravel()
    lab = np.zeros(w, dtype=np.int32)
    sc = _out(w, C) if return_scores else None
    _call("fpls_lda_predict", _p(T), w, k, _p(lin), _p(const), C, _p(lab), _p(sc))
    return dict(pred=lab, scores=sc) if return_scores else dict(pred=lab)


def lda_project_predict(X, R, offset, lda, return_scores=False):
    X = _f64(X)
    R = _f64(R)
    w, p = X.shape
    k = R.shape[1]
    lin = _f64(lda["linear"])
    C = lin.shape[0]
    const = np.ascontiguousarray(lda["constants"], dtype=np.float64).ravel()
    off = None if offset is None else np.ascontiguousarray(offset, dtype=np.float64).ravel()
    lab = np.zeros(w, dtype=np.int32)
    sc = _out(w, C) if return_scores else None
    _call("fpls_lda_project_predict", _p(X), w, p, _p(R), k, _p(off), _p(lin), _p(const), C,
          _p(lab), _p(sc))
    return dict(pred=lab, scores=sc) if return_scores else dict(pred=lab)


PREC = {"fp64": 0, "bf16x3": 1, "bf16x6": 2, "int8": 3}


def bf16x3_gemm(A, B):
    """C = A B through the BF16 split-precision tensor-core kernel (diagnostic)."""
    A = _f64(A)
    B = _f64(B)
    C = _out(A.shape[0], B.shape[1])
    _call("fpls_bf16x3_gemm", _p(A), A.shape[0], A.shape[1], _p(B), B.shape[1], _p(C))
    return C


def int8_gram(X, slices=4, mean=None):
    """(X - mean)(X - mean)^T through INT8 digit planes of the rows (fpls_int8_gram)."""
    f32 = np.asarray(X).dtype == np.float32
    Xa = np.asfortranarray(X, dtype=np.float32 if f32 else np.float64)
    n, p = Xa.shape
    mu = None if mean is None else np.ascontiguousarray(mean, dtype=np.float64).ravel()
    K = _out(n, n)
    _call("fpls_int8_gram", Xa.ctypes.data, int(f32), n, p, _p(mu), int(slices), _p(K))
    return K


def int8_emulated_gemm(A, B, slices=7):
    """C = A B through the INT8 tensor-core (Ozaki digit-plane) product."""
    A = _f64(A)
    B = _f64(B)
    C = _out(A.shape[0], B.shape[1])
    _call("fpls_int8_emulated_gemm", _p(A), A.shape[0], A.shape[1], _p(B), B.shape[1], int(slices), _p(C))
    return C


KERNEL_IDS = {"linear": 1, "rbf": 2, "poly": 3}


def kernel_matrix(X1, X2, kernel="rbf", gamma=None, degree=3, coef0=1.0):
    """kernel_matrix_cpp on the device (X1 n1 x p, X2 n2 x p)."""
    X1 = _f64(X1)
    X2 = X1 if X2 is None else _f64(X2)
    kid = KERNEL_IDS[kernel] if isinstance(kernel, str) else int(kernel)
    g = 1.0 / max(1, X1.shape[1]) if gamma is None else float(gamma)
    K = _out(X1.shape[0], X2.shape[0])
    _call("fpls_kernel_matrix", _p(X1), X1.shape[0], _p(X2), X2.shape[0], X1.shape[1], kid, g, int(degree),
          float(coef0), _p(K))
    return K


def center_kernel_train(K):
    K = _f64(K)
    n = K.shape[0]
    Kc = _out(n, n)
    cm = np.zeros(n)
    g = np.zeros(1)
    _call("fpls_center_kernel_train", _p(K), n, _p(Kc), _p(cm), _p(g))
    return dict(K=Kc, col_means=cm, grand_mean=float(g[0]))


def center_kernel_test(Ktest, col_means, grand_mean):
    Kt = _f64(Ktest)
    Kc = _out(*Kt.shape)
    _call("fpls_center_kernel_test", _p(Kt), Kt.shape[0], Kt.shape[1], _p(_f64(np.asarray(col_means))),
          float(grand_mean), _p(Kc))
    return Kc


def kernel_pls_model2_fast(X, Y, ncomp, kernel="rbf", gamma=None, degree=3, coef0=1.0, scaling=1, fit=False,
                           seed=1):
    """Kernel PLS fit in one device call (preprocess, kernel, centre, fast SIMPLS)."""
    X = _f64(X)
    Y = _f64(np.asarray(Y, dtype=np.float64).reshape(X.shape[0], -1))
    n, p = X.shape
    m = Y.shape[1]
    nc = _i32(np.atleast_1d(ncomp))
    L = nc.size
    K = int(nc.max())
    R = _out(n, K)
    Q = _out(m, K)
    mK, vK, mY = np.zeros(n), np.zeros(n), np.zeros(m)
    B = np.zeros((n, m, L), order="F")
    Yfit = np.zeros((n, m, L), order="F") if fit else None
    R2Y = np.zeros(L)
    ncd = ctypes.c_int(0)
    mX, vX, cm = np.zeros(p), np.zeros(p), np.zeros(n)
    g = np.zeros(1)
    gu = np.zeros(1)
    kid = KERNEL_IDS[kernel] if isinstance(kernel, str) else int(kernel)
    _call("fpls_kernel_pls_model2_fast", _p(X), n, p, _p(Y), m, _p(nc), L, int(scaling), kid,
          -1.0 if gamma is None else float(gamma), int(degree), float(coef0), int(bool(fit)), int(seed),
          _p(R), _p(Q), _p(mK), _p(vK), _p(mY), _p(B), None if Yfit is None else _p(Yfit), _p(R2Y),
          ctypes.byref(ncd), _p(mX), _p(vX), _p(cm), _p(g), _p(gu))
    inner = dict(R=R, Q=Q, mX=mK.reshape(1, n), vX=vK.reshape(1, n), mY=mY.reshape(1, m), B=B, R2Y=R2Y,
                 ncomp=nc, p=n, m=m, pls_method="simpls", n_components=ncd.value, B_stored=True,
                 compact_prediction=False)
    if fit:
        inner["Yfit"] = Yfit
    return dict(inner=inner, mX=mX, vX=vX, col_means=cm, grand_mean=float(g[0]), gamma=float(gu[0]),
                kernel_id=kid, degree=int(degree), coef0=float(coef0))


def _x_arg(X):
    if np.asarray(X).dtype == np.float32:
        Xa = np.asfortranarray(X, dtype=np.float32)
        return Xa, 1
    return _f64(X), 0


def cv_predict(X, y, fold, ncomp, n_classes, method=3, scaling=1, seed=1, precision="fp64",
               batched=True, return_scores=False):
    """Cross-validated class predictions (argmax classifier), folds 0-based.
    With return_scores, class_score (n x L x n_classes) holds the scores each
    argmax read (fpls_cv_predict_scores)."""
    Xa, is32 = _x_arg(X)
    n, p = Xa.shape
    yy = _i32(y)
    fd = _i32(fold)
    nc = _i32(np.atleast_1d(ncomp))
    L = nc.size
    kfold = int(fd.max()) + 1
    cp = np.zeros((n, L), dtype=np.int32, order="F")
    st = np.zeros(kfold, dtype=np.int32)
    args = (Xa.ctypes.data, is32, n, p, _p(yy), int(n_classes), _p(fd), kfold,
            _p(nc), L, int(method), int(scaling), int(seed), PREC[precision], int(bool(batched)),
            cp.ctypes.data_as(_c_int_p), _p(st))
    if not return_scores:
        _call("fpls_cv_predict", *args)
        return dict(class_pred=cp, status=st)
    sc = np.zeros((L, n, int(n_classes)))
    _call("fpls_cv_predict_scores", *args, _p(sc))
    return dict(class_pred=cp, status=st, class_score=np.ascontiguousarray(sc.transpose(1, 0, 2)))


def _double_cv_args(n, y, outer_fold, inner_fold, ncomp, return_inner, outer_ids):
    yy = _i32(y)
    of = _i32(outer_fold)
    inf_ = np.asfortranarray(np.asarray(inner_fold, dtype=np.int32))
    Ko = int(of.max()) + 1
    Ki = int(inf_.max()) + 1
    nc = _i32(np.atleast_1d(ncomp))
    L = nc.size
    ids = None if outer_ids is None else _i32(outer_ids)
    outs = dict(best_comp=np.zeros(Ko, dtype=np.int32), inner_accuracy=_out(Ko, L),
                pred=np.zeros(n, dtype=np.int32), fit_status=np.zeros(Ko * Ki + Ko, dtype=np.int32))
    if return_inner:
        outs["inner_pred"] = np.zeros((n, L, Ko), dtype=np.int32, order="F")
    return yy, of, inf_, Ko, Ki, nc, L, ids, outs


def _double_cv_result(outs, yy, ids, of):
    pred = outs["pred"]
    rows = np.ones(pred.size, dtype=bool) if ids is None else np.isin(of, ids)
    outs["accuracy"] = float(np.mean(pred[rows] == yy[rows])) if rows.any() else float("nan")
    return outs


def double_cv(X, y, outer_fold, inner_fold, ncomp, n_classes, scaling=1, seed=1, run=1,
              precision="fp64", batched=True, return_inner=False, outer_ids=None,
              return_scores=False):
    """Double CV of SIMPLS PLS-DA over the supplied outer/inner folds (0-based).

    outer_ids restricts the call to those outer folds (fpls_double_cv_outer_subset):
    only their entries of the outputs are written, the rest stay zero, and
    `accuracy` is taken over their rows.  return_scores (full calls only) adds
    inner_score (kfold_outer x L x n x n_classes), outer_score (n x n_classes)
    and inner_pred (fpls_double_cv_scores)."""
    Xa, is32 = _x_arg(X)
    n, p = Xa.shape
    if return_scores:
        if outer_ids is not None:
            raise ValueError("return_scores needs the full fold list")
        return_inner = True
    yy, of, inf_, Ko, Ki, nc, L, ids, o = _double_cv_args(n, y, outer_fold, inner_fold, ncomp,
                                                          return_inner, outer_ids)
    inner = o.get("inner_pred")
    tail = (_p(nc), L, int(scaling), int(seed), int(run), PREC[precision], int(bool(batched)),
            _p(o["best_comp"]), _p(o["inner_accuracy"]), _p(o["pred"]),
            None if inner is None else inner.ctypes.data_as(_c_int_p), _p(o["fit_status"]))
    head = (Xa.ctypes.data, is32, n, p, _p(yy), int(n_classes), _p(of), Ko,
            inf_.ctypes.data_as(_c_int_p), Ki)
    if return_scores:
        o["inner_score"] = np.zeros((Ko, L, n, int(n_classes)))
        o["outer_score"] = np.zeros((n, int(n_classes)))
        _call("fpls_double_cv_scores", *head, *tail, _p(o["inner_score"]), _p(o["outer_score"]))
    elif ids is None:
        _call("fpls_double_cv", *head, *tail)
    else:
        _call("fpls_double_cv_outer_subset", *head, _p(ids), ids.size, *tail)
    return _double_cv_result(o, yy, ids, of)


def pls_lda(Xtrain, Ytrain, y, Xtest, ncomp, n_classes, method=1, scaling=1, xprod=False, fit=False,
            oversample=10, power_iters=1, svds_tol=0.0, seed=1, lda_ridge=1e-8, store_B=True):
    """Fused PLS + LDA (fpls_pls_lda): fit, one LDA per distinct ncomp, test labels.
    Xtrain / Xtest: FP64 or FP32 (the same type for both)."""
    if _is_device(Xtrain):
        Xa = Xtrain if isinstance(Xtrain, DeviceMatrix) else DeviceMatrix(Xtrain, allow_f32=True)
        f32 = Xa.dtype == np.float32
        n, p = Xa.shape
        if Xtest is None:
            Xt = np.zeros((0, p), dtype=Xa.dtype)
        else:
            Xt = Xtest if isinstance(Xtest, DeviceMatrix) else DeviceMatrix(Xtest, allow_f32=True)
            if Xt.dtype != Xa.dtype:
                raise ValueError("Xtrain and Xtest must have the same type")
    else:
        f32 = np.asarray(Xtrain).dtype == np.float32
        dt = np.float32 if f32 else np.float64
        Xa = np.asfortranarray(Xtrain, dtype=dt)
        n, p = Xa.shape
        Xt = np.asfortranarray(np.zeros((0, p)) if Xtest is None else Xtest, dtype=dt)
    Y = _f64(Ytrain)
    m = Y.shape[1]
    yy = _i32(y)
    nc = _i32(np.maximum(np.atleast_1d(ncomp), 1))
    L = nc.size
    C = int(n_classes)
    K0 = int(nc.max()) if method == 3 else min(int(nc.max()), min(n, p, m))
    ntest = Xt.shape[0]
    o = dict(ncomp=np.zeros(L, dtype=np.int32), R=_out(p, K0), Q=_out(m, K0), mX=_out(1, p), vX=_out(1, p),
             mY=_out(1, m), B=_out(p, m, L) if store_B else None, Yfit=_out(n, m, L) if fit else None,
             R2Y=np.zeros(L), unique_ncomp=np.zeros(L, dtype=np.int32), lda_means=_out(C, K0, L),
             lda_linear=_out(C, K0, L), lda_constants=_out(C, L), lda_priors=np.zeros(C), lda_lambda=np.zeros(L),
             R_predict=_out(p, K0), R_offset=np.zeros(K0),
             pred_codes=np.zeros((max(ntest, 1), L), dtype=np.int32, order="F"))
    U = ctypes.c_int(0)
    xa_ptr = Xa.ptr if isinstance(Xa, DeviceMatrix) else Xa.ctypes.data
    xt_ptr = (Xt.ptr if isinstance(Xt, DeviceMatrix) else Xt.ctypes.data) if ntest else None
    _call("fpls_pls_lda", xa_ptr, int(f32), n, p, _p(Y), m, _p(yy), xt_ptr, ntest, _p(nc), L, C, int(method), int(scaling), int(bool(xprod)),
          int(bool(fit)), int(oversample), int(power_iters), float(svds_tol), int(seed), float(lda_ridge),
          _p(o["ncomp"]), _p(o["R"]), _p(o["Q"]), _p(o["mX"]), _p(o["vX"]), _p(o["mY"]), _p(o["B"]),
          _p(o["Yfit"]), _p(o["R2Y"]), ctypes.byref(U), _p(o["unique_ncomp"]), _p(o["lda_means"]),
          _p(o["lda_linear"]), _p(o["lda_constants"]), _p(o["lda_priors"]), _p(o["lda_lambda"]),
          _p(o["R_predict"]), _p(o["R_offset"]), _p(o["pred_codes"]) if ntest else None)
    u = U.value
    o["unique_ncomp"] = o["unique_ncomp"][:u]
    for k in ("lda_means", "lda_linear"):
        o[k] = o[k][:, :, :u]
    o["lda_constants"] = o["lda_constants"][:, :u]
    o["lda_lambda"] = o["lda_lambda"][:u]
    if not ntest:
        o.pop("pred_codes")
    if not store_B:
        o.pop("B")
    o.update(p=p, m=m, method=int(method))
    return o


def set_autotune(on=True):
    """Autotuning of the batched double-CV grids (fpls_set_autotune)."""
    _call("fpls_set_autotune", int(bool(on)))


def autotune_report():
    """The tuned grid shapes: list of dicts (shape, chosen configuration, candidates)."""
    import json
    need = ctypes.c_size_t(0)
    _call("fpls_autotune_report", None, 0, ctypes.byref(need))
    buf = ctypes.create_string_buffer(max(int(need.value), 1))
    _call("fpls_autotune_report", buf, ctypes.sizeof(buf), ctypes.byref(need))
    return [json.loads(line) for line in buf.value.decode().splitlines() if line.strip()]


def x_upload(X):
    """Registers X in device memory; returns a handle for double_cv_resident."""
    Xa, is32 = _x_arg(X)
    h = ctypes.c_int(-1)
    _call("fpls_x_upload", Xa.ctypes.data, is32, Xa.shape[0], Xa.shape[1], ctypes.byref(h))
    return h.value


class ResidentMatrix:
    """A registered device matrix seen as a column-major device matrix: pass it
    where the entry points accept device memory (fpls_x_device_pointer)."""

    def __init__(self, handle, n, p, f32=False):
        self.handle = handle
        ptr = ctypes.c_void_p(0)
        _call("fpls_x_device_pointer", int(handle), ctypes.byref(ptr))
        self.ptr = int(ptr.value)
        self.shape = (int(n), int(p))
        self.dtype = np.dtype(np.float32 if f32 else np.float64)

    @property
    def __cuda_array_interface__(self):
        n, p = self.shape
        esz = self.dtype.itemsize
        return dict(shape=(n, p), typestr="<f4" if esz == 4 else "<f8", data=(self.ptr, False),
                    strides=(esz, esz * n), version=3)

    def download(self):
        out = np.zeros(self.shape, dtype=self.dtype, order="F")
        _call("fpls_x_download", int(self.handle), out.ctypes.data_as(ctypes.c_void_p))
        return out

    def free(self):
        x_free(self.handle)


def x_resident(X):
    """Uploads X once and returns it as a ResidentMatrix."""
    Xa, is32 = _x_arg(X)
    return ResidentMatrix(x_upload(Xa), Xa.shape[0], Xa.shape[1], bool(is32))


def x_alloc(n, p, f32=False):
    """An empty resident matrix (zeros) for outputs that stay in HBM."""
    h = ctypes.c_int(-1)
    _call("fpls_x_alloc", int(n), int(p), int(bool(f32)), ctypes.byref(h))
    return ResidentMatrix(h.value, n, p, f32)


def x_free(handle):
    _call("fpls_x_free", int(handle))


def double_cv_resident(handle, n, y, outer_fold, inner_fold, ncomp, n_classes, scaling=1, seed=1,
                       run=1, precision="fp64", batched=True, return_inner=False, outer_ids=None):
    """double_cv on a registered predictor matrix (x_upload)."""
    yy, of, inf_, Ko, Ki, nc, L, ids, o = _double_cv_args(n, y, outer_fold, inner_fold, ncomp,
                                                          return_inner, outer_ids)
    inner = o.get("inner_pred")
    tail = (_p(nc), L, int(scaling), int(seed), int(run), PREC[precision], int(bool(batched)),
            _p(o["best_comp"]), _p(o["inner_accuracy"]), _p(o["pred"]),
            None if inner is None else inner.ctypes.data_as(_c_int_p), _p(o["fit_status"]))
    head = (int(handle), _p(yy), int(n_classes), _p(of), Ko, inf_.ctypes.data_as(_c_int_p), Ki)
    if ids is None:
        _call("fpls_double_cv_resident", *head, *tail)
    else:
        _call("fpls_double_cv_resident_outer_subset", *head, _p(ids), ids.size, *tail)
    return _double_cv_result(o, yy, ids, of)


def launch_count():
    return int(load().fpls_launch_count())


def last_call_ms():
    return float(load().fpls_last_call_ms())


def profile_begin():
    _call("fpls_profile", 1, None, None, None)


def profile_end():
    ms = ctypes.c_double(0.0)
    cnt = ctypes.c_longlong(0)
    by = ctypes.c_double(0.0)
    _call("fpls_profile", 0, ctypes.byref(ms), ctypes.byref(cnt), ctypes.byref(by))
    return dict(ms=ms.value, launches=cnt.value, bytes=by.value)


def profile_classes():
    """Per-kernel-class timings of the last closed profiling window."""
    out = []
    idx = 0
    lib = load()
    while True:
        name = ctypes.create_string_buffer(64)
        ms, by, fl = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
        cnt = ctypes.c_longlong(0)
        err = ctypes.create_string_buffer(256)
        rc = lib.fpls_profile_class(idx, name, 64, ctypes.byref(ms), ctypes.byref(cnt), ctypes.byref(by),
                                    ctypes.byref(fl), err, 256)
        if rc != 0:
            break
        out.append(dict(name=name.value.decode(), ms=ms.value, launches=cnt.value, bytes=by.value,
                        flops=fl.value))
        idx += 1
    return out


def gaussian_y_encode(Y, projection):
    """Regression response compression (R/main.R:2000-2064); projection q x d."""
    Y = _f64(Y)
    G = _f64(projection)
    n, q = Y.shape
    d = G.shape[1]
    Z, mu, dec = _out(n, d), np.zeros(q), _out(d, q)
    _call("fpls_gaussian_y_encode", _p(Y), n, q, _p(G), d, _p(Z), _p(mu), _p(dec))
    return dict(Z=Z, y_center=mu, decoder=dec)


def gaussian_y_decode(Z, decoder, y_center, out=None):
    Z = _f64(Z)
    D = _f64(decoder)
    mu = np.ascontiguousarray(y_center, dtype=np.float64).ravel()
    w, d = Z.shape
    q = D.shape[1]
    Y = _out(w, q) if out is None else _f64(out)
    _call("fpls_gaussian_y_decode", _p(Z), w, d, _p(D), _p(mu), q, _p(Y))
    return Y


def nearest_code_classes(Z, codes):
    Z = _f64(Z)
    C = _f64(codes)
    lab = np.zeros(Z.shape[0], dtype=np.int32)
    _call("fpls_nearest_code_classes", _p(Z), Z.shape[0], Z.shape[1], _p(C), C.shape[0], _p(lab))
    return lab


def opls_filter(X, Y, north, scaling=1, out=None):
    """OPLS filter; `out` (optional, n x p, host or device) receives the filtered X."""
    X = _f64(X)
    Y = _f64(Y)
    n, p = X.shape
    q = Y.shape[1]
    Xf = _out(n, p) if out is None else _f64(out)
    mX, vX = np.zeros(p), np.zeros(p)
    W, P = _out(p, max(north, 1)), _out(p, max(north, 1))
    used = ctypes.c_int(0)
    _call("fpls_opls_filter", _p(X), n, p, _p(Y), q, int(north), int(scaling), _p(Xf), _p(mX),
          _p(vX), _p(W), _p(P), ctypes.byref(used))
    k = used.value
    return dict(X=Xf, mX=mX, vX=vX, W_orth=W[:, :k], P_orth=P[:, :k], north=k)


def opls_apply_filter(X, mX, vX, W_orth, P_orth, out=None):
    X = _f64(X)
    w, p = X.shape
    W = _f64(W_orth)
    P = _f64(P_orth)
    out = _out(w, p) if out is None else _f64(out)
    _call("fpls_opls_apply_filter", _p(X), w, p, _p(np.ascontiguousarray(mX, dtype=np.float64).ravel()),
          _p(np.ascontiguousarray(vX, dtype=np.float64).ravel()), _p(W), _p(P), W.shape[1], _p(out))
    return out


def candidate_scores(T, Ck=None):
    """row_l2(T Ck) (R/main.R:657-662, 700-730)."""
    T = _f64(T)
    n, k = T.shape
    out = _out(n, k)
    _call("fpls_candidate_scores", _p(T), n, k, _p(_f64(Ck)) if Ck is not None else None, _p(out))
    return out


def candidate_centroids(Tn, y_codes, n_classes):
    Tn = _f64(Tn)
    n, k = Tn.shape
    y = np.ascontiguousarray(y_codes, dtype=np.int32)
    out = _out(n_classes, k)
    _call("fpls_candidate_centroids", _p(Tn), n, k, _p(y), int(n_classes), _p(out))
    return out


def candidate_knn_predict(Ttest_norm, Ttrain_norm, y_codes, centroids, bias=None, top_k=1,
                          top_m=20, knn_k=3, tau=0.2, alpha=0.5):
    Tt = _f64(Ttest_norm)
    Tr = _f64(Ttrain_norm)
    C = _f64(centroids)
    y = np.ascontiguousarray(y_codes, dtype=np.int32)
    ntest, k = Tt.shape
    nc = C.shape[0]
    tk = max(1, min(int(top_k), nc))
    ti = np.zeros((ntest, tk), dtype=np.int32, order="F")
    ts = _out(ntest, tk)
    b = None if bias is None else np.ascontiguousarray(bias, dtype=np.float64)
    _call("fpls_candidate_knn_predict", _p(Tt), ntest, _p(Tr), Tr.shape[0], k, _p(y), _p(C), nc,
          _p(b) if b is not None else None, int(top_k), int(top_m), int(knn_k), float(tau),
          float(alpha), _p(ti), _p(ts))
    return dict(top_index=ti, top_score=ts)


def plssvd_label_aware(X, y_codes, m, ncomp, scaling=1, svd_method=3, oversample=10,
                       power_iters=1, seed=1, keep_scores=False):
    """Label-aware PLSSVD (R/main.R:513-655); X float32 or float64, y_codes 1..m."""
    X = np.asfortranarray(X)
    f32 = X.dtype == np.float32
    if not f32:
        X = _f64(X)
    n, p = X.shape
    y = np.ascontiguousarray(y_codes, dtype=np.int32)
    nc = np.ascontiguousarray(ncomp, dtype=np.int32)
    L = len(nc)
    K = int(min(max(int(nc.max()), 1), n, p, m))
    out = dict(C_latent=np.zeros((K, K, L), order="F"), W_latent=np.zeros((K, m, L), order="F"),
               Q=_out(m, K), R=_out(p, K), mX=np.zeros(p), vX=np.zeros(p), mY=np.zeros(m),
               s=np.zeros(K))
    T = _out(n, K) if keep_scores else None
    nco = np.zeros(L, dtype=np.int32)
    kr = ctypes.c_int(0)
    _call("fpls_plssvd_label_aware", X.ctypes.data_as(ctypes.c_void_p), int(f32), n, p, _p(y), int(m),
          _p(nc), L, int(scaling), int(svd_method), int(oversample), int(power_iters), int(seed),
          _p(nco), _p(out["C_latent"]), _p(out["W_latent"]), _p(out["Q"]), _p(out["R"]),
          _p(out["mX"]), _p(out["vX"]), _p(out["mY"]), _p(out["s"]), _p(T), ctypes.byref(kr))
    out["ncomp"] = nco
    out["max_rank"] = kr.value
    if keep_scores:
        out["Ttrain"] = T
    return out


def _knn_out(ntest, m, top_k):
    tk = max(1, min(int(top_k), int(m)))
    return np.zeros((ntest, tk), dtype=np.int32, order="F"), _out(ntest, tk)


def label_aware_cknn(Xtrain, y_codes, m, Xtest, ncomp, scaling=1, svd_method=4, oversample=10,
                     power_iters=1, seed=1, knn_k=10, tau=0.2, alpha=0.75, top_m=20, top_k=5):
    """Label-aware PLSSVD + candidate-kNN on host buffers (FP32 or FP64, same type)."""
    f32 = np.asarray(Xtrain).dtype == np.float32
    dt = np.float32 if f32 else np.float64
    Xtr = np.asfortranarray(Xtrain, dtype=dt)
    Xte = np.asfortranarray(Xtest, dtype=dt)
    y = np.ascontiguousarray(y_codes, dtype=np.int32)
    ti, ts = _knn_out(Xte.shape[0], m, top_k)
    _call("fpls_label_aware_cknn", Xtr.ctypes.data_as(ctypes.c_void_p), int(f32), Xtr.shape[0],
          Xtr.shape[1], _p(y), int(m), Xte.ctypes.data_as(ctypes.c_void_p), Xte.shape[0], int(ncomp),
          int(scaling), int(svd_method), int(oversample), int(power_iters), int(seed), int(knn_k),
          float(tau), float(alpha), int(top_m), int(top_k), _p(ti), _p(ts))
    return dict(top_index=ti, top_score=ts)


def label_aware_cknn_resident(xtrain_handle, y_codes, m, xtest_handle, ntest, ncomp, scaling=1,
                              svd_method=4, oversample=10, power_iters=1, seed=1, knn_k=10, tau=0.2,
                              alpha=0.75, top_m=20, top_k=5):
    y = np.ascontiguousarray(y_codes, dtype=np.int32)
    ti, ts = _knn_out(ntest, m, top_k)
    _call("fpls_label_aware_cknn_resident", int(xtrain_handle), _p(y), int(m), int(xtest_handle),
          int(ncomp), int(scaling), int(svd_method), int(oversample), int(power_iters), int(seed),
          int(knn_k), float(tau), float(alpha), int(top_m), int(top_k), _p(ti), _p(ts))
    return dict(top_index=ti, top_score=ts)


def gaussian_sketch(rows, cols, seed):
    """The device-drawn Gaussian sketch (mt19937 + normal_distribution stream)."""
    out = _out(rows, cols)
    _call("fpls_gaussian_sketch", int(rows), int(cols), int(seed) & 0xFFFFFFFF, _p(out))
    return out


def host_register(a):
    """Pins the memory of numpy array `a` (page-locked) until host_unregister."""
    _call("fpls_host_register", ctypes.c_void_p(a.ctypes.data), ctypes.c_size_t(a.nbytes))


def host_unregister(a):
    _call("fpls_host_unregister", ctypes.c_void_p(a.ctypes.data))


def set_precision(precision):
    """Session precision of single fits and predictions: "fp64", "bf16x3" or "bf16x6"."""
    _call("fpls_set_precision", PREC[precision] if isinstance(precision, str) else int(precision))


def get_precision():
    return {v: k for k, v in PREC.items()}[int(load().fpls_get_precision())]

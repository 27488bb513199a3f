"""GPU tests of the FP64-accurate INT8 tensor-core product (digit planes on
tcgen05 kind::i8) against its CPU model and the FP64 product, and of its use
for the row-space K products of the mixed-precision CV grids."""
import os

import numpy as np
import pytest

import int8_model as im
from fastpls_b200 import synthetic
from fastpls_b200.folds import double_cv_folds

pytestmark = pytest.mark.gpu


def _model_close(C, A, B, slices):
    # the kernel and the model sum the same exact integer levels; only the FP64
    # combination order (per stream-K segment) differs
    ref = im.product(A, B, slices)
    scale = np.abs(A) @ np.abs(B)
    return np.all(np.abs(C - ref) <= 1e-14 * scale + 1e-300)


@pytest.mark.parametrize("M,K,N", [(128, 128, 64), (300, 257, 60), (3000, 3000, 60), (129, 1000, 65),
                                   (200, 1000, 240), (1, 1, 1), (77, 8300, 5)])
@pytest.mark.parametrize("slices", [7, 5])
def test_int8_product_random(lib, M, K, N, slices):
    rng = np.random.default_rng(M * 7 + K + N)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    C = lib.int8_emulated_gemm(A, B, slices)
    assert np.all(np.abs(C - A @ B) <= im.error_bound(A, B, slices))
    assert _model_close(C, A, B, slices)


def test_int8_product_dynamic_range_and_zeros(lib):
    rng = np.random.default_rng(4)
    A = rng.standard_normal((500, 700)) * np.logspace(-8, 8, 500)[:, None]
    B = rng.standard_normal((700, 90)) * np.logspace(5, -5, 90)[None, :]
    A[17] = 0.0
    B[:, 3] = 0.0
    C = lib.int8_emulated_gemm(A, B, 7)
    assert np.all(C[17] == 0.0) and np.all(C[:, 3] == 0.0)
    assert np.all(np.abs(C - A @ B) <= im.error_bound(A, B, 7))


def test_int8_product_integers_exact(lib):
    # one digit per entry: the product is exact whatever the slice count
    rng = np.random.default_rng(8)
    A = rng.integers(-100, 101, size=(640, 1500)).astype(np.float64)
    B = rng.integers(-100, 101, size=(1500, 64)).astype(np.float64)
    for slices in (4, 7):
        assert np.array_equal(lib.int8_emulated_gemm(A, B, slices), A @ B)


def test_int8_product_nonfinite_column(lib):
    rng = np.random.default_rng(9)
    A = rng.standard_normal((200, 300))
    B = rng.standard_normal((300, 10))
    B[5, 2] = np.nan
    C = lib.int8_emulated_gemm(A, B, 7)
    assert np.all(np.isnan(C[:, 2]))
    keep = [j for j in range(10) if j != 2]
    assert np.all(np.abs(C[:, keep] - A @ B[:, keep]) <= im.error_bound(A, B[:, keep], 7))


def test_int8_product_rejects_bad_slices(lib):
    with pytest.raises(lib.FastPLSError):
        lib.int8_emulated_gemm(np.ones((4, 4)), np.ones((4, 4)), 9)


@pytest.fixture(scope="module")
def c4_mid():
    return synthetic.c4_omics(seed=6, n=600, p=2400, n_informative=30)


def _double_cv(lib, d, kprod):
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=2)
    os.environ["FASTPLS_KPROD"] = kprod
    try:
        return lib.double_cv(d["X"], d["y"], outer, inner, ncomp=list(range(1, 16)),
                             n_classes=d["n_classes"], seed=3, precision="bf16x3")
    finally:
        os.environ.pop("FASTPLS_KPROD", None)


def test_row_space_int8_k_products_match_fp64(lib, c4_mid):
    # the mixed-precision grid with its K products on the INT8 tensor cores
    # against the same grid with FP64 DMMA K products
    a = _double_cv(lib, c4_mid, "int8")
    b = _double_cv(lib, c4_mid, "fp64")
    assert np.array_equal(a["best_comp"], b["best_comp"])
    assert np.mean(a["pred"] == b["pred"]) >= 0.999
    assert np.nanmax(np.abs(a["inner_accuracy"] - b["inner_accuracy"])) <= 2e-3

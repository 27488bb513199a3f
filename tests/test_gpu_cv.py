"""GPU tests of the BF16 split tensor-core GEMM and of the CV grids."""
import numpy as np
import pytest

from oracle import cv as ocv
from fastpls_b200 import synthetic
from fastpls_b200.folds import double_cv_folds, stratified_group_folds
from parity_utils import rel_err

pytestmark = pytest.mark.gpu

# BF16 hi/lo three-product error: ~3 * 2^-17 per product, accumulated in FP32.
SPLIT_REL_TOL = 1e-4


@pytest.mark.parametrize("M,K,N", [(128, 64, 64), (300, 1000, 50), (1000, 3000, 7), (20000, 700, 64),
                                   (257, 129, 130)])
def test_bf16x3_gemm_random(lib, M, K, N):
    rng = np.random.default_rng(M + K + N)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    C = lib.bf16x3_gemm(A, B)
    assert rel_err(C, A @ B) < SPLIT_REL_TOL


def test_bf16x3_gemm_exact_inputs(lib):
    # Inputs exactly representable in BF16 (lo = 0): the only error left is the
    # FP32 accumulation, so a layout or pipeline bug cannot hide in the tolerance.
    rng = np.random.default_rng(3)
    A = rng.integers(-8, 9, size=(777, 1024)).astype(np.float64) / 8.0
    B = rng.integers(-8, 9, size=(1024, 40)).astype(np.float64) / 4.0
    C = lib.bf16x3_gemm(A, B)
    assert np.array_equal(C, A @ B)


@pytest.fixture(scope="module")
def c4_small():
    d = synthetic.c4_omics(seed=2, n=360, p=600, n_informative=20)
    return d


def _labels_agree(a, b, frac=0.995):
    return np.mean(np.asarray(a) == np.asarray(b)) >= frac


@pytest.mark.parametrize("batched", [True, False])
def test_cv_predict_fp64_matches_oracle(lib, c4_small, batched):
    d = c4_small
    rng = np.random.default_rng(1)
    fold = stratified_group_folds(d["y"], d["groups"], 5, rng)
    nc = np.arange(1, 11)
    got = lib.cv_predict(d["X"], d["y"], fold, nc, d["n_classes"], seed=7, batched=batched)
    ref = ocv.pls_cv_predict_compiled(d["X"].astype(np.float64), d["y"], fold, nc, d["n_classes"],
                                      seed=7)
    assert np.array_equal(got["status"], ref["status"])
    assert _labels_agree(got["class_pred"], ref["class_pred"], 0.999)


def test_double_cv_fp64_matches_oracle(lib, c4_small):
    d = c4_small
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=5)
    nc = np.arange(1, 9)
    got = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, batched=True)
    seq = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, batched=False)
    ref = ocv.double_cv(d["X"].astype(np.float64), d["y"], outer, inner, nc, d["n_classes"], seed=1)
    assert np.array_equal(got["best_comp"], ref["best_comp"])
    assert np.allclose(got["inner_accuracy"], ref["inner_accuracy"], atol=2e-3)
    assert _labels_agree(got["pred"], ref["pred"], 0.99)
    assert np.array_equal(seq["best_comp"], ref["best_comp"])
    assert _labels_agree(seq["pred"], ref["pred"], 0.99)


def test_double_cv_bf16x3_close_to_fp64(lib, c4_small):
    d = c4_small
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=5)
    nc = np.arange(1, 9)
    a = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, precision="fp64")
    b = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, precision="bf16x3")
    assert np.allclose(a["inner_accuracy"], b["inner_accuracy"], atol=5e-3)
    assert _labels_agree(a["pred"], b["pred"], 0.99)

"""The row Gram on the INT8 tensor cores (fpls_int8_gram, the FPLS_PREC_INT8
CV grids): digit planes of the centred rows, exact int32 plane products on the
upper tiles with an L2-sharing stream-K plan, FP64 combination, mirrored lower
triangle.  Checked entry by entry against the Ozaki error bound
3 p 2^(e_i + e_j - 7 slices) around the exact FP64 product."""
import numpy as np
import pytest

from fastpls_b200 import synthetic
from fastpls_b200.folds import double_cv_folds
from parity_utils import REL_TOL, cv_labels_match, slice_score_rel_err

pytestmark = pytest.mark.gpu


def _bound(Xc, slices):
    e = np.frexp(np.abs(Xc).max(axis=1))[1].astype(np.float64)
    return 3.0 * Xc.shape[1] * np.exp2(e[:, None] + e[None, :] - 7.0 * slices)


@pytest.mark.parametrize("n,p,slices", [(700, 3000, 4), (257, 1000, 5), (1000, 700, 7), (129, 130, 6)])
def test_int8_gram_within_bound(lib, n, p, slices):
    rng = np.random.default_rng(n + p)
    X = rng.standard_normal((n, p)) * np.exp(rng.standard_normal((n, 1)))   # row scales differ
    mean = X.mean(axis=0)
    K = lib.int8_gram(X, slices=slices, mean=mean)
    Xc = X - mean
    ref = Xc @ Xc.T
    assert np.array_equal(K, K.T)
    assert np.all(np.abs(K - ref) <= _bound(Xc, slices))


def test_int8_gram_fp32_input_and_nonfinite_rows(lib):
    rng = np.random.default_rng(4)
    X32 = rng.standard_normal((300, 900)).astype(np.float32)
    K = lib.int8_gram(X32, slices=5)
    X = X32.astype(np.float64)
    assert np.all(np.abs(K - X @ X.T) <= _bound(X, 5))
    X[7, 3] = np.inf
    K = lib.int8_gram(X, slices=4)
    assert np.all(np.isnan(K[7])) and np.all(np.isnan(K[:, 7]))
    ok = np.setdiff1d(np.arange(300), [7])
    assert np.all(np.isfinite(K[np.ix_(ok, ok)]))


def test_int8_double_cv_close_to_fp64(lib):
    d = synthetic.c4_omics(seed=9, n=360, p=1500, n_informative=20)
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=3)
    nc = np.arange(1, 11)
    kw = dict(seed=1, return_scores=True)
    a = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], precision="fp64", **kw)
    b = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], precision="int8", **kw)
    assert np.array_equal(a["best_comp"], b["best_comp"])
    assert np.array_equal(a["pred"], b["pred"])
    assert slice_score_rel_err(b["inner_score"], a["inner_score"]) < 1e-5
    assert cv_labels_match(b["inner_pred"], a["inner_pred"], np.transpose(a["inner_score"], (2, 1, 0, 3)), 1e-5)[0]


def test_int8_double_cv_host_chunks(lib):
    """A host X wider than one upload chunk (bounds 0, 4096, 7936, 9000): each
    chunk's digit planes carry their own row scales and its share of the row
    Gram and of the sketch product is added as it lands.  The grid stays within
    1e-5 of the FP64 grid's class scores and agrees with the INT8 grid on the
    resident matrix (one set of row scales over all columns)."""
    d = synthetic.c4_omics(seed=11, n=300, p=9000, n_informative=20)
    outer, inner = double_cv_folds(d["y"], d["groups"], 3, 3, seed=5)
    nc = np.arange(1, 9)
    kw = dict(seed=1, return_scores=True)
    a = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], precision="fp64", **kw)
    b = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], precision="int8", **kw)
    assert np.array_equal(a["best_comp"], b["best_comp"])
    assert np.array_equal(a["pred"], b["pred"])
    assert slice_score_rel_err(b["inner_score"], a["inner_score"]) < 1e-5
    assert cv_labels_match(b["inner_pred"], a["inner_pred"], np.transpose(a["inner_score"], (2, 1, 0, 3)), 1e-5)[0]
    h = lib.x_upload(d["X"])
    try:
        r = lib.double_cv_resident(h, d["X"].shape[0], d["y"], outer, inner, nc, d["n_classes"], seed=1,
                                   precision="int8")
    finally:
        lib.x_free(h)
    assert np.array_equal(r["best_comp"], b["best_comp"])
    assert np.array_equal(r["pred"], b["pred"])
    assert np.max(np.abs(r["inner_accuracy"] - b["inner_accuracy"])) <= 2.0 / d["X"].shape[0]

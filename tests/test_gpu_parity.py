"""GPU parity of the FP64 drop-in against the CPU oracle, through the C ABI.

Sizes are the benchmark shapes where the oracle finishes in seconds (C1 at full
size) and scaled-down versions of the larger configs.
"""
import numpy as np
import pytest

from oracle import lda as olda
from oracle import pls as opls
from oracle import svd as osvd
from fastpls_b200 import synthetic
from parity_utils import ANGLE_TOL, REL_TOL, labels_match_beyond_margin, rel_err, sign_align, subspace_angle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    return synthetic.c1_simpls_regression(seed=1)


@pytest.fixture(scope="module")
def c2_small():
    d = synthetic.c2_plsda(seed=3, n=3000, n_test=600, p=800, n_classes=20)
    d["Y"] = opls.transformy(d["ytrain"])
    return d


def test_matrix_multiply(lib):
    rng = np.random.default_rng(0)
    for (m, k, n) in [(1, 1, 1), (37, 129, 3), (300, 1000, 70), (513, 65, 257)]:
        A = rng.standard_normal((m, k))
        B = rng.standard_normal((k, n))
        assert rel_err(lib.matrix_multiply(A, B), A @ B) < 1e-13


@pytest.mark.parametrize("method,power", [(4, 1), (4, 2), (4, 0), (3, 1)])
def test_truncated_svd(lib, method, power):
    rng = np.random.default_rng(5)
    U = np.linalg.qr(rng.standard_normal((400, 30)))[0]
    V = np.linalg.qr(rng.standard_normal((90, 30)))[0]
    s = 5.0 * 0.85 ** np.arange(30)
    A = (U * s) @ V.T + 1e-3 * rng.standard_normal((400, 90))
    k = 12
    got = lib.truncated_svd(A, k, svd_method=method, oversample=10, power_iters=power, seed=7)
    ref = osvd.truncated_svd(A, k, method, 10, power, 7, left_only=False)
    assert got["u"].shape == ref.U.shape
    assert rel_err(got["d"], ref.s) < REL_TOL
    assert subspace_angle(got["u"], ref.U) < ANGLE_TOL
    assert rel_err(sign_align(got["u"], ref.U), ref.U) < 1e-8
    assert rel_err((got["u"] * got["d"]) @ got["vt"], (ref.U * ref.s) @ ref.Vt) < REL_TOL


def test_truncated_svd_exact_small(lib):
    # fastsvd(...) on a 40 x 5 matrix equals a full SVD (test-svd-public-tools.R:42-61)
    rng = np.random.default_rng(11)
    A = rng.standard_normal((40, 5))
    got = lib.truncated_svd(A, 5, svd_method=4)
    U, s, Vt = np.linalg.svd(A, full_matrices=False)
    assert np.allclose(got["d"], s, atol=1e-12, rtol=1e-12)
    assert np.allclose(np.abs(got["u"]), np.abs(U), atol=1e-10)
    assert np.allclose(np.abs(got["vt"]), np.abs(Vt), atol=1e-10)


def _check_simpls(got, ref, L):
    assert rel_err(got["B"], ref["B"]) < REL_TOL
    K = ref["R"].shape[1]
    assert rel_err(sign_align(got["R"], ref["R"]), ref["R"]) < 1e-8
    assert rel_err(sign_align(got["Q"], ref["Q"]), ref["Q"]) < 1e-8
    assert np.allclose(got["mX"], ref["mX"], rtol=1e-13, atol=1e-14)
    assert K == got["R"].shape[1]


@pytest.mark.parametrize("scaling", [1, 2, 3])
def test_simpls_fast_c1(lib, c1, scaling):
    X, Y, Xt = c1["Xtrain"], c1["Ytrain"], c1["Xtest"]
    nc = [1, 3, 10]
    got = lib.pls_model2_fast(X, Y, nc, scaling=scaling, fit=True, seed=1)
    ref = opls.pls_model2_fast(X, Y, nc, scaling=scaling, fit=True, seed=1)
    assert got["n_components"] == 10
    _check_simpls(got, ref, len(nc))
    # reference signs: refresh vectors follow the Householder convention r[0] <= 0
    assert np.allclose(got["R"], ref["R"], rtol=1e-8, atol=1e-12)
    assert rel_err(got["Yfit"], ref["Yfit"]) < REL_TOL
    assert np.allclose(got["R2Y"], ref["R2Y"], rtol=1e-9, atol=1e-12)
    pg = lib.predict_lowrank(got, Xt)["Ypred"]
    pr = opls.pls_predict(ref, Xt)["Ypred"]
    assert rel_err(pg, pr) < REL_TOL


def test_simpls_fast_single_response(lib, c1):
    X, Y = c1["Xtrain"], c1["Ytrain"][:, :1]
    got = lib.pls_model2_fast(X, Y, [1, 2, 6], seed=3)
    ref = opls.pls_model2_fast(X, Y, [1, 2, 6], seed=3)
    assert rel_err(got["B"], ref["B"]) < REL_TOL


def test_simpls_fast_unsorted_ncomp(lib, c1):
    # slices are filled exactly where the reference's while-loop fills them
    X, Y = c1["Xtrain"], c1["Ytrain"]
    got = lib.pls_model2_fast(X, Y, [5, 2, 7], fit=True, seed=2)
    ref = opls.pls_model2_fast(X, Y, [5, 2, 7], fit=True, seed=2)
    assert rel_err(got["B"], ref["B"]) < REL_TOL
    assert rel_err(got["Yfit"], ref["Yfit"]) < REL_TOL


@pytest.mark.parametrize("method", [3, 4])
def test_simpls_classic_c1(lib, c1, method):
    X, Y = c1["Xtrain"], c1["Ytrain"]
    got = lib.pls_model2(X, Y, [2, 10], fit=True, svd_method=method, power_iters=2, seed=1)
    ref = opls.pls_model2(X, Y, [2, 10], fit=True, svd_method=method, rsvd_power=2, seed=1)
    assert rel_err(got["B"], ref["B"]) < REL_TOL
    assert rel_err(sign_align(got["R"], ref["R"]), ref["R"]) < 1e-8
    assert rel_err(got["Yfit"], ref["Yfit"]) < REL_TOL
    assert np.allclose(got["R2Y"], ref["R2Y"], rtol=1e-9)


@pytest.mark.parametrize("method,power", [(4, 2), (4, 1), (3, 1)])
def test_plssvd_c2_small(lib, c2_small, method, power):
    X = c2_small["Xtrain"].astype(np.float64)
    Y = c2_small["Y"]
    nc = [1, 5, 10, 15]
    got = lib.pls_model1(X, Y, nc, fit=True, svd_method=method, oversample=10, power_iters=power, seed=1)
    ref = opls.pls_model1(X, Y, nc, fit=True, svd_method=method, rsvd_oversample=10, rsvd_power=power, seed=1)
    assert np.array_equal(got["ncomp"], ref["ncomp"])
    assert rel_err(got["singular_values"], ref["singular_values"]) < REL_TOL
    assert subspace_angle(got["R"], ref["R"]) < ANGLE_TOL
    assert rel_err(got["B"], ref["B"]) < REL_TOL
    assert rel_err(got["Yfit"], ref["Yfit"]) < REL_TOL
    assert np.allclose(got["R2Y"], ref["R2Y"], rtol=1e-9)
    Xt = c2_small["Xtest"].astype(np.float64)
    pg = lib.predict_lowrank(got, Xt)["Ypred"]
    pr = opls.pls_predict(ref, Xt, use_B=True)["Ypred"]
    assert rel_err(pg, pr) < REL_TOL
    cls = lib.predict_classes(got, Xt)["top_index"][:, 0, :]
    for a in range(len(nc)):
        ok, _ = labels_match_beyond_margin(cls[:, a], opls.argmax_first(pr[:, :, a]), pr[:, :, a])
        assert ok


def test_plssvd_small_exact_route(lib, c1):
    # min(n, p, m) <= 32 takes the exact SVD (fastPLS.cpp:318-324)
    X, Y = c1["Xtrain"], c1["Ytrain"]
    got = lib.pls_model1(X, Y, [1, 3, 5], svd_method=4, seed=1)
    ref = opls.pls_model1(X, Y, [1, 3, 5], svd_method=4, seed=1)
    assert rel_err(got["B"], ref["B"]) < REL_TOL
    assert subspace_angle(got["R"], ref["R"]) < ANGLE_TOL


def test_topk_classes(lib, c2_small):
    X = c2_small["Xtrain"].astype(np.float64)
    Y = c2_small["Y"]
    model = lib.pls_model1(X, Y, [8], svd_method=4, power_iters=2, seed=1)
    Xt = c2_small["Xtest"].astype(np.float64)
    bias = np.linspace(-0.01, 0.01, Y.shape[1])
    got = lib.predict_classes(model, Xt, class_bias=bias, top_k=5, return_scores=True)
    pr = opls.pls_predict(model, Xt, use_B=False)["Ypred"][:, :, 0] + bias
    order = np.argsort(-pr, axis=1, kind="stable")[:, :5] + 1
    assert np.array_equal(got["top_index"][:, :, 0], order)
    assert rel_err(got["top_score"][:, :, 0], np.take_along_axis(pr, order - 1, axis=1)) < 1e-12


def test_lda_prefix(lib, c2_small):
    X = c2_small["Xtrain"].astype(np.float64)
    y = c2_small["ytrain"]
    C = c2_small["n_classes"]
    model = opls.pls_model1(X, opls.transformy(y), [12], svd_method=4, rsvd_power=2, seed=1)
    Rp = model["R"] / model["vX"].T
    off = (model["mX"] @ Rp).ravel()
    nc = [3, 7, 12]
    got = lib.lda_project_train_prefix(X, Rp, off, y, C, nc, ridge=1e-8)
    ref = olda.lda_project_train_prefix(X, Rp, off, y, C, nc, ridge=1e-8)
    for kk in nc:
        g, r = got[str(kk)], ref[str(kk)]
        assert rel_err(g["means"], r["means"]) < 1e-12
        assert rel_err(g["linear"], r["linear"]) < REL_TOL
        assert rel_err(g["constants"], r["constants"]) < REL_TOL
        assert abs(g["ridge"] - r["ridge"]) <= 1e-12 * abs(r["ridge"])
    Xt = c2_small["Xtest"].astype(np.float64)
    for kk in nc:
        g = lib.lda_project_predict(Xt, Rp[:, :kk], off[:kk], got[str(kk)], return_scores=True)
        r_lab, r_scores = olda.lda_project_predict(Xt, Rp[:, :kk], off[:kk], ref[str(kk)], return_scores=True)
        ok, nclear = labels_match_beyond_margin(g["pred"], r_lab, r_scores)
        assert ok and nclear > 0.9 * Xt.shape[0]
        assert rel_err(g["scores"], r_scores) < REL_TOL


def test_lda_train_on_scores(lib):
    rng = np.random.default_rng(2)
    T = rng.standard_normal((500, 6))
    y = rng.integers(1, 5, size=500).astype(np.int32)
    got = lib.lda_train_prefix(T, y, 4, [2, 6])
    ref = olda.lda_train_prefix(T, y, 4, [2, 6])
    for kk in ("2", "6"):
        assert rel_err(got[kk]["linear"], ref[kk]["linear"]) < 1e-11
        assert rel_err(got[kk]["constants"], ref[kk]["constants"]) < 1e-11
        lab = lib.lda_predict(T[:, :int(kk)], got[kk])["pred"]
        assert np.array_equal(lab, olda.lda_predict_labels(T[:, :int(kk)], ref[kk]))


def test_errors_are_status_codes(lib):
    from fastpls_b200._lib import FastPLSError
    with pytest.raises(FastPLSError):
        lib.lda_train_prefix(np.ones((4, 2)), np.array([1, 1, 1, 1], dtype=np.int32), 2, [1])
    with pytest.raises(FastPLSError):
        lib.lda_train_prefix(np.ones((4, 2)), np.array([1, 2, 3, 1], dtype=np.int32), 2, [1])


def test_fp64_runs_repeat_bit_for_bit(lib, c1, c2_small):
    # Split-K partial sums and LDA class sums are added in a fixed order (no
    # atomics), so the FP64 drop-in gives identical bits on every run.
    X, Y = c1["Xtrain"], c1["Ytrain"]
    a = lib.pls_model2_fast(X, Y, [3, 10], fit=True, seed=1)
    b = lib.pls_model2_fast(X, Y, [3, 10], fit=True, seed=1)
    assert np.array_equal(a["B"], b["B"]) and np.array_equal(a["Yfit"], b["Yfit"])
    Xc = c2_small["Xtrain"].astype(np.float64)
    y = c2_small["ytrain"]
    m1 = lib.pls_model1(Xc, c2_small["Y"], [8], svd_method=4, power_iters=2, seed=1)
    m2 = lib.pls_model1(Xc, c2_small["Y"], [8], svd_method=4, power_iters=2, seed=1)
    assert np.array_equal(m1["B"], m2["B"])
    Rp = m1["R"] / m1["vX"].T
    off = (m1["mX"] @ Rp).ravel()
    l1 = lib.lda_project_train_prefix(Xc, Rp, off, y, c2_small["n_classes"], [4, 8])
    l2 = lib.lda_project_train_prefix(Xc, Rp, off, y, c2_small["n_classes"], [4, 8])
    for kk in ("4", "8"):
        assert np.array_equal(l1[kk]["linear"], l2[kk]["linear"])
        assert np.array_equal(l1[kk]["constants"], l2[kk]["constants"])


@pytest.mark.parametrize("top_k,scores", [(5, True), (1, False)])
def test_class_prediction_streamed_in_row_blocks(lib, c2_small, monkeypatch, top_k, scores):
    # test rows scored in blocks (the copy of the next block in flight) give the
    # predictions of the one-block call
    X = c2_small["Xtrain"].astype(np.float64)
    model = lib.pls_model1(X, c2_small["Y"], [4, 8], svd_method=4, power_iters=2, seed=1)
    Xt = c2_small["Xtest"].astype(np.float64)
    bias = np.linspace(-0.02, 0.02, c2_small["Y"].shape[1])
    one = lib.predict_classes(model, Xt, class_bias=bias, top_k=top_k, return_scores=scores)
    monkeypatch.setenv("FASTPLS_PREDICT_BLOCK_ROWS", "37")
    blk = lib.predict_classes(model, Xt, class_bias=bias, top_k=top_k, return_scores=scores)
    assert np.array_equal(blk["top_index"], one["top_index"])
    if scores:
        assert np.max(np.abs(blk["top_score"] - one["top_score"])) < 1e-12

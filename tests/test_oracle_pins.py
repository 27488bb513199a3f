"""Pins the CPU oracle (no GPU).

The reference's tests hold no golden vectors; the oracle is pinned against the
C++ standard's RNG known answer, the identities the reference's own tests
assert, and closed-form known answers.
"""
import numpy as np
import pytest

from oracle import lda as olda
from oracle import pls as opls
from oracle import svd as osvd
from oracle.rng import gaussian_matrix, mt19937_raw
from fastpls_b200 import synthetic


def test_mt19937_known_answer():
    # C++ standard [rand.predef]: the 10000th draw of a default-constructed mt19937.
    assert int(mt19937_raw(10000, seed=5489)[-1]) == 4123659995


def test_gaussian_matrix_column_major_stream():
    a = gaussian_matrix(7, 3, 11)
    b = gaussian_matrix(21, 1, 11)
    assert np.array_equal(a.ravel(order="F"), b.ravel())
    assert not np.array_equal(gaussian_matrix(5, 1, 1), gaussian_matrix(5, 1, 2))


def test_exact_svd_matches_full_svd():
    # test-svd-public-tools.R:42-61 (fastsvd on 40 x 5 equals base::svd, 1e-8)
    rng = np.random.default_rng(4)
    A = rng.standard_normal((40, 5))
    r = osvd.truncated_svd(A, 5, osvd.SVD_METHOD_CPU_RSVD)
    U, s, Vt = np.linalg.svd(A, full_matrices=False)
    assert np.allclose(r.s, s, atol=1e-8)
    assert np.allclose(np.abs(r.U), np.abs(U), atol=1e-6)
    assert np.allclose(np.abs(r.Vt), np.abs(Vt), atol=1e-6)


def test_rsvd_recovers_exact_rank_k():
    rng = np.random.default_rng(9)
    U = np.linalg.qr(rng.standard_normal((300, 8)))[0]
    V = np.linalg.qr(rng.standard_normal((120, 8)))[0]
    s = np.array([9, 7, 5, 3, 2, 1.5, 1.0, 0.5])
    A = (U * s) @ V.T
    for power in (0, 1, 2):
        r = osvd.truncated_svd_cpu_rsvd(A, 8, oversample=5, power_iters=power, seed=3)
        assert np.allclose(r.s, s, rtol=1e-10)
        assert np.linalg.norm((r.U * r.s) @ r.Vt - A) < 1e-10 * np.linalg.norm(A)


def test_rsvd_singular_values_close_to_exact():
    # test-svd-rsvd.R:1-33 (rsvd vs exact singular values, tol 1e-2)
    rng = np.random.default_rng(1)
    A = rng.standard_normal((200, 60)) @ np.diag(0.9 ** np.arange(60)) @ rng.standard_normal((60, 60))
    r = osvd.truncated_svd_cpu_rsvd(A, 5, oversample=10, power_iters=2, seed=1)
    e = osvd.truncated_svd_cpu_exact(A, 5)
    assert np.allclose(r.s, e.s, rtol=1e-2)


def test_predict_identity_b_route_equals_latent_route():
    # test-predict-optimized.R:26-56 (pls_predict == (X - mX)/vX B + mY, 1e-12)
    d = synthetic.c1_simpls_regression(seed=2, n=220, p=24, m=2, rank=5)
    model = opls.pls_model2_fast(d["Xtrain"], d["Ytrain"], [1, 3, 5], fit=True, seed=123)
    a = opls.pls_predict(model, d["Xtest"], use_B=True)["Ypred"]
    b = opls.pls_predict(model, d["Xtest"], use_B=False)["Ypred"]
    legacy = np.stack([((d["Xtest"] - model["mX"]) / model["vX"]) @ model["B"][:, :, s] + model["mY"]
                       for s in range(3)], axis=2)
    assert np.allclose(a, legacy, atol=1e-12)
    assert np.allclose(b, legacy, atol=1e-12)


def test_plssvd_optimized_equals_legacy():
    # test-plssvd-optimized.R:40-73: C = G^-1 D  vs  G^-1 T^T Y V  (B and Yfit, 1e-8)
    d = synthetic.c1_simpls_regression(seed=4, n=300, p=80, m=6, rank=10)
    X, Y = d["Xtrain"], d["Ytrain"]
    model = opls.pls_model1(X, Y, [1, 3, 5], fit=True, svd_method=4, rsvd_power=1, seed=1)
    Xc = X - model["mX"]
    Yc = Y - model["mY"]
    for a, mc in enumerate([1, 3, 5]):
        U = model["R"][:, :mc]
        V = model["Q"][:, :mc]
        T = Xc @ U
        C = np.linalg.solve(T.T @ T, T.T @ (Yc @ V))
        B_legacy = U @ C @ V.T
        assert np.allclose(model["B"][:, :, a], B_legacy, atol=1e-8)


def test_onehot_class_sums_match_dense_product():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((500, 30))
    y = rng.integers(1, 8, size=500)
    Y = opls.transformy(y)
    sums = np.zeros((30, Y.shape[1]))
    for c in range(Y.shape[1]):
        sums[:, c] = X[y == c + 1].sum(axis=0)
    assert np.allclose(X.T @ Y, sums, atol=1e-12)


def test_lda_projected_equals_explicit():
    # test-lda-cuda-native.R:1-32: projected LDA == explicit C++ LDA (1e-12, same labels)
    rng = np.random.default_rng(8)
    X = rng.standard_normal((400, 20))
    y = rng.integers(1, 5, size=400)
    R = rng.standard_normal((20, 6))
    off = rng.standard_normal(6)
    a = olda.lda_project_train_prefix(X, R, off, y, 4, [2, 6])
    b = olda.lda_train_prefix(X @ R - off, y, 4, [2, 6])
    for k in ("2", "6"):
        assert np.allclose(a[k]["linear"], b[k]["linear"], atol=1e-12)
        lab1 = olda.lda_project_predict(X, R[:, :int(k)], off[:int(k)], a[k])
        lab2 = olda.lda_predict_labels((X @ R - off)[:, :int(k)], b[k])
        assert np.array_equal(lab1, lab2)


def test_simpls_fast_same_seed_same_result():
    # test-pls-rsvd.R:100-140: same seed => identical B; different seed => different
    d = synthetic.c1_simpls_regression(seed=5, n=120, p=40, m=3, rank=6)
    a = opls.pls_model2_fast(d["Xtrain"], d["Ytrain"], [4], seed=7)
    b = opls.pls_model2_fast(d["Xtrain"], d["Ytrain"], [4], seed=7)
    c = opls.pls_model2_fast(d["Xtrain"], d["Ytrain"], [4], seed=8)
    assert np.array_equal(a["B"], b["B"])
    assert not np.array_equal(a["B"], c["B"])


def test_simpls_refresh_sign_convention():
    # Householder QR of one column gives Q[0] <= 0, and gesvd of 1 x m keeps U = 1.
    d = synthetic.c1_simpls_regression(seed=6, n=100, p=50, m=4, rank=5)
    m = opls.pls_model2_fast(d["Xtrain"], d["Ytrain"], [5], seed=1)
    assert np.all(m["R"][0, :] <= 0)


def test_oracle_golden_fixtures():
    # The committed fixtures (tests/golden/make_golden.py) hold inputs and the
    # oracle's outputs; the oracle run again on those inputs must give them back.
    import glob
    import os
    from golden.make_golden import CASES, inputs_of
    from parity_utils import cv_labels_match, rel_err
    here = os.path.dirname(os.path.abspath(__file__))
    files = sorted(glob.glob(os.path.join(here, "golden", "*.npz")))
    assert {os.path.basename(f)[:-4] for f in files} == set(CASES), "golden fixtures missing"
    for f in files:
        name = os.path.basename(f)[:-4]
        want = dict(np.load(f))
        got = CASES[name][1](inputs_of(want))
        assert set(got) == {k for k in want if not k.startswith("in_")}, name
        for k, v in got.items():
            w = want[k]
            assert np.shape(v) == w.shape, (name, k)
            if w.dtype.kind == "f":
                assert rel_err(v, w) <= 1e-10, (name, k, rel_err(v, w))
            elif k in ("pred", "inner_pred"):
                sc = want["outer_score" if k == "pred" else "inner_score"]
                assert cv_labels_match(v, w, sc, 1e-9)[0], (name, k)
            else:
                assert np.array_equal(v, w), (name, k)


def test_gaussian_y_identities():
    # tests/testthat/test-gaussian-y.R: decoded predictions keep Y's shape and are
    # finite; the decoder solves the ridge normal equations of R/main.R:1968-1981.
    from oracle import gaussian_y as og
    rng = np.random.default_rng(120)
    Y = rng.standard_normal((70, 24))
    G = rng.standard_normal((24, 7)) / np.sqrt(7)
    enc = og.prepare_regression(Y, G)
    Z, D = enc["Z"], enc["decoder"]
    assert Z.shape == (70, 7) and D.shape == (7, 24)
    ztz = Z.T @ Z
    lhs = (ztz + 1e-8 * np.mean(np.diag(ztz)) * np.eye(7)) @ D
    assert np.allclose(lhs, Z.T @ (Y - Y.mean(axis=0)), rtol=1e-10, atol=1e-10)
    out = og.decode_regression(Z[:9], D, enc["y_center"])
    assert out.shape == (9, 24) and np.all(np.isfinite(out))
    # class codes: centred columns, unit rows; a code decodes to its own class
    codes = og.class_codes(rng.standard_normal((6, 5)) / np.sqrt(5))
    assert np.allclose(np.linalg.norm(codes, axis=1), 1.0)
    assert np.array_equal(og.nearest_code_classes(codes, codes), np.arange(1, 7))


def test_opls_filter_identities():
    # Each removed orthogonal score is orthogonal to the filtered X, weights are
    # unit vectors, and applying the stored filter to the training rows
    # reproduces the filtered training matrix (src/fastPLS.cpp:4377-4483).
    from oracle import opls as oo
    rng = np.random.default_rng(7)
    X = rng.standard_normal((60, 20)) + rng.standard_normal((60, 1)) * rng.standard_normal(20)
    Y = X[:, :3] @ rng.standard_normal((3, 2)) + 0.1 * rng.standard_normal((60, 2))
    for scaling in (1, 2, 3):
        f = oo.opls_filter(X, Y, 3, scaling=scaling)
        assert f["north"] == 3
        assert np.allclose(np.linalg.norm(f["W_orth"], axis=0), 1.0)
        again = oo.opls_apply_filter(X, f["mX"], f["vX"], f["W_orth"], f["P_orth"])
        assert np.allclose(again, f["X"], atol=1e-10)
    f0 = oo.opls_filter(X, Y, 0)
    assert f0["north"] == 0 and f0["W_orth"].shape == (20, 0)


def test_cknn_known_answer():
    # Two classes in 2-D, worked by hand from src/fastPLS.cpp:1287-1467.
    import math
    from oracle import cknn
    Tr = np.array([[1.0, 0.0], [0.8, 0.6], [0.0, 1.0]])
    y = np.array([1, 1, 2], dtype=np.int32)
    cents = cknn.centroids(Tr, y, 2)
    assert np.allclose(cents[0], np.array([0.9, 0.3]) / math.hypot(0.9, 0.3))
    Tt = np.array([[1.0, 0.0]])
    out = cknn.candidate_knn_predict(Tt, Tr, y, cents, top_k=2, top_m=2, knn_k=2, tau=0.2,
                                     alpha=0.75)
    base1 = cents[0] @ Tt[0]
    local1 = 1.0 + 0.2 * math.log((1.0 + math.exp((0.8 - 1.0) / 0.2)) / 2.0)
    assert out["top_index"].tolist() == [[1, 2]]
    assert np.allclose(out["top_score"], [[local1 + 0.75 * base1, 0.0]], atol=1e-15)
    # tau <= 0 falls back to 0.2; top is clamped to the class count (test-class-bias-top5.R:70-72)
    again = cknn.candidate_knn_predict(Tt, Tr, y, cents, top_k=5, top_m=9, knn_k=2, tau=-1.0,
                                       alpha=0.75)
    assert again["top_index"].shape == (1, 2)
    assert np.array_equal(again["top_score"], out["top_score"])


def test_cknn_insertion_ties_keep_first():
    from oracle import cknn
    s, ix = [-np.inf] * 3, [-1] * 3
    for c, v in enumerate([0.5, 0.7, 0.5, 0.7]):
        cknn.insert_top(s, ix, v, c + 1)
    assert ix == [2, 4, 1] and s == [0.7, 0.7, 0.5]


def test_xprod_oracle_equals_materialized():
    # The implicit operator applies the same A = XᵀY (and P_V A after deflation) as the
    # materialized paths, so the models agree to rounding (fastPLS.cpp:550-622, 936-1000).
    from oracle import xprod as ox
    d = synthetic.c1_simpls_regression(seed=3, n=300, p=120, m=60, rank=8)
    X, Y = d["Xtrain"], d["Ytrain"]
    a = ox.pls_model1_xprod(X, Y, [3, 6], rsvd_oversample=5, rsvd_power=2, seed=4)
    b = opls.pls_model1(X, Y, [3, 6], svd_method=4, rsvd_oversample=5, rsvd_power=2, seed=4)
    assert np.allclose(a["B"], b["B"], rtol=1e-10, atol=1e-12)
    c = ox.pls_model2_fast_xprod(X, Y, [2, 5, 9], seed=3)
    e = opls.pls_model2_fast(X, Y, [2, 5, 9], seed=3)
    assert np.linalg.norm(c["B"] - e["B"]) < 1e-10 * np.linalg.norm(e["B"])


def test_kernel_oracle_properties():
    # centring a linear kernel equals the Gram of the column-centred rows; an
    # RBF kernel has a unit diagonal and is symmetric; centred test kernels of
    # the training rows reproduce the centred training kernel
    from oracle import kernel as ok
    rng = np.random.default_rng(5)
    X = rng.standard_normal((40, 7))
    Xc = X - X.mean(axis=0)
    kc = ok.center_kernel_train(ok.kernel_matrix(X, X, 1, 1.0, 1, 0.0))
    assert np.allclose(kc["K"], Xc @ Xc.T, atol=1e-12)
    K = ok.kernel_matrix(X, X, 2, 0.2, 3, 1.0)
    assert np.allclose(np.diag(K), 1.0) and np.allclose(K, K.T)
    kc = ok.center_kernel_train(K)
    assert np.allclose(ok.center_kernel_test(K, kc["col_means"], kc["grand_mean"]), kc["K"], atol=1e-12)

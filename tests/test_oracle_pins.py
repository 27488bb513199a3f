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
    import glob
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    files = sorted(glob.glob(os.path.join(here, "golden", "*.npz")))
    if not files:
        pytest.skip("no golden fixtures committed")
    from golden.make_golden import CASES
    for f in files:
        name = os.path.basename(f)[:-4]
        want = dict(np.load(f))
        got = CASES[name]()
        for k, v in want.items():
            if k.startswith("in_"):
                continue
            assert np.allclose(got[k], v, rtol=1e-10, atol=1e-12), (name, k)

"""GPU parity of label-aware PLSSVD and of the whole-GPU exact SVD."""
import numpy as np
import pytest

from oracle import label_aware as ola
from parity_utils import rel_err, subspace_angle

pytestmark = pytest.mark.gpu


def _orth(rng, n, k):
    q, _ = np.linalg.qr(rng.standard_normal((n, k)))
    return q


@pytest.mark.parametrize("rows,cols", [(300, 500), (640, 200)])
def test_exact_svd_whole_gpu(lib, rows, cols):
    rng = np.random.default_rng(rows)
    r = min(rows, cols)
    s = np.linspace(10.0, 1.0, r)
    A = _orth(rng, rows, r) @ np.diag(s) @ _orth(rng, cols, r).T
    got = lib.truncated_svd(A, r, svd_method=3)
    assert rel_err(got["d"], s) < 1e-12
    U, V = got["u"], got["vt"].T
    sign = np.sign(np.sum(U * (A @ V), axis=0))
    assert np.all(sign > 0)
    assert rel_err(U * got["d"] @ V.T, A) < 1e-12
    assert np.max(np.abs(U.T @ U - np.eye(r))) < 1e-12
    assert np.max(np.abs(V.T @ V - np.eye(r))) < 1e-12


def test_exact_svd_rank_deficient_completion(lib):
    rng = np.random.default_rng(8)
    A = rng.standard_normal((150, 40)) @ rng.standard_normal((40, 120))
    got = lib.truncated_svd(A, 120, svd_method=3)
    U = got["u"]
    assert np.max(np.abs(U.T @ U - np.eye(120))) < 1e-10
    assert rel_err(got["d"][:40], np.linalg.svd(A, compute_uv=False)[:40]) < 1e-12
    assert np.all(got["d"][40:] < 1e-10 * got["d"][0])


def _zipf_data(seed, n, p, m, noise=0.3):
    rng = np.random.default_rng(seed)
    pr = 1.0 / np.arange(1, m + 1) ** 1.1
    pr /= pr.sum()
    y = rng.choice(m, size=n, p=pr) + 1
    y[:m] = np.arange(1, m + 1)  # every class present
    protos = rng.standard_normal((m, p))
    protos /= np.linalg.norm(protos, axis=1, keepdims=True)
    X = protos[y - 1] + noise * rng.standard_normal((n, p))
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    return X, y.astype(np.int32)


def _compare(got, ref, Xtest):
    K = got["max_rank"]
    assert np.array_equal(got["ncomp"], ref["ncomp"])
    assert rel_err(got["mX"], ref["mX"]) < 1e-12
    assert rel_err(got["vX"], ref["vX"]) < 1e-12
    assert rel_err(got["mY"], ref["mY"]) < 1e-15
    assert rel_err(got["s"], ref["d"]) < 1e-10
    sg = np.sign(np.sum(got["R"] * ref["R"], axis=0))
    assert rel_err(got["R"] * sg, ref["R"]) < 1e-9
    assert rel_err(got["Q"] * sg, ref["Q"]) < 1e-9
    D = np.diag(sg)
    for a in range(len(ref["ncomp"])):
        assert rel_err(D @ got["C_latent"][:, :, a] @ D, ref["C_latent"][:, :, a]) < 1e-9
        # predictions are sign-invariant
        Xc = (Xtest - ref["mX"]) / ref["vX"]
        pg = Xc @ got["R"] @ got["W_latent"][:, :, a]
        pr = Xc @ ref["R"] @ ref["W_latent"][:, :, a]
        assert rel_err(pg, pr) < 1e-9
    assert K == ref["R"].shape[1]


@pytest.mark.parametrize("scaling", [1, 2])
def test_label_aware_small_matches_oracle(lib, scaling):
    # S 1 = 0, so rank(S) <= m - 1 = 11: a 12th component is a null direction
    # whose singular vectors no two SVD routines choose alike.
    X, y = _zipf_data(3, 3000, 60, 12)
    got = lib.plssvd_label_aware(X, y, 12, [3, 8, 11], scaling=scaling)
    ref = ola.label_aware_plssvd(X, y, 12, [3, 8, 11], scaling=scaling)
    _compare(got, ref, X[:200])


def test_label_aware_whole_gpu_svd_fp32_input(lib):
    # min(p, m) = 120 > 96: the exact SVD runs as the cooperative Jacobi
    X, y = _zipf_data(4, 6000, 160, 120)
    X32 = X.astype(np.float32)
    got = lib.plssvd_label_aware(X32, y, 120, [10, 40], scaling=1)
    ref = ola.label_aware_plssvd(X32.astype(np.float64), y, 120, [10, 40], scaling=1)
    _compare(got, ref, X[:300])


def test_label_aware_rsvd_matches_oracle(lib):
    X, y = _zipf_data(5, 5000, 96, 80)
    got = lib.plssvd_label_aware(X, y, 80, [5, 20], svd_method=4, oversample=10, power_iters=1,
                                 seed=7)
    ref = ola.label_aware_plssvd(X, y, 80, [5, 20], svd_method=4, oversample=10, power_iters=1,
                                 seed=7)
    _compare(got, ref, X[:200])


def test_label_aware_scores_and_errors(lib):
    X, y = _zipf_data(6, 800, 30, 5)
    got = lib.plssvd_label_aware(X, y, 5, [2, 9], keep_scores=True)
    assert list(got["ncomp"]) == [2, 5]  # capped at min(n, p, m)
    Xc = X - X.mean(axis=0)
    assert rel_err(got["Ttrain"], Xc @ got["R"]) < 1e-12
    bad = y.copy()
    bad[0] = 6
    with pytest.raises(lib.FastPLSError):
        lib.plssvd_label_aware(X, bad, 5, [2])


def _oracle_pipeline(X, y, m, Xtest, ncomp, svd_method, knn_k, tau, alpha, top_m, top_k, **kw):
    from oracle import cknn as ok
    fit = ola.label_aware_plssvd(X, y, m, [ncomp], svd_method=svd_method, **kw)
    C = fit["C_latent"][:, :, 0]
    T = ((X - fit["mX"]) / fit["vX"]) @ fit["R"]
    Tn = ok.row_l2(T @ C)
    cents = ok.centroids(Tn, y, m)
    Tt = ok.row_l2((((Xtest - fit["mX"]) / fit["vX"]) @ fit["R"]) @ C)
    return ok.candidate_knn_predict(Tt, Tn, y, cents, top_k=top_k, top_m=top_m, knn_k=knn_k,
                                    tau=tau, alpha=alpha)


@pytest.mark.parametrize("svd_method", [3, 4])
def test_label_aware_cknn_pipeline(lib, svd_method):
    X, y = _zipf_data(9, 7000, 48, 40)
    Xte, _ = _zipf_data(10, 150, 48, 40)
    kw = dict(knn_k=10, tau=0.2, alpha=0.75, top_m=20, top_k=5)
    got = lib.label_aware_cknn(X, y, 40, Xte, 24, svd_method=svd_method, oversample=10,
                               power_iters=1, seed=3, **kw)
    extra = {} if svd_method == 3 else dict(oversample=10, power_iters=1, seed=3)
    ref = _oracle_pipeline(X, y, 40, Xte, 24, svd_method, **kw, **extra)
    assert np.array_equal(got["top_index"], ref["top_index"])
    assert np.max(np.abs(got["top_score"] - ref["top_score"])) < 1e-9


def test_label_aware_cknn_resident_matches_host(lib):
    X, y = _zipf_data(11, 5000, 64, 30)
    Xte, _ = _zipf_data(12, 100, 64, 30)
    X32, Xte32 = X.astype(np.float32), Xte.astype(np.float32)
    host = lib.label_aware_cknn(X32, y, 30, Xte32, 16, svd_method=4, seed=2)
    htr, hte = lib.x_upload(X32), lib.x_upload(Xte32)
    try:
        res = lib.label_aware_cknn_resident(htr, y, 30, hte, Xte32.shape[0], 16, svd_method=4, seed=2)
    finally:
        lib.x_free(htr)
        lib.x_free(hte)
    assert np.array_equal(host["top_index"], res["top_index"])
    assert np.max(np.abs(host["top_score"] - res["top_score"])) < 1e-12

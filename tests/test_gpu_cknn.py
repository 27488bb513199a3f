"""GPU parity of the candidate-kNN classifier (score space, centroids, predict)."""
import numpy as np
import pytest

from oracle import cknn as ok
from parity_utils import rel_err

pytestmark = pytest.mark.gpu


def _zipf_case(seed, n_train, n_test, n_classes, kdim, empty=()):
    rng = np.random.default_rng(seed)
    p = 1.0 / np.arange(1, n_classes + 1) ** 1.1
    p /= p.sum()
    protos = ok.row_l2(rng.standard_normal((n_classes, kdim)))
    y = rng.choice(n_classes, size=n_train, p=p) + 1
    for e in empty:
        y[y == e] = 1
    Tr = ok.row_l2(protos[y - 1] + 0.3 * rng.standard_normal((n_train, kdim)))
    yt = rng.choice(n_classes, size=n_test, p=p) + 1
    Tt = ok.row_l2(protos[yt - 1] + 0.3 * rng.standard_normal((n_test, kdim)))
    return Tr, y.astype(np.int32), Tt


def _check(got, ref):
    assert got["top_index"].shape == ref["top_index"].shape
    assert np.array_equal(got["top_index"], ref["top_index"])
    fin = np.isfinite(ref["top_score"])
    assert np.array_equal(np.isfinite(got["top_score"]), fin)
    assert np.max(np.abs(got["top_score"][fin] - ref["top_score"][fin])) < 1e-12


def test_scores_and_centroids(lib):
    rng = np.random.default_rng(5)
    T = rng.standard_normal((700, 12))
    T[3] = 0.0
    Ck = rng.standard_normal((12, 12))
    assert rel_err(lib.candidate_scores(T, Ck), ok.row_l2(T @ Ck)) < 1e-13
    Tn = lib.candidate_scores(T)
    assert rel_err(Tn, ok.row_l2(T)) < 1e-14
    y = rng.integers(1, 9, size=700).astype(np.int32)
    y[y == 4] = 2  # class 4 empty -> zero centroid
    got = lib.candidate_centroids(Tn, y, 8)
    ref = ok.centroids(Tn, y, 8)
    assert np.max(np.abs(got - ref)) < 1e-14
    assert np.all(got[3] == 0.0)


@pytest.mark.parametrize("knn_k,tau,top_k,top_m", [(10, 0.2, 5, 20), (3, 0.2, 1, 4), (40, -1.0, 3, 30)])
def test_candidate_knn_matches_oracle(lib, knn_k, tau, top_k, top_m):
    # 40 Zipf classes; the largest spans several 2048-row chunks.
    Tr, y, Tt = _zipf_case(11, 12000, 300, 40, 24, empty=(17,))
    cents = ok.centroids(Tr, y, 40)
    got = lib.candidate_knn_predict(Tt, Tr, y, cents, top_k=top_k, top_m=top_m, knn_k=knn_k,
                                    tau=tau, alpha=0.75)
    ref = ok.candidate_knn_predict(Tt, Tr, y, cents, top_k=top_k, top_m=top_m, knn_k=knn_k,
                                   tau=tau, alpha=0.75, knn_cap=32)
    _check(got, ref)


def test_candidate_knn_bias_small_classes_and_clamps(lib):
    # classes smaller than knn_k, a bias vector, top_k above the class count
    Tr, y, Tt = _zipf_case(12, 90, 20, 4, 9)
    cents = ok.centroids(Tr, y, 4)
    bias = np.array([0.0, 0.05, -0.02, 0.1])
    got = lib.candidate_knn_predict(Tt, Tr, y, cents, bias=bias, top_k=7, top_m=2, knn_k=10,
                                    tau=0.2, alpha=0.75)
    ref = ok.candidate_knn_predict(Tt, Tr, y, cents, bias=bias, top_k=7, top_m=2, knn_k=10,
                                   tau=0.2, alpha=0.75)
    assert got["top_index"].shape == (20, 4)
    _check(got, ref)


@pytest.mark.parametrize("kdim", [100, 150])
def test_candidate_knn_wide_scores(lib, kdim):
    # kdim > 16 * several K-blocks and a test count that is not a tile multiple;
    # 150 is past the staged kernels' 116-wide rows (the k-step kernel runs)
    Tr, y, Tt = _zipf_case(13, 5000, 131, 25, kdim)
    cents = ok.centroids(Tr, y, 25)
    got = lib.candidate_knn_predict(Tt, Tr, y, cents, top_k=5, top_m=10, knn_k=10, tau=0.2,
                                    alpha=0.75)
    ref = ok.candidate_knn_predict(Tt, Tr, y, cents, top_k=5, top_m=10, knn_k=10, tau=0.2,
                                   alpha=0.75)
    _check(got, ref)


@pytest.mark.parametrize("buffers", ["1", "2", "3", "4"])
@pytest.mark.parametrize("kdim", [9, 24, 100, 128])
def test_candidate_knn_staged_tiles_match_oracle(lib, monkeypatch, kdim, buffers):
    # every similarity-tile kernel (FASTPLS_CKNN_TILES=1: 16-wide k-steps;
    # 2: contraction staged, two training-row buffers; 3: one buffer, two
    # CTAs per SM; 4, the default: BF16 tensor-core filter with exact FP64
    # rescoring) gives the oracle's neighbours, for odd, small and wide score
    # spaces (128 is the filter's widest; the staged kernels hand it to the
    # k-step kernel)
    monkeypatch.setenv("FASTPLS_CKNN_TILES", buffers)
    Tr, y, Tt = _zipf_case(14 + kdim, 6000, 150, 30, kdim)
    cents = ok.centroids(Tr, y, 30)
    got = lib.candidate_knn_predict(Tt, Tr, y, cents, top_k=5, top_m=12, knn_k=10, tau=0.2, alpha=0.75)
    ref = ok.candidate_knn_predict(Tt, Tr, y, cents, top_k=5, top_m=12, knn_k=10, tau=0.2, alpha=0.75)
    _check(got, ref)


@pytest.mark.parametrize("copies", [8, 40])
def test_candidate_knn_filter_near_ties(lib, monkeypatch, copies):
    # training rows that are copies of one another up to 1e-7: many
    # approximate similarities fall inside the filter's error bar around a
    # pair's k-th neighbour, so the exact rescoring decides the list (8
    # copies); with 40 copies a pair has more such rows than its candidate
    # slots and the call falls back to the FP64 tiles
    monkeypatch.setenv("FASTPLS_CKNN_TILES", "4")
    rng = np.random.default_rng(21)
    base, y, Tt = _zipf_case(22, 400, 90, 6, 32)
    Tr = ok.row_l2(np.repeat(base, copies, axis=0) + 1e-7 * rng.standard_normal((400 * copies, 32)))
    y = np.repeat(y, copies).astype(np.int32)
    cents = ok.centroids(Tr, y, 6)
    got = lib.candidate_knn_predict(Tt, Tr, y, cents, top_k=3, top_m=4, knn_k=12, tau=0.2, alpha=0.75)
    ref = ok.candidate_knn_predict(Tt, Tr, y, cents, top_k=3, top_m=4, knn_k=12, tau=0.2, alpha=0.75)
    _check(got, ref)

"""The CUDA path against the committed golden fixtures (tests/golden/*.npz).

Each fixture holds a case's inputs and the CPU oracle's outputs on them (made
by tests/golden/make_golden.py); here the library, through its C ABI, runs the
same inputs and must reproduce those outputs within the FP64 drop-in
tolerances: coefficients, predictions and scores to relative 1e-9, subspace
quantities sign-aligned to 1e-8, labels identical wherever the oracle's
decision margin exceeds 1e-8 of the score scale, kNN indices equal.
"""
import os

import numpy as np
import pytest

from golden.make_golden import C1_NCOMP, C2_NCOMP, C5_NCOMP, inputs_of
from parity_utils import REL_TOL, cv_labels_match, labels_match_beyond_margin, rel_err, sign_align

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
MARGIN = 1e-8


def _fixture(name):
    fx = dict(np.load(os.path.join(HERE, "golden", name + ".npz")))
    return inputs_of(fx), fx


def test_golden_c1_simpls_regression(lib):
    x, want = _fixture("c1_simpls_regression")
    X, Y = x["X"], x["Y"]
    Xtr, Ytr, Xte = np.asfortranarray(X[:400]), np.asfortranarray(Y[:400]), np.asfortranarray(X[400:])
    fast = lib.pls_model2_fast(Xtr, Ytr, C1_NCOMP, fit=True, seed=1)
    assert rel_err(fast["B"], want["fast_B"]) < REL_TOL
    # the refresh vectors keep the reference's sign convention: compared as they are
    assert np.allclose(fast["R"], want["fast_R"], rtol=1e-8, atol=1e-12)
    assert rel_err(fast["Yfit"], want["fast_Yfit"]) < REL_TOL
    assert np.allclose(fast["R2Y"], want["fast_R2Y"], rtol=1e-9, atol=1e-12)
    assert rel_err(lib.predict_lowrank(fast, Xte)["Ypred"], want["fast_Ypred"]) < REL_TOL
    classic = lib.pls_model2(Xtr, Ytr, C1_NCOMP, svd_method=3, seed=1)
    assert rel_err(classic["B"], want["classic_B"]) < REL_TOL
    assert rel_err(lib.predict_lowrank(classic, Xte)["Ypred"], want["classic_Ypred"]) < REL_TOL
    svd = lib.pls_model1(Xtr, Ytr, C1_NCOMP, svd_method=4, seed=1)
    assert rel_err(svd["B"], want["plssvd_B"]) < REL_TOL
    assert rel_err(lib.predict_lowrank(svd, Xte)["Ypred"], want["plssvd_Ypred"]) < REL_TOL


def test_golden_c2_plssvd_lda(lib):
    from oracle import pls as opls
    x, want = _fixture("c2_plssvd_lda")
    m = int(x["n_classes"])
    X = x["Xtrain"].astype(np.float64)
    Xt = x["Xtest"].astype(np.float64)
    model = lib.pls_model1(X, opls.transformy(x["ytrain"]), C2_NCOMP, svd_method=4, oversample=10,
                           power_iters=2, seed=1)
    assert rel_err(lib.predict_lowrank(model, Xt)["Ypred"], want["Ypred"]) < REL_TOL
    Rp = model["R"] / model["vX"].T
    off = (model["mX"] @ Rp).ravel()
    lda = lib.lda_project_train_prefix(X, Rp, off, x["ytrain"], m, C2_NCOMP, ridge=1e-8)
    for kk in C2_NCOMP:
        g = lib.lda_project_predict(Xt, Rp[:, :kk], off[:kk], lda[str(kk)], return_scores=True)
        # each component of the rSVD is defined up to sign, and so is its LDA column
        lin = sign_align(lda[str(kk)]["linear"], want[f"lda{kk}_linear"])
        assert rel_err(lin, want[f"lda{kk}_linear"]) < REL_TOL
        assert rel_err(lda[str(kk)]["constants"], want[f"lda{kk}_constants"]) < REL_TOL
        assert rel_err(g["scores"], want[f"lda{kk}_scores"]) < REL_TOL
        ok, nclear = labels_match_beyond_margin(g["pred"], want[f"lda{kk}_pred"], want[f"lda{kk}_scores"],
                                                MARGIN)
        assert ok and nclear > 0.9 * Xt.shape[0]


def test_golden_c3_label_aware_cknn(lib):
    x, want = _fixture("c3_label_aware_cknn")
    got = lib.label_aware_cknn(x["Xtrain"], x["ytrain"], int(x["n_classes"]), x["Xtest"], 16, svd_method=3,
                               knn_k=10, tau=0.2, alpha=0.75, top_m=20, top_k=5)
    assert np.array_equal(got["top_index"], want["top_index"])
    assert np.max(np.abs(got["top_score"] - want["top_score"])) < 1e-9


@pytest.mark.parametrize("batched", [True, False])
def test_golden_c4_double_cv(lib, batched):
    x, want = _fixture("c4_double_cv")
    got = lib.double_cv(x["X"], x["y"], x["outer"], x["inner"], np.arange(1, 7), int(x["n_classes"]), seed=1,
                        batched=batched, return_scores=True)
    assert np.array_equal(got["best_comp"], want["best_comp"])
    assert np.allclose(got["inner_accuracy"], want["inner_accuracy"], rtol=0, atol=1e-12)
    gi = np.transpose(got["inner_pred"], (2, 1, 0))
    assert cv_labels_match(gi, want["inner_pred"], want["inner_score"], MARGIN)[0]
    assert cv_labels_match(got["pred"], want["pred"], want["outer_score"], MARGIN)[0]
    assert rel_err(got["inner_score"], want["inner_score"]) < REL_TOL
    assert rel_err(got["outer_score"], want["outer_score"]) < REL_TOL


def test_golden_c5_opls_gaussian_y(lib):
    x, want = _fixture("c5_opls_gaussian_y")
    X = x["Xtrain"].astype(np.float64)
    Y = x["Ytrain"].astype(np.float64)
    Xt = x["Xtest"].astype(np.float64)
    filt = lib.opls_filter(X, Y, 2)
    for a in range(2):
        s = np.sign(filt["W_orth"][:, a] @ want["W_orth"][:, a])
        assert rel_err(s * filt["W_orth"][:, a], want["W_orth"][:, a]) < 1e-8
        assert rel_err(s * filt["P_orth"][:, a], want["P_orth"][:, a]) < 1e-8
    enc = lib.gaussian_y_encode(Y, x["G"])
    assert rel_err(enc["decoder"], want["decoder"]) < REL_TOL
    model = lib.pls_model2_fast(filt["X"], enc["Z"], C5_NCOMP, seed=1)
    Xtf = lib.opls_apply_filter(Xt, filt["mX"], filt["vX"], filt["W_orth"], filt["P_orth"])
    Zp = lib.predict_lowrank(model, Xtf)["Ypred"]
    assert rel_err(Zp, want["Zpred"]) < 1e-8
    Yp = np.stack([lib.gaussian_y_decode(Zp[:, :, a], enc["decoder"], enc["y_center"])
                   for a in range(Zp.shape[2])], axis=2)
    assert rel_err(Yp, want["Ypred"]) < 1e-8

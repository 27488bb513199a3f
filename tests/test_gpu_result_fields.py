"""The model lists an R shim builds from the ABI outputs: field names and
shapes of pls_model1 (fastPLS.cpp:4966-4984), pls_model2_fast
(fastPLS.cpp:2759-2777) and pls_lda_gpu_native (fastPLS.cpp:6275-6437), as
the Python mirror returns them."""
import numpy as np
import pytest

from oracle import pls as opls
from fastpls_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def d():
    return synthetic.c1_simpls_regression(seed=3, n=300, p=400, m=4, rank=8)


def _shapes(model, spec):
    for k, shape in spec.items():
        assert k in model, k
        assert np.shape(model[k]) == shape, (k, np.shape(model[k]), shape)


def test_pls_model1_fields(lib, d):
    X, Y = d["Xtrain"], d["Ytrain"]
    n, p = X.shape
    m = Y.shape[1]
    nc = [2, 4]
    L, K = len(nc), 4
    mod = lib.pls_model1(X, Y, nc, fit=True, svd_method=4, seed=1)
    _shapes(mod, dict(C_latent=(K, K, L), W_latent=(K, m, L), Q=(m, K), Ttrain=(n, K), R=(p, K), mX=(1, p),
                      vX=(1, p), mY=(1, m), ncomp=(L,), Yfit=(n, m, L), R2Y=(L,), B=(p, m, L)))
    assert mod["p"] == p and mod["m"] == m and mod["B_stored"] and not mod["compact_prediction"]
    assert list(mod["ncomp"]) == nc
    lean = lib.pls_model1(X, Y, nc, svd_method=4, seed=1, store_B=False)
    assert "B" not in lean and lean["compact_prediction"]


def test_pls_model2_fast_fields(lib, d):
    X, Y = d["Xtrain"], d["Ytrain"]
    n, p = X.shape
    m = Y.shape[1]
    nc = [3, 6, 1]
    L, K = len(nc), 6
    mod = lib.pls_model2_fast(X, Y, nc, fit=True, seed=1)
    _shapes(mod, dict(Q=(m, K), R=(p, K), mX=(1, p), vX=(1, p), mY=(1, m), ncomp=(L,), Yfit=(n, m, L),
                      R2Y=(L,), B=(p, m, L)))
    assert mod["p"] == p and mod["m"] == m and mod["n_components"] == K
    assert mod["pls_method"] == "simpls" and mod["B_stored"]


def test_pls_lda_fields(lib):
    c = synthetic.c2_plsda(seed=8, n=600, n_test=50, p=120, n_classes=12)
    Y = opls.transformy(c["ytrain"])
    n, p = c["Xtrain"].shape
    nc = [4, 2, 4]
    mod = lib.pls_lda(c["Xtrain"], Y, c["ytrain"], c["Xtest"], nc, 12, method=1, fit=True)
    K, L, U, C = 4, 3, 2, 12
    _shapes(mod, dict(R=(p, K), Q=(12, K), mX=(1, p), vX=(1, p), mY=(1, 12), ncomp=(L,), B=(p, 12, L),
                      Yfit=(n, 12, L), R2Y=(L,), unique_ncomp=(U,), lda_means=(C, K, U), lda_linear=(C, K, U),
                      lda_constants=(C, U), lda_priors=(C,), lda_lambda=(U,), R_predict=(p, K), R_offset=(K,),
                      pred_codes=(50, L)))
    assert list(mod["unique_ncomp"]) == [2, 4]
    assert np.all((mod["pred_codes"] >= 1) & (mod["pred_codes"] <= C))

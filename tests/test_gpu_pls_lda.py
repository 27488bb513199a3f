"""The fused PLS + LDA entry (fpls_pls_lda, for _fastPLS_pls_lda_gpu_native)
against the oracle's composition of the same steps (oracle/pls_lda.py):
PLSSVD or fast SIMPLS fit, one LDA per distinct ncomp on the training scores,
test labels per ncomp slice.  FP64 tolerances; labels identical wherever the
oracle's LDA decision margin exceeds 1e-8 of the score scale."""
import numpy as np
import pytest

from oracle import pls as opls
from oracle import pls_lda as opl
from fastpls_b200 import synthetic
from parity_utils import REL_TOL, labels_match_beyond_margin, rel_err, sign_align, subspace_angle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data():
    return synthetic.c2_plsda(seed=5, n=1500, n_test=300, p=300, n_classes=40)


@pytest.mark.parametrize("method", [1, 3])
@pytest.mark.parametrize("f32", [True, False])
def test_pls_lda_matches_oracle(lib, data, method, f32):
    d = data
    Xtr = d["Xtrain"] if f32 else d["Xtrain"].astype(np.float64)
    Xte = d["Xtest"] if f32 else d["Xtest"].astype(np.float64)
    Y = opls.transformy(d["ytrain"])
    nc = [5, 12, 5]
    kw = dict(method=method, oversample=10, power_iters=2, seed=3)
    got = lib.pls_lda(Xtr, Y, d["ytrain"], Xte, nc, d["n_classes"], **kw)
    ref = opl.pls_lda(d["Xtrain"].astype(np.float64), Y, d["ytrain"], d["Xtest"].astype(np.float64), nc,
                      d["n_classes"], **kw)
    assert np.array_equal(got["ncomp"], ref["ncomp"])
    assert np.array_equal(got["unique_ncomp"], ref["unique_ncomp"])
    assert rel_err(got["B"], ref["model"]["B"]) < REL_TOL
    K0 = got["R_predict"].shape[1]
    assert subspace_angle(got["R_predict"], ref["R_predict"][:, :K0]) < 1e-8
    Rp = sign_align(got["R_predict"], ref["R_predict"][:, :K0])
    assert rel_err(Rp, ref["R_predict"][:, :K0]) < 1e-8
    for u, kk in enumerate(got["unique_ncomp"]):
        r = ref["lda"][str(int(kk))]
        lin = got["lda_linear"][:, :kk, u]
        assert rel_err(sign_align(lin, r["linear"]), r["linear"]) < 1e-8
        assert rel_err(got["lda_constants"][:, u], r["constants"]) < REL_TOL
    for i in range(len(nc)):
        ok, nclear = labels_match_beyond_margin(got["pred_codes"][:, i], ref["pred_codes"][:, i],
                                                ref["pred_scores"][i], 1e-8)
        assert ok and nclear > 0.9 * Xte.shape[0]


def test_pls_lda_equals_separate_calls(lib, data):
    # the fused call gives the labels of PLSSVD, LDA-project-train and
    # LDA-project-predict called one after another
    d = data
    X = d["Xtrain"].astype(np.float64)
    Xt = d["Xtest"].astype(np.float64)
    Y = opls.transformy(d["ytrain"])
    fused = lib.pls_lda(X, Y, d["ytrain"], Xt, [8], d["n_classes"], method=1, power_iters=2, seed=2)
    model = lib.pls_model1(X, Y, [8], svd_method=4, power_iters=2, seed=2)
    Rp = model["R"] / model["vX"].T
    off = (model["mX"] @ Rp).ravel()
    lda = lib.lda_project_train_prefix(X, Rp, off, d["ytrain"], d["n_classes"], [8])
    sep = lib.lda_project_predict(Xt, Rp, off, lda["8"], return_scores=True)
    ok, _ = labels_match_beyond_margin(fused["pred_codes"][:, 0], sep["pred"], sep["scores"], 1e-8)
    assert ok


def test_pls_lda_argument_errors(lib, data):
    d = data
    Y = opls.transformy(d["ytrain"])
    with pytest.raises(lib.FastPLSError):
        lib.pls_lda(d["Xtrain"], Y, d["ytrain"], d["Xtest"], [3], d["n_classes"], method=2)
    bad = d["ytrain"].copy()
    bad[0] = d["n_classes"] + 1
    with pytest.raises(lib.FastPLSError):
        lib.pls_lda(d["Xtrain"], Y, bad, d["Xtest"], [3], d["n_classes"])

"""Mixed-precision single fits against the FP64 drop-in on the same inputs:
PLSSVD + LDA (PLS-DA), fast SIMPLS on a compressed response, the matrix-free
PLSSVD and the predictions.  Bar for the three-plane BF16x6 mode: relative
prediction error within 1e-5 and identical class labels wherever the FP64
decision margin exceeds 1e-5.  The two-plane BF16x3 mode (the CV grids' mixed
mode) is checked at its own, looser, level."""
import numpy as np
import pytest

from oracle import pls as opls
from fastpls_b200 import synthetic
from parity_utils import labels_match_beyond_margin, rel_err

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5


@pytest.fixture
def both(lib):
    """Runs fn in FP64 and in BF16x6 session precision; restores FP64."""
    def run(fn, mode="bf16x6"):
        lib.set_precision("fp64")
        a = fn()
        lib.set_precision(mode)
        try:
            b = fn()
        finally:
            lib.set_precision("fp64")
        return a, b
    return run


@pytest.fixture(scope="module")
def c2_mid():
    return synthetic.c2_plsda(seed=3, n=3000, n_test=600, p=1500, n_classes=20)


def test_precision_setting(lib):
    assert lib.get_precision() == "fp64"
    with pytest.raises(lib.FastPLSError):
        lib.set_precision(7)
    for mode in ("bf16x3", "bf16x6"):
        lib.set_precision(mode)
        assert lib.get_precision() == mode
    lib.set_precision("fp64")


def test_plssvd_lda_mixed(lib, both, c2_mid):
    d = c2_mid
    X, Xt = d["Xtrain"].astype(np.float64), d["Xtest"].astype(np.float64)
    Y = opls.transformy(d["ytrain"])

    def fit():
        m = lib.pls_model1(X, Y, [5, 15], svd_method=4, power_iters=2, seed=1)
        pr = lib.predict_lowrank(m, Xt)["Ypred"]
        Rp = m["R"] / m["vX"].T
        off = (m["mX"] @ Rp).ravel()
        lda = lib.lda_project_train_prefix(X, Rp, off, d["ytrain"], d["n_classes"], [15])
        lp = lib.lda_project_predict(Xt, Rp, off, lda["15"], return_scores=True)
        return m, pr, lp

    (m64, p64, l64), (mbf, pbf, lbf) = both(fit)
    assert rel_err(mbf["singular_values"], m64["singular_values"]) < MIXED_TOL
    assert rel_err(pbf, p64) < MIXED_TOL
    ok, clear = labels_match_beyond_margin(lbf["pred"], l64["pred"], l64["scores"], margin=1e-5)
    assert ok and clear > 0.95 * Xt.shape[0]
    assert rel_err(lbf["scores"], l64["scores"]) < MIXED_TOL


def test_simpls_fast_mixed_compressed_response(lib, both):
    d = synthetic.c5_lowrank(seed=8, n=2500, p=2000, q=400, rank=12, n_test=300)
    X, Xt = d["Xtrain"].astype(np.float64), d["Xtest"].astype(np.float64)
    rng = np.random.default_rng(3)
    G = rng.standard_normal((400, 40)) / np.sqrt(40)

    def fit():
        enc = lib.gaussian_y_encode(d["Ytrain"].astype(np.float64), G)
        m = lib.pls_model2_fast(X, enc["Z"], [4, 12], seed=2)
        z = lib.predict_lowrank(m, Xt)["Ypred"]
        return [lib.gaussian_y_decode(z[:, :, a], enc["decoder"], enc["y_center"]) for a in range(2)]

    y64, ybf = both(fit)
    # 4 components (inside the latent rank): the 1e-5 bar.  12 components reach
    # the data's latent rank; the trailing components are weakly determined and
    # amplify any product error (FP64 rounding differences too), so their bar
    # is stated separately.
    assert rel_err(ybf[0], y64[0]) < MIXED_TOL
    assert rel_err(ybf[1], y64[1]) < 1e-4


def test_plssvd_xprod_mixed(lib, both):
    d = synthetic.c1_simpls_regression(seed=9, n=1200, p=900, m=300, rank=10)
    X, Y, Xt = d["Xtrain"], d["Ytrain"], d["Xtest"]

    def fit():
        m = lib.pls_model1(X, Y, [6], oversample=8, power_iters=2, seed=4, xprod=True)
        return lib.predict_lowrank(m, Xt)["Ypred"]

    p64, pbf = both(fit)
    assert rel_err(pbf, p64) < MIXED_TOL


def test_plssvd_two_plane_mode(lib, both, c2_mid):
    d = c2_mid
    X, Xt = d["Xtrain"].astype(np.float64), d["Xtest"].astype(np.float64)
    Y = opls.transformy(d["ytrain"])

    def fit():
        m = lib.pls_model1(X, Y, [15], svd_method=4, power_iters=2, seed=1)
        return lib.predict_lowrank(m, Xt)["Ypred"]

    p64, pbf = both(fit, "bf16x3")
    assert rel_err(pbf, p64) < 2e-4


def test_opls_filter_mixed_wide_tiles(lib, both):
    # X^T Y of the filter (2100 x 600) takes the 128 x 128 three-plane tiles
    d = synthetic.c5_lowrank(seed=11, n=2500, p=2100, q=600, rank=10, n_test=10)
    X = d["Xtrain"].astype(np.float64)
    Y = d["Ytrain"].astype(np.float64)
    ref, got = both(lambda: lib.opls_filter(X, Y, 2))
    assert got["north"] == ref["north"] == 2
    assert rel_err(got["X"], ref["X"]) < MIXED_TOL

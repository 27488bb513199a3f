"""GPU parity of Gaussian response compression and of the OPLS filter (C5 path)."""
import numpy as np
import pytest

from oracle import gaussian_y as og
from oracle import opls as oopls
from oracle import pls as opls
from fastpls_b200 import synthetic
from parity_utils import REL_TOL, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c5_small():
    return synthetic.c5_lowrank(seed=4, n=1500, p=700, q=300, rank=12, n_test=300)


def test_gaussian_y_regression_roundtrip(lib, c5_small):
    Y = c5_small["Ytrain"].astype(np.float64)
    rng = np.random.default_rng(1)
    G = rng.standard_normal((Y.shape[1], 40)) / np.sqrt(40)
    got = lib.gaussian_y_encode(Y, G)
    ref = og.prepare_regression(Y, G)
    assert rel_err(got["Z"], ref["Z"]) < 1e-12
    assert rel_err(got["y_center"], ref["y_center"]) < 1e-13
    assert rel_err(got["decoder"], ref["decoder"]) < REL_TOL
    Yd = lib.gaussian_y_decode(got["Z"], got["decoder"], got["y_center"])
    assert rel_err(Yd, og.decode_regression(ref["Z"], ref["decoder"], ref["y_center"])) < REL_TOL


def test_gaussian_y_simpls_pipeline(lib, c5_small):
    # SIMPLS on the compressed response, then decoding (the C5 regression route).
    X = c5_small["Xtrain"].astype(np.float64)
    Y = c5_small["Ytrain"].astype(np.float64)
    Xt = c5_small["Xtest"].astype(np.float64)
    rng = np.random.default_rng(2)
    G = rng.standard_normal((Y.shape[1], 30)) / np.sqrt(30)
    enc = lib.gaussian_y_encode(Y, G)
    ref_enc = og.prepare_regression(Y, G)
    got = lib.pls_model2_fast(X, enc["Z"], [5, 12], seed=1)
    ref = opls.pls_model2_fast(X, ref_enc["Z"], [5, 12], seed=1)
    zg = lib.predict_lowrank(got, Xt)["Ypred"]
    zr = opls.pls_predict(ref, Xt)["Ypred"]
    assert rel_err(zg, zr) < REL_TOL
    for a in range(2):
        yg = lib.gaussian_y_decode(zg[:, :, a], enc["decoder"], enc["y_center"])
        yr = og.decode_regression(zr[:, :, a], ref_enc["decoder"], ref_enc["y_center"])
        assert rel_err(yg, yr) < REL_TOL


def test_nearest_code_classes(lib):
    rng = np.random.default_rng(3)
    codes = og.class_codes(rng.standard_normal((12, 9)) / 3.0)
    Z = rng.standard_normal((400, 9))
    assert np.array_equal(lib.nearest_code_classes(Z, codes), og.nearest_code_classes(Z, codes))


@pytest.mark.parametrize("scaling,q", [(1, 300), (2, 8)])
def test_opls_filter_matches_oracle(lib, c5_small, scaling, q):
    X = c5_small["Xtrain"].astype(np.float64)
    Y = c5_small["Ytrain"][:, :q].astype(np.float64)
    got = lib.opls_filter(X, Y, 2, scaling=scaling)
    ref = oopls.opls_filter(X, Y, 2, scaling=scaling)
    assert got["north"] == ref["north"] == 2
    assert rel_err(got["X"], ref["X"]) < 1e-8
    # orthogonal weights are defined up to sign
    for a in range(2):
        s = np.sign(got["W_orth"][:, a] @ ref["W_orth"][:, a])
        assert rel_err(s * got["W_orth"][:, a], ref["W_orth"][:, a]) < 1e-8
        assert rel_err(s * got["P_orth"][:, a], ref["P_orth"][:, a]) < 1e-8
    Xt = c5_small["Xtest"].astype(np.float64)
    ft = lib.opls_apply_filter(Xt, got["mX"], got["vX"], got["W_orth"], got["P_orth"])
    fr = oopls.opls_apply_filter(Xt, ref["mX"], ref["vX"], ref["W_orth"], ref["P_orth"])
    assert rel_err(ft, fr) < 1e-8


def test_opls_filter_wide_response(lib):
    # p < q: the leading left vector comes from the p x p Gram side.
    d = synthetic.c5_lowrank(seed=9, n=900, p=120, q=400, rank=10, n_test=50)
    X = d["Xtrain"].astype(np.float64)
    Y = d["Ytrain"].astype(np.float64)
    got = lib.opls_filter(X, Y, 3)
    ref = oopls.opls_filter(X, Y, 3)
    assert got["north"] == ref["north"] == 3
    assert rel_err(got["X"], ref["X"]) < 1e-8
    for a in range(3):
        s = np.sign(got["P_orth"][:, a] @ ref["P_orth"][:, a])
        assert rel_err(s * got["P_orth"][:, a], ref["P_orth"][:, a]) < 1e-8


def test_opls_filter_zero_components(lib, c5_small):
    X = c5_small["Xtrain"][:200, :50].astype(np.float64)
    Y = c5_small["Ytrain"][:200, :4].astype(np.float64)
    got = lib.opls_filter(X, Y, 0)
    assert got["north"] == 0
    assert rel_err(got["X"], X - X.mean(axis=0)) < 1e-14

"""GPU parity of the matrix-free (implicit XᵀY) PLSSVD and SIMPLS paths."""
import numpy as np
import pytest

from oracle import pls as opls
from oracle import xprod as ox
from fastpls_b200 import synthetic
from parity_utils import REL_TOL, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    return synthetic.c1_simpls_regression(seed=21, n=400, p=300, m=120, rank=10)


@pytest.mark.parametrize("power", [1, 2])
def test_plssvd_xprod_matches_oracle(lib, c1, power):
    X, Y, Xt = c1["Xtrain"], c1["Ytrain"], c1["Xtest"]
    got = lib.pls_model1(X, Y, [4, 8], fit=True, oversample=6, power_iters=power, seed=5, xprod=True)
    ref = ox.pls_model1_xprod(X, Y, [4, 8], fit=True, rsvd_oversample=6, rsvd_power=power, seed=5)
    assert rel_err(got["singular_values"], ref["singular_values"][:8]) < REL_TOL
    for a in range(2):
        assert rel_err(got["B"][:, :, a], ref["B"][:, :, a]) < REL_TOL
        assert rel_err(got["Yfit"][:, :, a], ref["Yfit"][:, :, a]) < REL_TOL
    assert rel_err(got["R2Y"], ref["R2Y"]) < REL_TOL
    # the operator path agrees with the materialized rSVD path on the same data
    mat = lib.pls_model1(X, Y, [4, 8], oversample=6, power_iters=power, seed=5)
    assert rel_err(got["B"], mat["B"]) < 1e-8


def test_plssvd_xprod_exact_fallback(lib):
    # min(n, p, m) <= 32: the reference forms XᵀY and takes the exact SVD
    d = synthetic.c1_simpls_regression(seed=22, n=200, p=80, m=20, rank=6)
    got = lib.pls_model1(d["Xtrain"], d["Ytrain"], [3, 6], xprod=True)
    ref = ox.pls_model1_xprod(d["Xtrain"], d["Ytrain"], [3, 6])
    assert rel_err(got["B"], ref["B"]) < REL_TOL


@pytest.mark.parametrize("scaling", [1, 2])
def test_simpls_xprod_matches_oracle(lib, c1, scaling):
    X, Y, Xt = c1["Xtrain"], c1["Ytrain"], c1["Xtest"]
    got = lib.pls_model2_fast(X, Y, [2, 5, 12], scaling=scaling, fit=True, seed=7, xprod=True)
    ref = ox.pls_model2_fast_xprod(X, Y, [2, 5, 12], scaling=scaling, fit=True, seed=7)
    assert got["n_components"] == ref["n_components"] == 12
    for a in range(3):
        assert rel_err(got["B"][:, :, a], ref["B"][:, :, a]) < REL_TOL
        assert rel_err(got["Yfit"][:, :, a], ref["Yfit"][:, :, a]) < REL_TOL
    assert rel_err(got["R2Y"], ref["R2Y"]) < REL_TOL
    sg = np.sign(np.sum(got["R"] * ref["R"], axis=0))
    assert rel_err(got["R"] * sg, ref["R"]) < REL_TOL
    assert rel_err(got["Q"] * sg, ref["Q"]) < REL_TOL
    # same model as the materialized fast SIMPLS
    mat = opls.pls_model2_fast(X, Y, [2, 5, 12], scaling=scaling, seed=7)
    assert rel_err(got["B"], mat["B"]) < 1e-8


def test_xprod_precision_codes_rejected(lib, c1):
    X, Y = c1["Xtrain"], c1["Ytrain"]
    import ctypes
    nc = np.array([2], dtype=np.int32)
    R = np.zeros((300, 2), order="F")
    err = ctypes.create_string_buffer(256)
    rc = lib.load().fpls_pls_model2_fast_xprod(
        lib._p(lib._f64(X)), 400, 300, lib._p(lib._f64(Y)), 120, lib._p(nc), 1, 1, 0, 1, 5,
        lib._p(R), lib._p(np.zeros((120, 2), order="F")), lib._p(np.zeros(300)), lib._p(np.zeros(300)),
        lib._p(np.zeros(120)), None, None, None, None, err, 256)
    assert rc == 1 and b"CPU-only" in err.value

"""Kernel PLS on the device (kernel matrices, centring, fused fit) against the
oracle restatement of kernel_matrix_cpp / center_kernel_*_cpp and the kernel
PLS wrapper (src/fastPLS.cpp:4314-4375, R/main.R:2764-2917)."""
import numpy as np
import pytest

from oracle import kernel as ok
from oracle import pls as opls
from parity_utils import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["linear", "rbf", "poly"])
def test_kernel_matrix(lib, kernel):
    rng = np.random.default_rng(3)
    X1 = rng.standard_normal((300, 40))
    X2 = rng.standard_normal((170, 40))
    g, deg, c0 = 0.05, 3, 1.0
    kid = ok.KERNELS[kernel]
    for A, B in ((X1, X2), (X1, None)):
        got = lib.kernel_matrix(A, B, kernel, g, deg, c0)
        ref = ok.kernel_matrix(A, A if B is None else B, kid, g, deg, c0)
        assert rel_err(got, ref) < 1e-12
    sym = lib.kernel_matrix(X1, None, kernel, g, deg, c0)
    assert np.array_equal(sym, sym.T)
    if kernel == "rbf":
        assert np.allclose(np.diag(sym), 1.0, atol=1e-12)


def test_center_kernel(lib):
    rng = np.random.default_rng(4)
    X = rng.standard_normal((250, 30))
    Xt = rng.standard_normal((60, 30))
    K = ok.kernel_matrix(X, X, 2, 0.03, 3, 1.0)
    Kt = ok.kernel_matrix(Xt, X, 2, 0.03, 3, 1.0)
    got = lib.center_kernel_train(K)
    ref = ok.center_kernel_train(K)
    assert rel_err(got["K"], ref["K"]) < 1e-12
    assert rel_err(got["col_means"], ref["col_means"]) < 1e-14
    assert abs(got["grand_mean"] - ref["grand_mean"]) <= 1e-14 * abs(ref["grand_mean"])
    gt = lib.center_kernel_test(Kt, got["col_means"], got["grand_mean"])
    assert rel_err(gt, ok.center_kernel_test(Kt, ref["col_means"], ref["grand_mean"])) < 1e-12


@pytest.mark.parametrize("kernel,scaling", [("rbf", 1), ("poly", 2), ("rbf", 3)])
def test_kernel_pls_fit_and_predict(lib, kernel, scaling):
    # the shape of the reference's kernel PLS test (test-kernel-opls.R): a few
    # dozen rows, ten predictors, three classes, ncomp 1:2 -- here with more
    # rows and components to exercise the SIMPLS loop on the centred kernel
    rng = np.random.default_rng(2201 + scaling)
    X = rng.standard_normal((160, 10))
    y = rng.integers(1, 4, 160)
    X[:, 0] += 0.8 * y
    Y = opls.transformy(y)
    idx = np.arange(24)
    tr = np.setdiff1d(np.arange(160), idx)
    nc = [1, 2, 5]
    got = lib.kernel_pls_model2_fast(X[tr], Y[tr], nc, kernel=kernel, scaling=scaling, seed=3)
    ref = ok.kernel_pls_fit(X[tr], Y[tr], nc, kernel=kernel, scaling=scaling, seed=3)
    assert abs(got["gamma"] - ref["gamma"]) == 0.0
    assert rel_err(got["col_means"], ref["col_means"]) < 1e-12
    assert rel_err(got["inner"]["B"], ref["inner"]["B"]) < 1e-9
    # prediction through the drop-in kernel routines and the low-rank predict
    Xref = (X[tr] - got["mX"]) / got["vX"]
    Xn = (X[idx] - got["mX"]) / got["vX"]
    Kt = lib.kernel_matrix(Xn, Xref, kernel, got["gamma"], got["degree"], got["coef0"])
    Kc = lib.center_kernel_test(Kt, got["col_means"], got["grand_mean"])
    pred = lib.predict_lowrank(got["inner"], Kc)["Ypred"]
    pref = ok.kernel_pls_predict(ref, X[idx])["Ypred"]
    assert rel_err(pred, pref) < 1e-9
    assert np.array_equal(pred.argmax(axis=1), pref.argmax(axis=1))


def test_kernel_pls_rejects_bad_input(lib):
    with pytest.raises(lib.FastPLSError):
        lib.kernel_matrix(np.ones((4, 3)), np.ones((4, 3)), 7)
    with pytest.raises(lib.FastPLSError):
        lib.kernel_matrix(np.ones((4, 3)), np.ones((4, 3)), "rbf", gamma=-1.0)

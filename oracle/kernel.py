"""Kernel PLS restatement (test infrastructure only).

  * kernel_matrix_cpp (linear / rbf / poly)   src/fastPLS.cpp:4314-4340
  * center_kernel_train_cpp                   src/fastPLS.cpp:4344-4357
  * center_kernel_test_cpp                    src/fastPLS.cpp:4360-4375
  * .fastpls_preprocess_train / _test         R/main.R:2764-2785
  * .kernel_pls_gamma (default 1 / p)         R/main.R:2792-2801
  * .kernel_pls_fit (non-linear kernels: preprocess, kernel, centre, inner
    fit on the centred kernel with scaling "none")   R/main.R:2826-2917
  * predict.fastPLSKernel                     R/main.R:3035-3048
The inner fit is the SIMPLS restatement of oracle.pls (pls_model2_fast).
"""
import numpy as np

from . import pls as opls

KERNELS = {"linear": 1, "rbf": 2, "poly": 3}


def kernel_matrix(X1, X2, kernel, gamma, degree, coef0):
    X1 = np.asarray(X1, dtype=np.float64)
    X2 = np.asarray(X2, dtype=np.float64)
    dots = X1 @ X2.T
    if kernel == 1:
        return dots
    if kernel == 3:
        return np.power(gamma * dots + coef0, degree)
    if kernel != 2:
        raise ValueError("Unknown kernel id")
    n1 = np.sum(X1 * X1, axis=1)
    n2 = np.sum(X2 * X2, axis=1)
    d2 = n1[:, None] + n2[None, :] - 2.0 * dots
    d2 = np.where((d2 < 0.0) & (d2 > -1e-10), 0.0, d2)
    return np.exp(-gamma * d2)


def center_kernel_train(K):
    K = np.asarray(K, dtype=np.float64)
    col_means = K.mean(axis=0)
    row_means = K.mean(axis=1)
    grand = col_means.mean()
    Kc = K - col_means[None, :]
    Kc = Kc - row_means[:, None]
    return dict(K=Kc + grand, col_means=col_means, grand_mean=grand)


def center_kernel_test(Ktest, col_means, grand):
    Ktest = np.asarray(Ktest, dtype=np.float64)
    row_means = Ktest.mean(axis=1)
    Kc = Ktest - np.asarray(col_means)[None, :]
    Kc = Kc - row_means[:, None]
    return Kc + grand


def preprocess_train(X, scaling):
    X = np.asarray(X, dtype=np.float64)
    mX = np.zeros(X.shape[1])
    if scaling < 3:
        mX = X.mean(axis=0)
        X = X - mX
    vX = np.ones(X.shape[1])
    if scaling == 2:
        vX = X.std(axis=0, ddof=1)
        vX[~np.isfinite(vX) | (vX == 0)] = 1.0
        X = X / vX
    return X, mX, vX


def kernel_pls_fit(Xtrain, Ytrain, ncomp, kernel="rbf", gamma=None, degree=3, coef0=1.0, scaling=1, seed=1):
    Xp, mX, vX = preprocess_train(Xtrain, scaling)
    if gamma is None:
        gamma = 1.0 / max(1, Xp.shape[1])
    kid = KERNELS[kernel]
    kc = center_kernel_train(kernel_matrix(Xp, Xp, kid, gamma, degree, coef0))
    inner = opls.pls_model2_fast(kc["K"], np.asarray(Ytrain, dtype=np.float64), ncomp, scaling=3, seed=seed)
    return dict(inner=inner, Xref=Xp, mX=mX, vX=vX, kernel_id=kid, gamma=gamma, degree=degree, coef0=coef0,
                col_means=kc["col_means"], grand_mean=kc["grand_mean"])


def kernel_pls_predict(model, Xnew):
    Xn = (np.asarray(Xnew, dtype=np.float64) - model["mX"]) / model["vX"]
    Kt = kernel_matrix(Xn, model["Xref"], model["kernel_id"], model["gamma"], model["degree"], model["coef0"])
    Kc = center_kernel_test(Kt, model["col_means"], model["grand_mean"])
    return opls.pls_predict(model["inner"], Kc)

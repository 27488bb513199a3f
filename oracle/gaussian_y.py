"""Gaussian response compression restatement (test infrastructure only).

  * .gaussian_y_ridge_decoder     R/main.R:1968-1981
  * .gaussian_y_class_codes       R/main.R:1983-1998
  * .prepare_gaussian_y           R/main.R:2000-2064 (regression branch)
  * .decode_gaussian_y_matrix     R/main.R:2085-2104
  * nearest_code_classes          src/fastPLS.cpp:4203-4215

The projection and class codes come from R's RNG on the R side of the
boundary; here they are inputs.
"""
import numpy as np


def ridge_decoder(Z, Yc):
    ztz = Z.T @ Z
    ridge = 1e-8 * np.mean(np.diag(ztz))
    if not np.isfinite(ridge) or ridge <= 0:
        ridge = 1e-8
    rhs = Z.T @ Yc
    return np.linalg.solve(ztz + ridge * np.eye(ztz.shape[0]), rhs)


def prepare_regression(Y, projection):
    Y = np.asarray(Y, dtype=np.float64)
    y_center = Y.mean(axis=0)
    Yc = Y - y_center
    Z = Yc @ projection
    decoder = ridge_decoder(Z, Yc)
    return dict(Z=Z, y_center=y_center, decoder=decoder)


def decode_regression(Z, decoder, y_center):
    return np.asarray(Z) @ decoder + np.asarray(y_center)[None, :]


def class_codes(raw):
    """Centre, column-scale and row-normalise raw N(0,1)/sqrt(dim) codes."""
    codes = np.array(raw, dtype=np.float64)
    codes -= codes.mean(axis=0, keepdims=True)
    sds = np.sqrt((codes * codes).sum(axis=0))
    sds[~np.isfinite(sds) | (sds == 0)] = 1.0
    codes /= sds
    rn = np.sqrt((codes * codes).sum(axis=1))
    rn[~np.isfinite(rn) | (rn == 0)] = 1.0
    return codes / rn[:, None]


def nearest_code_classes(Z, codes):
    score = 2.0 * (np.asarray(Z) @ codes.T) - (codes * codes).sum(axis=1)[None, :]
    return (np.argmax(score, axis=1) + 1).astype(np.int32)

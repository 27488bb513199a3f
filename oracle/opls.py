"""OPLS orthogonal filter restatement (test infrastructure only).

  * opls_filter_cpp        src/fastPLS.cpp:4377-4460
  * opls_apply_filter_cpp  src/fastPLS.cpp:4463-4483
"""
import numpy as np
import scipy.linalg as sla


def opls_filter(X, Y, north, scaling=1):
    X = np.array(X, dtype=np.float64)
    Y = np.array(Y, dtype=np.float64)
    p = X.shape[1]
    mX = np.zeros(p)
    if scaling < 3:
        mX = X.mean(axis=0)
        X -= mX
    vX = np.ones(p)
    if scaling == 2:
        vX = X.std(axis=0, ddof=1)
        vX[~np.isfinite(vX) | (vX == 0)] = 1.0
        X /= vX
    Y = Y - Y.mean(axis=0)
    W = np.zeros((p, north))
    P = np.zeros((p, north))
    used = 0
    for _ in range(north):
        S = X.T @ Y
        U, d, Vt = sla.svd(S, full_matrices=False, lapack_driver="gesdd")
        w = U[:, 0]
        wn = np.linalg.norm(w)
        if not np.isfinite(wn) or wn <= 0:
            break
        w = w / wn
        t = X @ w
        tss = t @ t
        if not np.isfinite(tss) or tss <= 0:
            break
        pv = X.T @ t / tss
        wo = pv - w * ((w @ pv) / (w @ w))
        won = np.linalg.norm(wo)
        if not np.isfinite(won) or won <= 0:
            break
        wo = wo / won
        to = X @ wo
        toss = to @ to
        if not np.isfinite(toss) or toss <= 0:
            break
        po = X.T @ to / toss
        X -= np.outer(to, po)
        W[:, used] = wo
        P[:, used] = po
        used += 1
    return dict(X=X, mX=mX, vX=vX, W_orth=W[:, :used], P_orth=P[:, :used], north=used)


def opls_apply_filter(X, mX, vX, W, P):
    X = (np.asarray(X, dtype=np.float64) - mX) / vX
    for a in range(W.shape[1]):
        t = X @ W[:, a]
        X = X - np.outer(t, P[:, a])
    return X

"""LDA head restatement (test infrastructure only).

  * lda_train_prefix_cpp            src/fastPLS.cpp:1817-1927
  * lda_project_train_prefix_cpp    src/fastPLS.cpp:1930-1957
  * lda_labels_from_scores          src/fastPLS.cpp:1719-1733
  * lda_predict_labels_cpp          src/fastPLS.cpp:2080-2098
  * lda_project_predict_labels_cpp  src/fastPLS.cpp:2100-2147
"""
import numpy as np
import scipy.linalg as sla


def _inv_sympd(A):
    try:
        c = sla.cho_factor(A, lower=False)
        return sla.cho_solve(c, np.eye(A.shape[0]))
    except sla.LinAlgError:
        try:
            return sla.inv(A)
        except sla.LinAlgError:
            return sla.pinv(A)


def lda_train_prefix(T, y, n_classes, ncomp, ridge=1e-8):
    T = np.asarray(T, dtype=np.float64)
    y = np.asarray(y, dtype=np.int64)
    n = T.shape[0]
    ncomp = [int(c) for c in np.atleast_1d(ncomp)]
    kmax = max(ncomp)
    if n == 0 or T.shape[1] == 0:
        raise ValueError("lda_train_prefix_cpp requires a non-empty score matrix")
    if n_classes < 2:
        raise ValueError("lda_train_prefix_cpp requires at least two classes")
    if kmax < 1 or kmax > T.shape[1]:
        raise ValueError("component counts must be in 1..ncol(Ttrain)")
    Tk = T[:, :kmax]
    if y.min() < 1 or y.max() > n_classes:
        raise ValueError("lda_train_prefix_cpp labels must be encoded as 1..n_classes")
    counts = np.bincount(y - 1, minlength=n_classes).astype(np.float64)
    means = np.zeros((n_classes, kmax))
    np.add.at(means, y - 1, Tk)
    if np.any(counts <= 0):
        raise ValueError("lda_train_prefix_cpp received an empty class")
    means /= counts[:, None]
    G = Tk.T @ Tk
    pooled_full = np.triu(G) + np.triu(G, 1).T
    for c in range(n_classes):
        pooled_full -= counts[c] * np.outer(means[c], means[c])
    df = max(1.0, float(n) - float(n_classes))
    pooled_full /= df
    models = {}
    for kk in ncomp:
        pooled = pooled_full[:kk, :kk].copy()
        mk = means[:, :kk]
        scale = np.trace(pooled) / max(1, kk)
        if not np.isfinite(scale) or scale <= 0:
            scale = 1.0
        lam = ridge if (np.isfinite(ridge) and ridge >= 0) else 1e-8
        lam *= scale
        pooled[np.diag_indices(kk)] += lam
        inv_cov = _inv_sympd(pooled)
        linear = mk @ inv_cov
        prior = np.maximum(counts / n, np.finfo(np.float64).tiny)
        constants = -0.5 * np.sum(mk * linear, axis=1) + np.log(prior)
        models[str(kk)] = dict(means=mk.copy(), inv_cov=inv_cov, linear=linear,
                               constants=constants, priors=counts / n, ridge=lam)
    return models


def lda_project_train_prefix(X, R, offset, y, n_classes, ncomp, ridge=1e-8):
    T = np.asarray(X, dtype=np.float64) @ np.asarray(R, dtype=np.float64)
    if offset is not None and len(offset) >= R.shape[1]:
        T = T - np.asarray(offset)[None, :R.shape[1]]
    return lda_train_prefix(T, y, n_classes, ncomp, ridge)


def labels_from_scores(scores, constants):
    return (np.argmax(scores + np.asarray(constants)[None, :], axis=1) + 1).astype(np.int32)


def lda_predict_labels(T, lda):
    return labels_from_scores(np.asarray(T) @ lda["linear"].T, lda["constants"])


def lda_project_predict(X, R, offset, lda, return_scores=False):
    """Labels (and the score matrix incl. constants) with the reference's route rule."""
    X = np.asarray(X, dtype=np.float64)
    R = np.asarray(R, dtype=np.float64)
    linear = lda["linear"]
    constants = np.asarray(lda["constants"], dtype=np.float64)
    n, p = X.shape
    k = R.shape[1]
    C = linear.shape[0]
    latent_ops = n * k * (p + C)
    direct_ops = n * p * C
    if direct_ops < 0.5 * latent_ops:
        W = R @ linear.T
        cadj = constants.copy()
        if offset is not None and len(offset) >= k:
            cadj = cadj - np.asarray(offset)[:k] @ linear.T
        scores = X @ W + cadj[None, :]
    else:
        T = X @ R
        if offset is not None and len(offset) >= k:
            T = T - np.asarray(offset)[None, :k]
        scores = T @ linear.T + constants[None, :]
    lab = (np.argmax(scores, axis=1) + 1).astype(np.int32)
    if return_scores:
        return lab, scores
    return lab

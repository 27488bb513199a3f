"""Label-aware PLSSVD restatement (test infrastructure only).

  * .cap_plssvd_ncomp                   R/main.R:24-42
  * .plssvd_label_aware_stream_model    R/main.R:513-655

Blocks of ``block_size`` rows are centred / scaled and reduced exactly as the
R code does (column sums, class sums via rowsum, G = sum_b (X_b R)^T (X_b R));
the SVD of the class-sum cross-covariance is LAPACK gesdd (R's svd()).
"""
import numpy as np
import scipy.linalg as sla


def cap_ncomp(ncomp, n, p, m):
    max_rank = min(n, p, m)
    if max_rank < 1:
        raise ValueError("plssvd rank is < 1")
    nc = np.minimum(np.maximum(np.asarray(ncomp, dtype=np.int64), 1), max_rank)
    return nc.astype(np.int32), max_rank


def label_aware_plssvd(X, y_codes, m, ncomp, scaling=1, block_size=8192, svd_method=3,
                       oversample=10, power_iters=1, seed=1):
    """svd_method 3: R's svd() (gesdd) as the reference; 4 / 5: the seeded rSVD
    recipe of src/svd_cpu_rsvd.cpp:95-126 on the same S (the large-class
    configuration's variant)."""
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y_codes, dtype=np.int64)
    n, p = X.shape
    if n < 1 or p < 1 or m < 2:
        raise ValueError("label-aware PLSSVD requires non-empty X and at least two classes")
    ncomp, _ = cap_ncomp(ncomp, n, p, m)
    K = int(ncomp.max())
    sums = np.zeros(p)
    sums_sq = np.zeros(p)
    for s in range(0, n, block_size):
        Xb = X[s:s + block_size]
        sums += Xb.sum(axis=0)
        if scaling == 2:
            sums_sq += (Xb * Xb).sum(axis=0)
    mX = sums / n if scaling < 3 else np.zeros(p)
    vX = np.ones(p)
    if scaling == 2:
        css = np.maximum(sums_sq - n * mX * mX, 0.0)
        vX = np.sqrt(css / max(1, n - 1))
        vX[~np.isfinite(vX) | (vX == 0)] = 1.0
    counts = np.bincount(y - 1, minlength=m)[:m].astype(np.float64)
    mY = counts / n

    def prep(Xb):
        if scaling < 3:
            Xb = Xb - mX
        if scaling == 2:
            Xb = Xb / vX
        return Xb

    class_sums = np.zeros((p, m))
    for s in range(0, n, block_size):
        Xb = prep(X[s:s + block_size])
        rs = np.zeros((m, p))
        np.add.at(rs, y[s:s + block_size] - 1, Xb)
        class_sums += rs.T
    total = class_sums.sum(axis=1)
    S = class_sums - np.outer(total, mY)
    if svd_method == 3:
        U, d, Vt = sla.svd(S, full_matrices=False, lapack_driver="gesdd")
    else:
        from .svd import truncated_svd
        res = truncated_svd(S, K, svd_method=svd_method, oversample=oversample,
                            power_iters=power_iters, seed=seed)
        U, d, Vt = res.U, res.s, res.Vt
    R = np.zeros((p, K))
    Q = np.zeros((m, K))
    r = min(K, U.shape[1])
    R[:, :r] = U[:, :r]
    Q[:, :r] = Vt[:r].T
    d = np.concatenate([d[:r], np.zeros(K - r)])
    G = np.zeros((K, K))
    for s in range(0, n, block_size):
        Tb = prep(X[s:s + block_size]) @ R
        G += Tb.T @ Tb
    L = len(ncomp)
    C_latent = np.zeros((K, K, L))
    W_latent = np.zeros((K, m, L))
    for a, k in enumerate(ncomp):
        Gk = G[:k, :k]
        ridge = 1e-10 * np.mean(np.diag(Gk))
        if not np.isfinite(ridge) or ridge <= 0:
            ridge = 1e-10
        coeff = np.linalg.solve(Gk + ridge * np.eye(k), np.diag(d[:k]))
        C_latent[:k, :k, a] = coeff
        W_latent[:k, :, a] = coeff @ Q[:, :k].T
    return dict(C_latent=C_latent, W_latent=W_latent, Q=Q, R=R, mX=mX, vX=vX, mY=mY,
                ncomp=ncomp, d=d, S=S, G=G)

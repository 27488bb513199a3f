"""Matrix-free (implicit X^T Y) PLS restatement (test infrastructure only).

  * project_deflated_left_double          src/fastPLS.cpp:625-640
  * finalize_rsvd_from_q_b_double         src/fastPLS.cpp:434-473
  * truncated_rsvd_crossprod_double       src/fastPLS.cpp:550-622
  * refresh_deflated_crossprod_left_double src/fastPLS.cpp:936-1000
  * pls_model1_rsvd_xprod_precision (3)   src/fastPLS.cpp:5518-5690
  * pls_model2_fast_rsvd_xprod_precision  src/fastPLS.cpp:5695-5986 (3, default options)

The cross-covariance S = X^T Y is never formed except in the exact fallback
(use_full_svd or l >= min(p, m)), which the reference also takes.
"""
import numpy as np

from . import svd as osvd
from .pls import (RQ, _center_scale, _solve_likely_sympd, env_int_or,
                  plssvd_use_small_exact_svd, should_store_coefficients)
from .rng import gaussian_matrix


def project_deflated(M, V, n_prev):
    if n_prev > 0:
        Vp = V[:, :n_prev]
        M = M - Vp @ (Vp.T @ M)
    return M


def finalize_from_q_b(Q, B, k):
    max_rank = min(B.shape)
    rank = min(max_rank, max(int(k), 1))
    U_hat, s, V = osvd.svd_econ(B, left_only=False)
    actual = min(rank, U_hat.shape[1], s.size, V.shape[1])
    return osvd.SVDResult(Q @ U_hat[:, :actual], s[:actual].copy(), V[:, :actual].T.copy())


def truncated_rsvd_crossprod(X, Y, k, oversample=10, power_iters=1, seed=1, use_full_svd=False):
    p = X.shape[1]
    m = Y.shape[1]
    max_rank = min(p, m)
    target = min(max_rank, max(int(k), 1))
    l = min(max_rank, target + max(int(oversample), 0))
    if use_full_svd or l >= max_rank:
        S = X.T @ Y
        return osvd.truncated_svd(S, target, osvd.SVD_METHOD_CPU_RSVD, oversample, power_iters,
                                  seed, left_only=False, use_full_svd=True)

    def a_times(M):
        return X.T @ (Y @ M)

    def at_times(M):
        return Y.T @ (X @ M)

    Ys = a_times(gaussian_matrix(m, l, seed))
    if power_iters == 1:
        Ys = a_times(at_times(Ys))
    else:
        for _ in range(max(power_iters, 0)):
            Ys = a_times(osvd.qr_econ_q(at_times(Ys)))
    Q = osvd.qr_econ_q(Ys)
    B = (X @ Q).T @ Y
    return finalize_from_q_b(Q, B, target)


def pls_model1_xprod(Xtrain, Ytrain, ncomp, scaling=1, fit=False, rsvd_oversample=10,
                     rsvd_power=1, seed=1):
    X = np.array(Xtrain, dtype=np.float64)
    Y = np.array(Ytrain, dtype=np.float64)
    n, p = X.shape
    m = Y.shape[1]
    max_rank = min(n, p, m)
    ncomp = np.maximum(np.minimum(np.atleast_1d(np.asarray(ncomp, dtype=np.int64)), max_rank), 1)
    L = ncomp.size
    max_eff = min(int(ncomp.max()), max_rank)
    X, mX, vX = _center_scale(X, scaling)
    mY = Y.mean(axis=0)
    Y = Y - mY
    res = truncated_rsvd_crossprod(X, Y, max_eff, rsvd_oversample, rsvd_power, seed,
                                   plssvd_use_small_exact_svd(max_rank, osvd.SVD_METHOD_CPU_RSVD))
    U, s, V = res.U, res.s, res.Vt.T
    store_B = should_store_coefficients(p, m, L, True)
    K0 = max_eff
    C_latent = np.zeros((K0, K0, L))
    W_latent = np.zeros((K0, m, L))
    B = np.zeros((p, m, L)) if store_B else None
    Yfit = np.zeros((n, m, L)) if fit else None
    R2Y = np.zeros(L)
    max_eff = min(max_eff, U.shape[1], V.shape[1])
    U = U[:, :max_eff]
    V = V[:, :max_eff]
    T = X @ U
    G = T.T @ T
    for a in range(L):
        mc = min(int(ncomp[a]), max_eff)
        C = _solve_likely_sympd(G[:mc, :mc], np.diag(s[:mc]))
        C_latent[:mc, :mc, a] = C
        Wa = C @ V[:, :mc].T
        W_latent[:mc, :, a] = Wa
        if store_B:
            B[:, :, a] = U[:, :mc] @ Wa
        if fit:
            t1 = T[:, :mc] @ Wa
            R2Y[a] = RQ(Y, t1)
            Yfit[:, :, a] = t1 + mY
    out = dict(C_latent=C_latent, W_latent=W_latent, Q=V, Ttrain=T, R=U, mX=mX[None, :],
               vX=vX[None, :], mY=mY[None, :], ncomp=ncomp, Yfit=Yfit, R2Y=R2Y,
               singular_values=s, B_stored=store_B)
    if store_B:
        out["B"] = B
    return out


def refresh_crossprod_left(X, Y, V, n_prev, warm_start, power_iters, seed):
    """k_block = 1 (the default refresh block)."""
    p = X.shape[1]
    Ys = gaussian_matrix(p, 1, seed)
    if warm_start is not None and warm_start.size == p:
        Ys[:, 0] = warm_start
    Ys = project_deflated(Ys, V, n_prev)

    def a_times(M):
        return project_deflated(X.T @ (Y @ M), V, n_prev)

    def at_times(M):
        return Y.T @ (X @ project_deflated(M, V, n_prev))

    for _ in range(max(power_iters, 0)):
        Ys = a_times(at_times(Ys))
    Q = osvd.qr_econ_q(Ys)
    if Q.shape[1] < 1:
        return None
    Q = osvd.qr_econ_q(project_deflated(Q, V, n_prev))
    Bsmall = (X @ Q).T @ Y
    U_hat, _, _ = osvd.svd_econ(Bsmall, left_only=True)  # 1 x m: fewer rows than the eig threshold
    return project_deflated(Q @ U_hat, V, n_prev)[:, :1]


def pls_model2_fast_xprod(Xtrain, Ytrain, ncomp, scaling=1, fit=False, seed=1):
    X = np.array(Xtrain, dtype=np.float64)
    Y = np.array(Ytrain, dtype=np.float64)
    n, p = X.shape
    m = Y.shape[1]
    ncomp = np.maximum(np.atleast_1d(np.asarray(ncomp, dtype=np.int64)), 1)
    max_ncomp = int(ncomp.max())
    L = ncomp.size
    X, mX, vX = _center_scale(X, scaling)
    mY = Y.mean(axis=0)
    Y = Y - mY
    RR = np.zeros((p, max_ncomp))
    QQ = np.zeros((m, max_ncomp))
    VV = np.zeros((p, max_ncomp))
    store_B = should_store_coefficients(p, m, L, True)
    B = np.zeros((p, m, L)) if store_B else None
    Yfit = np.zeros((n, m, L)) if fit else None
    R2Y = np.zeros(L)
    Yfit_cur = np.zeros((n, m)) if fit else None
    Bcur = np.zeros((p, m))
    inc_power_iters = env_int_or("FASTPLS_FAST_INC_ITERS", 2, 1, 6)
    i_out = 0
    rr_prev = None
    a = 0
    while a < max_ncomp:
        Ub = refresh_crossprod_left(X, Y, VV, a, rr_prev, inc_power_iters, seed + a)
        if Ub is None or Ub.shape[1] < 1:
            break
        rr = Ub[:, 0].copy()
        tt = X @ rr
        tnorm = np.linalg.norm(tt)
        if not np.isfinite(tnorm) or tnorm <= 0:
            break
        tt = tt / tnorm
        rr = rr / tnorm
        pp = X.T @ tt
        qq = Y.T @ tt
        rr_prev = rr
        vv = pp.copy()
        if a > 0:
            Vp = VV[:, :a]
            vv = vv - Vp @ (Vp.T @ pp)
        vnorm = np.linalg.norm(vv)
        if not np.isfinite(vnorm) or vnorm <= 0:
            break
        vv = vv / vnorm
        RR[:, a] = rr
        QQ[:, a] = qq
        VV[:, a] = vv
        if store_B:
            Bcur = Bcur + np.outer(rr, qq)
        while i_out < L and a == ncomp[i_out] - 1:
            if store_B:
                B[:, :, i_out] = Bcur
            if fit:
                Yfit_cur = Yfit_cur + np.outer(tt, qq)
                R2Y[i_out] = RQ(Y, Yfit_cur)
                Yfit[:, :, i_out] = Yfit_cur + mY
            i_out += 1
        a += 1
    out = dict(R=RR, Q=QQ, mX=mX[None, :], vX=vX[None, :], mY=mY[None, :], ncomp=ncomp,
               Yfit=Yfit, R2Y=R2Y, B_stored=store_B, n_components=a)
    if store_B:
        out["B"] = B
    return out

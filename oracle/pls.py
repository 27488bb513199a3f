"""PLS fit and predict restatement (test infrastructure only).

  * variance (Welford, n-1)          src/fastPLS.cpp:1570-1589
  * RQ (R2 / Q2)                     src/fastPLS.cpp:1483-1500
  * transformy (one-hot)             src/fastPLS.cpp:1593-1604
  * should_store_coefficients        src/fastPLS.cpp:63-85
  * plssvd_use_small_exact_svd       src/fastPLS.cpp:318-324
  * pls_model1 (PLSSVD)              src/fastPLS.cpp:4780-4986
  * pls_model2 (classic SIMPLS)      src/fastPLS.cpp:2260-2451
  * leading_left_vec_dispatch        src/fastPLS.cpp:161-262
  * pls_model2_fast (SIMPLS)         src/fastPLS.cpp:2454-2778
    with SimplsFastRefreshWorkspace  src/fastPLS.cpp:1068-1190
    finalize_left_block_from_bsmall  src/fastPLS.cpp:264-291
  * pls_predict                      src/fastPLS.cpp:3211-3445
  * compact_prediction_weights       src/fastPLS.cpp:3737-3836
  * pls_predict_classes_compact_cpu  src/fastPLS.cpp:4115-4154
All arrays are float64; matrices are (rows, cols); cubes are (rows, cols, slices).
"""
import os

import numpy as np
import scipy.linalg as sla

from . import svd as osvd
from .rng import gaussian_matrix


def env_int_or(key, fallback, lo, hi):
    raw = os.environ.get(key)
    if raw is None:
        return fallback
    try:
        v = int(raw.strip().split()[0])
    except (ValueError, IndexError):
        return fallback
    return max(lo, min(hi, v))


def variance(X):
    """Column standard deviation by Welford's recurrence (fastPLS.cpp:1570-1589)."""
    X = np.asarray(X, dtype=np.float64)
    n = X.shape[0]
    mean = np.zeros(X.shape[1])
    m2 = np.zeros(X.shape[1])
    for i in range(n):
        xx = X[i]
        delta = xx - mean
        mean = mean + delta / (i + 1)
        m2 = m2 + delta * (xx - mean)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.sqrt(m2 / float(n - 1))


def RQ(y, yp):
    """1 - PRESS/TSS (fastPLS.cpp:1483-1500)."""
    y = np.asarray(y)
    yp = np.asarray(yp)
    my = y.mean(axis=0)
    press = np.sum((y - yp) ** 2)
    tss = np.sum((y - my) ** 2)
    return 1.0 - press / tss


def transformy(y):
    """One-hot of 1-based integer labels (fastPLS.cpp:1593-1604)."""
    y = np.asarray(y, dtype=np.int64)
    nc = int(y.max())
    return (y[:, None] == np.arange(1, nc + 1)[None, :]).astype(np.float64)


def should_store_coefficients(p, m, n_slices, compact_available=True):
    mode = os.environ.get("FASTPLS_STORE_B")
    if mode is not None:
        v = mode.lower()
        if v in ("always", "1", "true", "yes"):
            return True
        if v in ("never", "0", "false", "no"):
            return False
    if not compact_available:
        return True
    max_mb = env_int_or("FASTPLS_STORE_B_MAX_MB", 256, 0, 1048576)
    b_mb = float(p) * float(m) * float(max(n_slices, 1)) * 8.0 / (1024.0 * 1024.0)
    return b_mb <= float(max_mb)


def plssvd_use_small_exact_svd(max_rank, svd_method):
    if svd_method == osvd.SVD_METHOD_IRLBA:
        return max_rank < 6
    thr = env_int_or("FASTPLS_PLSSVD_SMALL_EXACT_MAX_RANK", 32, 5, 512)
    return max_rank <= thr


def _center_scale(X, scaling):
    n, p = X.shape
    mX = np.zeros(p)
    if scaling < 3:
        mX = X.mean(axis=0)
        X = X - mX
    vX = np.ones(p)
    if scaling == 2:
        vX = variance(X)
        X = X / vX
    return X, mX, vX


def _solve_likely_sympd(G, D):
    try:
        return sla.solve(G, D, assume_a="pos")
    except (sla.LinAlgError, ValueError):
        return sla.solve(G, D)


def pls_model1(Xtrain, Ytrain, ncomp, scaling=1, fit=False, svd_method=4,
               rsvd_oversample=10, rsvd_power=1, svds_tol=0.0, seed=1):
    """PLSSVD (fastPLS.cpp:4780-4986), optimized latent solve C = G^-1 D."""
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
    S = X.T @ Y
    res = osvd.truncated_svd(S, max_eff, svd_method, rsvd_oversample, rsvd_power, seed,
                             left_only=False,
                             use_full_svd=plssvd_use_small_exact_svd(max_rank, svd_method))
    U = res.U
    s = res.s
    V = res.Vt.T
    store_B = should_store_coefficients(p, m, L, True)
    K0 = max_eff
    C_latent = np.zeros((K0, K0, L))
    W_latent = np.zeros((K0, m, L))
    B = np.zeros((p, m, L)) if store_B else None
    Yfit = np.zeros((n, m, L)) if fit else None
    R2Y = np.zeros(L)
    max_eff = min(max_eff, U.shape[1])
    if V.shape[1] > 0:
        max_eff = min(max_eff, V.shape[1])
    if max_eff < 1:
        raise RuntimeError("plssvd effective rank is < 1 after SVD")
    U = U[:, :max_eff]
    V = V[:, :max_eff]
    T = X @ U
    G = T.T @ T
    for a in range(L):
        mc = min(int(ncomp[a]), max_eff)
        Ga = G[:mc, :mc]
        Da = np.diag(s[:mc])
        C = _solve_likely_sympd(Ga, Da)
        C_latent[:mc, :mc, a] = C
        Wa = C @ V[:, :mc].T
        W_latent[:mc, :, a] = Wa
        if store_B:
            B[:, :, a] = U[:, :mc] @ Wa
        if fit:
            t1 = T[:, :mc] @ Wa
            R2Y[a] = RQ(Y, t1)
            Yfit[:, :, a] = t1 + mY
    out = dict(C_latent=C_latent, W_latent=W_latent, Q=V, Ttrain=T, R=U,
               mX=mX[None, :], vX=vX[None, :], mY=mY[None, :], p=p, m=m,
               ncomp=ncomp, Yfit=Yfit, R2Y=R2Y, singular_values=s,
               pls_method="plssvd", B_stored=store_B, compact_prediction=not store_B)
    if store_B:
        out["B"] = B
    return out


def leading_left_vec_dispatch(S, svd_method, rsvd_oversample, rsvd_power, svds_tol, seed):
    """fastPLS.cpp:161-262 (CPU branches; the CUDA branch follows the CPU recipe)."""
    if S.shape[0] < 1 or S.shape[1] < 1:
        return None
    if svd_method in (osvd.SVD_METHOD_CPU_RSVD, osvd.SVD_METHOD_CUDA_RSVD):
        max_iters = env_int_or("FASTPLS_LEADING_LEFT_MAX_ITERS", max(rsvd_power + 2, 4), 1, 64)
        tol = max(svds_tol, 1e-8)
        omega = gaussian_matrix(S.shape[1], 1, seed + max(rsvd_oversample, 0))
        u = S @ omega[:, 0]
        un = np.linalg.norm(u)
        if not np.isfinite(un) or un <= 0:
            return None
        u = u / un
        for _ in range(max_iters):
            v = S.T @ u
            vn = np.linalg.norm(v)
            if not np.isfinite(vn) or vn <= 0:
                return None
            v = v / vn
            un_ = S @ v
            unn = np.linalg.norm(un_)
            if not np.isfinite(unn) or unn <= 0:
                return None
            un_ = un_ / unn
            resid = np.linalg.norm(un_ - u)
            u = un_
            if resid <= tol:
                break
        return u
    res = osvd.truncated_svd(S, 1, svd_method, rsvd_oversample, rsvd_power, seed,
                             left_only=True, use_full_svd=False)
    if res.U.shape[1] < 1:
        return None
    return res.U[:, 0].copy()


def pls_model2(Xtrain, Ytrain, ncomp, scaling=1, fit=False, svd_method=3,
               rsvd_oversample=10, rsvd_power=1, svds_tol=0.0, seed=1):
    """Classic SIMPLS with a fresh leading vector per component (fastPLS.cpp:2260-2451)."""
    X0 = np.array(Xtrain, dtype=np.float64)
    Ytr = np.array(Ytrain, dtype=np.float64)
    n, p = X0.shape
    m = Ytr.shape[1]
    ncomp = np.atleast_1d(np.asarray(ncomp, dtype=np.int64))
    max_ncomp = int(ncomp.max())
    L = ncomp.size
    X, mX, vX = _center_scale(X0, scaling)
    mY = Ytr.mean(axis=0)
    Y = Ytr - mY
    S = X.T @ Y
    RR = np.zeros((p, max_ncomp))
    PP = np.zeros((p, max_ncomp))
    QQ = np.zeros((m, max_ncomp))
    TT = np.zeros((n, max_ncomp))
    VV = np.zeros((p, max_ncomp))
    store_B = should_store_coefficients(p, m, L, True)
    B = np.zeros((p, m, L)) if store_B else None
    Yfit = np.zeros((n, m, L)) if fit else None
    R2Y = np.zeros(L)
    i_out = 0
    for a in range(max_ncomp):
        rr = leading_left_vec_dispatch(S, svd_method, rsvd_oversample, rsvd_power,
                                       svds_tol, seed + a)
        if rr is None or rr.size != S.shape[0]:
            break
        tt = X @ rr
        tt = tt - tt.mean()
        tnorm = np.sqrt(np.sum(tt * tt))
        tt = tt / tnorm
        rr = rr / tnorm
        pp = X.T @ tt
        qq = Y.T @ tt
        vv = pp.copy()
        if a > 0:
            vv = vv - VV[:, :a] @ (VV[:, :a].T @ pp)
        vv = vv / np.sqrt(np.sum(vv * vv))
        S = S - np.outer(vv, vv @ S)
        RR[:, a] = rr
        TT[:, a] = tt
        PP[:, a] = pp
        QQ[:, a] = qq
        VV[:, a] = vv
        if i_out < L and a == ncomp[i_out] - 1:
            if store_B:
                B[:, :, i_out] = RR[:, :a + 1] @ QQ[:, :a + 1].T
            if fit:
                t1 = TT[:, :a + 1] @ QQ[:, :a + 1].T + mY
                Yfit[:, :, i_out] = t1
                R2Y[i_out] = RQ(Ytr, t1)
            i_out += 1
    out = dict(P=PP, Q=QQ, Ttrain=TT, R=RR, mX=mX[None, :], vX=vX[None, :], mY=mY[None, :],
               p=p, m=m, ncomp=ncomp, Yfit=Yfit, R2Y=R2Y, pls_method="simpls",
               B_stored=store_B, compact_prediction=not store_B)
    if store_B:
        out["B"] = B
    return out


def simpls_fast_refresh(S, warm_start, power_iters, seed):
    """SimplsFastRefreshWorkspace::refresh, CPU branch, k_block = 1
    (fastPLS.cpp:1117-1189 with finalize_left_block_from_bsmall :264-291)."""
    p = S.shape[0]
    Omega = gaussian_matrix(p, 1, seed)
    if warm_start is not None and warm_start.size == p:
        Omega[:, 0] = warm_start
    Yb = Omega
    for _ in range(power_iters):
        Z = S.T @ Yb
        Yb = S @ Z
    Q = osvd.qr_econ_q(Yb)
    if Q.shape[1] < 1:
        return None
    Bsmall = Q.T @ S
    eig_threshold = env_int_or("FASTPLS_GPU_FINALIZE_THRESHOLD", 4, 1, 256)
    if Bsmall.shape[0] >= eig_threshold:
        _, Uhat = osvd.eig_sym_desc(Bsmall @ Bsmall.T)
    else:
        Uhat, _, _ = osvd.svd_econ(Bsmall, left_only=True)
    Ublock = Q @ Uhat
    return Ublock[:, :1]


def pls_model2_fast(Xtrain, Ytrain, ncomp, scaling=1, fit=False, svd_method=4,
                    rsvd_oversample=10, rsvd_power=1, svds_tol=0.0, seed=1):
    """Fast SIMPLS (fastPLS.cpp:2454-2778) with the default option set:
    refresh block 1, FASTPLS_FAST_INC_ITERS=2, no t-centring, no re-orthogonalisation,
    deflation cache on, adaptive policy off, top-1 rSVD off.

    Note (reference behaviour kept): the fitted values only accumulate t q^T at
    the requested ncomp indices (fastPLS.cpp:2648-2653)."""
    X0 = np.array(Xtrain, dtype=np.float64)
    Ytr = np.array(Ytrain, dtype=np.float64)
    n, p = X0.shape
    m = Ytr.shape[1]
    ncomp = np.maximum(np.atleast_1d(np.asarray(ncomp, dtype=np.int64)), 1)
    max_ncomp = int(ncomp.max())
    L = ncomp.size
    X, mX, vX = _center_scale(X0, scaling)
    mY = Ytr.mean(axis=0)
    Y = Ytr - mY
    S = X.T @ Y
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
    use_cache = (max_ncomp >= env_int_or("FASTPLS_FAST_CROSSPROD_MIN_NCOMP", 20, 1, 1024)
                 and p <= n
                 and n >= p * env_int_or("FASTPLS_FAST_CROSSPROD_MIN_N_TO_P_RATIO", 8, 1, 1024)
                 and p <= env_int_or("FASTPLS_FAST_CROSSPROD_MAX_P", 512, 16, 65536))
    XtX = X.T @ X if use_cache else None
    Sxy = S.copy() if use_cache else None
    state = dict(i_out=0, rr_prev=None)

    def append_component(rr, a):
        rr = rr.copy()
        tt = None
        if use_cache:
            pp = XtX @ rr
            tsq = float(rr @ pp)
            if not np.isfinite(tsq) or tsq <= 0:
                return False
            tnorm = np.sqrt(tsq)
            rr /= tnorm
            pp /= tnorm
            qq = Sxy.T @ rr
            if fit:
                tt = X @ rr
        else:
            tt = X @ rr
            tnorm = np.linalg.norm(tt)
            if not np.isfinite(tnorm) or tnorm <= 0:
                return False
            tt = tt / tnorm
            rr /= tnorm
            pp = X.T @ tt
            qq = Y.T @ tt
        state["rr_prev"] = rr
        vv = pp.copy()
        if a > 0:
            Vp = VV[:, :a]
            vv = vv - Vp @ (Vp.T @ pp)
        vnorm = np.linalg.norm(vv)
        if not np.isfinite(vnorm) or vnorm <= 0:
            return False
        vv = vv / vnorm
        vS = vv @ S
        S[:] = S - np.outer(vv, vS)
        RR[:, a] = rr
        QQ[:, a] = qq
        VV[:, a] = vv
        if store_B:
            Bcur[:] = Bcur + np.outer(rr, qq)
        while state["i_out"] < L and a == ncomp[state["i_out"]] - 1:
            io = state["i_out"]
            if store_B:
                B[:, :, io] = Bcur
            if fit:
                Yfit_cur[:] = Yfit_cur + np.outer(tt, qq)
                R2Y[io] = RQ(Y, Yfit_cur)
                Yfit[:, :, io] = Yfit_cur + mY
            state["i_out"] += 1
        return True

    can_incremental = S.shape[0] > 5 and S.shape[1] > 1
    a = 0
    while a < max_ncomp:
        if can_incremental:
            U = simpls_fast_refresh(S, state["rr_prev"], inc_power_iters, seed + a)
            if U is None:
                break
        else:
            res = osvd.truncated_svd(S, 1, svd_method, rsvd_oversample, rsvd_power, seed + a,
                                     left_only=True, use_full_svd=False)
            U = res.U
        if U.shape[1] < 1:
            break
        if not append_component(U[:, 0], a):
            break
        a += 1
    out = dict(P=np.zeros((0, 0)), Q=QQ, Ttrain=np.zeros((0, 0)), R=RR, mX=mX[None, :],
               vX=vX[None, :], mY=mY[None, :], p=p, m=m, ncomp=ncomp, Yfit=Yfit, R2Y=R2Y,
               pls_method="simpls", B_stored=store_B, compact_prediction=not store_B,
               n_components=a)
    if store_B:
        out["B"] = B
    return out


def compact_prediction_weights(model, m, ncomp):
    """fastPLS.cpp:3737-3836: per-slice latent weights (kmax x m x slices)."""
    R = model["R"]
    kmax = R.shape[1]
    L = len(ncomp)
    W = np.zeros((kmax, m, L))
    if model["pls_method"] in ("simpls", "simpls_fast"):
        Q = model["Q"]
        for a in range(L):
            mc = int(ncomp[a])
            W[:mc, :, a] = Q[:, :mc].T
        return W
    if "W_latent" in model:
        return model["W_latent"][:, :, :L].copy()
    C = model["C_latent"]
    Q = model["Q"]
    for a in range(L):
        mc = int(ncomp[a])
        W[:mc, :, a] = C[:mc, :mc, a] @ Q[:, :mc].T
    return W


def pls_predict(model, Xtest, proj=False, use_B=None):
    """pls_predict (fastPLS.cpp:3211-3445).  With ``use_B`` None the route is
    chosen as the reference does (latent when B is absent or >= 256 MB)."""
    Xt = (np.asarray(Xtest, dtype=np.float64) - model["mX"]) / model["vX"]
    mY = model["mY"]
    ncomp = np.atleast_1d(model["ncomp"])
    m = int(model["m"])
    L = ncomp.size
    Ypred = np.zeros((Xt.shape[0], m, L))
    has_B = "B" in model
    if use_B is None:
        latent_min = env_int_or("FASTPLS_PREDICT_LATENT_MIN_B_MB", 256, 0, 1048576)
        b_mb = Xt.shape[1] * m * 8 / (1024.0 * 1024.0)
        prefer_latent = latent_min == 0 or b_mb >= latent_min
        use_B = has_B and not prefer_latent
    if use_B:
        for a in range(L):
            Ypred[:, :, a] = Xt @ model["B"][:, :, a] + mY
    else:
        W = compact_prediction_weights(model, m, ncomp)
        R = model["R"]
        for a in range(L):
            mc = int(ncomp[a])
            Ypred[:, :, a] = (Xt @ R[:, :mc]) @ W[:mc, :, a] + mY
    out = dict(Ypred=Ypred)
    if proj:
        out["Ttest"] = Xt @ model["R"]
    return out


def argmax_first(scores):
    """1-based index of the first maximum per row (arma index_max / strict >)."""
    return np.argmax(scores, axis=1).astype(np.int32) + 1


def pls_predict_classes_compact(model, Xtest, return_scores=False):
    """pls_predict_classes_compact_cpu (fastPLS.cpp:4115-4154).  With
    return_scores the class scores the argmax reads (ntest x m x slices, the
    latent-route Ypred) come back too."""
    pred = pls_predict(model, Xtest, use_B=False)["Ypred"]
    labels = np.stack([argmax_first(pred[:, :, a]) for a in range(pred.shape[2])], axis=1)
    return (labels, pred) if return_scores else labels

"""Row-sharded PLSSVD and fast SIMPLS restated on the CPU (test infrastructure
only: the checker of the library's fpls_pls_model1_rows /
fpls_pls_model2_fast_rows, never a product path).

Each rank holds a block of the rows of X and Y.  `reduce(a)` returns the sum
of the array `a` over all ranks (the all-reduce); with one rank it is the
identity and the fits are pls.pls_model1 / pls.pls_model2_fast (without the
fast-SIMPLS crossprod cache, which the library does not use either).  The
sums are taken in the library's order and with the library's sizes, so a
recording `reduce` gives the sequence of all-reduce sizes the library must
make:

  * 1                 row count
  * p + m             column sums of X (zero when scaling = 3) and of Y
  * p, p              scaling = 2: sums of the centred columns, then their
                      squared deviations (sd with n - 1)
  * p m               S = XᵀY
  PLSSVD (src/fastPLS.cpp:4780-4986):
  * k k               G = TᵀT
  Fast SIMPLS (src/fastPLS.cpp:2454-2778), per component:
  * p + 2 + m         [Xᵀt | tᵀt, Σt | Yᵀt] for the unnormalised t = X r
  fit = True:
  * m                 column sums of the centred Y (the TSS centre)
  * 2 L               PRESS and TSS of every ncomp slice
"""
import numpy as np

from . import svd as osvd
from .pls import (_solve_likely_sympd, env_int_or, plssvd_use_small_exact_svd,
                  should_store_coefficients, simpls_fast_refresh)


def split_rows(n, world):
    """Contiguous row blocks, the first n % world one row longer."""
    base, extra = divmod(n, world)
    out, start = [], 0
    for r in range(world):
        stop = start + base + (1 if r < extra else 0)
        out.append((start, stop))
        start = stop
    return out


def _row_total(n, reduce):
    return int(round(float(reduce(np.array([float(n)]))[0])))


def _center_scale_rows(X, Y, scaling, reduce, n_all):
    """src/fastPLS.cpp:4817-4834 with the column statistics over all ranks."""
    p, m = X.shape[1], Y.shape[1]
    sx = X.sum(axis=0) if scaling < 3 else np.zeros(p)
    buf = reduce(np.concatenate([sx, Y.sum(axis=0)]))
    mX = buf[:p] / n_all if scaling < 3 else np.zeros(p)
    X = X - mX
    mY = buf[p:] / n_all
    Y = Y - mY
    vX = np.ones(p)
    if scaling == 2:
        mu = reduce(X.sum(axis=0)) / n_all
        q = reduce(((X - mu) ** 2).sum(axis=0))
        vX = np.sqrt(q / (n_all - 1))
        X = X / vX
    return X, mX, vX, Y, mY


def _rq_local(y, yp, my):
    return np.array([np.sum((y - yp) ** 2), np.sum((y - my) ** 2)])


def pls_model1_rows(Xtrain, Ytrain, ncomp, reduce, scaling=1, fit=False, svd_method=4,
                    rsvd_oversample=10, rsvd_power=1, svds_tol=0.0, seed=1):
    """PLSSVD over this rank's rows (src/fastPLS.cpp:4780-4986): S and TᵀT are
    summed over the ranks; Ttrain and Yfit are this rank's rows."""
    X = np.array(Xtrain, dtype=np.float64)
    Y = np.array(Ytrain, dtype=np.float64)
    n, p = X.shape
    m = Y.shape[1]
    n_all = _row_total(n, reduce)
    max_rank = min(n_all, p, m)
    ncomp = np.maximum(np.minimum(np.atleast_1d(np.asarray(ncomp, dtype=np.int64)), max_rank), 1)
    L = ncomp.size
    max_eff = min(int(ncomp.max()), max_rank)
    X, mX, vX, Y, mY = _center_scale_rows(X, Y, scaling, reduce, n_all)
    S = reduce(X.T @ Y)
    res = osvd.truncated_svd(S, max_eff, svd_method, rsvd_oversample, rsvd_power, seed,
                             left_only=False,
                             use_full_svd=plssvd_use_small_exact_svd(max_rank, svd_method))
    U, s, V = res.U, res.s, res.Vt.T
    store_B = should_store_coefficients(p, m, L, True)
    K0 = max_eff
    C_latent = np.zeros((K0, K0, L))
    W_latent = np.zeros((K0, m, L))
    B = np.zeros((p, m, L)) if store_B else None
    Yfit = np.zeros((n, m, L)) if fit else None
    max_eff = min(max_eff, U.shape[1], V.shape[1] if V.shape[1] > 0 else max_eff)
    if max_eff < 1:
        raise RuntimeError("plssvd effective rank is < 1 after SVD")
    U = U[:, :max_eff]
    V = V[:, :max_eff]
    T = X @ U
    G = reduce(T.T @ T)
    rq = np.zeros((L, 2))
    my = reduce(Y.sum(axis=0)) / n_all if fit else None
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
            rq[a] = _rq_local(Y, t1, my)
            Yfit[:, :, a] = t1 + mY
    R2Y = np.zeros(L)
    if fit:
        rq = reduce(rq.ravel()).reshape(L, 2)
        R2Y = 1.0 - rq[:, 0] / rq[:, 1]
    out = dict(C_latent=C_latent, W_latent=W_latent, Q=V, Ttrain=T, R=U,
               mX=mX[None, :], vX=vX[None, :], mY=mY[None, :], p=p, m=m,
               ncomp=ncomp, Yfit=Yfit, R2Y=R2Y, singular_values=s, n_total=n_all)
    if store_B:
        out["B"] = B
    return out


def pls_model2_fast_rows(Xtrain, Ytrain, ncomp, reduce, scaling=1, fit=False, seed=1):
    """Fast SIMPLS over this rank's rows (src/fastPLS.cpp:2454-2778, default
    options, no crossprod cache): one all-reduce of [Xᵀt | tᵀt, Σt | Yᵀt] per
    component; Yfit is this rank's rows."""
    X = np.array(Xtrain, dtype=np.float64)
    Y = np.array(Ytrain, dtype=np.float64)
    n, p = X.shape
    m = Y.shape[1]
    n_all = _row_total(n, reduce)
    ncomp = np.maximum(np.atleast_1d(np.asarray(ncomp, dtype=np.int64)), 1)
    max_ncomp = int(ncomp.max())
    L = ncomp.size
    X, mX, vX, Y, mY = _center_scale_rows(X, Y, scaling, reduce, n_all)
    S = reduce(X.T @ Y)
    RR = np.zeros((p, max_ncomp))
    QQ = np.zeros((m, max_ncomp))
    VV = np.zeros((p, max_ncomp))
    store_B = should_store_coefficients(p, m, L, True)
    B = np.zeros((p, m, L)) if store_B else None
    Yfit = np.zeros((n, m, L)) if fit else None
    Yfit_cur = np.zeros((n, m)) if fit else None
    Bcur = np.zeros((p, m))
    rq = np.zeros((L, 2))
    filled = np.zeros(L, dtype=bool)
    inc_power_iters = env_int_or("FASTPLS_FAST_INC_ITERS", 2, 1, 6)
    T_keep = []
    rr_prev = None
    i_out = 0
    a = 0
    can_incremental = p > 5 and m > 1
    while a < max_ncomp:
        if can_incremental:
            Ub = simpls_fast_refresh(S, rr_prev, inc_power_iters, seed + a)
            if Ub is None:
                break
            rr = Ub[:, 0].copy()
        else:
            res = osvd.truncated_svd(S, 1, 4, 10, 1, seed + a, left_only=True, use_full_svd=False)
            if res.U.shape[1] < 1:
                break
            rr = res.U[:, 0].copy()
        tt = X @ rr
        red = reduce(np.concatenate([X.T @ tt, [tt @ tt, tt.sum()], Y.T @ tt]))
        tsq = red[p]
        if not np.isfinite(tsq) or tsq <= 0:
            break
        tnorm = np.sqrt(tsq)
        tt = tt / tnorm
        rr = rr / tnorm
        pp = red[:p] / tnorm
        qq = red[p + 2:] / tnorm
        rr_prev = rr
        vv = pp.copy()
        if a > 0:
            Vp = VV[:, :a]
            vv = vv - Vp @ (Vp.T @ pp)
        vnorm = np.linalg.norm(vv)
        if not np.isfinite(vnorm) or vnorm <= 0:
            break
        vv = vv / vnorm
        S = S - np.outer(vv, vv @ S)
        RR[:, a] = rr
        QQ[:, a] = qq
        VV[:, a] = vv
        T_keep.append(tt)
        if store_B:
            Bcur = Bcur + np.outer(rr, qq)
        while i_out < L and a == ncomp[i_out] - 1:
            if store_B:
                B[:, :, i_out] = Bcur
            filled[i_out] = True
            i_out += 1
        a += 1
    done = a
    R2Y = np.zeros(L)
    if fit:
        # fitted values: t q^T accumulated at the requested ncomp indices
        # (src/fastPLS.cpp:2648-2653), after the loop as the library does
        my = reduce(Y.sum(axis=0)) / n_all
        i_out = 0
        for a in range(done):
            while i_out < L and a == ncomp[i_out] - 1:
                Yfit_cur = Yfit_cur + np.outer(T_keep[a], QQ[:, a])
                rq[i_out] = _rq_local(Y, Yfit_cur, my)
                Yfit[:, :, i_out] = Yfit_cur + mY
                i_out += 1
        rq = reduce(rq.ravel()).reshape(L, 2)
        with np.errstate(invalid="ignore", divide="ignore"):
            R2Y = np.where(filled, 1.0 - rq[:, 0] / rq[:, 1], 0.0)
    out = dict(Q=QQ, R=RR, mX=mX[None, :], vX=vX[None, :], mY=mY[None, :], p=p, m=m,
               ncomp=ncomp, Yfit=Yfit, R2Y=R2Y, n_components=done, n_total=n_all)
    if store_B:
        out["B"] = B
    return out

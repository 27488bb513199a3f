"""Fused PLS + LDA restatement (test infrastructure only).

  * pls_lda_gpu_native    src/fastPLS.cpp:6182-6443
    - PLSSVD (method 1, rSVD) or fast SIMPLS (method 3) fit      :6208-6311
    - R_predict = R / vX rows, offset = mX R_predict             :6318-6335
    - one LDA per distinct ncomp (arma::unique, increasing)      :6337-6371
    - predictions per ncomp slice with its LDA model             :6400-6429

The reference trains the LDA on the fit's training scores (Ttrain) when the
fit returns them, else on X R_predict - offset: the same matrix.
"""
import numpy as np

from . import lda as olda
from . import pls as opls


def pls_lda(Xtrain, Ytrain, y, Xtest, ncomp, n_classes, method=1, scaling=1, fit=False, oversample=10,
            power_iters=1, seed=1, lda_ridge=1e-8):
    X = np.asarray(Xtrain, dtype=np.float64)
    Y = np.asarray(Ytrain, dtype=np.float64)
    nc = np.maximum(np.atleast_1d(np.asarray(ncomp, dtype=np.int64)), 1)
    if method == 1:
        max_rank = min(X.shape[0], X.shape[1], Y.shape[1])
        nc = np.minimum(nc, max_rank)
        model = opls.pls_model1(X, Y, nc, scaling=scaling, fit=fit, svd_method=4,
                                rsvd_oversample=oversample, rsvd_power=power_iters, seed=seed)
    elif method == 3:
        model = opls.pls_model2_fast(X, Y, nc, scaling=scaling, fit=fit, seed=seed)
    else:
        raise ValueError("pls_lda_gpu_native currently supports method=1 (plssvd) or method=3 (simpls)")
    kmax = int(nc.max())
    R = model["R"][:, :kmax]
    vX = np.ravel(model["vX"]).copy()
    vX[~np.isfinite(vX) | (vX == 0)] = 1.0
    Rp = R / vX[:, None]
    off = np.ravel(model["mX"]) @ Rp
    uq = np.unique(nc)
    lda = olda.lda_project_train_prefix(X, Rp, off, y, n_classes, uq, ridge=lda_ridge)
    out = dict(model=model, ncomp=nc, unique_ncomp=uq, lda=lda, R_predict=Rp, R_offset=off)
    if Xtest is not None and len(Xtest):
        Xt = np.asarray(Xtest, dtype=np.float64)
        pred = np.zeros((Xt.shape[0], nc.size), dtype=np.int32)
        scores = []
        for i, kk in enumerate(nc):
            lab, sc = olda.lda_project_predict(Xt, Rp[:, :kk], off[:kk], lda[str(int(kk))], return_scores=True)
            pred[:, i] = lab
            scores.append(sc)
        out["pred_codes"] = pred
        out["pred_scores"] = scores
    return out

"""Candidate-kNN classifier restatement (test infrastructure only).

  * candidate_insert_top                   src/fastPLS.cpp:1249-1267
  * candidate_smoothed_class_knn           src/fastPLS.cpp:1287-1320
  * candidate_knn_predict_native_impl      src/fastPLS.cpp:1322-1467
  * .candidate_row_l2                      R/main.R:657-662
  * .candidate_centroids                   R/main.R:686-698
  * .candidate_score_space                 R/main.R:700-730 (T or T %*% C_k)

The device scorer replaces ``candidate_knn_predict_cuda``, whose kernel keeps at
most 32 neighbour similarities per (row, candidate) (src/lda_cuda_kernels.cu:206);
``knn_cap=32`` reproduces that, ``knn_cap=None`` the uncapped CPU routine.
"""
import math

import numpy as np


def insert_top(scores, index, value, cls):
    """Strict '>' insertion: earlier entries win ties (src/fastPLS.cpp:1249-1267)."""
    for j in range(len(scores)):
        if value > scores[j]:
            scores[j + 1:] = scores[j:-1]
            index[j + 1:] = index[j:-1]
            scores[j] = value
            index[j] = cls
            return


def row_l2(X):
    X = np.asarray(X, dtype=np.float64)
    nr = np.sqrt((X * X).sum(axis=1))
    nr[~np.isfinite(nr) | (nr == 0)] = 1.0
    return X / nr[:, None]


def score_space(T, ncomp, Ck=None):
    kk = min(int(ncomp), T.shape[1])
    T = np.asarray(T, dtype=np.float64)[:, :kk]
    if Ck is None:
        return T
    return T @ np.asarray(Ck, dtype=np.float64)[:kk, :kk]


def centroids(Tn, y_codes, n_classes):
    y = np.asarray(y_codes)
    sums = np.zeros((n_classes, Tn.shape[1]))
    np.add.at(sums, y - 1, Tn)
    counts = np.bincount(y - 1, minlength=n_classes).astype(np.float64)
    counts[counts == 0] = 1.0
    return row_l2(sums / counts[:, None])


def smoothed_class_knn(sims, knn_k, tau):
    if len(sims) == 0:
        return -math.inf
    use_k = max(1, min(knn_k, len(sims)))
    vals = np.sort(sims)[::-1][:use_k]
    if not math.isfinite(tau) or tau <= 0.0:
        total = 0.0
        for v in vals:
            total += v
        return total / use_k
    mx = vals[0]
    if not math.isfinite(mx):
        return mx
    acc = 0.0
    for v in vals:
        acc += math.exp((v - mx) / tau)
    return mx + tau * math.log(acc / use_k)


def candidate_knn_predict(Ttest_norm, Ttrain_norm, y_codes, cents, bias=None, top_k=1,
                          top_m=20, knn_k=3, tau=0.2, alpha=0.5, knn_cap=32):
    Tt = np.asarray(Ttest_norm, dtype=np.float64)
    Tr = np.asarray(Ttrain_norm, dtype=np.float64)
    y = np.asarray(y_codes)
    C = cents.shape[0]
    ntest = Tt.shape[0]
    top_k = max(1, min(top_k, C))
    top_m = max(top_k, min(max(1, top_m), C))
    knn_k = max(1, knn_k)
    if knn_cap is not None:
        knn_k = min(knn_k, knn_cap)
    tau = tau if (math.isfinite(tau) and tau > 0.0) else 0.2
    alpha = alpha if math.isfinite(alpha) else 0.5
    bias = np.zeros(C) if bias is None else np.asarray(bias, dtype=np.float64)
    base = Tt @ cents.T
    rows = [np.nonzero(y == c + 1)[0] for c in range(C)]
    top_index = np.zeros((ntest, top_k), dtype=np.int32)
    top_score = np.full((ntest, top_k), -math.inf)
    for i in range(ntest):
        sc = [-math.inf] * top_m
        ix = [-1] * top_m
        for c in range(C):
            insert_top(sc, ix, base[i, c], c + 1)
        rs = [-math.inf] * top_m
        ri = [-1] * top_m
        for j in range(top_m):
            cls = ix[j]
            if cls < 1 or cls > C:
                continue
            r = rows[cls - 1]
            local = smoothed_class_knn(Tr[r] @ Tt[i], knn_k, tau)
            insert_top(rs, ri, local + alpha * sc[j] + bias[cls - 1], cls)
        top_index[i] = ri[:top_k]
        top_score[i] = rs[:top_k]
    return dict(top_index=top_index, top_score=top_score)

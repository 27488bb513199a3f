"""Cross-validation restatement (test infrastructure only).

  * pls_cv_predict_compiled (folds supplied)   src/fastPLS.cpp:6615-7151
  * fold construction (stratified by the first class of each group)
                                                src/fastPLS.cpp:6720-6769, R/main.R:4011-4040
  * pls.double.cv / optim.pls.cv composition   R/main.R:6586-6760, 6399-6537
  * .cv_best_index (first maximum of accuracy)  R/main.R:6316-6330

Folds are supplied as 0-based integer vectors; the reference draws them from
R's RNG (set.seed + unif_rand), which stays on the R side of the boundary.
"""
import numpy as np

from . import pls as opls


def response_rows(y, idx, n_classes):
    Y = np.zeros((len(idx), n_classes))
    Y[np.arange(len(idx)), np.asarray(y)[idx] - 1] = 1.0
    return Y


def pls_cv_predict_compiled(X, y, fold, ncomp, n_classes, method=3, scaling=1, seed=1,
                            kfold=None):
    """Classification CV with the argmax classifier (classifier 0).
    Returns class_pred (n x L, 1-based), the fold status vector and, for the
    margin checks of the tests, class_score (n x L x m: the scores the argmax
    read; zero for rows of skipped folds)."""
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y)
    fold = np.asarray(fold)
    ncomp = np.maximum(np.atleast_1d(np.asarray(ncomp, dtype=np.int64)), 1)
    L = ncomp.size
    n = X.shape[0]
    kfold = int(fold.max()) + 1 if kfold is None else kfold
    class_pred = np.zeros((n, L), dtype=np.int32)
    class_score = np.zeros((n, L, n_classes))
    status = np.zeros(kfold, dtype=np.int32)
    for f in range(kfold):
        test = np.where(fold == f)[0]
        train = np.where(fold != f)[0]
        if test.size == 0:
            status[f] = 2
            continue
        if train.size == 0:
            class_pred[test, :] = y[test, None]
            status[f] = 3
            continue
        counts = np.bincount(y[train] - 1, minlength=n_classes)
        active = np.where(counts > 0)[0]
        if active.size <= 1:
            class_pred[test, :] = (active[0] + 1) if active.size == 1 else 1
            status[f] = 4
            continue
        Ytr = response_rows(y, train, n_classes)
        if method == 1:
            model = opls.pls_model1(X[train], Ytr, ncomp, scaling=scaling, fit=False,
                                    svd_method=4, seed=seed + f)
        else:
            model = opls.pls_model2_fast(X[train], Ytr, ncomp, scaling=scaling, fit=False,
                                         seed=seed + f)
        lab, sc = opls.pls_predict_classes_compact(model, X[test], return_scores=True)
        class_pred[test, :] = lab
        class_score[test] = np.transpose(sc, (0, 2, 1))
        status[f] = 1
    return dict(class_pred=class_pred, status=status, fold=fold + 1, class_score=class_score)


def accuracy_table(class_pred, y):
    return (np.asarray(class_pred) == np.asarray(y)[:, None]).mean(axis=0)


def best_index(acc):
    acc = np.asarray(acc, dtype=np.float64)
    finite = np.isfinite(acc)
    if not finite.any():
        return 0
    return int(np.argmax(np.where(finite, acc, -np.inf)))


def double_cv(X, y, outer_fold, inner_folds, ncomp, n_classes, scaling=1, seed=1, run=1,
              outer_ids=None):
    """pls.double.cv for one run with method simpls, argmax classifier.

    outer_ids (optional) restricts the loop to those outer folds; the entries of
    the other folds stay zero (the fold-sharded layout of the library's outputs).

    outer_fold: n 0-based outer fold ids.  inner_folds: n x kfold_outer matrix of
    inner fold ids of each row within outer fold o (-1 for the rows of fold o).
    Inner CV seed = seed + 1000 run + (o + 1), fits use + inner fold index;
    outer refit seed = seed + 2000 run + (o + 1) (R/main.R:6697-6730)."""
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y)
    n = X.shape[0]
    ncomp = np.atleast_1d(np.asarray(ncomp, dtype=np.int64))
    K_out = int(outer_fold.max()) + 1
    best = np.zeros(K_out, dtype=np.int32)
    inner_acc = np.zeros((K_out, ncomp.size))
    pred = np.zeros(n, dtype=np.int32)
    m = int(n_classes)
    # class scores behind the labels: inner (kfold_outer x L x n x m, at the
    # rows' own indices) and outer (n x m, at the chosen ncomp)
    inner_pred = np.zeros((K_out, ncomp.size, n), dtype=np.int32)
    inner_score = np.zeros((K_out, ncomp.size, n, m))
    outer_score = np.zeros((n, m))
    for o in (range(K_out) if outer_ids is None else outer_ids):
        test = np.where(outer_fold == o)[0]
        train = np.where(outer_fold != o)[0]
        inner = pls_cv_predict_compiled(X[train], y[train], inner_folds[train, o], ncomp,
                                        n_classes, method=3, scaling=scaling,
                                        seed=seed + 1000 * run + o + 1)
        acc = accuracy_table(inner["class_pred"], y[train])
        inner_acc[o] = acc
        inner_pred[o][:, train] = inner["class_pred"].T
        inner_score[o][:, train, :] = np.transpose(inner["class_score"], (1, 0, 2))
        best[o] = int(ncomp[best_index(acc)])
        Ytr = response_rows(y, train, n_classes)
        model = opls.pls_model2_fast(X[train], Ytr, [best[o]], scaling=scaling,
                                     seed=seed + 2000 * run + o + 1)
        lab, sc = opls.pls_predict_classes_compact(model, X[test], return_scores=True)
        pred[test] = lab[:, 0]
        outer_score[test] = sc[:, :, 0]
    return dict(best_comp=best, inner_accuracy=inner_acc, pred=pred,
                accuracy=float(np.mean(pred == y)), inner_pred=inner_pred,
                inner_score=inner_score, outer_score=outer_score)

"""Cross-validation fold assignment on the host.

Folds are assigned per constraint group and stratified by the class of each
group's first row, as `.make_single_cv_folds` (R/main.R:4011-4040) and the
compiled CV helper (src/fastPLS.cpp:6720-6769) do.  The reference permutes
with R's RNG (set.seed + sample / unif_rand); here the permutation comes from
numpy's PCG64 seeded with the same seed, so fold memberships follow the same
rule but not R's random stream.  Fold ids are 0-based.
"""
import numpy as np


def stratified_group_folds(y, groups, kfold, rng):
    y = np.asarray(y)
    groups = np.asarray(groups)
    ug, first = np.unique(groups, return_index=True)
    gfold = np.zeros(ug.size, dtype=np.int64)
    kfold = min(int(kfold), ug.size)
    first_cls = y[first]
    for cls in np.unique(first_cls):
        idx = np.where(first_cls == cls)[0]
        idx = rng.permutation(idx)
        gfold[idx] = np.arange(idx.size) % kfold
    pos = np.searchsorted(ug, groups)
    return gfold[pos].astype(np.int32)


def double_cv_folds(y, groups, kfold_outer, kfold_inner, seed=1):
    """Outer fold ids (n) and the inner fold id of every row within each outer
    fold (n x kfold_outer; -1 for the rows of that outer fold)."""
    rng = np.random.default_rng(seed)
    y = np.asarray(y)
    groups = np.asarray(groups)
    outer = stratified_group_folds(y, groups, kfold_outer, rng)
    Ko = int(outer.max()) + 1
    inner = -np.ones((y.size, Ko), dtype=np.int32)
    for o in range(Ko):
        tr = np.where(outer != o)[0]
        inner[tr, o] = stratified_group_folds(y[tr], groups[tr], kfold_inner, rng)
    return outer, np.asfortranarray(inner)

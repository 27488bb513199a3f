"""GPU tests of the BF16 split tensor-core GEMM and of the CV grids."""
import numpy as np
import pytest

from oracle import cv as ocv
from oracle import pls as opls
from fastpls_b200 import synthetic
from fastpls_b200.folds import double_cv_folds, stratified_group_folds
from parity_utils import REL_TOL, cv_labels_match, rel_err, slice_score_rel_err

pytestmark = pytest.mark.gpu

# BF16 hi/lo three-product error: ~3 * 2^-17 per product, accumulated in FP32.
SPLIT_REL_TOL = 1e-4


@pytest.mark.parametrize("M,K,N", [(128, 64, 64), (300, 1000, 50), (1000, 3000, 7), (20000, 700, 64),
                                   (257, 129, 130)])
def test_bf16x3_gemm_random(lib, M, K, N):
    rng = np.random.default_rng(M + K + N)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    C = lib.bf16x3_gemm(A, B)
    assert rel_err(C, A @ B) < SPLIT_REL_TOL


def test_bf16x3_gemm_exact_inputs(lib):
    # Inputs exactly representable in BF16 (lo = 0): the only error left is the
    # FP32 accumulation, so a layout or pipeline bug cannot hide in the tolerance.
    rng = np.random.default_rng(3)
    A = rng.integers(-8, 9, size=(777, 1024)).astype(np.float64) / 8.0
    B = rng.integers(-8, 9, size=(1024, 40)).astype(np.float64) / 4.0
    C = lib.bf16x3_gemm(A, B)
    assert np.array_equal(C, A @ B)


def test_bf16x3_gemm_wide_tiles_exact(lib):
    # a product with at least 2048 rows and 512 columns runs on 128 x 128
    # tiles: exact inputs must give the exact product there too, at the N edge
    # (700 columns: a partial last tile) included
    rng = np.random.default_rng(4)
    A = rng.integers(-8, 9, size=(2300, 320)).astype(np.float64) / 8.0
    B = rng.integers(-8, 9, size=(320, 700)).astype(np.float64) / 4.0
    C = lib.bf16x3_gemm(A, B)
    assert np.array_equal(C, A @ B)


@pytest.fixture(scope="module")
def c4_small():
    d = synthetic.c4_omics(seed=2, n=360, p=600, n_informative=20)
    return d


# FP64 CV labels must equal the oracle's wherever its decision margin exceeds
# this fraction of the row's score scale; scores agree to REL_TOL.
MARGIN = 1e-8
# The mixed grid (BF16x3 row Gram, INT8 K products) against FP64: measured class
# score error up to 3.2e-4 of a slice's scores on the 3000 x 20000 grid, so its
# labels are held to FP64's beyond a 1e-3 margin and its scores within 1e-3.
MIXED_TOL = 1e-3


def _inner(r):
    """inner predictions as kfold_outer x L x n (the oracle's layout)."""
    return np.transpose(r["inner_pred"], (2, 1, 0))


def _check_double_cv(got, ref, margin=MARGIN, score_tol=REL_TOL):
    """Double CV outputs against a reference run with scores (oracle or FP64)."""
    ok_in, _, bad_in, _ = cv_labels_match(_inner(got), ref["inner_pred"], ref["inner_score"], margin)
    ok_out, _, bad_out, _ = cv_labels_match(got["pred"], ref["pred"], ref["outer_score"], margin)
    assert ok_in and ok_out, (bad_in, bad_out)
    assert slice_score_rel_err(got["inner_score"], ref["inner_score"]) < score_tol
    assert slice_score_rel_err(got["outer_score"][None], ref["outer_score"][None]) < score_tol
    # accuracies differ only through rows inside the margin
    gap = np.sort(ref["inner_score"], axis=-1)
    unclear = (gap[..., -1] - gap[..., -2]) <= margin * np.abs(gap).max(axis=-1)
    pred_rows = np.abs(ref["inner_score"]).max(axis=-1) > 0
    slack = (unclear & pred_rows).sum(axis=-1).max() / max(1, pred_rows.sum(axis=-1).min())
    assert np.nanmax(np.abs(got["inner_accuracy"] - ref["inner_accuracy"])) <= slack + 1e-12


def _as_ref(r):
    return dict(r, inner_pred=_inner(r))


@pytest.mark.parametrize("batched", [True, False])
def test_cv_predict_fp64_matches_oracle(lib, c4_small, batched):
    d = c4_small
    rng = np.random.default_rng(1)
    fold = stratified_group_folds(d["y"], d["groups"], 5, rng)
    nc = np.arange(1, 11)
    got = lib.cv_predict(d["X"], d["y"], fold, nc, d["n_classes"], seed=7, batched=batched, return_scores=True)
    ref = ocv.pls_cv_predict_compiled(d["X"].astype(np.float64), d["y"], fold, nc, d["n_classes"],
                                      seed=7)
    assert np.array_equal(got["status"], ref["status"])
    assert cv_labels_match(got["class_pred"], ref["class_pred"], ref["class_score"], MARGIN)[0]
    assert slice_score_rel_err(np.transpose(got["class_score"], (1, 0, 2)),
                               np.transpose(ref["class_score"], (1, 0, 2))) < REL_TOL


def test_double_cv_fp64_matches_oracle(lib, c4_small):
    d = c4_small
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=5)
    nc = np.arange(1, 9)
    got = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, batched=True,
                        return_scores=True)
    seq = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, batched=False,
                        return_scores=True)
    ref = ocv.double_cv(d["X"].astype(np.float64), d["y"], outer, inner, nc, d["n_classes"], seed=1)
    for r in (got, seq):
        assert np.array_equal(r["best_comp"], ref["best_comp"])
        _check_double_cv(r, ref)


def test_double_cv_bf16x3_close_to_fp64(lib, c4_small):
    d = c4_small
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=5)
    nc = np.arange(1, 9)
    a = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, precision="fp64",
                      return_scores=True)
    b = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, precision="bf16x3",
                      return_scores=True)
    _check_double_cv(b, _as_ref(a), margin=MIXED_TOL, score_tol=MIXED_TOL)


def test_double_cv_fold_edge_cases(lib):
    # Outer fold 0 leaves only class 1 in its training rows (single-class
    # fallback: every fit of that fold is skipped, its rows get the majority
    # class of the outer training rows, best ncomp = the smallest), and inner
    # fold id 2 of outer fold 1 is never used (that inner fit has no test rows).
    # The other folds follow the oracle's double CV loop.
    rng = np.random.default_rng(11)
    n, p, m = 240, 300, 3
    y = np.repeat(np.arange(1, m + 1), n // m).astype(np.int32)
    X = rng.standard_normal((n, p)) + 0.8 * y[:, None] * (np.arange(p) < 10)[None, :]
    outer = np.where(y > 1, 0, 1 + rng.integers(0, 2, n)).astype(np.int32)
    idx1 = np.where(y == 1)[0]
    outer[idx1[:60]] = 1 + (np.arange(60) % 2)
    outer[idx1[60:]] = 0
    # outer 0 holds classes 2, 3 and 20 rows of class 1 -> its training rows are class 1 only
    Ko, Ki = 3, 4
    inner = np.full((n, Ko), -1, dtype=np.int32)
    for o in range(Ko):
        rows = np.where(outer != o)[0]
        ids = np.arange(rows.size) % Ki
        if o == 1:
            ids[ids == 2] = 3
        inner[rows, o] = ids
    nc = np.arange(1, 6)
    got = lib.double_cv(X, y, outer, inner, nc, m, seed=3, return_scores=True)
    st = got["fit_status"]
    assert np.all(st[0:Ki] == 2) and st[Ko * Ki + 0] == 2
    assert st[1 * Ki + 2] == 2
    tr0 = outer != 0
    fb = np.bincount(y[tr0], minlength=m + 1)[1:].argmax() + 1
    assert got["best_comp"][0] == nc.min()
    assert np.all(got["pred"][outer == 0] == fb)
    Xd = X.astype(np.float64)
    for o in (1, 2):
        test = np.where(outer == o)[0]
        train = np.where(outer != o)[0]
        inn = ocv.pls_cv_predict_compiled(Xd[train], y[train], inner[train, o], nc, m, seed=3 + 1000 + o + 1)
        acc = ocv.accuracy_table(inn["class_pred"], y[train])
        gi = _inner(got)[o][:, train].T
        assert cv_labels_match(gi, inn["class_pred"], inn["class_score"], MARGIN)[0]
        assert slice_score_rel_err(got["inner_score"][o][:, train], np.transpose(inn["class_score"], (1, 0, 2))) \
            < REL_TOL
        best = int(nc[ocv.best_index(acc)])
        assert got["best_comp"][o] == best
        model = opls.pls_model2_fast(Xd[train], ocv.response_rows(y, train, m), [best], seed=3 + 2000 + o + 1)
        ref, sc = opls.pls_predict_classes_compact(model, Xd[test], return_scores=True)
        assert cv_labels_match(got["pred"][test], ref[:, 0], sc[:, :, 0], MARGIN)[0]
        assert rel_err(got["outer_score"][test], sc[:, :, 0]) < REL_TOL


def _same_outputs(a, b, exact=True):
    assert np.array_equal(a["best_comp"], b["best_comp"])
    assert np.array_equal(a["fit_status"], b["fit_status"])
    if exact:
        assert np.array_equal(a["pred"], b["pred"])
        assert np.array_equal(a["inner_accuracy"], b["inner_accuracy"], equal_nan=True)
        assert np.array_equal(a["inner_pred"], b["inner_pred"])
    else:
        # mixed shards: the INT8 product plan depends on the batch width, so the
        # merge equals the full call beyond the mixed grid's margin
        assert cv_labels_match(a["pred"], b["pred"], b["outer_score"], MIXED_TOL)[0]
        assert cv_labels_match(_inner(a), _inner(b), b["inner_score"], MIXED_TOL)[0]


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
@pytest.mark.parametrize("world", [2, 3])
def test_fold_sharded_double_cv_merges_to_the_full_call(lib, c4_small, precision, world):
    # Each shard runs only its outer folds (own fit set, same seeds); merged, the
    # shards give the outputs of one call.  FP64 fits do not depend on which
    # other fits share the batch, so the merge is exact there.
    from fastpls_b200 import fold_shards
    d = c4_small
    outer, inner = double_cv_folds(d["y"], d["groups"], 5, 3, seed=5)
    nc = np.arange(1, 9)
    kw = dict(seed=1, precision=precision, return_inner=True)
    full = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, precision=precision,
                         return_scores=True)
    plan = fold_shards.assign_outer_folds(outer, world)
    parts = [lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], outer_ids=ids, **kw)
             for ids in plan]
    for ids, part in zip(plan, parts):
        rows = np.isin(outer, ids)
        assert np.all(part["pred"][~rows] == 0) and np.all(part["pred"][rows] >= 1)
        assert np.all(part["best_comp"][np.setdiff1d(np.arange(5), ids)] == 0)
    _same_outputs(fold_shards.merge_outputs(parts), full, exact=precision == "fp64")


def test_fold_sharded_resident_and_single_rank_driver(lib, c4_small):
    from fastpls_b200 import fold_shards
    d = c4_small
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=8)
    nc = np.arange(1, 7)
    kw = dict(seed=4, precision="fp64", return_inner=True)
    full = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], **kw)
    one = fold_shards.double_cv_sharded(d["X"], d["y"], outer, inner, nc, d["n_classes"], **kw)
    assert one["plan"] == [[0, 1, 2, 3]]
    _same_outputs(one, full)
    assert one["accuracy"] == full["accuracy"]
    h = lib.x_upload(d["X"])
    try:
        parts = [lib.double_cv_resident(h, d["X"].shape[0], d["y"], outer, inner, nc, d["n_classes"],
                                        outer_ids=ids, **kw) for ids in ([3, 0], [2], [1])]
    finally:
        lib.x_free(h)
    _same_outputs(fold_shards.merge_outputs(parts), full)


def test_fold_sharded_edge_folds(lib):
    # A single-class outer fold and an unused inner fold id, split across shards.
    from fastpls_b200 import fold_shards
    rng = np.random.default_rng(11)
    n, p, m = 240, 300, 3
    y = np.repeat(np.arange(1, m + 1), n // m).astype(np.int32)
    X = rng.standard_normal((n, p)) + 0.8 * y[:, None] * (np.arange(p) < 10)[None, :]
    outer = np.where(y > 1, 0, 1 + rng.integers(0, 2, n)).astype(np.int32)
    idx1 = np.where(y == 1)[0]
    outer[idx1[:60]] = 1 + (np.arange(60) % 2)
    outer[idx1[60:]] = 0
    Ko, Ki = 3, 4
    inner = np.full((n, Ko), -1, dtype=np.int32)
    for o in range(Ko):
        rows = np.where(outer != o)[0]
        ids = np.arange(rows.size) % Ki
        if o == 1:
            ids[ids == 2] = 3
        inner[rows, o] = ids
    nc = np.arange(1, 6)
    full = lib.double_cv(X, y, outer, inner, nc, m, seed=3, return_inner=True)
    parts = [lib.double_cv(X, y, outer, inner, nc, m, seed=3, return_inner=True, outer_ids=ids)
             for ids in ([0], [1, 2])]
    _same_outputs(fold_shards.merge_outputs(parts), full)


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_ncomp_list_order_and_repeats(lib, c4_small, precision):
    # The predictions of a slice depend only on its ncomp value: an unsorted
    # list with repeats gives, slice by slice, the predictions of the sorted
    # list without repeats (same folds, same sketches).
    d = c4_small
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=5)
    mixed = np.array([7, 2, 9, 2, 5])
    base = np.array([2, 5, 7, 9])
    kw = dict(seed=1, precision=precision, return_inner=True)
    a = lib.double_cv(d["X"], d["y"], outer, inner, mixed, d["n_classes"], **kw)
    b = lib.double_cv(d["X"], d["y"], outer, inner, base, d["n_classes"], **kw)
    for s, c in enumerate(mixed):
        t = int(np.where(base == c)[0][0])
        assert np.array_equal(a["inner_pred"][:, s, :], b["inner_pred"][:, t, :])
        assert np.array_equal(a["inner_accuracy"][:, s], b["inner_accuracy"][:, t], equal_nan=True)
    # first maximum: the chosen ncomp follows the list order on ties
    for o in range(a["best_comp"].size):
        acc = a["inner_accuracy"][o]
        assert a["best_comp"][o] == mixed[int(np.nanargmax(acc))]
    rng = np.random.default_rng(2)
    fold = stratified_group_folds(d["y"], d["groups"], 5, rng)
    pa = lib.cv_predict(d["X"], d["y"], fold, mixed, d["n_classes"], seed=3, precision=precision)
    pb = lib.cv_predict(d["X"], d["y"], fold, base, d["n_classes"], seed=3, precision=precision)
    for s, c in enumerate(mixed):
        t = int(np.where(base == c)[0][0])
        assert np.array_equal(np.asarray(pa["class_pred"])[:, s], np.asarray(pb["class_pred"])[:, t])


def test_double_cv_bf16x6_close_to_fp64(lib, c4_small):
    # three BF16 planes and six products in the row Gram: the mixed grid's
    # scores sit closer to FP64 than the two-plane form's
    d = c4_small
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=5)
    nc = np.arange(1, 9)
    kw = dict(seed=1, return_scores=True)
    a = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], precision="fp64", **kw)
    b = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], precision="bf16x6", **kw)
    c = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], precision="bf16x3", **kw)
    _check_double_cv(b, _as_ref(a), margin=MIXED_TOL, score_tol=MIXED_TOL)
    assert slice_score_rel_err(b["inner_score"], a["inner_score"]) < \
        slice_score_rel_err(c["inner_score"], a["inner_score"])

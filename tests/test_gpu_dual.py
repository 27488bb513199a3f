"""The row-space (dual) batched SIMPLS engine against the predictor-space engine
and the oracle on a short, wide predictor block (n <= p / 2)."""
import os

import numpy as np
import pytest

from oracle import cv as ocv
from fastpls_b200 import synthetic
from fastpls_b200.folds import double_cv_folds, stratified_group_folds
from parity_utils import REL_TOL, cv_labels_match, slice_score_rel_err

# FP64 labels equal wherever the reference margin exceeds 1e-8 of the score
# scale; the mixed grid is held to FP64 beyond a 1e-3 margin (its measured class
# score error reaches 3.2e-4 of a slice on the 3000 x 20000 grid).
MARGIN = 1e-8
MIXED_TOL = 1e-3

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wide():
    return synthetic.c4_omics(seed=3, n=300, p=1500, n_informative=25)


def _with_env(value, fn):
    old = os.environ.get("FASTPLS_DUAL")
    os.environ["FASTPLS_DUAL"] = value
    try:
        return fn()
    finally:
        if old is None:
            os.environ.pop("FASTPLS_DUAL")
        else:
            os.environ["FASTPLS_DUAL"] = old


@pytest.mark.parametrize("scaling", [1, 3])
def test_dual_matches_primal_fp64(lib, wide, scaling):
    d = wide
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=5)
    nc = np.arange(1, 13)
    run = lambda: lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], scaling=scaling,
                                seed=1, precision="fp64", return_scores=True)
    dual = _with_env("1", run)
    primal = _with_env("0", run)
    assert np.array_equal(dual["best_comp"], primal["best_comp"])
    assert np.max(np.abs(dual["inner_accuracy"] - primal["inner_accuracy"])) < 1e-12
    assert np.array_equal(dual["pred"], primal["pred"])
    assert cv_labels_match(dual["inner_pred"], primal["inner_pred"],
                           np.transpose(primal["inner_score"], (2, 1, 0, 3)), MARGIN)[0]
    assert slice_score_rel_err(dual["inner_score"], primal["inner_score"]) < REL_TOL


def test_dual_cv_predict_matches_oracle(lib, wide):
    d = wide
    rng = np.random.default_rng(4)
    fold = stratified_group_folds(d["y"], d["groups"], 5, rng)
    nc = np.arange(1, 11)
    got = lib.cv_predict(d["X"], d["y"], fold, nc, d["n_classes"], seed=7, batched=True, return_scores=True)
    ref = ocv.pls_cv_predict_compiled(d["X"].astype(np.float64), d["y"], fold, nc, d["n_classes"],
                                      seed=7)
    assert np.array_equal(got["status"], ref["status"])
    assert cv_labels_match(got["class_pred"], ref["class_pred"], ref["class_score"], MARGIN)[0]
    assert slice_score_rel_err(got["class_score"], ref["class_score"]) < REL_TOL


def test_dual_bf16x3_close_to_fp64(lib, wide):
    d = wide
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=5)
    nc = np.arange(1, 13)
    a = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, precision="fp64",
                      return_scores=True)
    b = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=1, precision="bf16x3",
                      return_scores=True)
    assert np.array_equal(a["best_comp"], b["best_comp"])
    assert cv_labels_match(b["pred"], a["pred"], a["outer_score"], MIXED_TOL)[0]
    assert cv_labels_match(b["inner_pred"], a["inner_pred"], np.transpose(a["inner_score"], (2, 1, 0, 3)),
                           MIXED_TOL)[0]
    assert slice_score_rel_err(b["inner_score"], a["inner_score"]) < MIXED_TOL


@pytest.mark.parametrize("dual", ["1", "0"])
def test_uncentred_predictors_match_oracle(lib, wide, dual):
    # scaling 3: X is not centred but the response still is (fold means)
    d = wide
    rng = np.random.default_rng(6)
    fold = stratified_group_folds(d["y"], d["groups"], 4, rng)
    nc = np.arange(1, 9)
    got = _with_env(dual, lambda: lib.cv_predict(d["X"], d["y"], fold, nc, d["n_classes"], scaling=3,
                                                 seed=3, batched=True, return_scores=True))
    ref = ocv.pls_cv_predict_compiled(d["X"].astype(np.float64), d["y"], fold, nc, d["n_classes"],
                                      scaling=3, seed=3)
    assert cv_labels_match(got["class_pred"], ref["class_pred"], ref["class_score"], MARGIN)[0]
    assert slice_score_rel_err(got["class_score"], ref["class_score"]) < REL_TOL


def test_step_layouts_agree(lib):
    # the 512-thread step layout (default for n <= 4096) against the 256-thread
    # layout with 8 rows per thread (FP64, same folds and sketches)
    d = synthetic.c4_omics(seed=12, n=500, p=1600, n_informative=20)
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=7)
    nc = np.arange(1, 11)

    def run(lay):
        if lay:
            os.environ["FASTPLS_DUAL_STEP"] = lay
        try:
            return lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=2,
                                 precision="fp64", return_scores=True)
        finally:
            os.environ.pop("FASTPLS_DUAL_STEP", None)

    a, b = run(None), run("deep")
    assert np.array_equal(a["best_comp"], b["best_comp"])
    assert cv_labels_match(b["inner_pred"], a["inner_pred"], np.transpose(a["inner_score"], (2, 1, 0, 3)),
                           MARGIN)[0]
    assert slice_score_rel_err(b["inner_score"], a["inner_score"]) < REL_TOL


def test_host_buffer_chunked_upload_matches_resident(lib):
    # The host-buffer call uploads X in column chunks overlapped with the column
    # means, the BF16 split and the row Gram (4096, 3840 and a narrow final chunk
    # of 1064 columns here); its predictions match the resident call's.  The chunked row
    # Gram sums its FP32 segments over different stream-K cuts, so the check is
    # agreement, not bit equality.
    d = synthetic.c4_omics(seed=21, n=400, p=9000, n_informative=25)
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=3)
    nc = np.arange(1, 13)
    host = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=5, precision="bf16x3",
                         return_scores=True)
    h = lib.x_upload(d["X"])
    try:
        res = lib.double_cv_resident(h, d["X"].shape[0], d["y"], outer, inner, nc, d["n_classes"], seed=5,
                                     precision="bf16x3", return_inner=True)
    finally:
        lib.x_free(h)
    assert np.array_equal(host["best_comp"], res["best_comp"])
    assert cv_labels_match(res["inner_pred"], host["inner_pred"], np.transpose(host["inner_score"], (2, 1, 0, 3)),
                           MIXED_TOL)[0]
    assert cv_labels_match(res["pred"], host["pred"], host["outer_score"], MIXED_TOL)[0]
    # FP64 runs the single upload: identical to the resident call
    a = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=5, precision="fp64")
    h = lib.x_upload(d["X"])
    try:
        b = lib.double_cv_resident(h, d["X"].shape[0], d["y"], outer, inner, nc, d["n_classes"], seed=5,
                                   precision="fp64")
    finally:
        lib.x_free(h)
    assert np.array_equal(a["pred"], b["pred"]) and np.array_equal(a["inner_accuracy"], b["inner_accuracy"])


@pytest.mark.parametrize("props", [(0.5, 0.3, 0.2), (0.25, 0.2, 0.2, 0.15, 0.1, 0.1),
                                   (0.2, 0.15, 0.15, 0.1, 0.1, 0.1, 0.1, 0.1)])
@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_merged_refresh_matches_separate_reductions(lib, props, precision):
    # Up to 6 classes a step launch takes the refresh of component a from the
    # Gram-Schmidt reduction of a - 1 (power iterations on S'^T S'); with
    # FASTPLS_DUAL_MERGE=0 every refresh runs its own reductions.  Same folds
    # and sketches: the two agree to rounding (8 classes never merge).
    d = synthetic.c4_omics(seed=14, n=420, p=1500, n_informative=30, props=props)
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=9)
    nc = np.arange(1, 16)

    def run(merge):
        if merge is not None:
            os.environ["FASTPLS_DUAL_MERGE"] = merge
        try:
            return lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], seed=4,
                                 precision=precision, return_scores=True)
        finally:
            os.environ.pop("FASTPLS_DUAL_MERGE", None)

    a, b = run(None), run("0")
    tol = MARGIN if precision == "fp64" else MIXED_TOL
    assert np.array_equal(a["fit_status"], b["fit_status"])
    assert np.array_equal(a["best_comp"], b["best_comp"])
    assert cv_labels_match(a["inner_pred"], b["inner_pred"], np.transpose(b["inner_score"], (2, 1, 0, 3)), tol)[0]
    assert cv_labels_match(a["pred"], b["pred"], b["outer_score"], tol)[0]
    assert slice_score_rel_err(a["inner_score"], b["inner_score"]) < (REL_TOL if precision == "fp64" else MIXED_TOL)
    if len(props) > 6:
        assert np.array_equal(a["inner_pred"], b["inner_pred"])
    if precision == "fp64":
        ref = ocv.double_cv(d["X"].astype(np.float64), d["y"], outer, inner, nc, d["n_classes"], seed=4)
        assert np.array_equal(a["best_comp"], ref["best_comp"])
        assert cv_labels_match(np.transpose(a["inner_pred"], (2, 1, 0)), ref["inner_pred"], ref["inner_score"],
                               MARGIN)[0]
        assert cv_labels_match(a["pred"], ref["pred"], ref["outer_score"], MARGIN)[0]
        assert slice_score_rel_err(a["inner_score"], ref["inner_score"]) < REL_TOL

"""The double-CV autotuner: the first call of a grid shape times the candidate
configurations (Gram tile width, step layout, merged refresh) on its own
inputs and caches the fastest one whose results equal the default
configuration's; tuned calls then give the default's outputs.  The INT8 digit
slices are not searched, so a tuned INT8 grid keeps the INT8 mode's class
scores."""
import numpy as np
import pytest

from fastpls_b200 import synthetic
from fastpls_b200.folds import double_cv_folds

pytestmark = pytest.mark.gpu


@pytest.fixture
def autotune(lib):
    lib.set_autotune(True)
    yield
    lib.set_autotune(False)


@pytest.mark.parametrize("precision", ["fp64", "bf16x3", "int8"])
def test_tuned_grid_reproduces_default(lib, autotune, precision):
    d = synthetic.c4_omics(seed=31, n=330 if precision == "fp64" else 340, p=1400, n_informative=20)
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=2)
    nc = np.arange(1, 9)
    kw = dict(seed=1, precision=precision, return_inner=True)
    tuned = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], **kw)
    code = lib.PREC[precision]
    rep = [r for r in lib.autotune_report()
           if r["n"] == d["X"].shape[0] and r["p"] == d["X"].shape[1] and r["precision"] == code]
    assert len(rep) == 1
    r = rep[0]
    assert r["fits"] == 4 * (3 + 1) and r["kmax"] == 8
    assert len(r["candidates"]) >= 4 and all(c["ms"] > 0 for c in r["candidates"])
    chosen = [c for c in r["candidates"] if c["config"] == r["chosen"]]
    assert chosen and chosen[0]["same_results"]
    again = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], **kw)   # cached: no new entry
    assert len([x for x in lib.autotune_report()
                if x["n"] == d["X"].shape[0] and x["precision"] == code]) == 1
    lib.set_autotune(False)
    default = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], **kw)
    for res in (tuned, again):
        assert np.array_equal(res["best_comp"], default["best_comp"])
        assert np.array_equal(res["pred"], default["pred"])
        assert np.array_equal(res["inner_accuracy"], default["inner_accuracy"])


def test_tuned_int8_grid_keeps_its_class_scores(lib, autotune):
    """Every candidate keeps the INT8 mode's slice count, so the tuned grid's
    class scores stay within the INT8 bound (1e-5 of the slice's scale) of the
    untuned grid's."""
    d = synthetic.c4_omics(seed=33, n=350, p=1500, n_informative=20)
    outer, inner = double_cv_folds(d["y"], d["groups"], 4, 3, seed=3)
    nc = np.arange(1, 9)
    kw = dict(seed=1, precision="int8")
    lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], **kw)   # tunes the shape
    kw["return_scores"] = True
    tuned = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], **kw)   # runs it tuned
    r = [x for x in lib.autotune_report() if x["n"] == 350 and x["precision"] == lib.PREC["int8"]][0]
    assert all(c["config"]["ozaki_slices"] == r["candidates"][0]["config"]["ozaki_slices"]
               for c in r["candidates"])
    lib.set_autotune(False)
    default = lib.double_cv(d["X"], d["y"], outer, inner, nc, d["n_classes"], **kw)
    a, b = tuned["inner_score"], default["inner_score"]
    scale = np.max(np.abs(b), axis=tuple(range(1, b.ndim)), keepdims=True)
    assert np.max(np.abs(a - b) / scale) < 1e-5

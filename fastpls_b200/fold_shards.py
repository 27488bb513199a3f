"""Fold-sharded double cross-validation: the outer folds of ONE pls.double.cv job
split across processes (one per GPU), X replicated on every GPU.

The outer folds of a double CV are independent units (R/main.R:6586-6760 loops
over them; each needs only its own training rows, inner folds and seeds), so a
rank runs the inner CV and the refit of its share of the outer folds through
fpls_double_cv_outer_subset and the ranks exchange nothing but the finished
outputs: best ncomp, inner accuracies, outer predictions, fit status (and, on
request, the inner predictions) -- one all-reduce of a few hundred kB at the
end.  Each call writes only its folds' entries of zero-initialised outputs, so
the element-wise sum over ranks is the merge.  Fold ids keep their seeds
(seed + 1000 run + o + 1 + inner fold; seed + 2000 run + o + 1), so the merged
outputs are those of one unsharded call.
"""
import numpy as np

from . import _lib

OUTPUT_KEYS = ("best_comp", "inner_accuracy", "pred", "fit_status", "inner_pred")


def assign_outer_folds(outer_fold, world, kfold_outer=None):
    """Outer fold ids per rank.  The cost of outer fold o grows with its training
    rows (n - n_o: the inner fits and the refit all run on them), so the folds
    go, largest training set first, to the rank with the least work so far (ties
    to the lower fold id and the lower rank); each rank's list is sorted.  Ranks
    beyond the number of folds get an empty list."""
    of = np.asarray(outer_fold).ravel()
    Ko = int(of.max()) + 1 if kfold_outer is None else int(kfold_outer)
    if world < 1:
        raise ValueError("world must be >= 1")
    sizes = np.bincount(of[(of >= 0) & (of < Ko)], minlength=Ko)
    cost = of.size - sizes
    order = sorted(range(Ko), key=lambda o: (-int(cost[o]), o))
    load = [0] * world
    plan = [[] for _ in range(world)]
    for o in order:
        r = min(range(world), key=lambda k: (load[k], k))
        plan[r].append(o)
        load[r] += int(cost[o])
    return [sorted(p) for p in plan]


def empty_outputs(n, kfold_outer, kfold_inner, L, return_inner=False):
    """Zero outputs of a rank that holds no outer fold (it still joins the merge)."""
    out = dict(best_comp=np.zeros(kfold_outer, dtype=np.int32),
               inner_accuracy=np.zeros((kfold_outer, L), dtype=np.float64, order="F"),
               pred=np.zeros(n, dtype=np.int32),
               fit_status=np.zeros(kfold_outer * kfold_inner + kfold_outer, dtype=np.int32))
    if return_inner:
        out["inner_pred"] = np.zeros((n, L, kfold_outer), dtype=np.int32, order="F")
    return out


def merge_outputs(parts):
    """Merges the outputs of calls over disjoint outer fold lists (in one process)."""
    out = {}
    for k in OUTPUT_KEYS:
        if k in parts[0]:
            acc = np.zeros_like(parts[0][k])
            for p in parts:
                acc += p[k]
            out[k] = acc
    return out


def allreduce_outputs(part, pg=None, device=None):
    """Sum of every rank's partial outputs over the process group `pg` (the
    torch.distributed module after init_process_group, or None for one rank).
    Integers travel as int64 and accuracies as float64; with the nccl backend
    the buffers go through `device` (this rank's GPU)."""
    out = {k: np.array(v, copy=True) for k, v in part.items() if k in OUTPUT_KEYS}
    if pg is None or pg.get_world_size() == 1:
        return out
    import torch
    for k, v in out.items():
        t = torch.from_numpy(np.asarray(v, dtype=np.float64 if v.dtype.kind == "f" else np.int64)
                             .ravel(order="F").copy())
        if device is not None:
            t = t.to(device)
        pg.all_reduce(t, op=pg.ReduceOp.SUM)
        out[k] = t.cpu().numpy().astype(v.dtype).reshape(v.shape, order="F")
    return out


def double_cv_sharded(X, y, outer_fold, inner_fold, ncomp, n_classes, pg=None, device=None,
                      handle=None, n=None, return_inner=False, **kw):
    """One double CV whose outer folds are split over the ranks of `pg`.

    Every rank passes the same arguments (X, or the handle of its own registered
    copy of X with `n` rows) and receives the merged outputs of the whole job,
    plus `plan` (the outer fold ids of each rank) and `accuracy` over all rows.
    The remaining keywords are those of fastpls_b200._lib.double_cv."""
    world = 1 if pg is None else pg.get_world_size()
    rank = 0 if pg is None else pg.get_rank()
    of = np.asarray(outer_fold).ravel()
    inner = np.asarray(inner_fold)
    Ko, Ki = int(of.max()) + 1, int(inner.max()) + 1
    L = np.atleast_1d(ncomp).size
    rows = of.size if handle is None or n is None else int(n)
    plan = assign_outer_folds(of, world, Ko)
    mine = plan[rank]
    if not mine:
        part = empty_outputs(rows, Ko, Ki, L, return_inner)
    elif handle is None:
        part = _lib.double_cv(X, y, of, inner, ncomp, n_classes, return_inner=return_inner,
                              outer_ids=mine if world > 1 else None, **kw)
    else:
        part = _lib.double_cv_resident(handle, rows, y, of, inner, ncomp, n_classes,
                                       return_inner=return_inner,
                                       outer_ids=mine if world > 1 else None, **kw)
    out = allreduce_outputs(part, pg, device)
    yy = np.asarray(y).ravel()
    out["accuracy"] = float(np.mean(out["pred"] == yy))
    out["plan"] = plan
    return out

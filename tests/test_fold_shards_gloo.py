"""Fold-sharded double CV on CPU: the fold assignment, the argument checks of the
outer-subset entry points, and the merge of two gloo ranks' partial outputs
(each rank runs the oracle's double CV over its own outer folds)."""
import os

import numpy as np
import pytest

from fastpls_b200 import fold_shards


def _small_problem(seed=4, n=72, p=40, m=3, Ko=3, Ki=3):
    rng = np.random.default_rng(seed)
    y = (np.arange(n) % m + 1).astype(np.int32)
    X = rng.standard_normal((n, p)) + 0.9 * y[:, None] * (np.arange(p) < 6)[None, :]
    outer = rng.permutation(np.arange(n) % Ko).astype(np.int32)
    inner = np.full((n, Ko), -1, dtype=np.int32)
    for o in range(Ko):
        rows = np.where(outer != o)[0]
        inner[rows, o] = rng.permutation(np.arange(rows.size) % Ki)
    return X, y, outer, np.asfortranarray(inner), m


def test_assign_covers_every_fold_once():
    outer = np.repeat(np.arange(10), [40, 31, 33, 29, 35, 30, 28, 36, 32, 30])
    for world in (1, 2, 3, 4, 8, 10, 12):
        plan = fold_shards.assign_outer_folds(outer, world)
        assert len(plan) == world
        flat = sorted(o for p in plan for o in p)
        assert flat == list(range(10))
        counts = [len(p) for p in plan]
        assert max(counts) - min(counts) <= 1          # near-equal training sizes
        assert all(p == sorted(p) for p in plan)
    assert fold_shards.assign_outer_folds(outer, 12)[10:] == [[], []]
    assert fold_shards.assign_outer_folds(outer, 3) == fold_shards.assign_outer_folds(outer, 3)


def test_assign_balances_uneven_folds():
    # Fold 0 holds most rows, so its training set (and cost) is the smallest.
    outer = np.repeat(np.arange(4), [100, 10, 10, 10])
    plan = fold_shards.assign_outer_folds(outer, 2)
    cost = {o: outer.size - np.sum(outer == o) for o in range(4)}
    loads = [sum(cost[o] for o in p) for p in plan]
    assert max(loads) - min(loads) <= max(cost.values())
    with pytest.raises(ValueError):
        fold_shards.assign_outer_folds(outer, 0)


def test_merge_outputs_of_disjoint_shards():
    a = fold_shards.empty_outputs(6, 3, 2, 2, return_inner=True)
    b = fold_shards.empty_outputs(6, 3, 2, 2, return_inner=True)
    a["best_comp"][0], b["best_comp"][[1, 2]] = 2, [3, 1]
    a["inner_accuracy"][0] = [0.5, np.nan]
    b["inner_accuracy"][1:] = [[0.25, 0.75], [1.0, 0.5]]
    a["pred"][[0, 3]] = [1, 2]
    b["pred"][[1, 2, 4, 5]] = [2, 2, 1, 1]
    a["fit_status"][[0, 1, 6]] = 1
    b["fit_status"][[2, 3, 4, 5, 7, 8]] = [1, 1, 2, 1, 1, 1]
    m = fold_shards.merge_outputs([a, b])
    assert m["best_comp"].tolist() == [2, 3, 1]
    assert np.isnan(m["inner_accuracy"][0, 1]) and m["inner_accuracy"][2, 0] == 1.0
    assert m["pred"].tolist() == [1, 2, 2, 2, 1, 1]
    assert m["fit_status"].tolist() == [1, 1, 1, 1, 2, 1, 1, 1, 1]
    assert m["inner_pred"].shape == (6, 2, 3)


def test_outer_subset_argument_errors():
    # The fold list is checked before the device is touched.
    from fastpls_b200 import _lib
    from fastpls_b200.build import build_library
    build_library()
    _lib.load()
    X, y, outer, inner, m = _small_problem()
    for ids in ([0, 0], [3], [-1], []):
        with pytest.raises(_lib.FastPLSError) as e:
            _lib.double_cv(X, y, outer, inner, [1, 2], m, outer_ids=ids)
        assert e.value.code == 1


def _oracle_part(X, y, outer, inner, nc, m, ids, seed):
    from oracle import cv as ocv
    Ko, Ki = int(outer.max()) + 1, int(inner.max()) + 1
    part = fold_shards.empty_outputs(y.size, Ko, Ki, len(nc))
    if not ids:
        return part
    r = ocv.double_cv(X, y, outer, inner, nc, m, seed=seed, outer_ids=ids)
    for o in ids:
        part["best_comp"][o] = r["best_comp"][o]
        part["inner_accuracy"][o] = r["inner_accuracy"][o]
        part["fit_status"][o * Ki:(o + 1) * Ki] = 1
        part["fit_status"][Ko * Ki + o] = 1
    rows = np.isin(outer, ids)
    part["pred"][rows] = r["pred"][rows]
    return part


def _worker(rank, world, port, q):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        X, y, outer, inner, m = _small_problem()
        nc = [1, 2, 3, 4]
        plan = fold_shards.assign_outer_folds(outer, world)
        part = _oracle_part(X, y, outer, inner, nc, m, plan[rank], seed=2)
        merged = fold_shards.allreduce_outputs(part, dist)
        q.put((rank, plan, {k: v.tolist() for k, v in merged.items()}))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_ranks_merge_to_the_unsharded_double_cv(world):
    import socket
    import torch.multiprocessing as mp
    from oracle import cv as ocv
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=240) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    X, y, outer, inner, m = _small_problem()
    full = ocv.double_cv(X, y, outer, inner, [1, 2, 3, 4], m, seed=2)
    plan = out[0][1]
    if world == 4:
        assert plan[3] == []                             # more ranks than outer folds
    for rank, plan_r, merged in out:
        assert plan_r == plan
        assert merged["best_comp"] == full["best_comp"].tolist()
        assert np.allclose(merged["inner_accuracy"], full["inner_accuracy"], atol=0, rtol=0)
        assert merged["pred"] == full["pred"].tolist()
        assert all(s == 1 for s in merged["fit_status"])

"""Row-sharded fits on the CPU: the row split, the oracle's sharded PLSSVD and
fast SIMPLS against the unsharded oracle (one rank, three threads summing in
rank order, and two gloo processes whose all-reduce is torch.distributed's),
the collective argument check, and the callback's error path."""
import os
import threading

import numpy as np
import pytest

from fastpls_b200 import row_shards
from oracle import pls as opls
from oracle import row_shards as orow

TOL = 1e-9


def _data(seed=3, n=150, p=40, m=4):
    rng = np.random.default_rng(seed)
    L = rng.standard_normal((n, 3))
    X = L @ rng.standard_normal((3, p)) + 0.3 * rng.standard_normal((n, p)) + 2.0
    Y = L @ rng.standard_normal((3, m)) + 0.2 * rng.standard_normal((n, m)) - 1.0
    return X, Y


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _aligned(a, b):
    # singular vectors of S: same up to the sign of each column
    s = np.sign(np.sum(a * b, axis=0))
    s[s == 0] = 1.0
    return a * s


def _check_plssvd(parts, full, blocks):
    for r in parts:
        assert r["n_total"] == full["Ttrain"].shape[0]
        for k in ("C_latent", "W_latent", "mX", "vX", "mY", "R2Y", "singular_values", "B"):
            assert _rel(r[k], full[k]) < TOL, k
        assert _rel(_aligned(r["R"], full["R"]), full["R"]) < TOL
    T = np.vstack([r["Ttrain"] for r in parts])
    assert _rel(_aligned(T, full["Ttrain"]), full["Ttrain"]) < TOL
    if full["Yfit"] is not None:
        assert _rel(np.concatenate([r["Yfit"] for r in parts], axis=0), full["Yfit"]) < TOL


def _check_simpls(parts, full):
    for r in parts:
        assert r["n_components"] == full["n_components"]
        for k in ("R", "Q", "mX", "vX", "mY", "R2Y", "B"):
            assert _rel(r[k], full[k]) < TOL, k
    if full["Yfit"] is not None:
        assert _rel(np.concatenate([r["Yfit"] for r in parts], axis=0), full["Yfit"]) < TOL


def test_split_rows():
    for n, w in [(10, 3), (7, 7), (100, 8), (5, 1)]:
        b = row_shards.split_rows(n, w)
        assert b == orow.split_rows(n, w)
        assert b[0][0] == 0 and b[-1][1] == n
        assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
        sizes = [e - s for s, e in b]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        row_shards.split_rows(4, 0)


@pytest.mark.parametrize("scaling", [1, 2, 3])
def test_one_rank_is_the_unsharded_oracle(scaling):
    X, Y = _data()
    nc = [1, 3, 5]
    full = opls.pls_model1(X, Y, nc, scaling=scaling, fit=True)
    one = orow.pls_model1_rows(X, Y, nc, lambda a: a, scaling=scaling, fit=True)
    _check_plssvd([one], full, [(0, X.shape[0])])
    # p > 512 keeps the unsharded oracle off the crossprod cache (the library never uses it)
    X2, Y2 = _data(seed=5, n=90, p=520, m=3)
    full = opls.pls_model2_fast(X2, Y2, [2, 4, 6], scaling=scaling, fit=True)
    one = orow.pls_model2_fast_rows(X2, Y2, [2, 4, 6], lambda a: a, scaling=scaling, fit=True)
    _check_simpls([one], full)


class _ThreadReducer:
    """Sum over `world` threads in rank order (every thread gets the same bits)."""

    def __init__(self, world):
        self.world = world
        self.slots = [None] * world
        self.barrier = threading.Barrier(world)
        self.sizes = [[] for _ in range(world)]

    def for_rank(self, r):
        def reduce(a):
            a = np.asarray(a, dtype=np.float64)
            self.sizes[r].append(a.size)
            self.slots[r] = a.copy()
            self.barrier.wait()
            total = self.slots[0].copy()
            for k in range(1, self.world):
                total = total + self.slots[k]
            self.barrier.wait()
            return total
        return reduce


def _run_threads(world, fn):
    red = _ThreadReducer(world)
    out = [None] * world
    errs = []

    def body(r):
        try:
            out[r] = fn(r, red.for_rank(r))
        except BaseException as e:   # reported below
            errs.append(e)
            red.barrier.abort()
    th = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(60)
    assert not errs, errs
    return out, red.sizes


@pytest.mark.parametrize("scaling", [1, 2])
def test_three_ranks_match_the_unsharded_oracle(scaling):
    X, Y = _data(seed=7, n=161)
    blocks = orow.split_rows(X.shape[0], 3)
    nc = [2, 4, 4, 6]
    full = opls.pls_model1(X, Y, nc, scaling=scaling, fit=True)
    parts, sizes = _run_threads(3, lambda r, red: orow.pls_model1_rows(
        X[slice(*blocks[r])], Y[slice(*blocks[r])], nc, red, scaling=scaling, fit=True))
    _check_plssvd(parts, full, blocks)
    p, m = X.shape[1], Y.shape[1]
    k = min(max(nc), p, m)
    expect = [1, p + m] + ([p, p] if scaling == 2 else []) + [p * m, k * k, m, 2 * len(nc)]
    assert all(s == expect for s in sizes)

    X2, Y2 = _data(seed=9, n=130, p=530, m=3)
    blocks = orow.split_rows(X2.shape[0], 3)
    full = opls.pls_model2_fast(X2, Y2, [1, 3, 7], scaling=scaling, fit=True)
    parts, sizes = _run_threads(3, lambda r, red: orow.pls_model2_fast_rows(
        X2[slice(*blocks[r])], Y2[slice(*blocks[r])], [1, 3, 7], red, scaling=scaling, fit=True))
    _check_simpls(parts, full)
    p, m = X2.shape[1], Y2.shape[1]
    expect = ([1, p + m] + ([p, p] if scaling == 2 else []) + [p * m] + [p + 2 + m] * 7 + [m, 6])
    assert all(s == expect for s in sizes)


def _gloo_worker(rank, world, port, q):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        def reduce(a):
            t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).copy())
            dist.all_reduce(t)
            return t.numpy()
        X, Y = _data(seed=11, n=121)
        b = orow.split_rows(X.shape[0], world)[rank]
        fit1 = orow.pls_model1_rows(X[b[0]:b[1]], Y[b[0]:b[1]], [2, 5], reduce, fit=True)
        X2, Y2 = _data(seed=12, n=100, p=515, m=3)
        b2 = orow.split_rows(X2.shape[0], world)[rank]
        fit2 = orow.pls_model2_fast_rows(X2[b2[0]:b2[1]], Y2[b2[0]:b2[1]], [3, 5], reduce, fit=True)
        # the collective argument check: equal shapes pass and give the row total
        total = row_shards.check_shards(b[1] - b[0], [40, 4, 2, 2, 5], None)
        # one rank passing other options fails on every rank
        try:
            row_shards.check_shards(b[1] - b[0], [40, 4, 2, 2, 5 + rank], None)
            mismatch = "passed"
        except ValueError:
            mismatch = "raised"
        q.put((rank, fit1, fit2, total, mismatch))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_the_unsharded_oracle():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=240) for _ in range(2)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    X, Y = _data(seed=11, n=121)
    _check_plssvd([o[1] for o in out], opls.pls_model1(X, Y, [2, 5], fit=True), None)
    X2, Y2 = _data(seed=12, n=100, p=515, m=3)
    _check_simpls([o[2] for o in out], opls.pls_model2_fast(X2, Y2, [3, 5], fit=True))
    assert [o[3] for o in out] == [121, 121]
    assert [o[4] for o in out] == ["raised", "raised"]


def test_callback_keeps_the_exception():
    from fastpls_b200 import _lib

    def bad(buf, count, stream):
        raise RuntimeError("peer lost")
    cb, errors = _lib.allreduce_callback(bad)
    assert cb(0, 3, 0, None) == 1
    assert isinstance(errors[0], RuntimeError)
    seen = []
    cb2, errors2 = _lib.allreduce_callback(lambda b, c, s: seen.append((b, c, s)))
    assert cb2(4096, 7, 16, None) == 0 and seen == [(4096, 7, 16)] and not errors2

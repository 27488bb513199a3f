"""Candidate-kNN prediction with the test rows split over ranks, on CPU: the row
blocks, the merge of placed blocks, and gloo ranks that each score their block
with the oracle and merge to the unsharded oracle's top-k lists entry for entry."""
import os

import numpy as np
import pytest

from fastpls_b200 import cknn_shards

KW = dict(top_k=3, top_m=4, knn_k=3, tau=0.2, alpha=0.75)


def _scores(seed=6, n=120, ntest=37, k=6, C=5):
    from oracle import cknn as ok
    rng = np.random.default_rng(seed)
    y = (rng.permutation(np.arange(n) % C) + 1).astype(np.int32)
    proto = rng.standard_normal((C, k))
    Tr = ok.row_l2(proto[y - 1] + 0.4 * rng.standard_normal((n, k)))
    yt = rng.integers(0, C, size=ntest)
    Tt = ok.row_l2(proto[yt] + 0.4 * rng.standard_normal((ntest, k)))
    return Tt, Tr, y, ok.centroids(Tr, y, C)


def test_blocks_cover_every_row_once():
    for ntest in (0, 1, 5, 37, 50000):
        for world in (1, 2, 3, 4, 8):
            b = cknn_shards.assign_test_rows(ntest, world)
            assert len(b) == world and b[0][0] == 0 and b[-1][1] == ntest
            assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
            sizes = [r1 - r0 for r0, r1 in b]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    assert cknn_shards.assign_test_rows(2, 4)[2:] == [(2, 2), (2, 2)]
    with pytest.raises(ValueError):
        cknn_shards.assign_test_rows(5, 0)


def test_placed_blocks_merge_to_the_whole():
    from oracle import cknn as ok
    Tt, Tr, y, cents = _scores()
    full = ok.candidate_knn_predict(Tt, Tr, y, cents, **KW)
    parts = []
    for r0, r1 in cknn_shards.assign_test_rows(Tt.shape[0], 3):
        blk = ok.candidate_knn_predict(Tt[r0:r1], Tr, y, cents, **KW)
        parts.append(cknn_shards.place_block(blk, Tt.shape[0], KW["top_k"], r0))
    for k in cknn_shards.OUTPUT_KEYS:
        merged = sum(p[k] for p in parts)
        assert np.array_equal(merged, full[k])


def _worker(rank, world, port, q):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    from oracle import cknn as ok
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        Tt, Tr, y, cents = _scores()
        out = cknn_shards.candidate_knn_predict_sharded(Tt, Tr, y, cents, pg=dist,
                                                        predict=ok.candidate_knn_predict, **KW)
        q.put((rank, out["bounds"], out["top_index"].tolist(), out["top_score"].tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_merge_to_the_unsharded_prediction(world):
    import socket
    import torch.multiprocessing as mp
    from oracle import cknn as ok
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
    Tt, Tr, y, cents = _scores()
    full = ok.candidate_knn_predict(Tt, Tr, y, cents, **KW)
    for rank, bounds, ti, ts in out:
        assert [tuple(b) for b in bounds] == cknn_shards.assign_test_rows(Tt.shape[0], world)
        assert np.array_equal(np.asarray(ti), full["top_index"])
        assert np.array_equal(np.asarray(ts), full["top_score"])

"""Multi-process replica plumbing of bench.py on CPU: two gloo ranks."""
import os

import pytest


def _worker(rank, world, port, q):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from fastpls_b200 import replicas
    w, r, local, pg = replicas.init_from_env(timeout_s=60)
    try:
        replicas.barrier(pg)
        t = 1.0 + rank              # per-rank "device time"
        tmax = replicas.reduce_max(pg, t)
        q.put((r, w, local, os.environ["FASTPLS_DEVICE"], tmax,
               replicas.job_rate(w, 1500, tmax)))
        replicas.barrier(pg)
    finally:
        pg.destroy_process_group()


def test_two_rank_replicas():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2 for o in out)
    assert [o[3] for o in out] == ["0", "1"]          # each rank pinned to its own GPU
    assert all(o[4] == 2.0 for o in out)              # time = max over ranks
    assert all(abs(o[5] - 2 * 1500 / 2.0) < 1e-9 for o in out)


def test_single_rank_defaults(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from fastpls_b200 import replicas
    w, r, local, pg = replicas.init_from_env()
    assert (w, r, local, pg) == (1, 0, 0, None)
    assert replicas.reduce_max(None, 3.5) == 3.5

"""Row-sharded fits through the C ABI (fpls_pls_model1_rows,
fpls_pls_model2_fast_rows).

* One rank: the sharded fit is the unsharded fit bit for bit, and the library
  calls the all-reduce with exactly the sizes, in the order, of the oracle's
  sharded restatement (oracle/row_shards.py).
* Two processes on one GPU, gloo through host memory (the host waits; no
  kernel waits on another process): the model equals the unsharded fit and
  the oracle's, the per-row outputs are each rank's rows.
* One NCCL rank: the collective is enqueued on the library's stream.
"""
import os

import numpy as np
import pytest

from oracle import pls as opls
from oracle import row_shards as orow

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _data(seed=3, n=600, p=300, m=5):
    rng = np.random.default_rng(seed)
    L = rng.standard_normal((n, 4))
    X = L @ rng.standard_normal((4, p)) + 0.3 * rng.standard_normal((n, p)) + 1.5
    Y = L @ rng.standard_normal((4, m)) + 0.2 * rng.standard_normal((n, m)) - 0.5
    return np.asfortranarray(X), np.asfortranarray(Y)


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _aligned(a, b):
    s = np.sign(np.sum(a * b, axis=0))
    s[s == 0] = 1.0
    return a * s


class _Recorder:
    def __init__(self):
        self.sizes = []

    def __call__(self, buf, count, stream):
        assert buf != 0 and stream != 0
        self.sizes.append(count)


def _oracle_sizes(fn, *a, **k):
    sizes = []

    def red(x):
        x = np.asarray(x, dtype=np.float64)
        sizes.append(x.size)
        return x
    fn(*a, red, **k)
    return sizes


PLSSVD_KEYS = ("C_latent", "W_latent", "Q", "Ttrain", "R", "mX", "vX", "mY", "B", "Yfit", "R2Y",
               "singular_values", "ncomp")
SIMPLS_KEYS = ("R", "Q", "mX", "vX", "mY", "B", "Yfit", "R2Y")


@pytest.mark.parametrize("scaling", [1, 2, 3])
def test_one_rank_is_the_unsharded_fit(lib, scaling):
    X, Y = _data()
    nc = [2, 4, 7]
    rec = _Recorder()
    one = lib.pls_model1(X, Y, nc, scaling=scaling, fit=True, allreduce=rec, n_total=X.shape[0])
    full = lib.pls_model1(X, Y, nc, scaling=scaling, fit=True)
    for k in PLSSVD_KEYS:
        assert np.array_equal(one[k], full[k]), k
    assert rec.sizes == _oracle_sizes(orow.pls_model1_rows, X, Y, nc, scaling=scaling, fit=True)

    rec = _Recorder()
    one = lib.pls_model2_fast(X, Y, nc, scaling=scaling, fit=True, allreduce=rec)
    full = lib.pls_model2_fast(X, Y, nc, scaling=scaling, fit=True)
    assert one["n_components"] == full["n_components"] == 7
    for k in SIMPLS_KEYS:
        assert np.array_equal(one[k], full[k]), k
    assert rec.sizes == _oracle_sizes(orow.pls_model2_fast_rows, X, Y, nc, scaling=scaling, fit=True)


def test_callback_failure_is_an_error(lib):
    X, Y = _data(n=100, p=40)

    def fail(buf, count, stream):
        if count > 100:
            raise RuntimeError("peer lost")
    with pytest.raises(RuntimeError, match="peer lost"):
        lib.pls_model2_fast(X, Y, [3], allreduce=fail)
    ok = lib.pls_model2_fast(X, Y, [3])          # the next call runs normally
    assert ok["n_components"] == 3


def _worker(rank, world, port, backend, q):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist
    from fastpls_b200 import _lib, row_shards
    _lib.load()
    torch.cuda.set_device(0)
    kw = dict(timeout=datetime.timedelta(seconds=60))
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", 0)
    dist.init_process_group(backend, **kw)
    try:
        X, Y = _data(seed=21)
        b = row_shards.split_rows(X.shape[0], world)[rank]
        Xl, Yl = np.asfortranarray(X[b[0]:b[1]]), np.asfortranarray(Y[b[0]:b[1]])
        f1 = row_shards.pls_model1_rows(Xl, Yl, [3, 6], scaling=2, fit=True)
        f2 = row_shards.pls_model2_fast_rows(Xl, Yl, [2, 5, 8], fit=True)
        q.put((rank, {k: np.asarray(v) for k, v in f1.items() if isinstance(v, np.ndarray)},
               {k: np.asarray(v) for k, v in f2.items() if isinstance(v, np.ndarray)}))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _spawn(world, backend):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, backend, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out


def _check_against_unsharded(lib, out):
    X, Y = _data(seed=21)
    full1 = lib.pls_model1(X, Y, [3, 6], scaling=2, fit=True)
    full2 = lib.pls_model2_fast(X, Y, [2, 5, 8], fit=True)
    ref1 = opls.pls_model1(X, Y, [3, 6], scaling=2, fit=True)
    for _, f1, f2 in out:
        for k in ("C_latent", "W_latent", "mX", "vX", "mY", "B", "R2Y", "singular_values"):
            assert _rel(f1[k], full1[k]) < TOL, k
            assert _rel(f1[k], ref1[k]) < TOL, k
        assert _rel(_aligned(f1["R"], full1["R"]), full1["R"]) < TOL
        for k in ("R", "Q", "mX", "vX", "mY", "B", "R2Y"):
            assert _rel(f2[k], full2[k]) < TOL, k
    T = np.vstack([f1["Ttrain"] for _, f1, _ in out])
    assert _rel(_aligned(T, full1["Ttrain"]), full1["Ttrain"]) < TOL
    assert _rel(np.concatenate([f1["Yfit"] for _, f1, _ in out], axis=0), full1["Yfit"]) < TOL
    assert _rel(np.concatenate([f2["Yfit"] for _, _, f2 in out], axis=0), full2["Yfit"]) < TOL


def test_two_ranks_on_one_gpu_match_the_unsharded_fit(lib):
    _check_against_unsharded(lib, _spawn(2, "gloo"))


def test_nccl_allreduce_on_the_library_stream(lib):
    _check_against_unsharded(lib, _spawn(1, "nccl"))

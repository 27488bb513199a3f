"""Row-sharded PLS fits: one process per GPU, each holding a block of the rows
of X and Y (the fits of src/fastPLS.cpp:4780-4986 and 2454-2778 over data
too tall for one GPU, or split for speed).

Every sum over rows is completed by an all-reduce that the library calls
through `fpls_allreduce_fn` on its own stream:
  * the row count, the column sums of X and Y (and, for scaling 2, the sums of
    the centred columns and their squared deviations);
  * S = XᵀY (p x m), once;
  * PLSSVD: G = TᵀT (k x k);
  * fast SIMPLS: per component one buffer [Xᵀt | tᵀt, Σt | Yᵀt] (p + 2 + m);
  * with fit: the TSS centre of Y (m) and the PRESS / TSS sums (2 L).
The model (R, Q, B, C_latent, W_latent, mX, vX, mY, R2Y) comes out the same on
every rank; the per-row outputs (Ttrain, Yfit) are each rank's own rows.

`nccl_allreduce` enqueues `torch.distributed.all_reduce` on the library's
stream (NCCL over NVLink between the GPUs of a node); `host_allreduce` sums
through host memory with any backend (gloo), synchronising the stream.
"""
import numpy as np

from . import _lib


def split_rows(n, world):
    """Contiguous row blocks [(start, stop)] per rank, the first n % world one
    row longer."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(int(n), int(world))
    out, start = [], 0
    for r in range(world):
        stop = start + base + (1 if r < extra else 0)
        out.append((start, stop))
        start = stop
    return out


def _device_tensor(ptr, count):
    import torch

    class _Buf:
        __cuda_array_interface__ = dict(shape=(int(count),), typestr="<f8", data=(int(ptr), False),
                                        version=3, strides=None, stream=None)
    return torch.as_tensor(_Buf())


def nccl_allreduce(group=None):
    """fn(buf, count, stream): NCCL all-reduce (sum) of the library's device
    buffer, enqueued on the library's stream: the collective waits for the
    work already on that stream and the work enqueued after it waits for the
    collective; the host does not block."""
    import torch
    import torch.distributed as dist

    def fn(buf, count, stream):
        t = _device_tensor(buf, count)
        with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=t.device)):
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return fn


def host_allreduce(group=None):
    """fn(buf, count, stream): all-reduce (sum) through host memory with any
    backend (gloo): synchronises the library's stream, reduces a host copy and
    writes it back before returning."""
    import torch
    import torch.distributed as dist

    def fn(buf, count, stream):
        t = _device_tensor(buf, count)
        torch.cuda.ExternalStream(stream, device=t.device).synchronize()
        h = t.cpu()
        dist.all_reduce(h, op=dist.ReduceOp.SUM, group=group)
        t.copy_(h)
        torch.cuda.current_stream(t.device).synchronize()
    return fn


def _agree(values, group, dist, device):
    """The same integers on every rank (min == max), else ValueError on all ranks."""
    import torch
    v = torch.tensor([float(x) for x in values], dtype=torch.float64, device=device)
    lo, hi = v.clone(), v.clone()
    dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX, group=group)
    return bool(torch.equal(lo, hi))


def check_shards(n_local, shape_args, group=None):
    """Collective argument check before a sharded fit (every rank calls it):
    each rank holds at least one row and all ranks pass the same p, m, ncomp
    and options, so no rank can fail alone inside the fit and leave the
    others waiting in an all-reduce.  Returns the total row count."""
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    ok = _agree(shape_args, group, dist, device)
    t = torch.tensor([float(n_local), 1.0 if n_local >= 1 else 0.0], dtype=torch.float64, device=device)
    mn = t.clone()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(mn, op=dist.ReduceOp.MIN, group=group)
    if not ok:
        raise ValueError("row-sharded fit: the ranks passed different shapes or options")
    if mn[1].item() < 1.0:
        raise ValueError("row-sharded fit: every rank needs at least one row")
    return int(round(t[0].item()))


def pls_model1_rows(X, Y, ncomp, allreduce=None, group=None, scaling=1, fit=False, svd_method=4,
                    oversample=10, power_iters=1, svds_tol=0.0, seed=1, store_B=True):
    """PLSSVD over this rank's rows X (n_local x p), Y (n_local x m)
    (fpls_pls_model1_rows).  allreduce defaults to nccl_allreduce(group)."""
    import torch.distributed as dist
    nc = np.atleast_1d(np.asarray(ncomp, dtype=np.int64))
    n_local, p = X.shape
    m = Y.shape[1]
    n_total = check_shards(n_local, [p, m, nc.size, *nc.tolist(), scaling, int(bool(fit)), svd_method,
                                     oversample, power_iters, seed, int(bool(store_B))], group)
    if allreduce is None:
        allreduce = nccl_allreduce(group) if dist.get_backend(group) == "nccl" else host_allreduce(group)
    out = _lib.pls_model1(X, Y, nc, scaling=scaling, fit=fit, svd_method=svd_method, oversample=oversample,
                          power_iters=power_iters, svds_tol=svds_tol, seed=seed, store_B=store_B,
                          allreduce=allreduce, n_total=n_total)
    out["n_total"] = n_total
    return out


def pls_model2_fast_rows(X, Y, ncomp, allreduce=None, group=None, scaling=1, fit=False, seed=1, store_B=True):
    """Fast SIMPLS over this rank's rows (fpls_pls_model2_fast_rows).
    allreduce defaults to nccl_allreduce(group)."""
    import torch.distributed as dist
    nc = np.maximum(np.atleast_1d(np.asarray(ncomp, dtype=np.int64)), 1)
    n_local, p = X.shape
    m = Y.shape[1]
    n_total = check_shards(n_local, [p, m, nc.size, *nc.tolist(), scaling, int(bool(fit)), seed,
                                     int(bool(store_B))], group)
    if allreduce is None:
        allreduce = nccl_allreduce(group) if dist.get_backend(group) == "nccl" else host_allreduce(group)
    out = _lib.pls_model2_fast(X, Y, nc, scaling=scaling, fit=fit, seed=seed, store_B=store_B,
                               allreduce=allreduce)
    out["n_total"] = n_total
    return out

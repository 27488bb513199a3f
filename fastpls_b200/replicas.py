"""Host plumbing for N independent double-CV replicas, one process per GPU.

`bench.py --gpus N` runs N weak-scaled replicas: rank r uses device LOCAL_RANK
and its own seeded workload, the ranks meet only at barriers, and the job's time
is the maximum of the ranks' device times (gloo all-reduce of one float; no
data-path collective).  Splitting ONE double CV across the ranks by outer fold
is fold_shards.double_cv_sharded.
"""
import datetime
import os


def init_from_env(timeout_s=300):
    """Reads WORLD_SIZE / RANK / LOCAL_RANK, pins the library to the rank's GPU
    (FASTPLS_DEVICE) and joins a gloo group when there is more than one rank."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    os.environ["FASTPLS_DEVICE"] = str(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, v):
    """Maximum of a float over the ranks (the job's time)."""
    if pg is None:
        return float(v)
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def job_rate(world, units_per_rank, max_seconds):
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / max_seconds

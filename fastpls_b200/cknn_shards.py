"""Candidate-kNN prediction with the test rows split across processes (one per
GPU), the training scores (or the training matrix) replicated on every GPU.

Every test row of the candidate-kNN classifier is scored on its own: its
candidate classes, their nearest training rows and the smoothed class score
read only that row and the (shared) training scores and centroids
(src/fastPLS.cpp:1322-1467, lda_cuda_kernels.cu:180-243 score one test row per
thread block).  So a rank predicts one contiguous block of the test rows and
the ranks exchange nothing but the finished top-k lists: each rank writes its
block into zero outputs of the full size and one all-reduce (a sum) merges
them.  The merged lists are those of one unsharded call, entry for entry.
"""
import numpy as np

from . import _lib

OUTPUT_KEYS = ("top_index", "top_score")


def assign_test_rows(ntest, world):
    """Contiguous blocks [r0, r1) of the test rows per rank: sizes differ by at
    most one, the larger blocks first; ranks beyond ntest get empty blocks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if ntest < 0:
        raise ValueError("ntest must be >= 0")
    base, extra = divmod(int(ntest), int(world))
    bounds, r0 = [], 0
    for r in range(world):
        r1 = r0 + base + (1 if r < extra else 0)
        bounds.append((r0, r1))
        r0 = r1
    return bounds


def empty_outputs(ntest, top_k):
    return dict(top_index=np.zeros((ntest, top_k), dtype=np.int32, order="F"),
                top_score=np.zeros((ntest, top_k), dtype=np.float64, order="F"))


def place_block(part, ntest, top_k, r0):
    """The full-size outputs holding one rank's block at rows r0.. (zeros elsewhere)."""
    out = empty_outputs(ntest, top_k)
    for k in OUTPUT_KEYS:
        blk = np.asarray(part[k])
        out[k][r0:r0 + blk.shape[0], :blk.shape[1]] = blk
    return out


def allreduce_outputs(part, pg=None, device=None):
    """Sum of every rank's full-size outputs over the process group `pg` (the
    torch.distributed module after init_process_group, or None for one rank);
    with the nccl backend the buffers go through `device`."""
    out = {k: np.array(part[k], copy=True) for k in OUTPUT_KEYS}
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


def _sharded(ntest, top_k, predict_block, pg, device):
    world = 1 if pg is None else pg.get_world_size()
    rank = 0 if pg is None else pg.get_rank()
    bounds = assign_test_rows(ntest, world)
    r0, r1 = bounds[rank]
    if r1 > r0:
        part = place_block(predict_block(r0, r1), ntest, top_k, r0)
    else:
        part = empty_outputs(ntest, top_k)
    out = allreduce_outputs(part, pg, device)
    out["bounds"] = bounds
    return out


def candidate_knn_predict_sharded(Ttest_norm, Ttrain_norm, y_codes, centroids, pg=None, device=None,
                                  predict=None, **kw):
    """candidate_knn_predict over the ranks of `pg`: every rank passes the same
    arguments and receives the merged top-k lists of all test rows (plus
    `bounds`, the row block of each rank).  `predict` is the per-block scorer
    (default: the library's fpls_candidate_knn_predict) with the keywords of
    fastpls_b200._lib.candidate_knn_predict."""
    fn = predict or _lib.candidate_knn_predict
    Tt = np.asarray(Ttest_norm)
    ncls = np.asarray(centroids).shape[0]
    top_k = max(1, min(int(kw.get("top_k", 1)), ncls))

    def block(r0, r1):
        return fn(np.asfortranarray(Tt[r0:r1]), Ttrain_norm, y_codes, centroids, **kw)
    return _sharded(Tt.shape[0], top_k, block, pg, device)


def label_aware_cknn_sharded(Xtrain, y_codes, m, Xtest, ncomp, pg=None, device=None, **kw):
    """label_aware_cknn over the ranks of `pg`: every rank fits the label-aware
    PLSSVD on the whole training matrix (the fit is replicated, not split) and
    predicts its block of the test rows; the merged top-k lists come back on
    every rank.  Keywords are those of fastpls_b200._lib.label_aware_cknn."""
    Xte = np.asarray(Xtest)
    top_k = max(1, min(int(kw.get("top_k", 5)), int(m)))

    def block(r0, r1):
        return _lib.label_aware_cknn(Xtrain, y_codes, m, np.asfortranarray(Xte[r0:r1]), ncomp, **kw)
    return _sharded(Xte.shape[0], top_k, block, pg, device)

"""Comparison helpers for the parity tests (FP64 tolerances of the drop-in)."""
import numpy as np

# Tolerances of the FP64 drop-in against the CPU oracle.
REL_TOL = 1e-9          # coefficients and predictions, relative Frobenius error
ANGLE_TOL = 1e-8        # largest principal angle between subspaces (radians)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    if nb == 0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)


def sign_align(A, B):
    """Flip columns of A to match the sign of B column by column."""
    A = np.array(A, dtype=np.float64, copy=True)
    for j in range(A.shape[1]):
        if np.dot(A[:, j], B[:, j]) < 0:
            A[:, j] = -A[:, j]
    return A


def subspace_angle(A, B):
    """Largest principal angle between span(A) and span(B)."""
    qa, _ = np.linalg.qr(np.asarray(A, dtype=np.float64))
    qb, _ = np.linalg.qr(np.asarray(B, dtype=np.float64))
    s = np.linalg.svd(qa.T @ qb, compute_uv=False)
    s = np.clip(s, -1.0, 1.0)
    # sin of the largest angle computed stably
    proj = qb - qa @ (qa.T @ qb)
    return float(np.arcsin(min(1.0, np.linalg.norm(proj, 2))))


def labels_match_beyond_margin(lab_a, lab_b, scores_ref, margin=1e-7):
    """Labels must agree wherever the reference decision margin exceeds `margin`
    (relative to the score scale)."""
    lab_a = np.asarray(lab_a).ravel()
    lab_b = np.asarray(lab_b).ravel()
    s = np.sort(np.asarray(scores_ref), axis=1)
    gap = s[:, -1] - s[:, -2] if s.shape[1] > 1 else np.full(s.shape[0], np.inf)
    scale = np.maximum(np.abs(s).max(axis=1), 1e-300)
    clear = gap > margin * scale
    return bool(np.all(lab_a[clear] == lab_b[clear])), int(clear.sum())


def score_margins(scores):
    """Per row: gap between the two largest class scores, and the score scale
    (largest absolute score).  scores: (..., m) with classes last."""
    s = np.sort(np.asarray(scores, dtype=np.float64), axis=-1)
    gap = s[..., -1] - s[..., -2] if s.shape[-1] > 1 else np.full(s.shape[:-1], np.inf)
    scale = np.abs(s).max(axis=-1)
    return gap, scale


def cv_labels_match(pred, pred_ref, score_ref, margin):
    """CV labels against the oracle's: identical wherever the oracle's decision
    margin (top-two score gap) exceeds `margin` times the row's score scale.
    Rows whose reference scores are all zero took a fallback class (or were
    not predicted) and must match exactly.  pred, pred_ref: (...) labels;
    score_ref: (..., m).  Returns (ok, rows checked by margin, mismatching
    rows beyond margin, all-zero rows that differ)."""
    pred = np.asarray(pred).ravel()
    pred_ref = np.asarray(pred_ref).ravel()
    sc = np.asarray(score_ref, dtype=np.float64)
    sc = sc.reshape(-1, sc.shape[-1])
    gap, scale = score_margins(sc)
    fallback = scale == 0
    clear = (~fallback) & (gap > margin * scale)
    bad_clear = int(np.sum(pred[clear] != pred_ref[clear]))
    bad_fallback = int(np.sum(pred[fallback] != pred_ref[fallback]))
    return bad_clear == 0 and bad_fallback == 0, int(clear.sum()), bad_clear, bad_fallback


def slice_score_rel_err(score, score_ref):
    """Largest relative Frobenius error of the class scores over the leading
    slices (e.g. outer fold x ncomp), rows that were not predicted excluded."""
    a = np.asarray(score, dtype=np.float64)
    b = np.asarray(score_ref, dtype=np.float64)
    a = a.reshape(-1, a.shape[-2], a.shape[-1])
    b = b.reshape(-1, b.shape[-2], b.shape[-1])
    worst = 0.0
    for k in range(a.shape[0]):
        rows = np.abs(b[k]).max(axis=1) > 0
        if not rows.any():
            continue
        nb = np.linalg.norm(b[k][rows])
        worst = max(worst, float(np.linalg.norm(a[k][rows] - b[k][rows]) / nb))
    return worst

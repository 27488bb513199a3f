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

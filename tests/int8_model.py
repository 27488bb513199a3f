"""CPU model of the INT8 digit-plane (Ozaki scheme) product used by the
tensor-core kernel: power-of-two row scales, signed 7-bit digits taken exactly
in FP64, exact integer products of the plane pairs with s + t <= S + 1 summed
per level, levels combined in FP64 from the smallest.  Test infrastructure."""
import numpy as np


def split_digits(rows, slices):
    """Digit planes (slices x rows x k, int64) and scales 2^e of the rows."""
    rows = np.asarray(rows, dtype=np.float64)
    m = np.max(np.abs(rows), axis=1) if rows.shape[1] else np.zeros(rows.shape[0])
    e = np.where(m > 0, np.frexp(m)[1], 0)
    a = rows * np.ldexp(1.0, -e)[:, None]
    planes = []
    for _ in range(slices):
        a = a * 128.0
        d = np.trunc(a)
        a = a - d
        planes.append(d.astype(np.int64))
    return planes, np.ldexp(1.0, e)


def product(A, B, slices):
    """A (M x K) @ B (K x N) as the kernel forms it (up to FP64 rounding)."""
    DA, sa = split_digits(A, slices)
    DB, sb = split_digits(np.asarray(B).T, slices)
    M, N = DA[0].shape[0], DB[0].shape[0]
    levels = [np.zeros((M, N), dtype=np.int64) for _ in range(slices)]
    for s in range(slices):
        for t in range(slices - s):
            levels[s + t] += DA[s] @ DB[t].T
    acc = np.zeros((M, N))
    for lv in reversed(range(slices)):
        acc += levels[lv].astype(np.float64) * 2.0 ** (-7 * (lv + 2))
    return acc * sa[:, None] * sb[None, :]


def error_bound(A, B, slices):
    """Entrywise bound 3 K 2^(eA_i + eB_j - 7 S) on |product - A @ B| (plus the
    FP64 rounding of the exact product, K 2^-52 sum |A||B|)."""
    _, sa = split_digits(A, 1)
    _, sb = split_digits(np.asarray(B).T, 1)
    K = np.asarray(A).shape[1]
    trunc = 3.0 * K * np.outer(sa, sb) * 2.0 ** (-7 * slices)
    return trunc + K * 2.0 ** -52 * (np.abs(A) @ np.abs(B))

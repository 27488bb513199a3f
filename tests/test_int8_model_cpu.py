"""The digit-plane model behind the INT8 tensor-core product, on the CPU:
digits are exact and bounded, and the product stays inside its stated bound."""
import numpy as np
import pytest

import int8_model as im


@pytest.mark.parametrize("slices", [4, 5, 6, 7])
def test_digits_reconstruct_rows(slices):
    rng = np.random.default_rng(slices)
    X = rng.standard_normal((40, 300)) * np.logspace(-6, 6, 40)[:, None]
    X[3] = 0.0
    D, sc = im.split_digits(X, slices)
    assert all(np.abs(d).max() <= 127 for d in D)
    rec = sum(d * 2.0 ** (-7 * (s + 1)) for s, d in enumerate(D)) * sc[:, None]
    # truncation residual below one unit of the last digit
    assert np.all(np.abs(rec - X) <= sc[:, None] * 2.0 ** (-7 * slices))
    assert np.all(rec[3] == 0.0)


@pytest.mark.parametrize("slices", [4, 5, 6, 7])
def test_product_within_bound(slices):
    rng = np.random.default_rng(10 + slices)
    A = rng.standard_normal((70, 500)) * np.logspace(-3, 3, 70)[:, None]
    B = rng.standard_normal((500, 30)) * np.logspace(2, -2, 30)[None, :]
    C = im.product(A, B, slices)
    assert np.all(np.abs(C - A @ B) <= im.error_bound(A, B, slices))


def test_integer_inputs_exact():
    # small integers need one digit: every slice count reproduces the product
    rng = np.random.default_rng(5)
    A = rng.integers(-100, 101, size=(50, 257)).astype(np.float64)
    B = rng.integers(-100, 101, size=(257, 20)).astype(np.float64)
    for slices in (4, 7):
        assert np.array_equal(im.product(A, B, slices), A @ B)


def test_level_sums_fit_int32():
    # the kernel's per-segment level accumulator: at most S pairs of at most
    # 64 * 128 terms of 127^2 each
    for s in range(4, 8):
        assert s * 64 * 128 * 127 ** 2 < 2 ** 31

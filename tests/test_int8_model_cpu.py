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


@pytest.mark.parametrize("slices", [4, 5, 6, 7])
def test_digit_fields_equal_iterated_digits(slices):
    """The split kernels take each entry's digits as the 7-bit fields of one
    truncation q = trunc(a 2^(7S)) (a = x 2^-e, |a| < 1), most significant
    first, with the sign of a.  They equal the S rounds of "times 128, take
    the integer part" of the model, entry for entry."""
    rng = np.random.default_rng(slices)
    rows = rng.standard_normal((40, 300)) * np.exp(rng.normal(0.0, 4.0, size=(40, 1)))
    rows[3, :7] = [0.0, -0.0, 1e-300, -1e-300, 2.0 ** -60, -(1.0 - 2.0 ** -53), 5e-324]
    rows[4] = np.nextafter(1.0, 0.0) * np.sign(rng.standard_normal(300))
    planes, scale = im.split_digits(rows, slices)
    a = rows / scale[:, None]
    q = np.trunc(a * 2.0 ** (7 * slices)).astype(np.int64)
    mag, sign = np.abs(q), np.where(q < 0, -1, 1)
    for s in range(slices):
        field = sign * ((mag >> (7 * (slices - 1 - s))) & 127)
        assert np.array_equal(field, planes[s]), f"plane {s}"

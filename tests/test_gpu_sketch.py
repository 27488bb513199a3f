"""The device-drawn Gaussian sketch against the host libstdc++ stream."""
import numpy as np
import pytest

from oracle.rng import gaussian_matrix

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,cols,seed", [(1, 1, 1), (7, 3, 11), (20001, 1, 5), (1000, 110, 1),
                                            (613, 7, 4294967295)])
def test_sketch_matches_host_stream(lib, rows, cols, seed):
    got = lib.gaussian_sketch(rows, cols, seed)
    ref = gaussian_matrix(rows, cols, seed)
    assert got.shape == ref.shape
    same = np.mean(got == ref)
    # identical except where the device log rounds differently in the last place
    assert same > 0.99
    assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)) < 4 * np.finfo(float).eps

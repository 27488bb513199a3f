"""Matrix arguments already in HBM: the entry points that copy X, Y, Xtest, the
response or the filtered X whole accept device pointers (unified addressing
tells them from host pointers) and give the results of the host-buffer calls.
The device buffers come from torch, standing in for a caller that keeps its
data on the GPU: same results bit for bit."""
import numpy as np
import pytest

from fastpls_b200 import synthetic
from parity_utils import rel_err

pytestmark = pytest.mark.gpu

TOL = 0.0


def _dev(torch, a):
    """Column-major device copy of a 2-D host array (transpose of a contiguous tensor)."""
    a = np.asarray(a, dtype=np.float64)
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().T


def test_fits_and_predictions_from_device_buffers(lib):
    torch = pytest.importorskip("torch")
    d = synthetic.c5_lowrank(seed=6, n=600, p=300, q=80, rank=6, n_test=100)
    X, Y, Xt = (d[k].astype(np.float64) for k in ("Xtrain", "Ytrain", "Xtest"))
    Xd, Yd, Xtd = _dev(torch, X), _dev(torch, Y), _dev(torch, Xt)
    torch.cuda.synchronize()
    host = lib.pls_model2_fast(X, Y, [3, 7], seed=2)
    dev = lib.pls_model2_fast(Xd, Yd, [3, 7], seed=2)
    assert rel_err(dev["B"], host["B"]) <= TOL and rel_err(dev["R"], host["R"]) <= TOL
    m1h = lib.pls_model1(X, Y, [4], svd_method=4, seed=3)
    m1d = lib.pls_model1(Xd, Yd, [4], svd_method=4, seed=3)
    assert rel_err(m1d["B"], m1h["B"]) <= TOL
    ph = lib.predict_lowrank(host, Xt)["Ypred"]
    pd = lib.predict_lowrank(host, Xtd)["Ypred"]
    assert rel_err(pd, ph) <= TOL
    # filtered X written straight into a device buffer
    out = torch.empty((X.shape[1], X.shape[0]), dtype=torch.float64, device="cuda").T
    fh = lib.opls_filter(X, Y, 2)
    fd = lib.opls_filter(Xd, Yd, 2, out=out)
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), fh["X"]) <= TOL
    assert rel_err(fd["W_orth"], fh["W_orth"]) <= TOL
    outt = torch.empty((Xt.shape[1], Xt.shape[0]), dtype=torch.float64, device="cuda").T
    lib.opls_apply_filter(Xtd, fd["mX"], fd["vX"], fd["W_orth"], fd["P_orth"], out=outt)
    torch.cuda.synchronize()
    assert rel_err(outt.cpu().numpy(),
                   lib.opls_apply_filter(Xt, fh["mX"], fh["vX"], fh["W_orth"], fh["P_orth"])) <= TOL
    G = np.random.default_rng(1).standard_normal((Y.shape[1], 10)) / np.sqrt(10.0)
    eh = lib.gaussian_y_encode(Y, G)
    ed = lib.gaussian_y_encode(Yd, G)
    assert rel_err(ed["Z"], eh["Z"]) <= TOL and rel_err(ed["decoder"], eh["decoder"]) <= TOL
    assert rel_err(lib.predict_lowrank(dev, Xtd)["Ypred"], ph) <= TOL


def test_device_matrix_layout_is_checked(lib):
    torch = pytest.importorskip("torch")
    X = torch.zeros((50, 40), dtype=torch.float64, device="cuda")  # row-major: not column-major
    with pytest.raises(ValueError):
        lib.DeviceMatrix(X)
    with pytest.raises(ValueError):
        lib.DeviceMatrix(torch.zeros((50, 40), dtype=torch.float32, device="cuda").T)


def test_resident_matrices_keep_a_pipeline_on_the_device(lib):
    # X sent once (fpls_x_upload), the filtered X written to a resident matrix
    # (fpls_x_alloc) and fed to the fit by its device pointer
    d = synthetic.c5_lowrank(seed=7, n=500, p=240, q=60, rank=5, n_test=50)
    X, Y = d["Xtrain"].astype(np.float64), d["Ytrain"].astype(np.float64)
    rx, ry = lib.x_resident(X), lib.x_resident(Y)
    rf = lib.x_alloc(*X.shape)
    try:
        fd = lib.opls_filter(rx, ry, 2, out=rf)
        fh = lib.opls_filter(X, Y, 2)
        assert rel_err(rf.download(), fh["X"]) <= TOL
        md = lib.pls_model2_fast(rf, ry, [4], seed=1)
        mh = lib.pls_model2_fast(fh["X"], Y, [4], seed=1)
        assert rel_err(md["B"], mh["B"]) <= TOL
        assert fd["north"] == 2
    finally:
        for r in (rx, ry, rf):
            r.free()

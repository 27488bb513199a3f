"""fpls_bf16x3_gemm_noalloc: the allocation-free tensor-core GEMM entry point.

It serves callers that cannot call cudaMalloc themselves (for instance code
running inside another runtime's fixed device-memory pool): they pass device
buffers they already own and the library uses only its fixed, load-time device
array for temporaries.  This test gives it device buffers (allocated here by
torch, standing in for such a host), calls it twice in a row through the C ABI
and checks both results against the ordinary allocating entry point
fpls_bf16x3_gemm, within the split-precision tolerance of the other tests.

The file name sorts last so a run that stops at the first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

from parity_utils import rel_err

pytestmark = pytest.mark.gpu

SPLIT_REL_TOL = 1e-4  # same bound as the allocating split GEMM tests


def _call_noalloc(lib_mod, A_dev, M, K, B_dev, N, C_dev):
    err = ctypes.create_string_buffer(512)
    rc = lib_mod.load().fpls_bf16x3_gemm_noalloc(
        ctypes.c_void_p(A_dev), M, K, ctypes.c_void_p(B_dev), N, ctypes.c_void_p(C_dev), err,
        ctypes.sizeof(err))
    return rc, err.value.decode(errors="replace")


def test_noalloc_gemm_matches_allocating_entry_point(lib):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    rng = np.random.default_rng(2024)
    # A large, block-aligned shape first, then a smaller one whose K is not a
    # multiple of the 64-wide K-block: the second call reuses scratch that still
    # holds the first call's planes and partials, so stale contents or padding
    # that is not rewritten would show up in its result.
    for M, K, N in ((700, 1536, 48), (333, 1000, 17)):
        A = rng.standard_normal((M, K))
        B = rng.standard_normal((K, N))
        # Column-major device copies (a transposed contiguous tensor is column-major).
        A_dev = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
        B_dev = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
        C_dev = torch.full((N, M), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        dev_before = torch.cuda.current_device()
        rc, msg = _call_noalloc(lib, A_dev.data_ptr(), M, K, B_dev.data_ptr(), N, C_dev.data_ptr())
        assert rc == 0, msg
        assert torch.cuda.current_device() == dev_before
        C = C_dev.cpu().numpy().T
        ref = lib.bf16x3_gemm(A, B)
        assert np.all(np.isfinite(C))
        assert rel_err(C, ref) < SPLIT_REL_TOL
        assert rel_err(C, A @ B) < SPLIT_REL_TOL


def test_noalloc_gemm_refuses_host_pointers(lib):
    # A host buffer passed as an operand is refused before any kernel runs.
    torch = pytest.importorskip("torch")
    dev = torch.zeros(64 * 64, dtype=torch.float64, device="cuda")
    host = np.zeros(64 * 64)
    rc, msg = _call_noalloc(lib, host.ctypes.data, 64, 64, dev.data_ptr(), 64, dev.data_ptr())
    assert rc == 1 and "device" in msg
    rc, msg = _call_noalloc(lib, dev.data_ptr(), 64, 64, dev.data_ptr(), 64, host.ctypes.data)
    assert rc == 1 and "device" in msg


def test_noalloc_gemm_rejects_oversized_shapes(lib):
    torch = pytest.importorskip("torch")
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc, msg = _call_noalloc(lib, dummy.data_ptr(), 20000, 4096, dummy.data_ptr(), 64,
                            dummy.data_ptr())
    assert rc == 1 and "scratch" in msg

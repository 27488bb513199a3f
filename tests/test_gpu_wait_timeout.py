"""The bounded waits of the tensor-core pipeline, made to run out on purpose.

With FASTPLS_TEST_WITHHOLD_LOADS=1 the split GEMM's producer issues no TMA load,
so the MMA issuer waits on a stage that nothing fills: its mbarrier wait gives
up after its clock budget (~4 s), raises the kernel's error flag, the other
roles see the flag and leave, and the CTA frees its tensor memory.  No copy
and no MMA is in flight at any point, so the GPU is never faulted; the call
returns FPLS_ERR_CUDA and the next call runs normally on the same context.
"""
import numpy as np
import pytest

from parity_utils import rel_err

pytestmark = pytest.mark.gpu


def test_split_gemm_wait_timeout_reports_and_recovers(lib, monkeypatch):
    rng = np.random.default_rng(5)
    A = rng.standard_normal((256, 192))
    B = rng.standard_normal((192, 40))
    monkeypatch.setenv("FASTPLS_TEST_WITHHOLD_LOADS", "1")
    with pytest.raises(lib.FastPLSError) as info:
        lib.bf16x3_gemm(A, B)
    assert info.value.code == 2 and "timed out" in str(info.value)
    monkeypatch.delenv("FASTPLS_TEST_WITHHOLD_LOADS")
    for _ in range(2):  # tensor memory was released: later calls allocate it again
        C = lib.bf16x3_gemm(A, B)
        assert rel_err(C, A @ B) < 1e-4

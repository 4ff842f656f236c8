"""Failure detection of the bounded device-side waits, without a GPU fault.

The tensor-core spreader and the FFT row kernel wait on mbarriers with a time
limit; a wait that gives up raises the kernel's abort flag and the device
error word, and the host turns the word into DNUFFT_ERR_TIMEOUT.  The test
hook runs the spreader's own wait routine, with a 2 ms limit, on a barrier
that nothing arrives at (no fault, no hang), checks the status and that the
context is still usable: the error word is cleared and the next transform
succeeds.
"""
import numpy as np
import pytest

from ducc_b200 import _capi as C
from ducc_b200 import nufft

pytestmark = pytest.mark.gpu

DNUFFT_ERR_TIMEOUT = 5


def test_bounded_wait_reports_timeout_and_context_survives():
    import torch
    st = ctypes_stream = torch.cuda.current_stream().cuda_stream
    L = C.lib()
    for _ in range(2):
        status = L.dnufft_selftest_wait_timeout(2_000_000, ctypes_stream)
        assert status == DNUFFT_ERR_TIMEOUT
        assert b"bounded device-side wait" in L.dnufft_last_error()
    assert L.dnufft_selftest_wait_timeout(0, st) != 0   # bad argument, no launch
    # the context and the error word are fine: a transform (tensor-core
    # spreader) runs and its result is finite
    rng = np.random.default_rng(0)
    M, shape = 30000, (96, 80)
    coord = torch.from_numpy(rng.uniform(-np.pi, np.pi, (M, 2)).astype(np.float32)).cuda()
    vals = torch.randn(M, dtype=torch.complex64, device="cuda")
    out = torch.empty(shape, dtype=torch.complex64, device="cuda")
    nufft.nu2u(points=vals, coord=coord, forward=True, epsilon=1e-5, out=out, spreader="tc")
    torch.cuda.synchronize()
    assert torch.isfinite(torch.view_as_real(out)).all()

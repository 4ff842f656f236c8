"""dnufft_nu2u_noalloc: the type-1 entry point for callers that cannot allocate
device memory while a transform runs (stream capture, plugins inside a
framework that owns the device memory pool, fixed-budget services).  It takes
every temporary from a fixed scratch area compiled into the library.

Called through the C-ABI and checked against the regular entry point
dnufft_nu2u on the same device inputs, with the tolerance the other parity
tests use (relative L2 below epsilon), on two calls in a row with different
problems, so that contents left in the shared scratch area by the first call
cannot leak into the second.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from ducc_b200 import _capi as C
from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu


def problem(seed, M, shape, cdtype, vdtype):
    rng = np.random.default_rng(seed)
    coord = rng.uniform(-np.pi, np.pi, (M, len(shape))).astype(cdtype)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(vdtype)
    return coord, vals


def call(fn, coord, vals, shape, eps, forward=True):
    import torch
    dc = torch.from_numpy(coord).cuda()
    dv = torch.from_numpy(vals).cuda()
    tdt = torch.complex64 if vals.dtype == np.complex64 else torch.complex128
    out = torch.full(shape, float("nan"), dtype=tdt, device="cuda")
    opts = C.make_opts(False, ndim=len(shape))
    a_p, a_c, a_o = C.describe(dv), C.describe(dc), C.describe(out)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    status = fn(ctypes.byref(a_p), ctypes.byref(a_c), 1 if forward else 0, float(eps),
                ctypes.byref(a_o), ctypes.byref(opts), st)
    torch.cuda.synchronize()
    return status, out.cpu().numpy()


CASES = [
    # seed, M, shape, coord dtype, value dtype, eps
    (1, 20000, (96, 80), np.float32, np.complex64, 1e-5),
    (2, 3000, (12, 14, 16), np.float64, np.complex128, 1e-9),
    (3, 50000, (200,), np.float64, np.complex64, 1e-4),
]


def test_noalloc_matches_regular_entry_point_twice():
    L = C.lib()
    assert L.dnufft_noalloc_scratch_bytes() == 32 << 20
    # two calls in a row through the no-allocation path, different problems,
    # each checked against the regular (allocating) entry point
    for seed, M, shape, cdt, vdt, eps in CASES[:2] + CASES[:2]:
        coord, vals = problem(seed, M, shape, cdt, vdt)
        s1, ref = call(L.dnufft_nu2u, coord, vals, shape, eps)
        assert s1 == 0, L.dnufft_last_error()
        s2, got = call(L.dnufft_nu2u_noalloc, coord, vals, shape, eps)
        assert s2 == 0, L.dnufft_last_error()
        assert np.all(np.isfinite(got))
        assert O.l2error(got, ref) < eps
    seed, M, shape, cdt, vdt, eps = CASES[2]
    coord, vals = problem(seed, M, shape, cdt, vdt)
    s1, ref = call(L.dnufft_nu2u, coord, vals, shape, eps)
    s2, got = call(L.dnufft_nu2u_noalloc, coord, vals, shape, eps)
    assert s1 == 0 and s2 == 0
    assert O.l2error(got, ref) < eps
    # and against the exact transform
    d = O.direct_nu2u(coord.astype(np.float64), vals, shape, True)
    assert O.l2error(got, d) < 4 * eps


def test_noalloc_rejects_oversized_problem():
    L = C.lib()
    coord, vals = problem(4, 1000, (4096, 4096), np.float32, np.complex64)
    status, _ = call(L.dnufft_nu2u_noalloc, coord, vals, (4096, 4096), 1e-5)
    assert status == 1
    assert b"no-allocation scratch" in L.dnufft_last_error()


def test_noalloc_allocates_no_device_memory():
    """The property the entry point exists for: a call whose problem is new in
    size (more points, so more scratch than any call before it) leaves the
    device's free memory unchanged.  Every device array of the test is
    allocated first, and one warm-up call loads the kernels the timed calls
    use (loading kernel code takes device memory once)."""
    import torch
    L = C.lib()
    shape, eps = (96, 80), 1e-5
    arrays = []
    for seed, M in ((5, 20000), (6, 70000)):
        coord, vals = problem(seed, M, shape, np.float32, np.complex64)
        dc = torch.from_numpy(coord).cuda()
        dv = torch.from_numpy(vals).cuda()
        out = torch.empty(shape, dtype=torch.complex64, device="cuda")
        arrays.append((dc, dv, out))
    opts = C.make_opts(False, ndim=2)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run(dc, dv, out):
        a_p, a_c, a_o = C.describe(dv), C.describe(dc), C.describe(out)
        s = L.dnufft_nu2u_noalloc(ctypes.byref(a_p), ctypes.byref(a_c), 1, eps,
                                  ctypes.byref(a_o), ctypes.byref(opts), st)
        torch.cuda.synchronize()
        return s

    assert run(*arrays[0]) == 0, L.dnufft_last_error()
    free0, _ = torch.cuda.mem_get_info()
    assert run(*arrays[1]) == 0, L.dnufft_last_error()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    # and the larger call is still right
    coord, vals = problem(6, 70000, shape, np.float32, np.complex64)
    s1, ref = call(L.dnufft_nu2u, coord, vals, shape, eps)
    assert s1 == 0
    assert O.l2error(arrays[1][2].cpu().numpy(), ref) < eps

"""DUCC's own NUFFT test sweep (python/test/test_nufft.py:46-230), run against
this library through the same call sequence.

Every parameter list of the reference's test_nufft_1d / 2d / 3d is kept, and
so is their cross product (about 12,500 cases, the single-precision cases
below eps=1e-6 skipped as there): grid sizes, 1 / 10 / 37 points, three
epsilons, both signs, single and double precision, scalar and per-axis
periodicity, both mode orders, nthreads 1 and 2 (which steer DUCC's
parameter cost model).  Each case checks, as the reference does:

* nu2u against the direct sum: relative L2 error <= {4, 2, 1} * eps in 1D /
  2D / 3D (DUCC's l2error, python/misc_pymod.cc:129-185);
* u2nu with the opposite sign is the adjoint: vdot(points, u2nu) equals
  vdot(nu2u, grid) within 3e-5 (single) / 2e-13 (double) of the largest norm;
* in double precision, the same through plans.

The 2D single-precision cases run once more with the split-precision
tensor-core spreader forced (unplanned and planned), against the same bound.

The reference imports ``ducc0``; here ``ducc0.nufft`` is this library's drop-in
module and ``ducc0.misc`` the oracle's long-double vdot / l2error.  The
reference's optional comparison against finufft is left out (finufft is not
installed).  The reference file itself is not read at run time: it does not
exist where the GPU tests run.
"""
import types

import numpy as np
import pytest
from numpy.testing import assert_allclose

from ducc_b200 import nufft as _nufft
from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu
pmp = pytest.mark.parametrize

ducc0 = types.SimpleNamespace(nufft=_nufft,
                              misc=types.SimpleNamespace(vdot=O.vdot, l2error=O.l2error))


def direct(uvw, ms, shape, forward, periodicity, fft_order):
    """Direct type-1 sum, modes from -N//2, in complex128."""
    sign = -1.0 if forward else 1.0
    per = np.ones(len(shape)) * np.asarray(periodicity, dtype=np.float64)
    out = np.zeros(shape, np.complex128)
    axes = [(np.arange(n) - n // 2) * (2 * np.pi / p) for n, p in zip(shape, per)]
    grids = np.meshgrid(*axes, indexing="ij")
    for j in range(ms.shape[0]):
        ph = sum(g * x for g, x in zip(grids, uvw[j]))
        out += complex(ms[j]) * np.exp(1j * sign * ph)
    return np.fft.ifftshift(out) if fft_order else out


def case_data(shape, npoints, periodicity, singleprec):
    rng = np.random.default_rng(42)
    uvw = (rng.random((npoints, len(shape))) - 0.5) * periodicity
    ms = rng.random(npoints) - 0.5 + 1j * (rng.random(npoints) - 0.5)
    dirty = rng.random(shape) - 0.5
    dirty = dirty + 1j * (rng.random(shape) - 0.5)
    if singleprec:
        ms = ms.astype(np.complex64)
        dirty = dirty.astype(np.complex64)
    return uvw, ms, dirty


def run_case(shape, npoints, epsilon, forward, singleprec, periodicity, fft_order, nthreads,
             tol_factor):
    if singleprec and epsilon < 1e-6:
        pytest.skip("single precision below 1e-6 (as in the reference)")
    uvw, ms, dirty = case_data(shape, npoints, periodicity, singleprec)

    def adjoint_ok(d2, m2):
        r = max(ducc0.misc.vdot(ms, ms).real, ducc0.misc.vdot(m2, m2).real,
                ducc0.misc.vdot(dirty, dirty).real, ducc0.misc.vdot(d2, d2).real)
        tol = 3e-5 * r if singleprec else 2e-13 * r
        assert_allclose(ducc0.misc.vdot(ms, m2), ducc0.misc.vdot(d2, dirty), rtol=tol)

    d2 = np.empty(shape, dtype=dirty.dtype)
    d2 = ducc0.nufft.nu2u(points=ms, coord=uvw, forward=forward, epsilon=epsilon,
                          nthreads=nthreads, out=d2, periodicity=periodicity,
                          fft_order=fft_order).astype(np.complex128)
    ref = direct(uvw, ms, shape, forward, periodicity, fft_order)
    assert ducc0.misc.l2error(d2, ref) <= tol_factor * epsilon
    m2 = ducc0.nufft.u2nu(grid=dirty, coord=uvw, forward=not forward, epsilon=epsilon,
                          nthreads=nthreads, periodicity=periodicity,
                          fft_order=fft_order).astype(np.complex128)
    adjoint_ok(d2, m2)
    if not singleprec:
        p1 = ducc0.nufft.plan(nu2u=True, coord=uvw, grid_shape=shape, epsilon=epsilon,
                              nthreads=nthreads, periodicity=periodicity, fft_order=fft_order)
        d3 = p1.nu2u(points=ms, forward=forward)
        p2 = ducc0.nufft.plan(nu2u=False, coord=uvw, grid_shape=shape, epsilon=epsilon,
                              nthreads=nthreads, periodicity=periodicity, fft_order=fft_order)
        m3 = p2.u2nu(grid=dirty, forward=not forward)
        adjoint_ok(d3, m3)


@pmp("nx", [1, 20, 21, 250, 257])
@pmp("npoints", (1, 37, 10))
@pmp("epsilon", (1e-1, 3e-5, 2e-13))
@pmp("forward", (True, False))
@pmp("singleprec", (True, False))
@pmp("periodicity", ([1.], 2 * np.pi))
@pmp("fft_order", (False, True))
@pmp("nthreads", (1, 2))
def test_nufft_1d(nx, npoints, epsilon, forward, singleprec, periodicity, fft_order, nthreads):
    run_case((nx,), npoints, epsilon, forward, singleprec, periodicity, fft_order, nthreads, 4)


@pmp("nx", [1, 20, 21, 250, 257])
@pmp("ny", [1, 21, 32, 257])
@pmp("npoints", (1, 37, 10))
@pmp("epsilon", (1e-1, 3e-5, 2e-13))
@pmp("forward", (True, False))
@pmp("singleprec", (True, False))
@pmp("periodicity", ((1., 1.), 2 * np.pi))
@pmp("fft_order", (False, True))
@pmp("nthreads", (1, 2))
def test_nufft_2d(nx, ny, npoints, epsilon, forward, singleprec, periodicity, fft_order,
                  nthreads):
    run_case((nx, ny), npoints, epsilon, forward, singleprec, periodicity, fft_order, nthreads,
             2)


@pmp("nx", [1, 20, 21])
@pmp("ny", [1, 21, 32])
@pmp("nz", [1, 22, 35])
@pmp("npoints", (1, 37, 10))
@pmp("epsilon", (1e-5, 3e-5, 5e-13))
@pmp("forward", (True, False))
@pmp("singleprec", (True, False))
@pmp("periodicity", (1., [1., np.pi, 7]))
@pmp("fft_order", (False, True))
@pmp("nthreads", (1, 2))
def test_nufft_3d(nx, ny, nz, npoints, epsilon, forward, singleprec, periodicity, fft_order,
                  nthreads):
    run_case((nx, ny, nz), npoints, epsilon, forward, singleprec, periodicity, fft_order,
             nthreads, 1)


@pmp("nx", [1, 20, 21, 250, 257])
@pmp("ny", [1, 21, 32, 257])
@pmp("npoints", (1, 37, 10))
@pmp("epsilon", (1e-1, 3e-5))
@pmp("forward", (True, False))
@pmp("periodicity", ((1., 1.), 2 * np.pi))
@pmp("fft_order", (False, True))
def test_nufft_2d_tensor_core_spreader(nx, ny, npoints, epsilon, forward, periodicity,
                                       fft_order):
    """The single-precision 2D cases of the sweep with the tensor-core
    spreader forced (the automatic choice takes it only from 0.5 points per
    mode): the same criterion against the direct sum, unplanned and planned."""
    shape = (nx, ny)
    uvw, ms, dirty = case_data(shape, npoints, periodicity, True)
    # float64 coordinates with complex64 values, as the reference's single
    # precision cases
    ref = direct(uvw, ms, shape, forward, periodicity, fft_order)
    d2 = np.empty(shape, np.complex64)
    d2 = _nufft.nu2u(points=ms, coord=uvw, forward=forward, epsilon=epsilon, out=d2,
                     periodicity=periodicity, fft_order=fft_order,
                     spreader="tc").astype(np.complex128)
    assert ducc0.misc.l2error(d2, ref) <= 2 * epsilon
    # a single-precision plan takes float32 coordinates
    u32 = uvw.astype(np.float32)
    ref32 = direct(u32.astype(np.float64), ms, shape, forward, periodicity, fft_order)
    p = _nufft.plan(nu2u=True, coord=u32, grid_shape=shape, epsilon=epsilon,
                    periodicity=periodicity, fft_order=fft_order, spreader="tc")
    d3 = p.nu2u(points=ms, forward=forward).astype(np.complex128)
    assert ducc0.misc.l2error(d3, ref32) <= 2 * epsilon

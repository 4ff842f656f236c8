"""Oversampled FFT lengths chosen to exercise the pencil passes of the row and
column FFT kernels: two, three and four passes, odd and even last radices,
composite radices, lengths whose plan is impossible under the register bounds
(which fall back to the single-pass line kernels), complex64 and complex128.

A small uniform grid is transformed on a forced large oversampled grid (any
oversampling above the kernel's own keeps the kernel's accuracy), so the
direct NUDFT is a cheap exact reference for both transform types and signs.
"""
import numpy as np
import pytest

from ducc_b200 import autotune, nufft
from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu

SHAPE = (48, 40)
CASES = [
    # (n0, n1), single precision
    ((1024, 8400), True),     # rows 21*20*20 / 3 passes, columns four-step
    ((8400, 1100), True),     # rows 5*20*11 (odd last radix)
    ((2310, 4096), True),     # 2*3*5*7*11 columns, rows 16*16*16
    ((4200, 1536), True),
    ((1250, 9604), True),     # rows beyond the register bounds: line-kernel fallback
    ((1024, 6600), False),    # rows 5*11*8*15 / 4 passes
    ((6050, 2310), False),    # columns 6050 = 2*5^2*11^2
    ((1100, 6250), False),    # rows beyond the register bounds: fallback
]


def problem(single, seed):
    rng = np.random.default_rng(seed)
    M = 3000
    coord = rng.uniform(-np.pi, np.pi, (M, 2))
    vals = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    grid = rng.standard_normal(SHAPE) + 1j * rng.standard_normal(SHAPE)
    if single:
        return coord.astype(np.float32), vals.astype(np.complex64), grid.astype(np.complex64)
    return coord, vals, grid


@pytest.mark.parametrize("nover,single", CASES)
def test_pencil_lengths(nover, single):
    eps = 1e-5 if single else 1e-10
    coord, vals, grid = problem(single, sum(nover))
    kidx = autotune.candidates(SHAPE, eps, single)[0][0]
    for forward in (True, False):
        p = nufft.plan(nu2u=True, coord=coord, grid_shape=SHAPE, epsilon=eps,
                       force_kernel=kidx, force_nover=list(nover))
        assert list(p.info()["nover"]) == list(nover)
        got1 = p.nu2u(points=vals, forward=forward)
        ref1 = O.direct_nu2u(coord, vals, SHAPE, forward)
        assert O.l2error(got1, ref1) < 4 * eps
        got2 = p.u2nu(grid=grid, forward=forward)
        ref2 = O.direct_u2nu(grid, coord, forward)
        assert O.l2error(got2, ref2) < 4 * eps

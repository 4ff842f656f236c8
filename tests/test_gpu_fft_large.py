"""2D transforms on oversampled grids with axes >= 1024 points, where the
row FFTs run in the persistent bulk-copy kernel and the column FFTs in two
four-step passes (with the single-pass kernels covering the short axes).

Checked against the oracle (FP64 restatement of DUCC's algorithm, same kernel
and oversampled sizes) and against the direct NUDFT on a few rows of modes;
odd sizes give kept ranges whose ends are not 16-byte aligned, both signs and
both output orders are covered, in complex64 and complex128.
"""
import numpy as np
import pytest

from ducc_b200 import nufft
from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    # shape, single precision, eps, forward, fft_order
    ((600, 700), True, 1e-5, True, False),
    ((613, 1031), True, 1e-6, False, True),
    ((1500, 64), True, 1e-5, True, True),
    ((64, 1500), True, 1e-5, False, False),
    ((1100, 1300), False, 1e-10, False, False),
    ((1013, 1201), False, 1e-9, True, True),
]


def problem(shape, single, seed):
    rng = np.random.default_rng(seed)
    M = 20000
    coord = rng.uniform(-np.pi, np.pi, (M, 2))
    vals = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    grid = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    if single:
        return coord.astype(np.float32), vals.astype(np.complex64), grid.astype(np.complex64)
    return coord, vals, grid


@pytest.mark.parametrize("shape,single,eps,forward,fft_order", CASES)
def test_type1_large_axes(shape, single, eps, forward, fft_order):
    coord, vals, _ = problem(shape, single, 1)
    kw = dict(epsilon=eps, nthreads=1, sigma_min=1.2, sigma_max=2.51, fft_order=fft_order)
    p = nufft.plan(nu2u=True, coord=coord, grid_shape=shape, **kw)
    assert max(p.info()["nover"]) >= 1024
    got = p.nu2u(points=vals, forward=forward)
    par = O.Params(shape, eps, single, coord.shape[0], True, 1)
    assert par.nover == p.info()["nover"]
    ref = O.nu2u(par, coord, vals, forward, fft_order)
    assert O.l2error(got, ref) < (3e-6 if single else 1e-11)
    # exact transform on a few rows of modes
    ku = np.arange(3) - shape[0] // 2
    kv = np.arange(shape[1]) - shape[1] // 2
    s = -1 if forward else 1
    c = coord.astype(np.float64)
    ex = np.einsum("m,mi,mj->ij", vals.astype(np.complex128), np.exp(s * 1j * np.outer(c[:, 0], ku)),
                   np.exp(s * 1j * np.outer(c[:, 1], kv)), optimize=True)
    rows = got[:3] if not fft_order else np.fft.fftshift(got)[:3]
    assert O.l2error(rows, ex) < 4 * eps


@pytest.mark.parametrize("shape,single,eps,forward,fft_order", CASES)
def test_type2_large_axes(shape, single, eps, forward, fft_order):
    coord, _, grid = problem(shape, single, 2)
    kw = dict(epsilon=eps, nthreads=1, sigma_min=1.2, sigma_max=2.51, fft_order=fft_order)
    p = nufft.plan(nu2u=False, coord=coord, grid_shape=shape, **kw)
    got = p.u2nu(grid=grid, forward=forward)
    par = O.Params(shape, eps, single, coord.shape[0], False, 1)
    assert par.nover == p.info()["nover"]
    ref = O.u2nu(par, grid, coord, forward, fft_order)
    assert O.l2error(got, ref) < (3e-6 if single else 1e-11)
    idx = np.arange(0, coord.shape[0], 997)
    ex = O.direct_u2nu(grid, coord[idx], forward, fft_order=fft_order)
    assert O.l2error(got[idx], ex) < 4 * eps


def test_unplanned_and_device_arrays_large():
    import torch
    coord, vals, grid = problem((1100, 900), True, 3)
    dc, dv, dg = (torch.from_numpy(x).cuda() for x in (coord, vals, grid))
    out = torch.empty((1100, 900), dtype=torch.complex64, device="cuda")
    nufft.nu2u(points=dv, coord=dc, forward=True, epsilon=1e-5, out=out)
    par = O.Params((1100, 900), 1e-5, True, coord.shape[0], True, 1)
    assert O.l2error(out.cpu().numpy(), O.nu2u(par, coord, vals, True)) < 3e-6
    r = nufft.u2nu(grid=dg, coord=dc, forward=False, epsilon=1e-5)
    par2 = O.Params((1100, 900), 1e-5, True, coord.shape[0], False, 1)
    assert O.l2error(r.cpu().numpy(), O.u2nu(par2, grid, coord, False)) < 3e-6

"""Unplanned calls on large host arrays run pipelined: the points are cut into
groups whose host->device copies (and, for type 2, device->host copies of the
results) overlap the sorting and spreading / interpolation of the other
groups.  Checked against the same calls on device arrays (one group, no
overlap), in complex64 (tensor-core spreader chosen by 'auto' at this density)
and complex128, both signs, and against the direct NUDFT on a sample of
modes / points.
"""
import numpy as np
import pytest

from ducc_b200 import nufft
from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu

M = 5_000_000          # above the pipelining threshold (4M points): 2 groups
SHAPE = (320, 288)


@pytest.mark.parametrize("single", [True, False])
def test_pipelined_host_calls_match_device_calls(single):
    import torch
    rng = np.random.default_rng(11)
    cdt, vdt = (np.float32, np.complex64) if single else (np.float64, np.complex128)
    eps = 1e-5 if single else 1e-10
    coord = rng.uniform(-np.pi, np.pi, (M, 2)).astype(cdt)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(vdt)
    grid = (rng.standard_normal(SHAPE) + 1j * rng.standard_normal(SHAPE)).astype(vdt)
    dc, dv, dg = (torch.from_numpy(x).cuda() for x in (coord, vals, grid))
    tol = 2e-6 if single else 1e-12
    for forward in (True, False):
        # type 1
        h_out = np.zeros(SHAPE, vdt)
        nufft.nu2u(points=vals, coord=coord, forward=forward, epsilon=eps, out=h_out)
        d_out = torch.zeros(SHAPE, dtype=dv.dtype, device="cuda")
        nufft.nu2u(points=dv, coord=dc, forward=forward, epsilon=eps, out=d_out)
        assert O.l2error(h_out, d_out.cpu().numpy()) < tol
        # a few modes against the direct sum over all points
        s = -1 if forward else 1
        ku = np.array([0, 1])
        kv = np.arange(8) - 4
        ex = np.zeros((2, 8), np.complex128)
        for i in range(0, M, 1000000):
            cc = coord[i:i + 1000000].astype(np.float64)
            ex += np.einsum("m,mi,mj->ij", vals[i:i + 1000000].astype(np.complex128),
                            np.exp(s * 1j * np.outer(cc[:, 0], ku)),
                            np.exp(s * 1j * np.outer(cc[:, 1], kv)), optimize=True)
        got = h_out[SHAPE[0] // 2:SHAPE[0] // 2 + 2, SHAPE[1] // 2 - 4:SHAPE[1] // 2 + 4]
        assert O.l2error(got, ex) < 2 * eps
        # type 2
        h_pts = np.empty(M, vdt)
        nufft.u2nu(grid=grid, coord=coord, forward=forward, epsilon=eps, out=h_pts)
        d_pts = nufft.u2nu(grid=dg, coord=dc, forward=forward, epsilon=eps)
        assert O.l2error(h_pts, d_pts.cpu().numpy()) < tol
        idx = rng.choice(M, 500, replace=False)
        ref = O.direct_u2nu(grid, coord[idx], forward)
        assert O.l2error(h_pts[idx], ref) < 2 * eps


def test_pipelined_mixed_host_and_device_arrays():
    """Host coordinates with device grids / outputs (the pipeline then uploads
    only the coordinates), and host values with a device output."""
    import torch
    rng = np.random.default_rng(12)
    eps = 1e-5
    coord = rng.uniform(-np.pi, np.pi, (M, 2)).astype(np.float32)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
    grid = (rng.standard_normal(SHAPE) + 1j * rng.standard_normal(SHAPE)).astype(np.complex64)
    dc, dv, dg = (torch.from_numpy(x).cuda() for x in (coord, vals, grid))
    # type 2: host coordinates, device grid and output (strided output view)
    big = torch.zeros(2 * M, dtype=torch.complex64, device="cuda")
    nufft.u2nu(grid=dg, coord=coord, forward=True, epsilon=eps, out=big[::2])
    ref = nufft.u2nu(grid=dg, coord=dc, forward=True, epsilon=eps)
    assert O.l2error(big[::2].cpu().numpy(), ref.cpu().numpy()) < 2e-6
    assert float(big[1::2].abs().max()) == 0.0
    # type 1: host coordinates and values, device output
    d_out = torch.zeros(SHAPE, dtype=torch.complex64, device="cuda")
    nufft.nu2u(points=vals, coord=coord, forward=False, epsilon=eps, out=d_out)
    ref1 = torch.zeros(SHAPE, dtype=torch.complex64, device="cuda")
    nufft.nu2u(points=dv, coord=dc, forward=False, epsilon=eps, out=ref1)
    assert O.l2error(d_out.cpu().numpy(), ref1.cpu().numpy()) < 2e-6


@pytest.mark.parametrize("shape,single", [((3000,), False), ((40, 36, 32), True),
                                          ((24, 20, 18), False)])
def test_pipelined_1d_3d(shape, single):
    """The pipelined host path in 1D and 3D (4.5M points: two groups) against
    the device-array path and direct sums on samples."""
    import torch
    rng = np.random.default_rng(13)
    M = 4_500_000
    nd = len(shape)
    cdt, vdt = (np.float32, np.complex64) if single else (np.float64, np.complex128)
    eps = 1e-5 if single else 1e-10
    coord = rng.uniform(-np.pi, np.pi, (M, nd)).astype(cdt)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(vdt)
    grid = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(vdt)
    dc, dv, dg = (torch.from_numpy(x).cuda() for x in (coord, vals, grid))
    tol = 2e-6 if single else 1e-12
    h_out = np.zeros(shape, vdt)
    nufft.nu2u(points=vals, coord=coord, forward=True, epsilon=eps, out=h_out)
    d_out = torch.zeros(shape, dtype=dv.dtype, device="cuda")
    nufft.nu2u(points=dv, coord=dc, forward=True, epsilon=eps, out=d_out)
    assert O.l2error(h_out, d_out.cpu().numpy()) < tol
    h_pts = np.empty(M, vdt)
    nufft.u2nu(grid=grid, coord=coord, forward=False, epsilon=eps, out=h_pts)
    d_pts = nufft.u2nu(grid=dg, coord=dc, forward=False, epsilon=eps)
    assert O.l2error(h_pts, d_pts.cpu().numpy()) < tol
    idx = rng.choice(M, 300, replace=False)
    ref = O.direct_u2nu(grid, coord[idx], False)
    assert O.l2error(h_pts[idx], ref) < 2 * eps


@pytest.mark.parametrize("single,spreader", [(True, "tc"), (True, "plain"), (False, "auto")])
def test_planned_host_groups_match_device_calls(single, spreader):
    """A plan made from host coordinates with many points keeps a per-group
    index: its calls on host arrays copy groups in / results out while other
    groups are spread / interpolated.  Same plan, same results as its calls on
    device arrays (one index over all points), repeated calls included."""
    import torch
    rng = np.random.default_rng(12)
    cdt, vdt = (np.float32, np.complex64) if single else (np.float64, np.complex128)
    eps = 1e-6 if single else 1e-10
    coord = rng.uniform(-np.pi, np.pi, (M, 2)).astype(cdt)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(vdt)
    grid = (rng.standard_normal(SHAPE) + 1j * rng.standard_normal(SHAPE)).astype(vdt)
    dv, dg = (torch.from_numpy(x).cuda() for x in (vals, grid))
    tol = 2e-6 if single else 1e-12
    p = nufft.plan(nu2u=True, coord=coord, grid_shape=SHAPE, epsilon=eps, spreader=spreader)
    for forward in (True, False):
        for _ in range(2):
            h_out = np.zeros(SHAPE, vdt)
            p.nu2u(points=vals, forward=forward, out=h_out)
            d_out = p.nu2u(points=dv, forward=forward)
            assert O.l2error(h_out, d_out.cpu().numpy()) < tol
            h_pts = np.empty(M, vdt)
            p.u2nu(grid=grid, forward=forward, out=h_pts)
            d_pts = p.u2nu(grid=dg, forward=forward)
            assert O.l2error(h_pts, d_pts.cpu().numpy()) < tol
        idx = rng.choice(M, 300, replace=False)
        assert O.l2error(h_pts[idx], O.direct_u2nu(grid, coord[idx], forward)) < 2 * eps
    # device uniform grid, host output: the grouped path reads the device array
    h_pts2 = np.empty(M, vdt)
    p.u2nu(grid=dg, forward=True, out=h_pts2)
    assert O.l2error(h_pts2, p.u2nu(grid=dg, forward=True).cpu().numpy()) < tol


def test_planned_host_groups_3d_and_ntrans():
    """The per-group path of a host-coordinate plan in 3D, and with several
    transforms per call (each transform through the groups), against the same
    plan on device arrays."""
    import torch
    rng = np.random.default_rng(13)
    M3, shape = 4_300_000, (40, 36, 44)
    coord = rng.uniform(-np.pi, np.pi, (M3, 3)).astype(np.float32)
    vals = (rng.standard_normal((2, M3)) + 1j * rng.standard_normal((2, M3))).astype(np.complex64)
    grid = (rng.standard_normal((2,) + shape) + 1j * rng.standard_normal((2,) + shape)).astype(
        np.complex64)
    p = nufft.plan(nu2u=True, coord=coord, grid_shape=shape, epsilon=1e-5, periodicity=[2 * np.pi, 3.0, 5.0])
    h = p.nu2u(points=vals, forward=True)
    d = p.nu2u(points=torch.from_numpy(vals).cuda(), forward=True).cpu().numpy()
    assert h.shape == (2,) + shape
    for t in range(2):
        assert O.l2error(h[t], d[t]) < 2e-6
    h2 = np.empty((2, M3), np.complex64)
    p.u2nu(grid=grid, forward=False, out=h2)
    d2 = p.u2nu(grid=torch.from_numpy(grid).cuda(), forward=False).cpu().numpy()
    for t in range(2):
        assert O.l2error(h2[t], d2[t]) < 2e-6

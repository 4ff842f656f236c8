"""Parity of the CUDA path (through the C-ABI) with DUCC and the oracle.

* golden fixtures produced by DUCC itself (tests/golden): outputs within the
  requested epsilon, tile permutation bit-exact;
* the oracle (numpy restatement, FP64) and direct FP64 sums on small problems
  (DUCC's own parameter sweep, with its tolerances, is tests/test_gpu_nufft_sweep.py);
* edge cases: zero points, strided device arrays, coordinates far outside
  the period, cfg1 at full size.
"""
import glob
import os

import numpy as np
import pytest

from ducc_b200 import nufft
from oracle import nufft_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "g*.npz")))

pytestmark = pytest.mark.gpu


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def torch_dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("device", [False, True])
def test_golden_nu2u(name, device):
    g = load(name)
    eps = float(g["eps"])
    per = list(g["periodicity"])
    shape = tuple(int(s) for s in g["shape"])
    vdt = g["values"].dtype
    if device:
        import torch
        out = torch.zeros(shape, dtype=torch.complex64 if vdt == np.complex64 else torch.complex128,
                          device="cuda")
        nufft.nu2u(points=torch_dev(g["values"]), coord=torch_dev(g["coord"]),
                   forward=bool(g["forward"]), epsilon=eps, out=out, periodicity=per,
                   fft_order=bool(g["fft_order"]))
        res = out.cpu().numpy()
    else:
        res = np.zeros(shape, dtype=vdt)
        nufft.nu2u(points=g["values"], coord=g["coord"], forward=bool(g["forward"]), epsilon=eps,
                   out=res, periodicity=per, fft_order=bool(g["fft_order"]))
    # both are approximations of the same transform with the same kernel:
    # they agree far better than eps
    assert O.l2error(res, g["nu2u"]) < eps
    ref = O.direct_nu2u(g["coord"], g["values"], shape, bool(g["forward"]), per,
                        bool(g["fft_order"]))
    assert O.l2error(res, ref) < 2 * eps * len(shape)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("device", [False, True])
def test_golden_u2nu(name, device):
    g = load(name)
    eps = float(g["eps"])
    per = list(g["periodicity"])
    if device:
        res = nufft.u2nu(grid=torch_dev(g["grid_in"]), coord=torch_dev(g["coord"]),
                         forward=bool(g["forward"]), epsilon=eps, periodicity=per,
                         fft_order=bool(g["fft_order"])).cpu().numpy()
    else:
        res = nufft.u2nu(grid=g["grid_in"], coord=g["coord"], forward=bool(g["forward"]),
                         epsilon=eps, periodicity=per, fft_order=bool(g["fft_order"]))
    assert res.dtype == g["u2nu"].dtype
    assert O.l2error(res, g["u2nu"]) < eps
    ref = O.direct_u2nu(g["grid_in"], g["coord"], bool(g["forward"]), per, bool(g["fft_order"]))
    assert O.l2error(res, ref) < 2 * eps * g["grid_in"].ndim


@pytest.mark.parametrize("name", CASES)
def test_golden_permutation_bit_exact(name):
    g = load(name)
    shape = tuple(int(s) for s in g["shape"])
    coord = g["coord"]
    sp = bool(g["singleprec"])
    # a plan's precision follows its coordinates; DUCC's function path for
    # mixed precision uses the data precision, so compare where they agree
    if sp != (coord.dtype == np.float32):
        pytest.skip("mixed-precision fixture (function path only)")
    p = nufft.plan(nu2u=True, coord=coord, grid_shape=shape, epsilon=float(g["eps"]),
                   nthreads=1, sigma_min=1.2, sigma_max=2.51, periodicity=list(g["periodicity"]),
                   fft_order=bool(g["fft_order"]))
    info = p.info()
    assert info["supp"] == int(g["W1"])
    assert info["nover"] == [int(x) for x in g["nover1"]]
    assert np.array_equal(p.permutation(), g["perm1"])


@pytest.mark.parametrize("name", ["g2d_f64", "g3d_f64", "g1d_f64", "g2d_f32", "g3d_f32"])
def test_golden_planned(name):
    g = load(name)
    shape = tuple(int(s) for s in g["shape"])
    coord = g["coord"]
    sp = bool(g["singleprec"])
    if sp != (coord.dtype == np.float32):
        pytest.skip("mixed precision")
    eps = float(g["eps"])
    kw = dict(epsilon=eps, nthreads=1, sigma_min=1.2, sigma_max=2.51,
              periodicity=list(g["periodicity"]), fft_order=bool(g["fft_order"]))
    p1 = nufft.plan(nu2u=True, coord=coord, grid_shape=shape, **kw)
    r1 = p1.nu2u(points=g["values"], forward=bool(g["forward"]))
    assert O.l2error(r1, g["nu2u"]) < eps
    p2 = nufft.plan(nu2u=False, coord=coord, grid_shape=shape, **kw)
    r2 = p2.u2nu(grid=g["grid_in"], forward=bool(g["forward"]))
    assert O.l2error(r2, g["u2nu"]) < eps


def test_zero_points():
    out = np.ones((16, 16), np.complex64)
    nufft.nu2u(points=np.zeros(0, np.complex64), coord=np.zeros((0, 2), np.float32),
               forward=True, epsilon=1e-5, out=out)
    assert np.all(out == 0)
    r = nufft.u2nu(grid=np.ones((16, 16), np.complex64), coord=np.zeros((0, 2), np.float32),
                   forward=True, epsilon=1e-5)
    assert r.shape == (0,)


def test_strided_device_arrays():
    import torch
    rng = np.random.default_rng(3)
    M, N = 500, (40, 44)
    coord = (rng.random((M, 2)) - 0.5) * 2 * np.pi
    vals = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    # coords as a transposed view, values with stride 2, output as a transposed view
    ct = torch.from_numpy(coord.T.copy()).cuda().t()
    vt = torch.from_numpy(np.repeat(vals, 2)).cuda()[::2]
    ot = torch.zeros((N[1], N[0]), dtype=torch.complex128, device="cuda").t()
    nufft.nu2u(points=vt, coord=ct, forward=True, epsilon=1e-9, out=ot)
    ref = O.direct_nu2u(coord, vals, N, True)
    assert O.l2error(ot.cpu().numpy(), ref) < 2e-9


def test_coordinates_far_outside_period():
    rng = np.random.default_rng(4)
    M, N = 300, (30, 31)
    coord = (rng.random((M, 2)) - 0.5) * 2 * np.pi * 50
    vals = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    out = np.empty(N, np.complex128)
    nufft.nu2u(points=vals, coord=coord, forward=False, epsilon=1e-10, out=out)
    assert O.l2error(out, O.direct_nu2u(coord, vals, N, False)) < 2e-10


def test_cfg1_full_size_vs_oracle():
    """2D type 1, M=2e5 float64 coords, 256^2 complex128, eps=1e-6."""
    rng = np.random.default_rng(11)
    M = 200000
    coord = rng.uniform(-np.pi, np.pi, (M, 2))
    vals = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    out = np.empty((256, 256), np.complex128)
    nufft.nu2u(points=vals, coord=coord, forward=True, epsilon=1e-6, out=out)
    p = O.Params((256, 256), 1e-6, False, M, True, 1)
    ref = O.nu2u(p, coord, vals, True)
    # same kernel, FP64 both: agreement to rounding
    assert O.l2error(out, ref) < 1e-12
    # and against the exact transform on a few rows of modes
    ku = np.arange(100, 104) - 128
    kv = np.arange(256) - 128
    eu = np.exp(-1j * np.outer(coord[:, 0], ku))
    ev = np.exp(-1j * np.outer(coord[:, 1], kv))
    exact = np.einsum("m,mi,mj->ij", vals, eu, ev, optimize=True)
    assert O.l2error(out[100:104], exact) < 1e-6


@pytest.mark.parametrize("shape,single", [((37,), False), ((40, 33), True), ((40, 33), False),
                                          ((12, 10, 14), True)])
@pytest.mark.parametrize("device", [False, True])
def test_plan_ntrans(shape, single, device):
    """Several transforms over one plan's points in one call (a leading ntrans
    axis): each equals the single-transform call."""
    rng = np.random.default_rng(31)
    M, nt = 3000, 3
    cdt, vdt = (np.float32, np.complex64) if single else (np.float64, np.complex128)
    eps = 1e-5 if single else 1e-10
    coord = rng.uniform(-np.pi, np.pi, (M, len(shape))).astype(cdt)
    vals = (rng.standard_normal((nt, M)) + 1j * rng.standard_normal((nt, M))).astype(vdt)
    grid = (rng.standard_normal((nt,) + shape) + 1j * rng.standard_normal((nt,) + shape)).astype(vdt)
    conv = torch_dev if device else (lambda x: x)
    back = (lambda x: x.cpu().numpy()) if device else (lambda x: x)
    p1 = nufft.plan(nu2u=True, coord=conv(coord), grid_shape=shape, epsilon=eps)
    r1 = back(p1.nu2u(points=conv(vals), forward=True))
    r2 = back(p1.u2nu(grid=conv(grid), forward=False))
    assert r1.shape == (nt,) + shape and r2.shape == (nt, M)
    # the spreaders add with atomics, whose order varies from call to call:
    # repeated single precision transforms agree to rounding, not bit for bit
    same = 1e-6 if single else 1e-12
    for t in range(nt):
        assert O.l2error(r1[t], back(p1.nu2u(points=conv(vals[t]), forward=True))) < same
        assert O.l2error(r2[t], back(p1.u2nu(grid=conv(grid[t]), forward=False))) < same
        ref = O.direct_nu2u(coord.astype(np.float64), vals[t], shape, True)
        assert O.l2error(r1[t], ref) < 4 * eps
    with pytest.raises(RuntimeError, match="leading extent"):
        p1.nu2u(points=conv(vals), forward=True, out=conv(np.empty((nt + 1,) + shape, vdt)))

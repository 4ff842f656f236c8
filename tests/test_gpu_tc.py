"""The split-precision tensor-core spreader (spreader='tc') against the plain
FP32 spreader and the FP64 oracle: same transform, same kernel, errors at the
FP32 level (DUCC's single-precision path reaches ~2e-7 relative L2)."""
import numpy as np
import pytest

from ducc_b200 import nufft
from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu


def run(spreader, coord, vals, shape, eps, **kw):
    out = np.empty(shape, np.complex64)
    nufft.nu2u(points=vals, coord=coord, forward=True, epsilon=eps, out=out, spreader=spreader,
               **kw)
    return out


@pytest.mark.parametrize("eps", [1e-2, 1e-3, 1e-4, 1e-5, 1e-6])
@pytest.mark.parametrize("shape", [(64, 48), (200, 300), (17, 1)])
def test_tc_matches_plain_and_oracle(eps, shape):
    rng = np.random.default_rng(5)
    M = 20000
    coord = rng.uniform(-np.pi, np.pi, (M, 2)).astype(np.float32)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
    a = run("tc", coord, vals, shape, eps)
    b = run("plain", coord, vals, shape, eps)
    p = O.Params(shape, eps, True, M, True, 1)
    ref = O.nu2u(p, coord, vals, True)
    ea, eb = O.l2error(a, ref), O.l2error(b, ref)
    assert ea < max(eps, 1e-6), (ea, eb)
    assert ea < 3 * eb + 5e-7, (ea, eb)


@pytest.mark.parametrize("scale", [1e-30, 1e-6, 1.0, 1e20])
def test_tc_value_scaling(scale):
    rng = np.random.default_rng(6)
    M, shape = 5000, (96, 96)
    coord = rng.uniform(-np.pi, np.pi, (M, 2)).astype(np.float32)
    vals = ((rng.standard_normal(M) + 1j * rng.standard_normal(M)) * scale).astype(np.complex64)
    a = run("tc", coord, vals, shape, 1e-5)
    b = run("plain", coord, vals, shape, 1e-5)
    assert O.l2error(a, b) < 2e-6


def test_tc_clustered_heavy_tiles():
    """Many points per tile: chunks split at 1024 points, many MMA rounds."""
    rng = np.random.default_rng(7)
    M, shape = 200000, (256, 256)
    cen = rng.uniform(-np.pi, np.pi, (4, 2))
    coord = (cen[rng.integers(0, 4, M)] + 0.05 * rng.standard_normal((M, 2)))
    coord = (np.mod(coord + np.pi, 2 * np.pi) - np.pi).astype(np.float32)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
    a = run("tc", coord, vals, shape, 1e-6)
    p = O.Params(shape, 1e-6, True, M, True, 1)
    ref = O.nu2u(p, coord, vals, True)
    assert O.l2error(a, ref) < 1e-6


def test_tc_planned_and_periodicity():
    rng = np.random.default_rng(8)
    M, shape = 30000, (120, 130)
    coord = rng.uniform(-3, 5, (M, 2)).astype(np.float32)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
    pl = nufft.plan(nu2u=True, coord=coord, grid_shape=shape, epsilon=1e-5,
                    periodicity=[2.0, 3.0], fft_order=True, spreader="tc")
    a = pl.nu2u(points=vals, forward=False)
    ref = O.direct_nu2u(coord, vals, shape, False, [2.0, 3.0], True)
    assert O.l2error(a, ref) < 2e-5


def test_tc_rejects_double():
    coord = np.zeros((10, 2))
    with pytest.raises(RuntimeError, match="tensor-core"):
        nufft.nu2u(points=np.zeros(10, np.complex128), coord=coord, forward=True, epsilon=1e-5,
                   out=np.zeros((8, 8), np.complex128), spreader="tc")


def test_tc_plan_permutation_is_duccs():
    """A tensor-core plan processes points in (tile, quadrant) order but still
    reports DUCC's stable tile permutation."""
    import os
    g = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "g2d_f32.npz")))
    shape = tuple(int(s) for s in g["shape"])
    for spreader in ("tc", "plain"):
        p = nufft.plan(nu2u=True, coord=g["coord"], grid_shape=shape, epsilon=float(g["eps"]),
                       nthreads=1, sigma_min=1.2, sigma_max=2.51,
                       periodicity=list(g["periodicity"]), spreader=spreader)
        assert np.array_equal(p.permutation(), g["perm1"])
        r = p.nu2u(points=g["values"], forward=bool(g["forward"]))
        assert O.l2error(r, g["nu2u"]) < float(g["eps"])
        r2 = p.u2nu(grid=g["grid_in"], forward=bool(g["forward"]))
        assert O.l2error(r2, g["u2nu"]) < float(g["eps"])


def test_tc_one_tile_long_accumulation_chains():
    """Every point in one tile quadrant: 4096-point chunks with 256 K-blocks
    into one accumulator, so the chain bound (drain into FP32 shared memory)
    is what keeps the error at the plain spreader's level."""
    rng = np.random.default_rng(9)
    M, shape = 300000, (64, 64)
    coord = (0.3 + 1e-3 * rng.standard_normal((M, 2))).astype(np.float32)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
    a = run("tc", coord, vals, shape, 1e-6)
    b = run("plain", coord, vals, shape, 1e-6)
    p = O.Params(shape, 1e-6, True, M, True, 1)
    ref = O.nu2u(p, coord, vals, True)
    ea, eb = O.l2error(a, ref), O.l2error(b, ref)
    assert ea < 3 * eb + 5e-7, (ea, eb)

"""The CPU oracle against DUCC: golden fixtures (always) and the compiled
reference (when oracle/_ref is built).  No GPU needed."""
import glob
import os

import numpy as np
import pytest

from oracle import nufft_oracle as O
from oracle import ref

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "g*.npz")))


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def params_for(g, gridding):
    shape = tuple(int(s) for s in g["shape"])
    k = "1" if gridding else "2"
    return O.Params(shape, float(g["eps"]), bool(g["singleprec"]), g["coord"].shape[0],
                    gridding, periodicity=list(g["periodicity"]),
                    force=(int(g["kidx" + k]), list(g["nover" + k])))


def test_kernel_table_matches_golden():
    rows = np.load(os.path.join(GOLD, "kernel_db.npz"))["rows"]
    mine = np.array([r[:6] + (float(r[6]),) for r in O.kernel_db()])
    assert rows.shape == mine.shape
    assert np.array_equal(rows, mine)


@pytest.mark.parametrize("name", CASES)
def test_parameter_choice_matches(name):
    g = load(name)
    shape = tuple(int(s) for s in g["shape"])
    for gridding, k in ((True, "1"), (False, "2")):
        kidx, nover = O.find_parameters(float(g["eps"]), 1.2, 2.51, shape,
                                        g["coord"].shape[0], gridding, 1,
                                        bool(g["singleprec"]))
        assert kidx == int(g["kidx" + k])
        assert list(nover) == list(g["nover" + k])


@pytest.mark.parametrize("name", CASES)
def test_index_bit_exact(name):
    g = load(name)
    p = params_for(g, True)
    i0, _ = O.getpix(p, g["coord"])
    assert np.array_equal(i0, g["i0_1"])
    assert np.array_equal(O.permutation(p, g["coord"]), g["perm1"])
    p2 = params_for(g, False)
    assert np.array_equal(O.permutation(p2, g["coord"]), g["perm2"])


@pytest.mark.parametrize("name", CASES)
def test_transforms_match_ducc(name):
    g = load(name)
    eps = float(g["eps"])
    fwd = bool(g["forward"])
    fo = bool(g["fft_order"])
    p = params_for(g, True)
    r1 = O.nu2u(p, g["coord"], g["values"], fwd, fo)
    # ducc computes in the data precision; the oracle in FP64
    assert O.l2error(r1, g["nu2u"]) < max(2 * eps, 1e-12)
    p2 = params_for(g, False)
    r2 = O.u2nu(p2, g["grid_in"], g["coord"], fwd, fo)
    assert O.l2error(r2, g["u2nu"]) < max(2 * eps, 1e-12)


@pytest.mark.parametrize("name", ["g1d_f64", "g2d_f64", "g3d_f64", "g2d_f32"])
def test_oracle_vs_direct(name):
    g = load(name)
    eps = float(g["eps"])
    fwd = bool(g["forward"])
    fo = bool(g["fft_order"])
    shape = tuple(int(s) for s in g["shape"])
    per = list(g["periodicity"])
    p = params_for(g, True)
    d1 = O.direct_nu2u(g["coord"], g["values"], shape, fwd, per, fo)
    assert O.l2error(O.nu2u(p, g["coord"], g["values"], fwd, fo), d1) < 2 * eps
    d2 = O.direct_u2nu(g["grid_in"], g["coord"], fwd, per, fo)
    p2 = params_for(g, False)
    assert O.l2error(O.u2nu(p2, g["grid_in"], g["coord"], fwd, fo), d2) < 2 * eps


def test_adjointness_oracle():
    g = load("g2d_f64")
    p = params_for(g, True)
    fwd = bool(g["forward"])
    a = O.nu2u(p, g["coord"], g["values"], fwd)
    b = O.u2nu(params_for(g, False), g["grid_in"], g["coord"], not fwd)
    lhs = O.vdot(g["values"], b)
    rhs = O.vdot(a, g["grid_in"])
    assert abs(lhs - rhs) < 1e-12 * max(abs(lhs), 1.0) * 100


def test_longdouble_fold_boundary():
    """Float64 coordinates fold in x87 long double: a value whose product with
    n lies just below an integer must not be rounded up by double arithmetic."""
    p = O.Params((4096,), 1e-9, False, 1, True)
    n = p.nover[0]
    # f*n = 1234 - tiny: representable in long double but rounds to 1234 in double
    f = np.nextafter(1234.0 / n, 0.0)
    coord = np.array([[f / p.coordfct[0]]])
    i0, frac = O.getpix(p, coord)
    tmp = coord[0, 0] * p.coordfct[0]
    tmp2 = np.longdouble(tmp - np.floor(tmp)) * np.longdouble(n)
    assert i0[0, 0] == min(int(tmp2 + np.longdouble(p.shift[0])) - n, p.maxi0[0])


@pytest.mark.skipif(ref.load() is None, reason="reference module not built")
def test_kernel_table_matches_reference():
    R = ref.load()
    assert [tuple(r) for r in R.kernel_db()] == [tuple(r) for r in O.kernel_db()]


@pytest.mark.skipif(ref.load() is None, reason="reference module not built")
@pytest.mark.parametrize("cdt", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(300,), (70, 90), (20, 24, 28)])
def test_index_vs_reference_random(cdt, shape):
    R = ref.load()
    rng = np.random.default_rng(7)
    M = 5000
    ndim = len(shape)
    coord = ((rng.random((M, ndim)) - 0.5) * 40).astype(cdt)
    sp = cdt == np.float32
    pr = R.index_probe(coord=coord, shape=list(shape), epsilon=1e-5, singleprec=sp,
                       gridding=True, nthreads=1, sigma_min=1.2, sigma_max=2.51,
                       periodicity=[2 * np.pi] * ndim)
    p = O.Params(shape, 1e-5, sp, M, True, 1, vlen=8 if sp else ref.simd_lanes_double())
    assert p.nover == list(pr["nover"])
    i0, _ = O.getpix(p, coord)
    assert np.array_equal(i0, pr["i0"])
    assert np.array_equal(O.permutation(p, coord), pr["coord_idx"])

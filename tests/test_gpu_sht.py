"""Spin-0 synthesis at arbitrary points and its adjoint on the GPU
(ducc_b200.sht) against the direct sums of oracle/sht_oracle.py, against the
golden fixtures made by DUCC itself, and against DUCC's compiled sht module
(oracle/_ref, where it was built) at sizes the direct sums cannot reach.

Restated from DUCC's python/test/test_sht.py (spin 0; nthreads only feeds
the cost model):
  test_adjointness_general   test_sht.py:234-262 (rtol 1e-9 at epsilon 1e-5)
  test_synthesis_general     test_sht.py:265-281 (l2 error below epsilon 1e-7)
"""
import glob
import os

import numpy as np
import pytest

from oracle import sht_oracle as O

pytestmark = pytest.mark.gpu
pmp = pytest.mark.parametrize
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def sht():
    from ducc_b200 import sht
    return sht


def l2err(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2))


def locs(rng, n, edges=True):
    loc = np.stack([rng.uniform(0., np.pi, n), rng.uniform(0., 2 * np.pi, n)], 1)
    if edges and n >= 6:
        # both poles, the equator, phi at both ends of its range
        loc[:6] = [[0., 0.3], [np.pi, 1.1], [np.pi / 2, 0.], [np.pi / 2, 2 * np.pi],
                   [0., 2 * np.pi], [1e-9, 4.]]
    return loc


def healpix_ring_centres(nside):
    """Pixel centres of the HEALPix RING scheme (theta, phi), the point set of
    DUCC's test_synthesis_general."""
    th, ph = [], []
    for i in range(1, 4 * nside):          # rings north to south
        if i < nside:
            z = 1 - i * i / (3. * nside * nside)
            n, shift = 4 * i, 0.5
        elif i <= 3 * nside:
            z = (2 * nside - i) * 2. / (3 * nside)
            n, shift = 4 * nside, 0.5 * ((i - nside + 1) % 2)
        else:
            k = 4 * nside - i
            z = -(1 - k * k / (3. * nside * nside))
            n, shift = 4 * k, 0.5
        t = np.arccos(z)
        th += [t] * n
        ph += list((np.arange(n) + shift) * 2 * np.pi / n)
    return np.stack([np.array(th), np.array(ph)], 1)


# ---------------------------------------------------------------- DUCC's tests
@pmp("lmmax", ((10, 8), (100, 100)))
@pmp("nside", (32,))
@pmp("nthreads", (1, 4))
def test_synthesis_general(sht, lmmax, nside, nthreads):
    rng = np.random.default_rng(48)
    lmax, mmax = lmmax
    epsilon = 1e-7
    slm = O.random_alm(lmax, mmax, rng)[None, :]
    loc = healpix_ring_centres(nside)
    assert loc.shape[0] == 12 * nside * nside
    v1 = sht.synthesis_general(lmax=lmax, mmax=mmax, alm=slm, loc=loc, spin=0,
                               epsilon=epsilon, nthreads=nthreads)
    v2 = O.synthesis(slm[0], lmax, mmax, loc)
    assert l2err(v1[0], v2) < epsilon


@pmp("nthreads", (1, 4))
@pmp("npix", (33, 200))
@pmp("lmmax", ((10, 8), (100, 100)))
def test_adjointness_general(sht, lmmax, npix, nthreads):
    rng = np.random.default_rng(48)
    lmax, mmax = lmmax
    epsilon = 1e-5
    slm1 = O.random_alm(lmax, mmax, rng)[None, :]
    loc = rng.uniform(0., 1., (npix, 2))
    loc[:, 0] *= np.pi
    loc[:, 1] *= 2 * np.pi
    points2 = rng.uniform(-0.5, 0.5, (loc.shape[0], 1)).T
    points1 = sht.synthesis_general(lmax=lmax, mmax=mmax, alm=slm1, loc=loc, spin=0,
                                    epsilon=epsilon, nthreads=nthreads)
    slm2 = sht.adjoint_synthesis_general(lmax=lmax, mmax=mmax, map=points2, loc=loc, spin=0,
                                         epsilon=epsilon, nthreads=nthreads)
    v1 = O.almdot(slm1[0], slm2[0], lmax)
    v2 = np.dot(points2[0], points1[0])
    np.testing.assert_allclose(v1, v2, rtol=1e-9)


# ---------------------------------------------------------------- direct sums
CASES = [
    # lmax, mmax, npoints, precision, epsilon
    (0, 0, 20, np.complex128, 1e-10),
    (1, 1, 40, np.complex128, 1e-12),
    (7, 0, 50, np.complex128, 1e-9),
    (13, 9, 300, np.complex128, 1e-11),
    (64, 64, 500, np.complex128, 1e-12),
    (150, 40, 400, np.complex128, 1e-8),
    (31, 31, 500, np.complex64, 1e-5),
    (90, 77, 700, np.complex64, 2e-6),
]


@pmp("case", CASES)
def test_against_direct_sums(sht, case):
    lmax, mmax, npts, cdt, eps = case
    rng = np.random.default_rng(lmax * 1000 + mmax)
    alm = O.random_alm(lmax, mmax, rng).astype(cdt)[None, :]
    loc = locs(rng, npts)
    rdt = np.float64 if cdt == np.complex128 else np.float32
    m1 = sht.synthesis_general(alm=alm, spin=0, lmax=lmax, mmax=mmax, loc=loc, epsilon=eps)
    assert m1.dtype == rdt and m1.shape == (1, npts)
    assert l2err(m1[0], O.synthesis(alm[0], lmax, mmax, loc)) < eps
    mp = rng.uniform(-1, 1, (1, npts)).astype(rdt)
    a1 = sht.adjoint_synthesis_general(map=mp, spin=0, lmax=lmax, mmax=mmax, loc=loc,
                                       epsilon=eps)
    assert a1.dtype == cdt and a1.shape == (1, O.nalm(lmax, mmax))
    ref = O.adjoint_synthesis(mp[0], lmax, mmax, loc)
    assert l2err(a1[0], ref) < eps
    assert np.all(a1[0, :lmax + 1].imag == 0)


def test_custom_layout(sht):
    """a_lm at mstart[m] + l * lstride with lstride 2 and a gap between m blocks."""
    rng = np.random.default_rng(5)
    lmax, mmax, npts, eps = 20, 12, 300, 1e-11
    ms = np.zeros(mmax + 1, np.int64)
    ofs = 3
    for m in range(mmax + 1):
        ms[m] = ofs - 2 * m
        ofs += 2 * (lmax + 1 - m) + 5
    size = ofs
    alm = np.zeros((1, size), np.complex128)
    dense = O.random_alm(lmax, mmax, rng)
    dms = O.default_mstart(lmax, mmax)
    for m in range(mmax + 1):
        ls = np.arange(m, lmax + 1)
        alm[0, ms[m] + 2 * ls] = dense[dms[m] + ls]
    loc = locs(rng, npts)
    m1 = sht.synthesis_general(alm=alm, spin=0, lmax=lmax, loc=loc, epsilon=eps, mstart=ms,
                               lstride=2)
    assert l2err(m1[0], O.synthesis(dense, lmax, mmax, loc)) < eps
    mp = rng.uniform(-1, 1, (1, npts))
    out = np.full((1, size), 7. + 7.j)
    sht.adjoint_synthesis_general(map=mp, spin=0, lmax=lmax, loc=loc, epsilon=eps, mstart=ms,
                                  lstride=2, alm=out)
    ref = O.adjoint_synthesis(mp[0], lmax, mmax, loc)
    got = np.zeros_like(ref)
    for m in range(mmax + 1):
        ls = np.arange(m, lmax + 1)
        got[dms[m] + ls] = out[0, ms[m] + 2 * ls]
    assert l2err(got, ref) < eps
    # entries outside the layout keep their values
    touched = np.zeros(size, bool)
    for m in range(mmax + 1):
        touched[ms[m] + 2 * np.arange(m, lmax + 1)] = True
    assert np.all(out[0, ~touched] == 7. + 7.j)


def test_golden_fixtures(sht):
    files = sorted(glob.glob(os.path.join(HERE, "golden", "sht_*.npz")))
    assert files
    for fn in files:
        g = np.load(fn)
        lmax, mmax = int(g["lmax"]), int(g["mmax"])
        f64 = g["alm"].dtype == np.complex128
        eps = 1e-11 if f64 else 1e-5
        m1 = sht.synthesis_general(alm=g["alm"], spin=0, lmax=lmax, mmax=mmax, loc=g["loc"],
                                   epsilon=eps)
        assert l2err(m1, g["synthesis"]) < eps, fn
        a1 = sht.adjoint_synthesis_general(map=g["map_in"], spin=0, lmax=lmax, mmax=mmax,
                                           loc=g["loc"], epsilon=eps)
        assert l2err(a1, g["adjoint"]) < eps, fn


def test_device_tensors_in_place(sht):
    import torch
    rng = np.random.default_rng(9)
    lmax, mmax, npts, eps = 30, 20, 400, 1e-10
    alm = O.random_alm(lmax, mmax, rng)[None, :]
    loc = locs(rng, npts)
    d_alm = torch.from_numpy(alm).cuda()
    d_loc = torch.from_numpy(loc).cuda()
    d_map = torch.zeros((1, npts), dtype=torch.float64, device="cuda")
    r = sht.synthesis_general(alm=d_alm, spin=0, lmax=lmax, mmax=mmax, loc=d_loc, epsilon=eps,
                              map=d_map)
    assert r is d_map
    assert l2err(d_map.cpu().numpy()[0], O.synthesis(alm[0], lmax, mmax, loc)) < eps
    # strided (non-contiguous) location columns
    wide = torch.zeros((npts, 3), dtype=torch.float64, device="cuda")
    wide[:, 0:2] = d_loc
    r2 = sht.synthesis_general(alm=d_alm, spin=0, lmax=lmax, mmax=mmax, loc=wide[:, 0:2],
                               epsilon=eps)
    assert torch.allclose(r2, d_map, rtol=0, atol=1e-12)


def test_errors(sht):
    rng = np.random.default_rng(1)
    alm = O.random_alm(10, 10, rng)[None, :]
    loc = locs(rng, 10)
    with pytest.raises(RuntimeError, match="spin"):
        sht.synthesis_general(alm=np.concatenate([alm, alm]), spin=1, lmax=10, loc=loc)
    with pytest.raises(RuntimeError):
        sht.synthesis_general(alm=alm[:, :-3], spin=0, lmax=10, loc=loc)
    with pytest.raises(RuntimeError):
        sht.synthesis_general(alm=alm, spin=0, lmax=10, loc=loc, mmax=11)
    with pytest.raises(RuntimeError):
        sht.synthesis_general(alm=alm, spin=0, lmax=10, loc=loc[:, :1].copy())
    with pytest.raises(RuntimeError):
        sht.synthesis_general(alm=alm, spin=0, lmax=10, loc=loc, epsilon=1e-30)
    with pytest.raises(TypeError):
        sht.synthesis_general(alm=alm, spin=0, lmax=10, loc=loc.astype(np.float32))
    # no points: an empty map, an all-zero adjoint
    e = sht.synthesis_general(alm=alm, spin=0, lmax=10, loc=np.zeros((0, 2)))
    assert e.shape == (1, 0)
    a = sht.adjoint_synthesis_general(map=np.zeros((1, 0)), spin=0, lmax=10, loc=np.zeros((0, 2)))
    assert a.shape == (1, O.nalm(10, 10)) and not np.any(a)


# ---------------------------------------------------------------- against DUCC, large
@pytest.fixture(scope="module")
def ducc():
    from oracle import ref
    m = ref.load()
    if m is None or not hasattr(m, "sht"):
        pytest.skip("DUCC's sht module (oracle/_ref) not built")
    return m.sht


@pmp("lmax,mmax,npts,cdt,eps", [
    (1023, 1023, 200000, np.complex128, 1e-10),
    (1023, 700, 200000, np.complex64, 1e-5),
    (4095, 4095, 50000, np.complex128, 1e-9),
])
def test_against_ducc_large(sht, ducc, lmax, mmax, npts, cdt, eps):
    """Sizes where the Legendre recurrence needs its carried exponent
    (sin^m theta below the double range for m in the thousands)."""
    rng = np.random.default_rng(lmax + npts)
    alm = O.random_alm(lmax, mmax, rng).astype(cdt)[None, :]
    loc = locs(rng, npts)
    nthr = os.cpu_count() or 1
    m1 = sht.synthesis_general(alm=alm, spin=0, lmax=lmax, mmax=mmax, loc=loc, epsilon=eps)
    m2 = ducc.synthesis_general(alm=alm.astype(np.complex128), spin=0, lmax=lmax, mmax=mmax,
                                loc=loc, epsilon=min(eps, 1e-12), nthreads=nthr)
    assert l2err(m1, m2) < eps
    rdt = np.float64 if cdt == np.complex128 else np.float32
    mp = rng.uniform(-1, 1, (1, npts)).astype(rdt)
    a1 = sht.adjoint_synthesis_general(map=mp, spin=0, lmax=lmax, mmax=mmax, loc=loc,
                                       epsilon=eps)
    a2 = ducc.adjoint_synthesis_general(map=mp.astype(np.float64), spin=0, lmax=lmax,
                                        mmax=mmax, loc=loc, epsilon=min(eps, 1e-12),
                                        nthreads=nthr)
    assert l2err(a1, a2) < eps

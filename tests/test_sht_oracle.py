"""The spin-0 spherical-harmonic oracle (oracle/sht_oracle.py) pinned against
DUCC: the golden fixtures made by DUCC's own synthesis_general /
adjoint_synthesis_general (tests/golden/make_golden_sht.py), its adjointness
(DUCC's test_sht.py:234-262 definition of the alm inner product), and, where
DUCC's compiled sht module is present (oracle/_ref), a fresh comparison."""
import glob
import os

import numpy as np
import pytest

from oracle import sht_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def l2err(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2))


def test_oracle_against_golden():
    files = sorted(glob.glob(os.path.join(HERE, "golden", "sht_*.npz")))
    assert len(files) >= 4
    for fn in files:
        g = np.load(fn)
        lmax, mmax = int(g["lmax"]), int(g["mmax"])
        tol = max(10 * float(g["eps"]), 1e-13)
        s = O.synthesis(g["alm"][0], lmax, mmax, g["loc"])
        a = O.adjoint_synthesis(g["map_in"][0], lmax, mmax, g["loc"])
        assert l2err(s, g["synthesis"][0]) < tol, fn
        assert l2err(a, g["adjoint"][0]) < tol, fn


@pytest.mark.parametrize("lmax,mmax", [(0, 0), (5, 5), (12, 3), (40, 40)])
def test_oracle_adjointness(lmax, mmax):
    rng = np.random.default_rng(lmax + 7 * mmax)
    alm = O.random_alm(lmax, mmax, rng)
    loc = np.stack([rng.uniform(0, np.pi, 60), rng.uniform(0, 2 * np.pi, 60)], 1)
    f = rng.uniform(-0.5, 0.5, 60)
    v1 = O.almdot(alm, O.adjoint_synthesis(f, lmax, mmax, loc), lmax)
    v2 = np.dot(f, O.synthesis(alm, lmax, mmax, loc))
    np.testing.assert_allclose(v1, v2, rtol=1e-12)


def test_oracle_known_values():
    """Y_00 = 1/sqrt(4 pi); Y_10 = sqrt(3/(4 pi)) cos theta;
    Y_11 = -sqrt(3/(8 pi)) sin theta e^{i phi} (Condon-Shortley)."""
    loc = np.array([[0.3, 1.2], [2.0, 5.0]])
    th, ph = loc[:, 0], loc[:, 1]
    # a_00 = 1
    np.testing.assert_allclose(O.synthesis(np.array([1, 0, 0]), 1, 1, loc),
                               np.full(2, 1 / np.sqrt(4 * np.pi)), rtol=1e-14)
    np.testing.assert_allclose(O.synthesis(np.array([0, 1, 0]), 1, 1, loc),
                               np.sqrt(3 / (4 * np.pi)) * np.cos(th), rtol=1e-14)
    y11 = -np.sqrt(3 / (8 * np.pi)) * np.sin(th) * np.exp(1j * ph)
    np.testing.assert_allclose(O.synthesis(np.array([0, 0, 1j]), 1, 1, loc),
                               2 * (1j * y11).real, rtol=1e-13)


def test_oracle_against_ducc_fresh():
    from oracle import ref
    R = ref.load()
    if R is None or not hasattr(R, "sht"):
        pytest.skip("DUCC's sht module (oracle/_ref) not built")
    rng = np.random.default_rng(3)
    lmax, mmax, n = 60, 45, 250
    alm = O.random_alm(lmax, mmax, rng)
    loc = np.stack([rng.uniform(0, np.pi, n), rng.uniform(0, 2 * np.pi, n)], 1)
    d = R.sht.synthesis_general(alm=alm[None], spin=0, lmax=lmax, mmax=mmax, loc=loc,
                                epsilon=1e-13)
    assert l2err(O.synthesis(alm, lmax, mmax, loc), d[0]) < 1e-12
    f = rng.uniform(-1, 1, (1, n))
    da = R.sht.adjoint_synthesis_general(map=f, spin=0, lmax=lmax, mmax=mmax, loc=loc,
                                         epsilon=1e-13)
    assert l2err(O.adjoint_synthesis(f[0], lmax, mmax, loc), da[0]) < 1e-12

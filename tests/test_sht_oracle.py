"""The spin-0 spherical-harmonic oracle (oracle/sht_oracle.py) pinned against
DUCC: the golden fixtures made by DUCC's own synthesis_general /
adjoint_synthesis_general (tests/golden/make_golden_sht.py; spin 0 to 3, the
modes STANDARD, GRAD_ONLY and DERIV1), its adjointness (DUCC's
test_sht.py:234-262 definition of the alm inner product), and, where
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
    assert len(files) >= 9
    for fn in files:
        g = np.load(fn)
        lmax, mmax, spin = int(g["lmax"]), int(g["mmax"]), int(g["spin"])
        tol = max(10 * float(g["eps"]), 1e-13)
        if spin == 0:
            s = O.synthesis(g["alm"][0], lmax, mmax, g["loc"])[None]
            a = O.adjoint_synthesis(g["map_in"][0], lmax, mmax, g["loc"])[None]
        else:
            mode = str(g["mode"])
            s = O.synthesis_spin(g["alm"], spin, lmax, mmax, g["loc"], mode)
            a = O.adjoint_synthesis_spin(g["map_in"], spin, lmax, mmax, g["loc"], mode)
        assert l2err(s, g["synthesis"]) < tol, fn
        assert l2err(a, g["adjoint"]) < tol, fn


def test_spin_recurrence_against_wigner_sum():
    """The oracle's Wigner-d recurrence against Wigner's explicit sum (small l,
    where the sum does not cancel), every m for spins 1..3."""
    th = np.linspace(0, np.pi, 9)
    for s in (1, 2, 3):
        for m in range(-8, 9):
            D = O.spin_D_all(10, m, s, th)
            for l in range(max(abs(m), s), 11):
                ref = np.sqrt((2 * l + 1) / (4 * np.pi)) * O.wigner_d(l, m, -s, th)
                assert np.abs(D[l] - ref).max() < 1e-11


@pytest.mark.parametrize("spin,mode", [(1, "STANDARD"), (2, "STANDARD"), (2, "GRAD_ONLY"),
                                       (1, "DERIV1")])
def test_oracle_spin_adjointness(spin, mode):
    rng = np.random.default_rng(spin + 11)
    lmax, mmax, n = 15, 11, 70
    nc = 2 if mode == "STANDARD" else 1
    alm = O.random_alm_spin(lmax, mmax, spin, nc, rng)
    loc = np.stack([rng.uniform(0, np.pi, n), rng.uniform(0, 2 * np.pi, n)], 1)
    p = rng.uniform(-0.5, 0.5, (2, n))
    a2 = O.adjoint_synthesis_spin(p, spin, lmax, mmax, loc, mode)
    v1 = sum(O.almdot(alm[c], a2[c], lmax) for c in range(nc))
    v2 = np.sum(p * O.synthesis_spin(alm, spin, lmax, mmax, loc, mode))
    np.testing.assert_allclose(v1, v2, rtol=1e-12)


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
    alm2 = O.random_alm_spin(lmax, mmax, 2, 2, rng)
    d = R.sht.synthesis_general(alm=alm2, spin=2, lmax=lmax, mmax=mmax, loc=loc, epsilon=1e-13)
    assert l2err(O.synthesis_spin(alm2, 2, lmax, mmax, loc), d) < 1e-12
    p = rng.uniform(-1, 1, (2, n))
    da = R.sht.adjoint_synthesis_general(map=p, spin=2, lmax=lmax, mmax=mmax, loc=loc,
                                         epsilon=1e-13)
    assert l2err(O.adjoint_synthesis_spin(p, 2, lmax, mmax, loc), da) < 1e-12

"""The host-side LSMR of ducc_b200.sht (the solver of pseudo_analysis_general)
against SciPy's LSMR (the same published algorithm) on small dense systems,
with numpy arrays as the vectors."""
import numpy as np
import pytest

scipy_lsmr = pytest.importorskip("scipy.sparse.linalg").lsmr


@pytest.mark.parametrize("shape,seed", [((60, 20), 0), ((40, 40), 1), ((200, 35), 2)])
def test_lsmr_matches_scipy(shape, seed):
    from ducc_b200.sht import lsmr
    rng = np.random.default_rng(seed)
    A = rng.standard_normal(shape)
    b = rng.standard_normal(shape[0])
    x, istop, itn, normr, normar, normA, condA, normx, normb = lsmr(
        lambda v: A @ v, lambda u: A.T @ u, np.linalg.norm, np.linalg.norm, b,
        np.zeros(shape[1]), 0., 1e-10, 1e-10, 1e8, 500)
    r = scipy_lsmr(A, b, atol=1e-10, btol=1e-10, conlim=1e8, maxiter=500)
    assert istop == r[1] and itn == r[2]
    np.testing.assert_allclose(x, r[0], rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose([normr, normar, normA, condA, normx],
                               [r[3], r[4], r[5], r[6], r[7]], rtol=1e-8)
    xls = np.linalg.lstsq(A, b, rcond=None)[0]
    np.testing.assert_allclose(x, xls, rtol=1e-6, atol=1e-8)


def test_lsmr_zero_rhs():
    from ducc_b200.sht import lsmr
    A = np.eye(5)
    x, istop, itn = lsmr(lambda v: A @ v, lambda u: A.T @ u, np.linalg.norm, np.linalg.norm,
                         np.zeros(5), np.zeros(5))[:3]
    assert itn == 0 and istop == 0 and not np.any(x)

"""Test infrastructure only (the checker, never the product): a CPU
restatement of DUCC's spin-0 ``synthesis_general`` / ``adjoint_synthesis_general``
as direct sums over the spherical harmonics, for sizes that finish in seconds.

Definitions (DUCC's, src/ducc0/sht/sht.cc:60-171 for the normalisation and
the Condon-Shortley sign of lambda_mm, sht.cc:2926-2994 for the two
functions): with a_lm stored at ``mstart[m] + l * lstride``,
    map(theta, phi) = sum_l a_l0 lambda_l0(theta)
                      + 2 Re sum_{m>0} sum_l a_lm lambda_lm(theta) e^{i m phi}
    a_lm = sum_i map_i lambda_lm(theta_i) e^{-i m phi_i}
where lambda_lm(theta) = Y_lm(theta, 0) is the orthonormal associated
Legendre function: lambda_mm = (-1)^m sqrt((2m+1)/(4 pi) prod_{k<=m}
(2k-1)/(2k)) sin^m theta, lambda_{m+1,m} = sqrt(2m+3) cos theta lambda_mm,
lambda_lm = alpha_l (cos theta lambda_{l-1,m} - beta_l lambda_{l-2,m}) with
alpha_l = sqrt((4l^2-1)/(l^2-m^2)), beta_l = sqrt(((l-1)^2-m^2)/(4(l-1)^2-1)).
Values below the double range (sin^m theta for large m near the poles) flush
to zero here, which is harmless at the small lmax this oracle is used for.
"""
import numpy as np


def default_mstart(lmax, mmax):
    """DUCC's default a_lm layout (python/sht_pymod.cc:124-134)."""
    ms = np.empty(mmax + 1, dtype=np.int64)
    idx = 0
    for m in range(mmax + 1):
        ms[m] = idx - m
        idx += lmax + 1 - m
    return ms


def nalm(lmax, mmax):
    return ((mmax + 1) * (mmax + 2)) // 2 + (mmax + 1) * (lmax - mmax)


def lambda_lm(lmax, m, theta):
    """lambda_lm(theta) for l = m .. lmax, shape (lmax - m + 1, len(theta))."""
    theta = np.asarray(theta, dtype=np.float64)
    x, s = np.cos(theta), np.sin(theta)
    nm = 1.0 / (4 * np.pi) * (2 * m + 1)
    for k in range(1, m + 1):
        nm *= (2 * k - 1) / (2 * k)
    out = np.zeros((lmax - m + 1, theta.size))
    lam = (-1) ** m * np.sqrt(nm) * s ** m
    out[0] = lam
    prev = np.zeros_like(lam)
    for l in range(m + 1, lmax + 1):
        alpha = np.sqrt((4.0 * l * l - 1) / (l * l - m * m))
        beta = np.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1) ** 2 - 1))
        new = alpha * (x * lam - beta * prev)
        prev, lam = lam, new
        out[l - m] = lam
    return out


def synthesis(alm, lmax, mmax, loc, mstart=None, lstride=1):
    """map (npoints,) of the spin-0 expansion alm (1D complex) at loc (n, 2)."""
    ms = default_mstart(lmax, mmax) if mstart is None else np.asarray(mstart)
    alm = np.asarray(alm).astype(np.complex128)
    theta, phi = loc[:, 0], loc[:, 1]
    res = np.zeros(theta.size)
    for m in range(mmax + 1):
        lam = lambda_lm(lmax, m, theta)
        idx = ms[m] + np.arange(m, lmax + 1) * lstride
        f = alm[idx] @ lam            # sum_l a_lm lambda_lm(theta_i)
        t = f * np.exp(1j * m * phi)
        res += t.real if m == 0 else 2 * t.real
    return res


def adjoint_synthesis(map_, lmax, mmax, loc, mstart=None, lstride=1):
    """alm (1D complex, DUCC's layout) = sum_i map_i conj(Y_lm(loc_i))."""
    ms = default_mstart(lmax, mmax) if mstart is None else np.asarray(mstart)
    size = 1 + max(max(int(ms[m]) + m * lstride, int(ms[m]) + lmax * lstride)
                   for m in range(mmax + 1))
    out = np.zeros(size, dtype=np.complex128)
    theta, phi = loc[:, 0], loc[:, 1]
    f = np.asarray(map_, dtype=np.float64)
    for m in range(mmax + 1):
        lam = lambda_lm(lmax, m, theta)
        w = f * np.exp(-1j * m * phi)
        idx = ms[m] + np.arange(m, lmax + 1) * lstride
        out[idx] = lam @ w
    return out


def random_alm(lmax, mmax, rng):
    """DUCC's test alm (python/test/test_sht.py random_alm, spin 0): uniform
    real and imaginary parts in [-1, 1), a_l0 real."""
    n = nalm(lmax, mmax)
    res = rng.uniform(-1., 1., n) + 1j * rng.uniform(-1., 1., n)
    res[0:lmax + 1].imag = 0.
    return res


def almdot(a1, a2, lmax):
    """The real inner product of two real-map alm vectors (m > 0 counted twice),
    as DUCC's test_sht.py myalmdot."""
    a1, a2 = np.asarray(a1), np.asarray(a2)
    v = np.vdot(a1[:lmax + 1], a2[:lmax + 1]).real
    return v + 2 * np.vdot(a1[lmax + 1:], a2[lmax + 1:]).real

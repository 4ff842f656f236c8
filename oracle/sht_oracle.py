"""Test infrastructure only (the checker, never the product): a CPU
restatement of DUCC's ``synthesis_general`` / ``adjoint_synthesis_general``
(spin 0 and spin > 0) as direct sums over the spherical harmonics, for sizes
that finish in seconds.

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

Spin s > 0 (DUCC's convention, pinned against its compiled functions by the
golden fixtures): two maps with
    Q + i U = (-1)^(s+1) sum_{l, |m| <= mmax} (E_lm + i B_lm) D_lm(theta) e^{i m phi}
with D_lm = sqrt((2l+1)/(4 pi)) d^l_{m,-s}(theta), d the Wigner d function
(from the single term of Wigner's sum at l0
and the three-term recurrence in l), l >= max(|m|, s) and
E_{l,-m} = (-1)^m conj(E_lm) (the same for B); GRAD_ONLY has B = 0, DERIV1
(spin 1) is GRAD_ONLY with E_lm sqrt(l (l+1)).  The adjoint is the transpose
for the inner product that counts m > 0 twice:
    W_lm = sum_i (Q_i + i U_i) D_lm(theta_i) e^{-i m phi_i},
    E'_lm = s (W_lm + (-1)^m conj W_l,-m) / 2, B'_lm = -i s (W_lm - (-1)^m conj W_l,-m) / 2,
s = (-1)^(s+1), zero for l < s.
"""
from math import lgamma

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


def wigner_d(l, mp, m, beta):
    """d^l_{mp,m}(beta) by Wigner's explicit sum (terms in logarithms)."""
    beta = np.asarray(beta, dtype=np.float64)
    c, s = np.cos(beta / 2), np.sin(beta / 2)
    pre = 0.5 * (lgamma(l + m + 1) + lgamma(l - m + 1) + lgamma(l + mp + 1) + lgamma(l - mp + 1))
    res = np.zeros_like(beta)
    for k in range(0, 2 * l + 1):
        a, b, cc, d = l + m - k, k, l - k - mp, k - m + mp
        if min(a, b, cc, d) < 0:
            continue
        mag = np.exp(pre - lgamma(a + 1) - lgamma(b + 1) - lgamma(cc + 1) - lgamma(d + 1))
        res += (-1) ** (k - m + mp) * mag * c ** (2 * l - 2 * k + m - mp) * s ** (2 * k - m + mp)
    return res


def spin_D_all(lmax, m, s, theta):
    """D_lm(theta) = sqrt((2l+1)/(4 pi)) d^l_{m,-s}(theta) for l = 0 .. lmax
    (zero below l0 = max(|m|, s)), shape (lmax + 1, len(theta)): the single
    term of Wigner's sum at l0, then the three-term recurrence of the Wigner
    d functions in l (Wigner's explicit sum cancels badly beyond l ~ 20)."""
    theta = np.asarray(theta, dtype=np.float64)
    mu = abs(m)
    l0 = max(mu, s)
    c, sn, x = np.cos(theta / 2), np.sin(theta / 2), np.cos(theta)
    sign = (-1.) ** (m + s)
    if mu >= s:
        k = l0 - s
        pc, ps = (l0 - s, l0 + s) if m >= 0 else (l0 + s, l0 - s)
        if m < 0:
            sign *= (-1.) ** (l0 - s)
    else:
        k = l0 - m
        pc, ps = l0 - m, l0 + m
    lognorm = 0.5 * (np.log((2 * l0 + 1) / (4 * np.pi)) + lgamma(2 * l0 + 1) - lgamma(k + 1)
                     - lgamma(2 * l0 - k + 1))
    out = np.zeros((lmax + 1, theta.size))
    if l0 > lmax:
        return out
    d1 = sign * np.exp(lognorm) * c ** pc * sn ** ps
    d2 = np.zeros_like(d1)
    out[l0] = d1
    for l in range(l0 + 1, lmax + 1):
        den = np.sqrt((l * l - m * m) * (l * l - s * s * 1.))
        al = l * np.sqrt((2 * l + 1.) * (2 * l - 1.)) / den
        be = -m * s / (l * (l - 1.))
        ga = (l / (l - 1.)) * np.sqrt((2 * l + 1.) / (2 * l - 3.)) * np.sqrt(
            max(((l - 1.) ** 2 - m * m) * ((l - 1.) ** 2 - s * s), 0.)) / den
        d1, d2 = al * (x - be) * d1 - ga * d2, d1
        out[l] = d1
    return out


def _spin_ab(alm, l, m, idx, mode):
    e = alm[0][idx]
    b = alm[1][idx] if mode == "STANDARD" else 0.
    if mode == "DERIV1":
        e = e * np.sqrt(l * (l + 1.))
    return e, b


def synthesis_spin(alm, spin, lmax, mmax, loc, mode="STANDARD", mstart=None, lstride=1):
    """(Q, U) of shape (2, npoints) of the spin-s a_lm (rows E[, B]) at loc."""
    ms = default_mstart(lmax, mmax) if mstart is None else np.asarray(mstart)
    alm = np.asarray(alm).astype(np.complex128)
    theta, phi = loc[:, 0], loc[:, 1]
    sig = (-1.) ** (spin + 1)
    G = np.zeros(theta.size, dtype=np.complex128)
    for m in range(mmax + 1):
        Dp = spin_D_all(lmax, m, spin, theta)
        Dn = spin_D_all(lmax, -m, spin, theta)
        for l in range(max(m, spin), lmax + 1):
            e, b = _spin_ab(alm, l, m, ms[m] + l * lstride, mode)
            G += sig * (e + 1j * b) * Dp[l] * np.exp(1j * m * phi)
            if m > 0:
                f = (-1.) ** m
                G += sig * f * (np.conj(e) + 1j * np.conj(b)) * Dn[l] * np.exp(-1j * m * phi)
    return np.stack([G.real, G.imag])


def adjoint_synthesis_spin(map_, spin, lmax, mmax, loc, mode="STANDARD", mstart=None,
                           lstride=1):
    """a_lm rows (E[, B]) of the adjoint of synthesis_spin for (Q, U) = map_."""
    ms = default_mstart(lmax, mmax) if mstart is None else np.asarray(mstart)
    size = 1 + max(max(int(ms[m]) + m * lstride, int(ms[m]) + lmax * lstride)
                   for m in range(mmax + 1))
    nrow = 2 if mode == "STANDARD" else 1
    out = np.zeros((nrow, size), dtype=np.complex128)
    theta, phi = loc[:, 0], loc[:, 1]
    P = np.asarray(map_[0], np.float64) + 1j * np.asarray(map_[1], np.float64)
    sig = (-1.) ** (spin + 1)
    for m in range(mmax + 1):
        Dp = spin_D_all(lmax, m, spin, theta)
        Dn = spin_D_all(lmax, -m, spin, theta)
        for l in range(m, lmax + 1):
            idx = ms[m] + l * lstride
            if l < spin:
                out[:, idx] = 0
                continue
            wp = np.sum(P * Dp[l] * np.exp(-1j * m * phi))
            wn = np.sum(P * Dn[l] * np.exp(1j * m * phi))
            f = (-1.) ** m
            e = sig * (wp + f * np.conj(wn)) / 2
            if mode == "DERIV1":
                e *= np.sqrt(l * (l + 1.))
            out[0, idx] = e
            if nrow == 2:
                out[1, idx] = -1j * sig * (wp - f * np.conj(wn)) / 2
    return out


def random_alm_spin(lmax, mmax, spin, ncomp, rng):
    """DUCC's test alm (python/test/test_sht.py random_alm): uniform parts in
    [-1, 1), a_l0 real, a_lm with l < spin zero."""
    n = nalm(lmax, mmax)
    res = rng.uniform(-1., 1., (ncomp, n)) + 1j * rng.uniform(-1., 1., (ncomp, n))
    res[:, 0:lmax + 1].imag = 0.
    ofs = 0
    for s in range(spin):
        res[:, ofs:ofs + spin - s] = 0.
        ofs += lmax + 1 - s
    return res

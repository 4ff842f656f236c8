"""Spherical-harmonic synthesis at arbitrary points on the sphere and its
adjoint on the GPU: a drop-in for ``ducc0.sht.synthesis_general`` and
``ducc0.sht.adjoint_synthesis_general`` (python/sht_pymod.cc:805-885,
:2299-2300 for the signatures and keyword defaults), any spin, modes
STANDARD, GRAD_ONLY and DERIV1.

The work runs in the CUDA library through the C-ABI
(``dnufft_synthesis_general`` / ``dnufft_adjoint_synthesis_general`` in
include/ducc_b200_sht.h): a Legendre (spin 0) or Wigner-d (spin > 0)
recurrence kernel onto equiangular rings, the DFT along the rings and one 2D
transform of this package at the points.  Arrays may be numpy arrays (copied to the current
CUDA device, the result copied back) or torch CUDA tensors (used in place;
the result is a tensor).  As in DUCC, the dtype of ``alm`` (synthesis) or
``map`` (adjoint) sets the precision and ``loc`` is float64 (theta, phi).
"""
import ctypes

import numpy as np

from . import _capi as C

__all__ = ["synthesis_general", "adjoint_synthesis_general", "pseudo_analysis_general", "lsmr"]


def _torch():
    import torch
    return torch


def _dev(x):
    torch = _torch()
    if C.is_torch(x):
        if not x.is_cuda:
            raise ValueError("torch tensors must live on a CUDA device")
        return x, False
    a = np.ascontiguousarray(np.asarray(x))
    if not a.flags.writeable:
        a = a.copy()
    return torch.from_numpy(a).cuda(), True


def _mstart(lmax, mmax, mstart):
    """DUCC's get_mstart (python/sht_pymod.cc:124-140)."""
    if mstart is None:
        mmax = lmax if mmax is None else int(mmax)
        if mmax > lmax:
            raise RuntimeError("mmax>lmax")
        ms = np.empty(mmax + 1, dtype=np.int64)
        idx = 0
        for m in range(mmax + 1):
            ms[m] = idx - m
            idx += lmax + 1 - m
        return ms
    ms = np.ascontiguousarray(np.asarray(mstart), dtype=np.int64)
    if mmax is not None and int(mmax) + 1 != ms.shape[0]:
        raise RuntimeError("mmax and mstart size mismatch")
    if ms.shape[0] > lmax + 1:
        raise RuntimeError("mmax>lmax")
    return ms


def _min_almdim(lmax, ms, lstride):
    """DUCC's min_almdim (python/sht_pymod.cc:168-182)."""
    res = 0
    for m in range(ms.shape[0]):
        first, last = int(ms[m]) + m * lstride, int(ms[m]) + lmax * lstride
        if first < 0 or last < 0:
            raise RuntimeError("impossible a_lm memory layout")
        res = max(res, first, last)
    return res + 1


def _opts(nthreads, sigma_min, sigma_max, verbose):
    o = C.ShtOpts()
    C.lib().dnufft_sht_default_opts(ctypes.byref(o))
    if int(nthreads) < 0:
        raise ValueError("nthreads must be >= 0")
    o.nthreads = int(nthreads)
    o.sigma_min = float(sigma_min)
    o.sigma_max = float(sigma_max)
    o.verbosity = 1 if verbose else 0
    return o


_MODES = {"STANDARD": 0, "GRAD_ONLY": 1, "DERIV1": 2}


def _mode(mode, spin):
    """DUCC's get_mode and component counts (python/sht_pymod.cc get_nalm,
    get_nmaps): (mode code, a_lm rows, map rows)."""
    if mode not in _MODES:
        raise RuntimeError("unknown SHT mode")
    nalm = 1 if (spin == 0 or mode != "STANDARD") else 2
    return _MODES[mode], nalm, (1 if spin == 0 else 2)


def _loc(loc):
    torch = _torch()
    d_loc, _ = _dev(loc)
    if d_loc.dtype != torch.float64:
        raise TypeError("unsupported combination of data types")
    if d_loc.dim() != 2 or d_loc.shape[1] != 2:
        raise RuntimeError("last dimension of loc must have size 2")
    return d_loc


def synthesis_general(*, alm, spin, lmax, loc, epsilon, mstart=None, lstride=1, mmax=None,
                      nthreads=1, map=None, sigma_min=1.1, sigma_max=2.6, mode="STANDARD",
                      verbose=False):
    """Evaluate the map(s) of ``alm`` at the points ``loc`` (theta, phi),
    returning ``map`` of shape (1, npoints) for spin 0, (2, npoints) (Q, U)
    otherwise (``ducc0.sht.synthesis_general``)."""
    torch = _torch()
    spin, lmax, lstride = int(spin), int(lmax), int(lstride)
    mcode, nalm_c, nmaps = _mode(mode, spin)
    d_alm, host = _dev(alm)
    if d_alm.dtype not in (torch.complex64, torch.complex128):
        raise TypeError("unsupported combination of data types")
    if d_alm.dim() != 2:
        raise RuntimeError("alm must be a 2D array")
    if d_alm.shape[0] != nalm_c:
        raise RuntimeError("number of components mismatch in alm")
    d_loc = _loc(loc)
    ms = _mstart(lmax, mmax, mstart)
    rdt = torch.float64 if d_alm.dtype == torch.complex128 else torch.float32
    npts = int(d_loc.shape[0])
    shape = (nmaps, npts)
    if map is not None and C.is_torch(map):
        d_map = map
    else:
        if map is not None and tuple(map.shape) != shape:
            raise RuntimeError("bad map shape")
        d_map = torch.empty(shape, dtype=rdt, device=d_alm.device)
    o = _opts(nthreads, sigma_min, sigma_max, verbose)
    st = ctypes.c_void_p(torch.cuda.current_stream(d_alm.device).cuda_stream)
    a_alm, a_loc, a_map = C.describe(d_alm), C.describe(d_loc), C.describe(d_map)
    C.check(C.lib().dnufft_synthesis_general(
        ctypes.byref(a_alm), spin, mcode, lmax,
        ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
        ms.shape[0], lstride, ctypes.byref(a_loc), float(epsilon), ctypes.byref(o),
        ctypes.byref(a_map), st))
    if map is not None and not C.is_torch(map):
        map[...] = d_map.cpu().numpy()
        return map
    return d_map.cpu().numpy() if host else d_map


def adjoint_synthesis_general(*, map, spin, lmax, loc, epsilon, mstart=None, lstride=1,
                              mmax=None, nthreads=1, alm=None, sigma_min=1.1, sigma_max=2.6,
                              mode="STANDARD", verbose=False):
    """The adjoint of ``synthesis_general`` for DUCC's inner product of a_lm
    (m > 0 counted twice): spin 0, a_lm = sum_i map_i conj(Y_lm(loc_i)); every
    a_lm with m <= l <= lmax is written (``ducc0.sht.adjoint_synthesis_general``)."""
    torch = _torch()
    spin, lmax, lstride = int(spin), int(lmax), int(lstride)
    mcode, nalm_c, nmaps = _mode(mode, spin)
    d_map, host = _dev(map)
    if d_map.dtype not in (torch.float32, torch.float64):
        raise TypeError("type matching failed: 'map' has neither type 'f4' nor 'f8'")
    if d_map.dim() != 2:
        raise RuntimeError("map must be a 2D array")
    if d_map.shape[0] != nmaps:
        raise RuntimeError("number of components mismatch in map")
    d_loc = _loc(loc)
    ms = _mstart(lmax, mmax, mstart)
    cdt = torch.complex128 if d_map.dtype == torch.float64 else torch.complex64
    nalm = _min_almdim(lmax, ms, lstride)
    if alm is not None and C.is_torch(alm):
        d_alm = alm
    elif alm is not None:
        if alm.shape[0] != nalm_c or alm.shape[1] < nalm:
            raise RuntimeError("bad alm shape")
        d_alm = torch.from_numpy(np.ascontiguousarray(alm)).to(d_map.device)
    else:
        d_alm = torch.zeros((nalm_c, nalm), dtype=cdt, device=d_map.device)
    o = _opts(nthreads, sigma_min, sigma_max, verbose)
    st = ctypes.c_void_p(torch.cuda.current_stream(d_map.device).cuda_stream)
    a_map, a_loc, a_alm = C.describe(d_map), C.describe(d_loc), C.describe(d_alm)
    C.check(C.lib().dnufft_adjoint_synthesis_general(
        ctypes.byref(a_map), spin, mcode, lmax,
        ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
        ms.shape[0], lstride, ctypes.byref(a_loc), float(epsilon), ctypes.byref(o),
        ctypes.byref(a_alm), st))
    if alm is not None and not C.is_torch(alm):
        alm[...] = d_alm.cpu().numpy()
        return alm
    return d_alm.cpu().numpy() if host else d_alm


def lsmr(op, op_adj, xnorm, bnorm, b, x0, damp=0., atol=1e-6, btol=1e-6, conlim=1e8,
         itnlim=None):
    """LSMR (Fong & Saunders, SIAM J. Sci. Comput. 33 (2011) 2950-2971), the
    least-squares solver DUCC's pseudo_analysis_general uses
    (src/ducc0/math/solvers.h), restated for any vectors with +, - and scalar
    * (numpy arrays, torch tensors): minimises |b - A x| given A x = op(x) and
    A^T y = op_adj(y), with the norms xnorm (solution space) and bnorm (data
    space).  Returns (x, istop, itn, normr, normar, normA, condA, normx, normb)."""
    x = x0
    u = b - op(x0)
    beta = bnorm(u)
    if beta > 0:
        u = u * (1. / beta)
    v = op_adj(u)
    alpha = xnorm(v)
    if alpha > 0:
        v = v * (1. / alpha)
    itnlim = itnlim if itnlim is not None else 1000000
    itn, zetabar, alphabar, rho, rhobar, cbar, sbar = 0, alpha * beta, alpha, 1., 1., 1., 0.
    h, hbar = v, v * 0.
    betadd, betad, rhodold, tautildeold, thetatilde, zeta, d = beta, 0., 1., 0., 0., 0., 0.
    normA2 = alpha * alpha
    maxrbar, minrbar = 0., 1e100
    normA, condA, normx = alpha, 1., 0.
    normb, istop = beta, 0
    ctol = 1. / conlim if conlim > 0 else 0.
    normr, normar = beta, alpha * beta
    if normar == 0:
        return x, istop, itn, normr, normar, normA, condA, normx, normb
    while itn < itnlim:
        itn += 1
        u = op(v) - u * alpha
        beta = bnorm(u)
        if beta > 0:
            u = u * (1. / beta)
            v = op_adj(u) - v * beta
            alpha = xnorm(v)
            if alpha > 0:
                v = v * (1. / alpha)
        # rotation that removes the damping term
        alphahat = np.hypot(alphabar, damp)
        chat, shat = alphabar / alphahat, damp / alphahat
        # plane rotation Q_k
        rhoold = rho
        rho = np.hypot(alphahat, beta)
        c, s = alphahat / rho, beta / rho
        thetanew = s * alpha
        alphabar = c * alpha
        # plane rotation Qbar_k
        rhobarold, zetaold = rhobar, zeta
        thetabar = sbar * rho
        rhotemp = cbar * rho
        rhobar = np.hypot(cbar * rho, thetanew)
        cbar, sbar = cbar * rho / rhobar, thetanew / rhobar
        zeta = cbar * zetabar
        zetabar = -sbar * zetabar
        # h, hbar, x
        hbar = h - hbar * (thetabar * rho / (rhoold * rhobarold))
        x = x + hbar * (zeta / (rho * rhobar))
        h = v - h * (thetanew / rho)
        # estimate of |r|
        betaacute = chat * betadd
        betacheck = -shat * betadd
        betahat = c * betaacute
        betadd = -s * betaacute
        thetatildeold = thetatilde
        rhotildeold = np.hypot(rhodold, thetabar)
        ctildeold, stildeold = rhodold / rhotildeold, thetabar / rhotildeold
        thetatilde = stildeold * rhobar
        rhodold = ctildeold * rhobar
        betad = -stildeold * betad + ctildeold * betahat
        tautildeold = (zetaold - thetatildeold * tautildeold) / rhotildeold
        taud = (zeta - thetatilde * tautildeold) / rhodold
        d += betacheck * betacheck
        normr = np.sqrt(d + (betad - taud) ** 2 + betadd * betadd)
        # estimates of |A| and cond(A)
        normA2 += beta * beta
        normA = np.sqrt(normA2)
        normA2 += alpha * alpha
        maxrbar = max(maxrbar, rhobarold)
        if itn > 1:
            minrbar = min(minrbar, rhobarold)
        condA = max(maxrbar, rhotemp) / min(minrbar, rhotemp)
        # stopping rules
        normar = abs(zetabar)
        normx = xnorm(x)
        test1 = normr / normb
        test2 = normar / (normA * normr) if normA * normr != 0 else np.inf
        test3 = 1. / condA
        t1 = test1 / (1. + normA * normx / normb)
        rtol = btol + atol * normA * normx / normb
        if itn >= itnlim:
            istop = 7
        if 1. + test3 <= 1.:
            istop = 6
        if 1. + test2 <= 1.:
            istop = 5
        if 1. + t1 <= 1.:
            istop = 4
        if test3 <= ctol:
            istop = 3
        if test2 <= atol:
            istop = 2
        if test1 <= rtol:
            istop = 1
        if istop > 0:
            break
    return x, istop, itn, normr, normar, normA, condA, normx, normb


def pseudo_analysis_general(*, lmax, map, loc, spin, nthreads, maxiter, epsilon=1e-5,
                            sigma_min=1.1, sigma_max=2.6, mstart=None, lstride=1, mmax=None,
                            alm=None, verbose=False):
    """a_lm whose synthesis at ``loc`` best fits ``map`` in the least-squares
    sense, by LSMR over ``synthesis_general`` and its adjoint at a tenth of
    ``epsilon`` (``ducc0.sht.pseudo_analysis_general``, src/ducc0/sht/sht.cc:3003-3057:
    atol = 1e-14 sqrt(npoints), btol = epsilon, conlim 1e8, the a_lm norm
    counting m > 0 twice).  Returns (alm, istop, itn, |r| / |map|,
    |A^T r| / (|A| |r|))."""
    torch = _torch()
    spin, lmax, lstride = int(spin), int(lmax), int(lstride)
    d_map, host = _dev(map)
    if d_map.dtype not in (torch.float32, torch.float64):
        raise TypeError("type matching failed: 'alm' has neither type 'c8' nor 'c16'")
    ncomp = 1 if spin == 0 else 2
    if d_map.dim() != 2 or d_map.shape[0] != ncomp:
        raise RuntimeError("number of components mismatch in map")
    d_loc = _loc(loc)
    ms = _mstart(lmax, mmax, mstart)
    nalm = _min_almdim(lmax, ms, lstride)
    cdt = torch.complex128 if d_map.dtype == torch.float64 else torch.complex64
    # weights of the a_lm norm: 1 for m = 0, 2 for m > 0, 0 off the layout
    w = np.zeros(nalm)
    for m in range(ms.shape[0]):
        w[int(ms[m]) + np.arange(m, lmax + 1) * lstride] = 1. if m == 0 else 2.
    d_w = torch.from_numpy(w).to(d_map.device)
    kw = dict(spin=spin, lmax=lmax, loc=d_loc, epsilon=0.1 * float(epsilon), mstart=ms,
              lstride=lstride, nthreads=nthreads, sigma_min=sigma_min, sigma_max=sigma_max,
              verbose=verbose)

    def op(x):
        return synthesis_general(alm=x, **kw)

    def op_adj(y):
        return adjoint_synthesis_general(map=y.contiguous(), **kw)

    def almnorm(x):
        return float(torch.sqrt(torch.sum(d_w * (x.real.double() ** 2 + x.imag.double() ** 2))))

    def mapnorm(y):
        return float(torch.sqrt(torch.sum(y.double() ** 2)))

    x0 = torch.zeros((ncomp, nalm), dtype=cdt, device=d_map.device)
    atol = 1e-14 * np.sqrt(d_map.shape[1])
    x, istop, itn, normr, normar, normA, condA, normx, normb = lsmr(
        op, op_adj, almnorm, mapnorm, d_map, x0, 0., atol, float(epsilon), 1e8, int(maxiter))
    rnorm = normr / normb if normb else 0.
    sqnorm = normar / (normA * normr) if normA * normr else 0.
    if alm is not None:
        if C.is_torch(alm):
            alm[:, :nalm] = x
        else:
            alm[:, :nalm] = x.cpu().numpy()
        res = alm
    else:
        res = x.cpu().numpy() if host else x
    return res, istop, itn, rnorm, sqnorm

"""CPU oracle for the NUFFT hot path - TEST INFRASTRUCTURE ONLY.

A numpy restatement of DUCC's type-1 / type-2 NUFFT (``ducc0.nufft.nu2u`` /
``u2nu``) used to check the CUDA product path.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it,
and only as the checker - the product never routes through it.

It restates, function by function (reference paths relative to DUCC's tree):

* parameter choice    ``findNufftParameters``      src/ducc0/nufft/nufft.h:155-208
                      ``getAvailableKernels``       src/ducc0/math/gridding_kernel.h:420-444
                      ``bestEpsilon``               src/ducc0/math/gridding_kernel.cc:1562-1576
                      ``good_size_cmplx``           src/ducc0/fft/fft.h:93-118
* kernel polynomial   ``getCoeffs``                 src/ducc0/math/gridding_kernel.cc:28-76
                      ``esknew``                    src/ducc0/math/gridding_kernel.cc:1539-1544
* correction factors  ``GLFullCorrection``/``corfunc`` src/ducc0/math/gridding_kernel.h:77-129
* folding             ``getpix``                    src/ducc0/nufft/nufft.h:285-298
* tile keys           ``get_tile``/``build_index``  src/ducc0/nufft/nufft.h:301-320,
                                                    :892-907, :1364-1381, :1862-1892
* stable tile sort    ``bucket_sort2``              src/ducc0/infra/bucket_sort.h:170-354
* spreading           ``HelperNu2u``/``spreading_helper`` nufft.h:917-993, :1141-1204
* interpolation       ``HelperU2nu``/``interpolation_helper`` nufft.h:995-1067, :1208-1272
* FFT + pruning       ``nonuni2uni``/``uni2nonuni`` nufft.h:1274-1362 (numpy.fft here)
* correction + crop   ``comp_indices``              nufft.h:142-151
* direct NUDFT        ``explicit_nufft``            python/test/test_nufft.py:32-43
* error metrics       ``l2error``/``vdot``           python/misc_pymod.cc:52-185

The arithmetic is FP64 throughout (folding in x87 long double where DUCC uses
it), so the oracle is at least as accurate as DUCC's own double path.  Its
parity is pinned against DUCC itself (``oracle/_ref``, built from source by
``oracle/Makefile``) and against the golden fixtures in ``tests/golden``.
"""
import math
import os
import re

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_DB_PATH = os.path.join(_HERE, "..", "ducc_b200", "csrc", "kernel_db.inc")

# ----------------------------------------------------------------------------
# kernel table and parameter choice
# ----------------------------------------------------------------------------

_KDB = None


def kernel_db():
    """Rows (W, ofactor, epsilon, beta, e0, ndim, singleprec) of the ES table."""
    global _KDB
    if _KDB is None:
        rows = []
        pat = re.compile(r"^\{(\d+),([^,]+),([^,]+),([^,]+),([^,]+),(\d),(\d)\},")
        with open(_DB_PATH) as f:
            for line in f:
                m = pat.match(line.strip())
                if m:
                    g = m.groups()
                    rows.append((int(g[0]), float(g[1]), float(g[2]), float(g[3]),
                                 float(g[4]), int(g[5]), g[6] == "1"))
        _KDB = rows
    return _KDB


def good_size_complex(n):
    """Smallest 2,3,5,7,11-smooth integer >= n (fft.h:93-118)."""
    n = int(n)
    if n <= 12:
        return n
    m = n
    while True:
        x = m
        for p in (2, 3, 5, 7, 11):
            while x % p == 0:
                x //= p
        if x == 1:
            return m
        m += 1


def wmax(singleprec):
    return 8 if singleprec else 16


def available_kernels(epsilon, ndim, singleprec, ofactor_min=1.1, ofactor_max=2.6):
    """Per support W, the row with the smallest ofactor reaching epsilon
    (gridding_kernel.h:420-444)."""
    db = kernel_db()
    ofc = [ofactor_max] * 20
    idx = [len(db)] * 20
    wlim = wmax(singleprec)
    for i, (W, of, eps, _b, _e, nd, sp) in enumerate(db):
        if (nd == ndim and sp == singleprec and W <= wlim and eps <= epsilon
                and of <= ofc[W] and of >= ofactor_min):
            ofc[W] = of
            idx[W] = i
    res = [v for v in idx if v < len(db)]
    if not res:
        raise RuntimeError("no appropriate kernel found")
    return res


def best_epsilon(ndim, singleprec, sigma_min=1.1, sigma_max=2.6):
    """gridding_kernel.cc:1562-1576."""
    res = 1000.0
    for (W, of, eps, _b, _e, nd, sp) in kernel_db():
        if nd == ndim and sp == singleprec and eps <= res and sigma_min <= of <= sigma_max:
            res = eps
    if res >= 1000.0:
        raise RuntimeError("no appropriate kernel found")
    return res


def find_parameters(epsilon, sigma_min, sigma_max, dims, npoints, gridding,
                    nthreads, singleprec, vlen=8):
    """Kernel row index and oversampled dims minimising DUCC's cost model
    (nufft.h:155-208).  ``vlen`` is the SIMD width DUCC's build uses for the
    accumulation type (8 on AVX-512 builds for float and double)."""
    ndim = len(dims)
    idx = available_kernels(epsilon, ndim, singleprec, sigma_min, sigma_max)
    db = kernel_db()
    mincost = 1e300
    nref_fft = 2048.0
    costref_fft = 0.0693
    best = None
    for i in idx:
        W, of = db[i][0], db[i][1]
        nvec = (W + vlen - 1) // vlen
        big = []
        gridsize = 1.0
        for d in dims:
            n = 2 * good_size_complex(int(d * of * 0.5) + 1)
            n = max(n, 16)
            big.append(n)
            gridsize *= n
        logterm = math.log(gridsize) / math.log(nref_fft * nref_fft)
        fftcost = gridsize / (nref_fft * nref_fft) * logterm * costref_fft
        kernelpoints = nvec * vlen
        for _ in range(ndim - 1):
            kernelpoints *= W
        gridcost = 2.2e-10 * npoints * (kernelpoints + (ndim * nvec * (W + 3) * vlen))
        gridcost /= nthreads
        x2 = nthreads - 1
        m2 = 6.0 - 1
        sig = 1.0 + x2 / (1.0 + (x2 / m2) ** 2.0) ** (1.0 / 2.0)
        fftcost /= sig
        cost = fftcost + gridcost
        if cost < mincost:
            mincost = cost
            best = (i, big)
    return best


def esk(v, beta, e0):
    """Generalised ES kernel (gridding_kernel.cc:1539-1544)."""
    tmp = (1 - v) * (1 + v)
    ok = tmp >= 0
    return np.where(ok, np.exp(beta * (np.power(np.where(ok, tmp, 0.0), e0) - 1)), 0.0)


def kernel_coeffs(W, beta_scaled, e0):
    """W piecewise polynomials of degree D=W+3, monomial coefficients from a
    Chebyshev interpolant on each sub-interval (gridding_kernel.cc:28-76).
    Returns coeff[(D+1)*W] laid out as coeff[j*W+i], j=0 highest power."""
    D = W + 3
    k = np.arange(D + 1)
    chebroot = np.cos((2 * k + 1.0) * math.pi / (2 * D + 2))
    coeff = np.zeros((D + 1) * W)
    # Chebyshev -> monomial conversion matrix
    C = np.zeros((D + 1, D + 1))
    C[0, 0] = 1.0
    C[1, 1] = 1.0
    for j in range(2, D + 1):
        C[j, 0] = -C[j - 2, 0]
        for kk in range(1, j + 1):
            C[j, kk] = 2 * C[j - 1, kk - 1] - C[j - 2, kk]
    for i in range(W):
        l = -1 + 2.0 * i / W
        r = -1 + 2.0 * (i + 1) / W
        y = esk(chebroot * (r - l) * 0.5 + (r + l) * 0.5, beta_scaled, e0)
        avg = y.mean()
        y = y - avg
        lcf = np.array([2.0 / (D + 1) * np.sum(y * np.cos(j * (2 * k + 1) * math.pi / (2 * D + 2)))
                        for j in range(D + 1)])
        lcf[0] *= 0.5
        lcf2 = C.T @ lcf
        lcf2[0] += avg
        for j in range(D + 1):
            coeff[j * W + i] = lcf2[D - j]
    return coeff


def gl_correction(W, beta_scaled, e0):
    """Nodes x>=0 and weights*psi*(W/2) for the correction integral
    (gridding_kernel.h:116-129), using numpy's Gauss-Legendre rule."""
    p = int(1.5 * W) + 2
    x, w = np.polynomial.legendre.leggauss(2 * p)
    sel = x >= 0
    x = x[sel]
    w = w[sel] * 2.0
    return x, w * esk(x, beta_scaled, e0) * W * 0.5


def corfac(n, dx, W, beta_scaled, e0):
    """1/psi_hat at 0, dx, ..., (n-1)dx (gridding_kernel.h:77-109)."""
    x, wgt = gl_correction(W, beta_scaled, e0)
    v = np.arange(n) * dx
    return 1.0 / (np.cos(np.outer(v, math.pi * W * x)) @ wgt)


class Params:
    """Everything DUCC's Nufft_ancestor constructor derives (nufft.h:392-433)."""

    def __init__(self, shape, epsilon, singleprec, npoints, gridding, nthreads=1,
                 sigma_min=1.2, sigma_max=2.51, periodicity=2 * math.pi,
                 coord_single=None, force=None, vlen=8):
        self.shape = tuple(int(s) for s in shape)
        self.ndim = len(self.shape)
        if np.ndim(periodicity) == 0:
            periodicity = [float(periodicity)] * self.ndim
        self.periodicity = [float(p) for p in periodicity]
        self.coordfct = [1.0 / p for p in self.periodicity]
        self.singleprec = singleprec
        if force is not None:
            kidx, nover = force
        else:
            kidx, nover = find_parameters(epsilon, sigma_min, sigma_max, self.shape,
                                          npoints, gridding, nthreads, singleprec, vlen)
        row = kernel_db()[kidx]
        self.kidx = kidx
        self.W = row[0]
        self.ofactor = row[1]
        self.beta = row[3] * self.W
        self.e0 = row[4]
        self.nover = [int(n) for n in nover]
        self.nsafe = (self.W + 1) // 2
        self.shift = [self.W * (-0.5) + 1 + n for n in self.nover]
        self.maxi0 = [(n + self.nsafe) - self.W for n in self.nover]
        if self.ndim == 1:
            self.log2tile = 9
        elif self.ndim == 2:
            self.log2tile = 5 if singleprec else 4
        else:
            self.log2tile = 4
        self.coeff = kernel_coeffs(self.W, self.beta, self.e0)
        self.corfac = [corfac(N // 2 + 1, 1.0 / n, self.W, self.beta, self.e0)
                       for N, n in zip(self.shape, self.nover)]


# ----------------------------------------------------------------------------
# folding, keys, sort
# ----------------------------------------------------------------------------

def getpix(p, coord):
    """Per point and axis: start index i0 and offset frac (nufft.h:285-298).

    Range reduction runs in long double for float64 coordinates and in double
    for float32 coordinates, exactly as DUCC does."""
    coord = np.asarray(coord)
    big = np.longdouble if coord.dtype == np.float64 else np.float64
    M = coord.shape[0]
    i0 = np.empty((M, p.ndim), dtype=np.int64)
    frac = np.empty((M, p.ndim), dtype=np.float64)
    for d in range(p.ndim):
        tmp = coord[:, d].astype(np.float64) * p.coordfct[d]
        tmp2 = (tmp - np.floor(tmp)).astype(big) * big(p.nover[d])
        s = (tmp2 + big(p.shift[d])).astype(np.int64) - p.nover[d]
        s = np.minimum(s, p.maxi0[d])
        i0[:, d] = s
        frac[:, d] = (tmp2 - s.astype(big)).astype(np.float64)
    return i0, frac


def tile_keys(p, i0):
    """Tile key per point (nufft.h:892-907, :1364-1381, :1862-1892)."""
    L = p.log2tile
    t = (i0 + p.nsafe) >> L
    if p.ndim == 1:
        return t[:, 0].astype(np.uint64)
    if p.ndim == 2:
        ntv = (p.nover[1] >> L) + 3
        return (t[:, 0] * ntv + t[:, 1]).astype(np.uint64)
    ntu, ntv, ntw = [(n >> L) + 3 for n in p.nover]
    lsq2 = L
    while lsq2 >= 1 and ((ntu * ntv * ntw) << (3 * (L - lsq2))) < (1 << 28):
        lsq2 -= 1
    ss = L - lsq2
    ms = (1 << ss) - 1
    t = (i0 + p.nsafe) >> lsq2
    low = ((t[:, 0] & ms) << (2 * ss)) | ((t[:, 1] & ms) << ss) | (t[:, 2] & ms)
    hi = ((t[:, 0] >> ss) * ntv * ntw) + ((t[:, 1] >> ss) * ntw) + (t[:, 2] >> ss)
    return ((hi << (3 * ss)) | low).astype(np.uint64)


def permutation(p, coord):
    """Stable argsort of tile keys: DUCC's coord_idx (bucket_sort.h:170)."""
    i0, _ = getpix(p, coord)
    return np.argsort(tile_keys(p, i0), kind="stable").astype(np.uint32)


# ----------------------------------------------------------------------------
# kernel weights, spreading, interpolation
# ----------------------------------------------------------------------------

def weights(p, frac):
    """W kernel weights per point for one axis: piecewise polynomial evaluated
    at x = W-1-2*frac (nufft.h:976-992, gridding_kernel.h:144-156)."""
    W, D = p.W, p.W + 3
    x = -2.0 * frac + (W - 1)
    c = p.coeff.reshape(D + 1, W)
    res = np.zeros((frac.shape[0], W))
    for j in range(D + 1):
        res = res * x[:, None] + c[j][None, :]
    return res


def _footprint(p, coord):
    i0, frac = getpix(p, coord)
    ws = [weights(p, frac[:, d]) for d in range(p.ndim)]
    return i0, ws


def spread(p, coord, values):
    """Type-1 spreading onto the periodic oversampled grid (FP64)."""
    grid = np.zeros(p.nover, dtype=np.complex128)
    i0, ws = _footprint(p, coord)
    vals = np.asarray(values).astype(np.complex128)
    W = p.W
    if p.ndim == 1:
        for a in range(W):
            np.add.at(grid, (i0[:, 0] + a) % p.nover[0], ws[0][:, a] * vals)
    elif p.ndim == 2:
        for a in range(W):
            iu = (i0[:, 0] + a) % p.nover[0]
            va = ws[0][:, a] * vals
            for b in range(W):
                np.add.at(grid, (iu, (i0[:, 1] + b) % p.nover[1]), va * ws[1][:, b])
    else:
        for a in range(W):
            iu = (i0[:, 0] + a) % p.nover[0]
            va = ws[0][:, a] * vals
            for b in range(W):
                iv = (i0[:, 1] + b) % p.nover[1]
                vb = va * ws[1][:, b]
                for c in range(W):
                    np.add.at(grid, (iu, iv, (i0[:, 2] + c) % p.nover[2]), vb * ws[2][:, c])
    return grid


def interpolate(p, grid, coord):
    """Type-2 interpolation from the periodic oversampled grid (FP64)."""
    i0, ws = _footprint(p, coord)
    W = p.W
    out = np.zeros(i0.shape[0], dtype=np.complex128)
    if p.ndim == 1:
        for a in range(W):
            out += ws[0][:, a] * grid[(i0[:, 0] + a) % p.nover[0]]
    elif p.ndim == 2:
        for a in range(W):
            iu = (i0[:, 0] + a) % p.nover[0]
            for b in range(W):
                out += ws[0][:, a] * ws[1][:, b] * grid[iu, (i0[:, 1] + b) % p.nover[1]]
    else:
        for a in range(W):
            iu = (i0[:, 0] + a) % p.nover[0]
            for b in range(W):
                iv = (i0[:, 1] + b) % p.nover[1]
                wab = ws[0][:, a] * ws[1][:, b]
                for c in range(W):
                    out += wab * ws[2][:, c] * grid[iu, iv, (i0[:, 2] + c) % p.nover[2]]
    return out


def comp_indices(idx, nuni, nbig, fft_order):
    """(corfac index, uniform index, oversampled index) (nufft.h:142-151)."""
    icf = abs(nuni // 2 - idx)
    i1 = nuni - nuni // 2 + idx if fft_order else idx
    if i1 >= nuni:
        i1 -= nuni
    i2 = nbig - nuni // 2 + idx
    if i2 >= nbig:
        i2 -= nbig
    return icf, i1, i2


def _index_maps(p, fft_order):
    maps = []
    for d in range(p.ndim):
        N, n = p.shape[d], p.nover[d]
        icf = np.empty(N, dtype=np.int64)
        iu = np.empty(N, dtype=np.int64)
        ig = np.empty(N, dtype=np.int64)
        for i in range(N):
            icf[i], iu[i], ig[i] = comp_indices(i, N, n, fft_order)
        maps.append((icf, iu, ig))
    return maps


def _fft(grid, forward):
    axes = tuple(range(grid.ndim))
    if forward:
        return np.fft.fftn(grid, axes=axes)
    return np.fft.ifftn(grid, axes=axes) * np.prod(grid.shape)


def nu2u(p, coord, values, forward, fft_order=False):
    """Full type-1 transform; returns the uniform grid (complex128)."""
    grid = _fft(spread(p, coord, values), forward)
    maps = _index_maps(p, fft_order)
    out = np.zeros(p.shape, dtype=np.complex128)
    fac = np.ones(())
    sel_g, sel_u = [], []
    for d, (icf, iu, ig) in enumerate(maps):
        shp = [1] * p.ndim
        shp[d] = -1
        fac = fac * p.corfac[d][icf].reshape(shp)
        sel_g.append(ig)
        sel_u.append(iu)
    out[np.ix_(*sel_u)] = grid[np.ix_(*sel_g)] * fac
    return out


def u2nu(p, uniform, coord, forward, fft_order=False):
    """Full type-2 transform; returns values at the points (complex128)."""
    maps = _index_maps(p, fft_order)
    grid = np.zeros(p.nover, dtype=np.complex128)
    fac = np.ones(())
    sel_g, sel_u = [], []
    for d, (icf, iu, ig) in enumerate(maps):
        shp = [1] * p.ndim
        shp[d] = -1
        fac = fac * p.corfac[d][icf].reshape(shp)
        sel_g.append(ig)
        sel_u.append(iu)
    grid[np.ix_(*sel_g)] = np.asarray(uniform)[np.ix_(*sel_u)] * fac
    grid = _fft(grid, forward)
    return interpolate(p, grid, coord)


# ----------------------------------------------------------------------------
# direct transforms and metrics
# ----------------------------------------------------------------------------

def direct_nu2u(coord, values, shape, forward, periodicity=2 * math.pi, fft_order=False,
                chunk=4096):
    """FP64 direct NUDFT, type 1 (python/test/test_nufft.py:32-43)."""
    coord = np.asarray(coord, dtype=np.float64)
    ndim = len(shape)
    if np.ndim(periodicity) == 0:
        periodicity = [periodicity] * ndim
    isign = -1 if forward else 1
    ks = [(-(s // 2) + np.arange(s)) * (2 * math.pi / per) for s, per in zip(shape, periodicity)]
    res = np.zeros(shape, dtype=np.complex128)
    vals = np.asarray(values).astype(np.complex128)
    for lo in range(0, coord.shape[0], chunk):
        c = coord[lo:lo + chunk]
        v = vals[lo:lo + chunk]
        facs = [np.exp(isign * 1j * np.outer(c[:, d], ks[d])) for d in range(ndim)]
        if ndim == 1:
            res += v @ facs[0]
        elif ndim == 2:
            res += np.einsum("m,mi,mj->ij", v, facs[0], facs[1], optimize=True)
        else:
            res += np.einsum("m,mi,mj,mk->ijk", v, facs[0], facs[1], facs[2], optimize=True)
    if fft_order:
        res = np.fft.ifftshift(res)
    return res


def direct_u2nu(uniform, coord, forward, periodicity=2 * math.pi, fft_order=False,
                chunk=4096):
    """FP64 direct NUDFT, type 2 (the adjoint of direct_nu2u)."""
    uniform = np.asarray(uniform).astype(np.complex128)
    shape = uniform.shape
    if fft_order:
        uniform = np.fft.fftshift(uniform)
    coord = np.asarray(coord, dtype=np.float64)
    ndim = len(shape)
    if np.ndim(periodicity) == 0:
        periodicity = [periodicity] * ndim
    isign = -1 if forward else 1
    ks = [(-(s // 2) + np.arange(s)) * (2 * math.pi / per) for s, per in zip(shape, periodicity)]
    out = np.zeros(coord.shape[0], dtype=np.complex128)
    for lo in range(0, coord.shape[0], chunk):
        c = coord[lo:lo + chunk]
        facs = [np.exp(isign * 1j * np.outer(c[:, d], ks[d])) for d in range(ndim)]
        if ndim == 1:
            out[lo:lo + chunk] = facs[0] @ uniform
        elif ndim == 2:
            out[lo:lo + chunk] = np.einsum("mi,mj,ij->m", facs[0], facs[1], uniform, optimize=True)
        else:
            out[lo:lo + chunk] = np.einsum("mi,mj,mk,ijk->m", facs[0], facs[1], facs[2],
                                           uniform, optimize=True)
    return out


def direct_u2nu_dcoord(uniform, coord, forward, weights, periodicity=2 * math.pi,
                       fft_order=False, chunk=2048):
    """FP64 direct coordinate gradient of the type-2 transform, contracted with
    weights: out[j, d] = Re(conj(w_j) * d/dx_{j,d} sum_k u_k exp(s i K.x_j)),
    K_d = k_d 2 pi / period_d.  DUCC has no counterpart; this is the derivative
    of direct_u2nu, used to pin the library's derivative-kernel gradients."""
    uniform = np.asarray(uniform).astype(np.complex128)
    shape = uniform.shape
    if fft_order:
        uniform = np.fft.fftshift(uniform)
    coord = np.asarray(coord, dtype=np.float64)
    w = np.asarray(weights).astype(np.complex128)
    ndim = len(shape)
    if np.ndim(periodicity) == 0:
        periodicity = [periodicity] * ndim
    isign = -1 if forward else 1
    ks = [(-(s // 2) + np.arange(s)) * (2 * math.pi / per) for s, per in zip(shape, periodicity)]
    out = np.zeros(coord.shape, dtype=np.float64)
    for lo in range(0, coord.shape[0], chunk):
        c = coord[lo:lo + chunk]
        facs = [np.exp(isign * 1j * np.outer(c[:, d], ks[d])) for d in range(ndim)]
        dfacs = [f * (isign * 1j * ks[d])[None, :] for d, f in enumerate(facs)]
        for d in range(ndim):
            fs = [dfacs[e] if e == d else facs[e] for e in range(ndim)]
            if ndim == 1:
                v = fs[0] @ uniform
            elif ndim == 2:
                v = np.einsum("mi,mj,ij->m", fs[0], fs[1], uniform, optimize=True)
            else:
                v = np.einsum("mi,mj,mk,ijk->m", fs[0], fs[1], fs[2], uniform, optimize=True)
            out[lo:lo + chunk, d] = (np.conj(w[lo:lo + chunk]) * v).real
    return out


def l2error(a, b):
    """sqrt(sum|a-b|^2 / max(sum|a|^2, sum|b|^2)) in long double (misc_pymod.cc:129-185)."""
    a = np.asarray(a).astype(np.clongdouble).ravel()
    b = np.asarray(b).astype(np.clongdouble).ravel()
    sa = np.sum(np.abs(a) ** 2)
    sb = np.sum(np.abs(b) ** 2)
    sd = np.sum(np.abs(a - b) ** 2)
    m = max(sa, sb)
    if m == 0:
        return 0.0
    return float(np.sqrt(sd / m))


def vdot(a, b):
    """sum(conj(a)*b) in long double (misc_pymod.cc:52-127)."""
    a = np.asarray(a).astype(np.clongdouble).ravel()
    b = np.asarray(b).astype(np.clongdouble).ravel()
    return complex(np.sum(np.conj(a) * b))

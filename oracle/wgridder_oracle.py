"""Direct (exact) sums of the w-gridder's operators - TEST INFRASTRUCTURE ONLY.

CPU restatement, in numpy, of the definitions DUCC's own tests check its
w-gridder against (python/test/test_wgridder.py:34-92, explicit_gridder /
explicit_degridder), used by tests/ as the checker of ``ducc_b200.wgridder``.
Nothing in the product imports this module.

For pixel (i, j) of an nx x ny image, x = l0 + (i - nx/2) pixsize_x and
y = m0 + (j - ny/2) pixsize_y, with the image centre (l0, m0) = (center_x,
center_y), each negated where that axis is flipped (DUCC's lshift / mshift,
src/ducc0/wgridder/wgridder.h:1648), n = sqrt(1 - x^2 - y^2) (its
continuation -sqrt(x^2 + y^2 - 1) beyond the horizon), and visibility
(row, chan) at (u, v, w) = uvw[row] freq[chan] / c:
    dirty(i, j) = sum Re(vis wgt e^{2 pi i (x u + y v - w (n - 1))}) / n
    vis(row, chan) = wgt sum_ij dirty(i, j) / n e^{-2 pi i (x u + y v - w (n - 1))}
without the w term, n = 1; masked visibilities take no part (and are 0).
Sums run over chunks of pixels in complex128.
"""
import numpy as np

SPEED_OF_LIGHT = 299792458.


def _pixels(nx, ny, psx, psy, center_x, center_y, apply_w):
    x, y = np.meshgrid(*[-ss / 2 + np.arange(ss) for ss in (nx, ny)], indexing="ij")
    x = x * psx + center_x
    y = y * psy + center_y
    if apply_w:
        eps = x ** 2 + y ** 2
        tmp = np.sqrt(np.abs(1. - eps))
        nm1 = np.where(eps <= 1, tmp - 1., -tmp - 1.)
    else:
        nm1 = np.zeros_like(x)
    return x.ravel(), y.ravel(), nm1.ravel()


def _uvw(uvw, freq, flip_u=False, flip_v=False, flip_w=False):
    f = np.asarray(freq, np.float64) / SPEED_OF_LIGHT
    s = np.array([-1. if flip_u else 1., -1. if flip_v else 1., -1. if flip_w else 1.])
    c = np.asarray(uvw, np.float64) * s
    return (np.outer(c[:, 0], f).ravel(), np.outer(c[:, 1], f).ravel(),
            np.outer(c[:, 2], f).ravel())


def explicit_gridder(uvw, freq, vis, wgt, nx, ny, psx, psy, apply_w, mask, divide_by_n=True,
                     center_x=0., center_y=0., flip_u=False, flip_v=False, flip_w=False):
    x, y, nm1 = _pixels(nx, ny, psx, psy, -center_x if flip_u else center_x,
                        -center_y if flip_v else center_y, apply_w)
    u, v, w = _uvw(uvw, freq, flip_u, flip_v, flip_w)
    c = np.asarray(vis, np.complex128).ravel().copy()
    if wgt is not None:
        c *= np.asarray(wgt, np.float64).ravel()
    if mask is not None:
        c *= (np.asarray(mask).ravel() != 0)
    res = np.zeros(nx * ny)
    for a in range(0, x.size, 4096):
        b = min(x.size, a + 4096)
        ph = 2j * np.pi * (np.outer(x[a:b], u) + np.outer(y[a:b], v) - np.outer(nm1[a:b], w))
        res[a:b] = (np.exp(ph) @ c).real
    res = res.reshape(nx, ny)
    if apply_w and divide_by_n:
        n = (nm1 + 1.).reshape(nx, ny)
        res = np.where(n > 0, res / np.where(n > 0, n, 1.), 0.)
    return res


def explicit_degridder(uvw, freq, dirty, wgt, psx, psy, apply_w, mask, divide_by_n=True,
                       center_x=0., center_y=0., flip_u=False, flip_v=False, flip_w=False):
    nx, ny = dirty.shape
    x, y, nm1 = _pixels(nx, ny, psx, psy, -center_x if flip_u else center_x,
                        -center_y if flip_v else center_y, apply_w)
    u, v, w = _uvw(uvw, freq, flip_u, flip_v, flip_w)
    d = np.asarray(dirty, np.float64).ravel()
    if apply_w and divide_by_n:
        n = nm1 + 1.
        d = np.where(n > 0, d / np.where(n > 0, n, 1.), 0.)
    res = np.zeros(u.size, np.complex128)
    for a in range(0, x.size, 4096):
        b = min(x.size, a + 4096)
        ph = -2j * np.pi * (np.outer(u, x[a:b]) + np.outer(v, y[a:b]) - np.outer(w, nm1[a:b]))
        res += np.exp(ph) @ d[a:b]
    res = res.reshape(np.asarray(uvw).shape[0], np.asarray(freq).shape[0])
    if wgt is not None:
        res = res * np.asarray(wgt, np.float64)
    if mask is not None:
        res = res * (np.asarray(mask) != 0)
    return res


def vdot(a, b):
    """sum(conj(a) * b) in extended precision (DUCC's ducc0.misc.vdot)."""
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    ca = a.astype(np.complex128) if np.iscomplexobj(a) else a.astype(np.float64)
    cb = b.astype(np.complex128) if np.iscomplexobj(b) else b.astype(np.float64)
    return np.vdot(ca, cb)


def l2error(a, b):
    """||a - b|| / max(||a||, ||b||) (DUCC's ducc0.misc.l2error)."""
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    nd = np.linalg.norm(a - b)
    m = max(np.linalg.norm(a), np.linalg.norm(b))
    return 0. if m == 0 else nd / m

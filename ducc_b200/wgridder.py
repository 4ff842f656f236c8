"""Radio-interferometric (de)gridding with w-stacking on the GPU: a drop-in for
``ducc0.wgridder`` (``vis2dirty``, ``dirty2vis``, ``ms2dirty``, ``dirty2ms``;
python/wgridder_pymod.cc:612-656 for the signatures and keyword defaults).

The work runs in the CUDA library through the C-ABI (``dnufft_vis2dirty``,
``dnufft_dirty2vis`` in include/ducc_b200.h): every w plane is a 2D type-1
(gridding) or type-2 (degridding) transform of this package, with the w
screens and the global corrections in their own kernels.  Arguments may be
numpy arrays (copied to the current CUDA device and the result copied back) or
torch CUDA tensors (used in place; the result is a tensor).  As in DUCC, the
data type of ``vis`` (gridding) or ``dirty`` (degridding) sets the precision.
"""
import ctypes

import numpy as np

from . import _capi as C

__all__ = ["vis2dirty", "dirty2vis", "ms2dirty", "dirty2ms", "wgrid_params"]


def _torch():
    import torch
    return torch


def _dev(x, dtype=None):
    """(tensor on the current CUDA device, was numpy) for an array or None."""
    if x is None:
        return None, False
    torch = _torch()
    if C.is_torch(x):
        if not x.is_cuda:
            raise ValueError("torch tensors must live on a CUDA device")
        return (x if dtype is None else x.to(dtype)), False
    a = np.asarray(x)
    if dtype is not None:
        a = a.astype(dtype, copy=False)
    a = np.ascontiguousarray(a)
    if not a.flags.writeable:   # (torch wraps only writable arrays)
        a = a.copy()
    return torch.from_numpy(a).cuda(), True


def _opts(nthreads, verbosity, sigma_min, sigma_max, center_x, center_y, do_wgridding, flip_u,
          flip_v, flip_w, divide_by_n, allow_nshift, double_precision_accumulation=False,
          planes=None):
    o = C.WgridOpts()
    C.lib().dnufft_wgrid_default_opts(ctypes.byref(o))
    if int(nthreads) < 0:
        raise ValueError("nthreads must be >= 0")
    o.nthreads = int(nthreads)
    o.verbosity = int(verbosity)
    o.sigma_min = float(sigma_min)
    o.sigma_max = float(sigma_max)
    o.center_x = float(center_x)
    o.center_y = float(center_y)
    o.do_wgridding = 1 if do_wgridding else 0
    o.flip_u = 1 if flip_u else 0
    o.flip_v = 1 if flip_v else 0
    o.flip_w = 1 if flip_w else 0
    o.divide_by_n = 1 if divide_by_n else 0
    o.allow_nshift = 1 if allow_nshift else 0
    o.double_precision_accumulation = 1 if double_precision_accumulation else 0
    if planes is not None:
        b, c = planes
        if int(b) < 0 or int(c) < 0:
            raise ValueError("planes must be (begin >= 0, count >= 0)")
        o.plane_begin, o.plane_count = int(b), int(c)
    return o


def _real_of(t):
    torch = _torch()
    return {torch.complex64: torch.float32, torch.complex128: torch.float64}[t.dtype]


def _complex_of(t):
    torch = _torch()
    return {torch.float32: torch.complex64, torch.float64: torch.complex128}[t.dtype]


def _common(uvw, freq, wgt, mask, data, real_dtype):
    torch = _torch()
    d_uvw, host = _dev(uvw, np.float64 if not C.is_torch(uvw) else None)
    d_freq, _ = _dev(freq, np.float64 if not C.is_torch(freq) else None)
    if d_uvw.dtype != torch.float64 or d_freq.dtype != torch.float64:
        raise TypeError("uvw and freq must be float64")
    d_wgt = None
    if wgt is not None:
        d_wgt, _ = _dev(wgt)
        if d_wgt.dtype != real_dtype:
            raise TypeError("wgt must be real with the precision of the data")
    d_mask = None
    if mask is not None:
        if C.is_torch(mask):
            d_mask = mask.to(torch.uint8)
        else:
            d_mask, _ = _dev(np.asarray(mask).astype(np.uint8))
    return d_uvw, d_freq, d_wgt, d_mask, host


def _desc(x):
    return None if x is None else ctypes.byref(C.describe(x))


def vis2dirty(*, uvw, freq, vis, wgt=None, npix_x=0, npix_y=0, pixsize_x, pixsize_y, epsilon,
              do_wgridding=False, nthreads=1, verbosity=0, mask=None, flip_u=False, flip_v=False,
              flip_w=False, divide_by_n=True, dirty=None, sigma_min=1.1, sigma_max=2.6,
              center_x=0., center_y=0., allow_nshift=True, gpu=False,
              double_precision_accumulation=False, planes=None):
    """Visibilities to dirty image (``ducc0.wgridder.vis2dirty``).  ``gpu``
    (DUCC's SYCL switch) is accepted and has no effect.  Addition:
    ``planes=(begin, count)`` grids only those w planes (a share of a split
    over processes: the images of a partition of the planes sum to the whole
    image; ``ducc_b200.distributed.vis2dirty_split`` does the split)."""
    torch = _torch()
    d_vis, host_vis = _dev(vis)
    if d_vis.dtype not in (torch.complex64, torch.complex128):
        raise TypeError("type matching failed: 'vis' has neither type 'c8' nor 'c16'")
    rdt = _real_of(d_vis)
    d_uvw, d_freq, d_wgt, d_mask, host = _common(uvw, freq, wgt, mask, d_vis, rdt)
    if (npix_x == 0) != (npix_y == 0):
        raise RuntimeError("inconsistent dirty image dimensions")
    host_out = False
    if dirty is None:
        if npix_x == 0:
            raise RuntimeError("npix_x and npix_y, or dirty, must be given")
        d_dirty = torch.empty((int(npix_x), int(npix_y)), dtype=rdt, device=d_vis.device)
        host_out = host_vis
    else:
        if npix_x and tuple(dirty.shape) != (int(npix_x), int(npix_y)):
            raise RuntimeError("dirty has the wrong shape")
        if C.is_torch(dirty):
            d_dirty = dirty
        else:
            d_dirty = torch.empty(tuple(dirty.shape), dtype=rdt, device=d_vis.device)
            host_out = True
    o = _opts(nthreads, verbosity, sigma_min, sigma_max, center_x, center_y, do_wgridding,
              flip_u, flip_v, flip_w, divide_by_n, allow_nshift, double_precision_accumulation,
              planes)
    st = ctypes.c_void_p(torch.cuda.current_stream(d_vis.device).cuda_stream)
    a_dirty = C.describe(d_dirty)
    C.check(C.lib().dnufft_vis2dirty(_desc(d_uvw), _desc(d_freq), _desc(d_vis), _desc(d_wgt),
                                     _desc(d_mask), float(pixsize_x), float(pixsize_y),
                                     float(epsilon), ctypes.byref(o), ctypes.byref(a_dirty), st))
    if dirty is not None and not C.is_torch(dirty):
        dirty[...] = d_dirty.cpu().numpy()
        return dirty
    return d_dirty.cpu().numpy() if host_out else d_dirty


def dirty2vis(*, uvw, freq, dirty, wgt=None, pixsize_x, pixsize_y, epsilon, do_wgridding=False,
              nthreads=1, verbosity=0, mask=None, flip_u=False, flip_v=False, flip_w=False,
              divide_by_n=True, vis=None, sigma_min=1.1, sigma_max=2.6, center_x=0.,
              center_y=0., allow_nshift=True, gpu=False, planes=None):
    """Dirty image to visibilities (``ducc0.wgridder.dirty2vis``).  ``gpu`` is
    accepted and has no effect.  Addition: ``planes=(begin, count)`` as in
    ``vis2dirty`` (the visibilities of a partition of the planes sum to the
    whole result)."""
    torch = _torch()
    d_dirty, host_dirty = _dev(dirty)
    if d_dirty.dtype not in (torch.float32, torch.float64):
        raise TypeError("type matching failed: 'dirty' has neither type 'f4' nor 'f8'")
    d_uvw, d_freq, d_wgt, d_mask, host = _common(uvw, freq, wgt, mask, d_dirty, d_dirty.dtype)
    nrows, nchan = int(d_uvw.shape[0]), int(d_freq.shape[0])
    cdt = _complex_of(d_dirty)
    if vis is not None and C.is_torch(vis):
        d_vis = vis
    else:
        d_vis = torch.empty((nrows, nchan), dtype=cdt, device=d_dirty.device)
    o = _opts(nthreads, verbosity, sigma_min, sigma_max, center_x, center_y, do_wgridding,
              flip_u, flip_v, flip_w, divide_by_n, allow_nshift, planes=planes)
    st = ctypes.c_void_p(torch.cuda.current_stream(d_dirty.device).cuda_stream)
    a_vis = C.describe(d_vis)
    C.check(C.lib().dnufft_dirty2vis(_desc(d_uvw), _desc(d_freq), _desc(d_dirty), _desc(d_wgt),
                                     _desc(d_mask), float(pixsize_x), float(pixsize_y),
                                     float(epsilon), ctypes.byref(o), ctypes.byref(a_vis), st))
    if vis is not None and not C.is_torch(vis):
        vis[...] = d_vis.cpu().numpy()
        return vis
    return d_vis.cpu().numpy() if (host_dirty and vis is None) else d_vis


def ms2dirty(uvw, freq, ms, wgt=None, npix_x=None, npix_y=None, pixsize_x=None, pixsize_y=None,
             nu=0, nv=0, epsilon=None, do_wstacking=False, nthreads=1, verbosity=0, mask=None,
             double_precision_accumulation=False, gpu=False):
    """``ducc0.wgridder.ms2dirty``: ``vis2dirty`` with its defaults (``nu``,
    ``nv`` ignored, as in DUCC)."""
    for name, val in (("npix_x", npix_x), ("npix_y", npix_y), ("pixsize_x", pixsize_x),
                      ("pixsize_y", pixsize_y), ("epsilon", epsilon)):
        if val is None:
            raise TypeError("ms2dirty(): missing argument '%s'" % name)
    return vis2dirty(uvw=uvw, freq=freq, vis=ms, wgt=wgt, npix_x=npix_x, npix_y=npix_y,
                     pixsize_x=pixsize_x, pixsize_y=pixsize_y, epsilon=epsilon,
                     do_wgridding=do_wstacking, nthreads=nthreads, verbosity=verbosity,
                     mask=mask, double_precision_accumulation=double_precision_accumulation)


def dirty2ms(uvw, freq, dirty, wgt=None, pixsize_x=None, pixsize_y=None, nu=0, nv=0,
             epsilon=None, do_wstacking=False, nthreads=1, verbosity=0, mask=None, gpu=False):
    """``ducc0.wgridder.dirty2ms``: ``dirty2vis`` with its defaults."""
    for name, val in (("pixsize_x", pixsize_x), ("pixsize_y", pixsize_y),
                      ("epsilon", epsilon)):
        if val is None:
            raise TypeError("dirty2ms(): missing argument '%s'" % name)
    return dirty2vis(uvw=uvw, freq=freq, dirty=dirty, wgt=wgt, pixsize_x=pixsize_x,
                     pixsize_y=pixsize_y, epsilon=epsilon, do_wgridding=do_wstacking,
                     nthreads=nthreads, verbosity=verbosity, mask=mask)


def wgrid_params(*, uvw, freq, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, vis=None,
                 wgt=None, mask=None, do_wgridding=False, nthreads=1,
                 sigma_min=1.1, sigma_max=2.6, center_x=0., center_y=0., flip_u=False,
                 flip_v=False, flip_w=False, allow_nshift=True):
    """The kernel, grid and w planes ``vis2dirty`` (``vis`` given) or
    ``dirty2vis`` (``vis`` None; the precision then is that of ``wgt``, double
    without it) would use, as a dict (no DUCC counterpart; DUCC prints them
    with ``verbosity=1``)."""
    torch = _torch()
    d_vis = None
    if vis is not None:
        d_vis, _ = _dev(vis)
        rdt = _real_of(d_vis)
    elif wgt is not None:
        rdt = _dev(wgt)[0].dtype
    else:
        rdt = torch.float64
    d_uvw, d_freq, d_wgt, d_mask, _ = _common(uvw, freq, wgt, mask, d_vis, rdt)
    o = _opts(nthreads, 0, sigma_min, sigma_max, center_x, center_y, do_wgridding, flip_u,
              flip_v, flip_w, True, allow_nshift)
    info = C.WgridInfo()
    st = ctypes.c_void_p(torch.cuda.current_stream(d_uvw.device).cuda_stream)
    C.check(C.lib().dnufft_wgrid_params(_desc(d_uvw), _desc(d_freq), _desc(d_vis), _desc(d_wgt),
                                        _desc(d_mask), int(npix_x), int(npix_y),
                                        float(pixsize_x), float(pixsize_y), float(epsilon),
                                        1 if vis is not None else 0, ctypes.byref(o),
                                        ctypes.byref(info), st))
    return {k: getattr(info, k) for k, _ in C.WgridInfo._fields_}

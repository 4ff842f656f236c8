"""Autotuner for the kernel support, oversampling factor and tile size of a
transform, by measurement on the GPU.

DUCC picks (W, sigma) with a CPU cost model (``findNufftParameters``,
src/ducc0/nufft/nufft.h:155-208) and a fixed tile size.  On a B200 the balance
between the spreading / interpolation work (grows with W) and the FFT work
(grows with sigma) differs, and so does the best tile size for small grids, so
``tune`` times every candidate on the actual coordinates: for each support W,
the smallest oversampling factor that reaches epsilon
(``dnufft_kernel_candidates``), for each tile size, a planned type 1 + type 2
pair over ``ntrans`` transforms, and keeps the fastest.  Results are cached per
(shape, epsilon, precision, npoints bucket, ntrans).

``plan_kwargs(choice)`` turns a result into ``nufft.plan`` keywords
(``force_kernel``, ``force_nover``, ``log2tile``).
"""
import ctypes
import math

import numpy as np

from . import _capi as C
from . import nufft

__all__ = ["candidates", "tune", "plan_kwargs"]

_CACHE = {}


def candidates(shape, epsilon, singleprec, sigma_min=1.1, sigma_max=2.6):
    """(kernel_index, W, ofactor, nover) for every usable kernel support."""
    nd = len(shape)
    mx = 32
    shp = (ctypes.c_int64 * 3)(*(list(shape) + [1] * (3 - nd)))
    kidx = (ctypes.c_int32 * mx)()
    supp = (ctypes.c_int32 * mx)()
    ofac = (ctypes.c_double * mx)()
    nov = (ctypes.c_int64 * (3 * mx))()
    cnt = ctypes.c_int()
    C.check(C.lib().dnufft_kernel_candidates(nd, shp, 1 if singleprec else 0, float(epsilon),
                                             float(sigma_min), float(sigma_max), mx, kidx, supp,
                                             ofac, nov, ctypes.byref(cnt)))
    return [(kidx[i], supp[i], ofac[i], [nov[3 * i + d] for d in range(nd)])
            for i in range(cnt.value)]


def plan_kwargs(choice):
    return {"force_kernel": choice["kernel_index"], "force_nover": choice["nover"],
            "log2tile": choice["log2tile"]}


def _time_candidate(coord, shape, epsilon, ntrans, kw, reps):
    import torch
    dev = coord.device
    f64 = coord.dtype == torch.float64
    cdt = torch.complex128 if f64 else torch.complex64
    M = coord.shape[0]
    g = torch.Generator(device=dev).manual_seed(0)
    vals = torch.randn((ntrans, M), dtype=cdt, device=dev, generator=g)
    grid = torch.randn((ntrans,) + tuple(shape), dtype=cdt, device=dev, generator=g)
    out = torch.empty((ntrans,) + tuple(shape), dtype=cdt, device=dev)
    pts = torch.empty((ntrans, M), dtype=cdt, device=dev)
    p = nufft.plan(nu2u=True, coord=coord, grid_shape=shape, epsilon=epsilon, **kw)

    def run():
        for t in range(ntrans):
            p.nu2u(points=vals[t], forward=True, out=out[t])
            p.u2nu(grid=grid[t], forward=False, out=pts[t])

    run()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / reps


def tune(coord, shape, epsilon, ntrans=1, sigma_min=1.1, sigma_max=2.6, reps=3, cache=True):
    """Fastest (kernel, oversampled size, tile) for this transform, measured
    on the GPU with the given coordinates (a torch CUDA tensor (M, ndim)).
    Returns a dict with kernel_index, supp, ofactor, nover, log2tile, ms and
    the measured table of all candidates."""
    import torch
    shape = tuple(int(s) for s in shape)
    single = coord.dtype == torch.float32
    M = coord.shape[0]
    key = (shape, float(epsilon), single, int(round(math.log2(max(M, 1)))), int(ntrans))
    if cache and key in _CACHE:
        return _CACHE[key]
    nd = len(shape)
    tiles = [None] if nd != 2 else [None, 4 if single else 5]
    table = []
    for kidx, W, of, nov in candidates(shape, epsilon, single, sigma_min, sigma_max):
        for lt in tiles:
            kw = {"force_kernel": kidx, "force_nover": nov, "log2tile": lt}
            ms = _time_candidate(coord, shape, epsilon, ntrans, kw, reps)
            dflt = (5 if single else 4) if nd == 2 else (9 if nd == 1 else 4)
            table.append({"kernel_index": kidx, "supp": W, "ofactor": of, "nover": nov,
                          "log2tile": lt if lt is not None else dflt, "ms": ms})
    best = dict(min(table, key=lambda r: r["ms"]))
    best["table"] = table
    if cache:
        _CACHE[key] = best
    return best

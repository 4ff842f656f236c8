"""Drop-in for ``ducc0.nufft`` running on a B200 GPU.

Same functions, keyword-only arguments, defaults and error behaviour as DUCC's
Python NUFFT module (python/nufft_pymod.cc:445-471):

* ``nu2u(*, points, coord, forward, epsilon, nthreads=1, out, verbosity=0,
  sigma_min=1.2, sigma_max=2.51, periodicity=2*pi, fft_order=False)``
* ``u2nu(*, grid, coord, forward, epsilon, nthreads=1, out=None, ...)``
* ``bestEpsilon(*, ndim, singleprec, sigma_min=1.1, sigma_max=2.6)``
* ``plan(*, nu2u, coord, grid_shape, epsilon, nthreads=0, sigma_min=1.1,
  sigma_max=2.6, periodicity=2*pi, fft_order=False)`` with ``.nu2u`` / ``.u2nu``

Arrays may be numpy arrays (host; copied through the device inside the call)
or torch CUDA tensors (used in place).  The computation precision is the data
precision, as in DUCC.  ``nthreads`` only feeds DUCC's parameter cost model, so
the same (kernel, oversampled size) is chosen as DUCC would choose.

Extensions beyond DUCC's signature (keyword-only, optional): ``spreader``
('auto' | 'plain' | 'tc') and ``stream`` (a CUDA stream handle), and the
coordinate-gradient transform ``u2nu_dcoord`` (function and plan method) used
by ``ducc_b200.autograd``.
"""
import ctypes
import math

import numpy as np

from . import _capi as C

__all__ = ["nu2u", "u2nu", "u2nu_dcoord", "bestEpsilon", "plan", "find_parameters"]


def _np_complex_for(code):
    return np.complex128 if code == C.C128 else np.complex64


def _prepare_in(x):
    """numpy inputs become C-contiguous; torch tensors pass through."""
    if C.is_torch(x):
        return x
    x = np.asarray(x)
    return np.ascontiguousarray(x)


class _OutProxy:
    """Output handling: numpy outputs that are not C-contiguous are computed
    into a contiguous temporary and copied back."""

    def __init__(self, out):
        self.user = out
        if C.is_torch(out) or out.flags.c_contiguous:
            self.buf = out
        else:
            self.buf = np.empty(out.shape, dtype=out.dtype)

    def finish(self):
        if self.buf is not self.user:
            self.user[...] = self.buf
        return self.user


def _check_types(data, coord):
    dc = C.dtype_code(data)
    cc = C.dtype_code(coord)
    if dc not in (C.C64, C.C128) or cc not in (C.F32, C.F64):
        raise RuntimeError("not yet supported")
    return dc, cc


def nu2u(*, points, coord, forward, epsilon, nthreads=1, out=None, verbosity=0,
         sigma_min=1.2, sigma_max=2.51, periodicity=2 * math.pi, fft_order=False,
         spreader="auto", stream=None):
    """Type 1 non-uniform FFT (non-uniform to uniform).  ``out`` is mandatory:
    its shape defines the uniform grid.  Returns ``out``."""
    if out is None:
        raise TypeError("nu2u(): 'out' is mandatory, since its shape defines the grid")
    points = _prepare_in(points)
    coord = _prepare_in(coord)
    _check_types(points, coord)
    op = _OutProxy(out)
    ndim = len(out.shape)
    o = C.make_opts(False, nthreads, sigma_min, sigma_max, periodicity, fft_order, verbosity,
                    spreader, ndim)
    a_p, a_c, a_o = C.describe(points), C.describe(coord), C.describe(op.buf)
    C.check(C.lib().dnufft_nu2u(ctypes.byref(a_p), ctypes.byref(a_c), 1 if forward else 0,
                                float(epsilon), ctypes.byref(a_o), ctypes.byref(o),
                                C.stream_of(points, coord, op.buf, stream=stream)))
    return op.finish()


def u2nu(*, grid, coord, forward, epsilon, nthreads=1, out=None, verbosity=0,
         sigma_min=1.2, sigma_max=2.51, periodicity=2 * math.pi, fft_order=False,
         stream=None):
    """Type 2 non-uniform FFT (uniform to non-uniform).  Returns the values at
    the points (``out`` if given)."""
    grid = _prepare_in(grid)
    coord = _prepare_in(coord)
    dc, _ = _check_types(grid, coord)
    npts = coord.shape[0]
    if out is None:
        if C.is_torch(grid):
            import torch
            out = torch.empty(npts, dtype=grid.dtype, device=grid.device)
        else:
            out = np.empty(npts, dtype=_np_complex_for(dc))
    op = _OutProxy(out)
    ndim = len(grid.shape)
    o = C.make_opts(False, nthreads, sigma_min, sigma_max, periodicity, fft_order, verbosity,
                    "auto", ndim)
    a_g, a_c, a_o = C.describe(grid), C.describe(coord), C.describe(op.buf)
    C.check(C.lib().dnufft_u2nu(ctypes.byref(a_g), ctypes.byref(a_c), 1 if forward else 0,
                                float(epsilon), ctypes.byref(a_o), ctypes.byref(o),
                                C.stream_of(grid, coord, op.buf, stream=stream)))
    return op.finish()


def _dcoord_out(coord, out):
    if out is not None:
        return out
    if C.is_torch(coord):
        import torch
        return torch.empty(tuple(coord.shape), dtype=coord.dtype, device=coord.device)
    return np.empty(coord.shape, dtype=np.asarray(coord).dtype)


def u2nu_dcoord(*, grid, coord, forward, epsilon, weights, nthreads=1, out=None,
                sigma_min=1.2, sigma_max=2.51, periodicity=2 * math.pi, fft_order=False,
                stream=None):
    """Coordinate gradient of the type-2 transform contracted with ``weights``:
    ``out[j, d] = Re(conj(weights[j]) * d/dcoord[j, d] u2nu(grid, coord)[j])``
    (real, the coordinates' dtype).  No counterpart in DUCC."""
    grid = _prepare_in(grid)
    coord = _prepare_in(coord)
    weights = _prepare_in(weights)
    _check_types(grid, coord)
    op = _OutProxy(_dcoord_out(coord, out))
    ndim = len(grid.shape)
    o = C.make_opts(False, nthreads, sigma_min, sigma_max, periodicity, fft_order, 0, "auto", ndim)
    a_g, a_c, a_w, a_o = C.describe(grid), C.describe(coord), C.describe(weights), C.describe(op.buf)
    C.check(C.lib().dnufft_u2nu_dcoord(ctypes.byref(a_g), ctypes.byref(a_c), 1 if forward else 0,
                                       float(epsilon), ctypes.byref(a_w), ctypes.byref(a_o),
                                       ctypes.byref(o),
                                       C.stream_of(grid, coord, weights, op.buf, stream=stream)))
    return op.finish()


def bestEpsilon(*, ndim, singleprec, sigma_min=1.1, sigma_max=2.6):
    """Smallest achievable epsilon for the given dimensionality / precision."""
    r = ctypes.c_double()
    C.check(C.lib().dnufft_best_epsilon(int(ndim), 1 if singleprec else 0, float(sigma_min),
                                        float(sigma_max), ctypes.byref(r)))
    return r.value


def find_parameters(*, nu2u, grid_shape, npoints, epsilon, singleprec, coord_single=None,
                    nthreads=0, sigma_min=1.1, sigma_max=2.6):
    """(kernel-table row, oversampled shape) that DUCC's parameter choice gives
    for a transform of ``npoints`` points (findNufftParameters,
    src/ducc0/nufft/nufft.h:155-216; plan defaults).  Processes that split the
    points of one transform pass the total count and plan with
    ``force_kernel`` / ``force_nover``.  Runs on the host only."""
    shape = [int(x) for x in grid_shape]
    ndim = len(shape)
    if coord_single is None:
        coord_single = singleprec
    o = C.make_opts(True, nthreads, sigma_min, sigma_max, 2 * math.pi, False, 0, "auto", ndim)
    shp = (ctypes.c_int64 * 3)(*(shape + [1] * (3 - ndim)))
    kidx = ctypes.c_int32()
    nover = (ctypes.c_int64 * 3)()
    C.check(C.lib().dnufft_find_parameters(1 if nu2u else 0, ndim, shp, int(npoints),
                                           float(epsilon), 0 if singleprec else 1,
                                           0 if coord_single else 1, ctypes.byref(o),
                                           ctypes.byref(kidx), nover))
    return kidx.value, [int(nover[d]) for d in range(ndim)]


class plan:
    """NUFFT plan for fixed coordinates (DUCC's ``ducc0.nufft.plan``).

    Float32 coordinates make a single-precision plan (complex64 data), float64
    coordinates a double-precision one (complex128 data)."""

    def __init__(self, *, nu2u, coord, grid_shape, epsilon, nthreads=0, sigma_min=1.1,
                 sigma_max=2.6, periodicity=2 * math.pi, fft_order=False, spreader="auto",
                 stream=None, force_kernel=None, force_nover=None, log2tile=None):
        self._ptr = None
        coord = _prepare_in(coord)
        if C.dtype_code(coord) not in (C.F32, C.F64):
            raise RuntimeError("unsupported")
        shape = [int(s) for s in grid_shape]
        ndim = len(shape)
        if not 1 <= ndim <= 3:
            raise RuntimeError("unsupported dimensionality")
        self.grid_shape = tuple(shape)
        self.npoints = coord.shape[0]
        self._f64 = C.dtype_code(coord) == C.F64
        self._torch_device = coord.device if C.is_torch(coord) else None
        o = C.make_opts(True, nthreads, sigma_min, sigma_max, periodicity, fft_order, 0,
                        spreader, ndim, force_kernel, force_nover, log2tile)
        a_c = C.describe(coord)
        shp = (ctypes.c_int64 * 3)(*(shape + [1] * (3 - ndim)))
        ptr = ctypes.c_void_p()
        C.check(C.lib().dnufft_plan_create(1 if nu2u else 0, ctypes.byref(a_c), shp, ndim,
                                           float(epsilon), ctypes.byref(o),
                                           C.stream_of(coord, stream=stream),
                                           ctypes.byref(ptr)))
        self._ptr = ptr

    def __del__(self):
        if getattr(self, "_ptr", None):
            try:
                C.lib().dnufft_plan_destroy(self._ptr)
            except Exception:
                pass
            self._ptr = None

    def _alloc(self, like, shape):
        dt = np.complex128 if self._f64 else np.complex64
        if like is not None and C.is_torch(like):
            import torch
            return torch.empty(shape, dtype=torch.complex128 if self._f64 else torch.complex64,
                               device=like.device)
        return np.empty(shape, dtype=dt)

    def nu2u(self, *, forward, verbosity=0, points, out=None, stream=None):
        """Type 1 over the plan's points.  ``points`` of shape ``(M,)``, or
        ``(ntrans, M)`` for ntrans transforms at once (then ``out`` is
        ``(ntrans,) + grid_shape``; an extension of DUCC's plan)."""
        points = _prepare_in(points)
        if out is None:
            lead = tuple(points.shape[:-1]) if len(points.shape) == 2 else ()
            out = self._alloc(points, lead + self.grid_shape)
        op = _OutProxy(out)
        a_p, a_o = C.describe(points), C.describe(op.buf)
        C.check(C.lib().dnufft_plan_nu2u(self._ptr, 1 if forward else 0, int(verbosity),
                                         ctypes.byref(a_p), ctypes.byref(a_o),
                                         C.stream_of(points, op.buf, stream=stream)))
        return op.finish()

    def u2nu(self, *, forward, verbosity=0, grid, out=None, stream=None):
        """Type 2 at the plan's points.  ``grid`` of shape ``grid_shape``, or
        ``(ntrans,) + grid_shape`` for ntrans transforms at once (then ``out``
        is ``(ntrans, M)``; an extension of DUCC's plan)."""
        grid = _prepare_in(grid)
        if out is None:
            lead = tuple(grid.shape[:1]) if len(grid.shape) == len(self.grid_shape) + 1 else ()
            out = self._alloc(grid, lead + (self.npoints,))
        op = _OutProxy(out)
        a_g, a_o = C.describe(grid), C.describe(op.buf)
        C.check(C.lib().dnufft_plan_u2nu(self._ptr, 1 if forward else 0, int(verbosity),
                                         ctypes.byref(a_g), ctypes.byref(a_o),
                                         C.stream_of(grid, op.buf, stream=stream)))
        return op.finish()

    # -- B200 extras
    def u2nu_dcoord(self, *, forward, grid, weights, out=None, stream=None):
        """Coordinate gradient of this plan's type-2 transform contracted with
        ``weights`` (see the module-level ``u2nu_dcoord``)."""
        grid = _prepare_in(grid)
        weights = _prepare_in(weights)
        if out is None:
            ct = np.float64 if self._f64 else np.float32
            if C.is_torch(grid):
                import torch
                out = torch.empty((self.npoints, len(self.grid_shape)),
                                  dtype=torch.float64 if self._f64 else torch.float32,
                                  device=grid.device)
            else:
                out = np.empty((self.npoints, len(self.grid_shape)), dtype=ct)
        op = _OutProxy(out)
        a_g, a_w, a_o = C.describe(grid), C.describe(weights), C.describe(op.buf)
        C.check(C.lib().dnufft_plan_u2nu_dcoord(self._ptr, 1 if forward else 0, ctypes.byref(a_g),
                                                ctypes.byref(a_w), ctypes.byref(a_o),
                                                C.stream_of(grid, weights, op.buf, stream=stream)))
        return op.finish()

    # -- type 1 in two halves (one transform's points split over several GPUs)
    def spread(self, *, points, out=None, stream=None):
        """Spread this plan's points with the values ``points`` into an
        oversampled grid: a C-contiguous CUDA tensor of the plan's data type and
        oversampled shape (``info()["nover"]``), zeroed first and returned.
        Summing such grids over plans of disjoint point sets and passing the sum
        to ``grid_to_uniform`` gives the type 1 of all points (the plans must
        share kernel and oversampled sizes, see ``find_parameters``)."""
        import torch
        points = _prepare_in(points)
        if out is None:
            dev = points.device if C.is_torch(points) else (
                self._torch_device or torch.device("cuda", torch.cuda.current_device()))
            out = torch.empty(tuple(self.info()["nover"]),
                              dtype=torch.complex128 if self._f64 else torch.complex64,
                              device=dev)
        a_p, a_g = C.describe(points), C.describe(out)
        C.check(C.lib().dnufft_plan_spread(self._ptr, ctypes.byref(a_p), ctypes.byref(a_g),
                                           C.stream_of(points, out, stream=stream)))
        return out

    def grid_to_uniform(self, *, forward, grid, out=None, stream=None):
        """FFT and correction of an oversampled grid (as from ``spread``, maybe
        summed over several plans; it is overwritten) into the uniform grid
        ``out`` (allocated like ``nu2u``'s when None); returns ``out``."""
        if out is None:
            out = self._alloc(grid, self.grid_shape)
        op = _OutProxy(out)
        a_g, a_o = C.describe(grid), C.describe(op.buf)
        C.check(C.lib().dnufft_plan_grid_to_uniform(self._ptr, 1 if forward else 0,
                                                    ctypes.byref(a_g), ctypes.byref(a_o),
                                                    C.stream_of(grid, op.buf, stream=stream)))
        return op.finish()

    def rows_fft(self, *, forward, rows, stream=None):
        """2D type 1: FFT along axis 1 of a slab of rows of an oversampled grid
        (a C-contiguous CUDA tensor of shape (r, nover[1])), in place; only the
        kept columns (the first (N1+1)//2 and the last N1//2) are written.
        Returns ``rows``."""
        a_r = C.describe(rows)
        C.check(C.lib().dnufft_plan_rows_fft(self._ptr, 1 if forward else 0, ctypes.byref(a_r),
                                             C.stream_of(rows, stream=stream)))
        return rows

    def cols_to_uniform(self, *, forward, grid, out=None, stream=None):
        """2D type 1: column FFTs of the kept columns of an oversampled grid
        whose rows ``rows_fft`` has transformed, correction and crop into
        ``out``; returns ``out``.  ``grid``: the whole (nover[0], nover[1])
        grid or its kept columns packed, (nover[0], N1) (the first (N1+1)//2
        and the last N1//2 of each row); it is overwritten."""
        if out is None:
            out = self._alloc(grid, self.grid_shape)
        op = _OutProxy(out)
        a_g, a_o = C.describe(grid), C.describe(op.buf)
        C.check(C.lib().dnufft_plan_cols_to_uniform(self._ptr, 1 if forward else 0,
                                                    ctypes.byref(a_g), ctypes.byref(a_o),
                                                    C.stream_of(grid, op.buf, stream=stream)))
        return op.finish()

    def cols_to_uniform_range(self, *, forward, cols, col0, out=None, stream=None):
        """Column pass, correction and crop of one block of kept columns:
        ``cols`` (nover[0], ncols), the kept columns col0 .. col0 + ncols - 1
        packed (transformed along axis 1; overwritten).  Returns ``out``
        (nuni[0], ncols): column x holds uniform column (col0 + x + s) mod N1,
        s = N1 // 2 (centred mode order) or 0 (fft_order)."""
        import torch
        if out is None:
            out = torch.empty((self.grid_shape[0], cols.shape[1]), dtype=cols.dtype,
                              device=cols.device)
        a_c, a_o = C.describe(cols), C.describe(out)
        C.check(C.lib().dnufft_plan_cols_to_uniform_range(
            self._ptr, 1 if forward else 0, ctypes.byref(a_c), int(col0), ctypes.byref(a_o),
            C.stream_of(cols, out, stream=stream)))
        return out

    def uniform_to_cols_range(self, *, forward, grid, col0, ncols, out=None, stream=None):
        """Type 2 first half for one block of kept columns: correction, zero
        padding and column FFTs of uniform columns of kept columns col0 ..
        col0 + ncols - 1 into ``out`` (nover[0], ncols)."""
        import torch
        if out is None:
            out = torch.empty((self.info()["nover"][0], int(ncols)), dtype=grid.dtype,
                              device=grid.device)
        a_g, a_o = C.describe(grid), C.describe(out)
        C.check(C.lib().dnufft_plan_uniform_to_cols_range(
            self._ptr, 1 if forward else 0, ctypes.byref(a_g), int(col0), ctypes.byref(a_o),
            C.stream_of(grid, out, stream=stream)))
        return out

    def rows_fft_kept_in(self, *, forward, rows, stream=None):
        """Type 2 row FFTs of a slab of rows whose kept columns are set; whole
        rows out, in place."""
        a_r = C.describe(rows)
        C.check(C.lib().dnufft_plan_rows_fft_kept_in(self._ptr, 1 if forward else 0,
                                                     ctypes.byref(a_r),
                                                     C.stream_of(rows, stream=stream)))
        return rows

    def interp(self, *, grid, out=None, stream=None):
        """Interpolation of the plan's points from an oversampled grid (type 2
        second half)."""
        if out is None:
            out = self._alloc(grid, (self.npoints,))
        a_g, a_o = C.describe(grid), C.describe(out)
        C.check(C.lib().dnufft_plan_interp(self._ptr, ctypes.byref(a_g), ctypes.byref(a_o),
                                           C.stream_of(grid, out, stream=stream)))
        return out

    def info(self):
        """Kernel support, oversampled sizes etc. of this plan."""
        inf = C.PlanInfo()
        C.check(C.lib().dnufft_plan_get_info(self._ptr, ctypes.byref(inf)))
        nd = inf.ndim
        return {"ndim": nd, "supp": inf.supp, "kernel_index": inf.kernel_index,
                "log2tile": inf.log2tile, "nuni": list(inf.nuni[:nd]),
                "nover": list(inf.nover[:nd]), "ofactor": inf.ofactor, "beta": inf.beta,
                "e0": inf.e0, "npoints": inf.npoints, "nchunks": inf.nchunks,
                "tc_records": inf.tc_records}

    def permutation(self):
        """The tile-order permutation of the points (DUCC's coord_idx)."""
        out = np.empty(self.npoints, dtype=np.uint32)
        C.check(C.lib().dnufft_plan_get_permutation(
            self._ptr, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), None))
        return out

"""ctypes binding of the C-ABI in include/ducc_b200.h.

Loads ``_lib/libducc_b200.so`` (built in-tree by ``ducc_b200.build``) and
describes numpy arrays (host memory) and torch CUDA tensors (device memory,
zero-copy) as ``dnufft_array``.  There is no fallback: if the library is
missing or fails to load, every call raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libducc_b200.so")

F32, F64, C64, C128, U8 = 1, 2, 3, 4, 5
SPREAD = {"auto": 0, "plain": 1, "tc": 2}


class Array(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("dtype", ctypes.c_int32), ("ndim", ctypes.c_int32),
                ("shape", ctypes.c_int64 * 4), ("stride", ctypes.c_int64 * 4)]


class Opts(ctypes.Structure):
    _fields_ = [("nthreads", ctypes.c_size_t), ("sigma_min", ctypes.c_double),
                ("sigma_max", ctypes.c_double), ("periodicity", ctypes.c_double * 3),
                ("fft_order", ctypes.c_int32), ("verbosity", ctypes.c_int32),
                ("spreader", ctypes.c_int32), ("simd_lanes", ctypes.c_int32),
                ("force_kernel", ctypes.c_int32), ("log2tile", ctypes.c_int32),
                ("force_nover", ctypes.c_int64 * 3)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int32), ("supp", ctypes.c_int32),
                ("kernel_index", ctypes.c_int32), ("log2tile", ctypes.c_int32),
                ("nuni", ctypes.c_int64 * 3), ("nover", ctypes.c_int64 * 3),
                ("ofactor", ctypes.c_double), ("beta", ctypes.c_double), ("e0", ctypes.c_double),
                ("npoints", ctypes.c_int64), ("coord_f64", ctypes.c_int32),
                ("calc_f64", ctypes.c_int32), ("nchunks", ctypes.c_int64),
                ("tc_records", ctypes.c_int64)]


class WgridOpts(ctypes.Structure):
    _fields_ = [("nthreads", ctypes.c_size_t), ("sigma_min", ctypes.c_double),
                ("sigma_max", ctypes.c_double), ("center_x", ctypes.c_double),
                ("center_y", ctypes.c_double), ("do_wgridding", ctypes.c_int32),
                ("flip_u", ctypes.c_int32), ("flip_v", ctypes.c_int32),
                ("flip_w", ctypes.c_int32), ("divide_by_n", ctypes.c_int32),
                ("allow_nshift", ctypes.c_int32),
                ("double_precision_accumulation", ctypes.c_int32),
                ("verbosity", ctypes.c_int32), ("plane_begin", ctypes.c_int32),
                ("plane_count", ctypes.c_int32)]


class ShtOpts(ctypes.Structure):
    _fields_ = [("nthreads", ctypes.c_size_t), ("sigma_min", ctypes.c_double),
                ("sigma_max", ctypes.c_double), ("verbosity", ctypes.c_int32)]


class WgridInfo(ctypes.Structure):
    _fields_ = [("kernel_index", ctypes.c_int32), ("supp", ctypes.c_int32),
                ("nu", ctypes.c_int64), ("nv", ctypes.c_int64), ("nplanes", ctypes.c_int64),
                ("dw", ctypes.c_double), ("wmin", ctypes.c_double), ("nshift", ctypes.c_double),
                ("nvis", ctypes.c_int64)]


_lib = None

EXPORTS = [
    "dnufft_default_opts", "dnufft_best_epsilon", "dnufft_nu2u", "dnufft_u2nu",
    "dnufft_plan_create", "dnufft_plan_nu2u", "dnufft_plan_u2nu", "dnufft_plan_destroy",
    "dnufft_plan_get_info", "dnufft_plan_get_permutation", "dnufft_last_error",
    "dnufft_kernel_launches", "dnufft_profile_enable", "dnufft_profile_json",
    "dnufft_nu2u_noalloc", "dnufft_noalloc_scratch_bytes", "dnufft_u2nu_dcoord",
    "dnufft_plan_u2nu_dcoord", "dnufft_batch_create", "dnufft_batch_nu2u", "dnufft_batch_u2nu",
    "dnufft_batch_destroy", "dnufft_kernel_candidates", "dnufft_selftest_wait_timeout",
    "dnufft_plan_spread", "dnufft_plan_grid_to_uniform", "dnufft_find_parameters",
    "dnufft_plan_rows_fft", "dnufft_plan_cols_to_uniform", "dnufft_plan_cols_to_uniform_range",
    "dnufft_plan_uniform_to_cols_range", "dnufft_plan_rows_fft_kept_in", "dnufft_plan_interp",
    "dnufft_wgrid_default_opts", "dnufft_vis2dirty", "dnufft_dirty2vis", "dnufft_wgrid_params",
    "dnufft_sht_default_opts", "dnufft_synthesis_general", "dnufft_adjoint_synthesis_general",
]


def lib():
    """The loaded CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("ducc_b200 CUDA library not built (%s); run "
                           "`python -m ducc_b200.build`" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    L.dnufft_default_opts.argtypes = [P(Opts), ctypes.c_int]
    L.dnufft_default_opts.restype = None
    L.dnufft_best_epsilon.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, P(ctypes.c_double)]
    for f in (L.dnufft_nu2u, L.dnufft_u2nu, L.dnufft_nu2u_noalloc):
        f.argtypes = [P(Array), P(Array), ctypes.c_int, ctypes.c_double, P(Array), P(Opts), vp]
    L.dnufft_noalloc_scratch_bytes.restype = ctypes.c_size_t
    L.dnufft_plan_create.argtypes = [ctypes.c_int, P(Array), P(ctypes.c_int64), ctypes.c_int,
                                     ctypes.c_double, P(Opts), vp, P(vp)]
    for f in (L.dnufft_plan_nu2u, L.dnufft_plan_u2nu):
        f.argtypes = [vp, ctypes.c_int, ctypes.c_int, P(Array), P(Array), vp]
    L.dnufft_u2nu_dcoord.argtypes = [P(Array), P(Array), ctypes.c_int, ctypes.c_double, P(Array),
                                     P(Array), P(Opts), vp]
    L.dnufft_plan_u2nu_dcoord.argtypes = [vp, ctypes.c_int, P(Array), P(Array), P(Array), vp]
    L.dnufft_plan_destroy.argtypes = [vp]
    L.dnufft_plan_spread.argtypes = [vp, P(Array), P(Array), vp]
    L.dnufft_plan_grid_to_uniform.argtypes = [vp, ctypes.c_int, P(Array), P(Array), vp]
    L.dnufft_plan_rows_fft.argtypes = [vp, ctypes.c_int, P(Array), vp]
    L.dnufft_plan_cols_to_uniform.argtypes = [vp, ctypes.c_int, P(Array), P(Array), vp]
    L.dnufft_plan_cols_to_uniform_range.argtypes = [vp, ctypes.c_int, P(Array), ctypes.c_int64,
                                                     P(Array), vp]
    L.dnufft_plan_uniform_to_cols_range.argtypes = [vp, ctypes.c_int, P(Array), ctypes.c_int64,
                                                     P(Array), vp]
    L.dnufft_plan_rows_fft_kept_in.argtypes = [vp, ctypes.c_int, P(Array), vp]
    L.dnufft_plan_interp.argtypes = [vp, P(Array), P(Array), vp]
    L.dnufft_find_parameters.argtypes = [ctypes.c_int, ctypes.c_int, P(ctypes.c_int64),
                                         ctypes.c_uint64, ctypes.c_double, ctypes.c_int,
                                         ctypes.c_int, P(Opts), P(ctypes.c_int32),
                                         P(ctypes.c_int64)]
    L.dnufft_batch_create.argtypes = [ctypes.c_int, P(vp), P(ctypes.c_int32), vp, P(vp)]
    for f in (L.dnufft_batch_nu2u, L.dnufft_batch_u2nu):
        f.argtypes = [vp, ctypes.c_int, P(Array), P(Array), vp]
    L.dnufft_batch_destroy.argtypes = [vp]
    L.dnufft_kernel_candidates.argtypes = [ctypes.c_int, P(ctypes.c_int64), ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int, P(ctypes.c_int32), P(ctypes.c_int32),
                                           P(ctypes.c_double), P(ctypes.c_int64),
                                           P(ctypes.c_int)]
    L.dnufft_plan_get_info.argtypes = [vp, P(PlanInfo)]
    L.dnufft_plan_get_permutation.argtypes = [vp, P(ctypes.c_uint32), vp]
    L.dnufft_last_error.restype = ctypes.c_char_p
    L.dnufft_kernel_launches.restype = ctypes.c_uint64
    L.dnufft_profile_enable.argtypes = [ctypes.c_int]
    L.dnufft_profile_enable.restype = None
    L.dnufft_profile_json.restype = ctypes.c_char_p
    L.dnufft_selftest_wait_timeout.argtypes = [ctypes.c_int64, vp]
    L.dnufft_wgrid_default_opts.argtypes = [P(WgridOpts)]
    L.dnufft_wgrid_default_opts.restype = None
    for f in (L.dnufft_vis2dirty, L.dnufft_dirty2vis):
        f.argtypes = [P(Array), P(Array), P(Array), P(Array), P(Array), ctypes.c_double,
                      ctypes.c_double, ctypes.c_double, P(WgridOpts), P(Array), vp]
    L.dnufft_wgrid_params.argtypes = [P(Array), P(Array), P(Array), P(Array), P(Array),
                                      ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      P(WgridOpts), P(WgridInfo), vp]
    L.dnufft_sht_default_opts.argtypes = [P(ShtOpts)]
    L.dnufft_sht_default_opts.restype = None
    for f in (L.dnufft_synthesis_general, L.dnufft_adjoint_synthesis_general):
        f.argtypes = [P(Array), ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t,
                      P(ctypes.c_int64), ctypes.c_size_t, ctypes.c_int64, P(Array),
                      ctypes.c_double, P(ShtOpts), P(Array), vp]
    _lib = L
    return L


def check(status):
    if status != 0:
        msg = lib().dnufft_last_error().decode()
        raise RuntimeError(msg or ("ducc_b200 error %d" % status))


# ------------------------------------------------------------------ arrays
_NP_CODES = {np.dtype(np.float32): F32, np.dtype(np.float64): F64,
             np.dtype(np.complex64): C64, np.dtype(np.complex128): C128}
_CODE_NP = {v: k for k, v in _NP_CODES.items()}


def is_torch(x):
    return type(x).__module__.split(".")[0] == "torch"


def torch_code(t):
    import torch
    return {torch.float32: F32, torch.float64: F64, torch.complex64: C64,
            torch.complex128: C128, torch.uint8: U8}.get(t.dtype)


def dtype_code(x):
    if is_torch(x):
        return torch_code(x)
    return _NP_CODES.get(np.asarray(x).dtype)


def describe(x):
    """dnufft_array for a numpy array (host, must be C-contiguous) or a torch
    CUDA tensor (device, any strides)."""
    a = Array()
    if is_torch(x):
        if not x.is_cuda:
            raise ValueError("torch tensors must live on a CUDA device")
        code = torch_code(x)
        if code is None:
            raise RuntimeError("not yet supported")
        a.data = x.data_ptr() if x.numel() else None
        a.dtype = code
        a.ndim = x.dim()
        for d in range(x.dim()):
            a.shape[d] = x.shape[d]
            a.stride[d] = x.stride(d)
        return a
    if not isinstance(x, np.ndarray):
        raise TypeError("expected a numpy array or a torch CUDA tensor")
    code = _NP_CODES.get(x.dtype)
    if code is None:
        raise RuntimeError("not yet supported")
    if not x.flags.c_contiguous:
        raise ValueError("host arrays passed to the C-ABI must be C-contiguous")
    a.data = x.ctypes.data if x.size else None
    a.dtype = code
    a.ndim = x.ndim
    for d in range(x.ndim):
        a.shape[d] = x.shape[d]
        a.stride[d] = x.strides[d] // x.itemsize
    return a


def stream_of(*xs, stream=None):
    if stream is not None:
        return ctypes.c_void_p(int(stream))
    for x in xs:
        if x is not None and is_torch(x) and x.is_cuda:
            import torch
            return ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
    return ctypes.c_void_p(0)


def make_opts(for_plan, nthreads=None, sigma_min=None, sigma_max=None, periodicity=None,
              fft_order=False, verbosity=0, spreader="auto", ndim=1, force_kernel=None,
              force_nover=None, log2tile=None):
    o = Opts()
    lib().dnufft_default_opts(ctypes.byref(o), 1 if for_plan else 0)
    if nthreads is not None:
        if int(nthreads) < 0:
            raise ValueError("nthreads must be >= 0")
        o.nthreads = int(nthreads)
    if sigma_min is not None:
        o.sigma_min = float(sigma_min)
    if sigma_max is not None:
        o.sigma_max = float(sigma_max)
    if periodicity is not None:
        if np.ndim(periodicity) == 0:
            per = [float(periodicity)] * ndim
        else:
            per = [float(p) for p in periodicity]
            if len(per) != ndim:
                raise RuntimeError("bad size of periodicity argument")
        for d in range(ndim):
            o.periodicity[d] = per[d]
    o.fft_order = 1 if fft_order else 0
    o.verbosity = int(verbosity)
    if spreader not in SPREAD:
        raise ValueError("spreader must be one of %s" % list(SPREAD))
    o.spreader = SPREAD[spreader]
    if force_kernel is not None:
        if force_nover is None or len(force_nover) != ndim:
            raise ValueError("force_kernel needs force_nover with one size per axis")
        o.force_kernel = int(force_kernel)
        for d in range(ndim):
            o.force_nover[d] = int(force_nover[d])
    if log2tile is not None:
        o.log2tile = int(log2tile)
    return o

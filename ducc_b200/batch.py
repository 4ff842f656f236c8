"""Batched transforms: many 2D plans of different sizes executed together.

``Batch(plans, ntrans=None)`` groups 2D plans of one precision (each with its
own grid size, points, epsilon and number of transforms over its
coordinates).  ``nu2u`` / ``u2nu`` run every instance at once: one
multi-instance launch per stage (grid zeroing, spreading or interpolation, the
two FFT line passes with the correction), recorded into a CUDA graph on the
first call of each direction and sign and replayed afterwards with the new
arrays.  DUCC has no batched interface; this module is an addition of this
library (the C-ABI ``dnufft_batch_*``).

Arrays are torch CUDA tensors: ``points[i]`` of shape ``(ntrans[i], M_i)`` (or
``(M_i,)`` when ``ntrans[i] == 1``) and uniform grids of shape
``(ntrans[i], N0, N1)`` (or ``(N0, N1)``), any strides.
"""
import ctypes

from . import _capi as C

__all__ = ["Batch"]


class Batch:
    def __init__(self, plans, ntrans=None, stream=None):
        self.plans = list(plans)   # the plans must outlive the batch
        n = len(self.plans)
        if n == 0:
            raise ValueError("empty batch")
        self.ntrans = [1] * n if ntrans is None else [int(t) for t in ntrans]
        if len(self.ntrans) != n:
            raise ValueError("one ntrans per plan")
        ptrs = (ctypes.c_void_p * n)(*[p._ptr.value for p in self.plans])
        nt = (ctypes.c_int32 * n)(*self.ntrans)
        h = ctypes.c_void_p()
        C.check(C.lib().dnufft_batch_create(n, ptrs, nt, C.stream_of(stream=stream), ctypes.byref(h)))
        self._ptr = h

    def __del__(self):
        if getattr(self, "_ptr", None):
            try:
                C.lib().dnufft_batch_destroy(self._ptr)
            except Exception:
                pass
            self._ptr = None

    def _arrays(self, xs):
        n = len(self.plans)
        if len(xs) != n:
            raise ValueError("one array per plan")
        descs = (C.Array * n)(*[C.describe(x) for x in xs])
        return descs

    def nu2u(self, *, points, out, forward, stream=None):
        """Type 1 for every instance: ``out[i] <- nu2u(points[i])``."""
        a_p, a_o = self._arrays(points), self._arrays(out)
        C.check(C.lib().dnufft_batch_nu2u(self._ptr, 1 if forward else 0, a_p, a_o,
                                          C.stream_of(points[0], out[0], stream=stream)))
        return out

    def u2nu(self, *, grids, out, forward, stream=None):
        """Type 2 for every instance: ``out[i] <- u2nu(grids[i])``."""
        a_g, a_o = self._arrays(grids), self._arrays(out)
        C.check(C.lib().dnufft_batch_u2nu(self._ptr, 1 if forward else 0, a_g, a_o,
                                          C.stream_of(grids[0], out[0], stream=stream)))
        return out

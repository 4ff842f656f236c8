"""Differentiable NUFFTs for PyTorch (``torch.autograd.Function``).

``u2nu(grid, coord, ...)`` (type 2) and ``nu2u(points, coord, shape, ...)``
(type 1) run the B200 transforms and differentiate with respect to both the
data and the coordinates:

* data: the adjoint transform (type 1 <-> type 2 with the opposite sign), the
  vector-Jacobian product of a complex-linear map, ``grad = A^H g``;
* coordinates: interpolation of the transformed grid with the derivative of
  the kernel (``dnufft_u2nu_dcoord``), one extra type-2 pass.  With cotangent
  ``g`` of the result, for type 2
      ``grad[j, d] = Re(conj(g_j) * d/dx_{j,d} u2nu(grid)(x_j))``
  and for type 1 (``out_k = sum_j c_j exp(s i k.x_j)``)
      ``grad[j, d] = Re(conj(c_j) * d/dx_{j,d} u2nu(g, sign -s)(x_j))``.

Complex gradients follow PyTorch's convention (the conjugate Wirtinger
derivative, so a complex-linear map's vector-Jacobian product is ``A^H g``).
Each forward call builds a plan for its coordinates (they may change between
steps); the backward pass reuses it.  Coordinates and data must have matching
precision: float32 with complex64, float64 with complex128.  DUCC has no
differentiable interface; this module is an addition of this library.
"""
import math

import torch

from . import nufft

__all__ = ["u2nu", "nu2u"]

_CPLX = {torch.float32: torch.complex64, torch.float64: torch.complex128}


def _check(data, coord, ndim):
    if not (data.is_cuda and coord.is_cuda):
        raise ValueError("ducc_b200.autograd works on CUDA tensors")
    if coord.dim() != 2 or coord.shape[1] != ndim:
        raise ValueError("coord must be (npoints, ndim)")
    if _CPLX.get(coord.dtype) != data.dtype:
        raise TypeError("coordinates and data must have matching precision "
                        "(float32 with complex64, float64 with complex128)")


class _Type2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, grid, coord, forward, epsilon, periodicity, fft_order, plan_kw):
        p = nufft.plan(nu2u=False, coord=coord.detach(), grid_shape=tuple(grid.shape),
                       epsilon=epsilon, periodicity=periodicity, fft_order=fft_order, **plan_kw)
        g = grid.detach().contiguous()
        out = p.u2nu(grid=g, forward=forward)
        ctx.plan, ctx.fwd = p, forward
        ctx.save_for_backward(g)
        return out

    @staticmethod
    def backward(ctx, gout):
        (grid,) = ctx.saved_tensors
        p, fwd = ctx.plan, ctx.fwd
        gout = gout.contiguous()
        g_grid = g_coord = None
        if ctx.needs_input_grad[0]:
            g_grid = p.nu2u(points=gout, forward=not fwd)
        if ctx.needs_input_grad[1]:
            g_coord = p.u2nu_dcoord(forward=fwd, grid=grid, weights=gout)
        return g_grid, g_coord, None, None, None, None, None


class _Type1(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, coord, shape, forward, epsilon, periodicity, fft_order, plan_kw):
        p = nufft.plan(nu2u=True, coord=coord.detach(), grid_shape=tuple(shape),
                       epsilon=epsilon, periodicity=periodicity, fft_order=fft_order, **plan_kw)
        c = points.detach().contiguous()
        out = p.nu2u(points=c, forward=forward)
        ctx.plan, ctx.fwd = p, forward
        ctx.save_for_backward(c)
        return out

    @staticmethod
    def backward(ctx, gout):
        (points,) = ctx.saved_tensors
        p, fwd = ctx.plan, ctx.fwd
        gout = gout.contiguous()
        g_pts = g_coord = None
        if ctx.needs_input_grad[0]:
            g_pts = p.u2nu(grid=gout, forward=not fwd)
        if ctx.needs_input_grad[1]:
            g_coord = p.u2nu_dcoord(forward=not fwd, grid=gout, weights=points)
        return g_pts, g_coord, None, None, None, None, None, None


def u2nu(grid, coord, *, forward=True, epsilon=1e-6, periodicity=2 * math.pi, fft_order=False,
         **plan_kw):
    """Differentiable type-2 NUFFT: values of ``grid`` (uniform modes) at the
    points ``coord`` (npoints, ndim).  Same conventions as
    ``ducc_b200.nufft.u2nu``; extra keywords go to ``nufft.plan``."""
    _check(grid, coord, grid.dim())
    return _Type2.apply(grid, coord, bool(forward), float(epsilon), periodicity, bool(fft_order),
                        plan_kw)


def nu2u(points, coord, shape, *, forward=True, epsilon=1e-6, periodicity=2 * math.pi,
         fft_order=False, **plan_kw):
    """Differentiable type-1 NUFFT onto a uniform grid of ``shape``.  Same
    conventions as ``ducc_b200.nufft.nu2u``; extra keywords go to
    ``nufft.plan``."""
    _check(points, coord, len(shape))
    return _Type1.apply(points, coord, tuple(int(s) for s in shape), bool(forward),
                        float(epsilon), periodicity, bool(fft_order), plan_kw)

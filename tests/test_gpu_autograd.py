"""Gradients of the differentiable NUFFT (ducc_b200.autograd).

DUCC has no differentiable interface, so these gradients are pinned by the
mathematics: the FP64 direct NUDFT and its analytic derivative (oracle
direct_nu2u / direct_u2nu / direct_u2nu_dcoord), central finite differences of
the loss, and - at the radial-trajectory size (1024^2 image, 2048 spokes x
2048 samples) - DUCC's own FP64 transforms (oracle/_ref) for the image
gradient and the direct FP64 derivative on a sample of the points.

Loss: L = sum_j |T(x)_j - y_j|^2, y the transform of a perturbed input.
"""
import math

import numpy as np
import pytest

from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    return t.detach().cpu().numpy()


CASES = [
    # shape, npoints, coord dtype, eps, forward, periodicity, fft_order
    ((24, 20), 40, np.float64, 1e-12, True, 2 * math.pi, False),
    ((17,), 30, np.float64, 1e-12, False, 1.0, True),
    ((8, 9, 10), 25, np.float64, 1e-11, True, [1.0, 2.0, 3.0], False),
    ((32, 30), 300, np.float32, 1e-6, True, 2 * math.pi, False),
    ((40,), 100, np.float32, 1e-5, False, 2 * math.pi, True),
]


def problem(shape, M, per, seed):
    rng = np.random.default_rng(seed)
    ndim = len(shape)
    pers = np.ones(ndim) * np.array(per, dtype=np.float64)
    x = (rng.random((M, ndim)) - 0.5) * pers * 1.3   # some points outside one period
    img = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    pert = 0.3 * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    cpert = 0.3 * (rng.standard_normal(M) + 1j * rng.standard_normal(M))
    return x, img, pert, c, cpert


def tolerances(cdt, eps):
    # data gradient: an adjoint transform of a residual known to ~eps; the
    # coordinate gradient differentiates the kernel approximation as well
    # (measured on B200: double <= 4e-12 / 9e-12 at eps 1e-11..1e-12, single
    # 5e-7..1.3e-5 / 7e-7..4e-5 at eps 1e-6..1e-5)
    if cdt == np.float64:
        return 50 * eps, 100 * eps
    return 5 * eps, 10 * eps


@pytest.mark.parametrize("shape,M,cdt,eps,forward,per,fft_order", CASES)
def test_type2_gradients_vs_fp64(shape, M, cdt, eps, forward, per, fft_order):
    from ducc_b200 import autograd as AG
    x, img, pert, _, _ = problem(shape, M, per, 1)
    ct = np.complex64 if cdt == np.float32 else np.complex128
    xs = x.astype(cdt)
    imgs = img.astype(ct)
    y = O.direct_u2nu(imgs + pert, xs, forward, per, fft_order)
    tx = dev(xs).requires_grad_()
    ti = dev(imgs).requires_grad_()
    out = AG.u2nu(ti, tx, forward=forward, epsilon=eps, periodicity=per, fft_order=fft_order)
    loss = (out - dev(y.astype(ct))).abs().pow(2).sum()
    loss.backward()
    g = 2 * (O.direct_u2nu(imgs, xs, forward, per, fft_order) - y)
    gimg = O.direct_nu2u(xs, g, shape, not forward, per, fft_order)
    gx = O.direct_u2nu_dcoord(imgs, xs, forward, g, per, fft_order)
    ti_tol, tx_tol = tolerances(cdt, eps)
    e_img = O.l2error(host(ti.grad), gimg)
    e_x = O.l2error(host(tx.grad), gx)
    print("type2 grad errors: image %.3e coord %.3e" % (e_img, e_x))
    assert e_img < ti_tol
    assert e_x < tx_tol


@pytest.mark.parametrize("shape,M,cdt,eps,forward,per,fft_order", CASES)
def test_type1_gradients_vs_fp64(shape, M, cdt, eps, forward, per, fft_order):
    from ducc_b200 import autograd as AG
    x, _, _, c, cpert = problem(shape, M, per, 2)
    ct = np.complex64 if cdt == np.float32 else np.complex128
    xs = x.astype(cdt)
    cs = c.astype(ct)
    Y = O.direct_nu2u(xs, cs + cpert, shape, forward, per, fft_order)
    tx = dev(xs).requires_grad_()
    tc = dev(cs).requires_grad_()
    out = AG.nu2u(tc, tx, shape, forward=forward, epsilon=eps, periodicity=per,
                  fft_order=fft_order)
    loss = (out - dev(Y.astype(ct))).abs().pow(2).sum()
    loss.backward()
    G = 2 * (O.direct_nu2u(xs, cs, shape, forward, per, fft_order) - Y)
    gc = O.direct_u2nu(G, xs, not forward, per, fft_order)
    gx = O.direct_u2nu_dcoord(G, xs, not forward, cs, per, fft_order)
    tc_tol, tx_tol = tolerances(cdt, eps)
    e_c = O.l2error(host(tc.grad), gc)
    e_x = O.l2error(host(tx.grad), gx)
    print("type1 grad errors: values %.3e coord %.3e" % (e_c, e_x))
    assert e_c < tc_tol
    assert e_x < tx_tol


@pytest.mark.parametrize("kind", ["type2", "type1"])
def test_coordinate_gradient_finite_differences(kind):
    """Central differences of the FP64 loss against the autograd gradient."""
    import torch
    from ducc_b200 import autograd as AG
    shape, M, per, eps = (20, 22), 30, 2 * math.pi, 1e-13
    x, img, pert, c, cpert = problem(shape, M, per, 3)
    if kind == "type2":
        y = dev(O.direct_u2nu(img + pert, x, True, per))
        ti = dev(img)

        def loss_of(tx):
            return (AG.u2nu(ti, tx, forward=True, epsilon=eps) - y).abs().pow(2).sum()
    else:
        Y = dev(O.direct_nu2u(x, c + cpert, shape, True, per))
        tc = dev(c)

        def loss_of(tx):
            return (AG.nu2u(tc, tx, shape, forward=True, epsilon=eps) - Y).abs().pow(2).sum()
    tx = dev(x).requires_grad_()
    loss_of(tx).backward()
    grad = host(tx.grad)
    h = 1e-5
    scale = np.abs(grad).max()
    for j, d in [(0, 0), (7, 1), (29, 0), (13, 1)]:
        xp, xm = x.copy(), x.copy()
        xp[j, d] += h
        xm[j, d] -= h
        with torch.no_grad():
            fd = (loss_of(dev(xp)).item() - loss_of(dev(xm)).item()) / (2 * h)
        assert abs(fd - grad[j, d]) < 1e-6 * scale, (j, d, fd, grad[j, d])


def radial(nspokes, nsamp):
    ang = np.pi * np.arange(nspokes) / nspokes
    rad = np.linspace(-np.pi, np.pi, nsamp, endpoint=False)
    kx = np.outer(np.cos(ang), rad).ravel()
    ky = np.outer(np.sin(ang), rad).ravel()
    return np.stack([kx, ky], axis=1).astype(np.float32)


def test_radial_trajectory_full_size():
    """1024^2 complex64 image, 2048 spokes x 2048 samples, float32 coordinates,
    eps 1e-6: image gradient against DUCC's FP64 transforms at 1e-13 (when the
    DUCC module is built), coordinate gradient against the FP64 direct
    derivative on 48 sampled points."""
    from ducc_b200 import autograd as AG
    from oracle import ref
    rng = np.random.default_rng(5)
    N, eps = 1024, 1e-6
    x = radial(2048, 2048)
    img = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)
    pert = (0.3 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)))).astype(
        np.complex64)
    R = ref.load()
    if R is not None:
        y = R.nufft.u2nu(grid=(img + pert).astype(np.complex128), coord=x.astype(np.float64),
                         forward=True, epsilon=1e-13, nthreads=0)
    else:
        y = None
    tx = dev(x).requires_grad_()
    ti = dev(img).requires_grad_()
    ty = None if y is None else dev(y.astype(np.complex64))
    out = AG.u2nu(ti, tx, forward=True, epsilon=eps)
    if ty is None:
        import torch
        with torch.no_grad():
            ty = AG.u2nu(dev(img + pert), dev(x), forward=True, epsilon=1e-6)
    loss = (out - ty).abs().pow(2).sum()
    loss.backward()
    gx = host(tx.grad)
    yh = host(ty).astype(np.complex128)
    # coordinate gradient on sampled points, FP64 direct
    idx = rng.choice(x.shape[0], 48, replace=False)
    xs = x[idx].astype(np.float64)
    g = 2 * (O.direct_u2nu(img, xs, True) - yh[idx])
    gx_ref = O.direct_u2nu_dcoord(img, xs, True, g)
    e_x = O.l2error(gx[idx], gx_ref)
    print("radial: coordinate gradient error on 48 points %.3e" % e_x)
    assert e_x < 10 * eps
    if R is not None:
        r = R.nufft.u2nu(grid=img.astype(np.complex128), coord=x.astype(np.float64), forward=True,
                         epsilon=1e-13, nthreads=0) - y
        gimg = np.zeros((N, N), np.complex128)
        R.nufft.nu2u(points=2 * r, coord=x.astype(np.float64), forward=False, epsilon=1e-13,
                     nthreads=0, out=gimg)
        e_img = O.l2error(host(ti.grad), gimg)
        print("radial: image gradient error %.3e" % e_img)
        assert e_img < 5 * eps

"""w-gridder on the GPU (ducc_b200.wgridder) against the direct sums and
against DUCC's own w-gridder.

The first six tests restate DUCC's python/test/test_wgridder.py (parameter
grids, inputs from the same seeded generators, the faceting helpers and the
tolerances; nthreads, which only feeds DUCC's cost model, at 1) against this
package:
  test_adjointness_ms2dirty            test_wgridder.py:190-260
  test_ms2dirty_against_wdft2          :263-318
  test_adjointness_wsclean             :321-356
  test_vis2dirty_wsclean               :359-394
  test_ms2dirty_against_wdft3          :397-437
  test_adjointness_ms2dirty_complex    :440-496
The direct sums are oracle/wgridder_oracle.py.  The last tests compare with
DUCC's compiled w-gridder (oracle/_ref, when it was built) on larger problems
over the options DUCC's tests leave at their defaults (axis flips, image
centre, divide_by_n, allow_nshift, double-precision accumulation).
"""
import numpy as np
import pytest

from oracle import wgridder_oracle as O

pytestmark = pytest.mark.gpu
pmp = pytest.mark.parametrize
SPEEDOFLIGHT = 299792458.


@pytest.fixture(scope="module")
def ng():
    from ducc_b200 import wgridder
    return wgridder


def vis2dirty_with_faceting(ng, *, nfacets_x=1, nfacets_y=1, npix_x, npix_y, center_x=0.,
                            center_y=0., dirty=None, **kwargs):
    """The image as nfacets_x x nfacets_y separate calls with shifted centres
    (even facet sides; partial facets at the far edges through a scratch)."""
    if dirty is None:
        dtype = np.float32 if kwargs["vis"].dtype == np.complex64 else np.float64
        dirty = np.zeros((npix_x, npix_y), dtype)
    istep = (npix_x + nfacets_x - 1) // nfacets_x
    istep += istep % 2
    jstep = (npix_y + nfacets_y - 1) // nfacets_y
    jstep += jstep % 2
    for i in range(nfacets_x):
        cx = center_x + kwargs["pixsize_x"] * 0.5 * ((2 * i + 1) * istep - npix_x)
        imax = min((i + 1) * istep, npix_x)
        for j in range(nfacets_y):
            cy = center_y + kwargs["pixsize_y"] * 0.5 * ((2 * j + 1) * jstep - npix_y)
            jmax = min((j + 1) * jstep, npix_y)
            t = ng.vis2dirty(**kwargs, center_x=cx, center_y=cy, npix_x=istep, npix_y=jstep)
            dirty[i * istep:imax, j * jstep:jmax] = t[:imax - i * istep, :jmax - j * jstep]
    return dirty


def dirty2vis_with_faceting(ng, *, nfacets_x=1, nfacets_y=1, center_x=0., center_y=0., dirty,
                            **kwargs):
    npix_x, npix_y = dirty.shape
    istep = (npix_x + nfacets_x - 1) // nfacets_x
    istep += istep % 2
    jstep = (npix_y + nfacets_y - 1) // nfacets_y
    jstep += jstep % 2
    vis = None
    for i in range(nfacets_x):
        cx = center_x + kwargs["pixsize_x"] * 0.5 * ((2 * i + 1) * istep - npix_x)
        imax = min((i + 1) * istep, npix_x)
        for j in range(nfacets_y):
            cy = center_y + kwargs["pixsize_y"] * 0.5 * ((2 * j + 1) * jstep - npix_y)
            jmax = min((j + 1) * jstep, npix_y)
            t = np.zeros((istep, jstep), dtype=dirty.dtype)
            t[:imax - i * istep, :jmax - j * jstep] = dirty[i * istep:imax, j * jstep:jmax]
            tv = ng.dirty2vis(**kwargs, dirty=t, center_x=cx, center_y=cy)
            vis = tv if vis is None else vis + tv
    return vis


def _adjoint_check(ms, dirty, d2, m2, singleprec):
    ref = max(O.vdot(ms, ms).real, O.vdot(m2, m2).real, O.vdot(dirty, dirty).real,
              O.vdot(d2, d2).real)
    tol = 3e-5 * ref if singleprec else 2e-13 * ref
    np.testing.assert_allclose(O.vdot(ms, m2).real, O.vdot(d2, dirty), rtol=3 * tol)


def _adjoint_inputs(nxdirty, nydirty, nrow, nchan, singleprec, use_wgt, use_mask, fov=None,
                    complex_dirty=False):
    rng = np.random.default_rng(43)
    if fov is None:
        pixsizex = np.pi / 180 / 60 / nxdirty * 0.2398
        pixsizey = np.pi / 180 / 60 / nxdirty
    else:
        pixsizex = fov * np.pi / 180 / nxdirty
        pixsizey = fov * np.pi / 180 / nydirty * 1.1
    f0 = 1e9
    freq = f0 + np.arange(nchan) * (f0 / nchan)
    uvw = (rng.random((nrow, 3)) - 0.5) / (pixsizey * f0 / SPEEDOFLIGHT)
    ms = rng.random((nrow, nchan)) - 0.5 + 1j * (rng.random((nrow, nchan)) - 0.5)
    wgt = rng.uniform(0.9, 1.1, (nrow, nchan)) if use_wgt else None
    mask = (rng.uniform(0, 1, (nrow, nchan)) > 0.5).astype(np.uint8) if use_mask else None
    dirty = rng.random((nxdirty, nydirty)) - 0.5
    if complex_dirty:
        dirty = dirty + 1j * (rng.random((nxdirty, nydirty)) - 0.5)
    if singleprec:
        ms = ms.astype("c8")
        dirty = dirty.astype("c8" if complex_dirty else "f4")
        if wgt is not None:
            wgt = wgt.astype("f4")
    return pixsizex, pixsizey, freq, uvw, ms, wgt, mask, dirty


@pmp('nx', [(2, 2), (32, 3), (128, 2)])
@pmp('ny', [(2, 2), (128, 2), (250, 5)])
@pmp("nrow", (1, 2, 27))
@pmp("nchan", (1, 5))
@pmp("epsilon", (1e-1, 3e-5, 2e-13))
@pmp("singleprec", (True, False))
@pmp("wstacking", (True, False))
@pmp("use_wgt", (True, False))
@pmp("use_mask", (False, True))
def test_adjointness_ms2dirty(ng, nx, ny, nrow, nchan, epsilon, singleprec, wstacking, use_wgt,
                              use_mask):
    (nxdirty, nxfacets), (nydirty, nyfacets) = nx, ny
    if singleprec and epsilon < 1e-6:
        pytest.skip()
    psx, psy, freq, uvw, ms, wgt, mask, dirty = _adjoint_inputs(
        nxdirty, nydirty, nrow, nchan, singleprec, use_wgt, use_mask)
    dirty2 = ng.ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, psx, psy, 0, 0, epsilon,
                         wstacking, 1, 0, mask).astype("f8")
    ms2 = ng.dirty2ms(uvw, freq, dirty, wgt, psx, psy, 0, 0, epsilon, wstacking, 1, 0,
                      mask).astype("c16")
    _adjoint_check(ms, dirty, dirty2, ms2, singleprec)
    kw = dict(uvw=uvw, freq=freq, wgt=wgt, pixsize_x=psx, pixsize_y=psy, epsilon=epsilon,
              do_wgridding=wstacking, nthreads=1, mask=mask)
    dirty2 = vis2dirty_with_faceting(ng, nfacets_x=nxfacets, nfacets_y=nyfacets, vis=ms,
                                     npix_x=nxdirty, npix_y=nydirty, **kw).astype("f8")
    ms2 = dirty2vis_with_faceting(ng, nfacets_x=nxfacets, nfacets_y=nyfacets, dirty=dirty,
                                  **kw).astype("c16")
    _adjoint_check(ms, dirty, dirty2, ms2, singleprec)


@pmp('nx', [(2, 2), (6, 2), (18, 2), (66, 4)])
@pmp('ny', [(2, 2), (64, 2)])
@pmp("nrow", (1, 2, 27))
@pmp("nchan", (1, 5))
@pmp("epsilon", (1e-2, 1e-4, 1e-7))
@pmp("wstacking", (False, True))
@pmp("fov", (0.001, 0.1, 20.))
def test_ms2dirty_against_wdft2(ng, nx, ny, nrow, nchan, epsilon, wstacking, fov):
    (nxdirty, nxfacets), (nydirty, nyfacets) = nx, ny
    rng = np.random.default_rng(42)
    psx = fov * np.pi / 180 / nxdirty
    psy = fov * np.pi / 180 / nydirty * 1.1
    f0 = 1e9
    freq = f0 + np.arange(nchan) * (f0 / nchan)
    uvw = (rng.random((nrow, 3)) - 0.5) / (psx * f0 / SPEEDOFLIGHT)
    ms = rng.random((nrow, nchan)) - 0.5 + 1j * (rng.random((nrow, nchan)) - 0.5)
    wgt = rng.uniform(0.9, 1.1, (nrow, nchan))
    mask = (rng.uniform(0, 1, (nrow, nchan)) > 0.5).astype(np.uint8)
    dirty = ng.ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, psx, psy, 0, 0, epsilon,
                        wstacking, 1, 0, mask).astype("f8")
    ref = O.explicit_gridder(uvw, freq, ms, wgt, nxdirty, nydirty, psx, psy, wstacking, mask)
    assert O.l2error(dirty, ref) <= epsilon
    dirty2 = vis2dirty_with_faceting(
        ng, nfacets_x=nxfacets, nfacets_y=nyfacets, uvw=uvw, freq=freq, vis=ms, wgt=wgt,
        npix_x=nxdirty, npix_y=nydirty, pixsize_x=psx, pixsize_y=psy, epsilon=epsilon,
        do_wgridding=wstacking, nthreads=1, mask=mask).astype("f8")
    assert O.l2error(dirty2, ref) <= epsilon


@pmp("use_wgt", (True, False))
@pmp("use_mask", (False, True))
@pmp("fov", (10., 120.))
def test_adjointness_wsclean(ng, use_wgt, use_mask, fov):
    nxdirty, nydirty, nrow, nchan, epsilon = 128, 250, 27, 5, 2e-10
    psx, psy, freq, uvw, ms, wgt, mask, dirty = _adjoint_inputs(
        nxdirty, nydirty, nrow, nchan, False, use_wgt, use_mask, fov=fov)
    dirty2 = ng.vis2dirty(uvw=uvw, freq=freq, vis=ms, wgt=wgt, npix_x=nxdirty, npix_y=nydirty,
                          pixsize_x=psx, pixsize_y=psy, epsilon=epsilon, do_wgridding=True,
                          nthreads=2, mask=mask, divide_by_n=False).astype("f8")
    ms2 = ng.dirty2vis(uvw=uvw, freq=freq, dirty=dirty, wgt=wgt, pixsize_x=psx, pixsize_y=psy,
                       epsilon=epsilon, do_wgridding=True, nthreads=2, mask=mask,
                       divide_by_n=False).astype("c16")
    _adjoint_check(ms, dirty, dirty2, ms2, False)


@pmp("fov", (10., 80., 90., 120.))
def test_vis2dirty_wsclean(ng, fov):
    nxdirty = nydirty = 50
    nrow, nchan, epsilon = 27, 5, 1e-7
    rng = np.random.default_rng(42)
    psx = fov * np.pi / 180 / nxdirty
    psy = fov * np.pi / 180 / nydirty * 1.1
    f0 = 1e9
    freq = f0 + np.arange(nchan) * (f0 / nchan)
    uvw = (rng.random((nrow, 3)) - 0.5) / (psx * f0 / SPEEDOFLIGHT)
    ms = rng.random((nrow, nchan)) - 0.5 + 1j * (rng.random((nrow, nchan)) - 0.5)
    wgt = rng.uniform(0.9, 1.1, (nrow, nchan))
    dirty = ng.vis2dirty(uvw=uvw, freq=freq, vis=ms, wgt=wgt, npix_x=nxdirty, npix_y=nydirty,
                         pixsize_x=psx, pixsize_y=psy, epsilon=epsilon, do_wgridding=True,
                         nthreads=1, verbosity=0, mask=None, divide_by_n=False).astype("f8")
    ref = O.explicit_gridder(uvw, freq, ms, wgt, nxdirty, nydirty, psx, psy, True, None,
                             divide_by_n=False)
    dirty[0, 0] = ref[0, 0]
    assert O.l2error(dirty, ref) <= epsilon


@pmp('nxdirty', [2, 16, 64])
@pmp('nydirty', [2, 64])
@pmp("nrow", (1, 100))
@pmp("nchan", (1, 7))
@pmp("epsilon", list(10. ** np.linspace(-2., -12., 20)))
def test_ms2dirty_against_wdft3(ng, nxdirty, nydirty, nrow, nchan, epsilon):
    fov = 10.
    rng = np.random.default_rng(42)
    psx = fov * np.pi / 180 / nxdirty
    psy = fov * np.pi / 180 / nydirty * 1.1
    f0 = 1e9
    freq = f0 + np.arange(nchan) * (f0 / nchan)
    uvw = (rng.random((nrow, 3)) - 0.5) / (psx * f0 / SPEEDOFLIGHT)
    ms = rng.random((nrow, nchan)) - 0.5 + 1j * (rng.random((nrow, nchan)) - 0.5)
    wgt = np.ascontiguousarray(np.broadcast_to(rng.random((nrow, 1)), (nrow, nchan)))
    try:
        dirty = ng.ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, psx, psy, 0, 0, epsilon,
                            True, 1, 0).astype("f8")
    except RuntimeError as e:
        # no kernel reaches this epsilon (DUCC's test skips the same way)
        assert "kernel" in str(e)
        pytest.skip()
    ref = O.explicit_gridder(uvw, freq, ms, wgt, nxdirty, nydirty, psx, psy, True, None)
    assert O.l2error(dirty, ref) <= 2 * epsilon
    x1 = O.explicit_degridder(uvw, freq, ref, wgt, psx, psy, True, None)
    x2 = ng.dirty2ms(uvw, freq, ref, wgt, psx, psy, 0, 0, epsilon, True, 1, 0).astype("c16")
    assert O.l2error(x1, x2) <= epsilon


@pmp('nx', [(2, 2), (30, 3), (128, 2)])
@pmp('ny', [(2, 2), (128, 2), (250, 5)])
@pmp("nrow", (1, 2, 27))
@pmp("nchan", (1, 5))
@pmp("epsilon", (1e-1, 3e-5, 2e-13))
@pmp("singleprec", (True, False))
@pmp("wstacking", (True, False))
@pmp("use_wgt", (True, False))
@pmp("use_mask", (False, True))
def test_adjointness_ms2dirty_complex(ng, nx, ny, nrow, nchan, epsilon, singleprec, wstacking,
                                      use_wgt, use_mask):
    (nxdirty, nxfacets), (nydirty, nyfacets) = nx, ny
    if singleprec and epsilon < 1e-6:
        pytest.skip()
    psx, psy, freq, uvw, ms, wgt, mask, dirty = _adjoint_inputs(
        nxdirty, nydirty, nrow, nchan, singleprec, use_wgt, use_mask, complex_dirty=True)
    # a complex image as two real ones: Re and Im of the adjoint pair
    dirty2 = (ng.ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, psx, psy, 0, 0, epsilon,
                          wstacking, 1, 0, mask).astype("c16")
              + 1j * ng.ms2dirty(uvw, freq, -1j * ms, wgt, nxdirty, nydirty, psx, psy, 0, 0,
                                 epsilon, wstacking, 1, 0, mask).astype("c16"))
    ms2 = (ng.dirty2ms(uvw, freq, np.ascontiguousarray(dirty.real), wgt, psx, psy, 0, 0,
                       epsilon, wstacking, 1, 0, mask).astype("c16")
           + 1j * ng.dirty2ms(uvw, freq, np.ascontiguousarray(dirty.imag), wgt, psx, psy, 0, 0,
                              epsilon, wstacking, 1, 0, mask).astype("c16"))
    ref = max(O.vdot(ms, ms).real, O.vdot(ms2, ms2).real, O.vdot(dirty, dirty).real,
              O.vdot(dirty2, dirty2).real)
    tol = 3e-5 * ref if singleprec else 2e-13 * ref
    np.testing.assert_allclose(O.vdot(ms, ms2), O.vdot(dirty2, dirty), rtol=3 * tol)


# ---------------------------------------------------------------- against DUCC
@pytest.fixture(scope="module")
def ducc():
    from oracle import ref
    m = ref.load()
    if m is None or not hasattr(m, "wgridder"):
        pytest.skip("DUCC's w-gridder (oracle/_ref) not built")
    return m.wgridder


def _ms_problem(seed, nrow, nchan, npix, fov_deg, singleprec, masked):
    rng = np.random.default_rng(seed)
    ps = fov_deg * np.pi / 180 / npix
    f0 = 1e9
    freq = f0 + np.arange(nchan) * (f0 / nchan / 4)
    uvw = (rng.random((nrow, 3)) - 0.5) / (ps * f0 / SPEEDOFLIGHT)
    uvw[:, 2] *= 0.3
    vis = rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))
    wgt = rng.uniform(0.5, 1.5, (nrow, nchan))
    mask = (rng.uniform(0, 1, (nrow, nchan)) > 0.2).astype(np.uint8) if masked else None
    dirty = rng.standard_normal((npix, npix))
    if singleprec:
        vis, wgt, dirty = vis.astype("c8"), wgt.astype("f4"), dirty.astype("f4")
    return ps, freq, uvw, vis, wgt, mask, dirty


OPTION_SETS = [
    dict(),
    dict(flip_u=True),
    dict(flip_v=True, flip_w=True),
    dict(center_x=3e-3, center_y=-2e-3),
    dict(center_x=-4e-3, center_y=1e-3, flip_u=True, flip_v=True),
    dict(divide_by_n=False),
    dict(allow_nshift=False),
    dict(sigma_min=1.5, sigma_max=2.0),
]


@pmp("singleprec,epsilon", [(True, 1e-4), (True, 2e-5), (False, 1e-6), (False, 1e-10)])
@pmp("do_w", (True, False))
@pmp("opt", range(len(OPTION_SETS)))
def test_against_ducc(ng, ducc, singleprec, epsilon, do_w, opt):
    """Both directions on 4000 x 4 visibilities and a 200^2 image at a 10 degree
    field of view (w terms matter), against DUCC with the same arguments."""
    kw = OPTION_SETS[opt]
    ps, freq, uvw, vis, wgt, mask, dirty = _ms_problem(7 + opt, 4000, 4, 200, 10., singleprec,
                                                       opt % 2 == 1)
    args = dict(uvw=uvw, freq=freq, wgt=wgt, mask=mask, pixsize_x=ps, pixsize_y=1.1 * ps,
                epsilon=epsilon, do_wgridding=do_w, nthreads=4, **kw)
    d_ours = ng.vis2dirty(vis=vis, npix_x=200, npix_y=200, **args)
    d_ref = ducc.vis2dirty(vis=vis, npix_x=200, npix_y=200, **args)
    assert d_ours.dtype == d_ref.dtype and d_ours.shape == d_ref.shape
    assert O.l2error(d_ours, d_ref) <= 2 * epsilon
    v_ours = ng.dirty2vis(dirty=dirty, **args)
    v_ref = ducc.dirty2vis(dirty=dirty, **args)
    assert v_ours.dtype == v_ref.dtype and v_ours.shape == v_ref.shape
    assert O.l2error(v_ours, v_ref) <= 2 * epsilon
    if mask is not None:
        assert np.all(v_ours[mask == 0] == 0)


def test_against_ducc_double_accumulation(ng, ducc):
    ps, freq, uvw, vis, wgt, mask, _ = _ms_problem(3, 20000, 2, 256, 5., True, False)
    args = dict(uvw=uvw, freq=freq, vis=vis, wgt=wgt, npix_x=256, npix_y=256, pixsize_x=ps,
                pixsize_y=ps, epsilon=1e-5, do_wgridding=True, nthreads=4,
                double_precision_accumulation=True)
    d_ours = ng.vis2dirty(**args)
    d_ref = ducc.vis2dirty(**args)
    assert d_ours.dtype == np.float32
    assert O.l2error(d_ours, d_ref) <= 2e-5


def test_parameters_and_no_visibilities(ng):
    ps, freq, uvw, vis, wgt, _, dirty = _ms_problem(5, 500, 3, 64, 10., False, False)
    p = ng.wgrid_params(uvw=uvw, freq=freq, vis=vis, wgt=wgt, npix_x=64, npix_y=64,
                        pixsize_x=ps, pixsize_y=ps, epsilon=1e-6, do_wgridding=True)
    assert p["nvis"] == 1500 and p["supp"] >= 4 and p["nplanes"] >= p["supp"]
    assert p["nu"] >= 64 and p["nu"] % 2 == 0 and p["dw"] > 0
    # every visibility masked out: zero image, zero visibilities
    mask = np.zeros((500, 3), np.uint8)
    d = ng.vis2dirty(uvw=uvw, freq=freq, vis=vis, wgt=wgt, mask=mask, npix_x=64, npix_y=64,
                     pixsize_x=ps, pixsize_y=ps, epsilon=1e-6, do_wgridding=True)
    assert np.all(d == 0)
    v = ng.dirty2vis(uvw=uvw, freq=freq, dirty=dirty, wgt=wgt, mask=mask, pixsize_x=ps,
                     pixsize_y=ps, epsilon=1e-6, do_wgridding=True)
    assert np.all(v == 0)


def test_bad_arguments(ng):
    ps, freq, uvw, vis, wgt, _, _ = _ms_problem(5, 50, 3, 64, 10., False, False)
    with pytest.raises(RuntimeError, match="even"):
        ng.vis2dirty(uvw=uvw, freq=freq, vis=vis, npix_x=63, npix_y=64, pixsize_x=ps,
                     pixsize_y=ps, epsilon=1e-6)
    with pytest.raises(RuntimeError, match="ascending"):
        ng.vis2dirty(uvw=uvw, freq=freq[::-1].copy(), vis=vis, npix_x=64, npix_y=64,
                     pixsize_x=ps, pixsize_y=ps, epsilon=1e-6)
    with pytest.raises(RuntimeError, match="kernel"):
        ng.vis2dirty(uvw=uvw, freq=freq, vis=vis.astype("c8"), npix_x=64, npix_y=64,
                     pixsize_x=ps, pixsize_y=ps, epsilon=1e-9)
    with pytest.raises(TypeError):
        ng.vis2dirty(uvw=uvw, freq=freq, vis=vis, wgt=wgt.astype("f4"), npix_x=64, npix_y=64,
                     pixsize_x=ps, pixsize_y=ps, epsilon=1e-6)


def test_torch_tensors_in_place(ng):
    """Device tensors in, results written into the given device tensors, the
    same numbers as the numpy path."""
    import torch
    ps, freq, uvw, vis, wgt, mask, dirty = _ms_problem(21, 3000, 4, 128, 10., True, True)
    args = dict(pixsize_x=ps, pixsize_y=ps, epsilon=1e-5, do_wgridding=True)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    out = torch.zeros((128, 128), dtype=torch.float32, device="cuda")
    r = ng.vis2dirty(uvw=t(uvw), freq=t(freq), vis=t(vis), wgt=t(wgt), mask=t(mask), dirty=out,
                     **args)
    assert r is out
    ref = ng.vis2dirty(uvw=uvw, freq=freq, vis=vis, wgt=wgt, mask=mask, npix_x=128, npix_y=128,
                       **args)
    assert O.l2error(out.cpu().numpy(), ref) < 1e-6
    vout = torch.empty(vis.shape, dtype=torch.complex64, device="cuda")
    r = ng.dirty2vis(uvw=t(uvw), freq=t(freq), dirty=t(dirty), wgt=t(wgt), mask=t(mask),
                     vis=vout, **args)
    assert r is vout
    vref = ng.dirty2vis(uvw=uvw, freq=freq, dirty=dirty, wgt=wgt, mask=mask, **args)
    assert O.l2error(vout.cpu().numpy(), vref) < 1e-6


@pmp("singleprec,epsilon", [(True, 1e-4), (True, 1e-5), (False, 1e-7), (False, 1e-11)])
@pmp("do_w", (True, False))
@pmp("nthreads", (1, 16))
def test_parameters_match_ducc(ng, ducc, capfd, singleprec, epsilon, do_w, nthreads):
    """The kernel support, oversampled grid and number of w planes are DUCC's
    (its cost model, printed with verbosity=1) for the same call."""
    import re
    from oracle import ref
    if not singleprec and ref.simd_lanes_double() != 8:
        pytest.skip("the reference build's float64 SIMD width is not the modelled one")
    ps, freq, uvw, vis, wgt, _, _ = _ms_problem(31, 20000, 8, 512, 8., singleprec, False)
    args = dict(uvw=uvw, freq=freq, wgt=wgt, npix_x=512, npix_y=384, pixsize_x=ps,
                pixsize_y=ps, epsilon=epsilon, do_wgridding=do_w, nthreads=nthreads)
    capfd.readouterr()
    ducc.vis2dirty(vis=vis, verbosity=1, **args)
    out = capfd.readouterr().out
    m = re.search(r"grid=\((\d+)x(\d+)(?:x(\d+))?\), supp=(\d+)", out)
    assert m, out
    mine = ng.wgrid_params(vis=vis, **args)
    assert (mine["nu"], mine["nv"], mine["supp"]) == (int(m.group(1)), int(m.group(2)),
                                                      int(m.group(4)))
    if do_w:
        assert mine["nplanes"] == int(m.group(3))


@pmp("singleprec,epsilon", [(True, 1e-5), (False, 1e-9)])
def test_against_ducc_large(ng, ducc, singleprec, epsilon):
    """400k visibilities on a 2048^2 image at a 5 degree field of view (some
    tens of w planes, about 4e5 tiles of the oversampled grid): both
    directions against DUCC."""
    ps, freq, uvw, vis, wgt, mask, dirty = _ms_problem(41, 50000, 8, 2048, 5., singleprec, True)
    args = dict(uvw=uvw, freq=freq, wgt=wgt, mask=mask, pixsize_x=ps, pixsize_y=ps,
                epsilon=epsilon, do_wgridding=True, nthreads=16)
    p = ng.wgrid_params(vis=vis, npix_x=2048, npix_y=2048, **args)
    assert p["nplanes"] >= 10
    d_ours = ng.vis2dirty(vis=vis, npix_x=2048, npix_y=2048, **args)
    d_ref = ducc.vis2dirty(vis=vis, npix_x=2048, npix_y=2048, **args)
    assert O.l2error(d_ours, d_ref) <= 2 * epsilon
    v_ours = ng.dirty2vis(dirty=dirty, **args)
    v_ref = ducc.dirty2vis(dirty=dirty, **args)
    assert O.l2error(v_ours, v_ref) <= 2 * epsilon


@pmp("singleprec", (False, True))
def test_plane_shares_sum_to_whole(ng, singleprec):
    """The planes=(begin, count) shares of ducc_b200.distributed's split: the
    results over a partition of the w planes sum to the whole call's, a share
    past the last plane gives zeros, and without w-stacking the one share is
    plane 0."""
    ps, freq, uvw, vis, wgt, mask, dirty = _ms_problem(51, 4000, 4, 200, 10., singleprec, True)
    args = dict(uvw=uvw, freq=freq, wgt=wgt, mask=mask, pixsize_x=ps, pixsize_y=ps,
                epsilon=1e-5 if singleprec else 1e-9, do_wgridding=True)
    nplanes = ng.wgrid_params(vis=vis, npix_x=200, npix_y=200, **args)["nplanes"]
    assert nplanes >= 4
    cuts = [0, 1, nplanes // 2, nplanes]
    shares = [(a, b - a) for a, b in zip(cuts[:-1], cuts[1:])]
    tol = 1e-5 if singleprec else 1e-12
    whole = ng.vis2dirty(vis=vis, npix_x=200, npix_y=200, **args)
    parts = sum(ng.vis2dirty(vis=vis, npix_x=200, npix_y=200, planes=s, **args).astype("f8")
                for s in shares)
    assert O.l2error(parts, whole) < tol
    assert np.all(ng.vis2dirty(vis=vis, npix_x=200, npix_y=200, planes=(nplanes, 1), **args) == 0)
    vwhole = ng.dirty2vis(dirty=dirty, **args)
    vparts = sum(ng.dirty2vis(dirty=dirty, planes=s, **args).astype("c16") for s in shares)
    assert O.l2error(vparts, vwhole) < tol
    assert np.all(ng.dirty2vis(dirty=dirty, planes=(nplanes, 1), **args) == 0)
    args["do_wgridding"] = False
    assert np.all(ng.vis2dirty(vis=vis, npix_x=200, npix_y=200, planes=(1, 1), **args) == 0)
    # (the spreader's atomic additions come in a different order each call)
    assert O.l2error(ng.vis2dirty(vis=vis, npix_x=200, npix_y=200, planes=(0, 1), **args),
                     ng.vis2dirty(vis=vis, npix_x=200, npix_y=200, **args)) < tol

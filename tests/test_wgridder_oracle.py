"""The w-gridder's direct sums (oracle/wgridder_oracle.py) pinned against DUCC's
own w-gridder (oracle/_ref, built from the reference sources) at epsilon =
1e-12 on small problems, over the options: with and without the w term, axis
flips, an image centre off the phase centre, and without the division by n.
CPU only."""
import numpy as np
import pytest

from oracle import wgridder_oracle as O

OPTS = [dict(), dict(flip_u=True, center_x=0.01, center_y=-0.02),
        dict(flip_v=True, flip_w=True, center_x=-0.03), dict(divide_by_n=False)]


@pytest.fixture(scope="module")
def ducc():
    from oracle import ref
    m = ref.load()
    if m is None or not hasattr(m, "wgridder"):
        pytest.skip("DUCC's w-gridder (oracle/_ref) not built")
    return m.wgridder


@pytest.mark.parametrize("do_w", (False, True))
@pytest.mark.parametrize("opt", range(len(OPTS)))
def test_direct_sums_match_ducc(ducc, do_w, opt):
    kw = OPTS[opt]
    rng = np.random.default_rng(1 + opt)
    nrow, nchan, nx, ny = 20, 3, 32, 40
    psx = 10. * np.pi / 180 / nx
    psy = 1.1 * psx
    f0 = 1e9
    freq = f0 + np.arange(nchan) * f0 / nchan
    uvw = (rng.random((nrow, 3)) - 0.5) / (psx * f0 / O.SPEED_OF_LIGHT)
    vis = rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))
    wgt = rng.uniform(0.5, 1.5, (nrow, nchan))
    mask = (rng.random((nrow, nchan)) > 0.3).astype(np.uint8)
    args = dict(uvw=uvw, freq=freq, wgt=wgt, mask=mask, pixsize_x=psx, pixsize_y=psy,
                epsilon=1e-12, do_wgridding=do_w, **kw)
    d = ducc.vis2dirty(vis=vis, npix_x=nx, npix_y=ny, **args)
    assert O.l2error(d, O.explicit_gridder(uvw, freq, vis, wgt, nx, ny, psx, psy, do_w, mask,
                                           **kw)) < 1e-11
    dirty = rng.standard_normal((nx, ny))
    v = ducc.dirty2vis(dirty=dirty, **args)
    assert O.l2error(v, O.explicit_degridder(uvw, freq, dirty, wgt, psx, psy, do_w, mask,
                                             **kw)) < 1e-11

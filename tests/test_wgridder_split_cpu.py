"""The w-gridder's split over processes (ducc_b200.distributed.vis2dirty_split
/ dirty2vis_split) on the CPU with two and three `gloo` ranks: the plane
shares cover every plane once (a rank without planes asks for an empty range,
never for "all"), and the one all-reduce of the partial images / visibilities
gives every rank the whole result.  Without a GPU the rank's computation is
a stand-in that returns the direct sum (oracle/wgridder_oracle.py) weighted by
the share of the planes it was given, so the sum over the ranks is the direct
sum itself; the GPU test of the shares (tests/test_gpu_wgridder.py) checks
that the library's partial results add up the same way."""
import json
import os
import socket

import numpy as np
import pytest

from oracle import wgridder_oracle as O

NPLANES = 7


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    rng = np.random.default_rng(3)
    nrow, nchan, n = 40, 3, 24
    ps = 5. * np.pi / 180 / n
    freq = 1e9 + np.arange(nchan) * 1e8
    uvw = (rng.random((nrow, 3)) - 0.5) / (ps * 1e9 / O.SPEED_OF_LIGHT)
    vis = rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))
    dirty = rng.standard_normal((n, n))
    return dict(uvw=uvw, freq=freq, pixsize_x=ps, pixsize_y=ps, epsilon=1e-6,
                do_wgridding=True), vis, dirty


def _fraction(planes):
    b, c = planes
    return max(0, min(NPLANES, b + c) - b) / NPLANES


def _worker(rank, world, port, outdir):
    import datetime

    import torch.distributed as td

    from ducc_b200 import distributed as D
    td.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                          world_size=world, timeout=datetime.timedelta(seconds=60))
    seen = []
    try:
        kw, vis, dirty = _problem()
        n = dirty.shape[0]

        def grid(planes, **a):
            seen.append(list(planes))
            return O.explicit_gridder(a["uvw"], a["freq"], a["vis"], None, n, n,
                                      a["pixsize_x"], a["pixsize_y"], True, None) * \
                _fraction(planes)

        def degrid(planes, **a):
            return O.explicit_degridder(a["uvw"], a["freq"], a["dirty"], None, a["pixsize_x"],
                                        a["pixsize_y"], True, None) * _fraction(planes)

        img = D.vis2dirty_split(_run=grid, _nplanes=NPLANES, vis=vis, npix_x=n, npix_y=n, **kw)
        v = D.dirty2vis_split(_run=degrid, _nplanes=NPLANES, dirty=dirty, **kw)
        e1 = O.l2error(img, O.explicit_gridder(kw["uvw"], kw["freq"], vis, None, n, n,
                                              kw["pixsize_x"], kw["pixsize_y"], True, None))
        e2 = O.l2error(v, O.explicit_degridder(kw["uvw"], kw["freq"], dirty, None,
                                              kw["pixsize_x"], kw["pixsize_y"], True, None))
        td.barrier()
    finally:
        td.destroy_process_group()
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump({"err": [e1, e2], "planes": seen}, f)


@pytest.mark.parametrize("world", [2, 3])
def test_plane_split_sums_over_gloo_ranks(tmp_path, world):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(world)]
    covered = []
    for r in res:
        assert r["err"][0] < 1e-13 and r["err"][1] < 1e-13
        b, c = r["planes"][0]
        covered += list(range(b, min(NPLANES, b + c)))
    assert sorted(covered) == list(range(NPLANES))


def test_plane_share_partition():
    from ducc_b200.distributed import plane_share
    for n in (1, 2, 7, 16, 100):
        for world in (1, 2, 3, 8, 20):
            got = []
            for r in range(world):
                b, c = plane_share(n, world, r)
                assert c in (n // world, n // world + 1)
                got += list(range(b, b + c))
            assert got == list(range(n))

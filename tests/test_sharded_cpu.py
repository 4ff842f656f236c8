"""Host side of one transform split over several ranks (ducc_b200.distributed),
on the CPU: the parameter choice of the whole transform (the library's
restatement of DUCC's findNufftParameters against the oracle's), its
agreement over two `gloo` ranks, and the grid sum of the type-1 exchange.
Without a GPU the oracle's FP64 spreading, FFT and correction stand in for
the two CUDA halves of the type 1 (plan.spread / plan.grid_to_uniform, which
the GPU tests check against the library's own one-piece transform), so what
runs here is exactly the collective logic: count agreement, broadcast of the
parameters, the all-reduce of the complex grid, and that the sum of the
per-rank grids gives the transform of all points.
"""
import json
import os
import socket

import numpy as np
import pytest

from ducc_b200 import nufft
from oracle import nufft_oracle as O


@pytest.mark.parametrize("shape,M,eps,single", [
    ((4096, 4096), 50_000_000, 1e-6, True),
    ((4096, 4096), 1_000_000, 1e-6, True),
    ((256, 256), 200_000, 1e-6, False),
    ((300,), 5_000, 1e-9, False),
    ((48, 40, 32), 100_000, 1e-5, True),
    ((64, 64, 64), 2_000_000, 1e-10, False),
])
def test_find_parameters_matches_oracle(shape, M, eps, single):
    for nthreads in (1, 8):
        k, n = nufft.find_parameters(nu2u=True, grid_shape=shape, npoints=M, epsilon=eps,
                                     singleprec=single, nthreads=nthreads)
        ko, no = O.find_parameters(eps, 1.1, 2.6, list(shape), M, True, nthreads, single)
        assert k == ko and list(n) == list(no)


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


SHAPE = (40, 36)
EPS = 1e-9
M_RANK = (700, 1100)   # uneven shards


def _inputs():
    rng = np.random.default_rng(21)
    M = sum(M_RANK)
    coord = rng.uniform(-np.pi, np.pi, (M, 2))
    vals = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    return coord, vals


def _worker(rank, world, port, outdir):
    import datetime

    import torch
    import torch.distributed as td

    from ducc_b200 import distributed as D
    td.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                          world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        coord, vals = _inputs()
        a = sum(M_RANK[:rank])
        mine = slice(a, a + M_RANK[rank])
        kidx, nover, total = D.global_parameters(nu2u=True, grid_shape=SHAPE,
                                                 npoints_local=M_RANK[rank], epsilon=EPS,
                                                 singleprec=False, nthreads=4)
        p = O.Params(SHAPE, EPS, False, total, True, force=(kidx, nover))
        # this rank's half of the type 1: its points spread on the oversampled grid
        g = torch.from_numpy(O.spread(p, coord[mine], vals[mine]))
        D.sum_grids(g)
        # the other half from the summed grid: FFT + correction of the oracle
        full = O._fft(g.numpy(), True)
        out = np.zeros(SHAPE, np.complex128)
        maps = O._index_maps(p, False)
        fac = np.ones(())
        for d, (icf, iu, ig) in enumerate(maps):
            shp = [1, 1]
            shp[d] = -1
            fac = fac * p.corfac[d][icf].reshape(shp)
        out[np.ix_(maps[0][1], maps[1][1])] = full[np.ix_(maps[0][2], maps[1][2])] * fac
        ref = O.nu2u(p, coord, vals, True)
        err = O.l2error(out, ref)
        td.barrier()
    finally:
        td.destroy_process_group()
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump({"kidx": kidx, "nover": nover, "total": total, "err": err}, f)


def test_two_gloo_ranks_type1_exchange(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(world)]
    k, n = nufft.find_parameters(nu2u=True, grid_shape=SHAPE, npoints=sum(M_RANK), epsilon=EPS,
                                 singleprec=False, nthreads=4)
    for r in res:
        assert r["total"] == sum(M_RANK)
        assert r["kidx"] == k and r["nover"] == list(n)
        # the summed shard grids give the transform of all points (FP64 sums
        # in another order)
        assert r["err"] < 1e-13


def test_find_parameters_argument_errors():
    import ctypes

    from ducc_b200 import _capi as C
    L = C.lib()
    o = C.make_opts(True, 0, 1.1, 2.6, 2 * np.pi, False, 0, "auto", 2)
    shp = (ctypes.c_int64 * 3)(64, 64, 1)
    k = ctypes.c_int32()
    n = (ctypes.c_int64 * 3)()
    assert L.dnufft_find_parameters(1, 4, shp, 1000, 1e-6, 1, 1, ctypes.byref(o),
                                    ctypes.byref(k), n) == 1
    assert b"dimensionality" in L.dnufft_last_error()
    assert L.dnufft_find_parameters(1, 2, shp, 1000, -1.0, 1, 1, ctypes.byref(o),
                                    ctypes.byref(k), n) == 1
    assert b"epsilon" in L.dnufft_last_error()
    # below the reachable accuracy of single precision
    assert L.dnufft_find_parameters(1, 2, shp, 1000, 1e-9, 0, 0, ctypes.byref(o),
                                    ctypes.byref(k), n) == 2
    with pytest.raises(RuntimeError):
        nufft.find_parameters(nu2u=True, grid_shape=(64, 64), npoints=10, epsilon=1e-9,
                              singleprec=True)


def _slab_worker(rank, world, port, outdir):
    import datetime

    import torch
    import torch.distributed as td

    from ducc_b200 import distributed as D
    td.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                          world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        coord, vals = _inputs()
        cuts = [0, 500, 1300, sum(M_RANK)]
        mine = slice(cuts[rank], cuts[rank + 1])
        kidx, nover, total = D.global_parameters(nu2u=True, grid_shape=SHAPE,
                                                 npoints_local=cuts[rank + 1] - cuts[rank],
                                                 epsilon=EPS, singleprec=False, nthreads=4)
        p = O.Params(SHAPE, EPS, False, total, True, force=(kidx, nover))
        maps = O._index_maps(p, False)
        fac = np.ones(())
        for d, (icf, iu, ig) in enumerate(maps):
            shp = [1, 1]
            shp[d] = -1
            fac = fac * p.corfac[d][icf].reshape(shp)
        rows_done = []

        def spread_into(buf):
            buf.copy_(torch.from_numpy(O.spread(p, coord[mine], vals[mine])))

        def rows_fft(rows):
            rows_done.append(rows.shape[0])
            rows.copy_(torch.from_numpy(np.fft.fft(rows.numpy(), axis=1)))

        def cols_to_uniform(kept):
            # packed kept columns back to their grid positions, then the columns
            lo, hi = (SHAPE[1] + 1) // 2, SHAPE[1] // 2
            g = np.zeros(tuple(nover), np.complex128)
            g[:, :lo] = kept.numpy()[:, :lo]
            g[:, nover[1] - hi:] = kept.numpy()[:, lo:]
            full = np.fft.fft(g, axis=0)
            out = np.zeros(SHAPE, np.complex128)
            out[np.ix_(maps[0][1], maps[1][1])] = full[np.ix_(maps[0][2], maps[1][2])] * fac
            return out

        got = D.type1_by_slabs(spread_into=spread_into, rows_fft=rows_fft,
                               cols_to_uniform=cols_to_uniform, nover=nover,
                               nkept=SHAPE[1], dtype=torch.complex128,
                               device=torch.device("cpu"))
        err = O.l2error(got, O.nu2u(p, coord, vals, True))
        td.barrier()
    finally:
        td.destroy_process_group()
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump({"err": err, "rows": rows_done, "nover": nover}, f)


def test_three_gloo_ranks_type1_slab_exchange(tmp_path):
    """Reduce-scatter of row slabs (88 oversampled rows over three ranks: the
    last slab holds padding rows), row FFTs per slab, all-gather of the kept
    columns, column pass on every rank: the type 1 of all points everywhere."""
    import torch.multiprocessing as mp
    world = 3
    mp.spawn(_slab_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(world)]
    n0 = res[0]["nover"][0]
    r = -(-n0 // world)
    assert sum(sum(x["rows"]) for x in res) == n0      # every row transformed once
    assert res[0]["rows"] == [r]
    for x in res:
        assert x["err"] < 1e-13


def test_exchange_helpers_one_rank():
    """The packing of the kept columns (first (N+1)//2 and last N//2 of each
    row) and the row-count check of the reduce-scatter, on a one-rank group."""
    import datetime

    import torch
    import torch.distributed as td

    from ducc_b200 import distributed as D
    td.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0,
                          world_size=1, timeout=datetime.timedelta(seconds=30))
    try:
        g = torch.arange(6 * 10, dtype=torch.float64).reshape(6, 10).to(torch.complex128)
        assert torch.equal(D.reduce_scatter_rows(g.clone()), g)
        for nk in (1, 4, 5, 10):
            k = D.gather_kept_columns(g, nk)
            lo, hi = (nk + 1) // 2, nk // 2
            assert k.shape == (6, nk)
            assert torch.equal(k[:, :lo], g[:, :lo])
            assert torch.equal(k[:, lo:], g[:, 10 - hi:])
        with pytest.raises(ValueError):
            D.reduce_scatter_rows(g[:, ::2])          # not contiguous
        s = torch.ones(4, 3, dtype=torch.complex64)
        assert torch.equal(D.sum_grids(s), torch.ones(4, 3, dtype=torch.complex64))
    finally:
        td.destroy_process_group()


def _rows_worker(rank, world, port, outdir):
    """Row-slab partition on `gloo` ranks: points routed to their slab owners,
    spread there (the oracle's FP64 spreading), halo rows exchanged, row FFTs
    per slab, kept columns transposed into column blocks, each block's column
    pass (numpy FFT + the oracle's correction factors) and the all-gather of
    the blocks; then type-2 results routed back to the points' own ranks."""
    import datetime

    import torch
    import torch.distributed as td

    from ducc_b200 import distributed as D
    td.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                          world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(33)
        M = 2600
        coord = rng.uniform(-np.pi, np.pi, (M, 2))
        coord[:40, 0] = np.pi * (1 - 1e-9)   # footprints across the periodic edge
        vals = rng.standard_normal(M) + 1j * rng.standard_normal(M)
        cuts = np.linspace(0, M, world + 1).astype(int)
        mine = slice(cuts[rank], cuts[rank + 1])
        kidx, nover, total = D.global_parameters(nu2u=True, grid_shape=SHAPE,
                                                 npoints_local=cuts[rank + 1] - cuts[rank],
                                                 epsilon=EPS, singleprec=False, nthreads=4)
        p = O.Params(SHAPE, EPS, False, total, True, force=(kidx, nover))
        slabs = D.RowSlabs(nover[0], SHAPE[1], world)
        c_mine = torch.from_numpy(coord[mine])
        owner = slabs.owner(D.row_estimate(c_mine[:, 0], nover[0], 2 * np.pi))
        order, send, recv, owned = D.route_points(owner, c_mine, world)
        ovals = D.route_values(torch.from_numpy(vals[mine]), order, send, recv)
        # every owned point's footprint stays within its owner's slab and halos
        s0, s1 = slabs.slab(rank)
        fold, _ = O.getpix(p, owned.numpy())
        W = p.W
        for i0 in fold[:, 0]:
            rows = np.arange(i0, i0 + W) % nover[0]
            rel = (rows - (s0 - slabs.HALO)) % nover[0]
            assert np.all(rel < (s1 - s0) + 2 * slabs.HALO)
        maps = O._index_maps(p, False)
        icf0, iu0, ig0 = maps[0]
        icf1, iu1, ig1 = maps[1]
        N0, N1 = SHAPE
        lo = (N1 + 1) // 2
        rows_done = []

        def spread_into(buf):
            buf.copy_(torch.from_numpy(O.spread(p, owned.numpy(), ovals.numpy())))

        def rows_fft(rows):
            rows_done.append(rows.shape[0])
            rows.copy_(torch.from_numpy(np.fft.fft(rows.numpy(), axis=1)))

        def cols_block(cols, c0):
            full = np.fft.fft(cols.numpy(), axis=0)
            w = cols.shape[1]
            out = np.zeros((N0, w), np.complex128)
            for x in range(w):
                xg = c0 + x
                gx = xg if xg < lo else nover[1] - N1 + xg
                j = int(np.nonzero(ig1 == gx)[0][0])
                out[iu0, x] = full[ig0, x] * p.corfac[0][icf0] * p.corfac[1][icf1[j]]
            return torch.from_numpy(out)

        got = D.type1_by_row_slabs(spread_into=spread_into, rows_fft=rows_fft,
                                   cols_block=cols_block, slabs=slabs, nover=nover,
                                   nuni0=N0, shift=N1 // 2, dtype=torch.complex128,
                                   device=torch.device("cpu"))
        err = O.l2error(got.numpy(), O.nu2u(p, coord, vals, True))
        # type 2: the owners evaluate their points, the results go back
        grid = rng.standard_normal(SHAPE) + 1j * rng.standard_normal(SHAPE)
        p2 = O.Params(SHAPE, EPS, False, total, False, force=(kidx, nover))
        back = D.route_back(torch.from_numpy(O.u2nu(p2, grid, owned.numpy(), False)), order,
                            send, recv)
        err2 = O.l2error(back.numpy(), O.u2nu(p2, grid, coord[mine], False))
        td.barrier()
    finally:
        td.destroy_process_group()
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump({"err": err, "err2": err2, "rows": rows_done, "nover": nover,
                   "owned": int(owned.shape[0])}, f)


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_type1_row_slab_partition(tmp_path, world):
    import torch.multiprocessing as mp
    mp.spawn(_rows_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(world)]
    n0 = res[0]["nover"][0]
    assert sum(sum(x["rows"]) for x in res) == n0       # every row transformed once
    assert sum(x["owned"] for x in res) == 2600          # every point owned once
    for x in res:
        assert x["err"] < 1e-13
        assert x["err2"] < 1e-13


def _rows2_worker(rank, world, port, outdir):
    """Row-slab type 2 on `gloo` ranks: column blocks of the uniform grid
    (numpy FFT with the oracle's correction and padding), blocks to row slabs,
    row FFTs of the slab, halo rows from the neighbours, the oracle's FP64
    interpolation of the owned points, results routed back."""
    import datetime

    import torch
    import torch.distributed as td

    from ducc_b200 import distributed as D
    td.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                          world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(34)
        M = 2400
        coord = rng.uniform(-np.pi, np.pi, (M, 2))
        coord[:30, 0] = -np.pi * (1 - 1e-9)
        cuts = np.linspace(0, M, world + 1).astype(int)
        mine = slice(cuts[rank], cuts[rank + 1])
        kidx, nover, total = D.global_parameters(nu2u=False, grid_shape=SHAPE,
                                                 npoints_local=cuts[rank + 1] - cuts[rank],
                                                 epsilon=EPS, singleprec=False, nthreads=4)
        p = O.Params(SHAPE, EPS, False, total, False, force=(kidx, nover))
        slabs = D.RowSlabs(nover[0], SHAPE[1], world)
        c_mine = torch.from_numpy(coord[mine])
        owner = slabs.owner(D.row_estimate(c_mine[:, 0], nover[0], 2 * np.pi))
        order, send, recv, owned = D.route_points(owner, c_mine, world)
        grid_u = rng.standard_normal(SHAPE) + 1j * rng.standard_normal(SHAPE)
        # the padded, corrected oversampled grid of the uniform array (the
        # oracle's type-2 first step) and its column FFT
        maps = O._index_maps(p, False)
        icf0, iu0, ig0 = maps[0]
        icf1, iu1, ig1 = maps[1]
        full = np.zeros(tuple(nover), np.complex128)
        full[np.ix_(ig0, ig1)] = grid_u[np.ix_(iu0, iu1)] * np.outer(p.corfac[0][icf0],
                                                                     p.corfac[1][icf1])
        colfft = np.fft.fft(full, axis=0)
        N1 = SHAPE[1]
        lo = (N1 + 1) // 2

        def uniform_to_cols(c0, nc):
            xs = np.arange(c0, c0 + nc)
            gx = np.where(xs < lo, xs, nover[1] - N1 + xs)
            return torch.from_numpy(np.ascontiguousarray(colfft[:, gx]))

        def rows_fft_kept_in(rows):
            rows.copy_(torch.from_numpy(np.fft.fft(rows.numpy(), axis=1)))

        def interp(g):
            return torch.from_numpy(O.interpolate(p, g.numpy(), owned.numpy()))

        res = D.type2_by_row_slabs(uniform_to_cols=uniform_to_cols,
                                   rows_fft_kept_in=rows_fft_kept_in, interp=interp,
                                   slabs=slabs, nover=nover, dtype=torch.complex128,
                                   device=torch.device("cpu"))
        back = D.route_back(res, order, send, recv)
        err = O.l2error(back.numpy(), O.u2nu(p, grid_u, coord[mine], True))
        td.barrier()
    finally:
        td.destroy_process_group()
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump({"err": err}, f)


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_type2_row_slab_partition(tmp_path, world):
    import torch.multiprocessing as mp
    mp.spawn(_rows2_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        assert json.load(open(tmp_path / ("rank%d.json" % r)))["err"] < 1e-13

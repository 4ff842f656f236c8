"""Type 1 in two halves (plan.spread + plan.grid_to_uniform), the pieces of a
transform whose points are split over several GPUs: the halves against the
plan's one-piece type 1, two shards whose summed grids give the transform of
all points (checked against the one-piece transform and direct sums), the
sharded plan over a one-rank NCCL group, and argument errors.
"""
import numpy as np
import pytest

from ducc_b200 import nufft
from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu


def _problem(ndim, M, single, seed):
    rng = np.random.default_rng(seed)
    coord = rng.uniform(-np.pi, np.pi, (M, ndim))
    vals = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    if single:
        return coord.astype(np.float32), vals.astype(np.complex64)
    return coord, vals


CASES = [((256, 240), 400_000, True, 1e-6),     # tensor-core spreader ('auto')
         ((96, 80), 30_000, True, 1e-5),        # plain
         ((96, 80), 30_000, False, 1e-11),
         ((400,), 20_000, False, 1e-10),
         ((24, 20, 16), 20_000, True, 1e-5)]


@pytest.mark.parametrize("shape,M,single,eps", CASES)
def test_halves_equal_one_piece(shape, M, single, eps):
    import torch
    coord, vals = _problem(len(shape), M, single, 3)
    dc, dv = torch.from_numpy(coord).cuda(), torch.from_numpy(vals).cuda()
    p = nufft.plan(nu2u=True, coord=dc, grid_shape=shape, epsilon=eps)
    for forward in (True, False):
        ref = p.nu2u(points=dv, forward=forward).cpu().numpy()
        g = p.spread(points=dv)
        assert tuple(g.shape) == tuple(p.info()["nover"]) and g.is_contiguous()
        got = p.grid_to_uniform(forward=forward, grid=g).cpu().numpy()
        # same kernels; float atomics may add in another order
        assert O.l2error(got, ref) < (1e-6 if single else 1e-14)


@pytest.mark.parametrize("shape,M,single,eps", CASES)
def test_two_shards_sum_to_whole(shape, M, single, eps):
    import torch
    coord, vals = _problem(len(shape), M, single, 4)
    k, n = nufft.find_parameters(nu2u=True, grid_shape=shape, npoints=M, epsilon=eps,
                                 singleprec=single)
    cut = M // 3
    parts = []
    for sl in (slice(0, cut), slice(cut, M)):
        dc = torch.from_numpy(np.ascontiguousarray(coord[sl])).cuda()
        parts.append((nufft.plan(nu2u=True, coord=dc, grid_shape=shape, epsilon=eps,
                                 force_kernel=k, force_nover=n),
                      torch.from_numpy(np.ascontiguousarray(vals[sl])).cuda()))
    whole = nufft.plan(nu2u=True, coord=torch.from_numpy(coord).cuda(), grid_shape=shape,
                       epsilon=eps, force_kernel=k, force_nover=n)
    g = parts[0][0].spread(points=parts[0][1])
    g += parts[1][0].spread(points=parts[1][1])
    got = parts[0][0].grid_to_uniform(forward=True, grid=g).cpu().numpy()
    ref = whole.nu2u(points=torch.from_numpy(vals).cuda(), forward=True).cpu().numpy()
    assert O.l2error(got, ref) < (2e-6 if single else 1e-13)
    # against the direct sum over a sample of points (all modes)
    sub = slice(0, 2000)
    p_sub = nufft.plan(nu2u=True, coord=torch.from_numpy(np.ascontiguousarray(coord[sub])).cuda(),
                       grid_shape=shape, epsilon=eps, force_kernel=k, force_nover=n)
    ga = p_sub.spread(points=torch.from_numpy(np.ascontiguousarray(vals[sub])).cuda())
    got_sub = p_sub.grid_to_uniform(forward=True, grid=ga).cpu().numpy()
    exact = O.direct_nu2u(coord[sub].astype(np.float64), vals[sub].astype(np.complex128), shape,
                          True)
    assert O.l2error(got_sub, exact) < 4 * eps


def test_sharded_plan_one_rank_nccl():
    import datetime
    import socket

    import torch
    import torch.distributed as td

    from ducc_b200 import distributed as D
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    td.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                          world_size=1, timeout=datetime.timedelta(seconds=60),
                          device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        shape, M, eps = (128, 112), 60_000, 1e-6
        coord, vals = _problem(2, M, True, 5)
        dc, dv = torch.from_numpy(coord).cuda(), torch.from_numpy(vals).cuda()
        sp = D.ShardedPlan(nu2u=True, coord=dc, grid_shape=shape, epsilon=eps)
        k, n = nufft.find_parameters(nu2u=True, grid_shape=shape, npoints=M, epsilon=eps,
                                     singleprec=True)
        assert sp.kernel_index == k and list(sp.nover) == list(n) and sp.npoints_total == M
        got = sp.nu2u(forward=False, points=dv).cpu().numpy()
        ref = nufft.plan(nu2u=True, coord=dc, grid_shape=shape, epsilon=eps, force_kernel=k,
                         force_nover=n).nu2u(points=dv, forward=False).cpu().numpy()
        assert O.l2error(got, ref) < 1e-6
        grid = torch.from_numpy((np.random.default_rng(6).standard_normal(shape)
                                 + 0j).astype(np.complex64)).cuda()
        pts = sp.u2nu(forward=True, grid=grid).cpu().numpy()
        idx = np.arange(0, M, 97)
        exact = O.direct_u2nu(grid.cpu().numpy().astype(np.complex128),
                              coord[idx].astype(np.float64), True)
        assert O.l2error(pts[idx], exact) < 4 * eps
        td.barrier()
    finally:
        td.destroy_process_group()


def test_split_type1_argument_errors():
    import torch
    coord, vals = _problem(2, 5000, True, 7)
    dc, dv = torch.from_numpy(coord).cuda(), torch.from_numpy(vals).cuda()
    p = nufft.plan(nu2u=True, coord=dc, grid_shape=(64, 64), epsilon=1e-5)
    nover = tuple(p.info()["nover"])
    with pytest.raises(RuntimeError, match="oversampled sizes"):
        p.spread(points=dv, out=torch.empty((nover[0], nover[1] + 2), dtype=torch.complex64,
                                            device="cuda"))
    with pytest.raises(RuntimeError, match="C-contiguous"):
        big = torch.empty((nover[1], nover[0]), dtype=torch.complex64, device="cuda")
        p.spread(points=dv, out=big.t())
    with pytest.raises(RuntimeError, match="data type"):
        p.spread(points=dv, out=torch.empty(nover, dtype=torch.complex128, device="cuda"))
    with pytest.raises(RuntimeError, match="device array"):
        p.grid_to_uniform(forward=True, grid=np.zeros(nover, np.complex64))
    with pytest.raises(RuntimeError, match="number of points"):
        p.spread(points=dv[:100])


def test_empty_shard_contributes_zero():
    """A rank without points: its plan spreads a zero grid, and the sum with a
    shard holding every point is that shard's transform."""
    import torch
    shape, eps = (64, 48), 1e-6
    coord, vals = _problem(2, 20_000, True, 8)
    k, n = nufft.find_parameters(nu2u=True, grid_shape=shape, npoints=20_000, epsilon=eps,
                                 singleprec=True)
    empty = nufft.plan(nu2u=True, coord=torch.zeros((0, 2), dtype=torch.float32, device="cuda"),
                       grid_shape=shape, epsilon=eps, force_kernel=k, force_nover=n)
    full = nufft.plan(nu2u=True, coord=torch.from_numpy(coord).cuda(), grid_shape=shape,
                      epsilon=eps, force_kernel=k, force_nover=n)
    g0 = empty.spread(points=torch.zeros(0, dtype=torch.complex64, device="cuda"))
    assert float(g0.abs().max()) == 0.0
    dv = torch.from_numpy(vals).cuda()
    g = full.spread(points=dv) + g0
    got = empty.grid_to_uniform(forward=True, grid=g).cpu().numpy()
    ref = full.nu2u(points=dv, forward=True).cpu().numpy()
    assert O.l2error(got, ref) < 1e-6


@pytest.mark.parametrize("shape", [(300, 260), (1100, 1000)])   # line kernels / row + four-step kernels
@pytest.mark.parametrize("single,eps", [(True, 1e-6), (False, 1e-11)])
def test_row_slabs_then_columns_equal_one_piece(single, eps, shape):
    """The 2D FFT half split into row slabs (each transformed on its own) and
    the column pass equals the plan's one-piece type 1."""
    import torch
    coord, vals = _problem(2, 200_000, single, 9)
    dc, dv = torch.from_numpy(coord).cuda(), torch.from_numpy(vals).cuda()
    p = nufft.plan(nu2u=True, coord=dc, grid_shape=shape, epsilon=eps)
    for forward in (True, False):
        ref = p.nu2u(points=dv, forward=forward).cpu().numpy()
        g = p.spread(points=dv)
        cut = g.shape[0] // 3
        p.rows_fft(forward=forward, rows=g[:cut])
        p.rows_fft(forward=forward, rows=g[cut:])
        # the kept columns packed, as the slab exchange gathers them
        lo, hi = (shape[1] + 1) // 2, shape[1] // 2
        packed = torch.cat([g[:, :lo], g[:, g.shape[1] - hi:]], dim=1).contiguous()
        got = p.cols_to_uniform(forward=forward, grid=g).cpu().numpy()
        got_p = p.cols_to_uniform(forward=forward, grid=packed).cpu().numpy()
        # two separate spreads: atomic additions in another order
        assert O.l2error(got, ref) < (1e-6 if single else 1e-13)
        assert O.l2error(got_p, got) < (1e-7 if single else 1e-15)


def test_sharded_plan_exchanges_agree():
    import datetime
    import socket

    import torch
    import torch.distributed as td

    from ducc_b200 import distributed as D
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    td.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                          world_size=1, timeout=datetime.timedelta(seconds=60),
                          device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        coord, vals = _problem(2, 80_000, True, 10)
        dc, dv = torch.from_numpy(coord).cuda(), torch.from_numpy(vals).cuda()
        sp = D.ShardedPlan(nu2u=True, coord=dc, grid_shape=(160, 144), epsilon=1e-6)
        a = sp.nu2u(forward=True, points=dv, exchange="slabs").cpu().numpy()
        b = sp.nu2u(forward=True, points=dv, exchange="grid").cpu().numpy()
        assert O.l2error(a, b) < 1e-6
        exact = O.direct_nu2u(coord[:3000].astype(np.float64), vals[:3000].astype(np.complex128),
                              (160, 144), True)
        sub = D.ShardedPlan(nu2u=True, coord=dc[:3000].contiguous(), grid_shape=(160, 144),
                            epsilon=1e-6)
        assert O.l2error(sub.nu2u(forward=True, points=dv[:3000].contiguous()).cpu().numpy(),
                         exact) < 4e-6
        td.barrier()
    finally:
        td.destroy_process_group()


def test_rows_cols_argument_errors():
    import torch
    coord, vals = _problem(3, 5000, True, 11)
    p3 = nufft.plan(nu2u=True, coord=torch.from_numpy(coord).cuda(), grid_shape=(16, 16, 16),
                    epsilon=1e-5)
    n3 = tuple(p3.info()["nover"])
    with pytest.raises(RuntimeError, match="2D plans only"):
        p3.rows_fft(forward=True, rows=torch.zeros((n3[0], n3[1] * n3[2]), dtype=torch.complex64,
                                                   device="cuda"))
    coord2, _ = _problem(2, 5000, True, 12)
    p = nufft.plan(nu2u=True, coord=torch.from_numpy(coord2).cuda(), grid_shape=(64, 64),
                   epsilon=1e-5)
    n = tuple(p.info()["nover"])
    with pytest.raises(RuntimeError, match="cells expected"):
        p.rows_fft(forward=True, rows=torch.zeros((4, n[1] + 1), dtype=torch.complex64,
                                                  device="cuda"))
    with pytest.raises(RuntimeError, match="device array"):
        p.rows_fft(forward=True, rows=np.zeros((4, n[1]), np.complex64))
    with pytest.raises(RuntimeError, match="oversampled sizes"):
        p.cols_to_uniform(forward=True, grid=torch.zeros((n[0] - 1, n[1]), dtype=torch.complex64,
                                                         device="cuda"))


@pytest.mark.parametrize("single,fft_order,shape", [(True, False, (600, 300)),
                                                    (False, True, (800, 300))])
def test_column_blocks_equal_one_piece(single, fft_order, shape):
    """The column pass split into blocks of kept columns (the sharded column
    pass), each block's uniform columns packed, reassembled by the documented
    column rule, equals the one-piece column pass."""
    import torch
    coord, vals = _problem(2, 100_000, single, 12)
    dc, dv = torch.from_numpy(coord).cuda(), torch.from_numpy(vals).cuda()
    p = nufft.plan(nu2u=True, coord=dc, grid_shape=shape, epsilon=1e-6 if single else 1e-11,
                   fft_order=fft_order)
    assert p.info()["nover"][0] >= 1024   # the four-step column passes
    N0, N1 = shape
    lo, hi = (N1 + 1) // 2, N1 // 2
    for forward in (True, False):
        g = p.spread(points=dv)
        p.rows_fft(forward=forward, rows=g)
        packed = torch.cat([g[:, :lo], g[:, g.shape[1] - hi:]], dim=1).contiguous()
        ref = p.cols_to_uniform(forward=forward, grid=packed.clone()).cpu().numpy()
        got = np.zeros(shape, ref.dtype)
        s = 0 if fft_order else N1 // 2
        for c0, c1 in ((0, 37), (37, 150), (150, 151), (151, N1)):
            blk = packed[:, c0:c1].contiguous()
            o = p.cols_to_uniform_range(forward=forward, cols=blk, col0=c0).cpu().numpy()
            got[:, (np.arange(c0, c1) + s) % N1] = o
        assert O.l2error(got, ref) < (1e-7 if single else 1e-15)
    with pytest.raises(RuntimeError, match="outside the kept columns"):
        p.cols_to_uniform_range(forward=True, cols=packed[:, :10].contiguous(), col0=N1 - 5)


def test_sharded_plan_row_partition_one_rank():
    """The row-slab partition on a one-rank NCCL group: points routed to their
    owner (itself), spread, row FFTs of the slab, the kept columns as one
    column block through the block column pass, the block gathered; type 2
    results routed back.  Equal to the plain plan's transforms."""
    import datetime
    import socket

    import torch
    import torch.distributed as td

    from ducc_b200 import distributed as D
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    td.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                          world_size=1, timeout=datetime.timedelta(seconds=60),
                          device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        shape = (600, 400)
        coord, vals = _problem(2, 150_000, True, 13)
        dc, dv = torch.from_numpy(coord).cuda(), torch.from_numpy(vals).cuda()
        for fo, per in ((False, 2 * np.pi), (True, [3.0, 2 * np.pi])):
            sp = D.ShardedPlan(nu2u=True, coord=dc, grid_shape=shape, epsilon=1e-6,
                               partition="rows", fft_order=fo, periodicity=per)
            assert sp.partition == "rows" and sp.nover[0] >= 1024
            ref_p = nufft.plan(nu2u=True, coord=dc, grid_shape=shape, epsilon=1e-6,
                               fft_order=fo, periodicity=per)
            for forward in (True, False):
                a = sp.nu2u(forward=forward, points=dv).cpu().numpy()
                b = ref_p.nu2u(points=dv, forward=forward).cpu().numpy()
                assert O.l2error(a, b) < 1e-6
                g = torch.randn(shape, dtype=torch.complex64, device="cuda")
                r2 = sp.u2nu(forward=forward, grid=g).cpu().numpy()
                assert O.l2error(r2, ref_p.u2nu(grid=g, forward=forward).cpu().numpy()) < 1e-6
        td.barrier()
    finally:
        td.destroy_process_group()


@pytest.mark.parametrize("single,fft_order,shape", [(True, True, (600, 300)),
                                                    (False, False, (800, 300))])
def test_type2_halves_equal_one_piece(single, fft_order, shape):
    """Type 2 in its three stages — column pass of blocks of kept columns from
    the uniform array, row FFTs of slabs with only the kept columns set,
    interpolation from the assembled grid — equals the plan's one-piece u2nu."""
    import torch
    coord, _ = _problem(2, 100_000, single, 14)
    dc = torch.from_numpy(coord).cuda()
    p = nufft.plan(nu2u=False, coord=dc, grid_shape=shape, epsilon=1e-6 if single else 1e-11,
                   fft_order=fft_order)
    n0, n1 = p.info()["nover"]
    assert n0 >= 1024
    N1 = shape[1]
    lo, hi = (N1 + 1) // 2, N1 // 2
    ct = torch.complex64 if single else torch.complex128
    for forward in (True, False):
        g = torch.randn(shape, dtype=ct, device="cuda")
        ref = p.u2nu(grid=g, forward=forward).cpu().numpy()
        blocks = [p.uniform_to_cols_range(forward=forward, grid=g, col0=a, ncols=b - a)
                  for a, b in ((0, 41), (41, 150), (150, N1))]
        packed = torch.cat(blocks, dim=1)
        grid = torch.zeros((n0, n1), dtype=ct, device="cuda")
        grid[:, :lo] = packed[:, :lo]
        grid[:, n1 - hi:] = packed[:, lo:]
        cut = n0 // 3
        p.rows_fft_kept_in(forward=forward, rows=grid[:cut])
        p.rows_fft_kept_in(forward=forward, rows=grid[cut:])
        got = p.interp(grid=grid).cpu().numpy()
        assert O.l2error(got, ref) < (1e-7 if single else 1e-14)

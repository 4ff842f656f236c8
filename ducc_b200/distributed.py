"""One NUFFT whose points are split over the GPUs of a node (one process per
GPU, ``torch.distributed``; NCCL over NVLink between GPUs).

Type 1 (``ShardedPlan.nu2u``): every rank spreads its own points into a full
oversampled grid (``plan.spread``); spreading is linear in the values, so the
sum of these grids over the ranks is the grid of all points, and summing them
is the real exchange step of the transform.  In 2D (``type1_by_slabs``) each
rank receives the sum of one slab of rows only (a reduce-scatter), transforms
those rows along axis 1 (``plan.rows_fft``), and the ranks gather the kept
columns of all rows (an all-gather of the N1 of n1 columns) for the column
pass, correction and crop, which every rank runs (``plan.cols_to_uniform``).
Against summing whole grids (``sum_grids`` + ``plan.grid_to_uniform``, the
1D / 3D path) this moves (1 + N1/n1) instead of 2 grids' worth of bytes per
rank and splits the row FFTs over the ranks.  Every rank holds the whole
uniform result.

Type 2 (``ShardedPlan.u2nu``): every rank has the whole uniform grid and
interpolates its own points; nothing crosses between ranks.

Both halves use the kernel and oversampled sizes that DUCC's parameter choice
(src/ducc0/nufft/nufft.h:155-216) gives for the total number of points,
agreed by one all-reduce of the counts (``global_parameters``), so the result
is the transform of all points on one GPU up to the order of the
floating-point sums.

Independent transforms (batches, separate problems) need no collective at
all: ``ducc_b200.shard`` splits them over the ranks by weight.
"""
import math

from . import nufft

__all__ = ["global_parameters", "sum_grids", "reduce_scatter_rows", "gather_kept_columns",
           "type1_by_slabs", "ShardedPlan"]


def _count_device(group):
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def global_parameters(*, nu2u, grid_shape, npoints_local, epsilon, singleprec,
                      coord_single=None, group=None, nthreads=0, sigma_min=1.1, sigma_max=2.6):
    """(kernel-table row, oversampled shape, total points) of the whole
    transform: the local point counts are summed over the group, DUCC's
    parameter choice is made for the total on the group's first rank and
    broadcast (its cost model with ``nthreads=0`` depends on the host's thread
    count, which need not be the same for every rank)."""
    import torch
    import torch.distributed as dist
    dev = _count_device(group)
    n = torch.tensor([int(npoints_local)], dtype=torch.int64, device=dev)
    dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
    total = int(n.item())
    ndim = len(grid_shape)
    kidx, nover = nufft.find_parameters(nu2u=nu2u, grid_shape=grid_shape, npoints=total,
                                        epsilon=epsilon, singleprec=singleprec,
                                        coord_single=coord_single, nthreads=nthreads,
                                        sigma_min=sigma_min, sigma_max=sigma_max)
    t = torch.tensor([kidx] + list(nover), dtype=torch.int64, device=dev)
    src = 0 if group is None else dist.get_global_rank(group, 0)
    dist.broadcast(t, src=src, group=group)
    v = [int(x) for x in t.tolist()]
    return v[0], v[1:1 + ndim], total


def sum_grids(grid, group=None):
    """Sum a complex oversampled grid over the ranks of the group, in place
    (an all-reduce of its real view); returns it."""
    import torch
    import torch.distributed as dist
    if not grid.is_contiguous():
        raise ValueError("sum_grids: the grid must be contiguous")
    dist.all_reduce(torch.view_as_real(grid), op=dist.ReduceOp.SUM, group=group)
    return grid


def reduce_scatter_rows(grid, group=None):
    """Sum a complex (world * r, ...) grid over the ranks of the group and
    return this rank's r rows of the sum (rank k: rows k*r .. k*r + r - 1)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if grid.shape[0] % world or not grid.is_contiguous():
        raise ValueError("reduce_scatter_rows: a contiguous grid of world * r rows expected")
    out = torch.empty((grid.shape[0] // world,) + tuple(grid.shape[1:]), dtype=grid.dtype,
                      device=grid.device)
    dist.reduce_scatter_tensor(torch.view_as_real(out), torch.view_as_real(grid),
                               op=dist.ReduceOp.SUM, group=group)
    return out


def _kept(n, N):
    """(first, last) counts of the kept indices of an axis: [0, (N+1)//2) and
    [n - N//2, n)."""
    return (N + 1) // 2, N // 2


def gather_kept_columns(rows, nkept, group=None):
    """All-gather the kept columns of every rank's (r, n1) rows: returns a
    (world * r, nkept) array, the first (nkept+1)//2 and the last nkept//2
    columns of each row, packed."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    n1 = rows.shape[1]
    lo, hi = _kept(n1, nkept)
    packed = torch.cat([rows[:, :lo], rows[:, n1 - hi:]], dim=1).contiguous()
    out = torch.empty((world * rows.shape[0], nkept), dtype=rows.dtype, device=rows.device)
    dist.all_gather_into_tensor(torch.view_as_real(out), torch.view_as_real(packed),
                                group=group)
    return out


def type1_by_slabs(*, spread_into, rows_fft, cols_to_uniform, nover, nkept, dtype, device,
                   group=None):
    """The slab exchange of a 2D type 1 with the local steps passed in:
    ``spread_into(buf)`` writes this rank's spread grid into ``buf`` (an
    (nover[0], nover[1]) C-contiguous tensor), ``rows_fft(rows)`` transforms
    rows along axis 1 in place, ``cols_to_uniform(kept)`` runs the column pass,
    correction and crop of the gathered kept columns (packed, (nover[0],
    nkept)) and returns the uniform result.  Collective over the group."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    n0, n1 = int(nover[0]), int(nover[1])
    r = -(-n0 // world)
    buf = torch.empty((r * world, n1), dtype=dtype, device=device)
    grid = buf[:n0]
    spread_into(grid)
    buf[n0:].zero_()
    slab = reduce_scatter_rows(buf, group)
    nr = max(0, min(r, n0 - rank * r))
    if nr:
        rows_fft(slab[:nr])
    kept = gather_kept_columns(slab, nkept, group)
    # the column pass takes the kept columns packed: no copy back into the grid
    return cols_to_uniform(kept[:n0])


class ShardedPlan:
    """Plan of this rank's points of one transform split over the ranks of a
    process group.  Arguments as ``ducc_b200.nufft.plan``; ``coord`` holds only
    this rank's points, ``epsilon`` and ``grid_shape`` are those of the whole
    transform and must be the same on every rank.  Construction is collective
    (every rank of the group calls it, in the same order as the other
    collectives)."""

    def __init__(self, *, nu2u, coord, grid_shape, epsilon, group=None, nthreads=0,
                 sigma_min=1.1, sigma_max=2.6, periodicity=2 * math.pi, fft_order=False,
                 spreader="auto"):
        import torch
        self.group = group
        if not torch.is_tensor(coord):
            raise TypeError("ShardedPlan: coord must be a torch CUDA tensor")
        single = coord.dtype == torch.float32
        kidx, nover, total = global_parameters(
            nu2u=nu2u, grid_shape=grid_shape, npoints_local=coord.shape[0], epsilon=epsilon,
            singleprec=single, coord_single=single, group=group, nthreads=nthreads,
            sigma_min=sigma_min, sigma_max=sigma_max)
        self.npoints_total = total
        self.kernel_index = kidx
        self.nover = nover
        self.plan = nufft.plan(nu2u=nu2u, coord=coord, grid_shape=grid_shape, epsilon=epsilon,
                               nthreads=nthreads, sigma_min=sigma_min, sigma_max=sigma_max,
                               periodicity=periodicity, fft_order=fft_order, spreader=spreader,
                               force_kernel=kidx, force_nover=nover)
        self.grid_shape = tuple(int(x) for x in grid_shape)
        self.npoints = coord.shape[0]
        self.device = coord.device

    def nu2u(self, *, forward, points, out=None, exchange=None):
        """Type 1 of all ranks' points (collective); every rank gets the whole
        uniform grid in ``out``.  ``exchange``: 'slabs' (the 2D default on
        several ranks: reduce-scatter of row slabs, row FFTs split over the
        ranks, all-gather of the kept columns) or 'grid' (all-reduce of whole
        grids, any dimension; the default otherwise)."""
        import torch
        import torch.distributed as dist
        if exchange is None:
            # one rank: nothing to exchange, and the grid path adds no copies
            multi = dist.get_world_size(self.group) > 1
            exchange = "slabs" if len(self.grid_shape) == 2 and multi else "grid"
        if exchange == "slabs":
            if len(self.grid_shape) != 2:
                raise ValueError("the slab exchange is for 2D transforms")
            dtype = torch.complex128 if self.plan._f64 else torch.complex64
            return type1_by_slabs(
                spread_into=lambda buf: self.plan.spread(points=points, out=buf),
                rows_fft=lambda rows: self.plan.rows_fft(forward=forward, rows=rows),
                cols_to_uniform=lambda g: self.plan.cols_to_uniform(forward=forward, grid=g,
                                                                    out=out),
                nover=self.nover, nkept=self.grid_shape[1], dtype=dtype,
                device=self.device, group=self.group)
        if exchange != "grid":
            raise ValueError("exchange must be 'slabs' or 'grid'")
        g = self.plan.spread(points=points)
        sum_grids(g, self.group)
        return self.plan.grid_to_uniform(forward=forward, grid=g, out=out)

    def u2nu(self, *, forward, grid, out=None):
        """Type 2 at this rank's points from the whole uniform grid (local,
        no collective)."""
        return self.plan.u2nu(forward=forward, grid=grid, out=out)

"""One NUFFT whose points are split over the GPUs of a node (one process per
GPU, ``torch.distributed``; NCCL over NVLink between GPUs).

Type 1 (``ShardedPlan.nu2u``): every rank spreads its own points into a full
oversampled grid (``plan.spread``), the grids are summed over the ranks with
one all-reduce (``sum_grids``), and every rank runs the FFT and the
correction of the sum (``plan.grid_to_uniform``), so each holds the whole
uniform result.  Spreading is linear in the values, so the summed grid is the
grid of all points: the single real exchange step of the transform.

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

__all__ = ["global_parameters", "sum_grids", "ShardedPlan"]


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

    def nu2u(self, *, forward, points, out=None):
        """Type 1 of all ranks' points (collective); every rank gets the whole
        uniform grid in ``out``."""
        g = self.plan.spread(points=points)
        sum_grids(g, self.group)
        return self.plan.grid_to_uniform(forward=forward, grid=g, out=out)

    def u2nu(self, *, forward, grid, out=None):
        """Type 2 at this rank's points from the whole uniform grid (local,
        no collective)."""
        return self.plan.u2nu(forward=forward, grid=grid, out=out)

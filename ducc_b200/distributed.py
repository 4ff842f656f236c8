"""One NUFFT whose points are split over the GPUs of a node (one process per
GPU, ``torch.distributed``; NCCL over NVLink between GPUs).

Type 1, row-slab partition (``ShardedPlan(partition="rows")``, 2D; the
default on several ranks): rank k owns the rows [k r, (k + 1) r) of the
oversampled grid (r = ceil(n0 / ranks)) and the points whose footprint starts
in them.  At plan time every rank sends each of its points' coordinates to the
owner (one all-to-all), per call the values follow the same route (one
all-to-all of M / ranks values per rank).  The owner spreads its points, which
touch only its slab and a halo of a few rows on either side; the halo rows go
to the neighbouring ranks and are added there (two sends and two receives of
H x n1 cells); each rank transforms its slab's rows along axis 1
(``plan.rows_fft``), the ranks exchange blocks of the kept columns (an
all-to-all that leaves rank j with all n0 rows of its block of N1 / ranks kept
columns), each runs the column pass, correction and crop of its block
(``plan.cols_to_uniform_range``), and an all-gather assembles the uniform
result on every rank.  Spreading, row FFTs and column passes are split over
the ranks; what crosses NVLink is the values, the halos, one transpose of the
kept columns and the result.

Type 1, point partition (``partition="points"``; also any dimension): every
rank spreads its own points into a full oversampled grid; in 2D each rank
receives the sum of one slab of rows (a reduce-scatter), transforms those rows
and the ranks gather the kept columns of all rows for a column pass that every
rank runs (``type1_by_slabs``), in 1D / 3D whole grids are summed
(``sum_grids``).

Type 2 (``ShardedPlan.u2nu``), every rank given the whole uniform grid: with
the row-slab partition the mirror of type 1 (the column pass of each rank's
block of kept columns, one all-to-all into row slabs, the slab's row FFTs,
halo rows copied from the neighbours, interpolation of the owned points, the
results routed back); with the point partition every rank runs the whole
transform head and interpolates its own points, nothing crossing between
ranks.

Both use the kernel and oversampled sizes that DUCC's parameter choice
(src/ducc0/nufft/nufft.h:155-216) gives for the total number of points,
agreed by one all-reduce of the counts (``global_parameters``), so the result
is the transform of all points on one GPU up to the order of the
floating-point sums.

Independent transforms (batches, separate problems) need no collective at
all: ``ducc_b200.shard`` splits them over the ranks by weight.

The w-gridder (``vis2dirty_split`` / ``dirty2vis_split``) splits its w
planes: each rank runs its consecutive share (spreading or interpolation and
the 2D FFT of each of its planes) into a partial image or partial
visibilities, and one all-reduce sums them.
"""
import math

from . import nufft

__all__ = ["global_parameters", "sum_grids", "reduce_scatter_rows", "gather_kept_columns",
           "type1_by_slabs", "RowSlabs", "row_estimate", "route_points", "route_values",
           "exchange_halos", "transpose_kept_columns", "gather_column_blocks",
           "route_back", "type1_by_row_slabs", "columns_to_row_slabs", "fill_halos",
           "type2_by_row_slabs", "ShardedPlan", "plane_share", "vis2dirty_split",
           "dirty2vis_split"]


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


# ---------------------------------------------------------------- row-slab partition
class RowSlabs:
    """Rank k owns the oversampled rows [start(k), start(k + 1)), start(k) =
    min(k * ceil(n0 / ranks), n0), and the kept columns [col(k), col(k + 1)),
    col(k) = min(k * ceil(N1 / ranks), N1).  A point whose footprint starts
    near row e (``row_estimate``) touches only rows e - HALO .. e + HALO
    (modulo n0): its owner's slab and at most HALO rows of each neighbour."""

    HALO = 11   # kernel support <= 16: footprints start within W/2 + 1 rows of e

    def __init__(self, n0, nkept, world):
        self.n0, self.nkept, self.world = int(n0), int(nkept), int(world)
        r = -(-self.n0 // self.world)
        self.rows = r
        self.starts = [min(k * r, self.n0) for k in range(self.world + 1)]
        c = -(-self.nkept // self.world)
        self.cols = [min(k * c, self.nkept) for k in range(self.world + 1)]
        if self.world > 1 and min(self.starts[k + 1] - self.starts[k]
                                  for k in range(self.world)) < self.HALO:
            raise ValueError("row slabs: %d oversampled rows are too few for %d ranks"
                             % (self.n0, self.world))

    def slab(self, k):
        return self.starts[k], self.starts[k + 1]

    def col_block(self, k):
        return self.cols[k], self.cols[k + 1]

    def owner(self, rows):
        """Owning rank of oversampled rows (a torch integer tensor)."""
        import torch
        return torch.clamp(torch.div(rows, self.rows, rounding_mode="floor"), max=self.world - 1)


def row_estimate(coord0, n0, period):
    """Oversampled row of each point along axis 0, floor(frac(x / period) * n0)
    in float64: DUCC's getpix (nufft.h:285-298) puts the first row of the
    footprint at this row minus W/2 - 1, up to one row of rounding."""
    import torch
    t = coord0.to(torch.float64) / float(period)
    f = t - torch.floor(t)
    return torch.remainder(torch.floor(f * n0).to(torch.int64), n0)


def route_points(owner, coord, world, group=None):
    """Send every point to its owner (collective).  Returns (order, send counts,
    receive counts, the owned points' coordinates): ``order`` sorts this
    rank's points by owner, stably."""
    import torch
    import torch.distributed as dist
    order = torch.argsort(owner, stable=True)
    send = torch.bincount(owner, minlength=world).to(torch.int64)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    send_l, recv_l = [int(x) for x in send.tolist()], [int(x) for x in recv.tolist()]
    owned = coord.new_empty((sum(recv_l),) + tuple(coord.shape[1:]))
    dist.all_to_all_single(owned, coord[order].contiguous(), recv_l, send_l, group=group)
    return order, send_l, recv_l, owned


def route_values(values, order, send, recv, group=None):
    """Values of this rank's points (in its own order) to their owners, in the
    order ``route_points`` delivered the coordinates (collective)."""
    import torch
    import torch.distributed as dist
    src = torch.view_as_real(values[order].contiguous())
    dst = src.new_empty((sum(recv), 2))
    dist.all_to_all_single(dst, src, recv, send, group=group)
    return torch.view_as_complex(dst)


def route_back(res, order, send, recv, group=None):
    """Results at the owned points (in ``route_points``' delivery order) back
    to the ranks the points came from, in each rank's own point order
    (collective)."""
    import torch
    import torch.distributed as dist
    r = torch.view_as_real(res).contiguous()
    back = r.new_empty((sum(send), 2))
    dist.all_to_all_single(back, r, send, recv, group=group)
    out = torch.empty((sum(send),), dtype=res.dtype, device=res.device)
    out[order] = torch.view_as_complex(back)
    return out


def _rows_mod(a, b, n0, device):
    import torch
    return torch.remainder(torch.arange(a, b, device=device), n0)


def exchange_halos(grid, slabs, group=None):
    """Add the halo rows of every rank's spread grid to the rank that owns
    them (collective; nothing to do on one rank): rank k sends its HALO rows
    below its slab to rank k + 1 and the HALO rows above it to rank k - 1, and
    adds what it receives into the first and last HALO rows of its slab."""
    import torch
    import torch.distributed as dist
    world, rank = slabs.world, dist.get_rank(group)
    if world == 1:
        return grid
    H, n0 = slabs.HALO, slabs.n0
    s0, s1 = slabs.slab(rank)
    nxt, prv = (rank + 1) % world, (rank - 1) % world
    if group is not None:
        nxt, prv = dist.get_global_rank(group, nxt), dist.get_global_rank(group, prv)
    below = _rows_mod(s1, s1 + H, n0, grid.device)
    above = _rows_mod(s0 - H, s0, n0, grid.device)
    send_below = torch.view_as_real(grid.index_select(0, below)).contiguous()
    send_above = torch.view_as_real(grid.index_select(0, above)).contiguous()
    from_prev = torch.empty_like(send_below)   # rank k - 1's rows below its slab: my first H
    from_next = torch.empty_like(send_above)   # rank k + 1's rows above its slab: my last H
    ops = [dist.P2POp(dist.isend, send_below, nxt, group),
           dist.P2POp(dist.isend, send_above, prv, group),
           dist.P2POp(dist.irecv, from_prev, prv, group),
           dist.P2POp(dist.irecv, from_next, nxt, group)]
    for r in dist.batch_isend_irecv(ops):
        r.wait()
    grid[s0:s0 + H] += torch.view_as_complex(from_prev)
    grid[s1 - H:s1] += torch.view_as_complex(from_next)
    return grid


def transpose_kept_columns(packed, slabs, group=None):
    """Rows -> column blocks (collective): ``packed`` is this rank's slab of
    rows, kept columns packed ((slab rows, N1)); returns (n0, N1 / ranks): all
    rows of this rank's block of kept columns."""
    import torch
    import torch.distributed as dist
    world, rank = slabs.world, dist.get_rank(group)
    nr = packed.shape[0]
    src = torch.cat([torch.view_as_real(packed[:, a:b]).reshape(-1)
                     for a, b in (slabs.col_block(j) for j in range(world))])
    c0, c1 = slabs.col_block(rank)
    w = c1 - c0
    send = [nr * (b - a) * 2 for a, b in (slabs.col_block(j) for j in range(world))]
    recv = [(slabs.slab(k)[1] - slabs.slab(k)[0]) * w * 2 for k in range(world)]
    dst = src.new_empty(sum(recv))
    dist.all_to_all_single(dst, src, recv, send, group=group)
    return torch.view_as_complex(dst.reshape(slabs.n0, w, 2))


def gather_column_blocks(block, slabs, shift, group=None):
    """Every rank's (N0, width) block of uniform columns -> the whole (N0, N1)
    uniform array on every rank (collective): block j's column x is uniform
    column (col(j) + x + shift) mod N1."""
    import torch
    import torch.distributed as dist
    world = slabs.world
    wmax = max(b - a for a, b in (slabs.col_block(j) for j in range(world)))
    N0 = block.shape[0]
    pad = torch.zeros((N0, wmax), dtype=block.dtype, device=block.device)
    pad[:, :block.shape[1]] = block
    allb = torch.empty((world * N0, wmax, 2), dtype=torch.view_as_real(pad).dtype,
                       device=block.device)
    dist.all_gather_into_tensor(allb, torch.view_as_real(pad).contiguous(), group=group)
    allb = torch.view_as_complex(allb).reshape(world, N0, wmax)
    full = torch.cat([allb[j, :, :b - a] for j, (a, b) in
                      enumerate(slabs.col_block(j) for j in range(world))], dim=1)
    return torch.roll(full, shifts=int(shift), dims=1)


def type1_by_row_slabs(*, spread_into, rows_fft, cols_block, slabs, nover, nuni0, shift,
                       dtype, device, group=None):
    """The row-slab type 1 with the local steps passed in: ``spread_into(buf)``
    writes this rank's (owned) points' spread grid into ``buf`` ((n0, n1),
    C-contiguous), ``rows_fft(rows)`` transforms rows along axis 1 in place,
    ``cols_block(cols, col0)`` runs the column pass, correction and crop of a
    block of packed kept columns ((n0, width) -> (N0, width)).  Collective."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    n0, n1 = int(nover[0]), int(nover[1])
    grid = torch.empty((n0, n1), dtype=dtype, device=device)
    spread_into(grid)
    exchange_halos(grid, slabs, group)
    s0, s1 = slabs.slab(rank)
    if s1 > s0:
        rows_fft(grid[s0:s1])
    lo, hi = (slabs.nkept + 1) // 2, slabs.nkept // 2
    packed = torch.cat([grid[s0:s1, :lo], grid[s0:s1, n1 - hi:]], dim=1)
    block = transpose_kept_columns(packed, slabs, group).contiguous()
    c0, c1 = slabs.col_block(rank)
    if c1 > c0:
        ob = cols_block(block, c0)
    else:   # an empty column block (more ranks than kept columns)
        ob = torch.empty((int(nuni0), 0), dtype=dtype, device=device)
    return gather_column_blocks(ob, slabs, shift, group)


def columns_to_row_slabs(block, slabs, group=None):
    """Column blocks -> rows (collective), the inverse of
    ``transpose_kept_columns``: ``block`` is this rank's (n0, width) block of
    kept columns; returns (slab rows, N1): this rank's rows, kept columns
    packed."""
    import torch
    import torch.distributed as dist
    world, rank = slabs.world, dist.get_rank(group)
    c0, c1 = slabs.col_block(rank)
    w = c1 - c0
    src = torch.cat([torch.view_as_real(block[a:b]).reshape(-1)
                     for a, b in (slabs.slab(k) for k in range(world))])
    send = [(b - a) * w * 2 for a, b in (slabs.slab(k) for k in range(world))]
    s0, s1 = slabs.slab(rank)
    nr = s1 - s0
    recv = [nr * (b - a) * 2 for a, b in (slabs.col_block(j) for j in range(world))]
    dst = src.new_empty(sum(recv))
    dist.all_to_all_single(dst, src, recv, send, group=group)
    parts, off = [], 0
    for j in range(world):
        a, b = slabs.col_block(j)
        n = nr * (b - a) * 2
        parts.append(dst[off:off + n].reshape(nr, b - a, 2))
        off += n
    return torch.view_as_complex(torch.cat(parts, dim=1).contiguous())


def fill_halos(grid, slabs, group=None):
    """Copy the HALO rows on either side of this rank's slab from the ranks
    that own them (collective; nothing to do on one rank): the interpolation
    of the owned points reads them."""
    import torch
    import torch.distributed as dist
    world, rank = slabs.world, dist.get_rank(group)
    if world == 1:
        return grid
    H, n0 = slabs.HALO, slabs.n0
    s0, s1 = slabs.slab(rank)
    nxt, prv = (rank + 1) % world, (rank - 1) % world
    if group is not None:
        nxt, prv = dist.get_global_rank(group, nxt), dist.get_global_rank(group, prv)
    first = torch.view_as_real(grid[s0:s0 + H]).contiguous()   # rank k - 1's rows below it
    last = torch.view_as_real(grid[s1 - H:s1]).contiguous()    # rank k + 1's rows above it
    from_prev = torch.empty_like(last)
    from_next = torch.empty_like(first)
    ops = [dist.P2POp(dist.isend, first, prv, group),
           dist.P2POp(dist.isend, last, nxt, group),
           dist.P2POp(dist.irecv, from_next, nxt, group),
           dist.P2POp(dist.irecv, from_prev, prv, group)]
    for r in dist.batch_isend_irecv(ops):
        r.wait()
    grid.index_copy_(0, _rows_mod(s0 - H, s0, n0, grid.device), torch.view_as_complex(from_prev))
    grid.index_copy_(0, _rows_mod(s1, s1 + H, n0, grid.device), torch.view_as_complex(from_next))
    return grid


def type2_by_row_slabs(*, uniform_to_cols, rows_fft_kept_in, interp, slabs, nover, dtype,
                       device, group=None):
    """The row-slab type 2 with the local steps passed in: ``uniform_to_cols(
    col0, ncols)`` returns the column pass of a block of kept columns ((n0,
    ncols)), ``rows_fft_kept_in(rows)`` transforms rows whose kept columns
    are set into whole rows in place, ``interp(grid)`` interpolates this
    rank's owned points from a (n0, n1) grid whose slab and halo rows are set.
    Collective; returns the owned points' results."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    n0, n1 = int(nover[0]), int(nover[1])
    c0, c1 = slabs.col_block(rank)
    block = (uniform_to_cols(c0, c1 - c0) if c1 > c0
             else torch.empty((n0, 0), dtype=dtype, device=device))
    packed = columns_to_row_slabs(block, slabs, group)
    s0, s1 = slabs.slab(rank)
    lo, hi = (slabs.nkept + 1) // 2, slabs.nkept // 2
    grid = torch.zeros((n0, n1), dtype=dtype, device=device)
    grid[s0:s1, :lo] = packed[:, :lo]
    grid[s0:s1, n1 - hi:] = packed[:, lo:]
    if s1 > s0:
        rows_fft_kept_in(grid[s0:s1])
    fill_halos(grid, slabs, group)
    return interp(grid)


class ShardedPlan:
    """Plan of this rank's points of one transform split over the ranks of a
    process group.  Arguments as ``ducc_b200.nufft.plan``; ``coord`` holds only
    this rank's points, ``epsilon`` and ``grid_shape`` are those of the whole
    transform and must be the same on every rank.  Construction is collective
    (every rank of the group calls it, in the same order as the other
    collectives).

    ``partition``: "rows" (2D, several ranks, oversampled rows >= 1024: the
    default there) routes every point to the rank owning its oversampled row
    slab at construction and its value at every type 1; "points" keeps every
    point on its rank (the only choice in 1D / 3D)."""

    def __init__(self, *, nu2u, coord, grid_shape, epsilon, group=None, nthreads=0,
                 sigma_min=1.1, sigma_max=2.6, periodicity=2 * math.pi, fft_order=False,
                 spreader="auto", partition=None):
        import torch
        import torch.distributed as dist
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
        self.grid_shape = tuple(int(x) for x in grid_shape)
        self.npoints = coord.shape[0]
        self.device = coord.device
        self.fft_order = bool(fft_order)
        world = dist.get_world_size(group)
        if partition is None:
            partition = ("rows" if len(self.grid_shape) == 2 and world > 1 and nover[0] >= 1024
                         else "points")
        if partition not in ("rows", "points"):
            raise ValueError("partition must be 'rows' or 'points'")
        if partition == "rows" and len(self.grid_shape) != 2:
            raise ValueError("the row-slab partition is for 2D transforms")
        self.partition = partition
        owned = coord
        if partition == "rows":
            self.slabs = RowSlabs(nover[0], self.grid_shape[1], world)
            per = periodicity if not hasattr(periodicity, "__len__") else periodicity[0]
            owner = self.slabs.owner(row_estimate(coord[:, 0], nover[0], per))
            self.route = route_points(owner, coord, world, group)
            owned = self.route[3]
        self.plan = nufft.plan(nu2u=nu2u, coord=owned, grid_shape=grid_shape, epsilon=epsilon,
                               nthreads=nthreads, sigma_min=sigma_min, sigma_max=sigma_max,
                               periodicity=periodicity, fft_order=fft_order, spreader=spreader,
                               force_kernel=kidx, force_nover=nover)

    def nu2u(self, *, forward, points, out=None, exchange=None):
        """Type 1 of all ranks' points (collective); every rank gets the whole
        uniform grid in ``out``.  With the point partition, ``exchange``:
        'slabs' (the 2D default on several ranks: reduce-scatter of row slabs,
        row FFTs split over the ranks, all-gather of the kept columns) or
        'grid' (all-reduce of whole grids, any dimension; the default
        otherwise)."""
        import torch
        import torch.distributed as dist
        dtype = torch.complex128 if self.plan._f64 else torch.complex64
        if self.partition == "rows":
            order, send, recv, _ = self.route
            vals = route_values(points, order, send, recv, self.group)
            res = type1_by_row_slabs(
                spread_into=lambda buf: self.plan.spread(points=vals, out=buf),
                rows_fft=lambda rows: self.plan.rows_fft(forward=forward, rows=rows),
                cols_block=lambda cols, c0: self.plan.cols_to_uniform_range(
                    forward=forward, cols=cols, col0=c0),
                slabs=self.slabs, nover=self.nover, nuni0=self.grid_shape[0],
                shift=0 if self.fft_order else self.grid_shape[1] // 2, dtype=dtype,
                device=self.device, group=self.group)
            if out is None:
                return res
            out.copy_(res)
            return out
        if exchange is None:
            # one rank: nothing to exchange, and the grid path adds no copies
            multi = dist.get_world_size(self.group) > 1
            exchange = "slabs" if len(self.grid_shape) == 2 and multi else "grid"
        if exchange == "slabs":
            if len(self.grid_shape) != 2:
                raise ValueError("the slab exchange is for 2D transforms")
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
        """Type 2 at this rank's points from the whole uniform grid.  With the
        point partition nothing crosses between ranks.  With the row partition
        (collective) each rank runs the column pass of its block of kept
        columns, the blocks become row slabs (one all-to-all), each rank
        transforms its slab's rows, copies the halo rows from its neighbours,
        interpolates its owned points, and the results go back to the ranks
        the points came from."""
        if self.partition != "rows":
            return self.plan.u2nu(forward=forward, grid=grid, out=out)
        import torch
        order, send, recv, _ = self.route
        dtype = torch.complex128 if self.plan._f64 else torch.complex64
        owned = type2_by_row_slabs(
            uniform_to_cols=lambda c0, nc: self.plan.uniform_to_cols_range(
                forward=forward, grid=grid, col0=c0, ncols=nc),
            rows_fft_kept_in=lambda rows: self.plan.rows_fft_kept_in(forward=forward,
                                                                     rows=rows),
            interp=lambda g: self.plan.interp(grid=g),
            slabs=self.slabs, nover=self.nover, dtype=dtype, device=self.device,
            group=self.group)
        res = route_back(owned, order, send, recv, self.group)
        if out is None:
            return res
        out.copy_(res)
        return out


# ---------------------------------------------------------------- w-gridder
def plane_share(nplanes, world, rank):
    """(begin, count) of rank's w planes: consecutive, sizes differing by at
    most one."""
    base, extra = divmod(int(nplanes), int(world))
    begin = rank * base + min(rank, extra)
    return begin, base + (1 if rank < extra else 0)


def _split_wgridder(run, nplanes, group):
    """run((begin, count)) -> this rank's partial result (a torch tensor on the
    communicator's device, or a numpy array); the partials of all ranks are
    summed (one all-reduce) and every rank gets the sum, in run's type.  A
    rank without planes asks for the empty range past the last plane (count
    0 would mean all planes), which gives zeros."""
    import numpy as np
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    begin, count = plane_share(nplanes, world, rank)
    if count == 0:
        begin, count = nplanes, 1
    part = run((begin, count))
    dev = _count_device(group)
    t = part if (torch.is_tensor(part) and part.device == dev) else \
        torch.as_tensor(np.asarray(part) if not torch.is_tensor(part) else part).to(dev)
    dist.all_reduce(t, group=group)
    if torch.is_tensor(part):
        return t if t.device == part.device else t.to(part.device)
    return t.cpu().numpy()


def vis2dirty_split(group=None, _run=None, **kwargs):
    """``ducc_b200.wgridder.vis2dirty`` with its w planes split over the ranks
    of ``group`` (every rank passes the same arguments): each rank grids its
    consecutive share of the planes into a partial image, and one all-reduce
    sums them, so every rank returns the whole dirty image.  What crosses
    between GPUs is one image per rank.  Without w-stacking rank 0 does the
    work.  ``_run`` replaces the rank's computation (``_run(planes=...,
    **kwargs)``; tests on the CPU)."""
    from . import wgridder
    run = _run or wgridder.vis2dirty
    nplanes = 1
    if kwargs.get("do_wgridding"):
        q = {k: kwargs[k] for k in ("uvw", "freq", "vis", "wgt", "mask", "npix_x", "npix_y",
                                    "pixsize_x", "pixsize_y", "epsilon", "do_wgridding",
                                    "nthreads", "sigma_min", "sigma_max", "center_x",
                                    "center_y", "flip_u", "flip_v", "flip_w", "allow_nshift")
             if k in kwargs}
        nplanes = int(kwargs.pop("_nplanes", 0)) or wgridder.wgrid_params(**q)["nplanes"]
    kwargs.pop("_nplanes", None)
    return _split_wgridder(lambda pl: run(planes=pl, **kwargs), max(nplanes, 1), group)


def dirty2vis_split(group=None, _run=None, **kwargs):
    """``ducc_b200.wgridder.dirty2vis`` with its w planes split over the ranks
    of ``group`` (every rank passes the same arguments): each rank degrids its
    share of the planes and one all-reduce sums the visibilities."""
    from . import wgridder
    run = _run or wgridder.dirty2vis
    nplanes = 1
    if kwargs.get("do_wgridding"):
        q = {k: kwargs[k] for k in ("uvw", "freq", "wgt", "mask", "pixsize_x", "pixsize_y",
                                    "epsilon", "do_wgridding", "nthreads", "sigma_min",
                                    "sigma_max", "center_x", "center_y", "flip_u", "flip_v",
                                    "flip_w", "allow_nshift")
             if k in kwargs}
        d = kwargs["dirty"]
        nplanes = int(kwargs.pop("_nplanes", 0)) or wgridder.wgrid_params(
            npix_x=d.shape[0], npix_y=d.shape[1], **q)["nplanes"]
    kwargs.pop("_nplanes", None)
    return _split_wgridder(lambda pl: run(planes=pl, **kwargs), max(nplanes, 1), group)


def _point_share(npts, group):
    """This rank's consecutive share [a, b) of npts points."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    b0, c = plane_share(npts, world, rank)
    return b0, b0 + c, world


def _to_comm(x, dev):
    import numpy as np
    import torch
    return x.to(dev) if torch.is_tensor(x) else torch.as_tensor(np.asarray(x)).to(dev)


def synthesis_general_split(group=None, _run=None, **kwargs):
    """``ducc_b200.sht.synthesis_general`` with the points split over the ranks
    of ``group`` (every rank passes the same arguments): each rank evaluates
    the expansion at its consecutive share of ``loc`` and one all-gather
    assembles the map on every rank.  The rings (Legendre part) are computed by
    every rank; what crosses between GPUs is the map.  ``_run`` replaces the
    rank's computation (``_run(loc=share, **kwargs)``; tests on the CPU)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    from . import sht
    run = _run or sht.synthesis_general
    loc = kwargs.pop("loc")
    npts = int(loc.shape[0])
    a, b, world = _point_share(npts, group)
    part = run(loc=loc[a:b], **kwargs)
    dev = _count_device(group)
    t = _to_comm(part, dev)
    # every share padded to the largest one for the all-gather
    width = (npts + world - 1) // world
    buf = torch.zeros((t.shape[0], width), dtype=t.dtype, device=dev)
    buf[:, :t.shape[1]] = t
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    pieces = []
    for r in range(world):
        ra, rb = plane_share(npts, world, r)[0], sum(plane_share(npts, world, r))
        pieces.append(parts[r][:, :rb - ra])
    full = torch.cat(pieces, dim=1)
    if torch.is_tensor(part):
        return full.to(part.device)
    return full.cpu().numpy()


def adjoint_synthesis_general_split(group=None, _run=None, **kwargs):
    """``ducc_b200.sht.adjoint_synthesis_general`` with the points split over
    the ranks of ``group`` (every rank passes the same arguments): each rank
    takes its consecutive share of ``loc`` and of the map's columns, and one
    all-reduce sums the partial a_lm (the adjoint is a sum over the points).
    ``_run`` replaces the rank's computation (tests on the CPU)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    from . import sht
    run = _run or sht.adjoint_synthesis_general
    loc = kwargs.pop("loc")
    mp = kwargs.pop("map")
    npts = int(loc.shape[0])
    a, b, _ = _point_share(npts, group)
    part = run(loc=loc[a:b], map=mp[:, a:b], **kwargs)
    dev = _count_device(group)
    t = _to_comm(part, dev)
    dist.all_reduce(t, group=group)
    if torch.is_tensor(part):
        return t if t.device == part.device else t.to(part.device)
    return t.cpu().numpy()

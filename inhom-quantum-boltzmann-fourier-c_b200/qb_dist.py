"""Multi-rank Strang step: x-cells sharded over ranks, 2-cell halos exchanged.

Upstream distributes contiguous blocks of x-cells over MPI ranks
(src/main_inhom.c:350-351) and swaps two boundary cells with each neighbour
before each half step of transport (src/simulation.c:341-384, 457-484); the
transport is then run on the haloed line (numVol + 4 cells) and the interior
kept.  Here one process drives one GPU, the halos travel through
torch.distributed (NCCL over NVLink on GPUs, gloo on CPU for tests), and the
collision stays cell-local.  The transport and collision callables are
injected so the same host logic runs with the CUDA kernels (bench) and with
the CPU oracle (tests).

`ShardedStrang` keeps the haloed lines [2 | local | 2] preallocated and
overlaps the second halo exchange with the collision: the two edge cells on
each side collide first, their halo messages are posted, and the interior
cells collide while the messages travel.  Every rank posts the same
operations in the same order in every step.
"""
import torch
import torch.distributed as dist


def partition(ncells_total, world, rank):
    """upstream src/main_inhom.c:350-351: [n*rank/world, n*(rank+1)/world)"""
    i0 = ncells_total * rank // world
    i1 = ncells_total * (rank + 1) // world
    return i0, i1


def _halo_ops(ext, n, group):
    """batched point-to-point operations that fill the halos of the haloed
    line `ext` ([2 | n local | 2], dim 0 = cells) on the periodic ring: the
    left halo receives the left neighbour's last two cells, the right halo
    the right neighbour's first two.  The same op order on every rank keeps
    the pairing unambiguous even when left == right (two ranks)."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    left, right = (rank - 1) % world, (rank + 1) % world
    return [dist.P2POp(dist.isend, ext[n:n + 2], right, group),          # my last cells -> right neighbour's left halo
            dist.P2POp(dist.irecv, ext[0:2], left, group),
            dist.P2POp(dist.isend, ext[2:4], left, group),                # my first cells -> left neighbour's right halo
            dist.P2POp(dist.irecv, ext[n + 2:n + 4], right, group)]


def _start_halos(ext, n, group):
    """post the halo exchange of `ext`; returns the requests (none on one rank,
    where the halos wrap around locally)"""
    if dist.get_world_size(group) == 1:
        ext[0:2].copy_(ext[n:n + 2])
        ext[n + 2:n + 4].copy_(ext[2:4])
        return []
    return dist.batch_isend_irecv(_halo_ops(ext, n, group))


def halo_exchange(W, group=None):
    """Return (left halo, right halo): the last two cells of the left neighbour
    and the first two cells of the right neighbour on the periodic ring."""
    if W.shape[0] < 2:
        raise ValueError("every rank needs at least two cells (upstream src/simulation.c:317)")
    n = W.shape[0]
    ext = torch.empty((n + 4,) + tuple(W.shape[1:]), dtype=W.dtype, device=W.device)
    ext[2:n + 2].copy_(W)
    for r in _start_halos(ext, n, group):
        r.wait()
    return ext[0:2].clone(), ext[n + 2:n + 4].clone()


class ShardedStrang:
    """InhomStepPeriodic (upstream src/simulation.c:307-555) on this rank's n
    cells of a sharded periodic domain: 1/2 transport, cell-local collision,
    1/2 transport.

    transport(ext, out): one limiter half step on the haloed line `ext`
    (n + 4 cells, periodic within itself) into `out` (same shape); only the
    local cells out[2:n + 2] are kept, their 5-point stencils never reach the
    wrapped ends.  collision(cells, start): the collision part in place on a
    block of consecutive cells (a view along dim 0) whose first cell is local
    cell `start` (for per-cell fields)."""

    def __init__(self, n, cell_shape, dtype, device, transport, collision, group=None):
        if n < 2:
            raise ValueError("every rank needs at least two cells (upstream src/simulation.c:317)")
        self.n, self.transport, self.collision, self.group = n, transport, collision, group
        shape = (n + 4,) + tuple(cell_shape)
        self.ext_a = torch.empty(shape, dtype=dtype, device=device)   # haloed line before a half step
        self.ext_b = torch.empty(shape, dtype=dtype, device=device)   # after it

    def step(self, W, out=None):
        n = self.n
        a, b = self.ext_a, self.ext_b
        a[2:n + 2].copy_(W)
        for r in _start_halos(a, n, self.group):
            r.wait()
        self.transport(a, b)
        cells = b[2:n + 2]
        # the edge cells collide first; their halos travel while the interior collides
        if n >= 6:
            self.collision(cells[:2], 0)
            self.collision(cells[n - 2:], n - 2)
            reqs = _start_halos(b, n, self.group)
            self.collision(cells[2:n - 2], 2)
        else:
            self.collision(cells, 0)
            reqs = _start_halos(b, n, self.group)
        for r in reqs:
            r.wait()
        self.transport(b, a)
        if out is None:
            return a[2:n + 2].clone()
        out.copy_(a[2:n + 2])
        return out


def transport_with_halo(W, transport, group=None):
    """One half step of periodic transport on this rank's cells: the limiter
    runs on [2 halo | local | 2 halo] and the local cells are kept."""
    hl, hr = halo_exchange(W, group)
    ext = torch.cat([hl, W, hr], dim=0).contiguous()
    out = transport(ext)
    return out[2:2 + W.shape[0]].contiguous()


def sharded_strang_step(W, transport, collision, group=None):
    """One Strang step without preallocated buffers or overlap (the reference
    form of ShardedStrang.step): transport(ext) returns the half-stepped
    haloed line, collision(cells) returns the collided cells."""
    Wt = transport_with_halo(W, transport, group)
    Wt = collision(Wt)
    return transport_with_halo(Wt, transport, group)

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
"""
import torch
import torch.distributed as dist


def partition(ncells_total, world, rank):
    """upstream src/main_inhom.c:350-351: [n*rank/world, n*(rank+1)/world)"""
    i0 = ncells_total * rank // world
    i1 = ncells_total * (rank + 1) // world
    return i0, i1


def halo_exchange(W, group=None):
    """Return (left halo, right halo): the last two cells of the left neighbour
    and the first two cells of the right neighbour on the periodic ring."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if W.shape[0] < 2:
        raise ValueError("every rank needs at least two cells (upstream src/simulation.c:317)")
    if world == 1:
        return W[-2:].clone(), W[:2].clone()
    left, right = (rank - 1) % world, (rank + 1) % world
    recv_left = torch.empty_like(W[:2])
    recv_right = torch.empty_like(W[:2])
    send_right = W[-2:].contiguous()      # my last cells are my right neighbour's left halo
    send_left = W[:2].contiguous()        # my first cells are my left neighbour's right halo
    # the same op order on every rank keeps the pairing unambiguous even when
    # left == right (two ranks)
    ops = [dist.P2POp(dist.isend, send_right, right, group),
           dist.P2POp(dist.irecv, recv_left, left, group),
           dist.P2POp(dist.isend, send_left, left, group),
           dist.P2POp(dist.irecv, recv_right, right, group)]
    for r in dist.batch_isend_irecv(ops):
        r.wait()
    return recv_left, recv_right


def transport_with_halo(W, transport, group=None):
    """One half step of periodic transport on this rank's cells: the limiter
    runs on [2 halo | local | 2 halo] and the local cells are kept (their
    5-point stencils never reach the wrapped ends)."""
    hl, hr = halo_exchange(W, group)
    ext = torch.cat([hl, W, hr], dim=0).contiguous()
    out = transport(ext)
    return out[2:2 + W.shape[0]].contiguous()


def sharded_strang_step(W, transport, collision, group=None):
    """InhomStepPeriodic (upstream src/simulation.c:307-555) on a sharded domain:
    1/2 transport, cell-local collision, 1/2 transport."""
    Wt = transport_with_halo(W, transport, group)
    Wt = collision(Wt)
    return transport_with_halo(Wt, transport, group)

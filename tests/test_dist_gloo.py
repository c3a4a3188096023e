"""Sharded Strang step on 2 and 3 ranks (gloo, CPU) against the single-domain oracle.

The host logic of the multi-GPU path (partitioning, 2-cell halo exchange on
the periodic ring, transport on the haloed block, cell-local collision) runs
here with the oracle's transport and collision as the callables; the gathered
result must equal the oracle's InhomStepPeriodic on the whole domain bit for
bit, because every cell sees the same neighbours and the same arithmetic.
Both forms run: `sharded_strang_step` and `ShardedStrang` (preallocated
haloed lines; edge cells collide first and their halos travel while the
interior collides; ranks of 6 or more cells take that overlapped path).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import PKG, REPO

N, J, M, L, R = 8, 2, 2, 6.0, 3.75


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, W, h, dt, out_path, form):
    import sys
    sys.path[:0] = [PKG, os.path.join(REPO, "oracle")]
    import orc
    import qb_dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    o = orc.Oracle(N, J, M, L, R)
    vg = np.where(np.arange(N) < N // 2, np.arange(N), np.arange(N) - N) * (2 * L / N)

    def transport_into(ext, out):
        a, o_ = ext.numpy(), out.numpy()
        for c in range(4):
            for l in range(N):
                for k in range(N):
                    o_[:, c, l, k] = orc.slope_periodic(h, 0.5 * dt, vg[l], a[:, c, l, k])
        return out

    def collide_in_place(cells, start=0):
        a = cells.numpy()
        for i in range(a.shape[0]):
            wf = orc.to_fourier(a[i])
            a[i] = orc.from_fourier(o.collision_step(wf, dt))
        return cells

    ncells = W.shape[0]
    i0, i1 = qb_dist.partition(ncells, world, rank)
    mine = torch.from_numpy(W[i0:i1].copy())
    if form == "overlapped":
        out = qb_dist.ShardedStrang(i1 - i0, (4, N, N), torch.float64, "cpu", transport_into, collide_in_place).step(mine)
    else:
        out = qb_dist.sharded_strang_step(mine, lambda e: transport_into(e, torch.empty_like(e)), collide_in_place)
    parts = [None] * world
    dist.all_gather_object(parts, (i0, out.numpy()))
    if rank == 0:
        full = np.zeros_like(W)
        for a, blk in parts:
            full[a:a + blk.shape[0]] = blk
        np.save(out_path, full)
    dist.barrier()
    dist.destroy_process_group()


# (ranks, cells): 7 cells split 3 + 4; 20 cells split 6 + 7 + 7 (every rank on the overlapped path)
@pytest.mark.parametrize("world,ncells,form", [(2, 7, "plain"), (2, 7, "overlapped"), (3, 20, "overlapped")])
def test_sharded_step_matches_single_domain(tmp_path, world, ncells, form):
    import sys
    sys.path[:0] = [PKG]
    import orc
    import qbgpu
    W = qbgpu.gaussian_mixture_state(N, L, seed=41, ncells=ncells)
    h = 1.0 / ncells
    dt = 0.4 * h / L
    out_path = str(tmp_path / "sharded.npy")
    mp.start_processes(_worker, args=(world, _free_port(), W, h, dt, out_path, form), nprocs=world, join=True, start_method="spawn")
    sharded = np.load(out_path)
    ref = orc.Oracle(N, J, M, L, R).inhom_step(W, h, dt)
    assert np.array_equal(sharded, ref)


def test_partition_covers_domain():
    import sys
    sys.path[:0] = [PKG]
    import qb_dist
    for n, w in ((64, 8), (7, 2), (10, 3)):
        blocks = [qb_dist.partition(n, w, r) for r in range(w)]
        assert blocks[0][0] == 0 and blocks[-1][1] == n
        assert all(blocks[r][1] == blocks[r + 1][0] for r in range(w - 1))
        assert all(b - a >= 2 for a, b in blocks)

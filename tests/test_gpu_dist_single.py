"""GPU: the sharded Strang step of bench.py's multi-GPU path, driven by the
same qbgpu calls (qb_transport, qb_fourier_collision) on one rank of a
gloo process group, against the single-domain step (qb_inhom_step)."""
import socket

import numpy as np
import pytest

import qb_dist
import qbgpu
from conftest import rel_l1

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_step_with_the_library_calls_matches_inhom_step():
    import torch.distributed as dist
    N, J, M, L, R = 16, 4, 3, 6.0, 3.75
    q, ws = qbgpu.Quad(N, J, M, L, R), qbgpu.Workspace(N)
    ncells = 6
    W = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=61, ncells=ncells)).cuda()
    B = torch.from_numpy(np.random.default_rng(4).standard_normal((ncells, 3)) * 0.05).cuda()
    h, dt = 1.0 / ncells, 0.4 / ncells / L
    ref = qbgpu.inhom_step(ws, q, W, h, dt, B).cpu().numpy()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{free_port()}", rank=0, world_size=1)
    try:
        out = qb_dist.sharded_strang_step(W, lambda e: qbgpu.transport(e, L, h, 0.5 * dt),
                                          lambda Wt: qbgpu.fourier_collision(ws, q, Wt, dt, B))
        ov = qb_dist.ShardedStrang(ncells, (4, N, N), torch.float64, W.device,
                                   lambda e, o: qbgpu.transport(e, L, h, 0.5 * dt, out=o),
                                   lambda c, i: qbgpu.fourier_collision(ws, q, c, dt, B[i:i + c.shape[0]]))
        out2 = ov.step(W)
        out3 = ov.step(W)                       # the preallocated lines are reused
    finally:
        dist.destroy_process_group()
    assert rel_l1(out.cpu().numpy(), ref) < 1e-14
    # edge cells and interior collide in separate launches (overlapped form): same arithmetic per cell
    assert rel_l1(out2.cpu().numpy(), ref) < 1e-14
    assert torch.equal(out2, out3)


@pytest.mark.parametrize("ncells", [8, 4])
def test_c_abi_sharded_step_with_exchange_callback(ncells):
    """qb_sharded_step (the C-ABI form of the sharded step, for hosts that
    exchange halos themselves) with a one-rank exchange callback (the periodic
    wrap, on the caller's stream): equal to qb_inhom_step; 8 cells take the
    overlapped path (edge cells first, interior on the workspace stream), 4
    the plain one"""
    import ctypes as C
    N, J, M, L, R = 16, 4, 3, 6.0, 3.75
    q, ws = qbgpu.Quad(N, J, M, L, R), qbgpu.Workspace(N)
    W = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=62, ncells=ncells)).cuda()
    B = torch.from_numpy(np.random.default_rng(5).standard_normal((ncells, 3)) * 0.05).cuda()
    h, dt = 1.0 / ncells, 0.4 / ncells / L
    ref = qbgpu.inhom_step(ws, q, W, h, dt, B).cpu().numpy()
    ext = {k: torch.zeros((ncells + 4, 4, N, N), dtype=torch.float64, device="cuda") for k in "ab"}
    ext["a"][2:ncells + 2].copy_(W)
    by_ptr = {t.data_ptr(): t for t in ext.values()}
    calls = []

    def exchange(ptr, n, stream, user):
        t = by_ptr[ptr]
        t[0:2].copy_(t[n:n + 2])
        t[n + 2:n + 4].copy_(t[2:4])
        calls.append(ptr)
        return 0
    cb = qbgpu.HALO_FN(exchange)
    ws2 = qbgpu.Workspace(N)
    rc = qbgpu.lib().qb_sharded_step(ws2.h, q.h, ncells, ext["a"].data_ptr(), ext["b"].data_ptr(), h, dt, qbgpu._ptr(B),
                                    cb, None, qbgpu._stream())
    assert rc == 0, qbgpu.lib().qb_last_error().decode()
    torch.cuda.synchronize()
    assert calls == [ext["a"].data_ptr(), ext["b"].data_ptr()]
    assert rel_l1(ext["a"][2:ncells + 2].cpu().numpy(), ref) < 1e-14

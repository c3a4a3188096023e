"""GPU: trajectory recording, diagnostics and CUDA-graph replay of the step."""
import os

import numpy as np
import pytest

import orc
import qbgpu
from conftest import rel_l1

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N, J, M, L, R = 16, 4, 3, 6.0, 3.75


@pytest.fixture(scope="module")
def env():
    return qbgpu.Quad(N, J, M, L, R), qbgpu.Workspace(N), orc.Oracle(N, J, M, L, R)


def test_diagnostics_match_numpy_restatement():
    W = qbgpu.gaussian_mixture_state(32, L, seed=51, ncells=5)
    W[2, 1] += 0.7 * W[2, 0]          # push eigenvalues outside (0, 1) somewhere
    out = qbgpu.diagnostics(torch.from_numpy(W).cuda(), L).cpu().numpy()
    ref = orc.diagnostics(W, L)
    assert np.allclose(out, ref, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("every", [1, 3])
def test_recorded_trajectory_matches_repeated_oracle_steps(env, tmp_path, every):
    q, ws, o = env
    W0 = qbgpu.gaussian_mixture_state(N, L, seed=52, ncells=6)
    B = np.random.default_rng(8).standard_normal((6, 3)) * 0.05
    h, dt, steps = 1 / 6, 0.4 / 6 / L, 7
    path = str(tmp_path / "traj.dat")
    final, frames = qbgpu.simulate_record(ws, q, W0, h, dt, steps, B, record_every=every, path=path)
    traj = np.fromfile(path).reshape(-1, 6, 4, N, N)
    expect_idx = [i for i in range(steps) if i % every == 0]
    assert frames == len(expect_idx) == traj.shape[0]
    ref = [W0]
    for _ in range(steps - 1):
        ref.append(o.inhom_step(ref[-1], h, dt, B))
    assert np.array_equal(traj[0], W0)
    for k, i in enumerate(expect_idx[1:], start=1):
        assert rel_l1(traj[k], ref[i]) < 1e-12
    assert rel_l1(final, ref[-1]) < 1e-12


def test_graph_replay_equals_direct_launches(env, monkeypatch):
    q, ws, _ = env
    W = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=53, ncells=4)).cuda()
    B = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    h, dt = 0.25, 0.01
    out = torch.empty_like(W)
    results = []
    for _ in range(4):                       # direct, capture+replay, replay, replay
        qbgpu.inhom_step(ws, q, W, h, dt, B, out=out)
        torch.cuda.synchronize()
        results.append(out.clone())
    for r in results[1:]:
        assert torch.equal(r, results[0])
    monkeypatch.setenv("QB_CUDA_GRAPHS", "0")
    ws2 = qbgpu.Workspace(N)
    direct = qbgpu.inhom_step(ws2, q, W, h, dt, B)
    torch.cuda.synchronize()
    assert torch.equal(direct, results[0])


def test_alternating_buffers_replay_their_graphs(env):
    """Steps that alternate two state buffers (A -> B, B -> A, ...) keep one
    graph per direction: from the third step of each direction on, every
    step is a graph replay, its kernels are counted, and the trajectory is
    bit-identical to kernel-by-kernel launches."""
    q, _, _ = env
    L_ = qbgpu.lib()
    ws = qbgpu.Workspace(N)
    W = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=54, ncells=4)).cuda()
    B = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    h, dt = 0.25, 0.01
    bufs = [W.clone(), torch.empty_like(W)]
    steps = 10
    counts = []
    for k in range(steps):
        c0 = L_.qb_launch_count()
        qbgpu.inhom_step(ws, q, bufs[k % 2], h, dt, B, out=bufs[(k + 1) % 2])
        counts.append(L_.qb_launch_count() - c0)
    torch.cuda.synchronize()
    # calls 0, 1 run directly (one per key), 2, 3 capture, 4.. replay
    assert ws.graph_replays == steps - 4
    assert len(set(counts)) == 1 and counts[0] > 0      # replays count the graph's kernel nodes
    ref = W.clone()
    wsd = qbgpu.Workspace(N)
    L_.qb_profile_enable(1)                             # profiling on: kernel-by-kernel launches
    try:
        for k in range(steps):
            ref = qbgpu.inhom_step(wsd, q, ref, h, dt, B)
        torch.cuda.synchronize()
    finally:
        L_.qb_profile_enable(0)
        L_.qb_profile_reset()
    assert wsd.graph_replays == 0
    assert torch.equal(bufs[steps % 2], ref)

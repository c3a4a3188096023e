"""GPU: homogeneous collision steps for a batch of instances of different grid
sizes (one batched launch sequence per size) against the oracle's
CollisionStep / RK4 per instance."""
import numpy as np
import pytest

import orc
import qbgpu
from conftest import rel_l1

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

J, M, L, R = 4, 3, 6.0, 3.75
TOL = 1e-12


@pytest.mark.parametrize("rk4", [True, False])
def test_mixed_size_batch_matches_oracle(rk4):
    sizes = [8, 16, 8, 32, 16, 8]
    rng = np.random.default_rng(11)
    Wf = [orc.to_fourier(qbgpu.gaussian_mixture_state(n, L, seed=100 + i, ncells=1))[0] for i, n in enumerate(sizes)]
    B = rng.standard_normal((len(sizes), 3)) * 0.1
    states = [torch.from_numpy(w.copy()).cuda() for w in Wf]
    dt, steps = 0.01, 2
    qbgpu.homogeneous_batch(states, dt, steps, B=B, rk4=rk4, J=J, M=M, L=L, R=R)
    oracles = {n: orc.Oracle(n, J, M, L, R) for n in set(sizes)}
    for i, n in enumerate(sizes):
        ref = Wf[i]
        for _ in range(steps):
            ref = oracles[n].collision_step(ref, dt, B[i], rk4=rk4)
        assert rel_l1(states[i].cpu().numpy(), ref) < TOL, (i, n)


def test_batch_rejects_unsupported_size():
    """N = 20 (2N = 40 has the factor 5: neither a fixed-size nor an any-N size)"""
    bad = [torch.zeros((4, 20, 20), dtype=torch.complex128, device="cuda")]
    with pytest.raises(RuntimeError, match="N=20"):
        qbgpu.homogeneous_batch(bad, 0.01, 1, J=J, M=M, L=L, R=R)


def test_fp32_batch_tracks_fp64_batch():
    """the FP32 form of the mixed-size batch (N = 8, 16, 32 and 64, the last
    through the whole-grid FP32 I3 kernel) within the 1e-5 bound of the FP64 one"""
    sizes = [8, 16, 32, 64, 16, 32]
    Wf = [orc.to_fourier(qbgpu.gaussian_mixture_state(n, L, seed=300 + i, ncells=1))[0] for i, n in enumerate(sizes)]
    B = np.random.default_rng(12).standard_normal((len(sizes), 3)) * 0.1
    out = {}
    for prec in (64, 32):
        states = [torch.from_numpy(w.copy()).cuda() for w in Wf]
        qbgpu.homogeneous_batch(states, 0.01, 2, B=B, rk4=True, J=J, M=M, L=L, R=R, precision=prec)
        out[prec] = [s.cpu().numpy() for s in states]
    for i in range(len(sizes)):
        a, b = out[32][i], out[64][i]
        e = float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
        assert 0 < e <= 1e-5, (sizes[i], e)
    with pytest.raises(RuntimeError):
        qbgpu.homogeneous_batch([torch.from_numpy(Wf[0].copy()).cuda()], 0.01, 1, precision=16)


def test_batch_graph_replay_and_tuned_schedules(monkeypatch):
    """a batch call of 7 steps: the groups' schedules are tuned on the first
    call, two direct steps size the buffers, then two-step CUDA graphs of all
    groups (each size on its own stream) are replayed; the result equals the
    same call with direct launches bit for bit, and the oracle within 1e-12"""
    sizes = [16, 8, 16, 32, 8]
    rng = np.random.default_rng(21)
    Wf = [orc.to_fourier(qbgpu.gaussian_mixture_state(n, L, seed=500 + i, ncells=1))[0] for i, n in enumerate(sizes)]
    B = rng.standard_normal((len(sizes), 3)) * 0.1
    dt, steps = 0.01, 7
    graphed = [torch.from_numpy(w.copy()).cuda() for w in Wf]
    qbgpu.homogeneous_batch(graphed, dt, steps, B=B, rk4=True, J=J, M=M, L=L, R=R)
    monkeypatch.setenv("QB_CUDA_GRAPHS", "0")
    direct = [torch.from_numpy(w.copy()).cuda() for w in Wf]
    qbgpu.homogeneous_batch(direct, dt, steps, B=B, rk4=True, J=J, M=M, L=L, R=R)
    torch.cuda.synchronize()
    for a, b in zip(graphed, direct):
        assert torch.equal(a, b)
    oracles = {n: orc.Oracle(n, J, M, L, R) for n in set(sizes)}
    for i, n in enumerate(sizes):
        ref = Wf[i]
        for _ in range(steps):
            ref = oracles[n].collision_step(ref, dt, B[i], rk4=True)
        assert rel_l1(graphed[i].cpu().numpy(), ref) < TOL, (i, n)
    tuned = [s for s in qbgpu.batch_schedules() if s["J"] == J and s["M"] == M and s["rk4"] == 1]
    assert {(s["N"], s["instances"]) for s in tuned} >= {(8, 2), (16, 2), (32, 1)}
    assert all(s["step_ms"] > 0 for s in tuned)


def test_fp32_any_n_batch_graph_replay_and_fp64_bound(monkeypatch):
    """the any-N sizes of the configuration (N = 24, 48, 96, 128) in the FP32
    form: a 7-step batch call replays its two-step CUDA graphs (the per-cell
    choice between the real and the complex form of the I3 sums is made on
    the device inside the graph) bit for bit like direct launches, and stays
    within the 1e-5 bound of the FP64 batch"""
    sizes = [24, 96, 48, 128, 24]
    Wf = [orc.to_fourier(qbgpu.gaussian_mixture_state(n, L, seed=700 + i, ncells=1))[0] for i, n in enumerate(sizes)]
    B = np.random.default_rng(27).standard_normal((len(sizes), 3)) * 0.1
    dt, steps = 0.01, 7
    graphed = [torch.from_numpy(w.copy()).cuda() for w in Wf]
    qbgpu.homogeneous_batch(graphed, dt, steps, B=B, rk4=True, J=J, M=M, L=L, R=R, precision=32)
    fp64 = [torch.from_numpy(w.copy()).cuda() for w in Wf]
    qbgpu.homogeneous_batch(fp64, dt, steps, B=B, rk4=True, J=J, M=M, L=L, R=R, precision=64)
    monkeypatch.setenv("QB_CUDA_GRAPHS", "0")
    direct = [torch.from_numpy(w.copy()).cuda() for w in Wf]
    qbgpu.homogeneous_batch(direct, dt, steps, B=B, rk4=True, J=J, M=M, L=L, R=R, precision=32)
    torch.cuda.synchronize()
    for a, b in zip(graphed, direct):
        assert torch.equal(a, b)
    for i, n in enumerate(sizes):
        a, b = graphed[i].cpu().numpy(), fp64[i].cpu().numpy()
        e = float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
        assert 0 < e <= 1e-5, (n, e)

"""The any-N engine (grid sizes without fixed-size kernels: N = 24, 48, 96 with
radix-3 transforms, N = 128 with 256 x 256 padded grids) against the oracle,
which restates upstream with N as a run-time parameter and a mixed-radix
(2, 3) FFT.  FP64 within 1e-12 relative L1, the FP32 form within 1e-5.
QB_ANYN=1 routes the fixed sizes through the same engine: a cross-check of the
two engines on identical inputs."""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "inhom-quantum-boltzmann-fourier-c_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

pytestmark = pytest.mark.gpu

L, R = 6.0, 3.75


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


@pytest.fixture(scope="module")
def mods():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    import qbgpu
    import orc
    return torch, qbgpu, orc


def _states(qbgpu, orc, N, ncells, seed):
    Wv = qbgpu.gaussian_mixture_state(N, L, seed=seed, ncells=ncells)
    return Wv, orc.to_fourier(Wv)


@pytest.mark.parametrize("N,J,M", [(24, 4, 3), (48, 4, 2), (12, 2, 3)])
def test_operators_fp64_vs_oracle(mods, N, J, M):
    torch, qbgpu, orc = mods
    ws, q = qbgpu.Workspace(N), qbgpu.Quad(N, J, M, L, R)
    o = orc.Oracle(N, J, M, L, R)
    _, WF = _states(qbgpu, orc, N, 3, 70 + N)
    cc, cd = qbgpu.collision_operators(ws, q, torch.from_numpy(WF).cuda())
    cc, cd = cc.cpu().numpy(), cd.cpu().numpy()
    for i in range(3):
        assert rel_l1(cc[i], o.cc(WF[i])) < 1e-12
        assert rel_l1(cd[i], o.cd(WF[i])) < 1e-12


@pytest.mark.parametrize("N,J,M", [(24, 4, 3), (96, 2, 2)])
def test_operators_fp32_vs_oracle(mods, N, J, M):
    torch, qbgpu, orc = mods
    ws, q = qbgpu.Workspace(N, precision=32), qbgpu.Quad(N, J, M, L, R)
    o = orc.Oracle(N, J, M, L, R)
    _, WF = _states(qbgpu, orc, N, 2, 90 + N)
    cc, cd = qbgpu.collision_operators(ws, q, torch.from_numpy(WF).cuda())
    cc, cd = cc.cpu().numpy(), cd.cpu().numpy()
    for i in range(2):
        assert rel_l1(cc[i], o.cc(WF[i])) < 1e-5
        assert rel_l1(cd[i], o.cd(WF[i])) < 1e-5


@pytest.mark.parametrize("prec,fused", [(32, "1"), (32, "0"), (64, "1")])
def test_i3_chain_paths_vs_oracle(mods, prec, fused):
    """The two I3 chain paths at N = 24: whole-grid chains (QB_ANYN_FUSED=1)
    and three global passes (QB_ANYN_FUSED=0, the default), on two smooth
    cells and one noisy cell: in FP32 the smooth cells take the real form and
    the noisy one the complex form, all within 1e-5 of the oracle; FP64
    within 1e-12."""
    torch, qbgpu, orc = mods
    N, J, M = 24, 4, 3
    ws, q = qbgpu.Workspace(N, precision=prec), qbgpu.Quad(N, J, M, L, R)
    o = orc.Oracle(N, J, M, L, R)
    Wv = qbgpu.gaussian_mixture_state(N, L, seed=124, ncells=3)
    Wv[2] += 1e-3 * np.random.default_rng(24).standard_normal(Wv[2].shape)
    WF = orc.to_fourier(Wv)
    old = os.environ.get("QB_ANYN_FUSED")
    os.environ["QB_ANYN_FUSED"] = fused
    try:
        cc, cd = qbgpu.collision_operators(ws, q, torch.from_numpy(WF).cuda())
    finally:
        if old is None:
            del os.environ["QB_ANYN_FUSED"]
        else:
            os.environ["QB_ANYN_FUSED"] = old
    # Nyquist fraction of the smooth cells: 2.3e-7 (bound 1e-6)
    assert ws.i3_forms() == ((2, 3) if prec == 32 else (0, 0))
    tol = 1e-5 if prec == 32 else 1e-12
    cc, cd = cc.cpu().numpy(), cd.cpu().numpy()
    for i in range(3):
        assert rel_l1(cc[i], o.cc(WF[i])) < tol
        assert rel_l1(cd[i], o.cd(WF[i])) < tol


def test_n128_fp64_collision_step_vs_oracle(mods):
    torch, qbgpu, orc = mods
    N, J, M = 128, 2, 2
    ws, q = qbgpu.Workspace(N), qbgpu.Quad(N, J, M, L, R)
    o = orc.Oracle(N, J, M, L, R)
    _, WF = _states(qbgpu, orc, N, 1, 128)
    B = np.array([[0.2, -0.1, 0.3]])
    out = qbgpu.collision_step(ws, q, torch.from_numpy(WF).cuda(), 0.01, torch.from_numpy(B).cuda(), rk4=True).cpu().numpy()
    assert rel_l1(out[0], o.collision_step(WF[0], 0.01, B[0], rk4=True)) < 1e-12


@pytest.mark.parametrize("N", [24, 48, 96])
def test_transforms_vs_oracle(mods, N):
    torch, qbgpu, orc = mods
    Wv = qbgpu.gaussian_mixture_state(N, L, seed=5, ncells=2)
    WF = qbgpu.to_fourier(torch.from_numpy(Wv).cuda()).cpu().numpy()
    assert rel_l1(WF, orc.to_fourier(Wv)) < 1e-14
    back = qbgpu.from_fourier(torch.from_numpy(WF).cuda()).cpu().numpy()
    assert rel_l1(back, orc.from_fourier(WF)) < 1e-14
    assert rel_l1(back, Wv) < 1e-14


def test_mixed_size_batch_rk4_vs_oracle(mods):
    """A batch of homogeneous instances of the configuration's sizes N = 16,
    24, 32, 48 (fixed-size and any-N groups side by side), RK4 steps, against
    the oracle's RK4 per instance."""
    torch, qbgpu, orc = mods
    J, M, dt, steps = 4, 3, 0.01, 2
    sizes = [24, 16, 48, 24, 32]
    W0 = [orc.to_fourier(qbgpu.gaussian_mixture_state(n, L, seed=400 + i, ncells=1))[0] for i, n in enumerate(sizes)]
    states = [torch.from_numpy(w.copy()).cuda() for w in W0]
    qbgpu.homogeneous_batch(states, dt, steps, rk4=True, J=J, M=M, L=L, R=R, precision=64)
    for i, n in enumerate(sizes):
        o = orc.Oracle(n, J, M, L, R)
        w = W0[i]
        for _ in range(steps):
            w = o.collision_step(w, dt, rk4=True)
        assert rel_l1(states[i].cpu().numpy(), w) < 1e-12, n


def test_fixed_sizes_through_the_any_n_engine():
    """QB_ANYN=1 (read per call) sends N = 16 and 32 through the any-N engine;
    both engines agree within FP64 rounding (run in a child process so the
    switch does not leak into other tests)."""
    code = r"""
import os, sys, numpy as np, torch
sys.path.insert(0, %r); sys.path.insert(0, %r)
import qbgpu, orc
for N in (16, 32):
    q = qbgpu.Quad(N, 4, 3, 6.0, 3.75)
    WF = orc.to_fourier(qbgpu.gaussian_mixture_state(N, 6.0, seed=9, ncells=2))
    W = torch.from_numpy(WF).cuda()
    os.environ["QB_ANYN"] = "0"
    a = [x.cpu().numpy() for x in qbgpu.collision_operators(qbgpu.Workspace(N), q, W)]
    os.environ["QB_ANYN"] = "1"
    b = [x.cpu().numpy() for x in qbgpu.collision_operators(qbgpu.Workspace(N), q, W)]
    for x, y in zip(a, b):
        r = np.abs(x - y).sum() / np.abs(x).sum()
        assert r < 1e-12, (N, r)
print("ok")
""" % (os.path.join(ROOT, "inhom-quantum-boltzmann-fourier-c_b200"), os.path.join(ROOT, "oracle"))
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("bc", ["periodic", "dirichlet"])
def test_inhomogeneous_strang_step_n24_vs_oracle(mods, bc):
    """The inhomogeneous Strang step (transport, Fourier representation,
    collision step, back, transport) at N = 24 through the any-N engine."""
    torch, qbgpu, orc = mods
    N, J, M, cells = 24, 4, 3, 5
    ws, q = qbgpu.Workspace(N), qbgpu.Quad(N, J, M, L, R)
    o = orc.Oracle(N, J, M, L, R)
    Wv = qbgpu.gaussian_mixture_state(N, L, seed=240, ncells=cells)
    Bext = np.random.default_rng(24).standard_normal((cells, 3)) * 0.2
    h, dt = 1.0 / cells, 0.4 / cells / L
    out = qbgpu.inhom_step(ws, q, torch.from_numpy(Wv).cuda(), h, dt, torch.from_numpy(Bext).cuda(), bc=bc).cpu().numpy()
    want = o.inhom_step(Wv, h, dt, Bext, bc=bc)
    assert rel_l1(out, want) < 1e-12


def test_inhomogeneous_graph_replay_n48(mods):
    """Strang steps at N = 48 that alternate two buffers replay their CUDA
    graphs from the third call of each direction on, bit-identical to
    kernel-by-kernel launches (profiling on)."""
    torch, qbgpu, orc = mods
    N, J, M, cells = 48, 4, 2, 3
    q = qbgpu.Quad(N, J, M, L, R)
    W0 = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=48, ncells=cells)).cuda()
    B = torch.zeros((cells, 3), dtype=torch.float64, device="cuda")
    h, dt, steps = 1.0 / cells, 0.4 / cells / L, 8
    ws = qbgpu.Workspace(N)
    bufs = [W0.clone(), torch.empty_like(W0)]
    for k in range(steps):
        qbgpu.inhom_step(ws, q, bufs[k % 2], h, dt, B, out=bufs[(k + 1) % 2])
    torch.cuda.synchronize()
    assert ws.graph_replays == steps - 4
    L_ = qbgpu.lib()
    ref, wsd = W0.clone(), qbgpu.Workspace(N)
    L_.qb_profile_enable(1)
    try:
        for k in range(steps):
            ref = qbgpu.inhom_step(wsd, q, ref, h, dt, B)
        torch.cuda.synchronize()
    finally:
        L_.qb_profile_enable(0)
        L_.qb_profile_reset()
    assert wsd.graph_replays == 0
    assert torch.equal(bufs[steps % 2], ref)


def test_waves_do_not_change_the_sums():
    """The I1-I4 sums run in waves of terms and, where one term of the batch
    overflows the scratch cap, in slices of cells; every cell still adds its
    terms in order.  A 1 MB wave budget and scratch cap (QB_ANYN_WAVE_MB,
    QB_ANYN_SLICE_MB, read per call) cut the batch into slices of one cell
    and one term a wave; Cc and Cd stay
    bit-identical to the default waves, FP32 real and complex forms (N = 96,
    three global passes), FP32 whole-grid chains (N = 48, QB_ANYN_FUSED=1) and
    FP64 (N = 48 with QB_ANYN_FUSED=0).  Run in a child process so the switches do not leak
    into other tests."""
    code = r"""
import os, sys, numpy as np, torch
sys.path.insert(0, %r); sys.path.insert(0, %r)
import qbgpu, orc
def run(N, prec, cells, seed, noisy):
    q = qbgpu.Quad(N, 2, 2, 6.0, 3.75)
    Wv = qbgpu.gaussian_mixture_state(N, 6.0, seed=seed, ncells=cells)
    if noisy:
        Wv[::2] += 1e-3 * np.random.default_rng(seed).standard_normal(Wv[::2].shape)
    W = torch.from_numpy(orc.to_fourier(Wv)).cuda()
    out = []
    for mb in ("", "1"):
        os.environ["QB_ANYN_WAVE_MB"] = mb
        os.environ["QB_ANYN_SLICE_MB"] = mb
        ws = qbgpu.Workspace(N, precision=prec)
        out.append([x.cpu().numpy() for x in qbgpu.collision_operators(ws, q, W)])
        forms = ws.i3_forms()
    os.environ["QB_ANYN_WAVE_MB"] = os.environ["QB_ANYN_SLICE_MB"] = ""
    for x, y in zip(*out):
        assert np.array_equal(x, y), (N, prec)
    return forms
assert run(96, 32, 5, 3, True) == (2, 5)
os.environ["QB_ANYN_FUSED"] = "1"
assert run(48, 32, 5, 4, True) == (2, 5)
os.environ["QB_ANYN_FUSED"] = "0"
assert run(48, 64, 3, 5, False) == (0, 0)
print("ok")
""" % (os.path.join(ROOT, "inhom-quantum-boltzmann-fourier-c_b200"), os.path.join(ROOT, "oracle"))
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr

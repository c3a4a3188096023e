"""GPU: the learned surrogate of the collision operator (qb_fno_*,
qb_surrogate_*), which has no upstream counterpart.

  - forward pass and every weight gradient against the float64 restatement
    oracle/fno_ref.py (itself pinned by finite differences);
  - training on homogeneous relaxation data cuts the held-out error;
  - the surrogate Strang step with tol = 0 is the exact step of qb_inhom_step;
  - a trained surrogate conserves mass, momentum and energy to round-off on
    its own steps and tracks the exact solver more closely than dropping the
    collision operator does;
  - a surrogate step is several times cheaper than an exact one.
"""
import math

import numpy as np
import pytest

import fno_ref
import qbgpu
from conftest import rel_l1

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

L, R = 6.0, 3.75


def rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def mixture_states(N, nseeds, seed):
    return qbgpu.mixture_cells(N, L, nseeds, seed)


def relaxation_pairs(N, J, M, nseeds, samples, seed):
    q = qbgpu.Quad(N, J, M, L, R)
    ws = qbgpu.Workspace(N)
    return qbgpu.relaxation_pairs(ws, q, torch.from_numpy(mixture_states(N, nseeds, seed)).cuda(), samples)


def test_forward_and_gradients_match_oracle():
    N, w, m, Ly, B = 16, 8, 4, 3, 3
    net = qbgpu.FNO(N, width=w, modes=m, layers=Ly, seed=3)
    assert net.num_params == fno_ref.num_params(w, m, Ly)
    W = mixture_states(N, B, seed=11)
    rng = np.random.default_rng(5)
    target = rng.standard_normal((B, 4, N, N)) * 0.1
    inscale = np.linspace(0.5, 2.0, fno_ref.NFEAT)
    scale = np.array([0.1, 0.2, 0.05, 0.3])
    net.set_input_scale(inscale)
    net.set_scale(scale)
    theta = net.get_params().astype(np.float64)
    x = fno_ref.features(W, inscale)
    y_ref = fno_ref.forward(theta, x, N, w, m, Ly) * scale[None, :, None]
    Wd = torch.from_numpy(W).cuda()
    y = net.forward(Wd).cpu().numpy().reshape(B, 4, -1)
    assert rel_l2(y, y_ref) < 1e-5
    loss, g = net.gradients(Wd, torch.from_numpy(target).cuda())
    loss_ref, g_ref = fno_ref.loss_and_grads(theta, x, target, scale, N, w, m, Ly)
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    gd, gr = fno_ref.unflatten(g.astype(np.float64), w, m, Ly), fno_ref.unflatten(g_ref, w, m, Ly)
    for name in gr:
        assert rel_l2(gd[name], gr[name]) < 1e-4, name
    # the gradient call left the weights alone; a train step moves them
    assert np.array_equal(net.get_params(), theta.astype(np.float32))
    net.train_step(Wd, torch.from_numpy(target).cuda(), 1e-3)
    assert not np.array_equal(net.get_params(), theta.astype(np.float32))


@pytest.mark.parametrize("N,w,m,Ly,B", [(16, 8, 4, 3, 3), (32, 32, 12, 4, 5), (16, 8, 4, 2, 130)])
def test_tensor_core_stages_against_oracle(N, w, m, Ly, B):
    """The pointwise channel maps, the truncated DFTs and (from 128 cells on)
    the mode mixing on the tensor cores (BF16 operands, FP32 accumulation):
    forward pass and weight gradients against the float64 restatement within
    BF16 accuracy (inputs and weights rounded to 8 significant bits), the MMA
    waits complete, and the FP32 path is untouched."""
    net = qbgpu.FNO(N, width=w, modes=m, layers=Ly, seed=7)
    W = mixture_states(N, B, seed=13)
    rng = np.random.default_rng(9)
    target = rng.standard_normal((B, 4, N, N)) * 0.1
    inscale = np.linspace(0.5, 2.0, fno_ref.NFEAT)
    scale = np.array([0.1, 0.2, 0.05, 0.3])
    net.set_input_scale(inscale)
    net.set_scale(scale)
    theta = net.get_params().astype(np.float64)
    x = fno_ref.features(W, inscale)
    y_ref = fno_ref.forward(theta, x, N, w, m, Ly) * scale[None, :, None]
    Wd = torch.from_numpy(W).cuda()
    y32 = net.forward(Wd).cpu().numpy().reshape(B, 4, -1)
    net.set_tensor_cores(True)
    ytc = net.forward(Wd).cpu().numpy().reshape(B, 4, -1)
    assert net.device_errors() == 0
    e_tc, e_32 = rel_l2(ytc, y_ref), rel_l2(y32, y_ref)
    assert e_32 < 1e-5
    assert 1e-5 < e_tc < 2e-2, e_tc
    loss, g = net.gradients(Wd, torch.from_numpy(target).cuda())
    loss_ref, g_ref = fno_ref.loss_and_grads(theta, x, target, scale, N, w, m, Ly)
    assert abs(loss - loss_ref) <= 3e-2 * loss_ref
    gd, gr = fno_ref.unflatten(g.astype(np.float64), w, m, Ly), fno_ref.unflatten(g_ref, w, m, Ly)
    for name in gr:
        assert rel_l2(gd[name], gr[name]) < 5e-2, name
    assert net.device_errors() == 0
    net.set_tensor_cores(False)
    assert np.array_equal(net.forward(Wd).cpu().numpy().reshape(B, 4, -1), y32)


def test_parameters_roundtrip_and_bad_arguments():
    net = qbgpu.FNO(8, width=4, modes=2, layers=1, seed=1)
    p = net.get_params()
    net.set_params(p * 2)
    assert np.array_equal(net.get_params(), p * 2)
    with pytest.raises(RuntimeError):
        net.set_scale([1.0, 0.0, 1.0, 1.0])
    with pytest.raises(RuntimeError):
        qbgpu.FNO(8, width=4, modes=5, layers=1)      # 2 modes - 1 > N
    with pytest.raises(RuntimeError):
        qbgpu.FNO(7, width=4, modes=2, layers=1)      # odd N
    # a network for another grid size than the workspace's
    q, ws = qbgpu.Quad(16, 4, 3, L, R), qbgpu.Workspace(16)
    sur = qbgpu.Surrogate(net, tol=1.0, check_every=2)
    W = torch.from_numpy(qbgpu.gaussian_mixture_state(16, L, seed=1, ncells=2)).cuda()
    with pytest.raises(RuntimeError):
        sur.step(ws, q, W, 0.5, 0.01)


@pytest.fixture(scope="module")
def trained16():
    N, J, M = 16, 8, 8
    X, Y = relaxation_pairs(N, J, M, 1024, 3, seed=5000)
    Xt, Yt = relaxation_pairs(N, J, M, 64, 2, seed=1)
    net = qbgpu.FNO(N, width=32, modes=6, layers=4, seed=2)
    net.fit_scales(X, Y)
    e0 = rel_l1(net.forward(Xt).cpu().numpy(), Yt.cpu().numpy())
    qbgpu.train_fno(net, X, Y, 4000, lr=5e-3, spin_rotations=True)
    e1 = rel_l1(net.forward(Xt).cpu().numpy(), Yt.cpu().numpy())
    return dict(N=N, J=J, M=M, net=net, e0=e0, e1=e1)


def test_training(trained16):
    assert trained16["e1"] < 0.4 * trained16["e0"] and trained16["e1"] < 0.4, (trained16["e0"], trained16["e1"])


def totals(W, N):
    """mass, momentum (x, y) and energy of the trace component over all cells"""
    v = qbgpu.velocity_grid(N, L)
    vx, vy = np.meshgrid(v, v, indexing="ij")
    w0 = W[:, 0]
    return np.array([w0.sum(), (w0 * vx).sum(), (w0 * vy).sum(), (w0 * (vx * vx + vy * vy)).sum()])


def test_surrogate_with_zero_tolerance_is_the_exact_step():
    N, J, M = 16, 4, 3
    q = qbgpu.Quad(N, J, M, L, R)
    ws = qbgpu.Workspace(N)
    net = qbgpu.FNO(N, width=8, modes=4, layers=2, seed=4)
    sur = qbgpu.Surrogate(net, tol=0.0, check_every=3)
    ncells, h = 6, 1.0 / 6
    dt = 0.4 * h / L
    W0 = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=21, ncells=ncells)).cuda()
    B = torch.from_numpy(np.random.default_rng(6).standard_normal((ncells, 3)) * 0.05).cuda()
    a, b = W0.clone(), W0.clone()
    for _ in range(5):
        a = qbgpu.inhom_step(ws, q, a, h, dt, B)
        b = sur.step(ws, q, b, h, dt, B)
    torch.cuda.synchronize()
    assert rel_l1(b.cpu().numpy(), a.cpu().numpy()) < 1e-12
    ns, ne, res = sur.stats()
    assert (ns, ne) == (0, 30) and res > 0


def transport_only(W, h, dt):
    return qbgpu.transport(qbgpu.transport(W, L, h, 0.5 * dt), L, h, 0.5 * dt)


def test_trained_surrogate_conserves_and_tracks_the_exact_solver(trained16):
    N, J, M, net = trained16["N"], trained16["J"], trained16["M"], trained16["net"]
    q = qbgpu.Quad(N, J, M, L, R)
    ws = qbgpu.Workspace(N)
    sur = qbgpu.Surrogate(net, tol=10.0, check_every=100)
    ncells, steps = 8, 10
    h = 1.0 / ncells
    dt = 0.4 * h / L
    W0 = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=77, ncells=ncells)).cuda()
    B = torch.from_numpy(np.random.default_rng(7).standard_normal((ncells, 3)) * 0.05).cuda()
    A, Bs, Cf = W0.clone(), W0.clone(), W0.clone()
    t1 = None
    for k in range(steps):
        A = qbgpu.inhom_step(ws, q, A, h, dt, B)
        Bs = sur.step(ws, q, Bs, h, dt, B)
        Cf = transport_only(Cf, h, dt)
        if k == 0:
            t1 = totals(Bs.cpu().numpy(), N)
    torch.cuda.synchronize()
    ns, ne, res = sur.stats()
    assert (ns, ne) == ((steps - 1) * ncells, ncells)
    assert 0 < res < math.inf
    # after the first (exact, checking) step only surrogate steps ran: their
    # projected C~ keeps the trace component's moments to round-off
    t = totals(Bs.cpu().numpy(), N)
    scale = np.array([abs(t1[0]), abs(t1[0]) * L, abs(t1[0]) * L, abs(t1[3])])
    assert np.all(np.abs(t - t1) / scale < 1e-12), np.abs(t - t1) / scale
    a, b, c = A.cpu().numpy(), Bs.cpu().numpy(), Cf.cpu().numpy()
    assert rel_l1(b, a) < 0.8 * rel_l1(c, a), (rel_l1(b, a), rel_l1(c, a))


def test_surrogate_step_is_cheaper_than_the_exact_step():
    N, J, M = 32, 16, 16
    q = qbgpu.Quad(N, J, M, L, R)
    ws = qbgpu.Workspace(N)
    net = qbgpu.FNO(N, width=32, modes=12, layers=4, seed=8)
    sur = qbgpu.Surrogate(net, tol=math.inf, check_every=1000)      # untrained: never fall back
    ncells, h = 64, 1.0 / 64
    dt = 0.4 * h / L
    W = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=31, ncells=ncells)).cuda()
    B = torch.zeros((ncells, 3), dtype=torch.float64, device="cuda")
    out = torch.empty_like(W)
    sur.step(ws, q, W, h, dt, B, out=out)               # the checking step

    def timed(f, n=5):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            f()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    t_ex = timed(lambda: qbgpu.inhom_step(ws, q, W, h, dt, B, out=out))
    t_sur = timed(lambda: sur.step(ws, q, W, h, dt, B, out=out))
    assert t_sur * 3 < t_ex, (t_sur, t_ex)

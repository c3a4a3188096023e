"""GPU: the FP32 precision form of the collision operator.

The FP32 form keeps the Wigner state, the Pauli-blocking assembly, the
magnetic term and the time update in FP64 and runs the spectra, the quadrature
tables and every FFT of the factored I1-I4 sums in FP32.  Its bound is the
relative error of C[W] against the FP64 operator: <= 1e-5 for each of Cc and
Cd (relative L2 over all cells and components), checked against the CPU
oracle on a small case and against the FP64 GPU path (itself pinned to the
oracle within 1e-12 by the parity tests) at the bench's table sizes.
"""
import numpy as np
import pytest

import orc
import qbgpu
from conftest import rel_l1

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

L, R = 6.0, 3.75
C_TOL = 1e-5


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def fourier_states(N, ncells, seed):
    Wv = qbgpu.gaussian_mixture_state(N, L, seed=seed, ncells=ncells)
    return Wv, np.stack([orc.to_fourier(w) for w in Wv])


def test_precision_selector():
    ws = qbgpu.Workspace(16)
    assert ws.precision == 64
    ws.set_precision(32)
    assert ws.precision == 32
    with pytest.raises(RuntimeError):
        ws.set_precision(16)
    assert ws.precision == 32


def test_fp32_operators_against_oracle():
    N, J, M = 16, 4, 3
    o = orc.Oracle(N, J, M, L, R)
    q = qbgpu.Quad(N, J, M, L, R)
    ws = qbgpu.Workspace(N, precision=32)
    _, Wf = fourier_states(N, 3, seed=71)
    cc, cd = qbgpu.collision_operators(ws, q, torch.from_numpy(Wf).cuda())
    cc, cd = cc.cpu().numpy(), cd.cpu().numpy()
    ref_cc = np.stack([o.cc(w) for w in Wf])
    ref_cd = np.stack([o.cd(w) for w in Wf])
    assert rel_l2(cc, ref_cc) <= C_TOL
    assert rel_l2(cd, ref_cd) <= C_TOL


@pytest.mark.parametrize("N,J,M", [(32, 16, 16), (32, 8, 4), (8, 4, 3), (64, 4, 3)])
def test_fp32_operators_against_fp64(N, J, M):
    q = qbgpu.Quad(N, J, M, L, R)
    ws64, ws32 = qbgpu.Workspace(N), qbgpu.Workspace(N, precision=32)
    _, Wf = fourier_states(N, 8, seed=72 + N)
    W = torch.from_numpy(Wf).cuda()
    cc64, cd64 = qbgpu.collision_operators(ws64, q, W)
    cc32, cd32 = qbgpu.collision_operators(ws32, q, W)
    e_cc = rel_l2(cc32.cpu().numpy(), cc64.cpu().numpy())
    e_cd = rel_l2(cd32.cpu().numpy(), cd64.cpu().numpy())
    assert e_cc <= C_TOL and e_cd <= C_TOL, (e_cc, e_cd)
    # the FP32 form is not the FP64 path under another name
    assert e_cc > 0 and e_cd > 0


def test_fp32_n64_real_form_and_guard():
    """N = 64 in FP32: cells with negligible Nyquist content run the I3 sums in
    real form (two chains per complex transform), cells with Nyquist content
    take the complex kernel; both stay within the FP32 bound of the oracle"""
    N, J, M = 64, 4, 3
    o = orc.Oracle(N, J, M, L, R)
    q = qbgpu.Quad(N, J, M, L, R)
    Wv = qbgpu.gaussian_mixture_state(N, L, seed=2, ncells=4)
    rng = np.random.default_rng(5)
    Wv[2:] += 1e-3 * rng.standard_normal(Wv[2:].shape)      # white noise: Nyquist fraction far above 1e-6
    Wf = np.stack([orc.to_fourier(w) for w in Wv])
    ws32, ws64 = qbgpu.Workspace(N, precision=32), qbgpu.Workspace(N)
    cc, cd = qbgpu.collision_operators(ws32, q, torch.from_numpy(Wf).cuda())
    qbgpu.collision_operators(ws64, q, torch.from_numpy(Wf).cuda())
    assert ws32.i3_forms() == (2, 4)
    assert ws64.i3_forms() == (0, 0)
    assert ws32.i3_forms(reset=True) == (2, 4) and ws32.i3_forms() == (0, 0)
    cc, cd = cc.cpu().numpy(), cd.cpu().numpy()
    for sl in (slice(0, 2), slice(2, 4)):
        ref_cc = np.stack([o.cc(w) for w in Wf[sl]])
        ref_cd = np.stack([o.cd(w) for w in Wf[sl]])
        assert rel_l2(cc[sl], ref_cc) <= C_TOL
        assert rel_l2(cd[sl], ref_cd) <= C_TOL


@pytest.mark.parametrize("N,J,M", [(32, 4, 3), (64, 4, 3), (48, 4, 3), (96, 2, 2), (128, 2, 2)])
def test_fp32_real_form_guard_routes_non_hermitian_states(N, J, M):
    """The real form of the FP32 I3 sums (N = 32: k_i3pr, N = 64:
    k_i3_full128r; N = 48 the whole-grid chains of the any-N engine, N = 96
    and 128 its three-pass chains, all with two chains packed in one complex
    transform) holds only for Fourier states of real velocity-space
    components (Hermitian, W(-k) = conj W(k)) without Nyquist content.  Two
    smooth cells take it; two cells with an anti-Hermitian part (a complex
    perturbation kept off the Nyquist row and column, so that only the
    Hermitian check can catch it) take the complex kernel, and all four stay
    within the FP32 bound of the oracle, which evaluates general complex
    states."""
    o = orc.Oracle(N, J, M, L, R)
    q = qbgpu.Quad(N, J, M, L, R)
    _, Wf = fourier_states(N, 4, seed=90 + N)
    rng = np.random.default_rng(N)
    noise = rng.standard_normal(Wf[2:].shape) + 1j * rng.standard_normal(Wf[2:].shape)
    noise[..., N // 2, :] = 0
    noise[..., :, N // 2] = 0
    Wf[2:] += 1e-4 * np.abs(Wf[2:]).max() * noise
    ws32 = qbgpu.Workspace(N, precision=32)
    cc, cd = qbgpu.collision_operators(ws32, q, torch.from_numpy(Wf).cuda())
    assert ws32.i3_forms() == (2, 4)
    cc, cd = cc.cpu().numpy(), cd.cpu().numpy()
    for sl in (slice(0, 2), slice(2, 4)):
        ref_cc = np.stack([o.cc(w) for w in Wf[sl]])
        ref_cd = np.stack([o.cd(w) for w in Wf[sl]])
        assert rel_l2(cc[sl], ref_cc) <= C_TOL, sl
        assert rel_l2(cd[sl], ref_cd) <= C_TOL, sl


def conserved_totals(W):
    """mass, momentum (x, y) and kinetic energy of the trace component summed over all cells"""
    d = orc.diagnostics(W, L)
    mass = d[:, 0]
    mom = mass[:, None] * d[:, 4:6]
    energy = mass * (d[:, 6] + 0.5 * (d[:, 4] ** 2 + d[:, 5] ** 2))
    return np.array([mass.sum(), mom[:, 0].sum(), mom[:, 1].sum(), energy.sum()])


def test_fp32_strang_steps_track_fp64():
    N, J, M = 32, 16, 16
    q = qbgpu.Quad(N, J, M, L, R)
    ws64, ws32 = qbgpu.Workspace(N), qbgpu.Workspace(N, precision=32)
    ncells, steps = 16, 20
    h = 1.0 / ncells
    dt = 0.4 * h / L
    W0 = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=73, ncells=ncells)).cuda()
    B = torch.from_numpy(np.random.default_rng(9).standard_normal((ncells, 3)) * 0.05).cuda()
    a, b = W0.clone(), W0.clone()
    for _ in range(steps):
        a = qbgpu.inhom_step(ws64, q, a, h, dt, B)
        b = qbgpu.inhom_step(ws32, q, b, h, dt, B)
    torch.cuda.synchronize()
    a, b = a.cpu().numpy(), b.cpu().numpy()
    assert rel_l1(b, a) <= 1e-6


@pytest.mark.parametrize("precision", [32, 64])
def test_conserved_moments_over_1000_steps(precision):
    """with conservation on, mass, momentum and energy drift <= 1e-9 (relative)
    over 1000 Strang steps (periodic, magnetic field on); the plain discrete
    operator keeps them only to its quadrature accuracy"""
    N, J, M = 32, 16, 16
    q = qbgpu.Quad(N, J, M, L, R)
    ws = qbgpu.Workspace(N, precision=precision, conserve=True)
    ncells, steps = 8, 1000
    h = 1.0 / ncells
    dt = 0.4 * h / L
    W0 = qbgpu.gaussian_mixture_state(N, L, seed=75, ncells=ncells)
    B = torch.from_numpy(np.random.default_rng(10).standard_normal((ncells, 3)) * 0.05).cuda()
    w = torch.from_numpy(W0).cuda()
    nxt = torch.empty_like(w)
    for _ in range(steps // 2):
        qbgpu.inhom_step(ws, q, w, h, dt, B, out=nxt)
        qbgpu.inhom_step(ws, q, nxt, h, dt, B, out=w)
    torch.cuda.synchronize()
    t0, t1 = conserved_totals(W0), conserved_totals(w.cpu().numpy())
    scale = np.array([abs(t0[0]), abs(t0[0]) * L, abs(t0[0]) * L, abs(t0[3])])
    drift = np.abs(t1 - t0) / scale
    assert np.all(drift <= 1e-9), drift


def test_fp32_graph_replay_equals_direct(monkeypatch):
    N, J, M = 16, 4, 3
    q = qbgpu.Quad(N, J, M, L, R)
    ws = qbgpu.Workspace(N, precision=32)
    W = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=74, ncells=4)).cuda()
    B = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    out = torch.empty_like(W)
    results = []
    for _ in range(3):
        qbgpu.inhom_step(ws, q, W, 0.25, 0.01, B, out=out)
        torch.cuda.synchronize()
        results.append(out.clone())
    assert all(torch.equal(r, results[0]) for r in results[1:])
    monkeypatch.setenv("QB_CUDA_GRAPHS", "0")
    ws2 = qbgpu.Workspace(N, precision=32)
    assert torch.equal(qbgpu.inhom_step(ws2, q, W, 0.25, 0.01, B), results[0])


def test_eigenvalues_stay_in_unit_interval_over_200_steps():
    """0 <= W <= 1 (the Pauli principle: eigenvalues w0 -+ |w|) along 200 Strang
    steps of the inhomogeneous workload (64 cells, N = 32, J = M = 16), in both
    precisions; the tails of the state dip below 0 by the discrete operator's
    error only (about 1e-7), and the FP32 form tracks the FP64 bounds"""
    N, J, M, cells, steps = 32, 16, 16, 64, 200
    q = qbgpu.Quad(N, J, M, L, R)
    h = 1.0 / cells
    dt = 0.4 * h / L
    W0 = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=1, ncells=cells)).cuda()
    bounds = {}
    for prec in (64, 32):
        ws = qbgpu.Workspace(N, precision=prec)
        w, nxt = W0.clone(), torch.empty_like(W0)
        lo, hi = np.inf, -np.inf
        for k in range(steps):
            qbgpu.inhom_step(ws, q, w, h, dt, out=nxt)
            w, nxt = nxt, w
            if k % 20 == 19:
                d = qbgpu.diagnostics(w, L).cpu().numpy()
                lo, hi = min(lo, d[:, 7].min()), max(hi, d[:, 8].max())
        assert -1e-6 <= lo and hi <= 1.0, (prec, lo, hi)
        bounds[prec] = (lo, hi)
    assert abs(bounds[32][0] - bounds[64][0]) <= 1e-8 and abs(bounds[32][1] - bounds[64][1]) <= 1e-8, bounds


def test_fp32_state_after_1000_steps():
    """the FP32 form's W against the FP64 path after 1000 Strang steps (8 cells,
    N = 32, J = M = 16, magnetic field on): within the 1e-5 bound of C"""
    N, J, M, cells, steps = 32, 16, 16, 8, 1000
    q = qbgpu.Quad(N, J, M, L, R)
    h = 1.0 / cells
    dt = 0.4 * h / L
    W0 = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=76, ncells=cells)).cuda()
    B = torch.from_numpy(np.random.default_rng(11).standard_normal((cells, 3)) * 0.05).cuda()
    out = {}
    for prec in (64, 32):
        ws = qbgpu.Workspace(N, precision=prec)
        w, nxt = W0.clone(), torch.empty_like(W0)
        for _ in range(steps):
            qbgpu.inhom_step(ws, q, w, h, dt, B, out=nxt)
            w, nxt = nxt, w
        out[prec] = w.cpu().numpy()
    e = rel_l1(out[32], out[64])
    assert 0 < e <= 1e-5, e

"""GPU: Fermi-Dirac equilibrium fit and quantum relative entropy diagnostics
against the numpy/scipy restatement of the upstream Matlab post-processing
(visualization/asymptoticFD.m, calculateFDparams.m, createFD.m,
relentropy.m).  The library solves the moment equations by Newton's method
with its own dilogarithm; the oracle uses scipy's least squares and
scipy.special.spence, so the two share no code."""
import numpy as np
import pytest

import orc
import qbgpu

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

L = 6.0


def fd_state(N, beta, mu, u, n):
    v = orc._vgrid(N, L)
    vx, vy = np.meshgrid(v, v, indexing="ij")
    e = 0.5 * ((vx - u[0]) ** 2 + (vy - u[1]) ** 2)
    f1 = 1 / (np.exp(beta * (e - mu[0])) + 1)
    f2 = 1 / (np.exp(beta * (e - mu[1])) + 1)
    n = np.asarray(n) / np.linalg.norm(n)
    return np.stack([0.5 * (f1 + f2)] + [0.5 * (f2 - f1) * c for c in n])


@pytest.mark.parametrize("N", [16, 32])
def test_equilibrium_matches_oracle(N):
    W = qbgpu.gaussian_mixture_state(N, L, seed=81 + N, ncells=3)
    WFD, par = qbgpu.fermi_dirac_equilibrium(torch.from_numpy(W).cuda(), L)
    ref_W, ref_par = orc.asymptotic_fd(W, L)
    assert np.all(par[:, 8] < 1e-10) and np.all(ref_par[:, 8] < 1e-10)
    assert np.allclose(par[:, :8], ref_par[:, :8], rtol=1e-8, atol=1e-10)
    assert np.allclose(WFD.cpu().numpy(), ref_W, rtol=1e-8, atol=1e-12)


def test_equilibrium_recovers_a_fermi_dirac_state():
    N = 32
    beta, mu, u, n = 1.3, (0.4, 1.1), (0.3, -0.2), (0.2, -0.5, 0.8)
    W = fd_state(N, beta, mu, u, n)[None]
    _, par = qbgpu.fermi_dirac_equilibrium(torch.from_numpy(W).cuda(), L)
    nn = np.asarray(n) / np.linalg.norm(n)
    # Riemann sums over the box against integrals over the plane: the tail
    # beyond [-L, L)^2 bounds the match
    assert np.allclose(par[0, :8], [beta, mu[0], mu[1], u[0], u[1], *nn], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("N", [16, 32])
def test_relative_entropy_matches_oracle(N):
    W = qbgpu.gaussian_mixture_state(N, L, seed=91 + N, ncells=2)
    Wd = torch.from_numpy(W).cuda()
    WFD, _ = qbgpu.fermi_dirac_equilibrium(Wd, L)
    out = qbgpu.relative_entropy(Wd, WFD, L).cpu().numpy()
    ref = orc.relative_entropy(W, WFD.cpu().numpy(), L)
    assert np.allclose(out, ref, rtol=1e-10, atol=1e-13)
    assert np.all(out[:, 0] > 0) and np.all(out[:, 1] > 0)
    # a state relative to itself
    self_kl = qbgpu.relative_entropy(WFD, WFD, L).cpu().numpy()
    assert np.all(np.abs(self_kl) < 1e-12)

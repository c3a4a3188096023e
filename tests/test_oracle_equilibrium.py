"""CPU: the oracle's restatement of the upstream Fermi-Dirac / relative-entropy
post-processing (visualization/asymptoticFD.m, relentropy.m) on states with
known answers.  No Matlab goldens exist for these, so they are pinned by
construction: a Fermi-Dirac state is its own equilibrium and has zero
relative entropy to it."""
import numpy as np

import orc

L = 6.0


def test_fd_fit_recovers_parameters_of_a_fd_state():
    N = 32
    beta, mu, u, n = 0.9, (-0.3, 0.7), (-0.4, 0.25), np.array([0.6, 0.0, -0.8])
    v = orc._vgrid(N, L)
    vx, vy = np.meshgrid(v, v, indexing="ij")
    e = 0.5 * ((vx - u[0]) ** 2 + (vy - u[1]) ** 2)
    f1, f2 = 1 / (np.exp(beta * (e - mu[0])) + 1), 1 / (np.exp(beta * (e - mu[1])) + 1)
    W = np.stack([0.5 * (f1 + f2)] + [0.5 * (f2 - f1) * c for c in n])[None]
    WFD, par = orc.asymptotic_fd(W, L)
    # the moments are Riemann sums over the box [-L, L)^2, the fit uses the
    # integrals over the plane: the state's tail beyond the box bounds the match
    assert np.allclose(par[0, :8], [beta, mu[0], mu[1], u[0], u[1], *n], rtol=1e-5, atol=1e-6)
    assert np.abs(WFD - W).max() < 1e-5
    kl = orc.relative_entropy(W, WFD, L)
    assert abs(kl[0, 0]) < 1e-8 and kl[0, 1] < 1e-4


def test_relative_entropy_is_positive_off_equilibrium():
    import qbgpu
    W = qbgpu.gaussian_mixture_state(16, L, seed=5, ncells=2)
    WFD, par = orc.asymptotic_fd(W, L)
    assert np.all(par[:, 8] < 1e-10)
    kl = orc.relative_entropy(W, WFD, L)
    assert np.all(kl > 0)

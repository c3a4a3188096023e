"""CPU: the float64 restatement of the Fourier-neural-operator surrogate
(oracle/fno_ref.py).  There is no upstream counterpart to pin it to, so its
analytic gradient is pinned by central finite differences of its own loss, and
its spectral layer by the properties of the transform it restates."""
import numpy as np
import pytest

import fno_ref


def small_case(seed=0):
    N, w, m, L, B = 8, 3, 2, 2, 2
    rng = np.random.default_rng(seed)
    theta = rng.standard_normal(fno_ref.num_params(w, m, L)) * 0.5
    x = rng.standard_normal((B, fno_ref.NFEAT, N * N))
    target = rng.standard_normal((B, 4, N * N))
    scale = np.array([1.0, 2.0, 0.5, 3.0])
    return N, w, m, L, theta, x, target, scale


def test_gradient_matches_finite_differences():
    N, w, m, L, theta, x, target, scale = small_case()
    loss, g = fno_ref.loss_and_grads(theta, x, target, scale, N, w, m, L)
    assert np.isfinite(loss) and g.shape == theta.shape
    rng = np.random.default_rng(1)
    eps = 1e-6
    for i in rng.choice(theta.size, 40, replace=False):
        tp, tm = theta.copy(), theta.copy()
        tp[i] += eps
        tm[i] -= eps
        lp, _ = fno_ref.loss_and_grads(tp, x, target, scale, N, w, m, L)
        lm, _ = fno_ref.loss_and_grads(tm, x, target, scale, N, w, m, L)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_every_weight_group_receives_gradient():
    N, w, m, L, theta, x, target, scale = small_case(2)
    _, g = fno_ref.loss_and_grads(theta, x, target, scale, N, w, m, L)
    for name, arr in fno_ref.unflatten(g, w, m, L).items():
        assert np.abs(arr).max() > 0, name


def test_truncated_dft_matches_the_full_fft():
    N, m = 8, 3
    rng = np.random.default_rng(3)
    h = rng.standard_normal((N, N))
    E = fno_ref.dft_mats(N, m)
    H = E @ h.ravel()
    F = np.fft.fft2(h)
    for kx in range(-(m - 1), m):
        for ky in range(m):
            assert abs(H[(kx + m - 1) * m + ky] - F[kx % N, ky]) < 1e-12


def test_features_layout():
    rng = np.random.default_rng(4)
    W = rng.standard_normal((2, 4, 4, 4))
    s = np.arange(1, 15, dtype=np.float64)
    x = fno_ref.features(W, s)
    assert x.shape == (2, 14, 16) and x.dtype == np.float32
    Wf = W.reshape(2, 4, 16)
    assert np.allclose(x[:, 2], 3 * Wf[:, 2], rtol=1e-6)
    # (0,0), (0,1), (0,2), (0,3), (1,1), ...: feature 8 is w1 w1
    assert np.allclose(x[:, 8], 9 * Wf[:, 1] ** 2, rtol=1e-6)
    assert np.allclose(x[:, 13], 14 * Wf[:, 3] ** 2, rtol=1e-6)


def test_flatten_roundtrip():
    w, m, L = 3, 2, 2
    theta = np.arange(fno_ref.num_params(w, m, L), dtype=np.float64)
    assert np.array_equal(fno_ref.flatten(fno_ref.unflatten(theta, w, m, L), w, m, L), theta)


def test_collision_operator_commutes_with_spin_rotations():
    """the premise of training the surrogate on spin-rotated pairs: for a global
    rotation R of the Pauli vector, C[R W] = R C[W] (oracle, N = 8)"""
    import orc
    import qbgpu
    N, J, M, L, R = 8, 4, 3, 6.0, 3.75
    o = orc.Oracle(N, J, M, L, R)
    W = qbgpu.gaussian_mixture_state(N, L, seed=3, ncells=1)[0]
    torch = pytest.importorskip("torch")
    Rm = qbgpu.random_rotations(1, torch.Generator().manual_seed(1))
    assert float((Rm[0] @ Rm[0].T - torch.eye(3, dtype=torch.float64)).abs().max()) < 1e-14
    Q = Rm[0].numpy()

    def rot(X):
        Y = X.copy()
        Y[1:4] = np.einsum("ij,jkl->ikl", Q, X[1:4])
        return Y
    # the device helper applies the same rotation
    Wt = torch.from_numpy(W[None].copy())
    assert np.abs(qbgpu.rotate_spin(Wt, Rm)[0].numpy() - rot(W)).max() < 1e-15
    Wf, WRf = orc.to_fourier(W[None])[0], orc.to_fourier(rot(W)[None])[0]
    c0 = o.cc(Wf) + o.cd(Wf)
    c1 = o.cc(WRf) + o.cd(WRf)
    assert np.abs(c1 - rot(c0)).max() <= 1e-12 * np.abs(c0).max()

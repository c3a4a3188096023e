"""CPU: the identity behind the real form of the FP32 I3 sums at N = 64.

One I3 chain is X_j += eta_i P_i . FFT2(psi2 . IFFT2(W^_i . P_j)) with
W^_i = FFT2(Pad(W_i)) and P_c = FFT2(Pad(psi1 . W_c)) (upstream I3integral,
src/integrals.c:332-379).  When the N x N Fourier states W_c have zero
Nyquist row and column, Pad(W_c) and Pad(psi1 . W_c) are Hermitian, so W^ and
P are real, and a -> FFT2(psi2 . IFFT2(a)) maps real grids to real grids
(psi2 real and even).  Two chains then share one complex transform and the
spectra of two components come out of one.  These tests restate both forms in
numpy at a small size: equal to rounding without Nyquist content, and apart by
a fraction of the Nyquist content otherwise (the bound the GPU guard uses).
"""
import math

import numpy as np

N, L, R = 16, 6.0, 3.75
P = 2 * N
ETA = (1.0, -1.0, -1.0, -1.0)


def pad(a):
    o = np.zeros((P, P), complex)
    h = N // 2
    o[:h, :h] = a[:h, :h]; o[:h, -h:] = a[:h, h:]; o[-h:, :h] = a[h:, :h]; o[-h:, -h:] = a[h:, h:]
    return o


def state(seed, nyquist):
    """4 Fourier-space Pauli components of a smooth real state; `nyquist`
    scales the entries on row and column N/2"""
    rng = np.random.default_rng(seed)
    v = np.array([k if k < N // 2 else k - N for k in range(N)]) * 2 * L / N
    vx, vy = np.meshgrid(v, v, indexing="ij")
    W = np.zeros((4, N, N))
    for _ in range(2):
        u, T, s = rng.uniform(-1, 1, 2), rng.uniform(0.5, 1.5), rng.uniform(-0.5, 0.5, 3)
        g = rng.uniform(0.3, 0.6) * np.exp(-((vx - u[0]) ** 2 + (vy - u[1]) ** 2) / (2 * T)) / 2
        W[0] += g
        W[1:] += g * s[:, None, None]
    F = np.fft.fft2(W, axes=(1, 2)) / N ** 2
    F[:, N // 2, :] *= nyquist
    F[:, :, N // 2] *= nyquist
    return F


def terms(J=3, M=2):
    kg = np.array([k if k < N // 2 else k - N for k in range(N)])
    k2 = np.array([k if k < N else k - P for k in range(P)])
    Kl, Kk = np.meshgrid(kg, kg, indexing="ij")
    K2l, K2k = np.meshgrid(k2, k2, indexing="ij")
    rho, w = np.polynomial.legendre.leggauss(M)
    for j in range(J):
        th = 2 * math.pi * j / J
        for m in range(M):
            r = (rho[m] + 1) * R / 2
            psi1 = np.exp(1j * r * math.pi / L * (Kl * math.cos(th) + Kk * math.sin(th)))
            psi2 = w[m] * np.sinc(R / L * (-K2l * math.sin(th) + K2k * math.cos(th)))
            yield psi1, psi2


def complex_sums(F):
    What = [np.fft.fft2(pad(F[c])) for c in range(4)]
    X = np.zeros((4, P, P), complex)
    for psi1, psi2 in terms():
        Pc = [np.fft.fft2(pad(psi1 * F[c])) for c in range(4)]
        for j in range(4):
            for i in range(4):
                X[j] += ETA[i] * Pc[i] * np.fft.fft2(psi2 * np.fft.ifft2(What[i] * Pc[j]))
    return X


def real_sums(F):
    """the packed real form: spectra of components (0, 1) and (2, 3) from one
    transform each, chains (i = 0, 1) and (2, 3) of every output in one each"""
    What = [np.fft.fft2(pad(F[c])).real for c in range(4)]
    X = np.zeros((4, P, P))
    for psi1, psi2 in terms():
        Pc = []
        for a in (0, 2):
            z = np.fft.fft2(pad(psi1 * (F[a] + 1j * F[a + 1])))
            Pc += [z.real, z.imag]
        for j in range(4):
            for i0 in (0, 2):
                z = np.fft.fft2(psi2 * np.fft.ifft2(Pc[j] * (What[i0] + 1j * What[i0 + 1])))
                X[j] += ETA[i0] * Pc[i0] * z.real + ETA[i0 + 1] * Pc[i0 + 1] * z.imag
    return X


def nyquist_fraction(F):
    a = np.abs(F)
    return (a[:, N // 2, :].sum() + a[:, :, N // 2].sum() - a[:, N // 2, N // 2].sum()) / a.sum()


def test_real_form_exact_without_nyquist_content():
    F = state(3, nyquist=0.0)
    Xc, Xr = complex_sums(F), real_sums(F)
    assert np.abs(Xc.imag).max() <= 1e-12 * np.abs(Xc).max()
    assert np.abs(Xc - Xr).max() <= 1e-12 * np.abs(Xc).max()


def test_real_form_error_bounded_by_nyquist_content():
    for seed in (3, 4):
        F = state(seed, nyquist=1.0)
        frac = nyquist_fraction(F)
        Xc, Xr = complex_sums(F), real_sums(F)
        err = np.abs(Xc - Xr).sum() / np.abs(Xc).sum()
        assert frac > 1e-8, frac
        assert err <= 2.0 * frac, (err, frac)

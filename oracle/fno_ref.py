"""ORACLE / TEST INFRASTRUCTURE ONLY: float64 numpy restatement of the
Fourier-neural-operator surrogate of the collision operator (the model of
csrc/qb_fno.cu, which has no upstream counterpart): forward pass, loss and
the analytic gradient of every weight.  The GPU kernels are checked against
it; its own gradient is checked against central finite differences.

Model, per cell (fields on the N x N velocity grid, point p = l N + k_v):
  x      = 14 input features: w_c (c = 0..3) and w_i w_j (i <= j), times scale
  h0     = A x + a
  layer  H = DFT_m(h), O[o] = sum_i R[i, o] H[i], s = Re IDFT_m(O) / N^2,
         u = s + W h + b, h' = gelu(u) (no gelu after the last layer)
  y      = Q h + q,  C~ = y * out_scale
DFT_m keeps the frequencies kx in [-(m-1), m-1], ky in [0, m):
  H(k) = sum_p h(p) exp(-i theta(k, p)), theta = 2 pi (kx l + ky k_v) / N,
frequency index k = (kx + m - 1) m + ky.  The weight vector is the flat
float32 array of qb_fno_get_params: A[w][14], a[w], per layer Rr[w][w][K],
Ri[w][w][K] (index [in][out][k]), W[w][w] ([out][in]), b[w], Q[4][w], q[4].
"""
import numpy as np
from scipy.special import erf

NFEAT = 14


def features(W, scale=None):
    """(B, 4, N, N) or (B, 4, P) float64 states -> (B, 14, P) float32 features
    (computed in float64 and rounded once, as the device kernel does)"""
    W = np.asarray(W, dtype=np.float64)
    B = W.shape[0]
    W = W.reshape(B, 4, -1)
    s = np.ones(NFEAT) if scale is None else np.asarray(scale, dtype=np.float64)
    out = []
    f = 0
    for c in range(4):
        out.append(s[f] * W[:, c])
        f += 1
    for i in range(4):
        for j in range(i, 4):
            out.append(s[f] * W[:, i] * W[:, j])
            f += 1
    return np.stack(out, axis=1).astype(np.float32)


def shapes(w, m, L):
    K = (2 * m - 1) * m
    sh = [("A", (w, NFEAT)), ("a", (w,))]
    for l in range(L):
        sh += [(f"Rr{l}", (w, w, K)), (f"Ri{l}", (w, w, K)), (f"W{l}", (w, w)), (f"b{l}", (w,))]
    sh += [("Q", (4, w)), ("q", (4,))]
    return sh


def num_params(w, m, L):
    return sum(int(np.prod(s)) for _, s in shapes(w, m, L))


def unflatten(theta, w, m, L):
    theta = np.asarray(theta, dtype=np.float64)
    out, o = {}, 0
    for name, s in shapes(w, m, L):
        n = int(np.prod(s))
        out[name] = theta[o:o + n].reshape(s)
        o += n
    assert o == theta.size
    return out


def flatten(d, w, m, L):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in shapes(w, m, L)])


def dft_mats(N, m):
    """E[k, p] = exp(-i theta(k, p))"""
    kx = np.arange(-(m - 1), m)
    ky = np.arange(m)
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    l = np.arange(N)
    L_, V_ = np.meshgrid(l, l, indexing="ij")
    th = 2 * np.pi * (KX.ravel()[:, None] * L_.ravel()[None, :] + KY.ravel()[:, None] * V_.ravel()[None, :]) / N
    return np.exp(-1j * th)


def gelu(u):
    return 0.5 * u * (1 + erf(u / np.sqrt(2)))


def dgelu(u):
    return 0.5 * (1 + erf(u / np.sqrt(2))) + u * np.exp(-0.5 * u * u) / np.sqrt(2 * np.pi)


def forward(theta, x, N, w, m, L, keep=False):
    """x: (B, 14, N*N) features; returns y (B, 4, N*N), unscaled network output"""
    p = unflatten(theta, w, m, L)
    x = np.asarray(x, dtype=np.float64)
    P = N * N
    E = dft_mats(N, m)
    h = np.einsum("oi,bip->bop", p["A"], x) + p["a"][None, :, None]
    hs, us, Hs = [h], [], []
    for l in range(L):
        H = h @ E.T
        R = p[f"Rr{l}"] + 1j * p[f"Ri{l}"]
        O = np.einsum("iok,bik->bok", R, H)
        s = np.real(O @ np.conj(E)) / P
        u = s + np.einsum("oi,bip->bop", p[f"W{l}"], h) + p[f"b{l}"][None, :, None]
        h = gelu(u) if l < L - 1 else u
        hs.append(h)
        us.append(u)
        Hs.append(H)
    y = np.einsum("oi,bip->bop", p["Q"], h) + p["q"][None, :, None]
    if keep:
        return y, (p, x, E, hs, us, Hs)
    return y


def loss_and_grads(theta, x, target, scale, N, w, m, L):
    """loss = mean((y - target / scale)^2) and its gradient (flat, float64)"""
    y, (p, x, E, hs, us, Hs) = forward(theta, x, N, w, m, L, keep=True)
    P = N * N
    t = np.asarray(target, dtype=np.float64).reshape(y.shape) / np.asarray(scale, dtype=np.float64)[None, :, None]
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2 * d / d.size
    g = {}
    g["Q"] = np.einsum("bop,bip->oi", dy, hs[L])
    g["q"] = dy.sum(axis=(0, 2))
    dh = np.einsum("oi,bop->bip", p["Q"], dy)
    for l in reversed(range(L)):
        du = dh * dgelu(us[l]) if l < L - 1 else dh
        g[f"W{l}"] = np.einsum("bop,bip->oi", du, hs[l])
        g[f"b{l}"] = du.sum(axis=(0, 2))
        GO = (du @ E.T) / P
        dR = np.einsum("bok,bik->iok", GO, np.conj(Hs[l]))
        g[f"Rr{l}"] = dR.real
        g[f"Ri{l}"] = dR.imag
        R = p[f"Rr{l}"] + 1j * p[f"Ri{l}"]
        GH = np.einsum("iok,bok->bik", np.conj(R), GO)
        dh = np.einsum("oi,bop->bip", p[f"W{l}"], du) + np.real(GH @ np.conj(E))
    g["A"] = np.einsum("bop,bip->oi", dh, x)
    g["a"] = dh.sum(axis=(0, 2))
    return loss, flatten(g, w, m, L)

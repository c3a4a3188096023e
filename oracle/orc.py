"""ORACLE / TEST INFRASTRUCTURE ONLY: ctypes access to the CPU checkers.

  Oracle  -- the C restatement (oracle/_build/liboracle.so, qb_oracle.c),
             run-time grid size N.
  Ref     -- the unmodified upstream C sources compiled with the project's CPU
             FFTW-API shim (oracle/_ref/libqbref_n32.so, N = 32), present
             only where the upstream checkout existed at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Arrays are numpy: complex grids complex128 of shape (..., N, N)
(element (l, k) = [l, k], the upstream index k + N*l), real grids float64.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqbref_n32.so")

_dp = C.POINTER(C.c_double)


def build():
    """Compile the checkers with oracle/Makefile (restatement always, upstream
    sources when their checkout exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _ptr(a):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _c(a):
    """complex128 C-contiguous copy/view"""
    return np.ascontiguousarray(a, dtype=np.complex128)


def _r(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _Quad(C.Structure):
    _fields_ = [("N", C.c_int), ("J", C.c_int), ("M", C.c_int), ("L", C.c_double), ("R", C.c_double),
                ("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int), ("n4", C.c_int)] + \
               [(n, _dp) for n in ("i1r1", "i1r2", "i2r1", "i2r2", "i3r1", "i3r2", "i4r1", "i4r2")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_quad_create.restype = C.POINTER(_Quad)
        L.orc_quad_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_flux_right.restype = C.c_double
        L.orc_flux_left.restype = C.c_double
        _lib = L
    return _lib


class Oracle:
    """Quadrature tables for (N, J, M, L, R) plus the restated operators."""

    def __init__(self, N, J, M, L, R):
        self.N, self.J, self.M, self.L, self.R = N, J, M, L, R
        self.q = lib().orc_quad_create(N, J, M, L, R)

    def __del__(self):
        if getattr(self, "q", None) is not None and _lib is not None:
            _lib.orc_quad_free(self.q)
            self.q = None

    # tables as numpy views (copied)
    def tables(self):
        N, P, q = self.N, 2 * self.N, self.q.contents
        def arr(p, n, shape, dt=np.float64):
            a = np.ctypeslib.as_array(p, shape=(n,)).copy()
            return a.view(dt).reshape(shape) if dt is not np.float64 else a.reshape(shape)
        return {
            "i1r1": arr(q.i1r1, q.n1 * P * P, (q.n1, P, P)), "i1r2": arr(q.i1r2, q.n1 * N * N, (q.n1, N, N)),
            "i2r1": arr(q.i2r1, q.n2 * N * N, (q.n2, N, N)), "i2r2": arr(q.i2r2, q.n2 * N * N, (q.n2, N, N)),
            "i3r1": np.ctypeslib.as_array(q.i3r1, shape=(q.n3 * 2 * N * N,)).copy().view(np.complex128).reshape(q.n3, N, N),
            "i3r2": arr(q.i3r2, q.n3 * P * P, (q.n3, P, P)),
            "i4r1": arr(q.i4r1, q.n4 * P * P, (q.n4, P, P)), "i4r2": arr(q.i4r2, q.n4 * N * N, (q.n4, N, N)),
        }

    def _int(self, fn, f, g, h, num, r1, r2):
        out = np.zeros((self.N, self.N), np.complex128)
        f, g, h = _c(f), _c(g), _c(h)
        fn(self.N, _ptr(f), _ptr(g), _ptr(h), num, r1, r2, _ptr(out))
        return out

    def i1(self, f, g, h):
        q = self.q.contents
        return self._int(lib().orc_i1, f, g, h, q.n1, q.i1r1, q.i1r2)

    def i4(self, f, g, h):
        q = self.q.contents
        return self._int(lib().orc_i1, f, g, h, q.n4, q.i4r1, q.i4r2)

    def i2(self, f, g, h):
        q = self.q.contents
        return self._int(lib().orc_i2, f, g, h, q.n2, q.i2r1, q.i2r2)

    def i3(self, f, g, h):
        q = self.q.contents
        return self._int(lib().orc_i3, f, g, h, q.n3, q.i3r1, q.i3r2)

    def cc(self, W):
        W = _c(W); out = np.zeros_like(W)
        lib().orc_cc(self.q, _ptr(W), _ptr(out)); return out

    def cd(self, W):
        W = _c(W); out = np.zeros_like(W)
        lib().orc_cd(self.q, _ptr(W), _ptr(out)); return out

    def collision_step(self, W, dt, B=(0.0, 0.0, 0.0), rk4=False):
        W = _c(W); out = np.zeros_like(W); Bv = _r(B)
        fn = lib().orc_collision_step_rk4 if rk4 else lib().orc_collision_step
        fn(self.q, _ptr(W), C.c_double(dt), _ptr(Bv), _ptr(out)); return out

    def inhom_step(self, W, h, dt, Bext=None, bc="periodic"):
        W = _r(W); n = W.shape[0]; out = np.zeros_like(W)
        Bext = _r(np.zeros((n, 3)) if Bext is None else Bext)
        lib().orc_inhom_step(self.q, 0 if bc == "periodic" else 1, n, _ptr(W), C.c_double(h), C.c_double(dt), _ptr(Bext), _ptr(out))
        return out

    def inhom_step_maxwell(self, W, h, dt, lam, WL, WR, Bext=None):
        W = _r(W); n = W.shape[0]; out = np.zeros_like(W)
        Bext = _r(np.zeros((n, 3)) if Bext is None else Bext)
        WL, WR = _r(WL), _r(WR)
        lib().orc_inhom_step_maxwell(self.q, n, _ptr(W), C.c_double(h), C.c_double(dt), C.c_double(lam),
                                     _ptr(WL), _ptr(WR), _ptr(Bext), _ptr(out))
        return out

    def simulation_homogeneous(self, W0, dt, numsteps, B=(0.0, 0.0, 0.0)):
        W0 = _r(W0); out = np.zeros((numsteps,) + W0.shape); Bv = _r(B)
        lib().orc_simulation_homogeneous(self.q, _ptr(W0), C.c_double(dt), numsteps, _ptr(Bv), _ptr(out))
        return out


def i2_raw(N, f, g, h, psiR1, psiR2):
    """I2 with caller-supplied tables (as test/I2_test.c builds them)."""
    f, g, h, r1, r2 = _c(f), _c(g), _c(h), _r(psiR1), _r(psiR2)
    out = np.zeros((N, N), np.complex128)
    lib().orc_i2(N, _ptr(f), _ptr(g), _ptr(h), r1.shape[0], _ptr(r1), _ptr(r2), _ptr(out))
    return out


def lgwt(M, a, b):
    x = np.zeros(M); w = np.zeros(M)
    lib().orc_lgwt(M, C.c_double(a), C.c_double(b), _ptr(x), _ptr(w))
    return x, w


def to_fourier(Wv):
    Wv = _r(Wv); N = Wv.shape[-1]; cells = Wv.size // (4 * N * N)
    out = np.zeros(Wv.shape, np.complex128)
    lib().orc_to_fourier(N, cells, _ptr(Wv), _ptr(out)); return out


def from_fourier(Wf):
    Wf = _c(Wf); N = Wf.shape[-1]; cells = Wf.size // (4 * N * N)
    out = np.zeros(Wf.shape, np.float64)
    lib().orc_from_fourier(N, cells, _ptr(Wf), _ptr(out)); return out


def slope_periodic(h, dt, A, Un):
    Un = _r(Un); out = np.zeros_like(Un)
    lib().orc_slope_periodic(C.c_double(h), C.c_double(dt), C.c_double(A), len(Un), _ptr(Un), _ptr(out)); return out


def slope_dirichlet(h, dt, A, Un):
    Un = _r(Un); out = np.zeros_like(Un)
    lib().orc_slope_dirichlet(C.c_double(h), C.c_double(dt), C.c_double(A), len(Un), _ptr(Un), _ptr(out)); return out


def slope_maxwell(h, dt, A, lam, fluxL, fluxR, UL, UR, Un):
    """Un: (N, m) cell-major, i.e. the upstream m x N matrix Un[i + m*j]."""
    A, UL, UR, Un = _r(A), _r(UL), _r(UR), _r(Un)
    out = np.zeros_like(Un)
    lib().orc_slope_maxwell(C.c_double(h), C.c_double(dt), len(A), _ptr(A), Un.shape[0], C.c_double(lam),
                            C.c_double(fluxL), C.c_double(fluxR), _ptr(UL), _ptr(UR), _ptr(Un), _ptr(out))
    return out


# ---------------------------------------------------------------------------
# The upstream sources themselves (N = 32), when built.

_ref = None


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            return None
        L = C.CDLL(REF_SO)
        L.ref_ctx_create.restype = C.c_void_p
        L.ref_ctx_create.argtypes = [C.c_uint, C.c_uint, C.c_double, C.c_double]
        for n in ("ref_ctx_free", "ref_table_num", "ref_table_copy", "ref_i1", "ref_i2", "ref_i3", "ref_cc", "ref_cd",
                  "ref_collision_step", "ref_inhom_step", "ref_inhom_step_maxwell", "ref_sim_hom",
                  "ref_sim_inhom_periodic"):
            getattr(L, n).argtypes = None
        L.ref_table_num.restype = C.c_uint
        L.CalculateRightwardFlux.restype = C.c_double
        L.CalculateLeftwardFlux.restype = C.c_double
        _ref = L
    return _ref


class Ref:
    """The upstream C functions at N = 32 with tables from the upstream builders."""
    N = 32

    def __init__(self, J, M, L, R):
        self.J, self.M, self.L, self.R = J, M, L, R
        self.h = C.c_void_p(ref_lib().ref_ctx_create(J, M, L, R))

    def __del__(self):
        if getattr(self, "h", None) is not None and _ref is not None:
            _ref.ref_ctx_free(self.h)
            self.h = None

    def table(self, which, part):
        N, P = self.N, 2 * self.N
        num = ref_lib().ref_table_num(self.h, which)
        shapes = {(1, 1): (num, P, P), (1, 2): (num, N, N), (2, 1): (num, N, N), (2, 2): (num, N, N),
                  (3, 1): (num, N, N, 2), (3, 2): (num, P, P), (4, 1): (num, P, P), (4, 2): (num, N, N)}
        a = np.zeros(shapes[(which, part)])
        ref_lib().ref_table_copy(self.h, which, part, _ptr(a))
        return a.view(np.complex128)[..., 0] if which == 3 and part == 1 else a

    def _int(self, fn, *args):
        args = [_c(a) for a in args]
        out = np.zeros((self.N, self.N), np.complex128)
        fn(self.h, *[_ptr(a) for a in args], _ptr(out))
        return out

    def i1(self, f, g, h):
        return self._int(lambda hh, *p: ref_lib().ref_i1(hh, 1, *p), f, g, h)

    def i4(self, f, g, h):
        return self._int(lambda hh, *p: ref_lib().ref_i1(hh, 4, *p), f, g, h)

    def i2(self, f, g, h):
        return self._int(ref_lib().ref_i2, f, g, h)

    def i3(self, f, g, h):
        return self._int(ref_lib().ref_i3, f, g, h)

    def cc(self, W):
        W = _c(W); out = np.zeros_like(W); ref_lib().ref_cc(self.h, _ptr(W), _ptr(out)); return out

    def cd(self, W):
        W = _c(W); out = np.zeros_like(W); ref_lib().ref_cd(self.h, _ptr(W), _ptr(out)); return out

    def collision_step(self, W, dt, B=(0.0, 0.0, 0.0)):
        W = _c(W); out = np.zeros_like(W); Bv = _r(B)
        ref_lib().ref_collision_step(self.h, _ptr(W), C.c_double(dt), _ptr(Bv), _ptr(out)); return out

    def inhom_step(self, W, h, dt, Bext=None, bc="periodic"):
        W = _r(W); n = W.shape[0]; out = np.zeros_like(W)
        Bext = _r(np.zeros((n, 3)) if Bext is None else Bext)
        ref_lib().ref_inhom_step(self.h, 0 if bc == "periodic" else 1, C.c_uint(n), C.c_double(self.L), _ptr(W),
                                 C.c_double(h), C.c_double(dt), _ptr(Bext), _ptr(out))
        return out

    def inhom_step_maxwell(self, W, h, dt, lam, WL, WR, Bext=None):
        W = _r(W); n = W.shape[0]; out = np.zeros_like(W)
        Bext = _r(np.zeros((n, 3)) if Bext is None else Bext)
        WL, WR = _r(WL), _r(WR)
        ref_lib().ref_inhom_step_maxwell(self.h, C.c_uint(n), C.c_double(self.L), _ptr(W), C.c_double(h), C.c_double(dt),
                                         C.c_double(lam), _ptr(WL), _ptr(WR), _ptr(Bext), _ptr(out))
        return out

    def simulation_homogeneous(self, W0, dt, numsteps, B=(0.0, 0.0, 0.0)):
        W0 = _r(W0); out = np.zeros((numsteps,) + W0.shape); Bv = _r(B)
        ref_lib().ref_sim_hom(self.h, _ptr(W0), C.c_double(dt), C.c_uint(numsteps), _ptr(Bv), _ptr(out)); return out

    def sim_inhom_periodic(self, W0, h, dt, steps, Bext=None):
        """SimulationInhomogeneousPeriodic over `steps` Strang steps: frames
        (steps + 1, cells, 4, N, N), frame 0 = W0."""
        W0 = _r(W0); n = W0.shape[0]; out = np.zeros((steps + 1,) + W0.shape)
        Bext = _r(np.zeros((n, 3)) if Bext is None else Bext)
        ref_lib().ref_sim_inhom_periodic(self.h, C.c_uint(n), C.c_double(self.L), _ptr(W0), C.c_double(h), C.c_double(dt),
                                         C.c_uint(steps + 1), _ptr(Bext), _ptr(out))
        return out


def ref_to_fourier(Wv):
    Wv = _r(Wv); out = np.zeros(Wv.shape, np.complex128)
    ref_lib().ref_to_fourier(_ptr(Wv), _ptr(out)); return out


def diagnostics(W, L):
    """Moments, eigenvalue bounds and Fermi-Dirac entropy per cell, restating
    visualization/wignerMoments.m:15-37 and visualization/entropy.m in numpy
    (float64).  W: (ncells, 4, N, N) velocity space; columns as qbgpu.DIAGNOSTICS."""
    W = np.asarray(W, dtype=np.float64)
    N = W.shape[-1]
    dv = 2.0 * L / N
    v = np.where(np.arange(N) < N // 2, np.arange(N), np.arange(N) - N) * dv
    vx, vy = np.meshgrid(v, v, indexing="ij")        # [l, k]: l is v_x
    out = np.zeros((W.shape[0], 10))
    for i, w in enumerate(W):
        t = w[0]
        r = np.sqrt(w[1] ** 2 + w[2] ** 2 + w[3] ** 2)
        ux, uy = (vx * t).sum() / t.sum(), (vy * t).sum() / t.sum()
        e = (0.5 * ((vx - ux) ** 2 + (vy - uy) ** 2) * t).sum() / t.sum()

        def S(p):
            ok = (p > 0) & (p < 1)
            q = p[ok]
            return -(q * np.log(q) + (1 - q) * np.log1p(-q)).sum()
        out[i] = [w[0].sum() * dv * dv, w[1].sum() * dv * dv, w[2].sum() * dv * dv, w[3].sum() * dv * dv,
                  ux, uy, e, (t - r).min(), (t + r).max(), (S(t - r) + S(t + r)) * dv * dv]
    return out



# ---------------------------------------------------------------------------
# Fermi-Dirac equilibrium and quantum relative entropy (test oracle), restating
# visualization/asymptoticFD.m, calculateFDparams.m, createFD.m and
# relentropy.m, and the relative-entropy / distance loops of
# visualization/visualizeHomBoltzmann.m:116-148, in numpy/scipy (float64).

def _vgrid(N, L):
    return np.where(np.arange(N) < N // 2, np.arange(N), np.arange(N) - N) * (2.0 * L / N)


def fd_params(lam, en):
    """calculateFDparams.m: (beta, mu) of the 2-D Fermi-Dirac distribution with
    spin densities lam (2,) and normalised energy en, by nonlinear least
    squares on (z_up, z_dn, beta) from (1, 1, 1), retried from beta = 0.5 when
    the residual stays above 1e-4 (as the Matlab does); returns (beta, mu, residual)."""
    from scipy.optimize import least_squares
    from scipy.special import spence
    lam = np.asarray(lam, dtype=np.float64)
    en_t = en * lam.sum()

    def li2(x):                       # Li_2(x) = spence(1 - x)
        return spence(1.0 - x)

    def F(x):
        zu, zd, b = x
        rho = lambda z: 2 * np.pi / b * np.log1p(z)
        ene = lambda z: -2 * np.pi / b ** 2 * li2(-z)
        return np.array([rho(zu) - lam[0], rho(zd) - lam[1], ene(zu) + ene(zd) - en_t])

    def Jac(x):
        zu, zd, b = x
        rho = lambda z: 2 * np.pi / b * np.log1p(z)
        ene = lambda z: -2 * np.pi / b ** 2 * li2(-z)
        dr = lambda z: (2 * np.pi / (b * (1 + z)), -rho(z) / b)
        de = lambda z: (rho(z) / (b * z), -2 * ene(z) / b)
        return np.array([[dr(zu)[0], 0, dr(zu)[1]], [0, dr(zd)[0], dr(zd)[1]], [de(zu)[0], de(zd)[0], de(zu)[1] + de(zd)[1]]])

    best = None
    for b0 in (1.0, 0.5):
        r = least_squares(F, [1.0, 1.0, b0], jac=Jac, bounds=([1e-300, 1e-300, 1e-300], [np.inf, np.inf, np.inf]),
                          ftol=1e-15, xtol=1e-15, gtol=1e-15, max_nfev=2000)
        md = float(np.linalg.norm(F(r.x)))
        if best is None or md < best[2]:
            best = (r.x, None, md)
        if md <= 1e-4:
            break
    x, _, md = best
    beta = x[2]
    return beta, np.log(x[:2]) / beta, md


def asymptotic_fd(W, L):
    """asymptoticFD.m per cell: W (ncells, 4, N, N) -> (WFD of the same shape,
    params (ncells, 9) = beta, mu_1, mu_2, u_x, u_y, n_x, n_y, n_z, residual)
    with n the unit spin direction of the larger density eigenvalue."""
    W = np.asarray(W, dtype=np.float64)
    N = W.shape[-1]
    d = diagnostics(W, L)
    v = _vgrid(N, L)
    vx, vy = np.meshgrid(v, v, indexing="ij")        # [l, k]: l is v_x
    out = np.zeros_like(W)
    par = np.zeros((W.shape[0], 9))
    for i in range(W.shape[0]):
        w = d[i, :4]
        r = np.sqrt(w[1] ** 2 + w[2] ** 2 + w[3] ** 2)
        lam = np.array([w[0] - r, w[0] + r])         # eig of pauliToMatrix(w), ascending
        n = w[1:] / r if r > 0 else np.array([0.0, 0.0, -1.0])
        beta, mu, md = fd_params(lam, d[i, 6])
        ux, uy = d[i, 4], d[i, 5]
        e = 0.5 * ((vx - ux) ** 2 + (vy - uy) ** 2)
        f1 = 1.0 / (np.exp(beta * (e - mu[0])) + 1.0)
        f2 = 1.0 / (np.exp(beta * (e - mu[1])) + 1.0)
        out[i, 0] = 0.5 * (f1 + f2)
        for c in range(3):
            out[i, c + 1] = 0.5 * (f2 - f1) * n[c]
        par[i] = [beta, mu[0], mu[1], ux, uy, n[0], n[1], n[2], md]
    return out, par


def relative_entropy(W, WFD, L):
    """per cell (KL, distFD): the quantum relative entropy (relentropy.m) of
    W(v) to WFD(v) summed over points with WFD_0(v) > 1e-6, times dv^2, and
    sum_j ||W_j - WFD_j||_1 dv^2 with the Matlab matrix 1-norm (largest column
    sum; a column is a fixed v_x)."""
    W = np.asarray(W, dtype=np.float64)
    WFD = np.asarray(WFD, dtype=np.float64)
    N = W.shape[-1]
    dv2 = (2.0 * L / N) ** 2
    eps = np.finfo(np.float64).eps
    sx = np.array([[0, 1], [1, 0]], complex)
    sy = np.array([[0, -1j], [1j, 0]], complex)
    sz = np.array([[1, 0], [0, -1]], complex)
    out = np.zeros((W.shape[0], 2))
    for i in range(W.shape[0]):
        kl = 0.0
        for l in range(N):
            for k in range(N):
                if not WFD[i, 0, l, k] > 1e-6:
                    continue
                a = W[i, :, l, k]
                b = WFD[i, :, l, k]
                rho = a[0] * np.eye(2) + a[1] * sx + a[2] * sy + a[3] * sz
                tau = b[0] * np.eye(2) + b[1] * sx + b[2] * sy + b[3] * sz
                mu, U = np.linalg.eigh(rho)
                nu, V = np.linalg.eigh(tau)
                mu = np.where(mu <= 0, eps, mu)
                mu = np.where(mu >= 1, 1 - eps, mu)
                nu = np.where(nu <= 0, eps, nu)
                nu = np.where(nu >= 1, 1 - eps, nu)
                Wm = U.conj().T @ V
                log_tau = Wm @ np.diag(np.log(nu)) @ Wm.conj().T
                log_1tau = Wm @ np.diag(np.log(1 - nu)) @ Wm.conj().T
                r = np.diag(mu)
                val = np.trace(r @ (np.diag(np.log(mu)) - log_tau)) + np.trace((np.eye(2) - r) @ (np.diag(np.log(1 - mu)) - log_1tau))
                kl += val.real * dv2
        dist = sum(np.abs(W[i, j] - WFD[i, j]).sum(axis=1).max() * dv2 for j in range(4))
        out[i] = [kl, dist]
    return out

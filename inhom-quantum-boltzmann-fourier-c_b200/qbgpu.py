"""Python binding of libqbgpu (ctypes) — used by the tests, the smoke check and bench.py.

Two surfaces:
  * ``Upstream`` — the upstream C API exactly as a C caller sees it (host
    buffers, struct pointers; N_GRID = 32 in lib/libqbgpu.so).  This is the
    drop-in boundary: the same entry points test/*_test.c and main_*.c call.
  * ``Quad`` / ``Workspace`` + module functions — the batched extension API of
    include/qbgpu.h on device tensors (torch CUDA tensors are used only as
    device memory and for the stream handle).

The module never computes anything on the CPU: every operator is a call into
the CUDA library, and loading fails loudly when the library is missing.

Layouts (upstream): velocity-space cell = 4 real N x N grids (float64),
Fourier-space cell = 4 complex N x N grids (complex128), element (l, k) at
[..., l, k] == upstream index k + N*l; cells consecutive.
"""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
N_GRID = 32

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p


def library_path(n_grid=N_GRID):
    name = "libqbgpu.so" if n_grid == 32 else f"libqbgpu_n{n_grid}.so"
    return os.path.join(LIB_DIR, name)


_libs = {}


# int exchange(double *ext, int ncells, void *stream, void *user) of qb_sharded_step
HALO_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p)


def lib(n_grid=N_GRID):
    """Load libqbgpu (raises if it has not been built)."""
    if n_grid in _libs:
        return _libs[n_grid]
    path = library_path(n_grid)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python inhom-quantum-boltzmann-fourier-c_b200/build.py`")
    L = C.CDLL(path)
    L.qb_last_error.restype = C.c_char_p
    L.qb_quad_create.restype = _vp
    L.qb_quad_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
    L.qb_quad_free.argtypes = [_vp]
    L.qb_workspace_create.restype = _vp
    L.qb_workspace_create.argtypes = [C.c_int]
    L.qb_workspace_free.argtypes = [_vp]
    L.qb_workspace_set_precision.argtypes = [_vp, C.c_int]
    L.qb_workspace_precision.argtypes = [_vp]
    L.qb_workspace_set_conservation.argtypes = [_vp, C.c_int]
    L.qb_workspace_i3_forms.argtypes = [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.c_int]
    L.qb_collision_operators.argtypes = [_vp, _vp, C.c_int, _vp, C.c_int, _vp, _vp, _vp]
    L.qb_collision_step.argtypes = [_vp, _vp, C.c_int, _vp, _vp, C.c_double, _vp, C.c_int, _vp]
    L.qb_inhom_step.argtypes = [_vp, _vp, C.c_int, _vp, _vp, C.c_double, C.c_double, _vp, C.c_int, _vp]
    L.qb_inhom_step_maxwell.argtypes = [_vp, _vp, C.c_int, _vp, _vp, C.c_double, C.c_double, C.c_double, _vp, _vp, _vp, _vp]
    L.qb_to_fourier.argtypes = [C.c_int, C.c_int, _vp, _vp, _vp]
    L.qb_from_fourier.argtypes = [C.c_int, C.c_int, _vp, _vp, _vp]
    L.qb_integral.argtypes = [_vp, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp]
    L.qb_transport.argtypes = [C.c_int, C.c_double, C.c_int, _vp, _vp, C.c_double, C.c_double, C.c_int, _vp]
    L.qb_fourier_collision.argtypes = [_vp, _vp, C.c_int, _vp, _vp, C.c_double, _vp]
    L.qb_launch_count.restype = C.c_long
    L.qb_workspace_graph_replays.restype = C.c_long
    L.qb_workspace_graph_replays.argtypes = [_vp]
    L.qb_workspace_set_i3_variant.argtypes = [_vp, C.c_int]
    L.qb_workspace_device_errors.argtypes = [_vp]
    L.qb_umma_selftest.argtypes = [_vp, _vp, _vp, _vp]
    L.qb_batch_schedules.argtypes = [C.c_char_p, C.c_int]
    L.qb_sharded_step.argtypes = [_vp, _vp, C.c_int, _vp, _vp, C.c_double, C.c_double, _vp, HALO_FN, _vp, _vp]
    L.qb_fp64_peak_tflops.restype = C.c_double
    L.qb_simulate_record.restype = C.c_long
    L.qb_simulate_record.argtypes = [_vp, _vp, C.c_int, _vp, C.c_double, C.c_double, C.c_uint, _vp, C.c_int, C.c_uint, C.c_char_p, _vp]
    L.qb_diagnostics.argtypes = [C.c_int, C.c_double, C.c_int, _vp, _vp, _vp]
    L.qb_homogeneous_batch.argtypes = [C.c_int, _vp, _vp, _vp, C.c_double, C.c_uint, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _vp]
    L.qb_homogeneous_batch_ex.argtypes = [C.c_int, _vp, _vp, _vp, C.c_double, C.c_uint, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                          C.c_double, _vp]
    L.qb_fermi_dirac_equilibrium.argtypes = [C.c_int, C.c_double, C.c_int, _vp, _vp, _vp, _vp]
    L.qb_relative_entropy.argtypes = [C.c_int, C.c_double, C.c_int, _vp, _vp, _vp, _vp]
    L.qb_fno_create.restype = _vp
    L.qb_fno_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong]
    L.qb_fno_free.argtypes = [_vp]
    L.qb_fno_num_params.restype = C.c_long
    L.qb_fno_num_params.argtypes = [_vp]
    L.qb_fno_grid_size.argtypes = [_vp]
    L.qb_fno_get_params.argtypes = [_vp, _vp]
    L.qb_fno_set_params.argtypes = [_vp, _vp]
    L.qb_fno_set_scale.argtypes = [_vp, _vp]
    L.qb_fno_set_input_scale.argtypes = [_vp, _vp]
    L.qb_fno_forward.argtypes = [_vp, C.c_int, _vp, _vp, _vp]
    L.qb_fno_set_tensor_cores.argtypes = [_vp, C.c_int]
    L.qb_fno_device_errors.argtypes = [_vp]
    L.qb_fno_gradients.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp]
    L.qb_fno_train_step.argtypes = [_vp, C.c_int, _vp, _vp, C.c_float, _vp, _vp]
    L.qb_surrogate_create.restype = _vp
    L.qb_surrogate_create.argtypes = [_vp, C.c_double, C.c_uint]
    L.qb_surrogate_free.argtypes = [_vp]
    L.qb_surrogate_inhom_step.argtypes = [_vp, _vp, _vp, C.c_int, _vp, _vp, C.c_double, C.c_double, _vp, _vp]
    L.qb_surrogate_stats.argtypes = [_vp, _vp, _vp, _vp]
    L.CalculateRightwardFlux.restype = C.c_double
    L.CalculateLeftwardFlux.restype = C.c_double
    _libs[n_grid] = L
    return L


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed: {lib().qb_last_error().decode()}")


# ---------------------------------------------------------------------------
# batched extension API on device tensors

def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("a CUDA device is required")
    return torch


def _stream():
    return _vp(_torch().cuda.current_stream().cuda_stream)


def _ptr(t):
    assert t.is_cuda and t.is_contiguous()
    return _vp(t.data_ptr())


class Quad:
    """Device quadrature tables (FourierI1..I4) for grid size N."""

    def __init__(self, N, J, M, L, R):
        self.N, self.J, self.M, self.L, self.R = N, J, M, L, R
        self.h = lib().qb_quad_create(N, J, M, L, R)
        if not self.h:
            raise RuntimeError(f"qb_quad_create failed: {lib().qb_last_error().decode()}")
        self._free = lib().qb_quad_free

    def __del__(self):
        # the bound function is kept on the object: module globals may already
        # be gone when this runs at interpreter exit
        if getattr(self, "h", None) and getattr(self, "_free", None):
            self._free(self.h)
            self.h = None


class Workspace:
    """Device scratch for one grid size (grows on demand).

    precision=64 evaluates the collision operator in FP64 (the upstream
    arithmetic); precision=32 selects the FP32 form (FP64 state and update,
    FP32 spectra, tables and FFTs).  conserve=True restores the trace
    component's mass, momentum and energy after each velocity-space collision."""

    def __init__(self, N, precision=64, conserve=False):
        self.N = N
        self.h = lib().qb_workspace_create(N)
        if not self.h:
            raise RuntimeError(f"qb_workspace_create failed: {lib().qb_last_error().decode()}")
        self._free = lib().qb_workspace_free
        if precision != 64:
            self.set_precision(precision)
        if conserve:
            _check(lib().qb_workspace_set_conservation(self.h, 1), "qb_workspace_set_conservation")

    def set_precision(self, bits):
        _check(lib().qb_workspace_set_precision(self.h, bits), "qb_workspace_set_precision")

    @property
    def precision(self):
        return lib().qb_workspace_precision(self.h)

    def i3_forms(self, reset=False):
        """(cells whose I3 sums ran in the real form, all cells) evaluated so
        far through this workspace in FP32 (zero in FP64)."""
        r, a = C.c_longlong(), C.c_longlong()
        _check(lib().qb_workspace_i3_forms(self.h, C.byref(r), C.byref(a), 1 if reset else 0), "qb_workspace_i3_forms")
        return r.value, a.value

    def set_i3_variant(self, variant):
        """0: FFT kernels for the I3 sums; 1: DFT-GEMMs on the tensor cores
        (FP32 form at N = 16)."""
        _check(lib().qb_workspace_set_i3_variant(self.h, variant), "qb_workspace_set_i3_variant")

    def device_errors(self):
        """device error word since the last call (0: no bounded wait ran out)"""
        return lib().qb_workspace_device_errors(self.h)

    @property
    def graph_replays(self):
        """Strang steps of inhom_step served by relaunching a captured CUDA graph."""
        return lib().qb_workspace_graph_replays(self.h)

    def __del__(self):
        if getattr(self, "h", None) and getattr(self, "_free", None):
            self._free(self.h)
            self.h = None


def collision_operators(ws, q, W, parts=3):
    """(Cc, Cd) of Fourier states W: complex128 CUDA tensor (ncells, 4, N, N)."""
    torch = _torch()
    n = W.shape[0]
    cc = torch.empty_like(W) if parts & 1 else None
    cd = torch.empty_like(W) if parts & 2 else None
    _check(lib().qb_collision_operators(ws.h, q.h, n, _ptr(W), parts, _ptr(cc) if cc is not None else None,
                                        _ptr(cd) if cd is not None else None, _stream()), "qb_collision_operators")
    return cc, cd


def collision_step(ws, q, W, dt, B=None, rk4=False, out=None):
    torch = _torch()
    n = W.shape[0]
    if B is None:
        B = torch.zeros((n, 3), dtype=torch.float64, device=W.device)
    out = torch.empty_like(W) if out is None else out
    _check(lib().qb_collision_step(ws.h, q.h, n, _ptr(W), _ptr(B), dt, _ptr(out), 1 if rk4 else 0, _stream()), "qb_collision_step")
    return out


def inhom_step(ws, q, W, h, dt, Bext=None, bc="periodic", out=None):
    """One Strang step; W: float64 CUDA tensor (ncells, 4, N, N)."""
    torch = _torch()
    n = W.shape[0]
    if Bext is None:
        Bext = torch.zeros((n, 3), dtype=torch.float64, device=W.device)
    out = torch.empty_like(W) if out is None else out
    _check(lib().qb_inhom_step(ws.h, q.h, n, _ptr(W), _ptr(out), h, dt, _ptr(Bext), 0 if bc == "periodic" else 1, _stream()),
           "qb_inhom_step")
    return out


def batch_schedules():
    """the schedules tuned so far by homogeneous_batch (list of dicts)"""
    import json
    n = lib().qb_batch_schedules(None, 0)
    buf = C.create_string_buffer(n + 1)
    lib().qb_batch_schedules(buf, n + 1)
    return json.loads(buf.value.decode())


def homogeneous_batch(states, dt, steps, B=None, rk4=True, J=16, M=16, L=6.0, R=3.75, precision=64):
    """Advance independent homogeneous instances of possibly different grid
    sizes in place: states is a list of complex128 CUDA tensors (4, N_i, N_i)
    (Fourier space), B an optional (ninst, 3) array; `steps` collision steps
    of size dt (RK4 or midpoint), one batched launch sequence per grid size;
    precision 64 or 32 (the FP32 form)."""
    n = len(states)
    sizes = (C.c_int * n)(*[int(s.shape[-1]) for s in states])
    ptrs = (C.c_void_p * n)(*[s.data_ptr() for s in states])
    for s in states:
        assert s.is_cuda and s.is_contiguous() and s.dtype == _torch().complex128
    Bh = None
    if B is not None:
        Bh = np.ascontiguousarray(np.asarray(B, dtype=np.float64).reshape(n, 3))
    _check(lib().qb_homogeneous_batch_ex(n, sizes, ptrs, Bh.ctypes.data_as(_vp) if Bh is not None else None, dt, steps,
                                         1 if rk4 else 0, precision, J, M, L, R, _stream()), "qb_homogeneous_batch_ex")
    return states


def transport(W, L, h, dt, bc="periodic", out=None):
    """One limiter step (qb_transport) of step dt on every x-line of the cells
    of W (float64 CUDA tensor (ncells, 4, N, N)) in a box of half-width L."""
    out = _torch().empty_like(W) if out is None else out
    N = W.shape[-1]
    _check(lib().qb_transport(N, L, W.shape[0], _ptr(W), _ptr(out), h, dt, 0 if bc == "periodic" else 1, _stream()), "qb_transport")
    return out


def fourier_collision(ws, q, W, dt, Bext=None):
    """The collision part of a Strang step in place on velocity-space cells
    W (qb_fourier_collision); returns W."""
    _check(lib().qb_fourier_collision(ws.h, q.h, W.shape[0], _ptr(W), _ptr(Bext) if Bext is not None else None, dt, _stream()),
           "qb_fourier_collision")
    return W


# ---------------------------------------------------------------------------
# learned surrogate of the collision operator (qb_fno_*, qb_surrogate_*)

def _features_np(W):
    """the 14 network input features of velocity-space states W (numpy,
    (B, 4, N, N)): w_c, then w_i w_j for i <= j"""
    W = np.asarray(W, dtype=np.float64).reshape(W.shape[0], 4, -1)
    f = [W[:, c] for c in range(4)] + [W[:, i] * W[:, j] for i in range(4) for j in range(i, 4)]
    return np.stack(f, axis=1)


class FNO:
    """Fourier neural operator W -> C~[W] ~ Cc + Cd on N x N velocity-space
    cells (qb_fno_*): FP32 weights on the device, forward, gradients and Adam
    steps in the library's own kernels."""

    NFEAT = 14

    def __init__(self, N, width=32, modes=8, layers=4, seed=0):
        self.N, self.width, self.modes, self.layers = N, width, modes, layers
        self.h = lib().qb_fno_create(N, width, modes, layers, seed)
        if not self.h:
            raise RuntimeError(f"qb_fno_create failed: {lib().qb_last_error().decode()}")
        self._free = lib().qb_fno_free
        self.scale = np.ones(4)
        self.input_scale = np.ones(self.NFEAT)

    def __del__(self):
        if getattr(self, "h", None) and getattr(self, "_free", None):
            self._free(self.h)
            self.h = None

    @property
    def num_params(self):
        return int(lib().qb_fno_num_params(self.h))

    def get_params(self):
        out = np.empty(self.num_params, dtype=np.float32)
        _check(lib().qb_fno_get_params(self.h, out.ctypes.data_as(_vp)), "qb_fno_get_params")
        return out

    def set_params(self, theta):
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        assert theta.size == self.num_params
        _check(lib().qb_fno_set_params(self.h, theta.ctypes.data_as(_vp)), "qb_fno_set_params")

    def set_scale(self, scale):
        s = np.ascontiguousarray(scale, dtype=np.float64)
        assert s.size == 4
        _check(lib().qb_fno_set_scale(self.h, s.ctypes.data_as(_vp)), "qb_fno_set_scale")
        self.scale = s.copy()

    def set_input_scale(self, scale):
        s = np.ascontiguousarray(scale, dtype=np.float64)
        assert s.size == self.NFEAT
        _check(lib().qb_fno_set_input_scale(self.h, s.ctypes.data_as(_vp)), "qb_fno_set_input_scale")
        self.input_scale = s.copy()

    def fit_scales(self, X, Y):
        """input scales = 1 / RMS of each feature over the states X, output
        scales = RMS of each Pauli component of the targets Y (numpy or CUDA
        tensors (B, 4, N, N))"""
        X = X.cpu().numpy() if hasattr(X, "cpu") else np.asarray(X)
        Y = Y.cpu().numpy() if hasattr(Y, "cpu") else np.asarray(Y)
        f = _features_np(X)
        rx = np.sqrt(np.mean(f * f, axis=(0, 2)))
        ry = np.sqrt(np.mean(np.asarray(Y, dtype=np.float64).reshape(Y.shape[0], 4, -1) ** 2, axis=(0, 2)))
        self.set_input_scale(1.0 / np.where(rx > 0, rx, 1.0))
        self.set_scale(np.where(ry > 0, ry, 1.0))

    def set_tensor_cores(self, on=True):
        """pointwise channel maps on the tensor cores (BF16 operands, FP32
        accumulation) when on; FP32 on the CUDA cores otherwise (the default)"""
        _check(lib().qb_fno_set_tensor_cores(self.h, 1 if on else 0), "qb_fno_set_tensor_cores")

    def device_errors(self):
        """nonzero when a tensor-core MMA did not complete within its poll limit"""
        return int(lib().qb_fno_device_errors(self.h))

    def forward(self, W, out=None):
        """C~[W] for float64 CUDA states W (B, 4, N, N)"""
        out = _torch().empty_like(W) if out is None else out
        _check(lib().qb_fno_forward(self.h, W.shape[0], _ptr(W), _ptr(out), _stream()), "qb_fno_forward")
        return out

    def gradients(self, W, target):
        """(loss, flat float32 gradient) of mean((y - target / scale)^2)"""
        g = np.empty(self.num_params, dtype=np.float32)
        loss = C.c_double()
        _check(lib().qb_fno_gradients(self.h, W.shape[0], _ptr(W), _ptr(target), g.ctypes.data_as(_vp), C.byref(loss), _stream()),
               "qb_fno_gradients")
        return loss.value, g

    def train_step(self, W, target, lr):
        loss = C.c_double()
        _check(lib().qb_fno_train_step(self.h, W.shape[0], _ptr(W), _ptr(target), float(lr), C.byref(loss), _stream()),
               "qb_fno_train_step")
        return loss.value


def mixture_cells(N, L, nseeds, seed):
    """one velocity-space cell per seed, numpy (nseeds, 4, N, N): seed k's
    Gaussian mixture at x-cell k mod 4 of a 4-cell box, so that the mixture
    amplitudes vary as well"""
    return np.stack([gaussian_mixture_state(N, L, seed=seed + k, ncells=4)[k % 4] for k in range(nseeds)])


def relaxation_pairs(ws, q, W, samples, every=5, dt=0.02):
    """training pairs (W, C[W] = Cc + Cd), both float64 CUDA tensors in
    velocity space: the states W (B, 4, N, N) and every `every`-th state of
    their spatially homogeneous relaxation (midpoint collision steps of size
    dt), `samples` states per trajectory"""
    torch = _torch()
    Wf = to_fourier(W)
    X, Y = [], []
    for k in range(samples):
        if k:
            for _ in range(every):
                Wf = collision_step(ws, q, Wf, dt)
        cc, cd = collision_operators(ws, q, Wf)
        X.append(from_fourier(Wf))
        Y.append(from_fourier(cc + cd))
    return torch.cat(X), torch.cat(Y)


def random_rotations(n, generator):
    """n uniformly distributed 3 x 3 rotation matrices (float64, CPU): unit
    quaternions from normal variates"""
    import torch
    qv = torch.randn((n, 4), dtype=torch.float64, generator=generator)
    a, b, c, d = (qv / qv.norm(dim=1, keepdim=True)).unbind(1)
    return torch.stack([
        torch.stack([a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)], 1),
        torch.stack([2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)], 1),
        torch.stack([2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d], 1)], 1)


def rotate_spin(W, Rm):
    """the Pauli vector components (1..3) of states or operators W (B, 4, N, N)
    rotated by the matrices Rm (B, 3, 3); component 0 is unchanged"""
    import torch
    out = W.clone()
    out[:, 1:4] = torch.einsum("bij,bjkl->bikl", Rm, W[:, 1:4])
    return out


def train_fno(net, X, Y, iters, batch=64, lr=2e-3, seed=0, spin_rotations=False):
    """`iters` Adam steps on random minibatches of the pairs (X, Y) with a
    cosine learning-rate schedule from lr to 0; returns the last loss.
    spin_rotations: rotate the Pauli vector of every pair of a minibatch by a
    random rotation, which maps a pair (W, C[W]) to the pair (RW, RC[W]) =
    (RW, C[RW]) of the same operator (the collision operator commutes with
    global spin rotations)."""
    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    loss = float("nan")
    for it in range(iters):
        idx = torch.randint(0, X.shape[0], (batch,), generator=g).to(X.device)
        a = lr * 0.5 * (1 + math.cos(math.pi * it / iters))
        xb, yb = X[idx], Y[idx]
        if spin_rotations:
            Rm = random_rotations(batch, g).to(X.device)
            xb, yb = rotate_spin(xb, Rm), rotate_spin(yb, Rm)
        loss = net.train_step(xb.contiguous(), yb.contiguous(), a)
    return loss


class Surrogate:
    """Strang steps whose collision half takes the network's C~ with the exact
    operator as judge every `check_every` steps and as per-cell fallback where
    the network's collision increment differed from the exact one by more
    than `tol`, relative L1 (qb_surrogate_inhom_step)."""

    def __init__(self, net, tol=0.3, check_every=10):
        self.net = net                       # the surrogate holds the network: keep it alive
        self.h = lib().qb_surrogate_create(net.h, tol, check_every)
        if not self.h:
            raise RuntimeError(f"qb_surrogate_create failed: {lib().qb_last_error().decode()}")
        self._free = lib().qb_surrogate_free

    def __del__(self):
        if getattr(self, "h", None) and getattr(self, "_free", None):
            self._free(self.h)
            self.h = None

    def step(self, ws, q, W, h, dt, Bext=None, out=None):
        out = _torch().empty_like(W) if out is None else out
        _check(lib().qb_surrogate_inhom_step(self.h, ws.h, q.h, W.shape[0], _ptr(W), _ptr(out), h, dt,
                                             _ptr(Bext) if Bext is not None else None, _stream()), "qb_surrogate_inhom_step")
        return out

    def stats(self):
        """(surrogate cell-steps, exact cell-steps, largest residual of the last check:
        the relative L1 difference of the network's collision increment)"""
        a, b, r = C.c_long(), C.c_long(), C.c_double()
        _check(lib().qb_surrogate_stats(self.h, C.byref(a), C.byref(b), C.byref(r)), "qb_surrogate_stats")
        return a.value, b.value, r.value


def inhom_step_maxwell(ws, q, W, h, dt, lam, WL, WR, Bext=None, out=None):
    torch = _torch()
    n = W.shape[0]
    if Bext is None:
        Bext = torch.zeros((n, 3), dtype=torch.float64, device=W.device)
    out = torch.empty_like(W) if out is None else out
    _check(lib().qb_inhom_step_maxwell(ws.h, q.h, n, _ptr(W), _ptr(out), h, dt, lam, _ptr(WL), _ptr(WR), _ptr(Bext), _stream()),
           "qb_inhom_step_maxwell")
    return out


DIAGNOSTICS = ("w_tr", "w_x", "w_y", "w_z", "u_x", "u_y", "energy", "lam_min", "lam_max", "entropy")


def diagnostics(W, L):
    """per-cell moments, eigenvalue bounds and entropy of velocity-space states
    W (float64 CUDA tensor (ncells, 4, N, N)); returns (ncells, 10) tensor with
    columns DIAGNOSTICS"""
    torch = _torch()
    N, n = W.shape[-1], W.shape[0]
    out = torch.empty((n, len(DIAGNOSTICS)), dtype=torch.float64, device=W.device)
    _check(lib().qb_diagnostics(N, L, n, _ptr(W), _ptr(out), _stream()), "qb_diagnostics")
    return out


FD_PARAMS = ("beta", "mu_1", "mu_2", "u_x", "u_y", "n_x", "n_y", "n_z", "residual")


def fermi_dirac_equilibrium(W, L):
    """Fermi-Dirac states with the conserved moments of each cell of W
    (float64 CUDA tensor (ncells, 4, N, N)); returns (WFD tensor, params numpy
    array (ncells, 9) with columns FD_PARAMS)"""
    torch = _torch()
    N, n = W.shape[-1], W.shape[0]
    WFD = torch.empty_like(W)
    par = np.zeros((n, len(FD_PARAMS)))
    _check(lib().qb_fermi_dirac_equilibrium(N, L, n, _ptr(W), _ptr(WFD), par.ctypes.data_as(_vp), _stream()),
           "qb_fermi_dirac_equilibrium")
    return WFD, par


def relative_entropy(W, WFD, L):
    """(ncells, 2) tensor: quantum relative entropy of W to WFD and the 1-norm distance"""
    torch = _torch()
    N, n = W.shape[-1], W.shape[0]
    out = torch.empty((n, 2), dtype=torch.float64, device=W.device)
    _check(lib().qb_relative_entropy(N, L, n, _ptr(W), _ptr(WFD), _ptr(out), _stream()), "qb_relative_entropy")
    return out


def simulate_record(ws, q, W0, h, dt, numsteps, Bext=None, bc="periodic", record_every=1, path=None):
    """numsteps frames (initial included) from host state W0 (numpy (ncells,4,N,N));
    frames 0, k, 2k, ... appended to `path` in the upstream trajectory format.
    Returns (final state, frames written)."""
    W0 = np.ascontiguousarray(W0, dtype=np.float64)
    n = W0.shape[0]
    Bv = np.ascontiguousarray(np.zeros((n, 3)) if Bext is None else Bext, dtype=np.float64)
    final = np.zeros_like(W0)
    frames = lib().qb_simulate_record(ws.h, q.h, n, W0.ctypes.data, h, dt, numsteps, Bv.ctypes.data,
                                      0 if bc == "periodic" else 1, record_every, path.encode() if path else None,
                                      final.ctypes.data)
    if frames < 0:
        raise RuntimeError(f"qb_simulate_record failed: {lib().qb_last_error().decode()}")
    return final, frames


def to_fourier(Wv):
    torch = _torch()
    N = Wv.shape[-1]
    out = torch.empty(Wv.shape, dtype=torch.complex128, device=Wv.device)
    _check(lib().qb_to_fourier(N, Wv.numel() // (N * N), _ptr(Wv), _ptr(out), _stream()), "qb_to_fourier")
    return out


def from_fourier(Wf):
    torch = _torch()
    N = Wf.shape[-1]
    out = torch.empty(Wf.shape, dtype=torch.float64, device=Wf.device)
    _check(lib().qb_from_fourier(N, Wf.numel() // (N * N), _ptr(Wf), _ptr(out), _stream()), "qb_from_fourier")
    return out


def integral(ws, q, which, f, g, h):
    torch = _torch()
    out = torch.empty_like(f)
    _check(lib().qb_integral(ws.h, q.h, which, _ptr(f), _ptr(g), _ptr(h), _ptr(out), _stream()), "qb_integral")
    return out


# ---------------------------------------------------------------------------
# the upstream C API (host buffers), N_GRID = 32

class quadI1_t(C.Structure):
    _fields_ = [("num", C.c_uint), ("psiR1", _dp), ("psiR2", _dp)]


quadI2_t = quadI1_t
quadI3_t = quadI1_t          # same layout: num + two pointers


class interm_t(C.Structure):   # I1/I2/I3/Cc/Cd/collision/simulationHom interm: one handle
    _fields_ = [("ws", _vp)]


def _inhom_interm_type(n):
    class inhomStepInterm_t(C.Structure):
        _fields_ = [("numVol", C.c_uint), ("vgrid", C.c_double * n), ("vxgridMaxw", C.c_double * (n * n)), ("ws", _vp)]
    return inhomStepInterm_t


def _np(a, dt):
    a = np.ascontiguousarray(a, dtype=dt)
    return a, a.ctypes.data_as(_dp)


class Upstream:
    """The upstream entry points of libqbgpu, called the way a C driver calls them."""

    def __init__(self, n_grid=N_GRID):
        self.N = n_grid
        self.L = lib(n_grid)
        self.inhom_t = _inhom_interm_type(n_grid)

    # quadrature structs -------------------------------------------------------
    def fourier(self, which, J, L, R, M=None):
        q = quadI1_t()
        fn = {1: self.L.FourierI1, 2: self.L.FourierI2, 3: self.L.FourierI3, 4: self.L.FourierI4}[which]
        if which == 3:
            fn(C.c_uint(J), C.c_double(L), C.c_double(R), C.c_uint(M), C.byref(q))
        else:
            fn(C.c_uint(J), C.c_double(L), C.c_double(R), C.byref(q))
        return q

    def quad_delete(self, which, q):
        {1: self.L.QuadI1_Delete, 2: self.L.QuadI2_Delete, 3: self.L.QuadI3_Delete, 4: self.L.QuadI1_Delete}[which](C.byref(q))

    def quad_arrays(self, which, q):
        N, P = self.N, 2 * self.N
        n = q.num
        sh1 = {1: (n, P, P), 2: (n, N, N), 3: (n, N, N, 2), 4: (n, P, P)}[which]
        sh2 = {1: (n, N, N), 2: (n, N, N), 3: (n, P, P), 4: (n, N, N)}[which]
        a1 = np.ctypeslib.as_array(q.psiR1, shape=(int(np.prod(sh1)),)).reshape(sh1).copy()
        a2 = np.ctypeslib.as_array(q.psiR2, shape=(int(np.prod(sh2)),)).reshape(sh2).copy()
        return (a1.view(np.complex128)[..., 0] if which == 3 else a1), a2

    def quad_from_arrays(self, which, psiR1, psiR2):
        """A caller-filled quad struct (as test/I2_test.c builds one)."""
        q = quadI1_t()
        {1: self.L.QuadI1_Allocate, 2: self.L.QuadI2_Allocate, 3: self.L.QuadI3_Allocate}[which](C.c_uint(len(psiR1)), C.byref(q))
        r1 = np.ascontiguousarray(psiR1.view(np.float64) if np.iscomplexobj(psiR1) else psiR1, dtype=np.float64).ravel()
        r2 = np.ascontiguousarray(psiR2, dtype=np.float64).ravel()
        C.memmove(q.psiR1, r1.ctypes.data, r1.nbytes)
        C.memmove(q.psiR2, r2.ctypes.data, r2.nbytes)
        return q

    # interms -------------------------------------------------------------------
    def _interm(self, kind):
        it = interm_t()
        getattr(self.L, f"{kind}_Create")(C.byref(it))
        return it

    def _interm_del(self, kind, it):
        getattr(self.L, f"{kind}_Delete")(C.byref(it))

    # operators -----------------------------------------------------------------
    def integral(self, which, f, g, h, q):
        kind = {1: "I1interm", 2: "I2interm", 3: "I3interm", 4: "I1interm"}[which]
        fn = {1: self.L.I1integral, 2: self.L.I2integral, 3: self.L.I3integral, 4: self.L.I1integral}[which]
        it = self._interm(kind)
        f, pf = _np(f, np.complex128); g, pg = _np(g, np.complex128); h, ph = _np(h, np.complex128)
        out = np.zeros((self.N, self.N), np.complex128)
        fn(pf, pg, ph, C.byref(q), C.byref(it), out.ctypes.data_as(_dp))
        self._interm_del(kind, it)
        return out

    def cc(self, W, q1):
        it = self._interm("CcInterm")
        W, pW = _np(W, np.complex128)
        out = np.zeros_like(W)
        self.L.CcInt(pW, C.byref(q1), C.byref(it), out.ctypes.data_as(_dp))
        self._interm_del("CcInterm", it)
        return out

    def cd(self, W, q2, q3, q4):
        it = self._interm("CdInterm")
        W, pW = _np(W, np.complex128)
        out = np.zeros_like(W)
        self.L.CdInt(pW, C.byref(q2), C.byref(q3), C.byref(q4), C.byref(it), out.ctypes.data_as(_dp))
        self._interm_del("CdInterm", it)
        return out

    def collision_step(self, W, quads, dt, B=(0.0, 0.0, 0.0)):
        it = self._interm("CollisionInterm")
        W, pW = _np(W, np.complex128)
        Bv, pB = _np(B, np.float64)
        out = np.zeros_like(W)
        self.L.CollisionStep(pW, *[C.byref(q) for q in quads], C.c_double(dt), pB, C.byref(it), out.ctypes.data_as(_dp))
        self._interm_del("CollisionInterm", it)
        return out

    def inhom_interm(self, numVol, L):
        it = self.inhom_t()
        self.L.InhomStepInterm_Create(C.c_uint(numVol), C.c_double(L), C.byref(it))
        return it

    def inhom_step(self, W, quads, h, dt, Bext=None, bc="periodic", L=12.0, interm=None, out=None):
        """InhomStepPeriodic / InhomStepDirichlet on host arrays; `out` (a
        C-contiguous float64 array shaped like W, e.g. pinned) receives Wnext"""
        n = W.shape[0]
        it = interm or self.inhom_interm(n, L)
        W, pW = _np(W, np.float64)
        Bv, pB = _np(np.zeros((n, 3)) if Bext is None else Bext, np.float64)
        if out is None:
            out = np.zeros_like(W)
        elif not (out.flags["C_CONTIGUOUS"] and out.dtype == np.float64 and out.shape == W.shape):
            raise ValueError("out must be a C-contiguous float64 array shaped like W")
        fn = {"periodic": self.L.InhomStepPeriodic, "dirichlet": self.L.InhomStepDirichlet}[bc]
        fn(pW, *[C.byref(q) for q in quads], C.c_double(h), C.c_double(dt), pB, C.byref(it), out.ctypes.data_as(_dp))
        if interm is None:
            self.L.InhomStepInterm_Delete(C.byref(it))
        return out

    def inhom_step_maxwell(self, W, quads, h, dt, lam, WL, WR, Bext=None, L=12.0):
        n = W.shape[0]
        it = self.inhom_interm(n, L)
        W, pW = _np(W, np.float64)
        WL, pL = _np(WL, np.float64); WR, pR = _np(WR, np.float64)
        Bv, pB = _np(np.zeros((n, 3)) if Bext is None else Bext, np.float64)
        out = np.zeros_like(W)
        self.L.InhomStepMaxwell(pW, *[C.byref(q) for q in quads], C.c_double(h), C.c_double(dt), C.c_double(lam), pL, pR, pB,
                                C.byref(it), out.ctypes.data_as(_dp))
        self.L.InhomStepInterm_Delete(C.byref(it))
        return out

    def simulation_inhom(self, W0, quads, h, dt, numsteps, Bext=None, bc="periodic", L=12.0):
        n = W0.shape[0]
        it = self.inhom_interm(n, L)
        W0, pW = _np(W0, np.float64)
        Bv, pB = _np(np.zeros((n, 3)) if Bext is None else Bext, np.float64)
        out = np.zeros((numsteps,) + W0.shape)
        fn = {"periodic": self.L.SimulationInhomogeneousPeriodic, "dirichlet": self.L.SimulationInhomogeneousDirichlet}[bc]
        fn(pW, *[C.byref(q) for q in quads], C.c_double(h), C.c_double(dt), C.c_uint(numsteps), pB, C.byref(it), out.ctypes.data_as(_dp))
        self.L.InhomStepInterm_Delete(C.byref(it))
        return out

    def simulation_hom(self, W0, quads, dt, numsteps, B=(0.0, 0.0, 0.0)):
        it = self._interm("SimulationHomInterm")
        W0, pW = _np(W0, np.float64)
        Bv, pB = _np(B, np.float64)
        out = np.zeros((numsteps,) + W0.shape)
        self.L.SimulationHomogeneous(pW, *[C.byref(q) for q in quads], C.c_double(dt), C.c_uint(numsteps), pB, C.byref(it), out.ctypes.data_as(_dp))
        self._interm_del("SimulationHomInterm", it)
        return out

    def to_fourier_r2c(self, Wv):
        """The upstream drivers' own transform to Fourier space through the FFTW
        API (test/Cc_test.c:99-136): r2c plan, 1/N^2, Hermitian completion."""
        N = self.N
        Wv = np.ascontiguousarray(Wv, dtype=np.float64).reshape(-1, N, N)
        out = np.zeros(Wv.shape, np.complex128)
        half = np.zeros((N, N // 2 + 1), np.complex128)
        self.L.fftw_plan_dft_r2c_2d.restype = _vp
        self.L.fftw_plan_dft_r2c_2d.argtypes = [C.c_int, C.c_int, _vp, _vp, C.c_uint]
        self.L.fftw_execute.argtypes = [_vp]
        self.L.fftw_destroy_plan.argtypes = [_vp]
        for i in range(Wv.shape[0]):
            src = np.ascontiguousarray(Wv[i])
            plan = self.L.fftw_plan_dft_r2c_2d(N, N, src.ctypes.data, half.ctypes.data, 1 << 6)
            self.L.fftw_execute(plan)
            self.L.fftw_destroy_plan(plan)
            h = half / (N * N)
            for l in range(N):
                lc = (N - l) % N
                out[i, l, :N // 2 + 1] = h[l]
                for k in range(N // 2 + 1, N):
                    out[i, l, k] = np.conj(h[lc, N - k])
        return out

    def slope(self, bc, h, dt, A, Un):
        Un, pU = _np(Un, np.float64)
        out = np.zeros_like(Un)
        fn = self.L.SlopeLimiterStepPeriodic if bc == "periodic" else self.L.SlopeLimiterStepDirichlet
        fn(C.c_double(h), C.c_double(dt), C.c_double(A), C.c_uint(len(Un)), pU, out.ctypes.data_as(_dp))
        return out

    def slope_maxwell(self, h, dt, A, lam, fluxL, fluxR, UL, UR, Un):
        A, pA = _np(A, np.float64); UL, pL = _np(UL, np.float64); UR, pR = _np(UR, np.float64)
        Un, pU = _np(Un, np.float64)
        out = np.zeros_like(Un)
        self.L.SlopeLimiterStepMaxwell(C.c_double(h), C.c_double(dt), C.c_uint(len(A)), pA, C.c_uint(Un.shape[0]), C.c_double(lam),
                                       C.c_double(fluxL), C.c_double(fluxR), pL, pR, pU, out.ctypes.data_as(_dp))
        return out

    def lgwt(self, M, a, b):
        x = np.zeros(M); w = np.zeros(M)
        self.L.LegendreGaussQuad(C.c_uint(M), C.c_double(a), C.c_double(b), x.ctypes.data_as(_dp), w.ctypes.data_as(_dp))
        return x, w


# ---------------------------------------------------------------------------
# seeded synthetic initial states (velocity box [-L, L)^2)

def _splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x, z ^ (z >> 31)


class _Rng:
    """counter-based uniform doubles (splitmix64), reproducible across platforms"""

    def __init__(self, seed):
        self.s = seed & 0xFFFFFFFFFFFFFFFF

    def uniform(self, a=0.0, b=1.0):
        self.s, z = _splitmix64(self.s)
        return a + (b - a) * ((z >> 11) * (1.0 / 9007199254740992.0))


def mixture_params(seed, max_tries=1000):
    """Two-component Gaussian mixture parameters: a_k ~ U[0.3,0.6], u_k ~ U[-1,1]^2,
    T_k ~ U[0.5,1.5], s_k uniform in the ball |s| <= 0.9, phi_k ~ U[0, 2 pi);
    redrawn until sum_k 1.3 a_k (1 + |s_k|)/2 <= 1 so that 0 <= W <= 1 holds
    pointwise even with the 30% spatial modulation.
    Returns (params, redraws)."""
    rng = _Rng(seed)
    for tries in range(max_tries):
        comps = []
        for _ in range(2):
            a = rng.uniform(0.3, 0.6)
            u = (rng.uniform(-1, 1), rng.uniform(-1, 1))
            T = rng.uniform(0.5, 1.5)
            while True:
                s = np.array([rng.uniform(-0.9, 0.9) for _ in range(3)])
                if np.linalg.norm(s) <= 0.9:
                    break
            phi = rng.uniform(0, 2 * math.pi)
            comps.append((a, u, T, s, phi))
        # largest eigenvalue <= sum_k (1 + 0.3) a_k (1 + |s_k|) / 2 (spatial modulation included)
        if sum(1.3 * c[0] * (1 + np.linalg.norm(c[3])) / 2 for c in comps) <= 1.0:
            return comps, tries
    raise RuntimeError("no admissible mixture found")


def velocity_grid(N, L):
    k = np.arange(N)
    return np.where(k < N // 2, k, k - N) * (2.0 * L / N)


def gaussian_mixture_state(N, L, seed, ncells=1, modulation=0.3):
    """Velocity-space Wigner states (ncells, 4, N, N) in Pauli form:
    w0 = sum_k a_k(x) g_k / 2, w_vec = sum_k a_k(x) g_k s_k / 2 with
    g_k = exp(-|v-u_k|^2 / (2 T_k)) and a_k(x) = a_k (1 + modulation sin(2 pi x + phi_k))
    at cell centres x_i = (i + 1/2)/ncells (no modulation for one cell)."""
    comps, _ = mixture_params(seed)
    v = velocity_grid(N, L)
    vx, vy = np.meshgrid(v, v, indexing="ij")        # [l, k]: l is v_x (slow), k is v_y
    W = np.zeros((ncells, 4, N, N))
    for i in range(ncells):
        x = (i + 0.5) / ncells
        for (a, u, T, s, phi) in comps:
            ax = a * (1 + modulation * math.sin(2 * math.pi * x + phi)) if ncells > 1 else a
            g = np.exp(-((vx - u[0]) ** 2 + (vy - u[1]) ** 2) / (2 * T))
            W[i, 0] += ax * g / 2
            for c in range(3):
                W[i, c + 1] += ax * g * s[c] / 2
    return W

"""The allocation-free I3 entry point (qb_integral_i3_noalloc).

Callers that cannot allocate device memory -- code recording a CUDA graph on
its stream, a host application that hands out all device memory itself, or a
loop that must never stall on an allocation -- call this variant.  It takes
its scratch from a fixed 4 MiB static device array inside the library instead
of allocating, so its results must equal those of the allocating entry point
qb_integral(q, 3, ...).  Two calls in a row check that nothing stale carries
over between calls sharing the array.  This file is collected last so that a
run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

import qbgpu
from conftest import rel_l1

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-12      # the plain FP64 parity bound used by every other GPU test


def _noalloc_fn():
    L = qbgpu.lib()
    fn = L.qb_integral_i3_noalloc
    fn.argtypes = [C.c_void_p] * 6
    fn.restype = C.c_int
    return fn


def _grids(N, seed):
    rng = np.random.default_rng(seed)
    return [torch.from_numpy(rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).cuda() for _ in range(3)]


@pytest.mark.parametrize("N,J,M", [(32, 32, 7), (16, 6, 5)])
def test_noalloc_matches_allocating_entry_point(N, J, M):
    fn = _noalloc_fn()
    q, ws = qbgpu.Quad(N, J, M, 12.0, 7.5), qbgpu.Workspace(N)
    for seed in (1, 2):                       # two calls in a row sharing the static scratch
        f, g, h = _grids(N, seed)
        ref = qbgpu.integral(ws, q, 3, f, g, h)
        out = torch.empty_like(f)
        rc = fn(q.h, qbgpu._ptr(f), qbgpu._ptr(g), qbgpu._ptr(h), qbgpu._ptr(out), qbgpu._stream())
        assert rc == 0, qbgpu.lib().qb_last_error().decode()
        torch.cuda.synchronize()
        err = rel_l1(out.cpu().numpy(), ref.cpu().numpy())
        assert err < TOL, (seed, err)

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

import orc
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


@pytest.mark.parametrize("N,J,M", [(32, 32, 7), (16, 6, 5), (8, 4, 3)])
def test_noalloc_matches_allocating_entry_point(N, J, M):
    """every grid size the entry point dispatches (N = 8, 16, 32), against the
    allocating entry point and against the CPU oracle's I3integral"""
    fn = _noalloc_fn()
    q, ws = qbgpu.Quad(N, J, M, 12.0, 7.5), qbgpu.Workspace(N)
    o = orc.Oracle(N, J, M, 12.0, 7.5)
    for seed in (1, 2):                       # two calls in a row sharing the static scratch
        f, g, h = _grids(N, seed)
        ref = qbgpu.integral(ws, q, 3, f, g, h)
        out = torch.empty_like(f)
        rc = fn(q.h, qbgpu._ptr(f), qbgpu._ptr(g), qbgpu._ptr(h), qbgpu._ptr(out), qbgpu._stream())
        assert rc == 0, qbgpu.lib().qb_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        err = rel_l1(got, ref.cpu().numpy())
        assert err < TOL, (seed, err)
        want = o.i3(f.cpu().numpy(), g.cpu().numpy(), h.cpu().numpy())
        assert rel_l1(got, want) < TOL, seed

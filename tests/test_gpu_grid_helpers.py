"""The exported grid helpers of the upstream API on the GPU, bit for bit.

MultiplyPointwise* (upstream src/grid.c:33-164), GridZeroPad and GridExtract
(src/grid.c:171-210) are called through libqbgpu's C ABI with host buffers,
the way the upstream test drivers call them, and compared with

  - the upstream functions themselves (oracle/_ref, built from the unmodified
    sources) where that build exists, and
  - a numpy restatement of the same element formulas (always),

both with exact equality: the products are single IEEE multiplies and one
add/subtract per component, which the GPU kernel issues unfused.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "inhom-quantum-boltzmann-fourier-c_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import qbgpu  # noqa: E402
import orc  # noqa: E402

pytestmark = pytest.mark.gpu
N = qbgpu.N_GRID
P = 2 * N

# name -> (kind of f, kind of g or None for the Assign forms, kind of ret, grid size)
PRODUCTS = {
    "MultiplyPointwiseRR": ("r", "r", "r", N),
    "MultiplyPointwiseRC": ("r", "c", "c", N),
    "MultiplyPointwiseCC": ("c", "c", "c", N),
    "MultiplyPointwiseRR2": ("r", "r", "r", P),
    "MultiplyPointwiseCC2": ("c", "c", "c", P),
    "MultiplyPointwiseAssignRR": ("r", None, "r", N),
    "MultiplyPointwiseAssignRC": ("r", None, "c", N),
    "MultiplyPointwiseAssignRC2": ("r", None, "c", P),
    "MultiplyPointwiseAssignCC2": ("c", None, "c", P),
}


def _grid(kind, n, rng):
    a = rng.standard_normal((n, n))
    if kind == "c":
        a = a + 1j * rng.standard_normal((n, n))
    # a spread of magnitudes, so that rounding differences would show
    return a * np.exp(rng.uniform(-20, 20, (n, n)))


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _call(lib, name, f, g, ret):
    fn = getattr(lib, name)
    fn.restype = None
    if g is None:
        fn(_ptr(f), _ptr(ret))
    else:
        fn(_ptr(f), _ptr(g), _ptr(ret))


def _cmul(a, b):
    """(a.re b.re - a.im b.im) + i (a.re b.im + a.im b.re), each product rounded"""
    return (a.real * b.real - a.imag * b.imag) + 1j * (a.real * b.imag + a.imag * b.real)


def _numpy_product(name, f, g, ret0):
    kf, kg, kr, _ = PRODUCTS[name]
    if kg is None:
        if kf == "r":
            return ret0 * f if kr == "r" else ret0.real * f + 1j * (ret0.imag * f)
        return _cmul(f, ret0)
    if kf == "r" and kg == "r":
        return f * g
    if kf == "r":
        return f * g.real + 1j * (f * g.imag)
    return _cmul(f, g)


@pytest.fixture(scope="module")
def libs():
    gpu = qbgpu.lib()
    ref = orc.ref_lib() if (orc.ref_available() and N == 32) else None
    return gpu, ref


@pytest.mark.parametrize("name", sorted(PRODUCTS))
def test_pointwise_products_bit_exact(libs, name):
    gpu, ref = libs
    kf, kg, kr, n = PRODUCTS[name]
    rng = np.random.default_rng(sum(name.encode()))
    f = np.ascontiguousarray(_grid(kf, n, rng))
    g = None if kg is None else np.ascontiguousarray(_grid(kg, n, rng))
    ret0 = np.ascontiguousarray(_grid(kr, n, rng))
    got = ret0.copy()
    _call(gpu, name, f, g, got)
    assert np.array_equal(got, _numpy_product(name, f, g, ret0))
    if ref is not None:
        want = ret0.copy()
        _call(ref, name, f, g, want)
        assert np.array_equal(got, want)


def test_zero_pad_and_extract_bit_exact(libs):
    gpu, ref = libs
    rng = np.random.default_rng(7)
    f = np.ascontiguousarray(_grid("c", N, rng))
    pad = np.full((P, P), np.nan + 1j * np.nan)          # every entry must be written
    _call(gpu, "GridZeroPad", f, None, pad)
    want = np.zeros((P, P), np.complex128)
    lo, hi = np.r_[0:N // 2], np.r_[N // 2:N]
    want[np.ix_(lo, lo)] = f[np.ix_(lo, lo)]
    want[np.ix_(lo, hi + N)] = f[np.ix_(lo, hi)]
    want[np.ix_(hi + N, lo)] = f[np.ix_(hi, lo)]
    want[np.ix_(hi + N, hi + N)] = f[np.ix_(hi, hi)]
    assert np.array_equal(pad, want)
    back = np.full((N, N), np.nan + 1j * np.nan)
    big = np.ascontiguousarray(_grid("c", P, rng))
    _call(gpu, "GridExtract", big, None, back)
    idx = np.r_[0:N // 2, 3 * N // 2:P]
    assert np.array_equal(back, big[np.ix_(idx, idx)])
    if ref is not None:
        pr = np.zeros((P, P), np.complex128)
        _call(ref, "GridZeroPad", f, None, pr)
        assert np.array_equal(pad, pr)
        er = np.zeros((N, N), np.complex128)
        _call(ref, "GridExtract", big, None, er)
        assert np.array_equal(back, er)

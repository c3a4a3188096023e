"""GPU parity: the CUDA path against the upstream goldens and the CPU oracle.

Two surfaces are checked:
  * the upstream C API (host buffers, N_GRID = 32) -- the drop-in boundary --
    on the upstream golden vectors with the upstream test drivers' parameters;
  * the batched device API (include/qbgpu.h) against the oracle on seeded
    Gaussian-mixture states at N = 8, 16, 32, 64, including magnetic fields and
    all three boundary conditions.  N = 64 runs the split-grid kernels (one
    padded 128 x 128 grid per CTA pair of a cluster).
Tolerance: the plain FP64 path must match the upstream C code within 1e-12
relative (L1, as test/Cc_test.c:177-189 measures); against the Matlab-made
I-integral goldens the bound is the upstream C code's own 5e-12 average
absolute error.  Transport is bit-exact.
"""
import numpy as np
import pytest

import orc
import qbgpu
from conftest import avg_abs_err, golden_c, golden_r, rel_l1

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
L_, R_ = 12.0, 7.5
TOL = 1e-12


@pytest.fixture(scope="module")
def up():
    return qbgpu.Upstream()


@pytest.fixture(scope="module")
def fgh():
    return golden_c("f.dat"), golden_c("g.dat"), golden_c("h.dat")


# ---------------------------------------------------------------------------
# upstream API on the upstream goldens

def test_fftw_api_transform_matches_oracle(up, golden_W):
    WF = up.to_fourier_r2c(golden_W)
    assert rel_l1(WF, orc.to_fourier(golden_W)) < 1e-14


@pytest.mark.parametrize("which,J,M,golden", [(1, 32, 2, "I1_ref.dat"), (2, 32, 2, "I2_ref2.dat"), (3, 32, 7, "I3_ref.dat"), (4, 32, 2, "I4_ref.dat")])
def test_integral_golden(up, fgh, which, J, M, golden):
    q = up.fourier(which, J, L_, R_, M)
    out = up.integral(which, *fgh, q)
    up.quad_delete(which, q)
    # the Matlab goldens carry ~1e-12 absolute error themselves (upstream C code:
    # 0.8-2.1e-12); the factored sums round differently, so bound the relative error
    assert rel_l1(out, golden_c(golden)) < 1e-13
    o = orc.Oracle(32, J, M, L_, R_)
    ref = {1: o.i1, 2: o.i2, 3: o.i3, 4: o.i4}[which](*fgh)
    assert rel_l1(out, ref) < TOL


def test_integral_i2_caller_tables(up, fgh):
    """test/I2_test.c fills quadI2_t by hand: generic (unregistered) tables"""
    w = golden_r("weight.dat", (7,))
    p1 = np.stack([golden_r(f"psiR1_{j}.dat", (32, 32)) for j in range(1, 8)])
    p2 = np.stack([golden_r(f"psiR2_{j}.dat", (32, 32)) * w[j - 1] for j in range(1, 8)])
    q = up.quad_from_arrays(2, p1, p2)
    out = up.integral(2, *fgh, q)
    up.quad_delete(2, q)
    assert avg_abs_err(out, golden_c("I2_ref.dat")) < 1e-13
    assert rel_l1(out, orc.i2_raw(32, *fgh, p1, p2)) < TOL


def test_quadrature_tables_match_oracle(up):
    o = orc.Oracle(32, 5, 4, 6.0, 3.75)
    T = o.tables()
    for which, keys in ((1, ("i1r1", "i1r2")), (2, ("i2r1", "i2r2")), (3, ("i3r1", "i3r2")), (4, ("i4r1", "i4r2"))):
        q = up.fourier(which, 5, 6.0, 3.75, 4)
        a1, a2 = up.quad_arrays(which, q)
        up.quad_delete(which, q)
        assert np.abs(a1 - T[keys[0]]).max() < 1e-13 * max(1.0, np.abs(T[keys[0]]).max()), keys[0]
        assert np.abs(a2 - T[keys[1]]).max() < 1e-13 * max(1.0, np.abs(T[keys[1]]).max()), keys[1]


def test_lgwt(up):
    x, w = up.lgwt(15, 0.5, 2.0)
    assert np.abs(x - golden_r("x_ref.dat", (15,))).max() < 1e-14
    assert np.abs(w - golden_r("w_ref.dat", (15,))).max() < 1e-14


def test_cc_golden(up, golden_W):
    q1 = up.fourier(1, 48, L_, R_)
    WF = up.to_fourier_r2c(golden_W)
    out = up.cc(WF, q1)
    up.quad_delete(1, q1)
    ref = np.stack([golden_c(f"Cc{i}_ref.dat") for i in range(4)])
    assert rel_l1(out, ref) < TOL
    assert np.all(out[0] == 0)


def test_cd_golden(up, golden_W):
    q2, q3, q4 = up.fourier(2, 17, L_, R_), up.fourier(3, 17, L_, R_, 15), up.fourier(4, 17, L_, R_)
    WF = up.to_fourier_r2c(golden_W)
    out = up.cd(WF, q2, q3, q4)
    for w, q in ((2, q2), (3, q3), (4, q4)):
        up.quad_delete(w, q)
    ref = np.stack([golden_c(f"Cd{i}_ref.dat") for i in range(4)])
    assert rel_l1(out, ref) < TOL


def _quads(up, J, M, L=L_, R=R_):
    return [up.fourier(1, J, L, R), up.fourier(2, J, L, R), up.fourier(3, J, L, R, M), up.fourier(4, J, L, R)]


def _free(up, quads):
    for w, q in zip((1, 2, 3, 4), quads):
        up.quad_delete(w, q)


def test_collision_step_golden(up, golden_W):
    quads = _quads(up, 32, 32)
    WF = up.to_fourier_r2c(golden_W)
    out = up.collision_step(WF, quads, 1e-3)
    _free(up, quads)
    ref = np.stack([golden_c(f"WFnext{i}_ref.dat") for i in range(4)])
    assert rel_l1(out, ref) < TOL


def test_simulation_homogeneous_frame_golden(up):
    quads = _quads(up, 32, 32)
    W0 = golden_r("W0_hom.dat", (4, 32, 32))
    ev = up.simulation_hom(W0, quads, 1e-3, 2)
    _free(up, quads)
    assert np.array_equal(ev[0], W0)
    assert rel_l1(ev[1], golden_r("Wevolv_hom_frame1.dat", (4, 32, 32))) < TOL


def test_inhom_step_golden(up):
    quads = _quads(up, 16, 32)
    Wx = golden_r("Wx.dat", (8, 4, 32, 32))
    out = up.inhom_step(Wx, quads, 0.08, 0.002, L=L_)
    _free(up, quads)
    assert rel_l1(out, golden_r("Wx_next_ref.dat", (8, 4, 32, 32))) < TOL


def test_upstream_api_n_grid_64():
    """the upstream entry points built with N_GRID = 64 (lib/libqbgpu_n64.so),
    called as a driver compiled for that grid calls them, against the oracle"""
    up64 = qbgpu.Upstream(64)
    J, M, L, R = 4, 3, 6.0, 3.75
    quads = _quads(up64, J, M, L, R)
    o = orc.Oracle(64, J, M, L, R)
    Wv = qbgpu.gaussian_mixture_state(64, L, seed=41, ncells=3)
    WF = up64.to_fourier_r2c(Wv[0])
    assert rel_l1(WF, orc.to_fourier(Wv[0])) < 1e-14
    assert rel_l1(up64.cc(WF, quads[0]), o.cc(WF)) < TOL
    assert rel_l1(up64.cd(WF, quads[1], quads[2], quads[3]), o.cd(WF)) < TOL
    h, dt = 1 / 3, 0.4 / 3 / L
    out = up64.inhom_step(Wv, quads, h, dt, L=L)
    assert rel_l1(out, o.inhom_step(Wv, h, dt)) < TOL
    _free(up64, quads)


def test_simulation_inhom_periodic_frame_golden(up):
    """bin/params_periodic_example.txt: 10 cells, J = M = 32, h = 0.1, dt = 0.008"""
    quads = _quads(up, 32, 32)
    W0 = golden_r("W0_inhom.dat", (10, 4, 32, 32))
    ev = up.simulation_inhom(W0, quads, 0.1, 0.008, 2, L=L_)
    _free(up, quads)
    assert np.array_equal(ev[0], W0)
    assert rel_l1(ev[1], golden_r("Wevolv_inhom_periodic_frame1.dat", (10, 4, 32, 32))) < TOL


def test_slope_limiters_bit_exact(up):
    Un = golden_r("Un.dat", (128,))
    assert np.array_equal(up.slope("periodic", 0.08, 0.02, -1.2, Un), golden_r("Un1_periodic_ref.dat", (128,)))
    assert np.array_equal(up.slope("dirichlet", 0.08, 0.02, -1.2, Un), golden_r("Un1_Dirichlet_ref.dat", (128,)))
    UnM = golden_r("UnM.dat", (101, 4))
    UL = np.array([0.2, -np.pi / 4, 0, 0]); UR = np.array([0, 0, 1 / np.e, -0.8])
    out = up.slope_maxwell(0.01, 0.005, np.array([1.0, 0.5, -0.5, -1.0]), 0.4, 0.7, 0.45, UL, UR, UnM)
    assert np.array_equal(out, golden_r("Un1_Maxwell_ref.dat", (101, 4)))


def test_slope_limiter_edge_cells(up):
    """two cells (smallest periodic/Dirichlet line) and both velocity signs"""
    rng = np.random.default_rng(3)
    for n in (2, 3, 5):
        Un = rng.random(n)
        for A in (-0.7, 0.0, 1.3):
            assert np.array_equal(up.slope("periodic", 0.1, 0.03, A, Un), orc.slope_periodic(0.1, 0.03, A, Un))
            assert np.array_equal(up.slope("dirichlet", 0.1, 0.03, A, Un), orc.slope_dirichlet(0.1, 0.03, A, Un))


def test_fluxes_bit_exact(up):
    rng = np.random.default_rng(4)
    A = np.concatenate([rng.random(50), -rng.random(50)])
    U = rng.random(100)
    pa, pu = A.ctypes.data_as(qbgpu._dp), U.ctypes.data_as(qbgpu._dp)
    assert up.L.CalculateRightwardFlux(100, pa, pu) == orc.lib().orc_flux_right(100, pa, pu)
    assert up.L.CalculateLeftwardFlux(100, pa, pu) == orc.lib().orc_flux_left(100, pa, pu)


def test_inhom_step_maxwell_upstream_api(up):
    quads = _quads(up, 4, 4, 6.0, 3.75)
    W = qbgpu.gaussian_mixture_state(32, 6.0, seed=21, ncells=5)
    WL = qbgpu.gaussian_mixture_state(32, 6.0, seed=22)[0]
    WR = qbgpu.gaussian_mixture_state(32, 6.0, seed=23)[0]
    B = np.random.default_rng(5).standard_normal((5, 3)) * 0.1
    out = up.inhom_step_maxwell(W, quads, 0.2, 0.01, 0.4, WL, WR, B, L=6.0)
    _free(up, quads)
    ref = orc.Oracle(32, 4, 4, 6.0, 3.75).inhom_step_maxwell(W, 0.2, 0.01, 0.4, WL, WR, B)
    assert rel_l1(out, ref) < TOL


# ---------------------------------------------------------------------------
# batched device API against the oracle at several grid sizes

# even J: with odd J the upstream I1 principal-value weight -1/cos(theta1_i - theta2_j)
# (src/quadrature.c:224) hits cos = 0 and the operator is singular
CASES = [(8, 4, 3), (16, 4, 3), (32, 2, 4), (64, 4, 3)]


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.to(device="cuda", dtype=dtype) if dtype else t.cuda()


@pytest.fixture(scope="module", params=CASES, ids=[f"N{c[0]}" for c in CASES])
def setup(request):
    N, J, M = request.param
    L, R = 6.0, 3.75
    return dict(N=N, J=J, M=M, L=L, R=R, q=qbgpu.Quad(N, J, M, L, R), ws=qbgpu.Workspace(N), o=orc.Oracle(N, J, M, L, R))


def test_operators_vs_oracle(setup):
    s = setup
    Wv = qbgpu.gaussian_mixture_state(s["N"], s["L"], seed=31, ncells=3)
    WF = orc.to_fourier(Wv)
    cc, cd = qbgpu.collision_operators(s["ws"], s["q"], dev(WF))
    cc, cd = cc.cpu().numpy(), cd.cpu().numpy()
    for i in range(3):
        assert rel_l1(cc[i], s["o"].cc(WF[i])) < TOL
        assert rel_l1(cd[i], s["o"].cd(WF[i])) < TOL


def test_transforms_vs_oracle(setup):
    Wv = qbgpu.gaussian_mixture_state(setup["N"], setup["L"], seed=32, ncells=2)
    WF = qbgpu.to_fourier(dev(Wv)).cpu().numpy()
    assert rel_l1(WF, orc.to_fourier(Wv)) < 1e-14
    back = qbgpu.from_fourier(dev(WF)).cpu().numpy()
    assert rel_l1(back, orc.from_fourier(WF)) < 1e-14
    assert rel_l1(back, Wv) < 1e-14


@pytest.mark.parametrize("rk4", [False, True])
def test_collision_step_vs_oracle(setup, rk4):
    s = setup
    Wv = qbgpu.gaussian_mixture_state(s["N"], s["L"], seed=33, ncells=2)
    WF = orc.to_fourier(Wv)
    B = np.array([[0.3, -0.1, 0.2], [0.0, 0.0, 0.0]])
    out = qbgpu.collision_step(s["ws"], s["q"], dev(WF), 0.01, dev(B), rk4=rk4).cpu().numpy()
    for i in range(2):
        assert rel_l1(out[i], s["o"].collision_step(WF[i], 0.01, B[i], rk4=rk4)) < TOL


@pytest.mark.parametrize("bc", ["periodic", "dirichlet"])
def test_inhom_step_vs_oracle(setup, bc):
    s = setup
    W = qbgpu.gaussian_mixture_state(s["N"], s["L"], seed=34, ncells=6)
    B = np.random.default_rng(6).standard_normal((6, 3)) * 0.05
    h, dt = 1 / 6, 0.4 * (1 / 6) / s["L"]
    out = qbgpu.inhom_step(s["ws"], s["q"], dev(W), h, dt, dev(B), bc=bc).cpu().numpy()
    assert rel_l1(out, s["o"].inhom_step(W, h, dt, B, bc=bc)) < TOL


def test_inhom_step_maxwell_vs_oracle(setup):
    s = setup
    W = qbgpu.gaussian_mixture_state(s["N"], s["L"], seed=35, ncells=4)
    WL = qbgpu.gaussian_mixture_state(s["N"], s["L"], seed=36)[0]
    WR = qbgpu.gaussian_mixture_state(s["N"], s["L"], seed=37)[0]
    h, dt = 0.25, 0.01
    out = qbgpu.inhom_step_maxwell(s["ws"], s["q"], dev(W), h, dt, 0.4, dev(WL), dev(WR)).cpu().numpy()
    assert rel_l1(out, s["o"].inhom_step_maxwell(W, h, dt, 0.4, WL, WR)) < TOL


def test_integrals_vs_oracle(setup):
    s = setup
    rng = np.random.default_rng(7)
    N = s["N"]
    f, g, h = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)) for _ in range(3))
    for which, fn in ((1, s["o"].i1), (2, s["o"].i2), (3, s["o"].i3), (4, s["o"].i4)):
        out = qbgpu.integral(s["ws"], s["q"], which, dev(f), dev(g), dev(h)).cpu().numpy()
        assert rel_l1(out, fn(f, g, h)) < TOL, which


def test_transport_only_is_bit_exact(setup):
    """zero collision time: dt = 0 leaves only the identity collision, so the
    Strang step is transport(transport(W)); compare the transport halves exactly"""
    s = setup
    W = qbgpu.gaussian_mixture_state(s["N"], s["L"], seed=38, ncells=5)
    out = qbgpu.inhom_step(s["ws"], s["q"], dev(W), 0.2, 0.0).cpu().numpy()
    # with dt = 0 the limiter is the identity and the collision adds 0 * C
    assert rel_l1(out, W) < 1e-15


def test_moments_match_oracle(setup):
    """density of each Pauli component, momentum and energy after a collision
    step (visualization/wignerMoments.m:15-37) agree with the oracle's; the
    discrete operator conserves them only up to the resolution error, so the
    drift itself is compared, not assumed zero"""
    s = setup
    N, L = s["N"], s["L"]
    Wv = qbgpu.gaussian_mixture_state(N, L, seed=39, ncells=1)
    WF = orc.to_fourier(Wv)
    gpu = orc.from_fourier(qbgpu.collision_step(s["ws"], s["q"], dev(WF), 0.05).cpu().numpy())[0]
    ref = orc.from_fourier(s["o"].collision_step(WF[0], 0.05))
    v = qbgpu.velocity_grid(N, L)
    vx, vy = np.meshgrid(v, v, indexing="ij")
    scale = abs(Wv[0, 0].sum())
    for c in range(4):
        assert abs(gpu[c].sum() - ref[c].sum()) < 1e-12 * scale
    for w in (vx, vy, vx ** 2 + vy ** 2):
        assert abs((w * gpu[0]).sum() - (w * ref[0]).sum()) < 1e-12 * abs(w * Wv[0, 0]).sum()

"""Pin the CPU oracle (oracle/qb_oracle.c) to the upstream golden vectors.

The goldens are the upstream project's own fixtures (test/data/*.dat, produced
by its Matlab reference scripts) and two trajectories written by its C
programs (data/Wevolv_*.dat), copied by tests/golden/make_fixtures.py.  The
tolerances are the agreement the upstream C code itself reaches against the
same files (Matlab goldens ~1e-12 absolute on the I-integrals, C-generated
data ~1e-15 relative).
"""
import numpy as np
import pytest

import orc
from conftest import avg_abs_err, golden_c, golden_r, rel_l1

L_, R_ = 12.0, 7.5          # test drivers' box (test/I1_test.c:39-40)


@pytest.fixture(scope="module")
def fgh():
    return golden_c("f.dat"), golden_c("g.dat"), golden_c("h.dat")


def test_i1_golden(fgh):                     # test/I1_test.c: J = 32
    o = orc.Oracle(32, 32, 2, L_, R_)
    assert avg_abs_err(o.i1(*fgh), golden_c("I1_ref.dat")) < 5e-12


def test_i2_handmade_tables_golden(fgh):     # test/I2_test.c: J = 7, tables from files
    w = golden_r("weight.dat", (7,))
    p1 = np.stack([golden_r(f"psiR1_{j}.dat", (32, 32)) for j in range(1, 8)])
    p2 = np.stack([golden_r(f"psiR2_{j}.dat", (32, 32)) * w[j - 1] for j in range(1, 8)])
    assert avg_abs_err(orc.i2_raw(32, *fgh, p1, p2), golden_c("I2_ref.dat")) < 1e-13


def test_i2_golden(fgh):                     # test/I2_test2.c: FourierI2, J = 32
    o = orc.Oracle(32, 32, 2, L_, R_)
    assert avg_abs_err(o.i2(*fgh), golden_c("I2_ref2.dat")) < 5e-12


def test_i3_golden(fgh):                     # test/I3_test.c: J = 32, M = 7
    o = orc.Oracle(32, 32, 7, L_, R_)
    assert avg_abs_err(o.i3(*fgh), golden_c("I3_ref.dat")) < 5e-12


def test_i4_golden(fgh):                     # test/I4_test.c: FourierI4, J = 32
    o = orc.Oracle(32, 32, 2, L_, R_)
    assert avg_abs_err(o.i4(*fgh), golden_c("I4_ref.dat")) < 5e-12


def test_lgwt_golden():                      # test/lgwt_test.c: M = 15 on [0.5, 2]
    x, w = orc.lgwt(15, 0.5, 2.0)
    assert np.array_equal(x, golden_r("x_ref.dat", (15,)))
    assert np.array_equal(w, golden_r("w_ref.dat", (15,)))


def test_slope_limiters_golden():            # test/slope_lim_test.c: N = 128, A = -1.2
    Un = golden_r("Un.dat", (128,))
    assert np.array_equal(orc.slope_periodic(0.08, 0.02, -1.2, Un), golden_r("Un1_periodic_ref.dat", (128,)))
    assert np.array_equal(orc.slope_dirichlet(0.08, 0.02, -1.2, Un), golden_r("Un1_Dirichlet_ref.dat", (128,)))


def test_slope_maxwell_golden():             # test/slope_lim_test2.c: m = 4, N = 101
    UnM = golden_r("UnM.dat", (101, 4))
    UL = np.array([0.2, -np.pi / 4, 0, 0]); UR = np.array([0, 0, 1 / np.e, -0.8])
    out = orc.slope_maxwell(0.01, 0.005, np.array([1.0, 0.5, -0.5, -1.0]), 0.4, 0.7, 0.45, UL, UR, UnM)
    assert np.array_equal(out, golden_r("Un1_Maxwell_ref.dat", (101, 4)))


def test_cc_golden(golden_W):                # test/Cc_test.c: J = 48
    o = orc.Oracle(32, 48, 2, L_, R_)
    ref = np.stack([golden_c(f"Cc{i}_ref.dat") for i in range(4)])
    assert rel_l1(o.cc(orc.to_fourier(golden_W)), ref) < 1e-13


def test_cd_golden(golden_W):                # test/Cd_test.c: J = 17, M = 15
    o = orc.Oracle(32, 17, 15, L_, R_)
    ref = np.stack([golden_c(f"Cd{i}_ref.dat") for i in range(4)])
    assert rel_l1(o.cd(orc.to_fourier(golden_W)), ref) < 1e-13


def test_collision_step_golden(golden_W):    # test/coll_step_test.c: J = M = 32, dt = 1e-3
    o = orc.Oracle(32, 32, 32, L_, R_)
    ref = np.stack([golden_c(f"WFnext{i}_ref.dat") for i in range(4)])
    assert rel_l1(o.collision_step(orc.to_fourier(golden_W), 1e-3), ref) < 1e-13


def test_homogeneous_frame_golden():         # src/main_hom.c: frame 1 of data/Wevolv_hom.dat
    o = orc.Oracle(32, 32, 32, L_, R_)
    W0 = golden_r("W0_hom.dat", (4, 32, 32))
    ev = o.simulation_homogeneous(W0, 1e-3, 2)
    assert np.array_equal(ev[0], W0)
    assert rel_l1(ev[1], golden_r("Wevolv_hom_frame1.dat", (4, 32, 32))) < 1e-13


def test_inhom_step_golden():                # test/sim_step_test.c: 8 cells, J = 16, M = 32
    o = orc.Oracle(32, 16, 32, L_, R_)
    Wx = golden_r("Wx.dat", (8, 4, 32, 32))
    assert rel_l1(o.inhom_step(Wx, 0.08, 0.002), golden_r("Wx_next_ref.dat", (8, 4, 32, 32))) < 1e-13


@pytest.mark.slow
def test_inhom_periodic_frame_golden():      # bin/params_periodic_example.txt: 10 cells, J = M = 32
    o = orc.Oracle(32, 32, 32, L_, R_)
    W0 = golden_r("W0_inhom.dat", (10, 4, 32, 32))
    assert rel_l1(o.inhom_step(W0, 0.1, 0.008), golden_r("Wevolv_inhom_periodic_frame1.dat", (10, 4, 32, 32))) < 1e-13

"""GPU parity on the seeded workloads, beyond single steps of small cases.

  * The headline configuration itself (64 x-cells, N = 32, J = M = 16,
    h = 1/64, dt = 0.4 h / L): one Strang step through the batched device API
    and through the upstream C API, against the upstream C code's own step
    (fixture made by tests/golden/make_seeded_fixtures.py from the unmodified
    upstream sources).
  * A 200-step trajectory of the same domain at the reduced quadrature
    J = M = 4 against upstream SimulationInhomogeneousPeriodic
    (src/simulation.c:1288-1301): parity over many steps, not just one.
  * N = 64 in FP64 with enough quadrature terms (J = M = 8, 64 I3 terms) that
    the I3 sums of the split-grid kernel run as several chunk partials per
    cell, reduced in a fixed order, against the oracle.

Bound: 1e-12 relative L1 (test/Cc_test.c:177-189), the plain FP64 parity gate.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import orc
import qbgpu
from conftest import GOLDEN, rel_l1

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
TOL = 1e-12

SEEDED = os.path.join(GOLDEN, "SEEDED.json")


def _fixture(name):
    if not os.path.exists(SEEDED):
        pytest.skip("seeded fixtures not generated (tests/golden/make_seeded_fixtures.py)")
    man = json.load(open(SEEDED))
    if name not in man:
        pytest.skip(f"{name} not generated")
    e = man[name]
    path = os.path.join(GOLDEN, name)
    blob = open(path, "rb").read()
    assert hashlib.sha256(blob).hexdigest() == e["sha256"]
    N = e["N"]
    data = np.frombuffer(blob, dtype="<f8").reshape(len(e["cells_stored"]), 4, N, N)
    W0 = qbgpu.gaussian_mixture_state(N, e["L"], seed=e["seed"], ncells=e["cells_total"])
    # the initial state is regenerated here; it must be the one the fixture started from
    assert hashlib.sha256(np.ascontiguousarray(W0, dtype="<f8").tobytes()).hexdigest() == e["initial_state_sha256"]
    return e, W0, data


def test_headline_step_matches_upstream():
    """64 cells, N = 32, J = M = 16: batched API and upstream C API against
    upstream InhomStepPeriodic"""
    e, W0, want = _fixture("inhom_step_n32_j16m16_step1.dat")
    q, ws = qbgpu.Quad(e["N"], e["J"], e["M"], e["L"], e["R"]), qbgpu.Workspace(e["N"])
    out = qbgpu.inhom_step(ws, q, torch.from_numpy(W0).cuda(), e["h"], e["dt"]).cpu().numpy()
    cells = e["cells_stored"]
    for k, c in enumerate(cells):
        assert rel_l1(out[c], want[k]) < TOL, c
    up = qbgpu.Upstream()
    quads = [up.fourier(1, e["J"], e["L"], e["R"]), up.fourier(2, e["J"], e["L"], e["R"]),
             up.fourier(3, e["J"], e["L"], e["R"], e["M"]), up.fourier(4, e["J"], e["L"], e["R"])]
    try:
        out_up = up.inhom_step(W0, quads, e["h"], e["dt"], L=e["L"])
    finally:
        for w, qq in zip((1, 2, 3, 4), quads):
            up.quad_delete(w, qq)
    for k, c in enumerate(cells):
        assert rel_l1(out_up[c], want[k]) < TOL, c


def test_trajectory_200_steps_matches_upstream():
    """200 Strang steps (graph replays after the first steps) against upstream
    SimulationInhomogeneousPeriodic; the eigenvalues w0 -+ |w| stay within
    [0, 1] up to the discrete operator's undershoot, as upstream's do"""
    e, W0, want = _fixture("inhom_traj_n32_j4m4_step200.dat")
    q, ws = qbgpu.Quad(e["N"], e["J"], e["M"], e["L"], e["R"]), qbgpu.Workspace(e["N"])
    bufs = [torch.from_numpy(W0).cuda(), torch.empty((e["cells_total"], 4, e["N"], e["N"]), dtype=torch.float64, device="cuda")]
    B = torch.zeros((e["cells_total"], 3), dtype=torch.float64, device="cuda")
    for k in range(e["steps"]):
        qbgpu.inhom_step(ws, q, bufs[k % 2], e["h"], e["dt"], B, out=bufs[(k + 1) % 2])
    out = bufs[e["steps"] % 2].cpu().numpy()
    assert ws.graph_replays >= e["steps"] - 4
    errs = [rel_l1(out[c], want[k]) for k, c in enumerate(e["cells_stored"])]
    assert max(errs) < TOL, max(errs)
    r = np.sqrt((out[:, 1:] ** 2).sum(axis=1))
    lo, hi = (out[:, 0] - r).min(), (out[:, 0] + r).max()
    assert lo > -1e-6 and hi <= 1.0, (lo, hi)


def test_n64_fp64_chunked_i3_sums_vs_oracle():
    """N = 64, J = M = 8 (64 I3 terms, several chunk partials per cell):
    Cc, Cd and a Strang step of 2 cells against the oracle"""
    N, J, M, L, R = 64, 8, 8, 6.0, 3.75
    q, ws = qbgpu.Quad(N, J, M, L, R), qbgpu.Workspace(N)
    o = orc.Oracle(N, J, M, L, R)
    Wv = qbgpu.gaussian_mixture_state(N, L, seed=47, ncells=2)
    WF = orc.to_fourier(Wv)
    cc, cd = qbgpu.collision_operators(ws, q, torch.from_numpy(WF).cuda())
    cc, cd = cc.cpu().numpy(), cd.cpu().numpy()
    for i in range(2):
        assert rel_l1(cc[i], o.cc(WF[i])) < TOL
        assert rel_l1(cd[i], o.cd(WF[i])) < TOL
    h, dt = 0.5, 0.4 * 0.5 / L
    out = qbgpu.inhom_step(ws, q, torch.from_numpy(Wv).cuda(), h, dt).cpu().numpy()
    assert rel_l1(out, o.inhom_step(Wv, h, dt)) < TOL

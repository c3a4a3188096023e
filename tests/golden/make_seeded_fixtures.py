"""Seeded parity fixtures from the upstream C code (test infrastructure).

Two fixtures pin the plain FP64 GPU path against the reference on the seeded
workload of the inhomogeneous periodic run (64 x-cells on [0,1), N = 32,
L = 6, R = 3.75, h = 1/64, dt = 0.4 h / L, Bext = 0, the two-Gaussian mixture
of `qbgpu.gaussian_mixture_state(32, 6, seed=1, ncells=64)`):

  inhom_traj_n32_j4m4_step200.dat
      200 Strang steps of upstream SimulationInhomogeneousPeriodic
      (src/simulation.c:1288-1301) at the reduced quadrature J = M = 4;
      frame 200 of every 4th cell (cells 0, 4, ..., 60).
  inhom_step_n32_j16m16_step1.dat
      one upstream InhomStepPeriodic (src/simulation.c:307-555) at the
      benchmark quadrature J = M = 16; every 8th cell (0, 8, ..., 56).

Both are raw little-endian float64 wignerV_t cells (4 x 32 x 32 each), as the
upstream test data.  SEEDED.json records the parameters, the sha256 of the
initial state the tests regenerate, and the sha256 of each fixture.

    make -C oracle                                   # builds oracle/_ref
    python tests/golden/make_seeded_fixtures.py [--only traj|step] [--source ref|oracle]

`--source oracle` runs the C restatement (oracle/_build, multi-threaded)
instead of the upstream build, for a quick local check; the committed
fixtures come from `--source ref`.  The upstream run of the trajectory is
single-threaded and takes a few hours on one core with the CPU FFT shim.
"""
import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "inhom-quantum-boltzmann-fourier-c_b200"))

N, L, R, CELLS, SEED = 32, 6.0, 3.75, 64, 1
H = 1.0 / CELLS
DT = 0.4 * H / L
FIXTURES = {
    "traj": dict(file="inhom_traj_n32_j4m4_step200.dat", J=4, M=4, steps=200, cells=list(range(0, CELLS, 4))),
    "step": dict(file="inhom_step_n32_j16m16_step1.dat", J=16, M=16, steps=1, cells=list(range(0, CELLS, 8))),
}


def initial_state():
    import qbgpu
    return qbgpu.gaussian_mixture_state(N, L, seed=SEED, ncells=CELLS)


def sha(b):
    return hashlib.sha256(b).hexdigest()


def run(name, source, outdir=HERE):
    import orc
    spec = FIXTURES[name]
    W0 = np.ascontiguousarray(initial_state())
    t0 = time.time()
    if source == "ref":
        r = orc.Ref(spec["J"], spec["M"], L, R)
        W = r.sim_inhom_periodic(W0, H, DT, spec["steps"])[-1]
    else:
        o = orc.Oracle(N, spec["J"], spec["M"], L, R)
        W = W0
        for _ in range(spec["steps"]):
            W = o.inhom_step(W, H, DT)
    sel = np.ascontiguousarray(W[spec["cells"]], dtype="<f8")
    sel.tofile(os.path.join(outdir, spec["file"]))
    return name, describe(name, source, outdir, seconds=round(time.time() - t0, 1))


def describe(name, source, outdir, seconds=None):
    """manifest entry of an already written fixture file"""
    spec = FIXTURES[name]
    path = os.path.join(outdir, spec["file"])
    W0 = np.ascontiguousarray(initial_state())
    return dict(source=("upstream SimulationInhomogeneousPeriodic (oracle/_ref)" if source == "ref"
                        else "oracle restatement (oracle/_build)"),
                N=N, J=spec["J"], M=spec["M"], L=L, R=R, cells_total=CELLS, seed=SEED, h=H, dt=DT,
                steps=spec["steps"], cells_stored=spec["cells"], bytes=os.path.getsize(path),
                sha256=sha(open(path, "rb").read()), initial_state_sha256=sha(W0.astype("<f8").tobytes()),
                seconds=seconds)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=sorted(FIXTURES))
    ap.add_argument("--source", choices=("ref", "oracle"), default="ref")
    ap.add_argument("--out", default=HERE, help="output directory (default: next to this script)")
    ap.add_argument("--record", action="store_true",
                    help="only (re)write the manifest entries of fixture files already written by --source")
    a = ap.parse_args()
    names = [a.only] if a.only else sorted(FIXTURES)
    if a.record:
        results = [(n, describe(n, a.source, a.out)) for n in names]
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(len(names)) as pool:
            results = pool.starmap(run, [(n, a.source, a.out) for n in names])
    man_path = os.path.join(a.out, "SEEDED.json")
    man = json.load(open(man_path)) if os.path.exists(man_path) else {}
    for name, entry in results:
        man[FIXTURES[name]["file"]] = entry
        print(name, entry)
    with open(man_path, "w") as fh:
        json.dump(man, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()

"""Generate the golden fixtures in this directory from the upstream repository.

The upstream project ships raw little-endian float64 golden vectors for its C
test drivers (test/data/*.dat, produced by its Matlab scripts) and two
end-to-end trajectories written by its own C programs (data/*.dat).  This
script copies the vectors the parity tests use and slices the first two
frames out of the trajectories, then writes MANIFEST.json with the source,
size and sha256 of every fixture.  Run it where the upstream checkout exists:

    python tests/golden/make_fixtures.py [--ref /root/reference]

The tests only read the files written here; they never read the upstream
checkout at run time.
"""
import argparse
import hashlib
import json
import os
import shutil

HERE = os.path.dirname(os.path.abspath(__file__))
N_GRID = 32
WIGNER_V_BYTES = 4 * N_GRID * N_GRID * 8          # one wignerV_t

TEST_DATA = [
    "f.dat", "g.dat", "h.dat", "W0.dat", "W1.dat", "W2.dat", "W3.dat",
    "I1_ref.dat", "I2_ref.dat", "I2_ref2.dat", "I3_ref.dat", "I4_ref.dat",
    "Cc0_ref.dat", "Cc1_ref.dat", "Cc2_ref.dat", "Cc3_ref.dat",
    "Cd0_ref.dat", "Cd1_ref.dat", "Cd2_ref.dat", "Cd3_ref.dat",
    "WFnext0_ref.dat", "WFnext1_ref.dat", "WFnext2_ref.dat", "WFnext3_ref.dat",
    "Wx.dat", "Wx_next_ref.dat",
    "Un.dat", "Un1_periodic_ref.dat", "Un1_Dirichlet_ref.dat",
    "UnM.dat", "Un1_Maxwell_ref.dat",
    "x_ref.dat", "w_ref.dat", "weight.dat",
] + [f"psiR1_{j}.dat" for j in range(1, 8)] + [f"psiR2_{j}.dat" for j in range(1, 8)]


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    manifest = {}
    for name in TEST_DATA:
        src = os.path.join(args.ref, "test", "data", name)
        dst = os.path.join(HERE, name)
        shutil.copyfile(src, dst)
        manifest[name] = {"source": f"test/data/{name}", "bytes": os.path.getsize(dst), "sha256": sha(dst)}
    # whole-file copies of the initial states
    for name in ("W0_hom.dat", "W0_inhom.dat"):
        src = os.path.join(args.ref, "data", name)
        dst = os.path.join(HERE, name)
        shutil.copyfile(src, dst)
        manifest[name] = {"source": f"data/{name}", "bytes": os.path.getsize(dst), "sha256": sha(dst)}
    # frame 1 of the end-to-end trajectories (frame 0 equals the initial state)
    for name, cells in (("Wevolv_hom.dat", 1), ("Wevolv_inhom_periodic.dat", 10)):
        src = os.path.join(args.ref, "data", name)
        frame = cells * WIGNER_V_BYTES
        with open(src, "rb") as fh:
            fh.seek(frame)
            blob = fh.read(frame)
        out = name.replace(".dat", "_frame1.dat")
        with open(os.path.join(HERE, out), "wb") as fh:
            fh.write(blob)
        manifest[out] = {"source": f"data/{name} bytes [{frame}, {2 * frame})",
                         "bytes": len(blob), "sha256": sha(os.path.join(HERE, out))}
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)
    print(f"wrote {len(manifest)} fixtures to {HERE}")


if __name__ == "__main__":
    main()

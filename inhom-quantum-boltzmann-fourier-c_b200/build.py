"""Build libqbgpu for sm_100a (B200) in-tree.

    python inhom-quantum-boltzmann-fourier-c_b200/build.py [--n-grid 32 --n-grid 64] [--jobs 8]

Outputs (git-ignored, shipped with the tree):
  lib/libqbgpu.so          upstream C API for N_GRID = 32 + batched extension API
  lib/libqbgpu_n64.so      the same with the upstream C API for N_GRID = 64
  lib/libqbgpu_nXX.so      other N_GRID values when requested (8, 16, 32, 64)

Every translation unit is compiled by nvcc with
  -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo
and linked into one shared library with the CUDA runtime linked statically.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(REPO, "include")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "_build")

SOURCES = ["qb_engine.cu", "qb_anyn.cu", "qb_tables.cu", "qb_abi.cu", "qb_fftw.cu", "qb_ext.cu", "qb_noalloc.cu", "qb_diag.cu", "qb_batch.cu",
           "qb_fno.cu", "qb_surrogate.cu", "qb_dftmma.cu"]
# sources that depend on N_GRID (the upstream ABI); the others are grid-size independent
NGRID_SOURCES = {"qb_abi.cu", "qb_ext.cu"}


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def flags(n_grid):
    return ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
            "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "-Drestrict_=__restrict__",
            f"-DN_GRID={n_grid}", "-I", INC, "-I", CSRC]


def compile_one(src, n_grid, verbose):
    out = os.path.join(OBJ, f"n{n_grid}_" + src.replace(".cu", ".o") if src in NGRID_SOURCES else src.replace(".cu", ".o"))
    inp = os.path.join(CSRC, src)
    deps = [inp] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
           [os.path.join(INC, f) for f in os.listdir(INC)]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    cmd = [nvcc(), "-c", inp, "-o", out] + flags(n_grid)
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed for {src}")
    if verbose:
        sys.stderr.write(r.stderr)
    return out


def build(n_grids=(32,), jobs=8, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    outs = []
    for n in n_grids:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            objs = list(ex.map(lambda s: compile_one(s, n, verbose), SOURCES))
        name = "libqbgpu.so" if n == 32 else f"libqbgpu_n{n}.so"
        target = os.path.join(LIB, name)
        cmd = [nvcc(), "-shared", "-o", target] + objs + ["-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static"]
        subprocess.run(cmd, check=True)
        outs.append(target)
    return outs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-grid", type=int, action="append")
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    for t in build(tuple(a.n_grid or [32, 64]), a.jobs, a.verbose):
        print(t)

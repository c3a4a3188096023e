"""The C-ABI library loads without a GPU and exports every declared entry point;
the upstream drivers compile against include/ and link against it unchanged."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

import qbgpu
from conftest import REPO

INCLUDE = os.path.join(REPO, "include")


def _upstream_dir():
    """The upstream checkout: $QB_REFERENCE_DIR, else the REF default of the
    oracle's build recipe (oracle/Makefile), which is overridable the same way."""
    d = os.environ.get("QB_REFERENCE_DIR")
    if d:
        return d
    try:
        r = subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "print-ref"], capture_output=True, text=True, timeout=30)
        return r.stdout.strip() if r.returncode == 0 else ""
    except (OSError, subprocess.SubprocessError):
        return ""


UPSTREAM = _upstream_dir()


def declared_functions():
    names = set()
    for fn in sorted(os.listdir(INCLUDE)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"^\s*(?!static|typedef|#)[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_declarations_found():
    names = declared_functions()
    for must in ("CcInt", "CdInt", "I1integral", "I2integral", "I3integral", "CollisionStep", "InhomStepPeriodic",
                 "InhomStepDirichlet", "InhomStepMaxwell", "SimulationHomogeneous", "SimulationInhomogeneousPeriodic",
                 "SlopeLimiterStepPeriodic", "SlopeLimiterStepMaxwell", "FourierI1", "FourierI3", "LegendreGaussQuad",
                 "GridZeroPad", "ReadData", "fftw_execute", "fftw_plan_dft_r2c_2d", "qb_inhom_step", "qb_last_error"):
        assert must in names, must


def test_library_exports_every_declared_symbol():
    L = qbgpu.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_library_links_cuda_runtime_statically():
    out = subprocess.run(["ldd", qbgpu.library_path()], capture_output=True, text=True).stdout
    assert "libcudart" not in out


def test_read_write_data_roundtrip(tmp_path):
    """util.c: ReadData checks the exact file size (-2 on mismatch)."""
    L = qbgpu.lib()
    import numpy as np
    a = np.arange(10, dtype=np.float64)
    p = str(tmp_path / "x.dat").encode()
    assert L.WriteData(p, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(8), ctypes.c_size_t(10), ctypes.c_bool(False)) == 0
    b = np.zeros(10)
    assert L.ReadData(p, b.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(8), ctypes.c_size_t(10)) == 0
    assert np.array_equal(a, b)
    assert L.ReadData(p, b.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(8), ctypes.c_size_t(9)) == -2
    assert L.ReadData(b"/nonexistent/file", b.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(8), ctypes.c_size_t(1)) == -1


DRIVERS = ["test/I1_test.c", "test/I2_test.c", "test/I2_test2.c", "test/I3_test.c", "test/I4_test.c", "test/Cc_test.c",
           "test/Cd_test.c", "test/coll_step_test.c", "test/sim_step_test.c", "test/lgwt_test.c", "test/slope_lim_test.c",
           "test/slope_lim_test2.c", "src/main_hom.c", "src/main_inhom.c"]


@pytest.mark.skipif(not UPSTREAM or not os.path.isdir(UPSTREAM) or shutil.which("gcc") is None, reason="upstream drivers not available here")
@pytest.mark.parametrize("driver", DRIVERS)
def test_upstream_driver_links_unchanged(driver, tmp_path):
    """Compile the unmodified upstream driver with its own flags against
    include/ and link it against libqbgpu (no run: that needs a GPU)."""
    src = os.path.join(UPSTREAM, driver)
    exe = str(tmp_path / "drv")
    cmd = ["gcc", "-w", "-m64", "-O3", "-DNDEBUG", "-Drestrict_=__restrict__", "-I", INCLUDE, src, "-o", exe,
           "-L", qbgpu.LIB_DIR, "-lqbgpu", f"-Wl,-rpath,{qbgpu.LIB_DIR}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

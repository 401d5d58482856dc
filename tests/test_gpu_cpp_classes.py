"""The C++ classes of include/wrapd_gpu.hpp on the GPU: a solve of the
8x8x32 bar through wrapd::gpu::Solver (tests/host/shim_solve.cpp) gives the
same final positions and energy log, bit for bit, as the same solve through
the Python mirror -- one library, and its device sums are deterministic."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from wrapd_b200 import bars
from wrapd_b200.solver import Solver

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_solver_matches_the_python_mirror(lib_built, tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    libdir = os.path.dirname(lib_built)
    exe = str(tmp_path / "shim_solve")
    subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "host", "shim_solve.cpp"), f"-L{libdir}", "-lwrapd_gpu",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    bar = bars.bar_8x8x32()
    files = {n: str(tmp_path / f"{n}.bin") for n in ("rest", "init", "tets", "pins", "x", "obj")}
    np.asarray(bar.rest, np.float64).tofile(files["rest"])
    np.asarray(bar.init, np.float64).tofile(files["init"])
    np.asarray(bar.tets, np.int32).tofile(files["tets"])
    np.asarray(bar.pins, np.int32).tofile(files["pins"])
    r = subprocess.run([exe, files["rest"], files["init"], files["tets"], files["pins"], "1e5", "60", files["x"],
                        files["obj"]], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    x_cpp = np.fromfile(files["x"]).reshape(-1, 3)
    obj_cpp = np.fromfile(files["obj"])

    s = Solver(youngs=1e5, max_iters=60)
    s.add_tetmesh(bar.rest, bar.init, bar.tets)
    s.set_pins(bar.pins)
    s.initialize()
    x = s.solve()
    d = s.algorithm_data()
    assert obj_cpp.size == d.objectives.size > 1
    assert np.array_equal(obj_cpp, d.objectives)
    assert np.array_equal(x_cpp, x)
    s.close()

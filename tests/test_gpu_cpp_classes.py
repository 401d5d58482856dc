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


QUASI_COMPAT = os.path.join(ROOT, "oracle", "_ref", "quasi_compat")


def test_reference_front_end_on_the_dropin_headers(lib_built, golden, tmp_path):
    """The reference's samples/tests/quasi.cpp, unchanged, built against
    include/wrapd and the GPU library (oracle/_ref/quasi_compat, made where the
    reference sources are present), run on the small bar: its own log and mesh
    writers give the reference's files (tests/golden/quasi_small.npz) within
    the FP64 parity tolerances of test_gpu_quasi.py."""
    from test_gpu_quasi import _compare
    if not os.path.exists(QUASI_COMPAT):
        pytest.skip("oracle/_ref/quasi_compat not built (needs the reference sources)")
    b = bars.make_bar(3, 3, 8, twist_deg=90.0, noise=0.02, seed=5)
    files = bars.write_bar(b, str(tmp_path), "q")
    run = tmp_path / "run"
    run.mkdir()
    r = subprocess.run([QUASI_COMPAT, "-rest", files["rest"], "-init", files["init"], "-handles", files["handles"],
                        "-youngs", "1e5", "-poisson", "0.45", "-it", "40", "-p", "0", "-s", "1"],
                       capture_output=True, text=True, timeout=300, cwd=str(run))
    assert r.returncode == 0, r.stdout + r.stderr
    ours = {name: (run / (name if "." in name else name + ".txt")).read_text()
            for name in ("objectives", "x_errors", "reweighted", "final_mesh.node", "final_mesh.ele",
                         "final_mesh.obj")}
    _compare(golden("quasi_small.npz"), "plain", ours)

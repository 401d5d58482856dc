"""The host-side setup on the CPU, through a small C++ driver
(tests/host/assembly_check.cpp) built against wrapd_b200/csrc/symbolic.cpp:
the assembly scatter map lists, for every entry of A, exactly the element
slots that hold both of its vertices in element order and puts the entry in
the lower triangle of the front that owns its column; and the free-vertex
graph, the analysis and the map do not change with the number of host
threads."""
import dataclasses
import os
import shutil
import subprocess

import numpy as np
import pytest

from wrapd_b200 import bars

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("host") / "assembly_check")
    subprocess.run([gxx, "-O2", "-std=c++17", "-pthread", os.path.join(ROOT, "tests", "host", "assembly_check.cpp"),
                    os.path.join(ROOT, "wrapd_b200", "csrc", "symbolic.cpp"), "-o", exe], check=True)
    return exe


def check(exe, bar, tmp_path, threads=8):
    paths = [str(tmp_path / n) for n in ("rest.bin", "tets.bin", "pins.bin")]
    np.asarray(bar.rest, np.float64).tofile(paths[0])
    np.asarray(bar.tets, np.int32).tofile(paths[1])
    np.asarray(bar.pins, np.int32).tofile(paths[2])
    r = subprocess.run([exe, *paths, str(threads)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr


def test_scatter_map_of_the_8x8x32_bar(checker, tmp_path):
    check(checker, bars.bar_8x8x32(), tmp_path)


def test_scatter_map_with_scattered_pins(checker, tmp_path):
    b = bars.make_bar(6, 5, 20, twist_deg=30.0, noise=0.03, seed=4)
    rng = np.random.default_rng(2)
    extra = rng.choice(np.setdiff1d(np.arange(b.n_verts), b.pins), 40, replace=False)
    check(checker, dataclasses.replace(b, pins=np.sort(np.concatenate([b.pins, extra])).astype(np.int32)), tmp_path)


def test_setup_of_the_786k_bar_is_thread_count_independent(checker, tmp_path):
    """138,303 free vertices: every threaded phase runs on several threads."""
    check(checker, bars.bar_32x32x128_bent(), tmp_path, threads=8)


def test_cpp_classes_over_the_abi(lib_built, tmp_path):
    """include/wrapd_gpu.hpp (wrapd::gpu::Solver, Settings, AlgorithmData):
    defaults, the reference's messages as std::runtime_error, and, with no
    usable GPU, initialize() failing loudly."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    libdir = os.path.dirname(lib_built)
    exe = str(tmp_path / "shim_check")
    subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "host", "shim_check.cpp"), f"-L{libdir}", "-lwrapd_gpu",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    try:
        import torch
        gpu = torch.cuda.is_available()
    except ImportError:
        gpu = False
    r = subprocess.run([exe] + ([] if gpu else ["nogpu"]), capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr

"""The drop-in headers (include/wrapd: Solver.hpp, System.hpp, TetElements.hpp,
Settings.hpp, ... with the reference's file and class names) on the CPU.

* The reference's own front end, samples/tests/quasi.cpp, unchanged, builds
  against them and the GPU library in place of the reference's src/ (only the
  include path differs), and so does the repository's driver of the reference
  (oracle/ref_quasi.cpp), which reaches further into the classes (m_system,
  AlgorithmData's members, the Lame parameters).  Both need the reference's
  sources and its vendored Eigen, so these skip where they are absent.
* Settings::parse_args keeps the reference's flags, defaults and errors, and
  to_c() hands them to the C ABI unchanged (tests/host/dropin_check.cpp).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ref_dir():
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"], capture_output=True,
                       text=True)
    ref = r.stdout.strip()
    return ref if ref and os.path.exists(os.path.join(ref, "samples", "tests", "quasi.cpp")) else None


def _compile(src, exe, lib_built, ref, extra=()):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    libdir = os.path.dirname(lib_built)
    cmd = [gxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include", "wrapd"),
           "-isystem", os.path.join(ref, "deps", "Eigen3"), *extra, src, f"-L{libdir}", "-lwrapd_gpu",
           f"-Wl,-rpath,{libdir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return r.stderr


def test_reference_front_end_builds_unchanged(lib_built, tmp_path):
    ref = _ref_dir()
    if ref is None:
        pytest.skip("reference sources not present")
    _compile(os.path.join(ref, "samples", "tests", "quasi.cpp"), str(tmp_path / "quasi"), lib_built, ref,
             ["-isystem", os.path.join(ref, "samples", "utils"), '-DWRAPD_OUTPUT_DIR="."'])


def test_reference_driver_builds_against_the_headers(lib_built, tmp_path):
    ref = _ref_dir()
    if ref is None:
        pytest.skip("reference sources not present")
    err = _compile(os.path.join(ROOT, "oracle", "ref_quasi.cpp"), str(tmp_path / "drv"), lib_built, ref,
                   ["-isystem", os.path.join(ref, "samples", "utils")])
    assert "include/wrapd" not in err    # no warning from the headers themselves


def test_settings_and_classes_on_the_cpu(lib_built, tmp_path):
    """Flags, defaults, errors and the no-GPU failure of the drop-in classes
    (tests/host/dropin_check.cpp needs Eigen: the reference's vendored copy)."""
    ref = _ref_dir()
    if ref is None:
        pytest.skip("no Eigen: the reference's vendored copy is absent")
    exe = str(tmp_path / "dropin_check")
    _compile(os.path.join(ROOT, "tests", "host", "dropin_check.cpp"), exe, lib_built, ref)
    try:
        import torch
        gpu = torch.cuda.is_available()
    except ImportError:
        gpu = False
    r = subprocess.run([exe] + ([] if gpu else ["nogpu"]), capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok" in r.stdout

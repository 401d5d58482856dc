"""The command-line front end (wrapd_b200/_lib/quasi, C++ over the C ABI)
against the reference's own front end on the same input files
(tests/golden/quasi_small.npz): the four logs, final_mesh.node/.ele and
final_mesh.obj, without and with -soln (which stops on the x error).

Tolerances: FP64 energies and positions within 1e-8 relative; the .ele file
byte for byte; the .obj boundary faces as a set of oriented triangles (the
reference emits them in hash-table order)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from wrapd_b200 import bars

pytestmark = pytest.mark.gpu
QUASI = os.path.join(ROOT, "wrapd_b200", "_lib", "quasi")


@pytest.fixture(scope="module", autouse=True)
def _built(lib_built):
    assert os.path.exists(QUASI)


def _text(g, key):
    return bytes(g[key]).decode()


def _log(txt):
    a = np.array([[float(v) for v in line.split()] for line in txt.strip().splitlines()])
    np.testing.assert_array_equal(a[:, 0], np.arange(a.shape[0]))
    return a[:, 1]


def _node(txt):
    lines = txt.splitlines()
    n = int(lines[0].split()[0])
    return np.array([[float(v) for v in l.split()[1:4]] for l in lines[1:1 + n]])


def _obj(txt):
    v, f = [], set()
    for line in txt.splitlines():
        p = line.split()
        if p and p[0] == "v":
            v.append([float(x) for x in p[1:4]])
        elif p and p[0] == "f":
            a, b, c = (int(x) for x in p[1:4])
            m = min(range(3), key=lambda i: (a, b, c)[i])   # rotate to the smallest id first
            f.add(tuple((a, b, c)[(m + k) % 3] for k in range(3)))
    return np.array(v), f


def _run(tmp_path, tag, extra, it):
    b = bars.make_bar(3, 3, 8, twist_deg=90.0, noise=0.02, seed=5)
    files = bars.write_bar(b, str(tmp_path), "q")
    od = tmp_path / tag
    od.mkdir()
    cmd = [QUASI, "-rest", files["rest"], "-init", files["init"], "-handles", files["handles"], "-youngs", "1e5",
           "-poisson", "0.45", "-it", str(it), "-p", "0", "-out", str(od), *extra]
    subprocess.run(cmd, check=True, capture_output=True, timeout=300)
    return {name: (od / (name if "." in name else name + ".txt")).read_text()
            for name in ("objectives", "x_errors", "reweighted", "final_mesh.node", "final_mesh.ele",
                         "final_mesh.obj")}


def _compare(g, tag, ours):
    ref_obj = _log(_text(g, f"{tag}/objectives"))
    obj = _log(ours["objectives"])
    assert len(obj) == len(ref_obj)
    np.testing.assert_allclose(obj, ref_obj, rtol=1e-8)
    # x errors are |x - x_soln| / |x_init - x_soln|: positions agreeing to 1e-8
    # give agreement to ~1e-7 absolute, also where x reaches x_soln
    np.testing.assert_allclose(_log(ours["x_errors"]), _log(_text(g, f"{tag}/x_errors")), rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(_log(ours["reweighted"]), _log(_text(g, f"{tag}/reweighted")))
    assert ours["final_mesh.ele"] == _text(g, f"{tag}/final_mesh.ele")
    Xr = _node(_text(g, f"{tag}/final_mesh.node"))
    X = _node(ours["final_mesh.node"])
    assert np.abs(X - Xr).max() <= 1e-8 * np.abs(Xr).max()
    assert ours["final_mesh.node"].splitlines()[0] == _text(g, f"{tag}/final_mesh.node").splitlines()[0]
    vo, fo = _obj(ours["final_mesh.obj"])
    vr, fr = _obj(_text(g, f"{tag}/final_mesh.obj"))
    assert fo == fr
    assert np.abs(vo - vr).max() <= 1e-8 * np.abs(vr).max()


def test_front_end_matches_reference_files(golden, tmp_path):
    g = golden("quasi_small.npz")
    _compare(g, "plain", _run(tmp_path, "plain", [], 40))


def test_front_end_soln_stops_on_x_error(golden, tmp_path):
    """-soln set to the reference's own iterate 40: both stop there on the
    x-error test (ADMM::converged, src/ADMM.cpp:158-169)."""
    g = golden("quasi_small.npz")
    soln = tmp_path / "soln_in"
    soln.mkdir()
    (soln / "m.node").write_text(_text(g, "plain/final_mesh.node"))
    (soln / "m.ele").write_text(_text(g, "plain/final_mesh.ele"))
    ours = _run(tmp_path, "soln", ["-soln", str(soln / "m")], 200)
    _compare(g, "soln", ours)
    assert len(_log(ours["objectives"])) == 41

"""bench.py's stdout carries exactly one JSON line: the reference's host code
(OBJ loader, mesh builder) logs progress to stdout, and bench.py points file
descriptor 1 at stderr while it runs.  CPU only."""

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SNIPPET = r"""
import os, sys
sys.path[:0] = [{root!r}, os.path.join({root!r}, "oracle"), os.path.join({root!r}, "embree-benchmark-protoray_b200")]
import numpy as np
import bench, oracle, scenes
m, _ = scenes.small_scene()
obj = os.path.join({tmp!r}, "s.obj")
with open(obj, "w") as f:
    np.savetxt(f, m.positions, fmt="v %.9g %.9g %.9g")
    np.savetxt(f, m.indices + 1, fmt="f %d %d %d")
R = oracle.Reference()
with bench.c_stdout_to_stderr():
    t, n = R.load_obj(obj)
    R.build_soup(t, n, os.path.join({tmp!r}, "s.mesh"))
print('{{"metric": "x"}}')
"""


def test_reference_logs_go_to_stderr(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.Reference.available():
        pytest.skip("oracle/_ref not built")
    code = SNIPPET.format(root=ROOT, tmp=str(tmp_path))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout == '{"metric": "x"}\n'
    assert "Loading OBJ file" in r.stderr

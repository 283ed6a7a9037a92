"""The C++ command line (`protoray render`) on the B200 device: the reference's
flags, its stats files and its PPM output."""

import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "embree-benchmark-protoray_b200", "protoray")


def _read_ppm(path):
    data = open(path, "rb").read()
    parts = data.split(b"\n", 3)
    assert parts[0] == b"P6" and parts[2] == b"255"
    w, h = map(int, parts[1].split())
    return w, h, np.frombuffer(parts[3], np.uint8).reshape(h, w, 3)


def test_cli_benchmark_run(tmp_path, small):
    import prt
    import scenes
    mesh, view = small
    path = scenes.write_scene(str(tmp_path), "small", mesh, view)
    prefix = str(tmp_path / "bench")
    r = subprocess.run([EXE, "render", path, "-no-mtl", "-r", "diffuse", "-spp", "6", "-size", "64,48",
                        "-maxDepth", "4", "-dev", "b200", "-benchmark", prefix], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    stats = dict(l.strip().split("=", 1) for l in open(prefix + ".txt") if "=" in l)
    for k in ("stats_mray", "stats_ray", "stats_buildMs", "stats_buildMprim", "stats_renderMs"):
        assert k in stats, stats
    assert float(stats["stats_mray"]) > 0
    rows = open(prefix + ".csv").read().strip().split("\n")
    assert len(rows) == 1 + (6 - 6 // 6)     # header + frames after the warm-up
    w, h, img = _read_ppm(prefix + ".ppm")
    assert (w, h) == (64, 48)
    # the same render through the C ABI
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.init_frame(64, 48)
    c.set_view(view, 64, 48)
    c.render(6, 4)
    ldr = c.read_ldr()
    bgr = np.stack([ldr & 0xFF, (ldr >> 8) & 0xFF, (ldr >> 16) & 0xFF], axis=-1).astype(np.int64)
    assert np.max(np.abs(img.astype(np.int64) - bgr)) <= 1


def test_cli_rejects_bad_options(tmp_path, small):
    import scenes
    path = scenes.write_scene(str(tmp_path), "small", *small)
    r = subprocess.run([EXE, "render", path, "-spp", "1", "-size", "63,48", "-o", str(tmp_path / "x")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "multiple of 8" in r.stderr
    r = subprocess.run([EXE, "render", path, "-spp", "1", "-r", "ao", "-o", str(tmp_path / "x")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "invalid renderer type" in r.stderr
    r = subprocess.run([EXE, "render", str(tmp_path / "none.mesh"), "-spp", "1", "-o", str(tmp_path / "x")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 1


def test_cli_config_file_and_default_view(tmp_path, small):
    import scenes
    mesh, _ = small
    mpath = str(tmp_path / "noview.mesh")
    scenes.write_mesh(mpath, mesh)            # no .view file: the default view
    cfg = tmp_path / "run.cfg"
    cfg.write_text("noview.mesh -spp 2 -size 32,32 -maxDepth 2\n")   # relative to the config file
    r = subprocess.run([EXE, "render", "-c", str(cfg), "-o", str(tmp_path / "cfg")], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Default view" in r.stdout
    assert os.path.exists(str(tmp_path / "cfg.ppm"))


def test_cli_checkpoint_images(tmp_path, small):
    """-checkpoint writes <prefix>_<spp>spp.ppm at every power-of-two spp
    (main/render/render_window.cpp:279-292); the last equals the final image."""
    import scenes
    path = scenes.write_scene(str(tmp_path), "small", *small)
    prefix = str(tmp_path / "cp")
    r = subprocess.run([EXE, "render", path, "-spp", "5", "-size", "32,24", "-maxDepth", "3", "-checkpoint",
                        "-o", prefix], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    for n in (1, 2, 4):
        assert os.path.exists(f"{prefix}_{n:06d}spp.ppm")
    assert not os.path.exists(f"{prefix}_000003spp.ppm") and not os.path.exists(f"{prefix}_000005spp.ppm")
    assert _read_ppm(f"{prefix}_000004spp.ppm")[2].shape == (24, 32, 3)

"""The reference's own render loop on the B200 device.

oracle/_ref/protoray_refloop links the reference's unmodified RenderWindow,
Window, StatsRecorder and ViewSet (main/render/render_window.cpp,
window.cpp, stats_recorder.cpp, view.cpp), its sys/ and image/ code, and
DeviceB200 (host/reference_device_b200.h) over the C ABI; oracle/Makefile
builds it from the reference sources (target refloop).  Run in benchmark
mode with 6 spp at 64x48 (render/device.h's Device interface driven one pass
per frame, main/render/render_window.cpp:164-305), the files the reference
writes must hold its stats (stats_mray, stats_ray, stats_buildMs, averaged
after the first spp/6 frames) and the image the library renders for the same
passes."""

import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "protoray_refloop")


def _read_ppm(path):
    data = open(path, "rb").read()
    parts = data.split(b"\n", 3)
    assert parts[0] == b"P6" and parts[2] == b"255"
    w, h = map(int, parts[1].split())
    return np.frombuffer(parts[3], np.uint8).reshape(h, w, 3)


@pytest.mark.skipif(not os.path.exists(EXE), reason="reference render loop not built (oracle/Makefile refloop)")
@pytest.mark.parametrize("renderer", ["diffuse", "diffuse2"])
def test_reference_render_loop_on_b200(renderer, tmp_path, small):
    import prt
    import scenes
    mesh, view = small
    scene = scenes.write_scene(str(tmp_path), "small", mesh, view)
    W, H, spp, depth = 64, 48, 6, 5
    prefix = str(tmp_path / "bench")
    r = subprocess.run([EXE, scene, str(W), str(H), str(spp), str(depth), renderer, prefix],
                       capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    stats = {}
    for line in open(prefix + ".txt"):
        k, v = line.strip().split("=", 1)
        stats[k] = v
    for k in ("stats_mray", "stats_ray", "stats_buildMs", "stats_buildMprim"):
        assert k in stats, (k, sorted(stats))
    assert float(stats["stats_mray"]) > 0 and float(stats["stats_buildMs"]) > 0
    csv = open(prefix + ".csv").read().splitlines()
    assert len(csv) >= spp - spp // 6   # one row per frame after the warm-up frames (plus a header)
    img = _read_ppm(prefix + ".ppm")
    assert img.shape == (H, W, 3)

    # the same passes through the library directly (one call of 6 passes)
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.set_integrator(renderer)
    c.build()
    c.init_frame(W, H)
    c.set_view(view, W, H)
    st = c.render(spp, depth)
    ldr = c.read_ldr().view(np.uint8).reshape(H, W, 4)[..., :3]
    # rays of one frame (one pass): the loop averages frames after the warm-up
    c.clear()
    one = c.render(1, depth)
    assert abs(float(stats["stats_ray"]) - one["ray"]) <= 0.05 * one["ray"]
    c.close()
    diff = np.abs(img.astype(int) - ldr.astype(int))
    # float sums in another order can move a byte by one
    assert diff.max() <= 1 and (diff > 0).mean() < 0.01, (diff.max(), (diff > 0).mean())
    assert st["ray"] > 0

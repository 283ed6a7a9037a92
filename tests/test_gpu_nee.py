"""The diffuse2 integrator (shadow ray toward the sky at every bounce, fixed
0.5 MIS weights; render/diffuse2_integrator_single.h:41-90) on the GPU
against the FP64 oracle, which the golden reference diffuse2 image pins."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_err(a, b):
    return float(np.mean(np.abs(a - b) / np.maximum(np.abs(b), 1e-2)))


@pytest.mark.parametrize("albedo", [False, True])
def test_nee_image_parity(small, small_oracle, oracle_mod, albedo):
    import prt
    import scenes
    mesh, view = small
    W, H, spp, depth = 128, 96, 8, 4
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.set_integrator("diffuse2")
    alb = scenes.albedo_for(mesh) if albedo else None
    if albedo:
        c.set_albedo(alb)
        c.set_sky(1.5)
    c.init_frame(W, H)
    c.set_view(view, W, H)
    st = c.render(spp, depth)
    img = c.read_accum()
    ref, rays = small_oracle.render(oracle_mod.Oracle().camera(view, W, H), W, H, 0, spp, depth, albedo=alb,
                                    sky=1.5 if albedo else 1.0, nee=True)
    assert np.all(img[..., 3] == spp)
    assert _rel_err(img[..., 0], ref[..., 0]) < 1e-3
    assert abs(st["ray"] - rays) <= 1e-3 * rays
    # the per-bounce profiling path runs the same kernels (it counts extension rays only)
    ms, r = c.render_profile(spp, depth)
    assert ms.sum() > 0 and r[0] == W * H * spp


def test_nee_differs_from_plain_and_cli(tmp_path, small):
    import subprocess
    import os
    import prt
    import scenes
    mesh, view = small
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.init_frame(32, 32)
    c.set_view(view, 32, 32)
    c.render(4, 3)
    plain = c.read_accum().copy()
    c.set_integrator("diffuse2")
    c.clear()
    c.render(4, 3)
    nee = c.read_accum()
    # both estimate the same image (same expectation), with different noise
    assert abs(plain[..., 0].mean() - nee[..., 0].mean()) < 0.1 * plain[..., 0].mean()
    assert not np.array_equal(plain, nee)
    with pytest.raises(ValueError):
        c.set_integrator("ao")
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "embree-benchmark-protoray_b200",
                       "protoray")
    path = scenes.write_scene(str(tmp_path), "small", mesh, view)
    r = subprocess.run([exe, "render", path, "-r", "diffuse2", "-spp", "2", "-size", "32,32", "-o",
                        str(tmp_path / "d2")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr

"""prt_render_noalloc — the render entry point for callers that cannot
allocate device memory at render time (an application that owns the GPU's
memory through its own pool, or a frame loop that cannot afford cudaMalloc's
implicit synchronisation).  Its scratch lives in a fixed device array inside
the library.

Checked through the C ABI against prt_render, the allocating entry point, on
two calls in a row (the second call reuses the array the first one left
behind), within the tolerance the other image tests use for float-atomic
reassociation: one wave, several waves (a frame that fills the array, one
pass per wave), per-triangle albedo, the diffuse2 integrator and primary rays
as warp packets (the context's launch configuration).  This file is collected
last on purpose."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _context(small, W, H, albedo=None, integrator="diffuse"):
    import prt
    mesh, view = small
    ctx = prt.Context(0)
    ctx.load_mesh(mesh.indices, mesh.positions)
    if albedo is not None:
        ctx.set_albedo(albedo)
    ctx.set_integrator(integrator)
    ctx.build()
    ctx.init_frame(W, H)
    cam = prt.camera_from_view(view, W, H)
    ctx.set_camera(cam)
    return ctx, cam


def _check_twice(ctx, cam, W, H, spp, depth):
    st = ctx.render(spp, depth)
    ref = ctx.read_accum().copy()
    for call in range(2):
        acc = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        rays = ctx.render_noalloc(cam, W, H, 0, spp, depth, acc)
        torch.cuda.synchronize()
        got = acc.cpu().numpy()
        assert rays == st["ray"], (call, rays, st["ray"])
        assert np.all(got[..., 3] == spp)
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5)


def test_noalloc_matches_render_twice(small):
    W, H = 200, 120
    ctx, cam = _context(small, W, H)
    _check_twice(ctx, cam, W, H, spp=4, depth=5)
    ctx.close()


def test_noalloc_multi_wave(small):
    # 1024 x 512 fills the fixed array: one pass per wave, three waves
    W, H = 1024, 512
    ctx, cam = _context(small, W, H)
    _check_twice(ctx, cam, W, H, spp=3, depth=5)
    ctx.close()


def test_noalloc_per_triangle_albedo(small):
    mesh, _ = small
    rng = np.random.default_rng(7)
    albedo = rng.uniform(0.2, 0.8, len(mesh.indices)).astype(np.float32)
    W, H = 160, 96
    ctx, cam = _context(small, W, H, albedo=albedo)
    _check_twice(ctx, cam, W, H, spp=4, depth=5)
    ctx.close()


@pytest.mark.parametrize("packets", [1, 2])
def test_noalloc_packet_primaries(small, packets):
    """Depth 0 as warp packets with per-ray (1) or interval (2) node tests:
    the entry point launches the context's configuration as prt_render does."""
    W, H = 200, 120
    ctx, cam = _context(small, W, H)
    ctx.set_tune(128, 0, 0, 0, packets)
    _check_twice(ctx, cam, W, H, spp=4, depth=5)
    ctx.close()


def test_noalloc_diffuse2(small):
    W, H = 160, 96
    ctx, cam = _context(small, W, H, integrator="diffuse2")
    _check_twice(ctx, cam, W, H, spp=4, depth=4)
    ctx.close()


def test_noalloc_rejects_oversized_frames(small):
    import prt
    W, H = 1920, 1080
    ctx, cam = _context(small, 64, 64)
    cam = prt.camera_from_view(small[1], W, H)
    acc = torch.zeros((8, 8, 4), dtype=torch.float32, device="cuda")   # never written
    with pytest.raises(prt.PrtError) as e:
        ctx.render_noalloc(cam, W, H, 0, 1, 5, acc)
    assert e.value.status == prt.PRT_EINVAL and "too large" in str(e.value)
    ctx.close()


def test_noalloc_rejects_unusable_accum(small):
    # a host buffer or a misaligned device pointer is refused on the host,
    # before anything is launched
    import prt
    W, H = 64, 48
    ctx, cam = _context(small, W, H)
    host = np.zeros((H, W, 4), np.float32)
    with pytest.raises(prt.PrtError) as e:
        ctx.render_noalloc(cam, W, H, 0, 1, 5, host)
    assert e.value.status == prt.PRT_EINVAL and "device memory" in str(e.value)
    dev = torch.zeros(H * W * 4 + 4, dtype=torch.float32, device="cuda")

    class Shifted:
        def data_ptr(self):
            return dev.data_ptr() + 4

    with pytest.raises(prt.PrtError) as e:
        ctx.render_noalloc(cam, W, H, 0, 1, 5, Shifted())
    assert e.value.status == prt.PRT_EINVAL
    assert float(dev.abs().sum()) == 0.0
    ctx.close()

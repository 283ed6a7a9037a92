"""prt_render_noalloc — the render entry point for callers that cannot
allocate device memory at render time (an application that owns the GPU's
memory through its own pool, or a frame loop that cannot afford cudaMalloc's
implicit synchronisation).  Its scratch lives in a fixed device array inside
the library.

Checked through the C ABI against prt_render, the allocating entry point, on
two calls in a row (the second call reuses the array the first one left
behind), within the tolerance the other image tests use for float-atomic
reassociation.  This file is collected last on purpose."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_noalloc_matches_render_twice(small):
    import prt
    mesh, view = small
    W, H, spp, depth = 200, 120, 4, 5
    ctx = prt.Context(0)
    ctx.load_mesh(mesh.indices, mesh.positions)
    ctx.build()
    ctx.init_frame(W, H)
    cam = prt.camera_from_view(view, W, H)
    ctx.set_camera(cam)
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
    ctx.close()


def test_noalloc_rejects_oversized_frames(small):
    import prt
    mesh, view = small
    ctx = prt.Context(0)
    ctx.load_mesh(mesh.indices, mesh.positions)
    ctx.build()
    W, H = 1920, 1080
    cam = prt.camera_from_view(view, W, H)
    acc = torch.zeros((8, 8, 4), dtype=torch.float32, device="cuda")   # never written
    with pytest.raises(prt.PrtError) as e:
        ctx.render_noalloc(cam, W, H, 0, 1, 5, acc)
    assert e.value.status == prt.PRT_EINVAL and "too large" in str(e.value)
    ctx.close()

"""Parity of the GPU's own ray generation with the FP64 oracle, per pixel.

Two checks pin the camera rays the renderer traces first
(generateRaysKernel, render/diffuse_renderer_cuda.cu:27-59;
RendererSingle::renderTile, render/renderer_single.h:107-124;
RandomSampler, sampling/random_sampler.h:44-73):

* prt_primary_rays writes the rays that the bounce kernels' first depth
  generates (same item -> pixel mapping, RNG seeding and camera_ray); they
  equal the oracle's primary rays to a few float ulps at every pixel, and the
  primitive ids they hit equal the oracle's at every pixel the oracle does
  not flag as grazing;
* a maxDepth-0 render (the fused render kernel itself, per-lane or as warp
  packets, with per-ray or interval node tests) adds 1 to a pixel whose primary ray escapes and 0 to one that hits:
  its per-pixel hit/miss mask equals the oracle's at every unflagged pixel.

C0 frame: 256 x 256, passes 0 and 7, pinhole and thin lens.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx_c0(small):
    import prt
    mesh, _ = small
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.init_frame(256, 256)
    yield c
    c.close()


def _view(small, lens):
    import scenes
    _, view = small
    if not lens:
        return view
    return scenes.View(view.pos, view.angleX, view.angleY, view.fovY, lens, 38.0)


@pytest.mark.parametrize("lens", [0.0, 0.3])
@pytest.mark.parametrize("pass_", [0, 7])
def test_primary_rays_match_oracle(ctx_c0, small, small_oracle, oracle_mod, lens, pass_):
    W, H = 256, 256
    view = _view(small, lens)
    ctx_c0.set_view(view, W, H)
    O = oracle_mod.Oracle()
    ref = O.primary_rays(O.camera(view, W, H), W, H, pass_)
    dev = torch.empty((W * H, 8), dtype=torch.float32, device="cuda")
    ctx_c0.primary_rays(pass_, dev)
    torch.cuda.synchronize()
    got = dev.cpu().numpy()
    # origins: the camera position (pinhole) or a point on the lens disk
    np.testing.assert_allclose(got[:, 0:3], ref[:, 0:3], rtol=1e-6, atol=4e-6)
    # unit directions: a few ulps (the reference normalises with rsqrt + Newton)
    np.testing.assert_allclose(got[:, 4:7], ref[:, 4:7], rtol=0, atol=6e-7)
    assert np.all(got[:, 3] == 0) and np.all(got[:, 7] == ref[:, 7])

    # the GPU's rays hit the oracle's primitives at every unflagged pixel
    want, flags = small_oracle.intersect(ref, flags=True)
    hits = torch.empty((W * H, 4), dtype=torch.float32, device="cuda")
    ctx_c0.intersect(dev, hits, W * H)
    torch.cuda.synchronize()
    gp = hits.cpu().numpy()[:, 1].view(np.int32)
    rp = want[:, 1].view(np.int32)
    bad = (gp != rp) & (flags == 0)
    assert bad.sum() == 0, (int(bad.sum()), int(((gp != rp)).sum()))
    assert (rp >= 0).mean() > 0.2 and (rp < 0).mean() > 0.05   # the view sees geometry and sky


@pytest.mark.parametrize("packets", [0, 1, 2])
@pytest.mark.parametrize("lens", [0.0, 0.3])
@pytest.mark.parametrize("pass_", [0, 7])
def test_depth0_render_hit_mask_matches_oracle(ctx_c0, small, small_oracle, oracle_mod, lens, pass_, packets):
    """packets 1: depth 0 runs the warp-packet kernel (k_primary_packet); 2: its
    interval traversal."""
    W, H = 256, 256
    view = _view(small, lens)
    ctx_c0.set_tune(128, 0, 0, 0, packets)
    ctx_c0.set_view(view, W, H)
    ctx_c0.set_pass(pass_)
    st = ctx_c0.render(1, 0, accumulate=False)
    img = ctx_c0.read_accum().reshape(W * H, 4)
    assert st["ray"] == W * H
    assert np.all(img[:, 3] == 1.0)
    assert np.all((img[:, 0] == 0.0) | (img[:, 0] == 1.0))
    O = oracle_mod.Oracle()
    ref = O.primary_rays(O.camera(view, W, H), W, H, pass_)
    want, flags = small_oracle.intersect(ref, flags=True)
    miss_ref = want[:, 1].view(np.int32) < 0
    miss_gpu = img[:, 0] == 1.0
    bad = (miss_gpu != miss_ref) & (flags == 0)
    assert bad.sum() == 0, (int(bad.sum()), int((miss_gpu != miss_ref).sum()))

"""Path-replay adjoint (prt_render_backward) of an L2 image loss with respect
to per-triangle albedo and sky radiance, through a torch.autograd.Function
(tests/autograd_fn.py).  Checked against the FP64 CPU adjoint of the oracle
and against central finite differences (eps 1e-3); tolerance 1e-2 relative."""

import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(small):
    import prt
    import scenes
    mesh, view = small
    W, H, spp, depth = 96, 96, 4, 3
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.init_frame(W, H)
    c.set_view(view, W, H)
    # one pass per wave: each pixel receives its samples in pass order, so
    # forward images are bit-reproducible for the finite differences
    c.set_tune(128, 0, 1)
    alb = scenes.albedo_for(mesh)
    rng = np.random.default_rng(9)
    target_alb = np.clip(alb + rng.normal(0, 0.05, size=alb.shape).astype(np.float32), 0.05, 0.95)
    return c, mesh, view, (W, H, spp, depth), alb, target_alb


def test_adjoint_matches_oracle_and_fd(setup, small_oracle, oracle_mod):
    from autograd_fn import PathTrace
    c, mesh, view, (W, H, spp, depth), alb, target_alb = setup
    dev = "cuda"
    sky0 = 1.3
    with torch.no_grad():
        target = PathTrace.apply(torch.from_numpy(target_alb).to(dev), torch.tensor([sky0], device=dev), c, spp,
                                 depth).clone()
    a = torch.from_numpy(alb).to(dev).requires_grad_(True)
    s = torch.tensor([sky0], device=dev, requires_grad=True)
    img = PathTrace.apply(a, s, c, spp, depth)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    g_alb = a.grad.cpu().numpy().astype(np.float64)
    g_sky = float(s.grad.item())

    # FP64 oracle adjoint with the same dL/dsum
    dimg = (2.0 * (img - target)).detach().cpu().numpy().astype(np.float64)
    cam = oracle_mod.Oracle().camera(view, W, H)
    o_alb, o_sky = small_oracle.render_backward(cam, W, H, 0, spp, depth, alb, sky0, dimg / spp)
    # every one of the 200 largest gradients within 1e-2 (observed: at most 2e-5)
    top = np.argsort(-np.abs(o_alb))[:200]
    rel = np.abs(g_alb[top] - o_alb[top]) / np.maximum(np.abs(o_alb[top]), 1e-12)
    assert np.median(rel) < 1e-4 and np.all(rel < 1e-2), (np.median(rel), rel.max())
    assert abs(g_sky - o_sky) <= 1e-2 * abs(o_sky)
    np.testing.assert_allclose(np.linalg.norm(g_alb), np.linalg.norm(o_alb), rtol=1e-2)

    # central finite differences on the largest gradients and on the sky
    eps = 1e-3

    def L(alb_np, sky):
        with torch.no_grad():
            im = PathTrace.apply(torch.from_numpy(alb_np).to(dev), torch.tensor([sky], device=dev), c, spp, depth)
            return float(((im.double() - target.double()) ** 2).sum())

    for i in np.argsort(-np.abs(g_alb))[:6]:
        ap = alb.copy(); ap[i] += eps
        am = alb.copy(); am[i] -= eps
        fd = (L(ap, sky0) - L(am, sky0)) / (2 * eps)
        assert abs(fd - g_alb[i]) <= 1e-2 * abs(fd) + 1e-6, (i, fd, g_alb[i])
    fd = (L(alb, sky0 + eps) - L(alb, sky0 - eps)) / (2 * eps)
    assert abs(fd - g_sky) <= 1e-2 * abs(fd), (fd, g_sky)


def test_replay_forward_equals_wavefront(setup):
    c, mesh, view, (W, H, spp, depth), alb, _ = setup
    c.set_albedo(alb)
    c.set_sky(1.0)
    c.clear()
    st1 = c.render(spp, depth)
    a = c.read_accum().copy()
    c.clear()
    st2 = c.render_replay(0, spp, depth)
    b = c.read_accum()
    assert st1["ray"] == st2["ray"]
    np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6)
    c.set_albedo(None)

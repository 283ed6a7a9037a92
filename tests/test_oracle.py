"""Pins the FP64 C restatement (oracle/prt_oracle.c) against vectors produced by
the reference's own CPU code (tests/golden/make_golden.py)."""

import hashlib

import numpy as np
import pytest


def test_small_scene_matches_golden_scene(small, golden):
    mesh, _ = small
    h = hashlib.sha256()
    h.update(mesh.positions.tobytes())
    h.update(mesh.indices.tobytes())
    assert h.hexdigest().encode() == bytes(golden["small_digest"])


def test_rng_streams_bit_exact(golden, oracle_mod):
    O = oracle_mod.Oracle()
    for (p, px), states, values in zip(golden["rng_pairs"], golden["rng_states"], golden["rng_values"]):
        s = O.rng_seed(int(p), int(px))
        assert s == int(states[0])
        for k in range(len(values)):
            s = O.lcg_next(s)
            assert s == int(states[k + 1])
            assert np.float32(O.unorm(s)) == values[k]


def test_unorm_rounds_to_nearest(oracle_mod):
    O = oracle_mod.Oracle()
    # 0xFFFFFF80 and above round up to 2^32 -> 1.0 (math/math.h:179)
    assert O.unorm(0xFFFFFFFF) == 1.0
    assert O.unorm(0) == 0.0
    assert O.unorm(0x80000000) == 0.5


def test_camera_fields(golden, oracle_mod):
    import scenes
    O = oracle_mod.Oracle()
    for v, (w, h), ref in zip(golden["cam_views"], golden["cam_sizes"], golden["cam_fields"]):
        view = scenes.View(tuple(v[:3]), *v[3:])
        cam = O.camera(view, int(w), int(h)).as_array()
        np.testing.assert_allclose(cam, ref, rtol=0, atol=2e-6)


def test_primary_rays(golden, oracle_mod):
    import scenes
    O = oracle_mod.Oracle()
    k = 0
    for v in golden["cam_views"]:
        view = scenes.View(tuple(v[:3]), *v[3:])
        cam = O.camera(view, 32, 24)
        for p in (0, 5):
            rays = O.primary_rays(cam, 32, 24, p)
            ref = golden["primary_rays"][k]
            k += 1
            # the reference normalises with rsqrt + one Newton step; the oracle in FP64
            np.testing.assert_allclose(rays[:, :3], ref[:, :3], atol=2e-5)
            np.testing.assert_allclose(rays[:, 4:7], ref[:, 4:7], atol=1e-6)


def test_cosine_sample_and_frame(golden, oracle_mod):
    O = oracle_mod.Oracle()
    for (a, b), ref in zip(golden["cosine_in"], golden["cosine_out"]):
        np.testing.assert_allclose(O.cosine_sample(float(a), float(b)), ref, atol=2e-6)
    for n, ref in zip(golden["frame_in"], golden["frame_out"]):
        U, V = O.make_frame(n.astype(np.float64))
        np.testing.assert_allclose(U, ref[:3], atol=2e-6)
        np.testing.assert_allclose(V, ref[3:], atol=2e-6)


def test_query_hits_match_reference(golden, small_oracle):
    q = golden["query_in"]
    hits = small_oracle.intersect(q)
    prims = hits[:, 1].view(np.int32)
    assert np.array_equal(prims, golden["query_prim"])
    np.testing.assert_allclose(hits[:, 0], golden["query_dist"], rtol=1e-6)


def test_post_intersect_and_bounce(golden, small_oracle, oracle_mod):
    O = oracle_mod.Oracle()
    for row, ref in zip(golden["shade_in"], golden["shade_out"]):
        org, d, t, prim = row[0:3], row[3:6], float(row[6]), int(row[7])
        sx, sy = float(row[10]), float(row[11])
        p, eps, ng = small_oracle.post_intersect(org.astype(np.float64), d.astype(np.float64), t, prim)
        np.testing.assert_allclose(p, ref[0:3], atol=1e-5)
        assert abs(eps - ref[3]) <= 1e-6 * max(1.0, abs(ref[3]))
        np.testing.assert_allclose(ng, ref[4:7], atol=2e-6)
        U, V = O.make_frame(ng)
        np.testing.assert_allclose(U, ref[7:10], atol=2e-6)
        np.testing.assert_allclose(V, ref[10:13], atol=2e-6)
        l = O.cosine_sample(sx, sy)
        nd = l[0] * U + l[1] * V + l[2] * ng
        np.testing.assert_allclose(nd, ref[16:19], atol=3e-6)
        np.testing.assert_allclose(p + eps * nd, ref[13:16], atol=1e-5)


def _image_rel_error(a, b):
    """Mean over pixels of |a - b| / max(b, 1e-2) on the red sums."""
    return float(np.mean(np.abs(a - b) / np.maximum(np.abs(b), 1e-2)))


def test_image_matches_reference_renderer(golden, small, small_oracle, oracle_mod):
    import scenes
    mesh, view = small
    W, H, spp, depth = (int(x) for x in golden["image_cfg"])
    cam = oracle_mod.Oracle().camera(view, W, H)
    acc, rays = small_oracle.render(cam, W, H, 0, spp, depth)
    ref = golden["image_sums"]
    assert np.all(acc[..., 3] == spp) and np.all(ref[..., 3] == spp)
    assert _image_rel_error(acc[..., 0], ref[..., 0]) < 1e-3
    assert abs(rays - golden["image_rays"][0]) <= 1e-3 * rays
    # thin lens
    v = golden["image_tl_view"]
    tl = scenes.View(tuple(v[:3]), *v[3:])
    cam = oracle_mod.Oracle().camera(tl, W, H)
    acc, rays = small_oracle.render(cam, W, H, 0, 2, 3)
    assert _image_rel_error(acc[..., 0], golden["image_tl_sums"][..., 0]) < 1e-3
    assert abs(rays - golden["image_tl_rays"][0]) <= 1e-3 * rays


def test_nee_image_matches_reference_diffuse2(golden, small, small_oracle, oracle_mod):
    """The oracle's next-event-estimation path against the reference's own
    diffuse2 renderer (render/diffuse2_integrator_single.h:41-90)."""
    mesh, view = small
    W, H, spp, depth = (int(x) for x in golden["image_d2_cfg"])
    cam = oracle_mod.Oracle().camera(view, W, H)
    acc, rays = small_oracle.render(cam, W, H, 0, spp, depth, nee=True)
    ref = golden["image_d2_sums"]
    assert np.all(acc[..., 3] == spp)
    assert _image_rel_error(acc[..., 0], ref[..., 0]) < 1e-3
    assert abs(rays - golden["image_d2_rays"][0]) <= 1e-3 * rays


@pytest.mark.parametrize("nee", [False, True])
def test_listed_pixels_equal_full_render(small, small_oracle, oracle_mod, nee):
    """render_pixels (the sampled-pixel checker of full-resolution frames)
    leaves exactly the sums and ray counts that render leaves at those pixels,
    pass range and thin lens included."""
    import scenes
    mesh, view = small
    W, H, p0, spp, depth = 40, 30, 3, 3, 4
    O = oracle_mod.Oracle()
    tl = scenes.View(view.pos, view.angleX, view.angleY, view.fovY, 0.3, 38.0)
    for v in (view, tl):
        cam = O.camera(v, W, H)
        full, rays = small_oracle.render(cam, W, H, p0, spp, depth, nee=nee)
        px = np.array([0, W - 1, W * H - 1, W * (H - 1), 17, 5 * W + 33, 611], np.int32)
        got, per = small_oracle.render_pixels(cam, W, H, px, p0, spp, depth, nee=nee)
        np.testing.assert_array_equal(got, full.reshape(-1, 4)[px])
        assert np.all(per >= spp)
        every, per_all = small_oracle.render_pixels(cam, W, H, np.arange(W * H), p0, spp, depth, nee=nee)
        np.testing.assert_array_equal(every, full.reshape(-1, 4))
        assert int(per_all.sum()) == rays
    with pytest.raises(ValueError):
        small_oracle.render_pixels(O.camera(view, W, H), W, H, np.array([W * H]), 0, 1, 1)


def test_oracle_adjoint_matches_finite_differences(small, small_oracle, oracle_mod):
    """The FP64 adjoint equals the derivative of the FP64 forward (paths do not
    depend on albedo, so central differences are exact up to rounding)."""
    import scenes
    mesh, view = small
    W, H = 24, 24
    O = oracle_mod.Oracle()
    cam = O.camera(view, W, H)
    alb = scenes.albedo_for(mesh)
    target = np.zeros((H, W, 3))
    acc, _ = small_oracle.render(cam, W, H, 0, 2, 3, albedo=alb, sky=1.3)
    g = 2.0 * (acc[..., :3] - target)          # L = sum (sum_rgb - target)^2
    d_alb, d_sky = small_oracle.render_backward(cam, W, H, 0, 2, 3, alb, 1.3, g)
    idx = np.argsort(-np.abs(d_alb))[:5]
    eps = 1e-3

    def loss(a, sky):
        r, _ = small_oracle.render(cam, W, H, 0, 2, 3, albedo=a, sky=sky)
        return float(np.sum((r[..., :3] - target) ** 2))

    for i in idx:
        ap = alb.copy(); ap[i] += eps
        am = alb.copy(); am[i] -= eps
        fd = (loss(ap, 1.3) - loss(am, 1.3)) / (2 * eps)
        assert abs(fd - d_alb[i]) <= 1e-2 * abs(fd) + 1e-6
    fd = (loss(alb, 1.3 + eps) - loss(alb, 1.3 - eps)) / (2 * eps)
    assert abs(fd - d_sky) <= 1e-2 * abs(fd)


def test_empty_and_invalid_scene(oracle_mod):
    O = oracle_mod.Oracle()
    empty = O.scene(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32))
    rays = np.array([[0, 0, 0, 0, 0, 0, 1, 3e38]], np.float32)
    assert empty.intersect(rays)[0, 0] == -1.0
    with pytest.raises(ValueError):
        O.scene(np.zeros((3, 3), np.float32), np.array([[0, 1, 5]], np.int32))

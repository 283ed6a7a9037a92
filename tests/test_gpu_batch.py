"""Batched rendering (prt_render_batch): each request of an uneven batch —
different scenes, resolutions (ragged ones included), spp and depth — equals
the same request rendered alone with prt_render, within float-atomic
reassociation tolerance; ray counts add up exactly."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("paths_per_wave,packets", [(0, 0), (65536, 0), (65536, 1), (0, 1), (0, 2)])
def test_batch_equals_individual_renders(small, paths_per_wave, packets):
    """paths_per_wave 65536 splits the batch into several waves, which run in
    two concurrent chains; packets 1 traces depth 0 as warp packets
    (k_batch_primary_packet), 2 as packets with interval node tests."""
    import prt
    import scenes
    mesh0, view0 = small
    mesh1, view1 = scenes.batch_scene(1)
    ctxs, views = [], [view0, view1]
    for m in (mesh0, mesh1):
        c = prt.Context(0)
        c.load_mesh(m.indices, m.positions)
        c.build()
        ctxs.append(c)
    reqs_spec = [(0, 64, 64, 3, 4), (1, 128, 72, 1, 5), (0, 37, 23, 5, 2), (1, 256, 128, 2, 0), (0, 8, 8, 7, 6),
                 (1, 200, 96, 4, 3)]
    reqs = []
    for k, (si, w, h, spp, d) in enumerate(reqs_spec):
        acc = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda") if k % 2 == 0 else \
            np.zeros((h, w, 4), np.float32)
        reqs.append({"scene": ctxs[si], "camera": prt.camera_from_view(views[si], w, h), "width": w, "height": h,
                     "spp": spp, "maxDepth": d, "accum": acc})
    ctxs[0].set_tune(128, 0, paths_per_wave, 2, packets)
    st = ctxs[0].render_batch(reqs)
    st2 = ctxs[0].render_batch(reqs)     # replayed graph gives the same result
    total = 0
    for (si, w, h, spp, d), q in zip(reqs_spec, reqs):
        c = ctxs[si]
        c.init_frame(w, h)
        c.set_view(views[si], w, h)
        s = c.render(spp, d)
        total += s["ray"]
        ref = c.read_accum()
        got = q["accum"].cpu().numpy() if hasattr(q["accum"], "cpu") else q["accum"]
        assert np.all(got[..., 3] == spp)
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5)
    assert st["ray"] == total and st2["ray"] == total


def test_batch_rejects_bad_requests(small):
    import prt
    mesh, view = small
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    acc = np.zeros((8, 8, 4), np.float32)
    good = {"scene": c, "camera": prt.camera_from_view(view, 8, 8), "width": 8, "height": 8, "spp": 1,
            "maxDepth": 2, "accum": acc}
    bad = dict(good, width=0)
    with pytest.raises(prt.PrtError):
        c.render_batch([good, bad])
    assert c.render_batch([])["ray"] == 0

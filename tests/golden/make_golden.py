"""Generates tests/golden/reference_kats.npz from the reference's own CPU code.

Run in a container that has the ProtoRay sources at /root/reference:

    make -C oracle all && python tests/golden/make_golden.py

The vectors come from oracle/_ref/libprotoray_ref.so, i.e. the reference's
renderers, samplers, cameras, .mesh loader and shading code compiled from
their unmodified sources (oracle/Makefile); the closest-hit queries inside the
reference image come from the FP64 intersector that stands in for Embree.
The tests compare the FP64 C restatement (oracle/prt_oracle.c) and the CUDA
library against these fixtures.
"""

import hashlib
import math
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "embree-benchmark-protoray_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import scenes  # noqa: E402
import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.npz")


def mesh_digest(mesh) -> str:
    h = hashlib.sha256()
    h.update(mesh.positions.tobytes())
    h.update(mesh.indices.tobytes())
    return h.hexdigest()


def main():
    R = oracle.Reference()
    out = {}

    # RNG streams (sampling/random_sampler.h:44-63)
    pairs = np.array([[0, 0], [0, 1], [1, 0], [3, 17], [63, 2073599], [7, 123456], [1000, 65535]], np.int32)
    states, values = [], []
    for p, px in pairs:
        s, v = R.rng(int(p), int(px), 24)
        states.append(s)
        values.append(v)
    out["rng_pairs"] = pairs
    out["rng_states"] = np.array(states, np.uint32)
    out["rng_values"] = np.array(values, np.float32)

    # cameras (camera/pinhole_camera.h:34-47, camera/thin_lens_camera.h:29-36)
    views = [
        scenes.View((0.0, 14.0, 42.0), 0.38, 0.0, float(np.float32(math.radians(45.0))), 0.0, 40.0),
        scenes.View((1.5, -2.0, 30.0), -0.2, 0.7, float(np.float32(math.radians(60.0))), 0.0, 10.0),
        scenes.View((0.0, 16.0, 34.0), 0.52, -0.3, float(np.float32(math.radians(50.0))), 0.25, 35.0),
    ]
    sizes = [(256, 256), (1920, 1080), (640, 360)]
    out["cam_views"] = np.array([oracle.view_array(v) for v in views], np.float32)
    out["cam_sizes"] = np.array(sizes, np.int32)
    out["cam_fields"] = np.array([R.camera(v, w, h) for v, (w, h) in zip(views, sizes)], np.float32)

    # primary rays of RendererSingle::renderTile (render/renderer_single.h:107-124)
    prim = []
    for v in views:
        for p in (0, 5):
            prim.append(R.primary_rays(v, 32, 24, p))
    out["primary_rays"] = np.array(prim, np.float32)    # [view*2 + pass_index][32*24][8]

    # cosineSampleHemisphere and makeFrame
    rs = np.random.default_rng(11)
    cs_in = rs.uniform(0, 1, size=(64, 2)).astype(np.float32)
    cs_in[0] = [0.0, 0.0]
    cs_in[1] = [1.0, 0.5]
    out["cosine_in"] = cs_in
    out["cosine_out"] = np.array([R.cosine_sample(float(a), float(b)) for a, b in cs_in], np.float32)
    nrm = rs.normal(size=(64, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm[0] = [0, 0, 1]
    nrm[1] = [0, 1, 0]
    nrm[2] = [1, 0, 0]
    nrm = nrm.astype(np.float32)
    out["frame_in"] = nrm
    out["frame_out"] = np.array([R.make_frame(n) for n in nrm], np.float32)

    # scene-dependent vectors on the small scene
    mesh, view = scenes.small_scene()
    out["small_digest"] = np.frombuffer(mesh_digest(mesh).encode(), np.uint8)
    with tempfile.TemporaryDirectory() as d:
        path = scenes.write_scene(d, "small", mesh, view)
        rsc = R.open(path)
        pos, idx = rsc.arrays()
        assert np.array_equal(pos, mesh.positions) and np.array_equal(idx, mesh.indices)
        lo, hi = rsc.info()[2:]
        out["small_bounds"] = np.array([lo, hi], np.float32)

        # shading + bounce KATs on hits of primary rays
        rays = R.primary_rays(view, 32, 24, 0)
        hits = []
        for r in rays[::7]:
            q = rsc.query_ray(r[:3], r[4:7])
            if q is None:
                continue
            hits.append((r, q))
        shade_in, shade_out = [], []
        # barycentrics from the oracle's FP64 query (the reference queryRay
        # reports dist and primId; u, v only matter for normals/uvs)
        for k, (r, q) in enumerate(hits[:40]):
            sx, sy = rs.uniform(0, 1, size=2).astype(np.float32)
            shade_in.append([*r[:3], *r[4:7], q["dist"], q["primId"], 0.25, 0.25, sx, sy])
            shade_out.append(rsc.shade(r[:3], r[4:7], q["dist"], q["primId"], 0.25, 0.25, float(sx), float(sy)))
        out["shade_in"] = np.array(shade_in, np.float32)
        out["shade_out"] = np.array(shade_out, np.float32)
        out["query_in"] = np.array([r for r, _ in hits], np.float32)
        out["query_prim"] = np.array([q["primId"] for _, q in hits], np.int32)
        out["query_dist"] = np.array([q["dist"] for _, q in hits], np.float32)
        out["query_Ng"] = np.array([q["Ng"] for _, q in hits], np.float32)

        # reference image: diffuse renderer, 64x64, 4 frames, maxDepth 5
        sums, st = rsc.render("diffuse", view, 64, 64, 4, 5, accel=0)
        out["image_sums"] = sums.astype(np.float32)
        out["image_rays"] = np.array([st["rays"]], np.float64)
        out["image_cfg"] = np.array([64, 64, 4, 5], np.int32)
        # same with a thin-lens view
        tl = scenes.View(view.pos, view.angleX, view.angleY, view.fovY, 0.3, 38.0)
        sums_tl, st_tl = rsc.render("diffuse", tl, 64, 64, 2, 3, accel=0)
        out["image_tl_view"] = oracle.view_array(tl)
        out["image_tl_sums"] = sums_tl.astype(np.float32)
        out["image_tl_rays"] = np.array([st_tl["rays"]], np.float64)
        # next-event-estimation renderer (render/diffuse2_integrator_single.h)
        sums_d2, st_d2 = rsc.render("diffuse2", view, 64, 64, 4, 3, accel=0)
        out["image_d2_sums"] = sums_d2.astype(np.float32)
        out["image_d2_rays"] = np.array([st_d2["rays"]], np.float64)
        out["image_d2_cfg"] = np.array([64, 64, 4, 3], np.int32)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()

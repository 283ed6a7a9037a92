"""Structural checks of the 8-wide BVH built on the GPU: every triangle in
exactly one leaf, leaf triangles carry their own vertices, child boxes
enclose their contents, the tree depth fits the traversal stack."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _decode(nodes):
    """Per node: origin (3), scale (3), imask, child base, tri base, meta[8],
    qlo[3][8], qhi[3][8]."""
    q = nodes.view(np.uint32)
    origin = q[:, 0:3].view(np.float32)
    e = q[:, 3]
    scale = np.stack([np.ldexp(1.0, ((e >> (8 * k)) & 0xFF).astype(np.int64) - 127) for k in range(3)], axis=1)
    imask = (e >> 24) & 0xFF
    child = q[:, 4].astype(np.int64)
    tbase = q[:, 5].astype(np.int64)
    b = nodes.view(np.uint8).reshape(len(nodes), 80)
    meta = b[:, 24:32]
    qlo = np.stack([b[:, 32:40], b[:, 40:48], b[:, 48:56]], axis=1)
    qhi = np.stack([b[:, 56:64], b[:, 64:72], b[:, 72:80]], axis=1)
    return origin, scale, imask, child, tbase, meta, qlo, qhi


def _chain(n, ratio):
    """n nested triangles whose sizes shrink geometrically (ratio per step)
    around one point, so that SAH splits peel the largest off one by one."""
    s = ratio ** np.arange(n, dtype=np.float64)
    c = np.stack([0.1 * s, 0.05 * s, 0 * s], axis=1)
    shape = np.array([[-0.5, -0.3, 0.0], [0.5, -0.3, 0.1], [0.0, 0.6, -0.1]])
    pos = (c[:, None, :] + s[:, None, None] * shape[None]).reshape(-1, 3).astype(np.float32)
    return pos, np.arange(3 * n, dtype=np.int32).reshape(n, 3)


@pytest.mark.parametrize("scene,leaf,high", [("small", 1, 1), ("small", 3, 1), ("batch3", 1, 1), ("batch3", 2, 1),
                                             ("one", 1, 1), ("two", 1, 1), ("two", 3, 1), ("small", 1, 0),
                                             ("batch3", 2, 0), ("dup", 1, 1), ("dup", 1, 0), ("chain200", 1, 1),
                                             ("chain1000", 1, 1), ("chain1000", 2, 0)])
def test_bvh_structure(scene, leaf, high, small):
    import prt
    import scenes
    if scene == "dup":
        # 5000 copies of one triangle: every centroid in one bin, across
        # several 4096-triangle chunks (the split by position)
        pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
        idx = np.zeros((5000, 3), np.int32) + np.array([0, 1, 2], np.int32)
    elif scene.startswith("chain"):
        n = int(scene[5:])
        pos, idx = _chain(n, 0.8 if n <= 256 else 0.95)
    elif scene == "small":
        mesh, _ = small
        pos, idx = mesh.positions, mesh.indices
    elif scene == "batch3":
        mesh, _ = scenes.batch_scene(3)
        pos, idx = mesh.positions, mesh.indices
    elif scene == "one":
        pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
        idx = np.array([[0, 1, 2]], np.int32)
    else:
        pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
        idx = np.array([[0, 1, 2], [0, 1, 3]], np.int32)
    c = prt.Context(0)
    c.load_mesh(idx, pos)
    c.set_leaf_size(leaf)
    c.set_build_quality(bool(high))
    st = c.build()
    nodes, tris = c.read_accel()
    assert 2 * st["levels"] <= 64
    n = len(idx)
    prims = tris[:, 3].view(np.int32)
    assert np.array_equal(np.sort(prims), np.arange(n))
    # leaf triangles hold their own vertices
    np.testing.assert_array_equal(tris[:, 0:3], pos[idx[prims, 0]])
    np.testing.assert_array_equal(tris[:, 4:7], pos[idx[prims, 1]])
    np.testing.assert_array_equal(tris[:, 8:11], pos[idx[prims, 2]])

    origin, scale, imask, child, tbase, meta, qlo, qhi = _decode(nodes)
    seen_nodes = np.zeros(len(nodes), np.int64)
    seen_tris = np.zeros(n, np.int64)
    seen_nodes[0] += 1
    for i in range(len(nodes)):
        rank = 0
        for s in range(8):
            m = int(meta[i, s])
            if m == 0:
                continue
            lo = origin[i] + qlo[i, :, s] * scale[i]
            hi = origin[i] + qhi[i, :, s] * scale[i]
            eps = 1e-6 * (np.abs(lo) + np.abs(hi) + 1)
            if (m & 0x1F) >= 24:
                assert (m & 0x1F) - 24 == s and (imask[i] >> s) & 1
                ci = child[i] + rank
                rank += 1
                seen_nodes[ci] += 1
                # the child node's own planes lie inside the slot box, up to the
                # child's conservative rounding (origin one step below its box,
                # planes rounded outwards)
                used = meta[ci] != 0
                clo = origin[ci][:, None] + qlo[ci][:, used] * scale[ci][:, None]
                chi = origin[ci][:, None] + qhi[ci][:, used] * scale[ci][:, None]
                slack = eps + 2 * scale[ci]
                assert np.all(clo.min(axis=1) >= lo - slack) and np.all(chi.max(axis=1) <= hi + slack)
            else:
                cnt = bin(m >> 5).count("1")
                assert (m >> 5) == (1 << cnt) - 1 and 1 <= cnt <= leaf
                off = m & 0x1F
                for k in range(cnt):
                    t = tbase[i] + off + k
                    seen_tris[prims[t]] += 1
                    v = tris[t].reshape(3, 4)[:, :3]
                    assert np.all(v >= lo - eps) and np.all(v <= hi + eps)
        assert rank == bin(int(imask[i])).count("1")
    assert np.all(seen_nodes == 1)
    assert np.all(seen_tris == 1)


def test_build_quality_changes_grouping_not_hits(small):
    """The SAH grouping (high quality, default) makes fewer, fuller 8-wide
    nodes than the greedy one (low quality, `-no-sbvh`); closest hits and the
    image are the same for both."""
    import prt
    mesh, view = small
    W, H = 96, 96
    out = {}
    for high in (True, False):
        c = prt.Context(0)
        c.load_mesh(mesh.indices, mesh.positions)
        c.set_build_quality(high)
        st = c.build()
        c.init_frame(W, H)
        c.set_view(view, W, H)
        r = c.render(4, 5)
        out[high] = (st["nodeCount"], c.read_accum(), r["ray"])
        c.close()
    assert out[True][0] < 0.8 * out[False][0]
    a, b = out[True][1][..., 0], out[False][1][..., 0]
    assert float(np.mean(np.abs(a - b) / np.maximum(a, 1e-2))) < 1e-4
    assert abs(out[True][2] - out[False][2]) <= 1e-4 * out[True][2]
    c = prt.Context(0)
    with pytest.raises(prt.PrtError):
        c._check(c.L.prt_set_build_quality(c.h, 2), "prt_set_build_quality")
    c.close()



def test_rebuilds_reuse_scratch(small):
    """A context keeps its build scratch between builds: rebuilding other
    meshes of other sizes in one context gives the same trees (node count,
    levels) and images as fresh contexts."""
    import prt
    import scenes
    W, H = 64, 48
    big, bview = scenes.batch_scene(5)
    mesh, view = small

    def run(c, m, v):
        c.load_mesh(m.indices, m.positions)
        st = c.build()
        c.init_frame(W, H)
        c.set_view(v, W, H)
        c.render(2, 4, accumulate=False)
        return st["nodeCount"], st["levels"], c.read_accum().copy()

    fresh = {}
    for name, m, v in (("small", mesh, view), ("big", big, bview)):
        c = prt.Context(0)
        fresh[name] = run(c, m, v)
        c.close()
    c = prt.Context(0)
    for name, m, v in (("big", big, bview), ("small", mesh, view), ("big", big, bview), ("small", mesh, view)):
        nodes, levels, img = run(c, m, v)
        assert (nodes, levels) == fresh[name][:2], name
        ref = fresh[name][2]
        assert float(np.mean(np.abs(img[..., 0] - ref[..., 0]) / np.maximum(ref[..., 0], 1e-2))) < 1e-5, name
        assert np.array_equal(img[..., 3], ref[..., 3]), name
    c.close()

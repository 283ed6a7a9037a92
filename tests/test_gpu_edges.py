"""Edge cases through the C ABI: empty and one-triangle scenes, ragged frame
sizes (the reference CUDA path rejects H % 16 != 0,
render/diffuse_renderer_cuda.cu:161-162), zero spp, bad inputs, .mesh errors."""

import math
import struct

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _ctx(idx, pos):
    import prt
    c = prt.Context(0)
    c.load_mesh(np.asarray(idx, np.int32).reshape(-1, 3), np.asarray(pos, np.float32).reshape(-1, 3))
    c.build()
    return c


def _view():
    import scenes
    return scenes.View((0.0, 0.0, 5.0), 0.0, 0.0, math.radians(45.0), 0.0, 5.0)


def test_empty_scene_all_miss():
    c = _ctx(np.zeros((0, 3)), np.zeros((0, 3)))
    c.init_frame(16, 8)
    c.set_view(_view(), 16, 8)
    st = c.render(2, 5)
    img = c.read_accum()
    assert np.all(img[..., 0] == 2.0) and np.all(img[..., 3] == 2.0)
    assert st["ray"] == 16 * 8 * 2
    assert c.query_ray((0, 0, 0), (0, 0, -1)) is None


def test_single_triangle(oracle_mod):
    pos = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], np.float32)
    idx = np.array([[0, 1, 2]], np.int32)
    c = _ctx(idx, pos)
    q = c.query_ray((0.0, 0.0, 5.0), (0.0, 0.0, -1.0))
    assert q["primId"] == 0 and abs(q["dist"] - 5.0) < 1e-5
    np.testing.assert_allclose(q["Ng"], [0, 0, 1], atol=1e-6)
    assert c.query_ray((3.0, 0.0, 5.0), (0.0, 0.0, -1.0)) is None
    # render parity with the oracle
    O = oracle_mod.Oracle()
    s = O.scene(pos, idx)
    W, H = 24, 16
    c.init_frame(W, H)
    c.set_view(_view(), W, H)
    c.render(3, 2)
    img = c.read_accum()
    ref, _ = s.render(O.camera(_view(), W, H), W, H, 0, 3, 2)
    np.testing.assert_allclose(img[..., 0], ref[..., 0], atol=1e-5)


@pytest.mark.parametrize("size", [(37, 23), (1, 1), (8, 1080 // 8), (130, 9)])
def test_ragged_frames(small, small_oracle, oracle_mod, size):
    import prt
    mesh, view = small
    W, H = size
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.init_frame(W, H)
    c.set_view(view, W, H)
    c.render(2, 3)
    img = c.read_accum()
    assert np.all(img[..., 3] == 2)
    ref, _ = small_oracle.render(oracle_mod.Oracle().camera(view, W, H), W, H, 0, 2, 3)
    assert np.mean(np.abs(img[..., 0] - ref[..., 0]) / np.maximum(ref[..., 0], 1e-2)) < 2e-2


def test_zero_spp_and_depth(small):
    import prt
    mesh, view = small
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.init_frame(16, 16)
    c.set_view(view, 16, 16)
    st = c.render(0, 5)
    assert st["ray"] == 0
    assert np.all(c.read_accum() == 0)
    st = c.render(1, 0)     # primary rays only: escaped -> 1, hit -> 0
    assert st["ray"] == 256
    img = c.read_accum()
    assert set(np.unique(img[..., 0])).issubset({0.0, 1.0})


def test_errors_are_status_codes(tmp_path, small):
    import prt
    c = prt.Context(0)
    with pytest.raises(prt.PrtError) as e:
        c.render(1, 1)
    assert e.value.status == prt.PRT_ESTATE
    with pytest.raises(prt.PrtError) as e:
        c.load_mesh(np.array([[0, 1, 7]], np.int32), np.zeros((3, 3), np.float32))
    assert e.value.status == prt.PRT_EINVAL
    with pytest.raises(prt.PrtError) as e:
        c.load_mesh_file(str(tmp_path / "missing.mesh"))
    assert e.value.status == prt.PRT_EIO
    bad = tmp_path / "bad.mesh"
    bad.write_bytes(struct.pack("<i", 7) + b"\0" * 64)
    with pytest.raises(prt.PrtError) as e:
        c.load_mesh_file(str(bad))
    assert e.value.status == prt.PRT_EIO and "blob ID" in str(e.value)
    import scenes
    p = scenes.write_scene(str(tmp_path), "s", *small)
    data = open(p, "rb").read()
    tr = tmp_path / "trunc.mesh"
    tr.write_bytes(data[: len(data) - 100])
    with pytest.raises(prt.PrtError) as e:
        c.load_mesh_file(str(tr))
    assert e.value.status == prt.PRT_EIO
    c.load_mesh_file(p)
    c.build()
    with pytest.raises(prt.PrtError):
        c.init_frame(0, 10)
    c.init_frame(8, 8)
    with pytest.raises(prt.PrtError):
        c.render(1, 1)      # no camera yet
    c.set_view(small[1], 8, 8)
    with pytest.raises(prt.PrtError):
        c.render(-1, 1)
    with pytest.raises(prt.PrtError):
        c.render(1, 65)
    with pytest.raises(prt.PrtError):
        c.set_albedo(np.ones(3, np.float32))


def test_mesh_file_matches_arrays(small, small_path):
    import prt
    mesh, view = small
    a = prt.Context(0)
    a.load_mesh_file(small_path)
    a.build()
    lo, hi = a.scene_bounds()
    mlo, mhi = mesh.bounds()
    assert np.array_equal(lo, mlo) and np.array_equal(hi, mhi)
    b = prt.Context(0)
    b.load_mesh(mesh.indices, mesh.positions)
    b.build()
    for c in (a, b):
        c.init_frame(32, 32)
        c.set_view(view, 32, 32)
        c.render(2, 3)
    np.testing.assert_array_equal(a.read_accum(), b.read_accum())


def test_mesh_file_with_normals_and_uvs(tmp_path):
    """Interleaved position/normal/uv attributes (stride 8) are de-interleaved
    on the GPU (geometry/triangle_mesh.cpp:29-56)."""
    import prt
    rng = np.random.default_rng(1)
    nv, nt = 50, 40
    pos = rng.uniform(-1, 1, (nv, 3)).astype(np.float32)
    nrm = rng.normal(size=(nv, 3)).astype(np.float32)
    uv = rng.uniform(0, 1, (nv, 2)).astype(np.float32)
    idx = rng.integers(0, nv, (nt, 3)).astype(np.int32)
    attrs = np.concatenate([pos, nrm, uv], axis=1)
    path = tmp_path / "nuv.mesh"
    with open(path, "wb") as f:
        f.write(struct.pack("<i", 0x04DF8666))
        f.write(struct.pack("<6f", *pos.min(0), *pos.max(0)))
        f.write(struct.pack("<ii??", nt, nv, True, True))
        f.write(idx.tobytes())
        f.write(np.zeros(nt, np.int32).tobytes())
        f.write(attrs.tobytes())
        f.write(struct.pack("<i", 1) + struct.pack("<i", 3) + b"mat")
    c = prt.Context(0)
    lo, hi = c.load_mesh_file(str(path))
    np.testing.assert_array_equal(lo, pos.min(0))
    c.build()
    _, tris = c.read_accel()
    prims = tris[:, 3].view(np.int32)
    np.testing.assert_array_equal(tris[:, 0:3], pos[idx[prims, 0]])
    np.testing.assert_array_equal(tris[:, 8:11], pos[idx[prims, 2]])

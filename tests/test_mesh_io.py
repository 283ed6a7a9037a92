"""`.mesh` / `.view` formats (geometry/triangle_mesh.cpp:305-337, sys/blob.h,
main/render/view.h): the writer's output is read back by the reference's own
loader when it is built, and by the Python reader; corrupt files are rejected."""

import os
import struct

import numpy as np
import pytest


def test_round_trip_python(tmp_path, small):
    import scenes
    mesh, view = small
    p = scenes.write_scene(str(tmp_path), "s", mesh, view)
    m2 = scenes.read_mesh(p)
    assert np.array_equal(m2.positions, mesh.positions)
    assert np.array_equal(m2.indices, mesh.indices)
    assert m2.material_names == ["default"]
    v2 = scenes.read_view(str(tmp_path / "s.view"))
    assert np.allclose(v2.pos, view.pos) and np.float32(v2.angleX) == np.float32(view.angleX)
    assert os.path.getsize(tmp_path / "s.view") == 320


def test_round_trip_reference_loader(small_path, small, oracle_mod):
    if not oracle_mod.Reference.available():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    mesh, _ = small
    rs = oracle_mod.Reference().open(small_path)
    pos, idx = rs.arrays()
    assert np.array_equal(pos, mesh.positions)
    assert np.array_equal(idx, mesh.indices)
    t, v, lo, hi = rs.info()
    assert t == mesh.tri_count and v == mesh.vert_count
    mlo, mhi = mesh.bounds()
    assert np.array_equal(lo, mlo) and np.array_equal(hi, mhi)


def test_reader_rejects_corrupt_files(tmp_path, small):
    import scenes
    mesh, view = small
    p = scenes.write_scene(str(tmp_path), "s", mesh, view)
    data = open(p, "rb").read()
    bad_id = tmp_path / "bad_id.mesh"
    bad_id.write_bytes(struct.pack("<i", 1234) + data[4:])
    with pytest.raises(ValueError, match="blob ID"):
        scenes.read_mesh(str(bad_id))
    trunc = tmp_path / "trunc.mesh"
    trunc.write_bytes(data[: len(data) // 2])
    with pytest.raises(ValueError, match="end of stream"):
        scenes.read_mesh(str(trunc))


def test_scene_sizes():
    import scenes
    m, _ = scenes.small_scene()
    assert m.tri_count == 2 + 64 * 1280
    m, _ = scenes.terrain_scene()
    assert m.tri_count == 1024 * 512 * 2 + 256 * 1280
    for k in range(8):
        m, _ = scenes.batch_scene(k)
        assert 10_000 <= m.tri_count <= 2_100_000

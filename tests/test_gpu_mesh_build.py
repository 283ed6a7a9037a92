"""GPU mesh builder (prt_build_mesh) against the reference's TriangleMeshBuilder
(geometry/triangle_mesh_builder.cpp): the same triangles and the same unique
vertices, bit for bit, in Morton order instead of the reference's median-split
order.  Fixtures come from tests/golden/make_obj_golden.py; larger cases run
the compiled reference builder live when oracle/_ref is present."""

import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import obj_cases  # noqa: E402

pytestmark = pytest.mark.gpu
OBJ_GOLDEN = os.path.join(HERE, "golden", "obj_build.npz")


@pytest.fixture(scope="module")
def obj_golden():
    return dict(np.load(OBJ_GOLDEN))


@pytest.fixture(scope="module")
def ctx():
    import prt
    c = prt.Context(0)
    yield c
    c.close()


def _names(arr) -> list:
    return arr.tobytes().decode().split("\n")


def _canon(m: dict):
    """Sorted unique-vertex records and the sorted (vertex rank x3, material)
    rows of the triangles: equal for two meshes with the same content."""
    a = np.ascontiguousarray(m["attrs"])
    v = a.view(np.dtype((np.void, a.shape[1] * 4))).ravel() if len(a) else np.zeros(0, "V12")
    order = np.argsort(v, kind="stable")
    rank = np.empty(len(v), np.int64)
    rank[order] = np.arange(len(v))
    idx = m["indices"]
    rows = np.stack([rank[idx[:, 0]], rank[idx[:, 1]], rank[idx[:, 2]], m["material_ids"]], 1) if len(idx) else \
        np.zeros((0, 4), np.int64)
    rows = rows[np.lexsort(rows.T[::-1])] if len(rows) else rows
    return v[order], rows


def _morton30(p: np.ndarray, lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """The builder's 30-bit Morton code, in float32 as on the device."""
    p = p.astype(np.float32)
    ext = (hi - lo).astype(np.float32)
    code = np.zeros(len(p), np.uint64)
    for k in range(3):
        u = np.where(ext[k] > 0, (p[:, k] - lo[k]) / np.where(ext[k] > 0, ext[k], 1), np.float32(0)).astype(np.float32)
        q = np.minimum(np.maximum(u * np.float32(1024), 0), 1023).astype(np.uint64)
        b = np.zeros(len(p), np.uint64)
        for bit in range(10):
            b |= ((q >> bit) & 1) << (3 * bit)
        code |= b << k
    return code


def assert_same_mesh(mine: dict, ref: dict, what: str):
    for k in ("tri", "vert", "has_normals", "has_texcoords", "names"):
        assert mine[k] == ref[k], (what, k, mine[k], ref[k])
    assert np.array_equal(mine["lo"], ref["lo"]) and np.array_equal(mine["hi"], ref["hi"]), what
    mv, mt = _canon(mine)
    rv, rt = _canon(ref)
    assert len(np.unique(mv)) == len(mv), f"{what}: duplicate vertices"
    assert mv.tobytes() == rv.tobytes(), f"{what}: vertex sets differ"
    assert np.array_equal(mt, rt), f"{what}: triangles differ"


def assert_morton_order(m: dict, what: str):
    if m["vert"] == 0:
        return
    pos = m["attrs"][:, :3]
    vc = _morton30(pos, m["lo"], m["hi"])
    assert np.all(np.diff(vc.astype(np.int64)) >= 0), f"{what}: vertices not in Morton order"
    tri = pos[m["indices"]]
    third = np.float32(1.0) / np.float32(3.0)
    cen = ((tri[:, 0] + tri[:, 1]) + tri[:, 2]) * third
    tc = _morton30(cen.astype(np.float32), m["lo"], m["hi"])
    assert np.all(np.diff(tc.astype(np.int64)) >= 0), f"{what}: triangles not in Morton order"


def _build(ctx, tris, names, path):
    import scenes
    info = ctx.build_mesh(tris, names)
    ctx.save_built_mesh(path)
    return info, scenes.read_mesh_blob(path)


def test_builder_matches_reference_blobs(obj_golden, ctx, tmp_path):
    import scenes
    names = list(obj_golden["mesh_names"])
    assert len(names) >= 7
    for j, name in enumerate(names):
        tris = obj_golden[f"mesh_soup_{j}"]
        mtl = _names(obj_golden[f"mesh_mtl_{j}"])
        info, mine = _build(ctx, tris, mtl, str(tmp_path / f"{name}.mesh"))
        ref = scenes.read_mesh_blob(obj_golden[f"mesh_blob_{j}"].tobytes())
        assert_same_mesh(mine, ref, name)
        assert_morton_order(mine, name)
        assert info["triCount"] == ref["tri"] and info["vertCount"] == ref["vert"]
        assert mine["size"] == os.path.getsize(str(tmp_path / f"{name}.mesh"))


def test_built_mesh_arrays_match_blob(obj_golden, ctx, tmp_path):
    import scenes
    j = list(obj_golden["mesh_names"]).index("random_normals")
    info, blob = _build(ctx, obj_golden[f"mesh_soup_{j}"], _names(obj_golden[f"mesh_mtl_{j}"]),
                        str(tmp_path / "a.mesh"))
    m = ctx.read_built_mesh()
    assert info["hasNormals"] and not info["hasTexcoords"] and info["hasMaterials"]
    assert np.array_equal(m["indices"], blob["indices"])
    assert np.array_equal(m["materialIds"], blob["material_ids"])
    assert np.array_equal(m["positions"], blob["attrs"][:, :3])
    assert np.array_equal(m["normals"], blob["attrs"][:, 3:6])
    assert m["texcoords"] is None


def test_builder_is_deterministic(obj_golden, ctx, tmp_path):
    j = list(obj_golden["mesh_names"]).index("grid_tex_materials")
    t, n = obj_golden[f"mesh_soup_{j}"], _names(obj_golden[f"mesh_mtl_{j}"])
    blobs = []
    for k in range(3):
        p = str(tmp_path / f"d{k}.mesh")
        _build(ctx, t, n, p)
        blobs.append(open(p, "rb").read())
    assert blobs[0] == blobs[1] == blobs[2]


def test_obj_soups_build_like_reference(obj_golden, ctx, tmp_path):
    """OBJ fixtures through both builders (live reference)."""
    import oracle
    import scenes
    if not os.path.exists(oracle.REF_SO):
        pytest.skip("the reference build (oracle/_ref) is not present")
    R = oracle.Reference()
    for i, name in enumerate(obj_golden["obj_names"]):
        # non-finite coordinates: the two builders' bounds follow different
        # min/max conventions for inf and nan (the parser test covers that file)
        if not obj_golden["obj_ok"][i] or name == "nonfinite":
            continue
        tris = obj_golden[f"obj_soup_{i}"]
        mtl = _names(obj_golden[f"obj_mtl_{i}"])
        rp = str(tmp_path / f"{name}_ref.mesh")
        R.build_soup(tris, mtl, rp)
        _, mine = _build(ctx, tris, mtl, str(tmp_path / f"{name}.mesh"))
        assert_same_mesh(mine, scenes.read_mesh_blob(rp), name)


def test_large_soup_matches_live_reference(ctx, tmp_path):
    """The terrain workload's heightfield as a soup (1M triangles sharing
    vertices, plus random normals on a fraction of the corners)."""
    import oracle
    import scenes
    if not os.path.exists(oracle.REF_SO):
        pytest.skip("the reference build (oracle/_ref) is not present")
    mesh, _ = scenes.terrain_scene()
    tris = np.zeros(mesh.tri_count, oracle.SOUP_DTYPE)
    tris["v"]["pos"] = mesh.positions[mesh.indices]
    rng = np.random.default_rng(4)
    pick = rng.uniform(size=(mesh.tri_count, 3)) < 0.02
    tris["v"]["normal"] = np.where(pick[..., None], rng.standard_normal((mesh.tri_count, 3, 3)), 0).astype(np.float32)
    tris["matId"] = 1
    rp = str(tmp_path / "t_ref.mesh")
    ref_ms = oracle.Reference().build_soup(tris, ["", "Default"], rp)
    info, mine = _build(ctx, tris, ["", "Default"], str(tmp_path / "t.mesh"))
    ref = scenes.read_mesh_blob(rp)
    assert_same_mesh(mine, ref, "terrain")
    assert_morton_order(mine, "terrain")
    print(f"terrain soup {mesh.tri_count} tris: GPU build {info['buildMs']:.1f} ms "
          f"(total {info['totalMs']:.1f} ms), reference {ref_ms:.0f} ms")


def test_built_mesh_renders_like_the_source(ctx, small, tmp_path):
    """OBJ -> soup -> GPU build -> .mesh -> render equals rendering the source mesh."""
    import prt
    import scenes
    mesh, view = small
    lines = ["v %.9g %.9g %.9g" % tuple(float(x) for x in p) for p in mesh.positions]
    lines += [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in mesh.indices]
    obj = str(tmp_path / "small.obj")
    with open(obj, "w") as f:
        f.write("\n".join(lines) + "\n")
    tris, names, dropped = prt.load_obj(obj)
    assert dropped == 0 and len(tris) == mesh.tri_count
    ctx.build_mesh(tris, names)
    out = str(tmp_path / "small.mesh")
    ctx.save_built_mesh(out)
    W, H = 64, 64
    imgs = []
    for path in (None, out):
        c = prt.Context(0)
        if path is None:
            c.load_mesh(mesh.indices, mesh.positions)
        else:
            c.load_mesh_file(path)
        c.build()
        c.init_frame(W, H)
        c.set_view(view, W, H)
        st = c.render(4, 5)
        imgs.append((c.read_accum(), st["ray"]))
        c.close()
    a, b = imgs[0][0][..., 0], imgs[1][0][..., 0]
    assert float(np.mean(np.abs(a - b) / np.maximum(a, 1e-2))) < 1e-3
    assert abs(imgs[0][1] - imgs[1][1]) <= 1e-3 * imgs[0][1]


def test_builder_errors(ctx, tmp_path):
    import prt
    c = prt.Context(0)
    with pytest.raises(prt.PrtError) as e:
        c.save_built_mesh(str(tmp_path / "x.mesh"))
    assert e.value.status == prt.PRT_ESTATE
    L = prt.lib()
    assert L.prt_build_mesh(c.h, None, -1, None, 0, None) == prt.PRT_EINVAL
    assert L.prt_build_mesh(c.h, None, 3, None, 0, None) == prt.PRT_EINVAL
    c.close()


def test_builder_allocation_failures(obj_golden):
    """Every device allocation of the builder failing in turn gives PRT_ENOMEM
    and leaves the context usable.  A fresh context allocates the build scratch
    (kept for later builds) and then the output, so two failures are seen."""
    import prt
    j = list(obj_golden["mesh_names"]).index("random_normals")
    t, n = obj_golden[f"mesh_soup_{j}"], _names(obj_golden[f"mesh_mtl_{j}"])
    ctx = prt.Context(0)
    seen = 0
    for k in range(40):
        prt.fail_allocations(k)
        try:
            ctx.build_mesh(t, n)
            break
        except prt.PrtError as e:
            assert e.status == prt.PRT_ENOMEM
            seen += 1
        finally:
            prt.fail_allocations(-1)
    assert seen >= 2
    ctx.build_mesh(t, n)
    ctx.close()


def test_cli_build(obj_golden, tmp_path):
    """`protoray build x.obj -o x.mesh`, and the .mesh re-save path."""
    import scenes
    exe = os.path.join(os.path.dirname(HERE), "embree-benchmark-protoray_b200", "protoray")
    i = list(obj_golden["obj_names"]).index("grid")
    obj = str(tmp_path / "grid.obj")
    with open(obj, "wb") as f:
        f.write(obj_golden[f"obj_text_{i}"].tobytes())
    r = subprocess.run([exe, "build", obj, "-threads", "2"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    built = scenes.read_mesh_blob(str(tmp_path / "grid.mesh"))
    assert built["tri"] == len(obj_golden[f"obj_soup_{i}"])
    assert built["names"] == _names(obj_golden[f"obj_mtl_{i}"])
    r = subprocess.run([exe, "build", str(tmp_path / "grid.mesh"), "-o", str(tmp_path / "copy.mesh")],
                       cwd=str(tmp_path), capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert open(tmp_path / "copy.mesh", "rb").read() == open(tmp_path / "grid.mesh", "rb").read()
    bad = str(tmp_path / "bad.obj")
    with open(bad, "w") as f:
        f.write("v 1 2\n")
    r = subprocess.run([exe, "build", bad], cwd=str(tmp_path), capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and not os.path.exists(str(tmp_path / "bad.mesh"))


def test_soup_path_equals_triangle_path(obj_golden, ctx, tmp_path):
    """prt_build_mesh_soup (indexed upload, expansion on the GPU) writes the
    same .mesh as prt_build_mesh on the expanded soup, for every accepted
    OBJ fixture and a larger multi-chunk file."""
    import prt
    files = []
    for i, name in enumerate(obj_golden["obj_names"]):
        if obj_golden["obj_ok"][i]:
            p = str(tmp_path / f"{name}.obj")
            with open(p, "wb") as f:
                f.write(obj_golden[f"obj_text_{i}"].tobytes())
            files.append((name, p))
    p = str(tmp_path / "large.obj")
    with open(p, "w") as f:
        f.write(obj_cases.large_obj(seed=13))
    files.append(("large", p))
    for name, path in files:
        soup = prt.Soup(path, 4)
        a, b = str(tmp_path / f"{name}_soup.mesh"), str(tmp_path / f"{name}_tris.mesh")
        ctx.build_mesh_soup(soup)
        ctx.save_built_mesh(a)
        ctx.build_mesh(soup.triangles(), soup.names)
        ctx.save_built_mesh(b)
        soup.close()
        assert open(a, "rb").read() == open(b, "rb").read(), name


"""OBJ -> triangle soup (prt_soup_load_obj, host code of libprt_b200.so) against
the reference's ObjLoader (main/build/obj_loader.cpp): the committed fixtures of
tests/golden/make_obj_golden.py, and live runs of the compiled reference
loader on larger files when oracle/_ref is built."""

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import obj_cases  # noqa: E402

OBJ_GOLDEN = os.path.join(HERE, "golden", "obj_build.npz")


@pytest.fixture(scope="module")
def obj_golden():
    return dict(np.load(OBJ_GOLDEN))


@pytest.fixture(scope="module")
def prt_mod():
    import prt
    prt.lib()
    return prt


def _reference_or_skip():
    import oracle
    if not os.path.exists(oracle.REF_SO):
        pytest.skip("the reference build (oracle/_ref) is not present")
    return oracle.Reference()


def _write(tmp_path, name, data: bytes) -> str:
    p = os.path.join(str(tmp_path), name + ".obj")
    with open(p, "wb") as f:
        f.write(data)
    return p


@pytest.mark.parametrize("threads", [1, 4])
def test_obj_cases_match_reference_loader(obj_golden, prt_mod, tmp_path, threads):
    names = list(obj_golden["obj_names"])
    assert len(names) >= 20
    for i, name in enumerate(names):
        path = _write(tmp_path, name, obj_golden[f"obj_text_{i}"].tobytes())
        if obj_golden["obj_ok"][i]:
            tris, mtl, _ = prt_mod.load_obj(path, threads)
            ref = obj_golden[f"obj_soup_{i}"]
            assert tris.tobytes() == ref.tobytes(), name
            assert mtl == obj_golden[f"obj_mtl_{i}"].tobytes().decode().split("\n"), name
        else:
            with pytest.raises(prt_mod.PrtError) as e:
                prt_mod.load_obj(path, threads)
            assert e.value.status == prt_mod.PRT_EIO, name


def test_degenerate_triangles_are_counted(obj_golden, prt_mod, tmp_path):
    i = list(obj_golden["obj_names"]).index("degenerate")
    path = _write(tmp_path, "degenerate", obj_golden[f"obj_text_{i}"].tobytes())
    tris, _, dropped = prt_mod.load_obj(path)
    # f 1 1 2 | f 1 2 -4 (-4 is vertex 1) | fan 1 2 3 3 4 drops (1,3,3) | f 2 2 2 | f 1 1 99
    assert dropped == 5
    assert len(tris) == 3


def test_material_ids_follow_usemtl(obj_golden, prt_mod, tmp_path):
    names = list(obj_golden["obj_names"])
    path = _write(tmp_path, "m", obj_golden[f"obj_text_{names.index('materials_first')}"].tobytes())
    tris, mtl, _ = prt_mod.load_obj(path)
    assert mtl == ["", "red", "blue", "green"]          # no "Default": usemtl precedes every face
    assert tris["matId"].tolist() == [1, 2, 1, 2]
    path = _write(tmp_path, "d", obj_golden[f"obj_text_{names.index('default_then_materials')}"].tobytes())
    tris, mtl, _ = prt_mod.load_obj(path)
    assert mtl == ["", "Default", "x"]
    assert tris["matId"].tolist() == [1, 1, 2, 1]


def test_chunked_parse_is_identical(prt_mod, tmp_path):
    """Many chunks (relative indices and usemtl state crossing chunk
    boundaries) give the same soup as one chunk."""
    path = _write(tmp_path, "large", obj_cases.large_obj().encode())
    assert os.path.getsize(path) > 2_000_000
    one, n1, d1 = prt_mod.load_obj(path, 1)
    many, n2, d2 = prt_mod.load_obj(path, 8)
    assert len(one) > 50000
    assert one.tobytes() == many.tobytes() and n1 == n2 and d1 == d2


def test_large_obj_matches_live_reference(prt_mod, tmp_path):
    R = _reference_or_skip()
    path = _write(tmp_path, "large", obj_cases.large_obj(seed=12).encode())
    ref = R.load_obj(path)
    tris, names, _ = prt_mod.load_obj(path, 8)
    assert tris.tobytes() == ref[0].tobytes()
    assert names == ref[1]


def test_missing_file(prt_mod, tmp_path):
    with pytest.raises(prt_mod.PrtError) as e:
        prt_mod.load_obj(os.path.join(str(tmp_path), "nope.obj"))
    assert e.value.status == prt_mod.PRT_EIO

"""Generates tests/golden/obj_build.npz from the reference's own `protoray build`
code: ObjLoader (main/build/obj_loader.cpp) and TriangleMeshBuilder
(geometry/triangle_mesh_builder.cpp) compiled from their unmodified sources
into oracle/_ref/libprotoray_ref.so (oracle/Makefile).

Run in a container that has the ProtoRay sources at /root/reference:

    make -C oracle ref && python tests/golden/make_obj_golden.py

Contents:
  obj_names, obj_texts      OBJ test files (grammar cases and error cases)
  obj_ok                    1 where ObjLoader::load accepts the file
  obj_soup_<i>, obj_mtl_<i> its triangle soup (FatTriangle records) and
                            material names ('\\n'-joined)
  mesh_names                builder cases
  mesh_soup_<j>, mesh_mtl_<j>  the soup given to TriangleMeshBuilder
  mesh_blob_<j>             the .mesh blob the reference wrote for it
"""

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "embree-benchmark-protoray_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
import obj_cases  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "obj_build.npz")


def main():
    R = oracle.Reference()
    out = {}
    cases = obj_cases.obj_cases()
    out["obj_names"] = np.array([c[0] for c in cases])
    out["obj_texts"] = np.array([c[1].encode() for c in cases], dtype=object)
    ok = []
    with tempfile.TemporaryDirectory() as d:
        for i, (name, text) in enumerate(cases):
            path = os.path.join(d, name + ".obj")
            with open(path, "wb") as f:
                f.write(text.encode())
            r = R.load_obj(path)
            ok.append(r is not None)
            if r is not None:
                out[f"obj_soup_{i}"] = r[0]
                out[f"obj_mtl_{i}"] = np.frombuffer("\n".join(r[1]).encode(), np.uint8)
        out["obj_ok"] = np.array(ok, np.int32)

        soups = obj_cases.builder_soups()
        out["mesh_names"] = np.array([s[0] for s in soups])
        for j, (name, tris, names) in enumerate(soups):
            path = os.path.join(d, name + ".mesh")
            R.build_soup(tris, names, path)
            with open(path, "rb") as f:
                out[f"mesh_blob_{j}"] = np.frombuffer(f.read(), np.uint8)
            out[f"mesh_soup_{j}"] = tris
            out[f"mesh_mtl_{j}"] = np.frombuffer("\n".join(names).encode(), np.uint8)
    obj_texts = out.pop("obj_texts")
    for i, t in enumerate(obj_texts):
        out[f"obj_text_{i}"] = np.frombuffer(t, np.uint8)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(cases)} OBJ cases ({sum(ok)} accepted), {len(soups)} builder cases")


if __name__ == "__main__":
    main()

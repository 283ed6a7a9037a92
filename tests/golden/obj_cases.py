"""OBJ files and triangle soups for the `protoray build` parity tests.

Everything here is generated from fixed seeds, so tests/golden/make_obj_golden.py
and the live comparisons in tests/test_obj_build.py see the same inputs.
"""

from typing import List, Tuple

import numpy as np

SOUP_VERTEX_DTYPE = np.dtype([("pos", "<f4", 3), ("normal", "<f4", 3), ("tex", "<f4", 2)])
SOUP_DTYPE = np.dtype([("v", SOUP_VERTEX_DTYPE, 3), ("matId", "<i4")])


def _grid_obj(nx: int, nz: int, seed: int, forms: bool = True, materials: int = 3) -> str:
    """A height-field grid as OBJ text with normals, texcoords, mixed corner
    forms (p, p/t, p//n, p/t/n), negative indices, quads and triangles, and
    material switches."""
    rng = np.random.default_rng(seed)
    lines = ["# grid", "mtllib none.mtl", "o grid"]
    vid = 0
    for z in range(nz + 1):
        for x in range(nx + 1):
            h = float(np.float32(rng.uniform(-0.5, 0.5)))
            lines.append(f"v {x * 0.25:.6g} {h:.7g} {z * 0.25:.6g}")
            vid += 1
    for z in range(nz + 1):
        for x in range(nx + 1):
            lines.append(f"vt {x / nx:.6g} {z / nz:.6g}")
    for k in range(7):
        a = rng.standard_normal(3)
        a /= np.linalg.norm(a)
        lines.append(f"vn {a[0]:.6g} {a[1]:.6g} {a[2]:.6g}")
    nv = (nx + 1) * (nz + 1)
    for z in range(nz):
        if materials and z % 3 == 0:
            lines.append(f"usemtl m{(z // 3) % materials}")
        for x in range(nx):
            i0 = z * (nx + 1) + x + 1
            q = [i0, i0 + 1, i0 + nx + 2, i0 + nx + 1]
            form = (x + z) % 5 if forms else 0
            if form == 0:
                toks = [f"{p}" for p in q]
            elif form == 1:
                toks = [f"{p}/{p}" for p in q]
            elif form == 2:
                toks = [f"{p}//{1 + (p % 7)}" for p in q]
            elif form == 3:
                toks = [f"{p}/{p}/{1 + (p % 7)}" for p in q]
            else:
                toks = [f"{p - nv - 1}/{p - nv - 1}/-{1 + (p % 7)}" for p in q]   # relative
            if (x * 7 + z) % 4 == 0:
                lines.append("f " + " ".join(toks))
            else:
                lines.append("f " + " ".join([toks[0], toks[1], toks[2]]))
                lines.append("f " + " ".join([toks[0], toks[2], toks[3]]))
    return "\n".join(lines) + "\n"


def obj_cases() -> List[Tuple[str, str]]:
    c = []
    c.append(("fan", "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv -1 0.5 0\nf 1 2 3 4\nf 1 2 3 4 5\nf 5 4 1\n"))
    c.append(("forms",
              "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\n"
              "vt 0 0\nvt 1 0\nvt 1 1\n"
              "vn 0 0 1\nvn 0 0 -1\n"
              "f 1/1/1 2/2/1 3/3/1\n"
              "f 1//2 3//2 4//2\n"
              "f 1/1 2/2 4/3\n"
              "f -4/-3/-2 -3/-2/-1 -2/-1/-1\n"
              "f 1/2/3/4 2/3/1/9 3/1/2\n"            # extra fields after p/t/n are ignored
              "f 1// 2// 3//\n"                     # p only
              "f 1abc 2x 3y\n"))                    # trailing junk after the number
    c.append(("materials_first",
              "usemtl red\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3\nusemtl blue\nf 2 4 3\n"
              "usemtl red\nf 1 3 4\nusemtl green\nusemtl blue\nf 1 2 4\n"))
    c.append(("default_then_materials",
              "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3\nusemtl Default\nf 2 4 3\nusemtl x\nf 1 2 4\n"
              "usemtl Default\nf 1 3 4\n"))
    c.append(("material_without_faces", "usemtl lonely\nv 0 0 0\n"))
    c.append(("degenerate",
              "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\n"
              "f 1 1 2\nf 1 2 -4\nf 1 2 3 3 4\nf 2 2 2\nf 1 2 3\n"
              "f 1 1 99\n"))                        # dropped before its index is checked
    c.append(("whitespace",
              "# comment line\r\n\r\n  v\t0 0 0\r\nv 1e0 0 +0\r\nv 0 1.0e+0 0\r\n"
              "v 1-2-3\r\n\t\ng group\r\ns 1\r\nvp 1 2 3\r\n#v 9 9 9\r\n"
              "f 1 2 3   \r\nf\t4\t1\t2\r\n"))
    c.append(("forward_reference", "f 1 2 3\nf 3 2 4\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 1\n"))
    c.append(("empty", ""))
    c.append(("comments_only", "# nothing\n\n# more\n"))
    c.append(("numbers",                                  # decimal -> float edge cases
              "v 16777217 0.1 -0.0\nv 1e22 1e23 3.4028235e38\nv 1e-45 1.4e-45 1e-38\n"
              "v 123456789012345678901234 0.000000000000000000000001 9007199254740993\n"
              "v .5 5. +1.5e+3\nv 1E3 2e-0 0e9\nv 0x1p3 0X1.8P-2 -0x10\n"
              "v 0.12345678901234567890123 -7.0000005 33554431\n"
              "v 1.00000005960464477539062 3.4028235e38 -1.17549435e-38\n"
              "f 1 2 3\nf 4 5 6\nf 7 8 9\n"))
    c.append(("nonfinite", "v 0 0 0\nv inf 1 nan\nv 1 3.4028236e38 -INFINITY\nf 1 2 3\n"))
    c.append(("grid", _grid_obj(24, 20, seed=7)))
    c.append(("grid_plain", _grid_obj(40, 30, seed=8, forms=False, materials=0)))
    # files the reference rejects
    c.append(("bad_position", "v 1 2\nv 0 0 0\n"))
    c.append(("bad_texcoord", "vt 1\n"))
    c.append(("bad_normal", "vn 1 x 2\n"))
    c.append(("bad_face_token", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 a 2\n"))
    c.append(("two_corner_face", "v 0 0 0\nv 1 0 0\nf 1 2\n"))
    c.append(("empty_face", "v 0 0 0\nf\n"))
    c.append(("bad_usemtl", "usemtl\n"))
    c.append(("position_out_of_range", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n"))
    c.append(("normal_out_of_range", "v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2//2 3//1\n"))
    c.append(("texcoord_out_of_range", "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nf 1/1 2/1 3/-2\n"))
    return c


def large_obj(seed: int = 11) -> str:
    """A larger grid (about 2.6 MB of text) for the multi-chunk parser."""
    return _grid_obj(180, 160, seed=seed)


def _soup_from_indexed(pos: np.ndarray, idx: np.ndarray) -> np.ndarray:
    t = np.zeros(len(idx), SOUP_DTYPE)
    t["v"]["pos"] = pos[idx]
    return t


def builder_soups() -> List[Tuple[str, np.ndarray, List[str]]]:
    """(name, soup, material names) cases for TriangleMeshBuilder."""
    out = []
    rng = np.random.default_rng(21)
    # a shared-vertex grid as a soup: heavy de-duplication, no attributes
    nx, nz = 30, 20
    xs, zs = np.meshgrid(np.arange(nx + 1, dtype=np.float32), np.arange(nz + 1, dtype=np.float32))
    pos = np.stack([xs.ravel() * 0.5, rng.uniform(0, 1, xs.size).astype(np.float32), zs.ravel()], 1).astype(np.float32)
    q = []
    for z in range(nz):
        for x in range(nx):
            i0 = z * (nx + 1) + x
            q += [[i0, i0 + 1, i0 + nx + 2], [i0, i0 + nx + 2, i0 + nx + 1]]
    grid = _soup_from_indexed(pos, np.array(q))
    out.append(("grid_positions", grid, ["", "Default"]))
    # same grid with material ids, texcoords and some duplicated triangles
    g2 = grid.copy()
    g2["matId"] = 1 + (np.arange(len(g2)) % 3)
    g2["v"]["tex"] = g2["v"]["pos"][..., [0, 2]] / np.float32(16)
    g2 = np.concatenate([g2, g2[::7]])
    out.append(("grid_tex_materials", g2, ["", "a", "b", "c"]))
    # random triangles with some normals given: zero normals are replaced by
    # the triangle's cross product
    n = 3000
    t = np.zeros(n, SOUP_DTYPE)
    t["v"]["pos"] = rng.standard_normal((n, 3, 3)).astype(np.float32)
    given = rng.uniform(size=(n, 3)) < 0.4
    nrm = rng.standard_normal((n, 3, 3)).astype(np.float32)
    t["v"]["normal"] = np.where(given[..., None], nrm, np.float32(0))
    t["matId"] = rng.integers(0, 4, n)
    # share some corners between triangles so that merging matters
    t["v"]["pos"][1::2, 0] = t["v"]["pos"][0::2, 1]
    out.append(("random_normals", t, ["", "Default", "x", "y"]))
    # integer coordinates and axis-aligned triangles: fixed normals collide exactly
    m = 400
    base = rng.integers(-20, 20, (m, 3)).astype(np.float32)
    tri = np.zeros(m, SOUP_DTYPE)
    tri["v"]["pos"][:, 0] = base
    tri["v"]["pos"][:, 1] = base + np.float32([1, 0, 0])
    tri["v"]["pos"][:, 2] = base + np.float32([0, 1, 0])
    tri["v"]["normal"][::5, 0] = [0, 0, 1]
    out.append(("integer_fixup", np.concatenate([tri, tri[::3]]), ["", "Default"]))
    # texcoords only
    u = grid[:200].copy()
    u["v"]["tex"] = rng.uniform(0, 1, (200, 3, 2)).astype(np.float32)
    u["v"]["tex"][::4] = 0
    out.append(("texcoords_only", u, ["", "Default"]))
    # one triangle, and an empty soup
    out.append(("single", grid[:1].copy(), ["", "Default"]))
    out.append(("empty", np.zeros(0, SOUP_DTYPE), [""]))
    return out

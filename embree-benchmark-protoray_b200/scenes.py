"""Seeded synthetic scenes in ProtoRay's `.mesh` / `.view` formats.

The reference benchmarks on downloaded production scenes that are not part of
its tree (benchmark/scenes.txt:1-15); these generators stand in for them with
the shapes, sizes and value distributions of the five workloads this library is
measured on:

* ``small``      ground quad 40x40 (2 tris) + 64 level-3 icospheres
                 (1280 tris each), centres U[-10,10]^3, radius U[0.5,2]
* ``terrain``    1024x512-quad heightfield (1,048,576 tris; heights = sum of
                 4 seeded sine octaves, amplitude 2) + 256 level-3 icospheres
* ``spheres10m`` 2000 level-4 icospheres (5120 tris each), radius
                 log-uniform [0.1, 5], centres in a 200^3 box
* ``batch_scene(k)`` eight icosphere / heightfield scenes of 10K-2M tris

File formats follow the reference byte for byte:

* ``.mesh`` blob (sys/blob.h:26-50, geometry/triangle_mesh.cpp:305-337):
  int32 blobId 0x04df8666; Box3f bounds (low xyz, high xyz);
  int32 triCount; int32 vertCount; uint8 hasNormals; uint8 hasTexcoords;
  int32[3] indices[triCount]; int32 materialIds[triCount];
  float32 vertexAttribs[vertCount*stride] (stride 3: positions only);
  Array<std::string> materialNames = int32 count + (int32 len + bytes) each
  (sys/array.h:357-392, sys/string.cpp:30-45).
* ``.view`` file (main/render/view.h:25-40, main/render/view.cpp:23-46):
  10 x View{float pos[3], angleX, angleY, fovY, radius, focus} = 320 bytes.
"""

from __future__ import annotations

import math
import os
import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

MESH_BLOB_ID = 0x04DF8666


@dataclass
class View:
    """Camera view record (main/render/view.h:25-33)."""

    pos: Tuple[float, float, float]
    angleX: float = 0.0
    angleY: float = 0.0
    fovY: float = math.radians(45.0)
    radius: float = 0.0   # lens radius; 0 selects the pinhole camera
    focus: float = 1.0    # focal distance

    def pack(self) -> bytes:
        return struct.pack("<8f", *self.pos, self.angleX, self.angleY, self.fovY, self.radius, self.focus)

    @staticmethod
    def unpack(b: bytes) -> "View":
        v = struct.unpack("<8f", b)
        return View((v[0], v[1], v[2]), v[3], v[4], v[5], v[6], v[7])


@dataclass
class Mesh:
    """Triangle mesh as stored in a `.mesh` blob (positions only)."""

    positions: np.ndarray          # (V,3) float32
    indices: np.ndarray            # (T,3) int32
    material_ids: Optional[np.ndarray] = None   # (T,) int32
    material_names: List[str] = field(default_factory=lambda: ["default"])
    albedo: Optional[np.ndarray] = None         # (T,) float32, not stored in .mesh

    def __post_init__(self):
        self.positions = np.ascontiguousarray(self.positions, dtype=np.float32)
        self.indices = np.ascontiguousarray(self.indices, dtype=np.int32)
        if self.material_ids is None:
            self.material_ids = np.zeros(len(self.indices), dtype=np.int32)
        self.material_ids = np.ascontiguousarray(self.material_ids, dtype=np.int32)

    @property
    def tri_count(self) -> int:
        return int(self.indices.shape[0])

    @property
    def vert_count(self) -> int:
        return int(self.positions.shape[0])

    def bounds(self) -> Tuple[np.ndarray, np.ndarray]:
        if self.vert_count == 0:
            return np.zeros(3, np.float32), np.zeros(3, np.float32)
        return self.positions.min(axis=0), self.positions.max(axis=0)


# --------------------------------------------------------------------------
# .mesh / .view I/O
# --------------------------------------------------------------------------

def write_mesh(path: str, mesh: Mesh) -> None:
    lo, hi = mesh.bounds()
    with open(path, "wb") as f:
        f.write(struct.pack("<i", MESH_BLOB_ID))
        f.write(struct.pack("<6f", *lo.tolist(), *hi.tolist()))
        f.write(struct.pack("<ii??", mesh.tri_count, mesh.vert_count, False, False))
        f.write(mesh.indices.astype("<i4").tobytes())
        f.write(mesh.material_ids.astype("<i4").tobytes())
        f.write(mesh.positions.astype("<f4").tobytes())
        f.write(struct.pack("<i", len(mesh.material_names)))
        for name in mesh.material_names:
            b = name.encode()
            f.write(struct.pack("<i", len(b)))
            f.write(b)


def read_mesh(path: str) -> Mesh:
    """Reads a `.mesh` blob; raises ValueError on a wrong id or truncation."""
    with open(path, "rb") as f:
        data = f.read()

    off = 0

    def take(n: int) -> bytes:
        nonlocal off
        if off + n > len(data):
            raise ValueError(f"{path}: unexpected end of stream")
        b = data[off:off + n]
        off += n
        return b

    (blob_id,) = struct.unpack("<i", take(4))
    if blob_id != MESH_BLOB_ID:
        raise ValueError(f"{path}: file has wrong blob ID")
    take(24)  # bounds
    tri, vert, has_n, has_t = struct.unpack("<ii??", take(10))
    if tri < 0 or vert < 0:
        raise ValueError(f"{path}: negative element count")
    stride = 3 + (3 if has_n else 0) + (2 if has_t else 0)
    idx = np.frombuffer(take(12 * tri), dtype="<i4").reshape(tri, 3).copy()
    mat = np.frombuffer(take(4 * tri), dtype="<i4").copy()
    attrs = np.frombuffer(take(4 * vert * stride), dtype="<f4").reshape(vert, stride)
    (count,) = struct.unpack("<i", take(4))
    names = []
    for _ in range(count):
        (n,) = struct.unpack("<i", take(4))
        names.append(take(n).decode())
    return Mesh(attrs[:, :3].copy(), idx, mat, names)


def read_mesh_blob(data) -> dict:
    """Every field of a `.mesh` blob (geometry/triangle_mesh.cpp:305-320) from
    a path or bytes: bounds, counts, normal/texcoord flags, indices, material
    ids, the interleaved vertex attributes and the material names."""
    if isinstance(data, str):
        with open(data, "rb") as f:
            data = f.read()
    data = bytes(data)
    (blob_id,) = struct.unpack_from("<i", data, 0)
    if blob_id != MESH_BLOB_ID:
        raise ValueError("file has wrong blob ID")
    b = np.frombuffer(data, "<f4", 6, 4)
    tri, vert, has_n, has_t = struct.unpack_from("<ii??", data, 28)
    stride = 3 + (3 if has_n else 0) + (2 if has_t else 0)
    off = 38
    idx = np.frombuffer(data, "<i4", 3 * tri, off).reshape(tri, 3)
    off += 12 * tri
    mat = np.frombuffer(data, "<i4", tri, off)
    off += 4 * tri
    attrs = np.frombuffer(data, "<f4", vert * stride, off).reshape(vert, stride)
    off += 4 * vert * stride
    (count,) = struct.unpack_from("<i", data, off)
    off += 4
    names = []
    for _ in range(count):
        (n,) = struct.unpack_from("<i", data, off)
        names.append(data[off + 4:off + 4 + n].decode())
        off += 4 + n
    return {"lo": b[:3].copy(), "hi": b[3:].copy(), "tri": tri, "vert": vert, "has_normals": bool(has_n),
            "has_texcoords": bool(has_t), "indices": idx.copy(), "material_ids": mat.copy(), "attrs": attrs.copy(),
            "names": names, "size": off}


def write_view(path: str, view: View) -> None:
    with open(path, "wb") as f:
        for _ in range(10):
            f.write(view.pack())


def read_view(path: str, view_id: int = 0) -> View:
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < 32 * (view_id + 1):
        raise ValueError(f"{path}: truncated view set")
    return View.unpack(data[32 * view_id:32 * (view_id + 1)])


def default_view(mesh: Mesh) -> View:
    """Default view of the reference viewer (main/render/render_window.cpp:400-426)."""
    lo, hi = mesh.bounds()
    lo = lo.astype(np.float32)
    hi = hi.astype(np.float32)
    center = (lo + hi) * np.float32(0.5)
    size = hi - lo
    pos = np.array([center[0], center[1], np.float32(1.7) * size.max() + center[2]], dtype=np.float32)
    focus = float(np.linalg.norm((center - pos).astype(np.float32)))
    return View((float(pos[0]), float(pos[1]), float(pos[2])), 0.0, 0.0, float(np.float32(math.radians(45.0))), 0.0, focus)


# --------------------------------------------------------------------------
# Primitive generators
# --------------------------------------------------------------------------

_ICO_CACHE: Dict[int, Tuple[np.ndarray, np.ndarray]] = {}


def icosphere(level: int) -> Tuple[np.ndarray, np.ndarray]:
    """Unit icosphere by midpoint subdivision: level 3 = 642 verts / 1280 tris,
    level 4 = 2562 verts / 5120 tris."""
    if level in _ICO_CACHE:
        return _ICO_CACHE[level]
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
             (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [tuple(np.array(v) / np.linalg.norm(v)) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache: Dict[Tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = (np.array(verts[a]) + np.array(verts[b])) * 0.5
                verts.append(tuple(m / np.linalg.norm(m)))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    out = (np.array(verts, dtype=np.float64), np.array(faces, dtype=np.int32))
    _ICO_CACHE[level] = out
    return out


def sphere_instances(level: int, centers: np.ndarray, radii: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    uv, uf = icosphere(level)
    n = len(centers)
    pos = (centers[:, None, :] + radii[:, None, None] * uv[None, :, :]).reshape(-1, 3)
    idx = (uf[None, :, :] + (np.arange(n, dtype=np.int64) * len(uv))[:, None, None]).reshape(-1, 3)
    return pos.astype(np.float32), idx.astype(np.int32)


def ground_quad(size: float = 40.0, y: float = 0.0) -> Tuple[np.ndarray, np.ndarray]:
    h = size * 0.5
    pos = np.array([[-h, y, -h], [h, y, -h], [h, y, h], [-h, y, h]], dtype=np.float32)
    idx = np.array([[0, 2, 1], [0, 3, 2]], dtype=np.int32)
    return pos, idx


def heightfield(nx: int, nz: int, extent_x: float, extent_z: float, amplitude: float,
                rng: np.random.Generator, octaves: int = 4) -> Tuple[np.ndarray, np.ndarray]:
    """(nx x nz)-quad heightfield in the x/z plane; height = sum of `octaves`
    seeded sine octaves scaled so that the peak amplitude is `amplitude`."""
    xs = np.linspace(-extent_x / 2, extent_x / 2, nx + 1)
    zs = np.linspace(-extent_z / 2, extent_z / 2, nz + 1)
    X, Z = np.meshgrid(xs, zs)                      # (nz+1, nx+1)
    Hgt = np.zeros_like(X)
    norm = 0.0
    for k in range(octaves):
        f = 2.0 ** k
        ang = rng.uniform(0, 2 * math.pi)
        base = rng.uniform(0.15, 0.3)
        ph = rng.uniform(0, 2 * math.pi, size=2)
        w = 0.5 ** k
        u = math.cos(ang) * X + math.sin(ang) * Z
        v = -math.sin(ang) * X + math.cos(ang) * Z
        Hgt += w * np.sin(f * base * u + ph[0]) * np.cos(f * base * 0.7 * v + ph[1])
        norm += w
    Hgt *= amplitude / norm
    pos = np.stack([X, Hgt, Z], axis=-1).reshape(-1, 3).astype(np.float32)
    i = np.arange(nx)[None, :]
    j = np.arange(nz)[:, None]
    v00 = j * (nx + 1) + i
    v10 = v00 + 1
    v01 = v00 + (nx + 1)
    v11 = v01 + 1
    t0 = np.stack([v00, v01, v10], axis=-1)
    t1 = np.stack([v10, v01, v11], axis=-1)
    idx = np.stack([t0, t1], axis=2).reshape(-1, 3).astype(np.int32)
    return pos, idx


def _merge(parts: List[Tuple[np.ndarray, np.ndarray]]) -> Tuple[np.ndarray, np.ndarray]:
    pos_l, idx_l, off = [], [], 0
    for p, i in parts:
        pos_l.append(p)
        idx_l.append(i + off)
        off += len(p)
    return np.concatenate(pos_l).astype(np.float32), np.concatenate(idx_l).astype(np.int32)


# --------------------------------------------------------------------------
# Workload scenes
# --------------------------------------------------------------------------

def small_scene(seed: int = 0) -> Tuple[Mesh, View]:
    """Ground quad + 64 level-3 icospheres (~82K tris)."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-10, 10, size=(64, 3))
    radii = rng.uniform(0.5, 2.0, size=64)
    pos, idx = _merge([ground_quad(40.0, -10.0), sphere_instances(3, centers, radii)])
    mesh = Mesh(pos, idx)
    view = View((0.0, 14.0, 42.0), angleX=0.38, angleY=0.0, fovY=float(np.float32(math.radians(45.0))),
                radius=0.0, focus=40.0)
    return mesh, view


def terrain_scene(seed: int = 1) -> Tuple[Mesh, View]:
    """1024x512-quad heightfield + 256 level-3 icospheres (~1.38M tris)."""
    rng = np.random.default_rng(seed)
    hf = heightfield(1024, 512, 64.0, 32.0, 2.0, rng)
    n = 256
    centers = np.stack([rng.uniform(-30, 30, n), rng.uniform(2.5, 9.0, n), rng.uniform(-15, 15, n)], axis=-1)
    radii = rng.uniform(0.5, 2.0, n)
    pos, idx = _merge([hf, sphere_instances(3, centers, radii)])
    mesh = Mesh(pos, idx)
    view = View((0.0, 16.0, 34.0), angleX=0.52, angleY=0.0, fovY=float(np.float32(math.radians(50.0))),
                radius=0.0, focus=35.0)
    return mesh, view


def spheres10m_scene(seed: int = 2, count: int = 2000) -> Tuple[Mesh, View]:
    """2000 level-4 icospheres (~10.24M tris), log-uniform radius in [0.1,5]."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-100, 100, size=(count, 3))
    radii = np.exp(rng.uniform(math.log(0.1), math.log(5.0), size=count))
    pos, idx = sphere_instances(4, centers, radii)
    mesh = Mesh(pos, idx)
    return mesh, default_view(mesh)


def field_view(mesh: Mesh) -> View:
    """Camera on the front face of a scene's bounding box (x/y centre, z at
    the box's far side), looking down -z with a 45-degree vertical field of
    view: for the 10M-triangle icosphere field, about 47% of the primary rays
    hit (12% from the default view outside the box)."""
    lo = mesh.positions.min(axis=0)
    hi = mesh.positions.max(axis=0)
    c = 0.5 * (lo + hi)
    return View((float(c[0]), float(c[1]), float(hi[2])), angleX=0.0, angleY=0.0,
                fovY=float(np.float32(math.radians(45.0))), radius=0.0, focus=float(hi[2] - lo[2]))


def batch_scene(k: int, seed: int = 100) -> Tuple[Mesh, View]:
    """Eight seeded scenes of 10K-2M tris for the uneven-batch workload."""
    rng = np.random.default_rng(seed + k)
    # triangle budgets between 10K and 2M, spread log-uniformly over k=0..7
    target = int(round(10_000 * (200.0 ** (k / 7.0))))
    if k % 2 == 0:
        n = max(8, -(-target // 1280))
        ext = 8.0 + 4.0 * math.sqrt(n)
        centers = rng.uniform(-ext, ext, size=(n, 3))
        radii = rng.uniform(0.5, 2.0, n)
        pos, idx = _merge([ground_quad(4 * ext, -ext - 2.0), sphere_instances(3, centers, radii)])
        view = View((0.0, 0.35 * ext, 2.2 * ext), angleX=0.2, fovY=float(np.float32(math.radians(50.0))), focus=2 * ext)
    else:
        quads = max(1, target // 2)
        nz = max(1, int(math.sqrt(quads / 2)))
        nx = max(1, quads // nz)
        hf = heightfield(nx, nz, 64.0, 32.0, 2.0, rng)
        n = 32
        centers = np.stack([rng.uniform(-30, 30, n), rng.uniform(2.5, 9.0, n), rng.uniform(-15, 15, n)], axis=-1)
        pos, idx = _merge([hf, sphere_instances(2, centers, rng.uniform(0.5, 2.0, n))])
        view = View((0.0, 16.0, 34.0), angleX=0.52, fovY=float(np.float32(math.radians(50.0))), focus=35.0)
    return Mesh(pos, idx), view


def albedo_for(mesh: Mesh, seed: int = 3, lo: float = 0.2, hi: float = 0.8) -> np.ndarray:
    """Per-triangle diffuse albedo U[lo, hi] (float32)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=mesh.tri_count).astype(np.float32)


SCENES = {
    "small": small_scene,
    "terrain": terrain_scene,
    "spheres10m": spheres10m_scene,
}


def write_scene(directory: str, name: str, mesh: Mesh, view: View) -> str:
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, name + ".mesh")
    write_mesh(path, mesh)
    write_view(os.path.join(directory, name + ".view"), view)
    return path


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="write a synthetic scene as .mesh + .view")
    ap.add_argument("scene", choices=sorted(SCENES) + ["batch0", "batch1", "batch2", "batch3",
                                                      "batch4", "batch5", "batch6", "batch7"])
    ap.add_argument("--out", default=".")
    a = ap.parse_args()
    if a.scene.startswith("batch"):
        m, v = batch_scene(int(a.scene[5:]))
    else:
        m, v = SCENES[a.scene]()
    p = write_scene(a.out, a.scene, m, v)
    print(p, m.tri_count, "tris", m.vert_count, "verts")

"""ctypes bindings of the CPU checkers — TEST INFRASTRUCTURE ONLY.

* ``Oracle``    — oracle/liboracle.so, the FP64 C restatement (prt_oracle.c).
* ``Reference`` — oracle/_ref/libprotoray_ref.so, the reference's own CPU
  renderers compiled from its sources, with project intersectors standing in
  for Embree (ref_driver.cpp).

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libprotoray_ref.so")
REF_TREE = "/root/reference"


def build(with_ref: Optional[bool] = None) -> None:
    """Compiles the oracle (and the reference build when its sources exist)."""
    targets = ["oracle"]
    if with_ref is None:
        with_ref = os.path.isdir(REF_TREE)
    if with_ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, *targets], check=True)


# the reference's FatTriangle (geometry/triangle.h:54-57, geometry/vertex.h:23-28):
# three {pos, normal, tex} vertices and a material id, 100 bytes
SOUP_VERTEX_DTYPE = np.dtype([("pos", "<f4", 3), ("normal", "<f4", 3), ("tex", "<f4", 2)])
SOUP_DTYPE = np.dtype([("v", SOUP_VERTEX_DTYPE, 3), ("matId", "<i4")])
assert SOUP_DTYPE.itemsize == 100


def _f32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _f64p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class OrView(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("angleX", C.c_float), ("angleY", C.c_float),
                ("fovY", C.c_float), ("radius", C.c_float), ("focus", C.c_float)]


class OrCamera(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("U", C.c_float * 3), ("V", C.c_float * 3), ("N", C.c_float * 3),
                ("imageO", C.c_float * 3), ("imageDx", C.c_float * 3), ("imageDy", C.c_float * 3),
                ("lensRadius", C.c_float), ("focalDistance", C.c_float), ("thinLens", C.c_int)]

    def as_array(self) -> np.ndarray:
        v = [*self.origin, *self.U, *self.V, *self.N, *self.imageO, *self.imageDx, *self.imageDy,
             self.lensRadius, self.focalDistance]
        return np.array(v, dtype=np.float32)


class OrHit(C.Structure):
    _fields_ = [("t", C.c_double), ("primId", C.c_int), ("u", C.c_double), ("v", C.c_double), ("grazing", C.c_int)]


def view_array(view) -> np.ndarray:
    return np.array([*view.pos, view.angleX, view.angleY, view.fovY, view.radius, view.focus], dtype=np.float32)


class Oracle:
    """FP64 C restatement of the diffuse path."""

    _lib = None

    def __init__(self):
        if Oracle._lib is None:
            if not os.path.exists(ORACLE_SO):
                build(with_ref=False)
            lib = C.CDLL(ORACLE_SO)
            lib.or_rng_seed.restype = C.c_uint32
            lib.or_rng_seed.argtypes = [C.c_int, C.c_int]
            lib.or_lcg_next.restype = C.c_uint32
            lib.or_lcg_next.argtypes = [C.c_uint32]
            lib.or_unorm.restype = C.c_float
            lib.or_unorm.argtypes = [C.c_uint32]
            lib.or_camera_from_view.argtypes = [C.POINTER(OrView), C.c_float, C.POINTER(OrCamera)]
            lib.or_scene_create.restype = C.c_void_p
            lib.or_scene_create.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
            lib.or_scene_destroy.argtypes = [C.c_void_p]
            lib.or_intersect_rays.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
            lib.or_occluded_rays.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
            lib.or_primary_rays.argtypes = [C.POINTER(OrCamera), C.c_int, C.c_int, C.c_int, C.c_void_p]
            lib.or_render.restype = C.c_int64
            lib.or_render.argtypes = [C.c_void_p, C.POINTER(OrCamera), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_void_p, C.c_float, C.c_void_p, C.c_int]
            lib.or_render_ex.restype = C.c_int64
            lib.or_render_ex.argtypes = [C.c_void_p, C.POINTER(OrCamera), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_int]
            lib.or_render_pixels.restype = C.c_int64
            lib.or_render_pixels.argtypes = [C.c_void_p, C.POINTER(OrCamera), C.c_int, C.c_int, C.c_void_p, C.c_int,
                                             C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_float, C.c_void_p,
                                             C.c_void_p, C.c_int, C.c_int]
            lib.or_render_backward.argtypes = [C.c_void_p, C.POINTER(OrCamera), C.c_int, C.c_int, C.c_int, C.c_int,
                                               C.c_int, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_int]
            lib.or_cosine_sample_hemisphere.argtypes = [C.c_double, C.c_double, C.c_void_p]
            lib.or_make_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
            lib.or_post_intersect.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                              C.c_void_p, C.POINTER(C.c_double), C.c_void_p]
            Oracle._lib = lib
        self.lib = Oracle._lib

    # RNG
    def rng_seed(self, pass_: int, pixel: int) -> int:
        return int(self.lib.or_rng_seed(pass_, pixel))

    def lcg_next(self, s: int) -> int:
        return int(self.lib.or_lcg_next(s))

    def unorm(self, s: int) -> float:
        return float(self.lib.or_unorm(s))

    def camera(self, view, width: int, height: int) -> OrCamera:
        v = OrView((C.c_float * 3)(*view.pos), view.angleX, view.angleY, view.fovY, view.radius, view.focus)
        cam = OrCamera()
        self.lib.or_camera_from_view(C.byref(v), C.c_float(np.float32(width) / np.float32(height)), C.byref(cam))
        return cam

    def scene(self, positions: np.ndarray, indices: np.ndarray) -> "OracleScene":
        return OracleScene(self, positions, indices)

    def cosine_sample(self, sx: float, sy: float) -> np.ndarray:
        out = np.zeros(3, np.float64)
        self.lib.or_cosine_sample_hemisphere(sx, sy, out.ctypes.data)
        return out

    def make_frame(self, n: Sequence[float]) -> Tuple[np.ndarray, np.ndarray]:
        N = np.asarray(n, np.float64)
        U = np.zeros(3)
        V = np.zeros(3)
        self.lib.or_make_frame(N.ctypes.data, U.ctypes.data, V.ctypes.data)
        return U, V

    def primary_rays(self, cam: OrCamera, width: int, height: int, pass_: int) -> np.ndarray:
        out = np.zeros((width * height, 8), np.float32)
        self.lib.or_primary_rays(C.byref(cam), width, height, pass_, out.ctypes.data)
        return out


class OracleScene:
    def __init__(self, oracle: Oracle, positions: np.ndarray, indices: np.ndarray):
        self.o = oracle
        self.pos = np.ascontiguousarray(positions, np.float32)
        self.idx = np.ascontiguousarray(indices, np.int32)
        self.h = oracle.lib.or_scene_create(self.pos.ctypes.data, len(self.pos), self.idx.ctypes.data, len(self.idx))
        if not self.h:
            raise ValueError("invalid mesh")

    def __del__(self):
        if getattr(self, "h", None):
            self.o.lib.or_scene_destroy(self.h)
            self.h = None

    @property
    def tri_count(self) -> int:
        return len(self.idx)

    def intersect(self, rays: np.ndarray, nthreads: int = 0, flags: bool = False):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.zeros((len(rays), 4), np.float32)
        fl = np.zeros(len(rays), np.int32) if flags else None
        self.o.lib.or_intersect_rays(self.h, rays.ctypes.data, len(rays), hits.ctypes.data,
                                     fl.ctypes.data if flags else None, nthreads)
        return (hits, fl) if flags else hits

    def occluded(self, rays: np.ndarray, nthreads: int = 0) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.zeros(len(rays), np.float32)
        self.o.lib.or_occluded_rays(self.h, rays.ctypes.data, len(rays), out.ctypes.data, nthreads)
        return out

    def render(self, cam: OrCamera, width: int, height: int, pass0: int, npass: int, max_depth: int,
               albedo: Optional[np.ndarray] = None, sky: float = 1.0, nthreads: int = 0, nee: bool = False):
        """nee=True evaluates the diffuse2 (next-event estimation) integrator."""
        accum = np.zeros((height, width, 4), np.float64)
        alb = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
        rays = self.o.lib.or_render_ex(self.h, C.byref(cam), width, height, pass0, npass, max_depth,
                                       None if alb is None else alb.ctypes.data, C.c_float(sky), accum.ctypes.data,
                                       nthreads, int(nee))
        return accum, int(rays)

    def render_pixels(self, cam: OrCamera, width: int, height: int, pixels: np.ndarray, pass0: int, npass: int,
                      max_depth: int, albedo: Optional[np.ndarray] = None, sky: float = 1.0, nthreads: int = 0,
                      nee: bool = False):
        """render() at the listed pixels (x + y * width) of a width x height
        frame only: (values (n, 4), per-pixel ray counts (n,))."""
        px = np.ascontiguousarray(pixels, np.int32).ravel()
        out = np.zeros((len(px), 4), np.float64)
        rays = np.zeros(len(px), np.int64)
        alb = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
        r = self.o.lib.or_render_pixels(self.h, C.byref(cam), width, height, px.ctypes.data, len(px), pass0, npass,
                                        max_depth, None if alb is None else alb.ctypes.data, C.c_float(sky),
                                        out.ctypes.data, rays.ctypes.data, nthreads, int(nee))
        if r < 0:
            raise ValueError("pixel index outside the frame")
        return out, rays

    def render_backward(self, cam: OrCamera, width: int, height: int, pass0: int, npass: int, max_depth: int,
                        albedo: Optional[np.ndarray], sky: float, dL_dsum: np.ndarray, nthreads: int = 0):
        alb = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
        g = np.ascontiguousarray(dL_dsum, np.float64).reshape(height, width, 3)
        d_alb = np.zeros(self.tri_count, np.float64)
        d_sky = C.c_double(0.0)
        self.o.lib.or_render_backward(self.h, C.byref(cam), width, height, pass0, npass, max_depth,
                                      None if alb is None else alb.ctypes.data, C.c_float(sky), g.ctypes.data,
                                      d_alb.ctypes.data, C.byref(d_sky), nthreads)
        return d_alb, float(d_sky.value)

    def post_intersect(self, org, dir_, t: float, prim: int):
        o = np.asarray(org, np.float64)
        d = np.asarray(dir_, np.float64)
        p = np.zeros(3)
        ng = np.zeros(3)
        eps = C.c_double(0)
        self.o.lib.or_post_intersect(self.h, o.ctypes.data, d.ctypes.data, t, prim, p.ctypes.data, C.byref(eps),
                                     ng.ctypes.data)
        return p, eps.value, ng


class Reference:
    """The reference's own CPU renderers (compiled from its sources)."""

    _lib = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self):
        if Reference._lib is None:
            if not os.path.exists(REF_SO):
                raise FileNotFoundError(REF_SO)
            lib = C.CDLL(REF_SO)
            lib.ref_scene_open.restype = C.c_void_p
            lib.ref_scene_open.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
            lib.ref_scene_close.argtypes = [C.c_void_p]
            lib.ref_scene_info.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p, C.c_void_p]
            lib.ref_scene_arrays.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
            lib.ref_scene_build.restype = C.c_double
            lib.ref_scene_build.argtypes = [C.c_void_p, C.c_int]
            lib.ref_render.restype = C.c_int
            lib.ref_render.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]
            lib.ref_fast_trace.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
            lib.ref_query_ray.restype = C.c_int
            lib.ref_query_ray.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
            lib.ref_rng.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
            lib.ref_obj_load.restype = C.c_void_p
            lib.ref_obj_load.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p]
            lib.ref_soup_get.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p]
            lib.ref_soup_free.argtypes = [C.c_void_p]
            lib.ref_build_soup.restype = C.c_double
            lib.ref_build_soup.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.c_char_p]
            lib.ref_camera.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
            lib.ref_primary_rays.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
            lib.ref_cosine_sample.argtypes = [C.c_float, C.c_float, C.c_void_p]
            lib.ref_make_frame.argtypes = [C.c_void_p, C.c_void_p]
            lib.ref_shade.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_float, C.c_float, C.c_float,
                                      C.c_float, C.c_void_p]
            Reference._lib = lib
        self.lib = Reference._lib

    def open(self, path: str) -> "RefScene":
        return RefScene(self, path)

    def load_obj(self, path: str):
        """ObjLoader::load: (soup records as a SOUP_DTYPE array, material
        names), or None when the reference loader rejects the file."""
        n, names, nbytes = C.c_int(), C.c_int(), C.c_int()
        h = self.lib.ref_obj_load(path.encode(), C.byref(n), C.byref(names), C.byref(nbytes))
        if not h:
            return None
        try:
            tris = np.zeros(n.value, SOUP_DTYPE)
            buf = C.create_string_buffer(max(1, nbytes.value))
            self.lib.ref_soup_get(h, tris.ctypes.data, buf)
            text = buf.raw[:nbytes.value].decode()
            return tris, text.split("\n")[:names.value]
        finally:
            self.lib.ref_soup_free(h)

    def build_soup(self, tris: np.ndarray, names, mesh_path: str) -> float:
        """TriangleMeshBuilder + saveBlob; returns the builder's time in ms."""
        tris = np.ascontiguousarray(tris, SOUP_DTYPE)
        joined = "".join(s + "\n" for s in names).encode()
        ms = self.lib.ref_build_soup(tris.ctypes.data, len(tris), joined, len(names), mesh_path.encode())
        if ms < 0:
            raise RuntimeError("reference TriangleMeshBuilder failed")
        return ms

    def rng(self, pass_: int, pixel: int, n: int):
        st = np.zeros(n + 1, np.uint32)
        vals = np.zeros(n, np.float32)
        self.lib.ref_rng(pass_, pixel, n, st.ctypes.data, vals.ctypes.data)
        return st, vals

    def camera(self, view, width: int, height: int) -> np.ndarray:
        out = np.zeros(23, np.float32)
        self.lib.ref_camera(view_array(view).ctypes.data, width, height, out.ctypes.data)
        return out

    def primary_rays(self, view, width: int, height: int, pass_: int) -> np.ndarray:
        out = np.zeros((width * height, 8), np.float32)
        self.lib.ref_primary_rays(view_array(view).ctypes.data, width, height, pass_, out.ctypes.data)
        return out

    def cosine_sample(self, sx: float, sy: float) -> np.ndarray:
        out = np.zeros(3, np.float32)
        self.lib.ref_cosine_sample(sx, sy, out.ctypes.data)
        return out

    def make_frame(self, n) -> np.ndarray:
        N = np.asarray(n, np.float32)
        out = np.zeros(6, np.float32)
        self.lib.ref_make_frame(N.ctypes.data, out.ctypes.data)
        return out


class RefScene:
    def __init__(self, ref: Reference, path: str):
        self.r = ref
        err = C.create_string_buffer(512)
        self.h = ref.lib.ref_scene_open(path.encode(), err, 512)
        if not self.h:
            raise ValueError(err.value.decode())

    def __del__(self):
        if getattr(self, "h", None):
            self.r.lib.ref_scene_close(self.h)
            self.h = None

    def info(self):
        t = C.c_int()
        v = C.c_int()
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        self.r.lib.ref_scene_info(self.h, C.byref(t), C.byref(v), lo.ctypes.data, hi.ctypes.data)
        return t.value, v.value, lo, hi

    def arrays(self):
        t, v, _, _ = self.info()
        pos = np.zeros((v, 3), np.float32)
        idx = np.zeros((t, 3), np.int32)
        self.r.lib.ref_scene_arrays(self.h, pos.ctypes.data, idx.ctypes.data)
        return pos, idx

    def build(self, accel: int) -> float:
        """accel: 0 = FP64 oracle BVH, 1 = 8-wide AVX2 BVH with 4-triangle
        leaves (timing), 2 = scalar binary FP32 BVH (timing)."""
        return float(self.r.lib.ref_scene_build(self.h, accel))

    def fast_trace(self, rays: np.ndarray, accel: int = 1, any_hit: bool = False) -> np.ndarray:
        """Closest hits (n x 4: t or -1, primId bits, u, v) or occlusion flags
        (n) of n x 8 rays through a timing BVH (accel 1 or 2)."""
        r = np.ascontiguousarray(rays, np.float32)
        out = np.zeros(len(r) if any_hit else (len(r), 4), np.float32)
        self.r.lib.ref_fast_trace(self.h, accel, int(any_hit), r.ctypes.data, len(r), out.ctypes.data)
        return out

    def render(self, renderer: str, view, width: int, height: int, frames: int, max_depth: int, accel: int = 0,
               want_sums: bool = True):
        sums = np.zeros((height, width, 4), np.float32) if want_sums else None
        stats = np.zeros(3, np.float64)
        err = C.create_string_buffer(512)
        rc = self.r.lib.ref_render(self.h, renderer.encode(), accel, width, height, frames, max_depth,
                                   view_array(view).ctypes.data, None if sums is None else sums.ctypes.data,
                                   stats.ctypes.data, err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return sums, {"rays": stats[0], "seconds": stats[1], "mray": stats[2]}

    def query_ray(self, org, dir_, far=3.4028234663852886e38):
        ray = np.array([*org, *dir_, far], np.float32)
        out = np.zeros(8, np.float32)
        ok = self.r.lib.ref_query_ray(self.h, ray.ctypes.data, out.ctypes.data)
        if not ok:
            return None
        return {"primId": int(out[0]), "dist": float(out[1]), "p": out[2:5].copy(), "Ng": out[5:8].copy()}

    def shade(self, org, dir_, t, prim, u, v, sx, sy) -> np.ndarray:
        ray = np.array([*org, *dir_], np.float32)
        out = np.zeros(19, np.float32)
        self.r.lib.ref_shade(self.h, ray.ctypes.data, t, prim, u, v, sx, sy, out.ctypes.data)
        return out

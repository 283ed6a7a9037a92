"""ctypes binding of libprt_b200.so (the C ABI in include/prt_b200.h).

`Device` mirrors the reference's Device interface (render/device.h:29-54):
initScene / getSceneBounds / initRenderer / render / queryPixel / queryRay /
initCamera / initFrame / clearFrame / blitFrame, with the reference's
property names (`spp`, `maxDepth`, `type`, `imageSize`) and stats keys
(`mray`, `ray`, `buildMs`, `buildMprim`).  There is no CPU fallback: loading
fails loudly when the CUDA library is missing.
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# PRT_B200_LIB selects another build of the same library (e.g. a variant
# compiled with different launch bounds); the default is the in-tree build.
LIB_PATH = os.environ.get("PRT_B200_LIB", os.path.join(HERE, "libprt_b200.so"))

PRT_OK, PRT_EINVAL, PRT_ENOMEM, PRT_ECUDA, PRT_ETIMEOUT, PRT_EINTERNAL, PRT_EIO, PRT_ESTATE = range(8)
STATUS_NAMES = {0: "PRT_OK", 1: "PRT_EINVAL", 2: "PRT_ENOMEM", 3: "PRT_ECUDA", 4: "PRT_ETIMEOUT",
                5: "PRT_EINTERNAL", 6: "PRT_EIO", 7: "PRT_ESTATE"}

# exported symbols, in the order of include/prt_b200.h
EXPORTS = [
    "prt_create", "prt_destroy", "prt_last_error", "prt_get_info",
    "prt_load_mesh", "prt_load_mesh_file", "prt_get_scene_bounds", "prt_set_albedo", "prt_set_sky",
    "prt_set_integrator",
    "prt_build_accel", "prt_set_leaf_size", "prt_set_build_quality", "prt_camera_from_view", "prt_set_camera",
    "prt_init_frame", "prt_clear", "prt_read_accum", "prt_read_ldr",
    "prt_render", "prt_render_profile", "prt_set_pass", "prt_get_pass", "prt_query_ray",
    "prt_intersect", "prt_occluded", "prt_render_backward", "prt_render_replay",
    "prt_render_batch", "prt_read_accel", "prt_read_counters", "prt_debug_fail_allocations", "prt_autotune", "prt_set_tune", "prt_get_tune", "prt_render_noalloc", "prt_launch_count", "prt_primary_rays",
    "prt_soup_load_obj", "prt_soup_info", "prt_soup_triangles", "prt_soup_material_name", "prt_soup_free",
    "prt_build_mesh", "prt_build_mesh_soup", "prt_read_built_mesh", "prt_save_built_mesh",
]


class PrtError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class View(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("angleX", C.c_float), ("angleY", C.c_float), ("fovY", C.c_float),
                ("radius", C.c_float), ("focus", C.c_float)]


class Camera(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("basisU", C.c_float * 3), ("basisV", C.c_float * 3),
                ("imageO", C.c_float * 3), ("imageDx", C.c_float * 3), ("imageDy", C.c_float * 3),
                ("lensRadius", C.c_float), ("focalDistance", C.c_float)]


class Ray(C.Structure):
    _fields_ = [("org", C.c_float * 3), ("tnear", C.c_float), ("dir", C.c_float * 3), ("tfar", C.c_float)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("primId", C.c_int), ("u", C.c_float), ("v", C.c_float)]


class BuildStats(C.Structure):
    _fields_ = [("buildMs", C.c_double), ("buildMprim", C.c_double), ("nodeCount", C.c_int), ("levels", C.c_int)]


class RenderStats(C.Structure):
    _fields_ = [("rays", C.c_longlong), ("ms", C.c_double), ("mray", C.c_double), ("passes", C.c_int)]


class Request(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", Camera), ("width", C.c_int), ("height", C.c_int),
                ("spp", C.c_int), ("maxDepth", C.c_int), ("accum", C.c_void_p)]


class MeshInfo(C.Structure):
    _fields_ = [("triCount", C.c_int), ("vertCount", C.c_int), ("hasNormals", C.c_int), ("hasTexcoords", C.c_int),
                ("hasMaterials", C.c_int), ("boundsLo", C.c_float * 3), ("boundsHi", C.c_float * 3),
                ("buildMs", C.c_double), ("totalMs", C.c_double)]


# prt_soup_triangle: three {pos, normal, tex} vertices and a material id, 100 bytes
SOUP_VERTEX_DTYPE = np.dtype([("pos", "<f4", 3), ("normal", "<f4", 3), ("tex", "<f4", 2)])
SOUP_DTYPE = np.dtype([("v", SOUP_VERTEX_DTYPE, 3), ("matId", "<i4")])


class Tune(C.Structure):
    _fields_ = [("blockSize", C.c_int), ("blocksPerSM", C.c_int), ("pathsPerWave", C.c_int),
                ("concurrentWaves", C.c_int), ("primaryPackets", C.c_int), ("mray", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    """Loads libprt_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    vp, ip, fp = C.c_void_p, C.c_int, C.c_float
    sig = {
        "prt_create": (ip, [ip, C.POINTER(vp)]),
        "prt_destroy": (ip, [vp]),
        "prt_last_error": (C.c_char_p, [vp]),
        "prt_get_info": (ip, [vp, C.c_char_p, ip]),
        "prt_load_mesh": (ip, [vp, vp, ip, vp, ip]),
        "prt_load_mesh_file": (ip, [vp, C.c_char_p, vp, vp]),
        "prt_get_scene_bounds": (ip, [vp, vp, vp]),
        "prt_set_albedo": (ip, [vp, vp, ip]),
        "prt_set_sky": (ip, [vp, fp]),
        "prt_set_integrator": (ip, [vp, ip]),
        "prt_build_accel": (ip, [vp, C.POINTER(BuildStats)]),
        "prt_set_leaf_size": (ip, [vp, ip]),
        "prt_set_build_quality": (ip, [vp, ip]),
        "prt_camera_from_view": (ip, [C.POINTER(View), ip, ip, C.POINTER(Camera)]),
        "prt_set_camera": (ip, [vp, C.POINTER(Camera)]),
        "prt_init_frame": (ip, [vp, ip, ip]),
        "prt_clear": (ip, [vp]),
        "prt_read_accum": (ip, [vp, vp]),
        "prt_read_ldr": (ip, [vp, vp]),
        "prt_render": (ip, [vp, ip, ip, ip, C.POINTER(RenderStats)]),
        "prt_render_profile": (ip, [vp, ip, ip, vp, vp]),
        "prt_set_pass": (ip, [vp, ip]),
        "prt_get_pass": (ip, [vp, C.POINTER(C.c_int)]),
        "prt_query_ray": (ip, [vp, C.POINTER(Ray), C.POINTER(Hit), vp, vp]),
        "prt_intersect": (ip, [vp, vp, vp, ip, vp]),
        "prt_occluded": (ip, [vp, vp, vp, ip, vp]),
        "prt_render_backward": (ip, [vp, ip, ip, ip, vp, vp, vp]),
        "prt_render_replay": (ip, [vp, ip, ip, ip, C.POINTER(RenderStats)]),
        "prt_render_batch": (ip, [vp, C.POINTER(Request), ip, C.POINTER(RenderStats)]),
        "prt_read_accel": (ip, [vp, vp, ip, vp, ip, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "prt_read_counters": (ip, [vp, vp, ip, ip]),
        "prt_debug_fail_allocations": (ip, [C.c_longlong]),
        "prt_autotune": (ip, [vp, ip, ip, C.POINTER(Tune)]),
        "prt_set_tune": (ip, [vp, C.POINTER(Tune)]),
        "prt_get_tune": (ip, [vp, C.POINTER(Tune)]),
        "prt_render_noalloc": (ip, [vp, C.POINTER(Camera), ip, ip, ip, ip, ip, vp, C.POINTER(C.c_longlong)]),
        "prt_launch_count": (C.c_longlong, [vp]),
        "prt_primary_rays": (ip, [vp, ip, vp, vp]),
        "prt_soup_load_obj": (ip, [C.c_char_p, ip, C.POINTER(vp), C.c_char_p, ip]),
        "prt_soup_info": (ip, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "prt_soup_triangles": (vp, [vp]),
        "prt_soup_material_name": (C.c_char_p, [vp, ip]),
        "prt_soup_free": (None, [vp]),
        "prt_build_mesh": (ip, [vp, vp, ip, C.POINTER(C.c_char_p), ip, C.POINTER(MeshInfo)]),
        "prt_build_mesh_soup": (ip, [vp, vp, C.POINTER(MeshInfo)]),
        "prt_read_built_mesh": (ip, [vp, vp, vp, vp, vp, vp]),
        "prt_save_built_mesh": (ip, [vp, C.c_char_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _ptr(a) -> int:
    """Address of a numpy array or a torch tensor."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def fail_allocations(after: int) -> None:
    """Test hook: the (after+1)-th library allocation from now fails (-1: off)."""
    lib().prt_debug_fail_allocations(after)


class Soup:
    """A parsed OBJ (prt_soup_load_obj, ObjLoader::load in the reference)."""

    def __init__(self, path: str, threads: int = 0):
        self.L = lib()
        self.h = C.c_void_p()
        err = C.create_string_buffer(512)
        st = self.L.prt_soup_load_obj(path.encode(), threads, C.byref(self.h), err, 512)
        if st != PRT_OK:
            self.h = None
            raise PrtError(st, err.value.decode())
        n, m, d = C.c_int(), C.c_int(), C.c_int()
        self.L.prt_soup_info(self.h, C.byref(n), C.byref(m), C.byref(d))
        self.tri_count, self.degenerate = n.value, d.value
        self.names = [self.L.prt_soup_material_name(self.h, i).decode() for i in range(m.value)]

    def triangles(self) -> np.ndarray:
        """The expanded soup records as a SOUP_DTYPE array."""
        tris = np.zeros(self.tri_count, SOUP_DTYPE)
        if self.tri_count:
            p = self.L.prt_soup_triangles(self.h)
            if not p:
                raise PrtError(PRT_ENOMEM, "prt_soup_triangles")
            C.memmove(tris.ctypes.data, p, self.tri_count * SOUP_DTYPE.itemsize)
        return tris

    def close(self):
        if getattr(self, "h", None):
            self.L.prt_soup_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def load_obj(path: str, threads: int = 0):
    """OBJ -> triangle soup (ObjLoader::load, main/build/obj_loader.cpp:35-53).

    Returns (triangles as a SOUP_DTYPE array, material names, dropped
    degenerate triangles); raises PrtError on a malformed file."""
    s = Soup(path, threads)
    try:
        return s.triangles(), s.names, s.degenerate
    finally:
        s.close()


def camera_from_view(view, width: int, height: int) -> Camera:
    v = View((C.c_float * 3)(*view.pos), view.angleX, view.angleY, view.fovY, view.radius, view.focus)
    cam = Camera()
    st = lib().prt_camera_from_view(C.byref(v), width, height, C.byref(cam))
    if st != PRT_OK:
        raise PrtError(st, "prt_camera_from_view")
    return cam


class Context:
    """One prt_ctx: a scene, its acceleration structure, a camera and a frame."""

    def __init__(self, device: int = 0):
        self.L = lib()
        h = C.c_void_p()
        st = self.L.prt_create(device, C.byref(h))
        if st != PRT_OK:
            raise PrtError(st, f"prt_create(device={device})")
        self.h = h
        self.width = 0
        self.height = 0
        self.tri_count = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.prt_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, st: int, what: str):
        if st != PRT_OK:
            raise PrtError(st, f"{what}: {self.L.prt_last_error(self.h).decode()}")

    def info(self) -> str:
        buf = C.create_string_buffer(256)
        self._check(self.L.prt_get_info(self.h, buf, 256), "prt_get_info")
        return buf.value.decode()

    def load_mesh(self, indices: np.ndarray, positions: np.ndarray):
        idx = np.ascontiguousarray(indices, np.int32).reshape(-1, 3)
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        self._check(self.L.prt_load_mesh(self.h, idx.ctypes.data, len(idx), pos.ctypes.data, len(pos)), "prt_load_mesh")
        self.tri_count = len(idx)

    def load_mesh_file(self, path: str):
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        self._check(self.L.prt_load_mesh_file(self.h, path.encode(), lo.ctypes.data, hi.ctypes.data),
                    "prt_load_mesh_file")
        return lo, hi

    def scene_bounds(self):
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        self._check(self.L.prt_get_scene_bounds(self.h, lo.ctypes.data, hi.ctypes.data), "prt_get_scene_bounds")
        return lo, hi

    def set_albedo(self, albedo):
        if albedo is None:
            self._check(self.L.prt_set_albedo(self.h, None, 0), "prt_set_albedo")
            return
        n = int(albedo.numel() if hasattr(albedo, "numel") else len(albedo))
        if not hasattr(albedo, "data_ptr"):
            albedo = np.ascontiguousarray(albedo, np.float32)
        self._check(self.L.prt_set_albedo(self.h, _ptr(albedo), n), "prt_set_albedo")

    def set_integrator(self, name: str):
        """'diffuse' or 'diffuse2' (next-event estimation)."""
        kinds = {"diffuse": 0, "diffuse2": 1}
        if name not in kinds:
            raise ValueError("invalid renderer type")
        self._check(self.L.prt_set_integrator(self.h, kinds[name]), "prt_set_integrator")

    def set_sky(self, sky: float):
        self._check(self.L.prt_set_sky(self.h, sky), "prt_set_sky")

    def set_leaf_size(self, n: int):
        self._check(self.L.prt_set_leaf_size(self.h, n), "prt_set_leaf_size")

    def set_build_quality(self, high: bool):
        """True: full SAH tree with SAH grouping into 8-wide nodes (default);
        False: Morton LBVH with greedy grouping (faster to build)."""
        self._check(self.L.prt_set_build_quality(self.h, 1 if high else 0), "prt_set_build_quality")

    def build(self) -> Dict[str, float]:
        s = BuildStats()
        self._check(self.L.prt_build_accel(self.h, C.byref(s)), "prt_build_accel")
        return {"buildMs": s.buildMs, "buildMprim": s.buildMprim, "nodeCount": s.nodeCount, "levels": s.levels}

    def set_camera(self, cam: Camera):
        self._check(self.L.prt_set_camera(self.h, C.byref(cam)), "prt_set_camera")

    def set_view(self, view, width: int, height: int):
        self.set_camera(camera_from_view(view, width, height))

    def init_frame(self, width: int, height: int):
        self._check(self.L.prt_init_frame(self.h, width, height), "prt_init_frame")
        self.width, self.height = width, height

    def clear(self):
        self._check(self.L.prt_clear(self.h), "prt_clear")

    def render(self, spp: int, max_depth: int, accumulate: bool = True) -> Dict[str, float]:
        s = RenderStats()
        self._check(self.L.prt_render(self.h, spp, max_depth, int(accumulate), C.byref(s)), "prt_render")
        return {"ray": s.rays, "ms": s.ms, "mray": s.mray, "passes": s.passes}

    def render_profile(self, spp: int, max_depth: int):
        ms = np.zeros(max_depth + 1, np.float64)
        rays = np.zeros(max_depth + 1, np.int64)
        self._check(self.L.prt_render_profile(self.h, spp, max_depth, ms.ctypes.data, rays.ctypes.data),
                    "prt_render_profile")
        return ms, rays

    def render_replay(self, pass0: int, spp: int, max_depth: int) -> Dict[str, float]:
        s = RenderStats()
        self._check(self.L.prt_render_replay(self.h, pass0, spp, max_depth, C.byref(s)), "prt_render_replay")
        return {"ray": s.rays, "ms": s.ms, "mray": s.mray}

    def render_backward(self, pass0: int, spp: int, max_depth: int, dL_dsum, d_albedo, d_sky):
        self._check(self.L.prt_render_backward(self.h, pass0, spp, max_depth, _ptr(dL_dsum), _ptr(d_albedo),
                                               _ptr(d_sky)), "prt_render_backward")

    def set_pass(self, p: int):
        self._check(self.L.prt_set_pass(self.h, p), "prt_set_pass")

    def get_pass(self) -> int:
        v = C.c_int()
        self._check(self.L.prt_get_pass(self.h, C.byref(v)), "prt_get_pass")
        return v.value

    def read_accum(self, out=None) -> np.ndarray:
        if out is None:
            out = np.zeros((self.height, self.width, 4), np.float32)
        self._check(self.L.prt_read_accum(self.h, _ptr(out)), "prt_read_accum")
        return out

    def read_ldr(self) -> np.ndarray:
        out = np.zeros((self.height, self.width), np.uint32)
        self._check(self.L.prt_read_ldr(self.h, out.ctypes.data), "prt_read_ldr")
        return out

    def query_ray(self, org, dir_, tnear: float = 0.0, tfar: float = 3.4028234663852886e38):
        r = Ray((C.c_float * 3)(*org), tnear, (C.c_float * 3)(*dir_), tfar)
        h = Hit()
        p = np.zeros(3, np.float32)
        ng = np.zeros(3, np.float32)
        self._check(self.L.prt_query_ray(self.h, C.byref(r), C.byref(h), p.ctypes.data, ng.ctypes.data),
                    "prt_query_ray")
        if h.t < 0:
            return None
        return {"primId": h.primId, "dist": h.t, "u": h.u, "v": h.v, "p": p, "Ng": ng}

    def intersect(self, rays_dev, hits_dev, n: int, stream: int = 0):
        """rays_dev / hits_dev: device tensors of n x 8 / n x 4 float32."""
        self._check(self.L.prt_intersect(self.h, _ptr(rays_dev), _ptr(hits_dev), n, stream or None), "prt_intersect")

    def primary_rays(self, pass_: int, rays_dev, stream: int = 0):
        """rays_dev: device tensor of (H*W) x 8 float32, filled row-major with
        the camera rays of pass `pass_` (prt_primary_rays)."""
        self._check(self.L.prt_primary_rays(self.h, pass_, _ptr(rays_dev), stream or None), "prt_primary_rays")

    def occluded(self, rays_dev, out_dev, n: int, stream: int = 0):
        self._check(self.L.prt_occluded(self.h, _ptr(rays_dev), _ptr(out_dev), n, stream or None), "prt_occluded")

    def autotune(self, spp: int, max_depth: int) -> Dict[str, float]:
        t = Tune()
        self._check(self.L.prt_autotune(self.h, spp, max_depth, C.byref(t)), "prt_autotune")
        return {"blockSize": t.blockSize, "blocksPerSM": t.blocksPerSM, "pathsPerWave": t.pathsPerWave,
                "concurrentWaves": t.concurrentWaves, "primaryPackets": t.primaryPackets, "mray": t.mray}

    def get_tune(self) -> Dict[str, int]:
        t = Tune()
        self._check(self.L.prt_get_tune(self.h, C.byref(t)), "prt_get_tune")
        return {"blockSize": t.blockSize, "blocksPerSM": t.blocksPerSM, "pathsPerWave": t.pathsPerWave,
                "concurrentWaves": t.concurrentWaves, "primaryPackets": t.primaryPackets}

    def set_tune(self, block: int, per_sm: int, paths_per_wave: int, concurrent_waves: int = 0,
                 primary_packets: int = 0):
        t = Tune(block, per_sm, paths_per_wave, concurrent_waves, primary_packets, 0.0)
        self._check(self.L.prt_set_tune(self.h, C.byref(t)), "prt_set_tune")

    def render_noalloc(self, cam: Camera, width: int, height: int, pass0: int, spp: int, max_depth: int,
                       accum_dev) -> int:
        """Allocation-free render into a caller-owned device buffer (see
        prt_render_noalloc in include/prt_b200.h); returns the ray count."""
        rays = C.c_longlong(0)
        self._check(self.L.prt_render_noalloc(self.h, C.byref(cam), width, height, pass0, spp, max_depth,
                                              _ptr(accum_dev), C.byref(rays)), "prt_render_noalloc")
        return rays.value

    def read_accel(self):
        """(nodes uint32[N, 20], tris float32[T, 12]) of the built 8-wide BVH."""
        n, t = C.c_int(), C.c_int()
        self._check(self.L.prt_read_accel(self.h, None, 0, None, 0, C.byref(n), C.byref(t)), "prt_read_accel")
        nodes = np.zeros((max(n.value, 1), 20), np.uint32)
        tris = np.zeros((max(t.value, 1), 12), np.float32)
        self._check(self.L.prt_read_accel(self.h, nodes.ctypes.data, len(nodes), tris.ctypes.data, len(tris),
                                          C.byref(n), C.byref(t)), "prt_read_accel")
        return nodes[: n.value], tris[: t.value]

    def read_counters(self, reset: bool = True):
        """Traversal counters (builds with -DPRT_COUNTERS=1), see include/prt_b200.h."""
        out = np.zeros(6, np.int64)
        self._check(self.L.prt_read_counters(self.h, out.ctypes.data, 6, int(reset)), "prt_read_counters")
        keys = ["nodes", "tris", "rays", "steps", "lane_steps", "tri_iters"]
        return dict(zip(keys, out.tolist()))

    def launch_count(self) -> int:
        return int(self.L.prt_launch_count(self.h))

    def build_mesh(self, tris: np.ndarray, names: Sequence[str]) -> Dict[str, object]:
        """TriangleMeshBuilder on the GPU (prt_build_mesh); the mesh stays on
        the device until read_built_mesh / save_built_mesh."""
        tris = np.ascontiguousarray(tris, SOUP_DTYPE)
        arr = (C.c_char_p * max(1, len(names)))(*[s.encode() for s in names])
        info = MeshInfo()
        self._check(self.L.prt_build_mesh(self.h, tris.ctypes.data if len(tris) else None, len(tris), arr, len(names),
                                          C.byref(info)), "prt_build_mesh")
        self._mesh_info = info
        return {"triCount": info.triCount, "vertCount": info.vertCount, "hasNormals": bool(info.hasNormals),
                "hasTexcoords": bool(info.hasTexcoords), "hasMaterials": bool(info.hasMaterials),
                "boundsLo": np.array(info.boundsLo[:], np.float32), "boundsHi": np.array(info.boundsHi[:], np.float32),
                "buildMs": info.buildMs, "totalMs": info.totalMs}

    def build_mesh_soup(self, soup: "Soup") -> Dict[str, object]:
        """prt_build_mesh_soup: the GPU builder on a parsed OBJ's indexed form."""
        info = MeshInfo()
        self._check(self.L.prt_build_mesh_soup(self.h, soup.h, C.byref(info)), "prt_build_mesh_soup")
        self._mesh_info = info
        return {"triCount": info.triCount, "vertCount": info.vertCount, "hasNormals": bool(info.hasNormals),
                "hasTexcoords": bool(info.hasTexcoords), "hasMaterials": bool(info.hasMaterials),
                "boundsLo": np.array(info.boundsLo[:], np.float32), "boundsHi": np.array(info.boundsHi[:], np.float32),
                "buildMs": info.buildMs, "totalMs": info.totalMs}

    def read_built_mesh(self) -> Dict[str, np.ndarray]:
        info = self._mesh_info
        idx = np.zeros((info.triCount, 3), np.int32)
        mat = np.zeros(info.triCount, np.int32)
        pos = np.zeros((info.vertCount, 3), np.float32)
        nrm = np.zeros((info.vertCount, 3), np.float32) if info.hasNormals else None
        tex = np.zeros((info.vertCount, 2), np.float32) if info.hasTexcoords else None

        def p(a):
            return None if a is None or a.size == 0 else a.ctypes.data

        self._check(self.L.prt_read_built_mesh(self.h, p(idx), p(mat), p(pos), p(nrm), p(tex)), "prt_read_built_mesh")
        return {"indices": idx, "materialIds": mat, "positions": pos, "normals": nrm, "texcoords": tex}

    def save_built_mesh(self, path: str):
        self._check(self.L.prt_save_built_mesh(self.h, path.encode()), "prt_save_built_mesh")

    def render_batch(self, requests: Sequence[dict]) -> Dict[str, float]:
        """requests: dicts with scene (Context), camera (Camera), width, height,
        spp, maxDepth, accum (numpy (H,W,4) float32 or a device tensor)."""
        arr = (Request * max(1, len(requests)))()
        for i, q in enumerate(requests):
            arr[i].scene = q["scene"].h
            arr[i].camera = q["camera"]
            arr[i].width = q["width"]
            arr[i].height = q["height"]
            arr[i].spp = q["spp"]
            arr[i].maxDepth = q["maxDepth"]
            arr[i].accum = _ptr(q["accum"])
        s = RenderStats()
        self._check(self.L.prt_render_batch(self.h, arr, len(requests), C.byref(s)), "prt_render_batch")
        return {"ray": s.rays, "ms": s.ms, "mray": s.mray}


class Device:
    """Mirror of the reference Device interface (render/device.h:29-54) on one B200."""

    def __init__(self, device: int = 0):
        self.ctx = Context(device)
        self.props: Dict[str, object] = {}
        self.spp = 0
        self.max_depth = 6
        self.accumulate = True

    def getInfo(self) -> str:
        return self.ctx.info()

    def initScene(self, path: str, props: Optional[dict] = None):
        self.ctx.load_mesh_file(path)

    def getSceneBounds(self):
        return self.ctx.scene_bounds()

    def initRenderer(self, props: dict, stats: dict):
        """props: type (diffuse | diffuseFast | diffuse2 | diffuse2Fast),
        maxDepth (default 6, render/diffuse_integrator_single.h:35)."""
        rtype = props.get("type", "diffuse")
        if rtype not in ("diffuse", "diffuseFast", "diffuse2", "diffuse2Fast"):
            raise ValueError("invalid renderer type")
        self.accumulate = rtype in ("diffuse", "diffuse2")
        self.ctx.set_integrator("diffuse2" if rtype.startswith("diffuse2") else "diffuse")
        self.max_depth = int(props.get("maxDepth", 6))
        stats.update({k: v for k, v in self.ctx.build().items() if k in ("buildMs", "buildMprim")})

    def render(self, stats: dict, spp: int = 1):
        r = self.ctx.render(spp, self.max_depth, self.accumulate)
        stats.update({"mray": r["mray"], "ray": r["ray"], "spp": spp})

    def queryRay(self, org, dir_, far=3.4028234663852886e38):
        return self.ctx.query_ray(org, dir_, 0.0, far) or {}

    def initCamera(self, view):
        self.ctx.set_view(view, self.ctx.width, self.ctx.height)

    def initFrame(self, size):
        self.ctx.init_frame(int(size[0]), int(size[1]))

    def clearFrame(self):
        self.ctx.clear()

    def blitFrame(self) -> np.ndarray:
        return self.ctx.read_ldr()

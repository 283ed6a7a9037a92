"""Host-side checks of the C-ABI library that need no GPU: it loads, exports
every entry point declared in include/prt_b200.h, and reports errors as
status codes."""

import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "prt_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:const\s+)?(?:int|void|long long|char|prt_\w+)\s*\*?\s+(prt_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    import prt
    L = prt.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(prt.EXPORTS) == syms


def test_create_without_gpu_fails_cleanly():
    import prt
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    st = prt.lib().prt_create(0, C.byref(h))
    assert st in (prt.PRT_ECUDA, prt.PRT_EINVAL)
    assert not h.value


def test_camera_from_view_matches_oracle(golden, oracle_mod):
    """prt_camera_from_view is host code; it must reproduce the reference camera."""
    import prt
    import scenes
    for v, (w, h), ref in zip(golden["cam_views"], golden["cam_sizes"], golden["cam_fields"]):
        view = scenes.View(tuple(v[:3]), *v[3:])
        cam = prt.camera_from_view(view, int(w), int(h))
        got = np.array([*cam.origin, *cam.basisU, *cam.basisV, *cam.imageO, *cam.imageDx, *cam.imageDy], np.float32)
        exp = np.concatenate([ref[0:9], ref[12:21]])
        np.testing.assert_allclose(got, exp, atol=2e-6)
        assert cam.lensRadius == ref[21] and cam.focalDistance == ref[22]


def test_camera_from_view_rejects_bad_size():
    import prt
    v = prt.View((C.c_float * 3)(0, 0, 0), 0, 0, 0.7, 0, 1)
    cam = prt.Camera()
    assert prt.lib().prt_camera_from_view(C.byref(v), 0, 10, C.byref(cam)) == prt.PRT_EINVAL
    assert prt.lib().prt_camera_from_view(None, 10, 10, C.byref(cam)) == prt.PRT_EINVAL


def test_null_context_is_rejected():
    import prt
    L = prt.lib()
    assert L.prt_destroy(None) == prt.PRT_EINVAL
    assert L.prt_render(None, 1, 1, 1, None) == prt.PRT_EINVAL
    assert L.prt_build_accel(None, None) == prt.PRT_EINVAL
    assert L.prt_launch_count(None) == 0

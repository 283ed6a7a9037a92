"""Failure handling without faulting the GPU: an out-of-memory condition is
injected on the host (prt_debug_fail_allocations makes the n-th library
allocation fail) at every allocation of a load -> build -> frame -> render
sequence; each call either succeeds or reports PRT_ENOMEM, and the context
keeps working once allocations succeed again."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _pipeline(prt, mesh, view, ctx=None, steps=None):
    c = ctx or prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.init_frame(24, 16)
    c.set_view(view, 24, 16)
    c.render(2, 3)
    return c, c.read_accum().copy()


def test_injected_allocation_failures(small):
    import prt
    mesh, view = small
    _, ref = _pipeline(prt, mesh, view)
    failures = 0
    try:
        for k in range(0, 60):
            prt.fail_allocations(k)
            ctx = None
            try:
                ctx = prt.Context(0)
                _pipeline(prt, mesh, view, ctx)
                prt.fail_allocations(-1)
                break   # k exceeds the number of allocations of the sequence
            except prt.PrtError as e:
                assert e.status == prt.PRT_ENOMEM, str(e)
                failures += 1
            prt.fail_allocations(-1)
            if ctx is not None:
                _, img = _pipeline(prt, mesh, view, ctx)
                np.testing.assert_allclose(img, ref, rtol=1e-6, atol=1e-6)
                ctx.close()
    finally:
        prt.fail_allocations(-1)
    assert failures >= 10


def test_noalloc_entry_point_allocates_nothing(small):
    import prt
    mesh, view = small
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    cam = prt.camera_from_view(view, 32, 32)
    acc = torch.zeros((32, 32, 4), dtype=torch.float32, device="cuda")
    c.render_noalloc(cam, 32, 32, 0, 1, 3, acc)     # first call on the device: address set-up
    try:
        prt.fail_allocations(0)
        c.render_noalloc(cam, 32, 32, 1, 2, 3, acc)
    finally:
        prt.fail_allocations(-1)
    torch.cuda.synchronize()
    assert float(acc[..., 3].min()) == 3.0

"""The launch-configuration autotuner (prt_autotune) in the loop: it returns
a configuration inside its search ranges, the context keeps it, renders with
it keep image parity with the FP64 oracle and equal the default
configuration's image, and it is not slower than the default beyond noise."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_err(a, b):
    return float(np.mean(np.abs(a - b) / np.maximum(np.abs(b), 1e-2)))


def test_autotune_config_parity_and_speed(small, small_oracle, oracle_mod):
    import prt
    mesh, view = small
    W, H, spp, depth = 256, 256, 16, 5
    c = prt.Context(0)
    c.load_mesh(mesh.indices, mesh.positions)
    c.build()
    c.init_frame(W, H)
    c.set_view(view, W, H)
    default = c.get_tune()
    c.set_pass(0)
    c.render(spp, depth, accumulate=False)
    img_default = c.read_accum().copy()

    def speed(n=5):
        best = 0.0
        for _ in range(n):
            c.set_pass(0)
            best = max(best, c.render(spp, depth, accumulate=False)["mray"])
        return best

    m_default = speed()
    t = c.autotune(spp, depth)
    assert t["blockSize"] in (64, 128)
    assert t["blocksPerSM"] in (0, 4, 6)
    assert t["pathsPerWave"] == 0 or 65536 <= t["pathsPerWave"] <= 1 << 26
    assert 1 <= t["concurrentWaves"] <= 4
    assert t["primaryPackets"] in (0, 1, 2)
    assert t["mray"] > 0
    kept = c.get_tune()
    assert all(kept[k] == t[k] for k in kept), (kept, t)
    assert c.get_pass() == 0

    c.set_pass(0)
    c.render(spp, depth, accumulate=False)
    img = c.read_accum().copy()
    assert np.all(img[..., 3] == spp)
    O = oracle_mod.Oracle()
    ref, _ = small_oracle.render(O.camera(view, W, H), W, H, 0, spp, depth)
    assert _rel_err(img[..., 0], ref[..., 0]) < 1e-3
    # same paths, only the float summation order of the accumulation differs
    np.testing.assert_allclose(img, img_default, rtol=1e-5, atol=1e-5)

    m_tuned = speed()
    assert m_tuned >= 0.95 * m_default, (m_tuned, m_default, t, default)
    c.close()

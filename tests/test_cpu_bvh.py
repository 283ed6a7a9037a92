"""The CPU intersectors that stand in for Embree behind the reference's
renderers in the timed CPU baseline (oracle/cpu_bvh8.hpp: 8-wide AVX2 BVH with
4-triangle leaves; oracle/cpu_bvh32.hpp: scalar binary BVH): their closest
hits equal the FP64 oracle's outside the rays it flags as grazing, and their
occlusion answers agree with their closest hits.  CPU only; skipped when the
reference library (oracle/_ref) was not built."""

import numpy as np
import pytest


@pytest.fixture(scope="module")
def ref_scene(tmp_path_factory, small):
    import oracle
    import scenes
    if not oracle.Reference.available():
        pytest.skip("oracle/_ref/libprotoray_ref.so not built")
    mesh, view = small
    d = tmp_path_factory.mktemp("cpu_bvh")
    path = scenes.write_scene(str(d), "small", mesh, view)
    return oracle.Reference().open(path)


def _rays(mesh, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = mesh.positions.min(axis=0), mesh.positions.max(axis=0)
    org = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[::11] = np.array([0.0, -1.0, 0.0])        # axis-aligned directions (zero components)
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = org
    rays[:, 4:7] = d
    rays[:, 7] = 3.0e38
    rays[::3, 7] = 5.0                          # short segments exercise tfar
    return rays


@pytest.mark.parametrize("accel", [1, 2])
def test_fast_bvh_matches_oracle(accel, ref_scene, small, small_oracle, oracle_mod):
    mesh, view = small
    O = oracle_mod.Oracle()
    rays = np.concatenate([_rays(mesh, 20000, 11), O.primary_rays(O.camera(view, 128, 128), 128, 128, 0)])
    want, flags = small_oracle.intersect(rays, flags=True)
    got = ref_scene.fast_trace(rays, accel)
    rp = want[:, 1].view(np.int32)
    gp = got[:, 1].view(np.int32)
    assert ((rp != gp) & (flags == 0)).sum() == 0
    ok = (rp >= 0) & (rp == gp)
    np.testing.assert_allclose(got[ok, 0], want[ok, 0], rtol=1e-4, atol=1e-5)
    assert np.all(got[rp < 0, 0] < 0) or np.any(flags)
    occ = ref_scene.fast_trace(rays, accel, any_hit=True)
    assert np.array_equal(occ > 0, gp >= 0)
    assert (rp >= 0).mean() > 0.2

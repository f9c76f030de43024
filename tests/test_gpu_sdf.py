"""SDF build (makeSDF kernels.cu:282-300) vs the FP64 oracle.

Tolerance: |got - want| <= 1e-4 cell widths at every node whose winding
number is not within 1e-3 of the 0.5 threshold (there the sign itself is
ill-conditioned; such nodes are counted and must be rare)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _meshes():
    from mpm_b200 import scenes
    return {
        "sphere": ((32, 32, 32), scenes.uv_sphere(9.0, (16.2, 15.7, 16.1))),
        "torus": ((48, 32, 48), scenes.torus(12.0, 4.0, (24.3, 15.9, 23.8), 24, 12)),
        "box": ((32, 24, 40), scenes.box_mesh((10.5, 6.25, 14.0), (15.5, 12.1, 20.3))),
        "sphere_257tris": ((24, 24, 24), scenes.uv_sphere(7.0, (12.0, 12.0, 12.0), 17, 8)),
        # edges that are no multiple of the 8 x 8 x 4 node bricks, two shapes
        # in one list (1,200 triangles, five tiles of the sorted copy)
        "two_shapes_ragged": ((30, 21, 27), np.concatenate([
            scenes.torus(7.0, 2.5, (14.3, 10.2, 13.1), 24, 12), scenes.uv_sphere(3.5, (5.1, 5.2, 20.7), 24, 13)])),
    }


@pytest.mark.parametrize("name", ["sphere", "torus", "box", "sphere_257tris", "two_shapes_ragged"])
def test_sdf_matches_oracle(gpu_ok, mpm, oracle64, name):
    from mpm_b200 import scenes
    size, tris = _meshes()[name]
    cfg = scenes._cfg(size)
    with mpm.Engine(cfg) as eng:
        eng.init_sdf(tris)
        got = eng.get_sdf()
    want, wn = oracle64.make_sdf(cfg, tris.astype(np.float64))
    ok = np.abs(wn - 0.5) >= 1e-3
    assert ok.mean() > 0.999
    err = np.abs(got.astype(np.float64) - want)[ok]
    assert err.max() <= 1e-4, f"max SDF error {err.max():.3e} cells"
    assert (want < 0).any() and (want > 0).any()


def test_sdf_empty(gpu_ok, mpm):
    from mpm_b200 import scenes
    cfg = scenes._cfg((16, 16, 16))
    with mpm.Engine(cfg) as eng:
        assert np.all(eng.get_sdf() == np.sqrt(np.float32(1e30)))
        eng.init_sdf(np.zeros((0, 9), np.float32))
        assert np.all(eng.get_sdf() == np.sqrt(np.float32(1e30)))


def test_sdf_dam_break_torus(gpu_ok, mpm, oracle64):
    """The benchmark obstacle on its 128^3 grid, checked on a slab of nodes."""
    from mpm_b200 import scenes
    cfg, _, tris = scenes.dam_break()
    with mpm.Engine(cfg) as eng:
        eng.init_sdf(tris)
        got = eng.get_sdf().reshape(128, 128, 128)
    sub = scenes._cfg((128, 128, 4))
    # oracle on z = 62..65 only: shift the mesh so the slab starts at z = 0
    t = tris.astype(np.float64).reshape(-1, 3, 3).copy()
    t[:, :, 2] -= 62.0
    want, wn = oracle64.make_sdf(sub, t.reshape(-1, 9))
    want = want.reshape(4, 128, 128)
    ok = np.abs(wn.reshape(4, 128, 128) - 0.5) >= 1e-3
    err = np.abs(got[62:66].astype(np.float64) - want)[ok]
    assert err.max() <= 1e-4
    assert (want < 0).sum() > 100


def test_sdf_scale_scene_sampled(gpu_ok, mpm, oracle64):
    """The 256^3 scene with its three obstacles (3,276 triangles): the SDF at
    6,000 random nodes and 6,000 random nodes within 3 cells of a surface
    against the FP64 oracle at the same nodes."""
    from mpm_b200 import scenes
    cfg, st, tris = scenes.scale_scene(1236)
    with mpm.Engine(cfg) as eng:
        eng.init(st[:, :1000])
        eng.init_sdf(tris)
        sdf = eng.get_sdf()
    rng = np.random.default_rng(3)
    near = np.flatnonzero(np.abs(sdf) < 3.0)
    assert near.size > 6000
    idx = np.concatenate([rng.choice(sdf.size, 6000, replace=False), rng.choice(near, 6000, replace=False)])
    want, wn = oracle64.make_sdf_nodes(cfg, tris.astype(np.float64), idx)
    ok = np.abs(wn - 0.5) >= 1e-3
    assert ok.mean() > 0.999
    err = np.abs(sdf[idx].astype(np.float64) - want)[ok]
    assert err.max() <= 1e-4, f"max SDF error {err.max():.3e} cells"
    assert (want < 0).any()

"""Procedural workloads: particle counts, layout, closed outward meshes."""
import numpy as np


def test_dam_break_counts():
    from mpm_b200 import scenes
    cfg, st, tris = scenes.dam_break()
    assert st.shape == (26, 1_989_120)
    assert tris.shape == (48 * 24 * 2, 9)
    assert (cfg.size_x, cfg.size_y, cfg.size_z, cfg.padding, cfg.substeps) == (128, 128, 128, 3, 4)
    assert (np.float32(cfg.gravity), np.float32(cfg.dt), cfg.gamma, cfg.compression, cfg.resolution) == \
        (np.float32(-0.3), np.float32(0.1), 7.0, 10.0, 0.5)
    p = st[0:3]
    assert p[0].min() >= 4 and p[0].max() < 60 and p[1].min() >= 4 and p[1].max() < 41
    assert p[2].min() >= 4 and p[2].max() < 124
    # one particle per 0.5^3 sub-cell
    sub = np.floor(p * 2).astype(np.int64)
    ids = sub[0] + 1000 * sub[1] + 1000000 * sub[2]
    assert np.unique(ids).size == st.shape[1]


def test_literal_dam_break_count():
    from mpm_b200 import scenes
    n = 56 * 96 * 120 * 8
    assert n == 5_160_960
    lo, hi = np.array([4.0, 4.0, 4.0]), np.array([60.0, 100.0, 124.0])
    assert int(np.prod(np.floor((hi - lo) / 0.5))) == n


def test_sphere_drop_count():
    from mpm_b200 import scenes
    cfg, st, tris = scenes.sphere_drop()
    assert abs(st.shape[1] - 4 / 3 * np.pi * 15 ** 3 * 8) / st.shape[1] < 0.01
    assert tris.shape[0] == 0 and cfg.size_x == 64


def test_pack_layout():
    from mpm_b200 import scenes
    st = scenes.pack_state(np.arange(12, dtype=np.float32).reshape(4, 3))
    assert st.shape == (26, 4)
    assert np.array_equal(st[0], [0, 3, 6, 9]) and not st[3:24].any() and np.all(st[24:26] == 1)


def test_meshes_closed_and_outward(oracle64):
    from mpm_b200 import scenes
    cfg = scenes._cfg((32, 32, 32))
    for tris, inside, outside in [
        (scenes.uv_sphere(8.0, (16, 16, 16)), (16, 16, 16), (2, 2, 2)),
        (scenes.torus(9.0, 3.0, (16, 16, 16), 24, 12), (25, 16, 16), (16, 16, 16)),
        (scenes.box_mesh((10, 6, 8), (16, 16, 16)), (16, 16, 16), (16, 22, 16)),
    ]:
        sdf, wn = oracle64.make_sdf(cfg, tris)
        idx = lambda p: p[0] + 32 * p[1] + 1024 * p[2]
        assert sdf[idx(inside)] < 0 and abs(wn[idx(inside)] - 1) < 1e-3
        assert sdf[idx(outside)] > 0 and abs(wn[idx(outside)]) < 1e-3
    assert scenes.uv_sphere(15.0, (0, 0, 0)).shape[0] == 960


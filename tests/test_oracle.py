"""The CPU oracle: known answers and invariants (host only).  The pin of the
oracle against the reference's own outputs is tests/test_golden.py."""
import numpy as np
import pytest

from parity import morton_reference, stable_sort_reference


def test_morton_known_answers(oracle64):
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1], [2, 0, 0], [3, 5, 6], [1023, 1023, 1023],
                    [-4.0, 0.5, 2.9999]], np.float64).T
    st = np.zeros((26, pts.shape[1]))
    st[0:3] = pts
    keys = oracle64.morton_keys(st)
    # z:y:x interleave from the top: x -> bit 0, y -> bit 1, z -> bit 2
    assert list(keys[:6]) == [0, 1, 2, 4, 7, 8]
    x, y, z = 3, 5, 6
    want = 0
    for b in range(10):
        want |= ((x >> b) & 1) << (3 * b) | ((y >> b) & 1) << (3 * b + 1) | ((z >> b) & 1) << (3 * b + 2)
    assert keys[6] == want
    assert keys[7] == (1 << 30) - 1
    assert keys[8] == 32  # (0, 0, 2): z bit 1 lands on bit 3*1+2
    assert np.array_equal(keys, morton_reference(pts.astype(np.float32)))


def test_morton_aliasing_and_specials(oracle64):
    vals = np.array([1024.0, 2047.9, 4096.0, 3.0e9, np.inf, np.nan, -np.inf, 2.0 ** 32], np.float64)
    st = np.zeros((26, vals.size * 3))
    st[0, : vals.size] = vals
    st[1, vals.size: 2 * vals.size] = vals
    st[2, 2 * vals.size:] = vals
    keys = oracle64.morton_keys(st)
    assert np.array_equal(keys, morton_reference(st[0:3].astype(np.float32)))
    assert (keys < 0).any()  # y-spread of a large coordinate sets the sign bit


def test_sort_is_stable(oracle64):
    rng = np.random.default_rng(3)
    keys = rng.integers(-5, 40, 100_000).astype(np.int32)
    assert np.array_equal(oracle64.sort_perm(keys), stable_sort_reference(keys))


def _scene(oracle, n=4000, seed=2, **kw):
    from mpm_b200 import scenes
    cfg, st, tris = scenes.small_scene(n, (32, 32, 32), seed=seed, **kw)
    st = oracle.init_particles(cfg, st)
    return cfg, st, tris


def test_init_rules(oracle64):
    cfg, st, _ = _scene(oracle64)
    assert np.all(st[15] == 1) and np.all(st[19] == 1) and np.all(st[23] == 1)
    assert np.all(st[24] == np.float32(0.5) ** 3) and np.all(st[25] == 1)


def test_mass_and_momentum_conservation(oracle64):
    """Free flight away from walls: grid mass = particle mass, and the
    substep's momentum change is exactly the gravity impulse."""
    from mpm_b200 import scenes
    cfg = scenes._cfg((40, 40, 40))
    rng = np.random.default_rng(5)
    pos = 12 + rng.random((3, 3000)) * 16
    st = np.zeros((26, 3000))
    st[0:3] = pos
    st[3:6] = rng.normal(0, 0.1, (3, 3000))
    st[6:15] = rng.normal(0, 0.05, (9, 3000))
    st = oracle64.init_particles(cfg, st)
    sdf = oracle64.empty_sdf(cfg)
    s1, grid, keys, perm = oracle64.substep(cfg, st, sdf)
    assert abs(grid[0].sum() - 3000) < 1e-9
    p0 = (st[25] * st[3:6]).sum(1)
    p1 = (s1[25] * s1[3:6]).sum(1)
    # the engine stores GRAVITY and DT as float (SimConfig)
    g = np.array([0, -float(np.float32(cfg.gravity)) * float(np.float32(cfg.dt)) * 3000, 0])
    assert np.abs(p1 - p0 - g).max() < 1e-9


def test_fp32_restatement_tracks_fp64(oracle64, oracle32):
    cfg, st, tris = _scene(oracle64)
    sdf, _ = oracle64.make_sdf(cfg, tris)
    want = oracle64.substep(cfg, st, sdf)[0]
    got = oracle32.substep(cfg, st.astype(np.float32), sdf.astype(np.float32))[0]
    from parity import assert_state_close
    assert_state_close(got, want, st)


def test_tile_drop_is_tiny(oracle64):
    cfg, st, tris = _scene(oracle64)
    sdf, _ = oracle64.make_sdf(cfg, tris)
    keys = oracle64.morton_keys(st)
    perm = oracle64.sort_perm(keys)
    g1 = oracle64.p2g(cfg, st, perm, 1)
    g0 = oracle64.p2g(cfg, st, perm, 0)
    assert np.abs(g1 - g0).max() < 1e-8


def test_sdf_of_sphere(oracle64):
    from mpm_b200 import scenes
    cfg = scenes._cfg((24, 24, 24))
    c = np.array([12.0, 12.0, 12.0])
    tris = scenes.uv_sphere(7.0, c, 32, 16)
    sdf, wn = oracle64.make_sdf(cfg, tris)
    g = np.stack(np.meshgrid(np.arange(24), np.arange(24), np.arange(24), indexing="ij")[::-1], 0).reshape(3, -1)
    r = np.linalg.norm(g.T - c, axis=1)
    assert np.all(np.sign(sdf[r < 6.5]) == -1) and np.all(np.sign(sdf[r > 7.5]) == 1)
    # the polyhedron lies within 0.1 cells of the analytic sphere
    far = np.abs(r - 7) > 1
    assert np.abs(np.abs(sdf[far]) - np.abs(r[far] - 7)).max() < 0.15
    assert np.all(np.abs(wn[r < 6] - 1.0) < 1e-3) and np.all(np.abs(wn[r > 8]) < 1e-3)


def test_g2p_is_order_independent(oracle64):
    cfg, st, tris = _scene(oracle64)
    sdf, _ = oracle64.make_sdf(cfg, tris)
    keys = oracle64.morton_keys(st)
    perm = oracle64.sort_perm(keys)
    grid = oracle64.grid_update(cfg, oracle64.p2g(cfg, st, perm, 0), sdf)
    a = oracle64.g2p(cfg, st, perm, grid, sdf)
    b = oracle64.g2p(cfg, st, None, grid, sdf)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("threads", [1, 3])
def test_thread_count_invariance(oracle64, threads):
    cfg, st, tris = _scene(oracle64, n=3000)
    sdf, _ = oracle64.make_sdf(cfg, tris)
    old = oracle64.threads()
    oracle64.set_threads(1)
    a = oracle64.substep(cfg, st, sdf)
    oracle64.set_threads(threads)
    b = oracle64.substep(cfg, st, sdf)
    oracle64.set_threads(old)
    assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
    assert np.abs(a[0] - b[0]).max() < 1e-12

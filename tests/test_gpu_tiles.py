"""The grid update over touched node tiles only (mpm_tuning.grid_block = 0)
against the FP64 oracle and against the update of every node (gridUpdate,
kernels.cu:144-196, which writes every node of the grid)."""
import numpy as np
import pytest

from parity import assert_normwise, assert_state_close

pytestmark = pytest.mark.gpu


def _scene(n, size, seed, **kw):
    from mpm_b200 import scenes
    return scenes.small_scene(n, size, seed=seed, **kw)


@pytest.mark.parametrize("case", [dict(n=8192, size=(32, 32, 32), seed=1),
                                  dict(n=12_345, size=(48, 32, 40), seed=2),
                                  dict(n=257, size=(16, 16, 16), seed=6, obstacle=False)])
def test_one_substep_tiles(gpu_ok, mpm, oracle64, case):
    cfg, st, tris = _scene(**case)
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        eng.set_tuning(grid_block=0)
        assert eng.tuning()["grid_block"] == 0
        sdf = eng.get_sdf()
        eng.step(1)
        got, grid = eng.get_buffer(), eng.get_grid()
    st0 = oracle64.init_particles(cfg, st)
    want, wgrid, _, _ = oracle64.substep(cfg, st0, sdf.astype(np.float64))
    assert_state_close(got, want, st0)
    assert_normwise("grid mass", grid[0], wgrid[0])
    assert_normwise("grid velocity", grid[1:4], wgrid[1:4])


def test_tiles_left_behind_are_reset(gpu_ok, mpm):
    """A block of fluid thrown across the grid: the tiles it leaves must read
    zero afterwards, as in the update of every node, and the next substep from
    the same particles must give the same grid either way."""
    from mpm_b200 import scenes
    rng = np.random.default_rng(11)
    cfg = scenes.small_scene(1, (48, 32, 32), seed=11, obstacle=False)[0]
    pos = np.array([4.0, 8.0, 8.0]) + rng.random((6000, 3)) * np.array([10.0, 16.0, 16.0])
    st = scenes.pack_state(pos.astype(np.float32))
    st[3] = 4.0  # 0.4 cells per substep along +x
    tris = np.zeros((0, 9), np.float32)
    with mpm.Engine(cfg) as tiles, mpm.Engine(cfg) as every:
        tiles.init(st)
        tiles.init_sdf(tris)
        tiles.set_tuning(grid_block=0)
        tiles.step(30)
        mid = tiles.get_buffer()
        every.init(st)
        every.init_sdf(tris)
        every.set_tuning(grid_block=256)
        every.set_state(mid)
        tiles.step(1)
        every.step(1)
        g_t, g_e = tiles.get_grid(), every.get_grid()
        s_t, s_e = tiles.get_buffer(), every.get_buffer()
    assert mid[0].min() > 12.0, "the block did not move far enough to leave tiles"
    empty = g_e[0] == 0
    assert empty.sum() > 0.5 * empty.size
    assert not np.any(g_t[:, empty]), "a node the particles left still holds values"
    assert_normwise("grid mass", g_t[0], g_e[0])
    assert_normwise("grid velocity", g_t[1:4], g_e[1:4])
    assert_state_close(s_t, s_e, mid)


def test_batch_one_substep_tiles(gpu_ok, mpm, oracle64):
    """Touched tiles in a batch: every scene (one of them empty) after one
    substep against the FP64 oracle on that scene alone."""
    from mpm_b200 import scenes
    sc = [scenes.small_scene(3000, (32, 32, 32), seed=41),
          scenes.small_scene(5000, (48, 24, 40), seed=42),
          scenes.small_scene(10, (16, 16, 16), seed=43, obstacle=False)]
    cfg, st, tris = scenes.small_scene(100, (20, 20, 20), seed=45, obstacle=False)
    sc.append((cfg, st[:, :0], tris))
    with mpm.Batch([c for c, _, _ in sc]) as b:
        b.init_all([s for _, s, _ in sc])
        for k, (_, _, t) in enumerate(sc):
            if len(t):
                b.init_scene_sdf(k, t)
        b.set_tuning(grid_block=0)
        sdfs = [b.scene_sdf(k) for k in range(len(sc))]
        b.step(1)
        got = [b.scene_buffer(k) for k in range(len(sc))]
        grids = [b.scene_grid(k) for k in range(len(sc))]
    for k, (c, st, _) in enumerate(sc):
        if st.shape[1] == 0:
            assert not grids[k].any()
            continue
        st0 = oracle64.init_particles(c, st)
        want, wgrid, _, _ = oracle64.substep(c, st0, sdfs[k].astype(np.float64))
        assert_state_close(got[k], want, st0)
        assert_normwise(f"scene {k} grid mass", grids[k][0], wgrid[0])
        assert_normwise(f"scene {k} grid velocity", grids[k][1:4], wgrid[1:4])

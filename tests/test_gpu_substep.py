"""One MLS-MPM substep on the GPU vs the FP64 oracle, whole and stage by stage
(p2GTransferScatter kernels.cu:6-142, gridUpdate 144-196, g2PTransfer 199-280)."""
import numpy as np
import pytest

from parity import RTOL, assert_normwise, assert_state_close

pytestmark = pytest.mark.gpu

SCENES = {
    "cube32_obstacle": dict(n=8192, size=(32, 32, 32), seed=1),
    "box48x32x40_obstacle": dict(n=12_345, size=(48, 32, 40), seed=2),
    "cube32_free": dict(n=6000, size=(32, 32, 32), seed=3, obstacle=False),
    "gamma_neg2_gravity": dict(n=5000, size=(32, 32, 32), seed=4, gamma=-2.0, compression=200.0, gravity=9.81,
                               dt=0.01, resolution=1.0, padding=2),
    "one_particle": dict(n=1, size=(16, 16, 16), seed=5, obstacle=False),
    "n257": dict(n=257, size=(16, 16, 16), seed=6, obstacle=False),
}


def _scene(name):
    from mpm_b200 import scenes
    kw = dict(SCENES[name])
    n, size = kw.pop("n"), kw.pop("size")
    return scenes.small_scene(n, size, **kw)


def _run(mpm, cfg, st, tris, nsub):
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        start = eng.get_buffer()
        sdf = eng.get_sdf()
        eng.step(nsub)
        return start, sdf, eng.get_buffer(), eng.get_grid(), eng.get_positions()


@pytest.mark.parametrize("name", sorted(SCENES))
def test_one_substep(gpu_ok, mpm, oracle64, name):
    cfg, st, tris = _scene(name)
    start, sdf, got, grid, pos = _run(mpm, cfg, st, tris, 1)
    st0 = oracle64.init_particles(cfg, st)
    assert np.array_equal(start, st0.astype(np.float32)), "init rules (initFMatrices) differ"
    want, wgrid, _, _ = oracle64.substep(cfg, st0, sdf.astype(np.float64))
    assert_state_close(got, want, st0)
    assert_normwise("grid mass", grid[0], wgrid[0])
    assert_normwise("grid velocity", grid[1:4], wgrid[1:4])
    assert np.array_equal(pos, got[0:3].T), "position export differs from the state"


def test_stage_p2g(gpu_ok, mpm, oracle64):
    cfg, st, tris = _scene("box48x32x40_obstacle")
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        eng.substep_partial(mpm.STAGE_P2G)
        grid = eng.get_grid()
        _, perm = eng.get_sort()
        eng.substep_partial(mpm.STAGE_GRID)
        vgrid = eng.get_grid()
        sdf = eng.get_sdf()
        after = eng.get_buffer()
    st0 = oracle64.init_particles(cfg, st)
    assert np.array_equal(after, st0.astype(np.float32)), "a partial substep changed the particles"
    for tile_mode in (0, 1):  # with and without the reference's 1e-9 tile drop
        want = oracle64.p2g(cfg, st0, perm, tile_mode)
        assert_normwise(f"P2G mass (tile_mode {tile_mode})", grid[0], want[0])
        assert_normwise(f"P2G momentum (tile_mode {tile_mode})", grid[1:4], want[1:4])
    # Grid update on the engine's own P2G grid isolates the update stage (the
    # second partial substep redoes P2G: equal up to float-atomic order).
    upd = oracle64.grid_update(cfg, grid.astype(np.float64), sdf.astype(np.float64))
    assert_normwise("mass after update", vgrid[0], grid[0])
    assert_normwise("updated velocity", vgrid[1:4], upd[1:4])


def test_stage_g2p(gpu_ok, mpm, oracle64):
    """G2P alone: the oracle's gather on the engine's own updated grid."""
    cfg, st, tris = _scene("cube32_obstacle")
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        eng.substep_partial(mpm.STAGE_GRID)
        vgrid = eng.get_grid()
        sdf = eng.get_sdf()
        eng.substep_partial(mpm.STAGE_G2P)  # completes this substep on the same grid
        got = eng.get_buffer()
        assert eng.stats()["substeps"] == 1
    st0 = oracle64.init_particles(cfg, st)
    want = oracle64.g2p(cfg, st0, None, vgrid.astype(np.float64), sdf.astype(np.float64))
    assert_state_close(got, want, st0, rtol=RTOL)


def test_ten_substeps(gpu_ok, mpm, oracle64):
    """Ten substeps: FP32 and FP64 trajectories stay within 1e-4 (errors of
    each substep compound, so the one-substep bound is scaled by the count)."""
    cfg, st, tris = _scene("cube32_obstacle")
    start, sdf, got, _, _ = _run(mpm, cfg, st, tris, 10)
    s = oracle64.init_particles(cfg, st)
    st0 = s.copy()
    for _ in range(10):
        s = oracle64.substep(cfg, s, sdf.astype(np.float64))[0]
    assert_state_close(got, s, st0, rtol=1e-4)


def test_zero_particles(gpu_ok, mpm):
    from mpm_b200 import scenes
    cfg, _, tris = scenes.small_scene(10, (16, 16, 16), seed=1, obstacle=False)
    with mpm.Engine(cfg) as eng:
        eng.init(np.zeros((26, 0), np.float32))
        eng.step(3)
        assert eng.get_number() == 0
        g = eng.get_grid()
        assert not g.any()


def test_reinit_and_counts(gpu_ok, mpm):
    from mpm_b200 import scenes
    cfg, st, tris = scenes.small_scene(3000, (32, 32, 32), seed=8)
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.step(2)
        cfg2, st2, _ = scenes.small_scene(5000, (32, 32, 32), seed=9)
        eng.init(st2)
        assert eng.get_number() == 5000
        eng.step(1)
        s = eng.stats()
        assert s["substeps"] == 1 and s["kernel_launches"] > 0


def test_reinit_reuses_buffers(gpu_ok, mpm, oracle64):
    """Re-initialising with no more particles than before keeps the device
    buffers (6000, then 2500, then 6000 again); the substep after each init
    still matches the oracle."""
    from mpm_b200 import scenes
    cfg, big, tris = scenes.small_scene(6000, (32, 32, 32), seed=10)
    _, small, _ = scenes.small_scene(2500, (32, 32, 32), seed=11)
    with mpm.Engine(cfg) as eng:
        eng.init(big)
        eng.init_sdf(tris)
        eng.step(2)
        for st in (small, big):
            eng.init(st)
            assert eng.get_number() == st.shape[1]
            sdf = eng.get_sdf()
            eng.step(1)
            got = eng.get_buffer()
            st0 = oracle64.init_particles(cfg, st)
            want = oracle64.substep(cfg, st0, sdf.astype(np.float64))[0]
            assert_state_close(got, want, st0)


@pytest.mark.parametrize("case", ["dense_cap4", "one_cell_pile"])
def test_crowded_cells_through_the_list(gpu_ok, mpm, oracle64, case):
    """Particles past a cell's cap go to the crowded-cell list, 256 per entry,
    and a second launch sums them.  In a dense scene at the smallest cap, every
    cell above 4 particles takes that path; a pile of 3000 particles in one
    cell makes several entries of one cell."""
    from mpm_b200 import scenes
    cfg, st, tris = scenes.small_scene(30_000 if case == "dense_cap4" else 6000, (16, 16, 16), seed=7,
                                       obstacle=False)
    if case == "one_cell_pile":
        rng = np.random.default_rng(8)
        st[0:3, :3000] = rng.uniform(8.5, 9.5, (3, 3000)).astype(np.float32)  # stencil base cell (8, 8, 8)
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        if case == "dense_cap4":
            eng.set_tuning(12, 256, 256, 4)
        sdf = eng.get_sdf()
        eng.step(1)
        got = eng.get_buffer()
    st0 = oracle64.init_particles(cfg, st)
    want, _, _, _ = oracle64.substep(cfg, st0, sdf.astype(np.float64))
    assert_state_close(got, want, st0)

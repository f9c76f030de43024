"""Batches of independent scenes (no counterpart in the reference): every
scene of a batch must evolve exactly as it would alone.

Tolerances as in test_gpu_substep: each scene's state after one substep within
1e-5 (normwise) of the FP64 oracle run on that scene alone; keys and
permutation bit-exact; several substeps batched vs the same scenes in
single-scene engines within 1e-4 (float sums in a different order)."""
import numpy as np
import pytest

from parity import assert_normwise, assert_state_close, morton_reference, stable_sort_reference

pytestmark = pytest.mark.gpu


def _scenes():
    from mpm_b200 import scenes
    out = [
        scenes.small_scene(3000, (32, 32, 32), seed=41),
        scenes.small_scene(5000, (48, 24, 40), seed=42, obstacle=True),
        scenes.small_scene(10, (16, 16, 16), seed=43, obstacle=False),
        scenes.small_scene(4000, (24, 40, 32), seed=44, gamma=-2.0, gravity=9.81, compression=200.0, dt=0.01),
    ]
    cfg, st, tris = scenes.small_scene(100, (20, 20, 20), seed=45, obstacle=False)
    out.append((cfg, st[:, :0], tris))  # a scene without particles
    return out


def _batch(mpm, sc):
    b = mpm.Batch([c for c, _, _ in sc])
    b.init_all([s for _, s, _ in sc])
    for k, (_, _, t) in enumerate(sc):
        if len(t):
            b.init_scene_sdf(k, t)
    return b


def test_batch_one_substep_vs_oracle(gpu_ok, mpm, oracle64):
    sc = _scenes()
    with _batch(mpm, sc) as b:
        assert b.scenes == len(sc)
        starts = [b.scene_buffer(k) for k in range(len(sc))]
        sdfs = [b.scene_sdf(k) for k in range(len(sc))]
        b.step(1)
        got = [b.scene_buffer(k) for k in range(len(sc))]
        grids = [b.scene_grid(k) for k in range(len(sc))]
        sorts = [b.scene_sort(k) for k in range(len(sc))]
        pos = [b.scene_positions(k) for k in range(len(sc))]
    for k, (cfg, st, _) in enumerate(sc):
        st0 = oracle64.init_particles(cfg, st)
        assert np.array_equal(starts[k], st0.astype(np.float32)), f"scene {k}: init rules"
        if st.shape[1] == 0:
            assert got[k].shape == (26, 0) and not grids[k].any()
            continue
        want, wgrid, _, _ = oracle64.substep(cfg, st0, sdfs[k].astype(np.float64))
        assert_state_close(got[k], want, st0)
        assert_normwise(f"scene {k} grid mass", grids[k][0], wgrid[0])
        assert_normwise(f"scene {k} grid velocity", grids[k][1:4], wgrid[1:4])
        keys, perm = sorts[k]
        assert np.array_equal(keys, morton_reference(starts[k][0:3]))
        assert np.array_equal(perm, stable_sort_reference(keys))
        assert np.array_equal(pos[k], got[k][0:3].T)


def test_batch_matches_single_engines(gpu_ok, mpm):
    sc = _scenes()
    with _batch(mpm, sc) as b:
        b.step(6)
        batched = [b.scene_buffer(k) for k in range(len(sc))]
        assert b.stats()["substeps"] == 6
    for k, (cfg, st, tris) in enumerate(sc):
        if st.shape[1] == 0:
            continue
        with mpm.Engine(cfg) as e:
            e.init(st)
            if len(tris):
                e.init_sdf(tris)
            start = e.get_buffer()
            e.step(6)
            alone = e.get_buffer()
        assert_state_close(batched[k], alone.astype(np.float64), start, rtol=1e-4)


def test_batch_errors(gpu_ok, mpm):
    from mpm_b200 import scenes
    cfg, st, _ = scenes.small_scene(100, (16, 16, 16), seed=46, obstacle=False)
    with mpm.Batch([cfg, cfg]) as b:
        with pytest.raises(mpm.MpmError) as ei:
            b.init(st)  # the single-scene init is refused for a batch
        assert ei.value.name == "MPM_ERR_UNSUPPORTED"
        b.init_all([st, st])
        with pytest.raises(mpm.MpmError) as ei:
            b.init_scene_sdf(2, np.zeros((0, 9), np.float32))
        assert ei.value.name == "MPM_ERR_INVALID_ARGUMENT"
        b.step(2)
        a0, a1 = b.scene_buffer(0), b.scene_buffer(1)
    assert np.array_equal(a0[24:26], a1[24:26])
    # identical scenes evolve identically up to float-sum order
    assert np.abs(a0[0:3].astype(np.float64) - a1[0:3]).max() < 1e-4


def test_autotune_keeps_state_and_results(gpu_ok, mpm):
    sc = _scenes()
    with _batch(mpm, sc) as b:
        b.step(2)
        before = [b.scene_buffer(k) for k in range(len(sc))]
        t = b.autotune(repeats=2)
        assert t["p2g_ctas_per_sm"] >= 1 and t["g2p_block"] in (128, 256, 512) and t["grid_block"] in (128, 256)
        assert t["p2g_cell_cap"] == 0  # chosen per work item
        assert t["p2g_ms"] > 0 and t["g2p_ms"] > 0 and t["grid_ms"] > 0
        assert b.tuning()["p2g_ctas_per_sm"] == t["p2g_ctas_per_sm"]
        after = [b.scene_buffer(k) for k in range(len(sc))]
        for x, y in zip(before, after):
            assert np.array_equal(x, y)  # tuning does not advance the state
        assert b.stats()["substeps"] == 2
        b.step(3)
        tuned = [b.scene_buffer(k) for k in range(len(sc))]
    with _batch(mpm, sc) as b:
        b.step(2)
        b.set_tuning(4, 128, 128, 32)
        b.step(3)
        other = [b.scene_buffer(k) for k in range(len(sc))]
        with pytest.raises(mpm.MpmError):
            b.set_tuning(0, 256, 256)
    for k, (x, y) in enumerate(zip(tuned, other)):
        if x.shape[1]:
            assert_state_close(x, y.astype(np.float64), before[k], rtol=1e-4)


def test_batch_beyond_shared_scene_table(gpu_ok, mpm):
    """More scenes than the kernels stage in shared memory (64): the scene
    lookup falls back to the global table; every scene still evolves as alone."""
    from mpm_b200 import scenes
    sc = [scenes.small_scene(200 + 37 * k, (16 + (k % 3) * 8, 16, 16 + (k % 2) * 8), seed=500 + k,
                             obstacle=(k % 4 == 0)) for k in range(70)]
    with _batch(mpm, sc) as b:
        assert b.scenes == 70
        b.step(3)
        got = [b.scene_buffer(k) for k in (0, 33, 64, 69)]
    for g, k in zip(got, (0, 33, 64, 69)):
        cfg, st, tris = sc[k]
        with mpm.Engine(cfg) as e:
            e.init(st)
            if len(tris):
                e.init_sdf(tris)
            start = e.get_buffer()
            e.step(3)
            alone = e.get_buffer()
        assert_state_close(g, alone.astype(np.float64), start, rtol=1e-4)

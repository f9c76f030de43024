"""Error paths of the C ABI on a GPU: every failure is a status code, the
engine stays usable afterwards.  Faults are made on the host (bad arguments,
NaN or out-of-grid values in the state); nothing here faults the GPU."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small(seed=1):
    from mpm_b200 import scenes
    return scenes.small_scene(2000, (32, 32, 32), seed=seed)


def test_not_initialized(gpu_ok, mpm):
    cfg, st, tris = _small()
    with mpm.Engine(cfg) as eng:
        with pytest.raises(mpm.MpmError) as ei:
            eng.step(1)
        assert ei.value.name == "MPM_ERR_NOT_INITIALIZED"
        eng.init(st)
        eng.step(1)


def test_bad_arguments(gpu_ok, mpm):
    cfg, st, tris = _small()
    lib = mpm.lib
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        assert lib.mpm_step(eng._h, -1) == 1
        assert lib.mpm_init_particles(eng._h, -5, None) == 1
        assert lib.mpm_init_particles(eng._h, 10, None) == 1
        assert lib.mpm_substep_partial(eng._h, 9) == 1
        assert lib.mpm_set_state(eng._h, 7, None) == 1
        assert lib.mpm_get_grid(eng._h, None) == 1
        assert b"NULL" in lib.mpm_last_error(eng._h) or lib.mpm_last_error(eng._h)
        eng.step(1)  # still usable
    assert lib.mpm_step(None, 1) == 1


def test_bad_config(gpu_ok, mpm):
    from mpm_b200 import Config
    for bad in (dict(size_x=0), dict(size_y=-3), dict(dt=float("nan")), dict(size_x=4096, size_y=4096, size_z=4096)):
        with pytest.raises(mpm.MpmError) as ei:
            mpm.Engine(Config(**bad))
        assert ei.value.name == "MPM_ERR_BAD_CONFIG"
    with pytest.raises(mpm.MpmError) as ei:
        mpm.Engine(Config(), device=99)
    assert ei.value.name == "MPM_ERR_INVALID_ARGUMENT"


def test_set_state_rejects_nonuniform_mass(gpu_ok, mpm):
    cfg, st, tris = _small()
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        s = eng.get_buffer()
        s[25, 3] = 2.0
        with pytest.raises(mpm.MpmError) as ei:
            eng.set_state(s)
        assert ei.value.name == "MPM_ERR_UNSUPPORTED"
        eng.step(1)


def test_health_nonfinite(gpu_ok, mpm):
    cfg, st, tris = _small()
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        s = eng.get_buffer()
        s[3, 17] = np.nan  # a NaN velocity reaches positions after one substep
        eng.set_state(s)
        eng.step(1)  # checks off: the reference also just continues
        assert eng.stats()["health"] & mpm.HEALTH_NONFINITE
        eng.set_checks(mpm.HEALTH_NONFINITE)
        with pytest.raises(mpm.MpmError) as ei:
            eng.step(1)
        assert ei.value.name == "MPM_ERR_NONFINITE_STATE"
        eng.stats(reset_health=True)
        eng.init(st)
        eng.step(2)  # clean state: no error
        assert eng.stats()["health"] == 0


def test_health_out_of_grid(gpu_ok, mpm):
    cfg, st, tris = _small()
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        s = eng.get_buffer()
        s[0, 5] = 40.0  # outside a 32-node grid on x
        eng.set_state(s)
        eng.set_checks(mpm.HEALTH_OUT_OF_GRID)
        with pytest.raises(mpm.MpmError) as ei:
            eng.step(1)
        assert ei.value.name == "MPM_ERR_OUT_OF_GRID"
        got = eng.get_buffer()
        assert got[0, 5] > 32.0  # like the reference, particles are never clamped


def test_stage_timing(gpu_ok, mpm):
    cfg, st, tris = _small()
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        eng.set_stage_timing(5)
        eng.step(8)  # more substeps than slots: the rest go to scratch events
        ms, cnt = eng.stage_times()
        assert cnt == 5 and all(v > 0 for v in ms.values())
        eng.set_stage_timing(0)
        eng.step(2)
        ms, cnt = eng.stage_times()
        assert cnt == 0


def test_async_and_stream(gpu_ok, mpm):
    cfg, st, tris = _small()
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        eng.step_async(3)
        eng.synchronize()
        assert eng.stream() != 0
        assert eng.positions_device_ptr() != 0
        assert eng.stats()["substeps"] == 3


def test_two_engines_one_process(gpu_ok, mpm):
    cfg, st, tris = _small(1)
    cfg2, st2, tris2 = _small(2)
    with mpm.Engine(cfg) as a, mpm.Engine(cfg2) as b:
        a.init(st)
        b.init(st2)
        a.init_sdf(tris)
        b.init_sdf(tris2)
        a.step(2)
        b.step(2)
        assert a.get_number() == b.get_number() == 2000
        assert not np.array_equal(a.get_buffer(), b.get_buffer())


# Bounded device waits.  The test hooks make the first wait of the SDF build
# (triangle tile copies) or of the learned step's tcgen05 MMAs give up, only
# after the real completion has been observed: *_GIVE_UP reports it at once,
# *_EXPIRE waits for a barrier phase that nothing completes until the 20 ms
# limit really runs out.  Nothing is in flight when the CTAs give up, free
# their TMEM and return, so the GPU context stays usable.
@pytest.mark.parametrize("hook", ["WAIT_TEST_SDF_GIVE_UP", "WAIT_TEST_SDF_EXPIRE"])
def test_sdf_wait_gives_up_and_engine_recovers(gpu_ok, mpm, oracle64, hook):
    from mpm_b200 import scenes
    cfg, st, _ = scenes.small_scene(2000, (32, 32, 32), seed=3)
    # Two tiles of triangles (the kernel streams 256 per tile).
    tris = np.concatenate([scenes.torus(8.0, 3.0, (16.2, 15.7, 16.1), 24, 12),
                           scenes.uv_sphere(4.0, (8.3, 9.1, 22.4), 16, 8)])
    assert len(tris) > 256
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.set_wait_test(getattr(mpm, hook))
        with pytest.raises(mpm.MpmError) as ei:
            eng.init_sdf(tris)
        assert ei.value.name == "MPM_ERR_TIMEOUT"
        eng.set_wait_test(0)
        eng.init_sdf(tris)  # the next call succeeds
        sdf = eng.get_sdf()
        want, _ = oracle64.make_sdf(cfg, tris)
        assert np.abs(sdf.astype(np.float64) - want).max() <= 1e-4
        eng.step(2)


@pytest.mark.parametrize("hook", ["WAIT_TEST_MMA_GIVE_UP", "WAIT_TEST_MMA_EXPIRE"])
def test_tcgen05_wait_gives_up_and_engine_recovers(gpu_ok, mpm, hook):
    from mpm_b200 import learned
    from mpm_b200 import scenes
    # Water at rest in the physical orientation (the corrector's training
    # regime): a large step of random C and F could invert F, which the
    # reference's J < 0.3 rescue turns into NaN.
    cfg, st, tris = scenes.small_scene(4096, (32, 32, 32), seed=11, randomize=False)
    cfg = learned.physical_config(cfg)
    params, _ = learned.load_params(learned.PHYSICAL_PARAMS)
    with mpm.Engine(cfg) as ref_eng:
        ref_eng.init(st)
        ref_eng.init_sdf(tris)
        ref_eng.set_corrector(params, ratio=4, max_density_change=-1.0)
        ref_eng.step_learned(1)
        want = ref_eng.get_buffer()
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        eng.set_corrector(params, ratio=4, max_density_change=-1.0)
        eng.set_wait_test(getattr(mpm, hook))
        with pytest.raises(mpm.MpmError) as ei:
            eng.step_learned(1)
        assert ei.value.name == "MPM_ERR_TIMEOUT"
        eng.set_wait_test(0)
        eng.init(st)  # the failed step's state is unspecified: start again
        eng.step_learned(1)
        got = eng.get_buffer()
    assert np.isfinite(want).all()
    assert np.abs(got.astype(np.float64) - want).max() <= 1e-4 * max(1.0, np.abs(want).max())


def test_wait_test_rejects_unknown_flags(gpu_ok, mpm):
    cfg, st, tris = _small()
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        with pytest.raises(mpm.MpmError) as ei:
            eng.set_wait_test(0x100)
        assert ei.value.name == "MPM_ERR_INVALID_ARGUMENT"

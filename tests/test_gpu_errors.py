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

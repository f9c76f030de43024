"""The engine against the reference's own CUDA engine (engine.cu/kernels.cu
compiled from the reference sources into oracle/_ref) on identical inputs:
keys and sort permutation bit-exact, state/grid/SDF within the parity
tolerances, and both FP32 engines against the FP64 oracle."""
import os

import numpy as np
import pytest

from parity import assert_normwise, assert_state_close

pytestmark = pytest.mark.gpu

REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libref_engine.so")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference engine not built")


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import RefEngine
    r = RefEngine()
    yield r
    r.destroy()


def _scene(seed, size=(32, 32, 32), n=8192, obstacle=True):
    from mpm_b200 import scenes
    return scenes.small_scene(n, size, seed=seed, obstacle=obstacle)


@needs_ref
@pytest.mark.parametrize("seed,size", [(21, (32, 32, 32)), (22, (64, 32, 48))])
def test_substep_vs_reference(gpu_ok, mpm, oracle64, ref, tmp_path, seed, size):
    cfg, st, tris = _scene(seed, size)
    ref.create(cfg, st, tris, str(tmp_path / "config.txt"))
    r_start = ref.state()
    r_keys = ref.keys()
    ref.step(1)
    r_state, r_grid, r_perm, r_sdf, r_pos = ref.state(), ref.grid(), ref.perm(), ref.sdf(), ref.positions()
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        start = eng.get_buffer()
        sdf = eng.get_sdf()
        eng.step(1)
        keys, perm = eng.get_sort()
        state, grid, pos = eng.get_buffer(), eng.get_grid(), eng.get_positions()
    assert np.array_equal(start, r_start), "initial state (initFMatrices) differs from the reference"
    assert np.array_equal(keys, r_keys), "Morton keys differ from the reference's setKeys"
    assert np.array_equal(perm, r_perm), "sort permutation differs from the reference's thrust sort"
    assert np.abs(sdf - r_sdf).max() <= 1e-4
    # Both FP32 engines against the FP64 oracle, then against each other.
    want, wgrid, _, _ = oracle64.substep(cfg, r_start.astype(np.float64), r_sdf.astype(np.float64))
    assert_state_close(r_state, want, r_start)
    assert_state_close(state, want, r_start)
    # Two FP32 results each within RTOL of FP64 are within 2 RTOL of each other.
    assert_state_close(state, r_state, r_start, rtol=2e-5)
    assert_normwise("grid mass vs reference", grid[0], r_grid[0], rtol=2e-5)
    assert_normwise("grid velocity vs reference", grid[1:4], r_grid[1:4], rtol=2e-5)
    assert np.abs(pos - r_pos).max() <= np.abs(r_pos).max() * 1e-6 + 1e-5


@needs_ref
def test_sdf_vs_reference(gpu_ok, mpm, ref, tmp_path):
    from mpm_b200 import scenes
    cfg, st, _ = _scene(23, (48, 32, 48), n=512, obstacle=False)
    tris = scenes.torus(12.0, 4.0, (24.3, 15.9, 23.8), 24, 12)
    ref.create(cfg, st, tris, str(tmp_path / "config.txt"))
    r_sdf = ref.sdf()
    with mpm.Engine(cfg) as eng:
        eng.init_sdf(tris)
        sdf = eng.get_sdf()
    err = np.abs(sdf.astype(np.float64) - r_sdf)
    assert err.max() <= 1e-4


@needs_ref
def test_sort_vs_reference_after_steps(gpu_ok, mpm, ref, tmp_path):
    """After several substeps the engine's sort of a state equals the
    reference's sort of the same state."""
    cfg, st, tris = _scene(24, (32, 32, 32), n=20_000)
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        eng.step(5)
        mid = eng.get_buffer()
        eng.step(1)
        keys, perm = eng.get_sort()
    ref.create(cfg, mid, tris, str(tmp_path / "config.txt"))
    # Engine::init re-applies initFMatrices to the diagonal of F; keys depend on positions only.
    assert np.array_equal(ref.keys(), keys)
    ref.sort_only()
    assert np.array_equal(ref.perm(), perm)


@needs_ref
def test_config_file_parity(gpu_ok, mpm, ref, tmp_path):
    """The same config.txt read by the reference's GameConfigData and by the
    engine's parser gives the same values."""
    text = ("SIZE_X = 1 28\nSIZE_Y=64\nSIZE_Z=32\n\nPADDING=3\nGRAVITY=-0.3\nDT=0.1\nGAMMA=7\n"
            "COMPRESSION=10.0\nRESOLUTION=0.5\nSUBSTEPS=4\nSDF_RESOLUTION=1.5e2\nnot a key line\n"
            "WATER=models/sphere.obj;15.0;0.0;20.0;25.0\nOBJECT=a b.obj; 110;0;-10;0;extra\nDT=0.05\n")
    p = tmp_path / "config.txt"
    p.write_text(text)
    ref.lib.ref_config_load(str(p).encode())
    cfg = mpm.parse_config_file(str(p))
    for key, val in [("SIZE_X", cfg.size_x), ("SIZE_Y", cfg.size_y), ("SIZE_Z", cfg.size_z),
                     ("PADDING", cfg.padding), ("SUBSTEPS", cfg.substeps), ("SDF_RESOLUTION", cfg.sdf_resolution)]:
        assert ref.lib.ref_config_get_int(key.encode()) == val, key
    for key, val in [("GRAVITY", cfg.gravity), ("DT", cfg.dt), ("GAMMA", cfg.gamma),
                     ("COMPRESSION", cfg.compression), ("RESOLUTION", cfg.resolution)]:
        assert np.float32(ref.lib.ref_config_get_float(key.encode())) == np.float32(val), key
    import ctypes
    vals = (ctypes.c_float * 16)()
    paths = ctypes.create_string_buffer(1024)
    for which, entries in ((0, cfg.waters), (1, cfg.objects)):
        cnt = ref.lib.ref_config_entries(which, vals, paths, 1024, 4)
        assert cnt == len(entries)
        names = paths.raw.split(b"\0")
        for i, e in enumerate(entries):
            assert names[i].decode() == e.model_path
            assert list(np.float32(vals[4 * i: 4 * i + 4])) == list(np.float32([e.scale, e.x, e.y, e.z]))

"""The C-ABI library loads on a CPU-only host and exports every entry point
declared in include/*.h; no compute call is made here."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(mpm_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = _declared()
    for must in ("mpm_create", "mpm_destroy", "mpm_init_particles", "mpm_init_sdf", "mpm_step", "mpm_get_state",
                 "mpm_get_positions", "mpm_positions_device", "mpm_get_grid", "mpm_get_sort",
                 "mpm_sort_particles_device", "mpm_config_parse_file"):
        assert must in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol(mpm):
    lib = ctypes.CDLL(mpm.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_abi_version_and_status_strings(mpm):
    assert mpm.lib.mpm_abi_version() == 1
    for code, name in mpm.STATUS.items():
        assert mpm.lib.mpm_status_string(code).decode() == name


def test_create_without_gpu_is_an_error(mpm):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(mpm.MpmError) as ei:
        mpm.Engine(mpm.Config())
    assert ei.value.name == "MPM_ERR_NO_DEVICE"
    assert mpm.lib.mpm_global_last_error()


def test_null_engine_calls(mpm):
    lib = mpm.lib
    assert lib.mpm_step(None, 1) == 1
    assert lib.mpm_get_state(None, None) == 1
    assert lib.mpm_num_particles(None) == 0
    assert lib.mpm_positions_device(None) is None
    assert lib.mpm_last_error(None) == b""
    lib.mpm_destroy(None)



def test_wrapper_marshalling_against_null_engine(mpm):
    """Every Engine method marshals its arguments (ctypes) and reaches the
    library, which rejects the NULL engine with MPM_ERR_INVALID_ARGUMENT."""
    import numpy as np
    e = mpm.Engine.__new__(mpm.Engine)
    e._h = None
    e.cfg = mpm.Config(size_x=8, size_y=8, size_z=8)
    e.n = 4
    st = np.zeros((26, 4), np.float32)
    calls = [lambda: e.init(st), lambda: e.init_sdf(np.zeros((2, 9), np.float32)), lambda: e.set_state(st),
             lambda: e.step(1), lambda: e.step_async(1), e.synchronize, lambda: e.substep_partial(2),
             lambda: e.set_checks(1), e.get_buffer, e.get_positions, e.get_grid, e.get_sdf, e.get_sort, e.stats,
             lambda: e.set_stage_timing(2), e.stage_times]
    for call in calls:
        with pytest.raises(mpm.MpmError) as ei:
            call()
        assert ei.value.name == "MPM_ERR_INVALID_ARGUMENT"
    assert e.get_number() == 0 and e.positions_device_ptr() == 0 and e.stream() == 0
    with pytest.raises(mpm.MpmError):
        mpm.sort_particles_device(0, 0, 0, 5, 0, 0, 0)
    assert mpm.lib.mpm_sort_particles_device(None, None, None, 0, None, None, None) == 0


def test_corrector_layout_matches_header():
    """The parameter offsets documented in mpm_b200.h match the reference MLP."""
    import re
    import mlp_ref
    hdr = open(os.path.join(ROOT, "include", "mpm_b200.h")).read()
    assert int(re.search(r"#define MPM_CORRECTOR_PARAMS (\d+)", hdr).group(1)) == mlp_ref.NPARAMS
    for name, label in (("in_mean", "input mean"), ("in_inv_std", "input 1/std"), ("out_std", "output scale"),
                        ("W1", "W1"), ("b1", "b1"), ("W2", "W2"), ("b2", "b2"), ("W3", "W3"), ("b3", "b3")):
        m = re.search(re.escape(label) + r" \[[^\]]*\](?:\[[^\]]*\])?[\s*]*@(\d+)", hdr)
        assert m and int(m.group(1)) == mlp_ref.OFF[name][0], name


def test_cli_usage_and_checkpoint_errors_without_gpu(tmp_path):
    import subprocess
    cli = os.path.join(ROOT, "water-sim-cuda_b200", "bin", "mpm_run")
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    import mpm_b200
    with pytest.raises(mpm_b200.MpmError) as ei:
        mpm_b200.checkpoint_info(str(tmp_path / "none.ckpt"))
    assert ei.value.name == "MPM_ERR_IO"
    (tmp_path / "x.ckpt").write_bytes(b"NOTACKPT" + bytes(200))
    with pytest.raises(mpm_b200.MpmError) as ei:
        mpm_b200.checkpoint_info(str(tmp_path / "x.ckpt"))
    assert "magic" in str(ei.value)


def test_scene_generation_maps_no_library():
    """The package maps libmpm_b200.so on its first library call, not at
    import: the reference arm of the benchmark builds its scenes with
    `mpm_b200.scenes` and must run without the engine's code mapped."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, sys.argv[1])\n"
            "from mpm_b200 import scenes\n"
            "cfg, st, tris = scenes.small_scene(512, (16, 16, 16), seed=1)\n"
            "import mpm_b200\n"
            "assert not mpm_b200.lib.loaded(), 'library mapped by scene generation'\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libmpm_b200' not in maps, 'libmpm_b200.so is mapped'\n")
    r = subprocess.run([sys.executable, "-c", code, os.path.join(ROOT, "water-sim-cuda_b200")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

"""config.txt parsing (GameConfigData, game_configdata.cpp:22-90;
Simulation::initDeviceParams, Simulation.cpp:56-77).  Host only."""
import os

import numpy as np
import pytest

BASE = ("SIZE_X=128\nSIZE_Y=128\nSIZE_Z=128\nPADDING=2\nGRAVITY=9.81\nDT=0.01\nGAMMA=-2.0\n"
        "COMPRESSION=200.0\nRESOLUTION=1.0\nSUBSTEPS=10\nSDF_RESOLUTION=256\n")


def test_reference_config_file(mpm):
    """The reference's own config.txt, values as std::stoi/std::stof read them
    (read as text from the reference tree when it is present)."""
    from conftest import reference_tree
    path = os.path.join(reference_tree() or "", "config.txt")
    text = open(path).read() if os.path.exists(path) else (
        BASE + "\n\nWATER=models/sphere.obj;15.0;0.0;20.0;25.0\nWATER=models/sphere.obj;15.0;10.0;20.0;25.0\n\n"
        "OBJECT=models/u.obj;110.0;0.0;-10.0;0.0")
    c = mpm.parse_config_string(text)
    assert (c.size_x, c.size_y, c.size_z, c.padding, c.substeps, c.sdf_resolution) == (128, 128, 128, 2, 10, 256)
    assert np.float32(c.gravity) == np.float32(9.81) and np.float32(c.dt) == np.float32(0.01)
    assert c.gamma == -2.0 and c.compression == 200.0 and c.resolution == 1.0
    assert [w.model_path for w in c.waters] == ["models/sphere.obj"] * 2
    assert [(w.scale, w.x, w.y, w.z) for w in c.waters] == [(15.0, 0.0, 20.0, 25.0), (15.0, 10.0, 20.0, 25.0)]
    assert [(o.model_path, o.scale, o.y) for o in c.objects] == [("models/u.obj", 110.0, -10.0)]


def test_spaces_removed_and_overrides(mpm):
    c = mpm.parse_config_string(BASE.replace("SIZE_X=128", "SIZE_X = 1 2 8") + "DT=0.05\n  \nno equals here\n")
    assert c.size_x == 128 and np.float32(c.dt) == np.float32(0.05)


def test_stoi_prefix_semantics(mpm):
    c = mpm.parse_config_string(BASE.replace("PADDING=2", "PADDING=3.9").replace("SUBSTEPS=10", "SUBSTEPS=+4abc")
                                .replace("SDF_RESOLUTION=256", "SDF_RESOLUTION=1e3"))
    assert (c.padding, c.substeps, c.sdf_resolution) == (3, 4, 1)
    # RESOLUTION is read as a float: 0.5 stays 0.5 (the kernels read it as float)
    c = mpm.parse_config_string(BASE.replace("RESOLUTION=1.0", "RESOLUTION=0.5"))
    assert c.resolution == 0.5


def test_stof_forms(mpm):
    c = mpm.parse_config_string(BASE.replace("GRAVITY=9.81", "GRAVITY=-3e-1").replace("DT=0.01", "DT=.1xyz"))
    assert np.float32(c.gravity) == np.float32(-0.3) and np.float32(c.dt) == np.float32(0.1)


@pytest.mark.parametrize("key", ["SIZE_X", "SIZE_Y", "SIZE_Z", "PADDING", "GRAVITY", "DT", "GAMMA", "COMPRESSION",
                                 "RESOLUTION", "SUBSTEPS", "SDF_RESOLUTION"])
def test_missing_key(mpm, key):
    text = "\n".join(l for l in BASE.splitlines() if not l.startswith(key + "="))
    with pytest.raises(mpm.MpmError) as ei:
        mpm.parse_config_string(text)
    assert ei.value.name == "MPM_ERR_BAD_CONFIG" and key in str(ei.value)


@pytest.mark.parametrize("bad", ["SIZE_X=abc", "SIZE_X=99999999999", "DT=x1", "GRAVITY=1e99"])
def test_unparsable_value(mpm, bad):
    key = bad.split("=")[0]
    text = "\n".join(bad if l.startswith(key + "=") else l for l in BASE.splitlines())
    with pytest.raises(mpm.MpmError) as ei:
        mpm.parse_config_string(text)
    assert ei.value.name == "MPM_ERR_BAD_CONFIG"


@pytest.mark.parametrize("entry", ["WATER=models/a.obj;1;2;3", "OBJECT=x", "WATER=a;b;1;2;3", "OBJECT=a;1;2;3;"])
def test_malformed_entry(mpm, entry):
    with pytest.raises(mpm.MpmError) as ei:
        mpm.parse_config_string(BASE + entry + "\n")
    assert ei.value.name == "MPM_ERR_BAD_CONFIG"


def test_entry_extra_fields_and_spaces(mpm):
    c = mpm.parse_config_string(BASE + "OBJECT = my model.obj ; 2.5 ;1;2;3;ignored\n")
    assert c.objects[0].model_path == "mymodel.obj" and c.objects[0].scale == 2.5


def test_file_errors(mpm, tmp_path):
    with pytest.raises(mpm.MpmError) as ei:
        mpm.parse_config_file(str(tmp_path / "missing.txt"))
    assert ei.value.name == "MPM_ERR_IO"
    p = tmp_path / "c.txt"
    p.write_text(BASE)
    assert mpm.parse_config_file(str(p)).size_x == 128


def test_round_trip_text(mpm):
    from mpm_b200 import scenes
    cfg = scenes._cfg((64, 32, 16))
    back = mpm.parse_config_string(cfg.to_text())
    for f in ("size_x", "size_y", "size_z", "padding", "substeps", "sdf_resolution"):
        assert getattr(back, f) == getattr(cfg, f)
    for f in ("gravity", "dt", "gamma", "compression", "resolution"):
        assert np.float32(getattr(back, f)) == np.float32(getattr(cfg, f))

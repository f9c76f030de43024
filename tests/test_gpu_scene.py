"""Scene construction on the GPU (voxelization and lattice snapping) against
the CPU restatement (oracle/scene_oracle.c), bit for bit, and the whole
WATER= / OBJECT= path of a config file."""
import numpy as np
import pytest

import objgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sco():
    from oracle.oracle import SceneOracle
    return SceneOracle()


MESHES = {
    "sphere": lambda: objgen.uv_sphere(15.0, 32, 16, (3.0, -2.0, 1.5)),
    "sphere_small": lambda: objgen.uv_sphere(1.0, 12, 8, style="v/t/n"),
    "torus": lambda: objgen.torus(25.0, 8.0, 48, 24),
    "flat_box": lambda: objgen.box((0.0, 0.0, 0.0), (10.0, 3.0, 7.0)),
}


@pytest.mark.parametrize("name", sorted(MESHES))
def test_voxelize_matches_oracle(gpu_ok, mpm, sco, name):
    text = MESHES[name]()
    mesh = mpm.Mesh.from_text(text)
    got = mesh.voxelize(100.0)
    v, f = sco.parse_obj(text)
    want = sco.voxelize(v, f, 100.0)
    assert got.shape == want.shape and np.array_equal(got, want)


def test_voxelize_known_answer(gpu_ok, mpm):
    got = mpm.Mesh.from_text(objgen.box((0.0, 0.0, 0.0), (100.0, 100.0, 100.0))).voxelize(100.0)
    assert len(got) == 100 ** 3 - 99 ** 3
    assert np.array_equal(np.unique(np.floor(got).astype(int)), np.arange(100))


@pytest.mark.parametrize("case", [(128.0, 30.0, (0.0, 20.0, 25.0), 1), (128.0, 66.0, (16.0, -34.0, 0.0), 1),
                                  (64.0, 40.0, (5.0, 5.0, 5.0), 2), (128.0, 300.0, (0.0, 0.0, 0.0), 1)])
def test_normalize_matches_oracle(gpu_ok, mpm, sco, case):
    size, scale, disp, step = case
    text = MESHES["sphere"]()
    vox = mpm.Mesh.from_text(text).voxelize(100.0)
    got = mpm.normalize_points(vox, size, scale, disp, step)
    want = sco.normalize(vox, size, scale, disp, step)
    assert got.shape == want.shape and np.array_equal(got, want)


def test_normalize_known_answers(gpu_ok, mpm):
    one = np.array([[1.5, 2.5, 3.5]], np.float32)
    assert np.array_equal(mpm.normalize_points(one, 64.0, 8.0, (0, 0, 0), 1), one)
    out = mpm.normalize_points(np.array([[0.0, 0, 0], [2.0, 0, 0]], np.float32), 64.0, 8.0, (0, 0, 0), 1)
    xs = set(range(26, 31)) | set(range(34, 39))
    want = sorted((x, y, z) for x in xs for y in range(30, 35) for z in range(30, 35))
    assert out.tolist() == [list(map(float, w)) for w in want]
    with pytest.raises(mpm.MpmError) as ei:
        mpm.normalize_points(np.zeros((3, 3), np.float32), 64.0, 8.0, (0, 0, 0), 0)
    assert ei.value.name == "MPM_ERR_BAD_CONFIG"


def _config(waters, objects, res="1.0", size=128):
    lines = [f"SIZE_X={size}", f"SIZE_Y={size}", f"SIZE_Z={size}", "PADDING=2", "GRAVITY=9.81", "DT=0.01",
             "GAMMA=-2.0", "COMPRESSION=200.0", f"RESOLUTION={res}", "SUBSTEPS=10", "SDF_RESOLUTION=256"]
    lines += [f"WATER={w}" for w in waters] + [f"OBJECT={o}" for o in objects]
    return "\n".join(lines) + "\n"


def test_build_scene_matches_oracle(gpu_ok, mpm, sco, tmp_path):
    (tmp_path / "models").mkdir()
    (tmp_path / "models" / "sphere.obj").write_text(MESHES["sphere"]())
    (tmp_path / "models" / "torus.obj").write_text(MESHES["torus"]())
    waters = ["models/sphere.obj;15.0;0.0;20.0;25.0", "models/sphere.obj;15.0;10.0;20.0;25.0"]
    objects = ["models/torus.obj;110.0;0.0;-10.0;0.0", "models/missing.obj;5;0;0;0"]
    cfg, st, tris, log = mpm.build_scene(_config(waters, objects), str(tmp_path))
    assert "missing.obj" in log
    parts = []
    for w in waters:
        path, scale, x, y, z = w.split(";")
        v, f = sco.parse_obj((tmp_path / path).read_text())
        parts.append(sco.normalize(sco.voxelize(v, f, 100.0), 128.0, float(scale), (float(x), float(y), float(z)), 1))
    want = np.concatenate(parts)
    assert st.shape == (26, len(want))
    assert np.array_equal(st[0:3].T, want)
    assert not st[3:24].any() and (st[24:26] == 1).all()
    v, f = sco.parse_obj((tmp_path / "models" / "torus.obj").read_text())
    wt = sco.normalize_triangles(v[f].reshape(-1, 9), 128.0, 110.0, (0.0, -10.0, 0.0))
    assert np.array_equal(tris, wt)
    # the scene runs: Engine::init + initSDF + a few substeps
    with mpm.Engine(cfg) as e:
        e.init(st)
        e.init_sdf(tris)
        e.step(3)
        assert np.isfinite(e.get_positions()).all()


def test_build_scene_errors(gpu_ok, mpm, tmp_path):
    (tmp_path / "s.obj").write_text(MESHES["sphere_small"]())
    with pytest.raises(mpm.MpmError) as ei:
        mpm.build_scene(_config(["s.obj;10;0;0;0"], [], res="0.5"), str(tmp_path))
    assert ei.value.name == "MPM_ERR_BAD_CONFIG"  # getInt("RESOLUTION") = 0
    with pytest.raises(mpm.MpmError) as ei:
        mpm.build_scene(_config(["nothere.obj;10;0;0;0"], []), str(tmp_path))
    assert ei.value.name == "MPM_ERR_IO"
    cfg, st, tris, _ = mpm.build_scene(_config([], []), str(tmp_path))
    assert st.shape == (26, 0) and tris.shape == (0, 9)

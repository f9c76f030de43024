"""Scene construction on the host (no GPU): OBJ reading and the obstacle
triangle transform against the CPU restatement (oracle/scene_oracle.c), and
hand-derived answers.  Bit-exact: both sides perform the same float
operations in the same order."""
import numpy as np
import pytest

import objgen


@pytest.fixture(scope="module")
def sco():
    from oracle.oracle import SceneOracle
    return SceneOracle()


OBJS = {
    "sphere_v": lambda: objgen.uv_sphere(15.0, 32, 16, (3.0, -2.0, 1.5)),
    "sphere_vtn": lambda: objgen.uv_sphere(1.0, 12, 8, style="v/t/n"),
    "sphere_vn": lambda: objgen.uv_sphere(2.5, 20, 10, style="v//n"),
    "torus_negative": lambda: objgen.torus(25.0, 8.0, 48, 24),
    "box": lambda: objgen.box((-1.0, 2.0, 0.5), (3.0, 2.5, 4.0)),
}


@pytest.mark.parametrize("name", sorted(OBJS))
def test_obj_matches_oracle(mpm, sco, name):
    text = OBJS[name]()
    v, f, t = mpm.Mesh.from_text(text).arrays()
    ov, of = sco.parse_obj(text)
    assert np.array_equal(v, ov) and np.array_equal(f, of)
    assert np.array_equal(t.reshape(-1, 3, 3), ov[of])


def test_obj_numbers(mpm, sco):
    vals = ["1", "-2.5", ".5", "-.25", "+7", "1e3", "1.5E-2", "3.14159265358979", "0.000001", "12abc",
            "123456789.123456789", "-0.0", "2.5e+1", "7E0", "0.1234567891234"]
    text = "".join(f"v {a} {b} 0\n" for a, b in zip(vals, vals[1:] + vals[:1]))
    v, _, _ = mpm.Mesh.from_text(text).arrays()
    ov, _ = sco.parse_obj(text)
    assert np.array_equal(v.view(np.uint32), ov.view(np.uint32))
    nice = [float(x) for x in vals if x != "12abc"]
    got = [float(a) for a, s in zip(v[:, 0], vals) if s != "12abc"]
    assert np.allclose(got, np.float32(nice), rtol=0, atol=0)
    assert v[vals.index("12abc"), 0] == 12.0
    # unparsable and missing fields read 0
    w, _, _ = mpm.Mesh.from_text("v x 1\n").arrays()
    assert np.array_equal(w, [[0, 1, 0]])


def test_quad_diagonal_rule(mpm):
    # |v2 - v0| < |v3 - v1|: [0,1,2], [0,2,3]; otherwise [0,1,3], [1,2,3]
    short02 = "v 0 0 0\nv 10 0 0\nv 1 1 0\nv 0 10 0\nf 1 2 3 4\n"
    long02 = "v 0 0 0\nv 1 0 0\nv 10 10 0\nv 0 1 0\nf 1 2 3 4\n"
    assert mpm.Mesh.from_text(short02).arrays()[1].tolist() == [[0, 1, 2], [0, 2, 3]]
    assert mpm.Mesh.from_text(long02).arrays()[1].tolist() == [[0, 1, 3], [1, 2, 3]]
    pent = "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0.5 2 0\nv 0 1 0\nf 1 2 3 4 5\nf 1 2\n"
    assert mpm.Mesh.from_text(pent).arrays()[1].tolist() == [[0, 1, 2], [0, 2, 3], [0, 3, 4]]


def test_obj_errors(mpm, tmp_path):
    for bad in ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 0\n", "v 0 0 0\nf 1 2 3\n", "v 0 0 0\nf 1/0/1 1 1\n"):
        with pytest.raises(mpm.MpmError) as ei:
            mpm.Mesh.from_text(bad)
        assert ei.value.name == "MPM_ERR_BAD_CONFIG"
    with pytest.raises(mpm.MpmError) as ei:
        mpm.Mesh.load(str(tmp_path / "missing.obj"))
    assert ei.value.name == "MPM_ERR_IO"
    p = tmp_path / "ok.obj"
    p.write_text(objgen.box())
    assert mpm.Mesh.load(str(p)).arrays()[1].shape == (12, 3)


@pytest.mark.parametrize("case", [(128.0, 66.0, (16.0, -34.0, 0.0)), (64.0, 30.0, (0.0, 0.0, 0.0)),
                                  (128.0, 200.0, (90.0, 10.0, -50.0))])
def test_triangle_normalize_matches_oracle(mpm, sco, case):
    size, scale, disp = case
    _, _, t = mpm.Mesh.from_text(objgen.torus(25.0, 8.0, 48, 24)).arrays()
    got = mpm.normalize_triangles(t, size, scale, disp)
    want = sco.normalize_triangles(t, size, scale, disp)
    assert got.shape == want.shape and np.array_equal(got, want)
    if case[2][0] == 90.0:
        assert 0 < len(got) < len(t)  # some culled, some kept


def test_triangle_normalize_known_answer(mpm):
    _, _, t = mpm.Mesh.from_text(objgen.box()).arrays()
    got = mpm.normalize_triangles(t, 64.0, 32.0, (1.0, 2.0, 3.0)).reshape(-1, 3)
    # unit cube -> [0, 64]^3 -> longest side 32 about 32 -> [16, 48] -> + displacement
    assert set(np.unique(got[:, 0])) == {17.0, 49.0}
    assert set(np.unique(got[:, 1])) == {18.0, 50.0}
    assert set(np.unique(got[:, 2])) == {19.0, 51.0}
    # a degenerate (point) mesh is left untouched
    pt = np.ones((2, 9), np.float32)
    assert np.array_equal(mpm.normalize_triangles(pt, 64.0, 5.0, (9.0, 9.0, 9.0)), pt)


def test_oracle_normalize_known_answers(sco):
    # one point: zero size, returned as is (VoxelEngine.cpp:280-284)
    assert np.array_equal(sco.normalize(np.array([[1.5, 2.5, 3.5]]), 64.0, 8.0, (0, 0, 0), 1), [[1.5, 2.5, 3.5]])
    # two points 2 apart on x: -> x in {28, 36}, y = z = 32, then 5^3 dilation each
    out = sco.normalize(np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]]), 64.0, 8.0, (0, 0, 0), 1)
    xs = set(range(26, 31)) | set(range(34, 39))
    want = sorted((x, y, z) for x in xs for y in range(30, 35) for z in range(30, 35))
    assert out.tolist() == [list(map(float, w)) for w in want]
    with pytest.raises(ValueError):
        sco.normalize(np.zeros((3, 3)), 64.0, 8.0, (0, 0, 0), 0)


def test_oracle_voxelize_known_answer(sco):
    # box [0,100]^3: voxel size 1; the faces at 0 fill the slabs x = 0, y = 0,
    # z = 0, while the faces at 100 have an empty index range (floor(100) = 100
    # > 99): 100^3 - 99^3 voxels.
    v, f = sco.parse_obj(objgen.box((0.0, 0.0, 0.0), (100.0, 100.0, 100.0)))
    vox = sco.voxelize(v, f, 100.0)
    assert len(vox) == 100 ** 3 - 99 ** 3
    idx = (vox - 0.5).astype(int)
    assert ((idx == 0).any(1)).all()
    # z, y, x order
    key = (idx[:, 2] * 100 + idx[:, 1]) * 100 + idx[:, 0]
    assert (np.diff(key) > 0).all()

"""The numpy restatement of the obstacle pass (shaders/dot.vert + dot.frag,
renderer.cpp:247-303) against hand-derived answers, on the CPU: it is the
checker of the library's obstacle rasteriser."""
import numpy as np


def _square(grid, half, z):
    """Two triangles forming a square facing the camera, centred on the
    camera axis at depth z (grid coordinates)."""
    cx, cy = grid[0] / 2.0, grid[1] / 2.0
    a, b, c, d = (cx - half, cy - half, z), (cx + half, cy - half, z), (cx + half, cy + half, z), (cx - half, cy + half, z)
    return np.array([a + b + c, a + c + d], np.float32)


def test_square_facing_the_camera():
    from oracle import render_oracle as ro
    grid, w, h = (32, 32, 32), 128, 128
    tris = _square(grid, 4.0, 16.0)
    bg, depth = ro.obstacles(tris, w, h, grid)
    # The camera sits at z = 64 looking at the grid centre: the square at
    # view distance 48 spans 8 / (2 * 48 * tan 22.5 deg) of the image height.
    side_px = 8.0 / (2 * 48.0 * np.tan(np.radians(22.5))) * h
    cov = depth < 1.0
    assert abs(cov.sum() - side_px ** 2) <= 4 * side_px + 4
    ys, xs = np.nonzero(cov)
    assert abs(xs.mean() - 63.5) < 0.6 and abs(ys.mean() - 63.5) < 0.6
    # no pixel on the shared diagonal is drawn twice or left out: the
    # covered region is a solid square
    assert cov.sum() == (xs.max() - xs.min() + 1) * (ys.max() - ys.min() + 1)
    # flat colour: n = +z, L = (0.2, 10, 0.5) / |.|: 0.15 + 0.5 * 0.5 / 10.0142
    want = int(np.floor((0.15 + 0.5 * 0.5 / np.linalg.norm([0.2, 10.0, 0.5])) * 255 + 0.5))
    assert (bg[cov] == want).all()
    assert (bg[~cov] == [217, 230, 242]).all()
    # window depth of a point at view distance 48 (near 0.1, far 5000)
    n, f = 0.1, 5000.0
    zw = ((-(f + n) / (f - n)) * -48.0 - 2 * f * n / (f - n)) / 48.0 * 0.5 + 0.5
    assert np.allclose(depth[cov], zw, atol=1e-6)


def test_nearer_triangle_wins_and_back_faces_are_drawn():
    from oracle import render_oracle as ro
    grid, w, h = (32, 32, 32), 96, 96
    far = _square(grid, 6.0, 10.0)
    near = _square(grid, 3.0, 20.0)[:, [0, 1, 2, 6, 7, 8, 3, 4, 5]]  # reversed winding: a back face
    bg1, d1 = ro.obstacles(np.concatenate([far, near]), w, h, grid)
    bg2, d2 = ro.obstacles(np.concatenate([near, far]), w, h, grid)
    assert np.array_equal(d1, d2) and np.array_equal(bg1, bg2)  # the depth test, not the order
    c = (d1 < 1.0)
    assert d1[h // 2, w // 2] < d1[c].max()  # the centre holds the nearer square

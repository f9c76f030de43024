"""TEST INFRASTRUCTURE: numpy restatement of the reference's screen-space
fluid passes, the checker of the library's mpm_render_* kernels.

  camera     renderer.cpp:95-96, 186-197 (glm::lookAt, perspective, the model
             rotation about the grid centre, the view-space light direction)
  splat      shaders/ssf_depth.vert + ssf_depth.frag: point sprites of
             radius * 1000 / |view pos| pixels, sphere-surface view depth,
             nearest fragment kept, 99999 where nothing is drawn
  blur       shaders/ssf_blur.frag, horizontal then vertical, wrapping
             texture coordinates (GL_REPEAT)
  composite  shaders/screen.frag: normal from depth differences, refracted
             background (bilinear, wrapping), Fresnel, specular; depth-tested
             against the obstacles (gl_FragDepth)
  obstacles  shaders/dot.vert + dot.frag, the default opaque mode
             (renderer.cpp:247-303): triangles rasterised at pixel centres
             (top-left rule), depth test GL_LESS from 1, flat Lambert colour
             0.3 C + max(n . L, 0) C with n the plane normal towards the eye,
             8-bit framebuffer

Arrays are (height, width[, 3]) with row 0 at the bottom (GL window
coordinates), float32 throughout like the shaders.

Parity: the reference renders through OpenGL, which this pool cannot run
(no graphics stack), so these passes are pinned by hand-derived answers in
tests/test_gpu_render.py, not by images of the reference.
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32


def camera(width, height, grid, zoom=None, rotation=0.0, rotation_vertical=0.0, fov=45.0, near=0.1, far=5000.0,
           light=(0.2, 10.0, 0.5)):
    """Model-view (4x4, applied to column vectors), p00, p11, view-space light."""
    cx, cy, cz = grid[0] / 2.0, grid[1] / 2.0, grid[2] / 2.0
    zoom = grid[2] * 2.0 if zoom is None else zoom
    eye = np.array([cx, cy, zoom])
    f = np.array([cx, cy, cz]) - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, [0.0, 1.0, 0.0])
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    view = np.eye(4)
    view[0, :3], view[1, :3], view[2, :3] = s, u, -f
    view[0, 3], view[1, 3], view[2, 3] = -s @ eye, -u @ eye, f @ eye

    def rot(a, axis):
        c, sn = math.cos(a), math.sin(a)
        x, y, z = axis
        return np.array([[c + (1 - c) * x * x, (1 - c) * x * y - sn * z, (1 - c) * x * z + sn * y, 0],
                         [(1 - c) * y * x + sn * z, c + (1 - c) * y * y, (1 - c) * y * z - sn * x, 0],
                         [(1 - c) * z * x - sn * y, (1 - c) * z * y + sn * x, c + (1 - c) * z * z, 0],
                         [0, 0, 0, 1.0]])

    def tr(x, y, z):
        m = np.eye(4)
        m[:3, 3] = (x, y, z)
        return m

    model = tr(cx, cy, cz) @ rot(rotation_vertical, (1, 0, 0)) @ rot(rotation, (0, 1, 0)) @ tr(-cx, -cy, -cz)
    mv = (view @ model).astype(F)
    fy = 1.0 / math.tan(math.radians(fov) / 2.0)
    L = np.array(light) / np.linalg.norm(light)
    lv = (view[:3, :3] @ L).astype(F)
    return mv, F(fy / (width / height)), F(fy), lv, F(near), F(far)


def _model(grid, rotation=0.0, rotation_vertical=0.0):
    cx, cy, cz = grid[0] / 2.0, grid[1] / 2.0, grid[2] / 2.0

    def rot(a, axis):
        c, sn = math.cos(a), math.sin(a)
        x, y, z = axis
        return np.array([[c + (1 - c) * x * x, (1 - c) * x * y - sn * z, (1 - c) * x * z + sn * y, 0],
                         [(1 - c) * y * x + sn * z, c + (1 - c) * y * y, (1 - c) * y * z - sn * x, 0],
                         [(1 - c) * z * x - sn * y, (1 - c) * z * y + sn * x, c + (1 - c) * z * z, 0],
                         [0, 0, 0, 1.0]])

    def tr(x, y, z):
        m = np.eye(4)
        m[:3, 3] = (x, y, z)
        return m

    return tr(cx, cy, cz) @ rot(rotation_vertical, (1, 0, 0)) @ rot(rotation, (0, 1, 0)) @ tr(-cx, -cy, -cz)


def _unorm8(v):
    return np.floor(np.clip(np.asarray(v, F), 0, 1) * F(255) + F(0.5)).astype(np.uint8)


def obstacles(tris, width, height, grid, zoom=None, rotation=0.0, rotation_vertical=0.0, fov=45.0, near=0.1,
              far=5000.0, light=(0.2, 10.0, 0.5), color=(0.5, 0.5, 0.5), clear=(0.85, 0.9, 0.95), background=None):
    """The framebuffer after the obstacle pass: (RGB8 (h, w, 3), window depth (h, w), 1 where empty)."""
    mv, p00, p11, _, near32, far32 = camera(width, height, grid, zoom, rotation, rotation_vertical, fov, near, far,
                                            light)
    p22 = F(-(far + near) / (far - near))
    p32 = F(-(2.0 * far * near) / (far - near))
    model = _model(grid, rotation, rotation_vertical)
    zoom = grid[2] * 2.0 if zoom is None else zoom
    eye = np.array([grid[0] / 2.0, grid[1] / 2.0, zoom])
    L = np.array(light) / np.linalg.norm(light)
    col = np.array(color, np.float64)
    if background is None:
        bg = np.broadcast_to(_unorm8(clear), (height, width, 3)).copy()
    else:
        bg = np.asarray(background, np.uint8).reshape(height, width, 3).copy()
    depth = np.ones((height, width), F)
    t = np.asarray(tris, F).reshape(-1, 9)
    for i in range(len(t)):
        V = t[i].reshape(3, 3)
        X, Y, Z = np.zeros(3, F), np.zeros(3, F), np.zeros(3, F)
        ok = True
        for k in range(3):
            x, y, z = V[k]
            vx = ((mv[0, 0] * x + mv[0, 1] * y) + mv[0, 2] * z) + mv[0, 3]
            vy = ((mv[1, 0] * x + mv[1, 1] * y) + mv[1, 2] * z) + mv[1, 3]
            vz = ((mv[2, 0] * x + mv[2, 1] * y) + mv[2, 2] * z) + mv[2, 3]
            wc = -vz
            if not wc > near32:
                ok = False
                break
            X[k] = (p00 * vx / wc * F(0.5) + F(0.5)) * F(width)
            Y[k] = (p11 * vy / wc * F(0.5) + F(0.5)) * F(height)
            Z[k] = (p22 * vz + p32) / wc * F(0.5) + F(0.5)
        if not ok:
            continue
        area = (X[1] - X[0]) * (Y[2] - Y[0]) - (X[2] - X[0]) * (Y[1] - Y[0])
        if area == 0 or not np.isfinite(area):
            continue
        sgn = F(1) if area > 0 else F(-1)
        area = area * sgn
        x0 = max(0, int(math.ceil(float(X.min()) - 0.5)))
        x1 = min(width - 1, int(math.floor(float(X.max()) - 0.5)))
        y0 = max(0, int(math.ceil(float(Y.min()) - 0.5)))
        y1 = min(height - 1, int(math.floor(float(Y.max()) - 0.5)))
        if x0 > x1 or y0 > y1:
            continue
        sx = (np.arange(x0, x1 + 1).astype(F) + F(0.5))[None, :]
        sy = (np.arange(y0, y1 + 1).astype(F) + F(0.5))[:, None]
        inside = np.ones((y1 - y0 + 1, x1 - x0 + 1), bool)
        e = []
        for k in range(3):
            a, b = (k + 1) % 3, (k + 2) % 3
            ek = ((X[b] - X[a]) * (sy - Y[a]) - (Y[b] - Y[a]) * (sx - X[a])) * sgn
            ex, ey = (X[b] - X[a]) * sgn, (Y[b] - Y[a]) * sgn
            tl = (ey == 0 and ex < 0) or ey < 0
            inside &= (ek > 0) | ((ek == 0) & tl)
            e.append(ek)
        zw = ((e[0] * Z[0] + e[1] * Z[1]) + e[2] * Z[2]) / area
        sub = depth[y0:y1 + 1, x0:x1 + 1]
        win = inside & (zw >= 0) & (zw <= 1) & (zw < sub)
        # flat colour: the plane normal in the model-rotated frame, towards the eye
        W = (model[:3, :3] @ V.astype(np.float64).T).T + model[:3, 3]
        n = np.cross(W[1] - W[0], W[2] - W[0])
        if np.linalg.norm(n) > 0:
            n = n / np.linalg.norm(n)
        if n @ (eye - W[0]) < 0:
            n = -n
        c8 = _unorm8(0.3 * col + max(float(n @ L), 0.0) * col)
        sub[win] = zw[win]
        bg[y0:y1 + 1, x0:x1 + 1][win] = c8
    return bg, depth


def splat(xyz, width, height, cam, radius=2.0):
    mv, p00, p11, _, near, far = cam
    radius = F(radius)
    p = np.asarray(xyz, F)
    # row r of the view position: m[r][0] x + m[r][1] y + m[r][2] z + m[r][3],
    # summed left to right in float32 (the kernel's order, no fused multiply-add)
    v = np.stack([((mv[r, 0] * p[:, 0] + mv[r, 1] * p[:, 1]) + mv[r, 2] * p[:, 2]) + mv[r, 3] for r in range(3)], 1)
    best = np.full((height, width), -np.inf, F)
    for (vx, vy, vz) in v:
        w = -vz
        if not (near < w < far):
            continue
        nx, ny = p00 * vx / w, p11 * vy / w
        if not (-1 <= nx <= 1 and -1 <= ny <= 1):
            continue
        size = radius * (F(1000.0) / np.sqrt(vx * vx + vy * vy + vz * vz))
        cx, cy = (nx * F(0.5) + F(0.5)) * F(width), (ny * F(0.5) + F(0.5)) * F(height)
        x0, y0 = cx - F(0.5) * size, cy - F(0.5) * size
        px = np.arange(max(0, int(math.ceil(x0 - 0.5))), min(width - 1, int(math.ceil(x0 + size - 0.5)) - 1) + 1)
        py = np.arange(max(0, int(math.ceil(y0 - 0.5))), min(height - 1, int(math.ceil(y0 + size - 0.5)) - 1) + 1)
        if not len(px) or not len(py):
            continue
        s = ((px.astype(F) + F(0.5)) - x0) / size
        t = F(1.0) - ((py.astype(F) + F(0.5)) - y0) / size
        nx2 = s * F(2) - F(1)
        ny2 = t * F(2) - F(1)
        r2 = ny2[:, None] * ny2[:, None] + nx2[None, :] * nx2[None, :]
        ok = r2 <= 1
        zz = vz + np.sqrt(np.maximum(F(1) - r2, F(0))) * radius
        sub = best[py[0]:py[-1] + 1, px[0]:px[-1] + 1]
        np.maximum(sub, np.where(ok, zz, -np.inf).astype(F), out=sub)
    return np.where(np.isfinite(best), best, F(99999.0)).astype(F)


def blur(depth, axis, filter_size=10.0, falloff=0.01):
    """One bilateral pass; axis 1 = horizontal, 0 = vertical."""
    d = np.asarray(depth, F)
    fs, fo = F(filter_size), F(falloff)
    s = np.zeros_like(d)
    ws = np.zeros_like(d)
    i = -fs
    while i <= fs:
        k = int(i)
        smp = np.roll(d, -k, axis=axis)
        r = i * F(1.0) / fs
        w = np.exp(-r * r).astype(F)
        r2 = (smp - d) * fo
        w = (w * np.exp(-r2 * r2)).astype(F)
        s += smp * w
        ws += w
        i += F(1)
    out = (s / ws).astype(F)
    return np.where(d > 5000, d, out)


def composite(depth, cam, background=None, clear=(0.85, 0.9, 0.95), obstacle_depth=None):
    _, p00, p11, L, near, far = cam
    h, w = depth.shape
    if background is None:
        q = np.floor(np.clip(np.array(clear, F), 0, 1) * F(255) + F(0.5)).astype(np.uint8)
        background = np.broadcast_to(q, (h, w, 3))
    bg = np.asarray(background, np.uint8).astype(F) / F(255)
    ys, xs = np.mgrid[0:h, 0:w]

    def pos(x, y):
        x, y = x % w, y % h
        d = depth[y, x]
        u = (x.astype(F) + F(0.5)) / F(w)
        v = (y.astype(F) + F(0.5)) / F(h)
        px = (u * F(2) - F(1)) / p00
        py = (v * F(2) - F(1)) / p11
        return np.stack([px * -d, py * -d, d], -1)

    pc, pr, pt = pos(xs, ys), pos(xs + 1, ys), pos(xs, ys + 1)
    n = np.cross(pr - pc, pt - pc).astype(F)
    n = (n / np.sqrt((n * n).sum(-1, keepdims=True))).astype(F)
    u = (xs.astype(F) + F(0.5)) / F(w) + n[..., 0] * F(0.05)
    v = (ys.astype(F) + F(0.5)) / F(h) + n[..., 1] * F(0.05)
    fx, fy = u * F(w) - F(0.5), v * F(h) - F(0.5)
    x0, y0 = np.floor(fx), np.floor(fy)
    ax, ay = (fx - x0)[..., None], (fy - y0)[..., None]
    x0, y0 = x0.astype(int) % w, y0.astype(int) % h
    x1, y1 = (x0 + 1) % w, (y0 + 1) % h
    b = (bg[y0, x0] * (1 - ax) + bg[y0, x1] * ax) * (1 - ay) + (bg[y1, x0] * (1 - ax) + bg[y1, x1] * ax) * ay
    ndl = (n * -L).sum(-1)
    rz = -L[2] - F(2) * ndl * n[..., 2]
    spec = np.power(np.maximum(rz, 0), F(128)).astype(F)
    fres = np.power(F(1) - np.maximum(n[..., 2], 0), F(4)).astype(F)
    a = (F(0.3) + fres * F(0.5))[..., None]
    water = np.array([0.1, 0.5, 0.8], F)
    col = b * (1 - a) + water * a + spec[..., None]
    keep = depth > 5000
    if obstacle_depth is not None:
        p22 = F(-(float(far) + float(near)) / (float(far) - float(near)))
        p32 = F(-(2.0 * float(far) * float(near)) / (float(far) - float(near)))
        with np.errstate(divide="ignore", invalid="ignore"):
            fz = ((p22 * depth + p32) / -depth) * F(0.5) + F(0.5)
        keep |= ~(fz < obstacle_depth)
    return np.where(keep[..., None], bg, col).astype(F)


def render(xyz, width, height, grid, **kw):
    cam = camera(width, height, grid, **{k: v for k, v in kw.items() if k in ("zoom", "rotation",
                                                                                  "rotation_vertical")})
    raw = splat(xyz, width, height, cam, kw.get("radius", 2.0))
    h1 = blur(raw, 1)
    fin = blur(h1, 0)
    return raw, h1, fin, composite(fin, cam)

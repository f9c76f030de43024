"""Procedural scenes: obstacle meshes, particle seeding and the standard configs.

The reference builds its particles by voxelizing WATER= OBJ files and its
obstacles from OBJECT= OBJ files (Simulation.cpp:19-36, VoxelEngine.cpp).
The workloads here are defined procedurally instead, seeded, so that the
engine, the CPU oracle and the reference engine receive identical inputs:

* meshes are closed, triangles only, wound counter-clockwise seen from
  outside, so the winding number is +1 inside and the SDF is negative there;
* particles fill a region one per RESOLUTION^3 sub-cell, jittered uniformly
  inside the sub-cell, and are packed in the 26-plane layout of
  VoxelPipeline::process (VoxelPipeline.cpp:5-33): positions, 21 zero
  planes (velocity, C, F), then ones for VOL and MASS.
"""
from __future__ import annotations

import numpy as np

from . import Config

# Physics of the benchmark configs (sphere drop, dam break, scale, batched).
BENCH_PHYSICS = dict(padding=3, gravity=-0.3, dt=0.1, gamma=7.0, compression=10.0,
                     resolution=0.5, substeps=4)


def pack_state(pos: np.ndarray) -> np.ndarray:
    """(n, 3) positions -> (26, n) float32 state as VoxelPipeline::process lays it out."""
    n = pos.shape[0]
    st = np.zeros((26, n), np.float32)
    st[0:3] = pos.T.astype(np.float32)
    st[24:26] = 1.0
    return st


def _jitter_cells(idx: np.ndarray, lo: np.ndarray, res: float, rng) -> np.ndarray:
    cells = lo[None, :] + idx.astype(np.float64) * res
    pos = (cells + rng.random(idx.shape) * res).astype(np.float32)
    # keep every particle strictly inside its sub-cell after rounding to float
    top = np.nextafter((cells + res).astype(np.float32), np.float32(-np.inf))
    return np.minimum(pos, top)


def seed_box(lo, hi, res: float, rng) -> np.ndarray:
    """One jittered particle per res-sized sub-cell of [lo, hi); x varies fastest."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    counts = np.floor((hi - lo) / res + 1e-9).astype(np.int64)
    zz, yy, xx = np.meshgrid(np.arange(counts[2]), np.arange(counts[1]), np.arange(counts[0]), indexing="ij")
    idx = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    return _jitter_cells(idx, lo, res, rng)


def seed_sphere(center, radius: float, res: float, rng) -> np.ndarray:
    """One jittered particle per sub-cell whose centre lies inside the sphere."""
    c = np.asarray(center, np.float64)
    lo = c - radius
    m = int(np.ceil(2 * radius / res)) + 1
    zz, yy, xx = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    idx = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    centres = lo[None, :] + (idx + 0.5) * res
    inside = np.sum((centres - c[None, :]) ** 2, axis=1) < radius * radius
    return _jitter_cells(idx[inside], lo, res, rng)


def uv_sphere(radius: float, center, seg_u: int = 32, seg_v: int = 16) -> np.ndarray:
    """Closed UV sphere: triangle fans at the poles, two triangles per band quad.
    32 x 16 segments give 960 triangles.  Returns (t, 9) float32."""
    c = np.asarray(center, np.float64)
    verts = [c + [0, radius, 0]]
    for i in range(1, seg_v):
        th = np.pi * i / seg_v
        for j in range(seg_u):
            ph = 2 * np.pi * j / seg_u
            verts.append(c + radius * np.array([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)]))
    verts.append(c + [0, -radius, 0])
    V = np.array(verts)
    top, bot = 0, len(verts) - 1
    ring = lambda i, j: 1 + (i - 1) * seg_u + (j % seg_u)
    tris = []
    for j in range(seg_u):
        tris.append((top, ring(1, j + 1), ring(1, j)))
    for i in range(1, seg_v - 1):
        for j in range(seg_u):
            a, b = ring(i, j), ring(i, j + 1)
            cc, d = ring(i + 1, j), ring(i + 1, j + 1)
            tris.append((a, b, d))
            tris.append((a, d, cc))
    for j in range(seg_u):
        tris.append((bot, ring(seg_v - 1, j), ring(seg_v - 1, j + 1)))
    return _orient_outward(V, np.array(tris))


def torus(major: float, minor: float, center, seg_major: int = 48, seg_minor: int = 24) -> np.ndarray:
    """Closed torus around the y axis: seg_major*seg_minor*2 triangles."""
    c = np.asarray(center, np.float64)
    V = np.zeros((seg_major, seg_minor, 3))
    for i in range(seg_major):
        u = 2 * np.pi * i / seg_major
        for j in range(seg_minor):
            v = 2 * np.pi * j / seg_minor
            rr = major + minor * np.cos(v)
            V[i, j] = c + [rr * np.cos(u), minor * np.sin(v), rr * np.sin(u)]
    V = V.reshape(-1, 3)
    k = lambda i, j: (i % seg_major) * seg_minor + (j % seg_minor)
    tris = []
    for i in range(seg_major):
        for j in range(seg_minor):
            a, b, cc, d = k(i, j), k(i + 1, j), k(i, j + 1), k(i + 1, j + 1)
            tris.append((a, b, d))
            tris.append((a, d, cc))
    return _orient_outward(V, np.array(tris), torus_axis=(c, major))


def box_mesh(extent, center) -> np.ndarray:
    """Closed axis-aligned box, 12 triangles."""
    c = np.asarray(center, np.float64)
    h = np.asarray(extent, np.float64) / 2
    V = np.array([[sx, sy, sz] for sz in (-1, 1) for sy in (-1, 1) for sx in (-1, 1)]) * h + c
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    tris = []
    for a, b, cc, d in quads:
        tris.append((a, b, cc))
        tris.append((a, cc, d))
    return _orient_outward(V, np.array(tris))


def _orient_outward(V: np.ndarray, T: np.ndarray, torus_axis=None) -> np.ndarray:
    """Flip triangles whose normal points toward the solid's interior."""
    A, B, Cc = V[T[:, 0]], V[T[:, 1]], V[T[:, 2]]
    nrm = np.cross(B - A, Cc - A)
    cen = (A + B + Cc) / 3
    if torus_axis is None:
        inner = V.mean(axis=0)[None, :]
    else:  # nearest point of the torus core circle
        c, major = torus_axis
        d = cen - c
        d[:, 1] = 0
        d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-12)
        inner = c + major * d
    flip = np.sum(nrm * (cen - inner), axis=1) < 0
    T = T.copy()
    T[flip] = T[flip][:, [0, 2, 1]]
    return np.concatenate([V[T[:, 0]], V[T[:, 1]], V[T[:, 2]]], axis=1).astype(np.float32)


def _cfg(size, **over) -> Config:
    d = dict(BENCH_PHYSICS)
    d.update(over)
    return Config(size_x=size[0], size_y=size[1], size_z=size[2], sdf_resolution=max(size), **d)


def sphere_drop(seed: int = 1234):
    """Sphere drop: radius-15 sphere of water centred at (32,40,32) in 64^3, no obstacle."""
    rng = np.random.default_rng(seed)
    cfg = _cfg((64, 64, 64))
    pos = seed_sphere((32.0, 40.0, 32.0), 15.0, cfg.resolution, rng)
    return cfg, pack_state(pos), np.zeros((0, 9), np.float32)


def dam_break(seed: int = 1235, literal_extent: bool = False):
    """Dam break with a torus obstacle in 128^3.

    Water box x in [4,60), y in [4,41), z in [4,124) at RESOLUTION 0.5:
    1,989,120 particles (the 2M headline case).  literal_extent=True uses
    y in [4,100): 5,160,960 particles.  Torus: major radius 25, minor 8,
    48 x 24 segments, centred at (80,30,64), axis y."""
    rng = np.random.default_rng(seed)
    cfg = _cfg((128, 128, 128))
    y_hi = 100.0 if literal_extent else 41.0
    pos = seed_box((4.0, 4.0, 4.0), (60.0, y_hi, 124.0), cfg.resolution, rng)
    tris = torus(25.0, 8.0, (80.0, 30.0, 64.0), 48, 24)
    return cfg, pack_state(pos), tris


def scale_scene(seed: int = 1236):
    """256^3: three water boxes with seeded extents in [40,90] per axis, and a
    sphere (r 30), a torus (50/12) and a box (60x20x60), each scaled by
    U[0.8,1.2] and placed at seeded positions."""
    rng = np.random.default_rng(seed)
    cfg = _cfg((256, 256, 256))
    parts = []
    for _ in range(3):
        ext = rng.uniform(40, 90, size=3)
        lo = rng.uniform(8, 248 - ext)
        parts.append(seed_box(lo, lo + ext, cfg.resolution, rng))
    pos = np.concatenate(parts)
    tris = []
    s = rng.uniform(0.8, 1.2, size=3)
    for k, make in enumerate((lambda c, f: uv_sphere(30 * f, c),
                              lambda c, f: torus(50 * f, 12 * f, c),
                              lambda c, f: box_mesh((60 * f, 20 * f, 60 * f), c))):
        c = rng.uniform(70, 186, size=3)
        tris.append(make(c, s[k]))
    return cfg, pack_state(pos), np.concatenate(tris)


def small_scene(n: int, size=(32, 32, 32), seed: int = 7, obstacle: bool = True, randomize: bool = True,
                **physics):
    """A small seeded scene for parity tests: n particles uniform in the
    interior, random velocity, C and F near the identity (so every term of the
    substep is exercised), and an optional sphere obstacle."""
    rng = np.random.default_rng(seed)
    cfg = _cfg(size, **physics)
    lo = np.array([3.0, 3.0, 3.0])
    hi = np.array(size, np.float64) - 3.0
    c = np.array(size, np.float64) / 2
    r = min(size) / 6
    pos = np.zeros((0, 3))
    while pos.shape[0] < n:
        cand = lo + rng.random((2 * n, 3)) * (hi - lo)
        if obstacle:
            # Water starts outside the obstacle: deep inside, the SDF gradient
            # vanishes (the centre node of a symmetric mesh) and the collision
            # normal is undefined.
            cand = cand[np.linalg.norm(cand - c, axis=1) > r + 1.5]
        pos = np.concatenate([pos, cand])
    pos = pos[:n].astype(np.float32)
    st = pack_state(pos)
    if randomize:
        st[3:6] = rng.normal(0, 1.0, (3, n))
        st[6:15] = rng.normal(0, 0.3, (9, n))
        F = np.eye(3).reshape(9, 1) + rng.normal(0, 0.05, (9, n))
        st[15:24] = F
    tris = np.zeros((0, 9), np.float32)
    if obstacle:
        tris = uv_sphere(r, c, 16, 8)
    return cfg, st.astype(np.float32), tris


def batched_scenes(count: int = 64, seed: int = 1237):
    """Independent scenes for the batched engine: grid size per axis uniform in
    [32, 96]; one water sphere whose particle count is log-uniform in
    [10k, 500k] (its radius, from 8 particles per cell, is clamped to
    0.2-0.4 of the smallest grid extent and the sphere kept 4 cells off the
    walls); 0-2 obstacles, a torus or a box, at seeded positions.  Returns a
    list of (cfg, state26, triangles)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        size = tuple(int(v) for v in rng.integers(32, 97, size=3))
        cfg = _cfg(size)
        ext = float(min(size))
        target = float(np.exp(rng.uniform(np.log(1e4), np.log(5e5))))
        r = (3.0 * target / (4.0 * np.pi * 8.0)) ** (1.0 / 3.0)
        r = float(np.clip(r, 0.2 * ext, 0.4 * ext))
        lo = np.array([4.0 + r] * 3)
        hi = np.array(size, np.float64) - 4.0 - r
        c = rng.uniform(lo, np.maximum(hi, lo))
        pos = seed_sphere(tuple(c), r, cfg.resolution, rng)
        tris = []
        for _k in range(int(rng.integers(0, 3))):
            oc = rng.uniform(0.2, 0.8, size=3) * np.array(size)
            s = float(rng.uniform(0.1, 0.2) * ext)
            if rng.random() < 0.5:
                tris.append(torus(s, s / 3.0, tuple(oc), 24, 12))
            else:
                tris.append(box_mesh((s, s / 2.0, s), tuple(oc)))
        t = np.concatenate(tris) if tris else np.zeros((0, 9), np.float32)
        out.append((cfg, pack_state(pos), t))
    return out

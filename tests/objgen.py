"""OBJ texts for the scene-construction tests, written procedurally: a
Blender-style UV sphere (quads with triangle fans at the poles), a torus of
quads with relative (negative) indices, and an axis-aligned box."""
import math


def _fmt(x):
    return f"{x:.6f}"


def uv_sphere(radius=1.0, nu=32, nv=16, center=(0.0, 0.0, 0.0), style="v"):
    """style: 'v', 'v/t/n' or 'v//n' face tokens."""
    cx, cy, cz = center
    lines = ["# uv sphere", "mtllib sphere.mtl", "o Sphere"]
    verts = [(cx, cy + radius, cz)]
    for i in range(1, nv):
        th = math.pi * i / nv
        for j in range(nu):
            ph = 2 * math.pi * j / nu
            verts.append((cx + radius * math.sin(th) * math.cos(ph), cy + radius * math.cos(th),
                          cz + radius * math.sin(th) * math.sin(ph)))
    verts.append((cx, cy - radius, cz))
    for v in verts:
        lines.append("v " + " ".join(_fmt(c) for c in v))
    lines.append("vt 0.5 0.5")
    lines.append("vn 0 1 0")
    tok = {"v": lambda i: f"{i}", "v/t/n": lambda i: f"{i}/1/1", "v//n": lambda i: f"{i}//1"}[style]
    ring = lambda i, j: 2 + (i - 1) * nu + (j % nu)  # 1-based
    lines.append("s 0")
    for j in range(nu):
        lines.append(f"f {tok(1)} {tok(ring(1, j + 1))} {tok(ring(1, j))}")
    for i in range(1, nv - 1):
        for j in range(nu):
            a, b, c, d = ring(i, j), ring(i, j + 1), ring(i + 1, j + 1), ring(i + 1, j)
            lines.append(f"f {tok(a)} {tok(b)} {tok(c)} {tok(d)}")
    last = len(verts)
    for j in range(nu):
        lines.append(f"f {tok(ring(nv - 1, j))} {tok(ring(nv - 1, j + 1))} {tok(last)}")
    return "\r\n".join(lines) + "\r\n"


def torus(major=1.0, minor=0.3, nu=24, nv=12):
    """Quads written with negative indices right after each ring pair."""
    lines = ["o Torus", "g ring"]
    rings = []
    for i in range(nu):
        u = 2 * math.pi * i / nu
        rings.append([((major + minor * math.cos(2 * math.pi * j / nv)) * math.cos(u),
                       minor * math.sin(2 * math.pi * j / nv),
                       (major + minor * math.cos(2 * math.pi * j / nv)) * math.sin(u)) for j in range(nv)])
    for ring in rings:
        for v in ring:
            lines.append("v  " + "\t".join(_fmt(c) for c in v) + " 1.0")
    total = nu * nv
    for i in range(nu):
        for j in range(nv):
            a = i * nv + j
            b = i * nv + (j + 1) % nv
            c = ((i + 1) % nu) * nv + (j + 1) % nv
            d = ((i + 1) % nu) * nv + j
            lines.append("f " + " ".join(str(k - total) for k in (a, b, c, d)))
    return "\n".join(lines) + "\n"


def box(lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = [(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0), (x0, y0, z1), (x1, y0, z1), (x1, y1, z1),
         (x0, y1, z1)]
    faces = [(1, 4, 3, 2), (5, 6, 7, 8), (1, 2, 6, 5), (2, 3, 7, 6), (3, 4, 8, 7), (4, 1, 5, 8)]
    lines = ["v " + " ".join(repr(float(c)) for c in p) for p in v]
    lines += ["f " + " ".join(map(str, f)) for f in faces]
    return "\n".join(lines) + "\n"

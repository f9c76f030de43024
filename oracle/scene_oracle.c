/*
 * TEST INFRASTRUCTURE: CPU restatement of the reference's scene construction
 * (OBJ -> particles and obstacle triangles), the checker of the library's
 * mpm_scene_* / mpm_voxelize / mpm_points_normalize / mpm_triangles_normalize.
 * Plain C, single-threaded, float arithmetic without contraction
 * (-ffp-contract=off), loops in the reference's order.
 *
 *   sco_parse_obj            ObjLoader::loadObj (tinyobjloader LoadObj with
 *                            triangulation) + VoxelEngine::extractTriangles
 *                            (VoxelEngine.cpp:860-898)
 *   sco_voxelize             VoxelEngine::voxelize (VoxelEngine.cpp:120-243),
 *                            triangleAABBIntersection (902-962),
 *                            calculateBoundingBox (829-858)
 *   sco_normalize            VoxelEngine::normalize(VoxelData&) (245-494):
 *                            the std::set of lattice points becomes a sorted,
 *                            de-duplicated array of (x, y, z) triples
 *   sco_normalize_triangles  VoxelEngine::normalize(std::vector<Triangle>&)
 *                            (601-827)
 *
 * Parity: the reference's scene code needs glm and tinyobjloader (vcpkg
 * packages that are not in the reference tree), so it cannot be compiled
 * here and there are no golden outputs of it; this restatement is checked
 * against hand-derived answers (tests/test_scene.py).
 */
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static float mins(float a, float b) { return (b < a) ? b : a; } /* std::min */
static float maxs(float a, float b) { return (a < b) ? b : a; } /* std::max */
static float min3(float a, float b, float c) { return mins(mins(a, b), c); }
static float max3(float a, float b, float c) { return maxs(maxs(a, b), c); }

void sco_free(void* p) { free(p); }

/* ---------------------------------------------------------------- OBJ ---- */
/* tinyobjloader's tryParseDouble scheme: integer digits accumulated as
 * m = 10 m + d in double, fraction digit k (k = 1, 2, ...) adds d * 10^-k
 * taken from a table for k < 8, exponent e applied as ldexp(m * 5^e, e). */
static int obj_number(const char* s, const char* e, double* out) {
    static const double tab[8] = {1.0, 0.1, 0.01, 0.001, 0.0001, 0.00001, 0.000001, 0.0000001};
    double m = 0.0;
    int ex = 0, neg = 0, eneg = 0, k = 0, frac_only = 0;
    const char* c = s;
    if (c >= e) return 0;
    if (*c == '+' || *c == '-') {
        neg = *c == '-';
        ++c;
        if (c < e && *c == '.') frac_only = 1;
    } else if (*c == '.') {
        frac_only = 1;
    } else if (!(*c >= '0' && *c <= '9')) {
        return 0;
    }
    if (!frac_only) {
        for (; c < e && *c >= '0' && *c <= '9'; ++c, ++k) m = m * 10 + (*c - '0');
        if (k == 0) return 0;
    }
    if (c < e && *c == '.') {
        ++c;
        for (k = 1; c < e && *c >= '0' && *c <= '9'; ++c, ++k) m += (*c - '0') * (k < 8 ? tab[k] : pow(10.0, -k));
    } else if (c < e && *c != 'e' && *c != 'E') {
        c = e; /* anything else ends the number */
    }
    if (c < e && (*c == 'e' || *c == 'E')) {
        ++c;
        if (c < e && (*c == '+' || *c == '-')) {
            eneg = *c == '-';
            ++c;
        } else if (!(c < e && *c >= '0' && *c <= '9')) {
            return 0;
        }
        for (k = 0; c < e && *c >= '0' && *c <= '9'; ++c, ++k) {
            if (ex > INT_MAX / 10) return 0;
            ex = ex * 10 + (*c - '0');
        }
        if (k == 0) return 0;
        if (eneg) ex = -ex;
    }
    *out = (neg ? -1 : 1) * (ex ? ldexp(m * pow(5.0, ex), ex) : m);
    return 1;
}

static float obj_real(const char** t) {
    const char* s = *t + strspn(*t, " \t");
    const char* e = s + strcspn(s, " \t\r");
    double v = 0.0;
    obj_number(s, e, &v);
    *t = e;
    return (float)v;
}

static int obj_index(long idx, long n, long* out) {
    if (idx == 0) return 0;
    *out = idx > 0 ? idx - 1 : n + idx;
    return 1;
}

typedef struct {
    float* v;
    long nv, cv;
    int* f;
    long nf, cf;
} Mesh;

static void push_v(Mesh* m, float x) {
    if (m->nv == m->cv) {
        m->cv = m->cv ? 2 * m->cv : 256;
        m->v = (float*)realloc(m->v, m->cv * sizeof(float));
    }
    m->v[m->nv++] = x;
}
static void push_f(Mesh* m, int i) {
    if (m->nf == m->cf) {
        m->cf = m->cf ? 2 * m->cf : 256;
        m->f = (int*)realloc(m->f, m->cf * sizeof(int));
    }
    m->f[m->nf++] = i;
}

/* Returns 0 on success, else the 1-based line number of the failure.
 * *v: 3 floats per vertex, *f: 3 vertex indices per triangle. */
long sco_parse_obj(const char* text, float** v, long* nv, int** f, long* nt) {
    Mesh m = {0};
    long nvt = 0, nvn = 0, line = 0;
    long face[4096];
    const char* p = text;
    while (*p) {
        const char* eol = p + strcspn(p, "\n");
        size_t len = (size_t)(eol - p);
        char* buf = (char*)malloc(len + 1);
        memcpy(buf, p, len);
        buf[len] = 0;
        while (len && (buf[len - 1] == '\r')) buf[--len] = 0;
        p = *eol ? eol + 1 : eol;
        ++line;
        const char* t = buf + strspn(buf, " \t");
        int sp1 = t[0] && (t[1] == ' ' || t[1] == '\t');
        if (t[0] == 'v' && sp1) {
            t += 2;
            float x = obj_real(&t), y = obj_real(&t), z = obj_real(&t);
            push_v(&m, x);
            push_v(&m, y);
            push_v(&m, z);
        } else if (t[0] == 'v' && (t[1] == 't' || t[1] == 'n') && (t[2] == ' ' || t[2] == '\t')) {
            if (t[1] == 't') ++nvt;
            else ++nvn;
        } else if (t[0] == 'f' && sp1) {
            long k = 0, n = m.nv / 3;
            t += 2;
            t += strspn(t, " \t");
            while (*t && *t != '\r') {
                long vi, dummy;
                if (!obj_index(strtol(t, NULL, 10), n, &vi) || vi < 0 || vi >= n || k >= 4096) goto bad;
                t += strcspn(t, "/ \t\r");
                if (*t == '/') {
                    ++t;
                    if (*t == '/') {
                        ++t;
                        if (!obj_index(strtol(t, NULL, 10), nvn, &dummy)) goto bad;
                        t += strcspn(t, "/ \t\r");
                    } else {
                        if (!obj_index(strtol(t, NULL, 10), nvt, &dummy)) goto bad;
                        t += strcspn(t, "/ \t\r");
                        if (*t == '/') {
                            ++t;
                            if (!obj_index(strtol(t, NULL, 10), nvn, &dummy)) goto bad;
                            t += strcspn(t, "/ \t\r");
                        }
                    }
                }
                face[k++] = vi;
                t += strspn(t, " \t\r");
            }
            if (k == 4) {
                const float *a = m.v + 3 * face[0], *b = m.v + 3 * face[1], *c = m.v + 3 * face[2],
                            *d = m.v + 3 * face[3];
                float ex = c[0] - a[0], ey = c[1] - a[1], ez = c[2] - a[2];
                float gx = d[0] - b[0], gy = d[1] - b[1], gz = d[2] - b[2];
                float s02 = ex * ex + ey * ey + ez * ez, s13 = gx * gx + gy * gy + gz * gz;
                if (s02 < s13) {
                    push_f(&m, face[0]), push_f(&m, face[1]), push_f(&m, face[2]);
                    push_f(&m, face[0]), push_f(&m, face[2]), push_f(&m, face[3]);
                } else {
                    push_f(&m, face[0]), push_f(&m, face[1]), push_f(&m, face[3]);
                    push_f(&m, face[1]), push_f(&m, face[2]), push_f(&m, face[3]);
                }
            } else if (k >= 3) {
                for (long i = 2; i < k; ++i) push_f(&m, face[0]), push_f(&m, face[i - 1]), push_f(&m, face[i]);
            }
        }
        free(buf);
        continue;
    bad:
        free(buf);
        free(m.v);
        free(m.f);
        return line;
    }
    *v = m.v;
    *nv = m.nv / 3;
    *f = m.f;
    *nt = m.nf / 3;
    return 0;
}

/* ------------------------------------------------------- voxelization ---- */
static float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static int tri_aabb(const float* t0, const float* t1, const float* t2, const float* bmin, const float* bmax) {
    float c[3], h[3], v0[3], v1[3], v2[3], e0[3], e1[3], e2[3], axes[9][3];
    for (int i = 0; i < 3; ++i) {
        c[i] = (bmin[i] + bmax[i]) * 0.5f;
        h[i] = (bmax[i] - bmin[i]) * 0.5f;
    }
    for (int i = 0; i < 3; ++i) {
        v0[i] = t0[i] - c[i];
        v1[i] = t1[i] - c[i];
        v2[i] = t2[i] - c[i];
    }
    for (int i = 0; i < 3; ++i) {
        e0[i] = v1[i] - v0[i];
        e1[i] = v2[i] - v1[i];
        e2[i] = v0[i] - v2[i];
    }
    const float* es[3] = {e0, e1, e2};
    for (int k = 0; k < 3; ++k) {
        const float* e = es[k];
        axes[3 * k][0] = 0, axes[3 * k][1] = -e[2], axes[3 * k][2] = e[1];
        axes[3 * k + 1][0] = e[2], axes[3 * k + 1][1] = 0, axes[3 * k + 1][2] = -e[0];
        axes[3 * k + 2][0] = -e[1], axes[3 * k + 2][1] = e[0], axes[3 * k + 2][2] = 0;
    }
    for (int i = 0; i < 9; ++i) {
        float p0 = dot3(v0, axes[i]), p1 = dot3(v1, axes[i]), p2 = dot3(v2, axes[i]);
        float r = h[0] * fabsf(axes[i][0]) + h[1] * fabsf(axes[i][1]) + h[2] * fabsf(axes[i][2]);
        if (maxs(-max3(p0, p1, p2), min3(p0, p1, p2)) > r) return 0;
    }
    for (int i = 0; i < 3; ++i)
        if (max3(v0[i], v1[i], v2[i]) < -h[i] || min3(v0[i], v1[i], v2[i]) > h[i]) return 0;
    float n[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0]};
    float d = dot3(n, v0);
    float r = h[0] * fabsf(n[0]) + h[1] * fabsf(n[1]) + h[2] * fabsf(n[2]);
    return !(fabsf(d) > r);
}

/* Voxel centres (x y z per voxel) in z, y, x order; returns the count or -1. */
long sco_voxelize(const float* v, long nv, const int* f, long nt, float resolution, float** out) {
    *out = NULL;
    if (nv <= 0) return -1;
    float mn[3] = {v[0], v[1], v[2]}, mx[3] = {v[0], v[1], v[2]};
    for (long i = 0; i < nv; ++i)
        for (int c = 0; c < 3; ++c) {
            mn[c] = mins(mn[c], v[3 * i + c]);
            mx[c] = maxs(mx[c], v[3 * i + c]);
        }
    float sx = mx[0] - mn[0], sy = mx[1] - mn[1], sz = mx[2] - mn[2];
    float maxsize = maxs(sx, maxs(sy, sz));
    float res = maxsize / resolution;
    if (!(res > 0.0f)) return -1;
    int g[3];
    for (int c = 0; c < 3; ++c) g[c] = (int)ceilf((mx[c] - mn[c]) / res);
    long total = (long)g[0] * g[1] * g[2];
    unsigned char* filled = (unsigned char*)calloc(total > 0 ? total : 1, 1);
    for (long t = 0; t < nt; ++t) {
        const float *a = v + 3 * f[3 * t], *b = v + 3 * f[3 * t + 1], *c = v + 3 * f[3 * t + 2];
        int lo[3], hi[3];
        for (int k = 0; k < 3; ++k) {
            float tmin = min3(a[k], b[k], c[k]), tmax = max3(a[k], b[k], c[k]);
            int l = (int)floorf((tmin - mn[k]) / res), h = (int)ceilf((tmax - mn[k]) / res);
            lo[k] = l > 0 ? l : 0;
            hi[k] = h < g[k] - 1 ? h : g[k] - 1;
        }
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int x = lo[0]; x <= hi[0]; ++x) {
                    float bmin[3] = {mn[0] + x * res, mn[1] + y * res, mn[2] + z * res};
                    float bmax[3] = {bmin[0] + res, bmin[1] + res, bmin[2] + res};
                    if (tri_aabb(a, b, c, bmin, bmax)) filled[((long)z * g[1] + y) * g[0] + x] = 1;
                }
    }
    long count = 0;
    for (long i = 0; i < total; ++i) count += filled[i];
    float* o = (float*)malloc((count > 0 ? count : 1) * 3 * sizeof(float));
    long k = 0;
    for (int z = 0; z < g[2]; ++z)
        for (int y = 0; y < g[1]; ++y)
            for (int x = 0; x < g[0]; ++x)
                if (filled[((long)z * g[1] + y) * g[0] + x]) {
                    o[3 * k] = mn[0] + (x + 0.5f) * res;
                    o[3 * k + 1] = mn[1] + (y + 0.5f) * res;
                    o[3 * k + 2] = mn[2] + (z + 0.5f) * res;
                    ++k;
                }
    free(filled);
    *out = o;
    return count;
}

/* ---------------------------------------------------------- normalize ---- */
static int cmp_triple(const void* a, const void* b) {
    const int* x = (const int*)a;
    const int* y = (const int*)b;
    for (int i = 0; i < 3; ++i)
        if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
    return 0;
}

static void bounds(const float* p, long n, float* lo, float* hi) {
    for (int c = 0; c < 3; ++c) lo[c] = hi[c] = p[c];
    for (long i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            lo[c] = mins(lo[c], p[3 * i + c]);
            hi[c] = maxs(hi[c], p[3 * i + c]);
        }
}

/* In: n points (x y z each).  Out: the normalised, snapped, dilated points
 * (malloc'd, sorted like std::set<std::tuple<int,int,int>>); returns their
 * count, or -1 for step < 1. */
long sco_normalize(const float* in, long n, float size, float scale, const float* disp, int step, float** out) {
    *out = NULL;
    if (n <= 0) return 0;
    if (step < 1) return -1;
    float* p = (float*)malloc(3 * n * sizeof(float));
    memcpy(p, in, 3 * n * sizeof(float));
    float lo[3], hi[3];
    bounds(p, n, lo, hi);
    float maxdim = max3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    if (maxdim < 1e-6f) {
        *out = p;
        return n;
    }
    float ns = size / maxdim;
    float ctr[3] = {(lo[0] + hi[0]) * 0.5f, (lo[1] + hi[1]) * 0.5f, (lo[2] + hi[2]) * 0.5f};
    for (long i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            p[3 * i + c] -= ctr[c];
            p[3 * i + c] *= ns;
            p[3 * i + c] += size * 0.5f;
        }
    bounds(p, n, lo, hi);
    float cur = max3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    float s2 = (cur > 1e-6f) ? (scale / cur) : 1.0f;
    float half = size * 0.5f;
    for (long i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            p[3 * i + c] -= half;
            p[3 * i + c] *= s2;
            p[3 * i + c] += half;
        }
    for (long i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) p[3 * i + c] += disp[c];
    float gres = (float)step;
    int M = (int)(size / gres);
    int* tr = (int*)malloc(125 * 3 * n * sizeof(int));
    long k = 0;
    for (long i = 0; i < n; ++i) {
        int g[3];
        for (int c = 0; c < 3; ++c) {
            int q = (int)roundf(p[3 * i + c] / gres);
            g[c] = q < 0 ? 0 : (q > M ? M : q);
        }
        for (int a = -2; a <= 2; ++a)
            for (int b = -2; b <= 2; ++b)
                for (int c = -2; c <= 2; ++c) {
                    int x = g[0] + a, y = g[1] + b, z = g[2] + c;
                    if (x < 0 || x > M || y < 0 || y > M || z < 0 || z > M) continue;
                    tr[3 * k] = x, tr[3 * k + 1] = y, tr[3 * k + 2] = z;
                    ++k;
                }
    }
    qsort(tr, k, 3 * sizeof(int), cmp_triple);
    long u = 0;
    for (long i = 0; i < k; ++i)
        if (u == 0 || cmp_triple(tr + 3 * i, tr + 3 * (u - 1)) != 0) {
            memmove(tr + 3 * u, tr + 3 * i, 3 * sizeof(int));
            ++u;
        }
    float* o = (float*)malloc((u > 0 ? u : 1) * 3 * sizeof(float));
    for (long i = 0; i < u; ++i)
        for (int c = 0; c < 3; ++c) o[3 * i + c] = tr[3 * i + c] * gres;
    free(tr);
    free(p);
    *out = o;
    return u;
}

/* In place on 9 floats per triangle; returns the number kept. */
long sco_normalize_triangles(float* t, long nt, float size, float scale, const float* disp) {
    if (nt <= 0) return nt;
    float lo[3], hi[3];
    bounds(t, nt * 3, lo, hi);
    float maxdim = max3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    if (maxdim < 1e-6f) return nt;
    float ns = size / maxdim;
    float ctr[3] = {(lo[0] + hi[0]) * 0.5f, (lo[1] + hi[1]) * 0.5f, (lo[2] + hi[2]) * 0.5f};
    for (long i = 0; i < nt * 3; ++i)
        for (int c = 0; c < 3; ++c) {
            t[3 * i + c] -= ctr[c];
            t[3 * i + c] *= ns;
            t[3 * i + c] += size * 0.5f;
        }
    bounds(t, nt * 3, lo, hi);
    float cur = max3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    float s2 = (cur > 1e-6f) ? (scale / cur) : 1.0f;
    float half = size * 0.5f;
    for (long i = 0; i < nt * 3; ++i)
        for (int c = 0; c < 3; ++c) {
            t[3 * i + c] -= half;
            t[3 * i + c] *= s2;
            t[3 * i + c] += half;
        }
    for (long i = 0; i < nt * 3; ++i)
        for (int c = 0; c < 3; ++c) t[3 * i + c] += disp[c];
    long k = 0;
    for (long i = 0; i < nt; ++i) {
        const float* q = t + 9 * i;
        int any = 0;
        for (int j = 0; j < 3; ++j) {
            const float* v = q + 3 * j;
            if (v[0] >= 0.0f && v[0] <= size && v[1] >= 0.0f && v[1] <= size && v[2] >= 0.0f && v[2] <= size) any = 1;
        }
        if (any) {
            memmove(t + 9 * k, q, 9 * sizeof(float));
            ++k;
        }
    }
    return k;
}

/*
 * mpm_oracle.c - CPU restatement of the reference MLS-MPM substep and SDF
 * build.  TEST INFRASTRUCTURE ONLY: the parity tests use it as the checker
 * and the benchmark times its FP32 build as the CPU baseline.  No product
 * code path links or calls it.
 *
 * It follows the reference's CUDA sources line by line, in plain C:
 *   kernels.cu:361-371  setKeys            -> orc_morton_keys
 *   engine.cu:98-99     sequence+sort      -> orc_sort_perm (stable LSD radix)
 *   kernels.cu:311-318  emptyGrid          \
 *   kernels.cu:6-142    p2GTransferScatter -> orc_p2g (incl. the 11^3 shared
 *                                             tile of 256-particle blocks and
 *                                             its mass > 1e-9 flush rule)
 *   kernels.cu:144-196  gridUpdate         -> orc_grid_update
 *   kernels.cu:199-280  g2PTransfer        -> orc_g2p
 *   engine.cu:54-70     Engine::step       -> orc_substep
 *   kernels.cu:349-358  initFMatrices      -> orc_init_particles
 *   kernels.cu:341-347  changeFormat       -> orc_positions
 *   kernels.cu:282-300  makeSDF            -> orc_make_sdf
 *   common.cuh:131-378  device helpers     -> static functions below
 *
 * `real` is double (ORC_REAL=double: the FP64 oracle of the parity tests) or
 * float (ORC_REAL=float: the FP32 transcription timed as the CPU baseline).
 * Built with -ffp-contract=off so that no multiply-add is fused behind the
 * source's back; the float build then evaluates the spline exactly as the
 * reference does (x*x rounded to float, the rest in double, one rounding).
 * Integer conversions emulate the GPU's saturating cvt.rzi (NaN -> 0), which
 * C leaves undefined.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL real;

#define SHARED_H 11
#define SHARED_N (SHARED_H * SHARED_H * SHARED_H)

enum { POS_X = 0, VEL_X = 3, C00 = 6, F00 = 15, VOL = 24, MASS = 25, PLANES = 26 };

typedef struct orc_params {
    int32_t sx, sy, sz, padding;
    float gravity, dt, gamma, compression, resolution;
} orc_params;

/* cvt.rzi.s32 / cvt.rzi.u32: truncate toward zero, saturate, NaN -> 0. */
static inline int32_t to_i32(real v) {
    if (v != v) return 0;
    if (v >= (real)2147483647.0) return INT32_MAX;
    if (v <= (real)-2147483648.0) return INT32_MIN;
    return (int32_t)v;
}
static inline uint32_t to_u32(real v) {
    if (v != v || v <= 0) return 0u;
    if (v >= (real)4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

/* getGridIdx (common.cuh:131-134) */
static inline long gidx(const orc_params* p, int x, int y, int z) {
    return ((long)z * p->sy + y) * p->sx + x;
}
/* isInBounds (common.cuh:212-218) */
static inline int inb(const orc_params* p, int x, int y, int z) {
    return x >= 0 && x < p->sx && y >= 0 && y < p->sy && z >= 0 && z < p->sz;
}
/* spline (common.cuh:205-210) */
static inline real spline(real x) {
    real ax = (real)fabs((double)x);
    if (ax < 0.5) return (real)(0.75 - x * x);
    if (ax >= 0.5 && ax < 1.5) return (real)((1.5 - ax) * (1.5 - ax) * 0.5);
    return 0;
}
/* det3x3 (common.cuh:250-253) */
static inline real det3(const real* A) {
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) + A[2] * (A[3] * A[7] - A[4] * A[6]);
}
/* getSDF (common.cuh:136-167) */
static real sdf_at(const orc_params* p, const real* sdf, real qx, real qy, real qz) {
    int i = to_i32(floor(qx)), j = to_i32(floor(qy)), k = to_i32(floor(qz));
    real tx = qx - (real)i, ty = qy - (real)j, tz = qz - (real)k;
#define CL(v, hi) ((v) < 0 ? 0 : ((v) > (hi) ? (hi) : (v)))
#define S(a, b, c) sdf[gidx(p, CL(a, p->sx - 1), CL(b, p->sy - 1), CL(c, p->sz - 1))]
    /* i+1 in 64-bit: the device wraps, but only for |q| >= 2^31, never in tests */
    long i1 = (long)i + 1, j1 = (long)j + 1, k1 = (long)k + 1;
    real N0 = S(i, j, k), N1 = S(i1, j, k), N2 = S(i, j1, k), N3 = S(i1, j1, k);
    real N4 = S(i, j, k1), N5 = S(i1, j, k1), N6 = S(i, j1, k1), N7 = S(i1, j1, k1);
#undef S
#undef CL
    real x0 = N0 * (1 - tx) + N1 * tx, x1 = N2 * (1 - tx) + N3 * tx;
    real x2 = N4 * (1 - tx) + N5 * tx, x3 = N6 * (1 - tx) + N7 * tx;
    real y0 = x0 * (1 - ty) + x1 * ty, y1 = x2 * (1 - ty) + x3 * ty;
    return y0 * (1 - tz) + y1 * tz;
}
/* calculateNormal (common.cuh:169-182) */
static void sdf_normal(const orc_params* p, const real* sdf, real qx, real qy, real qz, real* n) {
    const real eps = (real)0.1f;
    n[0] = sdf_at(p, sdf, qx + eps, qy, qz) - sdf_at(p, sdf, qx - eps, qy, qz);
    n[1] = sdf_at(p, sdf, qx, qy + eps, qz) - sdf_at(p, sdf, qx, qy - eps, qz);
    n[2] = sdf_at(p, sdf, qx, qy, qz + eps) - sdf_at(p, sdf, qx, qy, qz - eps);
    real len = (real)sqrt((double)(n[0] * n[0] + n[1] * n[1] + n[2] * n[2])) + (real)1e-6f;
    n[0] /= len;
    n[1] /= len;
    n[2] /= len;
}
/* getNormalAtNode (common.cuh:195-203) */
static void node_normal(const orc_params* p, const real* sdf, int x, int y, int z, real* n) {
    int xp = x + 1 < p->sx - 1 ? x + 1 : p->sx - 1, xm = x - 1 > 0 ? x - 1 : 0;
    int yp = y + 1 < p->sy - 1 ? y + 1 : p->sy - 1, ym = y - 1 > 0 ? y - 1 : 0;
    int zp = z + 1 < p->sz - 1 ? z + 1 : p->sz - 1, zm = z - 1 > 0 ? z - 1 : 0;
    n[0] = sdf[gidx(p, xp, y, z)] - sdf[gidx(p, xm, y, z)];
    n[1] = sdf[gidx(p, x, yp, z)] - sdf[gidx(p, x, ym, z)];
    n[2] = sdf[gidx(p, x, y, zp)] - sdf[gidx(p, x, y, zm)];
    real len = (real)sqrt((double)(n[0] * n[0] + n[1] * n[1] + n[2] * n[2])) + (real)1e-9f;
    n[0] /= len;
    n[1] /= len;
    n[2] /= len;
}
/* expandBits + calculateMorton (common.cuh:277-284, 304-307): the published
 * multiply-and-mask bit spread (Karras 2012) */
static inline uint32_t spread3(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

/* ------------------------------------------------------------------ */

/* initFMatrices (kernels.cu:349-358) */
void orc_init_particles(const orc_params* p, real* st, long n) {
    float r = p->resolution;
    for (long i = 0; i < n; ++i) {
        st[(F00 + 0) * n + i] = 1;
        st[(F00 + 4) * n + i] = 1;
        st[(F00 + 8) * n + i] = 1;
        st[VOL * n + i] = (real)(r * r * r);
        st[MASS * n + i] = 1;
    }
}

/* setKeys (kernels.cu:361-371) */
void orc_morton_keys(const real* st, long n, int32_t* keys) {
    long i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; ++i) {
        real x = st[(POS_X + 0) * n + i], y = st[(POS_X + 1) * n + i], z = st[(POS_X + 2) * n + i];
        /* fmaxf(0, NaN) = 0 */
        uint32_t ux = to_u32(x > 0 ? x : 0), uy = to_u32(y > 0 ? y : 0), uz = to_u32(z > 0 ? z : 0);
        keys[i] = (int32_t)((spread3(uz) << 2) | (spread3(uy) << 1) | spread3(ux));
    }
}

/* thrust::sequence + thrust::sort_by_key on int keys (engine.cu:98-99):
 * stable ascending signed order, ties by index.  LSD radix, 8-bit digits;
 * each pass splits the input into per-thread chunks in order, so it stays
 * stable with any thread count. */
void orc_sort_perm(const int32_t* keys, long n, int32_t* perm) {
    if (n <= 0) return;
    uint32_t* k0 = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* k1 = (uint32_t*)malloc(sizeof(uint32_t) * n);
    int32_t* v1 = (int32_t*)malloc(sizeof(int32_t) * n);
    long i;
    for (i = 0; i < n; ++i) {
        k0[i] = (uint32_t)keys[i] ^ 0x80000000u;
        perm[i] = (int32_t)i;
    }
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    long* hist = (long*)calloc((size_t)nt * 256, sizeof(long));
    for (int pass = 0; pass < 4; ++pass) {
        int sh = 8 * pass;
        memset(hist, 0, sizeof(long) * nt * 256);
#pragma omp parallel num_threads(nt)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            long lo = n * t / nt, hi = n * (t + 1) / nt;
            for (long q = lo; q < hi; ++q) hist[t * 256 + ((k0[q] >> sh) & 255u)]++;
#pragma omp barrier
#pragma omp single
            {
                long run = 0;
                for (int d = 0; d < 256; ++d)
                    for (int u = 0; u < nt; ++u) {
                        long c = hist[u * 256 + d];
                        hist[u * 256 + d] = run;
                        run += c;
                    }
            }
            for (long q = lo; q < hi; ++q) {
                long dst = hist[t * 256 + ((k0[q] >> sh) & 255u)]++;
                k1[dst] = k0[q];
                v1[dst] = perm[q];
            }
        }
        uint32_t* tk = k0;
        k0 = k1;
        k1 = tk;
        memcpy(perm, v1, sizeof(int32_t) * n);
    }
    free(hist);
    free(k0);
    free(k1);
    free(v1);
}

static inline void grid_add(real* g, long G, long c, real m, real x, real y, real z) {
#pragma omp atomic
    g[c] += m;
#pragma omp atomic
    g[G + c] += x;
#pragma omp atomic
    g[2 * G + c] += y;
#pragma omp atomic
    g[3 * G + c] += z;
}

/* emptyGrid + p2GTransferScatter (kernels.cu:311-318, 6-142).  grid holds
 * 4 planes (mass, momentum x/y/z).  tile_mode 1 reproduces the reference's
 * blocks of 256 sorted particles and their 11^3 tile anchored one node below
 * the block's first particle, with the mass > 1e-9 flush; tile_mode 0 adds
 * every contribution straight to the grid. */
void orc_p2g(const orc_params* p, const real* st, long n, const int32_t* perm, real* grid, int tile_mode) {
    const long G = (long)p->sx * p->sy * p->sz;
    memset(grid, 0, sizeof(real) * 4 * G);
    const long nblocks = (n + 255) / 256;
    long b;
#pragma omp parallel for schedule(dynamic, 4)
    for (b = 0; b < nblocks; ++b) {
        real* tile = tile_mode ? (real*)calloc(4 * SHARED_N, sizeof(real)) : NULL;
        const long first = perm[b * 256];
        const int minX = to_i32(st[(POS_X + 0) * n + first] - (real)0.5f);
        const int minY = to_i32(st[(POS_X + 1) * n + first] - (real)0.5f);
        const int minZ = to_i32(st[(POS_X + 2) * n + first] - (real)0.5f);
        for (long t = b * 256; t < n && t < (b + 1) * 256; ++t) {
            const long q = perm[t];
            real pos[3], vel[3], C[9], F[9];
            for (int k = 0; k < 3; ++k) pos[k] = st[(POS_X + k) * n + q];
            for (int k = 0; k < 3; ++k) vel[k] = st[(VEL_X + k) * n + q];
            for (int k = 0; k < 9; ++k) C[k] = st[(C00 + k) * n + q];
            for (int k = 0; k < 9; ++k) F[k] = st[(F00 + k) * n + q];
            const real pm = st[MASS * n + q];
            const int bx = to_i32(pos[0] - (real)0.5f), by = to_i32(pos[1] - (real)0.5f), bz = to_i32(pos[2] - (real)0.5f);
            real J = det3(F);
            J = J > (real)1.1f ? (real)1.1f : J;
            J = J < (real)0.9f ? (real)0.9f : J;
            real pressure = (real)p->compression * ((real)pow((double)J, (double)p->gamma) - 1);
            if (pressure < 0) pressure = 0;
            const real volume = st[VOL * n + q] * J;
            const real multi = (real)4.0f * (real)p->dt * volume * pressure / pm;
            for (int k = 0; k < 9; ++k) C[k] = C[k] + multi * ((k % 4 == 0) ? 1 : 0);
            real wx[3], wy[3], wz[3];
            for (int a = 0; a < 3; ++a) {
                wx[a] = spline(pos[0] - (real)(bx + a));
                wy[a] = spline(pos[1] - (real)(by + a));
                wz[a] = spline(pos[2] - (real)(bz + a));
            }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        const int x = bx + i, y = by + j, z = bz + k;
                        if (!inb(p, x, y, z)) continue;
                        const real dx = -(pos[0] - (real)x), dy = -(pos[1] - (real)y), dz = -(pos[2] - (real)z);
                        const real w = wx[i] * wy[j] * wz[k];
                        const real wm = pm * w * 1;
                        const real mx = wm * (vel[0] + (C[0] * dx + C[1] * dy + C[2] * dz));
                        const real my = wm * (vel[1] + (C[3] * dx + C[4] * dy + C[5] * dz));
                        const real mz = wm * (vel[2] + (C[6] * dx + C[7] * dy + C[8] * dz));
                        const int lx = x - minX + 1, ly = y - minY + 1, lz = z - minZ + 1;
                        if (tile_mode && lx >= 0 && lx < SHARED_H && ly >= 0 && ly < SHARED_H && lz >= 0 &&
                            lz < SHARED_H) {
                            const long l = ((long)lz * SHARED_H + ly) * SHARED_H + lx;
                            tile[l] += wm;
                            tile[SHARED_N + l] += mx;
                            tile[2 * SHARED_N + l] += my;
                            tile[3 * SHARED_N + l] += mz;
                        } else {
                            grid_add(grid, G, gidx(p, x, y, z), wm, mx, my, mz);
                        }
                    }
        }
        if (tile_mode) {
            for (long l = 0; l < SHARED_N; ++l) {
                const int gx = minX + (int)(l % SHARED_H) - 1;
                const int gy = minY + (int)((l / SHARED_H) % SHARED_H) - 1;
                const int gz = minZ + (int)(l / (SHARED_H * SHARED_H)) - 1;
                if (inb(p, gx, gy, gz) && tile[l] > (real)1e-9)
                    grid_add(grid, G, gidx(p, gx, gy, gz), tile[l], tile[SHARED_N + l], tile[2 * SHARED_N + l],
                             tile[3 * SHARED_N + l]);
            }
            free(tile);
        }
    }
}

/* gridUpdate (kernels.cu:144-196); SimConfig fields are uint32, so the wall
 * tests compare unsigned. */
void orc_grid_update(const orc_params* p, real* grid, const real* sdf) {
    const long G = (long)p->sx * p->sy * p->sz;
    long idx;
#pragma omp parallel for schedule(static)
    for (idx = 0; idx < G; ++idx) {
        const int x = (int)(idx % p->sx), y = (int)((idx / p->sx) % p->sy), z = (int)(idx / ((long)p->sx * p->sy));
        const real mass = grid[idx];
        real v[3] = {0, 0, 0};
        if (mass > (real)1e-9f) {
            v[0] = grid[G + idx] / mass;
            v[1] = grid[2 * G + idx] / mass - (real)p->gravity * (real)p->dt;
            v[2] = grid[3 * G + idx] / mass;
            if (sdf[idx] < 0) {
                real nn[3];
                node_normal(p, sdf, x, y, z, nn);
                const real vdn = v[0] * nn[0] + v[1] * nn[1] + v[2] * nn[2];
                if (vdn < 0) {
                    v[0] -= nn[0] * vdn;
                    v[1] -= nn[1] * vdn;
                    v[2] -= nn[2] * vdn;
                }
            }
            const uint32_t pad = (uint32_t)p->padding;
            if ((uint32_t)x < pad && v[0] < 0) v[0] = 0;
            if ((uint32_t)y < pad && v[1] < 0) v[1] = 0;
            if ((uint32_t)z < pad && v[2] < 0) v[2] = 0;
            if ((uint32_t)x > (uint32_t)p->sx - 1u - pad && v[0] > 0) v[0] = 0;
            if ((uint32_t)y > (uint32_t)p->sy - 1u - pad && v[1] > 0) v[1] = 0;
            if ((uint32_t)z > (uint32_t)p->sz - 1u - pad && v[2] > 0) v[2] = 0;
        }
        grid[G + idx] = v[0];
        grid[2 * G + idx] = v[1];
        grid[3 * G + idx] = v[2];
    }
}

/* g2PTransfer (kernels.cu:199-280).  Order-independent: each particle reads
 * the grid and writes its own slot, so perm only fixes the loop order. */
void orc_g2p(const orc_params* p, real* st, long n, const int32_t* perm, const real* grid, const real* sdf) {
    const long G = (long)p->sx * p->sy * p->sz;
    const real dt = (real)p->dt;
    long t;
#pragma omp parallel for schedule(static)
    for (t = 0; t < n; ++t) {
        const long q = perm ? perm[t] : t;
        real pos[3], F[9];
        for (int k = 0; k < 3; ++k) pos[k] = st[(POS_X + k) * n + q];
        for (int k = 0; k < 9; ++k) F[k] = st[(F00 + k) * n + q];
        const int bx = to_i32(pos[0] - (real)0.5f), by = to_i32(pos[1] - (real)0.5f), bz = to_i32(pos[2] - (real)0.5f);
        real wx[3], wy[3], wz[3];
        for (int a = 0; a < 3; ++a) {
            wx[a] = spline(pos[0] - (real)(bx + a));
            wy[a] = spline(pos[1] - (real)(by + a));
            wz[a] = spline(pos[2] - (real)(bz + a));
        }
        real tv[3] = {0, 0, 0}, tc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    const int x = bx + i, y = by + j, z = bz + k;
                    if (!inb(p, x, y, z)) continue;
                    const long c = gidx(p, x, y, z);
                    const real d[3] = {-(pos[0] - (real)x), -(pos[1] - (real)y), -(pos[2] - (real)z)};
                    const real w = wx[i] * wy[j] * wz[k];
                    const real gv[3] = {grid[G + c], grid[2 * G + c], grid[3 * G + c]};
                    for (int r = 0; r < 3; ++r) tv[r] += w * gv[r];
                    const real term = 4 * w;
                    for (int r = 0; r < 3; ++r)
                        for (int s = 0; s < 3; ++s) tc[r * 3 + s] += term * gv[r] * d[s];
                }
        real T[9], NF[9];
        for (int k = 0; k < 9; ++k) T[k] = ((k % 4 == 0) ? 1 : 0) + dt * tc[k];
        for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s)
                NF[r * 3 + s] = T[r * 3 + 0] * F[s] + T[r * 3 + 1] * F[3 + s] + T[r * 3 + 2] * F[6 + s];
        const real J = det3(NF);
        if (J < (real)0.3f) {
            const real scale = (real)pow((double)((real)0.3f / J), (double)(1.0f / 3.0f));
            for (int k = 0; k < 9; ++k) NF[k] *= scale;
        }
        real nx = pos[0] + tv[0] * dt, ny = pos[1] + tv[1] * dt, nz = pos[2] + tv[2] * dt;
        const real dist = sdf_at(p, sdf, nx, ny, nz);
        if (dist < 0) {
            real nn[3];
            sdf_normal(p, sdf, nx, ny, nz, nn);
            nx -= nn[0] * dist;
            ny -= nn[1] * dist;
            nz -= nn[2] * dist;
            const real vdn = tv[0] * nn[0] + tv[1] * nn[1] + tv[2] * nn[2];
            if (vdn < 0) {
                tv[0] -= nn[0] * vdn;
                tv[1] -= nn[1] * vdn;
                tv[2] -= nn[2] * vdn;
            }
        }
        st[(POS_X + 0) * n + q] = nx;
        st[(POS_X + 1) * n + q] = ny;
        st[(POS_X + 2) * n + q] = nz;
        for (int k = 0; k < 3; ++k) st[(VEL_X + k) * n + q] = tv[k];
        for (int k = 0; k < 9; ++k) st[(C00 + k) * n + q] = tc[k];
        for (int k = 0; k < 9; ++k) st[(F00 + k) * n + q] = NF[k];
    }
}

/* Engine::step (engine.cu:54-70): keys, stable sort, clear, P2G, grid update,
 * G2P.  keys/perm (n ints each, may be NULL) receive this substep's sort. */
void orc_substep(const orc_params* p, real* st, long n, real* grid, const real* sdf, int32_t* keys_out,
                 int32_t* perm_out, int tile_mode) {
    int32_t* keys = keys_out ? keys_out : (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    int32_t* perm = perm_out ? perm_out : (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    orc_morton_keys(st, n, keys);
    orc_sort_perm(keys, n, perm);
    orc_p2g(p, st, n, perm, grid, tile_mode);
    orc_grid_update(p, grid, sdf);
    orc_g2p(p, st, n, perm, grid, sdf);
    if (!keys_out) free(keys);
    if (!perm_out) free(perm);
}

/* changeFormat (kernels.cu:341-347) */
void orc_positions(const real* st, long n, real* xyz) {
    for (long i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = st[(POS_X + k) * n + i];
}

static inline real dot3(const real* a, const real* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* calculateSolidAngle (common.cuh:310-323) */
static real solid_angle(const real* P, const real* t) {
    real a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = t[k] - P[k];
        b[k] = t[3 + k] - P[k];
        c[k] = t[6 + k] - P[k];
    }
    const real la = (real)sqrt((double)dot3(a, a)), lb = (real)sqrt((double)dot3(b, b)),
               lc = (real)sqrt((double)dot3(c, c));
    const real det = a[0] * (b[1] * c[2] - b[2] * c[1]) + a[1] * (b[2] * c[0] - b[0] * c[2]) +
                     a[2] * (b[0] * c[1] - b[1] * c[0]);
    const real div = la * lb * lc + dot3(a, b) * lc + dot3(a, c) * lb + dot3(b, c) * la;
    return 2 * (real)atan2((double)det, (double)div);
}

/* pointTriangleDistanceSq (common.cuh:325-378) */
static real tri_dist2(const real* P, const real* t) {
    const real* A = t;
    const real* B = t + 3;
    const real* Cv = t + 6;
    real ab[3], ac[3], ap[3], bp[3], cp[3], q[3], d[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = B[k] - A[k];
        ac[k] = Cv[k] - A[k];
        ap[k] = P[k] - A[k];
    }
    const real d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0 && d2 <= 0) return dot3(ap, ap);
    for (int k = 0; k < 3; ++k) bp[k] = P[k] - B[k];
    const real d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0 && d4 <= d3) return dot3(bp, bp);
    const real vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const real v = d1 / (d1 - d3);
        for (int k = 0; k < 3; ++k) d[k] = P[k] - (A[k] + v * ab[k]);
        return dot3(d, d);
    }
    for (int k = 0; k < 3; ++k) cp[k] = P[k] - Cv[k];
    const real d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0 && d5 <= d6) return dot3(cp, cp);
    const real vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const real w = d2 / (d2 - d6);
        for (int k = 0; k < 3; ++k) d[k] = P[k] - (A[k] + w * ac[k]);
        return dot3(d, d);
    }
    const real va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        const real w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int k = 0; k < 3; ++k) d[k] = P[k] - (B[k] + w * (Cv[k] - B[k]));
        return dot3(d, d);
    }
    const real denom = 1 / (va + vb + vc);
    const real v = vb * denom, w = vc * denom;
    for (int k = 0; k < 3; ++k) {
        q[k] = A[k] + ab[k] * v + ac[k] * w;
        d[k] = P[k] - q[k];
    }
    return dot3(d, d);
}

/* makeSDF (kernels.cu:282-300).  wn_out (may be NULL) receives the winding
 * number of each node, so a test can set aside nodes where the sign is
 * ill-conditioned. */
void orc_make_sdf(const orc_params* p, const real* tris, long t, real* sdf, real* wn_out) {
    const long G = (long)p->sx * p->sy * p->sz;
    const real four_pi_ref = (real)(4.0f * 3.1415f);
    long idx;
#pragma omp parallel for schedule(dynamic, 64)
    for (idx = 0; idx < G; ++idx) {
        const real P[3] = {(real)(idx % p->sx), (real)((idx / p->sx) % p->sy), (real)(idx / ((long)p->sx * p->sy))};
        real wsum = 0, dmin = (real)1e30f;
        for (long i = 0; i < t; ++i) {
            wsum += solid_angle(P, tris + 9 * i);
            const real d2 = tri_dist2(P, tris + 9 * i);
            if (d2 < dmin) dmin = d2;
        }
        const real wn = wsum / four_pi_ref;
        sdf[idx] = (wn > (real)0.5f ? -1 : 1) * (real)sqrt((double)dmin);
        if (wn_out) wn_out[idx] = wn;
    }
}

/* makeSDF at `count` chosen nodes (grid indices `nodes`): the same per-node
 * loop as orc_make_sdf, for grids whose full SDF is too costly on the CPU. */
void orc_make_sdf_nodes(const orc_params* p, const real* tris, long t, const long* nodes, long count, real* sdf,
                        real* wn_out) {
    const real four_pi_ref = (real)(4.0f * 3.1415f);
    long k;
#pragma omp parallel for schedule(dynamic, 16)
    for (k = 0; k < count; ++k) {
        const long idx = nodes[k];
        const real P[3] = {(real)(idx % p->sx), (real)((idx / p->sx) % p->sy), (real)(idx / ((long)p->sx * p->sy))};
        real wsum = 0, dmin = (real)1e30f;
        for (long i = 0; i < t; ++i) {
            wsum += solid_angle(P, tris + 9 * i);
            const real d2 = tri_dist2(P, tris + 9 * i);
            if (d2 < dmin) dmin = d2;
        }
        const real wn = wsum / four_pi_ref;
        sdf[k] = (wn > (real)0.5f ? -1 : 1) * (real)sqrt((double)dmin);
        if (wn_out) wn_out[k] = wn;
    }
}

int orc_real_bytes(void) { return (int)sizeof(real); }

int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

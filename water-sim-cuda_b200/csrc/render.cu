// Headless screen-space fluid rendering: the reference's OpenGL SSF passes
// (renderer.cpp:199-338 with shaders/ssf_depth.*, ssf_blur.frag and
// screen.frag) restated as CUDA kernels into device image buffers.  No
// graphics API is involved.
//
//  1. Depth splat (ssf_depth.vert/.frag): each particle is a point sprite of
//     radius * 1000 / |view position| pixels; a covered pixel at sprite
//     coordinate (s, t) with r2 = |(s, t) * 2 - 1|^2 <= 1 sees the sphere
//     surface at view z' = z + sqrt(1 - r2) * radius.  The depth test keeps
//     the nearest fragment (largest z'); the colour target holds z'.  Pixels
//     no sprite covers keep the clear value 99999.
//  2. Bilateral blur (ssf_blur.frag), horizontal then vertical: 2 F + 1 taps,
//     weight exp(-(i / F)^2) * exp(-((d_i - d_c) * falloff)^2), texture
//     coordinates wrapping (GL_REPEAT, the textures' default wrap mode);
//     pixels deeper than 5000 pass through.
//  3. Composite (screen.frag): view position from depth, normal from the
//     cross product of the right and top differences, background sampled at
//     uv + 0.05 n.xy (bilinear, wrapping), Fresnel (1 - n.z)^4, specular
//     (reflect(-L, n) . z)^128, colour mix(bg, water, 0.3 + 0.5 fresnel) + spec.
//
// Camera (renderer.cpp:95-96, 186-195): eye (SX/2, SY/2, zoom), looking at
// the grid centre, up +y; model = rotation about the centre by the vertical
// angle (x axis) then the horizontal angle (y axis); perspective 45 degrees,
// near 0.1, far 5000.
//
//  0. Obstacles (dot.vert + dot.frag, renderer.cpp:247-303, the default
//     opaque mode), drawn once per renderer into the background: each
//     triangle in grid coordinates goes through the model, view and
//     projection matrices, covers the pixels whose centres lie inside it
//     (top-left rule on shared edges), and the depth test (GL_LESS, depth
//     cleared to 1) keeps the nearest fragment, the earlier triangle on a
//     tie.  Its colour is flat: dot.frag's normal, the cross product of the
//     screen-space derivatives of the world position, is the triangle's plane
//     normal turned towards the eye; colour = 0.3 C + max(n . L, 0) C with
//     C = (0.5, 0.5, 0.5) and L the normalised world light, stored as 8 bits
//     like the framebuffer that glCopyTexSubImage2D turns into the
//     background texture.  The fluid's composite then passes the depth test
//     against the obstacles' window depth (screen.frag's gl_FragDepth).
//
// Differences from the GL pipeline, where the rasteriser's choices are not
// observable in the shaders: a sprite whose centre lies outside the clip
// volume is dropped whole; an obstacle triangle with a vertex behind the
// near plane is dropped whole (GL clips it); depths are compared as floats
// (GL's 24-bit depth buffer can keep the earlier of two fragments closer
// than its resolution); the glass and wireframe modes, keyboard toggles of
// the interactive viewer, are not restated.  Without obstacles the
// background is the clear colour as stored in the 8-bit framebuffer, or an
// image the caller supplies.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "kernels.h"

namespace {

struct Cam {
    float m[16];    // model-view (column-major: m[col * 4 + row])
    float p00, p11, p22, p32;  // perspective terms
    int w, h;
    float radius, far_clip, near_clip;
};

__device__ __forceinline__ unsigned ord_enc(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_dec(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// One thread per particle: the pixels of its sprite.
__global__ void splat_kernel(const float* __restrict__ xyz, long long n, Cam c, unsigned* __restrict__ zbuf) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = xyz[i * 3], y = xyz[i * 3 + 1], z = xyz[i * 3 + 2];
    const float vx = c.m[0] * x + c.m[4] * y + c.m[8] * z + c.m[12];
    const float vy = c.m[1] * x + c.m[5] * y + c.m[9] * z + c.m[13];
    const float vz = c.m[2] * x + c.m[6] * y + c.m[10] * z + c.m[14];
    const float w = -vz;
    if (!(w > c.near_clip && w < c.far_clip)) return;
    const float nx = c.p00 * vx / w, ny = c.p11 * vy / w;
    if (!(nx >= -1.0f && nx <= 1.0f && ny >= -1.0f && ny <= 1.0f)) return;
    const float size = c.radius * (1000.0f / sqrtf(vx * vx + vy * vy + vz * vz));
    const float cx = (nx * 0.5f + 0.5f) * (float)c.w, cy = (ny * 0.5f + 0.5f) * (float)c.h;
    const float x0 = cx - 0.5f * size, y0 = cy - 0.5f * size;
    // pixel centres (px + 0.5) in [x0, x0 + size)
    const int px0 = max(0, (int)ceilf(x0 - 0.5f)), px1 = min(c.w - 1, (int)ceilf(x0 + size - 0.5f) - 1);
    const int py0 = max(0, (int)ceilf(y0 - 0.5f)), py1 = min(c.h - 1, (int)ceilf(y0 + size - 0.5f) - 1);
    for (int py = py0; py <= py1; ++py) {
        const float t = 1.0f - (((float)py + 0.5f) - y0) / size;  // gl_PointCoord.t, origin upper left
        const float ny2 = t * 2.0f - 1.0f;
        for (int px = px0; px <= px1; ++px) {
            const float s = (((float)px + 0.5f) - x0) / size;
            const float nx2 = s * 2.0f - 1.0f;
            const float r2 = nx2 * nx2 + ny2 * ny2;
            if (r2 > 1.0f) continue;
            const float zz = vz + sqrtf(1.0f - r2) * c.radius;
            atomicMax(zbuf + (size_t)py * c.w + px, ord_enc(zz));
        }
    }
}

__global__ void resolve_kernel(const unsigned* __restrict__ zbuf, long long npix, float* __restrict__ depth) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const unsigned u = zbuf[i];
    depth[i] = u == 0u ? 99999.0f : ord_dec(u);
}

// One bilateral pass along (dx, dy) in {(1, 0), (0, 1)}.
__global__ void blur_kernel(const float* __restrict__ in, float* __restrict__ out, int w, int h, int dx, int dy,
                            float filter, float falloff) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const float dc = in[(size_t)y * w + x];
    if (dc > 5000.0f) {
        out[(size_t)y * w + x] = dc;
        return;
    }
    float sum = 0.0f, wsum = 0.0f;
    for (float i = -filter; i <= filter; i += 1.0f) {
        const int k = (int)i;
        int sx = x + k * dx, sy = y + k * dy;
        sx %= w;
        sy %= h;
        if (sx < 0) sx += w;
        if (sy < 0) sy += h;
        const float ds = in[(size_t)sy * w + sx];
        const float r = i * 1.0f / filter;
        float wt = expf(-r * r);
        const float r2 = (ds - dc) * falloff;
        wt *= expf(-r2 * r2);
        sum += ds * wt;
        wsum += wt;
    }
    out[(size_t)y * w + x] = sum / wsum;
}

__device__ __forceinline__ float3 view_pos(const float* __restrict__ depth, int w, int h, int x, int y, float p00,
                                           float p11) {
    x %= w;
    y %= h;
    const float d = depth[(size_t)y * w + x];
    const float u = ((float)x + 0.5f) / (float)w, v = ((float)y + 0.5f) / (float)h;
    const float px = (u * 2.0f - 1.0f) / p00, py = (v * 2.0f - 1.0f) / p11;
    return make_float3(px * -d, py * -d, d);
}

// Bilinear, wrapping sample of an RGB8 image at (u, v) (texel centres at
// (i + 0.5) / w).
__device__ float3 sample_rgb8(const unsigned char* __restrict__ img, int w, int h, float u, float v) {
    const float fx = u * (float)w - 0.5f, fy = v * (float)h - 0.5f;
    const float x0f = floorf(fx), y0f = floorf(fy);
    const float ax = fx - x0f, ay = fy - y0f;
    int x0 = (int)x0f % w, y0 = (int)y0f % h;
    if (x0 < 0) x0 += w;
    if (y0 < 0) y0 += h;
    const int x1 = (x0 + 1) % w, y1 = (y0 + 1) % h;
    float3 r;
    float* rp = &r.x;
    for (int c = 0; c < 3; ++c) {
        const float a = img[((size_t)y0 * w + x0) * 3 + c] / 255.0f, b = img[((size_t)y0 * w + x1) * 3 + c] / 255.0f;
        const float d = img[((size_t)y1 * w + x0) * 3 + c] / 255.0f, e = img[((size_t)y1 * w + x1) * 3 + c] / 255.0f;
        rp[c] = (a * (1.0f - ax) + b * ax) * (1.0f - ay) + (d * (1.0f - ax) + e * ax) * ay;
    }
    return r;
}

// One thread per obstacle triangle: the pixels whose centres it covers, as
// 64-bit keys (window depth bits, triangle index) kept by atomicMin, so the
// nearest fragment wins and, at equal depth, the earlier triangle.
__global__ void obstacle_raster_kernel(const float* __restrict__ tris, int t, Cam c,
                                       unsigned long long* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t) return;
    float X[3], Y[3], Z[3];
    for (int k = 0; k < 3; ++k) {
        const float x = tris[i * 9 + 3 * k], y = tris[i * 9 + 3 * k + 1], z = tris[i * 9 + 3 * k + 2];
        const float vx = c.m[0] * x + c.m[4] * y + c.m[8] * z + c.m[12];
        const float vy = c.m[1] * x + c.m[5] * y + c.m[9] * z + c.m[13];
        const float vz = c.m[2] * x + c.m[6] * y + c.m[10] * z + c.m[14];
        const float wc = -vz;
        if (!(wc > c.near_clip)) return;  // GL would clip at the near plane
        X[k] = (c.p00 * vx / wc * 0.5f + 0.5f) * (float)c.w;
        Y[k] = (c.p11 * vy / wc * 0.5f + 0.5f) * (float)c.h;
        Z[k] = (c.p22 * vz + c.p32) / wc * 0.5f + 0.5f;
    }
    float area = (X[1] - X[0]) * (Y[2] - Y[0]) - (X[2] - X[0]) * (Y[1] - Y[0]);
    if (area == 0.0f || !isfinite(area)) return;
    const float sgn = area > 0.0f ? 1.0f : -1.0f;
    area *= sgn;
    // Edge k runs from vertex k + 1 to k + 2; with the counter-clockwise
    // orientation (sgn applied) a top edge is horizontal and points left, a
    // left edge points down.
    bool tl[3];
    for (int k = 0; k < 3; ++k) {
        const int a = (k + 1) % 3, b = (k + 2) % 3;
        const float ex = (X[b] - X[a]) * sgn, ey = (Y[b] - Y[a]) * sgn;
        tl[k] = (ey == 0.0f && ex < 0.0f) || ey < 0.0f;
    }
    const int x0 = max(0, (int)ceilf(fminf(X[0], fminf(X[1], X[2])) - 0.5f));
    const int x1 = min(c.w - 1, (int)floorf(fmaxf(X[0], fmaxf(X[1], X[2])) - 0.5f));
    const int y0 = max(0, (int)ceilf(fminf(Y[0], fminf(Y[1], Y[2])) - 0.5f));
    const int y1 = min(c.h - 1, (int)floorf(fmaxf(Y[0], fmaxf(Y[1], Y[2])) - 0.5f));
    for (int py = y0; py <= y1; ++py) {
        const float sy = (float)py + 0.5f;
        for (int px = x0; px <= x1; ++px) {
            const float sx = (float)px + 0.5f;
            float e[3];
            bool in = true;
            for (int k = 0; k < 3; ++k) {
                const int a = (k + 1) % 3, b = (k + 2) % 3;
                e[k] = ((X[b] - X[a]) * (sy - Y[a]) - (Y[b] - Y[a]) * (sx - X[a])) * sgn;
                in = in && (e[k] > 0.0f || (e[k] == 0.0f && tl[k]));
            }
            if (!in) continue;
            const float zw = (e[0] * Z[0] + e[1] * Z[1] + e[2] * Z[2]) / area;
            if (!(zw >= 0.0f && zw <= 1.0f)) continue;
            atomicMin(key + (size_t)py * c.w + px,
                      ((unsigned long long)__float_as_uint(zw) << 32) | (unsigned long long)(unsigned)i);
        }
    }
}

// The framebuffer after the obstacle pass: the winning triangle's flat
// colour over the base image, and its window depth (1 where none).
__global__ void obstacle_resolve_kernel(const unsigned long long* __restrict__ key,
                                        const unsigned char* __restrict__ tri_rgb8,
                                        const unsigned char* __restrict__ base, long long npix,
                                        unsigned char* __restrict__ bg, float* __restrict__ odepth) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const unsigned long long k = key[i];
    if (k == ~0ull) {
        for (int c = 0; c < 3; ++c) bg[i * 3 + c] = base[i * 3 + c];
        odepth[i] = 1.0f;
        return;
    }
    const unsigned tri = (unsigned)(k & 0xffffffffull);
    for (int c = 0; c < 3; ++c) bg[i * 3 + c] = tri_rgb8[(size_t)tri * 3 + c];
    odepth[i] = __uint_as_float((unsigned)(k >> 32));
}

__global__ void composite_kernel(const float* __restrict__ depth, const unsigned char* __restrict__ bg, int w, int h,
                                 float p00, float p11, float p22, float p32, float lx, float ly, float lz,
                                 const float* __restrict__ odepth, float* __restrict__ rgb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t o = ((size_t)y * w + x) * 3;
    const float d = depth[(size_t)y * w + x];
    // discard, or the fluid surface behind an obstacle (gl_FragDepth of
    // screen.frag against the obstacles' depth, GL_LESS): the framebuffer
    // keeps the background
    const bool hidden = odepth && !(((p22 * d + p32) / -d) * 0.5f + 0.5f < odepth[(size_t)y * w + x]);
    if (d > 5000.0f || hidden) {
        for (int c = 0; c < 3; ++c) rgb[o + c] = bg[o + c] / 255.0f;
        return;
    }
    const float3 pc = view_pos(depth, w, h, x, y, p00, p11);
    const float3 pr = view_pos(depth, w, h, x + 1, y, p00, p11);
    const float3 pt = view_pos(depth, w, h, x, y + 1, p00, p11);
    const float ax = pr.x - pc.x, ay = pr.y - pc.y, az = pr.z - pc.z;
    const float bx = pt.x - pc.x, by = pt.y - pc.y, bz = pt.z - pc.z;
    float nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
    const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
    nx *= inv, ny *= inv, nz *= inv;
    const float u = ((float)x + 0.5f) / (float)w + nx * 0.05f, v = ((float)y + 0.5f) / (float)h + ny * 0.05f;
    const float3 b = sample_rgb8(bg, w, h, u, v);
    // reflect(-L, n) = -L - 2 dot(n, -L) n; its z
    const float ndl = nx * -lx + ny * -ly + nz * -lz;
    const float rz = -lz - 2.0f * ndl * nz;
    const float spec = powf(fmaxf(rz, 0.0f), 128.0f);
    const float fres = powf(1.0f - fmaxf(nz, 0.0f), 4.0f);
    const float a = 0.3f + fres * 0.5f;
    const float wc[3] = {0.1f, 0.5f, 0.8f};
    const float bc[3] = {b.x, b.y, b.z};
    for (int c = 0; c < 3; ++c) rgb[o + c] = bc[c] * (1.0f - a) + wc[c] * a + spec;
}

inline unsigned char unorm8(float f) {
    f = f < 0.0f ? 0.0f : (f > 1.0f ? 1.0f : f);
    return (unsigned char)std::floor(f * 255.0f + 0.5f);
}

// glm::lookAt / perspective / translate / rotate restated (column-major).
void mat_mul(const float* a, const float* b, float* out) {
    float r[16];
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) {
            float s = 0.0f;
            for (int k = 0; k < 4; ++k) s += a[k * 4 + rr] * b[c * 4 + k];
            r[c * 4 + rr] = s;
        }
    std::memcpy(out, r, sizeof(r));
}
void identity(float* m) {
    std::memset(m, 0, 16 * sizeof(float));
    m[0] = m[5] = m[10] = m[15] = 1.0f;
}
void translation(float* m, float x, float y, float z) {
    identity(m);
    m[12] = x, m[13] = y, m[14] = z;
}
void rotation(float* m, float angle, float ax, float ay, float az) {
    const float c = std::cos(angle), s = std::sin(angle);
    const float len = std::sqrt(ax * ax + ay * ay + az * az);
    ax /= len, ay /= len, az /= len;
    const float t[3] = {(1.0f - c) * ax, (1.0f - c) * ay, (1.0f - c) * az};
    identity(m);
    m[0] = c + t[0] * ax, m[1] = t[0] * ay + s * az, m[2] = t[0] * az - s * ay;
    m[4] = t[1] * ax - s * az, m[5] = c + t[1] * ay, m[6] = t[1] * az + s * ax;
    m[8] = t[2] * ax + s * ay, m[9] = t[2] * ay - s * ax, m[10] = c + t[2] * az;
}

}  // namespace

struct mpm_renderer {
    int device = 0;
    mpm_render_params prm{};
    Cam cam{};
    float light[3] = {0, 0, 1};
    unsigned* zbuf = nullptr;
    float* depth = nullptr;  // splat depth
    float* tmp = nullptr;    // after the horizontal blur
    float* fin = nullptr;    // after the vertical blur
    float* rgb = nullptr;
    unsigned char* bg = nullptr;       // the background texture: base + obstacles
    unsigned char* base = nullptr;     // clear colour or the caller's image
    float* odepth = nullptr;           // obstacles' window depth; null without obstacles
    unsigned long long* okey = nullptr;
    float* otris = nullptr;            // obstacle triangles (grid coordinates)
    unsigned char* ocolor = nullptr;   // their flat colours, 8 bits
    int ntris = 0;
    std::string last_error;
};

namespace {

mpm_status rfail(mpm_renderer* r, mpm_status s, const std::string& msg) {
    if (r) r->last_error = msg;
    mpm::set_global_error(msg);
    return s;
}

#define RK(r, call)                                                                                      \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            cudaGetLastError();                                                                          \
            return rfail((r), e_ == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA,     \
                         std::string("CUDA error in ") + #call + ": " + cudaGetErrorString(e_));         \
        }                                                                                                \
    } while (0)

void setup_camera(mpm_renderer* r) {
    const mpm_render_params& p = r->prm;
    const float cx = p.grid[0] / 2.0f, cy = p.grid[1] / 2.0f, cz = p.grid[2] / 2.0f;
    // view = lookAt(eye, centre, up)
    const float eye[3] = {cx, cy, p.zoom_distance};
    float f[3] = {cx - eye[0], cy - eye[1], cz - eye[2]};
    float fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (float& v : f) v /= fl;
    const float up[3] = {0.f, 1.f, 0.f};
    float s[3] = {f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]};
    const float sl = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (float& v : s) v /= sl;
    const float u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
    float view[16];
    identity(view);
    view[0] = s[0], view[4] = s[1], view[8] = s[2];
    view[1] = u[0], view[5] = u[1], view[9] = u[2];
    view[2] = -f[0], view[6] = -f[1], view[10] = -f[2];
    view[12] = -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2]);
    view[13] = -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2]);
    view[14] = f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2];
    // model = T(c) Rx(vertical) Ry(horizontal) T(-c)
    float m[16], t[16];
    translation(m, cx, cy, cz);
    rotation(t, p.rotation_vertical, 1, 0, 0);
    mat_mul(m, t, m);
    rotation(t, p.rotation, 0, 1, 0);
    mat_mul(m, t, m);
    translation(t, -cx, -cy, -cz);
    mat_mul(m, t, m);
    mat_mul(view, m, r->cam.m);
    const float fy = 1.0f / std::tan(p.fov_y_degrees * 3.14159265358979f / 180.0f / 2.0f);
    const float aspect = (float)p.width / (float)p.height;
    r->cam.p00 = fy / aspect;
    r->cam.p11 = fy;
    r->cam.p22 = -(p.far_clip + p.near_clip) / (p.far_clip - p.near_clip);
    r->cam.p32 = -(2.0f * p.far_clip * p.near_clip) / (p.far_clip - p.near_clip);
    r->cam.w = p.width;
    r->cam.h = p.height;
    r->cam.radius = p.radius;
    r->cam.far_clip = p.far_clip;
    r->cam.near_clip = p.near_clip;
    // lightDir = view * (normalised world light, 0)
    float L[3] = {p.light_dir[0], p.light_dir[1], p.light_dir[2]};
    const float ll = std::sqrt(L[0] * L[0] + L[1] * L[1] + L[2] * L[2]);
    for (float& v : L) v /= ll;
    for (int k = 0; k < 3; ++k) r->light[k] = view[k] * L[0] + view[4 + k] * L[1] + view[8 + k] * L[2];
}

}  // namespace

extern "C" {

void mpm_render_params_default(mpm_render_params* p, int32_t size_x, int32_t size_y, int32_t size_z) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->width = 1920;   // SCREEN_WIDTH, renderer.h:11
    p->height = 1600;  // SCREEN_HEIGHT, renderer.h:12
    p->grid[0] = size_x, p->grid[1] = size_y, p->grid[2] = size_z;
    p->fov_y_degrees = 45.0f;
    p->near_clip = 0.1f;
    p->far_clip = 5000.0f;
    p->zoom_distance = (float)size_z * 2.0f;  // renderer.cpp:95
    p->radius = 2.0f;                         // renderer.cpp:210
    p->filter_size = 10.0f;                   // renderer.cpp:223
    p->depth_falloff = 0.01f;                 // renderer.cpp:225
    p->light_dir[0] = 0.2f, p->light_dir[1] = 10.0f, p->light_dir[2] = 0.5f;  // renderer.cpp:197
    p->clear_color[0] = 0.85f, p->clear_color[1] = 0.9f, p->clear_color[2] = 0.95f;  // renderer.cpp:243
}

mpm_status mpm_renderer_create(const mpm_render_params* params, int32_t device, mpm_renderer** out) {
    if (!params || !out) return rfail(nullptr, MPM_ERR_INVALID_ARGUMENT, "params and out must be non-NULL");
    *out = nullptr;
    const mpm_render_params& p = *params;
    if (p.width <= 0 || p.height <= 0 || p.width > 16384 || p.height > 16384)
        return rfail(nullptr, MPM_ERR_INVALID_ARGUMENT, "image size out of range");
    if (!(p.radius > 0.f) || !(p.filter_size >= 0.f) || p.filter_size > 256.f || !(p.far_clip > p.near_clip) ||
        !(p.near_clip > 0.f) || !(p.fov_y_degrees > 0.f && p.fov_y_degrees < 180.f))
        return rfail(nullptr, MPM_ERR_INVALID_ARGUMENT, "render parameters out of range");
    auto* r = new mpm_renderer();
    r->device = device;
    r->prm = p;
    setup_camera(r);
    auto bad = [&](mpm_status s) {
        mpm_renderer_destroy(r);
        return s;
    };
    cudaError_t err = cudaSetDevice(device);
    const size_t npix = (size_t)p.width * p.height;
    if (err == cudaSuccess) err = cudaMalloc(&r->zbuf, npix * sizeof(unsigned));
    if (err == cudaSuccess) err = cudaMalloc(&r->depth, npix * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc(&r->tmp, npix * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc(&r->fin, npix * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc(&r->rgb, npix * 3 * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc(&r->bg, npix * 3);
    if (err == cudaSuccess) err = cudaMalloc(&r->base, npix * 3);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return bad(rfail(nullptr, MPM_ERR_OUT_OF_MEMORY, std::string("renderer allocation: ") + cudaGetErrorString(err)));
    }
    std::vector<unsigned char> bg(npix * 3);
    for (size_t i = 0; i < npix; ++i)
        for (int c = 0; c < 3; ++c) bg[i * 3 + c] = unorm8(p.clear_color[c]);
    if (cudaMemcpy(r->bg, bg.data(), bg.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(r->base, bg.data(), bg.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return bad(rfail(nullptr, MPM_ERR_CUDA, "background upload"));
    *out = r;
    return MPM_OK;
}

void mpm_renderer_destroy(mpm_renderer* r) {
    if (!r) return;
    cudaSetDevice(r->device);
    for (void* p : {(void*)r->zbuf, (void*)r->depth, (void*)r->tmp, (void*)r->fin, (void*)r->rgb, (void*)r->bg,
                    (void*)r->base, (void*)r->odepth, (void*)r->okey, (void*)r->otris, (void*)r->ocolor})
        if (p) cudaFree(p);
    delete r;
}

const char* mpm_renderer_last_error(const mpm_renderer* r) { return r ? r->last_error.c_str() : ""; }

// Draws the obstacle triangles (if any) over the base image into the
// background texture and the obstacle depth buffer; without obstacles the
// background is the base image.
static mpm_status draw_background(mpm_renderer* r) {
    const size_t npix = (size_t)r->prm.width * r->prm.height;
    if (r->ntris == 0) {
        RK(r, cudaMemcpy(r->bg, r->base, npix * 3, cudaMemcpyDeviceToDevice));
        return MPM_OK;
    }
    RK(r, cudaMemset(r->okey, 0xff, npix * sizeof(unsigned long long)));
    obstacle_raster_kernel<<<(r->ntris + 127) / 128, 128>>>(r->otris, r->ntris, r->cam, r->okey);
    obstacle_resolve_kernel<<<(unsigned)((npix + 255) / 256), 256>>>(r->okey, r->ocolor, r->base, (long long)npix, r->bg,
                                                                     r->odepth);
    RK(r, cudaGetLastError());
    RK(r, cudaDeviceSynchronize());
    return MPM_OK;
}

mpm_status mpm_renderer_set_background(mpm_renderer* r, const uint8_t* rgb8_host) {
    if (!r || !rgb8_host) return rfail(r, MPM_ERR_INVALID_ARGUMENT, "renderer and image must be non-NULL");
    RK(r, cudaSetDevice(r->device));
    RK(r, cudaMemcpy(r->base, rgb8_host, (size_t)r->prm.width * r->prm.height * 3, cudaMemcpyHostToDevice));
    return draw_background(r);
}

mpm_status mpm_renderer_set_obstacles(mpm_renderer* r, const float* tris_host, int64_t t, const float* rgb_host) {
    if (!r || t < 0 || (t > 0 && !tris_host) || t > 0x7fffffffLL)
        return rfail(r, MPM_ERR_INVALID_ARGUMENT, "bad obstacle arguments");
    RK(r, cudaSetDevice(r->device));
    for (void** p : {(void**)&r->otris, (void**)&r->ocolor, (void**)&r->okey, (void**)&r->odepth})
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
    r->ntris = 0;
    if (t == 0) return draw_background(r);
    // Flat colours (dot.frag): the world frame is the model-rotated grid
    // frame, the eye sits at (SX/2, SY/2, zoom) in it, the light direction is
    // the normalised world light.
    const mpm_render_params& p = r->prm;
    float M[16], T[16];
    const float cx = p.grid[0] / 2.0f, cy = p.grid[1] / 2.0f, cz = p.grid[2] / 2.0f;
    translation(M, cx, cy, cz);
    rotation(T, p.rotation_vertical, 1, 0, 0);
    mat_mul(M, T, M);
    rotation(T, p.rotation, 0, 1, 0);
    mat_mul(M, T, M);
    translation(T, -cx, -cy, -cz);
    mat_mul(M, T, M);
    const float eye[3] = {cx, cy, p.zoom_distance};
    float L[3] = {p.light_dir[0], p.light_dir[1], p.light_dir[2]};
    const float ll = std::sqrt(L[0] * L[0] + L[1] * L[1] + L[2] * L[2]);
    for (float& v : L) v /= ll;
    const float col[3] = {rgb_host ? rgb_host[0] : 0.5f, rgb_host ? rgb_host[1] : 0.5f, rgb_host ? rgb_host[2] : 0.5f};
    std::vector<unsigned char> rgb8((size_t)t * 3);
    for (int64_t i = 0; i < t; ++i) {
        float w[3][3];
        for (int k = 0; k < 3; ++k) {
            const float* v = tris_host + i * 9 + 3 * k;
            for (int a = 0; a < 3; ++a) w[k][a] = M[a] * v[0] + M[4 + a] * v[1] + M[8 + a] * v[2] + M[12 + a];
        }
        const float e1[3] = {w[1][0] - w[0][0], w[1][1] - w[0][1], w[1][2] - w[0][2]};
        const float e2[3] = {w[2][0] - w[0][0], w[2][1] - w[0][1], w[2][2] - w[0][2]};
        float n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const float nl = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nl > 0.0f)
            for (float& v : n) v /= nl;
        const float toward = n[0] * (eye[0] - w[0][0]) + n[1] * (eye[1] - w[0][1]) + n[2] * (eye[2] - w[0][2]);
        if (toward < 0.0f)
            for (float& v : n) v = -v;
        const float diff = std::max(n[0] * L[0] + n[1] * L[1] + n[2] * L[2], 0.0f);
        for (int c = 0; c < 3; ++c) rgb8[(size_t)i * 3 + c] = unorm8(0.3f * col[c] + diff * col[c]);
    }
    const size_t npix = (size_t)p.width * p.height;
    RK(r, cudaMalloc(&r->otris, (size_t)t * 9 * sizeof(float)));
    RK(r, cudaMalloc(&r->ocolor, (size_t)t * 3));
    RK(r, cudaMalloc(&r->okey, npix * sizeof(unsigned long long)));
    RK(r, cudaMalloc(&r->odepth, npix * sizeof(float)));
    RK(r, cudaMemcpy(r->otris, tris_host, (size_t)t * 9 * sizeof(float), cudaMemcpyHostToDevice));
    RK(r, cudaMemcpy(r->ocolor, rgb8.data(), rgb8.size(), cudaMemcpyHostToDevice));
    r->ntris = (int)t;
    return draw_background(r);
}

mpm_status mpm_renderer_get_background(mpm_renderer* r, uint8_t* rgb8_host, float* depth_host) {
    if (!r) return rfail(r, MPM_ERR_INVALID_ARGUMENT, "renderer is NULL");
    RK(r, cudaSetDevice(r->device));
    RK(r, cudaDeviceSynchronize());
    const size_t npix = (size_t)r->prm.width * r->prm.height;
    if (rgb8_host) RK(r, cudaMemcpy(rgb8_host, r->bg, npix * 3, cudaMemcpyDeviceToHost));
    if (depth_host) {
        if (r->odepth) {
            RK(r, cudaMemcpy(depth_host, r->odepth, npix * sizeof(float), cudaMemcpyDeviceToHost));
        } else {
            for (size_t i = 0; i < npix; ++i) depth_host[i] = 1.0f;
        }
    }
    return MPM_OK;
}

mpm_status mpm_render_points(mpm_renderer* r, const float* xyz_device, int64_t n, void* stream) {
    if (!r || (n > 0 && !xyz_device) || n < 0) return rfail(r, MPM_ERR_INVALID_ARGUMENT, "bad render arguments");
    RK(r, cudaSetDevice(r->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int w = r->prm.width, h = r->prm.height;
    const long long npix = (long long)w * h;
    RK(r, cudaMemsetAsync(r->zbuf, 0, npix * sizeof(unsigned), st));
    if (n > 0) splat_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(xyz_device, n, r->cam, r->zbuf);
    resolve_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(r->zbuf, npix, r->depth);
    const dim3 blk(32, 8), grd((w + 31) / 32, (h + 7) / 8);
    blur_kernel<<<grd, blk, 0, st>>>(r->depth, r->tmp, w, h, 1, 0, r->prm.filter_size, r->prm.depth_falloff);
    blur_kernel<<<grd, blk, 0, st>>>(r->tmp, r->fin, w, h, 0, 1, r->prm.filter_size, r->prm.depth_falloff);
    composite_kernel<<<grd, blk, 0, st>>>(r->fin, r->bg, w, h, r->cam.p00, r->cam.p11, r->cam.p22, r->cam.p32,
                                          r->light[0], r->light[1], r->light[2], r->odepth, r->rgb);
    RK(r, cudaGetLastError());
    return MPM_OK;
}

mpm_status mpm_render_frame(mpm_renderer* r, mpm_engine* engine) {
    if (!r || !engine) return rfail(r, MPM_ERR_INVALID_ARGUMENT, "renderer and engine must be non-NULL");
    const float* pos = mpm_positions_device(engine);
    const int64_t n = mpm_num_particles(engine);
    return mpm_render_points(r, pos, n, mpm_stream(engine));
}

// which: 0 = splat depth, 1 = after the horizontal blur, 2 = final depth.
mpm_status mpm_renderer_get_depth(mpm_renderer* r, int32_t which, float* host) {
    if (!r || !host || which < 0 || which > 2) return rfail(r, MPM_ERR_INVALID_ARGUMENT, "bad depth request");
    RK(r, cudaSetDevice(r->device));
    RK(r, cudaDeviceSynchronize());
    const size_t npix = (size_t)r->prm.width * r->prm.height;
    const float* src = which == 0 ? r->depth : (which == 1 ? r->tmp : r->fin);
    RK(r, cudaMemcpy(host, src, npix * sizeof(float), cudaMemcpyDeviceToHost));
    return MPM_OK;
}

mpm_status mpm_renderer_get_image(mpm_renderer* r, float* rgb_host, uint8_t* rgb8_host) {
    if (!r) return rfail(r, MPM_ERR_INVALID_ARGUMENT, "renderer is NULL");
    RK(r, cudaSetDevice(r->device));
    RK(r, cudaDeviceSynchronize());
    const size_t npix = (size_t)r->prm.width * r->prm.height;
    std::vector<float> tmp;
    float* dst = rgb_host;
    if (!dst) {
        tmp.resize(npix * 3);
        dst = tmp.data();
    }
    RK(r, cudaMemcpy(dst, r->rgb, npix * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    if (rgb8_host)
        for (size_t i = 0; i < npix * 3; ++i) rgb8_host[i] = unorm8(dst[i]);
    return MPM_OK;
}

}  // extern "C"

// Scene construction from a config's WATER= / OBJECT= entries: the part of
// Simulation::Simulation() (Simulation.cpp:4-38) that turns OBJ models into
// the particle buffer and the obstacle triangles.
//
//   WATER:  ObjLoader::loadObj -> VoxelEngine::voxelize(obj, 100) (surface
//           voxels, VoxelEngine.cpp:120-243) -> VoxelEngine::normalize
//           (centre, scale to SIZE_X, scale the longest side to `scale`,
//           displace, snap to the lattice of step getInt("RESOLUTION") with a
//           5x5x5 dilation, VoxelEngine.cpp:245-494) -> MergeVoxelData ->
//           VoxelPipeline::process (26 planes, VoxelPipeline.cpp:5-33)
//   OBJECT: ObjLoader::loadObj -> VoxelEngine::extractTriangles
//           (VoxelEngine.cpp:860-898) -> VoxelEngine::normalize(triangles)
//           (VoxelEngine.cpp:601-827, culls triangles with no vertex inside
//           [0, SIZE_X]^3) -> MergeTriangles
//
// The triangle-box tests of the voxelization and the dilation run on the GPU
// (this file is compiled without FMA contraction, so every float operation
// rounds as the reference's host code does); OBJ parsing and the per-triangle
// transform are host code.  The reference's std::set of lattice points
// becomes a bit set over the lattice, read back in the set's (x, y, z)
// lexicographic order.
//
// OBJ reading restates what the reference gets from tinyobjloader (a vcpkg
// dependency, not part of the reference tree; LoadObj with triangulation on):
// `v` lines give x y z (further values ignored; a field that does not parse
// reads 0), `f` lines give vertex indices (1-based, negative = relative, the
// forms v, v/t, v//n, v/t/n; an index 0 fails the load); a face of 4 vertices
// is split along its shorter diagonal ([0,1,2],[0,2,3] if |v2-v0|^2 < |v3-v1|^2,
// else [0,1,3],[1,2,3]); faces of fewer than 3 vertices are dropped.  Numbers
// are read with tinyobjloader's published scheme (mantissa digits accumulated
// in double, fraction digits scaled by a table of 10^-k, exponent applied as
// ldexp(m * 5^e, e)), then rounded to float.  Differences: faces of more than
// 4 vertices are split as a fan (tinyobjloader clips ears; for a planar convex
// polygon both cover the same set), and an index beyond the vertices read so
// far fails the load (the reference reads out of bounds).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "kernels.h"

namespace mpm {
bool config_text_int(const char* text, const char* key, int32_t* out, std::string& err);
}

struct mpm_mesh {
    std::vector<float> v;    // x y z per vertex (every `v` line)
    std::vector<int32_t> f;  // 3 vertex indices per triangle, 0-based
};

struct mpm_points {
    std::vector<float> p;  // x y z per point
};

struct mpm_scene_data {
    std::vector<float> p;     // particle positions, x y z per particle
    std::vector<float> tris;  // 9 floats per triangle
    std::string log;
};

namespace {

thread_local std::string g_scene_error;

mpm_status fail(mpm_status s, const std::string& msg) {
    g_scene_error = msg;
    mpm::set_global_error(msg);
    return s;
}

// ------------------------------------------------------------- OBJ ----
bool is_digit(char c) { return c >= '0' && c <= '9'; }

// tinyobjloader's number scheme on [s, e).
bool parse_double(const char* s, const char* e, double* result) {
    if (s >= e) return false;
    double mant = 0.0;
    int expo = 0;
    char sign = '+', exp_sign = '+';
    const char* cur = s;
    int read = 0;
    bool leading_dot = false;
    if (*cur == '+' || *cur == '-') {
        sign = *cur;
        ++cur;
        if (cur != e && *cur == '.') leading_dot = true;
    } else if (is_digit(*cur)) {
    } else if (*cur == '.') {
        leading_dot = true;
    } else {
        return false;
    }
    bool more = cur != e;
    if (!leading_dot) {
        while (more && is_digit(*cur)) {
            mant = mant * 10 + (*cur - '0');
            ++cur;
            ++read;
            more = cur != e;
        }
        if (read == 0) return false;
    }
    if (!more) goto assemble;
    if (*cur == '.') {
        static const double kPow10Neg[] = {1.0, 0.1, 0.01, 0.001, 0.0001, 0.00001, 0.000001, 0.0000001};
        ++cur;
        read = 1;
        more = cur != e;
        while (more && is_digit(*cur)) {
            mant += (*cur - '0') * (read < 8 ? kPow10Neg[read] : std::pow(10.0, -read));
            ++read;
            ++cur;
            more = cur != e;
        }
    } else if (*cur == 'e' || *cur == 'E') {
    } else {
        goto assemble;
    }
    if (!more) goto assemble;
    if (*cur == 'e' || *cur == 'E') {
        ++cur;
        more = cur != e;
        if (more && (*cur == '+' || *cur == '-')) {
            exp_sign = *cur;
            ++cur;
        } else if (more && is_digit(*cur)) {
        } else {
            return false;
        }
        read = 0;
        more = cur != e;
        while (more && is_digit(*cur)) {
            if (expo > INT_MAX / 10) return false;
            expo = expo * 10 + (*cur - '0');
            ++cur;
            ++read;
            more = cur != e;
        }
        expo *= exp_sign == '+' ? 1 : -1;
        if (read == 0) return false;
    }
assemble:
    *result = (sign == '+' ? 1 : -1) * (expo ? std::ldexp(mant * std::pow(5.0, expo), expo) : mant);
    return true;
}

float parse_real(const char*& tok, double def) {
    tok += std::strspn(tok, " \t");
    const char* end = tok + std::strcspn(tok, " \t\r");
    double v = def;
    parse_double(tok, end, &v);
    tok = end;
    return (float)v;
}

// One index field: 1-based or negative (relative to n); 0 fails.
bool fix_index(long idx, long n, long* out) {
    if (idx > 0) {
        *out = idx - 1;
        return true;
    }
    if (idx == 0) return false;
    *out = n + idx;
    return true;
}

bool parse_vertex_ref(const char*& tok, long nv, long nvt, long nvn, long* vi) {
    if (!fix_index(std::strtol(tok, nullptr, 10), nv, vi)) return false;
    tok += std::strcspn(tok, "/ \t\r");
    if (tok[0] != '/') return true;
    ++tok;
    long dummy = 0;
    if (tok[0] == '/') {
        ++tok;
        if (!fix_index(std::strtol(tok, nullptr, 10), nvn, &dummy)) return false;
        tok += std::strcspn(tok, "/ \t\r");
        return true;
    }
    if (!fix_index(std::strtol(tok, nullptr, 10), nvt, &dummy)) return false;
    tok += std::strcspn(tok, "/ \t\r");
    if (tok[0] != '/') return true;
    ++tok;
    if (!fix_index(std::strtol(tok, nullptr, 10), nvn, &dummy)) return false;
    tok += std::strcspn(tok, "/ \t\r");
    return true;
}

bool parse_obj(std::istream& in, mpm_mesh& m, std::string& err) {
    std::string line;
    long nvt = 0, nvn = 0, lineno = 0;
    std::vector<long> face;
    while (std::getline(in, line)) {
        ++lineno;
        while (!line.empty() && (line.back() == '\r' || line.back() == '\n')) line.pop_back();
        const char* tok = line.c_str();
        tok += std::strspn(tok, " \t");
        if (tok[0] == '\0' || tok[0] == '#') continue;
        const bool sp1 = tok[1] == ' ' || tok[1] == '\t';
        if (tok[0] == 'v' && sp1) {
            tok += 2;
            const float x = parse_real(tok, 0.0), y = parse_real(tok, 0.0), z = parse_real(tok, 0.0);
            m.v.push_back(x);
            m.v.push_back(y);
            m.v.push_back(z);
        } else if (tok[0] == 'v' && tok[1] == 't' && (tok[2] == ' ' || tok[2] == '\t')) {
            ++nvt;
        } else if (tok[0] == 'v' && tok[1] == 'n' && (tok[2] == ' ' || tok[2] == '\t')) {
            ++nvn;
        } else if (tok[0] == 'f' && sp1) {
            tok += 2;
            tok += std::strspn(tok, " \t");
            face.clear();
            const long nv = (long)(m.v.size() / 3);
            while (tok[0] != '\0' && tok[0] != '\r' && tok[0] != '\n') {
                long vi = 0;
                if (!parse_vertex_ref(tok, nv, nvt, nvn, &vi)) {
                    err = "OBJ line " + std::to_string(lineno) + ": malformed face index";
                    return false;
                }
                if (vi < 0 || vi >= nv) {
                    err = "OBJ line " + std::to_string(lineno) + ": face index outside the vertices read so far";
                    return false;
                }
                face.push_back(vi);
                tok += std::strspn(tok, " \t\r");
            }
            const size_t k = face.size();
            if (k < 3) continue;
            if (k == 4) {
                const float* v0 = &m.v[3 * face[0]];
                const float* v1 = &m.v[3 * face[1]];
                const float* v2 = &m.v[3 * face[2]];
                const float* v3 = &m.v[3 * face[3]];
                const float e02x = v2[0] - v0[0], e02y = v2[1] - v0[1], e02z = v2[2] - v0[2];
                const float e13x = v3[0] - v1[0], e13y = v3[1] - v1[1], e13z = v3[2] - v1[2];
                const float s02 = e02x * e02x + e02y * e02y + e02z * e02z;
                const float s13 = e13x * e13x + e13y * e13y + e13z * e13z;
                const long t[6] = {face[0], face[1], face[2], face[0], face[2], face[3]};
                const long u[6] = {face[0], face[1], face[3], face[1], face[2], face[3]};
                const long* pick = s02 < s13 ? t : u;
                for (int i = 0; i < 6; ++i) m.f.push_back((int32_t)pick[i]);
            } else {
                for (size_t i = 2; i < k; ++i) {
                    m.f.push_back((int32_t)face[0]);
                    m.f.push_back((int32_t)face[i - 1]);
                    m.f.push_back((int32_t)face[i]);
                }
            }
        }
    }
    return true;
}

std::vector<float> mesh_triangles(const mpm_mesh& m) {
    std::vector<float> t(m.f.size() * 3);
    for (size_t i = 0; i < m.f.size(); ++i)
        for (int c = 0; c < 3; ++c) t[3 * i + c] = m.v[3 * (size_t)m.f[i] + c];
    return t;
}

// ------------------------------------------------------ voxelization ----
struct VoxGrid {
    float minx, miny, minz, res;
    int gx, gy, gz;
};

// std::min / std::max on floats: (b < a) ? b : a and (a < b) ? b : a.
__host__ __device__ inline float min_std(float a, float b) { return (b < a) ? b : a; }
__host__ __device__ inline float max_std(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ inline float min3f(float a, float b, float c) { return min_std(min_std(a, b), c); }
__host__ __device__ inline float max3f(float a, float b, float c) { return max_std(max_std(a, b), c); }

// Separating-axis triangle / box test (VoxelEngine::triangleAABBIntersection,
// VoxelEngine.cpp:902-962): 9 edge-cross axes, the 3 box axes, the plane.
__device__ bool tri_box(const float* t, float bminx, float bminy, float bminz, float bmaxx, float bmaxy,
                        float bmaxz) {
    const float cx = (bminx + bmaxx) * 0.5f, cy = (bminy + bmaxy) * 0.5f, cz = (bminz + bmaxz) * 0.5f;
    const float hx = (bmaxx - bminx) * 0.5f, hy = (bmaxy - bminy) * 0.5f, hz = (bmaxz - bminz) * 0.5f;
    const float v0x = t[0] - cx, v0y = t[1] - cy, v0z = t[2] - cz;
    const float v1x = t[3] - cx, v1y = t[4] - cy, v1z = t[5] - cz;
    const float v2x = t[6] - cx, v2y = t[7] - cy, v2z = t[8] - cz;
    const float e[3][3] = {{v1x - v0x, v1y - v0y, v1z - v0z},
                           {v2x - v1x, v2y - v1y, v2z - v1z},
                           {v0x - v2x, v0y - v2y, v0z - v2z}};
    for (int k = 0; k < 3; ++k) {
        const float ax[3][3] = {{0.0f, -e[k][2], e[k][1]}, {e[k][2], 0.0f, -e[k][0]}, {-e[k][1], e[k][0], 0.0f}};
        for (int a = 0; a < 3; ++a) {
            const float p0 = v0x * ax[a][0] + v0y * ax[a][1] + v0z * ax[a][2];
            const float p1 = v1x * ax[a][0] + v1y * ax[a][1] + v1z * ax[a][2];
            const float p2 = v2x * ax[a][0] + v2y * ax[a][1] + v2z * ax[a][2];
            const float r = hx * fabsf(ax[a][0]) + hy * fabsf(ax[a][1]) + hz * fabsf(ax[a][2]);
            if (max_std(-max3f(p0, p1, p2), min3f(p0, p1, p2)) > r) return false;
        }
    }
    if (max3f(v0x, v1x, v2x) < -hx || min3f(v0x, v1x, v2x) > hx) return false;
    if (max3f(v0y, v1y, v2y) < -hy || min3f(v0y, v1y, v2y) > hy) return false;
    if (max3f(v0z, v1z, v2z) < -hz || min3f(v0z, v1z, v2z) > hz) return false;
    const float nx = e[0][1] * e[1][2] - e[0][2] * e[1][1];
    const float ny = e[0][2] * e[1][0] - e[0][0] * e[1][2];
    const float nz = e[0][0] * e[1][1] - e[0][1] * e[1][0];
    const float d = nx * v0x + ny * v0y + nz * v0z;
    const float r = hx * fabsf(nx) + hy * fabsf(ny) + hz * fabsf(nz);
    return !(fabsf(d) > r);
}

// One warp per triangle: every voxel of the triangle's index box that the
// triangle touches gets its bit (voxel (x, y, z) = bit (z*gy + y)*gx + x).
__global__ void voxel_mark_kernel(const float* __restrict__ tris, int nt, VoxGrid g, uint32_t* __restrict__ bits) {
    const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nt) return;
    float t[9];
    for (int k = 0; k < 9; ++k) t[k] = tris[w * 9 + k];
    const float tminx = min3f(t[0], t[3], t[6]), tminy = min3f(t[1], t[4], t[7]), tminz = min3f(t[2], t[5], t[8]);
    const float tmaxx = max3f(t[0], t[3], t[6]), tmaxy = max3f(t[1], t[4], t[7]), tmaxz = max3f(t[2], t[5], t[8]);
    const int x0 = max(0, (int)floorf((tminx - g.minx) / g.res));
    const int y0 = max(0, (int)floorf((tminy - g.miny) / g.res));
    const int z0 = max(0, (int)floorf((tminz - g.minz) / g.res));
    const int x1 = min(g.gx - 1, (int)ceilf((tmaxx - g.minx) / g.res));
    const int y1 = min(g.gy - 1, (int)ceilf((tmaxy - g.miny) / g.res));
    const int z1 = min(g.gz - 1, (int)ceilf((tmaxz - g.minz) / g.res));
    if (x1 < x0 || y1 < y0 || z1 < z0) return;
    const long long nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1;
    for (long long k = lane; k < nx * ny * nz; k += 32) {
        const int x = x0 + (int)(k % nx), y = y0 + (int)((k / nx) % ny), z = z0 + (int)(k / (nx * ny));
        const float bx = g.minx + (float)x * g.res, by = g.miny + (float)y * g.res, bz = g.minz + (float)z * g.res;
        if (tri_box(t, bx, by, bz, bx + g.res, by + g.res, bz + g.res)) {
            const long long idx = ((long long)z * g.gy + y) * g.gx + x;
            atomicOr(bits + (idx >> 5), 1u << (idx & 31));
        }
    }
}

// -------------------------------------------------------- normalize ----
__device__ __forceinline__ unsigned ord_enc(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
inline float ord_dec(unsigned u) {
    const unsigned b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

// mm[0..2] = min x, y, z, mm[3..5] = max (order-preserving encodings).
__global__ void minmax_kernel(const float* __restrict__ p, long long n, unsigned* __restrict__ mm) {
    unsigned lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) {
            const unsigned u = ord_enc(p[i * 3 + c]);
            lo[c] = min(lo[c], u);
            hi[c] = max(hi[c], u);
        }
    for (int c = 0; c < 3; ++c) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = min(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = max(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(mm + c, lo[c]);
            atomicMax(mm + 3 + c, hi[c]);
        }
    }
}

// p = (p - centre) * scale + half, one rounding per operation (VoxelEngine.cpp:298-306).
__global__ void recentre_kernel(float* __restrict__ p, long long n, float cx, float cy, float cz, float s,
                                float half) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float c[3] = {cx, cy, cz};
    for (int k = 0; k < 3; ++k) {
        float v = p[i * 3 + k];
        v = v - c[k];
        v = v * s;
        v = v + half;
        p[i * 3 + k] = v;
    }
}

// Second scaling about half, displacement, lattice snap with clamping and the
// 5x5x5 dilation into the lattice bit set (x-major: bit (x*L + y)*L + z,
// L = M + 1) (VoxelEngine.cpp:336-433).
__global__ void snap_dilate_kernel(const float* __restrict__ p, long long n, float half, float s2, float dx, float dy,
                                   float dz, float step, int M, uint32_t* __restrict__ lattice) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float d[3] = {dx, dy, dz};
    int gi[3];
    for (int k = 0; k < 3; ++k) {
        float v = p[i * 3 + k];
        v = v - half;
        v = v * s2;
        v = v + half;
        v = v + d[k];
        gi[k] = min(M, max(0, (int)roundf(v / step)));
    }
    const long long L = (long long)M + 1;
    for (int a = -2; a <= 2; ++a)
        for (int b = -2; b <= 2; ++b)
            for (int c = -2; c <= 2; ++c) {
                const int x = gi[0] + a, y = gi[1] + b, z = gi[2] + c;
                if (x < 0 || x > M || y < 0 || y > M || z < 0 || z > M) continue;
                const long long idx = ((long long)x * L + y) * L + z;
                atomicOr(lattice + (idx >> 5), 1u << (idx & 31));
            }
}

inline int blocks_of(long long n, int t) { return (int)((n + t - 1) / t); }

// Device buffers of one call, freed on every exit path.
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

#define SK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            cudaGetLastError();                                                                       \
            return fail(e_ == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA,       \
                        std::string("CUDA error in ") + #call + ": " + cudaGetErrorString(e_));       \
        }                                                                                             \
    } while (0)

mpm_status voxelize(const mpm_mesh& m, float resolution, int device, std::vector<float>& out) {
    out.clear();
    if (m.v.empty()) return fail(MPM_ERR_BAD_CONFIG, "voxelize: the mesh has no vertices");
    if (!(resolution > 0.0f)) return fail(MPM_ERR_INVALID_ARGUMENT, "voxelize: resolution must be positive");
    // calculateBoundingBox over every vertex (VoxelEngine.cpp:829-858).
    float mn[3] = {m.v[0], m.v[1], m.v[2]}, mx[3] = {m.v[0], m.v[1], m.v[2]};
    for (size_t i = 0; i < m.v.size(); i += 3)
        for (int c = 0; c < 3; ++c) {
            mn[c] = min_std(mn[c], m.v[i + c]);
            mx[c] = max_std(mx[c], m.v[i + c]);
        }
    const float sx = mx[0] - mn[0], sy = mx[1] - mn[1], sz = mx[2] - mn[2];
    const float maxsize = max_std(sx, max_std(sy, sz));
    const float res = maxsize / resolution;
    if (!(res > 0.0f) || !std::isfinite(res))
        return fail(MPM_ERR_BAD_CONFIG, "voxelize: the mesh's bounding box is a point (voxel size 0)");
    const float fg[3] = {std::ceil((mx[0] - mn[0]) / res), std::ceil((mx[1] - mn[1]) / res),
                         std::ceil((mx[2] - mn[2]) / res)};
    for (float f : fg)
        if (!(f >= 0.0f && f < 65536.0f)) return fail(MPM_ERR_BAD_CONFIG, "voxelize: voxel grid too large");
    VoxGrid g{mn[0], mn[1], mn[2], res, (int)fg[0], (int)fg[1], (int)fg[2]};
    const long long total = (long long)g.gx * g.gy * g.gz;
    if (total > (1LL << 34)) return fail(MPM_ERR_BAD_CONFIG, "voxelize: voxel grid too large");
    const long long nt = (long long)(m.f.size() / 3);
    if (total == 0 || nt == 0) return MPM_OK;
    if (nt > INT_MAX) return fail(MPM_ERR_BAD_CONFIG, "voxelize: too many triangles");
    SK(cudaSetDevice(device));
    const std::vector<float> tris = mesh_triangles(m);
    const size_t words = (size_t)((total + 31) / 32);
    DevBuf d_tris, d_bits;
    SK(cudaMalloc(&d_tris.p, tris.size() * sizeof(float)));
    SK(cudaMalloc(&d_bits.p, words * sizeof(uint32_t)));
    SK(cudaMemcpy(d_tris.p, tris.data(), tris.size() * sizeof(float), cudaMemcpyHostToDevice));
    SK(cudaMemset(d_bits.p, 0, words * sizeof(uint32_t)));
    voxel_mark_kernel<<<blocks_of(nt * 32, 256), 256>>>(static_cast<const float*>(d_tris.p), (int)nt, g,
                                                         static_cast<uint32_t*>(d_bits.p));
    SK(cudaGetLastError());
    std::vector<uint32_t> bits(words);
    SK(cudaMemcpy(bits.data(), d_bits.p, words * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    // Voxel centres in the reference's z, y, x order (VoxelEngine.cpp:208-225).
    for (size_t wd = 0; wd < words; ++wd) {
        uint32_t b = bits[wd];
        while (b) {
            const int k = __builtin_ctz(b);
            b &= b - 1;
            const long long idx = (long long)wd * 32 + k;
            const int x = (int)(idx % g.gx), y = (int)((idx / g.gx) % g.gy), z = (int)(idx / ((long long)g.gx * g.gy));
            out.push_back(g.minx + ((float)x + 0.5f) * res);
            out.push_back(g.miny + ((float)y + 0.5f) * res);
            out.push_back(g.minz + ((float)z + 0.5f) * res);
        }
    }
    return MPM_OK;
}

mpm_status normalize_points(std::vector<float>& p, float size, float scale, const float disp[3], int step,
                            int device) {
    const long long n = (long long)(p.size() / 3);
    if (n == 0) return MPM_OK;
    if (step < 1)
        return fail(MPM_ERR_BAD_CONFIG,
                    "lattice step getInt(\"RESOLUTION\") is below 1 (the reference divides by it, "
                    "VoxelEngine.cpp:369-381)");
    SK(cudaSetDevice(device));
    DevBuf d_p, d_mm;
    SK(cudaMalloc(&d_p.p, p.size() * sizeof(float)));
    SK(cudaMalloc(&d_mm.p, 6 * sizeof(unsigned)));
    SK(cudaMemcpy(d_p.p, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice));
    float* dp = static_cast<float*>(d_p.p);
    unsigned* dmm = static_cast<unsigned*>(d_mm.p);
    const unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    unsigned mm[6];
    const int mgrid = std::min(blocks_of(n, 256), 148 * 4);
    auto bounds = [&](float* lo, float* hi) -> mpm_status {
        SK(cudaMemcpy(dmm, init, sizeof(init), cudaMemcpyHostToDevice));
        minmax_kernel<<<mgrid, 256>>>(dp, n, dmm);
        SK(cudaGetLastError());
        SK(cudaMemcpy(mm, dmm, sizeof(mm), cudaMemcpyDeviceToHost));
        for (int c = 0; c < 3; ++c) lo[c] = ord_dec(mm[c]), hi[c] = ord_dec(mm[3 + c]);
        return MPM_OK;
    };
    float lo[3], hi[3];
    mpm_status st = bounds(lo, hi);
    if (st != MPM_OK) return st;
    const float maxdim = max3f(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    if (maxdim < 1e-6f) return MPM_OK;  // VoxelEngine.cpp:280-284: left as it is
    const float ns = size / maxdim;
    const float half = size * 0.5f;
    recentre_kernel<<<blocks_of(n, 256), 256>>>(dp, n, (lo[0] + hi[0]) * 0.5f, (lo[1] + hi[1]) * 0.5f,
                                                (lo[2] + hi[2]) * 0.5f, ns, half);
    SK(cudaGetLastError());
    if ((st = bounds(lo, hi)) != MPM_OK) return st;
    const float cur = max3f(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    const float s2 = (cur > 1e-6f) ? (scale / cur) : 1.0f;
    const float gres = (float)step;
    const int M = (int)(size / gres);
    if (M < 0 || M > 4095) return fail(MPM_ERR_BAD_CONFIG, "lattice too large (SIZE_X / RESOLUTION > 4095)");
    const long long L = (long long)M + 1;
    const size_t words = (size_t)((L * L * L + 31) / 32);
    DevBuf d_lat;
    SK(cudaMalloc(&d_lat.p, words * sizeof(uint32_t)));
    SK(cudaMemset(d_lat.p, 0, words * sizeof(uint32_t)));
    snap_dilate_kernel<<<blocks_of(n, 256), 256>>>(dp, n, half, s2, disp[0], disp[1], disp[2], gres, M,
                                                   static_cast<uint32_t*>(d_lat.p));
    SK(cudaGetLastError());
    std::vector<uint32_t> bits(words);
    SK(cudaMemcpy(bits.data(), d_lat.p, words * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    p.clear();
    for (size_t wd = 0; wd < words; ++wd) {
        uint32_t b = bits[wd];
        while (b) {
            const int k = __builtin_ctz(b);
            b &= b - 1;
            const long long idx = (long long)wd * 32 + k;
            const int x = (int)(idx / (L * L)), y = (int)((idx / L) % L), z = (int)(idx % L);
            p.push_back((float)x * gres);
            p.push_back((float)y * gres);
            p.push_back((float)z * gres);
        }
    }
    return MPM_OK;
}

// VoxelEngine::normalize(std::vector<Triangle>&, ...) (VoxelEngine.cpp:601-827).
void normalize_triangles(std::vector<float>& t, float size, float scale, const float disp[3]) {
    const size_t nt = t.size() / 9;
    if (nt == 0) return;
    auto bounds = [&](float* lo, float* hi) {
        for (int c = 0; c < 3; ++c) lo[c] = hi[c] = t[c];
        for (size_t i = 0; i < nt; ++i) {
            const float* q = &t[9 * i];
            for (int c = 0; c < 3; ++c) {
                lo[c] = min_std(min3f(lo[c], q[c], q[3 + c]), q[6 + c]);
                hi[c] = max_std(max3f(hi[c], q[c], q[3 + c]), q[6 + c]);
            }
        }
    };
    float lo[3], hi[3];
    bounds(lo, hi);
    const float maxdim = max3f(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    if (maxdim < 1e-6f) return;
    const float ns = size / maxdim;
    const float ctr[3] = {(lo[0] + hi[0]) * 0.5f, (lo[1] + hi[1]) * 0.5f, (lo[2] + hi[2]) * 0.5f};
    const float half = size * 0.5f;
    for (size_t i = 0; i < nt * 3; ++i)
        for (int c = 0; c < 3; ++c) {
            float v = t[3 * i + c];
            v = v - ctr[c];
            v = v * ns;
            v = v + half;
            t[3 * i + c] = v;
        }
    bounds(lo, hi);
    const float cur = max3f(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    const float s2 = (cur > 1e-6f) ? (scale / cur) : 1.0f;
    for (size_t i = 0; i < nt * 3; ++i)
        for (int c = 0; c < 3; ++c) {
            float v = t[3 * i + c];
            v = v - half;
            v = v * s2;
            v = v + half;
            t[3 * i + c] = v;
        }
    for (size_t i = 0; i < nt * 3; ++i)
        for (int c = 0; c < 3; ++c) t[3 * i + c] = t[3 * i + c] + disp[c];
    std::vector<float> keep;
    keep.reserve(t.size());
    for (size_t i = 0; i < nt; ++i) {
        const float* q = &t[9 * i];
        bool any = false;
        for (int k = 0; k < 3; ++k) {
            const float* v = q + 3 * k;
            any = any || (v[0] >= 0.0f && v[0] <= size && v[1] >= 0.0f && v[1] <= size && v[2] >= 0.0f &&
                          v[2] <= size);
        }
        if (any) keep.insert(keep.end(), q, q + 9);
    }
    t.swap(keep);
}

mpm_status load_obj_file(const std::string& path, mpm_mesh& m) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return fail(MPM_ERR_IO, "cannot open OBJ file " + path);
    std::string err;
    if (!parse_obj(in, m, err)) return fail(MPM_ERR_BAD_CONFIG, path + ": " + err);
    return MPM_OK;
}

std::string join_path(const char* base, const std::string& p) {
    if (!base || !base[0] || (!p.empty() && p[0] == '/')) return p;
    std::string b = base;
    if (b.back() != '/') b.push_back('/');
    return b + p;
}

}  // namespace

extern "C" {

const char* mpm_scene_last_error(void) { return g_scene_error.c_str(); }

mpm_status mpm_mesh_load_obj(const char* path, mpm_mesh** out) {
    if (!path || !out) return fail(MPM_ERR_INVALID_ARGUMENT, "path and out must be non-NULL");
    *out = nullptr;
    auto* m = new mpm_mesh();
    const mpm_status s = load_obj_file(path, *m);
    if (s != MPM_OK) {
        delete m;
        return s;
    }
    *out = m;
    return MPM_OK;
}

mpm_status mpm_mesh_from_obj_text(const char* text, mpm_mesh** out) {
    if (!text || !out) return fail(MPM_ERR_INVALID_ARGUMENT, "text and out must be non-NULL");
    *out = nullptr;
    auto* m = new mpm_mesh();
    std::istringstream in(text);
    std::string err;
    if (!parse_obj(in, *m, err)) {
        delete m;
        return fail(MPM_ERR_BAD_CONFIG, err);
    }
    *out = m;
    return MPM_OK;
}

void mpm_mesh_free(mpm_mesh* m) { delete m; }

int64_t mpm_mesh_num_vertices(const mpm_mesh* m) { return m ? (int64_t)(m->v.size() / 3) : -1; }
int64_t mpm_mesh_num_triangles(const mpm_mesh* m) { return m ? (int64_t)(m->f.size() / 3) : -1; }

mpm_status mpm_mesh_get(const mpm_mesh* m, float* vertices3_host, int32_t* faces3_host, float* triangles9_host) {
    if (!m) return fail(MPM_ERR_INVALID_ARGUMENT, "mesh is NULL");
    if (vertices3_host) std::memcpy(vertices3_host, m->v.data(), m->v.size() * sizeof(float));
    if (faces3_host) std::memcpy(faces3_host, m->f.data(), m->f.size() * sizeof(int32_t));
    if (triangles9_host) {
        const std::vector<float> t = mesh_triangles(*m);
        std::memcpy(triangles9_host, t.data(), t.size() * sizeof(float));
    }
    return MPM_OK;
}

mpm_status mpm_voxelize(const mpm_mesh* m, float resolution, int32_t device, mpm_points** out) {
    if (!m || !out) return fail(MPM_ERR_INVALID_ARGUMENT, "mesh and out must be non-NULL");
    *out = nullptr;
    auto* pts = new mpm_points();
    const mpm_status s = voxelize(*m, resolution, device, pts->p);
    if (s != MPM_OK) {
        delete pts;
        return s;
    }
    *out = pts;
    return MPM_OK;
}

mpm_status mpm_points_create(const float* xyz_host, int64_t n, mpm_points** out) {
    if (!out || n < 0 || (n > 0 && !xyz_host)) return fail(MPM_ERR_INVALID_ARGUMENT, "bad points arguments");
    auto* pts = new mpm_points();
    pts->p.assign(xyz_host, xyz_host + 3 * n);
    *out = pts;
    return MPM_OK;
}

int64_t mpm_points_count(const mpm_points* p) { return p ? (int64_t)(p->p.size() / 3) : -1; }

mpm_status mpm_points_get(const mpm_points* p, float* xyz_host) {
    if (!p || (!p->p.empty() && !xyz_host)) return fail(MPM_ERR_INVALID_ARGUMENT, "bad points arguments");
    std::memcpy(xyz_host, p->p.data(), p->p.size() * sizeof(float));
    return MPM_OK;
}

void mpm_points_free(mpm_points* p) { delete p; }

mpm_status mpm_points_normalize(mpm_points* p, float normalize_size, float scale, const float* displacement3,
                                int32_t lattice_step, int32_t device) {
    if (!p || !displacement3) return fail(MPM_ERR_INVALID_ARGUMENT, "points and displacement must be non-NULL");
    return normalize_points(p->p, normalize_size, scale, displacement3, lattice_step, device);
}

mpm_status mpm_triangles_normalize(float* triangles9_host, int64_t* t, float normalize_size, float scale,
                                   const float* displacement3) {
    if (!t || *t < 0 || (*t > 0 && !triangles9_host) || !displacement3)
        return fail(MPM_ERR_INVALID_ARGUMENT, "bad triangle arguments");
    std::vector<float> v(triangles9_host, triangles9_host + 9 * *t);
    normalize_triangles(v, normalize_size, scale, displacement3);
    std::memcpy(triangles9_host, v.data(), v.size() * sizeof(float));
    *t = (int64_t)(v.size() / 9);
    return MPM_OK;
}

mpm_status mpm_scene_build(const char* config_text, const char* base_dir, int32_t device, mpm_scene_data** out) {
    if (!config_text || !out) return fail(MPM_ERR_INVALID_ARGUMENT, "config_text and out must be non-NULL");
    *out = nullptr;
    mpm_config cfg;
    std::vector<mpm_scene_entry> waters(4096), objects(4096);
    int32_t nw = 0, no = 0;
    char err[1024];
    mpm_status s = mpm_config_parse_string(config_text, &cfg, waters.data(), (int32_t)waters.size(), &nw,
                                           objects.data(), (int32_t)objects.size(), &no, err, sizeof(err));
    if (s != MPM_OK) return fail(s, err);
    if (nw > (int32_t)waters.size() || no > (int32_t)objects.size())
        return fail(MPM_ERR_BAD_CONFIG, "more than 4096 WATER or OBJECT entries");
    int32_t step = 0;
    std::string e2;
    if (!mpm::config_text_int(config_text, "RESOLUTION", &step, e2)) return fail(MPM_ERR_BAD_CONFIG, e2);
    const float size = (float)cfg.size_x;  // getInt("SIZE_X") for every axis (Simulation.cpp:94,114)
    auto* sd = new mpm_scene_data();
    for (int32_t i = 0; i < nw; ++i) {
        const mpm_scene_entry& en = waters[i];
        mpm_mesh m;
        std::vector<float> pts;
        const float disp[3] = {en.x, en.y, en.z};
        if ((s = load_obj_file(join_path(base_dir, en.model_path), m)) != MPM_OK ||
            (s = voxelize(m, 100.0f, device, pts)) != MPM_OK) {
            delete sd;
            return s;
        }
        if (pts.empty()) {
            delete sd;
            return fail(MPM_ERR_BAD_CONFIG, std::string("WATER model ") + en.model_path + " gave no voxels");
        }
        if ((s = normalize_points(pts, size, en.scale, disp, step, device)) != MPM_OK) {
            delete sd;
            return s;
        }
        sd->p.insert(sd->p.end(), pts.begin(), pts.end());
    }
    for (int32_t i = 0; i < no; ++i) {
        const mpm_scene_entry& en = objects[i];
        mpm_mesh m;
        const std::string path = join_path(base_dir, en.model_path);
        if (load_obj_file(path, m) != MPM_OK) {
            sd->log += "OBJECT " + std::string(en.model_path) + " skipped: " + g_scene_error + "\n";
            continue;  // Prepare_triangles returns no triangles (Simulation.cpp:100-105)
        }
        std::vector<float> t = mesh_triangles(m);
        const float disp[3] = {en.x, en.y, en.z};
        normalize_triangles(t, size, en.scale, disp);
        sd->tris.insert(sd->tris.end(), t.begin(), t.end());
    }
    g_scene_error.clear();
    *out = sd;
    return MPM_OK;
}

void mpm_scene_data_free(mpm_scene_data* d) { delete d; }
int64_t mpm_scene_data_num_particles(const mpm_scene_data* d) { return d ? (int64_t)(d->p.size() / 3) : -1; }
int64_t mpm_scene_data_num_triangles(const mpm_scene_data* d) { return d ? (int64_t)(d->tris.size() / 9) : -1; }
const char* mpm_scene_data_log(const mpm_scene_data* d) { return d ? d->log.c_str() : ""; }

mpm_status mpm_scene_data_state(const mpm_scene_data* d, float* soa26_host) {
    if (!d) return fail(MPM_ERR_INVALID_ARGUMENT, "scene data is NULL");
    const size_t n = d->p.size() / 3;
    if (n > 0 && !soa26_host) return fail(MPM_ERR_INVALID_ARGUMENT, "soa26_host is NULL");
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) soa26_host[c * n + i] = d->p[3 * i + c];
    std::memset(soa26_host + 3 * n, 0, 21 * n * sizeof(float));
    for (size_t i = 0; i < 2 * n; ++i) soa26_host[24 * n + i] = 1.0f;
    return MPM_OK;
}

mpm_status mpm_scene_data_triangles(const mpm_scene_data* d, float* triangles9_host) {
    if (!d) return fail(MPM_ERR_INVALID_ARGUMENT, "scene data is NULL");
    if (!d->tris.empty() && !triangles9_host) return fail(MPM_ERR_INVALID_ARGUMENT, "triangles9_host is NULL");
    std::memcpy(triangles9_host, d->tris.data(), d->tris.size() * sizeof(float));
    return MPM_OK;
}

}  // extern "C"

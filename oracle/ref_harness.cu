// ref_harness.cu - headless C entry points around the reference's own Engine.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together
// with the reference's unmodified engine.cu, kernels.cu, config.cu and
// game_configdata.cpp (read in place from the reference tree, -rdc because
// d_config is an extern __constant__, common.cuh:81-83) into
// oracle/_ref/libref_engine.so.  Parity tests use it as a second witness next
// to the CPU oracle, and `bench.py --impl reference` times it.
//
// What it restates from the reference application (not compilable here: it
// needs GL, GLFW, glm and tinyobjloader):
//  - Simulation::initDeviceParams (Simulation.cpp:56-77): SimConfig from the
//    config map, GRID_SIZE/GRID_NUMBER/GRID_BLOCKS injected with setNewInt,
//    uploadConfigToGPU;
//  - Simulation::Simulation's hand-off (Simulation.cpp:19-36): a new[] 26*n
//    buffer owned by Engine::init, then Engine::initSDF.
// Private members are read through the explicit-instantiation access rule
// ([temp.explicit]/12), which leaves the reference sources untouched.
#include <cuda_runtime.h>
#include <thrust/binary_search.h>
#include <thrust/device_vector.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/sort.h>

#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "game_configdata.h"

__global__ void setKeys(Particles p, int* keys, int number);                                   // kernels.cu:361
__global__ void makeSDF(float* sdfGrid, const Triangle* __restrict__ triangles, int triangleNumber);  // kernels.cu:282
__global__ void p2GTransferScatter(Particles p, Grid g, int number, int* sortedIndices);  // kernels.cu:6
__global__ void gridUpdate(Grid g);                                                      // kernels.cu:144
__global__ void g2PTransfer(Particles p, Grid g, int number, int* sortedIndices);        // kernels.cu:199
__global__ void emptyGrid(Grid g);                                                       // kernels.cu:311
__global__ void changeFormat(Particles p, float3* buf, int number);                      // kernels.cu:341

namespace {

template <typename Tag, typename Tag::type M>
struct Expose {
    friend typename Tag::type get(Tag) { return M; }
};
struct ValuesTag {
    typedef int* Engine::*type;
    friend type get(ValuesTag);
};
template struct Expose<ValuesTag, &Engine::d_values>;
struct SdfTag {
    typedef float* Engine::*type;
    friend type get(SdfTag);
};
template struct Expose<SdfTag, &Engine::d_sdf_buffer>;
struct PositionsTag {
    typedef float3* Engine::*type;
    friend type get(PositionsTag);
};
template struct Expose<PositionsTag, &Engine::positionsToOpenGL>;
struct MapTag {
    typedef std::unordered_map<std::string, std::string>* type;
    friend type get(MapTag);
};
template struct Expose<MapTag, &GameConfigData::configMap>;
struct WatersTag {
    typedef std::vector<ConfigObject>* type;
    friend type get(WatersTag);
};
template struct Expose<WatersTag, &GameConfigData::waters>;
struct ObjectsTag {
    typedef std::vector<ConfigObject>* type;
    friend type get(ObjectsTag);
};
template struct Expose<ObjectsTag, &GameConfigData::objects>;

Engine* g_engine = nullptr;
long g_n = 0;

// Simulation::initDeviceParams (Simulation.cpp:56-77).
void init_device_params() {
    SimConfig h;
    h.SIZE_X = GameConfigData::getInt("SIZE_X");
    h.SIZE_Y = GameConfigData::getInt("SIZE_Y");
    h.SIZE_Z = GameConfigData::getInt("SIZE_Z");
    h.PADDING = GameConfigData::getInt("PADDING");
    h.GRAVITY = GameConfigData::getFloat("GRAVITY");
    h.DT = GameConfigData::getFloat("DT");
    h.GAMMA = GameConfigData::getFloat("GAMMA");
    h.COMPRESSION = GameConfigData::getFloat("COMPRESSION");
    h.RESOLUTION = GameConfigData::getFloat("RESOLUTION");
    h.SUBSTEPS = GameConfigData::getInt("SUBSTEPS");
    h.SDF_RESOLUTION = GameConfigData::getInt("SDF_RESOLUTION");
    h.GRID_SIZE = h.SIZE_X * h.SIZE_Y * h.SIZE_Z * CELL_SIZE;
    h.GRID_NUMBER = h.SIZE_X * h.SIZE_Y * h.SIZE_Z;
    h.GRID_BLOCKS = (h.GRID_NUMBER + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK;
    GameConfigData::setNewInt("GRID_SIZE", std::to_string(h.GRID_SIZE));
    GameConfigData::setNewInt("GRID_NUMBER", std::to_string(h.GRID_NUMBER));
    GameConfigData::setNewInt("GRID_BLOCKS", std::to_string(h.GRID_BLOCKS));
    uploadConfigToGPU(h);
}

}  // namespace

extern "C" {

// Clears the reference's process-global config store.
void ref_config_reset() {
    get(MapTag())->clear();
    get(WatersTag())->clear();
    get(ObjectsTag())->clear();
}

// GameConfigData::setConfigDataFromFile on `path`.  Only call it with files
// the reference accepts: on a malformed entry it exits the process.
void ref_config_load(const char* path) {
    ref_config_reset();
    GameConfigData::setConfigDataFromFile(path);
}

// 1 if the key is present (getInt/getFloat exit on a missing key).
int ref_config_has(const char* key) { return get(MapTag())->count(key) ? 1 : 0; }
int ref_config_get_int(const char* key) { return GameConfigData::getInt(key); }
float ref_config_get_float(const char* key) { return GameConfigData::getFloat(key); }

// Copies up to max WATER (which=0) or OBJECT (which=1) entries as
// (scale, x, y, z) quadruples and their paths (NUL-separated, path_cap bytes).
int ref_config_entries(int which, float* vals, char* paths, int path_cap, int max) {
    std::vector<ConfigObject> v = which == 0 ? GameConfigData::getWaters() : GameConfigData::getObjects();
    int off = 0;
    for (int i = 0; i < (int)v.size() && i < max; ++i) {
        vals[4 * i + 0] = v[i].scale;
        vals[4 * i + 1] = v[i].x;
        vals[4 * i + 2] = v[i].y;
        vals[4 * i + 3] = v[i].z;
        const std::string& s = v[i].modelPath;
        if (off + (int)s.size() + 1 <= path_cap) {
            std::memcpy(paths + off, s.c_str(), s.size() + 1);
            off += (int)s.size() + 1;
        }
    }
    return (int)v.size();
}

// Builds an Engine on the loaded config and an n-particle 26-plane state.
// Returns 0, or -1 when the grid node count is not a multiple of 256: the
// reference's emptyGrid/gridUpdate have no bounds check (kernels.cu:311-318,
// 144-150) and would write out of bounds, so such grids are not run.
int ref_engine_create(long n, const float* soa26) {
    if (g_engine) {
        delete g_engine;
        g_engine = nullptr;
    }
    init_device_params();
    const long g = (long)GameConfigData::getInt("GRID_NUMBER");
    if (g % 256 != 0 || n <= 0) return -1;
    float* buf = new float[26 * n];
    std::memcpy(buf, soa26, sizeof(float) * 26 * n);
    g_engine = new Engine();
    g_engine->init((int)n, buf);  // takes ownership (engine.cu:38)
    g_n = n;
    return 0;
}

// Engine::initSDF (engine.cu:105-114).  With t == 0 the harness allocates the
// SDF and launches makeSDF with no triangles itself, exactly what initSDF
// does, without its zero-byte host copy from a null vector pointer.
int ref_engine_init_sdf(const float* tris, long t) {
    if (!g_engine) return -1;
    if (t > 0) {
        std::vector<Triangle> v((size_t)t);
        std::memcpy(v.data(), tris, sizeof(Triangle) * t);
        g_engine->initSDF(v);
    } else {
        float*& sdf = g_engine->*get(SdfTag());
        if (cudaMalloc((void**)&sdf, GameConfigData::getInt("GRID_SIZE")) != cudaSuccess) return -2;
        makeSDF<<<GameConfigData::getInt("GRID_BLOCKS"), THREADS_PER_BLOCK>>>(sdf, nullptr, 0);
        if (cudaDeviceSynchronize() != cudaSuccess) return -3;
    }
    return 0;
}

// Overwrites the engine's particle buffer (getBuffer, 26 planes of g_n
// floats) with a state as it is: Engine::init applies initFMatrices
// (kernels.cu:349-358), which resets F's diagonal, so a state taken after
// some substeps is loaded through init and then written over with this.
int ref_engine_set_state(const float* soa26) {
    if (!g_engine) return -1;
    return cudaMemcpy(g_engine->getBuffer(), soa26, sizeof(float) * 26 * g_n, cudaMemcpyHostToDevice) == cudaSuccess
               ? 0
               : -2;
}

int ref_engine_step(int nsub) {
    if (!g_engine) return -1;
    for (int i = 0; i < nsub; ++i) g_engine->step();
    return 0;
}

// Device time of nsub Engine::step() calls, CUDA events on the default stream.
float ref_engine_time_steps(int nsub) {
    if (!g_engine) return -1.0f;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    for (int i = 0; i < nsub; ++i) g_engine->step();
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

int ref_engine_get_state(float* out) {
    if (!g_engine) return -1;
    return cudaMemcpy(out, g_engine->getBuffer(), sizeof(float) * 26 * g_n, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -2;
}

int ref_engine_get_grid(float* out) {
    if (!g_engine) return -1;
    const long g = GameConfigData::getInt("GRID_NUMBER");
    return cudaMemcpy(out, g_engine->getGrid().mass, sizeof(float) * 4 * g, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -2;
}

int ref_engine_get_sdf(float* out) {
    if (!g_engine) return -1;
    const long g = GameConfigData::getInt("GRID_NUMBER");
    return cudaMemcpy(out, g_engine->getGrid().sdf, sizeof(float) * g, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -2;
}

int ref_engine_get_positions(float* out) {
    if (!g_engine) return -1;
    return cudaMemcpy(out, g_engine->getPositions(), sizeof(float) * 3 * g_n, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -2;
}

// d_values after the last sortParticles: the sort permutation.
int ref_engine_get_perm(int* out) {
    if (!g_engine) return -1;
    int* v = g_engine->*get(ValuesTag());
    return cudaMemcpy(out, v, sizeof(int) * g_n, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -2;
}

// Engine::step (engine.cu:54-70) with CUDA events between its stages: the
// same calls in the same order and with the same launch shapes
// (sortParticles, emptyGrid, p2GTransferScatter, gridUpdate, g2PTransfer,
// changeFormat), without the host synchronisation after each launch.  Sums
// each stage's device time over nsub substeps into ms6[0..5] in that order;
// the sort includes the reference's per-call cudaMalloc/cudaFree of its key
// buffer, as Engine::sortParticles does it.
int ref_engine_time_stages(int nsub, float* ms6) {
    if (!g_engine) return -1;
    cudaEvent_t ev[7];
    for (auto& x : ev) cudaEventCreate(&x);
    for (int k = 0; k < 6; ++k) ms6[k] = 0.0f;
    const int n = (int)g_n;
    const int blocks = (n + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK;
    const int gblocks = GameConfigData::getInt("GRID_BLOCKS");
    int* values = g_engine->*get(ValuesTag());
    float3* positions = g_engine->*get(PositionsTag());
    cudaDeviceSynchronize();
    for (int i = 0; i < nsub; ++i) {
        cudaEventRecord(ev[0]);
        g_engine->sortParticles();
        cudaEventRecord(ev[1]);
        emptyGrid<<<gblocks, THREADS_PER_BLOCK>>>(g_engine->getGrid());
        cudaEventRecord(ev[2]);
        p2GTransferScatter<<<blocks, THREADS_PER_BLOCK>>>(g_engine->getParticles(), g_engine->getGrid(), n, values);
        cudaEventRecord(ev[3]);
        gridUpdate<<<gblocks, THREADS_PER_BLOCK>>>(g_engine->getGrid());
        cudaEventRecord(ev[4]);
        g2PTransfer<<<blocks, THREADS_PER_BLOCK>>>(g_engine->getParticles(), g_engine->getGrid(), n, values);
        cudaEventRecord(ev[5]);
        changeFormat<<<blocks, THREADS_PER_BLOCK>>>(g_engine->getParticles(), positions, n);
        cudaEventRecord(ev[6]);
        cudaEventSynchronize(ev[6]);
        for (int k = 0; k < 6; ++k) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            ms6[k] += t;
        }
    }
    for (auto& x : ev) cudaEventDestroy(x);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// Device time of one makeSDF launch (kernels.cu:282-300) over the loaded
// config's grid with Engine::initSDF's launch shape (engine.cu:105-114), the
// triangles already on the device.
float ref_time_make_sdf(const float* tris, long t) {
    const long g = (long)GameConfigData::getInt("GRID_NUMBER");
    float* sdf = nullptr;
    Triangle* d_tris = nullptr;
    if (cudaMalloc((void**)&sdf, sizeof(float) * g) != cudaSuccess) return -1.0f;
    if (t > 0 && cudaMalloc((void**)&d_tris, sizeof(Triangle) * t) != cudaSuccess) {
        cudaFree(sdf);
        return -1.0f;
    }
    if (t > 0) cudaMemcpy(d_tris, tris, sizeof(Triangle) * t, cudaMemcpyHostToDevice);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    makeSDF<<<GameConfigData::getInt("GRID_BLOCKS"), THREADS_PER_BLOCK>>>(sdf, d_tris, (int)t);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sdf);
    if (d_tris) cudaFree(d_tris);
    return cudaGetLastError() == cudaSuccess ? ms : -2.0f;
}

// Device time of `reps` reference sorts of n keys (setKeys on the engine's
// particles, then thrust::sequence + thrust::sort_by_key as
// Engine::sortParticles runs them, engine.cu:92-102), the key buffer
// allocated once outside the timed region.
float ref_time_sort(int reps) {
    if (!g_engine) return -1.0f;
    const int n = (int)g_n;
    int* keys = nullptr;
    if (cudaMalloc((void**)&keys, sizeof(int) * n) != cudaSuccess) return -1.0f;
    int* values = g_engine->*get(ValuesTag());
    const int blocks = (n + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    for (int r = 0; r < reps; ++r) {
        setKeys<<<blocks, THREADS_PER_BLOCK>>>(g_engine->getParticles(), keys, n);
        thrust::sequence(thrust::device, values, values + n);
        thrust::sort_by_key(thrust::device, keys, keys + n, values);
    }
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(keys);
    return cudaGetLastError() == cudaSuccess ? ms / (float)reps : -2.0f;
}

// setKeys on the current particle state (the keys the next substep sorts).
int ref_engine_keys(int* out) {
    if (!g_engine) return -1;
    int* d = nullptr;
    if (cudaMalloc((void**)&d, sizeof(int) * g_n) != cudaSuccess) return -2;
    setKeys<<<(g_n + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK, THREADS_PER_BLOCK>>>(g_engine->getParticles(), d, (int)g_n);
    int rc = cudaMemcpy(out, d, sizeof(int) * g_n, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -3;
    cudaFree(d);
    return rc;
}

// Engine::sortParticles alone (engine.cu:92-102).
int ref_engine_sort_only() {
    if (!g_engine) return -1;
    g_engine->sortParticles();
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

void ref_engine_destroy() {
    delete g_engine;
    g_engine = nullptr;
    g_n = 0;
}

}  // extern "C"

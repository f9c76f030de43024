/*
 * mpm_b200.h - C ABI of the B200 MLS-MPM substep engine.
 *
 * This is the drop-in boundary for the simulation step of water-sim-cuda.
 * The reference exposes the step as the C++ class `Engine` (engine.h:14-43),
 * configured through `GameConfigData` (game_configdata.h:15-32) and a
 * process-global `__constant__ SimConfig d_config` (common.cuh:65-83,
 * config.cu:3-8).  Each entry point below names the reference member it
 * replaces.  Differences that a caller can observe are stated beside it.
 *
 * Conventions
 *  - Plain pointers and sizes only.  `*_host` buffers are host memory (pinned
 *    or pageable); `*_device` / `d_*` buffers are device memory on the
 *    engine's device.
 *  - Every call returns an mpm_status; nothing here exits the process or
 *    traps the GPU (the reference calls exit(1) on any CUDA or config error,
 *    engine.cu:21-28, game_configdata.cpp:49,56-61).
 *  - One engine = one device, one CUDA stream, no process-global state, so
 *    several engines may live in one process (the reference allows one).
 *  - An engine is not thread-safe; use one engine per host thread.
 */
#ifndef MPM_B200_H
#define MPM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_ABI_VERSION 1

/* Particle state planes: n floats each, plane-major (SoA), in the order of
 * `enum ParticleAttr` (common.cuh:12-29).  A state buffer holds 26*n floats,
 * the layout `VoxelPipeline::process` builds (VoxelPipeline.cpp:5-33). */
enum {
    MPM_POS_X = 0, MPM_POS_Y, MPM_POS_Z,
    MPM_VEL_X, MPM_VEL_Y, MPM_VEL_Z,
    MPM_C00, MPM_C01, MPM_C02, MPM_C10, MPM_C11, MPM_C12, MPM_C20, MPM_C21, MPM_C22,
    MPM_F00, MPM_F01, MPM_F02, MPM_F10, MPM_F11, MPM_F12, MPM_F20, MPM_F21, MPM_F22,
    MPM_VOL, MPM_MASS,
    MPM_PARTICLE_PLANES /* = 26 */
};

/* Grid planes: G = size_x*size_y*size_z floats each, node index
 * z*size_x*size_y + y*size_x + x (common.cuh:110-121, 131-134).  After a
 * substep the momentum planes hold the updated node velocities, exactly as
 * the reference's gridUpdate leaves them (kernels.cu:193). */
enum {
    MPM_GRID_MASS = 0, MPM_GRID_MOM_X, MPM_GRID_MOM_Y, MPM_GRID_MOM_Z,
    MPM_GRID_PLANES /* = 4 */
};

typedef enum mpm_status {
    MPM_OK = 0,
    MPM_ERR_INVALID_ARGUMENT = 1,
    MPM_ERR_BAD_CONFIG = 2,      /* missing key, unparsable value, bad WATER/OBJECT entry */
    MPM_ERR_IO = 3,              /* config file cannot be opened */
    MPM_ERR_CUDA = 4,            /* a CUDA runtime call failed; see mpm_last_error */
    MPM_ERR_OUT_OF_MEMORY = 5,
    MPM_ERR_NOT_INITIALIZED = 6, /* step/readback before mpm_init_particles */
    MPM_ERR_NONFINITE_STATE = 7, /* checks on: a particle position/velocity became NaN/Inf */
    MPM_ERR_OUT_OF_GRID = 8,     /* checks on: a particle left [0,SIZE) on some axis */
    MPM_ERR_TIMEOUT = 9,         /* a bounded device-side wait gave up */
    MPM_ERR_UNSUPPORTED = 10,
    MPM_ERR_NO_DEVICE = 11       /* no CUDA device, or the device is not sm_100 */
} mpm_status;

/* Simulation parameters: the config.txt keys read by
 * Simulation::initDeviceParams (Simulation.cpp:56-77) into SimConfig
 * (common.cuh:65-79).  GRID_SIZE/GRID_NUMBER/GRID_BLOCKS are derived, as in
 * the reference, and not stored.  sdf_resolution is accepted and ignored:
 * no reference kernel reads SDF_RESOLUTION, the SDF lives on the simulation
 * grid. */
typedef struct mpm_config {
    int32_t size_x, size_y, size_z; /* SIZE_X/Y/Z (grid nodes per axis) */
    int32_t padding;                /* PADDING (wall thickness in nodes) */
    float gravity;                  /* GRAVITY: subtracted from v.y each substep (kernels.cu:155) */
    float dt;                       /* DT */
    float gamma;                    /* GAMMA: Tait exponent (kernels.cu:28) */
    float compression;              /* COMPRESSION: Tait stiffness (kernels.cu:28) */
    float resolution;               /* RESOLUTION: particle volume = RESOLUTION^3 (kernels.cu:356) */
    int32_t substeps;               /* SUBSTEPS: substeps per frame (Simulation.cpp:46) */
    int32_t sdf_resolution;         /* SDF_RESOLUTION: accepted, unused */
} mpm_config;

#define MPM_PATH_MAX 512

/* One `WATER=` or `OBJECT=` entry, `path;scale;x;y;z` (game_configdata.cpp:35-49,
 * struct ConfigObject game_configdata.h:7-12). */
typedef struct mpm_scene_entry {
    char model_path[MPM_PATH_MAX];
    float scale;
    float x, y, z;
} mpm_scene_entry;

typedef struct mpm_engine mpm_engine;

/* Health bits reported by mpm_get_stats (always recorded) and turned into
 * step errors by mpm_set_checks. */
enum {
    MPM_HEALTH_NONFINITE = 1u << 0,   /* some particle position or velocity is NaN/Inf */
    MPM_HEALTH_OUT_OF_GRID = 1u << 1  /* some particle position is outside [0,SIZE) */
};

typedef struct mpm_stats {
    int64_t substeps;          /* substeps completed since mpm_init_particles */
    int64_t kernel_launches;   /* kernels this engine launched since creation */
    int64_t sort_passes;       /* radix-sort passes run since creation (mpm_get_sort) */
    uint32_t health;           /* MPM_HEALTH_* bits seen since init or the last reset */
    uint32_t reserved;
} mpm_stats;

/* Stages of one substep, for mpm_substep_partial. */
enum {
    MPM_STAGE_SORT = 1,  /* particle ordering (the reference's Morton keys + stable sort,
                          * engine.cu:92-102); here the ordering by stencil cell */
    MPM_STAGE_P2G = 2,   /* + grid clear + particle-to-grid scatter (kernels.cu:6-142, 311-318) */
    MPM_STAGE_GRID = 3,  /* + grid update (kernels.cu:144-196) */
    MPM_STAGE_G2P = 4    /* + grid-to-particle gather: a full substep (kernels.cu:199-280) */
};

/* ------------------------------------------------------------------ */
/* Library                                                              */
/* ------------------------------------------------------------------ */

int32_t mpm_abi_version(void);
const char* mpm_status_string(mpm_status status);

/* ------------------------------------------------------------------ */
/* Configuration (no GPU needed)                                        */
/* ------------------------------------------------------------------ */

/* Replaces GameConfigData::setConfigDataFromFile (game_configdata.cpp:22-54)
 * followed by the getInt/getFloat reads of Simulation::initDeviceParams
 * (Simulation.cpp:56-77).  Same format: `KEY=value` lines, every space
 * removed before parsing, blank lines skipped, lines without '=' ignored,
 * later keys overwrite earlier ones, integer keys parsed like std::stoi
 * (leading integer prefix, so "0.5" reads as 0), float keys like std::stof.
 * Repeated WATER=/OBJECT= entries are appended (at most max_* are stored,
 * n_* counts all).  Where the reference exits, this returns
 * MPM_ERR_BAD_CONFIG with the reason in err (if err_len > 0):
 * a required key missing or unparsable, or a WATER/OBJECT value with fewer
 * than 5 ';'-separated fields.  Any of waters/objects/n_* may be NULL. */
mpm_status mpm_config_parse_file(const char* path, mpm_config* cfg,
                                 mpm_scene_entry* waters, int32_t max_waters, int32_t* n_waters,
                                 mpm_scene_entry* objects, int32_t max_objects, int32_t* n_objects,
                                 char* err, int32_t err_len);

/* As mpm_config_parse_file, from the text of a config file. */
mpm_status mpm_config_parse_string(const char* text, mpm_config* cfg,
                                   mpm_scene_entry* waters, int32_t max_waters, int32_t* n_waters,
                                   mpm_scene_entry* objects, int32_t max_objects, int32_t* n_objects,
                                   char* err, int32_t err_len);

/* ------------------------------------------------------------------ */
/* Engine lifetime                                                      */
/* ------------------------------------------------------------------ */

/* Replaces `Engine engine;` plus uploadConfigToGPU (config.cu:5-8) and
 * Engine::initGrid (engine.cu:86-90).  Allocates the grid and SDF on
 * `device`; the SDF starts at +1e15 everywhere, the value the reference's
 * makeSDF writes for an empty triangle list (kernels.cu:289,299), so a scene
 * without OBJECT entries may skip mpm_init_sdf.  Rejects sizes <= 0,
 * padding < 0, and non-finite floats with MPM_ERR_BAD_CONFIG. */
mpm_status mpm_create(const mpm_config* cfg, int32_t device, mpm_engine** out);

/* Replaces Engine::~Engine (engine.cu:36-43).  Frees every buffer, including
 * the SDF and position buffers the reference leaks.  NULL is a no-op. */
void mpm_destroy(mpm_engine* engine);

/* Replaces Engine::init(int n, float* h_buffer) (engine.cu:45-52, 72-83).
 * For an engine of one scene (mpm_create); batches use
 * mpm_init_particles_batch.
 * soa26_host holds 26*n floats (layout above).  Unlike the reference, the
 * buffer is COPIED, not adopted (the reference delete[]s it in ~Engine).
 * As the reference's initFMatrices does (kernels.cu:349-358), F00/F11/F22
 * are set to 1, VOL to resolution^3 and MASS to 1; all other planes are
 * taken from the buffer.  n may be 0 (the reference cannot launch a
 * zero-block grid and exits).  May be called again to replace the scene. */
mpm_status mpm_init_particles(mpm_engine* engine, int64_t n, const float* soa26_host);

/* Replaces Engine::initSDF(std::vector<Triangle>) (engine.cu:105-114,
 * kernels.cu:282-300).  triangles_host holds t triangles of 9 floats
 * (v0.xyz, v1.xyz, v2.xyz) already placed in grid coordinates, the layout of
 * `struct Triangle` (common.cuh:123-126).  Each node at integer coordinates
 * gets sign(winding number > 0.5 ? -1 : +1) * distance to the closest
 * triangle.  t = 0 gives +1e15 everywhere. */
mpm_status mpm_init_sdf(mpm_engine* engine, const float* triangles_host, int64_t t);

/* ------------------------------------------------------------------ */
/* Stepping                                                             */
/* ------------------------------------------------------------------ */

/* Replaces `for (s < nsub) engine.step();` (Simulation.cpp:46-49,
 * engine.cu:54-70): nsub MLS-MPM substeps (keys, stable sort, clear, P2G,
 * grid update, G2P), then the float3 position export (kernels.cu:341-347).
 * Synchronous: returns after the device finished, like the reference's
 * per-kernel cudaDeviceSynchronize.  nsub = 0 only refreshes the export. */
mpm_status mpm_step(mpm_engine* engine, int32_t nsub);

/* As mpm_step but only enqueues the work on the engine's stream. */
mpm_status mpm_step_async(mpm_engine* engine, int32_t nsub);

/* Waits for the engine's stream and reports any asynchronous error. */
mpm_status mpm_synchronize(mpm_engine* engine);

/* Runs one substep stage by stage, so that a test can read the grid after
 * P2G or after the grid update: continues the substep in progress with the
 * stages after the last one run, up to `upto` (MPM_STAGE_*), or starts a new
 * substep when none is in progress or `upto` is not past the last stage run.
 * MPM_STAGE_G2P completes the substep exactly as mpm_step(engine, 1) would.
 * Particles only change at MPM_STAGE_G2P; mpm_step discards an unfinished
 * substep.  Synchronous.  No counterpart in the reference. */
mpm_status mpm_substep_partial(mpm_engine* engine, int32_t upto);

/* Health checks: when `flags` holds MPM_HEALTH_* bits, mpm_step returns
 * MPM_ERR_NONFINITE_STATE / MPM_ERR_OUT_OF_GRID after a step in which the
 * matching condition appeared (the step itself still completes).  Default 0:
 * like the reference, the step never fails on state contents. */
mpm_status mpm_set_checks(mpm_engine* engine, uint32_t flags);

/* Test hooks of the bounded device-side waits (failure detection without a
 * GPU fault).  Every mbarrier wait of the SDF build's triangle copies and of
 * the learned step's tcgen05 MMAs has a time limit; when it runs out the
 * kernel drains what it has in flight, records a status bit, frees its TMEM
 * and returns, and the call fails with MPM_ERR_TIMEOUT while the context stays
 * usable.  These flags make the first such wait of the next mpm_init_sdf /
 * mpm_scene_init_sdf (SDF_*) or mpm_step_learned on tcgen05 (MMA_*) give up,
 * always after the real completion has been observed, so that nothing is in
 * flight when it does:
 *   *_GIVE_UP  reports the give-up at once;
 *   *_EXPIRE   then waits for the barrier's next phase, which nothing
 *              completes, until a 20 ms limit really runs out.
 * The outputs of a call that failed this way are unspecified (an SDF left
 * unbuilt, a large step without its correction); the engine is usable for
 * the next call.  0 (the default) clears the hooks.  No counterpart in the
 * reference, which has no bounded waits. */
#define MPM_WAIT_TEST_SDF_GIVE_UP 0x1u
#define MPM_WAIT_TEST_SDF_EXPIRE 0x2u
#define MPM_WAIT_TEST_MMA_GIVE_UP 0x4u
#define MPM_WAIT_TEST_MMA_EXPIRE 0x8u
mpm_status mpm_set_wait_test(mpm_engine* engine, uint32_t flags);

/* ------------------------------------------------------------------ */
/* Readback                                                             */
/* ------------------------------------------------------------------ */

/* Replaces Engine::getNumber (engine.h:28). */
int64_t mpm_num_particles(const mpm_engine* engine);

/* Replaces Engine::getBuffer (engine.h:29) + a device-to-host copy: the
 * 26*n state in ORIGINAL particle order (the order of mpm_init_particles). */
mpm_status mpm_get_state(mpm_engine* engine, float* soa26_host);

/* Loads a 26*n state saved by mpm_get_state (checkpoint resume), for an
 * engine of one scene.  n must
 * equal the engine's particle count.  Unlike mpm_init_particles no plane is
 * overwritten.  VOL and MASS must each hold one value for all particles, as
 * every state the reference can produce does (initFMatrices sets them and
 * no kernel writes them); otherwise MPM_ERR_UNSUPPORTED.  No counterpart in
 * the reference. */
mpm_status mpm_set_state(mpm_engine* engine, int64_t n, const float* soa26_host);

/* Replaces Engine::getPositions (engine.h:23): n float3 positions in original
 * order, as changeFormat writes them (kernels.cu:341-347).  The pointer is
 * owned by the engine and valid until the next step, init or destroy. */
const float* mpm_positions_device(mpm_engine* engine);

/* mpm_positions_device + a device-to-host copy of 3*n floats. */
mpm_status mpm_get_positions(mpm_engine* engine, float* xyz_host);
/* As mpm_get_positions, without waiting: the copy runs on the engine's copy
 * stream, after the export it reads and alongside the substeps that follow,
 * and xyz_host holds the positions once mpm_positions_wait returns.  Exports
 * alternate between two device buffers, and an export waits for the read-back
 * of its buffer, so one frame can be read while the next computes.  Pinned
 * host memory makes the copy asynchronous. */
mpm_status mpm_get_positions_async(mpm_engine* engine, float* xyz_host);
mpm_status mpm_positions_wait(mpm_engine* engine);

/* Replaces Engine::getGrid (engine.h:22) + a copy of its 4 planes (4*G
 * floats, plane order MPM_GRID_*).  After a substep: mass from P2G and the
 * updated node velocities in the momentum planes. */
mpm_status mpm_get_grid(mpm_engine* engine, float* grid4_host);

/* Copies the G-float signed distance field (Grid::sdf, common.cuh:114). */
mpm_status mpm_get_sdf(mpm_engine* engine, float* sdf_host);

/* The Morton keys and sort permutation of the most recent substep, as the
 * reference's sortParticles leaves them (engine.cu:92-102): keys_host[i] is
 * setKeys' key of particle i (original order, kernels.cu:361-371) and
 * perm_host[j] is the original index of the j-th particle in stable
 * ascending key order (d_values after thrust::sort_by_key).  The engine
 * itself orders particles by stencil cell, which its P2G needs, not by this
 * key; it computes the reference's keys and permutation on request,
 * bit-exactly, from the state that substep started from (kept until the
 * next substep).  Either pointer may be NULL.  Before any substep: keys of
 * the current state, identity. */
mpm_status mpm_get_sort(mpm_engine* engine, int32_t* keys_host, int32_t* perm_host);

/* Counters and accumulated health bits; reset_health clears the bits. */
mpm_status mpm_get_stats(mpm_engine* engine, mpm_stats* stats, int32_t reset_health);

/* Per-stage device timing.  With max_substeps > 0 the substep graphs also
 * record CUDA events between the stages (sort, P2G, grid update, G2P) of the
 * next max_substeps substeps; 0 turns it off and frees the events.  No
 * counterpart in the reference (it has no timers). */
mpm_status mpm_set_stage_timing(mpm_engine* engine, int32_t max_substeps);

/* Sums of the recorded stage durations in milliseconds, ms[0..3] = sort,
 * P2G, grid update, G2P, over *count substeps, then clears the record.
 * Synchronizes the engine's stream. */
mpm_status mpm_get_stage_times(mpm_engine* engine, double* ms, int32_t* count);

/* The engine's cudaStream_t, for callers that order their own work after it. */
void* mpm_stream(mpm_engine* engine);

/* Text of the engine's last error ("" if none).  Never NULL. */
const char* mpm_last_error(const mpm_engine* engine);

/* Text of the last error of a call that had no engine to record it on
 * (mpm_create, mpm_sort_particles_device).  Thread-local.  Never NULL. */
const char* mpm_global_last_error(void);

/* ------------------------------------------------------------------ */
/* Batches of independent scenes                                        */
/* ------------------------------------------------------------------ */

/* No counterpart in the reference (one scene per process, its config lives
 * in a process-global __constant__).  An engine of nscenes independent
 * scenes, each with its own grid size, physics constants, particles and
 * obstacles, on one device.  Every substep stage runs as one launch over all
 * scenes, and mpm_step / mpm_step_async / mpm_synchronize /
 * mpm_substep_partial / mpm_set_stage_timing act on all of them.  An engine
 * from mpm_create is the batch of one scene, and the single-scene calls
 * (mpm_init_sdf, mpm_get_state, ...) address its scene 0. */
mpm_status mpm_create_batch(const mpm_config* cfgs, int32_t nscenes, int32_t device, mpm_engine** out);

/* Number of scenes (0 for NULL). */
int32_t mpm_num_scenes(const mpm_engine* engine);

/* Engine::init for every scene at once: scene s gets counts[s] particles
 * from soa26_host[s] (26 * counts[s] floats, copied; the same rules as
 * mpm_init_particles).  counts[s] may be 0. */
mpm_status mpm_init_particles_batch(mpm_engine* engine, const int64_t* counts, const float* const* soa26_host);

/* Per-scene forms of mpm_init_sdf, mpm_num_particles, mpm_get_state,
 * mpm_positions_device, mpm_get_positions, mpm_get_grid, mpm_get_sdf and
 * mpm_get_sort.  scene outside [0, mpm_num_scenes) is
 * MPM_ERR_INVALID_ARGUMENT (0 / NULL for the value-returning ones). */
mpm_status mpm_scene_init_sdf(mpm_engine* engine, int32_t scene, const float* triangles_host, int64_t t);
int64_t mpm_scene_num_particles(const mpm_engine* engine, int32_t scene);
mpm_status mpm_scene_get_state(mpm_engine* engine, int32_t scene, float* soa26_host);
const float* mpm_scene_positions_device(mpm_engine* engine, int32_t scene);
mpm_status mpm_scene_get_positions(mpm_engine* engine, int32_t scene, float* xyz_host);
mpm_status mpm_scene_get_grid(mpm_engine* engine, int32_t scene, float* grid4_host);
mpm_status mpm_scene_get_sdf(mpm_engine* engine, int32_t scene, float* sdf_host);
mpm_status mpm_scene_get_sort(mpm_engine* engine, int32_t scene, int32_t* keys_host, int32_t* perm_host);

/* ------------------------------------------------------------------ */
/* Stand-alone device operators                                         */
/* ------------------------------------------------------------------ */

/* Replaces Engine::sortParticles (engine.cu:92-102) as a free operator on
 * caller-owned device buffers: d_keys[i] = Morton key of particle i
 * (setKeys, kernels.cu:361-371) and d_perm = the stable ascending sort
 * permutation of those keys (thrust::sequence + thrust::sort_by_key).
 * Positions are three device arrays of n floats.  Work is enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream); scratch memory is
 * taken with cudaMallocAsync on that stream and released before return, as
 * the reference allocates its key buffer each call (engine.cu:95,101).
 * Returns after enqueueing; synchronize the stream before reading. */
mpm_status mpm_sort_particles_device(const float* d_pos_x, const float* d_pos_y, const float* d_pos_z,
                                     int64_t n, int32_t* d_keys, int32_t* d_perm, void* stream);

/* Largest n mpm_sort_particles_device_static accepts. */
#define MPM_SORT_STATIC_MAX_PARTICLES (1 << 20)

/* mpm_sort_particles_device for callers that cannot allocate device memory:
 * the same keys and permutation, bit for bit, with no cudaMalloc, cudaFree or
 * other allocating call.  It has no counterpart in the reference, which
 * allocates its key buffer on every sort (engine.cu:95,101).
 * Who needs it: hosts whose device memory belongs to another allocator (a
 * game engine's or framework's pool that reserved it up front), real-time
 * frame loops that must not block on an allocator or on the device-wide
 * synchronisation of cudaFree, and stacks without stream-ordered
 * allocation.
 * How: the sort scratch is one fixed array in device memory, about
 * 16 MiB + 1 MiB, that every device which loads this library holds until the
 * process exits.  n above MPM_SORT_STATIC_MAX_PARTICLES is rejected with
 * MPM_ERR_INVALID_ARGUMENT (mpm_global_last_error says why); use
 * mpm_sort_particles_device for larger inputs.
 * Runs on the calling thread's current device; `stream` must belong to it.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) and caches it, so make that first call before any
 * stream capture begins.  The cached address assumes the device is not reset
 * (cudaDeviceReset) while the process runs; after a reset, do not call it.
 * All calls on a device share the one array and nothing clears it between
 * calls (no part of it needs to start at zero).  Calls that overlap on the
 * GPU, on different streams or from different threads, race on it and give
 * wrong results: order them on one stream or serialise them.
 * Returns after enqueueing; synchronize the stream before reading. */
mpm_status mpm_sort_particles_device_static(const float* d_pos_x, const float* d_pos_y, const float* d_pos_z,
                                            int64_t n, int32_t* d_keys, int32_t* d_perm, void* stream);

/* ------------------------------------------------------------------ */
/* Headless screen-space fluid rendering                                */
/* ------------------------------------------------------------------ */
/* The reference's SSF passes (renderer.cpp:199-338; shaders ssf_depth.vert/
 * .frag, ssf_blur.frag, screen.frag) as CUDA kernels writing device image
 * buffers; no graphics API.  Images are width x height, row 0 at the bottom
 * (GL window coordinates), RGB float in [0, 1+] (the composite can exceed 1
 * by the specular term; the 8-bit copy clamps like a framebuffer). */
typedef struct mpm_render_params {
    int32_t width, height;        /* 1920 x 1600 (renderer.h:11-12) */
    int32_t grid[3];              /* SIZE_X, SIZE_Y, SIZE_Z: camera and centre */
    float fov_y_degrees;          /* 45 */
    float near_clip, far_clip;    /* 0.1, 5000 */
    float zoom_distance;          /* camera z: SIZE_Z * 2 */
    float rotation;               /* about y through the grid centre (radians) */
    float rotation_vertical;      /* about x */
    float radius;                 /* sprite radius 2 */
    float filter_size;            /* blur half-width 10 */
    float depth_falloff;          /* 0.01 */
    float light_dir[3];           /* world, (0.2, 10, 0.5) */
    float clear_color[3];         /* background (0.85, 0.9, 0.95) */
} mpm_render_params;
typedef struct mpm_renderer mpm_renderer;
void mpm_render_params_default(mpm_render_params* params, int32_t size_x, int32_t size_y, int32_t size_z);
mpm_status mpm_renderer_create(const mpm_render_params* params, int32_t device, mpm_renderer** out);
void mpm_renderer_destroy(mpm_renderer* renderer);
const char* mpm_renderer_last_error(const mpm_renderer* renderer);
/* Background image (width x height RGB8, row 0 at the bottom) in place of
 * the clear colour: what the framebuffer held before the fluid pass. */
mpm_status mpm_renderer_set_background(mpm_renderer* renderer, const uint8_t* rgb8_host);
/* The obstacle pass (shaders/dot.vert + dot.frag, renderer.cpp:247-303, the
 * default opaque mode): t triangles (9 floats each, grid coordinates, the
 * same list as mpm_init_sdf) drawn once over the background with a depth
 * test, flat Lambert shading 0.3 C + max(n . L, 0) C (rgb NULL: C = 0.5 grey)
 * and stored as 8 bits; the fluid's composite is depth-tested against them.
 * t = 0 removes them.  The glass and wireframe toggles are not restated; a
 * triangle with a vertex behind the near plane is dropped (GL would clip it). */
mpm_status mpm_renderer_set_obstacles(mpm_renderer* renderer, const float* tris_host, int64_t t,
                                      const float* rgb_host);
/* The background texture (RGB8, after the obstacle pass) and / or the
 * obstacles' window depth in [0, 1] (1 where none); either may be NULL. */
mpm_status mpm_renderer_get_background(mpm_renderer* renderer, uint8_t* rgb8_host, float* depth_host);
/* All passes for n positions (float3, device memory), enqueued on `stream`. */
mpm_status mpm_render_points(mpm_renderer* renderer, const float* xyz_device, int64_t n, void* stream);
/* All passes for the engine's current positions, on the engine's stream. */
mpm_status mpm_render_frame(mpm_renderer* renderer, mpm_engine* engine);
/* which: 0 = splat depth (view z, 99999 where no sprite), 1 = after the
 * horizontal blur, 2 = after the vertical blur. */
mpm_status mpm_renderer_get_depth(mpm_renderer* renderer, int32_t which, float* depth_host);
/* Final colour as float RGB and / or 8-bit RGB (either may be NULL). */
mpm_status mpm_renderer_get_image(mpm_renderer* renderer, float* rgb_host, uint8_t* rgb8_host);

/* ------------------------------------------------------------------ */
/* Checkpoints (no counterpart in the reference)                        */
/* ------------------------------------------------------------------ */
/* One file per engine of one scene, little-endian: a 128-byte header
 * ("MPMCKPT1", version 1, header size 128, n, substeps done, the config
 * fields, VOL, MASS, note length), the note (e.g. the config text), the state
 * in the 26-plane layout of mpm_get_state (original particle order), the SDF
 * (G floats), and a CRC-32 of everything before it.  Written to PATH.part and
 * renamed, so a crash never leaves a truncated file under PATH.  Loading
 * creates an engine with the state taken as it is (no initFMatrices) and the
 * SDF restored; it continues as the saved engine would, up to the order of
 * float sums. */
mpm_status mpm_checkpoint_save(mpm_engine* engine, const char* path, const char* note);
mpm_status mpm_checkpoint_load(const char* path, int32_t device, mpm_engine** out);
/* Header and note of a checkpoint (any output may be NULL). */
mpm_status mpm_checkpoint_info(const char* path, mpm_config* cfg, int64_t* n, int64_t* substeps, char* note,
                               int32_t note_len);

/* ------------------------------------------------------------------ */
/* Scene construction from WATER= / OBJECT= entries                     */
/* ------------------------------------------------------------------ */
/* Simulation::Simulation()'s scene part (Simulation.cpp:4-38): each WATER
 * model is loaded (ObjLoader::loadObj), voxelised at 100 voxels along its
 * longest side (VoxelEngine::voxelize, VoxelEngine.cpp:120-243: the voxels
 * the surface triangles touch), normalised into a SIZE_X cube, scaled so the
 * longest side is `scale` cells, displaced, and snapped to the lattice of
 * step getInt("RESOLUTION") with a 5x5x5 dilation (VoxelEngine::normalize,
 * VoxelEngine.cpp:245-494); the particles of all WATER entries are
 * concatenated (MergeVoxelData) in the layout of VoxelPipeline::process.
 * OBJECT models give triangles (extractTriangles), normalised the same way
 * and culled to those with a vertex in [0, SIZE_X]^3 (VoxelEngine.cpp:601-827).
 * The triangle-box tests and the dilation run on `device`.  Model paths are
 * relative to base_dir (the reference opens them from the working directory;
 * NULL or "" = as given).  A WATER model that cannot be read, or that gives
 * no voxels, fails the build (the reference throws); an OBJECT model that
 * cannot be read is skipped and noted in mpm_scene_data_log.  A lattice step
 * below 1 (RESOLUTION < 1, where the reference divides by zero,
 * VoxelEngine.cpp:369-381) is MPM_ERR_BAD_CONFIG. */
typedef struct mpm_scene_data mpm_scene_data;
mpm_status mpm_scene_build(const char* config_text, const char* base_dir, int32_t device, mpm_scene_data** out);
void mpm_scene_data_free(mpm_scene_data* scene);
int64_t mpm_scene_data_num_particles(const mpm_scene_data* scene);
int64_t mpm_scene_data_num_triangles(const mpm_scene_data* scene);
/* 26 * n floats: positions, zeros, VOL = MASS = 1 (VoxelPipeline.cpp:5-33);
 * mpm_init_particles applies initFMatrices to it. */
mpm_status mpm_scene_data_state(const mpm_scene_data* scene, float* soa26_host);
mpm_status mpm_scene_data_triangles(const mpm_scene_data* scene, float* triangles9_host);
const char* mpm_scene_data_log(const mpm_scene_data* scene);
const char* mpm_scene_last_error(void);

/* The stages one by one.  A mesh is an OBJ's vertices and triangles (faces
 * triangulated as tinyobjloader's LoadObj does; see csrc/scene.cu). */
typedef struct mpm_mesh mpm_mesh;
mpm_status mpm_mesh_load_obj(const char* path, mpm_mesh** out);
mpm_status mpm_mesh_from_obj_text(const char* text, mpm_mesh** out);
void mpm_mesh_free(mpm_mesh* mesh);
int64_t mpm_mesh_num_vertices(const mpm_mesh* mesh);
int64_t mpm_mesh_num_triangles(const mpm_mesh* mesh);
/* Any output may be NULL: 3 floats per vertex, 3 indices per triangle,
 * 9 floats per triangle (VoxelEngine::extractTriangles). */
mpm_status mpm_mesh_get(const mpm_mesh* mesh, float* vertices3_host, int32_t* faces3_host, float* triangles9_host);

/* A point set (x y z per point). */
typedef struct mpm_points mpm_points;
/* VoxelEngine::voxelize(obj, resolution): voxel centres in z, y, x order. */
mpm_status mpm_voxelize(const mpm_mesh* mesh, float resolution, int32_t device, mpm_points** out);
mpm_status mpm_points_create(const float* xyz_host, int64_t n, mpm_points** out);
int64_t mpm_points_count(const mpm_points* points);
mpm_status mpm_points_get(const mpm_points* points, float* xyz_host);
void mpm_points_free(mpm_points* points);
/* VoxelEngine::normalize(VoxelData&, normalizeSize, scale, displacement) in
 * place, with the lattice step getInt("RESOLUTION"); the result is in
 * (x, y, z) lexicographic order. */
mpm_status mpm_points_normalize(mpm_points* points, float normalize_size, float scale, const float* displacement3,
                                int32_t lattice_step, int32_t device);
/* VoxelEngine::normalize(std::vector<Triangle>&, ...) in place; *t shrinks
 * by the culled triangles.  Host only. */
mpm_status mpm_triangles_normalize(float* triangles9_host, int64_t* t, float normalize_size, float scale,
                                   const float* displacement3);

/* ------------------------------------------------------------------ */
/* Launch-shape tuning                                                   */
/* ------------------------------------------------------------------ */
/* The substep's launch shapes: persistent P2G CTAs per SM and P2G's
 * crowded-cell threshold, and the CTA sizes of the plain G2P and of the grid
 * update.  mpm_autotune leaves the threshold to P2G's per-item choice (0).  mpm_autotune times each
 * candidate on the engine's current particles (each stage on its own, the
 * median of `repeats` runs; every timed substep is undone, so the state does
 * not advance) and keeps the fastest; results are identical for every shape
 * up to the order of float sums. */
typedef struct mpm_tuning {
    int32_t p2g_ctas_per_sm;  /* 1 .. the most that fit (default 12) */
    int32_t g2p_block;        /* 128 or 256 (default 256); 512 = 256-thread CTAs free to use up to
                               * 255 registers (more loads in flight, fewer warps) */
    int32_t grid_block;       /* 128 or 256: the update visits every node in CTAs of that size;
                               * 0: only the node tiles this substep's particles reach, plus a
                               * reset of tiles they left (default for one scene of 2^23 nodes
                               * or more, else 256) */
    float p2g_ms, g2p_ms, grid_ms;  /* stage times of the chosen shapes (mpm_autotune) */
    int32_t p2g_cell_cap;     /* 4 .. 64: particles of a cell one lane sums before the
                               * rest goes, in chunks, to all warps; 0 (default): chosen
                               * per work item from its cells' particle counts */
} mpm_tuning;
mpm_status mpm_autotune(mpm_engine* engine, int32_t repeats, mpm_tuning* out);
mpm_status mpm_set_tuning(mpm_engine* engine, const mpm_tuning* tuning);
mpm_status mpm_get_tuning(mpm_engine* engine, mpm_tuning* tuning);

/* ------------------------------------------------------------------ */
/* Learned large step (no counterpart in the reference)                 */
/* ------------------------------------------------------------------ */
/* Beside the plain substep, never replacing it: one substep of RATIO x DT
 * (particles advect with v_old + (RATIO + 1) / (2 RATIO) (v_new - v_old),
 * the displacement of RATIO substeps under a constant acceleration) whose
 * G2P adds a velocity correction predicted per particle by a small MLP
 * (16 -> 64 -> 64 -> 3, GELU, bf16 weights on the tensor cores, fp32
 * accumulation).  Inputs: the particle's APIC matrix C (9), grid velocity
 * (3), interpolated grid mass over the seeding density, minus 1 (1), and the
 * obstacle SDF folded into one vector n * phi * max(0, 1 - |phi| / 4) (3), all
 * gathered from the large step's grid at the particle's start position.
 * The plain substep is the fallback and the yardstick: a large step whose
 * fallback statistic (mpm_set_fallback_rule) exceeds max_density_change is
 * undone and replaced by RATIO plain substeps.  Engines of one scene only. */
#define MPM_CORRECTOR_PARAMS 5478   /* fp32 parameter vector, layout below */
#define MPM_CORRECTOR_FEATURES 16
#define MPM_CORRECTOR_OUTPUTS 3
/* Parameter layout (offsets in floats): input mean [16] @0, input 1/std [16]
 * @16, output scale [3] @32, W1 [64][16] @35, b1 [64] @1059, W2 [64][64]
 * @1123, b2 [64] @5219, W3 [3][64] @5283, b3 [3] @5475.  W rows are outputs.
 * out = (W3 g(W2 g(W1 x' + b1) + b2) + b3) * scale, x' = (x - mean) / std,
 * g = GELU (tanh form); x', the weights and g's outputs rounded to bf16. */

typedef struct mpm_learned_stats {
    int64_t large_steps;         /* large steps accepted since creation */
    int64_t fallbacks;           /* large steps replaced by RATIO plain substeps */
    double last_density_change;  /* the statistic of the last large step that was checked
                                  * (large steps are checked only when the fallback is on) */
} mpm_learned_stats;

/* Sets the corrector (params_host: MPM_CORRECTOR_PARAMS floats, or NULL for
 * the uncorrected large step, which has no fallback), the step ratio and the
 * fallback threshold (negative: never fall back). */
mpm_status mpm_set_corrector(mpm_engine* engine, const float* params_host, int32_t ratio,
                             float max_density_change);
/* Which tensor-core path evaluates the MLP inside the large step's G2P:
 * tcgen05.mma with TMEM accumulators, 256 particles per CTA (default), or
 * warp-level mma.sync (the same operands and roundings). */
#define MPM_CORRECTOR_TCGEN05 0
#define MPM_CORRECTOR_MMA_SYNC 1
mpm_status mpm_set_corrector_kernel(mpm_engine* engine, int32_t kind);
/* nlarge large steps (each RATIO x DT of simulated time); stats optional. */
mpm_status mpm_step_learned(mpm_engine* engine, int32_t nlarge, mpm_learned_stats* stats);
/* The fallback statistic, a mean over particles computed by the large step's
 * G2P from the step's own grid (J = det(I + RATIO DT C) the predicted volume
 * change, rho / rho0 the interpolated grid mass over the seeding density):
 *   MPM_FALLBACK_DENSITY_CHANGE       |1 / J - 1|: the density change the
 *                                     step predicts (default);
 *   MPM_FALLBACK_REST_DENSITY         |rho / rho0 / J - 1|: how far the
 *                                     predicted density lies from rest
 *                                     density (free-surface particles, with
 *                                     part of their stencil empty, count too);
 *   MPM_FALLBACK_REST_DENSITY_EXCESS  the mean above minus the mean of
 *                                     |rho / rho0 - 1| before the step: how
 *                                     much the step moves the density away
 *                                     from rest. */
#define MPM_FALLBACK_DENSITY_CHANGE 0
#define MPM_FALLBACK_REST_DENSITY 1
#define MPM_FALLBACK_REST_DENSITY_EXCESS 2
mpm_status mpm_set_fallback_rule(mpm_engine* engine, int32_t rule);
/* Where a checked large step (a corrector set, max_density_change >= 0) is
 * accepted or rejected.  On the device (1, the default): each large step is
 * one CUDA graph (large step, a one-thread decision kernel, and a conditional
 * node whose body is the fallback: RATIO plain substeps from the start state,
 * then the result moved to where an accepted step leaves its own), so a call
 * of nlarge steps reads back only its counters, once.  On the host (0): the
 * statistic is read back after every large step and the fallback enqueued
 * from the host.  Both give the same results; after device-decided steps
 * mpm_get_sort reports the sort of the current state. */
mpm_status mpm_set_fallback_on_device(mpm_engine* engine, int32_t on_device);
/* The three means above (in that order: |1/J - 1|, |rho/rho0/J - 1|,
 * |rho/rho0 - 1|) of the last large step that was checked. */
mpm_status mpm_learned_statistics(mpm_engine* engine, double* out3);

/* Training data and training.  A corrector holds a dataset of (features,
 * target) pairs on the device and the parameters with their Adam state. */
typedef struct mpm_corrector mpm_corrector;
mpm_status mpm_corrector_create(int32_t device, int64_t capacity, mpm_corrector** out);
void mpm_corrector_destroy(mpm_corrector* corrector);
const char* mpm_corrector_last_error(const mpm_corrector* corrector);
int64_t mpm_corrector_size(const mpm_corrector* corrector);
mpm_status mpm_corrector_clear(mpm_corrector* corrector);
/* The collection probe on the engine's current state: one uncorrected large
 * step records every particle's features and velocity, the state goes back
 * to the start of that step, RATIO plain substeps follow (the engine keeps
 * their result: the plain trajectory goes on), and `samples` particles drawn
 * with replacement (seeded) are appended with target = velocity after the
 * plain substeps - velocity after the large step. */
mpm_status mpm_corrector_collect(mpm_corrector* corrector, mpm_engine* engine, int64_t samples, uint64_t seed);
mpm_status mpm_corrector_add_data(mpm_corrector* corrector, int64_t count, const float* features_host,
                                  const float* targets_host);
mpm_status mpm_corrector_get_data(mpm_corrector* corrector, int64_t first, int64_t count, float* features_host,
                                  float* targets_host);
/* Input normalisation and output scale from the dataset, seeded random
 * weights, Adam state reset. */
mpm_status mpm_corrector_init(mpm_corrector* corrector, uint64_t seed);
/* `steps` Adam steps (lr, beta 0.9 / 0.999) on batches of `batch` samples
 * (a multiple of 64) drawn with replacement; mean_loss: mean squared error of
 * the scaled targets over the steps. */
mpm_status mpm_corrector_train(mpm_corrector* corrector, int32_t steps, int32_t batch, float lr, uint64_t seed,
                               float* mean_loss);
/* Gradient of the loss on the samples idx_host[0..count) (count a multiple
 * of 64) at the current parameters, without a step. */
mpm_status mpm_corrector_gradient(mpm_corrector* corrector, int64_t count, const int64_t* idx_host,
                                  float* grad_host, float* loss_host);
/* Which kernel computes the training gradient: tcgen05.mma with TMEM
 * accumulators, 128 samples per tile, every GEMM of the forward and backward
 * pass on the tensor cores with bf16 operands (default); or FP32 on the CUDA
 * cores with the forward roundings of the inference.  A bounded wait of the
 * tcgen05 kernel that gives up is reported as MPM_ERR_TIMEOUT. */
#define MPM_TRAIN_TCGEN05 0
#define MPM_TRAIN_FP32 1
mpm_status mpm_corrector_set_train_kernel(mpm_corrector* corrector, int32_t kind);
mpm_status mpm_corrector_get_params(mpm_corrector* corrector, float* params_host);
mpm_status mpm_corrector_set_params(mpm_corrector* corrector, const float* params_host);
/* The tensor-core inference of the learned G2P on n feature rows
 * (warp-level mma.sync, bf16, fp32 accumulation). */
mpm_status mpm_corrector_forward(mpm_corrector* corrector, int64_t n, const float* features_host, float* out_host);
/* The same MLP on the 5th-generation tensor cores: tcgen05.mma with operands
 * in shared memory and accumulators in tensor memory, 256 rows per CTA. */
mpm_status mpm_corrector_forward_tc(mpm_corrector* corrector, int64_t n, const float* features_host,
                                    float* out_host);

#ifdef __cplusplus
}
#endif

#endif /* MPM_B200_H */

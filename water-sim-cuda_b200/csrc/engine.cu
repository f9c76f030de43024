// Host engine behind the C ABI (include/mpm_b200.h).
//
// Restates the reference's `Engine` (engine.h:14-43, engine.cu:36-114) and
// the config upload (config.cu:5-8, Simulation.cpp:56-77) with per-engine
// state: one device, one stream, and a CUDA graph per substep parity.  An
// engine holds one or more independent scenes (the batched form): their
// particle, grid, cell and bin arrays are concatenated, a device table of
// SimParams carries each scene's constants and offsets, and every substep
// stage is one launch over all scenes.  The reference's single Engine is an
// engine of one scene.
//
// Particle order.  The reference never moves particle data: every substep it
// sorts (Morton key, 0..n-1) and gathers through the permutation, so that
// the particles of a CTA are likely to share its shared-memory tile.  Here
// the particles are ordered by stencil base cell, grouped in bins of
// 8 x 4 x 4 cells, which is what the P2G kernel needs: all particles of a
// cell scatter to the same 27 nodes.  A substep from parity p, state P[p]
// filed into counter set p:
//   bin order: bin and cell starts from set p, gidx[new slot] = old slot;
//   P2G: one warp per (bin, layer) item, lane = cell, reading P[p] via gidx;
//   grid update;
//   G2P reads P[p] through gidx and writes P[1-p] at the new slot, i.e. the
//       state is regrouped for free, carries sigma (slot -> original slot)
//       along and files every particle into set 1-p for the next substep.
// The reference's keys and sort permutation of a substep are a function of
// the state the substep started from, which stays intact in P[p] until the
// next substep; mpm_get_sort recomputes them from it with the bit-exact key
// kernel and radix sort of sort.cu.  Readback scatters through sigma back to
// the original order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.h"
#include "mpm_b200.h"

using mpm::SimParams;

namespace {

thread_local std::string g_global_error;

constexpr int kNoSort = -1;
enum class GridView { kVelocity, kAccum };

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace

struct mpm_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    uint32_t checks = 0;

    // Scenes: config, constants and offsets (host copy of the device table).
    std::vector<mpm_config> cfg;
    std::vector<SimParams> prm;
    int scenes = 0;
    long long g_total = 0;      // grid nodes
    long long cells_total = 0;  // cells of all bins (incl. each overflow bin)
    long long bins_total = 0;   // bin entries: nb + 2 per scene
    long long bins_scan = 0;    // bins scanned: nb + 1 per scene
    SimParams* d_prm = nullptr;
    long long* d_poff = nullptr;     // S + 1 first slots
    long long* d_goff = nullptr;     // S + 1 first nodes
    long long* d_itemoff = nullptr;  // S + 1 first P2G items
    long long* d_clroff = nullptr;   // S + 1 first listed bins of the set being cleared
    mpm::SceneTable table{};

    bool initialized = false;
    long long n = 0;  // particles of all scenes
    int max_n = 0;    // largest scene
    long long cap_n = 0;     // particles, largest scene and sort scratch bytes the
    int cap_max_n = 0;       // particle buffers were allocated for
    size_t cap_sort = 0;
    float* P[2] = {nullptr, nullptr};        // particle-major state, 24 floats per particle
    int32_t* sigma[2] = {nullptr, nullptr};  // slot -> original slot (global)
    int32_t* gidx = nullptr;                 // new slot -> old slot of the current binning
    int4* crowd = nullptr;                   // P2G's crowded-cell list
    int crowd_cap = 0;
    int32_t* pcell = nullptr;                // global cell of each slot of P[parity]
    int32_t* ccur = nullptr;                 // slot cursor of every cell (the ordering's scatter)
    int32_t* ref_keys = nullptr;             // mpm_get_sort: keys in original order (one scene)
    int32_t* ref_perm = nullptr;             // mpm_get_sort: stable sort permutation
    void* sort_mem = nullptr;
    // float3 positions, all scenes, original order: two buffers written by
    // alternate exports, so that the host can read one back on copy_stream
    // while the next frame computes (pos_ready: export done; copy_done: the
    // read-back of that buffer done).
    float* pos_buf[2] = {nullptr, nullptr};
    int pos_cur = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t pos_ready[2] = {nullptr, nullptr};
    cudaEvent_t copy_done[2] = {nullptr, nullptr};

    float4* accum = nullptr;
    float4* vgrid = nullptr;
    float* sdf = nullptr;
    // Binning: two counter sets (cell counts, bin counts, bin lists) in one
    // allocation, the bin and cell starts of the current order, and ctl =
    // {list lengths of set 0 (S), of set 1 (S), P2G work, G2P work, crowded-cell
    // list length, crowded-cell entries taken}.
    void* bins_mem = nullptr;
    void* tiles_mem = nullptr;  // grid-update tile marks: stamp, mark[bins_total], dirty[bins_total]
    mpm::TileMarks tiles{};
    mpm::BinSet bins[2] = {};
    int32_t* bstart = nullptr;
    int32_t* cstart = nullptr;
    uint8_t* corder = nullptr;  // P2G's order of each listed bin's cells
    int32_t* bpart = nullptr;  // chunk sums of the bin scan: scenes x scan_chunks
    int scan_chunks = 1;
    uint32_t* ctl = nullptr;
    uint32_t* d_flags = nullptr;  // [0] health bits, [1] kernel status bits
    uint32_t wait_test = 0;       // MPM_WAIT_TEST_* (test hooks of the bounded device waits)

    float* staging = nullptr;  // device staging for imports/exports
    size_t staging_bytes = 0;

    int parity = 0;
    int sort_src = kNoSort;
    int partial_stage = 0;  // last MPM_STAGE_* run by mpm_substep_partial, 0 = none
    bool accum_dirty = false;
    GridView grid_view = GridView::kVelocity;

    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaGraph_t graph_src[2] = {nullptr, nullptr};
    int graph_kernels[2] = {0, 0};

    // Stage timing: kTimingMarks event-record nodes per substep graph, pointed
    // at a fresh slot of `tev` before each launch (scratch events once full).
    static constexpr int kTimingMarks = 5;
    int timing_cap = 0;
    int timing_used = 0;
    cudaEvent_t* tev = nullptr;
    cudaEvent_t tscratch[kTimingMarks] = {};
    cudaGraphNode_t tnode[2][kTimingMarks] = {};

    int64_t substeps = 0;
    int64_t kernel_launches = 0;
    int64_t sort_passes = 0;
    uint32_t health = 0;

    // Learned large step (engines of one scene): the RATIO x DT parameter
    // table, the packed corrector, the per-step density-change statistic and
    // the buffers of the collection probe (by original index).
    int ratio = 4;
    float max_density_change = 0.02f;
    bool mlp_set = false;
    SimParams* d_prm_large = nullptr;
    mpm::SceneTable table_large{};
    mpm::MlpPacked* mlp = nullptr;
    mpm::MlpTc* mlp_tc = nullptr;
    int corrector_kernel = MPM_CORRECTOR_TCGEN05;
    float* d_params = nullptr;
    float* d_stat = nullptr;
    float* feat_all = nullptr;  // [n][16]
    float* vlarge = nullptr;    // [n][3]
    float* vplain = nullptr;    // [n][3]
    int64_t large_steps = 0;
    int64_t fallbacks = 0;
    double last_density_change = 0.0;
    int fallback_rule = MPM_FALLBACK_DENSITY_CHANGE;
    // The checked learned step with its fallback decided on the device: a
    // graph per parity (large step, decision, conditional fallback body).
    bool fallback_on_device = true;
    bool l2_window = false;  // the accumulation grid is a persisting L2 window on `stream`
    cudaGraph_t lgraph_src[2] = {nullptr, nullptr};
    cudaGraphExec_t lgraph[2] = {nullptr, nullptr};
    int lgraph_kernels[2] = {0, 0};
    long long* d_lcount = nullptr;  // accepted, rejected large steps (device decision)
    float* d_llast = nullptr;       // the last decision's three means and its statistic
    long long lcount_host[2] = {0, 0};  // d_lcount as last read
    int lbody_kernels = 0;              // kernels of one fallback body
    double last_stats[3] = {0.0, 0.0, 0.0};  // the three means of the last checked large step

    // Launch shapes of the substep (mpm_autotune / mpm_set_tuning).
    mpm_tuning tune{12, 256, 256, 0.f, 0.f, 0.f, 0};
};

namespace {

mpm_status record(mpm_engine* e, mpm_status s, const std::string& msg) {
    if (e) e->last_error = msg;
    else g_global_error = msg;
    return s;
}

mpm_status cuda_fail(mpm_engine* e, cudaError_t err, const char* what) {
    cudaGetLastError();  // clear a non-sticky error
    std::string msg = std::string("CUDA error in ") + what + ": " + cudaGetErrorName(err) + " (" +
                      cudaGetErrorString(err) + ")";
    return record(e, err == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA, msg);
}

#define CK(e, call)                                                  \
    do {                                                             \
        cudaError_t err_ = (call);                                   \
        if (err_ != cudaSuccess) return cuda_fail((e), err_, #call); \
    } while (0)

template <typename T>
void free_dev(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// The learned-step graphs depend on the corrector, the rule, the threshold,
// the launch shapes and the buffers: rebuilt when any of them changes.
void destroy_learned_graphs(mpm_engine* e) {
    for (int k = 0; k < 2; ++k) {
        if (e->lgraph[k]) cudaGraphExecDestroy(e->lgraph[k]);
        if (e->lgraph_src[k]) cudaGraphDestroy(e->lgraph_src[k]);
        e->lgraph[k] = nullptr;
        e->lgraph_src[k] = nullptr;
        e->lgraph_kernels[k] = 0;
    }
}

// Buffers of the learned large step, sized by the particle count; allocated
// when first needed after an init.
void free_learned_buffers(mpm_engine* e) {
    free_dev(e->feat_all);
    free_dev(e->vlarge);
    free_dev(e->vplain);
}

void free_particles(mpm_engine* e) {
    destroy_learned_graphs(e);
    for (int k = 0; k < 2; ++k) {
        free_dev(e->P[k]);
        free_dev(e->sigma[k]);
        if (e->graph[k]) cudaGraphExecDestroy(e->graph[k]);
        if (e->graph_src[k]) cudaGraphDestroy(e->graph_src[k]);
        e->graph[k] = nullptr;
        e->graph_src[k] = nullptr;
        e->graph_kernels[k] = 0;
    }
    free_dev(e->gidx);
    free_dev(e->crowd);
    free_dev(e->pcell);
    free_dev(e->ref_keys);
    free_dev(e->ref_perm);
    free_dev(e->sort_mem);
    free_dev(e->pos_buf[0]);
    free_dev(e->pos_buf[1]);
    free_learned_buffers(e);
    // No buffer is left: the reuse test in alloc_particles must fail.
    e->cap_n = 0;
    e->cap_max_n = 0;
    e->cap_sort = 0;
    e->initialized = false;
}

mpm_status ensure_staging(mpm_engine* e, size_t bytes) {
    if (e->staging_bytes >= bytes) return MPM_OK;
    free_dev(e->staging);
    e->staging_bytes = 0;
    CK(e, cudaMalloc(&e->staging, bytes));
    e->staging_bytes = bytes;
    return MPM_OK;
}

mpm_status alloc_particles(mpm_engine* e, long long n, int max_n, size_t sort_bytes) {
    if (e->cap_n > 0 && n <= e->cap_n && max_n <= e->cap_max_n && sort_bytes <= e->cap_sort) {
        // The buffers of an earlier init are large enough: keep them (freeing
        // and allocating half a gigabyte takes from a few to hundreds of
        // milliseconds).  The substep graphs are captured again by the caller;
        // the learned-step buffers, sized by the earlier n, are allocated
        // again when next needed.  Work of the earlier state (an asynchronous
        // positions read-back on the copy stream included) ends first.
        CK(e, cudaStreamSynchronize(e->stream));
        CK(e, cudaStreamSynchronize(e->copy_stream));
        destroy_learned_graphs(e);
        for (int k = 0; k < 2; ++k) {
            if (e->graph[k]) cudaGraphExecDestroy(e->graph[k]);
            if (e->graph_src[k]) cudaGraphDestroy(e->graph_src[k]);
            e->graph[k] = nullptr;
            e->graph_src[k] = nullptr;
            e->graph_kernels[k] = 0;
        }
        free_learned_buffers(e);
        e->n = n;
        e->max_n = max_n;
        e->initialized = false;
        return MPM_OK;
    }
    free_particles(e);  // also zeroes the recorded capacities
    e->n = n;
    e->max_n = max_n;
    const size_t cap = (size_t)std::max(n, 1LL);
    const size_t ibytes = cap * sizeof(int32_t);
    for (int k = 0; k < 2; ++k) {
        CK(e, cudaMalloc(&e->P[k], cap * mpm::kAFloats * sizeof(float)));
        CK(e, cudaMalloc(&e->sigma[k], ibytes));
    }
    CK(e, cudaMalloc(&e->gidx, ibytes));
    // A crowded-cell entry holds at least one particle beyond a cap of 4 or
    // more (the smallest mpm_set_tuning accepts), and a cell yields one entry
    // per 256 of them: fewer than n / 4 entries.
    e->crowd_cap = (int)std::min<long long>(cap / 4 + 64, 0x7fffffffLL);
    CK(e, cudaMalloc(&e->crowd, (size_t)e->crowd_cap * sizeof(int4)));
    CK(e, cudaMalloc(&e->pcell, ibytes));
    const size_t sbytes = (size_t)std::max(max_n, 1) * sizeof(int32_t);
    CK(e, cudaMalloc(&e->ref_keys, sbytes));
    CK(e, cudaMalloc(&e->ref_perm, sbytes));
    CK(e, cudaMalloc(&e->sort_mem, sort_bytes));
    CK(e, cudaMalloc(&e->pos_buf[0], cap * 3 * sizeof(float)));
    CK(e, cudaMalloc(&e->pos_buf[1], cap * 3 * sizeof(float)));
    // Recorded only now: after a failed allocation above the capacities stay
    // zero, so the next init allocates again instead of reusing null buffers.
    e->cap_n = std::max(n, 1LL);
    e->cap_max_n = max_n;
    e->cap_sort = sort_bytes;
    return MPM_OK;
}

// Words of one counter set: cell counts, bin counts and bin lists, rounded up
// to 256 bytes so that the second set's cell counts stay 16-byte aligned for
// vector access.
size_t bins_set_words(const mpm_engine* e) {
    return align_up((size_t)e->cells_total + 2 * (size_t)e->bins_total, 64);
}
size_t bins_bytes(const mpm_engine* e) { return 2 * bins_set_words(e) * sizeof(uint32_t); }
size_t tiles_bytes(const mpm_engine* e) { return (size_t)(1 + e->bins_total) * sizeof(uint32_t) + (size_t)e->bins_total; }

void carve_bins(mpm_engine* e) {
    uint32_t* base = static_cast<uint32_t*>(e->bins_mem);
    for (int k = 0; k < 2; ++k) {
        uint32_t* s = base + k * bins_set_words(e);  // cell counts first: 16-byte aligned
        e->bins[k].ccount = s;
        e->bins[k].bcount = s + e->cells_total;
        e->bins[k].blist = reinterpret_cast<int32_t*>(e->bins[k].bcount + e->bins_total);
        e->bins[k].nlist = e->ctl + k * e->scenes;
    }
}

// Uploads the scene table (after the particle offsets change).
mpm_status upload_table(mpm_engine* e) {
    std::vector<long long> poff(e->scenes + 1), goff(e->scenes + 1);
    for (int s = 0; s < e->scenes; ++s) {
        poff[s] = e->prm[s].poff;
        goff[s] = e->prm[s].goff;
    }
    poff[e->scenes] = e->n;
    goff[e->scenes] = e->g_total;
    CK(e, cudaMemcpyAsync(e->d_prm, e->prm.data(), e->scenes * sizeof(SimParams), cudaMemcpyHostToDevice, e->stream));
    CK(e, cudaMemcpyAsync(e->d_poff, poff.data(), poff.size() * sizeof(long long), cudaMemcpyHostToDevice, e->stream));
    CK(e, cudaMemcpyAsync(e->d_goff, goff.data(), goff.size() * sizeof(long long), cudaMemcpyHostToDevice, e->stream));
    // Pageable host copies: wait before the vectors go out of scope.
    CK(e, cudaStreamSynchronize(e->stream));
    return MPM_OK;
}

// The tile marks when the grid update works on touched tiles only
// (grid_block 0), else none: every node is updated.
mpm::TileMarks active_tiles(const mpm_engine* e) { return e->tune.grid_block == 0 ? e->tiles : mpm::TileMarks{}; }

// Enqueues stages `from`..`upto` (MPM_STAGE_*) of one substep from parity
// `par`, for all scenes.  With `marks` (only while capturing a graph), records
// marks[0..4] as event-record nodes before the ordering and after each stage.
int enqueue_substep(mpm_engine* e, int par, int from, int upto, const cudaEvent_t* marks = nullptr) {
    const mpm::SceneTable& sc = e->table;
    cudaStream_t st = e->stream;
    auto mark = [&](int k) {
        if (marks) cudaEventRecordWithFlags(marks[k], st, cudaEventRecordExternal);
    };
    int launches = 0;
    uint32_t* work = e->ctl + 2 * e->scenes;
    mark(0);
    if (from <= MPM_STAGE_SORT && upto >= MPM_STAGE_SORT)
        launches += mpm::launch_bin_order(sc, e->n, e->bins_scan, e->bins[par], e->bins[1 - par], e->bstart, e->cstart,
                                          e->pcell, e->ccur, e->gidx, e->corder, e->d_itemoff, e->d_clroff, work, e->bpart,
                                          e->scan_chunks, active_tiles(e), st);
    mark(1);
    if (from <= MPM_STAGE_P2G && upto >= MPM_STAGE_P2G)
        launches += mpm::launch_p2g(sc, e->n, e->bins_scan, e->P[par], e->gidx, e->cstart, e->bins[par], e->corder, e->d_itemoff,
                                    work, e->accum, e->crowd, e->crowd_cap, e->d_flags + 1, st, e->tune.p2g_ctas_per_sm,
                                    e->tune.p2g_cell_cap);
    mark(2);
    if (from <= MPM_STAGE_GRID && upto >= MPM_STAGE_GRID)
        launches += mpm::launch_grid_update(sc, e->prm[0], e->g_total, e->accum, e->vgrid, e->sdf, active_tiles(e), st,
                                            e->tune.grid_block);
    mark(3);
    if (from <= MPM_STAGE_G2P && upto >= MPM_STAGE_G2P)
        launches += mpm::launch_g2p(sc, e->prm[0], e->n, e->P[par], e->P[1 - par], e->gidx, e->sigma[par],
                                    e->sigma[1 - par], e->vgrid, e->sdf, e->pcell, e->bins[1 - par],
                                    e->d_flags, st, nullptr, e->tune.g2p_block);
    mark(4);
    return launches;
}

mpm_status capture_graphs(mpm_engine* e) {
    destroy_learned_graphs(e);  // they embed the launch shapes too
    // Touched tiles only: after updates of every node any tile may hold
    // velocities, so the first tile update resets every tile not marked.
    if (active_tiles(e).mark) CK(e, cudaMemsetAsync(e->tiles.dirty, 1, (size_t)e->bins_total, e->stream));
    const bool timed = e->timing_cap > 0;
    for (int par = 0; par < 2; ++par) {
        if (e->graph[par]) cudaGraphExecDestroy(e->graph[par]);
        if (e->graph_src[par]) cudaGraphDestroy(e->graph_src[par]);
        e->graph[par] = nullptr;
        e->graph_src[par] = nullptr;
        cudaGraph_t g = nullptr;
        CK(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        const int launches = enqueue_substep(e, par, MPM_STAGE_SORT, MPM_STAGE_G2P, timed ? e->tscratch : nullptr);
        const cudaError_t launch_err = cudaGetLastError();
        const cudaError_t end_err = cudaStreamEndCapture(e->stream, &g);
        if (launch_err != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(e, launch_err, "substep capture");
        }
        CK(e, end_err);
        e->graph_src[par] = g;
        if (timed) {
            for (int k = 0; k < mpm_engine::kTimingMarks; ++k) e->tnode[par][k] = nullptr;
            // Find the event-record nodes by the scratch event each records.
            size_t count = 0;
            CK(e, cudaGraphGetNodes(g, nullptr, &count));
            std::vector<cudaGraphNode_t> nodes(count);
            CK(e, cudaGraphGetNodes(g, nodes.data(), &count));
            for (cudaGraphNode_t nd : nodes) {
                cudaGraphNodeType type;
                CK(e, cudaGraphNodeGetType(nd, &type));
                if (type != cudaGraphNodeTypeEventRecord) continue;
                cudaEvent_t ev;
                CK(e, cudaGraphEventRecordNodeGetEvent(nd, &ev));
                for (int k = 0; k < mpm_engine::kTimingMarks; ++k)
                    if (ev == e->tscratch[k]) e->tnode[par][k] = nd;
            }
            for (int k = 0; k < mpm_engine::kTimingMarks; ++k)
                if (!e->tnode[par][k]) return record(e, MPM_ERR_CUDA, "stage-timing event node missing from the graph");
        }
        CK(e, cudaGraphInstantiate(&e->graph[par], g, 0));
        e->graph_kernels[par] = launches;
    }
    return MPM_OK;
}

void free_timing(mpm_engine* e) {
    if (e->tev) {
        for (int i = 0; i < e->timing_cap * mpm_engine::kTimingMarks; ++i) cudaEventDestroy(e->tev[i]);
        delete[] e->tev;
    }
    e->tev = nullptr;
    for (int k = 0; k < mpm_engine::kTimingMarks; ++k) {
        if (e->tscratch[k]) cudaEventDestroy(e->tscratch[k]);
        e->tscratch[k] = nullptr;
    }
    e->timing_cap = 0;
    e->timing_used = 0;
}

mpm_status sync_and_collect(mpm_engine* e) {
    uint32_t flags[2] = {0, 0};
    CK(e, cudaMemcpyAsync(flags, e->d_flags, sizeof(flags), cudaMemcpyDeviceToHost, e->stream));
    CK(e, cudaStreamSynchronize(e->stream));
    e->health |= flags[0];
    if (flags[1] & (mpm::kStatusTimeout | mpm::kStatusBinning | mpm::kStatusCrowdList)) {
        CK(e, cudaMemsetAsync(e->d_flags + 1, 0, sizeof(uint32_t), e->stream));
        if (flags[1] & mpm::kStatusBinning)
            return record(e, MPM_ERR_CUDA, "internal error: a particle was not in the cell it was filed under");
        if (flags[1] & mpm::kStatusCrowdList)
            return record(e, MPM_ERR_CUDA, "internal error: the crowded-cell list of P2G overflowed");
        return record(e, MPM_ERR_TIMEOUT, "a bounded device-side wait gave up");
    }
    return MPM_OK;
}

mpm_status check_health(mpm_engine* e) {
    const uint32_t seen = e->health & e->checks;
    if (seen & MPM_HEALTH_NONFINITE)
        return record(e, MPM_ERR_NONFINITE_STATE, "a particle position or velocity is not finite");
    if (seen & MPM_HEALTH_OUT_OF_GRID)
        return record(e, MPM_ERR_OUT_OF_GRID, "a particle position is outside the grid");
    return MPM_OK;
}

bool finite_cfg(const mpm_config* c) {
    return std::isfinite(c->gravity) && std::isfinite(c->dt) && std::isfinite(c->gamma) &&
           std::isfinite(c->compression) && std::isfinite(c->resolution);
}

mpm_status export_positions(mpm_engine* e);

// Uploads each scene's 26-plane host state and imports it (init_rules:
// Engine::init), then files all particles into counter set 0.
mpm_status load_states(mpm_engine* e, const float* const* soa26_host, bool init_rules) {
    for (int s = 0; s < e->scenes; ++s) {
        const SimParams& p = e->prm[s];
        if (p.n <= 0) continue;
        const size_t plane = (size_t)p.n * sizeof(float);
        mpm_status st = ensure_staging(e, (size_t)MPM_PARTICLE_PLANES * plane);
        if (st != MPM_OK) return st;
        // Only the planes the import reads cross the bus: VOL and MASS are
        // uniform and live in SimParams, and with the init rules
        // (initFMatrices) F's diagonal is overwritten with 1 (21 of 26
        // planes; the import reads the skipped diagonal planes and discards
        // them).
        const char* src = reinterpret_cast<const char*>(soa26_host[s]);
        char* dst = reinterpret_cast<char*>(e->staging);
        if (init_rules) {
            const int runs[3][2] = {{0, MPM_F00}, {MPM_F00 + 1, MPM_F00 + 4}, {MPM_F00 + 5, MPM_F00 + 8}};
            for (const auto& r : runs)
                CK(e, cudaMemcpyAsync(dst + r[0] * plane, src + r[0] * plane, (size_t)(r[1] - r[0]) * plane,
                                      cudaMemcpyHostToDevice, e->stream));
        } else {
            CK(e, cudaMemcpyAsync(dst, src, (size_t)MPM_VOL * plane, cudaMemcpyHostToDevice, e->stream));
        }
        e->kernel_launches += mpm::launch_state_import(p, e->staging, e->P[0] + p.poff * mpm::kAFloats,
                                                       e->sigma[0] + p.poff, init_rules, e->stream);
        CK(e, cudaGetLastError());
    }
    // Both counter sets empty, then the imported particles filed into set 0.
    CK(e, cudaMemsetAsync(e->bins_mem, 0, bins_bytes(e), e->stream));
    CK(e, cudaMemsetAsync(e->ctl, 0, (2 * e->scenes + 4) * sizeof(uint32_t), e->stream));
    e->kernel_launches += mpm::launch_bin_count(e->table, e->n, e->P[0], e->pcell, e->bins[0], e->stream);
    CK(e, cudaGetLastError());
    e->parity = 0;
    e->sort_src = kNoSort;
    e->partial_stage = 0;
    CK(e, cudaMemsetAsync(e->accum, 0, (size_t)e->g_total * sizeof(float4), e->stream));
    CK(e, cudaMemsetAsync(e->vgrid, 0, (size_t)e->g_total * sizeof(float4), e->stream));
    CK(e, cudaMemsetAsync(e->tiles.dirty, 0, (size_t)e->bins_total, e->stream));  // the velocity grid is zero
    CK(e, cudaMemsetAsync(e->d_flags, 0, 2 * sizeof(uint32_t), e->stream));
    e->accum_dirty = false;
    e->grid_view = GridView::kVelocity;
    e->health = 0;
    mpm_status st = export_positions(e);
    if (st != MPM_OK) return st;
    st = capture_graphs(e);
    if (st != MPM_OK) return st;
    e->initialized = true;
    return sync_and_collect(e);
}

mpm_status enter(mpm_engine* e) {
    if (!e) return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "engine is NULL");
    e->last_error.clear();
    CK(e, cudaSetDevice(e->device));
    return MPM_OK;
}

mpm_status enter_scene(mpm_engine* e, int32_t scene) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (scene < 0 || scene >= e->scenes) return record(e, MPM_ERR_INVALID_ARGUMENT, "scene index out of range");
    return MPM_OK;
}

// Exports the current positions into the other position buffer, once any
// read-back of that buffer has finished, and makes it the current one.
mpm_status export_positions(mpm_engine* e) {
    const int b = 1 - e->pos_cur;
    CK(e, cudaStreamWaitEvent(e->stream, e->copy_done[b], 0));
    for (int sc = 0; sc < e->scenes; ++sc) {
        const SimParams& p = e->prm[sc];
        e->kernel_launches += mpm::launch_positions_export(p, e->P[e->parity] + p.poff * mpm::kAFloats,
                                                           e->sigma[e->parity] + p.poff, e->pos_buf[b] + p.poff * 3,
                                                           e->stream);
    }
    CK(e, cudaGetLastError());
    CK(e, cudaEventRecord(e->pos_ready[b], e->stream));
    e->pos_cur = b;
    return MPM_OK;
}

mpm_status run_steps(mpm_engine* e, int32_t nsub) {
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    if (nsub < 0) return record(e, MPM_ERR_INVALID_ARGUMENT, "nsub < 0");
    e->partial_stage = 0;  // a partial substep in progress is discarded (it changed no particle)
    if (e->accum_dirty) {
        CK(e, cudaMemsetAsync(e->accum, 0, (size_t)e->g_total * sizeof(float4), e->stream));
        e->accum_dirty = false;
    }
    for (int s = 0; s < nsub; ++s) {
        if (e->timing_cap > 0) {
            const int par = e->parity;
            const bool slot = e->timing_used < e->timing_cap;
            const cudaEvent_t* evs = slot ? e->tev + (size_t)e->timing_used * mpm_engine::kTimingMarks : e->tscratch;
            for (int k = 0; k < mpm_engine::kTimingMarks; ++k)
                CK(e, cudaGraphExecEventRecordNodeSetEvent(e->graph[par], e->tnode[par][k], evs[k]));
            if (slot) ++e->timing_used;
        }
        CK(e, cudaGraphLaunch(e->graph[e->parity], e->stream));
        e->kernel_launches += e->graph_kernels[e->parity];
        e->sort_src = e->parity;
        e->parity ^= 1;
        ++e->substeps;
    }
    if (nsub > 0) e->grid_view = GridView::kVelocity;
    return export_positions(e);
}

// Engine with `count` scenes; grid arrays, counter sets and the scene table
// are allocated here, particle arrays by the first init.
// The P2G accumulation grid as a persisting L2 window on the engine's
// stream (the substep graphs captured from it carry the window): its
// red.global.add reductions and the grid update's pass over it then hit L2
// while the particle streams go by.  Measured on the 2M dam break: P2G 15 %
// and the grid update 10 % faster in crowded states, the substep 1-8 %; no
// effect on G2P.  Only a grid that fits in the largest set-aside gets the
// window: on the 256^3 grid (268 MB) a partial window took 83 MB of L2 from
// the other arrays and made G2P 50 % and the grid update 2.3x slower.  The
// set-aside is a limit of this process's CUDA context (grown to the window
// when smaller, never shrunk); mpm_destroy resets the persisting lines.
// Failures are ignored: the window is only a hint.
void keep_accum_in_l2(mpm_engine* e, int device) {
    int max_persist = 0, max_window = 0;
    if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, device) != cudaSuccess ||
        max_persist <= 0 || max_window <= 0) {
        cudaGetLastError();
        return;
    }
    const size_t bytes = (size_t)e->g_total * sizeof(float4);
    if (bytes > (size_t)max_persist || bytes > (size_t)max_window) return;
    size_t limit = 0;
    if (cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize) == cudaSuccess && limit < bytes)
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, std::min(bytes, (size_t)max_persist));
    if (cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize) != cudaSuccess || limit == 0) {
        cudaGetLastError();
        return;
    }
    cudaStreamAttrValue av{};
    av.accessPolicyWindow.base_ptr = e->accum;
    av.accessPolicyWindow.num_bytes = bytes;
    av.accessPolicyWindow.hitRatio = std::min(1.0f, (float)limit / (float)bytes);
    av.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    av.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cudaStreamSetAttribute(e->stream, cudaStreamAttributeAccessPolicyWindow, &av);
    cudaGetLastError();
    e->l2_window = true;
}

mpm_status create_engine(const mpm_config* cfgs, int32_t count, int32_t device, mpm_engine** out) {
    g_global_error.clear();
    if (!cfgs || !out) return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "configs and out must be non-NULL");
    *out = nullptr;
    if (count <= 0 || count > 65536) return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "scene count out of range");
    long long g_total = 0, cells_total = 0, bins_total = 0;
    std::vector<SimParams> prm(count);
    for (int s = 0; s < count; ++s) {
        const mpm_config* cfg = cfgs + s;
        if (cfg->size_x <= 0 || cfg->size_y <= 0 || cfg->size_z <= 0)
            return record(nullptr, MPM_ERR_BAD_CONFIG, "SIZE_X/Y/Z must be positive");
        const long long g = (long long)cfg->size_x * cfg->size_y * cfg->size_z;
        if (g > 0x7fffffffLL) return record(nullptr, MPM_ERR_BAD_CONFIG, "grid has more than 2^31-1 nodes");
        if (!finite_cfg(cfg)) return record(nullptr, MPM_ERR_BAD_CONFIG, "a float parameter is not finite");
        SimParams& p = prm[s];
        p.sx = cfg->size_x;
        p.sy = cfg->size_y;
        p.sz = cfg->size_z;
        p.padding = cfg->padding;
        p.gravity = cfg->gravity;
        p.dt = cfg->dt;
        p.gamma = cfg->gamma;
        p.compression = cfg->compression;
        p.pvol = cfg->resolution * cfg->resolution * cfg->resolution;  // kernels.cu:356
        p.pmass = 1.0f;                                                // kernels.cu:357
        p.n = 0;
        p.g = (int)g;
        p.nbx = (cfg->size_x + 2 + mpm::kBinX - 1) / mpm::kBinX;
        p.nby = (cfg->size_y + 2 + mpm::kBinY - 1) / mpm::kBinY;
        p.nbz = (cfg->size_z + 2 + mpm::kBinZ - 1) / mpm::kBinZ;
        p.nb = p.nbx * p.nby * p.nbz;
        p.poff = 0;
        p.goff = g_total;
        p.coff = cells_total;
        p.boff = bins_total;
        g_total += g;
        cells_total += (long long)(p.nb + 1) * mpm::kBinCells;
        bins_total += p.nb + 2;
    }
    if (cells_total >= 0x7fffffffLL || g_total >= (1LL << 40))
        return record(nullptr, MPM_ERR_BAD_CONFIG, "grids too large for the cell index");

    int ndev = 0;
    cudaError_t err = cudaGetDeviceCount(&ndev);
    if (err != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return record(nullptr, MPM_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(err));
    }
    if (device < 0 || device >= ndev) return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "device index out of range");
    cudaDeviceProp prop;
    err = cudaGetDeviceProperties(&prop, device);
    if (err != cudaSuccess) return cuda_fail(nullptr, err, "cudaGetDeviceProperties");
    if (prop.major != 10 || prop.minor != 0)
        return record(nullptr, MPM_ERR_NO_DEVICE,
                      std::string("this library is built for sm_100a (B200); device is ") + prop.name);

    mpm_engine* e = new mpm_engine();
    e->device = device;
    e->cfg.assign(cfgs, cfgs + count);
    e->prm = prm;
    e->scenes = count;
    e->g_total = g_total;
    e->cells_total = cells_total;
    e->bins_total = bins_total;
    e->bins_scan = bins_total - count;
    for (const SimParams& p : prm) e->scan_chunks = std::max(e->scan_chunks, mpm::bin_scan_chunks(p.nb + 1));

    auto fail = [&](mpm_status s) {
        g_global_error = e->last_error;
        mpm_destroy(e);
        return s;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(cuda_fail(e, cudaGetLastError(), "cudaSetDevice"));
    if ((err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (err = cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(cuda_fail(e, err, "cudaStreamCreate"));
    for (int k = 0; k < 2; ++k)
        if ((err = cudaEventCreateWithFlags(&e->pos_ready[k], cudaEventDisableTiming)) != cudaSuccess ||
            (err = cudaEventCreateWithFlags(&e->copy_done[k], cudaEventDisableTiming)) != cudaSuccess)
            return fail(cuda_fail(e, err, "cudaEventCreate"));
    if ((err = cudaMalloc(&e->accum, (size_t)g_total * sizeof(float4))) != cudaSuccess ||
        (err = cudaMalloc(&e->vgrid, (size_t)g_total * sizeof(float4))) != cudaSuccess ||
        (err = cudaMalloc(&e->sdf, (size_t)g_total * sizeof(float))) != cudaSuccess ||
        (err = cudaMalloc(&e->d_flags, 2 * sizeof(uint32_t))) != cudaSuccess ||
        (err = cudaMalloc(&e->ctl, (2 * count + 4) * sizeof(uint32_t))) != cudaSuccess ||
        (err = cudaMalloc(&e->bins_mem, bins_bytes(e))) != cudaSuccess ||
        (err = cudaMalloc(&e->tiles_mem, tiles_bytes(e))) != cudaSuccess ||
        (err = cudaMalloc(&e->bstart, (size_t)bins_total * sizeof(int32_t))) != cudaSuccess ||
        (err = cudaMalloc(&e->bpart, (size_t)count * e->scan_chunks * sizeof(int32_t))) != cudaSuccess ||
        (err = cudaMalloc(&e->cstart, (size_t)cells_total * sizeof(int32_t))) != cudaSuccess ||
        (err = cudaMalloc(&e->ccur, (size_t)cells_total * sizeof(int32_t))) != cudaSuccess ||
        (err = cudaMalloc(&e->corder, (size_t)cells_total)) != cudaSuccess ||
        (err = cudaMalloc(&e->d_prm, count * sizeof(SimParams))) != cudaSuccess ||
        (err = cudaMalloc(&e->d_poff, (count + 1) * sizeof(long long))) != cudaSuccess ||
        (err = cudaMalloc(&e->d_goff, (count + 1) * sizeof(long long))) != cudaSuccess ||
        (err = cudaMalloc(&e->d_itemoff, (count + 1) * sizeof(long long))) != cudaSuccess ||
        (err = cudaMalloc(&e->d_clroff, (count + 1) * sizeof(long long))) != cudaSuccess)
        return fail(cuda_fail(e, err, "cudaMalloc(grid)"));
    carve_bins(e);
    e->tiles.stamp = static_cast<uint32_t*>(e->tiles_mem);
    e->tiles.mark = e->tiles.stamp + 1;
    e->tiles.dirty = reinterpret_cast<uint8_t*>(e->tiles.mark + e->bins_total);
    e->tiles.count = e->bins_total;
    keep_accum_in_l2(e, device);
    e->table.prm = e->d_prm;
    e->table.poff = e->d_poff;
    e->table.goff = e->d_goff;
    e->table.count = count;
    // A grid of 2^23 nodes or more (256^3) is mostly empty in the workloads
    // measured; there the touched-tile update is 2.7x faster than the update
    // of every node, while on 128^3 it ties and on 64^3 it is slower.
    if (count == 1 && g_total >= (1LL << 23)) e->tune.grid_block = 0;
    cudaMemsetAsync(e->accum, 0, (size_t)g_total * sizeof(float4), e->stream);
    cudaMemsetAsync(e->vgrid, 0, (size_t)g_total * sizeof(float4), e->stream);
    cudaMemsetAsync(e->tiles_mem, 0, tiles_bytes(e), e->stream);
    cudaMemsetAsync(e->d_flags, 0, 2 * sizeof(uint32_t), e->stream);
    // An empty triangle list leaves sqrt(1e30) everywhere (kernels.cu:289,299).
    e->kernel_launches += mpm::launch_fill(e->sdf, g_total, sqrtf(1e30f), e->stream);
    if ((err = cudaGetLastError()) != cudaSuccess) return fail(cuda_fail(e, err, "sdf fill"));
    if (upload_table(e) != MPM_OK) return fail(MPM_ERR_CUDA);
    if ((err = cudaStreamSynchronize(e->stream)) != cudaSuccess) return fail(cuda_fail(e, err, "create sync"));
    *out = e;
    return MPM_OK;
}

// init_rules: Engine::init's initFMatrices (false: the state is taken as it
// is, with VOL and MASS from vol / mass when given).
mpm_status init_all(mpm_engine* e, const int64_t* counts, const float* const* soa26_host, bool init_rules = true,
                    const float* vol = nullptr, const float* mass = nullptr) {
    long long total = 0;
    int max_n = 0;
    size_t sort_bytes = mpm::sort_scratch_bytes(1);  // radix-sort scratch of mpm_get_sort: any scene
    for (int s = 0; s < e->scenes; ++s) {
        if (counts[s] < 0 || counts[s] > 0x7fffffffLL - 64) return record(e, MPM_ERR_INVALID_ARGUMENT, "n out of range");
        if (counts[s] > 0 && !soa26_host[s]) return record(e, MPM_ERR_INVALID_ARGUMENT, "soa26_host is NULL");
        total += counts[s];
        max_n = std::max(max_n, (int)counts[s]);
        sort_bytes = std::max(sort_bytes, mpm::sort_scratch_bytes(std::max((int)counts[s], 1)));
    }
    if (total > 0x7fffffffLL - 64) return record(e, MPM_ERR_INVALID_ARGUMENT, "more than 2^31 particles in total");
    mpm_status st = alloc_particles(e, total, max_n, sort_bytes);
    if (st != MPM_OK) return st;
    long long off = 0;
    for (int s = 0; s < e->scenes; ++s) {
        SimParams& p = e->prm[s];
        p.n = (int)counts[s];
        p.poff = off;
        p.pvol = vol ? vol[s] : e->cfg[s].resolution * e->cfg[s].resolution * e->cfg[s].resolution;
        p.pmass = mass ? mass[s] : 1.0f;
        off += counts[s];
    }
    if ((st = upload_table(e)) != MPM_OK) return st;
    e->substeps = 0;
    return load_states(e, soa26_host, init_rules);
}

// ------------------------------------------------------ learned step ----
// Parameters of the large step: every scene's with DT x RATIO.
SimParams large_params(const mpm_engine* e, int s) {
    SimParams p = e->prm[s];
    p.dt = e->prm[s].dt * (float)e->ratio;
    return p;
}

mpm_status prepare_large(mpm_engine* e) {
    if (!e->d_prm_large) {
        CK(e, cudaMalloc(&e->d_prm_large, e->scenes * sizeof(SimParams)));
        CK(e, cudaMalloc(&e->d_stat, 3 * sizeof(float)));
    }
    std::vector<SimParams> big(e->scenes);
    for (int s = 0; s < e->scenes; ++s) big[s] = large_params(e, s);
    CK(e, cudaMemcpyAsync(e->d_prm_large, big.data(), big.size() * sizeof(SimParams), cudaMemcpyHostToDevice,
                          e->stream));
    CK(e, cudaStreamSynchronize(e->stream));
    e->table_large = e->table;
    e->table_large.prm = e->d_prm_large;
    if (e->accum_dirty) {
        CK(e, cudaMemsetAsync(e->accum, 0, (size_t)e->g_total * sizeof(float4), e->stream));
        e->accum_dirty = false;
    }
    e->partial_stage = 0;
    return MPM_OK;
}

// Advection blend of the large step: RATIO substeps under a constant
// acceleration move a particle by RATIO DT (v_old + (RATIO + 1) / (2 RATIO)
// (v_new - v_old)).
float large_blend(const mpm_engine* e) { return (float)(e->ratio + 1) / (float)(2 * e->ratio); }

// One substep of RATIO x DT from parity `par` into 1 - par (learn: the
// learned, collection or uncorrected large-step G2P).
int enqueue_large(mpm_engine* e, int par, const mpm::LearnArgs* learn) {
    cudaStream_t st = e->stream;
    uint32_t* work = e->ctl + 2 * e->scenes;
    const SimParams big = large_params(e, 0);
    int launches = 0;
    launches += mpm::launch_bin_order(e->table, e->n, e->bins_scan, e->bins[par], e->bins[1 - par], e->bstart,
                                      e->cstart, e->pcell, e->ccur, e->gidx, e->corder, e->d_itemoff, e->d_clroff, work, e->bpart,
                                          e->scan_chunks, active_tiles(e), st);
    launches += mpm::launch_p2g(e->table_large, e->n, e->bins_scan, e->P[par], e->gidx, e->cstart, e->bins[par],
                                e->corder, e->d_itemoff, work, e->accum, e->crowd, e->crowd_cap, e->d_flags + 1, st, e->tune.p2g_ctas_per_sm,
                                e->tune.p2g_cell_cap);
    launches += mpm::launch_grid_update(e->table_large, big, e->g_total, e->accum, e->vgrid, e->sdf, active_tiles(e), st,
                                        e->tune.grid_block);
    launches += mpm::launch_g2p(e->table_large, big, e->n, e->P[par], e->P[1 - par], e->gidx, e->sigma[par],
                                e->sigma[1 - par], e->vgrid, e->sdf, e->pcell, e->bins[1 - par], e->d_flags,
                                st, learn);
    return launches;
}

// Files the particles of P[par] afresh into counter set `par` (both sets
// emptied first): the state of parity `par` becomes the current one again.
mpm_status rebin(mpm_engine* e, int par) {
    CK(e, cudaMemsetAsync(e->bins_mem, 0, bins_bytes(e), e->stream));
    CK(e, cudaMemsetAsync(e->ctl, 0, (2 * e->scenes + 4) * sizeof(uint32_t), e->stream));
    e->kernel_launches += mpm::launch_bin_count(e->table, e->n, e->P[par], e->pcell, e->bins[par], e->stream);
    CK(e, cudaGetLastError());
    e->parity = par;
    return MPM_OK;
}

// `count` plain substeps through the captured graphs.
mpm_status plain_substeps(mpm_engine* e, int count) {
    for (int s = 0; s < count; ++s) {
        CK(e, cudaGraphLaunch(e->graph[e->parity], e->stream));
        e->kernel_launches += e->graph_kernels[e->parity];
        e->sort_src = e->parity;
        e->parity ^= 1;
        ++e->substeps;
    }
    return MPM_OK;
}

// The fallback of a rejected large step from parity `par`, enqueued on the
// engine's stream (captured into the conditional body of the learned-step
// graph): the counter sets emptied and the start state, still intact in
// P[par], filed into set par (rebin); RATIO plain substeps; then, when RATIO
// is even, the result moved to parity 1 - par, where an accepted large step
// leaves its own: the state, its slot-to-particle map, and the counter set
// the last substep filled (its slot order and cells stay valid, so the next
// substep orders by it and clears the other set as usual).
int enqueue_fallback(mpm_engine* e, int par) {
    cudaStream_t st = e->stream;
    int launches = 0;
    launches += mpm::launch_fill(static_cast<float*>(e->bins_mem), (long long)(bins_bytes(e) / sizeof(float)), 0.0f, st);
    launches += mpm::launch_fill(reinterpret_cast<float*>(e->ctl), 2 * e->scenes + 4, 0.0f, st);
    launches += mpm::launch_bin_count(e->table, e->n, e->P[par], e->pcell, e->bins[par], st);
    int q = par;
    for (int r = 0; r < e->ratio; ++r) {
        launches += enqueue_substep(e, q, MPM_STAGE_SORT, MPM_STAGE_G2P);
        q ^= 1;
    }
    if (q != 1 - par) {
        uint32_t* sets = static_cast<uint32_t*>(e->bins_mem);
        launches += mpm::launch_copy_words(e->P[1 - par], e->P[q], e->n * mpm::kAFloats, st);
        launches += mpm::launch_copy_words(e->sigma[1 - par], e->sigma[q], e->n, st);
        launches += mpm::launch_copy_words(sets + (size_t)(1 - par) * bins_set_words(e), sets + (size_t)q * bins_set_words(e),
                                           (long long)bins_set_words(e), st);
        launches += mpm::launch_copy_words(e->ctl + (1 - par) * e->scenes, e->ctl + q * e->scenes, e->scenes, st);
    }
    return launches;
}

// Captures the checked learned step as one graph per parity: the statistic
// sums cleared, the large step (ordering, P2G, grid update, learned G2P),
// the decision kernel, and a conditional node whose body is the fallback,
// run only when the decision kernel sets its condition.  The step then costs
// no host round trip, and the state ends at parity 1 - par either way.
mpm_status capture_learned_graphs(mpm_engine* e) {
    destroy_learned_graphs(e);
    if (!e->d_lcount) {
        CK(e, cudaMalloc(&e->d_lcount, 2 * sizeof(long long)));
        CK(e, cudaMalloc(&e->d_llast, 4 * sizeof(float)));
        CK(e, cudaMemsetAsync(e->d_lcount, 0, 2 * sizeof(long long), e->stream));
        CK(e, cudaMemsetAsync(e->d_llast, 0, 4 * sizeof(float), e->stream));
        CK(e, cudaStreamSynchronize(e->stream));
        e->lcount_host[0] = e->lcount_host[1] = 0;
    }
    cudaStream_t st = e->stream;
    const bool tc = e->corrector_kernel == MPM_CORRECTOR_TCGEN05;
    for (int par = 0; par < 2; ++par) {
        mpm::LearnArgs la{e->mlp, nullptr, nullptr, e->d_stat, large_blend(e), tc ? e->mlp_tc : nullptr, e->d_flags + 1,
                          (e->wait_test & (MPM_WAIT_TEST_MMA_GIVE_UP | MPM_WAIT_TEST_MMA_EXPIRE)) >> 2};
        CK(e, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int launches = mpm::launch_fill(e->d_stat, 3, 0.0f, st);
        launches += enqueue_large(e, par, &la);
        cudaError_t err = cudaGetLastError();
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        cudaGraphConditionalHandle handle = 0;
        cudaGraphNode_t cnode = nullptr;
        cudaGraph_t body = nullptr;
        if (err == cudaSuccess) err = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd);
        if (err == cudaSuccess) err = cudaGraphConditionalHandleCreate(&handle, cg, 0, cudaGraphCondAssignDefault);
        if (err == cudaSuccess) {
            launches += mpm::launch_learned_decide(e->d_stat, e->n, e->fallback_rule, e->max_density_change, handle,
                                                   e->d_lcount, e->d_llast, st);
            err = cudaGetLastError();
        }
        if (err == cudaSuccess) err = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd);
        if (err == cudaSuccess) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeIf;
            cp.conditional.size = 1;
            err = cudaGraphAddNode(&cnode, cg, deps, nd, &cp);
            if (err == cudaSuccess) body = cp.conditional.phGraph_out[0];
        }
        if (err == cudaSuccess) err = cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies);
        cudaGraph_t g = nullptr;
        const cudaError_t end_err = cudaStreamEndCapture(st, &g);
        if (err == cudaSuccess) err = end_err;
        if (err != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return cuda_fail(e, err, "learned-step graph capture");
        }
        e->lgraph_src[par] = g;
        // The fallback body, captured into the conditional node's graph.
        CK(e, cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        const int body_launches = enqueue_fallback(e, par);
        err = cudaGetLastError();
        cudaGraph_t b2 = nullptr;
        const cudaError_t bend = cudaStreamEndCapture(st, &b2);
        if (err == cudaSuccess) err = bend;
        if (err != cudaSuccess) {
            cudaGetLastError();
            return cuda_fail(e, err, "learned-step fallback capture");
        }
        CK(e, cudaGraphInstantiate(&e->lgraph[par], g, 0));
        e->lgraph_kernels[par] = launches;
        e->lbody_kernels = body_launches;
    }
    return MPM_OK;
}

mpm_status learned_ready(mpm_engine* e) {
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    if (e->scenes != 1) return record(e, MPM_ERR_UNSUPPORTED, "the learned large step serves engines of one scene");
    return prepare_large(e);
}

}  // namespace

// -------------------------------------------------------------------------

extern "C" int32_t mpm_abi_version(void) { return MPM_ABI_VERSION; }

extern "C" const char* mpm_status_string(mpm_status s) {
    switch (s) {
        case MPM_OK: return "MPM_OK";
        case MPM_ERR_INVALID_ARGUMENT: return "MPM_ERR_INVALID_ARGUMENT";
        case MPM_ERR_BAD_CONFIG: return "MPM_ERR_BAD_CONFIG";
        case MPM_ERR_IO: return "MPM_ERR_IO";
        case MPM_ERR_CUDA: return "MPM_ERR_CUDA";
        case MPM_ERR_OUT_OF_MEMORY: return "MPM_ERR_OUT_OF_MEMORY";
        case MPM_ERR_NOT_INITIALIZED: return "MPM_ERR_NOT_INITIALIZED";
        case MPM_ERR_NONFINITE_STATE: return "MPM_ERR_NONFINITE_STATE";
        case MPM_ERR_OUT_OF_GRID: return "MPM_ERR_OUT_OF_GRID";
        case MPM_ERR_TIMEOUT: return "MPM_ERR_TIMEOUT";
        case MPM_ERR_UNSUPPORTED: return "MPM_ERR_UNSUPPORTED";
        case MPM_ERR_NO_DEVICE: return "MPM_ERR_NO_DEVICE";
    }
    return "MPM_ERR_UNKNOWN";
}

extern "C" mpm_status mpm_create(const mpm_config* cfg, int32_t device, mpm_engine** out) {
    return create_engine(cfg, 1, device, out);
}

extern "C" mpm_status mpm_create_batch(const mpm_config* cfgs, int32_t nscenes, int32_t device, mpm_engine** out) {
    return create_engine(cfgs, nscenes, device, out);
}

extern "C" int32_t mpm_num_scenes(const mpm_engine* e) { return e ? e->scenes : 0; }

extern "C" void mpm_destroy(mpm_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    free_particles(e);
    free_timing(e);
    if (e->l2_window) {
        cudaCtxResetPersistingL2Cache();
        cudaGetLastError();
    }
    free_dev(e->accum);
    free_dev(e->vgrid);
    free_dev(e->sdf);
    free_dev(e->bins_mem);
    free_dev(e->tiles_mem);
    free_dev(e->bstart);
    free_dev(e->ccur);
    free_dev(e->bpart);
    free_dev(e->corder);
    free_dev(e->cstart);
    free_dev(e->ctl);
    free_dev(e->d_prm);
    free_dev(e->d_poff);
    free_dev(e->d_goff);
    free_dev(e->d_itemoff);
    free_dev(e->d_clroff);
    free_dev(e->d_flags);
    free_dev(e->staging);
    free_dev(e->d_prm_large);
    free_dev(e->mlp);
    free_dev(e->mlp_tc);
    free_dev(e->d_params);
    free_dev(e->d_stat);
    free_dev(e->d_lcount);
    free_dev(e->d_llast);
    if (e->copy_stream) cudaStreamSynchronize(e->copy_stream);
    for (int k = 0; k < 2; ++k) {
        if (e->pos_ready[k]) cudaEventDestroy(e->pos_ready[k]);
        if (e->copy_done[k]) cudaEventDestroy(e->copy_done[k]);
    }
    if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

extern "C" mpm_status mpm_init_particles(mpm_engine* e, int64_t n, const float* soa26_host) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (e->scenes != 1) return record(e, MPM_ERR_UNSUPPORTED, "engine holds several scenes: use mpm_init_particles_batch");
    return init_all(e, &n, &soa26_host);
}

extern "C" mpm_status mpm_init_particles_batch(mpm_engine* e, const int64_t* counts, const float* const* soa26_host) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!counts || !soa26_host) return record(e, MPM_ERR_INVALID_ARGUMENT, "counts and soa26_host must be non-NULL");
    return init_all(e, counts, soa26_host);
}

extern "C" mpm_status mpm_set_state(mpm_engine* e, int64_t n, const float* soa26_host) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    if (e->scenes != 1) return record(e, MPM_ERR_UNSUPPORTED, "mpm_set_state serves engines of one scene");
    if (n != e->n) return record(e, MPM_ERR_INVALID_ARGUMENT, "n differs from the engine's particle count");
    if (n > 0 && !soa26_host) return record(e, MPM_ERR_INVALID_ARGUMENT, "soa26_host is NULL");
    if (n > 0) {
        const float* vol = soa26_host + (size_t)MPM_VOL * n;
        const float* mass = soa26_host + (size_t)MPM_MASS * n;
        for (int64_t i = 1; i < n; ++i) {
            if (std::memcmp(&vol[i], &vol[0], sizeof(float)) != 0 || std::memcmp(&mass[i], &mass[0], sizeof(float)) != 0)
                return record(e, MPM_ERR_UNSUPPORTED, "VOL and MASS must each be uniform over the particles");
        }
        e->prm[0].pvol = vol[0];
        e->prm[0].pmass = mass[0];
        if ((s = upload_table(e)) != MPM_OK) return s;
    }
    return load_states(e, &soa26_host, false);
}

extern "C" mpm_status mpm_scene_init_sdf(mpm_engine* e, int32_t scene, const float* tris, int64_t t) {
    mpm_status s = enter_scene(e, scene);
    if (s != MPM_OK) return s;
    if (t < 0 || t > 0x7fffffffLL / 9) return record(e, MPM_ERR_INVALID_ARGUMENT, "triangle count out of range");
    if (t > 0 && !tris) return record(e, MPM_ERR_INVALID_ARGUMENT, "triangles_host is NULL");
    const SimParams& p = e->prm[scene];
    float* sdf = e->sdf + p.goff;
    if (t == 0) {
        e->kernel_launches += mpm::launch_fill(sdf, p.g, sqrtf(1e30f), e->stream);
        CK(e, cudaGetLastError());
        CK(e, cudaStreamSynchronize(e->stream));
        return MPM_OK;
    }
    // One allocation: the triangles as given, then the sorted copy with its
    // tile boxes (sdf.cu).  cudaMalloc: 256-byte aligned, as the kernel's
    // 16-byte bulk copies need; each part starts on a 16-byte boundary and 16
    // spare bytes cover the last tile's copy rounded up to 16 bytes.
    const size_t bytes = (size_t)t * 9 * sizeof(float);
    const size_t off = align_up(bytes, 16) + 16;
    const size_t aux_floats = mpm::sdf_aux_floats((int)t);
    std::vector<float> aux(aux_floats, 0.0f);
    mpm::sdf_prepare_host(tris, (int)t, aux.data());
    float* d_tris = nullptr;
    CK(e, cudaMalloc(&d_tris, off + aux_floats * sizeof(float) + 16));
    float* d_aux = reinterpret_cast<float*>(reinterpret_cast<char*>(d_tris) + off);
    cudaError_t err = cudaMemsetAsync(d_tris, 0, off + aux_floats * sizeof(float) + 16, e->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(d_tris, tris, bytes, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(d_aux, aux.data(), aux_floats * sizeof(float), cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess) {
        e->kernel_launches += mpm::launch_sdf_build(p, d_tris, d_aux, (int)t, sdf, e->d_flags + 1, e->stream,
                                                    e->wait_test & (MPM_WAIT_TEST_SDF_GIVE_UP | MPM_WAIT_TEST_SDF_EXPIRE));
        err = cudaGetLastError();
    }
    // aux is pageable host memory: the synchronisation below ends its copy.
    const mpm_status s2 = err != cudaSuccess ? cuda_fail(e, err, "sdf build") : sync_and_collect(e);
    if (err != cudaSuccess) cudaStreamSynchronize(e->stream);
    cudaFree(d_tris);
    return s2;
}

extern "C" mpm_status mpm_set_wait_test(mpm_engine* e, uint32_t flags) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (flags & ~(uint32_t)(MPM_WAIT_TEST_SDF_GIVE_UP | MPM_WAIT_TEST_SDF_EXPIRE | MPM_WAIT_TEST_MMA_GIVE_UP |
                            MPM_WAIT_TEST_MMA_EXPIRE))
        return record(e, MPM_ERR_INVALID_ARGUMENT, "unknown wait-test flag");
    e->wait_test = flags;
    destroy_learned_graphs(e);
    return MPM_OK;
}

extern "C" mpm_status mpm_init_sdf(mpm_engine* e, const float* tris, int64_t t) {
    return mpm_scene_init_sdf(e, 0, tris, t);
}

extern "C" mpm_status mpm_step_async(mpm_engine* e, int32_t nsub) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    return run_steps(e, nsub);
}

extern "C" mpm_status mpm_synchronize(mpm_engine* e) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if ((s = sync_and_collect(e)) != MPM_OK) return s;
    return check_health(e);
}

extern "C" mpm_status mpm_step(mpm_engine* e, int32_t nsub) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if ((s = run_steps(e, nsub)) != MPM_OK) return s;
    if ((s = sync_and_collect(e)) != MPM_OK) return s;
    return check_health(e);
}

extern "C" mpm_status mpm_substep_partial(mpm_engine* e, int32_t upto) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    if (upto < MPM_STAGE_SORT || upto > MPM_STAGE_G2P) return record(e, MPM_ERR_INVALID_ARGUMENT, "bad stage");
    // Continue the substep in progress, or start a new one.
    int from = e->partial_stage + 1;
    if (upto <= e->partial_stage) from = MPM_STAGE_SORT;
    if (from == MPM_STAGE_SORT && e->accum_dirty) {
        CK(e, cudaMemsetAsync(e->accum, 0, (size_t)e->g_total * sizeof(float4), e->stream));
        e->accum_dirty = false;
    }
    e->kernel_launches += enqueue_substep(e, e->parity, from, upto);
    CK(e, cudaGetLastError());
    if (from == MPM_STAGE_SORT) e->sort_src = e->parity;
    e->partial_stage = upto;
    if (upto == MPM_STAGE_P2G) {
        e->accum_dirty = true;
        e->grid_view = GridView::kAccum;
    } else if (upto >= MPM_STAGE_GRID && from <= MPM_STAGE_GRID) {
        e->accum_dirty = false;
        e->grid_view = GridView::kVelocity;
    }
    if (upto == MPM_STAGE_G2P) {
        e->partial_stage = 0;
        e->parity ^= 1;
        ++e->substeps;
        if ((s = export_positions(e)) != MPM_OK) return s;
    }
    if ((s = sync_and_collect(e)) != MPM_OK) return s;
    return upto == MPM_STAGE_G2P ? check_health(e) : MPM_OK;
}

extern "C" mpm_status mpm_set_checks(mpm_engine* e, uint32_t flags) {
    if (!e) return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "engine is NULL");
    e->checks = flags & (MPM_HEALTH_NONFINITE | MPM_HEALTH_OUT_OF_GRID);
    return MPM_OK;
}

extern "C" int64_t mpm_scene_num_particles(const mpm_engine* e, int32_t scene) {
    if (!e || !e->initialized || scene < 0 || scene >= e->scenes) return 0;
    return e->prm[scene].n;
}

extern "C" int64_t mpm_num_particles(const mpm_engine* e) { return mpm_scene_num_particles(e, 0); }

extern "C" mpm_status mpm_scene_get_state(mpm_engine* e, int32_t scene, float* out) {
    mpm_status s = enter_scene(e, scene);
    if (s != MPM_OK) return s;
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    const SimParams& p = e->prm[scene];
    if (p.n == 0) return MPM_OK;
    if (!out) return record(e, MPM_ERR_INVALID_ARGUMENT, "soa26_host is NULL");
    const size_t bytes = (size_t)MPM_PARTICLE_PLANES * p.n * sizeof(float);
    if ((s = ensure_staging(e, bytes)) != MPM_OK) return s;
    e->kernel_launches += mpm::launch_state_export(p, e->P[e->parity] + p.poff * mpm::kAFloats,
                                                   e->sigma[e->parity] + p.poff, e->staging, e->stream);
    CK(e, cudaGetLastError());
    CK(e, cudaMemcpyAsync(out, e->staging, bytes, cudaMemcpyDeviceToHost, e->stream));
    CK(e, cudaStreamSynchronize(e->stream));
    return MPM_OK;
}

extern "C" mpm_status mpm_get_state(mpm_engine* e, float* out) { return mpm_scene_get_state(e, 0, out); }

extern "C" const float* mpm_scene_positions_device(mpm_engine* e, int32_t scene) {
    if (!e || !e->initialized || scene < 0 || scene >= e->scenes) return nullptr;
    return e->pos_buf[e->pos_cur] + e->prm[scene].poff * 3;
}

namespace {
// Enqueues the read-back of the current positions of `scene` (-1: all
// scenes) on the copy stream, after the export that wrote them.
mpm_status enqueue_positions_copy(mpm_engine* e, int32_t scene, float* xyz) {
    const int b = e->pos_cur;
    const long long first = scene < 0 ? 0 : e->prm[scene].poff;
    const long long count = scene < 0 ? e->n : e->prm[scene].n;
    CK(e, cudaStreamWaitEvent(e->copy_stream, e->pos_ready[b], 0));
    if (count > 0)
        CK(e, cudaMemcpyAsync(xyz, e->pos_buf[b] + first * 3, (size_t)count * 3 * sizeof(float),
                              cudaMemcpyDeviceToHost, e->copy_stream));
    CK(e, cudaEventRecord(e->copy_done[b], e->copy_stream));
    return MPM_OK;
}
}  // namespace

extern "C" mpm_status mpm_get_positions_async(mpm_engine* e, float* xyz) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    if (e->n > 0 && !xyz) return record(e, MPM_ERR_INVALID_ARGUMENT, "xyz_host is NULL");
    return enqueue_positions_copy(e, -1, xyz);
}

extern "C" mpm_status mpm_positions_wait(mpm_engine* e) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    CK(e, cudaStreamSynchronize(e->copy_stream));
    return MPM_OK;
}

extern "C" const float* mpm_positions_device(mpm_engine* e) { return mpm_scene_positions_device(e, 0); }

extern "C" mpm_status mpm_scene_get_positions(mpm_engine* e, int32_t scene, float* xyz) {
    mpm_status s = enter_scene(e, scene);
    if (s != MPM_OK) return s;
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    const SimParams& p = e->prm[scene];
    if (p.n == 0) return MPM_OK;
    if (!xyz) return record(e, MPM_ERR_INVALID_ARGUMENT, "xyz_host is NULL");
    if ((s = enqueue_positions_copy(e, scene, xyz)) != MPM_OK) return s;
    CK(e, cudaStreamSynchronize(e->copy_stream));
    return MPM_OK;
}

extern "C" mpm_status mpm_get_positions(mpm_engine* e, float* xyz) { return mpm_scene_get_positions(e, 0, xyz); }

extern "C" mpm_status mpm_scene_get_grid(mpm_engine* e, int32_t scene, float* out) {
    mpm_status s = enter_scene(e, scene);
    if (s != MPM_OK) return s;
    if (!out) return record(e, MPM_ERR_INVALID_ARGUMENT, "grid4_host is NULL");
    const SimParams& p = e->prm[scene];
    const size_t bytes = (size_t)MPM_GRID_PLANES * p.g * sizeof(float);
    if ((s = ensure_staging(e, bytes)) != MPM_OK) return s;
    const float4* src = (e->grid_view == GridView::kAccum ? e->accum : e->vgrid) + p.goff;
    e->kernel_launches += mpm::launch_grid_export(p, src, e->staging, e->stream);
    CK(e, cudaGetLastError());
    CK(e, cudaMemcpyAsync(out, e->staging, bytes, cudaMemcpyDeviceToHost, e->stream));
    CK(e, cudaStreamSynchronize(e->stream));
    return MPM_OK;
}

extern "C" mpm_status mpm_get_grid(mpm_engine* e, float* out) { return mpm_scene_get_grid(e, 0, out); }

extern "C" mpm_status mpm_scene_get_sdf(mpm_engine* e, int32_t scene, float* out) {
    mpm_status s = enter_scene(e, scene);
    if (s != MPM_OK) return s;
    if (!out) return record(e, MPM_ERR_INVALID_ARGUMENT, "sdf_host is NULL");
    const SimParams& p = e->prm[scene];
    CK(e, cudaMemcpyAsync(out, e->sdf + p.goff, (size_t)p.g * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    CK(e, cudaStreamSynchronize(e->stream));
    return MPM_OK;
}

extern "C" mpm_status mpm_get_sdf(mpm_engine* e, float* out) { return mpm_scene_get_sdf(e, 0, out); }

extern "C" mpm_status mpm_scene_get_sort(mpm_engine* e, int32_t scene, int32_t* keys_host, int32_t* perm_host) {
    mpm_status s = enter_scene(e, scene);
    if (s != MPM_OK) return s;
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    const SimParams& p = e->prm[scene];
    if (p.n == 0) return MPM_OK;
    const size_t bytes = (size_t)p.n * sizeof(int32_t);
    // The state the most recent substep started from (intact until the next
    // substep), or the current state before any substep.
    const int src = e->sort_src == kNoSort ? e->parity : e->sort_src;
    e->kernel_launches += mpm::launch_reference_keys(p, e->P[src] + p.poff * mpm::kAFloats, e->sigma[src] + p.poff,
                                                     e->ref_keys, e->stream);
    if (e->sort_src == kNoSort) {
        e->kernel_launches += mpm::launch_identity(e->ref_perm, p.n, e->stream);
    } else {
        mpm::SortScratch sort;
        mpm::sort_scratch_carve(e->sort_mem, p.n, &sort);
        e->kernel_launches +=
            mpm::launch_radix_sort(e->ref_keys, p.n, sort, e->ref_perm, nullptr, nullptr, nullptr, e->stream);
        e->sort_passes += 4;
    }
    CK(e, cudaGetLastError());
    if (keys_host) CK(e, cudaMemcpyAsync(keys_host, e->ref_keys, bytes, cudaMemcpyDeviceToHost, e->stream));
    if (perm_host) CK(e, cudaMemcpyAsync(perm_host, e->ref_perm, bytes, cudaMemcpyDeviceToHost, e->stream));
    CK(e, cudaStreamSynchronize(e->stream));
    return MPM_OK;
}

extern "C" mpm_status mpm_get_sort(mpm_engine* e, int32_t* keys_host, int32_t* perm_host) {
    return mpm_scene_get_sort(e, 0, keys_host, perm_host);
}

extern "C" mpm_status mpm_get_stats(mpm_engine* e, mpm_stats* st, int32_t reset_health) {
    if (!e || !st) return record(e, MPM_ERR_INVALID_ARGUMENT, "engine and stats must be non-NULL");
    st->substeps = e->substeps;
    st->kernel_launches = e->kernel_launches;
    st->sort_passes = e->sort_passes;
    st->health = e->health;
    st->reserved = 0;
    if (reset_health) e->health = 0;
    return MPM_OK;
}

extern "C" void* mpm_stream(mpm_engine* e) { return e ? (void*)e->stream : nullptr; }

extern "C" const char* mpm_last_error(const mpm_engine* e) { return e ? e->last_error.c_str() : ""; }

extern "C" const char* mpm_global_last_error(void) { return g_global_error.c_str(); }

// Lets the free operators of other translation units report through
// mpm_global_last_error.
void mpm::set_global_error(const std::string& msg) { g_global_error = msg; }

extern "C" mpm_status mpm_sort_particles_device(const float* px, const float* py, const float* pz, int64_t n,
                                                int32_t* d_keys, int32_t* d_perm, void* stream) {
    g_global_error.clear();
    if (n < 0 || n > 0x7fffffffLL - 64) return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "n out of range");
    if (n == 0) return MPM_OK;
    if (!px || !py || !pz || !d_keys || !d_perm)
        return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "device pointers must be non-NULL");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int ni = (int)n;
    void* scratch = nullptr;
    CK(nullptr, cudaMallocAsync(&scratch, mpm::sort_scratch_bytes(ni), st));
    mpm::SortScratch s;
    mpm::sort_scratch_carve(scratch, ni, &s);
    mpm::launch_morton_keys(px, py, pz, ni, d_keys, st);
    mpm::launch_radix_sort(d_keys, ni, s, d_perm, nullptr, nullptr, nullptr, st);
    const cudaError_t launch_err = cudaGetLastError();
    const cudaError_t free_err = cudaFreeAsync(scratch, st);
    if (launch_err != cudaSuccess) return cuda_fail(nullptr, launch_err, "sort launch");
    CK(nullptr, free_err);
    return MPM_OK;
}

extern "C" mpm_status mpm_set_stage_timing(mpm_engine* e, int32_t max_substeps) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (max_substeps < 0 || max_substeps > (1 << 20))
        return record(e, MPM_ERR_INVALID_ARGUMENT, "max_substeps out of range");
    CK(e, cudaStreamSynchronize(e->stream));
    free_timing(e);
    if (max_substeps > 0) {
        for (int k = 0; k < mpm_engine::kTimingMarks; ++k) CK(e, cudaEventCreate(&e->tscratch[k]));
        const int total = max_substeps * mpm_engine::kTimingMarks;
        e->tev = new cudaEvent_t[total]();
        e->timing_cap = max_substeps;
        for (int i = 0; i < total; ++i) CK(e, cudaEventCreate(&e->tev[i]));
    }
    if (e->initialized) return capture_graphs(e);
    return MPM_OK;
}

extern "C" mpm_status mpm_get_stage_times(mpm_engine* e, double* ms, int32_t* count) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!ms || !count) return record(e, MPM_ERR_INVALID_ARGUMENT, "ms and count must be non-NULL");
    CK(e, cudaStreamSynchronize(e->stream));
    for (int k = 0; k < 4; ++k) ms[k] = 0.0;
    for (int sidx = 0; sidx < e->timing_used; ++sidx) {
        const cudaEvent_t* ev = e->tev + (size_t)sidx * mpm_engine::kTimingMarks;
        for (int k = 0; k < 4; ++k) {
            float t = 0.0f;
            CK(e, cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
            ms[k] += t;
        }
    }
    *count = e->timing_used;
    e->timing_used = 0;
    return MPM_OK;
}

// ------------------------------------------------------- learned step ----
namespace mpm {
mpm_status corrector_append(mpm_corrector* c, const float* feat_all, const float* vplain, const float* vlarge,
                            long long n, long long samples, unsigned long long seed, cudaStream_t st);
int launch_mlp_pack(const float* params, MlpPacked* out, cudaStream_t st);
int launch_mlp_pack_tc(const float* params, MlpTc* out, cudaStream_t st);
int launch_velocity_export(const float* P, const int32_t* sigma, long long n, float* out, cudaStream_t st);
}  // namespace mpm

extern "C" mpm_status mpm_set_corrector(mpm_engine* e, const float* params_host, int32_t ratio,
                                        float max_density_change) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (ratio < 1 || ratio > 64) return record(e, MPM_ERR_INVALID_ARGUMENT, "ratio must be in [1, 64]");
    if (std::isnan(max_density_change)) return record(e, MPM_ERR_INVALID_ARGUMENT, "max_density_change is NaN");
    if (params_host) {
        for (int i = 0; i < MPM_CORRECTOR_PARAMS; ++i)
            if (!std::isfinite(params_host[i])) return record(e, MPM_ERR_INVALID_ARGUMENT, "a parameter is not finite");
        if (!e->mlp) {
            CK(e, cudaMalloc(&e->mlp, sizeof(mpm::MlpPacked)));
            CK(e, cudaMalloc(&e->mlp_tc, sizeof(mpm::MlpTc)));
            CK(e, cudaMalloc(&e->d_params, MPM_CORRECTOR_PARAMS * sizeof(float)));
        }
        CK(e, cudaMemcpyAsync(e->d_params, params_host, MPM_CORRECTOR_PARAMS * sizeof(float), cudaMemcpyHostToDevice,
                              e->stream));
        e->kernel_launches += mpm::launch_mlp_pack(e->d_params, e->mlp, e->stream);
        e->kernel_launches += mpm::launch_mlp_pack_tc(e->d_params, e->mlp_tc, e->stream);
        CK(e, cudaGetLastError());
        CK(e, cudaStreamSynchronize(e->stream));
    }
    e->mlp_set = params_host != nullptr;
    e->ratio = ratio;
    e->max_density_change = max_density_change;
    destroy_learned_graphs(e);
    return MPM_OK;
}

extern "C" mpm_status mpm_step_learned(mpm_engine* e, int32_t nlarge, mpm_learned_stats* stats) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (nlarge < 0) return record(e, MPM_ERR_INVALID_ARGUMENT, "nlarge < 0");
    if ((s = learned_ready(e)) != MPM_OK) return s;
    const int32_t requested = nlarge;
    const bool checked_on_device = e->mlp_set && e->max_density_change >= 0.f && e->fallback_on_device;
    if (checked_on_device && nlarge > 0) {
        if (!e->lgraph[0] && (s = capture_learned_graphs(e)) != MPM_OK) return s;
        for (int k = 0; k < nlarge; ++k) {
            CK(e, cudaGraphLaunch(e->lgraph[e->parity], e->stream));
            e->kernel_launches += e->lgraph_kernels[e->parity];
            e->parity ^= 1;
        }
        // One read-back per call: the decisions' counters and the last means.
        long long cnt[2] = {0, 0};
        float last[4] = {0.f, 0.f, 0.f, 0.f};
        CK(e, cudaMemcpyAsync(cnt, e->d_lcount, sizeof(cnt), cudaMemcpyDeviceToHost, e->stream));
        CK(e, cudaMemcpyAsync(last, e->d_llast, sizeof(last), cudaMemcpyDeviceToHost, e->stream));
        CK(e, cudaStreamSynchronize(e->stream));
        const long long acc = cnt[0] - e->lcount_host[0], rej = cnt[1] - e->lcount_host[1];
        e->lcount_host[0] = cnt[0];
        e->lcount_host[1] = cnt[1];
        e->large_steps += acc;
        e->fallbacks += rej;
        e->substeps += rej * e->ratio;
        e->kernel_launches += rej * e->lbody_kernels;
        for (int q = 0; q < 3; ++q) e->last_stats[q] = last[q];
        e->last_density_change = last[3];
        // The state a fallback's last substep started from is overwritten by
        // the move to parity 1 - par: mpm_get_sort reports the current state.
        e->sort_src = kNoSort;
        nlarge = 0;  // done; the host-decided loop below runs no step
    }
    for (int k = 0; k < nlarge; ++k) {
        const int par = e->parity;
        const bool tc = e->mlp_set && e->corrector_kernel == MPM_CORRECTOR_TCGEN05;
        mpm::LearnArgs la{e->mlp_set ? e->mlp : nullptr, nullptr, nullptr, e->d_stat, large_blend(e),
                          tc ? e->mlp_tc : nullptr, e->d_flags + 1,
                          (e->wait_test & (MPM_WAIT_TEST_MMA_GIVE_UP | MPM_WAIT_TEST_MMA_EXPIRE)) >> 2};
        // The statistic is read back (a host sync per large step) only when
        // it can trigger the fallback.
        const bool checked = e->mlp_set && e->max_density_change >= 0.f;
        if (e->mlp_set) CK(e, cudaMemsetAsync(e->d_stat, 0, 3 * sizeof(float), e->stream));
        e->kernel_launches += enqueue_large(e, par, &la);
        CK(e, cudaGetLastError());
        e->sort_src = par;
        bool accept = true;
        if (checked) {
            float sum[3] = {0.f, 0.f, 0.f};
            CK(e, cudaMemcpyAsync(sum, e->d_stat, sizeof(sum), cudaMemcpyDeviceToHost, e->stream));
            CK(e, cudaStreamSynchronize(e->stream));
            for (int q = 0; q < 3; ++q) e->last_stats[q] = e->n > 0 ? (double)sum[q] / (double)e->n : 0.0;
            // The statistic the rule compares with max_density_change.
            double stat = e->last_stats[0];
            if (e->fallback_rule == MPM_FALLBACK_REST_DENSITY) stat = e->last_stats[1];
            if (e->fallback_rule == MPM_FALLBACK_REST_DENSITY_EXCESS) stat = e->last_stats[1] - e->last_stats[2];
            e->last_density_change = stat;
            accept = stat <= e->max_density_change;
        }
        if (accept) {
            e->parity = 1 - par;
            ++e->large_steps;
        } else {
            if ((s = rebin(e, par)) != MPM_OK) return s;
            if ((s = plain_substeps(e, e->ratio)) != MPM_OK) return s;
            ++e->fallbacks;
        }
    }
    if (requested > 0) e->grid_view = GridView::kVelocity;
    if ((s = export_positions(e)) != MPM_OK) return s;
    if (stats) {
        stats->large_steps = e->large_steps;
        stats->fallbacks = e->fallbacks;
        stats->last_density_change = e->last_density_change;
    }
    if ((s = sync_and_collect(e)) != MPM_OK) return s;
    return check_health(e);
}

extern "C" mpm_status mpm_corrector_collect(mpm_corrector* c, mpm_engine* e, int64_t samples, uint64_t seed) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!c) return record(e, MPM_ERR_INVALID_ARGUMENT, "corrector is NULL");
    if (samples < 0) return record(e, MPM_ERR_INVALID_ARGUMENT, "samples < 0");
    if ((s = learned_ready(e)) != MPM_OK) return s;
    if (e->n <= 0) return MPM_OK;
    if (!e->feat_all) {
        CK(e, cudaMalloc(&e->feat_all, (size_t)e->n * mpm::kMlpIn * sizeof(float)));
        CK(e, cudaMalloc(&e->vlarge, (size_t)e->n * 3 * sizeof(float)));
        CK(e, cudaMalloc(&e->vplain, (size_t)e->n * 3 * sizeof(float)));
    }
    // The uncorrected large step, recording features and final velocities;
    // then back to its start state for RATIO plain substeps.
    const int par = e->parity;
    mpm::LearnArgs la{nullptr, e->feat_all, e->vlarge, nullptr, large_blend(e), nullptr, nullptr, 0u};
    e->kernel_launches += enqueue_large(e, par, &la);
    CK(e, cudaGetLastError());
    if ((s = rebin(e, par)) != MPM_OK) return s;
    if ((s = plain_substeps(e, e->ratio)) != MPM_OK) return s;
    e->kernel_launches += mpm::launch_velocity_export(e->P[e->parity], e->sigma[e->parity], e->n, e->vplain, e->stream);
    CK(e, cudaGetLastError());
    s = mpm::corrector_append(c, e->feat_all, e->vplain, e->vlarge, e->n, samples, seed, e->stream);
    if (s != MPM_OK) {
        cudaStreamSynchronize(e->stream);
        return record(e, s, mpm_corrector_last_error(c));
    }
    ++e->kernel_launches;
    e->grid_view = GridView::kVelocity;
    if ((s = export_positions(e)) != MPM_OK) return s;
    if ((s = sync_and_collect(e)) != MPM_OK) return s;
    return check_health(e);
}

// ---------------------------------------------------------- checkpoint ----
namespace {

constexpr char kCkptMagic[8] = {'M', 'P', 'M', 'C', 'K', 'P', 'T', '1'};
constexpr uint32_t kCkptVersion = 1;
constexpr uint32_t kCkptHeader = 128;

uint32_t crc32_update(uint32_t crc, const void* data, size_t len) {
    static uint32_t table[256];
    static bool ready = false;
    if (!ready) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        ready = true;
    }
    const unsigned char* b = static_cast<const unsigned char*>(data);
    crc = ~crc;
    for (size_t i = 0; i < len; ++i) crc = table[(crc ^ b[i]) & 0xffu] ^ (crc >> 8);
    return ~crc;
}

template <typename T>
void put(std::vector<unsigned char>& h, size_t off, T v) {
    std::memcpy(h.data() + off, &v, sizeof(T));
}
template <typename T>
T get(const std::vector<unsigned char>& h, size_t off) {
    T v;
    std::memcpy(&v, h.data() + off, sizeof(T));
    return v;
}

struct CkptHeader {
    int64_t n = 0, substeps = 0;
    mpm_config cfg{};
    float pvol = 0.f, pmass = 0.f;
    uint64_t note_bytes = 0;
};

bool parse_header(const std::vector<unsigned char>& h, CkptHeader* out, std::string& err) {
    if (h.size() < kCkptHeader || std::memcmp(h.data(), kCkptMagic, 8) != 0) {
        err = "not an MPM checkpoint (bad magic)";
        return false;
    }
    if (get<uint32_t>(h, 8) != kCkptVersion || get<uint32_t>(h, 12) != kCkptHeader) {
        err = "unsupported checkpoint version";
        return false;
    }
    out->n = get<int64_t>(h, 16);
    out->substeps = get<int64_t>(h, 24);
    out->cfg.size_x = get<int32_t>(h, 32);
    out->cfg.size_y = get<int32_t>(h, 36);
    out->cfg.size_z = get<int32_t>(h, 40);
    out->cfg.padding = get<int32_t>(h, 44);
    out->cfg.gravity = get<float>(h, 48);
    out->cfg.dt = get<float>(h, 52);
    out->cfg.gamma = get<float>(h, 56);
    out->cfg.compression = get<float>(h, 60);
    out->cfg.resolution = get<float>(h, 64);
    out->cfg.substeps = get<int32_t>(h, 68);
    out->cfg.sdf_resolution = get<int32_t>(h, 72);
    out->pvol = get<float>(h, 76);
    out->pmass = get<float>(h, 80);
    out->note_bytes = get<uint64_t>(h, 84);
    if (out->n < 0 || out->n > 0x7fffffffLL - 64 || out->cfg.size_x <= 0 || out->cfg.size_y <= 0 ||
        out->cfg.size_z <= 0 || out->note_bytes > (1u << 24)) {
        err = "corrupt checkpoint header";
        return false;
    }
    return true;
}

}  // namespace

extern "C" mpm_status mpm_checkpoint_save(mpm_engine* e, const char* path, const char* note) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!path) return record(e, MPM_ERR_INVALID_ARGUMENT, "path is NULL");
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    if (e->scenes != 1) return record(e, MPM_ERR_UNSUPPORTED, "checkpoints hold engines of one scene");
    const long long n = e->n;
    const long long g = e->g_total;
    std::vector<float> state((size_t)MPM_PARTICLE_PLANES * n), sdf((size_t)g);
    if (n > 0 && (s = mpm_get_state(e, state.data())) != MPM_OK) return s;
    if ((s = mpm_get_sdf(e, sdf.data())) != MPM_OK) return s;
    const std::string txt = note ? note : "";
    std::vector<unsigned char> h(kCkptHeader, 0);
    std::memcpy(h.data(), kCkptMagic, 8);
    const mpm_config& c = e->cfg[0];
    put<uint32_t>(h, 8, kCkptVersion);
    put<uint32_t>(h, 12, kCkptHeader);
    put<int64_t>(h, 16, n);
    put<int64_t>(h, 24, e->substeps);
    put<int32_t>(h, 32, c.size_x);
    put<int32_t>(h, 36, c.size_y);
    put<int32_t>(h, 40, c.size_z);
    put<int32_t>(h, 44, c.padding);
    put<float>(h, 48, c.gravity);
    put<float>(h, 52, c.dt);
    put<float>(h, 56, c.gamma);
    put<float>(h, 60, c.compression);
    put<float>(h, 64, c.resolution);
    put<int32_t>(h, 68, c.substeps);
    put<int32_t>(h, 72, c.sdf_resolution);
    put<float>(h, 76, e->prm[0].pvol);
    put<float>(h, 80, e->prm[0].pmass);
    put<uint64_t>(h, 84, (uint64_t)txt.size());
    const std::string tmp = std::string(path) + ".part";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return record(e, MPM_ERR_IO, std::string("cannot write ") + tmp);
    uint32_t crc = 0;
    auto write = [&](const void* d, size_t len) {
        crc = crc32_update(crc, d, len);
        return std::fwrite(d, 1, len, f) == len;
    };
    bool ok = write(h.data(), h.size()) && write(txt.data(), txt.size()) &&
              write(state.data(), state.size() * sizeof(float)) && write(sdf.data(), sdf.size() * sizeof(float));
    ok = ok && std::fwrite(&crc, 1, sizeof(crc), f) == sizeof(crc);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return record(e, MPM_ERR_IO, std::string("cannot write checkpoint ") + path);
    }
    return MPM_OK;
}

namespace {
mpm_status read_checkpoint(const char* path, CkptHeader* hd, std::string* note, std::vector<float>* state,
                           std::vector<float>* sdf) {
    if (!path) return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "path is NULL");
    FILE* f = std::fopen(path, "rb");
    if (!f) return record(nullptr, MPM_ERR_IO, std::string("cannot open checkpoint ") + path);
    std::vector<unsigned char> data;
    unsigned char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) data.insert(data.end(), buf, buf + got);
    std::fclose(f);
    std::string err;
    if (!parse_header(data, hd, err)) return record(nullptr, MPM_ERR_IO, err);
    const size_t g = (size_t)hd->cfg.size_x * hd->cfg.size_y * hd->cfg.size_z;
    const size_t sbytes = (size_t)MPM_PARTICLE_PLANES * hd->n * sizeof(float);
    const size_t want = kCkptHeader + hd->note_bytes + sbytes + g * sizeof(float) + 4;
    if (data.size() != want) return record(nullptr, MPM_ERR_IO, "checkpoint size does not match its header");
    uint32_t crc;
    std::memcpy(&crc, data.data() + want - 4, 4);
    if (crc32_update(0, data.data(), want - 4) != crc) return record(nullptr, MPM_ERR_IO, "checkpoint CRC mismatch");
    size_t off = kCkptHeader;
    if (note) note->assign(reinterpret_cast<const char*>(data.data() + off), hd->note_bytes);
    off += hd->note_bytes;
    if (state) {
        state->resize((size_t)MPM_PARTICLE_PLANES * hd->n);
        std::memcpy(state->data(), data.data() + off, sbytes);
    }
    off += sbytes;
    if (sdf) {
        sdf->resize(g);
        std::memcpy(sdf->data(), data.data() + off, g * sizeof(float));
    }
    return MPM_OK;
}
}  // namespace

extern "C" mpm_status mpm_checkpoint_info(const char* path, mpm_config* cfg, int64_t* n, int64_t* substeps,
                                          char* note, int32_t note_len) {
    g_global_error.clear();
    CkptHeader hd;
    std::string txt;
    mpm_status s = read_checkpoint(path, &hd, &txt, nullptr, nullptr);
    if (s != MPM_OK) return s;
    if (cfg) *cfg = hd.cfg;
    if (n) *n = hd.n;
    if (substeps) *substeps = hd.substeps;
    if (note && note_len > 0) {
        const size_t k = std::min((size_t)note_len - 1, txt.size());
        std::memcpy(note, txt.data(), k);
        note[k] = '\0';
    }
    return MPM_OK;
}

extern "C" mpm_status mpm_checkpoint_load(const char* path, int32_t device, mpm_engine** out) {
    g_global_error.clear();
    if (!out) return record(nullptr, MPM_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    CkptHeader hd;
    std::vector<float> state, sdf;
    mpm_status s = read_checkpoint(path, &hd, nullptr, &state, &sdf);
    if (s != MPM_OK) return s;
    mpm_engine* e = nullptr;
    if ((s = create_engine(&hd.cfg, 1, device, &e)) != MPM_OK) return s;
    const int64_t n = hd.n;
    const float* planes = state.data();
    s = init_all(e, &n, &planes, false, &hd.pvol, &hd.pmass);
    if (s == MPM_OK) {
        cudaError_t err = cudaMemcpyAsync(e->sdf, sdf.data(), sdf.size() * sizeof(float), cudaMemcpyHostToDevice,
                                          e->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
        if (err != cudaSuccess) s = cuda_fail(e, err, "checkpoint sdf upload");
    }
    if (s != MPM_OK) {
        g_global_error = e->last_error;
        mpm_destroy(e);
        return s;
    }
    e->substeps = hd.substeps;
    *out = e;
    return MPM_OK;
}

// ------------------------------------------------------------ autotune ----
namespace {
bool valid_tuning(const mpm_tuning& t) {
    return t.p2g_ctas_per_sm >= 1 && t.p2g_ctas_per_sm <= mpm::p2g_max_ctas_per_sm() &&
           (t.g2p_block == 128 || t.g2p_block == 256 || t.g2p_block == 512) &&
           (t.grid_block == 0 || t.grid_block == 128 || t.grid_block == 256) &&
           (t.p2g_cell_cap == 0 || (t.p2g_cell_cap >= 4 && t.p2g_cell_cap <= 64));
}

// Times stage `stage` of one substep from the current state and undoes the
// substep (the state of the current parity is untouched by it; the counter
// sets are rebuilt from it).
mpm_status time_stage(mpm_engine* e, int stage, cudaEvent_t a, cudaEvent_t b, float* ms) {
    const int par = e->parity;
    e->kernel_launches += enqueue_substep(e, par, MPM_STAGE_SORT, stage - 1);
    CK(e, cudaEventRecord(a, e->stream));
    e->kernel_launches += enqueue_substep(e, par, stage, stage);
    CK(e, cudaEventRecord(b, e->stream));
    e->kernel_launches += enqueue_substep(e, par, stage + 1, MPM_STAGE_G2P);
    CK(e, cudaGetLastError());
    CK(e, cudaEventSynchronize(b));
    CK(e, cudaEventElapsedTime(ms, a, b));
    mpm_status s = rebin(e, par);
    if (s != MPM_OK) return s;
    return sync_and_collect(e);
}
}  // namespace

extern "C" mpm_status mpm_set_tuning(mpm_engine* e, const mpm_tuning* t) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!t || !valid_tuning(*t)) return record(e, MPM_ERR_INVALID_ARGUMENT, "tuning out of range");
    e->tune.p2g_ctas_per_sm = t->p2g_ctas_per_sm;
    e->tune.g2p_block = t->g2p_block;
    e->tune.grid_block = t->grid_block;
    e->tune.p2g_cell_cap = t->p2g_cell_cap;
    return e->initialized ? capture_graphs(e) : MPM_OK;
}

extern "C" mpm_status mpm_get_tuning(mpm_engine* e, mpm_tuning* t) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!t) return record(e, MPM_ERR_INVALID_ARGUMENT, "out is NULL");
    *t = e->tune;
    return MPM_OK;
}

extern "C" mpm_status mpm_autotune(mpm_engine* e, int32_t repeats, mpm_tuning* out) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!e->initialized) return record(e, MPM_ERR_NOT_INITIALIZED, "mpm_init_particles has not been called");
    if (repeats < 1 || repeats > 100) return record(e, MPM_ERR_INVALID_ARGUMENT, "repeats must be in [1, 100]");
    if (e->accum_dirty) {
        CK(e, cudaMemsetAsync(e->accum, 0, (size_t)e->g_total * sizeof(float4), e->stream));
        e->accum_dirty = false;
    }
    e->partial_stage = 0;
    cudaEvent_t a = nullptr, b = nullptr;
    CK(e, cudaEventCreate(&a));
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return cuda_fail(e, cudaGetLastError(), "cudaEventCreate");
    }
    mpm_tuning best = e->tune;
    best.p2g_cell_cap = e->tune.p2g_cell_cap = 0;
    auto median_time = [&](int stage, float* ms) -> mpm_status {
        std::vector<float> t(repeats);
        for (int r = 0; r < repeats; ++r) {
            mpm_status st = time_stage(e, stage, a, b, &t[r]);
            if (st != MPM_OK) return st;
        }
        std::sort(t.begin(), t.end());
        *ms = t[repeats / 2];
        return MPM_OK;
    };
    // Each stage is its own kernel: tune them one at a time.
    const int max_p2g = mpm::p2g_max_ctas_per_sm();
    float tbest = 1e30f, ms = 0.f;
    for (int k : {4, 6, 8, 10, 12, 14, 16, 20, 24}) {
        if (k > max_p2g) break;
        e->tune.p2g_ctas_per_sm = k;
        if ((s = median_time(MPM_STAGE_P2G, &ms)) != MPM_OK) break;
        if (ms < tbest) tbest = ms, best.p2g_ctas_per_sm = k, best.p2g_ms = ms;
    }
    e->tune.p2g_ctas_per_sm = best.p2g_ctas_per_sm;
    // The crowded-cell threshold is not tuned here: P2G chooses it per work
    // item from the counts it sees, which follows the state as it evolves,
    // while a fixed value timed on one state can cost far more later.
    tbest = 1e30f;
    for (int k : {128, 256, 0}) {
        if (s != MPM_OK) break;
        e->tune.grid_block = k;
        if ((s = median_time(MPM_STAGE_GRID, &ms)) != MPM_OK) break;
        if (ms < tbest) tbest = ms, best.grid_block = k, best.grid_ms = ms;
    }
    e->tune.grid_block = best.grid_block;
    tbest = 1e30f;
    for (int k : {128, 256, 512}) {
        if (s != MPM_OK) break;
        e->tune.g2p_block = k;
        if ((s = median_time(MPM_STAGE_G2P, &ms)) != MPM_OK) break;
        if (ms < tbest) tbest = ms, best.g2p_block = k, best.g2p_ms = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    e->tune = best;
    if (s != MPM_OK) return s;
    if ((s = capture_graphs(e)) != MPM_OK) return s;
    if (out) *out = best;
    return MPM_OK;
}

extern "C" mpm_status mpm_set_fallback_rule(mpm_engine* e, int32_t rule) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (rule != MPM_FALLBACK_DENSITY_CHANGE && rule != MPM_FALLBACK_REST_DENSITY &&
        rule != MPM_FALLBACK_REST_DENSITY_EXCESS)
        return record(e, MPM_ERR_INVALID_ARGUMENT, "unknown fallback rule");
    e->fallback_rule = rule;
    destroy_learned_graphs(e);
    return MPM_OK;
}

extern "C" mpm_status mpm_set_fallback_on_device(mpm_engine* e, int32_t on_device) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    e->fallback_on_device = on_device != 0;
    return MPM_OK;
}

extern "C" mpm_status mpm_learned_statistics(mpm_engine* e, double* out3) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (!out3) return record(e, MPM_ERR_INVALID_ARGUMENT, "out is NULL");
    for (int q = 0; q < 3; ++q) out3[q] = e->last_stats[q];
    return MPM_OK;
}

extern "C" mpm_status mpm_set_corrector_kernel(mpm_engine* e, int32_t kind) {
    mpm_status s = enter(e);
    if (s != MPM_OK) return s;
    if (kind != MPM_CORRECTOR_TCGEN05 && kind != MPM_CORRECTOR_MMA_SYNC)
        return record(e, MPM_ERR_INVALID_ARGUMENT, "unknown corrector kernel");
    e->corrector_kernel = kind;
    destroy_learned_graphs(e);
    return MPM_OK;
}

// Host-side launchers of the engine's CUDA kernels.  Each launcher enqueues
// its kernels on `st` and returns how many kernel launches it issued, so the
// engine can count the launches of a step.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "corrector.cuh"
#include "corrector_tc.cuh"
#include "device_math.cuh"

namespace mpm {

// ---------------------------------------------------------------- sort ----
// Stable LSD radix sort of 32-bit signed keys, 8-bit digits, 4 passes.
// Each pass is histogram -> per-digit spine scan -> scatter; no kernel waits
// on another CTA, so nothing can spin on the GPU.
struct SortScratch {
    int32_t* key_a = nullptr;
    int32_t* val_a = nullptr;
    int32_t* key_b = nullptr;
    int32_t* val_b = nullptr;
    uint32_t* hist = nullptr;    // [256][nb] per-CTA digit counts, scanned in place
    uint32_t* totals = nullptr;  // [256] digit totals of the pass
    int n = 0;
    int nb = 0;       // CTAs per pass
    int per_cta = 0;  // keys per CTA (multiple of the 2048-key tile)
};

// Bytes of scratch for sorting n keys (256-byte aligned sub-buffers).
size_t sort_scratch_bytes(int n);
// Points the scratch sub-buffers into `base` (sort_scratch_bytes(n) bytes).
void sort_scratch_carve(void* base, int n, SortScratch* s);

// keys[i] = Morton key of (px[i], py[i], pz[i]) (setKeys, kernels.cu:361-371).
int launch_morton_keys(const float* px, const float* py, const float* pz, int n, int32_t* keys, cudaStream_t st);

// Sorts `keys` (n signed ints, left unchanged) with values 0..n-1, stable, and
// writes the permutation sigma[j] = index of the j-th smallest key, the
// result of thrust::sequence + thrust::sort_by_key (engine.cu:98-99).
// If rank_out is non-null it also writes rank_out[sigma[j]] = j, and if gidx
// is non-null gidx[j] = rank_in[sigma[j]] (rank_in null: sigma[j]).
int launch_radix_sort(const int32_t* keys, int n, const SortScratch& s, int32_t* sigma, int32_t* rank_out,
                      const int32_t* rank_in, int32_t* gidx, cudaStream_t st);

// ------------------------------------------------------------- substep ----
// The substep kernels work on all scenes of a SceneTable at once; particle
// slots, cells and bins are global (device_math.cuh).  P is the
// particle-major state, ordered by cell of the binning that produced it.
// pcell[j] is the global cell of slot j; ccur holds one slot cursor per
// cell, which the ordering's scatter draws the cell's slots from.  A counter set holds the cell counts (global cells), the
// bin counts and the per-scene lists of bins that hold particles (global bin
// entries: nb + 2 per scene), and the per-scene list lengths nlist[scene].
// Two sets alternate: a substep orders the particles by one and its G2P
// fills the other, which that substep clears first.
struct BinSet {
    uint32_t* ccount;
    uint32_t* bcount;
    int32_t* blist;
    uint32_t* nlist;
};

// Node tiles of the grid update, one per bin: tile (bx, by, bz) of a scene
// holds the nodes x in [8 bx - 2, 8 bx + 6), y in [4 by - 2, 4 by + 2), z in
// [4 bz - 2, 4 bz + 2), so that the 10 x 6 x 6 nodes a bin's particles reach
// lie in tiles bx..bx+1 x by..by+1 x bz..bz+1.  stamp[0] counts orderings;
// mark[global bin] = the stamp of the last ordering whose listed bins reach
// the tile; dirty[global bin] = 1 while the tile's velocity nodes may hold
// values other than zero.
struct TileMarks {
    uint32_t* stamp;
    uint32_t* mark;
    uint8_t* dirty;
    long long count;  // global bin entries (nb + 2 per scene)
};

// Files the n particles of P (all scenes, slot order) into an empty set.
int launch_bin_count(const SceneTable& sc, long long n, const float* P, int32_t* pcell, const BinSet& set,
                     cudaStream_t st);
// Order by cell from set `cur`: bstart (global first slots of every bin), cstart
// (first slot of every cell of a listed bin), corder (P2G's order of each
// listed bin's cells, one byte per cell, indexed like the cells), gidx[new
// slot] = old slot, itemoff (the P2G work items of each scene: kBinZ per
// listed bin, prefix, S + 1 entries) and clroff (the same prefix of `other`'s
// listed bins, one per bin); clears `other` and the work counters work[0..1];
// with tiles.mark set, advances tiles.stamp and marks the tiles the listed
// bins of `cur` reach.
// bins_total: sum over scenes of nb + 1.  bpart: scenes x scan_chunks ints of
// scratch; scan_chunks = bin_scan_chunks(largest nb + 1).
int launch_bin_order(const SceneTable& sc, long long n, long long bins_total, const BinSet& cur, const BinSet& other,
                     int32_t* bstart, int32_t* cstart, const int32_t* pcell, int32_t* ccur, int32_t* gidx,
                     uint8_t* corder, long long* itemoff, long long* clroff, uint32_t* work, int32_t* bpart,
                     int scan_chunks, const TileMarks& tiles, cudaStream_t st);
// Chunks of the bin scan for a scene of `bins` scanned bins.
int bin_scan_chunks(long long bins);
// P2G over the items of `cur`; gidx maps slots of the new order to P.  Two
// launches: the items, then the crowded-cell list they fill (crowd: scratch of
// crowd_cap entries, at least n / 4 + 64; work[2..3] are its counters, reset
// by the bin scan).  ctas_per_sm: persistent single-warp CTAs per SM (0 = the
// default 12); cell_cap: particles of a cell its own lane sums before the rest
// goes to the list (0 = chosen per work item from its cells' counts).
int launch_p2g(const SceneTable& sc, long long n, long long bins_total, const float* P, const int32_t* gidx,
               const int32_t* cstart, const BinSet& cur, const uint8_t* corder, const long long* itemoff,
               uint32_t* work, float4* accum, int4* crowd, int crowd_cap, uint32_t* status, cudaStream_t st,
               int ctas_per_sm = 0, int cell_cap = 0);
// Most P2G CTAs that fit on one SM.
int p2g_max_ctas_per_sm();
// p0: the parameters of scene 0, used directly when the table holds one scene.
// With tiles.mark set: only the tiles marked by this substep's ordering are
// updated, and tiles updated before but not marked now are reset to zero;
// else every node.
int launch_grid_update(const SceneTable& sc, const SimParams& p0, long long g_total, float4* accum, float4* vgrid,
                       const float* sdf, const TileMarks& tiles, cudaStream_t st, int block = 256);
// Large-step G2P (one scene): particles advect with v_old + blend (v_new -
// v_old).  With mlp set: the corrector's correction is added to each
// particle's velocity and stat[0] += sum over particles of |1 / det(I + dt C)
// - 1| (the step's predicted relative density change).  With feat set
// (collection probe): feat[orig] receives the 16 features and vel[orig] the
// final velocity, by original index.  Neither: the uncorrected large step.
struct LearnArgs {
    const MlpPacked* mlp;
    float* feat;
    float* vel;
    float* stat;
    float blend;
    const MlpTc* mlp_tc;  // set: the MLP runs on tcgen05 (mlp unused)
    uint32_t* status;     // kStatusTimeout when a tcgen05 wait gives up
    uint32_t wait_test;   // test hooks of the first tcgen05 wait (kWaitTest*, corrector_tc.cuh)
};

// G2P: slot j of Pout = particle gidx[j] of Pin advanced one substep;
// sig_out[j] = sig_in[gidx[j]]; files slot j into `next`.  learn: a large
// step of one scene (LearnArgs), else null.
int launch_g2p(const SceneTable& sc, const SimParams& p0, long long n, const float* Pin, float* Pout,
               const int32_t* gidx, const int32_t* sig_in, int32_t* sig_out, const float4* vgrid, const float* sdf,
               int32_t* pcell, const BinSet& next, uint32_t* health, cudaStream_t st,
               const LearnArgs* learn = nullptr, int block = 256);

// The kernels below take one scene's SimParams and pointers already offset to
// that scene's part of the arrays.
// ------------------------------------------------------ state transfer ----
// Loads a 26-plane host-layout state (already on the device, stride n) into
// P (original order) and sets sigma[i] = p.poff + i (global slots).
// init_rules applies initFMatrices (kernels.cu:349-358): F diagonal = 1.
int launch_state_import(const SimParams& p, const float* soa26, float* P, int32_t* sigma, bool init_rules,
                        cudaStream_t st);
// keys[sigma[j] - p.poff] = setKeys' Morton key of slot j of P (original order).
int launch_reference_keys(const SimParams& p, const float* P, const int32_t* sigma, int32_t* keys, cudaStream_t st);
// Writes the 26-plane state in original order: plane k of particle sigma[j]
// from slot j of P (VOL and MASS from the scalars).
int launch_state_export(const SimParams& p, const float* P, const int32_t* sigma, float* soa26, cudaStream_t st);
// Float3 positions in original order (changeFormat, kernels.cu:341-347).
int launch_positions_export(const SimParams& p, const float* P, const int32_t* sigma, float* xyz, cudaStream_t st);
// Node float4 (mass, x, y, z) -> 4 planes.
int launch_grid_export(const SimParams& p, const float4* grid, float* planes4, cudaStream_t st);

// ----------------------------------------------------------------- sdf ----
// tris: 9*t floats on the device, allocation padded by >= 16 bytes.  aux:
// sdf_aux_floats(t) floats on the device (16-byte aligned, padded by >= 16
// bytes) holding what sdf_prepare_host wrote: the triangles sorted by the
// Morton code of their centroids and a bounding box per 256 of them.
// wait_test: test hooks of the first triangle tile's wait (kWaitTestGiveUp /
// kWaitTestExpire, corrector_tc.cuh), acted on after the real completion.
size_t sdf_aux_floats(int t);
void sdf_prepare_host(const float* tris, int t, float* aux);
int launch_sdf_build(const SimParams& p, const float* tris, const float* aux, int t, float* sdf, uint32_t* status,
                     cudaStream_t st, uint32_t wait_test = 0u);
int launch_fill(float* dst, long long count, float value, cudaStream_t st);
// The learned step's fallback decision (one thread): rule 0 / 1 / 2 =
// MPM_FALLBACK_DENSITY_CHANGE / REST_DENSITY / REST_DENSITY_EXCESS on the
// means of stat[0..2] over n particles; sets `fallback` to 1 to reject.
int launch_learned_decide(const float* stat, long long n, int rule, float threshold,
                          cudaGraphConditionalHandle fallback, long long* counters, float* last, cudaStream_t st);
// count 32-bit words from src to dst (device memory, not overlapping).
int launch_copy_words(void* dst, const void* src, long long count, cudaStream_t st);
// dst[i] = i for i < n.
int launch_identity(int32_t* dst, int n, cudaStream_t st);

// Device status bits written by kernels with bounded waits.
enum : uint32_t {
    kStatusTimeout = 1u << 0,  // a bounded wait gave up
    kStatusBinning = 1u << 1,  // P2G met a particle outside the cell it was filed under
    kStatusCrowdList = 1u << 2 // the crowded-cell list of P2G overflowed
};

// Sets the thread's mpm_global_last_error text (engine.cu).
void set_global_error(const std::string& msg);

}  // namespace mpm

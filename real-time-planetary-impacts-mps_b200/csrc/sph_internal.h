// sph_internal.h -- the context behind the C ABI and the launchers each .cu
// file provides.  Device memory layout (all per-particle arrays in the
// original particle order unless named s*):
//
//   pos4 (x, y, z, mass)  vel4 (vx, vy, vz, 0)  acc4 (ax, ay, az, 0)  float4
//   rho u P h f c du B dhdt gnorm                                       float
//   mat next_active                                                     int32
//   active                                                              uint8
//   globals[0] global time, globals[1] dt (ticks)                       int32
//   cell_range[2^24] (first, last sorted index; UINT_MAX/0 when empty)  uint2
//   sorted working set, index = sorted slot:
//     sp4 (x, y, z, m)  sv4 (vx, vy, vz, 0)        gathered before density
//     sA (x, y, z, h)   sB (vx, vy, vz, c)   sC (m, f P / rho^2, rho, B)
//                                               written by density, read by acceleration
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/sph.h"
#include "sph_common.cuh"

namespace sph {

// FP64 diagnostics sums: kDiag values (M, Ekin, Eint, Epot, P xyz, L xyz),
// partials of kDiagBlocks blocks followed by the totals.
constexpr int kDiag = 10;
constexpr int kDiagBlocks = 148 * 4;
constexpr int kDiagDoubles = (kDiagBlocks + 1) * kDiag;

// One-sweep LSD radix sorter for (uint32 key, uint32 value) pairs.
struct RadixSorter {
    uint32_t *keys[2] = {nullptr, nullptr};
    uint32_t *vals[2] = {nullptr, nullptr};
    uint32_t *hist = nullptr;     // [kMaxPasses][256] digit counts, filled by the key producer
    uint32_t *status = nullptr;   // [kMaxPasses][tiles][256] look-back words
    uint32_t *counters = nullptr; // [kMaxPasses] tile tickets
    int n_cap = 0;
    int tiles_cap = 0;
    int spin_limit = 1 << 22;     // polls before a look-back wait gives up
    static constexpr int kThreads = 256;
    static constexpr int kItems = 16;
    static constexpr int kTile = kThreads * kItems;
    static constexpr int kMaxPasses = 4;
};

// Device-resident octree in the reference's flattened format plus the node
// records of the FMM passes.
struct Tree {
    int32_t *tree = nullptr;        // flattened ints
    int64_t tree_cap = 0;
    int32_t *level_nodes = nullptr; // [max_levels][level_cap] tree offsets, DFS order within a level
    int32_t *level_count = nullptr; // [max_levels] (device)
    int32_t *list_slot = nullptr;   // [node_cap] by data pointer: branch rank within its level, -1 leaf
    int32_t *parent_slot = nullptr; // [node_cap] by data pointer: the parent's list slot (M2M writes it)
    float4 *poles = nullptr;        // [node_cap][kPoleQ]
    float4 *locals = nullptr;       // [node_cap][kLocalQ]
    int32_t *lists[2] = {nullptr, nullptr}; // unchecked-node lists, [branch_cap][list_cap] each
    int32_t *meta = nullptr;        // device: [0] n_levels, [1] n_nodes, [2] tree_len
    int2 *node_range = nullptr;     // [node_cap] by data pointer: (first, count) in the GPU tree's key order
    int64_t node_cap = 0;
    int64_t level_cap = 0;
    int64_t branch_cap = 0;         // list slots per level
    int max_levels = 0;
    int list_cap = 1024;
    bool valid = false;
    // host mirror of the level sizes (known for host trees; upper bounds for GPU trees)
    int n_levels_host = 0;
    int level_count_host[16] = {0};
};

// Scratch of the GPU tree builder (sph_tree.cu).
struct TreeBuild {
    RadixSorter sorter;
    int32_t *nstart = nullptr;  // [max_levels][level_cap]
    int32_t *ncount = nullptr;  // [max_levels][level_cap]
    int32_t *nparent = nullptr; // [max_levels][level_cap] parent index in previous level (or -1), octant in high bits
    int64_t *scan = nullptr;    // [level_cap * 8 + 1] scan scratch
    int64_t *scan_blocks = nullptr;
    int32_t *per_particle = nullptr; // [3][n+1] ints at start, nodes at start, first level
    int32_t *noffset = nullptr; // [max_levels][level_cap] tree offset of each node
    int32_t *ndp = nullptr;     // [max_levels][level_cap] data pointer
    float *bbox = nullptr;      // device [6] lo.xyz, hi.xyz as ordered ints
    int64_t scan_cap = 0;
    const uint32_t *order = nullptr;  // particle ids in the tree's key order (last GPU build)
    int32_t *walk_queues = nullptr;   // theta-form walk: node queues of the resident warps
    uint32_t *walk_counter = nullptr; // theta-form walk: group ticket
    int64_t walk_queue_ints = 0;
};

// Learned smoothing-length seed (sph_hseed.cu): FP32 master weights and Adam
// state, the feature normalisation, the captured training set and the seed.
struct HSeed {
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    float *norm = nullptr;
    double *norm_part = nullptr;
    float *X = nullptr;     // [n][8] raw features of the captured pass
    float *y = nullptr;     // [n] targets log(h_fix / h0)
    float *h0 = nullptr;    // [n] h at the start of the captured pass
    float *nn = nullptr;    // [n] neighbour count of the last density pass
    float *seed = nullptr;  // [n] predicted starting h
    float *loss = nullptr;  // running loss of a training call
    uint32_t *stats = nullptr;  // density-pass counters: [0] NR iterations, [1] fallbacks, [2] max, [3] particles
    uint32_t *adam_step = nullptr;  // device: Adam steps taken (bias correction, sample rows)
    bool have_data = false, have_norm = false, capture = false;
    // online refresh (sph_hseed_online): Adam steps per full step on the
    // previous density pass's recorded pairs, run before the next density
    // pass (beside the tree, sort and gravity passes in a full step)
    int online_iters = 0, online_batch = 16384;
    float online_lr = 1e-3f;
    bool trained_ahead = false;  // this step's refresh is already enqueued
};

struct HSeedArgs {
    int n;
    const float4 *pos4;  // (x, y, z, mass)
    const float *h, *dhdt, *rho, *u;
    const int32_t *mat, *nat;
    const uint8_t *active;
    const int32_t *globals;
    const float *nn;
    float *X, *y, *h0, *seed;
    const float *params;
    float *grads;
    const float *norm;
    float *loss;
    uint32_t *health;
    uint32_t salt;
};

}  // namespace sph

struct sph_ctx {
    int n = 0;
    int device = 0;
    sph_params params{};
    std::string forsterite_path, fe_path;

    float4 *pos4 = nullptr, *vel4 = nullptr, *acc4 = nullptr;
    float *rho = nullptr, *u = nullptr, *P = nullptr, *h = nullptr, *f = nullptr, *c = nullptr;
    float *du = nullptr, *B = nullptr, *dhdt = nullptr, *gnorm = nullptr;
    float *phi = nullptr;  // potential (theta gravity form)
    // mixed-precision form: FP64 master positions (x, y, z, -) and FP64 globals
    // ([0] global time in seconds); the float positions are their roundings
    double4 *pos64 = nullptr;
    double *dglob = nullptr;
    double *diag = nullptr;  // diagnostics: block partials, then the totals
    sph_form form{SPH_GRAVITY_REFERENCE, 0.5f, SPH_HSEED_PLAIN, SPH_PRECISION_REFERENCE, 0.f, SPH_TIMESTEP_GLOBAL};
    int32_t *mat = nullptr, *nat = nullptr;
    uint8_t *active = nullptr;
    int32_t *globals = nullptr;
    uint32_t *health = nullptr;

    sph::RadixSorter cell_sort;
    uint2 *cell_range = nullptr;
    bool cells_have_prev = false;  // cell_range holds the entries of cell_sort.keys[1]
    int cell_final = 1;            // buffer index of the sorted cell keys

    float4 *sp4 = nullptr, *sv4 = nullptr, *sA = nullptr, *sB = nullptr, *sC = nullptr;
    // density and acceleration over cell tiles: (first, end) sorted range of
    // each tile; counters [0] tiles, [1] tile ticket, [2] deferred, [3] spare
    // of the density pass's cell tiles, [4] tiles and [5] ticket of its coarse
    // tiles, [8..13] the same for the acceleration pass; the sorted indices
    // handed to the per-particle pass
    uint2 *tiles = nullptr;
    uint32_t *tile_ctr = nullptr;
    uint32_t *deferred = nullptr;
    // tile sizes: a 128-cell block is one tile up to tile_big_max particles
    // (0: never; measured slower at N = 1e6: such tiles overflow shared memory
    // and fall back to octets), else its 64-cell halves up to tile_block_max,
    // else their 16-cell quarters up to tile_half_max, else their octets
    uint32_t tile_big_max = 0;
    uint32_t tile_block_max = 320;
    uint32_t tile_half_max = 256;
    // coarse tiles, for particles whose boxes reach past the cell tiles'
    // limit: 64-cell units (4 x 4 x 4 cells, indexed by the cell key >> 6)
    // with their (first, last) sorted index, rebuilt by every sort; a flag per
    // 512-cell block that holds such a particle, set by the cell-tile passes
    // and cleared when the coarse tiles are listed.  tile_coarse 0 hands
    // those particles to the per-particle pass instead.
    uint2 *units = nullptr;
    uint8_t *coarse_flags = nullptr;
    int tile_coarse = 1;
    float2 *eos_forsterite = nullptr, *eos_fe = nullptr;
    sph::EosTables eos{};

    sph::Tree tree;
    sph::TreeBuild tb;

    void *stage = nullptr;  // device staging for uploads/downloads
    size_t stage_bytes = 0;
    int32_t *snapshot = nullptr;

    sph::HSeed hs;

    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    cudaStream_t own_stream = nullptr;
    // sph_step_host: its graph, the host buffers it was captured for, and the
    // side stream and events of the overlapped input copies
    cudaGraphExec_t host_graph = nullptr;
    sph_host_state host_in{}, host_out{};
    cudaStream_t side_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

namespace sph {

// sph_sort.cu
sph_status sort_alloc(RadixSorter &s, int n);
void sort_free(RadixSorter &s);
// Sort keys[0]/vals[0] (n pairs, `bits` significant key bits) whose digit
// histograms the producer already accumulated into s.hist.  Returns the buffer
// index (0/1) that holds the result.
int radix_sort_pairs(RadixSorter &s, int n, int bits, cudaStream_t st, uint32_t *health);
sph_status launch_sort(sph_ctx *ctx, cudaStream_t st);
void launch_init_cells(sph_ctx *ctx, cudaStream_t st);
// 64-bit exclusive scan of `count` values (count read on the host side bound
// `n_max`, actual count from *d_count when non-null) into out; *total at out[count].
void scan_exclusive_i64(const int64_t *in, int64_t *out, int64_t *block_scratch, int n_max, const int32_t *d_count,
                        cudaStream_t st);

// sph_hydro.cu
sph_status launch_density(sph_ctx *ctx, cudaStream_t st);
sph_status launch_acceleration(sph_ctx *ctx, cudaStream_t st);
sph_status launch_step(sph_ctx *ctx, cudaStream_t st);
sph_status launch_snapshot(sph_ctx *ctx, cudaStream_t st);
// FP64 copies of the float positions (entering the mixed-precision form)
sph_status launch_pos_to64(sph_ctx *ctx, cudaStream_t st);
// FP64 conservation sums into ctx->diag (see sph_diagnostics)
sph_status launch_diag_sums(sph_ctx *ctx, cudaStream_t st);

// sph_gravity.cu
sph_status launch_gravity(sph_ctx *ctx, cudaStream_t st);

// sph_hseed.cu
sph_status hseed_alloc(sph_ctx *ctx);
void hseed_free(sph_ctx *ctx);
int hseed_num_params();
int hseed_norm_size();
sph_status launch_hseed_capture(sph_ctx *ctx, cudaStream_t st);
sph_status launch_hseed_targets(sph_ctx *ctx, cudaStream_t st);
sph_status launch_hseed_infer(sph_ctx *ctx, cudaStream_t st);
sph_status launch_hseed_norm(sph_ctx *ctx, cudaStream_t st);
sph_status launch_hseed_grad(sph_ctx *ctx, uint32_t it, bool counted, int batch, uint32_t salt, cudaStream_t st);
sph_status launch_hseed_adam(sph_ctx *ctx, float lr, cudaStream_t st);

// sph_gravity_theta.cu
sph_status launch_gravity_theta(sph_ctx *ctx, cudaStream_t st);
// the potential alone (acceleration and |a| untouched), opening angle theta,
// on the current GPU tree
sph_status launch_potential_theta(sph_ctx *ctx, float theta, cudaStream_t st);
sph_status launch_direct_f64(sph_ctx *ctx, const int32_t *d_targets, int nt, double *d_out, cudaStream_t st);

// sph_tree.cu
sph_status tree_alloc(sph_ctx *ctx);
void tree_free(sph_ctx *ctx);
sph_status launch_tree_build(sph_ctx *ctx, cudaStream_t st);

// sph_api.cu
// One full step (tree, sort, gravity, density, acceleration, step) on st.
sph_status full_step(sph_ctx *ctx, cudaStream_t st);
// sph_hseed.cu: the online refresh of the learned seed (standardisation and
// Adam steps on the last recorded pass) on st; whether one is due this step
bool hseed_online_due(const sph_ctx *ctx);
sph_status launch_hseed_online(sph_ctx *ctx, cudaStream_t st);
// Destroy the captured step graphs (sph_step_all's and sph_step_host's):
// called whenever what they replay changes.
void drop_graphs(sph_ctx *ctx);
void set_error(const char *fmt, ...);
sph_status cuda_status(cudaError_t e, const char *what);

}  // namespace sph

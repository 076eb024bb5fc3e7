/*
 * sph.h -- C ABI of the B200 SPH + FMM step (libsph_b200.so).
 *
 * Drop-in for the reference's pass API, class Compute
 * (SPH/Compute/Compute.hpp:40-59).  A context owns every device buffer of one
 * simulation; each pass is stream-ordered and asynchronous, like the
 * reference's encoders into a caller-owned MTL::CommandBuffer, and the caller
 * synchronises (sph_synchronize) where the reference commits and waits
 * (SPH/Rendering/Headless.cpp:53-54).
 *
 * Plain types only: no CUDA or torch types cross this boundary.  A stream is
 * passed as `void*` holding a cudaStream_t (NULL = the legacy default stream).
 * Every call returns an sph_status; no exception crosses the ABI.  A context
 * is used by one host thread at a time.
 */
#ifndef SPH_B200_H
#define SPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SPH_OK = 0,
    SPH_ERR_INVALID_ARG = 1,
    SPH_ERR_OOM = 2,
    SPH_ERR_IO = 3,
    SPH_ERR_CUDA = 4,
    SPH_ERR_DEVICE_HEALTH = 5, /* a kernel raised a health bit (see SPH_HEALTH_*) */
    SPH_ERR_TIMEOUT = 6,       /* a bounded device wait gave up */
    SPH_ERR_UNSUPPORTED = 7
} sph_status;

/* Health bits raised by kernels instead of trapping (sph_get_health). */
#define SPH_HEALTH_SORT_TIMEOUT      0x0001u /* radix-sort look-back wait gave up */
#define SPH_HEALTH_LIST_CAPACITY     0x0002u /* a tree level exceeded the unchecked-list storage */
#define SPH_HEALTH_TREE_CAPACITY     0x0004u /* the tree outgrew its preallocated storage */
#define SPH_HEALTH_NAN_DENSITY       0x0008u /* a density or pressure came out non-finite */
#define SPH_HEALTH_SCAN_TIMEOUT      0x0010u /* a scan look-back wait gave up */
#define SPH_HEALTH_ROOT_LEAF         0x0020u /* the root is a leaf: gravity pass skipped */
#define SPH_HEALTH_MLP_TIMEOUT       0x0040u /* a tensor-core wait of the h-seed network gave up */
#define SPH_HEALTH_BAD_INPUT         0x0080u /* sph_step_host received an h outside (0, 10] */

typedef struct sph_ctx sph_ctx;

/* Tree sources for the gravity pass. */
#define SPH_TREE_GPU  0 /* Morton octree built on the GPU from sorted keys every sph_update_tree */
#define SPH_TREE_HOST 1 /* a host-built tree in the reference format, given by sph_set_tree */

/* Runtime knobs.  The physics constants of SPH/Parameters.h:11-53 are
 * compiled into the kernels; these are the structural ones. */
typedef struct {
    int32_t max_children_in_leaf;   /* MAX_CHILDREN_IN_LEAF (Parameters.h:43), default 4 */
    int32_t max_tree_depth;         /* MAX_TREE_DEPTH (Parameters.h:39), default 7, 1..10 */
    int32_t max_unchecked_pointers; /* MAX_UNCHECKED_POINTERS (Parameters.h:42), default 1024 */
    int32_t aneos_resolution;       /* ANEOS_TEXTURE_RESOLUTION (Parameters.h:20), default 2048 */
    int32_t tree_source;            /* SPH_TREE_GPU (default) or SPH_TREE_HOST */
    const char *forsterite_table;   /* ANEOS text table for material 400 (Compute.cpp:45) */
    const char *fe85si15_table;     /* ANEOS text table for every other material (Compute.cpp:46) */
} sph_params;

/* Initial conditions: the fields of DataStruct that Compute loads
 * (SPH/hdfHandler/hdfHandler.hpp:15-26, Compute.cpp:52-77).  Host pointers. */
typedef struct {
    int32_t n;
    const float *pos;        /* 3n, xyz interleaved */
    const float *vel;        /* 3n */
    const float *rho;        /* n */
    const float *u;          /* n, specific internal energy */
    const float *mass;       /* n */
    const float *pressure;   /* n */
    const float *h;          /* n, smoothing length */
    const int32_t *material; /* n, ANEOS material id (400 forsterite) */
} sph_ic;

/* Per-particle and global fields (sph_upload / sph_download / sph_get_buffer).
 * Host-side element types: F3 = 3 floats per particle, F = float, I = int32,
 * U = uint32, B = uint8.  Per-particle fields are in the original particle
 * order.  CELL_* are the sorted cell arrays of Compute::sort. */
typedef enum {
    SPH_FIELD_POS = 0,          /* F3  positionBuffer */
    SPH_FIELD_VEL = 1,          /* F3  _velocityBuffer */
    SPH_FIELD_ACC = 2,          /* F3  _accelerationBuffer */
    SPH_FIELD_RHO = 3,          /* F   densityBuffer */
    SPH_FIELD_U = 4,            /* F   _internalEnergyBuffer */
    SPH_FIELD_MASS = 5,         /* F   _massBuffer */
    SPH_FIELD_PRESSURE = 6,     /* F   _pressureBuffer */
    SPH_FIELD_H = 7,            /* F   _smoothingLengthBuffer */
    SPH_FIELD_GRAD_TERM = 8,    /* F   _gradientTermsBuffer */
    SPH_FIELD_SOUND_SPEED = 9,  /* F   _speedOfSoundBuffer */
    SPH_FIELD_DU = 10,          /* F   _dInternalEnergyBuffer */
    SPH_FIELD_BALSARA = 11,     /* F   _balsara */
    SPH_FIELD_DHDT = 12,        /* F   _dhdt */
    SPH_FIELD_GRAV_NORM = 13,   /* F   _gravAbs */
    SPH_FIELD_MATERIAL = 14,    /* I   materialIdBuffer */
    SPH_FIELD_ACTIVE = 15,      /* B   _active */
    SPH_FIELD_NEXT_ACTIVE = 16, /* I   _nextActiveTime */
    SPH_FIELD_GLOBAL_TIME = 17, /* I   _globalTime (1 value, ticks of 32/65536 s); an upload in the mixed form
                                       also sets the FP64 time to ticks x 2^-11 s */
    SPH_FIELD_DT = 18,          /* I   _dt (1 value, ticks) */
    SPH_FIELD_CELL_KEY = 19,    /* U   _cellArrayi[].x after sort (n) */
    SPH_FIELD_CELL_INDEX = 20,  /* U   _cellArrayi[].y after sort (n) */
    SPH_FIELD_CELL_START = 21,  /* U   _cellStart (2^24), UINT_MAX when empty; download only */
    SPH_FIELD_CELL_END = 22,    /* U   _cellEnd (2^24), 0 when empty; download only */
    SPH_FIELD_POTENTIAL = 23,   /* F   gravitational potential G phi (SPH_GRAVITY_THETA only; no reference buffer) */
    SPH_FIELD_POS64 = 24,       /* D3  FP64 master positions (3n doubles) of SPH_PRECISION_MIXED; an upload also
                                       sets the float positions to their roundings */
    SPH_FIELD_NEIGHBOURS = 25,  /* F   neighbour count of the last density pass, a feature of the learned h
                                       seed (present once the seed is in use or recording; no reference buffer) */
    SPH_FIELD_COUNT = 26
} sph_field;

/* Defaults equal to SPH/Parameters.h (table paths are the reference's names). */
void sph_params_default(sph_params *p);

/* Compute::Compute (Compute.cpp:22-36, 44-132): allocate, load the two EOS
 * tables, upload the initial state (active = 1, nextActiveTime = 0, time = 0),
 * select the current CUDA device.  For SPH_TREE_GPU the first tree is built
 * here; for SPH_TREE_HOST call sph_set_tree before sph_gravity. */
sph_status sph_create(const sph_params *params, const sph_ic *ic, sph_ctx **out);
sph_status sph_destroy(sph_ctx *ctx);
int32_t sph_num_particles(const sph_ctx *ctx);

/* Compute::updateOctreeBuffer (Compute.cpp:456-508): rebuild the octree on the
 * GPU from the current positions (SPH_TREE_GPU).  No host thread. */
sph_status sph_update_tree(sph_ctx *ctx, void *stream);
/* Give the context a tree in the reference's flattened format (octree.cpp:24-109):
 * leaf [n, dataPtr, p0..], branch [0, dataPtr, c0..c7 or -1]; levels as node
 * offsets (level_offsets has n_levels+1 entries into level_nodes). */
sph_status sph_set_tree(sph_ctx *ctx, const int32_t *tree, int32_t tree_len, const int32_t *level_offsets,
                        const int32_t *level_nodes, int32_t n_levels, int32_t n_nodes);

/* Read back the current tree (synchronous).  Any output pointer may be NULL to
 * query sizes only; level_offsets needs room for 17 entries. */
sph_status sph_get_tree(sph_ctx *ctx, int32_t *tree, int64_t tree_room, int32_t *tree_len, int32_t *level_offsets,
                        int32_t *level_nodes, int64_t level_nodes_room, int32_t *n_levels, int32_t *n_nodes);

/* Read back the FMM node records of the last gravity pass (synchronous), by
 * data pointer: poles 24 floats per node (com.xyz, size | M, XX, XY, XZ | YY,
 * YZ, ZZ, power2 | min.xyz, minGrav | max.xyz, active | X, Y, Z, 0), locals 16
 * floats per node (pos.xyz, e0 | e1..e4 | e5..e8 | e9, 0, 0, 0).  Either
 * pointer may be NULL; n_nodes is the node count of the current tree. */
sph_status sph_get_tree_nodes(sph_ctx *ctx, float *poles, float *locals, int32_t n_nodes);

/* The passes of Headless::step (Headless.cpp:43-51), in order. */
sph_status sph_sort(sph_ctx *ctx, void *stream);         /* Compute::sort (Compute.cpp:265-326) */
sph_status sph_gravity(sph_ctx *ctx, void *stream);      /* Compute::gravitationalPass (:328-377) */
sph_status sph_density(sph_ctx *ctx, void *stream);      /* Compute::densityPass (:179-208) */
sph_status sph_acceleration(sph_ctx *ctx, void *stream); /* Compute::accelerationPass (:210-240) */
sph_status sph_step(sph_ctx *ctx, void *stream);         /* Compute::stepPass (:242-263) */

/* Numerical forms beside the reference's own.  None has a counterpart in the
 * reference; the default form (all zero) reproduces the reference's logic,
 * quirks included, and is what the parity tests check against it. */
#define SPH_GRAVITY_REFERENCE 0 /* adaptive acceptance, forced leaf M2L, truncated softening (Compute.cpp:328-377) */
#define SPH_GRAVITY_THETA     1 /* opening-angle group walk: quadrupole M2P, exact softened P2P, Kahan sums;
                                   needs the GPU-built tree (SPH_TREE_GPU) */
#define SPH_PRECISION_REFERENCE 0 /* float positions drifted in float, as the reference (step.metal:45) */
#define SPH_PRECISION_MIXED     1 /* FP64 master positions and global time (float working copies), Kahan-
                                     compensated acceleration, du/dt and dh/dt sums */
#define SPH_TIMESTEP_GLOBAL     0 /* the reference's active test as shipped, globalTime <= nextActiveTime
                                     (P2M.metal:31): every particle is active every step */
#define SPH_TIMESTEP_INDIVIDUAL 1 /* README.md:60-64 as described: a particle is active once the global time
                                     reaches its next active time; a leaf with an active particle, and a branch
                                     of leaves with an active leaf, activate all their particles; inactive
                                     particles are only integrated (no gravity, neighbour or acceleration
                                     work); the global step never passes an inactive particle's next
                                     active time */
#define SPH_HSEED_PLAIN   0 /* the iteration starts from the particle's own h (density.metal:73-74) */
#define SPH_HSEED_LEARNED 1 /* it starts from the learned seed (sph_hseed_train), with fallback */
typedef struct {
    int32_t gravity;   /* SPH_GRAVITY_* */
    float theta;       /* opening angle of SPH_GRAVITY_THETA: a node of radius r_node (about its centre of
                          mass) is accepted for a group of particles when r_node < theta d, d = the distance
                          from its centre of mass to the group's bounding box, and d > 2 x softening */
    int32_t h_seed;    /* SPH_HSEED_* */
    int32_t precision; /* SPH_PRECISION_* */
    float h_tolerance; /* convergence test of the h iteration, |dh| / h <= tol; 0 = DENSITY_ETA (0.005) */
    int32_t timestep;  /* SPH_TIMESTEP_* */
} sph_form;
void sph_form_default(sph_form *f); /* reference form, theta 0.5 */
/* Select the form for the following passes (drops a captured step graph).
 * Entering SPH_PRECISION_MIXED takes the current float positions as the FP64
 * master positions and the current global time as the FP64 time. */
sph_status sph_set_form(sph_ctx *ctx, const sph_form *f);
sph_status sph_get_form(const sph_ctx *ctx, sph_form *f);

/* Tiling of the product build's density and acceleration passes.  It changes
 * how the work is scheduled, not what is computed (up to the float summation
 * order).  A 128-cell block of the sorted particles is one tile when it holds
 * at most big_max particles (0: never), else each 64-cell half is one up to
 * block_max, else each 16-cell quarter up to half_max, else each octet.
 * coarse != 0 runs the particles whose neighbour boxes reach more than 3 cells
 * past their own in coarse tiles (512-cell blocks staged by 4 x 4 x 4-cell
 * units); coarse = 0 hands them to the per-particle walk.  The parity build
 * (one lane per particle) ignores the tiling.  Drops a captured step graph. */
typedef struct {
    uint32_t big_max;   /* default 0 */
    uint32_t block_max; /* default 320 */
    uint32_t half_max;  /* default 256 */
    int32_t coarse;     /* default 1 */
} sph_tiling;
sph_status sph_set_tiling(sph_ctx *ctx, const sph_tiling *t);
sph_status sph_get_tiling(const sph_ctx *ctx, sph_tiling *t);

/* FP64 direct-sum gravity at n_targets particles (host array of particle
 * indices), from the current positions and masses of all particles, with the
 * cubic-spline softened kernel and its exact coefficients: out receives
 * (ax, ay, az, phi) per target, G included.  The accuracy reference for the
 * gravity forms; no counterpart in the reference.  Synchronous. */
sph_status sph_gravity_direct_f64(sph_ctx *ctx, const int32_t *targets, int32_t n_targets, double *out,
                                  void *stream);

/* Learned smoothing-length seed (no counterpart in the reference).  An
 * 8 -> 64 -> 64 -> 1 MLP, run and trained on the tensor cores (BF16 operands,
 * FP32 accumulation), predicts from a particle's state at the start of the
 * density pass the fixed point its iteration approaches, h_fix =
 * RESOLUTION_ETA (m / rho)^(1/3) at the converged density; SPH_HSEED_LEARNED
 * starts the iteration there (density.metal:73-143), falling back to the
 * plain guess when the first sweep moves the seed by more than 5%.
 * sph_hseed_capture(ctx, 1): every following density pass records its
 *   (features, log(h_fix / h0)) pairs as the training set (the last pass's).
 * sph_hseed_train: `iterations` Adam steps (learning rate lr) on minibatches
 *   of `batch` rows drawn from the recorded set, after deriving the feature
 *   and target standardisation from it.  *loss = the last minibatch's mean
 *   squared error (standardised target), may be NULL.  Synchronous.
 * sph_hseed_gradient: the loss gradient of one minibatch (row r of the batch
 *   is particle ((r * 0x9E3779B97F4A7C15) ^ salt) mod n, arithmetic modulo
 *   2^64) without updating the weights: grads receives
 *   sph_hseed_num_params() floats, in the order W1[64][8], b1[64],
 *   W2[64][64], b2[64], w3[64], b3.  Synchronous.
 * sph_hseed_params: copy the FP32 weights out (get) and/or in (set); either
 *   may be NULL.  sph_hseed_dataset: the recorded raw features [n][8],
 *   targets log(h_fix / h0) [n] and the standardisation (feature means
 *   [8], feature 1/deviations [8], target mean, target deviation); any may be
 *   NULL.
 * sph_hseed_stats: counters of the last density pass. */
typedef struct {
    uint32_t sweeps;     /* density sweeps of the h iteration, summed over particles */
    uint32_t fallbacks;  /* particles whose learned seed was abandoned */
    uint32_t max_sweeps; /* most sweeps of one particle */
    uint32_t particles;  /* particles iterated */
    uint32_t tiles;      /* cell tiles the product build's density pass staged */
    uint32_t deferred;   /* particles it handed from the tiles to the per-particle walk */
    uint32_t accel_deferred; /* the same count of the last acceleration pass */
    uint32_t coarse_tiles;   /* coarse tiles (512-cell blocks) of the density pass: blocks
                                holding particles whose boxes reach past the cell tiles */
    uint32_t accel_coarse_tiles; /* the same count of the last acceleration pass */
} sph_hseed_stats;
int32_t sph_hseed_num_params(void);
sph_status sph_hseed_capture(sph_ctx *ctx, int32_t on);
sph_status sph_hseed_train(sph_ctx *ctx, int32_t iterations, int32_t batch, float lr, float *loss, void *stream);
sph_status sph_hseed_gradient(sph_ctx *ctx, int32_t batch, uint32_t salt, float *grads, float *loss, void *stream);
/* Online refresh of the learned seed: with iterations > 0, every density pass
 * records its pairs (as sph_hseed_capture) and, while the learned seed is the
 * form's start, each step first takes `iterations` Adam steps (minibatch
 * `batch`, rate lr) on the previous pass's pairs, after re-deriving the
 * standardisation from them.  In sph_step_all, sph_step_host and ensembles
 * these steps run on a second stream beside the tree, sort and gravity
 * passes and are joined before the density pass; in a lone sph_density they
 * run at its start.  The seed otherwise drifts from the state it was trained
 * on: its sweeps per particle grow step by step.  iterations = 0 turns the
 * refresh and the recording off.  Drops a captured step graph. */
sph_status sph_hseed_online(sph_ctx *ctx, int32_t iterations, int32_t batch, float lr);
sph_status sph_hseed_params(sph_ctx *ctx, float *get, const float *set);
sph_status sph_hseed_dataset(sph_ctx *ctx, float *features, float *targets, float *norm);
/* The seed network's input/target standardisation (18 floats, the layout of
 * sph_hseed_dataset's norm): get it (after training), and/or set it, which
 * with sph_hseed_params restores a trained network, e.g. on resume from a
 * checkpoint.  Either pointer may be NULL.  Synchronous. */
sph_status sph_hseed_norm(sph_ctx *ctx, float *get, const float *set);
sph_status sph_hseed_get_stats(sph_ctx *ctx, sph_hseed_stats *out);

/* FP64 conservation diagnostics (no counterpart in the reference, which
 * computes no potential: L2P.metal:12-32 returns only the acceleration).
 * Sums over all particles in FP64, in a fixed order: mass, kinetic energy
 * 1/2 m v^2, internal energy m u, potential energy 1/2 m phi, momentum m v and
 * angular momentum m x v about the origin (FP64 positions in the mixed form).
 * phi is evaluated for the current positions by the opening-angle walk at
 * theta_potential (0 = 0.5) on a freshly built GPU tree, without touching the
 * accelerations; with a host tree (SPH_TREE_HOST) no potential is computed
 * and potential_valid is 0.  Synchronous on `stream`. */
typedef struct {
    double mass, kinetic, internal, potential, total;
    double momentum[3], angular_momentum[3];
    double time;             /* global time, seconds (FP64 in the mixed form) */
    int32_t potential_valid;
    uint32_t health;         /* the device health word */
} sph_diag;
sph_status sph_diagnostics(sph_ctx *ctx, void *stream, float theta_potential, sph_diag *out);

/* Cell sort for callers that cannot allocate device memory.  No counterpart in
 * the reference.  Meant for code whose host framework owns every device
 * allocation (pools, arenas, memory accounting), or that must not call
 * cudaMalloc/cudaFree on a latency-critical thread because those calls can
 * synchronise the device.  From positions the caller already holds on the
 * device (pos_xyz: 3n floats, xyz interleaved) it writes the same sorted
 * (cell key, particle index) pairs that sph_sort produces (SPH_FIELD_CELL_KEY,
 * SPH_FIELD_CELL_INDEX) into cell_key and cell_index (n entries each, device
 * memory).  It allocates nothing: its scratch is one fixed array inside the
 * library, present on every GPU that loads the library until the process
 * exits, which bounds n to SPH_SORT_NOALLOC_MAX_N (larger n is rejected with
 * SPH_ERR_INVALID_ARG).  The first call on each device looks up that array's
 * device address; make that first call before any stream capture.  Every call
 * reuses the array, so calls that overlap on the GPU (unordered streams,
 * several host threads) race; order them on one stream.  Asynchronous on
 * `stream`; no context is needed. */
#define SPH_SORT_NOALLOC_MAX_N 262144
sph_status sph_sort_cells_noalloc(const float *pos_xyz, int32_t n, uint32_t *cell_key, uint32_t *cell_index,
                                  void *stream);
/* Health of the last sph_sort_cells_noalloc call on the current device: waits
 * for `stream`, reads the health word kept inside the library's fixed scratch
 * (cudaMemcpyFromSymbol, no allocation) into *word (may be NULL) and returns
 * SPH_ERR_TIMEOUT when a bounded look-back wait gave up, in which case the
 * call's outputs are incomplete.  The next sph_sort_cells_noalloc call clears
 * the word.  No counterpart in the reference. */
sph_status sph_sort_cells_noalloc_health(void *stream, uint32_t *word);

/* Self-test of the radix sort's bounded look-back wait (no counterpart in the
 * reference): one sort tile is launched whose predecessor's status words are
 * withheld, so its wait gives up after spin_limit polls (1..2^22) and raises
 * SPH_HEALTH_SORT_TIMEOUT without touching any key.  With ctx, the context's
 * health word is raised (sph_synchronize then returns SPH_ERR_TIMEOUT); with
 * ctx NULL, the allocation-free sort's (sph_sort_cells_noalloc_health then
 * returns SPH_ERR_TIMEOUT).  The GPU stays usable; clear the word afterwards
 * (sph_clear_health, or the next sph_sort_cells_noalloc call). */
sph_status sph_selftest_lookback_timeout(sph_ctx *ctx, int32_t spin_limit, void *stream);
/* Self-test of the GPU tree build's capacity check (no counterpart in the
 * reference): one tree build runs with its storage bound lowered to 16 ints,
 * so the layout kernels find the tree too large, skip the writes that would
 * not fit and raise SPH_HEALTH_TREE_CAPACITY (sph_synchronize then returns
 * SPH_ERR_DEVICE_HEALTH).  The storage itself is untouched beyond the bound;
 * the tree is marked stale, the next tree build (sph_update_tree, sph_step)
 * makes a whole one.  SPH_TREE_GPU contexts only. */
sph_status sph_selftest_tree_capacity(sph_ctx *ctx, void *stream);

/* n_steps x (tree, sort, gravity, density, acceleration, step), replayed from
 * a CUDA graph captured on first use (Headless::step without the snapshot). */
sph_status sph_step_all(sph_ctx *ctx, void *stream, int32_t n_steps);

/* One full step whose state travels through host memory (no counterpart in
 * the reference, whose Headless loop keeps the state on the device): the
 * non-NULL fields of `in` are copied to the device at the start of the step
 * and the non-NULL fields of `out` back at its end, all on `stream` and
 * asynchronous to the host.  Layouts are sph_upload's: x y z per particle for
 * the vector fields; pos64 (FP64 positions) in the mixed-precision form and
 * pos (float positions, the mass kept) in the others.  Every buffer must be
 * page-locked (cudaHostAlloc, cudaHostRegister) and stay valid until the
 * stream passes the step.  The positions are copied first; velocity, u, h
 * and rho are copied on a second stream while the tree, sort and gravity
 * passes run, and joined before the density pass.  An h outside (0, 10] is
 * replaced by MAX_SMOOTHING_LENGTH (1) and raises SPH_HEALTH_BAD_INPUT
 * (sph_synchronize then returns SPH_ERR_DEVICE_HEALTH) rather than being
 * checked on the host.  The
 * first call with a set of buffers runs eagerly and waits, then captures a
 * CUDA graph that later calls with the same buffers replay. */
typedef struct {
    double *pos64;
    float *pos;
    float *vel;
    float *u;
    float *h;
    float *rho;
} sph_host_state;
sph_status sph_step_host(sph_ctx *ctx, const sph_host_state *in, const sph_host_state *out, void *stream);

/* Compute::drawSnapshot (Compute.cpp:396-448, render.metal:49-66): splat the
 * material ids into a 1024x1024 int image by atomic max.  When image is not
 * NULL it receives the image (synchronous). */
sph_status sph_draw_snapshot(sph_ctx *ctx, void *stream, int32_t *image);

/* Buffers.hpp:14-59 (writeDataToPrivateBuffer): synchronous host<->device copies.
 * count = number of host elements (3n floats for F3 fields, n otherwise).
 * They wait for all device work before and after the copy, like the
 * reference's blit followed by waitUntilCompleted (Buffers.hpp:39-59). */
sph_status sph_upload(sph_ctx *ctx, sph_field field, const void *host, size_t count);
sph_status sph_download(sph_ctx *ctx, sph_field field, void *host, size_t count);
/* The same copies ordered on `stream` and asynchronous to the host: copy,
 * then the pack/unpack kernel of F3 and mass fields, all on `stream`, through
 * one device staging buffer of the context (calls on one stream are ordered,
 * so consecutive transfers may share it; do not interleave transfers of one
 * context on two streams).  With pinned host memory the copies overlap host
 * work; the host buffer must stay valid until the stream reaches them. */
sph_status sph_upload_async(sph_ctx *ctx, sph_field field, const void *host, size_t count, void *stream);
sph_status sph_download_async(sph_ctx *ctx, sph_field field, void *host, size_t count, void *stream);
/* Borrow the device buffer behind a field (valid until sph_destroy).  F3 fields
 * are stored as 16-byte float4 records; the reported stride is in *stride. */
sph_status sph_get_buffer(sph_ctx *ctx, sph_field field, void **device_ptr, size_t *bytes, size_t *stride);

/* Wait for the stream, then report SPH_ERR_DEVICE_HEALTH if a health bit is set. */
sph_status sph_synchronize(sph_ctx *ctx, void *stream);
sph_status sph_get_health(sph_ctx *ctx, uint32_t *word);
sph_status sph_clear_health(sph_ctx *ctx);

/* Measurement probe (no counterpart in the reference): `blocks` x 256 threads
 * each run 8 independent FP32 FMA chains of `iters` steps, 16 x iters flops
 * per thread; sink is device memory of `blocks` floats (written only to keep
 * the result alive).  Asynchronous on `stream`; time it with events to get the
 * FP32 FMA peak of the device. */
sph_status sph_probe_fp32_fma(int32_t blocks, int32_t iters, float *sink, void *stream);

/* Batched ensemble (no counterpart in the reference, which runs one impact per
 * process: Headless.cpp:43-51).  n_instances independent impacts on the
 * current device, each with its own initial conditions and form (forms may be
 * NULL: all defaults) and the shared params; each instance is a full context
 * (reachable through sph_ensemble_instance for uploads, downloads and
 * diagnostics).  sph_ensemble_step advances every instance by n_steps steps,
 * one launch of one CUDA graph per step whose branches are the instances'
 * full steps, so small instances run side by side on the device.
 * With autotune != 0 the tuner picks per instance, on a scratch copy made from
 * the same initial conditions (the instance itself is not advanced): the
 * density / acceleration tile size, by timing, and for SPH_GRAVITY_THETA the
 * leaf capacity among 1, 2 and 4 times params->max_children_in_leaf, by timing
 * among those whose gravity has a median relative error <= 1e-3 against the
 * FP64 direct sum on 512 targets.  sph_ensemble_get_tuning reports the choice.
 * Creation synchronises the device.  Stepping is asynchronous on `stream`;
 * the first sph_ensemble_step call runs its first step eagerly, waits for it
 * and captures the step graph (so make it outside any stream capture), as
 * sph_step_all does.  sph_ensemble_synchronize waits and checks every
 * instance's health word. */
typedef struct sph_ensemble sph_ensemble;
typedef struct {
    int32_t max_children_in_leaf; /* leaf capacity the instance runs with */
    uint32_t tile_block_max;      /* particles of a 64-cell density / acceleration tile before it is split */
    float ms_per_step;            /* the tuner's time of one full step with this choice (0: not tuned) */
    float gravity_median_error;   /* its gravity error on the tuning sample (-1: not checked) */
} sph_ensemble_tuning;
sph_status sph_ensemble_create(const sph_params *params, int32_t n_instances, const sph_ic *ics,
                               const sph_form *forms, int32_t autotune, sph_ensemble **out);
sph_status sph_ensemble_destroy(sph_ensemble *e);
int32_t sph_ensemble_size(const sph_ensemble *e);
sph_status sph_ensemble_instance(sph_ensemble *e, int32_t i, sph_ctx **ctx);
sph_status sph_ensemble_get_tuning(const sph_ensemble *e, int32_t i, sph_ensemble_tuning *out);
sph_status sph_ensemble_step(sph_ensemble *e, void *stream, int32_t n_steps);
sph_status sph_ensemble_synchronize(sph_ensemble *e, void *stream);

/* Host-only helpers (no GPU work). */
/* ANEOS.cpp:21-175: parse a table and resample it to res x res (pressure,
 * sound speed) pairs, rho rows, u columns.  out holds 2*res*res floats. */
sph_status sph_eos_resample(const char *path, int32_t res, float *out);
const char *sph_status_string(sph_status s);
const char *sph_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SPH_B200_H */

/*
 * oracle.h -- CPU restatement of the reference's per-step SPH + FMM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library under
 * real-time-planetary-impacts-mps_b200/) links, loads or calls this code.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the
 * checker.
 *
 * Every pass mirrors one reference kernel (file:line of the reference project
 * given beside each function in oracle.cpp).  The state layout is plain SoA
 * with xyz-interleaved vectors (3 floats per particle), all in the original
 * particle order, exactly like the reference's Compute buffers.
 *
 * Parity pin: oracle/ref_build.sh compiles the reference's own Metal kernels
 * (through a host shim) and octree.cpp into oracle/_ref/libref.so; the golden
 * fixtures under tests/golden/ come from that build and the CPU tests check
 * this restatement against them.
 */
#ifndef SPH_ORACLE_H
#define SPH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t n;
    float *pos, *vel, *acc;              /* 3n each, xyz interleaved */
    float *rho, *u, *mass, *pressure, *h;
    float *grad_term, *sound_speed, *du, *balsara, *dhdt, *grav_norm;
    int32_t *material;
    uint8_t *active;
    int32_t *next_active_time;
    int32_t *global_time;                /* scalar, ticks of DT_MIN1 */
    int32_t *dt;                         /* scalar, ticks */
    uint32_t *cell_key, *cell_index;     /* n: the sorted (key, particle) pairs */
    uint32_t *cell_start, *cell_end;     /* 2^(3*CELL_POWER) each */
    const float *eos_forsterite, *eos_fe;/* res*res*2 (pressure, sound speed) */
    int32_t eos_res;
    const int32_t *tree;                 /* flattened octree, reference format */
    int32_t tree_len;
    const int32_t *level_offsets;        /* n_levels+1 prefix into level_nodes */
    const int32_t *level_nodes;          /* node offsets into tree, per level */
    int32_t n_levels, n_nodes;
    int32_t max_unchecked;               /* unchecked-list capacity per node (1024) */
} ora_state;

/* Passes, in the reference's dispatch order (Headless.cpp:43-51). */
void ora_sort(ora_state *st);
void ora_gravity(ora_state *st);
void ora_density(ora_state *st);
void ora_acceleration(ora_state *st);
void ora_step(ora_state *st);

/* Octree builders.  Output is the reference's flattened format
 * (octree.cpp:24-109): leaf [n, dataPtr, p0..], branch [0, dataPtr, c0..c7]. */
typedef struct ora_tree ora_tree;
ora_tree *ora_tree_build_reference(int n, const float *pos3, int max_leaf, int max_depth);
ora_tree *ora_tree_build_morton(int n, const float *pos3, int max_leaf, int max_depth);
void ora_tree_sizes(const ora_tree *t, int32_t *tree_len, int32_t *n_levels, int32_t *n_nodes);
void ora_tree_export(const ora_tree *t, int32_t *tree, int32_t *level_offsets, int32_t *level_nodes);
void ora_tree_free(ora_tree *t);

/* Node records of the last ora_gravity call, in the CUDA library's layout
 * (24 floats per multipole, 16 per local, by data pointer); returns the node count. */
int ora_last_tree_nodes(float *poles, float *locals, int n_nodes);

/* ANEOS text table -> res*res (pressure, sound speed) grid, ANEOS.cpp:21-175.
 * Returns 0 on success, -1 if the file cannot be opened, -2 on short data. */
int ora_aneos_load(const char *path, int res, float *out);

/* Morton cell key of one position (sort.metal:15-44), exposed for tests. */
uint32_t ora_cell_key(float x, float y, float z);

/* FP64 direct-sum gravity at nt target particles: out[4 t] = (ax, ay, az, phi),
 * G included, exact cubic-spline softening (no reference counterpart). */
void ora_gravity_direct_f64(int n, const float *pos3, const float *mass, const int32_t *targets, int nt,
                            double *out);

/* An all-FP64 run of the step (fp64.cpp): FP64 direct-sum gravity, then the
 * reference's density, acceleration and step passes in double (no
 * counterpart in the reference; the yardstick of the mixed-precision form). */
typedef struct {
    int32_t n;
    double *pos, *vel, *acc;             /* 3n each */
    double *rho, *u, *mass, *pressure, *h, *grad_term, *sound_speed, *du, *balsara, *dhdt;
    int32_t *material, *next_active_time;
    int32_t *global_time, *dt;           /* scalars, ticks of DT_MIN1 */
    double *time_s;                      /* scalar, seconds */
    const float *eos_forsterite, *eos_fe;
    int32_t eos_res;
} ora_f64;
void ora_f64_steps(ora_f64 *st, int n_steps);
/* kinetic, internal, potential (exact softening), total energy */
void ora_f64_energy(const ora_f64 *st, double *out);

/* Threads used by the OpenMP loops (0 = library default). */
void ora_set_threads(int n);
int ora_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif

// ref_driver.cpp -- host dispatcher for the reference's own kernels.
//
// TEST INFRASTRUCTURE ONLY.  oracle/ref_build.sh compiles the reference's
// Metal kernels (SPH/Shaders/*.metal, through oracle/ref_shim), its CPU
// octree (SPH/octree/octree.cpp) and its ANEOS loader (SPH/ANEOS/ANEOS.cpp)
// unchanged, straight from the reference tree, and links them with this file
// into oracle/_ref/libref.so.  This file restates only the dispatch order of
// SPH/Compute/Compute.cpp:179-376 (one OpenMP loop per Metal dispatch, one
// loop per encoder in encoder order) over the same ora_state buffers that the
// oracle restatement uses, so the two can be compared value for value.

#include <metal_stdlib>
#include <simd/simd.h>

#include <string>
#include <vector>

#include "oracle.h"
#include "poles.h"  // reference: SPH/Shaders/gravity/poles/poles.h (Multipole, Local)

using metal::atomic_int;
using metal::atomic_uint;
using metal::float3;
using metal::uint2;
typedef metal::texture2d<float, metal::access::sample> tex2d;

// ---- kernel entry points of the reference (compiled from its .metal files) --
void hash(float3 *, float *, int *, uint2 *, uint);
void hist(uint2 *, uint *, uint *, uint *, const int *, uint);
void scan(uint2 *, uint *, uint *, uint *, uint *, const int *, uint);
void sum(uint *, uint *, uint);
void sort(uint2 *, uint2 *, uint *, uint *, uint *, uint *, uint);
void initialise(uint *, uint *, uint);
void findCellPositions(uint2 *, atomic_uint *, atomic_uint *, uint);
void upPass(float3 *, float *, int *, Multipole *, Local *, int *, uint *, float *, bool *, int *, int *, uint);
void downPass(float3 *, float3 *, float *, int *, Multipole *, Local *, int *, uint *, int *, int *, float *, bool *,
              uint);
void density(float3 *, float3 *, float *, float *, float *, float *, float *, int *, float *, float *, float *, uint2 *,
             int *, int *, float *, int *, bool *, int *, tex2d, tex2d, uint);
void acceleration(float3 *, float3 *, float3 *, float *, float *, float *, float *, float *, float *, float *, float *,
                  float *, float *, uint2 *, int *, int *, float *, int *, bool *, int *, int *, atomic_int *, uint);
void step(float3 *, float3 *, float3 *, float *, float *, float *, float *, float *, bool *, int *, int *, int *, uint);
void drawToSnapshot(float3 *, int *, atomic_int *, uint);  // render.metal:49-66

// ---- reference host routines (octree.cpp, ANEOS.cpp) ------------------------
#include <vector>
void buildOctree(const simd_float3 *positions, int positionCount, std::vector<int> &octreeData,
                 std::vector<std::vector<int>> &treeLevels, int &nodeValues, int maxLeafSize);
struct ANEOSTable {  // reference: SPH/ANEOS/ANEOS.hpp:16-29
    int resolution;
    float *rho;
    float *u;
    simd_float2 *data;
    float minRho, maxRho, minU, maxU;
};
ANEOSTable loadANEOSDataFromFile(const std::string &filePath, const int resolution);
namespace MTL {
struct CommandQueue;
struct Texture;
}  // namespace MTL
void copyDataToTexture(MTL::CommandQueue *, MTL::Texture *, MTL::Texture *) {}

namespace {

const int kCellsPerDim = 256;
const float kCellSize = 0.18f;
const size_t kCells = (size_t)1 << 24;

std::vector<float3> to3(const float *a, int n) {
    std::vector<float3> v(n);
    for (int i = 0; i < n; ++i) v[i] = float3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
    return v;
}
void from3(const std::vector<float3> &v, float *a) {
    for (size_t i = 0; i < v.size(); ++i) {
        a[3 * i] = v[i].x;
        a[3 * i + 1] = v[i].y;
        a[3 * i + 2] = v[i].z;
    }
}
// the reference's `bool*` buffers are 1 byte per particle, like uint8_t
bool *as_bool(uint8_t *p) { return reinterpret_cast<bool *>(p); }

std::vector<uint2> sorted_pairs(const ora_state *st) {
    std::vector<uint2> cd(st->n);
    for (int i = 0; i < st->n; ++i) cd[i] = uint2(st->cell_key[i], st->cell_index[i]);
    return cd;
}

}  // namespace

extern "C" {

// Compute.cpp:265-326
void ref_sort(ora_state *st) {
    const int n = st->n;
    const int nBlocks = n / 256 + 1;  // Compute.cpp:93
    std::vector<float3> pos = to3(st->pos, n);
    std::vector<uint2> ci(n), cj(n);
    std::vector<uint> bucketHist((size_t)nBlocks * 256), bucketOffset(256), particleOffset(n);
    float cellSize = kCellSize;
    int cellsPerDim = kCellsPerDim;
#pragma omp parallel for
    for (int i = 0; i < n; ++i) hash(pos.data(), &cellSize, &cellsPerDim, ci.data(), (uint)i);
    for (uint it = 0; it < 4; ++it) {
        uint2 *src = (it % 2 == 0) ? ci.data() : cj.data();
        uint2 *dst = (it % 2 == 0) ? cj.data() : ci.data();
        uint ittr = it;
#pragma omp parallel for
        for (int b = 0; b < nBlocks; ++b)
            hist(src, bucketHist.data(), particleOffset.data(), &ittr, &n, (uint)b);
#pragma omp parallel for
        for (int b = 0; b < 256; ++b)
            scan(src, bucketHist.data(), bucketOffset.data(), particleOffset.data(), &ittr, &nBlocks, (uint)b);
        sum(bucketHist.data(), bucketOffset.data(), 0u);
#pragma omp parallel for
        for (int i = 0; i < n; ++i)
            sort(src, dst, bucketHist.data(), bucketOffset.data(), particleOffset.data(), &ittr, (uint)i);
    }
#pragma omp parallel for
    for (long c = 0; c < (long)kCells; ++c) initialise(st->cell_start, st->cell_end, (uint)c);
#pragma omp parallel for
    for (int i = 0; i < n; ++i)
        findCellPositions(ci.data(), reinterpret_cast<atomic_uint *>(st->cell_start),
                          reinterpret_cast<atomic_uint *>(st->cell_end), (uint)i);
    for (int i = 0; i < n; ++i) {
        st->cell_key[i] = ci[i].x;
        st->cell_index[i] = ci[i].y;
    }
}

// Compute.cpp:328-377 (+ the list sizing of updateOctreeBuffer, :484-502)
void ref_gravity(ora_state *st) {
    const int n = st->n;
    if (st->n_levels <= 0) return;
    std::vector<float3> pos = to3(st->pos, n), acc = to3(st->acc, n);
    std::vector<Multipole> mp(st->n_nodes);
    std::vector<Local> lc(st->n_nodes);
    std::vector<uint> parent(st->n_nodes, 0u);
    std::vector<int> tree(st->tree, st->tree + st->tree_len);
    const int L = st->n_levels;
    long maxSize = 0;
    std::vector<std::vector<int>> levels(L);
    for (int l = 0; l < L; ++l) {
        levels[l].assign(st->level_nodes + st->level_offsets[l], st->level_nodes + st->level_offsets[l + 1]);
        if (l != L - 1) maxSize = std::max(maxSize, (long)levels[l].size());
    }
    const size_t cap = 1024;  // MAX_UNCHECKED_POINTERS
    std::vector<int> gi(std::max<long>(maxSize, 1) * cap + 2, -1), gj(std::max<long>(maxSize, 1) * cap + 2, -1);
    for (int l = L - 1; l >= 0; --l) {
        const int cnt = (int)levels[l].size();
#pragma omp parallel for schedule(dynamic, 16)
        for (int t = 0; t < cnt; ++t)
            upPass(pos.data(), st->mass, tree.data(), mp.data(), lc.data(), levels[l].data(), parent.data(),
                   st->grav_norm, as_bool(st->active), st->next_active_time, st->global_time, (uint)t);
    }
    if (tree[0] == 0) {
        for (int l = 0; l < L; ++l) {
            const int cnt = (int)levels[l].size();
            int *in = (l % 2 == 0) ? gi.data() : gj.data();
            int *out = (l % 2 == 0) ? gj.data() : gi.data();
#pragma omp parallel for schedule(dynamic, 4)
            for (int t = 0; t < cnt; ++t)
                downPass(pos.data(), acc.data(), st->mass, tree.data(), mp.data(), lc.data(), levels[l].data(),
                         parent.data(), in, out, st->grav_norm, as_bool(st->active), (uint)t);
        }
    }
    from3(acc, st->acc);
}

// Compute.cpp:179-208
void ref_density(ora_state *st) {
    const int n = st->n;
    std::vector<float3> pos = to3(st->pos, n), vel = to3(st->vel, n);
    std::vector<uint2> cd = sorted_pairs(st);
    float cellSize = kCellSize;
    int cellsPerDim = kCellsPerDim;
    tex2d tf{st->eos_forsterite, st->eos_res, st->eos_res};
    tex2d te{st->eos_fe, st->eos_res, st->eos_res};
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i)
        density(pos.data(), vel.data(), st->rho, st->u, st->mass, st->pressure, st->h, st->material, st->grad_term,
                st->sound_speed, st->balsara, cd.data(), reinterpret_cast<int *>(st->cell_start),
                reinterpret_cast<int *>(st->cell_end), &cellSize, &cellsPerDim, as_bool(st->active), st->dt, tf, te,
                (uint)i);
}

// Compute.cpp:210-240
void ref_acceleration(ora_state *st) {
    const int n = st->n;
    std::vector<float3> pos = to3(st->pos, n), vel = to3(st->vel, n), acc = to3(st->acc, n);
    std::vector<uint2> cd = sorted_pairs(st);
    float cellSize = kCellSize;
    int cellsPerDim = kCellsPerDim;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i)
        acceleration(pos.data(), vel.data(), acc.data(), st->rho, st->u, st->mass, st->pressure, st->h,
                     st->grad_term, st->sound_speed, st->du, st->balsara, st->dhdt, cd.data(),
                     reinterpret_cast<int *>(st->cell_start), reinterpret_cast<int *>(st->cell_end), &cellSize,
                     &cellsPerDim, as_bool(st->active), st->next_active_time, st->global_time,
                     reinterpret_cast<atomic_int *>(st->dt), (uint)i);
    from3(acc, st->acc);
}

// Compute.cpp:242-263.  Thread 0 advances the global time while the others
// only read dt; the dispatch is otherwise element-wise.
void ref_step(ora_state *st) {
    const int n = st->n;
    std::vector<float3> pos = to3(st->pos, n), vel = to3(st->vel, n), acc = to3(st->acc, n);
    step(pos.data(), vel.data(), acc.data(), st->rho, st->u, st->du, st->dhdt, st->h, as_bool(st->active),
         st->next_active_time, st->global_time, st->dt, 0u);
#pragma omp parallel for
    for (int i = 1; i < n; ++i)
        step(pos.data(), vel.data(), acc.data(), st->rho, st->u, st->du, st->dhdt, st->h, as_bool(st->active),
             st->next_active_time, st->global_time, st->dt, (uint)i);
    from3(pos, st->pos);
    from3(vel, st->vel);
}

// octree.cpp:111-141 (buildOctree) on the given positions; depth cap is the
// compiled-in MAX_TREE_DEPTH (7).
struct ref_tree {
    std::vector<int> data;
    std::vector<std::vector<int>> levels;
    int nodes = 0;
};
ref_tree *ref_tree_build(int n, const float *pos3, int max_leaf) {
    std::vector<simd_float3> p(n);
    for (int i = 0; i < n; ++i) p[i] = simd_float3(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]);
    ref_tree *t = new ref_tree();
    buildOctree(p.data(), n, t->data, t->levels, t->nodes, max_leaf);
    return t;
}
void ref_tree_sizes(const ref_tree *t, int32_t *len, int32_t *nl, int32_t *nn) {
    *len = (int32_t)t->data.size();
    *nl = (int32_t)t->levels.size();
    *nn = t->nodes;
}
void ref_tree_export(const ref_tree *t, int32_t *tree, int32_t *off, int32_t *nodes) {
    for (size_t i = 0; i < t->data.size(); ++i) tree[i] = t->data[i];
    int32_t o = 0;
    for (size_t l = 0; l < t->levels.size(); ++l) {
        off[l] = o;
        for (int v : t->levels[l]) nodes[o++] = v;
    }
    off[t->levels.size()] = o;
}
void ref_tree_free(ref_tree *t) { delete t; }

// Compute::drawSnapshot (Compute.cpp:395-412): clear the image, then the
// reference's drawToSnapshot kernel for every particle
void ref_draw_snapshot(int n, const float *pos3, const int *mat, int *img) {
    std::vector<float3> p = to3(pos3, n);
    std::vector<int> m(mat, mat + n);
    for (size_t i = 0; i < (size_t)1024 * 1024; ++i) img[i] = 0;
    atomic_int *out = reinterpret_cast<atomic_int *>(img);
    for (int i = 0; i < n; ++i) drawToSnapshot(p.data(), m.data(), out, (uint)i);
}

// ANEOS.cpp:21-175
int ref_aneos_load(const char *path, int res, float *out) {
    try {
        ANEOSTable t = loadANEOSDataFromFile(path, res);
        for (size_t i = 0; i < (size_t)res * res; ++i) {
            out[2 * i] = t.data[i].x;
            out[2 * i + 1] = t.data[i].y;
        }
        delete[] t.rho;
        delete[] t.u;
        delete[] t.data;
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"

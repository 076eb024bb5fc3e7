// sph_tree.cu -- the octree build, moved from the reference's detached CPU
// thread (SPH/octree/octree.cpp:14-141 via Compute::updateOctreeData,
// Compute.cpp:510-516) onto the GPU.
//
// Tree definition (restated on the CPU by the oracle's ora_tree_build_morton):
//   * keys: each coordinate quantised to D = max_tree_depth bits over the
//     bounding cube (side = largest extent), interleaved with x on bit 0 of
//     each triplet (the reference's morton3D convention);
//   * particles stable-sorted by key (one-sweep radix sort, ties by index);
//   * a node is a leaf if it holds <= max_children_in_leaf particles or sits
//     at depth D; otherwise its children are the non-empty octants of the next
//     key triplet (octant bit x = 1, y = 2, z = 4, the reference's order);
//   * flattened in DFS preorder in the reference's int format
//     (leaf [n, dataPtr, ids...], branch [0, dataPtr, 8 child offsets or -1]),
//     with per-level node lists in DFS order, so the same up/down passes run
//     on it.  The split is geometric (cube midpoints) instead of the
//     reference's per-subset mean.
//
// Build: bounding box -> keys (+ digit histograms) -> sort -> per level, each
// branch finds its 8 octant ranges by binary search and a scan compacts the
// children into the next level -> every node adds its size at its first
// particle -> two scans give DFS offsets and data pointers -> nodes write
// themselves and link into their parents.  Every launch size is a host-side
// upper bound and the true counts stay on the device, so the whole build can
// be captured in a CUDA graph.
#include <cuda_runtime.h>

#include "sph_internal.h"

namespace sph {

void tree_bounds(int n, int leafcap, int depth, int64_t &nodes, int64_t &ints, int64_t &branches);

namespace {

__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_bbox_init(uint32_t *bb) {
    if (threadIdx.x < 3) bb[threadIdx.x] = 0xffffffffu;
    else if (threadIdx.x < 6) bb[threadIdx.x] = 0u;
}

__global__ void k_bbox(const float4 *__restrict__ pos4, int n, uint32_t *bb) {
    float lo[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float hi[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 p = pos4[i];
        lo[0] = fminf(lo[0], p.x);
        lo[1] = fminf(lo[1], p.y);
        lo[2] = fminf(lo[2], p.z);
        hi[0] = fmaxf(hi[0], p.x);
        hi[1] = fmaxf(hi[1], p.y);
        hi[2] = fmaxf(hi[2], p.z);
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(bb + a, f2ord(lo[a]));
            atomicMax(bb + 3 + a, f2ord(hi[a]));
        }
    }
}

__global__ void k_tree_keys(const float4 *__restrict__ pos4, int n, int depth, const uint32_t *__restrict__ bb,
                            uint32_t *__restrict__ keys, uint32_t *__restrict__ vals, uint32_t *__restrict__ hist,
                            int passes) {
    __shared__ uint32_t sh[RadixSorter::kMaxPasses][256];
    for (int i = threadIdx.x; i < RadixSorter::kMaxPasses * 256; i += blockDim.x) (&sh[0][0])[i] = 0u;
    __syncthreads();
    const float lx = ord2f(bb[0]), ly = ord2f(bb[1]), lz = ord2f(bb[2]);
    const float hx = ord2f(bb[3]), hy = ord2f(bb[4]), hz = ord2f(bb[5]);
    float span = fmaxf(hx - lx, fmaxf(hy - ly, hz - lz));
    if (!(span > 0.f)) span = 1.f;
    const int cells = 1 << depth;
    const float scale = __fdiv_rn((float)cells, span);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 p = pos4[i];
        int qx = (int)__fmul_rn(__fsub_rn(p.x, lx), scale);
        int qy = (int)__fmul_rn(__fsub_rn(p.y, ly), scale);
        int qz = (int)__fmul_rn(__fsub_rn(p.z, lz), scale);
        qx = min(max(qx, 0), cells - 1);
        qy = min(max(qy, 0), cells - 1);
        qz = min(max(qz, 0), cells - 1);
        uint32_t k = morton3((uint32_t)qx, (uint32_t)qy, (uint32_t)qz);
        keys[i] = k;
        vals[i] = (uint32_t)i;
        for (int q = 0; q < passes; ++q) atomicAdd(&sh[q][(k >> (8 * q)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
        uint32_t v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

struct LevelArgs {
    int32_t *nstart, *ncount, *nparent, *nrank, *noffset;
    int32_t *level_count;  // Tree::level_count
    int32_t *scan_n;       // [16] 8 * level count
    int64_t level_cap;
    int64_t *cand;         // [8 * level_cap + 1]
    int64_t *cand_scan;
    int32_t *cstart;       // [8 * level_cap]
    const uint32_t *keys;  // sorted tree keys
    int depth, leafcap, n;
};

__global__ void k_root(LevelArgs a) {
    a.nstart[0] = 0;
    a.ncount[0] = a.n;
    a.nparent[0] = -1;
    a.level_count[0] = 1;
    for (int l = 1; l < 16; ++l) a.level_count[l] = 0;
}

// first index in [lo, hi) whose octant digit (key >> shift & 7) is >= o
__device__ __forceinline__ int digit_lower_bound(const uint32_t *keys, int lo, int hi, int shift, uint32_t o) {
    while (lo < hi) {
        int mid = lo + ((hi - lo) >> 1);
        if (((keys[mid] >> shift) & 7u) < o)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_children(LevelArgs a, int l) {
    const int cnt = a.level_count[l];
    if (blockIdx.x == 0 && threadIdx.x == 0) a.scan_n[l] = 8 * cnt;
    const int32_t *ns = a.nstart + (size_t)l * a.level_cap, *nc = a.ncount + (size_t)l * a.level_cap;
    const int shift = 3 * (a.depth - l - 1);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int s = ns[t], c = nc[t];
        const bool branch = c > a.leafcap;
        int b = s;
        for (int o = 0; o < 8; ++o) {
            int e = branch ? ((o == 7) ? s + c : digit_lower_bound(a.keys, b, s + c, shift, (uint32_t)o + 1u)) : b;
            const int64_t nonempty = (e > b) ? 1 : 0;
            const int64_t brf = (o == 0 && branch) ? 1 : 0;
            a.cand[(size_t)t * 8 + o] = nonempty | (brf << 32);
            a.cstart[(size_t)t * 8 + o] = b;
            b = e;
        }
    }
}

__global__ void k_emit(LevelArgs a, int l) {
    const int cnt = a.level_count[l];
    const int64_t *sc = a.cand_scan;
    const int32_t *nc = a.ncount + (size_t)l * a.level_cap;
    int32_t *rank = a.nrank + (size_t)l * a.level_cap;
    const size_t nb = (size_t)(l + 1) * a.level_cap;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int64_t first = sc[(size_t)t * 8];
        rank[t] = (nc[t] > a.leafcap) ? (int32_t)(first >> 32) : -1;
        for (int o = 0; o < 8; ++o) {
            const size_t q = (size_t)t * 8 + o;
            const int64_t v = a.cand[q];
            if ((v & 0xffffffffll) == 0) continue;
            const int pos = (int)(sc[q] & 0xffffffffll);
            const int s = a.cstart[q];
            const int e = (o == 7) ? (a.cstart[(size_t)t * 8] + nc[t]) : a.cstart[q + 1];
            a.nstart[nb + pos] = s;
            a.ncount[nb + pos] = e - s;
            a.nparent[nb + pos] = t | (o << 28);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.level_count[l + 1] = (int32_t)(sc[(size_t)cnt * 8] & 0xffffffffll);
}

// leaf-level nodes get rank -1 (no list)
__global__ void k_rank_leaves(LevelArgs a, int l) {
    const int cnt = a.level_count[l];
    int32_t *rank = a.nrank + (size_t)l * a.level_cap;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) rank[t] = -1;
}

struct LayoutArgs {
    const int32_t *nstart, *ncount, *nparent, *nrank;
    int32_t *noffset;
    const int32_t *level_count;
    int64_t level_cap;
    int64_t *ints_at, *nodes_at;  // per particle (n + 1)
    int32_t *first_level;
    const int64_t *ints_off, *dp_off;
    int32_t *tree, *level_nodes, *list_slot;
    int2 *node_range;  // by data pointer: (first particle in key order, count)
    const uint32_t *order;
    int depth, leafcap, n;
    int64_t tree_cap, node_cap;
    uint32_t *health;
    int32_t *meta;
};

__global__ void k_layout_reset(LayoutArgs a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= a.n; i += gridDim.x * blockDim.x) {
        a.ints_at[i] = 0;
        a.nodes_at[i] = 0;
        a.first_level[i] = 0x7fffffff;
    }
}

__device__ __forceinline__ bool is_branch(const LayoutArgs &a, int l, int count) {
    return l < a.depth && count > a.leafcap;
}

__global__ void k_marks(LayoutArgs a, int l) {
    const int cnt = a.level_count[l];
    const int32_t *ns = a.nstart + (size_t)l * a.level_cap, *nc = a.ncount + (size_t)l * a.level_cap;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int s = ns[t], c = nc[t];
        const int size = is_branch(a, l, c) ? 10 : 2 + c;
        atomicAdd((unsigned long long *)(a.ints_at + s), (unsigned long long)size);
        atomicAdd((unsigned long long *)(a.nodes_at + s), 1ull);
        atomicMin(a.first_level + s, l);
    }
}

__global__ void k_write(LayoutArgs a, int l) {
    const int cnt = a.level_count[l];
    const size_t base = (size_t)l * a.level_cap;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int s = a.nstart[base + t], c = a.ncount[base + t];
        const int d = l - a.first_level[s];
        const int64_t off = a.ints_off[s] + 10 * (int64_t)d;
        const int64_t dp = a.dp_off[s] + d;
        const bool br = is_branch(a, l, c);
        if (off + (br ? 10 : 2 + c) > a.tree_cap || dp >= a.node_cap) {
            raise_health(a.health, SPH_HEALTH_TREE_CAPACITY);
            a.noffset[base + t] = 0;
            continue;
        }
        a.noffset[base + t] = (int32_t)off;
        a.level_nodes[base + t] = (int32_t)off;
        int32_t *T = a.tree + off;
        T[0] = br ? 0 : c;
        T[1] = (int32_t)dp;
        if (br) {
            for (int k = 0; k < 8; ++k) T[2 + k] = -1;
        } else {
            for (int k = 0; k < c; ++k) T[2 + k] = (int32_t)a.order[s + k];
        }
        a.list_slot[dp] = br ? a.nrank[base + t] : -1;
        a.node_range[dp] = make_int2(s, c);
    }
    if (l == 0 && blockIdx.x == 0 && threadIdx.x == 0) {
        a.meta[1] = (int32_t)a.dp_off[a.n];
        a.meta[2] = (int32_t)a.ints_off[a.n];
    }
}

__global__ void k_link(LayoutArgs a, int l) {
    // l >= 1: every node writes its offset into its parent's child slot
    const int cnt = a.level_count[l];
    const size_t base = (size_t)l * a.level_cap, pbase = (size_t)(l - 1) * a.level_cap;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int pr = a.nparent[base + t];
        const int pt = pr & 0x0fffffff, o = (pr >> 28) & 7;
        const int32_t poff = a.noffset[pbase + pt];
        a.tree[poff + 2 + o] = a.noffset[base + t];
    }
}

inline int grid_for(int64_t bound, int threads = 256) {
    int64_t b = (bound + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return (int)b;
}

}  // namespace

sph_status tree_alloc(sph_ctx *ctx) {
    TreeBuild &tb = ctx->tb;
    if (tb.nstart) return SPH_OK;
    const int n = ctx->n;
    const int D = ctx->params.max_tree_depth;
    const int64_t cap = ctx->tree.level_cap;  // n
    const int levels = D + 1;
    sph_status s = sort_alloc(tb.sorter, n);
    if (s != SPH_OK) return s;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    chk(cudaMalloc(&tb.nstart, sizeof(int32_t) * levels * cap));
    chk(cudaMalloc(&tb.ncount, sizeof(int32_t) * levels * cap));
    chk(cudaMalloc(&tb.nparent, sizeof(int32_t) * levels * cap));
    chk(cudaMalloc(&tb.noffset, sizeof(int32_t) * levels * cap));
    chk(cudaMalloc(&tb.ndp, sizeof(int32_t) * levels * cap));  // branch ranks per level
    tb.scan_cap = 8 * cap + 1;
    chk(cudaMalloc(&tb.scan, sizeof(int64_t) * 2 * tb.scan_cap));
    chk(cudaMalloc(&tb.scan_blocks, sizeof(int64_t) * (tb.scan_cap / 2048 + 16)));
    chk(cudaMalloc(&tb.per_particle, sizeof(int32_t) * 8 * (cap + 1)));  // cstart: 8 per node slot
    chk(cudaMalloc(&tb.bbox, sizeof(uint32_t) * 8 + sizeof(int32_t) * 16));
    return cuda_status(e, "tree_alloc");
}

void tree_free(sph_ctx *ctx) {
    TreeBuild &tb = ctx->tb;
    sort_free(tb.sorter);
    cudaFree(tb.nstart);
    cudaFree(tb.ncount);
    cudaFree(tb.nparent);
    cudaFree(tb.noffset);
    cudaFree(tb.ndp);
    cudaFree(tb.scan);
    cudaFree(tb.scan_blocks);
    cudaFree(tb.per_particle);
    cudaFree(tb.bbox);
    cudaFree(tb.walk_queues);
    cudaFree(tb.walk_counter);
    tb = TreeBuild();
}

sph_status launch_tree_build(sph_ctx *ctx, cudaStream_t st) {
    sph_status s = tree_alloc(ctx);
    if (s != SPH_OK) return s;
    TreeBuild &tb = ctx->tb;
    Tree &tr = ctx->tree;
    const int n = ctx->n;
    const int D = ctx->params.max_tree_depth;
    const int leafcap = ctx->params.max_children_in_leaf;
    const int64_t cap = tr.level_cap;
    const int bits = 3 * D;
    const int passes = (bits + 7) / 8;
    uint32_t *bb = (uint32_t *)tb.bbox;
    int32_t *scan_n = (int32_t *)(bb + 8);

    k_bbox_init<<<1, 32, 0, st>>>(bb);
    k_bbox<<<grid_for(n), 256, 0, st>>>(ctx->pos4, n, bb);
    cudaMemsetAsync(tb.sorter.hist, 0, sizeof(uint32_t) * 256 * RadixSorter::kMaxPasses, st);
    k_tree_keys<<<grid_for(n), 256, 0, st>>>(ctx->pos4, n, D, bb, tb.sorter.keys[0], tb.sorter.vals[0],
                                              tb.sorter.hist, passes);
    const int fin = radix_sort_pairs(tb.sorter, n, bits, st, ctx->health);
    const uint32_t *keys = tb.sorter.keys[fin];
    const uint32_t *order = tb.sorter.vals[fin];

    LevelArgs la;
    la.nstart = tb.nstart;
    la.ncount = tb.ncount;
    la.nparent = tb.nparent;
    la.nrank = tb.ndp;
    la.noffset = tb.noffset;
    la.level_count = tr.level_count;
    la.scan_n = scan_n;
    la.level_cap = cap;
    la.cand = tb.scan;
    la.cand_scan = tb.scan + tb.scan_cap;
    la.cstart = tb.per_particle;
    la.keys = keys;
    la.depth = D;
    la.leafcap = leafcap;
    la.n = n;
    k_root<<<1, 1, 0, st>>>(la);
    int64_t bound = 1;
    for (int l = 0; l < D; ++l) {
        k_children<<<grid_for(bound), 256, 0, st>>>(la, l);
        scan_exclusive_i64(la.cand, la.cand_scan, tb.scan_blocks, (int)std::min<int64_t>(8 * bound, 8 * cap),
                           scan_n + l, st);
        k_emit<<<grid_for(bound), 256, 0, st>>>(la, l);
        bound = std::min<int64_t>(bound * 8, cap);
    }
    k_rank_leaves<<<grid_for(bound), 256, 0, st>>>(la, D);

    // DFS layout: per-particle size sums, then offsets
    int64_t *ints_at = tb.scan, *nodes_at = tb.scan + (n + 1);
    int64_t *ints_off = tb.scan + tb.scan_cap, *dp_off = tb.scan + tb.scan_cap + (n + 1);
    int32_t *first_level = tb.per_particle;  // cstart no longer needed
    LayoutArgs ya;
    ya.nstart = tb.nstart;
    ya.ncount = tb.ncount;
    ya.nparent = tb.nparent;
    ya.nrank = tb.ndp;
    ya.noffset = tb.noffset;
    ya.level_count = tr.level_count;
    ya.level_cap = cap;
    ya.ints_at = ints_at;
    ya.nodes_at = nodes_at;
    ya.first_level = first_level;
    ya.ints_off = ints_off;
    ya.dp_off = dp_off;
    ya.tree = tr.tree;
    ya.level_nodes = tr.level_nodes;
    ya.list_slot = tr.list_slot;
    ya.order = order;
    ya.depth = D;
    ya.leafcap = leafcap;
    ya.n = n;
    ya.tree_cap = tr.tree_cap;
    ya.node_cap = tr.node_cap;
    ya.health = ctx->health;
    ya.meta = tr.meta;
    ya.node_range = tr.node_range;
    tb.order = order;
    k_layout_reset<<<grid_for(n + 1), 256, 0, st>>>(ya);
    int64_t lb[16];
    bound = 1;
    for (int l = 0; l <= D; ++l) {
        lb[l] = bound;
        k_marks<<<grid_for(bound), 256, 0, st>>>(ya, l);
        bound = std::min<int64_t>(bound * 8, cap);
    }
    scan_exclusive_i64(ints_at, ints_off, tb.scan_blocks, n, nullptr, st);
    scan_exclusive_i64(nodes_at, dp_off, tb.scan_blocks, n, nullptr, st);
    for (int l = 0; l <= D; ++l) k_write<<<grid_for(lb[l]), 256, 0, st>>>(ya, l);
    for (int l = 1; l <= D; ++l) k_link<<<grid_for(lb[l]), 256, 0, st>>>(ya, l);

    tr.n_levels_host = D + 1;
    for (int l = 0; l < 16; ++l) tr.level_count_host[l] = (l <= D) ? (int)lb[l] : 0;
    tr.valid = true;
    return cuda_status(cudaGetLastError(), "tree build");
}

}  // namespace sph

extern "C" sph_status sph_selftest_tree_capacity(sph_ctx *ctx, void *stream) {
    using namespace sph;
    if (!ctx || ctx->params.tree_source != SPH_TREE_GPU) {
        set_error("sph_selftest_tree_capacity: needs a context with the GPU tree");
        return SPH_ERR_INVALID_ARG;
    }
    cudaSetDevice(ctx->device);
    const int64_t cap = ctx->tree.tree_cap;
    ctx->tree.tree_cap = 16;  // room for one branch record at most
    const sph_status s = launch_tree_build(ctx, (cudaStream_t)stream);
    ctx->tree.tree_cap = cap;
    ctx->tree.valid = false;  // the next tree build replaces the partial one
    return s;
}

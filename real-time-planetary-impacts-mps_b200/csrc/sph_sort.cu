// sph_sort.cu -- Compute::sort (SPH/Compute/Compute.cpp:265-326) for sm_100a.
//
// The reference hashes every particle to a 24-bit Morton cell key
// (sort.metal:15-44), sorts (key, index) pairs with four stable 8-bit LSD
// passes of hist/scan/sum/scatter dispatches (sort.metal:46-129), then
// re-initialises all 2^24 cell entries and finds each cell's first and last
// sorted index with atomics (sort.metal:131-148).
//
// Here:
//  * k_hash_hist computes the keys and, in the same sweep, the global digit
//    histograms of all passes (the one-sweep "upsweep"); it also clears only
//    the cell entries the previous sort filled, instead of all 2^24;
//  * k_onesweep does one stable 8-bit pass per launch: warp-level ranking
//    with match_any, a decoupled look-back across tiles for each digit (every
//    wait is bounded and raises a health bit instead of hanging), scatter;
//    the top byte of the 24-bit keys is always zero, so three passes give the
//    reference's four-pass order exactly;
//  * k_cells writes each occupied cell's (first, last) sorted index from
//    neighbouring keys, without atomics.
#include <cuda_runtime.h>

#include <cstdio>

#include "sph_internal.h"

namespace sph {

namespace {

constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1u;
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Keys of the cell grid + all three digit histograms; clears the previous
// sort's occupied cells first (they are read from the previous sorted keys,
// which live in the buffer the first pass is about to overwrite).
__global__ void k_hash_hist(const float4 *__restrict__ pos4, int n, uint32_t *__restrict__ keys,
                            uint32_t *__restrict__ vals, uint32_t *__restrict__ hist,
                            const uint32_t *__restrict__ prev_keys, uint2 *__restrict__ cell_range, int clear_prev) {
    __shared__ uint32_t sh[3][256];
    for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) (&sh[0][0])[i] = 0u;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (clear_prev) {
            uint32_t pk = prev_keys[i];
            if (i == 0 || prev_keys[i - 1] != pk) cell_range[pk] = make_uint2(0xffffffffu, 0u);
        }
        float4 p = pos4[i];
        uint32_t k = cell_key(p.x, p.y, p.z);
        keys[i] = k;
        vals[i] = (uint32_t)i;
        atomicAdd(&sh[0][k & 255u], 1u);
        atomicAdd(&sh[1][(k >> 8) & 255u], 1u);
        atomicAdd(&sh[2][(k >> 16) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) {
        uint32_t v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// One stable 8-bit LSD pass.
__global__ void __launch_bounds__(RadixSorter::kThreads)
    k_onesweep(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
               uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out, int n, int shift,
               const uint32_t *__restrict__ hist, uint32_t *status, uint32_t *counter, uint32_t *health,
               int spin_limit) {
    constexpr int T = RadixSorter::kThreads, I = RadixSorter::kItems, W = T / 32;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[W][256];
    __shared__ uint32_t s_base[256];
    __shared__ uint32_t s_scan[256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(counter, 1u);
    for (int i = tid; i < W * 256; i += T) (&s_warp[0][0])[i] = 0u;
    // exclusive prefix of the global histogram over digits (Hillis-Steele in smem)
    s_scan[tid] = hist[tid];
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        uint32_t v = (tid >= off) ? s_scan[tid - off] : 0u;
        __syncthreads();
        s_scan[tid] += v;
        __syncthreads();
    }
    const uint32_t global_excl = s_scan[tid] - hist[tid];
    const uint32_t tile = s_tile;
    const int64_t base = (int64_t)tile * RadixSorter::kTile + (int64_t)warp * (I * 32);
    const uint32_t lt = lanemask_lt();

    uint32_t k[I], v[I], rank[I];
#pragma unroll
    for (int it = 0; it < I; ++it) {
        int64_t idx = base + it * 32 + lane;
        bool ok = idx < n;
        k[it] = ok ? keys_in[idx] : 0u;
        v[it] = ok ? vals_in[idx] : 0u;
    }
#pragma unroll
    for (int it = 0; it < I; ++it) {
        int64_t idx = base + it * 32 + lane;
        bool ok = idx < n;
        uint32_t d = ok ? ((k[it] >> shift) & 255u) : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = ok ? s_warp[warp][d] : 0u;
        rank[it] = before + __popc(peers & lt);
        __syncwarp();
        if (ok && (peers & lt) == 0u) s_warp[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: offsets of the warps inside the tile, and the tile total
    uint32_t tile_count = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        uint32_t c = s_warp[w][tid];
        s_warp[w][tid] = tile_count;
        tile_count += c;
    }
    // decoupled look-back for digit `tid`
    uint32_t excl = 0;
    volatile uint32_t *vs = status;
    if (tile == 0) {
        vs[tid] = kFlagPrefix | tile_count;
    } else {
        vs[(size_t)tile * 256 + tid] = kFlagAgg | tile_count;
        int64_t j = (int64_t)tile - 1;
        int spins = 0;
        while (j >= 0) {
            uint32_t s = vs[(size_t)j * 256 + tid];
            uint32_t flag = s & ~kValueMask;
            if (flag == 0u) {
                if (++spins > spin_limit) {
                    raise_health(health, SPH_HEALTH_SORT_TIMEOUT);
                    break;
                }
                __nanosleep(64);
                continue;
            }
            excl += s & kValueMask;
            if (flag == kFlagPrefix) break;
            --j;
        }
        __threadfence();
        vs[(size_t)tile * 256 + tid] = kFlagPrefix | ((excl + tile_count) & kValueMask);
    }
    s_base[tid] = global_excl + excl;
    __syncthreads();
#pragma unroll
    for (int it = 0; it < I; ++it) {
        int64_t idx = base + it * 32 + lane;
        if (idx < n) {
            uint32_t d = (k[it] >> shift) & 255u;
            uint32_t dst = s_base[d] + s_warp[warp][d] + rank[it];
            if (dst < (uint32_t)n) {  // only a timed-out look-back can break this
                keys_out[dst] = k[it];
                vals_out[dst] = v[it];
            }
        }
    }
}

__global__ void k_cells(const uint32_t *__restrict__ keys, int n, uint2 *__restrict__ cell_range) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k = keys[i];
    if (i == 0 || keys[i - 1] != k) cell_range[k].x = (uint32_t)i;
    if (i == n - 1 || keys[i + 1] != k) cell_range[k].y = (uint32_t)i;
}

// The unit table: (first, last) sorted index of every occupied 64-cell unit
// (cell key >> 6); the table is cleared to 0xff bytes before.
__global__ void k_units(const uint32_t *__restrict__ keys, int n, uint2 *__restrict__ units) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t u = keys[i] >> (3 * kUnitShift);
    if (i == 0 || (keys[i - 1] >> (3 * kUnitShift)) != u) units[u].x = (uint32_t)i;
    if (i == n - 1 || (keys[i + 1] >> (3 * kUnitShift)) != u) units[u].y = (uint32_t)i;
}

__global__ void k_init_cells(uint2 *cell_range, uint32_t count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        cell_range[i] = make_uint2(0xffffffffu, 0u);
}

// ---- 64-bit exclusive scan (reduce, scan of block sums, apply) -------------
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t *total) {
    __shared__ int64_t warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int64_t s = (lane < kScanThreads / 32) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    int64_t prefix = (warp > 0) ? warp_sums[warp - 1] : 0;
    *total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return prefix + x - v;
}

__global__ void k_scan_reduce(const int64_t *__restrict__ in, int64_t *__restrict__ blocks, int n_max,
                              const int32_t *d_count) {
    const int n = d_count ? min(*d_count, n_max) : n_max;
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int64_t s = 0;
    for (int it = 0; it < kScanItems; ++it) {
        int64_t i = base + (int64_t)it * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    int64_t total;
    block_excl_scan(s, &total);
    if (threadIdx.x == 0) blocks[blockIdx.x] = total;
}

__global__ void k_scan_blocks(int64_t *blocks, int nb) {
    // single block: exclusive scan of nb block sums in place, total at blocks[nb]
    int64_t carry = 0;
    for (int b0 = 0; b0 < nb; b0 += kScanThreads) {
        int i = b0 + threadIdx.x;
        int64_t v = (i < nb) ? blocks[i] : 0;
        int64_t total;
        int64_t e = block_excl_scan(v, &total);
        if (i < nb) blocks[i] = carry + e;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) blocks[nb] = carry;
}

__global__ void k_scan_apply(const int64_t *__restrict__ in, int64_t *__restrict__ out,
                             const int64_t *__restrict__ blocks, int n_max, const int32_t *d_count) {
    const int n = d_count ? min(*d_count, n_max) : n_max;
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t loc[kScanItems];
    int64_t s = 0;
    for (int it = 0; it < kScanItems; ++it) {
        int64_t i = base + it;
        loc[it] = (i < n) ? in[i] : 0;
        s += loc[it];
    }
    int64_t total;
    int64_t e = block_excl_scan(s, &total) + blocks[blockIdx.x];
    for (int it = 0; it < kScanItems; ++it) {
        int64_t i = base + it;
        if (i < n) out[i] = e;
        e += loc[it];
    }
}

__global__ void k_scan_total(const int64_t *__restrict__ in, int64_t *__restrict__ out, int n_max,
                             const int32_t *d_count) {
    const int n = d_count ? min(*d_count, n_max) : n_max;
    out[n] = (n > 0) ? out[n - 1] + in[n - 1] : 0;
}

}  // namespace

void scan_exclusive_i64(const int64_t *in, int64_t *out, int64_t *blocks, int n_max, const int32_t *d_count,
                        cudaStream_t st) {
    int nb = (n_max + kScanTile - 1) / kScanTile;
    if (nb < 1) nb = 1;
    k_scan_reduce<<<nb, kScanThreads, 0, st>>>(in, blocks, n_max, d_count);
    k_scan_blocks<<<1, kScanThreads, 0, st>>>(blocks, nb);
    k_scan_apply<<<nb, kScanThreads, 0, st>>>(in, out, blocks, n_max, d_count);
    k_scan_total<<<1, 1, 0, st>>>(in, out, n_max, d_count);
}

sph_status sort_alloc(RadixSorter &s, int n) {
    s.n_cap = n;
    s.tiles_cap = (n + RadixSorter::kTile - 1) / RadixSorter::kTile;
    if (s.tiles_cap < 1) s.tiles_cap = 1;
    size_t nb = sizeof(uint32_t) * (size_t)(n > 0 ? n : 1);
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2; ++b) {
        if (e == cudaSuccess) e = cudaMalloc(&s.keys[b], nb);
        if (e == cudaSuccess) e = cudaMalloc(&s.vals[b], nb);
    }
    if (e == cudaSuccess) e = cudaMalloc(&s.hist, sizeof(uint32_t) * 256 * RadixSorter::kMaxPasses);
    if (e == cudaSuccess)
        e = cudaMalloc(&s.status, sizeof(uint32_t) * 256 * (size_t)s.tiles_cap * RadixSorter::kMaxPasses);
    if (e == cudaSuccess) e = cudaMalloc(&s.counters, sizeof(uint32_t) * RadixSorter::kMaxPasses);
    return cuda_status(e, "sort_alloc");
}

void sort_free(RadixSorter &s) {
    for (int b = 0; b < 2; ++b) {
        cudaFree(s.keys[b]);
        cudaFree(s.vals[b]);
        s.keys[b] = s.vals[b] = nullptr;
    }
    cudaFree(s.hist);
    cudaFree(s.status);
    cudaFree(s.counters);
    s.hist = s.status = s.counters = nullptr;
}

int radix_sort_pairs(RadixSorter &s, int n, int bits, cudaStream_t st, uint32_t *health) {
    const int passes = (bits + 7) / 8;
    const int tiles = (n + RadixSorter::kTile - 1) / RadixSorter::kTile;
    int cur = 0;
    if (n <= 0) return 0;
    cudaMemsetAsync(s.status, 0, sizeof(uint32_t) * 256 * (size_t)tiles * passes, st);
    cudaMemsetAsync(s.counters, 0, sizeof(uint32_t) * RadixSorter::kMaxPasses, st);
    for (int p = 0; p < passes; ++p) {
        k_onesweep<<<tiles, RadixSorter::kThreads, 0, st>>>(s.keys[cur], s.vals[cur], s.keys[cur ^ 1],
                                                             s.vals[cur ^ 1], n, 8 * p, s.hist + 256 * p,
                                                             s.status + (size_t)256 * tiles * p, s.counters + p,
                                                             health, s.spin_limit);
        cur ^= 1;
    }
    return cur;
}

void launch_init_cells(sph_ctx *ctx, cudaStream_t st) {
    k_init_cells<<<148 * 8, 256, 0, st>>>(ctx->cell_range, kNumCells);
    ctx->cells_have_prev = false;
}

sph_status launch_sort(sph_ctx *ctx, cudaStream_t st) {
    RadixSorter &s = ctx->cell_sort;
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * 256 * RadixSorter::kMaxPasses, st);
    const int prev = ctx->cell_final;
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    // the previous sorted keys live in keys[prev]; the hash writes keys[0] and
    // the first pass writes keys[1], so clearing must use keys[prev] before that
    uint32_t *clear_src = s.keys[prev];
    if (prev == 0) {
        // never the case with 3 passes (result in buffer 1); kept for safety
        launch_init_cells(ctx, st);
    }
    k_hash_hist<<<blocks, 256, 0, st>>>(ctx->pos4, n, s.keys[0], s.vals[0], s.hist, clear_src, ctx->cell_range,
                                        (ctx->cells_have_prev && prev == 1) ? 1 : 0);
    int fin = radix_sort_pairs(s, n, 24, st, ctx->health);
    ctx->cell_final = fin;
    k_cells<<<(n + 255) / 256, 256, 0, st>>>(s.keys[fin], n, ctx->cell_range);
    ctx->cells_have_prev = true;
    if (ctx->units) {
        cudaMemsetAsync(ctx->units, 0xff, sizeof(uint2) * kNumUnits, st);
        k_units<<<(n + 255) / 256, 256, 0, st>>>(s.keys[fin], n, ctx->units);
    }
    return cuda_status(cudaGetLastError(), "sort");
}

}  // namespace sph

// ---------------------------------------------------------------------------
// Cell sort without allocation.
//
// Some callers cannot allocate device memory at all: code that runs inside a
// host framework which owns every allocation (a pool or arena it hands out,
// memory-accounting or sandboxing layers), or code that must not call
// cudaMalloc/cudaFree on a latency-critical thread because those calls may
// synchronise the device.  For them, sph_sort_cells_noalloc computes the same
// sorted (cell key, particle index) pairs as sph_sort from positions the
// caller already holds on the device, using only caller-provided inputs and
// outputs plus one fixed scratch array compiled into this library.
//
// The scratch is a file-scope __device__ array, so every GPU that loads the
// library carries it (kNoAllocScratchBytes, about 2.2 MiB) until the process
// exits.  On the host, the array's name is only a stand-in symbol, not a
// device address; its device address is looked up with cudaGetSymbolAddress
// on every call, for the device current at that call (the first lookup on a
// device loads the module there, which is why the first call should come
// before any stream capture).  Every call shares the array and it keeps the
// last call's contents, so the parts that must start at zero (histograms,
// tile tickets, the health word and the look-back words this call's size
// uses) are cleared on the caller's stream at each call, and calls whose work
// overlaps on the GPU (different streams without ordering, or several host
// threads) race on it.  A look-back wait that gives up raises the health word
// inside the scratch; sph_sort_cells_noalloc_health reads it back.
// ---------------------------------------------------------------------------
namespace sph {
namespace {

constexpr int kNoAllocPasses = 3;  // 24-bit cell keys
constexpr int kNoAllocTiles = (SPH_SORT_NOALLOC_MAX_N + RadixSorter::kTile - 1) / RadixSorter::kTile;
constexpr size_t kNoAllocKeysOff = 0;
constexpr size_t kNoAllocValsOff = kNoAllocKeysOff + sizeof(uint32_t) * SPH_SORT_NOALLOC_MAX_N;
// the words that must be zero when a call starts sit together from here on:
// histograms, tile tickets, the health word, then the look-back words of the
// three passes, each pass using 256 x (tiles of this call) words
constexpr size_t kNoAllocHistOff = kNoAllocValsOff + sizeof(uint32_t) * SPH_SORT_NOALLOC_MAX_N;
constexpr size_t kNoAllocCountOff = kNoAllocHistOff + sizeof(uint32_t) * 256 * kNoAllocPasses;
constexpr size_t kNoAllocHealthOff = kNoAllocCountOff + sizeof(uint32_t) * kNoAllocPasses;
constexpr size_t kNoAllocStatusOff = kNoAllocHealthOff + sizeof(uint32_t);
constexpr size_t kNoAllocScratchBytes = kNoAllocStatusOff + sizeof(uint32_t) * 256 * kNoAllocTiles * kNoAllocPasses;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// sort.metal:15-44 from xyz-interleaved positions, plus the digit histograms
// of the three passes (same keys as k_hash_hist; no cell table to clear).
__global__ void k_hash_hist_xyz(const float *__restrict__ pos, int n, uint32_t *__restrict__ keys,
                                uint32_t *__restrict__ vals, uint32_t *__restrict__ hist) {
    __shared__ uint32_t sh[3][256];
    for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) (&sh[0][0])[i] = 0u;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = cell_key(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        keys[i] = k;
        vals[i] = (uint32_t)i;
        atomicAdd(&sh[0][k & 255u], 1u);
        atomicAdd(&sh[1][(k >> 8) & 255u], 1u);
        atomicAdd(&sh[2][(k >> 16) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) {
        const uint32_t v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// Device address of the scratch array on the current device.
sph_status noalloc_scratch(unsigned char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "sph_sort_cells_noalloc: cudaGetSymbolAddress");
    *out = static_cast<unsigned char *>(p);
    return SPH_OK;
}

}  // namespace

}  // namespace sph

extern "C" sph_status sph_sort_cells_noalloc(const float *pos_xyz, int32_t n, uint32_t *cell_key,
                                            uint32_t *cell_index, void *stream) {
    using namespace sph;
    if (n < 0 || n > SPH_SORT_NOALLOC_MAX_N) {
        set_error("sph_sort_cells_noalloc: n = %d is outside 0..%d (the size of the library's fixed scratch)", n,
                  SPH_SORT_NOALLOC_MAX_N);
        return SPH_ERR_INVALID_ARG;
    }
    if (n == 0) return SPH_OK;
    if (!pos_xyz || !cell_key || !cell_index) {
        set_error("sph_sort_cells_noalloc: null device pointer");
        return SPH_ERR_INVALID_ARG;
    }
    unsigned char *s = nullptr;
    sph_status st = noalloc_scratch(&s);
    if (st != SPH_OK) return st;
    cudaStream_t cs = (cudaStream_t)stream;
    const int tiles = (n + RadixSorter::kTile - 1) / RadixSorter::kTile;
    uint32_t *tk = reinterpret_cast<uint32_t *>(s + kNoAllocKeysOff);
    uint32_t *tv = reinterpret_cast<uint32_t *>(s + kNoAllocValsOff);
    uint32_t *hist = reinterpret_cast<uint32_t *>(s + kNoAllocHistOff);
    uint32_t *counters = reinterpret_cast<uint32_t *>(s + kNoAllocCountOff);
    uint32_t *health = reinterpret_cast<uint32_t *>(s + kNoAllocHealthOff);
    uint32_t *status = reinterpret_cast<uint32_t *>(s + kNoAllocStatusOff);
    const size_t zero_bytes = (kNoAllocStatusOff - kNoAllocHistOff) + sizeof(uint32_t) * 256 * (size_t)tiles * kNoAllocPasses;
    cudaError_t e = cudaMemsetAsync(s + kNoAllocHistOff, 0, zero_bytes, cs);
    if (e != cudaSuccess) return cuda_status(e, "sph_sort_cells_noalloc: clear scratch");
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_hash_hist_xyz<<<blocks, 256, 0, cs>>>(pos_xyz, n, tk, tv, hist);
    // three stable 8-bit passes: scratch -> out -> scratch -> out
    uint32_t *kin[kNoAllocPasses] = {tk, cell_key, tk};
    uint32_t *vin[kNoAllocPasses] = {tv, cell_index, tv};
    uint32_t *kout[kNoAllocPasses] = {cell_key, tk, cell_key};
    uint32_t *vout[kNoAllocPasses] = {cell_index, tv, cell_index};
    for (int p = 0; p < kNoAllocPasses; ++p)
        k_onesweep<<<tiles, RadixSorter::kThreads, 0, cs>>>(kin[p], vin[p], kout[p], vout[p], n, 8 * p, hist + 256 * p,
                                                            status + (size_t)256 * tiles * p, counters + p, health,
                                                            kSpinLimit);
    return cuda_status(cudaGetLastError(), "sph_sort_cells_noalloc");
}

extern "C" sph_status sph_sort_cells_noalloc_health(void *stream, uint32_t *word) {
    using namespace sph;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_status(e, "sph_sort_cells_noalloc_health: stream");
    uint32_t w = 0;
    e = cudaMemcpyFromSymbol(&w, g_noalloc_scratch, sizeof(uint32_t), kNoAllocHealthOff, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "sph_sort_cells_noalloc_health: read");
    if (word) *word = w;
    if (w & SPH_HEALTH_SORT_TIMEOUT) {
        set_error("sph_sort_cells_noalloc: a look-back wait gave up (health 0x%x); the outputs are incomplete", w);
        return SPH_ERR_TIMEOUT;
    }
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// Self-test of the bounded look-back wait.  One k_onesweep tile is launched
// whose ticket is preset to 1, so it waits on tile 0's status words, which
// nothing writes: the wait must give up after spin_limit polls, raise
// SPH_HEALTH_SORT_TIMEOUT and return.  The tile holds no elements (n = 0), so
// it reads and writes no key or value.  With ctx the context's sorter scratch
// and health word are used (sph_synchronize then reports SPH_ERR_TIMEOUT);
// without, the allocation-free sort's static scratch is used
// (sph_sort_cells_noalloc_health then reports it).
// ---------------------------------------------------------------------------
namespace sph {
namespace {
__global__ void k_selftest_prepare(uint32_t *hist, uint32_t *status, uint32_t *counter) {
    const int t = threadIdx.x;  // 256 threads
    hist[t] = 0u;
    status[t] = 0u;
    status[256 + t] = 0u;
    if (t == 0) *counter = 1u;
}
}  // namespace
}  // namespace sph

extern "C" sph_status sph_selftest_lookback_timeout(sph_ctx *ctx, int32_t spin_limit, void *stream) {
    using namespace sph;
    if (spin_limit < 1 || spin_limit > (1 << 22)) {
        set_error("sph_selftest_lookback_timeout: spin_limit %d is outside 1..%d", spin_limit, 1 << 22);
        return SPH_ERR_INVALID_ARG;
    }
    cudaStream_t cs = (cudaStream_t)stream;
    uint32_t *hist, *status, *counter, *health, *kbuf, *vbuf;
    if (ctx) {
        cudaSetDevice(ctx->device);
        RadixSorter &r = ctx->cell_sort;  // status holds >= 4 x 256 words
        hist = r.hist;
        status = r.status;
        counter = r.counters;
        health = ctx->health;
        kbuf = r.keys[0];
        vbuf = r.vals[0];
    } else {
        unsigned char *s = nullptr;
        sph_status st = noalloc_scratch(&s);
        if (st != SPH_OK) return st;
        hist = reinterpret_cast<uint32_t *>(s + kNoAllocHistOff);
        counter = reinterpret_cast<uint32_t *>(s + kNoAllocCountOff);
        health = reinterpret_cast<uint32_t *>(s + kNoAllocHealthOff);
        status = reinterpret_cast<uint32_t *>(s + kNoAllocStatusOff);
        kbuf = reinterpret_cast<uint32_t *>(s + kNoAllocKeysOff);
        vbuf = reinterpret_cast<uint32_t *>(s + kNoAllocValsOff);
    }
    // the key/value buffers are valid device memory, though n = 0 touches none
    k_selftest_prepare<<<1, 256, 0, cs>>>(hist, status, counter);
    k_onesweep<<<1, RadixSorter::kThreads, 0, cs>>>(kbuf, vbuf, kbuf, vbuf, 0, 0, hist, status, counter,
                                                    health, spin_limit);
    return cuda_status(cudaGetLastError(), "sph_selftest_lookback_timeout");
}

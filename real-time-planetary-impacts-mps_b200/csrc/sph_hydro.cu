// sph_hydro.cu -- density, acceleration and step passes for sm_100a.
//
// density      SPH/Shaders/density.metal:12-239        (Compute.cpp:179-208)
// acceleration SPH/Shaders/accelerations.metal:12-141  (Compute.cpp:210-240)
// step         SPH/Shaders/step.metal:12-46            (Compute.cpp:242-263)
// snapshot     SPH/Shaders/render.metal:49-66          (Compute.cpp:396-448)
//
// A small group of lanes per particle in sorted (Morton cell) order (see
// group_walk), so a warp's groups walk neighbouring cells together.
// Neighbour data are read from sorted, 16-byte records (sp4/sv4, then
// sA/sB/sC written by the density epilogue), so every cell's particles are
// one contiguous run of float4 loads instead of the reference's index-chased
// float3 gathers.  The neighbour walks visit the reference's cells and
// particles; each lane sums its slice in the reference's order and the slices
// are combined at the end (with one lane per particle, in the parity build,
// the order is the reference's exactly).
//
// The reference's 128-entry per-thread neighbour cache (density.metal:67-70)
// is replaced by rescanning the same cell box with the same filters: the
// visited set and order are identical (see k_density), and no thread carries
// 1 KiB of local memory.
#include <cuda_runtime.h>

#include <algorithm>

#include "sph_internal.h"

namespace sph {

namespace {

// Margin on the distance from a particle to a cell box: positions near 318 Mm
// carry ~3e-5 Mm of float32 rounding, and a particle's cell comes from
// floor(x / CELL_WIDTH); 2e-4 Mm keeps every particle of a cell inside its box.
constexpr float kCellMargin = 2e-4f;

// Square root of a pair distance.  The parity build keeps the correctly
// rounded sqrtf of the reference; the product uses the hardware reciprocal
// square root (within 2 ulp), a rounding-level difference.
__device__ __forceinline__ float pair_sqrt(float r2) {
#ifdef SPH_PARITY
    return sqrtf(r2);
#else
    return r2 > 0.f ? r2 * rsqrtf(r2) : 0.f;
#endif
}

// 1 / r for a pair at r = pair_sqrt(r2) > 0: the correctly rounded quotient
// in the parity build, the hardware reciprocal square root in the product.
__device__ __forceinline__ float pair_rinv(float r2, float r) {
#ifdef SPH_PARITY
    return 1.f / r;
#else
    (void)r;
    return rsqrtf(r2);
#endif
}

// a / b in the pair arithmetic: the correctly rounded quotient in the parity
// build, the hardware approximation (within 2 ulp) in the product.
__device__ __forceinline__ float pdiv(float a, float b) {
#ifdef SPH_PARITY
    return a / b;
#else
    return __fdividef(a, b);
#endif
}

// Lanes per particle in the density and acceleration walks.  The parity
// build (SPH_PARITY) uses one, which sums in the reference's sequential order.
#ifdef SPH_PARITY
constexpr int kLanesPerParticle = 1;
#else
#ifndef SPH_HYDRO_LANES
#define SPH_HYDRO_LANES 8
#endif
constexpr int kLanesPerParticle = SPH_HYDRO_LANES;
#endif

// Squared distance from (px, py, pz) to the box of cell (x, y, z), each axis
// gap shortened by the margin.
__device__ __forceinline__ float cell_gap2(float px, float py, float pz, int x, int y, int z) {
    const float w = kCellWidth;
    const float gx = fmaxf(fmaxf((float)x * w - px, px - (float)(x + 1) * w) - kCellMargin, 0.f);
    const float gy = fmaxf(fmaxf((float)y * w - py, py - (float)(y + 1) * w) - kCellMargin, 0.f);
    const float gz = fmaxf(fmaxf((float)z * w - pz, pz - (float)(z + 1) * w) - kCellMargin, 0.f);
    return gx * gx + gy * gy + gz * gz;
}

__global__ void k_gather(int n, const uint32_t *__restrict__ cidx, const float4 *__restrict__ pos4,
                         const float4 *__restrict__ vel4, float4 *__restrict__ sp4, float4 *__restrict__ sv4) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t i = cidx[k];
    sp4[k] = pos4[i];
    sv4[k] = vel4[i];
}

// ---- neighbour walk shared by the lanes of one particle -------------------
//
// Each particle gets a group of L consecutive lanes (L = 1, 2, 4 or 8); a
// warp holds 32 / L consecutive particles of the sorted order.  The group
// walks the particle's own cell box of radius 2h in the reference's order
// (x outer, z inner; sorted index within a cell): its lanes look up L cells
// at a time (cells farther than the search radius are not looked up), the
// particles of those cells are numbered consecutively, and lane `sub` takes
// every L-th of them.  So each lane sees a slice of exactly the candidates the
// reference's box walk visits, the lanes stay busy although a cell holds only
// a few particles, and the cell table is read once per cell and particle
// group instead of once per lane.  Partial sums are combined across the
// group by a butterfly (every lane ends with the same bits).  With L = 1 the
// walk is the reference's sequential order exactly.

template <int L>
__device__ __forceinline__ unsigned group_mask(int lane) {
    return L == 32 ? 0xffffffffu : (((1u << L) - 1u) << (lane & ~(L - 1)));
}
template <int L>
__device__ __forceinline__ float group_sum(float v, unsigned gm) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gm, v, o, L);
    return v;
}
template <int L>
__device__ __forceinline__ int group_sum_i(int v, unsigned gm) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gm, v, o, L);
    return v;
}
template <int L>
__device__ __forceinline__ float group_max(float v, unsigned gm) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v = fmax_ref(v, __shfl_xor_sync(gm, v, o, L));
    return v;
}

// s_off / s_start: this warp's 32-entry scratch in shared memory; gbase =
// the group's first lane within the warp.
template <int L, class Body>
__device__ __forceinline__ void group_walk(float px, float py, float pz, float h, float r2cull,
                                           const uint2 *__restrict__ cells, int sub, unsigned gm, int gbase,
                                           uint32_t *s_off, uint32_t *s_start, Body &&body) {
    const CellBox b = cell_box(px, py, pz, h);
    const int ny = b.hi1 - b.lo1 + 1, nz = b.hi2 - b.lo2 + 1;
    const int nyz = ny * nz;
    const int nc = (b.hi0 - b.lo0 + 1) * nyz;
    for (int c0 = 0; c0 < nc; c0 += L) {
        const int c = c0 + sub;
        uint32_t st = 0u, cnt = 0u;
        if (c < nc) {
            const int ix = c / nyz, rem = c - ix * nyz;
            const int iy = rem / nz, iz = rem - iy * nz;
            const int x = b.lo0 + ix, y = b.lo1 + iy, z = b.lo2 + iz;
            if (cell_gap2(px, py, pz, x, y, z) <= r2cull) {
                const uint2 r = __ldg(cells + cell_index_of(x, y, z));
                if (r.x != 0xffffffffu) {
                    st = r.x;
                    cnt = r.y - r.x + 1u;
                }
            }
        }
        if (L == 1) {
            for (uint32_t k = st; k < st + cnt; ++k) body(k);
            continue;
        }
        uint32_t inc = cnt;
#pragma unroll
        for (int o = 1; o < L; o <<= 1) {
            const uint32_t y = __shfl_up_sync(gm, inc, o, L);
            if (sub >= o) inc += y;
        }
        const uint32_t tot = __shfl_sync(gm, inc, L - 1, L);
        if (tot == 0u) continue;
        s_off[gbase + sub] = inc - cnt;
        s_start[gbase + sub] = st;
        __syncwarp(gm);
        for (uint32_t j = sub; j < tot; j += L) {
            int q = 0;  // the last cell whose first candidate number is <= j
#pragma unroll
            for (int step = L / 2; step > 0; step >>= 1)
                if (s_off[gbase + q + step] <= j) q += step;
            body(s_start[gbase + q] + (j - s_off[gbase + q]));
        }
        __syncwarp(gm);
    }
}

// Collect, in the walk's order, the indices of the candidates of the
// particle's box of radius 2 hbox that pass `test` into the group's list in
// shared memory: each round of L candidates is ordered by a ballot, so the
// list keeps the reference's visiting order.  Whenever the list could
// overflow, `drain(count)` consumes it and the list restarts; a drain that
// returns false keeps the list instead and the walk only counts from then on,
// so the return value (the number of candidates found) may exceed cap.
template <int L, class Test, class Drain>
__device__ __forceinline__ int group_collect(float px, float py, float pz, float hbox, float r2cull,
                                             const uint2 *__restrict__ cells, int sub, unsigned gm, int gbase,
                                             uint32_t *s_off, uint32_t *s_start, uint32_t *list, int cap,
                                             Test &&test, Drain &&drain) {
    const CellBox b = cell_box(px, py, pz, hbox);
    const int ny = b.hi1 - b.lo1 + 1, nz = b.hi2 - b.lo2 + 1;
    const int nyz = ny * nz;
    const int nc = (b.hi0 - b.lo0 + 1) * nyz;
    int cnt = 0;
    for (int c0 = 0; c0 < nc; c0 += L) {
        const int c = c0 + sub;
        uint32_t st = 0u, n_in = 0u;
        if (c < nc) {
            const int ix = c / nyz, rem = c - ix * nyz;
            const int iy = rem / nz, iz = rem - iy * nz;
            const int x = b.lo0 + ix, y = b.lo1 + iy, z = b.lo2 + iz;
            if (cell_gap2(px, py, pz, x, y, z) <= r2cull) {
                const uint2 r = __ldg(cells + cell_index_of(x, y, z));
                if (r.x != 0xffffffffu) {
                    st = r.x;
                    n_in = r.y - r.x + 1u;
                }
            }
        }
        uint32_t inc = n_in;
#pragma unroll
        for (int o = 1; o < L; o <<= 1) {
            const uint32_t y = __shfl_up_sync(gm, inc, o, L);
            if (sub >= o) inc += y;
        }
        const uint32_t tot = __shfl_sync(gm, inc, L - 1, L);
        if (tot == 0u) continue;
        s_off[gbase + sub] = inc - n_in;
        s_start[gbase + sub] = st;
        __syncwarp(gm);
        for (uint32_t j0 = 0; j0 < tot; j0 += L) {
            const uint32_t j = j0 + sub;
            uint32_t k = 0u;
            bool hit = false;
            if (j < tot) {
                int q = 0;  // the last cell whose first candidate number is <= j
#pragma unroll
                for (int step = L / 2; step > 0; step >>= 1)
                    if (s_off[gbase + q + step] <= j) q += step;
                k = s_start[gbase + q] + (j - s_off[gbase + q]);
                hit = test(k);
            }
            const unsigned hm = (__ballot_sync(gm, hit) >> gbase) & (L == 32 ? 0xffffffffu : ((1u << L) - 1u));
            const int nh = __popc(hm);
            if (cnt + nh > cap) {
                if (!drain(cnt)) {
                    cnt += nh;  // overflow: keep counting, store nothing more
                    continue;
                }
                cnt = 0;
            }
            if (hit) list[cnt + __popc(hm & ((1u << sub) - 1u))] = k;
            cnt += nh;
            __syncwarp(gm);
        }
        __syncwarp(gm);
    }
    return cnt;
}

struct DensityArgs {
    int n;
    const uint32_t *cidx;
    const uint32_t *skey;  // sorted cell keys (tile passes)
    const uint2 *cells;
    const uint2 *units;    // 64-cell unit ranges (coarse tiles)
    uint8_t *cflags;       // per 512-cell block: holds a coarse-tile particle
    int coarse;            // coarse tiles on
    const float4 *sp4, *sv4;
    float *h, *rho, *f, *P, *c, *B;
    const float *u;
    const int32_t *mat;
    const uint8_t *active;
    float4 *sA, *sB, *sC;
    int32_t *globals;
    uint32_t *health;
    EosTables eos;
    float eta;            // convergence tolerance of the h iteration (DENSITY_ETA in the reference)
    const float *seed;    // learned starting h per particle, or null (the plain guess, h itself)
    float *nn_out;        // neighbour count per particle, or null
    uint32_t *stats;      // [0] sweeps, [1] fallbacks, [2] most sweeps, [3] particles; or null
};

// A learned seed whose first sweep moves h by more than this relative amount
// is abandoned for the plain initial guess.
constexpr float kSeedFallback = 0.05f;

// Per-particle neighbour list of the density pass, in shared memory: the
// sorted indices of every candidate within kListReach x the smoothing length
// the list was built for, in the reference's visiting order.  The iteration's
// sweeps and the gradient sweep read it instead of walking the cells again
// (recomputing each distance exactly as the walk does); a sweep whose radius
// the list does not cover rebuilds it, and a particle whose list overflows
// walks the cells in every sweep.
constexpr int kListMax = 192;       // list entries per particle
// particles per block: 16 groups, but never fewer than a warp's worth of lanes
template <int L>
__host__ __device__ constexpr int parts_per_block() { return 16 * L >= 32 ? 16 : 32 / L; }
constexpr float kListReach = 1.15f; // list radius / (2 h)

// density.metal:12-239 for one sorted particle per lane group.  The group
// keeps the reference's per-particle iteration state (h, the int max_h, the
// cached scan's h and neighbour count) identically in all its lanes.
// w_off / w_start: the warp's 32-entry walk scratch; list: the group's
// kListMax-entry neighbour list.
template <int L>
__device__ __forceinline__ void density_particle(const DensityArgs &a, int index, int sub, unsigned gm, int gbase,
                                                 uint32_t *w_off, uint32_t *w_start, uint32_t *list) {
    const uint32_t ind = a.cidx[index];
    const float4 me = a.sp4[index];
    const float4 mv = a.sv4[index];
    if (!a.active[ind]) {
        // density.metal:40-55: EOS only
        if (sub != 0) return;
        float2 pc = eos_lookup(a.eos, a.mat[ind], a.rho[ind], a.u[ind]);
        a.P[ind] = pc.x;
        a.c[ind] = pc.y;
        float hi = a.h[ind], rho = a.rho[ind], fi = a.f[ind];
        a.sA[index] = make_float4(me.x, me.y, me.z, hi);
        a.sB[index] = make_float4(mv.x, mv.y, mv.z, pc.y);
        a.sC[index] = make_float4(me.w, (fi * pc.x / (rho * rho)), rho, a.B[ind]);
        return;
    }
    const float px = me.x, py = me.y, pz = me.z, mi = me.w;
    const float h_plain = a.h[ind];
    float hi = h_plain;
    // a learned seed replaces the plain guess when it is finite and within a
    // factor two of it
    bool seeded = false;
    if (a.seed) {
        const float sd = a.seed[ind];
        if (sd >= 0.5f * h_plain && sd <= 2.f * h_plain && sd <= kMaxH) {
            hi = sd;
            seeded = true;
        }
    }
    bool first = true, fell_back = false;
    int sweeps = 0;
    int max_h = 0;  // an int in the reference (truncates h < 1 to 0)
    float h2x4 = 4.f * hi * hi;
    float h1 = 1.f / hi;
    float dens = 0.f;
    float eps = 1.f;
    int count = 0;
    // State of the reference's neighbour cache, which holds the neighbours of
    // the last full scan: that scan's h (box and filter), and its count capped
    // at N_NEIGHBOURS_ESTIM.  A "cached" sweep is a rescan with those filters.
    int nn = 0;
    float hs = hi, hs2x4 = h2x4;
    const uint2 *cells = a.cells;
    const float4 *sp4 = a.sp4;
    // the list: entries within sqrt(list_r2); n_list < 0 = none
    int n_list = -1;
    float list_r2 = 0.f;
    auto build = [&](float hb) {
        const float rl = 2.f * hb * kListReach;
        list_r2 = rl * rl;
        const float r2max = list_r2;
        n_list = group_collect<L>(
            px, py, pz, hb * kListReach, r2max, cells, sub, gm, gbase, w_off, w_start, list, kListMax,
            [&](uint32_t k) {
                const float4 q = __ldg(sp4 + k);
                const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                return dx * dx + dy * dy + dz * dz <= r2max;
            },
            [](int) { return false; });
        __syncwarp(gm);
    };
    while (eps > a.eta && count < kMaxNR) {
        const bool cached = hi < (float)max_h && nn < kNeighbourCache;
        if (!cached) {
            hs = hi;
            hs2x4 = h2x4;
        }
        const float h2 = hi + hi;
        if (n_list < 0 || (n_list <= kListMax && hs2x4 > list_r2)) build(hs);
        float part = 0.f;
        int found = 0;
        if (n_list <= kListMax) {
#pragma unroll 4
            for (int i = sub; i < n_list; i += L) {
                const float4 q = __ldg(sp4 + list[i]);
                const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > hs2x4) continue;
                const float r = pair_sqrt(r2);
                if (cached && r > h2) continue;
                ++found;
                part += kernel_w(r, h1) * q.w;
            }
        } else {
            group_walk<L>(px, py, pz, hs, hs2x4, cells, sub, gm, gbase, w_off, w_start, [&](uint32_t k) {
                const float4 q = __ldg(sp4 + k);
                const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > hs2x4) return;
                const float r = pair_sqrt(r2);
                if (cached && r > h2) return;
                ++found;
                part += kernel_w(r, h1) * q.w;
            });
        }
        dens = group_sum<L>(part, gm);
        if (!cached) nn = min(group_sum_i<L>(found, gm), kNeighbourCache);
        float nh = fmin_ref(kResolutionEta * powf(mi / dens, 1.f / 3), kMaxH);
        nh = 0.5f * (hi + nh);
        eps = fabsf(nh - hi) / hi;
        ++sweeps;
        if (first && seeded && eps > kSeedFallback) {
            // the seed disagrees with its own first sweep: start again from
            // the plain guess, with the iteration state of a fresh start
            first = false;
            fell_back = true;
            hi = h_plain;
            h1 = 1.f / hi;
            h2x4 = 4.f * hi * hi;
            max_h = 0;
            nn = 0;
            eps = 1.f;
            continue;
        }
        first = false;
        if (eps > a.eta) {
            max_h = (int)fmax_ref((float)max_h, hi);
            hi = nh;
            h1 = 1.f / hi;
            h2x4 = 4.f * hi * hi;
            count++;
        }
    }
    // gradient sweep (density.metal:145-213): below N_NEIGHBOURS_ESTIM the
    // cached neighbours (last full scan) within 2h; above, a full scan at h
    // that adds to the converged density again
    const bool gcached = nn < kNeighbourCache;
    const float gh = gcached ? hs : hi;
    const float g2 = gcached ? hs2x4 : h2x4;
    const float h2 = hi + hi;
    const float vix = mv.x, viy = mv.y, viz = mv.z;
    const float4 *sv4 = a.sv4;
    float pdens = 0.f, dens_h = 0.f, vdiv = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    auto grad = [&](uint32_t k, float r, float mj, float dx, float dy, float dz) {
        if (!gcached) pdens += kernel_w(r, h1) * mj;
        dens_h += mj * kernel_dwdh(r, h1);
        if (r > 1e-12f) {
            const float r1 = 1.f / r;
            const float4 vj = __ldg(sv4 + k);
            const float vx = vj.x - vix, vy = vj.y - viy, vz = vj.z - viz;
            const float sc = kernel_gradw_scale(r, h1);
            const float gx = sc * (dx * r1), gy = sc * (dy * r1), gz = sc * (dz * r1);
            vdiv += mj * (vx * gx + vy * gy + vz * gz);
            cx += mj * (vy * gz - vz * gy);
            cy += mj * (vz * gx - vx * gz);
            cz += mj * (vx * gy - vy * gx);
        }
    };
    if (n_list <= kListMax && g2 > list_r2) build(gh);
    if (n_list <= kListMax) {
#pragma unroll 4
        for (int i = sub; i < n_list; i += L) {
            const uint32_t k = list[i];
            const float4 q = __ldg(sp4 + k);
            const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > g2) continue;
            const float r = pair_sqrt(r2);
            if (gcached && r > h2) continue;
            grad(k, r, q.w, dx, dy, dz);
        }
    } else {
        group_walk<L>(px, py, pz, gh, g2, cells, sub, gm, gbase, w_off, w_start, [&](uint32_t k) {
            const float4 q = __ldg(sp4 + k);
            const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > g2) return;
            const float r = pair_sqrt(r2);
            if (gcached && r > h2) return;
            grad(k, r, q.w, dx, dy, dz);
        });
    }
    if (!gcached) dens += group_sum<L>(pdens, gm);
    dens_h = group_sum<L>(dens_h, gm);
    vdiv = group_sum<L>(vdiv, gm);
    cx = group_sum<L>(cx, gm);
    cy = group_sum<L>(cy, gm);
    cz = group_sum<L>(cz, gm);
    if (a.stats) {
        // counters of the iteration (one group member per particle)
        const unsigned am = __activemask();
        const uint32_t mine = sub == 0 ? 1u : 0u;
        const uint32_t sw = __reduce_add_sync(am, mine * (uint32_t)sweeps);
        const uint32_t fb = __reduce_add_sync(am, mine * (fell_back ? 1u : 0u));
        const uint32_t mx = __reduce_max_sync(am, mine * (uint32_t)sweeps);
        const uint32_t np = __reduce_add_sync(am, mine);
        if ((threadIdx.x & 31) == (uint32_t)(__ffs(am) - 1)) {
            atomicAdd(a.stats + 0, sw);
            if (fb) atomicAdd(a.stats + 1, fb);
            atomicMax(a.stats + 2, mx);
            atomicAdd(a.stats + 3, np);
        }
    }
    if (sub != 0) return;
    if (a.nn_out) a.nn_out[ind] = (float)nn;
    vdiv = fabsf(vdiv) / dens;
    float acurl = sqrtf(cx * cx + cy * cy + cz * cz) / dens;
    float fi = 1.f / (1.f + (hi / (3.f * dens)) * dens_h);
    float2 pc = eos_lookup(a.eos, a.mat[ind], dens, a.u[ind]);
    float bal = vdiv / (vdiv + acurl + 1e-4f * (pc.y / hi));
    a.h[ind] = hi;
    a.rho[ind] = dens;
    a.f[ind] = fi;
    a.P[ind] = pc.x;
    a.c[ind] = pc.y;
    a.B[ind] = bal;
    if (!(dens == dens) || !(pc.x == pc.x)) raise_health(a.health, SPH_HEALTH_NAN_DENSITY);
    a.sA[index] = make_float4(px, py, pz, hi);
    a.sB[index] = make_float4(vix, viy, viz, pc.y);
    a.sC[index] = make_float4(mi, (fi * pc.x / (dens * dens)), dens, bal);
}

// One lane group per sorted particle, every particle.
template <int L>
__global__ void __launch_bounds__(parts_per_block<L>() * L) k_density(DensityArgs a) {
    extern __shared__ uint32_t s_lists[];
    __shared__ uint32_t s_off[parts_per_block<L>() * L], s_start[parts_per_block<L>() * L];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, sub = lane & (L - 1), gbase = lane & ~(L - 1);
    const int index = t / L;
    if (index >= a.n) return;  // whole groups leave together
    if (t == 0) a.globals[1] = (int32_t)(kDT0 * 1 / kDtMin1);  // density.metal:34-36
    density_particle<L>(a, index, sub, group_mask<L>(lane), gbase, s_off + (threadIdx.x & ~31),
                        s_start + (threadIdx.x & ~31), s_lists + (size_t)(threadIdx.x / L) * kListMax);
}

// The particles the tile pass handed on (sorted indices idx[0, *count)),
// one lane group each, grid-stride.
template <int L>
__global__ void __launch_bounds__(parts_per_block<L>() * L)
    k_density_deferred(DensityArgs a, const uint32_t *__restrict__ idx, const uint32_t *__restrict__ count) {
    extern __shared__ uint32_t s_lists[];
    __shared__ uint32_t s_off[parts_per_block<L>() * L], s_start[parts_per_block<L>() * L];
    const int lane = threadIdx.x & 31, sub = lane & (L - 1), gbase = lane & ~(L - 1);
    const uint32_t cnt = *count;
    constexpr int per_block = parts_per_block<L>();
    for (uint32_t base = blockIdx.x * per_block; base < cnt; base += gridDim.x * per_block) {
        const uint32_t j = base + threadIdx.x / L;
        if (j < cnt)
            density_particle<L>(a, (int)idx[j], sub, group_mask<L>(lane), gbase, s_off + (threadIdx.x & ~31),
                                s_start + (threadIdx.x & ~31), s_lists + (size_t)(threadIdx.x / L) * kListMax);
    }
}

// ---- density over cell tiles (product build) --------------------------------
//
// A tile is an aligned Morton block of cells -- 64 cells (4 x 4 x 4), or, where
// such a block holds many particles, its 16-cell halves of halves or its
// octets -- so its particles are one contiguous run of the sorted order.  A CTA
// takes tiles from a ticket counter; per tile it stages, once, every particle
// of the box of cells that the tile's neighbour lists can reach (float4
// position + mass and the sorted index) into shared memory, in cell order
// x-major, then y, z innermost, so a row of cells along z is one contiguous
// run of staged slots.  Warps then take the tile's particles four at a time
// (density_tile_warp): the list build reads the particles' rows of the staged
// box, every h-iteration sweep reads the list, and no sweep touches the cell
// table or global positions again.  A particle whose list box reaches more
// than kTileReach cells beyond its own cell, whose h is at least
// MAX_SMOOTHING_LENGTH (where the reference's neighbour cache comes into play),
// whose list overflows or whose growing h leaves the staged box is handed to
// k_density_deferred, which runs the per-particle walk above; so is every
// particle of a tile whose box exceeds the shared-memory budget.
constexpr int kTileThreads = 384;
#ifndef SPH_TILE_LANES
#define SPH_TILE_LANES 8
#endif
constexpr int kTileLanes = SPH_TILE_LANES;                  // lanes per particle
constexpr int kTileGpw = 32 / kTileLanes;                   // particles per warp
constexpr int kTileGroups = kTileThreads / kTileLanes;      // particles in flight per CTA
constexpr int kTileStageMax = 3840;                         // staged particles per tile
constexpr int kTileCellsMax = 1024;                         // cells of a tile's staged box
constexpr int kTileCellsPerThread = (kTileCellsMax + kTileThreads - 1) / kTileThreads;
#ifndef SPH_TILE_REACH_CELLS
#define SPH_TILE_REACH_CELLS 3
#endif
constexpr int kTileReach = SPH_TILE_REACH_CELLS;            // cells a list box may extend past its own cell
constexpr int kTileList = 256;                              // list entries per particle (staged slots)
#ifndef SPH_TILE_LIST_REACH
#define SPH_TILE_LIST_REACH 1.05f
#endif
constexpr float kTileListReach = SPH_TILE_LIST_REACH;       // list radius / (2 h)
#ifndef SPH_TILE_STAGE_REACH
#define SPH_TILE_STAGE_REACH 1.15f
#endif
// staged box radius / (2 h): room for h to grow before a list rebuild leaves
// the staged box
constexpr float kTileStageReach = SPH_TILE_STAGE_REACH;

struct TileShared {
    float4 pos[kTileStageMax];          // staged (x, y, z, m)
    uint32_t gidx[kTileStageMax];       // staged sorted index
    uint32_t off[kTileCellsMax + 1];    // first staged slot of each box cell; off[cells] = staged count
    uint32_t first[kTileCellsMax];      // first sorted index of each box cell
    uint16_t list[kTileGroups][kTileList];
    int box[6];                         // staged box: lo x y z, hi x y z (unwrapped cell coordinates)
    uint32_t wsum[kTileThreads / 32];
    uint32_t start, end, tile, next;
    uint32_t stats[4];
    int defer_all;
    int need;                           // some particle of the range needs the warp pass
};

// The list box of a tile particle at smoothing length hb: the cells within
// 2 hb reach, widened by 1e-3 of a cell so that float rounding of the cell
// coordinates (|x| / CELL_WIDTH < 2^12, a few 1e-4 of a cell) never drops a
// cell.
__device__ __forceinline__ void tile_box(float px, float py, float pz, float hb, CellBox &b,
                                         float reach = kTileListReach) {
    constexpr float iw = 1.f / kCellWidth;
    constexpr float widen = 1e-3f;
    const float rl = 2.f * hb * reach;
    b.lo0 = (int)floorf((px - rl) * iw - widen);
    b.lo1 = (int)floorf((py - rl) * iw - widen);
    b.lo2 = (int)floorf((pz - rl) * iw - widen);
    b.hi0 = (int)floorf((px + rl) * iw + widen);
    b.hi1 = (int)floorf((py + rl) * iw + widen);
    b.hi2 = (int)floorf((pz + rl) * iw + widen);
}

// The (first, last) sorted range of tiling unit (x, y, z): a cell (U = 0) or a
// 64-cell unit (U = kUnitShift); first is 0xffffffff when it is empty.
template <int U>
__device__ __forceinline__ uint2 unit_range(const uint2 *cells, const uint2 *units, int x, int y, int z) {
    if (U == 0) return __ldg(cells + cell_index_of(x, y, z));
    return __ldg(units + unit_index_of(x, y, z));
}

// Whether a cell box reaches at most kTileReach tiling units (cells for U = 0,
// 64-cell units for U = kUnitShift) past the unit of cell (ox, oy, oz).
template <int U>
__device__ __forceinline__ bool within_reach(int ox, int oy, int oz, const CellBox &b) {
    return (ox >> U) - (b.lo0 >> U) <= kTileReach && (b.hi0 >> U) - (ox >> U) <= kTileReach &&
           (oy >> U) - (b.lo1 >> U) <= kTileReach && (b.hi1 >> U) - (oy >> U) <= kTileReach &&
           (oz >> U) - (b.lo2 >> U) <= kTileReach && (b.hi2 >> U) - (oz >> U) <= kTileReach;
}

// The pass that takes a density particle whose iteration starts from list
// radius 2 hb kTileListReach: 0 the cell tiles, kUnitShift the coarse tiles
// (a box past kTileReach cells, within kTileReach units), -1 the per-particle
// pass (h at MAX_H, where the reference's neighbour cache comes into play, or
// coarse tiles off).  Every pass evaluates it from the same inputs, so each
// particle is taken by exactly one.
__device__ __forceinline__ int density_mode(float px, float py, float pz, float hb, int coarse) {
    if (!(hb < kMaxH)) return -1;
    constexpr float iw = 1.f / kCellWidth;
    CellBox b;
    tile_box(px, py, pz, hb, b);
    const int ox = (int)floorf(px * iw), oy = (int)floorf(py * iw), oz = (int)floorf(pz * iw);
    if (within_reach<0>(ox, oy, oz, b)) return 0;
    if (coarse && within_reach<kUnitShift>(ox, oy, oz, b)) return kUnitShift;
    return -1;
}

// The starting h of an active particle's iteration (the learned seed when it
// is accepted, as in density_particle) and the h its staged box is built for.
__device__ __forceinline__ float tile_start_h(const DensityArgs &a, uint32_t ind, float h_plain, bool &seeded) {
    seeded = false;
    if (a.seed) {
        const float sd = a.seed[ind];
        if (sd >= 0.5f * h_plain && sd <= 2.f * h_plain && sd <= kMaxH) {
            seeded = true;
            return sd;
        }
    }
    return h_plain;
}

// Tiles: at the first sorted particle of every occupied 128-cell block (the
// cells whose keys differ in the low seven bits, 4 x 4 x 8), the block's
// octet ranges (from its 128 cell ranges); the block is one tile when it
// holds at most big_max particles, else each 64-cell half is one when it
// holds at most block_max, else each 16-cell quarter when it holds at most
// half_max, else each octet.  (first, one past last) per tile, in ticket
// order.  ctr[0] counts tiles; ctr[1] is the CTAs' tile ticket, ctr[2] the
// deferred count.
__global__ void k_tile_starts(int n, const uint32_t *__restrict__ skey, const uint2 *__restrict__ cells,
                              uint2 *__restrict__ tiles, uint32_t *ctr, int32_t *globals, uint32_t block_max,
                              uint32_t half_max, uint32_t big_max) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0 && globals) globals[1] = (int32_t)(kDT0 * 1 / kDtMin1);  // density.metal:34-36
    if (k >= n) return;
    const uint32_t blk = skey[k] >> 7;
    if (k > 0 && (skey[k - 1] >> 7) == blk) return;
    uint32_t ofirst[16], oend[16];  // octet ranges; oend == 0 when empty
#pragma unroll
    for (int o = 0; o < 16; ++o) {
        uint32_t f = 0xffffffffu, l = 0u;
        for (int j = 0; j < 8; ++j) {
            const uint2 r = cells[blk * 128u + (uint32_t)(o * 8 + j)];
            if (r.x != 0xffffffffu) {
                f = min(f, r.x);
                l = max(l, r.y + 1u);
            }
        }
        ofirst[o] = f;
        oend[o] = l;
    }
    auto emit = [&](uint32_t f, uint32_t l) {
        if (l > f) tiles[atomicAdd(ctr, 1u)] = make_uint2(f, l);
    };
    auto span = [&](int o0, int o1, uint32_t &f, uint32_t &l) {  // octets o0 .. o1 - 1
        f = 0xffffffffu;
        l = 0u;
        for (int o = o0; o < o1; ++o)
            if (oend[o]) {
                f = min(f, ofirst[o]);
                l = max(l, oend[o]);
            }
    };
    uint32_t f, l;
    span(0, 16, f, l);
    if (l - f <= big_max) {
        emit(f, l);
        return;
    }
    for (int hh = 0; hh < 2; ++hh) {
        span(8 * hh, 8 * hh + 8, f, l);
        if (l <= f) continue;
        if (l - f <= block_max) {
            emit(f, l);
            continue;
        }
        for (int q = 4 * hh; q < 4 * hh + 4; ++q) {
            span(2 * q, 2 * q + 2, f, l);
            if (l <= f) continue;
            if (l - f <= half_max) {
                emit(f, l);
            } else {
                emit(ofirst[2 * q], oend[2 * q]);
                emit(ofirst[2 * q + 1], oend[2 * q + 1]);
            }
        }
    }
}

// Coarse tiles: at the first sorted particle of every 512-cell block (2 x 2 x
// 2 units) that a cell-tile pass flagged, the block's (first, one past last)
// sorted range; the flag is cleared for the next pass.  ctr[0] counts tiles.
__global__ void k_coarse_starts(int n, const uint32_t *__restrict__ skey, const uint2 *__restrict__ units,
                                uint8_t *__restrict__ flags, uint2 *__restrict__ tiles, uint32_t *ctr) {
    constexpr int kShift = 3 * kUnitShift + 3;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t blk = skey[k] >> kShift;
    if (k > 0 && (skey[k - 1] >> kShift) == blk) return;
    if (!flags[blk]) return;
    flags[blk] = 0;
    uint32_t l = (uint32_t)k + 1u;
    for (int j = 0; j < 8; ++j) {
        const uint2 r = units[blk * 8u + (uint32_t)j];
        if (r.x != 0xffffffffu) l = max(l, r.y + 1u);
    }
    tiles[atomicAdd(ctr, 1u)] = make_uint2((uint32_t)k, l);
}

// One warp: the density pass of sorted particles p0 .. p0 + 3 of the staged
// tile (lane group g = lane / 8 takes p0 + g) whose pass is U (0 cell tiles,
// kUnitShift coarse tiles; the staged box counts U-units), in lockstep so the warp never
// runs its groups one after another: the list build is transposed (each lane
// takes one staged slot of a row and tests it against all four particles), and
// the sweeps run over the longest of the four lists with the others predicated
// off.  A particle that the tile path cannot finish is appended to `deferred`
// (sorted index) with nothing written; k_density_deferred takes it from the
// start.  The iteration is density_particle's with the neighbour cache never
// in use (h < MAX_H throughout, so the reference's int max_h stays 0).
template <int U, class Stage>
__device__ __forceinline__ void density_tile_warp(const DensityArgs &a, Stage &S, uint32_t *stats, uint32_t p0,
                                                  uint32_t end, int lane, uint16_t (*lists)[kTileList],
                                                  uint32_t *deferred, uint32_t *dctr) {
    constexpr int L = kTileLanes;
    constexpr unsigned kFull = 0xffffffffu;
    constexpr int kBig = 0x3fffffff;
    const int g = lane / L, sub = lane & (L - 1);
    uint16_t *list = lists[g];
    const uint32_t p = p0 + (uint32_t)g;
    bool live = p < end;  // the group iterates its particle (uniform within the group)
    uint32_t ind = 0u;
    float4 me = make_float4(0.f, 0.f, 0.f, 0.f), mv = me;
    if (live) {
        ind = a.cidx[p];
        me = a.sp4[p];
        mv = a.sv4[p];
        if (!a.active[ind]) {
            // density.metal:40-55: EOS only (in the cell-tile pass)
            if (U == 0 && sub == 0) {
                float2 pc = eos_lookup(a.eos, a.mat[ind], a.rho[ind], a.u[ind]);
                a.P[ind] = pc.x;
                a.c[ind] = pc.y;
                float hh = a.h[ind], rho = a.rho[ind], fi = a.f[ind];
                a.sA[p] = make_float4(me.x, me.y, me.z, hh);
                a.sB[p] = make_float4(mv.x, mv.y, mv.z, pc.y);
                a.sC[p] = make_float4(me.w, (fi * pc.x / (rho * rho)), rho, a.B[ind]);
            }
            live = false;
        }
    }
    auto defer = [&]() {
        if (sub == 0) deferred[atomicAdd(dctr, 1u)] = p;
        live = false;
    };
    const float px = me.x, py = me.y, pz = me.z, mi = me.w;
    float h_plain = 0.5f, hi = 0.5f;
    bool seeded = false;
    if (live) {
        h_plain = a.h[ind];
        hi = tile_start_h(a, ind, h_plain, seeded);
        const int m = density_mode(px, py, pz, fmaxf(hi, h_plain), a.coarse);
        if (m != U) {
            if (U == 0 && m < 0) defer();
            else live = false;  // another tile pass takes it
        } else if (S.defer_all) {
            defer();
        }
    }
    const int lo0 = S.box[0], lo1 = S.box[1], lo2 = S.box[2];
    const int ny = S.box[4] - lo1 + 1, nz = S.box[5] - lo2 + 1;
    // the group's list: staged slots within 2 hb kTileListReach
    int n_list = -1;
    float list_r2 = 0.f;
    auto build = [&](bool want, float hb) {
        CellBox b;
        if (want) {
            tile_box(px, py, pz, hb, b);
            b.lo0 >>= U, b.lo1 >>= U, b.lo2 >>= U, b.hi0 >>= U, b.hi1 >>= U, b.hi2 >>= U;  // U-units
            if (!(hb < kMaxH) || b.lo0 < lo0 || b.lo1 < lo1 || b.lo2 < lo2 || b.hi0 > S.box[3] || b.hi1 > S.box[4] ||
                b.hi2 > S.box[5]) {
                defer();
                want = false;
            }
        }
        if (!want) {
            b.lo0 = b.lo1 = b.lo2 = kBig;
            b.hi0 = b.hi1 = b.hi2 = -kBig;
        }
        const float rl = 2.f * hb * kTileListReach;
        const float r2 = want ? rl * rl : -1.f;
        const int u0 = __reduce_min_sync(kFull, b.lo0), u1 = __reduce_min_sync(kFull, b.lo1),
                  u2 = __reduce_min_sync(kFull, b.lo2);
        const int v0 = __reduce_max_sync(kFull, b.hi0), v1 = __reduce_max_sync(kFull, b.hi1),
                  v2 = __reduce_max_sync(kFull, b.hi2);
        if (u0 > v0) return;  // no group builds
        float qx[kTileGpw], qy[kTileGpw], qz[kTileGpw], qr[kTileGpw];
#pragma unroll
        for (int k = 0; k < kTileGpw; ++k) {
            qx[k] = __shfl_sync(kFull, px, k * L);
            qy[k] = __shfl_sync(kFull, py, k * L);
            qz[k] = __shfl_sync(kFull, pz, k * L);
            qr[k] = __shfl_sync(kFull, r2, k * L);
        }
        int cnt[kTileGpw] = {};
        const unsigned below = (1u << lane) - 1u;
        constexpr float w = kCellWidth;
        constexpr float iw = 1.f / kCellWidth;
        // Rows (x, y) of the union box, 32 at a time, one per lane; each row is
        // trimmed to the z cells that one of the four spheres reaches, and the
        // trimmed rows are walked as one flat sequence of staged slots, 32
        // slots per step.
        const int nyu = v1 - u1 + 1;
        const int rows = (v0 - u0 + 1) * nyu;
        for (int rb = 0; rb < rows; rb += 32) {
            const int r = rb + lane;
            uint32_t len = 0u, s0 = 0u;
            if (r < rows) {
                const int x = u0 + r / nyu, y = u1 + r % nyu;
                // the row's extent in x and y
                const float x0 = (float)(x * (1 << U)) * w, x1 = (float)((x + 1) * (1 << U)) * w;
                const float y0 = (float)(y * (1 << U)) * w, y1 = (float)((y + 1) * (1 << U)) * w;
                int zl = 0x3fffffff, zh = -0x3fffffff;
#pragma unroll
                for (int k = 0; k < kTileGpw; ++k) {
                    const float gx = fmaxf(fmaxf(x0 - qx[k], qx[k] - x1) - kCellMargin, 0.f);
                    const float gy = fmaxf(fmaxf(y0 - qy[k], qy[k] - y1) - kCellMargin, 0.f);
                    const float g2 = gx * gx + gy * gy;
                    if (g2 <= qr[k]) {
                        const float dz = sqrtf(qr[k] - g2);
                        zl = min(zl, (int)floorf((qz[k] - dz) * iw - 1e-3f) >> U);
                        zh = max(zh, (int)floorf((qz[k] + dz) * iw + 1e-3f) >> U);
                    }
                }
                zl = max(zl, u2);
                zh = min(zh, v2);
                if (zl <= zh) {
                    const int c0 = ((x - lo0) * ny + (y - lo1)) * nz;
                    s0 = S.off[c0 + (zl - lo2)];
                    len = S.off[c0 + (zh - lo2) + 1] - s0;
                }
            }
            uint32_t pre = len;  // inclusive scan of the row lengths
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(kFull, pre, o);
                if (lane >= o) pre += t;
            }
            const uint32_t excl = pre - len;
            const uint32_t total = __shfl_sync(kFull, pre, 31);
            for (uint32_t vb = 0; vb < total; vb += 32u) {
                const uint32_t v = vb + (uint32_t)lane;
                int j = 0;  // the last row whose first flat index is <= v
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const uint32_t e = __shfl_sync(kFull, excl, j + step);
                    if (e <= v) j += step;
                }
                const uint32_t sj = __shfl_sync(kFull, s0, j), ej = __shfl_sync(kFull, excl, j);
                float4 q = make_float4(3e38f, 3e38f, 3e38f, 0.f);
                const uint32_t s = sj + (v - ej);
                if (v < total) q = S.pos[s];
#pragma unroll
                for (int k = 0; k < kTileGpw; ++k) {
                    const float dx = q.x - qx[k], dy = q.y - qy[k], dz = q.z - qz[k];
                    const bool hit = dx * dx + dy * dy + dz * dz <= qr[k];
                    const unsigned bal = __ballot_sync(kFull, hit);
                    if (hit) {
                        const int at = cnt[k] + __popc(bal & below);
                        if (at < kTileList) lists[k][at] = (uint16_t)s;
                    }
                    cnt[k] += __popc(bal);
                }
            }
        }
        __syncwarp();
        if (want) {
            int c = 0;
#pragma unroll
            for (int k = 0; k < kTileGpw; ++k)
                if (g == k) c = cnt[k];
            if (c > kTileList) {
                defer();
            } else {
                n_list = c;
                list_r2 = r2;
            }
        }
    };
    bool iter = live;
    bool first = true, fell_back = false;
    int sweeps = 0, count = 0, nn = 0;
    float h2x4 = 4.f * hi * hi;
    float h1 = 1.f / hi;
    float dens = 0.f, eps = 1.f;
    float hs = hi, hs2x4 = h2x4;  // the h of the last full sweep
    while (__any_sync(kFull, iter)) {
        if (iter) {
            hs = hi;
            hs2x4 = h2x4;
        }
        const bool want = iter && (n_list < 0 || hs2x4 > list_r2);
        if (__any_sync(kFull, want)) {
            build(want, hs);
            iter = iter && live;
        }
        const int maxn = __reduce_max_sync(kFull, iter ? n_list : 0);
        float part = 0.f;
        int found = 0;
#pragma unroll 4
        for (int i = sub; i < maxn; i += L) {
            if (iter && i < n_list) {
                const float4 q = S.pos[list[i]];
                const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 <= hs2x4) {
                    const float r = pair_sqrt(r2);
                    ++found;
                    part += kernel_w(r, h1) * q.w;
                }
            }
        }
        const float dsum = group_sum<L>(part, kFull);
        const int fsum = group_sum_i<L>(found, kFull);
        if (iter) {
            dens = dsum;
            nn = min(fsum, kNeighbourCache);
            float nh = fmin_ref(kResolutionEta * powf(mi / dens, 1.f / 3), kMaxH);
            nh = 0.5f * (hi + nh);
            eps = fabsf(nh - hi) / hi;
            ++sweeps;
            if (first && seeded && eps > kSeedFallback) {
                // the seed disagrees with its own first sweep: start again from
                // the plain guess
                first = false;
                fell_back = true;
                hi = h_plain;
                h1 = 1.f / hi;
                h2x4 = 4.f * hi * hi;
                nn = 0;
                eps = 1.f;
            } else {
                first = false;
                if (eps > a.eta) {
                    if (nh >= kMaxH) {
                        defer();  // the reference's int max_h would leave 0 from here
                    } else {
                        hi = nh;
                        h1 = 1.f / hi;
                        h2x4 = 4.f * hi * hi;
                        count++;
                    }
                }
            }
            iter = live && eps > a.eta && count < kMaxNR;
        }
    }
    // gradient sweep (density.metal:145-213), as in density_particle
    const bool gcached = nn < kNeighbourCache;
    const float g2 = gcached ? hs2x4 : h2x4;
    const float h2 = hi + hi;
    {
        const bool want = live && g2 > list_r2;
        if (__any_sync(kFull, want)) build(want, gcached ? hs : hi);
    }
    const int maxn = __reduce_max_sync(kFull, live ? n_list : 0);
    const float vix = mv.x, viy = mv.y, viz = mv.z;
    float pdens = 0.f, dens_h = 0.f, vdiv = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
#pragma unroll 2
    for (int i = sub; i < maxn; i += L) {
        if (!(live && i < n_list)) continue;
        const uint32_t s = list[i];
        const float4 q = S.pos[s];
        const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > g2) continue;
        const float r = pair_sqrt(r2);
        if (gcached && r > h2) continue;
        const float mj = q.w;
        if (!gcached) pdens += kernel_w(r, h1) * mj;
        dens_h += mj * kernel_dwdh(r, h1);
        if (r > 1e-12f) {
            const float r1 = pair_rinv(r2, r);
            const float4 vj = __ldg(a.sv4 + S.gidx[s]);
            const float vx = vj.x - vix, vy = vj.y - viy, vz = vj.z - viz;
            const float sc = kernel_gradw_scale(r, h1);
            const float gx = sc * (dx * r1), gy = sc * (dy * r1), gz = sc * (dz * r1);
            vdiv += mj * (vx * gx + vy * gy + vz * gz);
            cx += mj * (vy * gz - vz * gy);
            cy += mj * (vz * gx - vx * gz);
            cz += mj * (vx * gy - vy * gx);
        }
    }
    pdens = group_sum<L>(pdens, kFull);
    dens_h = group_sum<L>(dens_h, kFull);
    vdiv = group_sum<L>(vdiv, kFull);
    cx = group_sum<L>(cx, kFull);
    cy = group_sum<L>(cy, kFull);
    cz = group_sum<L>(cz, kFull);
    if (!live || sub != 0) return;
    if (!gcached) dens += pdens;
    if (a.stats) {
        atomicAdd(&stats[0], (uint32_t)sweeps);
        if (fell_back) atomicAdd(&stats[1], 1u);
        atomicMax(&stats[2], (uint32_t)sweeps);
        atomicAdd(&stats[3], 1u);
    }
    if (a.nn_out) a.nn_out[ind] = (float)nn;
    vdiv = fabsf(vdiv) / dens;
    float acurl = sqrtf(cx * cx + cy * cy + cz * cz) / dens;
    float fi = 1.f / (1.f + (hi / (3.f * dens)) * dens_h);
    float2 pc = eos_lookup(a.eos, a.mat[ind], dens, a.u[ind]);
    float bal = vdiv / (vdiv + acurl + 1e-4f * (pc.y / hi));
    a.h[ind] = hi;
    a.rho[ind] = dens;
    a.f[ind] = fi;
    a.P[ind] = pc.x;
    a.c[ind] = pc.y;
    a.B[ind] = bal;
    if (!(dens == dens) || !(pc.x == pc.x)) raise_health(a.health, SPH_HEALTH_NAN_DENSITY);
    a.sA[p] = make_float4(px, py, pz, hi);
    a.sB[p] = make_float4(vix, viy, viz, pc.y);
    a.sC[p] = make_float4(mi, (fi * pc.x / (dens * dens)), dens, bal);
}

// The density tile pass U over the tiles of `tiles` (ctr[0] of them, ctr[1]
// the tile ticket): U = 0 the cell tiles, whose staged box counts cells;
// U = kUnitShift the coarse tiles (512-cell blocks), whose staged box counts
// 64-cell units.  Deferred particles are appended to `deferred`, counted in
// *dctr.
template <int U>
__global__ void __launch_bounds__(kTileThreads, 2)
    k_density_tile(DensityArgs a, const uint2 *__restrict__ tiles, uint32_t *ctr, uint32_t *__restrict__ deferred,
                   uint32_t *dctr) {
    extern __shared__ float4 s_tile_raw[];
    TileShared &S = *reinterpret_cast<TileShared *>(s_tile_raw);
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid < 4) S.stats[tid] = 0u;
    const uint32_t ntiles = ctr[0];
    for (;;) {
        __syncthreads();  // the previous tile is done with the staged data
        if (tid == 0) {
            const uint32_t t = atomicAdd(ctr + 1, 1u);
            S.tile = t;
            if (t < ntiles) {
                const uint2 r = tiles[t];
                S.start = r.x;
                S.end = r.y;
            }
        }
        __syncthreads();
        if (S.tile >= ntiles) break;
        const uint32_t tstart = S.start, tend = S.end;
        // a tile whose staged box overflows shared memory is taken again as
        // its octets (coarse tiles: its units), one at a time; one that still
        // overflows is handed to the per-particle pass
        constexpr int kSplit = U == 0 ? 3 : 3 * U;
        const bool splittable = (a.skey[tstart] >> kSplit) != (a.skey[tend - 1] >> kSplit);
        bool whole = true;
        uint32_t r0 = tstart;
        while (r0 < tend) {
            __syncthreads();
            if (tid == 0) {
                uint32_t r1 = tend;
                if (!whole) {  // the rest of r0's octet / unit
                    const uint32_t o = a.skey[r0] >> kSplit;
                    r1 = r0 + 1u;
                    if (U == 0) {
                        for (int j = 0; j < 8; ++j) {
                            const uint2 r = a.cells[o * 8u + (uint32_t)j];
                            if (r.x != 0xffffffffu) r1 = max(r1, r.y + 1u);
                        }
                    } else {
                        r1 = max(r1, a.units[o].y + 1u);
                    }
                }
                S.end = r1;
                S.next = 0u;
                S.box[0] = S.box[1] = S.box[2] = 0x7fffffff;
                S.box[3] = S.box[4] = S.box[5] = -0x7fffffff;
                S.defer_all = 0;
                S.need = 0;
            }
            __syncthreads();
            const uint32_t start = r0, end = S.end;
            // the staged box: union of the list boxes of the tile's active particles
            {
                int b[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, -0x7fffffff, -0x7fffffff, -0x7fffffff};
                // the warp pass is needed for this pass's particles and, in the
                // cell-tile pass, for the inactive (EOS only) and deferred ones
                bool need = false;
                for (uint32_t p = start + tid; p < end; p += kTileThreads) {
                    const uint32_t ind = a.cidx[p];
                    if (!a.active[ind]) {
                        need |= U == 0;
                        continue;
                    }
                    const float4 me = a.sp4[p];
                    const float h_plain = a.h[ind];
                    bool seeded;
                    const float h0 = tile_start_h(a, ind, h_plain, seeded);
                    const float hb = fmaxf(h0, h_plain);
                    const int m = density_mode(me.x, me.y, me.z, hb, a.coarse);
                    if (U == 0 && m == kUnitShift) a.cflags[a.skey[p] >> (3 * kUnitShift + 3)] = 1;
                    need |= m == U || (U == 0 && m < 0);
                    if (m != U) continue;
                    CellBox cb;
                    tile_box(me.x, me.y, me.z, hb, cb, fmaxf(kTileStageReach, kTileListReach));
                    b[0] = min(b[0], cb.lo0 >> U);
                    b[1] = min(b[1], cb.lo1 >> U);
                    b[2] = min(b[2], cb.lo2 >> U);
                    b[3] = max(b[3], cb.hi0 >> U);
                    b[4] = max(b[4], cb.hi1 >> U);
                    b[5] = max(b[5], cb.hi2 >> U);
                }
    #pragma unroll
                for (int k = 0; k < 3; ++k) {
                    b[k] = __reduce_min_sync(0xffffffffu, b[k]);
                    b[k + 3] = __reduce_max_sync(0xffffffffu, b[k + 3]);
                }
                if (__any_sync(0xffffffffu, need) && lane == 0) S.need = 1;
                if (lane == 0) {
    #pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        atomicMin(&S.box[k], b[k]);
                        atomicMax(&S.box[k + 3], b[k + 3]);
                    }
                }
            }
            __syncthreads();
            const int lo0 = S.box[0], lo1 = S.box[1], lo2 = S.box[2];
            const bool any = lo0 <= S.box[3];  // some particle of the tile takes the tile path
            const int nx = any ? S.box[3] - lo0 + 1 : 0, ny = any ? S.box[4] - lo1 + 1 : 0,
                      nz = any ? S.box[5] - lo2 + 1 : 0;
            int ncell = 0;
            if (any) {
                if (nx * ny * nz > kTileCellsMax) {
                    if (tid == 0) S.defer_all = 1;
                } else {
                    ncell = nx * ny * nz;
                }
            }
            // cell counts (kTileCellsPerThread consecutive cells per thread) and
            // their exclusive scan
            uint32_t c_cnt[kTileCellsPerThread];
            uint32_t tsum = 0u;
    #pragma unroll
            for (int k = 0; k < kTileCellsPerThread; ++k) {
                const int c = kTileCellsPerThread * tid + k;
                c_cnt[k] = 0u;
                if (c < ncell) {
                    const int ix = c / (ny * nz), rem = c - ix * ny * nz, iy = rem / nz, iz = rem - iy * nz;
                    const uint2 r = unit_range<U>(a.cells, a.units, lo0 + ix, lo1 + iy, lo2 + iz);
                    if (r.x != 0xffffffffu) {
                        c_cnt[k] = r.y - r.x + 1u;
                        S.first[c] = r.x;
                    }
                }
                tsum += c_cnt[k];
            }
            uint32_t inc = tsum;
    #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (lane == 31) S.wsum[tid >> 5] = inc;
            __syncthreads();
            uint32_t wbase = 0u;
            for (int w = 0; w < (tid >> 5); ++w) wbase += S.wsum[w];
            uint32_t run = wbase + inc - tsum;
    #pragma unroll
            for (int k = 0; k < kTileCellsPerThread; ++k) {
                const int c = kTileCellsPerThread * tid + k;
                if (c < ncell) S.off[c] = run;
                run += c_cnt[k];
            }
            if (tid == kTileThreads - 1) {
                S.off[ncell] = run;
                if (run > (uint32_t)kTileStageMax) S.defer_all = 1;
            }
            __syncthreads();
            if (S.defer_all && whole && splittable) {
                whole = false;
                continue;
            }
            if (!S.defer_all) {
                const uint32_t total = S.off[ncell];
                for (uint32_t s = tid; s < total; s += kTileThreads) {
                    int lo = 0, hi = ncell - 1;  // the last cell whose first slot is <= s
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (S.off[mid] <= s) lo = mid;
                        else hi = mid - 1;
                    }
                    const uint32_t g = S.first[lo] + (s - S.off[lo]);
                    S.pos[s] = __ldg(a.sp4 + g);
                    S.gidx[s] = g;
                }
            }
            __syncthreads();
            // warps take the tile's particles four at a time (none when no
            // particle of the range needs this pass)
            for (bool more = S.need != 0; more;) {
                uint32_t j = 0u;
                if (lane == 0) j = atomicAdd(&S.next, (uint32_t)kTileGpw);
                j = __shfl_sync(0xffffffffu, j, 0);
                more = start + j < end;
                if (!more) break;
                density_tile_warp<U>(a, S, S.stats, start + j, end, lane, &S.list[(tid >> 5) * kTileGpw], deferred,
                                     dctr);
            }
            r0 = end;
        }
    }
    if (a.stats && tid == 0) {
        if (S.stats[3]) {
            atomicAdd(a.stats + 0, S.stats[0]);
            if (S.stats[1]) atomicAdd(a.stats + 1, S.stats[1]);
            atomicMax(a.stats + 2, S.stats[2]);
            atomicAdd(a.stats + 3, S.stats[3]);
        }
    }
}

struct AccelArgs {
    int n;
    const uint32_t *cidx;
    const uint32_t *skey;  // sorted cell keys (tile passes)
    const uint2 *cells;
    const uint2 *units;    // 64-cell unit ranges (coarse tiles)
    uint8_t *cflags;       // per 512-cell block: holds a coarse-tile particle
    int coarse;            // coarse tiles on
    const float4 *sA, *sB, *sC;
    float4 *acc4;
    float *du, *dhdt;
    int32_t *nat;
    const uint8_t *active;
    int32_t *globals;
    int individual;  // SPH_TIMESTEP_INDIVIDUAL: inactive particles bound the global step
};

// The ticks an inactive particle allows the global step: INT_MAX with the
// reference's test (all particles active anyway); with individual timesteps
// the time left to its next active time, so no step passes it.
__device__ __forceinline__ int inactive_ticks(const AccelArgs &a, uint32_t ind) {
    if (!a.individual) return 0x7fffffff;
    return max(a.nat[ind] - a.globals[0], 1);
}

// The particle's own terms of accelerations.metal:60-141.
struct AccelI {
    float xi, yi, zi, hi, vxi, vyi, vzi, ci, facti, rhoi, Bi, hi1, hi2x4;
};
__device__ __forceinline__ AccelI accel_i(const float4 A, const float4 Bv, const float4 Cv) {
    AccelI I;
    I.xi = A.x;
    I.yi = A.y;
    I.zi = A.z;
    I.hi = A.w;
    I.vxi = Bv.x;
    I.vyi = Bv.y;
    I.vzi = Bv.z;
    I.ci = Bv.w;
    I.facti = Cv.y;
    I.rhoi = Cv.z;
    I.Bi = Cv.w;
    I.hi1 = 1.f / I.hi;
    I.hi2x4 = I.hi * I.hi * 4.f;
    return I;
}
// Running sums of one particle (a slice of its pairs): acceleration, du/dt,
// dh/dt, with Kahan compensations in the mixed-precision form, and the
// largest signal speed.
struct AccelSum {
    float dvx = 0.f, dvy = 0.f, dvz = 0.f, du = 0.f, dh = 0.f;
    float kx = 0.f, ky = 0.f, kz = 0.f, ku = 0.f, kh = 0.f;
    float vsig = 1e-12f;
};
template <bool KAHAN>
__device__ __forceinline__ void accel_add(float &sum, float &comp, float v) {
    if (KAHAN) {
        const float y = v - comp;
        const float t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    } else {
        sum += v;
    }
}
// accelerations.metal:75-124: one accepted pair (Aj = (x, y, z, h),
// Bj = (v, c), Cj = (m, f P / rho^2, rho, B) of the neighbour).
template <bool KAHAN>
__device__ __forceinline__ void accel_pair(const AccelI &I, AccelSum &S, const float4 Aj, const float4 Bj,
                                           const float4 Cj) {
    const float dx = I.xi - Aj.x, dy = I.yi - Aj.y, dz = I.zi - Aj.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float hj = Aj.w;
    const float r = pair_sqrt(r2);
    const float r1 = pair_rinv(r2, r);
    const float mj = Cj.x, factj = Cj.y, rhoj = Cj.z, Balj = Cj.w;
    const float hj1 = pdiv(1.f, hj);
    const float vx = I.vxi - Bj.x, vy = I.vyi - Bj.y, vz = I.vzi - Bj.z;
    const float rhoij = 0.5f * (I.rhoi + rhoj);
    const float vdr = vx * dx + vy * dy + vz * dz;
    const float mu = vdr < 0.f ? vdr * r1 : 0.f;
    const float vsig = I.ci + Bj.w - 3.f * mu;
    S.vsig = fmax_ref(vsig, S.vsig);
    const float Bij = 0.5f * (I.Bi + Balj);
    const float nu = pdiv(-0.5f * kViscosityAlpha * Bij * mu * vsig, rhoij);
    const float rhx = dx * r1, rhy = dy * r1, rhz = dz * r1;
    const float si = kernel_gradw_scale(r, I.hi1), sj = kernel_gradw_scale(r, hj1);
    const float gix = si * rhx, giy = si * rhy, giz = si * rhz;
    const float gjx = sj * rhx, gjy = sj * rhy, gjz = sj * rhz;
    const float gx = 0.5f * (gix + gjx), gy = 0.5f * (giy + gjy), gz = 0.5f * (giz + gjz);
    accel_add<KAHAN>(S.dvx, S.kx, -(mj * (I.facti * gix + factj * gjx + nu * gx)));
    accel_add<KAHAN>(S.dvy, S.ky, -(mj * (I.facti * giy + factj * gjy + nu * gy)));
    accel_add<KAHAN>(S.dvz, S.kz, -(mj * (I.facti * giz + factj * gjz + nu * gz)));
    accel_add<KAHAN>(S.du, S.ku,
                     mj * (I.facti * (vx * gix + vy * giy + vz * giz) + 0.5f * nu * (vx * gx + vy * gy + vz * gz)));
    accel_add<KAHAN>(S.dh, S.kh, pdiv(mj, rhoj) * (vx * gix + vy * giy + vz * giz));
}
// The group's sums combined (every lane ends with the same bits).
template <int L, bool KAHAN>
__device__ __forceinline__ void accel_reduce(AccelSum &S, unsigned gm) {
    if (KAHAN) {
        S.dvx -= S.kx;
        S.dvy -= S.ky;
        S.dvz -= S.kz;
        S.du -= S.ku;
        S.dh -= S.kh;
    }
    S.dvx = group_sum<L>(S.dvx, gm);
    S.dvy = group_sum<L>(S.dvy, gm);
    S.dvz = group_sum<L>(S.dvz, gm);
    S.du = group_sum<L>(S.du, gm);
    S.dh = group_sum<L>(S.dh, gm);
    S.vsig = group_max<L>(S.vsig, gm);
}
// accelerations.metal:129-140: the particle's timestep in ticks.
__device__ __forceinline__ int accel_ticks(const AccelI &I, float vsig) {
    const float goal = 2.0f * kCFL * kGamma * I.hi / vsig;
    int r = 0;
    float cand = kDT0;
    while (cand > goal && r < kRMax) {
        cand *= 0.5f;
        r++;
    }
    return (int)ceilf(1 / kDtMin1 * cand);
}
__device__ __forceinline__ void accel_store(const AccelArgs &a, uint32_t ind, const AccelSum &S, int idt) {
    float4 acc = a.acc4[ind];
    acc.x += S.dvx;
    acc.y += S.dvy;
    acc.z += S.dvz;
    a.acc4[ind] = acc;
    a.du[ind] = S.du;
    a.dhdt[ind] = S.dh;
    a.nat[ind] = a.globals[0] + idt;
}

// accelerations.metal:12-141 for one sorted particle per lane group.  The
// walk covers the particle's own box of radius 2 min(h, MAX_SMOOTHING_LENGTH)
// (the reference's box, which also decides which pairs with r < 2 h_j are
// seen, Q8).  The pairs that pass the reference's test are first collected in
// order into the group's list, then evaluated by all lanes of the group
// together, so the long pair computation runs with every lane busy.  Returns
// the particle's timestep in ticks (INT_MAX when inactive).
template <int L, bool KAHAN>
__device__ __forceinline__ int accel_particle(const AccelArgs &a, int index, int sub, unsigned gm, int gbase,
                                              uint32_t *w_off, uint32_t *w_start, uint32_t *list) {
    const uint32_t ind = a.cidx[index];
    if (!a.active[ind]) return inactive_ticks(a, ind);
    const AccelI I = accel_i(a.sA[index], a.sB[index], a.sC[index]);
    AccelSum S;
    const float4 *sA = a.sA, *sB = a.sB, *sC = a.sC;
    auto drain = [&](int cnt) {
        __syncwarp(gm);
        for (int i = sub; i < cnt; i += L) {
            const uint32_t k = list[i];
            accel_pair<KAHAN>(I, S, __ldg(sA + k), __ldg(sB + k), __ldg(sC + k));
        }
        __syncwarp(gm);
        return true;
    };
    const int rest = group_collect<L>(
        I.xi, I.yi, I.zi, fmin_ref(I.hi, kMaxH), 3.402823466e+38f, a.cells, sub, gm, gbase, w_off, w_start, list,
        kListMax,
        [&](uint32_t k) {
            const float4 Aj = __ldg(sA + k);
            const float dx = I.xi - Aj.x, dy = I.yi - Aj.y, dz = I.zi - Aj.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            const float hj2x4 = Aj.w * Aj.w * 4.f;
            return !((r2 > I.hi2x4 && r2 > hj2x4) || r2 < 1e-12f);
        },
        drain);
    drain(rest);
    accel_reduce<L, KAHAN>(S, gm);
    const int idt = accel_ticks(I, S.vsig);
    if (sub == 0) accel_store(a, ind, S, idt);
    return idt;
}

// Block-wide minimum of the timesteps, then one atomic per block.
__device__ __forceinline__ void block_min_dt(int idt, int32_t *dt) {
    __shared__ int wmin[32];
    const int lane = threadIdx.x & 31;
    for (int o = 16; o > 0; o >>= 1) idt = min(idt, __shfl_xor_sync(0xffffffffu, idt, o));
    if (lane == 0) wmin[threadIdx.x >> 5] = idt;
    __syncthreads();
    if (threadIdx.x < 32) {
        int v = (threadIdx.x < ((blockDim.x + 31) >> 5)) ? wmin[threadIdx.x] : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0 && v != 0x7fffffff) atomicMin(dt, v);
    }
}

template <int L, bool KAHAN>
__global__ void __launch_bounds__(parts_per_block<L>() * L) k_acceleration(AccelArgs a) {
    extern __shared__ uint32_t s_lists[];
    __shared__ uint32_t s_off[parts_per_block<L>() * L], s_start[parts_per_block<L>() * L];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, sub = lane & (L - 1), gbase = lane & ~(L - 1);
    const int index = t / L;
    int idt = 0x7fffffff;
    if (index < a.n)
        idt = accel_particle<L, KAHAN>(a, index, sub, group_mask<L>(lane), gbase, s_off + (threadIdx.x & ~31),
                                       s_start + (threadIdx.x & ~31),
                                       s_lists + (size_t)(threadIdx.x / L) * kListMax);
    block_min_dt(idt, a.globals + 1);
}

// The particles the tile pass handed on (sorted indices idx[0, *count)).
template <int L, bool KAHAN>
__global__ void __launch_bounds__(parts_per_block<L>() * L)
    k_acceleration_deferred(AccelArgs a, const uint32_t *__restrict__ idx, const uint32_t *__restrict__ count) {
    extern __shared__ uint32_t s_lists[];
    __shared__ uint32_t s_off[parts_per_block<L>() * L], s_start[parts_per_block<L>() * L];
    const int lane = threadIdx.x & 31, sub = lane & (L - 1), gbase = lane & ~(L - 1);
    const uint32_t cnt = *count;
    constexpr int per_block = parts_per_block<L>();
    int idt = 0x7fffffff;
    for (uint32_t base = blockIdx.x * per_block; base < cnt; base += gridDim.x * per_block) {
        const uint32_t j = base + threadIdx.x / L;
        if (j < cnt)
            idt = min(idt, accel_particle<L, KAHAN>(a, (int)idx[j], sub, group_mask<L>(lane), gbase,
                                                    s_off + (threadIdx.x & ~31), s_start + (threadIdx.x & ~31),
                                                    s_lists + (size_t)(threadIdx.x / L) * kListMax));
    }
    block_min_dt(idt, a.globals + 1);
}

// ---- acceleration over cell tiles (product build) ---------------------------
//
// The tiles of the density pass (k_tile_starts), staged the same way with the
// sA records (x, y, z, h) of the union of the tile particles' boxes of radius
// 2 min(h, MAX_H) -- the reference's box, exact (cell_box) -- plus each staged
// particle's cell within the staged box.  Warps take four particles at a time:
// the transposed list build walks the rows of the four boxes as one flat
// sequence and keeps a pair when r <= 2 h_i, or when r <= 2 h_j and the
// neighbour's cell lies in the particle's box (the reference sees such a pair
// only there, Q8); then the pair arithmetic runs over the lists with every
// lane busy, reading the neighbour's sB / sC records by its sorted index.
// Particles whose box reaches more than kTileReach cells past their own cell,
// whose list overflows, and every particle of a tile whose staged box exceeds
// the budget go to k_acceleration_deferred.
constexpr int kTileAccStage = 3072;  // staged particles per tile

struct TileAccShared {
    float4 pos[kTileAccStage];          // staged sA (x, y, z, h)
    uint32_t gidx[kTileAccStage];       // staged sorted index
    uint32_t scell[kTileAccStage];      // staged cell, box-relative: x | y << 10 | z << 20
    uint32_t off[kTileCellsMax + 1];
    uint32_t first[kTileCellsMax];
    uint16_t list[kTileGroups][kTileList];
    int gbox[kTileGroups][6];           // each group's box, box-relative lo xyz, hi xyz
    int box[6];
    uint32_t wsum[kTileThreads / 32];
    uint32_t start, end, tile, next;
    int defer_all;
    int need;                           // some particle of the range needs the warp pass
    int dtmin;
    int hmax_bits;                      // largest staged h (float bits; h > 0)
};

// The reference's box of an acceleration particle (cells) and the pass that
// takes it: 0 the cell tiles (reach within kTileReach cells of its own),
// kUnitShift the coarse tiles (within kTileReach units), -1 the per-particle
// pass (h at MAX_H, or coarse tiles off).
__device__ __forceinline__ int accel_mode(float px, float py, float pz, float h, CellBox &b, int coarse) {
    b = cell_box(px, py, pz, fmin_ref(h, kMaxH));
    if (!(h < kMaxH)) return -1;
    const int ox = (int)floorf(__fdiv_rn(px, kCellWidth)), oy = (int)floorf(__fdiv_rn(py, kCellWidth)),
              oz = (int)floorf(__fdiv_rn(pz, kCellWidth));
    if (within_reach<0>(ox, oy, oz, b)) return 0;
    if (coarse && within_reach<kUnitShift>(ox, oy, oz, b)) return kUnitShift;
    return -1;
}

// One warp: the acceleration pass of sorted particles p0 .. p0 + 3 of the
// staged tile (lane group g takes p0 + g) whose pass is U (the staged box
// counts U-units; the group boxes and staged cells stay in cells, relative to
// the box's first cell).  Returns the warp's smallest timestep in ticks
// (INT_MAX when none).
template <bool KAHAN, int U>
__device__ __forceinline__ int accel_tile_warp(const AccelArgs &a, TileAccShared &S, uint32_t p0, uint32_t end,
                                               int lane, int wslot, uint32_t *deferred, uint32_t *dctr) {
    constexpr int L = kTileLanes;
    constexpr unsigned kFull = 0xffffffffu;
    constexpr int kBig = 0x3fffffff;
    const int g = lane / L, sub = lane & (L - 1);
    uint16_t *list = S.list[wslot * kTileGpw + g];
    const uint32_t p = p0 + (uint32_t)g;
    bool live = p < end;
    uint32_t ind = 0u;
    int idt_inactive = 0x7fffffff;
    if (live) {
        ind = a.cidx[p];
        live = a.active[ind] != 0;
        if (!live && U == 0) idt_inactive = inactive_ticks(a, ind);
    }
    float4 A = make_float4(0.f, 0.f, 0.f, 1.f), Bv = A, Cv = A;
    if (live) {
        A = a.sA[p];
        Bv = a.sB[p];
        Cv = a.sC[p];
    }
    const AccelI I = accel_i(A, Bv, Cv);
    const int lo0 = S.box[0], lo1 = S.box[1], lo2 = S.box[2];
    const int ny = S.box[4] - lo1 + 1, nz = S.box[5] - lo2 + 1;
    CellBox b;
    bool want = false;
    if (live) {
        const int m = accel_mode(I.xi, I.yi, I.zi, I.hi, b, a.coarse);
        if (m != U) {
            if (U == 0 && m < 0 && sub == 0) deferred[atomicAdd(dctr, 1u)] = p;
            live = false;  // deferred, or another tile pass takes it
        } else if (S.defer_all) {
            if (sub == 0) deferred[atomicAdd(dctr, 1u)] = p;
            live = false;
        } else {
            want = true;
        }
    }
    if (!want) {
        b.lo0 = b.lo1 = b.lo2 = kBig;
        b.hi0 = b.hi1 = b.hi2 = -kBig;
    }
    if (want && sub == 0) {
        int *gb = S.gbox[wslot * kTileGpw + g];
        gb[0] = b.lo0 - lo0 * (1 << U);
        gb[1] = b.lo1 - lo1 * (1 << U);
        gb[2] = b.lo2 - lo2 * (1 << U);
        gb[3] = b.hi0 - lo0 * (1 << U);
        gb[4] = b.hi1 - lo1 * (1 << U);
        gb[5] = b.hi2 - lo2 * (1 << U);
    }
    const int u0 = __reduce_min_sync(kFull, b.lo0) >> U, u1 = __reduce_min_sync(kFull, b.lo1) >> U,
              u2 = __reduce_min_sync(kFull, b.lo2) >> U;
    const int v0 = __reduce_max_sync(kFull, b.hi0) >> U, v1 = __reduce_max_sync(kFull, b.hi1) >> U,
              v2 = __reduce_max_sync(kFull, b.hi2) >> U;
    if (u0 > v0) return __reduce_min_sync(kFull, idt_inactive);  // no active particle takes the tile path
    __syncwarp();
    // every accepted pair lies within 2 max(h_i, largest staged h) of the particle
    const float hm = fmaxf(I.hi, __int_as_float(S.hmax_bits));
    float qx[kTileGpw], qy[kTileGpw], qz[kTileGpw], qr[kTileGpw], qR[kTileGpw];
#pragma unroll
    for (int k = 0; k < kTileGpw; ++k) {
        qx[k] = __shfl_sync(kFull, I.xi, k * L);
        qy[k] = __shfl_sync(kFull, I.yi, k * L);
        qz[k] = __shfl_sync(kFull, I.zi, k * L);
        qr[k] = __shfl_sync(kFull, want ? I.hi2x4 : -1.f, k * L);
        qR[k] = __shfl_sync(kFull, want ? 4.f * hm * hm : -1.f, k * L);
    }
    // box bounds of the four groups, for the row test (lane k * L holds group k's)
    int cnt[kTileGpw] = {};
    const unsigned below = (1u << lane) - 1u;
    const int nyu = v1 - u1 + 1;
    const int rows = (v0 - u0 + 1) * nyu;
    for (int rb = 0; rb < rows; rb += 32) {
        const int r = rb + lane;
        uint32_t len = 0u, s0 = 0u;
        int zl = kBig, zh = -kBig;
        int x = 0, y = 0;
        if (r < rows) {
            x = u0 + r / nyu;
            y = u1 + r % nyu;
        }
        // the z range of the boxes that contain row (x, y), trimmed to the
        // sphere that holds every accepted pair
        constexpr float w = kCellWidth;
        constexpr float iw = 1.f / kCellWidth;
        const float x0 = (float)(x * (1 << U)) * w, x1 = (float)((x + 1) * (1 << U)) * w;
        const float y0 = (float)(y * (1 << U)) * w, y1 = (float)((y + 1) * (1 << U)) * w;
#pragma unroll
        for (int k = 0; k < kTileGpw; ++k) {
            // group k's box in U-units (empty boxes stay empty: kBig >> U > -kBig >> U)
            const int bl0 = __shfl_sync(kFull, b.lo0, k * L) >> U, bh0 = __shfl_sync(kFull, b.hi0, k * L) >> U;
            const int bl1 = __shfl_sync(kFull, b.lo1, k * L) >> U, bh1 = __shfl_sync(kFull, b.hi1, k * L) >> U;
            const int bl2 = __shfl_sync(kFull, b.lo2, k * L) >> U, bh2 = __shfl_sync(kFull, b.hi2, k * L) >> U;
            if (r < rows && x >= bl0 && x <= bh0 && y >= bl1 && y <= bh1) {
                const float gx = fmaxf(fmaxf(x0 - qx[k], qx[k] - x1) - kCellMargin, 0.f);
                const float gy = fmaxf(fmaxf(y0 - qy[k], qy[k] - y1) - kCellMargin, 0.f);
                const float g2 = gx * gx + gy * gy;
                if (g2 <= qR[k]) {
                    const float dz = sqrtf(qR[k] - g2);
                    zl = min(zl, max(bl2, (int)floorf((qz[k] - dz) * iw - 1e-3f) >> U));
                    zh = max(zh, min(bh2, (int)floorf((qz[k] + dz) * iw + 1e-3f) >> U));
                }
            }
        }
        if (zl <= zh) {
            const int c0 = ((x - lo0) * ny + (y - lo1)) * nz;
            s0 = S.off[c0 + (zl - lo2)];
            len = S.off[c0 + (zh - lo2) + 1] - s0;
        }
        uint32_t pre = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, pre, o);
            if (lane >= o) pre += t;
        }
        const uint32_t excl = pre - len;
        const uint32_t total = __shfl_sync(kFull, pre, 31);
        for (uint32_t vb = 0; vb < total; vb += 32u) {
            const uint32_t v = vb + (uint32_t)lane;
            int j = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const uint32_t e = __shfl_sync(kFull, excl, j + step);
                if (e <= v) j += step;
            }
            const uint32_t sj = __shfl_sync(kFull, s0, j), ej = __shfl_sync(kFull, excl, j);
            const uint32_t s = sj + (v - ej);
            float4 q = make_float4(3e38f, 3e38f, 3e38f, 0.f);
            uint32_t sc = 0u;
            if (v < total) {
                q = S.pos[s];
                sc = S.scell[s];
            }
            const float hj2x4 = q.w * q.w * 4.f;
#pragma unroll
            for (int k = 0; k < kTileGpw; ++k) {
                const float dx = qx[k] - q.x, dy = qy[k] - q.y, dz = qz[k] - q.z;
                const float r2 = dx * dx + dy * dy + dz * dz;
                const bool near = r2 >= 1e-12f;
                bool hit = near && r2 <= qr[k];
                // r > 2 h_i but r <= 2 h_j: only when the neighbour's cell is in the box
                const bool maybe = near && !hit && qr[k] >= 0.f && r2 <= hj2x4;
                if (__any_sync(kFull, maybe)) {
                    const int *gb = S.gbox[wslot * kTileGpw + k];
                    const int cx = (int)(sc & 1023u), cy = (int)((sc >> 10) & 1023u), cz = (int)(sc >> 20);
                    if (maybe && cx >= gb[0] && cx <= gb[3] && cy >= gb[1] && cy <= gb[4] && cz >= gb[2] &&
                        cz <= gb[5])
                        hit = true;
                }
                const unsigned bal = __ballot_sync(kFull, hit);
                if (hit) {
                    const int at = cnt[k] + __popc(bal & below);
                    if (at < kTileList) S.list[wslot * kTileGpw + k][at] = (uint16_t)s;
                }
                cnt[k] += __popc(bal);
            }
        }
    }
    __syncwarp();
    int n_list = 0;
#pragma unroll
    for (int k = 0; k < kTileGpw; ++k)
        if (g == k) n_list = cnt[k];
    if (live && n_list > kTileList) {
        if (sub == 0) deferred[atomicAdd(dctr, 1u)] = p;
        live = false;
    }
    const int maxn = __reduce_max_sync(kFull, live ? n_list : 0);
    AccelSum Sm;
#pragma unroll 2
    for (int i = sub; i < maxn; i += L) {
        if (live && i < n_list) {
            const uint32_t s = list[i];
            const uint32_t gj = S.gidx[s];
            accel_pair<KAHAN>(I, Sm, S.pos[s], __ldg(a.sB + gj), __ldg(a.sC + gj));
        }
    }
    accel_reduce<L, KAHAN>(Sm, kFull);
    int idt = idt_inactive;
    if (live) {
        idt = accel_ticks(I, Sm.vsig);
        if (sub == 0) accel_store(a, ind, Sm, idt);
    }
    return __reduce_min_sync(kFull, idt);
}

// The acceleration tile pass U over `tiles` (ctr[0] of them, ctr[1] the
// ticket), as k_density_tile; deferred particles are counted in *dctr.
template <bool KAHAN, int U>
__global__ void __launch_bounds__(kTileThreads, 2)
    k_acceleration_tile(AccelArgs a, const uint2 *__restrict__ tiles, uint32_t *ctr, uint32_t *__restrict__ deferred,
                        uint32_t *dctr) {
    extern __shared__ float4 s_tile_raw[];
    TileAccShared &S = *reinterpret_cast<TileAccShared *>(s_tile_raw);
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) S.dtmin = 0x7fffffff;
    const uint32_t ntiles = ctr[0];
    for (;;) {
        __syncthreads();
        if (tid == 0) {
            const uint32_t t = atomicAdd(ctr + 1, 1u);
            S.tile = t;
            if (t < ntiles) {
                const uint2 r = tiles[t];
                S.start = r.x;
                S.end = r.y;
            }
        }
        __syncthreads();
        if (S.tile >= ntiles) break;
        const uint32_t tstart = S.start, tend = S.end;
        // a tile whose staged box overflows shared memory is taken again as
        // its octets (coarse tiles: its units), one at a time; one that still
        // overflows is handed to the per-particle pass
        constexpr int kSplit = U == 0 ? 3 : 3 * U;
        const bool splittable = (a.skey[tstart] >> kSplit) != (a.skey[tend - 1] >> kSplit);
        bool whole = true;
        uint32_t r0 = tstart;
        while (r0 < tend) {
            __syncthreads();
            if (tid == 0) {
                uint32_t r1 = tend;
                if (!whole) {  // the rest of r0's octet / unit
                    const uint32_t o = a.skey[r0] >> kSplit;
                    r1 = r0 + 1u;
                    if (U == 0) {
                        for (int j = 0; j < 8; ++j) {
                            const uint2 r = a.cells[o * 8u + (uint32_t)j];
                            if (r.x != 0xffffffffu) r1 = max(r1, r.y + 1u);
                        }
                    } else {
                        r1 = max(r1, a.units[o].y + 1u);
                    }
                }
                S.end = r1;
                S.next = 0u;
                S.box[0] = S.box[1] = S.box[2] = 0x7fffffff;
                S.box[3] = S.box[4] = S.box[5] = -0x7fffffff;
                S.defer_all = 0;
                S.need = 0;
                S.hmax_bits = 0;
            }
            __syncthreads();
            const uint32_t start = r0, end = S.end;
            {
                int b[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, -0x7fffffff, -0x7fffffff, -0x7fffffff};
                // the warp pass is needed for this pass's particles and, in the
                // cell-tile pass, for the inactive (their next active time bounds
                // the step) and deferred ones
                bool need = false;
                for (uint32_t p = start + tid; p < end; p += kTileThreads) {
                    if (!a.active[a.cidx[p]]) {
                        need |= U == 0;
                        continue;
                    }
                    const float4 A = a.sA[p];
                    CellBox cb;
                    const int m = accel_mode(A.x, A.y, A.z, A.w, cb, a.coarse);
                    if (U == 0 && m == kUnitShift) a.cflags[a.skey[p] >> (3 * kUnitShift + 3)] = 1;
                    need |= m == U || (U == 0 && m < 0);
                    if (m != U) continue;
                    b[0] = min(b[0], cb.lo0 >> U);
                    b[1] = min(b[1], cb.lo1 >> U);
                    b[2] = min(b[2], cb.lo2 >> U);
                    b[3] = max(b[3], cb.hi0 >> U);
                    b[4] = max(b[4], cb.hi1 >> U);
                    b[5] = max(b[5], cb.hi2 >> U);
                }
    #pragma unroll
                for (int k = 0; k < 3; ++k) {
                    b[k] = __reduce_min_sync(0xffffffffu, b[k]);
                    b[k + 3] = __reduce_max_sync(0xffffffffu, b[k + 3]);
                }
                if (__any_sync(0xffffffffu, need) && lane == 0) S.need = 1;
                if (lane == 0) {
    #pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        atomicMin(&S.box[k], b[k]);
                        atomicMax(&S.box[k + 3], b[k + 3]);
                    }
                }
            }
            __syncthreads();
            const int lo0 = S.box[0], lo1 = S.box[1], lo2 = S.box[2];
            const bool any = lo0 <= S.box[3];
            const int nx = any ? S.box[3] - lo0 + 1 : 0, ny = any ? S.box[4] - lo1 + 1 : 0,
                      nz = any ? S.box[5] - lo2 + 1 : 0;
            int ncell = 0;
            if (any) {
                if (nx * ny * nz > kTileCellsMax) {
                    if (tid == 0) S.defer_all = 1;
                } else {
                    ncell = nx * ny * nz;
                }
            }
            uint32_t c_cnt[kTileCellsPerThread];
            uint32_t tsum = 0u;
    #pragma unroll
            for (int k = 0; k < kTileCellsPerThread; ++k) {
                const int c = kTileCellsPerThread * tid + k;
                c_cnt[k] = 0u;
                if (c < ncell) {
                    const int ix = c / (ny * nz), rem = c - ix * ny * nz, iy = rem / nz, iz = rem - iy * nz;
                    const uint2 r = unit_range<U>(a.cells, a.units, lo0 + ix, lo1 + iy, lo2 + iz);
                    if (r.x != 0xffffffffu) {
                        c_cnt[k] = r.y - r.x + 1u;
                        S.first[c] = r.x;
                    }
                }
                tsum += c_cnt[k];
            }
            uint32_t inc = tsum;
    #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (lane == 31) S.wsum[tid >> 5] = inc;
            __syncthreads();
            uint32_t wbase = 0u;
            for (int w = 0; w < (tid >> 5); ++w) wbase += S.wsum[w];
            uint32_t run = wbase + inc - tsum;
    #pragma unroll
            for (int k = 0; k < kTileCellsPerThread; ++k) {
                const int c = kTileCellsPerThread * tid + k;
                if (c < ncell) S.off[c] = run;
                run += c_cnt[k];
            }
            if (tid == kTileThreads - 1) {
                S.off[ncell] = run;
                if (run > (uint32_t)kTileAccStage) S.defer_all = 1;
            }
            __syncthreads();
            if (S.defer_all && whole && splittable) {
                whole = false;
                continue;
            }
            float hmax = 0.f;
            if (!S.defer_all) {
                const uint32_t total = S.off[ncell];
                for (uint32_t s = tid; s < total; s += kTileThreads) {
                    int lo = 0, hi = ncell - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (S.off[mid] <= s) lo = mid;
                        else hi = mid - 1;
                    }
                    const uint32_t gi = S.first[lo] + (s - S.off[lo]);
                    const float4 q = __ldg(a.sA + gi);
                    S.pos[s] = q;
                    S.gidx[s] = gi;
                    int ix = lo / (ny * nz), rem = lo - ix * ny * nz, iy = rem / nz, iz = rem - iy * nz;
                    if (U > 0) {
                        // the particle's cell within its unit: the low 3U bits of its key
                        const uint32_t key = a.skey[gi];
                        int dx = 0, dy = 0, dz = 0;
#pragma unroll
                        for (int bit = 0; bit < U; ++bit) {
                            dx |= (int)((key >> (3 * bit)) & 1u) << bit;
                            dy |= (int)((key >> (3 * bit + 1)) & 1u) << bit;
                            dz |= (int)((key >> (3 * bit + 2)) & 1u) << bit;
                        }
                        ix = (ix << U) | dx;
                        iy = (iy << U) | dy;
                        iz = (iz << U) | dz;
                    }
                    S.scell[s] = (uint32_t)ix | ((uint32_t)iy << 10) | ((uint32_t)iz << 20);
                    hmax = fmaxf(hmax, q.w);
                }
            }
            {
                float v = hmax;
    #pragma unroll
                for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
                if (lane == 0 && v > 0.f) atomicMax(&S.hmax_bits, __float_as_int(v));
            }
            __syncthreads();
            int wmin = 0x7fffffff;
            for (bool more = S.need != 0; more;) {  // none when no particle of the range needs this pass
                uint32_t j = 0u;
                if (lane == 0) j = atomicAdd(&S.next, (uint32_t)kTileGpw);
                j = __shfl_sync(0xffffffffu, j, 0);
                more = start + j < end;
                if (!more) break;
                wmin = min(wmin, accel_tile_warp<KAHAN, U>(a, S, start + j, end, lane, tid >> 5, deferred, dctr));
            }
            if (lane == 0 && wmin != 0x7fffffff) atomicMin(&S.dtmin, wmin);
            r0 = end;
        }
    }
    if (tid == 0 && S.dtmin != 0x7fffffff) atomicMin(a.globals + 1, S.dtmin);
}

struct StepArgs {
    int n;
    float4 *pos4, *vel4;
    const float4 *acc4;
    float *rho, *u, *h;
    const float *du, *dhdt;
    int32_t *globals;
    double4 *pos64;  // mixed-precision form: FP64 master positions
    double *dglob;   // mixed-precision form: [0] global time in seconds
};

// step.metal:12-46.  Every thread reads dt before thread 0 advances the
// global time in a separate word, as in the reference.  MIXED: the drift is
// added to FP64 positions, and the float positions are their roundings; the
// global time is also kept in FP64 seconds.
template <bool MIXED>
__global__ void k_step(StepArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int32_t ticks = a.globals[1];
    const float dt = kDtMin1 * (float)ticks;
    if (i == 0) {
        a.globals[0] += ticks;
        if (MIXED) a.dglob[0] += (double)kDtMin1 * (double)ticks;
    }
    float4 v = a.vel4[i];
    const float4 ac = a.acc4[i];
    const float hi = a.h[i];
    const float h1 = 1.f / hi;
    const float dh = a.dhdt[i];
    a.h[i] = fmin_ref(hi * expf(h1 * dh * dt), kMaxH);
    a.rho[i] *= expf(-3.f * h1 * dh * dt);
    a.vel4[i] = make_float4(v.x + dt * ac.x, v.y + dt * ac.y, v.z + dt * ac.z, v.w);
    a.u[i] += dt * a.du[i];
    float4 p = a.pos4[i];
    const float dx = dt * v.x + 0.5f * ac.x * dt * dt;
    const float dy = dt * v.y + 0.5f * ac.y * dt * dt;
    const float dz = dt * v.z + 0.5f * ac.z * dt * dt;
    if (MIXED) {
        double4 q = a.pos64[i];
        q.x += (double)dx;
        q.y += (double)dy;
        q.z += (double)dz;
        a.pos64[i] = q;
        p.x = (float)q.x;
        p.y = (float)q.y;
        p.z = (float)q.z;
    } else {
        p.x += dx;
        p.y += dy;
        p.z += dz;
    }
    a.pos4[i] = p;
}

__global__ void k_pos_to64(int n, const float4 *__restrict__ pos4, double4 *__restrict__ pos64) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos4[i];
    pos64[i] = make_double4((double)p.x, (double)p.y, (double)p.z, 0.0);
}

// FP64 conservation sums per block: mass, kinetic, internal and potential
// energy, momentum, angular momentum about the origin (FP64 positions when
// present); one record of kDiag doubles per block, summed in block order by
// k_diag_total so the result does not depend on scheduling.
constexpr int kDiagThreads = 256;
__global__ void __launch_bounds__(kDiagThreads) k_diag_block(int n, const float4 *__restrict__ pos4,
                                                                const double4 *__restrict__ pos64,
                                                                const float4 *__restrict__ vel4,
                                                                const float *__restrict__ u,
                                                                const float *__restrict__ phi, double *out) {
    __shared__ double red[kDiag][kDiagThreads / 32];
    double v[kDiag];
#pragma unroll
    for (int k = 0; k < kDiag; ++k) v[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pos4[i];
        const double m = (double)p.w;
        double x = p.x, y = p.y, z = p.z;
        if (pos64) {
            const double4 q = pos64[i];
            x = q.x;
            y = q.y;
            z = q.z;
        }
        const float4 w = vel4[i];
        const double vx = w.x, vy = w.y, vz = w.z;
        v[0] += m;
        v[1] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        v[2] += m * (double)u[i];
        v[3] += 0.5 * m * (double)phi[i];
        v[4] += m * vx;
        v[5] += m * vy;
        v[6] += m * vz;
        v[7] += m * (y * vz - z * vy);
        v[8] += m * (z * vx - x * vz);
        v[9] += m * (x * vy - y * vx);
    }
#pragma unroll
    for (int k = 0; k < kDiag; ++k) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < kDiag) {
        double t = 0.0;
        for (int w = 0; w < kDiagThreads / 32; ++w) t += red[threadIdx.x][w];
        out[(size_t)blockIdx.x * kDiag + threadIdx.x] = t;
    }
}

__global__ void k_diag_total(int blocks, double *partials, double *total) {
    const int k = threadIdx.x;
    if (k >= kDiag) return;
    double t = 0.0;
    for (int b = 0; b < blocks; ++b) t += partials[(size_t)b * kDiag + k];
    total[k] = t;
}

// render.metal:49-66
__global__ void k_snapshot(int n, const float4 *__restrict__ pos4, const int32_t *__restrict__ mat, int32_t *img) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float R_E = 6.3710f;
    float4 p = pos4[i];
    float ux = p.x, uy = p.y;
    ux -= 250.f;
    uy -= 250.f;
    const float s = kSnapshotRes / (20.f * R_E);
    ux *= s;
    uy *= s;
    if (ux < 0.f || uy < 0.f || ux > (float)kSnapshotRes || uy > (float)kSnapshotRes) return;
    int px = (int)ux, py = (int)uy;
    long pixel = (long)px + (long)(kSnapshotRes - 1 - py) * kSnapshotRes;
    // uv == SNAPSHOT_RESOLUTION exactly would index one past the image in the
    // reference; those splats are dropped here
    if (pixel < 0 || pixel >= (long)kSnapshotRes * kSnapshotRes || px >= kSnapshotRes) return;
    atomicMax(img + pixel, mat[i]);
}

// Dynamic shared memory of the list kernels; above 48 KiB (the one-lane
// parity build) it needs the per-device opt-in, set once per device.
size_t list_smem_opt_in() {
    const size_t smem = sizeof(uint32_t) * parts_per_block<kLanesPerParticle>() * kListMax;
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (smem > 48 * 1024 && dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(k_density<kLanesPerParticle>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_acceleration<kLanesPerParticle, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        cudaFuncSetAttribute(k_acceleration<kLanesPerParticle, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        done[dev] = true;
    }
    return smem;
}

// Shared memory of the tile kernel (above 48 KiB: the per-device opt-in) and
// the device's SM count, set up once per device.
int tile_smem_opt_in() {
    static int sms[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!sms[dev]) {
        cudaFuncSetAttribute(k_density_tile<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileShared));
        cudaFuncSetAttribute(k_density_tile<kUnitShift>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TileShared));
        cudaFuncSetAttribute(k_acceleration_tile<false, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TileAccShared));
        cudaFuncSetAttribute(k_acceleration_tile<true, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TileAccShared));
        cudaFuncSetAttribute(k_acceleration_tile<false, kUnitShift>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TileAccShared));
        cudaFuncSetAttribute(k_acceleration_tile<true, kUnitShift>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TileAccShared));
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        sms[dev] = v > 0 ? v : 148;
    }
    return sms[dev];
}

// Persistent CTAs of the tile passes: two per SM, but no more than one per
// ~48 particles (a tile holds ~100-300), so a small context -- an ensemble
// instance -- leaves the rest of the device to the others.
unsigned tile_grid(int n, int sms) {
    const int want = (n + 47) / 48;
    return (unsigned)std::max(1, std::min(sms * 2, want));
}

}  // namespace

sph_status launch_density(sph_ctx *ctx, cudaStream_t st) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    const uint32_t *cidx = ctx->cell_sort.vals[ctx->cell_final];
    k_gather<<<(n + 255) / 256, 256, 0, st>>>(n, cidx, ctx->pos4, ctx->vel4, ctx->sp4, ctx->sv4);
    DensityArgs a;
    a.n = n;
    a.cidx = cidx;
    a.skey = ctx->cell_sort.keys[ctx->cell_final];
    a.cells = ctx->cell_range;
    a.units = ctx->units;
    a.cflags = ctx->coarse_flags;
    a.coarse = ctx->tile_coarse;
    a.sp4 = ctx->sp4;
    a.sv4 = ctx->sv4;
    a.h = ctx->h;
    a.rho = ctx->rho;
    a.f = ctx->f;
    a.P = ctx->P;
    a.c = ctx->c;
    a.B = ctx->B;
    a.u = ctx->u;
    a.mat = ctx->mat;
    a.active = ctx->active;
    a.sA = ctx->sA;
    a.sB = ctx->sB;
    a.sC = ctx->sC;
    a.globals = ctx->globals;
    a.health = ctx->health;
    a.eos = ctx->eos;
    a.eta = ctx->form.h_tolerance > 0.f ? ctx->form.h_tolerance : kDensityEta;
    a.seed = nullptr;
    a.nn_out = ctx->hs.nn;
    a.stats = ctx->hs.stats;
    sph_status s = SPH_OK;
    // the learned seed's online refresh, unless a full step ran it ahead
    if (hseed_online_due(ctx) && !ctx->hs.trained_ahead) s = launch_hseed_online(ctx, st);
    if (s != SPH_OK) return s;
    if (ctx->hs.stats) cudaMemsetAsync(ctx->hs.stats, 0, sizeof(uint32_t) * 4, st);
    if (ctx->hs.capture) s = launch_hseed_capture(ctx, st);
    if (s == SPH_OK && ctx->form.h_seed == SPH_HSEED_LEARNED) {
        s = launch_hseed_infer(ctx, st);
        a.seed = ctx->hs.seed;
    }
    if (s != SPH_OK) return s;
    a.nn_out = ctx->hs.nn;
    a.stats = ctx->hs.stats;
    constexpr int parts = parts_per_block<kLanesPerParticle>();
    const size_t smem = list_smem_opt_in();
#ifdef SPH_PARITY
    // one lane per particle, in the reference's order
    k_density<kLanesPerParticle><<<(unsigned)((n + parts - 1) / parts), parts * kLanesPerParticle, smem, st>>>(a);
#else
    // cell tiles, then the coarse tiles of the blocks they flagged (the tile
    // list is reused), then the per-particle pass over what both deferred
    const int sms = tile_smem_opt_in();
    uint32_t *ctr = ctx->tile_ctr;
    cudaMemsetAsync(ctr, 0, sizeof(uint32_t) * 8, st);
    k_tile_starts<<<(n + 255) / 256, 256, 0, st>>>(n, a.skey, ctx->cell_range, ctx->tiles, ctr, ctx->globals,
                                                   ctx->tile_block_max, ctx->tile_half_max, ctx->tile_big_max);
    const unsigned tgrid = tile_grid(n, sms);
    k_density_tile<0><<<tgrid, kTileThreads, sizeof(TileShared), st>>>(a, ctx->tiles, ctr, ctx->deferred, ctr + 2);
    if (a.coarse) {
        k_coarse_starts<<<(n + 255) / 256, 256, 0, st>>>(n, a.skey, ctx->units, ctx->coarse_flags, ctx->tiles,
                                                         ctr + 4);
        k_density_tile<kUnitShift>
            <<<tgrid, kTileThreads, sizeof(TileShared), st>>>(a, ctx->tiles, ctr + 4, ctx->deferred, ctr + 2);
    }
    k_density_deferred<kLanesPerParticle><<<tgrid * 4, parts * kLanesPerParticle, smem, st>>>(a, ctx->deferred,
                                                                                           ctr + 2);
#endif
    if (ctx->hs.capture) s = launch_hseed_targets(ctx, st);
    if (s != SPH_OK) return s;
    return cuda_status(cudaGetLastError(), "density");
}

sph_status launch_acceleration(sph_ctx *ctx, cudaStream_t st) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    AccelArgs a;
    a.n = n;
    a.cidx = ctx->cell_sort.vals[ctx->cell_final];
    a.skey = ctx->cell_sort.keys[ctx->cell_final];
    a.cells = ctx->cell_range;
    a.units = ctx->units;
    a.cflags = ctx->coarse_flags;
    a.coarse = ctx->tile_coarse;
    a.sA = ctx->sA;
    a.sB = ctx->sB;
    a.sC = ctx->sC;
    a.acc4 = ctx->acc4;
    a.du = ctx->du;
    a.dhdt = ctx->dhdt;
    a.nat = ctx->nat;
    a.active = ctx->active;
    a.globals = ctx->globals;
    a.individual = ctx->form.timestep == SPH_TIMESTEP_INDIVIDUAL;
    constexpr int parts = parts_per_block<kLanesPerParticle>();
    const size_t smem = list_smem_opt_in();
    const bool kahan = ctx->form.precision == SPH_PRECISION_MIXED;
#ifdef SPH_PARITY
    // one lane per particle, in the reference's order
    const unsigned blocks = (unsigned)((n + parts - 1) / parts);
    if (kahan)
        k_acceleration<kLanesPerParticle, true><<<blocks, parts * kLanesPerParticle, smem, st>>>(a);
    else
        k_acceleration<kLanesPerParticle, false><<<blocks, parts * kLanesPerParticle, smem, st>>>(a);
#else
    // the density pass's tiles, rebuilt so the pass also stands alone; its own
    // counters (tile_ctr[8..15]); then the coarse tiles and the deferred
    const int sms = tile_smem_opt_in();
    uint32_t *ctr = ctx->tile_ctr + 8;
    cudaMemsetAsync(ctr, 0, sizeof(uint32_t) * 8, st);
    k_tile_starts<<<(n + 255) / 256, 256, 0, st>>>(n, a.skey, ctx->cell_range, ctx->tiles, ctr, nullptr,
                                                   ctx->tile_block_max, ctx->tile_half_max, ctx->tile_big_max);
    const unsigned tgrid = tile_grid(n, sms);
    const size_t tsm = sizeof(TileAccShared);
    if (kahan)
        k_acceleration_tile<true, 0><<<tgrid, kTileThreads, tsm, st>>>(a, ctx->tiles, ctr, ctx->deferred, ctr + 2);
    else
        k_acceleration_tile<false, 0><<<tgrid, kTileThreads, tsm, st>>>(a, ctx->tiles, ctr, ctx->deferred, ctr + 2);
    if (a.coarse) {
        k_coarse_starts<<<(n + 255) / 256, 256, 0, st>>>(n, a.skey, ctx->units, ctx->coarse_flags, ctx->tiles,
                                                         ctr + 4);
        if (kahan)
            k_acceleration_tile<true, kUnitShift>
                <<<tgrid, kTileThreads, tsm, st>>>(a, ctx->tiles, ctr + 4, ctx->deferred, ctr + 2);
        else
            k_acceleration_tile<false, kUnitShift>
                <<<tgrid, kTileThreads, tsm, st>>>(a, ctx->tiles, ctr + 4, ctx->deferred, ctr + 2);
    }
    if (kahan)
        k_acceleration_deferred<kLanesPerParticle, true>
            <<<tgrid * 4, parts * kLanesPerParticle, smem, st>>>(a, ctx->deferred, ctr + 2);
    else
        k_acceleration_deferred<kLanesPerParticle, false>
            <<<tgrid * 4, parts * kLanesPerParticle, smem, st>>>(a, ctx->deferred, ctr + 2);
#endif
    return cuda_status(cudaGetLastError(), "acceleration");
}

sph_status launch_step(sph_ctx *ctx, cudaStream_t st) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    StepArgs a;
    a.n = n;
    a.pos4 = ctx->pos4;
    a.vel4 = ctx->vel4;
    a.acc4 = ctx->acc4;
    a.rho = ctx->rho;
    a.u = ctx->u;
    a.h = ctx->h;
    a.du = ctx->du;
    a.dhdt = ctx->dhdt;
    a.globals = ctx->globals;
    a.pos64 = ctx->pos64;
    a.dglob = ctx->dglob;
    if (ctx->form.precision == SPH_PRECISION_MIXED)
        k_step<true><<<(n + 255) / 256, 256, 0, st>>>(a);
    else
        k_step<false><<<(n + 255) / 256, 256, 0, st>>>(a);
    return cuda_status(cudaGetLastError(), "step");
}

sph_status launch_pos_to64(sph_ctx *ctx, cudaStream_t st) {
    if (ctx->n > 0 && ctx->pos64) k_pos_to64<<<(ctx->n + 255) / 256, 256, 0, st>>>(ctx->n, ctx->pos4, ctx->pos64);
    return cuda_status(cudaGetLastError(), "positions to FP64");
}

// ctx->diag: [kDiagBlocks * kDiag] partials, then kDiag totals
sph_status launch_diag_sums(sph_ctx *ctx, cudaStream_t st) {
    double *tot = ctx->diag + (size_t)kDiagBlocks * kDiag;
    k_diag_block<<<kDiagBlocks, kDiagThreads, 0, st>>>(ctx->n, ctx->pos4,
                                                       ctx->form.precision == SPH_PRECISION_MIXED ? ctx->pos64 : nullptr,
                                                       ctx->vel4, ctx->u, ctx->phi, ctx->diag);
    k_diag_total<<<1, 32, 0, st>>>(kDiagBlocks, ctx->diag, tot);
    return cuda_status(cudaGetLastError(), "diagnostics");
}

sph_status launch_snapshot(sph_ctx *ctx, cudaStream_t st) {
    const int n = ctx->n;
    cudaMemsetAsync(ctx->snapshot, 0, sizeof(int32_t) * kSnapshotRes * kSnapshotRes, st);
    if (n > 0) k_snapshot<<<(n + 255) / 256, 256, 0, st>>>(n, ctx->pos4, ctx->mat, ctx->snapshot);
    return cuda_status(cudaGetLastError(), "snapshot");
}

}  // namespace sph

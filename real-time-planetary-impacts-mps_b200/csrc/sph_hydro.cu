// sph_hydro.cu -- density, acceleration and step passes for sm_100a.
//
// density      SPH/Shaders/density.metal:12-239        (Compute.cpp:179-208)
// acceleration SPH/Shaders/accelerations.metal:12-141  (Compute.cpp:210-240)
// step         SPH/Shaders/step.metal:12-46            (Compute.cpp:242-263)
// snapshot     SPH/Shaders/render.metal:49-66          (Compute.cpp:396-448)
//
// One thread per particle, in sorted (Morton cell) order, so a warp's threads
// walk neighbouring cells together.  Neighbour data are read from sorted,
// 16-byte records (sp4/sv4 gathered before density; sA/sB/sC written by the
// density epilogue), so a cell's particles are one contiguous run instead of
// the reference's index-chased float3 gathers.
//
// The reference walks the cell box of radius 2h (x outer, z inner; sorted
// index within a cell) once per smoothing-length iteration and once more for
// the gradient terms, and the box holds several times more candidates than
// neighbours.  Here:
//  * cells whose box lies farther than the filter radius (with a margin for
//    the rounding of cell boundaries) are skipped: none of their particles
//    passes the filter, so the visited set and its order are unchanged;
//  * the first sweep also records, in visiting order, every candidate within
//    2.5 h of the initial h; later sweeps walk that list with the same
//    filters while 4h^2 stays inside its radius, and fall back to the box
//    otherwise.  The list holds every candidate that a later box walk would
//    accept, in the same order; the two can differ only for candidates at
//    exactly the kernel's support radius, where W, dW/dh and grad W are zero.
// The reference's 128-entry per-thread neighbour cache (density.metal:67-70)
// becomes a walk with that cache's filters (its count is kept, capped).
#include <cuda_runtime.h>

#include "sph_internal.h"

namespace sph {

namespace {

constexpr int kHydroThreads = 128;
// Margin on the distance from a particle to a cell box: positions near 318 Mm
// carry ~3e-5 Mm of float32 rounding, and a particle's cell comes from
// floor(x / CELL_WIDTH); 2e-4 Mm keeps every particle of the cell inside.
constexpr float kCellMargin = 2e-4f;

// Squared distance from (px, py, pz) to the box of cell (x, y, z), each axis
// gap shortened by the margin.
__device__ __forceinline__ float cell_gap2(float px, float py, float pz, int x, int y, int z) {
    const float w = kCellWidth;
    float gx = fmaxf(fmaxf((float)x * w - px, px - (float)(x + 1) * w) - kCellMargin, 0.f);
    float gy = fmaxf(fmaxf((float)y * w - py, py - (float)(y + 1) * w) - kCellMargin, 0.f);
    float gz = fmaxf(fmaxf((float)z * w - pz, pz - (float)(z + 1) * w) - kCellMargin, 0.f);
    return gx * gx + gy * gy + gz * gz;
}

// The reference's walk over the cell box of radius 2h, skipping cells farther
// than sqrt(r2cull): body(k) for every remaining candidate, in visiting order.
//
// A lane first gathers up to kWalkChunk non-empty cell ranges of its box (in
// walk order), then runs one flat loop that takes exactly one candidate per
// iteration and steps to the next range when one runs out.  The lanes of a
// warp stay in step candidate by candidate, instead of idling while their
// neighbours finish a longer cell.
constexpr int kWalkChunk = 32;

template <class F>
__device__ __forceinline__ void walk_cells(float px, float py, float pz, float h, float r2cull,
                                           const uint2 *__restrict__ cells, F &&body) {
    const CellBox b = cell_box(px, py, pz, h);
    uint2 rg[kWalkChunk];
    int x = b.lo0, y = b.lo1, z = b.lo2;
    bool more = true;
    while (more) {
        int nc = 0;
        while (nc < kWalkChunk) {
            if (cell_gap2(px, py, pz, x, y, z) <= r2cull) {
                const uint2 r = __ldg(cells + cell_index_of(x, y, z));
                if (r.x != 0xffffffffu) rg[nc++] = r;
            }
            if (++z > b.hi2) {
                z = b.lo2;
                if (++y > b.hi1) {
                    y = b.lo1;
                    if (++x > b.hi0) {
                        more = false;
                        break;
                    }
                }
            }
        }
        if (nc == 0) continue;
        int ci = 0;
        uint32_t k = rg[0].x, e = rg[0].y;
        for (;;) {
            body(k);
            if (++k > e) {
                if (++ci >= nc) break;
                k = rg[ci].x;
                e = rg[ci].y;
            }
        }
    }
}

__global__ void k_gather(int n, const uint32_t *__restrict__ cidx, const float4 *__restrict__ pos4,
                         const float4 *__restrict__ vel4, float4 *__restrict__ sp4, float4 *__restrict__ sv4) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t i = cidx[k];
    sp4[k] = pos4[i];
    sv4[k] = vel4[i];
}

struct DensityArgs {
    int n;
    const uint32_t *cidx;
    const uint2 *cells;
    const float4 *sp4, *sv4;
    float *h, *rho, *f, *P, *c, *B;
    const float *u;
    const int32_t *mat;
    const uint8_t *active;
    float4 *sA, *sB, *sC;
    int32_t *globals;
    uint32_t *health;
    uint32_t *nlist;  // [kNeighbourListCap][n]: entry s of sorted particle i at s * n + i
    EosTables eos;
};

__global__ void __launch_bounds__(kHydroThreads) k_density(DensityArgs a) {
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= a.n) return;
    if (index == 0) a.globals[1] = (int32_t)(kDT0 * 1 / kDtMin1);  // density.metal:34-36
    const uint32_t ind = a.cidx[index];
    const float4 me = a.sp4[index];
    const float4 mv = a.sv4[index];
    if (!a.active[ind]) {
        // density.metal:40-55: EOS only
        const float2 pc = eos_lookup(a.eos, a.mat[ind], a.rho[ind], a.u[ind]);
        a.P[ind] = pc.x;
        a.c[ind] = pc.y;
        const float hv = a.h[ind], rho = a.rho[ind], fv = a.f[ind];
        a.sA[index] = make_float4(me.x, me.y, me.z, hv);
        a.sB[index] = make_float4(mv.x, mv.y, mv.z, pc.y);
        a.sC[index] = make_float4(me.w, (fv * pc.x / (rho * rho)), rho, a.B[ind]);
        return;
    }
    const float px = me.x, py = me.y, pz = me.z, mi = me.w;
    const float4 *__restrict__ sp4 = a.sp4;
    const uint2 *__restrict__ cells = a.cells;
    const size_t n = (size_t)a.n;
    uint32_t *__restrict__ list = a.nlist + index;
    float hi = a.h[ind];
    int max_h = 0;  // an int in the reference (truncates h < 1 to 0)
    float h2x4 = 4.f * hi * hi;
    float h1 = 1.f / hi;
    float dens = 0.f;
    float eps = 1.f;
    int count = 0;
    // The reference's neighbour cache holds the neighbours of the last full
    // scan: that scan's h (box and filter) and its count capped at
    // N_NEIGHBOURS_ESTIM.  A "cached" sweep walks again with those filters.
    int nn = 0;
    float hs = hi, hs2x4 = h2x4;
    // neighbour list of radius 2.5 h0, built by the first sweep
    const float lr = 2.5f * hi;
    const float lr2 = lr * lr;
    int nl = 0;
    bool list_ok = true;
    bool first = true;
    while (eps > kDensityEta && count < kMaxNR) {
        const bool cached = hi < (float)max_h && nn < kNeighbourCache;
        if (!cached) {
            hs = hi;
            hs2x4 = h2x4;
            nn = 0;
        }
        const float r2max = cached ? hs2x4 : h2x4;
        const float rlim = cached ? hi + hi : 3.402823466e+38f;
        dens = 0.f;
        auto visit = [&](float4 q) {
            const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > r2max) return;
            const float r = sqrtf(r2);
            if (r > rlim) return;
            if (!cached && nn < kNeighbourCache) nn++;
            dens += kernel_w(r, h1) * q.w;
        };
        if (first) {
            // first sweep (never a cached one): walk the 2.5 h box once,
            // recording the list while summing the sweep of radius 2h
            first = false;
            walk_cells(px, py, pz, 1.25f * hi, lr2, cells, [&](uint32_t k) {
                const float4 q = __ldg(sp4 + k);
                const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 <= lr2) {
                    if (nl < kNeighbourListCap)
                        list[(size_t)nl * n] = k;
                    else
                        list_ok = false;
                    ++nl;
                }
                if (r2 > h2x4) return;
                const float r = sqrtf(r2);
                if (nn < kNeighbourCache) nn++;
                dens += kernel_w(r, h1) * q.w;
            });
        } else if (list_ok && r2max <= lr2) {
            for (int s = 0; s < nl; ++s) visit(__ldg(sp4 + list[(size_t)s * n]));
        } else {
            walk_cells(px, py, pz, cached ? hs : hi, r2max, cells, [&](uint32_t k) { visit(__ldg(sp4 + k)); });
        }
        float nh = fmin_ref(kResolutionEta * powf(mi / dens, 1.f / 3), kMaxH);
        nh = 0.5f * (hi + nh);
        eps = fabsf(nh - hi) / hi;
        if (eps > kDensityEta) {
            max_h = (int)fmax_ref((float)max_h, hi);
            hi = nh;
            h1 = 1.f / hi;
            h2x4 = 4.f * hi * hi;
            count++;
        }
    }
    // gradient sweep (density.metal:145-213); with an overflowing cache the
    // reference adds to the converged density again, and so does this
    const bool cached = nn < kNeighbourCache;
    const float r2max = cached ? hs2x4 : h2x4;
    const float rlim = cached ? hi + hi : 3.402823466e+38f;
    const float vix = mv.x, viy = mv.y, viz = mv.z;
    const float4 *__restrict__ sv4 = a.sv4;
    float dens_h = 0.f, vdiv = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    auto grad = [&](uint32_t k) {
        const float4 q = __ldg(sp4 + k);
        const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > r2max) return;
        const float r = sqrtf(r2);
        if (r > rlim) return;
        const float mj = q.w;
        if (!cached) dens += kernel_w(r, h1) * mj;
        dens_h += mj * kernel_dwdh(r, h1);
        if (r > 1e-12f) {
            const float r1 = 1.f / r;
            const float4 vj = __ldg(sv4 + k);
            const float vx = vj.x - vix, vy = vj.y - viy, vz = vj.z - viz;
            const float s = kernel_gradw_scale(r, h1);
            const float gx = s * (dx * r1), gy = s * (dy * r1), gz = s * (dz * r1);
            vdiv += mj * (vx * gx + vy * gy + vz * gz);
            cx += mj * (vy * gz - vz * gy);
            cy += mj * (vz * gx - vx * gz);
            cz += mj * (vx * gy - vy * gx);
        }
    };
    if (list_ok && r2max <= lr2) {
        for (int s = 0; s < nl; ++s) grad(list[(size_t)s * n]);
    } else {
        walk_cells(px, py, pz, cached ? hs : hi, r2max, cells, grad);
    }
    vdiv = fabsf(vdiv) / dens;
    const float acurl = sqrtf(cx * cx + cy * cy + cz * cz) / dens;
    const float fi = 1.f / (1.f + (hi / (3.f * dens)) * dens_h);
    const float2 pc = eos_lookup(a.eos, a.mat[ind], dens, a.u[ind]);
    const float bal = vdiv / (vdiv + acurl + 1e-4f * (pc.y / hi));
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

struct AccelArgs {
    int n;
    const uint32_t *cidx;
    const uint2 *cells;
    const float4 *sA, *sB, *sC;
    float4 *acc4;
    float *du, *dhdt;
    int32_t *nat;
    const uint8_t *active;
    int32_t *globals;
    uint32_t *plist;  // accepted pairs, [kNeighbourListCap][n] (the density list's storage)
};

__global__ void __launch_bounds__(kHydroThreads) k_acceleration(AccelArgs a) {
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    int idt = 0x7fffffff;
    if (index < a.n) {
        const uint32_t ind = a.cidx[index];
        if (a.active[ind]) {
            const float4 A = a.sA[index], Bv = a.sB[index], Cv = a.sC[index];
            const float xi = A.x, yi = A.y, zi = A.z, hi = A.w;
            const float vxi = Bv.x, vyi = Bv.y, vzi = Bv.z, ci = Bv.w;
            const float facti = Cv.y, rhoi = Cv.z, Bi = Cv.w;
            const float hi1 = 1.f / hi;
            const float hi2x4 = hi * hi * 4.f;
            const float4 *__restrict__ sA = a.sA;
            const float4 *__restrict__ sB = a.sB;
            const float4 *__restrict__ sC = a.sC;
            const size_t n = (size_t)a.n;
            uint32_t *__restrict__ list = a.plist + index;
            float dvx = 0.f, dvy = 0.f, dvz = 0.f, du = 0.f, dh = 0.f;
            float vsig_i = 1e-12f;
            // accelerations.metal:73-120 for one accepted pair
            auto pair = [&](uint32_t k) {
                const float4 Aj = __ldg(sA + k);
                const float4 Bj = __ldg(sB + k);
                const float4 Cj = __ldg(sC + k);
                const float dx = xi - Aj.x, dy = yi - Aj.y, dz = zi - Aj.z;
                const float r2 = dx * dx + dy * dy + dz * dz;
                const float hj = Aj.w;
                const float r = sqrtf(r2);
                const float r1 = 1.f / r;
                const float mj = Cj.x, factj = Cj.y, rhoj = Cj.z, Balj = Cj.w;
                const float hj1 = 1.f / hj;
                const float vx = vxi - Bj.x, vy = vyi - Bj.y, vz = vzi - Bj.z;
                const float rhoij = 0.5f * (rhoi + rhoj);
                const float vdr = vx * dx + vy * dy + vz * dz;
                const float mu = vdr < 0.f ? vdr * r1 : 0.f;
                const float vsig = ci + Bj.w - 3.f * mu;
                vsig_i = fmax_ref(vsig, vsig_i);
                const float Bij = 0.5f * (Bi + Balj);
                const float nu = -0.5f * kViscosityAlpha * Bij * mu * vsig / rhoij;
                const float rhx = dx * r1, rhy = dy * r1, rhz = dz * r1;
                const float si = kernel_gradw_scale(r, hi1), sj = kernel_gradw_scale(r, hj1);
                const float gix = si * rhx, giy = si * rhy, giz = si * rhz;
                const float gjx = sj * rhx, gjy = sj * rhy, gjz = sj * rhz;
                const float gx = 0.5f * (gix + gjx), gy = 0.5f * (giy + gjy), gz = 0.5f * (giz + gjz);
                dvx -= mj * (facti * gix + factj * gjx + nu * gx);
                dvy -= mj * (facti * giy + factj * gjy + nu * gy);
                dvz -= mj * (facti * giz + factj * gjz + nu * gz);
                du += mj * (facti * (vx * gix + vy * giy + vz * giz) + 0.5f * nu * (vx * gx + vy * gy + vz * gz));
                dh += (mj / rhoj) * (vx * gix + vy * giy + vz * giz);
            };
            // walk: keep the accepted pairs, in visiting order, then evaluate
            // them in one uniform loop (a full list is evaluated and emptied)
            int nl = 0;
            walk_cells(xi, yi, zi, fmin_ref(hi, kMaxH), 3.402823466e+38f, a.cells, [&](uint32_t k) {
                const float4 Aj = __ldg(sA + k);
                const float dx = xi - Aj.x, dy = yi - Aj.y, dz = zi - Aj.z;
                const float r2 = dx * dx + dy * dy + dz * dz;
                const float hj = Aj.w;
                const float hj2x4 = hj * hj * 4.f;
                if ((r2 > hi2x4 && r2 > hj2x4) || r2 < 1e-12f) return;  // accelerations.metal:80
                if (nl == kNeighbourListCap) {
                    for (int s = 0; s < nl; ++s) pair(list[(size_t)s * n]);
                    nl = 0;
                }
                list[(size_t)nl * n] = k;
                ++nl;
            });
            for (int s = 0; s < nl; ++s) pair(list[(size_t)s * n]);
            float4 acc = a.acc4[ind];
            acc.x += dvx;
            acc.y += dvy;
            acc.z += dvz;
            a.acc4[ind] = acc;
            a.du[ind] = du;
            a.dhdt[ind] = dh;
            // accelerations.metal:129-140
            const float goal = 2.0f * kCFL * kGamma * hi / vsig_i;
            int rr = 0;
            float cand = kDT0;
            while (cand > goal && rr < kRMax) {
                cand *= 0.5f;
                rr++;
            }
            idt = (int)ceilf(1 / kDtMin1 * cand);
            a.nat[ind] = a.globals[0] + idt;
        }
    }
    // block-wide minimum, then one atomic per block
    for (int o = 16; o > 0; o >>= 1) idt = min(idt, __shfl_xor_sync(0xffffffffu, idt, o));
    __shared__ int wmin[kHydroThreads / 32];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = idt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int v = wmin[0];
        for (int w = 1; w < kHydroThreads / 32; ++w) v = min(v, wmin[w]);
        if (v != 0x7fffffff) atomicMin(&a.globals[1], v);
    }
}

struct StepArgs {
    int n;
    float4 *pos4, *vel4;
    const float4 *acc4;
    float *rho, *u, *h;
    const float *du, *dhdt;
    int32_t *globals;
};

// step.metal:12-46.  Every thread reads dt before thread 0 advances the
// global time in a separate word, as in the reference.
__global__ void k_step(StepArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int32_t ticks = a.globals[1];
    const float dt = kDtMin1 * (float)ticks;
    if (i == 0) a.globals[0] += ticks;
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
    p.x += dt * v.x + 0.5f * ac.x * dt * dt;
    p.y += dt * v.y + 0.5f * ac.y * dt * dt;
    p.z += dt * v.z + 0.5f * ac.z * dt * dt;
    a.pos4[i] = p;
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

}  // namespace

sph_status launch_density(sph_ctx *ctx, cudaStream_t st) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    const uint32_t *cidx = ctx->cell_sort.vals[ctx->cell_final];
    k_gather<<<(n + 255) / 256, 256, 0, st>>>(n, cidx, ctx->pos4, ctx->vel4, ctx->sp4, ctx->sv4);
    DensityArgs a;
    a.n = n;
    a.cidx = cidx;
    a.cells = ctx->cell_range;
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
    a.nlist = ctx->nlist;
    a.eos = ctx->eos;
    k_density<<<(n + kHydroThreads - 1) / kHydroThreads, kHydroThreads, 0, st>>>(a);
    return cuda_status(cudaGetLastError(), "density");
}

sph_status launch_acceleration(sph_ctx *ctx, cudaStream_t st) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    AccelArgs a;
    a.n = n;
    a.cidx = ctx->cell_sort.vals[ctx->cell_final];
    a.cells = ctx->cell_range;
    a.sA = ctx->sA;
    a.sB = ctx->sB;
    a.sC = ctx->sC;
    a.acc4 = ctx->acc4;
    a.du = ctx->du;
    a.dhdt = ctx->dhdt;
    a.nat = ctx->nat;
    a.active = ctx->active;
    a.globals = ctx->globals;
    a.plist = ctx->nlist;
    k_acceleration<<<(n + kHydroThreads - 1) / kHydroThreads, kHydroThreads, 0, st>>>(a);
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
    k_step<<<(n + 255) / 256, 256, 0, st>>>(a);
    return cuda_status(cudaGetLastError(), "step");
}

sph_status launch_snapshot(sph_ctx *ctx, cudaStream_t st) {
    const int n = ctx->n;
    cudaMemsetAsync(ctx->snapshot, 0, sizeof(int32_t) * kSnapshotRes * kSnapshotRes, st);
    if (n > 0) k_snapshot<<<(n + 255) / 256, 256, 0, st>>>(n, ctx->pos4, ctx->mat, ctx->snapshot);
    return cuda_status(cudaGetLastError(), "snapshot");
}

}  // namespace sph

// sph_hydro.cu -- density, acceleration and step passes for sm_100a.
//
// density      SPH/Shaders/density.metal:12-239        (Compute.cpp:179-208)
// acceleration SPH/Shaders/accelerations.metal:12-141  (Compute.cpp:210-240)
// step         SPH/Shaders/step.metal:12-46            (Compute.cpp:242-263)
// snapshot     SPH/Shaders/render.metal:49-66          (Compute.cpp:396-448)
//
// One thread per particle in sorted (Morton cell) order, so a warp's threads
// walk neighbouring cells together.  Neighbour data are read from sorted,
// 16-byte records (sp4/sv4, then sA/sB/sC written by the density epilogue),
// so every cell's particles are one contiguous run of float4 loads instead of
// the reference's index-chased float3 gathers.  The neighbour loops visit
// cells and particles in the reference's order and accumulate in the same
// order, so sums agree with it to rounding.
//
// The reference's 128-entry per-thread neighbour cache (density.metal:67-70)
// is replaced by rescanning the same cell box with the same filters: the
// visited set and order are identical (see k_density), and no thread carries
// 1 KiB of local memory.
#include <cuda_runtime.h>

#include "sph_internal.h"

namespace sph {

namespace {

// Margin on the distance from a particle to a cell box: positions near 318 Mm
// carry ~3e-5 Mm of float32 rounding, and a particle's cell comes from
// floor(x / CELL_WIDTH); 2e-4 Mm keeps every particle of a cell inside its box.
constexpr float kCellMargin = 2e-4f;

// Squared distance from (px, py, pz) to the box of cell (x, y, z), each axis
// gap shortened by the margin.
__device__ __forceinline__ float cell_gap2(float px, float py, float pz, int x, int y, int z) {
    const float w = kCellWidth;
    const float gx = fmaxf(fmaxf((float)x * w - px, px - (float)(x + 1) * w) - kCellMargin, 0.f);
    const float gy = fmaxf(fmaxf((float)y * w - py, py - (float)(y + 1) * w) - kCellMargin, 0.f);
    const float gz = fmaxf(fmaxf((float)z * w - pz, pz - (float)(z + 1) * w) - kCellMargin, 0.f);
    return gx * gx + gy * gy + gz * gz;
}

// Visit the neighbours of (px, py, pz) in the cell box of radius 2h, in the
// reference's order (x outer, z inner; sorted index within a cell).  Cells
// farther than sqrt(r2cull) are skipped: when r2cull bounds the caller's own
// distance filter, none of their particles would pass it, so the visited set
// and its order are unchanged.
template <class F>
__device__ __forceinline__ void for_cells(float px, float py, float pz, float h, float r2cull,
                                          const uint2 *__restrict__ cells, F &&body) {
    CellBox b = cell_box(px, py, pz, h);
    for (int x = b.lo0; x <= b.hi0; ++x)
        for (int y = b.lo1; y <= b.hi1; ++y)
            for (int z = b.lo2; z <= b.hi2; ++z) {
                if (cell_gap2(px, py, pz, x, y, z) > r2cull) continue;
                uint2 r = __ldg(cells + cell_index_of(x, y, z));
                if (r.x == 0xffffffffu) continue;
                for (uint32_t k = r.x; k <= r.y; ++k) body(k);
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
    EosTables eos;
};

__global__ void __launch_bounds__(128) k_density(DensityArgs a) {
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= a.n) return;
    if (index == 0) a.globals[1] = (int32_t)(kDT0 * 1 / kDtMin1);  // density.metal:34-36
    const uint32_t ind = a.cidx[index];
    const float4 me = a.sp4[index];
    const float4 mv = a.sv4[index];
    if (!a.active[ind]) {
        // density.metal:40-55: EOS only
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
    float hi = a.h[ind];
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
    while (eps > kDensityEta && count < kMaxNR) {
        dens = 0.f;
        if (hi < (float)max_h && nn < kNeighbourCache) {
            const float h2 = hi + hi;
            for_cells(px, py, pz, hs, hs2x4, cells, [&](uint32_t k) {
                float4 q = __ldg(sp4 + k);
                float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > hs2x4) return;
                float r = sqrtf(r2);
                if (r > h2) return;
                dens += kernel_w(r, h1) * q.w;
            });
        } else {
            hs = hi;
            hs2x4 = h2x4;
            nn = 0;
            for_cells(px, py, pz, hi, h2x4, cells, [&](uint32_t k) {
                float4 q = __ldg(sp4 + k);
                float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
                float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > h2x4) return;
                float r = sqrtf(r2);
                if (nn < kNeighbourCache) nn++;
                dens += kernel_w(r, h1) * q.w;
            });
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
    // gradient sweep (density.metal:145-213)
    float dens_h = 0.f, vdiv = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    const float vix = mv.x, viy = mv.y, viz = mv.z;
    const float4 *sv4 = a.sv4;
    auto grad = [&](uint32_t k, const float4 &q, float r, float dx, float dy, float dz) {
        float mj = q.w;
        dens_h += mj * kernel_dwdh(r, h1);
        if (r > 1e-12f) {
            float r1 = 1.f / r;
            float4 vj = __ldg(sv4 + k);
            float vx = vj.x - vix, vy = vj.y - viy, vz = vj.z - viz;
            float s = kernel_gradw_scale(r, h1);
            float gx = s * (dx * r1), gy = s * (dy * r1), gz = s * (dz * r1);
            vdiv += mj * (vx * gx + vy * gy + vz * gz);
            cx += mj * (vy * gz - vz * gy);
            cy += mj * (vz * gx - vx * gz);
            cz += mj * (vx * gy - vy * gx);
        }
    };
    if (nn < kNeighbourCache) {
        const float h2 = hi + hi;
        for_cells(px, py, pz, hs, hs2x4, cells, [&](uint32_t k) {
            float4 q = __ldg(sp4 + k);
            float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
            float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > hs2x4) return;
            float r = sqrtf(r2);
            if (r > h2) return;
            grad(k, q, r, dx, dy, dz);
        });
    } else {
        // cache overflow: the reference adds to the converged density again
        for_cells(px, py, pz, hi, h2x4, cells, [&](uint32_t k) {
            float4 q = __ldg(sp4 + k);
            float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
            float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > h2x4) return;
            float r = sqrtf(r2);
            dens += kernel_w(r, h1) * q.w;
            grad(k, q, r, dx, dy, dz);
        });
    }
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
};

__global__ void __launch_bounds__(128) k_acceleration(AccelArgs a) {
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
            float dvx = 0.f, dvy = 0.f, dvz = 0.f, du = 0.f, dh = 0.f;
            float vsig_i = 1e-12f;
            const float4 *sA = a.sA, *sB = a.sB, *sC = a.sC;
            for_cells(xi, yi, zi, fmin_ref(hi, kMaxH), 3.402823466e+38f, a.cells, [&](uint32_t k) {
                const float4 Aj = __ldg(sA + k);
                const float dx = xi - Aj.x, dy = yi - Aj.y, dz = zi - Aj.z;
                const float r2 = dx * dx + dy * dy + dz * dz;
                const float hj = Aj.w;
                const float hj2x4 = hj * hj * 4.f;
                if ((r2 > hi2x4 && r2 > hj2x4) || r2 < 1e-12f) return;
                const float4 Cj = __ldg(sC + k);
                const float4 Bj = __ldg(sB + k);
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
            });
            float4 acc = a.acc4[ind];
            acc.x += dvx;
            acc.y += dvy;
            acc.z += dvz;
            a.acc4[ind] = acc;
            a.du[ind] = du;
            a.dhdt[ind] = dh;
            // accelerations.metal:129-140
            const float goal = 2.0f * kCFL * kGamma * hi / vsig_i;
            int r = 0;
            float cand = kDT0;
            while (cand > goal && r < kRMax) {
                cand *= 0.5f;
                r++;
            }
            idt = (int)ceilf(1 / kDtMin1 * cand);
            a.nat[ind] = a.globals[0] + idt;
        }
    }
    // block-wide minimum, then one atomic per block
    for (int o = 16; o > 0; o >>= 1) idt = min(idt, __shfl_xor_sync(0xffffffffu, idt, o));
    __shared__ int wmin[32];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = idt;
    __syncthreads();
    if (threadIdx.x < 32) {
        int v = (threadIdx.x < (blockDim.x >> 5)) ? wmin[threadIdx.x] : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0 && v != 0x7fffffff) atomicMin(&a.globals[1], v);
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
    a.eos = ctx->eos;
    k_density<<<(n + 127) / 128, 128, 0, st>>>(a);
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
    k_acceleration<<<(n + 127) / 128, 128, 0, st>>>(a);
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

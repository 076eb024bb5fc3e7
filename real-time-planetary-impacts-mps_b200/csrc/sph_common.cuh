// sph_common.cuh -- constants and device helpers shared by the SPH + FMM kernels.
//
// The physics constants mirror SPH/Parameters.h:11-53 of the reference (as
// single-precision values, since Metal reads unsuffixed literals as float).
// Every helper states the reference function it computes; arithmetic is kept
// in the reference's operation order so results match it to rounding.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sph {

// ---- SPH/Parameters.h ------------------------------------------------------
constexpr float kViscosityAlpha = 1.5f;   // VISCOSITY_ALPHA
constexpr float kDensityEta = 0.005f;     // DENSITY_ETA
constexpr float kMaxH = 1.f;              // MAX_SMOOTHING_LENGTH
constexpr int kMaxNR = 50;                // MAX_DENSITY_NR_ITTERATIONS
constexpr int kNeighbourCache = 128;      // N_NEIGHBOURS_ESTIM
constexpr float kResolutionEta = 1.2348f; // RESOLUTION_ETA
constexpr float kAneosMinU = 1e-10f;      // ANEOS_MIN_U
constexpr float kAneosMinRho = 1e-6f;     // ANEOS_MIN_RHO
constexpr float kCFL = 0.2f;              // CFL
constexpr float kDT0 = 32.f;              // DT0
constexpr int kRMax = 16;                 // R_MAX
constexpr float kDtMin1 = kDT0 / (1 << kRMax); // DT_MIN1 (seconds per tick)
constexpr float kGamma = 1.825742f;       // GAMMA
constexpr float kGravityEta = 0.005f;     // GRAVITY_ETA
constexpr float kGravSoft = 0.04f;        // GRAVITY_SMOOTHING_LENGTH
constexpr float kCellWidth = 0.18f;       // CELL_WIDTH
constexpr int kCellPower = 8;             // CELL_POWER
constexpr int kCellsPerDim = 1 << kCellPower;
constexpr uint32_t kNumCells = 1u << (3 * kCellPower);
constexpr float kG = 6.67e-5f;                       // gravity/poles/poles.h:16
constexpr float kPi1 = 1 / 3.14159265358979323846f;  // utils/kernels.h:14
constexpr int kSnapshotRes = 1024;                   // SNAPSHOT_RESOLUTION
// Largest accepted initial smoothing length: the first density sweep scans a
// box of floor(4h / CELL_WIDTH) + 1 <= 223 cells per axis, inside the 256-cell grid.
constexpr float kMaxInitialH = 10.f;
// Multipole record, 6 float4 per node (gravity/poles/poles.h:46-55):
//   q0 = (com.x, com.y, com.z, size)   q1 = (M, XX, XY, XZ)
//   q2 = (YY, YZ, ZZ, power[2])       q3 = (min.x, min.y, min.z, minGrav)
//   q4 = (max.x, max.y, max.z, active) q5 = (X, Y, Z, 0)
// power[0] is M and power[1] is 0 by construction (helpers.metal:63-89).
constexpr int kPoleQ = 6;
// Local record, 4 float4 per node (poles.h:58-61):
//   l0 = (pos.x, pos.y, pos.z, e0)  l1 = (e1..e4)  l2 = (e5..e8)  l3 = (e9, 0, 0, 0)
constexpr int kLocalQ = 4;

enum { M = 0, X = 1, Y = 2, Z = 3, XX = 4, XY = 5, XZ = 6, YY = 7, YZ = 8, ZZ = 9 };

__device__ __forceinline__ float fmin_ref(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float fmax_ref(float a, float b) { return a < b ? b : a; }

// ---- utils/morton.h:16-34 ----------------------------------------------------
// Spread the low 10 bits of v so that bit b lands on bit 3b.
__host__ __device__ __forceinline__ uint32_t spread_bits3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__host__ __device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    return spread_bits3(x) | (spread_bits3(y) << 1) | (spread_bits3(z) << 2);
}

// ---- sort.metal:15-44 (hash) -------------------------------------------------
__device__ __forceinline__ uint32_t cell_key(float px, float py, float pz) {
    float nx = __fdiv_rn(px, kCellWidth), ny = __fdiv_rn(py, kCellWidth), nz = __fdiv_rn(pz, kCellWidth);
    int cx = (int)floorf(nx) % kCellsPerDim;
    int cy = (int)floorf(ny) % kCellsPerDim;
    int cz = (int)floorf(nz) % kCellsPerDim;
    if (cx < 0) cx += kCellsPerDim;
    if (cy < 0) cy += kCellsPerDim;
    if (cz < 0) cz += kCellsPerDim;
    return morton3((uint32_t)cx, (uint32_t)cy, (uint32_t)cz);
}

// ---- utils/cellsToScan.h:21-59 ----------------------------------------------
__device__ __forceinline__ uint32_t cell_index_of(int x, int y, int z) {
    const int mask = kCellsPerDim - 1;
    return morton3((uint32_t)(x & mask), (uint32_t)(y & mask), (uint32_t)(z & mask));
}
// Coarse units: 4 x 4 x 4 cells, the cells whose keys agree above the low six
// bits (unit index = cell key >> 6); 512-cell blocks are 2 x 2 x 2 units.
constexpr int kUnitShift = 2;  // cells per unit edge = 1 << kUnitShift
constexpr uint32_t kNumUnits = kNumCells >> (3 * kUnitShift);
constexpr uint32_t kNumCoarseBlocks = kNumUnits >> 3;
__device__ __forceinline__ uint32_t unit_index_of(int x, int y, int z) {
    const int mask = (kCellsPerDim >> kUnitShift) - 1;
    return morton3((uint32_t)(x & mask), (uint32_t)(y & mask), (uint32_t)(z & mask));
}
struct CellBox {
    int lo0, lo1, lo2, hi0, hi1, hi2;
};
__device__ __forceinline__ CellBox cell_box(float px, float py, float pz, float h) {
    float radius = 2.f * h;
    CellBox b;
    b.lo0 = (int)floorf(__fdiv_rn(__fsub_rn(px, radius), kCellWidth));
    b.lo1 = (int)floorf(__fdiv_rn(__fsub_rn(py, radius), kCellWidth));
    b.lo2 = (int)floorf(__fdiv_rn(__fsub_rn(pz, radius), kCellWidth));
    b.hi0 = (int)floorf(__fdiv_rn(__fadd_rn(px, radius), kCellWidth));
    b.hi1 = (int)floorf(__fdiv_rn(__fadd_rn(py, radius), kCellWidth));
    b.hi2 = (int)floorf(__fdiv_rn(__fadd_rn(pz, radius), kCellWidth));
    return b;
}

// ---- utils/kernels.h:35-85: cubic spline (M4), support 2h --------------------
__device__ __forceinline__ float kernel_w(float r, float h1) {
    float q = r * h1;
    if (q > 2.f) return 0.f;
    float fac = kPi1 * h1 * h1 * h1;
    if (q > 1.f) {
        float t = 2.f - q;
        return fac * 0.25f * t * t * t;
    }
    return fac * (1.f - 1.5f * q * q * (1.f - 0.5f * q));
}
// kernels.h:52-69; returns the scalar s with gradW = s * x_ij * r1 (or 0).
__device__ __forceinline__ float kernel_gradw_scale(float r, float h1) {
    float q = r * h1;
    if (q > 2.f || q < 1e-12f) return 0.f;
    float fac = kPi1 * h1 * h1 * h1 * h1;
    if (q > 1.f) {
        float t = 2.f - q;
        return -0.75f * fac * t * t;
    }
    return 3.f * fac * (0.75f * q - 1.f) * q;
}
__device__ __forceinline__ float kernel_dwdh(float r, float h1) {
    float q = r * h1;
    if (q > 2.f) return 0.f;
    float fac = -3.f * kPi1 * h1 * h1 * h1 * h1;
    if (q > 1.f) return fac * (2.f - 4.f * q + 2.5f * q * q - 0.5f * q * q * q);
    return fac * (1.f + 0.5f * (3.f * q - 5.f) * q * q);
}
// kernels.h:87-102 with the reference's integer-division coefficients
// ((4/3)=1, (6/5)=1, (8/3)=2, (1/6)=0, (1/15)=0) and h = min(0.04, 0.16).
__device__ __forceinline__ float grav_dphi_dr(float r) {
    const float h1 = 1.f / fmin_ref(kGravSoft, 0.16f);
    float q = r * h1;
    if (q <= 1.f) return (h1 * h1) * (q - q * q * q + 0.5f * q * q * q * q);
    if (q <= 2.f) return (h1 * h1) * (2.f * q - 3.f * q * q + q * q * q);
    float r1 = 1.f / r;
    return r1 * r1;
}

// ---- EOS: bilinear sample of a res x res (P, c) grid in normalised
// coordinates, texel centres at (i+0.5)/res, clamp-to-edge (density.metal:45-53).
__device__ __forceinline__ float2 eos_sample(const float2 *__restrict__ tab, int res, float u, float v) {
    float x = u * (float)res - 0.5f;
    float y = v * (float)res - 0.5f;
    float xf = floorf(x), yf = floorf(y);
    float fx = x - xf, fy = y - yf;
    int x0 = (int)xf, y0 = (int)yf, x1 = x0 + 1, y1 = y0 + 1;
    x0 = min(max(x0, 0), res - 1);
    x1 = min(max(x1, 0), res - 1);
    y0 = min(max(y0, 0), res - 1);
    y1 = min(max(y1, 0), res - 1);
    float2 t00 = __ldg(tab + (size_t)y0 * res + x0), t10 = __ldg(tab + (size_t)y0 * res + x1);
    float2 t01 = __ldg(tab + (size_t)y1 * res + x0), t11 = __ldg(tab + (size_t)y1 * res + x1);
    float gx = 1.f - fx, gy = 1.f - fy;
    float2 o;
    o.x = (t00.x * gx + t10.x * fx) * gy + (t01.x * gx + t11.x * fx) * fy;
    o.y = (t00.y * gx + t10.y * fx) * gy + (t01.y * gx + t11.y * fx) * fy;
    return o;
}

struct EosTables {
    const float2 *forsterite;
    const float2 *fe;
    int res;
    float log_u_range;    // log(1 / ANEOS_MIN_U)
    float log_rho_range;  // log(1 / ANEOS_MIN_RHO)
};

// density.metal:45-53 / :228-235: (P, c) of a particle.
__device__ __forceinline__ float2 eos_lookup(const EosTables &e, int mat, float rho, float u) {
    float uc = logf(u / kAneosMinU) / e.log_u_range;
    float rc = logf(rho / kAneosMinRho) / e.log_rho_range;
    // clamp(v, 0, 1) with NaN passed through, as min(max(v, 0), 1) in C++
    uc = (uc < 0.f) ? 0.f : uc;
    uc = (1.f < uc) ? 1.f : uc;
    rc = (rc < 0.f) ? 0.f : rc;
    rc = (1.f < rc) ? 1.f : rc;
    const float2 *tab = ((float)mat == 400.f) ? e.forsterite : e.fe;
    return eos_sample(tab, e.res, uc, rc);
}

// Health word helpers.
__device__ __forceinline__ void raise_health(uint32_t *word, uint32_t bit) { atomicOr(word, bit); }

}  // namespace sph

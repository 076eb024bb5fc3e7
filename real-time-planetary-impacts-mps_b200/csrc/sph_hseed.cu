// sph_hseed.cu -- the learned smoothing-length seed: an 8 -> 64 -> 64 -> 1
// MLP that predicts, from a particle's state at the start of the density
// pass, the smoothing length the density iteration (density.metal:73-143)
// converges to.  The prediction only seeds that iteration; the iteration's
// own test still decides convergence, and a seed whose first sweep moves h by
// more than 5 % falls back to the plain initial guess (the density kernels,
// sph_hydro.cu).
// No counterpart in the reference.
//
// Features (per particle, before the pass): log h0, (dh/dt) dt / h0, the last
// pass's neighbour count / 64, log rho, log u, material (400 -> 0, else 1),
// the active flag, log2(1 + own timestep ticks) / 16; standardised by the mean
// and deviation of the first training set.  Target: log(h_converged / h0),
// standardised the same way.  Prediction: h_seed = h0 exp(target).
//
// Both the inference and the training kernels run the two 64-wide layers on
// the tensor cores with tcgen05: BF16 operands staged in shared memory in the
// canonical K-major layout, FP32 accumulators in tensor memory (TMEM), one
// thread issuing the MMAs and an mbarrier signalling their completion.  Each
// CTA takes a tile of 128 particles (thread t = row t = TMEM lane t):
//   forward   D1 = X W1^T (K 16), H1 = relu(D1 + b1);  D2 = H1 W2^T (K 64),
//             H2 = relu(D2 + b2);  y = H2 . w3 + b3 on the CUDA cores;
//   backward  dH2 = dy w3 (.) [D2 + b2 > 0];  D3 = dH2 W2 (K 64) -> dH1 = D3 (.) [D1 + b1 > 0];
//             dW2 = dH2^T H1 (K 128 rows) and dW1 = dH1^T X (K 128 rows) as
//             128-row MMAs whose upper 64 rows are zero; bias and w3
//             gradients by warp reductions; FP32 atomics into the gradient.
// Adam updates the FP32 master weights; the kernels convert them to BF16.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "sph_internal.h"
#include "sph_tc.cuh"

namespace sph {

namespace {

constexpr int kIn = 8, kInPad = 16, kHid = 64;
// parameter block (FP32): W1 [64][8], b1 [64], W2 [64][64], b2 [64], w3 [64], b3
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid, kNParams = kOffB3 + 1;
// normalisation block: feature mean [8], feature 1/deviation [8], target mean, target deviation
constexpr int kNorm = 2 * kIn + 2;
constexpr int kTile = 128;
constexpr int kMbarLimit = 1 << 24;

// shared-memory map of the MLP kernel (bytes)
constexpr uint32_t kSA1 = 0;                         // X        [128 x 16]
constexpr uint32_t kSW1 = kSA1 + kTile * kInPad * 2; // W1       [64 x 16]
constexpr uint32_t kSA2 = kSW1 + kHid * kInPad * 2;  // H1       [128 x 64]
constexpr uint32_t kSW2 = kSA2 + kTile * kHid * 2;   // W2       [64 x 64]  (B of layer 2)
constexpr uint32_t kFwdBytes = kSW2 + kHid * kHid * 2;
constexpr uint32_t kSW2T = kFwdBytes;                // W2^T     [64 x 64]  (B of dH1)
constexpr uint32_t kSA3 = kSW2T + kHid * kHid * 2;   // dH2      [128 x 64]
constexpr uint32_t kSA4 = kSA3 + kTile * kHid * 2;   // dH2^T    [128 x 128] (rows >= 64 zero)
constexpr uint32_t kSB4 = kSA4 + kTile * kTile * 2;  // H1^T     [64 x 128]
constexpr uint32_t kSA5 = kSB4 + kHid * kTile * 2;   // dH1^T    [128 x 128] (rows >= 64 zero)
constexpr uint32_t kSB5 = kSA5 + kTile * kTile * 2;  // X^T      [16 x 128]  (rows >= 8 zero)
constexpr uint32_t kTrainBytes = kSB5 + kInPad * kTile * 2;
// TMEM columns of the accumulators
constexpr uint32_t kD1 = 0, kD2 = 64, kD3 = 128, kD4 = 192, kD5 = 256;
// TMEM columns allocated: inference needs D1 and D2 only (several CTAs of it
// share an SM's 512 columns), training all five
template <int MODE>
__host__ __device__ constexpr uint32_t tmem_cols() { return MODE == 0 ? 128u : 512u; }

__device__ __forceinline__ void st_bf16(unsigned char *base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}

// The 8 raw features of particle i at the start of a density pass.
__device__ __forceinline__ void raw_features(const HSeedArgs &a, int i, float *f) {
    const float h0 = a.h[i];
    const float dt = kDtMin1 * (float)a.globals[1];
    f[0] = logf(h0);
    f[1] = a.dhdt[i] * dt / h0;
    f[2] = a.nn[i] * (1.f / 64.f);
    f[3] = logf(fmaxf(a.rho[i], 1e-30f));
    f[4] = logf(fmaxf(a.u[i], 1e-30f));
    f[5] = ((float)a.mat[i] == 400.f) ? 0.f : 1.f;
    f[6] = a.active[i] ? 1.f : 0.f;
    f[7] = log2f(1.f + (float)max(a.nat[i] - a.globals[0], 0)) * (1.f / 16.f);
}

// Record the features of every particle (training set, before the pass).
__global__ void k_hs_capture(HSeedArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    float f[kIn];
    raw_features(a, i, f);
#pragma unroll
    for (int k = 0; k < kIn; ++k) a.X[(size_t)i * kIn + k] = f[k];
    a.h0[i] = a.h[i];
}

// Training targets after the pass: log(h_fix / h0), h_fix = RESOLUTION_ETA
// (m / rho)^(1/3) (capped at MAX_H) from the converged density -- the fixed
// point the iteration approaches.  The converged h itself stops within
// DENSITY_ETA of it on the side the iteration came from, so it depends on
// the start: trained on it, a seed learns the plain start's lag, and once
// the seed starts the iteration the next step's h0 carries a different lag
// than the training pairs did, and the seed drifts off.  The fixed point does
// not depend on the start, and a seed at it converges in one sweep.
__global__ void k_hs_targets(HSeedArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float m = a.pos4[i].w, rho = fmaxf(a.rho[i], 1e-30f);
    const float h_fix = fminf(kResolutionEta * cbrtf(m / rho), kMaxH);
    a.y[i] = logf(h_fix / a.h0[i]);
}

// FP64 mean and second moment of the features and the target (block partials
// [blocks][2 * 9], summed in block order by k_hs_norm_total).
constexpr int kNormBlocks = 256;
__global__ void __launch_bounds__(256) k_hs_norm_partial(int n, const float *X, const float *y, double *part) {
    __shared__ double red[2 * (kIn + 1)][8];
    double s[2 * (kIn + 1)];
#pragma unroll
    for (int k = 0; k < 2 * (kIn + 1); ++k) s[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k <= kIn; ++k) {
            const double v = (k < kIn) ? (double)X[(size_t)i * kIn + k] : (double)y[i];
            s[2 * k] += v;
            s[2 * k + 1] += v * v;
        }
    }
#pragma unroll
    for (int k = 0; k < 2 * (kIn + 1); ++k) {
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 2 * (kIn + 1)) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[threadIdx.x][w];
        part[(size_t)blockIdx.x * 2 * (kIn + 1) + threadIdx.x] = t;
    }
}

__global__ void k_hs_norm_total(int n, const double *part, float *norm) {
    const int k = threadIdx.x;
    if (k > kIn) return;
    double s = 0.0, q = 0.0;
    for (int b = 0; b < kNormBlocks; ++b) {
        s += part[(size_t)b * 2 * (kIn + 1) + 2 * k];
        q += part[(size_t)b * 2 * (kIn + 1) + 2 * k + 1];
    }
    const double mean = s / n, var = fmax(q / n - mean * mean, 0.0);
    const double dev = sqrt(var) > 1e-6 ? sqrt(var) : 1.0;
    if (k < kIn) {
        norm[k] = (float)mean;
        norm[kIn + k] = (float)(1.0 / dev);
    } else {
        norm[2 * kIn] = (float)mean;
        norm[2 * kIn + 1] = (float)dev;
    }
}

// Row index of a training sample: a multiplicative hash of the global row.
__device__ __forceinline__ int sample_row(uint32_t it, uint32_t row, int batch, int n, uint32_t salt) {
    const uint64_t g = (uint64_t)it * (uint64_t)batch + row;
    return (int)(((g * 0x9E3779B97F4A7C15ull) ^ salt) % (uint64_t)n);
}

// MODE 0: inference (features from the state, writes the seed); MODE 1:
// gradients of the loss 1/2 mean (y - t)^2 over `batch` sampled rows.
// MODE 1 samples its rows for iteration it + *it_base (it_base may be null).
template <int MODE>
__global__ void __launch_bounds__(kTile) k_mlp(HSeedArgs a, uint32_t it, int batch, const uint32_t *it_base) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    __shared__ float red_w3[4][kHid], red_b2[4][kHid], red_b1[4][kHid], red_b3[4];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const float *P = a.params;
    const float *norm = a.norm;
    // --- set-up: TMEM, barrier, weights in BF16 -----------------------------
    if (warp == 0) {
        tc::tmem_alloc(&tmem_slot, tmem_cols<MODE>());
        tc::fence_before_sync();
    }
    if (t == 0) tc::mbar_init(&bar, 1);
    for (int q = t; q < kHid * kInPad; q += kTile) {
        const int j = q / kInPad, i = q % kInPad;
        st_bf16(sm + kSW1, tc::kmajor_off(j, i, kInPad), i < kIn ? P[kOffW1 + j * kIn + i] : 0.f);
    }
    for (int q = t; q < kHid * kHid; q += kTile) {
        const int j = q / kHid, i = q % kHid;
        const float w = P[kOffW2 + j * kHid + i];
        st_bf16(sm + kSW2, tc::kmajor_off(j, i, kHid), w);
        if (MODE == 1) st_bf16(sm + kSW2T, tc::kmajor_off(i, j, kHid), w);
    }
    if (MODE == 1) {
        // zero rows of the padded operands
        for (int q = t; q < (kTile - kHid) * kTile; q += kTile) {
            const int row = kHid + q / kTile, k = q % kTile;
            st_bf16(sm + kSA4, tc::kmajor_off(row, k, kTile), 0.f);
            st_bf16(sm + kSA5, tc::kmajor_off(row, k, kTile), 0.f);
        }
        for (int q = t; q < (kInPad - kIn) * kTile; q += kTile)
            st_bf16(sm + kSB5, tc::kmajor_off(kIn + q / kTile, q % kTile, kTile), 0.f);
    }
    // --- this thread's row: features -> X ------------------------------------
    int row = -1;
    bool valid = false;
    float x[kIn];
    float target = 0.f;
    if (MODE == 0) {
        row = blockIdx.x * kTile + t;
        valid = row < a.n;
        if (valid) raw_features(a, row, x);
    } else {
        valid = (int)(blockIdx.x * kTile + t) < batch;
        if (valid) {
            row = sample_row(it + (it_base ? *it_base : 0u), blockIdx.x * kTile + t, batch, a.n, a.salt);
#pragma unroll
            for (int k = 0; k < kIn; ++k) x[k] = a.X[(size_t)row * kIn + k];
            target = (a.y[row] - norm[2 * kIn]) / norm[2 * kIn + 1];
        }
    }
#pragma unroll
    for (int k = 0; k < kIn; ++k) x[k] = valid ? (x[k] - norm[k]) * norm[kIn + k] : 0.f;
#pragma unroll
    for (int k = 0; k < kInPad; ++k) {
        const float v = k < kIn ? x[k] : 0.f;
        st_bf16(sm + kSA1, tc::kmajor_off(t, k, kInPad), v);
        if (MODE == 1 && k < kIn) st_bf16(sm + kSB5, tc::kmajor_off(k, t, kTile), v);
    }
    tc::fence_async_smem();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tmem_slot;
    const uint32_t lane_base = tm + ((uint32_t)(warp * 32) << 16);
    const uint32_t sbase = tc::smem_u32(sm);
    uint32_t phase = 0;
    bool ok = true;
    auto run = [&](auto &&issue) {
        if (t == 0) {
            issue();
            tc::mma_commit(&bar);
        }
        if (!tc::mbar_wait(&bar, phase, kMbarLimit)) ok = false;
        phase ^= 1u;
        tc::fence_after_sync();
    };
    // --- layer 1 --------------------------------------------------------------
    run([&] {
        tc::mma_bf16(tm + kD1, tc::kmajor_desc(sbase + kSA1, kInPad), tc::kmajor_desc(sbase + kSW1, kInPad),
                     tc::idesc_bf16_m128(kHid), false);
    });
    uint64_t mask1 = 0ull;
    float v[16];
#pragma unroll
    for (int c = 0; c < kHid; c += 16) {
        tc::tmem_ld16(lane_base + kD1 + c, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int j = c + q;
            const float z = v[q] + P[kOffB1 + j];
            const float hval = z > 0.f ? z : 0.f;
            if (z > 0.f) mask1 |= 1ull << j;
            st_bf16(sm + kSA2, tc::kmajor_off(t, j, kHid), hval);
            if (MODE == 1) st_bf16(sm + kSB4, tc::kmajor_off(j, t, kTile), hval);
        }
    }
    tc::fence_before_sync();
    tc::fence_async_smem();
    __syncthreads();
    tc::fence_after_sync();
    // --- layer 2 --------------------------------------------------------------
    run([&] {
        for (int s = 0; s < kHid / 16; ++s)
            tc::mma_bf16(tm + kD2, tc::kmajor_desc(sbase + kSA2 + s * 256, kHid),
                         tc::kmajor_desc(sbase + kSW2 + s * 256, kHid), tc::idesc_bf16_m128(kHid), s > 0);
    });
    float yhat = P[kOffB3];
    uint64_t mask2 = 0ull;
    float h2[kHid];
#pragma unroll
    for (int c = 0; c < kHid; c += 16) {
        tc::tmem_ld16(lane_base + kD2 + c, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int j = c + q;
            const float z = v[q] + P[kOffB2 + j];
            h2[j] = z > 0.f ? z : 0.f;
            if (z > 0.f) mask2 |= 1ull << j;
            yhat += h2[j] * P[kOffW3 + j];
        }
    }
    if (MODE == 0) {
        if (valid && ok) {
            const float pred = norm[2 * kIn] + norm[2 * kIn + 1] * yhat;
            a.seed[row] = a.h[row] * expf(pred);
        }
    } else {
        // --- backward -----------------------------------------------------------
        const float dy = valid ? (yhat - target) / (float)batch : 0.f;
        if (valid) atomicAdd(a.loss, 0.5f * (yhat - target) * (yhat - target) / (float)batch);
#pragma unroll
        for (int j = 0; j < kHid; ++j) {
            const float g = ((mask2 >> j) & 1ull) ? dy * P[kOffW3 + j] : 0.f;
            st_bf16(sm + kSA3, tc::kmajor_off(t, j, kHid), g);
            st_bf16(sm + kSA4, tc::kmajor_off(j, t, kTile), g);
            // sums over the tile's rows: w3, b2
            float s3 = dy * h2[j], s2 = g;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                s3 += __shfl_xor_sync(0xffffffffu, s3, o);
                s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            }
            if (lane == 0) {
                red_w3[warp][j] = s3;
                red_b2[warp][j] = s2;
            }
        }
        float s = dy;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red_b3[warp] = s;
        tc::fence_before_sync();
        tc::fence_async_smem();
        __syncthreads();
        tc::fence_after_sync();
        if (t < kHid) {
            atomicAdd(a.grads + kOffW3 + t, red_w3[0][t] + red_w3[1][t] + red_w3[2][t] + red_w3[3][t]);
            atomicAdd(a.grads + kOffB2 + t, red_b2[0][t] + red_b2[1][t] + red_b2[2][t] + red_b2[3][t]);
        }
        if (t == 0) atomicAdd(a.grads + kOffB3, red_b3[0] + red_b3[1] + red_b3[2] + red_b3[3]);
        // dH1 = dH2 W2 and dW2 = dH2^T H1
        run([&] {
            for (int s2 = 0; s2 < kHid / 16; ++s2)
                tc::mma_bf16(tm + kD3, tc::kmajor_desc(sbase + kSA3 + s2 * 256, kHid),
                             tc::kmajor_desc(sbase + kSW2T + s2 * 256, kHid), tc::idesc_bf16_m128(kHid), s2 > 0);
            for (int s2 = 0; s2 < kTile / 16; ++s2)
                tc::mma_bf16(tm + kD4, tc::kmajor_desc(sbase + kSA4 + s2 * 256, kTile),
                             tc::kmajor_desc(sbase + kSB4 + s2 * 256, kTile), tc::idesc_bf16_m128(kHid), s2 > 0);
        });
#pragma unroll
        for (int c = 0; c < kHid; c += 16) {
            tc::tmem_ld16(lane_base + kD3 + c, v);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int j = c + q;
                const float g = ((mask1 >> j) & 1ull) ? v[q] : 0.f;
                st_bf16(sm + kSA5, tc::kmajor_off(j, t, kTile), g);
                float s1 = g;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                if (lane == 0) red_b1[warp][j] = s1;
            }
        }
#pragma unroll
        for (int c = 0; c < kHid; c += 16) {
            tc::tmem_ld16(lane_base + kD4 + c, v);  // row t of dW2 (t < 64)
            if (t < kHid && ok)
#pragma unroll
                for (int q = 0; q < 16; ++q) atomicAdd(a.grads + kOffW2 + t * kHid + c + q, v[q]);
        }
        tc::fence_before_sync();
        tc::fence_async_smem();
        __syncthreads();
        tc::fence_after_sync();
        if (t < kHid) atomicAdd(a.grads + kOffB1 + t, red_b1[0][t] + red_b1[1][t] + red_b1[2][t] + red_b1[3][t]);
        // dW1 = dH1^T X
        run([&] {
            for (int s2 = 0; s2 < kTile / 16; ++s2)
                tc::mma_bf16(tm + kD5, tc::kmajor_desc(sbase + kSA5 + s2 * 256, kTile),
                             tc::kmajor_desc(sbase + kSB5 + s2 * 256, kTile), tc::idesc_bf16_m128(kInPad), s2 > 0);
        });
        tc::tmem_ld16(lane_base + kD5, v);
        if (t < kHid && ok)
#pragma unroll
            for (int q = 0; q < kIn; ++q) atomicAdd(a.grads + kOffW1 + t * kIn + q, v[q]);
    }
    if (!ok && t == 0) raise_health(a.health, SPH_HEALTH_MLP_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tm, tmem_cols<MODE>());
}

// Adam on the FP32 master weights (one CTA); clears the gradient and counts
// the step in the device counter *step, so that replays of a captured graph
// keep counting (bias correction, sample rows).
constexpr int kAdamThreads = 1024;
__global__ void __launch_bounds__(kAdamThreads) k_adam(float *params, float *grads, float *m, float *v,
                                                        uint32_t *step, float lr) {
    const float s = (float)(*step + 1u);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - powf(b1, s), c2 = 1.f - powf(b2, s);
    for (int k = threadIdx.x; k < kNParams; k += kAdamThreads) {
        const float g = grads[k];
        const float mk = b1 * m[k] + (1.f - b1) * g;
        const float vk = b2 * v[k] + (1.f - b2) * g * g;
        m[k] = mk;
        v[k] = vk;
        params[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
        grads[k] = 0.f;
    }
    __syncthreads();  // every thread has read *step
    if (threadIdx.x == 0) *step += 1u;
}

}  // namespace

size_t hseed_smem_bytes(bool train) { return train ? kTrainBytes : kFwdBytes; }
int hseed_num_params() { return kNParams; }
int hseed_norm_size() { return kNorm; }

sph_status hseed_alloc(sph_ctx *ctx) {
    HSeed &hs = ctx->hs;
    if (hs.params) return SPH_OK;
    const size_t n = (size_t)ctx->n;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    chk(cudaMalloc(&hs.params, sizeof(float) * kNParams));
    chk(cudaMalloc(&hs.grads, sizeof(float) * kNParams));
    chk(cudaMalloc(&hs.adam_m, sizeof(float) * kNParams));
    chk(cudaMalloc(&hs.adam_v, sizeof(float) * kNParams));
    chk(cudaMalloc(&hs.norm, sizeof(float) * kNorm));
    chk(cudaMalloc(&hs.norm_part, sizeof(double) * kNormBlocks * 2 * (kIn + 1)));
    chk(cudaMalloc(&hs.X, sizeof(float) * kIn * n));
    chk(cudaMalloc(&hs.y, sizeof(float) * n));
    chk(cudaMalloc(&hs.h0, sizeof(float) * n));
    chk(cudaMalloc(&hs.nn, sizeof(float) * n));
    chk(cudaMalloc(&hs.seed, sizeof(float) * n));
    chk(cudaMalloc(&hs.loss, sizeof(float)));
    chk(cudaMalloc(&hs.stats, sizeof(uint32_t) * 4));
    chk(cudaMalloc(&hs.adam_step, sizeof(uint32_t)));
    if (e != cudaSuccess) return cuda_status(e, "learned h seed buffers");
    // He-style initialisation, seeded (the host draws, the device keeps)
    std::vector<float> p(kNParams, 0.f);
    uint64_t state = 0x2545F4914F6CDD1Dull;
    auto uni = [&]() {
        state ^= state << 13;
        state ^= state >> 7;
        state ^= state << 17;
        return (float)((state >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    for (int k = 0; k < kHid * kIn; ++k) p[kOffW1 + k] = uni() * std::sqrt(6.f / kIn);
    for (int k = 0; k < kHid * kHid; ++k) p[kOffW2 + k] = uni() * std::sqrt(6.f / kHid);
    for (int k = 0; k < kHid; ++k) p[kOffW3 + k] = uni() * std::sqrt(3.f / kHid) * 0.1f;
    std::vector<float> nrm(kNorm, 0.f);
    for (int k = 0; k < kIn; ++k) nrm[kIn + k] = 1.f;
    nrm[2 * kIn + 1] = 1.f;
    chk(cudaMemcpy(hs.params, p.data(), sizeof(float) * kNParams, cudaMemcpyHostToDevice));
    chk(cudaMemcpy(hs.norm, nrm.data(), sizeof(float) * kNorm, cudaMemcpyHostToDevice));
    chk(cudaMemset(hs.grads, 0, sizeof(float) * kNParams));
    chk(cudaMemset(hs.adam_m, 0, sizeof(float) * kNParams));
    chk(cudaMemset(hs.adam_v, 0, sizeof(float) * kNParams));
    chk(cudaMemset(hs.nn, 0, sizeof(float) * n));
    chk(cudaMemset(hs.stats, 0, sizeof(uint32_t) * 4));
    chk(cudaMemset(hs.adam_step, 0, sizeof(uint32_t)));
    if (e == cudaSuccess) {
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_mlp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdBytes);
            cudaFuncSetAttribute(k_mlp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainBytes);
            attr = true;
        }
    }
    return cuda_status(e, "learned h seed init");
}

void hseed_free(sph_ctx *ctx) {
    HSeed &hs = ctx->hs;
    void *bufs[] = {hs.params, hs.grads, hs.adam_m, hs.adam_v, hs.norm,  hs.norm_part, hs.X,
                    hs.y,      hs.h0,    hs.nn,     hs.seed,   hs.loss, hs.stats,     hs.adam_step};
    for (void *b : bufs) cudaFree(b);
    hs = HSeed();
}

HSeedArgs hseed_args(sph_ctx *ctx) {
    HSeed &hs = ctx->hs;
    HSeedArgs a;
    a.n = ctx->n;
    a.pos4 = ctx->pos4;
    a.h = ctx->h;
    a.dhdt = ctx->dhdt;
    a.rho = ctx->rho;
    a.u = ctx->u;
    a.mat = ctx->mat;
    a.nat = ctx->nat;
    a.active = ctx->active;
    a.globals = ctx->globals;
    a.nn = hs.nn;
    a.X = hs.X;
    a.y = hs.y;
    a.h0 = hs.h0;
    a.seed = hs.seed;
    a.params = hs.params;
    a.grads = hs.grads;
    a.norm = hs.norm;
    a.loss = hs.loss;
    a.health = ctx->health;
    a.salt = 0u;
    return a;
}

sph_status launch_hseed_capture(sph_ctx *ctx, cudaStream_t st) {
    sph_status s = hseed_alloc(ctx);
    if (s != SPH_OK) return s;
    k_hs_capture<<<(ctx->n + 255) / 256, 256, 0, st>>>(hseed_args(ctx));
    return cuda_status(cudaGetLastError(), "h seed capture");
}

sph_status launch_hseed_targets(sph_ctx *ctx, cudaStream_t st) {
    k_hs_targets<<<(ctx->n + 255) / 256, 256, 0, st>>>(hseed_args(ctx));
    ctx->hs.have_data = true;
    return cuda_status(cudaGetLastError(), "h seed targets");
}

sph_status launch_hseed_infer(sph_ctx *ctx, cudaStream_t st) {
    sph_status s = hseed_alloc(ctx);
    if (s != SPH_OK) return s;
    const int tiles = (ctx->n + kTile - 1) / kTile;
    k_mlp<0><<<tiles, kTile, kFwdBytes, st>>>(hseed_args(ctx), 0u, 0, nullptr);
    return cuda_status(cudaGetLastError(), "h seed inference");
}

sph_status launch_hseed_norm(sph_ctx *ctx, cudaStream_t st) {
    HSeed &hs = ctx->hs;
    k_hs_norm_partial<<<kNormBlocks, 256, 0, st>>>(ctx->n, hs.X, hs.y, hs.norm_part);
    k_hs_norm_total<<<1, 32, 0, st>>>(ctx->n, hs.norm_part, hs.norm);
    hs.have_norm = true;
    return cuda_status(cudaGetLastError(), "h seed normalisation");
}

// Gradients of a minibatch: rows of iteration it (+ the Adam step counter
// when counted).
sph_status launch_hseed_grad(sph_ctx *ctx, uint32_t it, bool counted, int batch, uint32_t salt, cudaStream_t st) {
    HSeedArgs a = hseed_args(ctx);
    a.salt = salt;
    const int tiles = (batch + kTile - 1) / kTile;
    k_mlp<1><<<tiles, kTile, kTrainBytes, st>>>(a, it, batch, counted ? ctx->hs.adam_step : nullptr);
    return cuda_status(cudaGetLastError(), "h seed gradient");
}

sph_status launch_hseed_adam(sph_ctx *ctx, float lr, cudaStream_t st) {
    HSeed &hs = ctx->hs;
    k_adam<<<1, kAdamThreads, 0, st>>>(hs.params, hs.grads, hs.adam_m, hs.adam_v, hs.adam_step, lr);
    return cuda_status(cudaGetLastError(), "h seed update");
}

// Standardisation from the recorded pass, then `iterations` Adam steps (the
// minibatch of step s is drawn by s + 1); stream-ordered, graph-capturable.
sph_status launch_hseed_steps(sph_ctx *ctx, int iterations, int batch, float lr, cudaStream_t st) {
    sph_status s = launch_hseed_norm(ctx, st);
    for (int i = 0; i < iterations && s == SPH_OK; ++i) {
        s = launch_hseed_grad(ctx, 1u, true, batch, 0x5bd1e995u, st);
        if (s == SPH_OK) s = launch_hseed_adam(ctx, lr, st);
    }
    return s;
}

bool hseed_online_due(const sph_ctx *ctx) {
    return ctx->form.h_seed == SPH_HSEED_LEARNED && ctx->hs.online_iters > 0 && ctx->hs.have_data;
}

sph_status launch_hseed_online(sph_ctx *ctx, cudaStream_t st) {
    return launch_hseed_steps(ctx, ctx->hs.online_iters, ctx->hs.online_batch, ctx->hs.online_lr, st);
}

}  // namespace sph

using namespace sph;

extern "C" {

int32_t sph_hseed_num_params(void) { return kNParams; }

sph_status sph_hseed_capture(sph_ctx *ctx, int32_t on) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (on) {
        sph_status s = hseed_alloc(ctx);
        if (s != SPH_OK) return s;
    }
    drop_graphs(ctx);
    ctx->hs.capture = on != 0;
    return SPH_OK;
}

sph_status sph_hseed_train(sph_ctx *ctx, int32_t iterations, int32_t batch, float lr, float *loss, void *stream) {
    if (!ctx || iterations < 0 || batch < 1 || batch > (1 << 22) || !(lr > 0.f)) {
        set_error("sph_hseed_train: bad arguments");
        return SPH_ERR_INVALID_ARG;
    }
    if (!ctx->hs.have_data) {
        set_error("sph_hseed_train: no recorded density pass (sph_hseed_capture, then a density pass)");
        return SPH_ERR_INVALID_ARG;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    // the standardisation follows the recorded pass (the first pass after the
    // initial conditions has no neighbour counts or dh/dt yet)
    sph_status s = iterations > 0 ? launch_hseed_steps(ctx, iterations - 1, batch, lr, st) : SPH_OK;
    float last = 0.f;
    if (s == SPH_OK && iterations > 0) {
        // the last step also reports its minibatch loss
        cudaMemsetAsync(ctx->hs.loss, 0, sizeof(float), st);
        s = launch_hseed_grad(ctx, 1u, true, batch, 0x5bd1e995u, st);
        if (s == SPH_OK) s = launch_hseed_adam(ctx, lr, st);
    }
    if (s != SPH_OK) return s;
    if (iterations > 0) {
        cudaError_t e = cudaMemcpyAsync(&last, ctx->hs.loss, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e, "sph_hseed_train");
    }
    if (loss) *loss = last;
    return SPH_OK;
}

sph_status sph_hseed_online(sph_ctx *ctx, int32_t iterations, int32_t batch, float lr) {
    if (!ctx || iterations < 0 || iterations > 4096 || batch < 1 || batch > (1 << 22) || !(lr > 0.f)) {
        set_error("sph_hseed_online: bad arguments");
        return SPH_ERR_INVALID_ARG;
    }
    cudaSetDevice(ctx->device);
    if (iterations > 0) {
        sph_status s = hseed_alloc(ctx);
        if (s != SPH_OK) return s;
    }
    drop_graphs(ctx);
    ctx->hs.online_iters = iterations;
    ctx->hs.online_batch = batch;
    ctx->hs.online_lr = lr;
    // every density pass records its pairs while the refresh is on
    ctx->hs.capture = iterations > 0;
    return SPH_OK;
}

sph_status sph_hseed_gradient(sph_ctx *ctx, int32_t batch, uint32_t salt, float *grads, float *loss, void *stream) {
    if (!ctx || batch < 1 || batch > (1 << 22) || !grads) {
        set_error("sph_hseed_gradient: bad arguments");
        return SPH_ERR_INVALID_ARG;
    }
    if (!ctx->hs.have_data) {
        set_error("sph_hseed_gradient: no recorded density pass");
        return SPH_ERR_INVALID_ARG;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    sph_status s = SPH_OK;
    if (!ctx->hs.have_norm) s = launch_hseed_norm(ctx, st);
    if (s != SPH_OK) return s;
    cudaMemsetAsync(ctx->hs.grads, 0, sizeof(float) * kNParams, st);
    cudaMemsetAsync(ctx->hs.loss, 0, sizeof(float), st);
    s = launch_hseed_grad(ctx, 0u, false, batch, salt, st);
    if (s != SPH_OK) return s;
    float l = 0.f;
    cudaError_t e = cudaMemcpyAsync(grads, ctx->hs.grads, sizeof(float) * kNParams, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&l, ctx->hs.loss, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->hs.grads, 0, sizeof(float) * kNParams, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "sph_hseed_gradient");
    if (loss) *loss = l;
    return SPH_OK;
}

sph_status sph_hseed_params(sph_ctx *ctx, float *get, const float *set) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    sph_status s = hseed_alloc(ctx);
    if (s != SPH_OK) return s;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && get)
        e = cudaMemcpy(get, ctx->hs.params, sizeof(float) * kNParams, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && set)
        e = cudaMemcpy(ctx->hs.params, set, sizeof(float) * kNParams, cudaMemcpyHostToDevice);
    return cuda_status(e, "sph_hseed_params");
}

sph_status sph_hseed_norm(sph_ctx *ctx, float *get, const float *set) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    sph_status s = hseed_alloc(ctx);
    if (s != SPH_OK) return s;
    if (get && !ctx->hs.have_norm) {
        set_error("sph_hseed_norm: no standardisation yet (sph_hseed_train computes it)");
        return SPH_ERR_INVALID_ARG;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && get) e = cudaMemcpy(get, ctx->hs.norm, sizeof(float) * kNorm, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && set) {
        e = cudaMemcpy(ctx->hs.norm, set, sizeof(float) * kNorm, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) ctx->hs.have_norm = true;
    }
    return cuda_status(e, "sph_hseed_norm");
}

sph_status sph_hseed_dataset(sph_ctx *ctx, float *features, float *targets, float *norm) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    if (!ctx->hs.have_data) {
        set_error("sph_hseed_dataset: no recorded density pass");
        return SPH_ERR_INVALID_ARG;
    }
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaDeviceSynchronize();
    const size_t n = (size_t)ctx->n;
    if (e == cudaSuccess && features)
        e = cudaMemcpy(features, ctx->hs.X, sizeof(float) * kIn * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && targets) e = cudaMemcpy(targets, ctx->hs.y, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && norm) e = cudaMemcpy(norm, ctx->hs.norm, sizeof(float) * kNorm, cudaMemcpyDeviceToHost);
    return cuda_status(e, "sph_hseed_dataset");
}

sph_status sph_hseed_get_stats(sph_ctx *ctx, sph_hseed_stats *out) {
    if (!ctx || !out) return SPH_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    std::memset(out, 0, sizeof(*out));
    uint32_t v[4] = {0, 0, 0, 0}, t[16] = {};
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && ctx->tile_ctr) e = cudaMemcpy(t, ctx->tile_ctr, sizeof(t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "sph_hseed_get_stats");
    out->tiles = t[0];
    out->deferred = t[2];
    out->accel_deferred = t[10];
    out->coarse_tiles = t[4];
    out->accel_coarse_tiles = t[12];
    if (!ctx->hs.stats) return SPH_OK;
    e = cudaMemcpy(v, ctx->hs.stats, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "sph_hseed_get_stats");
    out->sweeps = v[0];
    out->fallbacks = v[1];
    out->max_sweeps = v[2];
    out->particles = v[3];
    return SPH_OK;
}

}  // extern "C"

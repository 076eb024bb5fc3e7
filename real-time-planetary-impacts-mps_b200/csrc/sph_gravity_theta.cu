// sph_gravity_theta.cu -- the opening-angle gravity form and the FP64 direct
// sum it is measured against.  Neither has a counterpart in the reference,
// whose gravity (Compute.cpp:328-377, sph_gravity.cu here) uses an adaptive
// acceptance test without an opening angle, force-accepts failing leaves and
// keeps integer-truncated softening coefficients (kernels.h:93,97).
//
// Tree: the GPU Morton octree (sph_tree.cu), whose leaves hold contiguous
// runs of the particles in key order.  Up pass, one launch per level: per
// node the mass, centre of mass, the second moments Q_jk = sum m r_j r_k about
// the centre of mass, and the radius of the smallest sphere about the centre
// of mass that holds the node's box.
//
// Evaluation is a group walk: a warp takes 32 consecutive particles in key
// order (a compact group) and traverses the tree from the root, 32 nodes at a
// time from a queue.  A node is accepted for the whole group when
//     r_node < theta * d   and   d > 2 eps,
// d being the distance from its centre of mass to the group's bounding box
// (so every particle of the group sees it under an angle below theta and
// outside the softening support); accepted nodes are evaluated at each
// particle (M2P: monopole + quadrupole, potential and acceleration), rejected
// leaves are summed particle by particle (P2P with the cubic-spline softened
// kernel and its exact coefficients), rejected branches put their children on
// the queue.  Accepted nodes and rejected leaves are staged in shared memory
// and evaluated in batches with every lane busy; each batch's partial sums
// are added into Kahan-compensated per-particle accumulators.  The walk
// writes acc = G a, |a| (the reference's gravNorm) and the potential G phi.
#include <cuda_runtime.h>

#include "sph_internal.h"

namespace sph {

namespace {

// Layout of a theta-form node record (kPoleQ float4 per node):
//   q0 (com.xyz, radius)  q1 (M, Qxx, Qxy, Qxz)  q2 (Qyy, Qyz, Qzz, 0)
//   q3 (bbox min, 0)      q4 (bbox max, 1)

__device__ __forceinline__ float corner_radius(float cx, float cy, float cz, float mnx, float mny, float mnz,
                                               float mxx, float mxy, float mxz) {
    const float dx = fmaxf(cx - mnx, mxx - cx), dy = fmaxf(cy - mny, mxy - cy), dz = fmaxf(cz - mnz, mxz - cz);
    return sqrtf(dx * dx + dy * dy + dz * dz);
}

struct ThetaUpArgs {
    const int32_t *T;
    const int32_t *level_nodes;
    const int32_t *level_count;
    const int32_t *list_slot;
    int32_t *parent_slot;
    float4 *poles;
    const float4 *pos4;
    uint8_t *active;
    const int32_t *nat;
    const int32_t *globals;
    int individual;  // SPH_TIMESTEP_INDIVIDUAL: activity from the next active times, synced per leaf
};

__device__ void p2m_theta(const ThetaUpArgs &a, int tp, int dp) {
    const int32_t *T = a.T;
    const int np = T[tp];
    const int s = tp + 2;
    // sums relative to the first particle: no cancellation at large |x|
    const float4 x0 = a.pos4[T[s]];
    float m = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
    float mnx = x0.x, mny = x0.y, mnz = x0.z, mxx = x0.x, mxy = x0.y, mxz = x0.z;
    // individual timesteps: the leaf is active when one of its particles is
    // due, and then all of them are (README.md:62-64); otherwise all are
    bool act = true;
    if (a.individual) {
        const int gt = a.globals[0];
        act = false;
        for (int i = 0; i < np && !act; ++i) act = gt >= a.nat[T[s + i]];
    }
    for (int i = 0; i < np; ++i) {
        const int p = T[s + i];
        const float4 q = a.pos4[p];
        a.active[p] = act ? 1 : 0;
        m += q.w;
        sx += q.w * (q.x - x0.x);
        sy += q.w * (q.y - x0.y);
        sz += q.w * (q.z - x0.z);
        mnx = fminf(mnx, q.x);
        mny = fminf(mny, q.y);
        mnz = fminf(mnz, q.z);
        mxx = fmaxf(mxx, q.x);
        mxy = fmaxf(mxy, q.y);
        mxz = fmaxf(mxz, q.z);
    }
    const float ox = sx / m, oy = sy / m, oz = sz / m;  // com - x0
    float qxx = 0.f, qxy = 0.f, qxz = 0.f, qyy = 0.f, qyz = 0.f, qzz = 0.f;
    for (int i = 0; i < np; ++i) {
        const float4 q = a.pos4[T[s + i]];
        const float rx = (q.x - x0.x) - ox, ry = (q.y - x0.y) - oy, rz = (q.z - x0.z) - oz;
        qxx += q.w * rx * rx;
        qxy += q.w * rx * ry;
        qxz += q.w * rx * rz;
        qyy += q.w * ry * ry;
        qyz += q.w * ry * rz;
        qzz += q.w * rz * rz;
    }
    const float cx = x0.x + ox, cy = x0.y + oy, cz = x0.z + oz;
    float4 *pr = a.poles + (size_t)dp * kPoleQ;
    pr[0] = make_float4(cx, cy, cz, corner_radius(cx, cy, cz, mnx, mny, mnz, mxx, mxy, mxz));
    pr[1] = make_float4(m, qxx, qxy, qxz);
    pr[2] = make_float4(qyy, qyz, qzz, 0.f);
    pr[3] = make_float4(mnx, mny, mnz, 0.f);
    pr[4] = make_float4(mxx, mxy, mxz, act ? 1.f : 0.f);
    pr[5] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__device__ void m2m_theta(const ThetaUpArgs &a, int tp, int dp) {
    const int32_t *T = a.T;
    const int my_slot = a.list_slot[dp];
    int first = -1;
    float4 c0f = make_float4(0.f, 0.f, 0.f, 0.f);
    float m = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
    float mnx = 3.402823466e+38f, mny = mnx, mnz = mnx, mxx = -mnx, mxy = -mnx, mxz = -mnx;
    for (int k = 0; k < 8; ++k) {
        const int c = T[tp + 2 + k];
        if (c == -1) continue;
        const int cdp = T[c + 1];
        a.parent_slot[cdp] = my_slot;
        const float4 *cp = a.poles + (size_t)cdp * kPoleQ;
        const float4 q0 = cp[0], q1 = cp[1], q3 = cp[3], q4 = cp[4];
        if (first < 0) {
            first = k;
            c0f = q0;
        }
        m += q1.x;
        sx += q1.x * (q0.x - c0f.x);
        sy += q1.x * (q0.y - c0f.y);
        sz += q1.x * (q0.z - c0f.z);
        mnx = fminf(mnx, q3.x);
        mny = fminf(mny, q3.y);
        mnz = fminf(mnz, q3.z);
        mxx = fmaxf(mxx, q4.x);
        mxy = fmaxf(mxy, q4.y);
        mxz = fmaxf(mxz, q4.z);
    }
    const float ox = sx / m, oy = sy / m, oz = sz / m;
    float qxx = 0.f, qxy = 0.f, qxz = 0.f, qyy = 0.f, qyz = 0.f, qzz = 0.f;
    for (int k = 0; k < 8; ++k) {
        const int c = T[tp + 2 + k];
        if (c == -1) continue;
        const float4 *cp = a.poles + (size_t)T[c + 1] * kPoleQ;
        const float4 q0 = cp[0], q1 = cp[1], q2 = cp[2];
        const float rx = (q0.x - c0f.x) - ox, ry = (q0.y - c0f.y) - oy, rz = (q0.z - c0f.z) - oz;
        const float mc = q1.x;
        qxx += q1.y + mc * rx * rx;
        qxy += q1.z + mc * rx * ry;
        qxz += q1.w + mc * rx * rz;
        qyy += q2.x + mc * ry * ry;
        qyz += q2.y + mc * ry * rz;
        qzz += q2.z + mc * rz * rz;
    }
    // individual timesteps: a branch is active when a child is; a branch
    // whose children are all leaves activates every leaf and particle under
    // it when one leaf is active (README.md:64)
    bool act = true;
    if (a.individual) {
        act = false;
        bool all_leaves = true;
        for (int k = 0; k < 8; ++k) {
            const int c = T[tp + 2 + k];
            if (c == -1) continue;
            if (a.poles[(size_t)T[c + 1] * kPoleQ + 4].w != 0.f) act = true;
            if (T[c] == 0) all_leaves = false;
        }
        if (act && all_leaves) {
            for (int k = 0; k < 8; ++k) {
                const int c = T[tp + 2 + k];
                if (c == -1) continue;
                a.poles[(size_t)T[c + 1] * kPoleQ + 4].w = 1.f;
                for (int j = 0; j < T[c]; ++j) a.active[T[c + 2 + j]] = 1;
            }
        }
    }
    const float cx = c0f.x + ox, cy = c0f.y + oy, cz = c0f.z + oz;
    float4 *pr = a.poles + (size_t)dp * kPoleQ;
    pr[0] = make_float4(cx, cy, cz, corner_radius(cx, cy, cz, mnx, mny, mnz, mxx, mxy, mxz));
    pr[1] = make_float4(m, qxx, qxy, qxz);
    pr[2] = make_float4(qyy, qyz, qzz, 0.f);
    pr[3] = make_float4(mnx, mny, mnz, 0.f);
    pr[4] = make_float4(mxx, mxy, mxz, act ? 1.f : 0.f);
    pr[5] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void k_up_theta(ThetaUpArgs a, int level, int64_t level_cap) {
    const int cnt = a.level_count[level];
    const int32_t *nodes = a.level_nodes + (size_t)level * level_cap;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int tp = nodes[t];
        const int dp = a.T[tp + 1];
        if (a.T[tp] == 0)
            m2m_theta(a, tp, dp);
        else
            p2m_theta(a, tp, dp);
    }
}

// Cubic-spline softened pair kernel with its exact coefficients (the
// reference's kernels.h:87-102 truncates them): force factor f(r) with
// a = -m f(r) R / r, and potential phi(r) (both -> Newtonian for r >= 2 eps).
__device__ __forceinline__ void soft_pair(float r, float &fr, float &pot) {
    const float h = kGravSoft;
    const float h1 = 1.f / h;
    const float q = r * h1;
    if (q >= 2.f) {
        const float r1 = 1.f / r;
        fr = r1 * r1;
        pot = -r1;
    } else if (q > 1.f) {
        const float q2 = q * q;
        fr = (h1 * h1) * ((8.f / 3.f) * q - 3.f * q2 + 1.2f * q2 * q - (1.f / 6.f) * q2 * q2 -
                          1.f / (15.f * q2));
        pot = h1 * ((4.f / 3.f) * q2 - q2 * q + 0.3f * q2 * q2 - (1.f / 30.f) * q2 * q2 * q - 1.6f +
                    1.f / (15.f * q));
    } else {
        const float q2 = q * q;
        fr = (h1 * h1) * ((4.f / 3.f) * q - 1.2f * q2 * q + 0.5f * q2 * q2);
        pot = h1 * ((2.f / 3.f) * q2 - 0.3f * q2 * q2 + 0.1f * q2 * q2 * q - 1.4f);
    }
}

__device__ __forceinline__ float warp_reduce_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_reduce_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_reduce_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void kahan_add(float &s, float &c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// ---- the group walk ----------------------------------------------------------
constexpr int kWalkWarps = 4;    // warps per block
constexpr int kCellCap = 64;     // accepted nodes staged per warp before evaluation
constexpr int kLeafCap = 64;     // rejected leaves staged per warp before evaluation
constexpr int kStackInts = 8192; // per warp, in global memory (depth-first: <= depth x 256 in use)

__global__ void k_gather_key_order(int n, const uint32_t *__restrict__ order, const float4 *__restrict__ pos4,
                                   float4 *__restrict__ kp4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) kp4[i] = pos4[order[i]];
}

struct WalkArgs {
    const int32_t *T;
    const float4 *poles;
    const int2 *node_range;
    const float4 *kp4;        // positions and masses in key order
    const uint32_t *order;    // key order -> particle id
    int n, ngroups;
    float theta2;
    float4 *acc4;
    float *gnorm, *phi;
    int32_t *queues;
    uint32_t *counter;
    uint32_t *health;
    const uint8_t *active;  // individual timesteps: only active particles are walked for and written
};

// Acceleration (and potential) of the staged nodes at x, per unit G.
__device__ __forceinline__ void eval_cells(const float4 (*cell)[3], int ncell, float4 x, float &sx, float &sy, float &sz,
                                           float &sp) {
    for (int j = 0; j < ncell; ++j) {
        const float4 c0 = cell[j][0], c1 = cell[j][1], c2 = cell[j][2];
        // c0 = (com, M), c1 = (Qxx, Qxy, Qxz, Qyy), c2 = (Qyz, Qzz, -, -)
        const float Rx = x.x - c0.x, Ry = x.y - c0.y, Rz = x.z - c0.z;
        const float r2 = Rx * Rx + Ry * Ry + Rz * Rz;
        const float rinv = rsqrtf(r2);
        const float rinv2 = rinv * rinv;
        const float rinv3 = rinv * rinv2;
        const float rinv5 = rinv3 * rinv2;
        const float M = c0.w, Qxx = c1.x, Qxy = c1.y, Qxz = c1.z, Qyy = c1.w, Qyz = c2.x, Qzz = c2.y;
        const float QRx = Qxx * Rx + Qxy * Ry + Qxz * Rz;
        const float QRy = Qxy * Rx + Qyy * Ry + Qyz * Rz;
        const float QRz = Qxz * Rx + Qyz * Ry + Qzz * Rz;
        const float RQR = Rx * QRx + Ry * QRy + Rz * QRz;
        const float trQ = Qxx + Qyy + Qzz;
        const float q5 = RQR * rinv5;
        sp -= M * rinv + 0.5f * (3.f * q5 - trQ * rinv3);
        const float radial = -M * rinv3 - 7.5f * q5 * rinv2 + 1.5f * trQ * rinv5;
        const float t3 = 3.f * rinv5;
        sx += radial * Rx + t3 * QRx;
        sy += radial * Ry + t3 * QRy;
        sz += radial * Rz + t3 * QRz;
    }
}

// Softened pair sums of the staged particles at x, per unit G.
__device__ __forceinline__ void eval_parts(const float4 *part, int np, float4 x, float &sx, float &sy, float &sz,
                                           float &sp) {
    const float soft2x4 = 4.f * kGravSoft * kGravSoft;
    for (int j = 0; j < np; ++j) {
        const float4 q = part[j];
        const float rx = x.x - q.x, ry = x.y - q.y, rz = x.z - q.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        if (r2 >= soft2x4) {
            const float rinv = rsqrtf(r2);
            const float mr = q.w * rinv;
            const float s = -mr * rinv * rinv;
            sx += s * rx;
            sy += s * ry;
            sz += s * rz;
            sp -= mr;
        } else if (r2 > 0.f) {
            const float r = sqrtf(r2);
            float fr, pot;
            soft_pair(r, fr, pot);
            const float s = -q.w * fr / r;
            sx += s * rx;
            sy += s * ry;
            sz += s * rz;
            sp += q.w * pot;
        }
    }
}

template <bool ACC>
__global__ void __launch_bounds__(32 * kWalkWarps) k_walk(WalkArgs a) {
    __shared__ float4 s_cell[kWalkWarps][kCellCap][3];
    __shared__ int2 s_leaf[kWalkWarps][kLeafCap];
    __shared__ int s_loff[kWalkWarps][kLeafCap];
    __shared__ float4 s_part[kWalkWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned full = 0xffffffffu;
    const unsigned lt = (1u << lane) - 1u;
    int32_t *stk = a.queues + (size_t)(blockIdx.x * kWalkWarps + w) * kStackInts;
    const int32_t *T = a.T;
    const float soft2x4 = 4.f * kGravSoft * kGravSoft;
    while (true) {
        int g = 0;
        if (lane == 0) g = (int)atomicAdd(a.counter, 1u);
        g = __shfl_sync(full, g, 0);
        if (g >= a.ngroups) break;
        const int i = g * 32 + lane;
        const bool valid = i < a.n;
        // individual timesteps: only active particles get gravity, and a
        // group without one is skipped (the down-pass culling of README.md:64)
        const bool act = valid && (!a.active || a.active[a.order[i]]);
        if (!__any_sync(full, act)) continue;
        const float4 xi = a.kp4[valid ? i : g * 32];
        float ax = 0.f, ay = 0.f, az = 0.f, ph = 0.f, cax = 0.f, cay = 0.f, caz = 0.f, cph = 0.f;
        int ncell = 0, nleaf = 0;
        // the box the walk tests nodes against, and whether this lane's
        // particle belongs to the particles being walked for
        float bx0, by0, bz0, bx1, by1, bz1;
        bool mine = true;
        auto flush_cells = [&]() {
            __syncwarp();
            float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f;
            eval_cells(s_cell[w], ncell, xi, sx, sy, sz, sp);
            if (mine) {
                kahan_add(ax, cax, sx);
                kahan_add(ay, cay, sy);
                kahan_add(az, caz, sz);
                kahan_add(ph, cph, sp);
            }
            ncell = 0;
            __syncwarp();
        };
        auto flush_leaves = [&]() {
            __syncwarp();
            // number the staged leaves' particles consecutively
            const int c0 = (lane < nleaf) ? s_leaf[w][lane].y : 0;
            const int c1 = (lane + 32 < nleaf) ? s_leaf[w][lane + 32].y : 0;
            int inc0 = c0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(full, inc0, o);
                if (lane >= o) inc0 += y;
            }
            const int tot0 = __shfl_sync(full, inc0, 31);
            int inc1 = c1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(full, inc1, o);
                if (lane >= o) inc1 += y;
            }
            const int tot = tot0 + __shfl_sync(full, inc1, 31);
            if (lane < nleaf) s_loff[w][lane] = inc0 - c0;
            if (lane + 32 < nleaf) s_loff[w][lane + 32] = tot0 + inc1 - c1;
            __syncwarp();
            float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f;
            for (int j0 = 0; j0 < tot; j0 += 32) {
                const int j = j0 + lane;
                if (j < tot) {
                    int q = 0;  // the last leaf whose first particle number is <= j
#pragma unroll
                    for (int step = kLeafCap / 2; step > 0; step >>= 1)
                        if (q + step < nleaf && s_loff[w][q + step] <= j) q += step;
                    s_part[w][lane] = a.kp4[s_leaf[w][q].x + (j - s_loff[w][q])];
                }
                __syncwarp();
                eval_parts(s_part[w], min(32, tot - j0), xi, sx, sy, sz, sp);
                __syncwarp();
            }
            if (mine) {
                kahan_add(ax, cax, sx);
                kahan_add(ay, cay, sy);
                kahan_add(az, caz, sz);
                kahan_add(ph, cph, sp);
            }
            nleaf = 0;
        };
        auto walk = [&]() {
            // depth-first: each round pops up to 32 nodes off the top of the
            // stack and pushes the children of the rejected branches
            if (lane == 0) stk[0] = 0;  // the root
            __syncwarp();
            int size = 1;
            while (size > 0) {
                const int take = min(size, 32);
                size -= take;
                const bool v = lane < take;
                const int tp = v ? stk[size + lane] : 0;
                __syncwarp();
                const int dp = T[tp + 1];
                const int cnt = T[tp];
                const float4 *pr = a.poles + (size_t)dp * kPoleQ;
                const float4 c0 = pr[0];
                const float dx = fmaxf(fmaxf(bx0 - c0.x, c0.x - bx1), 0.f);
                const float dy = fmaxf(fmaxf(by0 - c0.y, c0.y - by1), 0.f);
                const float dz = fmaxf(fmaxf(bz0 - c0.z, c0.z - bz1), 0.f);
                const float d2 = dx * dx + dy * dy + dz * dz;
                bool acc = v && c0.w * c0.w < a.theta2 * d2 && d2 > soft2x4;
                const bool rleaf = v && !acc && cnt != 0;
                bool rbr = v && !acc && cnt == 0;
                int nch = 0;
                if (rbr)
                    for (int c = 0; c < 8; ++c) nch += (T[tp + 2 + c] != -1) ? 1 : 0;
                int inc = nch;
    #pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(full, inc, o);
                    if (lane >= o) inc += y;
                }
                const int tot = __shfl_sync(full, inc, 31);
                if (size + tot > kStackInts) {
                    // no room (deeper than the stack allows): the rejected branches
                    // are taken as accepted nodes, flagged in the health word
                    if (lane == 0) raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
                    acc = acc || rbr;
                    rbr = false;
                } else {
                    if (rbr) {
                        // reversed, so that the first child is popped first
                        int o = size + inc - 1;
                        for (int c = 0; c < 8; ++c) {
                            const int ch = T[tp + 2 + c];
                            if (ch != -1) stk[o--] = ch;
                        }
                    }
                    size += tot;
                }
                // accepted nodes: stage their records
                if (ncell + 32 > kCellCap) flush_cells();
                const unsigned ma = __ballot_sync(full, acc);
                if (acc) {
                    const int o = ncell + __popc(ma & lt);
                    const float4 p1 = pr[1], p2 = pr[2];
                    s_cell[w][o][0] = make_float4(c0.x, c0.y, c0.z, p1.x);
                    s_cell[w][o][1] = make_float4(p1.y, p1.z, p1.w, p2.x);
                    s_cell[w][o][2] = make_float4(p2.y, p2.z, 0.f, 0.f);
                }
                ncell += __popc(ma);
                // rejected leaves: stage their particle ranges
                if (nleaf + 32 > kLeafCap) flush_leaves();
                const unsigned ml = __ballot_sync(full, rleaf);
                if (rleaf) s_leaf[w][nleaf + __popc(ml & lt)] = a.node_range[dp];
                nleaf += __popc(ml);
                __syncwarp();
            }
            flush_cells();
            flush_leaves();
        };
        // A group that straddles a jump of the key order (two distant clusters
        // of particles) is cut there: consecutive particles farther apart
        // than 6x the group's typical step (the mean of the steps no longer
        // than twice the mean step) start a new segment, and every segment is
        // walked against its own box.  Almost every group is one segment.
        {
            const float4 xn = make_float4(__shfl_down_sync(full, xi.x, 1), __shfl_down_sync(full, xi.y, 1),
                                          __shfl_down_sync(full, xi.z, 1), 0.f);
            const bool has_next = lane < 31;
            const float ddx = xn.x - xi.x, ddy = xn.y - xi.y, ddz = xn.z - xi.z;
            const float step = has_next ? sqrtf(ddx * ddx + ddy * ddy + ddz * ddz) : 0.f;
            const float mean1 = warp_reduce_sum(step) * (1.f / 31.f);
            const bool small = has_next && step <= 2.f * mean1;
            const float n2 = warp_reduce_sum(small ? 1.f : 0.f);
            const float mean2 = warp_reduce_sum(small ? step : 0.f) / fmaxf(n2, 1.f);
            const bool cut = has_next && step > 6.f * mean2 && step > 0.f;
            // segment of this lane = number of cuts before it
            const unsigned cuts = __ballot_sync(full, cut);
            const int seg = __popc(cuts & lt);
            const int nseg = __popc(cuts) + 1;
            for (int q = 0; q < nseg; ++q) {
                mine = seg == q;
                const float big = 3.402823466e+38f;
                bx0 = warp_reduce_min(mine ? xi.x : big);
                by0 = warp_reduce_min(mine ? xi.y : big);
                bz0 = warp_reduce_min(mine ? xi.z : big);
                bx1 = warp_reduce_max(mine ? xi.x : -big);
                by1 = warp_reduce_max(mine ? xi.y : -big);
                bz1 = warp_reduce_max(mine ? xi.z : -big);
                walk();
            }
        }
        if (act) {
            const uint32_t id = a.order[i];
            if (ACC) {
                const float4 old = a.acc4[id];
                a.acc4[id] = make_float4(kG * ax, kG * ay, kG * az, old.w);
                a.gnorm[id] = sqrtf(ax * ax + ay * ay + az * az);
            }
            a.phi[id] = kG * ph;
        }
        __syncwarp();
    }
}
// FP64 direct sum over all particles at the given targets, with the exact
// softened kernel: out[4 t] = (ax, ay, az, phi) including G.  One block per
// target; positions are the float32 working positions promoted to double.
__global__ void __launch_bounds__(256) k_direct_f64(const float4 *__restrict__ pos4, int n,
                                                    const int32_t *__restrict__ targets, int nt,
                                                    double *__restrict__ out) {
    __shared__ double red[4][8];
    const int t = blockIdx.x;
    if (t >= nt) return;
    const int ip = targets[t];
    const float4 xi = pos4[ip];
    const double xx = xi.x, xy = xi.y, xz = xi.z;
    const double h = (double)kGravSoft, h1 = 1.0 / h;
    double ax = 0.0, ay = 0.0, az = 0.0, ph = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        if (j == ip) continue;
        const float4 xj = pos4[j];
        const double rx = xx - (double)xj.x, ry = xy - (double)xj.y, rz = xz - (double)xj.z;
        const double r2 = rx * rx + ry * ry + rz * rz;
        if (r2 == 0.0) continue;
        const double r = sqrt(r2);
        const double q = r * h1;
        double fr, pot;
        if (q >= 2.0) {
            fr = 1.0 / r2;
            pot = -1.0 / r;
        } else if (q > 1.0) {
            const double q2 = q * q;
            fr = h1 * h1 * ((8.0 / 3.0) * q - 3.0 * q2 + 1.2 * q2 * q - (1.0 / 6.0) * q2 * q2 - 1.0 / (15.0 * q2));
            pot = h1 * ((4.0 / 3.0) * q2 - q2 * q + 0.3 * q2 * q2 - (1.0 / 30.0) * q2 * q2 * q - 1.6 +
                        1.0 / (15.0 * q));
        } else {
            const double q2 = q * q;
            fr = h1 * h1 * ((4.0 / 3.0) * q - 1.2 * q2 * q + 0.5 * q2 * q2);
            pot = h1 * ((2.0 / 3.0) * q2 - 0.3 * q2 * q2 + 0.1 * q2 * q2 * q - 1.4);
        }
        const double m = (double)xj.w;
        const double s = -m * fr / r;
        ax += s * rx;
        ay += s * ry;
        az += s * rz;
        ph += m * pot;
    }
    double v[4] = {ax, ay, az, ph};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        out[4 * (size_t)t + threadIdx.x] = (double)kG * s;
    }
}

}  // namespace

static sph_status theta_pass(sph_ctx *ctx, float theta, bool acc, cudaStream_t st) {
    Tree &tr = ctx->tree;
    TreeBuild &tb = ctx->tb;
    if (!tr.valid || ctx->n <= 0) return SPH_OK;
    if (ctx->params.tree_source != SPH_TREE_GPU || !tb.order) {
        set_error("the theta gravity form walks the GPU-built tree (tree_source SPH_TREE_GPU)");
        return SPH_ERR_UNSUPPORTED;
    }
    const int n = ctx->n;
    const int L = tr.n_levels_host;
    ThetaUpArgs u;
    u.T = tr.tree;
    u.level_nodes = tr.level_nodes;
    u.level_count = tr.level_count;
    u.list_slot = tr.list_slot;
    u.parent_slot = tr.parent_slot;
    u.poles = tr.poles;
    u.pos4 = ctx->pos4;
    u.active = ctx->active;
    u.nat = ctx->nat;
    u.globals = ctx->globals;
    // activity follows the next active times only when the accelerations are
    // computed (the potential for the diagnostics covers every particle)
    u.individual = acc && ctx->form.timestep == SPH_TIMESTEP_INDIVIDUAL;
    for (int l = L - 1; l >= 0; --l) {
        int64_t bound = tr.level_count_host[l];
        int blocks = (int)((bound + 127) / 128);
        blocks = blocks < 1 ? 1 : (blocks > 148 * 32 ? 148 * 32 : blocks);
        k_up_theta<<<blocks, 128, 0, st>>>(u, l, tr.level_cap);
    }
    // resident warps of the walk, each with its two node queues
    static int max_blocks_per_sm = 0;
    if (max_blocks_per_sm == 0) {
        int b0 = 0, b1 = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_walk<true>, 32 * kWalkWarps, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_walk<false>, 32 * kWalkWarps, 0);
        max_blocks_per_sm = b0 < b1 ? b0 : b1;
        if (max_blocks_per_sm < 1) max_blocks_per_sm = 1;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const int ngroups = (n + 31) / 32;
    int blocks = sms * max_blocks_per_sm;
    if (blocks * kWalkWarps > ngroups) blocks = (ngroups + kWalkWarps - 1) / kWalkWarps;
    const int64_t qints = (int64_t)blocks * kWalkWarps * kStackInts;
    if (qints > tb.walk_queue_ints) {
        cudaFree(tb.walk_queues);
        tb.walk_queues = nullptr;
        tb.walk_queue_ints = 0;
        cudaError_t e = cudaMalloc(&tb.walk_queues, sizeof(int32_t) * qints);
        if (e != cudaSuccess) return cuda_status(e, "gravity (theta) walk queues");
        tb.walk_queue_ints = qints;
    }
    if (!tb.walk_counter) {
        cudaError_t e = cudaMalloc(&tb.walk_counter, sizeof(uint32_t));
        if (e != cudaSuccess) return cuda_status(e, "gravity (theta) walk counter");
    }
    float4 *kp4 = ctx->sp4;  // free until the density pass gathers its own records
    k_gather_key_order<<<(n + 255) / 256, 256, 0, st>>>(n, tb.order, ctx->pos4, kp4);
    cudaMemsetAsync(tb.walk_counter, 0, sizeof(uint32_t), st);
    WalkArgs w;
    w.T = tr.tree;
    w.poles = tr.poles;
    w.node_range = tr.node_range;
    w.kp4 = kp4;
    w.order = tb.order;
    w.n = n;
    w.ngroups = ngroups;
    w.theta2 = theta * theta;
    w.acc4 = ctx->acc4;
    w.gnorm = ctx->gnorm;
    w.phi = ctx->phi;
    w.queues = tb.walk_queues;
    w.counter = tb.walk_counter;
    w.health = ctx->health;
    w.active = u.individual ? ctx->active : nullptr;
    if (acc)
        k_walk<true><<<blocks, 32 * kWalkWarps, 0, st>>>(w);
    else
        k_walk<false><<<blocks, 32 * kWalkWarps, 0, st>>>(w);
    return cuda_status(cudaGetLastError(), "gravity (theta)");
}

sph_status launch_gravity_theta(sph_ctx *ctx, cudaStream_t st) { return theta_pass(ctx, ctx->form.theta, true, st); }

sph_status launch_potential_theta(sph_ctx *ctx, float theta, cudaStream_t st) {
    return theta_pass(ctx, theta, false, st);
}

sph_status launch_direct_f64(sph_ctx *ctx, const int32_t *d_targets, int nt, double *d_out, cudaStream_t st) {
    if (nt <= 0) return SPH_OK;
    k_direct_f64<<<nt, 256, 0, st>>>(ctx->pos4, ctx->n, d_targets, nt, d_out);
    return cuda_status(cudaGetLastError(), "direct f64");
}

}  // namespace sph

// sph_gravity_theta.cu -- the opening-angle gravity form and the FP64 direct
// sum it is measured against.  Neither has a counterpart in the reference,
// whose gravity (Compute.cpp:328-377, sph_gravity.cu here) uses an adaptive
// acceptance test without an opening angle, force-accepts failing leaves and
// keeps integer-truncated softening coefficients (kernels.h:93,97).
//
// Tree and passes keep the reference's structure (flattened int tree, one
// launch per level, lists inherited from the parent), with these changes:
//   * multipoles: mass, centre of mass, the full second moments
//     Q_jk = sum m r_j r_k about the centre of mass, and the radius of the
//     smallest sphere about the centre of mass that holds the node's box;
//   * acceptance: (r_A + r_B) < theta * |com_A - com_B|, and never closer than
//     the softening support 2 eps (so every softened pair is summed exactly);
//   * branch targets: accepted nodes go through M2L into a local expansion of
//     the potential, the acceleration (monopole + quadrupole) and its gradient
//     (monopole); a rejected node is passed to the target's list, or opened
//     one level first when it is larger than the target;
//   * leaf targets resolve their list completely: accepted nodes are
//     evaluated at each particle (M2P, monopole + quadrupole), rejected
//     leaves are summed particle by particle (P2P, the cubic-spline softened
//     kernel with its exact coefficients), rejected branches are opened
//     through a small per-warp stack.  Per-particle sums are Kahan-compensated.
// Locals hold no factor G, like the reference's; the leaf writes
// acc = G a, |a| (the reference's gravNorm) and the potential G phi.
#include <cuda_runtime.h>

#include "sph_internal.h"

namespace sph {

namespace {

// Layout of a theta-form node record (kPoleQ float4 per node):
//   q0 (com.xyz, radius)  q1 (M, Qxx, Qxy, Qxz)  q2 (Qyy, Qyz, Qzz, 0)
//   q3 (bbox min, 0)      q4 (bbox max, 1)
// and of a local (kLocalQ float4): l0 (centre.xyz, phi0)  l1 (ax, ay, az, Txx)
//   l2 (Txy, Txz, Tyy, Tyz)  l3 (Tzz, 0, 0, 0)   with T_ij = d a_i / d x_j.

constexpr int kStack = 128;  // per-warp stack of opened branches at a leaf

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
};

__device__ void p2m_theta(const ThetaUpArgs &a, int tp, int dp) {
    const int32_t *T = a.T;
    const int np = T[tp];
    const int s = tp + 2;
    // sums relative to the first particle: no cancellation at large |x|
    const float4 x0 = a.pos4[T[s]];
    float m = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
    float mnx = x0.x, mny = x0.y, mnz = x0.z, mxx = x0.x, mxy = x0.y, mxz = x0.z;
    for (int i = 0; i < np; ++i) {
        const int p = T[s + i];
        const float4 q = a.pos4[p];
        a.active[p] = 1;
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
    pr[4] = make_float4(mxx, mxy, mxz, 1.f);
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
    const float cx = c0f.x + ox, cy = c0f.y + oy, cz = c0f.z + oz;
    float4 *pr = a.poles + (size_t)dp * kPoleQ;
    pr[0] = make_float4(cx, cy, cz, corner_radius(cx, cy, cz, mnx, mny, mnz, mxx, mxy, mxz));
    pr[1] = make_float4(m, qxx, qxy, qxz);
    pr[2] = make_float4(qyy, qyz, qzz, 0.f);
    pr[3] = make_float4(mnx, mny, mnz, 0.f);
    pr[4] = make_float4(mxx, mxy, mxz, 1.f);
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

// Field of a node (mass M, second moments Q about its centre of mass) at
// R = x - com: potential (without the factor -G... see below), acceleration
// and, for M2L, the monopole gradient.  With D = 1/|R|:
//   phi  = -(M D + 1/2 Q_jk d_j d_k D)
//   a_i  =   M d_i D + 1/2 Q_jk d_i d_j d_k D
//   T_ij =   M d_i d_j D
struct Field {
    float phi, ax, ay, az;
};

__device__ __forceinline__ Field node_field(float Rx, float Ry, float Rz, const float4 &q1, const float4 &q2) {
    const float r2 = Rx * Rx + Ry * Ry + Rz * Rz;
    const float rinv = 1.f / sqrtf(r2);
    const float rinv2 = rinv * rinv;
    const float rinv3 = rinv * rinv2;
    const float rinv5 = rinv3 * rinv2;
    const float rinv7 = rinv5 * rinv2;
    const float M = q1.x, Qxx = q1.y, Qxy = q1.z, Qxz = q1.w, Qyy = q2.x, Qyz = q2.y, Qzz = q2.z;
    const float QRx = Qxx * Rx + Qxy * Ry + Qxz * Rz;
    const float QRy = Qxy * Rx + Qyy * Ry + Qyz * Rz;
    const float QRz = Qxz * Rx + Qyz * Ry + Qzz * Rz;
    const float RQR = Rx * QRx + Ry * QRy + Rz * QRz;
    const float trQ = Qxx + Qyy + Qzz;
    Field f;
    f.phi = -(M * rinv + 0.5f * (3.f * RQR * rinv5 - trQ * rinv3));
    const float radial = -M * rinv3 - 7.5f * RQR * rinv7 + 1.5f * trQ * rinv5;
    f.ax = radial * Rx + 3.f * QRx * rinv5;
    f.ay = radial * Ry + 3.f * QRy * rinv5;
    f.az = radial * Rz + 3.f * QRz * rinv5;
    return f;
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

__device__ __forceinline__ void kahan_add(float &s, float &c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

struct ThetaDownArgs {
    const int32_t *T;
    const int32_t *level_nodes;
    const int32_t *level_count;
    const int32_t *list_slot;
    const int32_t *parent_slot;
    const float4 *poles;
    float4 *locals;
    const int32_t *list_in;
    int32_t *list_out;
    int list_cap;
    int64_t branch_cap;
    int64_t tree_cap;
    float theta;
    const float4 *pos4;
    float4 *acc4;
    float *gnorm;
    float *phi;
    uint32_t *health;
};

__device__ __forceinline__ bool accept_theta(float ax, float ay, float az, float ra, const float4 &b0, float theta) {
    const float dx = ax - b0.x, dy = ay - b0.y, dz = az - b0.z;
    const float d2 = dx * dx + dy * dy + dz * dz;
    const float rs = ra + b0.w;
    const float dmin = 2.f * kGravSoft;
    return rs * rs < theta * theta * d2 && d2 > dmin * dmin;
}

// M2L of node b into the local accumulators at centre (lx, ly, lz).
__device__ __forceinline__ void m2l_theta(float lx, float ly, float lz, const float4 *bp, float *acc) {
    const float4 b0 = bp[0], b1 = bp[1], b2 = bp[2];
    const float Rx = lx - b0.x, Ry = ly - b0.y, Rz = lz - b0.z;
    const Field f = node_field(Rx, Ry, Rz, b1, b2);
    const float r2 = Rx * Rx + Ry * Ry + Rz * Rz;
    const float rinv = 1.f / sqrtf(r2);
    const float rinv3 = rinv * rinv * rinv;
    const float m3 = 3.f * b1.x * rinv3 * rinv * rinv;
    const float m1 = b1.x * rinv3;
    acc[0] += f.phi;
    acc[1] += f.ax;
    acc[2] += f.ay;
    acc[3] += f.az;
    acc[4] += m3 * Rx * Rx - m1;
    acc[5] += m3 * Rx * Ry;
    acc[6] += m3 * Rx * Rz;
    acc[7] += m3 * Ry * Ry - m1;
    acc[8] += m3 * Ry * Rz;
    acc[9] += m3 * Rz * Rz - m1;
}

__device__ void branch_target(const ThetaDownArgs &a, int tp, int dp, int lane) {
    const int32_t *T = a.T;
    const int cap = a.list_cap;
    const float4 *sp = a.poles + (size_t)dp * kPoleQ;
    const float4 s0 = sp[0];
    const int slot = a.list_slot[dp];
    const int pslot = a.parent_slot[dp];
    if (slot < 0 || slot >= a.branch_cap || pslot < 0 || pslot >= a.branch_cap) {
        if (lane == 0) raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
        return;
    }
    int32_t *out = a.list_out + (size_t)slot * cap;
    const int32_t *in = a.list_in + (size_t)pslot * cap;
    const float4 *lp = a.locals + (size_t)dp * kLocalQ;
    const float4 L0 = lp[0];
    const float lx = L0.x, ly = L0.y, lz = L0.z;
    float acc[10];
#pragma unroll
    for (int j = 0; j < 10; ++j) acc[j] = 0.f;
    int op = 0;
    for (int c0 = 0; c0 < cap; c0 += 32) {
        const int i = c0 + lane;
        int e = (i < cap) ? in[i] : -1;
        if (e < -1 || e > a.tree_cap - 10) {
            raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
            e = -1;
        }
        const uint32_t stop = __ballot_sync(0xffffffffu, e == -1);
        const int nvalid = stop ? (__ffs(stop) - 1) : 32;
        // bit 8: pass e itself; bits 0..7: pass child k of e
        uint32_t pass = 0u;
        if (lane < nvalid) {
            const float4 *bp = a.poles + (size_t)T[e + 1] * kPoleQ;
            const float4 b0 = bp[0];
            if (accept_theta(lx, ly, lz, s0.w, b0, a.theta)) {
                m2l_theta(lx, ly, lz, bp, acc);
            } else if (T[e] != 0 || b0.w <= s0.w) {
                pass = 1u << 8;
            } else {
                for (int k = 0; k < 8; ++k) {
                    const int c = T[e + 2 + k];
                    if (c == -1) continue;
                    const float4 *cp = a.poles + (size_t)T[c + 1] * kPoleQ;
                    if (accept_theta(lx, ly, lz, s0.w, cp[0], a.theta))
                        m2l_theta(lx, ly, lz, cp, acc);
                    else
                        pass |= 1u << k;
                }
            }
        }
        const int mine = __popc(pass);
        int incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        int pos = op + incl - mine;
        while (pass) {
            const int k = __ffs(pass) - 1;
            pass &= pass - 1u;
            const int c = (k == 8) ? e : T[e + 2 + k];
            if (pos < cap - 1) {
                out[pos] = c;
            } else {
                // list full: the node is accepted although the opening test
                // failed; the health bit tells the caller the result is degraded
                raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
                m2l_theta(lx, ly, lz, a.poles + (size_t)T[c + 1] * kPoleQ, acc);
            }
            ++pos;
        }
        op = min(op + total, cap - 1);
        if (stop) break;
    }
    if (lane == 0) out[op] = -1;
#pragma unroll
    for (int j = 0; j < 10; ++j) {
        float v = acc[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        acc[j] = v;
    }
    const float4 L1 = lp[1], L2 = lp[2], L3 = lp[3];
    const float phi0 = L0.w + acc[0];
    const float ax = L1.x + acc[1], ay = L1.y + acc[2], az = L1.z + acc[3];
    const float txx = L1.w + acc[4], txy = L2.x + acc[5], txz = L2.y + acc[6];
    const float tyy = L2.z + acc[7], tyz = L2.w + acc[8], tzz = L3.x + acc[9];
    // L2L to every child, expanded about the child's centre of mass
    if (lane < 8) {
        const int c = T[tp + 2 + lane];
        if (c != -1) {
            const int cdp = T[c + 1];
            const float4 cpos = a.poles[(size_t)cdp * kPoleQ];
            const float sx = cpos.x - lx, sy = cpos.y - ly, sz = cpos.z - lz;
            const float tsx = txx * sx + txy * sy + txz * sz;
            const float tsy = txy * sx + tyy * sy + tyz * sz;
            const float tsz = txz * sx + tyz * sy + tzz * sz;
            const float cphi = phi0 - (ax * sx + ay * sy + az * sz) - 0.5f * (sx * tsx + sy * tsy + sz * tsz);
            float4 *clp = a.locals + (size_t)cdp * kLocalQ;
            clp[0] = make_float4(cpos.x, cpos.y, cpos.z, cphi);
            clp[1] = make_float4(ax + tsx, ay + tsy, az + tsz, txx);
            clp[2] = make_float4(txy, txz, tyy, tyz);
            clp[3] = make_float4(tzz, 0.f, 0.f, 0.f);
        }
    }
}

__device__ void leaf_target(const ThetaDownArgs &a, int tp, int dp, int lane, int32_t *stk) {
    const int32_t *T = a.T;
    const int cap = a.list_cap;
    const int np = T[tp];
    const float4 s0 = a.poles[(size_t)dp * kPoleQ];
    const int pslot = a.parent_slot[dp];
    if (pslot < 0 || pslot >= a.branch_cap) {
        if (lane == 0) raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
        return;
    }
    const int32_t *in = a.list_in + (size_t)pslot * cap;
    const float4 *lp = a.locals + (size_t)dp * kLocalQ;
    const float4 L0 = lp[0], L1 = lp[1], L2 = lp[2], L3 = lp[3];
    for (int i0 = 0; i0 < np; i0 += 32) {
        const bool mine = i0 + lane < np;
        const int p = mine ? T[tp + 2 + i0 + lane] : -1;
        const float4 xi = mine ? a.pos4[p] : s0;
        // L2P
        const float dx = xi.x - L0.x, dy = xi.y - L0.y, dz = xi.z - L0.z;
        const float tdx = L1.w * dx + L2.x * dy + L2.y * dz;
        const float tdy = L2.x * dx + L2.z * dy + L2.w * dz;
        const float tdz = L2.y * dx + L2.w * dy + L3.x * dz;
        float ax = L1.x + tdx, ay = L1.y + tdy, az = L1.z + tdz;
        float ph = L0.w - (L1.x * dx + L1.y * dy + L1.z * dz) - 0.5f * (dx * tdx + dy * tdy + dz * tdz);
        float cax = 0.f, cay = 0.f, caz = 0.f, cph = 0.f;
        int sp = 0;
        int li = 0;
        while (true) {
            int e;
            if (sp > 0) {
                e = stk[--sp];
            } else {
                if (li >= cap) break;
                e = in[li++];
                if (e == -1) break;
                if (e < -1 || e > a.tree_cap - 10) {
                    if (lane == 0) raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
                    break;
                }
            }
            const float4 *bp = a.poles + (size_t)T[e + 1] * kPoleQ;
            const float4 b0 = bp[0];
            const int ne = T[e];
            if (accept_theta(s0.x, s0.y, s0.z, s0.w, b0, a.theta)) {
                const Field f = node_field(xi.x - b0.x, xi.y - b0.y, xi.z - b0.z, bp[1], bp[2]);
                kahan_add(ax, cax, f.ax);
                kahan_add(ay, cay, f.ay);
                kahan_add(az, caz, f.az);
                kahan_add(ph, cph, f.phi);
            } else if (ne != 0) {
                for (int j = 0; j < ne; ++j) {
                    const int pj = T[e + 2 + j];
                    const float4 xj = a.pos4[pj];
                    const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                    const float r = sqrtf(rx * rx + ry * ry + rz * rz);
                    if (pj == p || r == 0.f) continue;
                    float fr, pot;
                    soft_pair(r, fr, pot);
                    const float s = -xj.w * fr / r;
                    kahan_add(ax, cax, s * rx);
                    kahan_add(ay, cay, s * ry);
                    kahan_add(az, caz, s * rz);
                    kahan_add(ph, cph, xj.w * pot);
                }
            } else {
                // open the branch: children pushed in reverse, popped in order
                for (int k = 7; k >= 0; --k) {
                    const int c = T[e + 2 + k];
                    if (c == -1) continue;
                    if (sp < kStack) {
                        if (lane == 0) stk[sp] = c;
                        ++sp;
                    } else {
                        if (lane == 0) raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
                        const float4 *cp = a.poles + (size_t)T[c + 1] * kPoleQ;
                        const float4 c0 = cp[0];
                        const Field f = node_field(xi.x - c0.x, xi.y - c0.y, xi.z - c0.z, cp[1], cp[2]);
                        kahan_add(ax, cax, f.ax);
                        kahan_add(ay, cay, f.ay);
                        kahan_add(az, caz, f.az);
                        kahan_add(ph, cph, f.phi);
                    }
                }
                __syncwarp();
            }
        }
        __syncwarp();
        if (mine) {
            const float4 old = a.acc4[p];
            a.acc4[p] = make_float4(kG * ax, kG * ay, kG * az, old.w);
            a.gnorm[p] = sqrtf(ax * ax + ay * ay + az * az);
            a.phi[p] = kG * ph;
        }
    }
}

constexpr int kDownWarps = 4;

__global__ void __launch_bounds__(32 * kDownWarps) k_down_theta(ThetaDownArgs a, int level, int64_t level_cap) {
    __shared__ int32_t stacks[kDownWarps][kStack];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int cnt = a.level_count[level];
    const int32_t *nodes = a.level_nodes + (size_t)level * level_cap;
    const int32_t *T = a.T;
    for (int t = warp0; t < cnt; t += nwarps) {
        const int tp = nodes[t];
        if (tp == 0) {
            if (T[0] != 0) {
                if (lane == 0) raise_health(a.health, SPH_HEALTH_ROOT_LEAF);
                continue;
            }
            // the root: zero locals at its children's centres, list = [root]
            if (lane < 8) {
                const int c = T[2 + lane];
                if (c != -1) {
                    const int cdp = T[c + 1];
                    const float4 cp = a.poles[(size_t)cdp * kPoleQ];
                    float4 *lp = a.locals + (size_t)cdp * kLocalQ;
                    lp[0] = make_float4(cp.x, cp.y, cp.z, 0.f);
                    lp[1] = make_float4(0.f, 0.f, 0.f, 0.f);
                    lp[2] = make_float4(0.f, 0.f, 0.f, 0.f);
                    lp[3] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
            if (lane == 0) {
                a.list_out[0] = 0;
                a.list_out[1] = -1;
            }
            continue;
        }
        const int dp = T[tp + 1];
        if (T[tp] == 0)
            branch_target(a, tp, dp, lane);
        else
            leaf_target(a, tp, dp, lane, stacks[wib]);
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

sph_status launch_gravity_theta(sph_ctx *ctx, cudaStream_t st) {
    Tree &tr = ctx->tree;
    if (!tr.valid || ctx->n <= 0) return SPH_OK;
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
    for (int l = L - 1; l >= 0; --l) {
        int64_t bound = tr.level_count_host[l];
        int blocks = (int)((bound + 127) / 128);
        blocks = blocks < 1 ? 1 : (blocks > 148 * 32 ? 148 * 32 : blocks);
        k_up_theta<<<blocks, 128, 0, st>>>(u, l, tr.level_cap);
    }
    ThetaDownArgs d;
    d.T = tr.tree;
    d.level_nodes = tr.level_nodes;
    d.level_count = tr.level_count;
    d.list_slot = tr.list_slot;
    d.parent_slot = tr.parent_slot;
    d.poles = tr.poles;
    d.locals = tr.locals;
    d.list_cap = tr.list_cap;
    d.branch_cap = tr.branch_cap;
    d.tree_cap = tr.tree_cap;
    d.theta = ctx->form.theta;
    d.pos4 = ctx->pos4;
    d.acc4 = ctx->acc4;
    d.gnorm = ctx->gnorm;
    d.phi = ctx->phi;
    d.health = ctx->health;
    for (int l = 0; l < L; ++l) {
        d.list_in = (l % 2 == 0) ? tr.lists[0] : tr.lists[1];
        d.list_out = (l % 2 == 0) ? tr.lists[1] : tr.lists[0];
        int64_t bound = tr.level_count_host[l];
        int blocks = (int)((bound * 32 + 32 * kDownWarps - 1) / (32 * kDownWarps));
        blocks = blocks < 1 ? 1 : (blocks > 148 * 32 ? 148 * 32 : blocks);
        k_down_theta<<<blocks, 32 * kDownWarps, 0, st>>>(d, l, tr.level_cap);
    }
    return cuda_status(cudaGetLastError(), "gravity (theta)");
}

sph_status launch_direct_f64(sph_ctx *ctx, const int32_t *d_targets, int nt, double *d_out, cudaStream_t st) {
    if (nt <= 0) return SPH_OK;
    k_direct_f64<<<nt, 256, 0, st>>>(ctx->pos4, ctx->n, d_targets, nt, d_out);
    return cuda_status(cudaGetLastError(), "direct f64");
}

}  // namespace sph

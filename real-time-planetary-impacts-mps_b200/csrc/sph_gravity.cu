// sph_gravity.cu -- Compute::gravitationalPass (SPH/Compute/Compute.cpp:328-377).
//
// up pass   gravity.metal:36-62 -> P2M.metal:12-107, M2M.metal:12-160 (p = 2)
// down pass gravity.metal:64-143 -> helpers.h:15-147, accept.metal:14-55,
//           M2L.metal:12-108, derivatives.metal:12-156, L2L.metal:12-104,
//           L2P.metal:12-32, helpers.h:47-81 (leaf P2P)
//
// The tree is the reference's flattened int format.  Levels run in order
// (deepest first up, root first down) as one launch each.  The up pass is one
// thread per node.  The down pass gives each node a warp: the 32 lanes take
// consecutive entries of the parent's unchecked list, evaluate the acceptance
// test and the M2L kernels in parallel, and append rejected branch children
// to the node's own list with a warp prefix sum, so the list keeps the
// reference's order (entry-major, child-slot-minor) and the reference's
// overflow rule (a child that finds the list full is force-accepted).  The
// per-lane partial local expansions are summed across the warp at the end.
// Leaves hand one particle to each lane for L2P plus the intra-leaf P2P sum,
// which runs over the leaf's particles in the reference's order.
//
// Lists are addressed by each branch's rank among the branches of its level
// (the reference uses the node's index in its level list); only branches
// write lists, so storage is bounded by the branch count.
#include <cuda_runtime.h>

#include "sph_internal.h"

namespace sph {

namespace {

struct Pole {
    float4 q0, q1, q2, q3, q4, q5;
};

__device__ __forceinline__ void store_pole(float4 *poles, int dp, const Pole &r) {
    float4 *p = poles + (size_t)dp * kPoleQ;
    p[0] = r.q0;
    p[1] = r.q1;
    p[2] = r.q2;
    p[3] = r.q3;
    p[4] = r.q4;
    p[5] = r.q5;
}

// helpers.metal:63-89 (p = 2); e = {M, X, Y, Z, XX, XY, XZ, YY, YZ, ZZ}
__device__ __forceinline__ float power2(const float *e) {
    float s = e[ZZ] * e[ZZ];
    s += 0.5f * e[YZ] * e[YZ];
    s += e[YY] * e[YY];
    s += 0.5f * e[XZ] * e[XZ];
    s += 0.5f * e[XY] * e[XY];
    s += 0.5f * e[XX] * e[XX];
    return sqrtf(s);
}

__device__ __forceinline__ Pole pack_pole(float cx, float cy, float cz, float size, const float *e, float mnx, float mny,
                                          float mnz, float min_grav, float mxx, float mxy, float mxz, bool active) {
    Pole r;
    r.q0 = make_float4(cx, cy, cz, size);
    r.q1 = make_float4(e[M], e[XX], e[XY], e[XZ]);
    r.q2 = make_float4(e[YY], e[YZ], e[ZZ], power2(e));
    r.q3 = make_float4(mnx, mny, mnz, min_grav);
    r.q4 = make_float4(mxx, mxy, mxz, active ? 1.f : 0.f);
    r.q5 = make_float4(e[X], e[Y], e[Z], 0.f);
    return r;
}

struct UpArgs {
    const int32_t *T;
    const int32_t *level_nodes;
    const int32_t *level_count;
    const int32_t *list_slot;
    int32_t *parent_slot;
    float4 *poles;
    const float4 *pos4;
    const float *gnorm;
    uint8_t *active;
    const int32_t *nat;
    const int32_t *globals;
    int individual;  // SPH_TIMESTEP_INDIVIDUAL: active once the time reaches nextActiveTime
};

// P2M.metal:12-107
__device__ void p2m(const UpArgs &a, int tp, int dp) {
    const int32_t *T = a.T;
    const int np = T[tp];
    const int s = tp + 2, e = s + np;
    float px = 0.f, py = 0.f, pz = 0.f, m0 = 0.f;
    float mg = 3.402823466e+38f;
    bool act = false;
    float mxx = -3.402823466e+38f, mxy = mxx, mxz = mxx, mnx = 3.402823466e+38f, mny = mnx, mnz = mnx;
    const int gt = a.globals[0];
    for (int i = s; i < e; ++i) {
        const int p = T[i];
        const float4 q = a.pos4[p];
        // the reference's test as shipped is time <= next (every particle
        // active every step); the individual form uses README.md:62's
        const bool ia = a.individual ? gt >= a.nat[p] : gt <= a.nat[p];
        if (!act && ia) act = true;
        mxx = fmax_ref(mxx, q.x);
        mxy = fmax_ref(mxy, q.y);
        mxz = fmax_ref(mxz, q.z);
        mnx = fmin_ref(mnx, q.x);
        mny = fmin_ref(mny, q.y);
        mnz = fmin_ref(mnz, q.z);
        m0 += q.w;
        px += q.x * q.w;
        py += q.y * q.w;
        pz += q.z * q.w;
        if (ia) mg = fmin_ref(mg, a.gnorm[p]);
    }
    for (int i = s; i < e; ++i) a.active[T[i]] = act ? 1 : 0;
    px = px / m0;
    py = py / m0;
    pz = pz / m0;
    float ex[10] = {m0, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int i = s; i < e; ++i) {
        const float4 q = a.pos4[T[i]];
        const float m = q.w;
        const float rx = q.x - px, ry = q.y - py, rz = q.z - pz;
        ex[X] -= rx * m;
        ex[Y] -= ry * m;
        ex[Z] -= rz * m;
        ex[XX] += m * rx * rx;
        ex[XY] += m * rx * ry;
        ex[XZ] += m * rx * rz;
        ex[YY] += m * ry * ry;
        ex[YZ] += m * ry * rz;
        ex[ZZ] += m * rz * rz;
    }
    ex[XX] *= 0.5f;
    ex[YY] *= 0.5f;
    ex[ZZ] *= 0.5f;
    const float dx = mxx - mnx, dy = mxy - mny, dz = mxz - mnz;
    const float size = fmax_ref(dx, fmax_ref(dy, dz));
    store_pole(a.poles, dp, pack_pole(px, py, pz, size, ex, mnx, mny, mnz, mg, mxx, mxy, mxz, act));
}

// M2M.metal:75-160 (Q5: the ZZ shift multiplies the child's Z term; Q6: the
// leaf-sync loop bound uses the parent's start).
__device__ void m2m(const UpArgs &a, int tp, int dp) {
    const int32_t *T = a.T;
    float mg = 3.402823466e+38f, px = 0.f, py = 0.f, pz = 0.f, mass = 0.f;
    bool act = false, all_leaves = true;
    float mxx = -3.402823466e+38f, mxy = mxx, mxz = mxx, mnx = 3.402823466e+38f, mny = mnx, mnz = mnx;
    const int s = tp + 2, e = s + 8;
    const int my_slot = a.list_slot[dp];
    for (int i = s; i < e; ++i) {
        const int c = T[i];
        if (c == -1) continue;
        const int cdp = T[c + 1];
        a.parent_slot[cdp] = my_slot;
        const float4 *cp = a.poles + (size_t)cdp * kPoleQ;
        const float4 c0 = cp[0], c1 = cp[1], c3 = cp[3], c4 = cp[4];
        mg = fmin_ref(c3.w, mg);
        mass += c1.x;
        px += c0.x * c1.x;
        py += c0.y * c1.x;
        pz += c0.z * c1.x;
        if (!act && c4.w != 0.f) act = true;
        if (all_leaves && T[c] == 0) all_leaves = false;
        mxx = fmax_ref(mxx, c4.x);
        mxy = fmax_ref(mxy, c4.y);
        mxz = fmax_ref(mxz, c4.z);
        mnx = fmin_ref(mnx, c3.x);
        mny = fmin_ref(mny, c3.y);
        mnz = fmin_ref(mnz, c3.z);
    }
    const float dx = mxx - mnx, dy = mxy - mny, dz = mxz - mnz;
    const float size = fmax_ref(dx, fmax_ref(dy, dz));
    px = px / mass;
    py = py / mass;
    pz = pz / mass;
    float ex[10] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int i = s; i < e; ++i) {
        const int c = T[i];
        if (c == -1) continue;
        const int cdp = T[c + 1];
        float4 *cp = a.poles + (size_t)cdp * kPoleQ;
        const float4 c0 = cp[0], c1 = cp[1], c2 = cp[2], c4 = cp[4], c5 = cp[5];
        const float rx = px - c0.x, ry = py - c0.y, rz = pz - c0.z;
        const float cm = c1.x;
        ex[M] += cm;
        // transformed X, Y, Z are zero (M2M.metal:17-19)
        ex[X] += 0.f;
        ex[Y] += 0.f;
        ex[Z] += 0.f;
        ex[XX] += c1.y + 0.5f * rx * rx * cm;
        ex[XY] += c1.z + rx * ry * cm;
        ex[XZ] += c1.w + rx * rz * cm;
        ex[YY] += c2.x + 0.5f * ry * ry * cm;
        ex[YZ] += c2.y + ry * rz * cm;
        ex[ZZ] += c2.z + 0.5f * rz * rz * c5.z;
        if (all_leaves && act && c4.w == 0.f) {
            cp[4].w = 1.f;
            const int cnp = T[c];
            const int cs = c + 2, ce = s + cnp;
            for (int j = cs; j < ce; ++j) a.active[T[j]] = 1;
        }
    }
    store_pole(a.poles, dp, pack_pole(px, py, pz, size, ex, mnx, mny, mnz, mg, mxx, mxy, mxz, act));
}

__global__ void k_up(UpArgs a, int level, int64_t level_cap) {
    const int cnt = a.level_count[level];
    const int32_t *nodes = a.level_nodes + (size_t)level * level_cap;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int tp = nodes[t];
        const int dp = a.T[tp + 1];
        if (a.T[tp] == 0)
            m2m(a, tp, dp);
        else
            p2m(a, tp, dp);
    }
}

// accept.metal:14-55.  A = (size, pos, minGrav) of the target; B = candidate.
__device__ __forceinline__ bool mac_accept(float ra, float ax, float ay, float az, float a_min_grav, const float4 &b0,
                                           const float4 &b1, const float4 &b2) {
    const float rb = b0.w;
    const float dx = ax - b0.x, dy = ay - b0.y, dz = az - b0.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float rs = ra + rb;
    if (rs * rs > r2) return false;
    const float rmax = fmax_ref(ra, rb);
    float e = 0.f;
    e += 1.f * b1.x * (ra * ra);
    e += 2.f * 0.f * ra;
    e += 1.f * b2.w * 1.f;
    e *= 8.f;
    if (ra + rb > 0.f) {
        e *= rmax;
        e /= (ra + rb);
    }
    return e < kGravityEta * a_min_grav * r2 * r2;
}

// derivatives.metal + M2L.metal (p = 2), added into acc[10].
__device__ __forceinline__ void m2l_add(float lx, float ly, float lz, const float4 &b0, const float4 &b1,
                                        const float4 &b2, float *acc) {
    const float vx = lx - b0.x, vy = ly - b0.y, vz = lz - b0.z;
    const float r2 = vx * vx + vy * vy + vz * vz;
    const float r = sqrtf(r2);
    const float rinv = r > 1e-6f ? 1.f / r : 0.f;
    const float eps = kGravSoft;
    const float eps2 = eps * eps;
    float d1, d2, d3;
    if (r2 < eps2) {
        const float ei = 1.f / eps;
        const float u = r * ei;
        float s1 = -3.f * u + 15.f;
        s1 = s1 * u - 28.f;
        s1 = s1 * u + 21.f;
        s1 = s1 * u;
        s1 = s1 * u - 7.f;
        s1 = s1 * u;
        s1 = s1 * u + 3.f;
        float s2 = -21.f * u + 90.f;
        s2 = s2 * u - 140.f;
        s2 = s2 * u + 84.f;
        s2 = s2 * u;
        s2 = s2 * u - 14.f;
        s2 = s2 * u;
        float s3 = -105.f * u + 360.f;
        s3 = s3 * u - 420.f;
        s3 = s3 * u + 168.f;
        s3 = s3 * u;
        s3 = s3 * u;
        d1 = ei * s1;
        const float ei2 = ei * ei;
        d2 = ei2 * s2;
        d3 = (ei2 * ei) * s3;
    } else {
        d1 = rinv;
        d2 = -1.f * d1 * rinv;
        d3 = -3.f * d2 * rinv;
    }
    const float rx = vx * rinv, ry = vy * rinv, rz = vz * rinv;
    float D[10];
    D[M] = d1;
    D[X] = rx * d2;
    D[Y] = ry * d2;
    D[Z] = rz * d2;
    d2 *= rinv;
    D[XX] = rx * rx * d3 + d2;
    D[XY] = rx * ry * d3;
    D[XZ] = rx * rz * d3;
    D[YY] = ry * ry * d3 + d2;
    D[YZ] = ry * rz * d3;
    D[ZZ] = rz * rz * d3 + d2;
    const float m0 = b1.x;
    float L0 = m0 * D[M];
    L0 += b1.y * D[XX] + b2.x * D[YY] + b2.z * D[ZZ];
    L0 += b1.z * D[XY] + b1.w * D[XZ] + b2.y * D[YZ];
    acc[M] += L0;
    acc[X] += m0 * D[X];
    acc[Y] += m0 * D[Y];
    acc[Z] += m0 * D[Z];
    acc[XX] += m0 * D[XX];
    acc[XY] += m0 * D[XY];
    acc[XZ] += m0 * D[XZ];
    acc[YY] += m0 * D[YY];
    acc[YZ] += m0 * D[YZ];
    acc[ZZ] += m0 * D[ZZ];
}

struct DownArgs {
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
    const float4 *pos4;
    float4 *acc4;
    float *gnorm;
    const uint8_t *active;
    uint32_t *health;
};

__device__ __forceinline__ void m2l_node(const DownArgs &a, int node, float lx, float ly, float lz, float *acc) {
    const float4 *bp = a.poles + (size_t)a.T[node + 1] * kPoleQ;
    m2l_add(lx, ly, lz, bp[0], bp[1], bp[2], acc);
}

__global__ void __launch_bounds__(128) k_down(DownArgs a, int level, int64_t level_cap) {
    const int lane = threadIdx.x & 31;
    const int warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int cnt = a.level_count[level];
    const int32_t *nodes = a.level_nodes + (size_t)level * level_cap;
    const int32_t *T = a.T;
    const int cap = a.list_cap;
    for (int t = warp0; t < cnt; t += nwarps) {
        const int tp = nodes[t];
        if (tp == 0 && T[0] != 0) {
            // the root is a leaf: the reference would read particle ids as
            // child pointers here; no down pass is run
            if (lane == 0) raise_health(a.health, SPH_HEALTH_ROOT_LEAF);
            continue;
        }
        if (tp == 0) {
            // helpers.h:15-32 (zeroFirstBranches); the root's list is slot 0
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
        const float4 *sp = a.poles + (size_t)dp * kPoleQ;
        const float4 s0 = sp[0];
        const float s_min_grav = sp[3].w;
        if (sp[4].w == 0.f) continue;  // inactive node: no local field
        const int np = T[tp];
        const int slot = (np == 0) ? a.list_slot[dp] : 0;
        const int pslot = a.parent_slot[dp];
        if ((np == 0 && (slot < 0 || slot >= a.branch_cap)) || pslot < 0 || pslot >= a.branch_cap) {
            if (lane == 0) raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
            continue;
        }
        int32_t *out = a.list_out + (size_t)slot * cap;
        const int32_t *in = a.list_in + (size_t)pslot * cap;
        int op = 0;
        if (np == 0) {
            if (lane == 0) out[0] = tp;
            op = 1;
        }
        const float4 *lp = a.locals + (size_t)dp * kLocalQ;
        const float4 L0 = lp[0], L1 = lp[1], L2 = lp[2], L3 = lp[3];
        const float lx = L0.x, ly = L0.y, lz = L0.z;
#ifdef SPH_PARITY
        // Parity build: one lane walks the list in order and adds every
        // contribution straight into the node's local expansion, which is the
        // reference's summation order (helpers.h:34-45, 125-147).
        float le[10] = {L0.w, L1.x, L1.y, L1.z, L1.w, L2.x, L2.y, L2.z, L2.w, L3.x};
        if (lane == 0) {
            for (int i = 0; i < cap; ++i) {
                int e = in[i];
                if (e < -1 || e > a.tree_cap - 10) {
                    raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
                    e = -1;
                }
                if (e == -1) break;
                const float4 *bp = a.poles + (size_t)T[e + 1] * kPoleQ;
                const float4 b0 = bp[0], b1 = bp[1], b2 = bp[2];
                if ((np != 0 && T[e] != 0) || mac_accept(s0.w, s0.x, s0.y, s0.z, s_min_grav, b0, b1, b2)) {
                    m2l_add(lx, ly, lz, b0, b1, b2, le);
                    continue;
                }
                for (int k = 0; k < 8; ++k) {
                    const int c = T[e + 2 + k];
                    if (c == tp || c == -1) continue;
                    const float4 *cp = a.poles + (size_t)T[c + 1] * kPoleQ;
                    const float4 c0v = cp[0], c1v = cp[1], c2v = cp[2];
                    const bool force = np != 0 || T[c] != 0 || op == cap;
                    if (force || mac_accept(s0.w, s0.x, s0.y, s0.z, s_min_grav, c0v, c1v, c2v))
                        m2l_add(lx, ly, lz, c0v, c1v, c2v, le);
                    else
                        out[op++] = c;
                }
            }
            if (np == 0 && op < cap) out[op] = -1;
        }
#pragma unroll
        for (int j = 0; j < 10; ++j) le[j] = __shfl_sync(0xffffffffu, le[j], 0);
#else
        float acc[10];
#pragma unroll
        for (int j = 0; j < 10; ++j) acc[j] = 0.f;
        for (int c0 = 0; c0 < cap; c0 += 32) {
            const int i = c0 + lane;
            int e = (i < cap) ? in[i] : -1;
            if (e < -1 || e > a.tree_cap - 10) {  // a corrupt list entry ends the list
                raise_health(a.health, SPH_HEALTH_LIST_CAPACITY);
                e = -1;
            }
            const uint32_t stop = __ballot_sync(0xffffffffu, e == -1);
            const int nvalid = stop ? (__ffs(stop) - 1) : 32;
            uint32_t cand = 0u;
            if (lane < nvalid) {
                const float4 *bp = a.poles + (size_t)T[e + 1] * kPoleQ;
                const float4 b0 = bp[0], b1 = bp[1], b2 = bp[2];
                if (mac_accept(s0.w, s0.x, s0.y, s0.z, s_min_grav, b0, b1, b2)) {
                    m2l_add(lx, ly, lz, b0, b1, b2, acc);
                } else {
                    for (int k = 0; k < 8; ++k) {
                        const int c = T[e + 2 + k];
                        if (c == tp || c == -1) continue;
                        if (np != 0 || T[c] != 0) {
                            // leaf target: every child forced (helpers.h:83-123, depth 1);
                            // leaf child of a branch target: forced (helpers.h:141)
                            m2l_node(a, c, lx, ly, lz, acc);
                        } else {
                            const float4 *cp = a.poles + (size_t)T[c + 1] * kPoleQ;
                            const float4 c0v = cp[0], c1v = cp[1], c2v = cp[2];
                            if (mac_accept(s0.w, s0.x, s0.y, s0.z, s_min_grav, c0v, c1v, c2v))
                                m2l_add(lx, ly, lz, c0v, c1v, c2v, acc);
                            else
                                cand |= 1u << k;
                        }
                    }
                }
            }
            if (np == 0) {
                // ordered append of the rejected branch children (entry-major)
                const int mine = __popc(cand);
                int incl = mine;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                int pos = op + incl - mine;
                while (cand) {
                    const int k = __ffs(cand) - 1;
                    cand &= cand - 1u;
                    const int c = T[e + 2 + k];
                    if (pos < cap)
                        out[pos] = c;
                    else
                        m2l_node(a, c, lx, ly, lz, acc);  // list full: forced accept
                    ++pos;
                }
                op = min(op + total, cap);
            }
            if (stop) break;
        }
        if (np == 0 && lane == 0 && op < cap) out[op] = -1;
        // sum the lanes' partial expansions
#pragma unroll
        for (int j = 0; j < 10; ++j) {
            float v = acc[j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            acc[j] = v;
        }
        float le[10] = {L0.w + acc[0], L1.x + acc[1], L1.y + acc[2], L1.z + acc[3], L1.w + acc[4],
                        L2.x + acc[5], L2.y + acc[6], L2.z + acc[7], L2.w + acc[8], L3.x + acc[9]};
#endif
        if (np == 0) {
            // L2L.metal:56-70 to every active child (empty slots skipped)
            if (lane < 8) {
                const int c = T[tp + 2 + lane];
                if (c != -1) {
                    const int cdp = T[c + 1];
                    const float4 *cp = a.poles + (size_t)cdp * kPoleQ;
                    if (cp[4].w != 0.f) {
                        const float4 cpos = cp[0];
                        const float rx = cpos.x - lx, ry = cpos.y - ly, rz = cpos.z - lz;
                        float o[10];
                        o[M] = le[M];
                        o[M] += rx * le[X] + ry * le[Y] + rz * le[Z];
                        o[X] = le[X];
                        o[Y] = le[Y];
                        o[Z] = le[Z];
                        o[M] += 0.5f * (rx * rx * le[XX] + ry * ry * le[YY] + rz * rz * le[ZZ]);
                        o[M] += rx * ry * le[XY] + rx * rz * le[XZ] + ry * rz * le[YZ];
                        o[X] += rx * le[XX] + ry * le[XY] + rz * le[XZ];
                        o[Y] += rx * le[XY] + ry * le[YY] + rz * le[YZ];
                        o[Z] += rx * le[XZ] + ry * le[YZ] + rz * le[ZZ];
                        float4 *clp = a.locals + (size_t)cdp * kLocalQ;
                        clp[0] = make_float4(lx + rx, ly + ry, lz + rz, o[M]);
                        clp[1] = make_float4(o[X], o[Y], o[Z], le[XX]);
                        clp[2] = make_float4(le[XY], le[XZ], le[YY], le[YZ]);
                        clp[3] = make_float4(le[ZZ], 0.f, 0.f, 0.f);
                    }
                }
            }
        } else {
            // helpers.h:47-81: L2P + P2P inside the leaf
            const int s = tp + 2;
            for (int i0 = 0; i0 < np; i0 += 32) {
                const int ii = i0 + lane;
                if (ii >= np) continue;
                const int p = T[s + ii];
                if (!a.active[p]) continue;
                const float4 xi = a.pos4[p];
                const float qx = xi.x - lx, qy = xi.y - ly, qz = xi.z - lz;
                float ax = le[X], ay = le[Y], az = le[Z];
                ax += qx * le[XX] + qy * le[XY] + qz * le[XZ];
                ay += qx * le[XY] + qy * le[YY] + qz * le[YZ];
                az += qx * le[XZ] + qy * le[YZ] + qz * le[ZZ];
                for (int j = 0; j < np; ++j) {
                    if (j == ii) continue;
                    const float4 xj = a.pos4[T[s + j]];
                    const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
                    const float r = sqrtf(dx * dx + dy * dy + dz * dz);
                    if (r == 0.f) continue;
                    const float rhx = dx / r, rhy = dy / r, rhz = dz / r;
                    const float fm = xj.w * grav_dphi_dr(r);
                    ax -= fm * rhx;
                    ay -= fm * rhy;
                    az -= fm * rhz;
                }
                const float4 old = a.acc4[p];
                a.acc4[p] = make_float4(kG * ax, kG * ay, kG * az, old.w);
                a.gnorm[p] = sqrtf(ax * ax + ay * ay + az * az);
            }
        }
    }
}

}  // namespace

sph_status launch_gravity(sph_ctx *ctx, cudaStream_t st) {
    Tree &tr = ctx->tree;
    if (!tr.valid || ctx->n <= 0) return SPH_OK;
    const int L = tr.n_levels_host;
    UpArgs u;
    u.T = tr.tree;
    u.level_nodes = tr.level_nodes;
    u.level_count = tr.level_count;
    u.list_slot = tr.list_slot;
    u.parent_slot = tr.parent_slot;
    u.poles = tr.poles;
    u.pos4 = ctx->pos4;
    u.gnorm = ctx->gnorm;
    u.active = ctx->active;
    u.nat = ctx->nat;
    u.globals = ctx->globals;
    u.individual = ctx->form.timestep == SPH_TIMESTEP_INDIVIDUAL;
    for (int l = L - 1; l >= 0; --l) {
        int64_t bound = tr.level_count_host[l];
        int blocks = (int)((bound + 127) / 128);
        blocks = blocks < 1 ? 1 : (blocks > 148 * 32 ? 148 * 32 : blocks);
        k_up<<<blocks, 128, 0, st>>>(u, l, tr.level_cap);
    }
    DownArgs d;
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
    d.pos4 = ctx->pos4;
    d.acc4 = ctx->acc4;
    d.gnorm = ctx->gnorm;
    d.active = ctx->active;
    d.health = ctx->health;
    for (int l = 0; l < L; ++l) {
        d.list_in = (l % 2 == 0) ? tr.lists[0] : tr.lists[1];
        d.list_out = (l % 2 == 0) ? tr.lists[1] : tr.lists[0];
        int64_t bound = tr.level_count_host[l];
        int blocks = (int)((bound * 32 + 127) / 128);
        blocks = blocks < 1 ? 1 : (blocks > 148 * 32 ? 148 * 32 : blocks);
        k_down<<<blocks, 128, 0, st>>>(d, l, tr.level_cap);
    }
    return cuda_status(cudaGetLastError(), "gravity");
}

}  // namespace sph

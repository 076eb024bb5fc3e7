// oracle.cpp -- CPU restatement of the reference's per-step hot path.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  The product never links this file.
//
// Each function below restates one reference kernel or host routine and
// cites it as `file:line` within the reference project (SPH/...).  The
// arithmetic is written operation-for-operation in the reference's order and
// in single precision (Metal treats unsuffixed literals as float, so every
// literal here carries an `f`), and the library is compiled with
// -ffp-contract=off so that it is bit-reproducible against the reference
// kernels compiled through oracle/ref_shim (oracle/_ref/libref.so).
//
// Quirks of the reference are reproduced on purpose (each one is described
// where it occurs, with the reference line it comes from); the two places
// where the reference reads out of bounds are given defined behaviour and say
// so.

#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---- SPH/Parameters.h:11-53, as single-precision values -------------------
constexpr float kViscosityAlpha = 1.5f;         // :12
constexpr float kDensityEta = 0.005f;           // :13
constexpr float kMaxH = 1.f;                    // :14
constexpr int kMaxNR = 50;                      // :15
constexpr int kNeighbourCache = 128;            // :16
constexpr float kResolutionEta = 1.2348f;       // :17
constexpr float kAneosMinU = 1e-10f;            // :23
constexpr float kAneosMinRho = 1e-6f;           // :21
constexpr float kCFL = 0.2f;                    // :27
constexpr float kDT0 = 32.f;                    // :28
constexpr int kRMax = 16;                       // :29
constexpr float kDtMin1 = kDT0 / (1 << kRMax);  // :30
constexpr float kGamma = 1.825742f;             // :33
constexpr float kGravityEta = 0.005f;           // :36
constexpr float kGravSoft = 0.04f;              // :40
constexpr float kCellWidth = 0.18f;             // :47
constexpr int kCellPower = 8;                   // :48
constexpr int kCellsPerDim = 1 << kCellPower;
constexpr float kG = 6.67e-5f;                  // gravity/poles/poles.h:16
constexpr float kPi1 = 1 / 3.14159265358979323846f;  // utils/kernels.h:14

int g_threads = 0;

inline float fminf_(float a, float b) { return b < a ? b : a; }
inline float fmaxf_(float a, float b) { return a < b ? b : a; }

struct F3 {
    float x, y, z;
};
inline F3 ld3(const float *a, int i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
inline void st3(float *a, int i, F3 v) {
    a[3 * i] = v.x;
    a[3 * i + 1] = v.y;
    a[3 * i + 2] = v.z;
}
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float len2(F3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// ---- utils/morton.h:16-34: interleave 8-bit cell coordinates --------------
// Bit b of x lands on bit 3b, of y on 3b+1, of z on 3b+2.
inline uint32_t spread3(uint32_t v) {
    uint32_t out = 0;
    for (int b = 0; b < 10; ++b) out |= ((v >> b) & 1u) << (3 * b);
    return out;
}
inline uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// ---- sort.metal:15-44 (hash) ----------------------------------------------
inline uint32_t cell_key(F3 p) {
    float nx = p.x / kCellWidth, ny = p.y / kCellWidth, nz = p.z / kCellWidth;
    int cx = (int)std::floor(nx) % kCellsPerDim;
    int cy = (int)std::floor(ny) % kCellsPerDim;
    int cz = (int)std::floor(nz) % kCellsPerDim;
    if (cx < 0) cx += kCellsPerDim;
    if (cy < 0) cy += kCellsPerDim;
    if (cz < 0) cz += kCellsPerDim;
    return morton3((uint32_t)cx, (uint32_t)cy, (uint32_t)cz);
}

// ---- utils/cellsToScan.h:21-59 --------------------------------------------
inline uint32_t cell_index_of(int x, int y, int z) {
    const int mask = kCellsPerDim - 1;
    return morton3((uint32_t)(x & mask), (uint32_t)(y & mask), (uint32_t)(z & mask));
}
struct CellBox {
    int lo[3], hi[3];
};
inline CellBox cell_box(F3 p, float h) {
    float radius = 2.f * h;
    F3 mn = {p.x - radius, p.y - radius, p.z - radius};
    F3 mx = {p.x + radius, p.y + radius, p.z + radius};
    CellBox b;
    b.lo[0] = (int)std::floor(mn.x / kCellWidth);
    b.lo[1] = (int)std::floor(mn.y / kCellWidth);
    b.lo[2] = (int)std::floor(mn.z / kCellWidth);
    b.hi[0] = (int)std::floor(mx.x / kCellWidth);
    b.hi[1] = (int)std::floor(mx.y / kCellWidth);
    b.hi[2] = (int)std::floor(mx.z / kCellWidth);
    return b;
}

// ---- utils/kernels.h:35-85: cubic spline M4, support 2h -------------------
inline float kernel_w(float r, float h1) {  // :35-50
    float q = r * h1;
    if (q > 2.f) return 0.f;
    float fac = kPi1 * h1 * h1 * h1;
    if (q > 1.f) {
        float t = 2.f - q;
        return fac * 0.25f * t * t * t;
    }
    return fac * (1.f - 1.5f * q * q * (1.f - 0.5f * q));
}
inline F3 kernel_gradw(F3 xij, float r, float r1, float h1) {  // :52-69
    float q = r * h1;
    if (q > 2.f || q < 1e-12f) return {0.f, 0.f, 0.f};
    F3 rh = {xij.x * r1, xij.y * r1, xij.z * r1};
    float fac = kPi1 * h1 * h1 * h1 * h1;
    float s;
    if (q > 1.f) {
        float t = 2.f - q;
        s = -0.75f * fac * t * t;
    } else {
        s = 3.f * fac * (0.75f * q - 1.f) * q;
    }
    return {s * rh.x, s * rh.y, s * rh.z};
}
inline float kernel_dwdh(float r, float h1) {  // :71-85
    float q = r * h1;
    if (q > 2.f) return 0.f;
    float fac = -3.f * kPi1 * h1 * h1 * h1 * h1;
    if (q > 1.f) return fac * (2.f - 4.f * q + 2.5f * q * q - 0.5f * q * q * q);
    return fac * (1.f + 0.5f * (3.f * q - 5.f) * q * q);
}
// kernels.h:87-102 with the reference's integer-division coefficients (Q2):
// (4/3)=1, (6/5)=1, (8/3)=2, (1/6)=0, (1/15)=0; h is min(0.04, 0.16).
inline float grav_dphi_dr(F3 xij) {
    float h1 = 1.f / fminf_(kGravSoft, 0.16f);
    float r = std::sqrt(len2(xij));
    float q = r * h1;
    if (q <= 1.f) return (h1 * h1) * (1.f * q - 1.f * q * q * q + 0.5f * q * q * q * q);
    if (q <= 2.f) {
        float q1 = 1.f / q;
        return (h1 * h1) * (2.f * q - 3.f * q * q + 1.f * q * q * q - 0.f * q * q * q * q - 0.f * q1 * q1);
    }
    float r1 = 1.f / r;
    return r1 * r1;
}

// ---- EOS sample: bilinear, normalised coordinates, texel centres at (i+0.5)/res,
// clamp-to-edge (density.metal:45-53 sampler).  Same formula as the CUDA path.
inline void eos_sample(const float *tab, int res, float u, float v, float &p, float &c) {
    float x = u * (float)res - 0.5f;
    float y = v * (float)res - 0.5f;
    float xf = std::floor(x), yf = std::floor(y);
    float fx = x - xf, fy = y - yf;
    int x0 = (int)xf, y0 = (int)yf;
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = std::min(std::max(x0, 0), res - 1);
    x1 = std::min(std::max(x1, 0), res - 1);
    y0 = std::min(std::max(y0, 0), res - 1);
    y1 = std::min(std::max(y1, 0), res - 1);
    const float *t00 = tab + 2 * ((size_t)y0 * res + x0);
    const float *t10 = tab + 2 * ((size_t)y0 * res + x1);
    const float *t01 = tab + 2 * ((size_t)y1 * res + x0);
    const float *t11 = tab + 2 * ((size_t)y1 * res + x1);
    float gx = 1.f - fx, gy = 1.f - fy;
    p = (t00[0] * gx + t10[0] * fx) * gy + (t01[0] * gx + t11[0] * fx) * fy;
    c = (t00[1] * gx + t10[1] * fx) * gy + (t01[1] * gx + t11[1] * fx) * fy;
}
// density.metal:45-50 / :228-233: coordinates of the (rho, u) lookup.
inline void eos_lookup(const ora_state *st, int mat, float rho, float u, float &p, float &c) {
    float uc = std::log(u / kAneosMinU) / std::log(1.f / kAneosMinU);
    float rc = std::log(rho / kAneosMinRho) / std::log(1.f / kAneosMinRho);
    uc = std::min(std::max(uc, 0.f), 1.f);
    rc = std::min(std::max(rc, 0.f), 1.f);
    const float *tab = ((float)mat == 400.f) ? st->eos_forsterite : st->eos_fe;
    eos_sample(tab, st->eos_res, uc, rc, p, c);
}

// ---- gravity/poles/poles.h:46-61 ------------------------------------------
enum { M = 0, X = 1, Y = 2, Z = 3, XX = 4, XY = 5, XZ = 6, YY = 7, YZ = 8, ZZ = 9 };
struct Pole {
    F3 pos, mn, mx;
    float size;
    float e[10];
    float power[3];
    float min_grav;
    bool active;
};
struct Loc {
    F3 pos;
    float e[10];
};

// gravity/poles/helpers.metal:63-89 (p = 2): note the 0.5 weights on XX, XY,
// XZ, YZ but not on YY, ZZ -- reproduced as written.
inline void add_powers(Pole &mp) {
    mp.power[0] = mp.e[M];
    mp.power[1] = 0.f;
    float s = mp.e[ZZ] * mp.e[ZZ];
    s += 0.5f * mp.e[YZ] * mp.e[YZ];
    s += mp.e[YY] * mp.e[YY];
    s += 0.5f * mp.e[XZ] * mp.e[XZ];
    s += 0.5f * mp.e[XY] * mp.e[XY];
    s += 0.5f * mp.e[XX] * mp.e[XX];
    mp.power[2] = std::sqrt(s);
}

// gravity/poles/accept.metal:14-55 (SWIFT-style adaptive MAC, no opening angle).
inline bool mac_accept(const Pole &A, const Pole &B) {
    const float ra = A.size, rb = B.size;
    F3 d = sub(A.pos, B.pos);
    const float r2 = len2(d);
    const float rs = ra + rb;
    if (rs * rs > r2) return false;
    const float rmax = fmaxf_(ra, rb);
    float e = 0.f;
    e += 1.f * B.power[0] * (ra * ra);  // binomial(2,0) * P0 * ra^2
    e += 2.f * B.power[1] * ra;         // binomial(2,1) * P1 * ra
    e += 1.f * B.power[2] * 1.f;        // binomial(2,2) * P2
    e *= 8.f;
    if (ra + rb > 0.f) {
        e *= rmax;
        e /= (ra + rb);
    }
    const float r_to_p = r2;  // integer_powf(r2, p/2)
    return e < kGravityEta * A.min_grav * r_to_p * r2;
}

// gravity/poles/derivatives.metal:12-156 (p = 2, softened inside eps).
inline void derivs(F3 v, float eps, float D[10]) {
    float r2 = len2(v);
    float r = std::sqrt(r2);
    float rinv = r > 1e-6f ? 1.f / r : 0.f;
    float eps2 = eps * eps;
    float d1, d2, d3;
    if (r2 < eps2) {
        const float ei = 1.f / eps;
        const float u = r * ei;
        float s1 = -3.f * u + 15.f;  // D_soft_1
        s1 = s1 * u - 28.f;
        s1 = s1 * u + 21.f;
        s1 = s1 * u;
        s1 = s1 * u - 7.f;
        s1 = s1 * u;
        s1 = s1 * u + 3.f;
        float s2 = -21.f * u + 90.f;  // D_soft_2
        s2 = s2 * u - 140.f;
        s2 = s2 * u + 84.f;
        s2 = s2 * u;
        s2 = s2 * u - 14.f;
        s2 = s2 * u;
        float s3 = -105.f * u + 360.f;  // D_soft_3
        s3 = s3 * u - 420.f;
        s3 = s3 * u + 168.f;
        s3 = s3 * u;
        s3 = s3 * u;
        d1 = ei * s1;
        const float ei2 = ei * ei;
        d2 = ei2 * s2;
        const float ei3 = ei2 * ei;
        d3 = ei3 * s3;
    } else {
        d1 = rinv;
        d2 = -1.f * d1 * rinv;
        d3 = -3.f * d2 * rinv;
    }
    const float rx = v.x * rinv, ry = v.y * rinv, rz = v.z * rinv;
    const float rx2 = rx * rx, ry2 = ry * ry, rz2 = rz * rz;
    D[M] = d1;
    D[X] = rx * d2;
    D[Y] = ry * d2;
    D[Z] = rz * d2;
    d2 *= rinv;
    D[XX] = rx2 * d3 + d2;
    D[XY] = rx * ry * d3;
    D[XZ] = rx * rz * d3;
    D[YY] = ry2 * d3 + d2;
    D[YZ] = ry * rz * d3;
    D[ZZ] = rz2 * d3 + d2;
}

// gravity/poles/M2L.metal:12-108 (p = 2), added into `acc` in the order of
// helpers.h:39-42.
inline void m2l_add(F3 x, const Pole &mp, float acc[10]) {
    float D[10];
    derivs(sub(x, mp.pos), kGravSoft, D);
    float L[10];
    const float m0 = mp.e[M];
    L[M] = m0 * D[M];
    L[X] = m0 * D[X];
    L[Y] = m0 * D[Y];
    L[Z] = m0 * D[Z];
    L[M] += mp.e[XX] * D[XX] + mp.e[YY] * D[YY] + mp.e[ZZ] * D[ZZ];
    L[M] += mp.e[XY] * D[XY] + mp.e[XZ] * D[XZ] + mp.e[YZ] * D[YZ];
    L[XX] = m0 * D[XX];
    L[YY] = m0 * D[YY];
    L[ZZ] = m0 * D[ZZ];
    L[XY] = m0 * D[XY];
    L[XZ] = m0 * D[XZ];
    L[YZ] = m0 * D[YZ];
    for (int j = 0; j < 10; ++j) acc[j] += L[j];
}

// gravity/poles/L2L.metal:12-54 (transformLocal, p = 2).
inline Loc shift_local(const Loc &l, F3 r) {
    Loc o;
    o.pos = {l.pos.x + r.x, l.pos.y + r.y, l.pos.z + r.z};
    o.e[M] = l.e[M];
    o.e[M] += r.x * l.e[X] + r.y * l.e[Y] + r.z * l.e[Z];
    o.e[X] = l.e[X];
    o.e[Y] = l.e[Y];
    o.e[Z] = l.e[Z];
    o.e[M] += 0.5f * (r.x * r.x * l.e[XX] + r.y * r.y * l.e[YY] + r.z * r.z * l.e[ZZ]);
    o.e[M] += r.x * r.y * l.e[XY] + r.x * r.z * l.e[XZ] + r.y * r.z * l.e[YZ];
    o.e[X] += r.x * l.e[XX] + r.y * l.e[XY] + r.z * l.e[XZ];
    o.e[Y] += r.x * l.e[XY] + r.y * l.e[YY] + r.z * l.e[YZ];
    o.e[Z] += r.x * l.e[XZ] + r.y * l.e[YZ] + r.z * l.e[ZZ];
    o.e[XX] = l.e[XX];
    o.e[XY] = l.e[XY];
    o.e[XZ] = l.e[XZ];
    o.e[YY] = l.e[YY];
    o.e[YZ] = l.e[YZ];
    o.e[ZZ] = l.e[ZZ];
    return o;
}

// gravity/poles/L2P.metal:12-32 (p = 2).
inline F3 l2p(const Loc &l, F3 p) {
    F3 r = sub(p, l.pos);
    F3 a = {l.e[X], l.e[Y], l.e[Z]};
    a.x += r.x * l.e[XX] + r.y * l.e[XY] + r.z * l.e[XZ];
    a.y += r.x * l.e[XY] + r.y * l.e[YY] + r.z * l.e[YZ];
    a.z += r.x * l.e[XZ] + r.y * l.e[YZ] + r.z * l.e[ZZ];
    return a;
}

// gravity/poles/P2M.metal:12-107 (leaf multipole; writes active[] of the leaf).
Pole p2m(const ora_state *st, int tp) {
    const int32_t *T = st->tree;
    Pole mp;
    int n = T[tp];
    int s = tp + 2, e = s + n;
    mp.pos = {0.f, 0.f, 0.f};
    for (float &v : mp.e) v = 0.f;
    mp.min_grav = FLT_MAX;
    mp.active = false;
    mp.mx = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    mp.mn = {FLT_MAX, FLT_MAX, FLT_MAX};
    const int gt = *st->global_time;
    for (int i = s; i < e; ++i) {
        int p = T[i];
        float m = st->mass[p];
        F3 x = ld3(st->pos, p);
        bool act = gt <= st->next_active_time[p];  // Q1
        if (!mp.active && act) mp.active = true;
        mp.mx = {fmaxf_(mp.mx.x, x.x), fmaxf_(mp.mx.y, x.y), fmaxf_(mp.mx.z, x.z)};
        mp.mn = {fminf_(mp.mn.x, x.x), fminf_(mp.mn.y, x.y), fminf_(mp.mn.z, x.z)};
        mp.e[M] += m;
        mp.pos.x += x.x * m;
        mp.pos.y += x.y * m;
        mp.pos.z += x.z * m;
        if (act) mp.min_grav = fminf_(mp.min_grav, st->grav_norm[p]);
    }
    for (int i = s; i < e; ++i) st->active[T[i]] = mp.active;
    mp.pos = {mp.pos.x / mp.e[M], mp.pos.y / mp.e[M], mp.pos.z / mp.e[M]};
    for (int i = s; i < e; ++i) {
        int p = T[i];
        float m = st->mass[p];
        F3 r = sub(ld3(st->pos, p), mp.pos);
        mp.e[X] -= r.x * m;
        mp.e[Y] -= r.y * m;
        mp.e[Z] -= r.z * m;
        mp.e[XX] += m * r.x * r.x;
        mp.e[XY] += m * r.x * r.y;
        mp.e[XZ] += m * r.x * r.z;
        mp.e[YY] += m * r.y * r.y;
        mp.e[YZ] += m * r.y * r.z;
        mp.e[ZZ] += m * r.z * r.z;
    }
    mp.e[XX] *= 0.5f;
    mp.e[YY] *= 0.5f;
    mp.e[ZZ] *= 0.5f;
    F3 d = sub(mp.mx, mp.mn);
    mp.size = fmaxf_(d.x, fmaxf_(d.y, d.z));
    add_powers(mp);
    return mp;
}

// gravity/poles/M2M.metal:12-160 (branch multipole).  Q5: the ZZ shift uses
// the child's expansion[Z]; Q6: the leaf-sync loop bound uses the parent's start.
Pole m2m(const ora_state *st, std::vector<Pole> &poles, std::vector<uint32_t> &parent, uint32_t index, int tp) {
    const int32_t *T = st->tree;
    Pole mp;
    mp.min_grav = FLT_MAX;
    mp.pos = {0.f, 0.f, 0.f};
    mp.active = false;
    for (float &v : mp.e) v = 0.f;
    float mass = 0.f;
    mp.mx = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    mp.mn = {FLT_MAX, FLT_MAX, FLT_MAX};
    int s = tp + 2, e = s + 8;
    bool all_leaves = true;
    for (int i = s; i < e; ++i) {
        int c = T[i];
        if (c == -1) continue;
        int cdp = T[c + 1];
        parent[cdp] = index;
        const Pole &cm = poles[cdp];
        mp.min_grav = fminf_(cm.min_grav, mp.min_grav);
        mass += cm.e[M];
        mp.pos.x += cm.pos.x * cm.e[M];
        mp.pos.y += cm.pos.y * cm.e[M];
        mp.pos.z += cm.pos.z * cm.e[M];
        if (!mp.active && cm.active) mp.active = true;
        if (all_leaves && T[c] == 0) all_leaves = false;
        mp.mx = {fmaxf_(mp.mx.x, cm.mx.x), fmaxf_(mp.mx.y, cm.mx.y), fmaxf_(mp.mx.z, cm.mx.z)};
        mp.mn = {fminf_(mp.mn.x, cm.mn.x), fminf_(mp.mn.y, cm.mn.y), fminf_(mp.mn.z, cm.mn.z)};
    }
    F3 d = sub(mp.mx, mp.mn);
    mp.size = fmaxf_(d.x, fmaxf_(d.y, d.z));
    mp.pos = {mp.pos.x / mass, mp.pos.y / mass, mp.pos.z / mass};
    for (int i = s; i < e; ++i) {
        int c = T[i];
        if (c == -1) continue;
        int cdp = T[c + 1];
        const Pole cm = poles[cdp];
        F3 r = sub(mp.pos, cm.pos);
        float t[10];
        t[M] = cm.e[M];
        t[X] = 0.f;
        t[Y] = 0.f;
        t[Z] = 0.f;
        t[XX] = cm.e[XX] + 0.5f * r.x * r.x * cm.e[M];
        t[XY] = cm.e[XY] + r.x * r.y * cm.e[M];
        t[XZ] = cm.e[XZ] + r.x * r.z * cm.e[M];
        t[YY] = cm.e[YY] + 0.5f * r.y * r.y * cm.e[M];
        t[YZ] = cm.e[YZ] + r.y * r.z * cm.e[M];
        t[ZZ] = cm.e[ZZ] + 0.5f * r.z * r.z * cm.e[Z];
        for (int j = 0; j < 10; ++j) mp.e[j] += t[j];
        if (all_leaves && mp.active && !cm.active) {
            poles[cdp].active = true;
            int np = T[c];
            int cs = c + 2;
            int ce = s + np;  // Q6
            for (int j = cs; j < ce; ++j) st->active[T[j]] = true;
        }
    }
    add_powers(mp);
    return mp;
}

struct Gravity {
    ora_state *st;
    std::vector<Pole> poles;
    std::vector<Loc> locals;
    std::vector<uint32_t> parent;
    std::vector<int32_t> lists[2];
    int cap;

    const int32_t *level(int l, int &count) const {
        count = st->level_offsets[l + 1] - st->level_offsets[l];
        return st->level_nodes + st->level_offsets[l];
    }

    // gravity/helpers.h:34-45
    bool check_add(const Pole &self, Loc &loc, int node, bool force) {
        const Pole &nm = poles[st->tree[node + 1]];
        if (force || mac_accept(self, nm)) {
            m2l_add(loc.pos, nm, loc.e);
            return true;
        }
        return false;
    }

    // gravity/helpers.h:15-32
    void zero_first_branches(int32_t *out) {
        const int32_t *T = st->tree;
        for (int i = 2; i < 10; ++i) {
            int np = T[i];
            if (np == -1) continue;
            int dp = T[np + 1];
            locals[dp].pos = poles[dp].pos;
            for (float &v : locals[dp].e) v = 0.f;
        }
        out[0] = 0;
        out[1] = -1;
    }

    // gravity/helpers.h:47-81 (L2P plus the intra-leaf P2P, Q3)
    void local_to_leaf(const Loc &loc, int tp, int n) {
        const int32_t *T = st->tree;
        int s = tp + 2, e = s + n;
        for (int i = s; i < e; ++i) {
            int p = T[i];
            if (!st->active[p]) continue;
            F3 xi = ld3(st->pos, p);
            F3 a = l2p(loc, xi);
            for (int j = s; j < e; ++j) {
                if (i == j) continue;
                int pj = T[j];
                F3 xj = ld3(st->pos, pj);
                float mj = st->mass[pj];
                F3 xij = sub(xi, xj);
                const float r = std::sqrt(len2(xij));
                if (r == 0.f) continue;
                F3 rh = {xij.x / r, xij.y / r, xij.z / r};
                float f = mj * grav_dphi_dr(xij);
                a.x -= f * rh.x;
                a.y -= f * rh.y;
                a.z -= f * rh.z;
            }
            st3(st->acc, p, {kG * a.x, kG * a.y, kG * a.z});
            st->grav_norm[p] = std::sqrt(len2(a));
        }
    }

    // gravity.metal:64-143 for one node of level l, thread index t.
    void down_node(int l, int t, const int32_t *in, int32_t *out) {
        const int32_t *T = st->tree;
        int cnt;
        const int32_t *nodes = level(l, cnt);
        int tp = nodes[t];
        if (tp == 0) {
            zero_first_branches(out);
            return;
        }
        int dp = T[tp + 1];
        const Pole mp = poles[dp];
        if (!mp.active) return;
        uint32_t op = (uint32_t)t * cap, op_max = (uint32_t)(t + 1) * cap;
        int np = T[tp];
        if (np == 0) out[op++] = tp;
        uint32_t pi = parent[dp];
        uint32_t s0 = pi * cap, s1 = (pi + 1) * cap;
        Loc loc = locals[dp];
        for (uint32_t i = s0; i < s1; ++i) {
            int e = in[i];
            if (e == -1) break;
            if (np != 0) {
                // helpers.h:83-123 with GRAVITY_MAX_RECURSION = 1: every child forced.
                if (check_add(mp, loc, e, T[e] != 0)) continue;
                for (int k = e + 2; k < e + 10; ++k) {
                    int c = T[k];
                    if (c == tp || c == -1) continue;
                    check_add(mp, loc, c, true);
                }
            } else {
                // helpers.h:125-147
                if (check_add(mp, loc, e, false)) continue;
                for (int k = e + 2; k < e + 10; ++k) {
                    int c = T[k];
                    if (c == tp || c == -1) continue;
                    if (!check_add(mp, loc, c, T[c] != 0 || op == op_max)) out[op++] = c;
                }
            }
        }
        if (op < op_max && np == 0) out[op] = -1;
        if (np == 0) {
            // L2L.metal:56-70 (slots holding -1 are skipped; the reference then
            // writes a transformed copy into the root's unused local)
            for (int k = tp + 2; k < tp + 10; ++k) {
                int c = T[k];
                if (c == -1) continue;
                int cdp = T[c + 1];
                const Pole &cm = poles[cdp];
                if (!cm.active) continue;
                F3 r = sub(cm.pos, loc.pos);
                locals[cdp] = shift_local(loc, r);
            }
        } else {
            local_to_leaf(loc, tp, np);
        }
    }

    void run() {
        const int32_t *T = st->tree;
        int nn = st->n_nodes;
        poles.assign(nn, Pole{});
        locals.assign(nn, Loc{});
        parent.assign(nn, 0u);
        int L = st->n_levels;
        int max_level = 1;
        for (int l = 0; l + 1 < L; ++l) {
            int c;
            level(l, c);
            max_level = std::max(max_level, c);
        }
        lists[0].assign((size_t)max_level * cap + 2, -1);
        lists[1].assign((size_t)max_level * cap + 2, -1);
        // upPass, deepest level first (gravity.metal:36-62, Compute.cpp:330-351)
        for (int l = L - 1; l >= 0; --l) {
            int cnt;
            const int32_t *nodes = level(l, cnt);
#pragma omp parallel for schedule(dynamic, 16)
            for (int t = 0; t < cnt; ++t) {
                int tp = nodes[t];
                int dp = T[tp + 1];
                if (T[tp] == 0)
                    poles[dp] = m2m(st, poles, parent, (uint32_t)t, tp);
                else
                    poles[dp] = p2m(st, tp);
            }
        }
        if (T[0] != 0) return;  // root is a leaf: the reference's down pass is undefined here
        // downPass, root first (Compute.cpp:353-376); lists ping-pong by level parity
        for (int l = 0; l < L; ++l) {
            int cnt;
            level(l, cnt);
            const int32_t *in = (l % 2 == 0) ? lists[0].data() : lists[1].data();
            int32_t *out = (l % 2 == 0) ? lists[1].data() : lists[0].data();
#pragma omp parallel for schedule(dynamic, 4)
            for (int t = 0; t < cnt; ++t) down_node(l, t, in, out);
        }
    }
};

inline void set_threads() {
#ifdef _OPENMP
    if (g_threads > 0) omp_set_num_threads(g_threads);
#endif
}

}  // namespace

extern "C" {

uint32_t ora_cell_key(float x, float y, float z) { return cell_key({x, y, z}); }

void ora_set_threads(int n) { g_threads = n; }
int ora_get_threads(void) {
#ifdef _OPENMP
    set_threads();
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Compute.cpp:265-326 driving sort.metal:15-148: hash, 4 stable 8-bit LSD
// counting passes (the reference's hist/scan/sum/sort), then the per-cell
// first/last sorted index (initialise + findCellPositions).
void ora_sort(ora_state *st) {
    set_threads();
    const int n = st->n;
    std::vector<uint32_t> k0(n), v0(n), k1(n), v1(n);
#pragma omp parallel for
    for (int i = 0; i < n; ++i) {
        k0[i] = cell_key(ld3(st->pos, i));
        v0[i] = (uint32_t)i;
    }
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 8 * pass;
        uint32_t count[257] = {0};
        for (int i = 0; i < n; ++i) count[((k0[i] >> shift) & 255u) + 1]++;
        for (int b = 0; b < 256; ++b) count[b + 1] += count[b];
        for (int i = 0; i < n; ++i) {
            uint32_t d = (k0[i] >> shift) & 255u;
            uint32_t dst = count[d]++;
            k1[dst] = k0[i];
            v1[dst] = v0[i];
        }
        k0.swap(k1);
        v0.swap(v1);
    }
    std::memcpy(st->cell_key, k0.data(), sizeof(uint32_t) * n);
    std::memcpy(st->cell_index, v0.data(), sizeof(uint32_t) * n);
    const size_t ncell = (size_t)1 << (3 * kCellPower);
    for (size_t c = 0; c < ncell; ++c) {
        st->cell_start[c] = UINT_MAX;
        st->cell_end[c] = 0u;
    }
    for (int i = 0; i < n; ++i) {
        uint32_t c = k0[i];
        st->cell_start[c] = std::min(st->cell_start[c], (uint32_t)i);
        st->cell_end[c] = std::max(st->cell_end[c], (uint32_t)i);
    }
}

static std::vector<float> g_last_poles, g_last_locals;

void ora_gravity(ora_state *st) {
    set_threads();
    if (st->n_levels <= 0 || st->tree_len <= 0) return;
    Gravity g;
    g.st = st;
    g.cap = st->max_unchecked > 0 ? st->max_unchecked : 1024;
    g.run();
    // keep the node records, in the CUDA library's layout, for diagnostics
    const size_t nn = g.poles.size();
    g_last_poles.assign(nn * 24, 0.f);
    g_last_locals.assign(nn * 16, 0.f);
    for (size_t i = 0; i < nn; ++i) {
        const Pole &p = g.poles[i];
        float *q = &g_last_poles[i * 24];
        const float v[24] = {p.pos.x, p.pos.y, p.pos.z, p.size, p.e[M], p.e[XX], p.e[XY], p.e[XZ],
                             p.e[YY], p.e[YZ], p.e[ZZ], p.power[2], p.mn.x, p.mn.y, p.mn.z, p.min_grav,
                             p.mx.x, p.mx.y, p.mx.z, p.active ? 1.f : 0.f, p.e[X], p.e[Y], p.e[Z], 0.f};
        std::memcpy(q, v, sizeof(v));
        const Loc &l = g.locals[i];
        float *r = &g_last_locals[i * 16];
        const float w[16] = {l.pos.x, l.pos.y, l.pos.z, l.e[0], l.e[1], l.e[2], l.e[3], l.e[4],
                             l.e[5], l.e[6], l.e[7], l.e[8], l.e[9], 0.f, 0.f, 0.f};
        std::memcpy(r, w, sizeof(w));
    }
}

int ora_last_tree_nodes(float *poles, float *locals, int n_nodes) {
    const int nn = (int)(g_last_poles.size() / 24);
    if (n_nodes > nn) return -1;
    if (poles) std::memcpy(poles, g_last_poles.data(), sizeof(float) * 24 * n_nodes);
    if (locals) std::memcpy(locals, g_last_locals.data(), sizeof(float) * 16 * n_nodes);
    return nn;
}

// density.metal:12-239
void ora_density(ora_state *st) {
    set_threads();
    const int n = st->n;
    *st->dt = (int32_t)(kDT0 * 1 / kDtMin1);  // Q11: thread 0 resets the global dt
#pragma omp parallel for schedule(dynamic, 64)
    for (int index = 0; index < n; ++index) {
        const int ind = (int)st->cell_index[index];
        if (!st->active[ind]) {
            float p, c;
            eos_lookup(st, st->material[ind], st->rho[ind], st->u[ind], p, c);
            st->pressure[ind] = p;
            st->sound_speed[ind] = c;
            continue;
        }
        const F3 pi = ld3(st->pos, ind);
        float hi = st->h[ind];
        int max_h = 0;  // Q7: integer
        float h2x4 = 4.f * hi * hi;
        float h1 = 1.f / hi;
        const float mi = st->mass[ind];
        float dens = 0.f;
        float eps = 1.f;
        int count = 0;
        int nn = 0;
        uint32_t nidx[kNeighbourCache];
        float nr[kNeighbourCache];
        while (eps > kDensityEta && count < kMaxNR) {
            dens = 0.f;
            if (hi < (float)max_h && nn < kNeighbourCache) {
                for (int q = 0; q < nn; ++q) {
                    float r = nr[q];
                    if (r > hi + hi) continue;
                    dens += kernel_w(r, h1) * st->mass[nidx[q]];
                }
            } else {
                CellBox b = cell_box(pi, hi);
                nn = 0;
                for (int x = b.lo[0]; x <= b.hi[0]; ++x)
                    for (int y = b.lo[1]; y <= b.hi[1]; ++y)
                        for (int z = b.lo[2]; z <= b.hi[2]; ++z) {
                            uint32_t ci = cell_index_of(x, y, z);
                            uint32_t s = st->cell_start[ci];
                            if (s == UINT_MAX) continue;
                            uint32_t e = st->cell_end[ci] + 1;
                            for (uint32_t k = s; k < e; ++k) {
                                uint32_t j = st->cell_index[k];
                                F3 xij = sub(ld3(st->pos, j), pi);
                                float r2 = len2(xij);
                                if (r2 > h2x4) continue;
                                float r = std::sqrt(r2);
                                if (nn < kNeighbourCache) {
                                    nidx[nn] = j;
                                    nr[nn] = r;
                                    nn++;
                                }
                                dens += kernel_w(r, h1) * st->mass[j];
                            }
                        }
            }
            float nh = fminf_(kResolutionEta * std::pow(mi / dens, 1.f / 3), kMaxH);
            nh = 0.5f * (hi + nh);
            eps = std::fabs(nh - hi) / hi;
            if (eps > kDensityEta) {
                max_h = (int)fmaxf_((float)max_h, hi);
                hi = nh;
                h1 = 1.f / hi;
                h2x4 = 4.f * hi * hi;
                count++;
            }
        }
        float dens_h = 0.f, vdiv = 0.f;
        F3 curl = {0.f, 0.f, 0.f};
        const F3 vi = ld3(st->vel, ind);
        auto grad_terms = [&](uint32_t j, float r, F3 xij) {
            float mj = st->mass[j];
            dens_h += mj * kernel_dwdh(r, h1);
            if (r > 1e-12f) {
                float r1 = 1.f / r;
                F3 vij = sub(ld3(st->vel, j), vi);
                F3 g = kernel_gradw(xij, r, r1, h1);
                vdiv += mj * dot3(vij, g);
                F3 cr = {vij.y * g.z - vij.z * g.y, vij.z * g.x - vij.x * g.z, vij.x * g.y - vij.y * g.x};
                curl.x += mj * cr.x;
                curl.y += mj * cr.y;
                curl.z += mj * cr.z;
            }
        };
        if (nn < kNeighbourCache) {
            for (int q = 0; q < nn; ++q) {
                uint32_t j = nidx[q];
                float r = nr[q];
                if (r > hi + hi) continue;
                grad_terms(j, r, sub(ld3(st->pos, j), pi));
            }
        } else {
            // Q7: overflow path adds to the converged density again
            CellBox b = cell_box(pi, hi);
            for (int x = b.lo[0]; x <= b.hi[0]; ++x)
                for (int y = b.lo[1]; y <= b.hi[1]; ++y)
                    for (int z = b.lo[2]; z <= b.hi[2]; ++z) {
                        uint32_t ci = cell_index_of(x, y, z);
                        uint32_t s = st->cell_start[ci];
                        if (s == UINT_MAX) continue;
                        uint32_t e = st->cell_end[ci] + 1;
                        for (uint32_t k = s; k < e; ++k) {
                            uint32_t j = st->cell_index[k];
                            F3 xij = sub(ld3(st->pos, j), pi);
                            float r2 = len2(xij);
                            if (r2 > h2x4) continue;
                            float r = std::sqrt(r2);
                            dens += kernel_w(r, h1) * st->mass[j];
                            grad_terms(j, r, xij);
                        }
                    }
        }
        vdiv = std::fabs(vdiv) / dens;
        float acurl = std::sqrt(len2(curl)) / dens;
        st->h[ind] = hi;
        st->rho[ind] = dens;
        st->grad_term[ind] = 1.f / (1.f + (hi / (3.f * dens)) * dens_h);
        float p, c;
        eos_lookup(st, st->material[ind], dens, st->u[ind], p, c);
        st->pressure[ind] = p;
        st->sound_speed[ind] = c;
        st->balsara[ind] = vdiv / (vdiv + acurl + 1e-4f * (c / hi));
    }
}

// accelerations.metal:12-141
void ora_acceleration(ora_state *st) {
    set_threads();
    const int n = st->n;
    int dt_min = *st->dt;
    const int gt = *st->global_time;
#pragma omp parallel for schedule(dynamic, 64) reduction(min : dt_min)
    for (int index = 0; index < n; ++index) {
        const int ind = (int)st->cell_index[index];
        if (!st->active[ind]) continue;
        const float fi = st->grad_term[ind], Pi = st->pressure[ind], rhoi = st->rho[ind];
        const float facti = (fi * Pi / (rhoi * rhoi));
        const F3 xi = ld3(st->pos, ind), vi = ld3(st->vel, ind);
        const float ci = st->sound_speed[ind], hi = st->h[ind], Bi = st->balsara[ind];
        const float hi1 = 1.f / hi;
        const float hi2x4 = hi * hi * 4.f;
        F3 dv = {0.f, 0.f, 0.f};
        float du = 0.f, dh = 0.f;
        CellBox b = cell_box(xi, fminf_(hi, kMaxH));
        float vsig_i = 1e-12f;
        for (int x = b.lo[0]; x <= b.hi[0]; ++x)
            for (int y = b.lo[1]; y <= b.hi[1]; ++y)
                for (int z = b.lo[2]; z <= b.hi[2]; ++z) {
                    uint32_t cidx = cell_index_of(x, y, z);
                    uint32_t s = st->cell_start[cidx];
                    if (s == UINT_MAX) continue;
                    uint32_t e = st->cell_end[cidx] + 1;
                    for (uint32_t k = s; k < e; ++k) {
                        const uint32_t j = st->cell_index[k];
                        F3 xij = sub(xi, ld3(st->pos, j));
                        float r2 = len2(xij);
                        float hj = st->h[j];
                        float hj2x4 = hj * hj * 4.f;
                        if ((r2 > hi2x4 && r2 > hj2x4) || r2 < 1e-12f) continue;  // Q8
                        float r = std::sqrt(r2);
                        float r1 = 1.f / r;
                        float mj = st->mass[j];
                        float fj = st->grad_term[j], Pj = st->pressure[j], rhoj = st->rho[j];
                        float factj = (fj * Pj / (rhoj * rhoj));
                        F3 vj = ld3(st->vel, j);
                        float cj = st->sound_speed[j];
                        float hj1 = 1.f / hj;
                        F3 vij = sub(vi, vj);
                        float rhoij = 0.5f * (rhoi + rhoj);
                        const float vdr = dot3(vij, xij);
                        float mu = vdr < 0.f ? vdr * r1 : 0.f;
                        float vsig = ci + cj - 3.f * mu;
                        vsig_i = fmaxf_(vsig, vsig_i);
                        float Bj = st->balsara[j];
                        float Bij = 0.5f * (Bi + Bj);
                        float nu = -0.5f * kViscosityAlpha * Bij * mu * vsig / rhoij;
                        F3 gi = kernel_gradw(xij, r, r1, hi1);
                        F3 gj = kernel_gradw(xij, r, r1, hj1);
                        F3 gij = {0.5f * (gi.x + gj.x), 0.5f * (gi.y + gj.y), 0.5f * (gi.z + gj.z)};
                        F3 ti = {facti * gi.x, facti * gi.y, facti * gi.z};
                        F3 tj = {factj * gj.x, factj * gj.y, factj * gj.z};
                        F3 tv = {nu * gij.x, nu * gij.y, nu * gij.z};
                        dv.x -= mj * (ti.x + tj.x + tv.x);
                        dv.y -= mj * (ti.y + tj.y + tv.y);
                        dv.z -= mj * (ti.z + tj.z + tv.z);
                        du += mj * (facti * dot3(vij, gi) + 0.5f * nu * dot3(vij, gij));
                        dh += (mj / rhoj) * dot3(vij, gi);
                    }
                }
        F3 a = ld3(st->acc, ind);
        st3(st->acc, ind, {a.x + dv.x, a.y + dv.y, a.z + dv.z});
        st->du[ind] = du;
        st->dhdt[ind] = dh;
        float goal = 2.0f * kCFL * kGamma * hi / vsig_i;
        int r = 0;
        float cand = kDT0;
        while (cand > goal && r < kRMax) {
            cand *= 0.5f;
            r++;
        }
        int idt = (int)std::ceil(1 / kDtMin1 * cand);
        st->next_active_time[ind] = gt + idt;
        dt_min = std::min(dt_min, idt);
    }
    *st->dt = dt_min;
}

// step.metal:12-46
void ora_step(ora_state *st) {
    set_threads();
    const int n = st->n;
    const float dt = kDtMin1 * (float)(*st->dt);
    *st->global_time += *st->dt;
#pragma omp parallel for
    for (int i = 0; i < n; ++i) {
        F3 v = ld3(st->vel, i);
        const F3 a = ld3(st->acc, i);
        float hi = st->h[i];
        float h1 = 1.f / hi;
        float dh = st->dhdt[i];
        st->h[i] = fminf_(hi * std::exp(h1 * dh * dt), kMaxH);
        st->rho[i] *= std::exp(-3.f * h1 * dh * dt);
        st3(st->vel, i, {v.x + dt * a.x, v.y + dt * a.y, v.z + dt * a.z});
        st->u[i] += dt * st->du[i];
        F3 x = ld3(st->pos, i);
        st3(st->pos, i,
            {x.x + (dt * v.x + 0.5f * a.x * dt * dt), x.y + (dt * v.y + 0.5f * a.y * dt * dt),
             x.z + (dt * v.z + 0.5f * a.z * dt * dt)});
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Octree builders.
// ---------------------------------------------------------------------------
struct ora_tree {
    std::vector<int32_t> data;
    std::vector<std::vector<int32_t>> levels;
    int32_t nodes = 0;
};

namespace {

// octree.cpp:14-109: split at the arithmetic mean of the subset (sequential
// float sum, then divide by the count), octant bit x=1, y=2, z=4 for "greater
// than the mean"; leaf if count <= max_leaf or level == max_depth.
int build_mean(const float *pos, const std::vector<int> &subset, int level, int max_leaf, int max_depth,
               ora_tree &t) {
    if ((int)subset.size() <= max_leaf || level == max_depth) {
        int start = (int)t.data.size();
        if (level >= (int)t.levels.size()) t.levels.resize(level + 1);
        t.levels[level].push_back(start);
        t.data.push_back((int)subset.size());
        t.data.push_back(t.nodes++);
        for (int p : subset) t.data.push_back(p);
        return start;
    }
    int start = (int)t.data.size();
    for (int i = 0; i < 10; ++i) t.data.push_back(-1);
    t.data[start] = 0;
    t.data[start + 1] = t.nodes++;
    if (level >= (int)t.levels.size()) t.levels.resize(level + 1);
    t.levels[level].push_back(start);
    float cx = 0.f, cy = 0.f, cz = 0.f;
    for (int p : subset) {
        cx += pos[3 * p];
        cy += pos[3 * p + 1];
        cz += pos[3 * p + 2];
    }
    const float cnt = (float)subset.size();
    cx /= cnt;
    cy /= cnt;
    cz /= cnt;
    std::vector<std::vector<int>> child(8);
    for (int p : subset) {
        int o = 0;
        o |= (pos[3 * p] > cx) ? 1 : 0;
        o |= (pos[3 * p + 1] > cy) ? 2 : 0;
        o |= (pos[3 * p + 2] > cz) ? 4 : 0;
        child[o].push_back(p);
    }
    for (int c = 0; c < 8; ++c) {
        int ci = -1;
        if (!child[c].empty()) ci = build_mean(pos, child[c], level + 1, max_leaf, max_depth, t);
        t.data[start + 2 + c] = ci;
    }
    return start;
}

// The GPU builder's tree: a Morton octree over the bounding cube.  Keys of
// 3*max_depth bits (x on bit 0 of each triplet, like morton3D), particles
// stable-sorted by key, children are the non-empty octants of the next key
// triplet, leaf if count <= max_leaf or level == max_depth.  Flattened in the
// reference format, preorder, so the same up/down passes consume it.
struct MortonBuild {
    const std::vector<uint64_t> &key;
    const std::vector<int> &order;
    int max_leaf, depth;
    ora_tree &t;
    int build(int s, int e, int level) {
        int n = e - s;
        if (level >= (int)t.levels.size()) t.levels.resize(level + 1);
        int start = (int)t.data.size();
        t.levels[level].push_back(start);
        if (n <= max_leaf || level == depth) {
            t.data.push_back(n);
            t.data.push_back(t.nodes++);
            for (int i = s; i < e; ++i) t.data.push_back(order[i]);
            return start;
        }
        for (int i = 0; i < 10; ++i) t.data.push_back(-1);
        t.data[start] = 0;
        t.data[start + 1] = t.nodes++;
        const int shift = 3 * (depth - level - 1);
        int i = s;
        while (i < e) {
            int oct = (int)((key[i] >> shift) & 7u);
            int j = i;
            while (j < e && (int)((key[j] >> shift) & 7u) == oct) ++j;
            int ci = build(i, j, level + 1);
            t.data[start + 2 + oct] = ci;
            i = j;
        }
        return start;
    }
};

}  // namespace

extern "C" {

ora_tree *ora_tree_build_reference(int n, const float *pos3, int max_leaf, int max_depth) {
    ora_tree *t = new ora_tree();
    if (n <= 0) return t;
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    build_mean(pos3, all, 0, max_leaf, max_depth, *t);
    return t;
}

ora_tree *ora_tree_build_morton(int n, const float *pos3, int max_leaf, int max_depth) {
    ora_tree *t = new ora_tree();
    if (n <= 0) return t;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], pos3[3 * i + a]);
            hi[a] = std::max(hi[a], pos3[3 * i + a]);
        }
    float span = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    if (!(span > 0.f)) span = 1.f;
    const int cells = 1 << max_depth;
    const float scale = (float)cells / span;
    std::vector<uint64_t> key(n);
    for (int i = 0; i < n; ++i) {
        uint64_t k = 0;
        for (int a = 0; a < 3; ++a) {
            float f = (pos3[3 * i + a] - lo[a]) * scale;
            int q = (int)f;
            q = std::min(std::max(q, 0), cells - 1);
            for (int b = 0; b < max_depth; ++b) k |= (uint64_t)((q >> b) & 1) << (3 * b + a);
        }
        key[i] = k;
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
    std::vector<uint64_t> skey(n);
    for (int i = 0; i < n; ++i) skey[i] = key[order[i]];
    MortonBuild mb{skey, order, max_leaf, max_depth, *t};
    mb.build(0, n, 0);
    return t;
}

void ora_tree_sizes(const ora_tree *t, int32_t *tree_len, int32_t *n_levels, int32_t *n_nodes) {
    *tree_len = (int32_t)t->data.size();
    *n_levels = (int32_t)t->levels.size();
    *n_nodes = t->nodes;
}

void ora_tree_export(const ora_tree *t, int32_t *tree, int32_t *level_offsets, int32_t *level_nodes) {
    std::memcpy(tree, t->data.data(), sizeof(int32_t) * t->data.size());
    int32_t off = 0;
    for (size_t l = 0; l < t->levels.size(); ++l) {
        level_offsets[l] = off;
        std::memcpy(level_nodes + off, t->levels[l].data(), sizeof(int32_t) * t->levels[l].size());
        off += (int32_t)t->levels[l].size();
    }
    level_offsets[t->levels.size()] = off;
}

void ora_tree_free(ora_tree *t) { delete t; }

// ANEOS.cpp:21-175.  The resampled grid is row-major (rho rows, u columns),
// each entry (pressure * 1e-18, sound speed * 1e-6).  Q10 is reproduced: the
// upper-row u index advances under the lower row's loop bound and the two
// interpolation weights of each pair are swapped.  Where the reference would
// read past the end of the whole u table, the scan stops instead.
int ora_aneos_load(const char *path, int res, float *out) {
    std::ifstream in(path);
    if (!in.is_open()) return -1;
    std::string line;
    for (int i = 0; i < 13; ++i) std::getline(in, line);
    int nrho = 0, nt = 0;
    {
        std::getline(in, line);
        std::istringstream iss(line);
        iss >> nrho >> nt;
    }
    if (nrho < 2 || nt < 2) return -2;
    std::vector<float> rho_t(nrho), t_t(nt);
    {
        int count = 0;
        while (count < nrho && std::getline(in, line)) {
            std::istringstream iss(line);
            float v;
            while (count < nrho && (iss >> v)) rho_t[count++] = v;
        }
    }
    {
        int count = 0;
        while (count < nt && std::getline(in, line)) {
            std::istringstream iss(line);
            float v;
            while (count < nt && (iss >> v)) t_t[count++] = v;
        }
    }
    std::vector<float> ut((size_t)nrho * nt), pt((size_t)nrho * nt), ct((size_t)nrho * nt);
    {
        int ri = 0, ti = 0;
        while (ti < nt && std::getline(in, line)) {
            std::istringstream iss(line);
            float u = 0.f, p = 0.f, c = 0.f;
            iss >> u;
            iss >> p;
            iss >> c;
            size_t k = (size_t)ri * nt + ti;
            ut[k] = u;
            pt[k] = p * std::pow(10.f, -18.f);
            ct[k] = c * std::pow(10.f, -6.f);
            if (++ri == nrho) {
                ri = 0;
                ++ti;
            }
        }
        if (ti < nt) return -2;
    }
    const float min_rho = (float)(1e-6 * 1e+6), max_rho = (float)(1.0 * 1e+6);
    const float min_u = (float)(1e-10 * 1e+12), max_u = (float)(1.0 * 1e+12);
    std::vector<float> grid_rho(res), grid_u(res);
    for (int i = 0; i < res; ++i) {
        grid_rho[i] = min_rho * std::pow((max_rho / min_rho), (float)i / res);
        grid_u[i] = min_u * std::pow((max_u / min_u), (float)i / res);
    }
    const size_t total = (size_t)nrho * nt;
    auto U = [&](int r, int t) -> float { return ut[(size_t)r * nt + t]; };
    int rti = 0;
    for (int ri = 0; ri < res; ++ri) {
        float rho = grid_rho[ri];
        while (rho > rho_t[rti + 1] && rti < nrho - 2) rti++;
        float rl = (rho - rho_t[rti]) / (rho_t[rti + 1] - rho_t[rti]);
        float rh = 1.f - rl;
        int ul = 0, uh = 0;
        for (int ui = 0; ui < res; ++ui) {
            float u = grid_u[ui];
            while (u > U(rti, ul + 1) && ul < nt - 2) ul++;
            while (ul < nt - 2 && (size_t)(rti + 1) * nt + uh + 1 < total &&
                   u > ut[(size_t)(rti + 1) * nt + uh + 1])
                uh++;
            const size_t kl0 = (size_t)rti * nt + ul, kl1 = kl0 + 1;
            const size_t kh0 = (size_t)(rti + 1) * nt + uh, kh1 = kh0 + 1;
            float ull = (u - ut[kl0]) / (ut[kl1] - ut[kl0]);
            float ulh = (u - ut[kh0]) / (ut[kh1] - ut[kh0]);
            float uhl = 1.f - ull;
            float uhh = 1.f - ulh;
            float *o = out + 2 * ((size_t)ri * res + ui);
            o[0] = rl * (pt[kl0] * ull + pt[kl1] * uhl) + rh * (pt[kh0] * ulh + pt[kh1] * uhh);
            o[1] = rl * (ct[kl0] * ull + ct[kl1] * uhl) + rh * (ct[kh0] * ulh + ct[kh1] * uhh);
        }
    }
    return 0;
}

// FP64 direct-sum gravity (no reference counterpart): the accuracy reference
// of the gravity forms.  Cubic-spline softened kernel with its exact
// coefficients (Price & Monaghan 2007 form; the reference's kernels.h:87-102
// truncates them), softening length GRAVITY_SMOOTHING_LENGTH = 0.04
// (Parameters.h), G = 6.67e-5 in code units (gravity/poles/poles.h:16).
void ora_gravity_direct_f64(int n, const float *pos3, const float *mass, const int32_t *targets, int nt,
                            double *out) {
    set_threads();
    const double G = (double)6.67e-5f, h = (double)0.04f, h1 = 1.0 / h;
#pragma omp parallel for schedule(dynamic, 4)
    for (int t = 0; t < nt; ++t) {
        const int i = targets[t];
        const double xi = pos3[3 * i], yi = pos3[3 * i + 1], zi = pos3[3 * i + 2];
        double ax = 0.0, ay = 0.0, az = 0.0, ph = 0.0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const double rx = xi - pos3[3 * j], ry = yi - pos3[3 * j + 1], rz = zi - pos3[3 * j + 2];
            const double r2 = rx * rx + ry * ry + rz * rz;
            if (r2 == 0.0) continue;
            const double r = std::sqrt(r2), q = r * h1;
            double fr, pot;
            if (q >= 2.0) {
                fr = 1.0 / r2;
                pot = -1.0 / r;
            } else if (q > 1.0) {
                const double q2 = q * q;
                fr = h1 * h1 * ((8.0 / 3.0) * q - 3.0 * q2 + 1.2 * q2 * q - q2 * q2 / 6.0 - 1.0 / (15.0 * q2));
                pot = h1 * ((4.0 / 3.0) * q2 - q2 * q + 0.3 * q2 * q2 - q2 * q2 * q / 30.0 - 1.6 + 1.0 / (15.0 * q));
            } else {
                const double q2 = q * q;
                fr = h1 * h1 * ((4.0 / 3.0) * q - 1.2 * q2 * q + 0.5 * q2 * q2);
                pot = h1 * ((2.0 / 3.0) * q2 - 0.3 * q2 * q2 + 0.1 * q2 * q2 * q - 1.4);
            }
            const double m = mass[j];
            const double s = -m * fr / r;
            ax += s * rx;
            ay += s * ry;
            az += s * rz;
            ph += m * pot;
        }
        out[4 * (size_t)t + 0] = G * ax;
        out[4 * (size_t)t + 1] = G * ay;
        out[4 * (size_t)t + 2] = G * az;
        out[4 * (size_t)t + 3] = G * ph;
    }
}

}  // extern "C"

// fp64.cpp -- an all-FP64 run of the SPH + gravity step, for stating the
// mixed-precision form's error against it.
//
// TEST INFRASTRUCTURE ONLY (built into liboracle.so beside oracle.cpp; only
// tests/ use it).  It is the reference's step (Headless.cpp:43-51) with every
// quantity in double and gravity summed directly:
//   gravity      the FP64 direct sum with the exact cubic-spline softening
//                (the accuracy target of the opening-angle form; the
//                reference's own FMM is not what an FP64 run is compared to);
//   density      density.metal:12-239: the damped h iteration from the
//                particle's h to |dh|/h <= DENSITY_ETA, the gradient sweep,
//                Balsara switch, EOS from the float tables by bilinear
//                interpolation evaluated in double;
//   acceleration accelerations.metal:12-141, including which pairs count: a
//                pair is seen from i when j's cell lies in i's box of radius
//                2 min(h_i, MAX_H) and r <= 2 h_i or r <= 2 h_j (Q8);
//                CFL timesteps quantised to ticks as the reference does;
//   step         step.metal:12-46 with the global time in ticks and seconds.
// The neighbour search uses the reference's cell grid (CELL_WIDTH) on double
// positions, sorted by unwrapped cell so no two regions alias.
#include <omp.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <vector>

#include "oracle.h"

namespace {

constexpr double kCellW = 0.18;
constexpr double kEta = 0.005;
constexpr int kMaxNRd = 50;
constexpr int kNNCache = 128;
constexpr double kResEta = 1.2348;
constexpr double kMaxHd = 1.0;
constexpr double kAlpha = 1.5;
constexpr double kCFLd = 0.2;
constexpr double kGammaD = 1.825742;
constexpr double kDT0d = 32.0;
constexpr int kRMaxD = 16;
constexpr double kTick = 32.0 / 65536.0;
constexpr double kPi1d = 1.0 / 3.14159265358979323846;
constexpr double kG = 6.67e-5;
constexpr double kSoft = 0.04;
constexpr double kMinU = 1e-10, kMinRho = 1e-6;

double w_kernel(double r, double h1) {
    const double q = r * h1;
    if (q > 2.0) return 0.0;
    const double fac = kPi1d * h1 * h1 * h1;
    if (q > 1.0) {
        const double t = 2.0 - q;
        return fac * 0.25 * t * t * t;
    }
    return fac * (1.0 - 1.5 * q * q * (1.0 - 0.5 * q));
}
double gradw_scale(double r, double h1) {  // gradW = s * x_ij / r
    const double q = r * h1;
    if (q > 2.0 || q < 1e-12) return 0.0;
    const double fac = kPi1d * h1 * h1 * h1 * h1;
    if (q > 1.0) {
        const double t = 2.0 - q;
        return -0.75 * fac * t * t;
    }
    return 3.0 * fac * (0.75 * q - 1.0) * q;
}
double dwdh(double r, double h1) {
    const double q = r * h1;
    if (q > 2.0) return 0.0;
    const double fac = -3.0 * kPi1d * h1 * h1 * h1 * h1;
    if (q > 1.0) return fac * (2.0 - 4.0 * q + 2.5 * q * q - 0.5 * q * q * q);
    return fac * (1.0 + 0.5 * (3.0 * q - 5.0) * q * q);
}

void eos(const ora_f64 *st, int mat, double rho, double u, double &p, double &c) {
    double uc = std::log(u / kMinU) / std::log(1.0 / kMinU);
    double rc = std::log(rho / kMinRho) / std::log(1.0 / kMinRho);
    uc = std::min(std::max(uc, 0.0), 1.0);
    rc = std::min(std::max(rc, 0.0), 1.0);
    const float *tab = ((float)mat == 400.f) ? st->eos_forsterite : st->eos_fe;
    const int res = st->eos_res;
    const double x = uc * res - 0.5, y = rc * res - 0.5;
    const double xf = std::floor(x), yf = std::floor(y), fx = x - xf, fy = y - yf;
    int x0 = (int)xf, y0 = (int)yf, x1 = x0 + 1, y1 = y0 + 1;
    x0 = std::min(std::max(x0, 0), res - 1);
    x1 = std::min(std::max(x1, 0), res - 1);
    y0 = std::min(std::max(y0, 0), res - 1);
    y1 = std::min(std::max(y1, 0), res - 1);
    const float *t00 = tab + 2 * ((size_t)y0 * res + x0), *t10 = tab + 2 * ((size_t)y0 * res + x1);
    const float *t01 = tab + 2 * ((size_t)y1 * res + x0), *t11 = tab + 2 * ((size_t)y1 * res + x1);
    const double gx = 1.0 - fx, gy = 1.0 - fy;
    p = (t00[0] * gx + t10[0] * fx) * gy + (t01[0] * gx + t11[0] * fx) * fy;
    c = (t00[1] * gx + t10[1] * fx) * gy + (t01[1] * gx + t11[1] * fx) * fy;
}

// Particles sorted by unwrapped cell (x, y, z), with the z-row lookup.
struct Grid {
    std::vector<int64_t> key;  // sorted keys
    std::vector<int> idx;      // particle of each sorted slot
    static int64_t pack(int64_t x, int64_t y, int64_t z) {
        const int64_t o = 1 << 20;
        return ((x + o) << 42) | ((y + o) << 21) | (z + o);
    }
    void build(int n, const double *pos) {
        std::vector<std::pair<int64_t, int>> kv(n);
        for (int i = 0; i < n; ++i)
            kv[i] = {pack((int64_t)std::floor(pos[3 * i] / kCellW), (int64_t)std::floor(pos[3 * i + 1] / kCellW),
                          (int64_t)std::floor(pos[3 * i + 2] / kCellW)),
                     i};
        std::sort(kv.begin(), kv.end());
        key.resize(n);
        idx.resize(n);
        for (int i = 0; i < n; ++i) {
            key[i] = kv[i].first;
            idx[i] = kv[i].second;
        }
    }
    // slots of the cells (x, y, z0 .. z1)
    std::pair<int, int> row(int64_t x, int64_t y, int64_t z0, int64_t z1) const {
        const auto a = std::lower_bound(key.begin(), key.end(), pack(x, y, z0));
        const auto b = std::upper_bound(key.begin(), key.end(), pack(x, y, z1));
        return {(int)(a - key.begin()), (int)(b - key.begin())};
    }
};

struct Box {
    int64_t lo[3], hi[3];
};
Box box_of(const double *p, double h) {
    Box b;
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = (int64_t)std::floor((p[k] - 2.0 * h) / kCellW);
        b.hi[k] = (int64_t)std::floor((p[k] + 2.0 * h) / kCellW);
    }
    return b;
}
template <class F>
void for_box(const Grid &g, const Box &b, F &&f) {
    for (int64_t x = b.lo[0]; x <= b.hi[0]; ++x)
        for (int64_t y = b.lo[1]; y <= b.hi[1]; ++y) {
            const auto r = g.row(x, y, b.lo[2], b.hi[2]);
            for (int s = r.first; s < r.second; ++s) f(g.idx[s]);
        }
}

void gravity(ora_f64 *st) {
    const int n = st->n;
    const double h1 = 1.0 / kSoft;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        const double *xi = st->pos + 3 * (size_t)i;
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const double rx = xi[0] - st->pos[3 * j], ry = xi[1] - st->pos[3 * j + 1], rz = xi[2] - st->pos[3 * j + 2];
            const double r2 = rx * rx + ry * ry + rz * rz;
            if (r2 == 0.0) continue;
            const double r = std::sqrt(r2), q = r * h1;
            double fr;
            if (q >= 2.0) {
                fr = 1.0 / r2;
            } else if (q > 1.0) {
                const double q2 = q * q;
                fr = h1 * h1 * ((8.0 / 3.0) * q - 3.0 * q2 + 1.2 * q2 * q - q2 * q2 / 6.0 - 1.0 / (15.0 * q2));
            } else {
                const double q2 = q * q;
                fr = h1 * h1 * ((4.0 / 3.0) * q - 1.2 * q2 * q + 0.5 * q2 * q2);
            }
            const double s = -st->mass[j] * fr / r;
            ax += s * rx;
            ay += s * ry;
            az += s * rz;
        }
        st->acc[3 * i] = kG * ax;
        st->acc[3 * i + 1] = kG * ay;
        st->acc[3 * i + 2] = kG * az;
    }
}

void density(ora_f64 *st, const Grid &g) {
    const int n = st->n;
#pragma omp parallel for schedule(dynamic, 32)
    for (int i = 0; i < n; ++i) {
        const double *pi = st->pos + 3 * (size_t)i;
        const double mi = st->mass[i];
        double hi = st->h[i], dens = 0.0, eps = 1.0, hs = hi;
        int count = 0, nn = 0;
        while (eps > kEta && count < kMaxNRd) {
            hs = hi;
            const double h1 = 1.0 / hi, h2x4 = 4.0 * hi * hi;
            dens = 0.0;
            int found = 0;
            for_box(g, box_of(pi, hi), [&](int j) {
                const double dx = st->pos[3 * j] - pi[0], dy = st->pos[3 * j + 1] - pi[1], dz = st->pos[3 * j + 2] - pi[2];
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > h2x4) return;
                ++found;
                dens += w_kernel(std::sqrt(r2), h1) * st->mass[j];
            });
            nn = std::min(found, kNNCache);
            double nh = std::min(kResEta * std::pow(mi / dens, 1.0 / 3.0), kMaxHd);
            nh = 0.5 * (hi + nh);
            eps = std::fabs(nh - hi) / hi;
            if (eps > kEta) {
                hi = nh;
                count++;
            }
        }
        // gradient sweep (density.metal:145-213): the last scan's neighbours
        // within 2h; past N_NEIGHBOURS_ESTIM a full scan that adds to the
        // density again (Q7)
        const bool cached = nn < kNNCache;
        const double gh = cached ? hs : hi, h1 = 1.0 / hi, h2 = 2.0 * hi;
        double dens_h = 0.0, vdiv = 0.0, cx = 0.0, cy = 0.0, cz = 0.0, pd = 0.0;
        const double *vi = st->vel + 3 * (size_t)i;
        for_box(g, box_of(pi, gh), [&](int j) {
            const double dx = st->pos[3 * j] - pi[0], dy = st->pos[3 * j + 1] - pi[1], dz = st->pos[3 * j + 2] - pi[2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > 4.0 * gh * gh) return;
            const double r = std::sqrt(r2);
            if (cached && r > h2) return;
            const double mj = st->mass[j];
            if (!cached) pd += w_kernel(r, h1) * mj;
            dens_h += mj * dwdh(r, h1);
            if (r > 1e-12) {
                const double vx = st->vel[3 * j] - vi[0], vy = st->vel[3 * j + 1] - vi[1], vz = st->vel[3 * j + 2] - vi[2];
                const double s = gradw_scale(r, h1) / r;
                const double gx = s * dx, gy = s * dy, gz = s * dz;
                vdiv += mj * (vx * gx + vy * gy + vz * gz);
                cx += mj * (vy * gz - vz * gy);
                cy += mj * (vz * gx - vx * gz);
                cz += mj * (vx * gy - vy * gx);
            }
        });
        dens += pd;
        vdiv = std::fabs(vdiv) / dens;
        const double acurl = std::sqrt(cx * cx + cy * cy + cz * cz) / dens;
        double p, c;
        eos(st, st->material[i], dens, st->u[i], p, c);
        st->h[i] = hi;
        st->rho[i] = dens;
        st->grad_term[i] = 1.0 / (1.0 + (hi / (3.0 * dens)) * dens_h);
        st->pressure[i] = p;
        st->sound_speed[i] = c;
        st->balsara[i] = vdiv / (vdiv + acurl + 1e-4 * (c / hi));
    }
}

void acceleration(ora_f64 *st, const Grid &g) {
    const int n = st->n;
    int dt_min = (int)(kDT0d / kTick);
    const int gt = *st->global_time;
#pragma omp parallel for schedule(dynamic, 32) reduction(min : dt_min)
    for (int i = 0; i < n; ++i) {
        const double *xi = st->pos + 3 * (size_t)i, *vi = st->vel + 3 * (size_t)i;
        const double hi = st->h[i], hi1 = 1.0 / hi, hi2x4 = 4.0 * hi * hi;
        const double rhoi = st->rho[i], facti = st->grad_term[i] * st->pressure[i] / (rhoi * rhoi);
        const double ci = st->sound_speed[i], Bi = st->balsara[i];
        double dvx = 0.0, dvy = 0.0, dvz = 0.0, du = 0.0, dh = 0.0, vsig_i = 1e-12;
        for_box(g, box_of(xi, std::min(hi, kMaxHd)), [&](int j) {
            const double dx = xi[0] - st->pos[3 * j], dy = xi[1] - st->pos[3 * j + 1], dz = xi[2] - st->pos[3 * j + 2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            const double hj = st->h[j];
            if ((r2 > hi2x4 && r2 > 4.0 * hj * hj) || r2 < 1e-12) return;
            const double r = std::sqrt(r2), r1 = 1.0 / r, hj1 = 1.0 / hj;
            const double rhoj = st->rho[j], factj = st->grad_term[j] * st->pressure[j] / (rhoj * rhoj);
            const double vx = vi[0] - st->vel[3 * j], vy = vi[1] - st->vel[3 * j + 1], vz = vi[2] - st->vel[3 * j + 2];
            const double rhoij = 0.5 * (rhoi + rhoj);
            const double vdr = vx * dx + vy * dy + vz * dz;
            const double mu = vdr < 0.0 ? vdr * r1 : 0.0;
            const double vsig = ci + st->sound_speed[j] - 3.0 * mu;
            vsig_i = std::max(vsig, vsig_i);
            const double Bij = 0.5 * (Bi + st->balsara[j]);
            const double nu = -0.5 * kAlpha * Bij * mu * vsig / rhoij;
            const double si = gradw_scale(r, hi1) * r1, sj = gradw_scale(r, hj1) * r1;
            const double gix = si * dx, giy = si * dy, giz = si * dz;
            const double gjx = sj * dx, gjy = sj * dy, gjz = sj * dz;
            const double gx = 0.5 * (gix + gjx), gy = 0.5 * (giy + gjy), gz = 0.5 * (giz + gjz);
            const double mj = st->mass[j];
            dvx -= mj * (facti * gix + factj * gjx + nu * gx);
            dvy -= mj * (facti * giy + factj * gjy + nu * gy);
            dvz -= mj * (facti * giz + factj * gjz + nu * gz);
            du += mj * (facti * (vx * gix + vy * giy + vz * giz) + 0.5 * nu * (vx * gx + vy * gy + vz * gz));
            dh += (mj / rhoj) * (vx * gix + vy * giy + vz * giz);
        });
        st->acc[3 * i] += dvx;
        st->acc[3 * i + 1] += dvy;
        st->acc[3 * i + 2] += dvz;
        st->du[i] = du;
        st->dhdt[i] = dh;
        const double goal = 2.0 * kCFLd * kGammaD * hi / vsig_i;
        int r = 0;
        double cand = kDT0d;
        while (cand > goal && r < kRMaxD) {
            cand *= 0.5;
            r++;
        }
        const int idt = (int)std::ceil(cand / kTick);
        st->next_active_time[i] = gt + idt;
        dt_min = std::min(dt_min, idt);
    }
    *st->dt = dt_min;
}

void step(ora_f64 *st) {
    const int n = st->n;
    const double dt = kTick * (double)(*st->dt);
    *st->global_time += *st->dt;
    *st->time_s += dt;
#pragma omp parallel for
    for (int i = 0; i < n; ++i) {
        const double hi = st->h[i], h1 = 1.0 / hi, dh = st->dhdt[i];
        st->h[i] = std::min(hi * std::exp(h1 * dh * dt), kMaxHd);
        st->rho[i] *= std::exp(-3.0 * h1 * dh * dt);
        for (int k = 0; k < 3; ++k) {
            const double v = st->vel[3 * i + k], a = st->acc[3 * i + k];
            st->vel[3 * i + k] = v + dt * a;
            st->pos[3 * i + k] += dt * v + 0.5 * a * dt * dt;
        }
        st->u[i] += dt * st->du[i];
    }
}

}  // namespace

extern "C" void ora_f64_steps(ora_f64 *st, int n_steps) {
    const int th = ora_get_threads();
    if (th > 0) omp_set_num_threads(th);
    Grid g;
    for (int s = 0; s < n_steps; ++s) {
        gravity(st);
        g.build(st->n, st->pos);
        density(st, g);
        acceleration(st, g);
        step(st);
    }
}

extern "C" void ora_f64_energy(const ora_f64 *st, double *out) {
    // kinetic, internal, potential (exact softening, FP64 pairs), total
    const int n = st->n;
    const double h1 = 1.0 / kSoft;
    double ek = 0.0, ei = 0.0, ep = 0.0;
#pragma omp parallel for reduction(+ : ek, ei, ep) schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        const double m = st->mass[i];
        const double *v = st->vel + 3 * (size_t)i;
        ek += 0.5 * m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        ei += m * st->u[i];
        double ph = 0.0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const double rx = st->pos[3 * i] - st->pos[3 * j], ry = st->pos[3 * i + 1] - st->pos[3 * j + 1],
                         rz = st->pos[3 * i + 2] - st->pos[3 * j + 2];
            const double r = std::sqrt(rx * rx + ry * ry + rz * rz), q = r * h1;
            double pot;
            if (q >= 2.0) {
                pot = -1.0 / r;
            } else if (q > 1.0) {
                const double q2 = q * q;
                pot = h1 * ((4.0 / 3.0) * q2 - q2 * q + 0.3 * q2 * q2 - q2 * q2 * q / 30.0 - 1.6 + 1.0 / (15.0 * q));
            } else {
                const double q2 = q * q;
                pot = h1 * ((2.0 / 3.0) * q2 - 0.3 * q2 * q2 + 0.1 * q2 * q2 * q - 1.4);
            }
            ph += st->mass[j] * pot;
        }
        ep += 0.5 * m * kG * ph;
    }
    out[0] = ek;
    out[1] = ei;
    out[2] = ep;
    out[3] = ek + ei + ep;
}

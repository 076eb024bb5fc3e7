// sph_api.cu -- the C ABI (include/sph.h): context lifetime, buffer transfer,
// host-built trees, the graph-captured step loop and the EOS table loader.
//
// Reference counterparts: Compute::Compute / buildBuffers / loadInitialConditions
// (SPH/Compute/Compute.cpp:22-132), Buffers.hpp:14-59 (staging copies),
// updateOctreeBuffer (Compute.cpp:456-508), ANEOS.cpp:21-175 (table loader),
// Headless::step (SPH/Rendering/Headless.cpp:37-55).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "sph_internal.h"

namespace sph {

namespace {
thread_local std::string g_error;

template <class T>
cudaError_t dmalloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void **)p, sizeof(T) * count);
}

__global__ void k_pack3(const float *__restrict__ src, float4 *__restrict__ dst, int n, int keep_w) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float w = keep_w ? dst[i].w : 0.f;
    dst[i] = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], w);
}
__global__ void k_unpack3(const float4 *__restrict__ src, float *__restrict__ dst, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = src[i];
    dst[3 * i] = v.x;
    dst[3 * i + 1] = v.y;
    dst[3 * i + 2] = v.z;
}
__global__ void k_set_w(const float *__restrict__ src, float4 *__restrict__ dst, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i].w = src[i];
}
__global__ void k_get_w(const float4 *__restrict__ src, float *__restrict__ dst, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i].w;
}
__global__ void k_pack3d(const double *__restrict__ src, double4 *__restrict__ dst64, float4 *__restrict__ dst,
                         int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = src[3 * i], y = src[3 * i + 1], z = src[3 * i + 2];
    dst64[i] = make_double4(x, y, z, 0.0);
    const float w = dst[i].w;
    dst[i] = make_float4((float)x, (float)y, (float)z, w);
}
__global__ void k_unpack3d(const double4 *__restrict__ src, double *__restrict__ dst, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 v = src[i];
    dst[3 * i] = v.x;
    dst[3 * i + 1] = v.y;
    dst[3 * i + 2] = v.z;
}
// FP32 FMA throughput probe: 8 independent FMA chains per thread.
__global__ void __launch_bounds__(256) k_fma_probe(int iters, float seed, float *sink) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + (float)(threadIdx.x + k);
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 1234.5678f) sink[blockIdx.x] = s;  // keeps the chains alive
}
__global__ void k_time_to64(const int32_t *globals, double *dglob) {
    dglob[0] = (double)kDtMin1 * (double)globals[0];
}
__global__ void k_split_cells(const uint2 *__restrict__ src, uint32_t *__restrict__ dst, uint32_t count, int which) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        dst[i] = which ? src[i].y : src[i].x;
}
}  // namespace

void set_error(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

sph_status cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return SPH_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA;
}

// ANEOS.cpp:21-175: parse the text table, resample on a log-uniform
// res x res (rho, u) grid.  Reproduces the reference's swapped interpolation
// weights and the upper-row u index that advances under the lower row's loop
// bound; where that index would leave the whole table, the scan stops.
static sph_status eos_resample_host(const char *path, int res, std::vector<float> &out) {
    std::ifstream in(path);
    if (!in.is_open()) {
        set_error("cannot open ANEOS table %s", path);
        return SPH_ERR_IO;
    }
    std::string line;
    for (int i = 0; i < 13; ++i) std::getline(in, line);
    int nrho = 0, nt = 0;
    std::getline(in, line);
    {
        std::istringstream iss(line);
        iss >> nrho >> nt;
    }
    if (nrho < 2 || nt < 2) {
        set_error("bad ANEOS table header in %s", path);
        return SPH_ERR_IO;
    }
    std::vector<float> rho_t(nrho), t_t(nt);
    for (int cnt = 0; cnt < nrho && std::getline(in, line);) {
        std::istringstream iss(line);
        float v;
        while (cnt < nrho && (iss >> v)) rho_t[cnt++] = v;
    }
    for (int cnt = 0; cnt < nt && std::getline(in, line);) {
        std::istringstream iss(line);
        float v;
        while (cnt < nt && (iss >> v)) t_t[cnt++] = v;
    }
    const size_t total = (size_t)nrho * nt;
    std::vector<float> ut(total), pt(total), ct(total);
    int ri = 0, ti = 0;
    while (ti < nt && std::getline(in, line)) {
        std::istringstream iss(line);
        float u = 0.f, p = 0.f, c = 0.f;
        iss >> u;
        iss >> p;
        iss >> c;
        const size_t k = (size_t)ri * nt + ti;
        ut[k] = u;
        pt[k] = p * std::pow(10.f, -18.f);
        ct[k] = c * std::pow(10.f, -6.f);
        if (++ri == nrho) {
            ri = 0;
            ++ti;
        }
    }
    if (ti < nt) {
        set_error("not enough pressure data in %s", path);
        return SPH_ERR_IO;
    }
    const float min_rho = (float)(1e-6 * 1e+6), max_rho = (float)(1.0 * 1e+6);
    const float min_u = (float)(1e-10 * 1e+12), max_u = (float)(1.0 * 1e+12);
    std::vector<float> grid_rho(res), grid_u(res);
    for (int i = 0; i < res; ++i) {
        grid_rho[i] = min_rho * std::pow((max_rho / min_rho), (float)i / res);
        grid_u[i] = min_u * std::pow((max_u / min_u), (float)i / res);
    }
    out.assign((size_t)2 * res * res, 0.f);
    int rti = 0;
    for (int r = 0; r < res; ++r) {
        const float rho = grid_rho[r];
        while (rho > rho_t[rti + 1] && rti < nrho - 2) rti++;
        const float rl = (rho - rho_t[rti]) / (rho_t[rti + 1] - rho_t[rti]);
        const float rh = 1.f - rl;
        int ul = 0, uh = 0;
        for (int q = 0; q < res; ++q) {
            const float u = grid_u[q];
            while (u > ut[(size_t)rti * nt + ul + 1] && ul < nt - 2) ul++;
            while (ul < nt - 2 && (size_t)(rti + 1) * nt + uh + 1 < total && u > ut[(size_t)(rti + 1) * nt + uh + 1])
                uh++;
            const size_t kl0 = (size_t)rti * nt + ul, kl1 = kl0 + 1;
            const size_t kh0 = (size_t)(rti + 1) * nt + uh, kh1 = kh0 + 1;
            const float ull = (u - ut[kl0]) / (ut[kl1] - ut[kl0]);
            const float ulh = (u - ut[kh0]) / (ut[kh1] - ut[kh0]);
            const float uhl = 1.f - ull, uhh = 1.f - ulh;
            float *o = out.data() + 2 * ((size_t)r * res + q);
            o[0] = rl * (pt[kl0] * ull + pt[kl1] * uhl) + rh * (pt[kh0] * ulh + pt[kh1] * uhh);
            o[1] = rl * (ct[kl0] * ull + ct[kl1] * uhl) + rh * (ct[kh0] * ulh + ct[kh1] * uhh);
        }
    }
    return SPH_OK;
}

static void tree_storage_free(Tree &t) {
    cudaFree(t.tree);
    cudaFree(t.level_nodes);
    cudaFree(t.level_count);
    cudaFree(t.list_slot);
    cudaFree(t.parent_slot);
    cudaFree(t.poles);
    cudaFree(t.locals);
    cudaFree(t.lists[0]);
    cudaFree(t.lists[1]);
    cudaFree(t.meta);
    cudaFree(t.node_range);
    Tree fresh;
    fresh.list_cap = t.list_cap;
    t = fresh;
}

// Storage for a tree of at most node_cap nodes, tree_cap ints, max_levels
// levels of at most level_cap nodes and branch_cap branches each.
static sph_status tree_storage_alloc(Tree &t, int64_t node_cap, int64_t tree_cap, int max_levels, int64_t level_cap,
                                     int64_t branch_cap, int list_cap) {
    tree_storage_free(t);
    t.node_cap = node_cap;
    t.tree_cap = tree_cap;
    t.max_levels = max_levels;
    t.level_cap = level_cap;
    t.branch_cap = branch_cap;
    t.list_cap = list_cap;
    cudaError_t e = dmalloc(&t.tree, tree_cap);
    if (e == cudaSuccess) e = dmalloc(&t.level_nodes, (size_t)max_levels * level_cap);
    if (e == cudaSuccess) e = dmalloc(&t.level_count, 16);
    if (e == cudaSuccess) e = dmalloc(&t.list_slot, node_cap);
    if (e == cudaSuccess) e = dmalloc(&t.parent_slot, node_cap);
    if (e == cudaSuccess) e = dmalloc(&t.poles, (size_t)node_cap * kPoleQ);
    if (e == cudaSuccess) e = dmalloc(&t.locals, (size_t)node_cap * kLocalQ);
    if (e == cudaSuccess) e = dmalloc(&t.lists[0], (size_t)branch_cap * list_cap + 2);
    if (e == cudaSuccess) e = dmalloc(&t.lists[1], (size_t)branch_cap * list_cap + 2);
    if (e == cudaSuccess) e = dmalloc(&t.meta, 4);
    if (e == cudaSuccess) e = dmalloc(&t.node_range, node_cap);
    if (e == cudaSuccess) e = cudaMemset(t.level_count, 0, sizeof(int32_t) * 16);
    if (e == cudaSuccess) e = cudaMemset(t.parent_slot, 0, sizeof(int32_t) * node_cap);
    return cuda_status(e, "tree storage");
}

// Capacity bounds for trees whose leaves hold <= leafcap particles or sit at
// depth `depth`: every branch holds more than leafcap particles, so a level
// has at most n / (leafcap + 1) branches.
void tree_bounds(int n, int leafcap, int depth, int64_t &nodes, int64_t &ints, int64_t &branches) {
    branches = (int64_t)n / (leafcap + 1) + 1;
    nodes = (int64_t)n + (int64_t)depth * branches + 1;
    ints = 10 * (int64_t)depth * branches + 3 * (int64_t)n + 16;
}

}  // namespace sph

using namespace sph;

extern "C" {

void sph_params_default(sph_params *p) {
    if (!p) return;
    p->max_children_in_leaf = 4;
    p->max_tree_depth = 7;
    p->max_unchecked_pointers = 1024;
    p->aneos_resolution = 2048;
    p->tree_source = SPH_TREE_GPU;
    p->forsterite_table = "ANEOS_forsterite_S19.txt";
    p->fe85si15_table = "ANEOS_Fe85Si15_S20.txt";
}

const char *sph_status_string(sph_status s) {
    switch (s) {
        case SPH_OK: return "ok";
        case SPH_ERR_INVALID_ARG: return "invalid argument";
        case SPH_ERR_OOM: return "out of device memory";
        case SPH_ERR_IO: return "i/o error";
        case SPH_ERR_CUDA: return "cuda error";
        case SPH_ERR_DEVICE_HEALTH: return "device health bit raised";
        case SPH_ERR_TIMEOUT: return "bounded device wait timed out";
        case SPH_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown";
}

const char *sph_last_error(void) { return g_error.c_str(); }

sph_status sph_eos_resample(const char *path, int32_t res, float *out) {
    if (!path || !out || res < 2) {
        set_error("sph_eos_resample: bad arguments");
        return SPH_ERR_INVALID_ARG;
    }
    std::vector<float> v;
    sph_status s = eos_resample_host(path, res, v);
    if (s != SPH_OK) return s;
    std::memcpy(out, v.data(), sizeof(float) * v.size());
    return SPH_OK;
}

int32_t sph_num_particles(const sph_ctx *ctx) { return ctx ? ctx->n : 0; }

sph_status sph_destroy(sph_ctx *ctx) {
    if (!ctx) return SPH_OK;
    cudaSetDevice(ctx->device);
    drop_graphs(ctx);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    void *bufs[] = {ctx->pos4, ctx->vel4, ctx->acc4, ctx->rho, ctx->u, ctx->P, ctx->h, ctx->f, ctx->c,
                    ctx->du, ctx->B, ctx->dhdt, ctx->gnorm, ctx->phi, ctx->mat, ctx->nat, ctx->active, ctx->globals,
                    ctx->health, ctx->cell_range, ctx->sp4, ctx->sv4, ctx->sA, ctx->sB, ctx->sC,
                    ctx->eos_forsterite, ctx->eos_fe, ctx->stage, ctx->snapshot, ctx->pos64, ctx->dglob,
                    ctx->diag, ctx->tiles, ctx->tile_ctr, ctx->deferred, ctx->units, ctx->coarse_flags};
    for (void *b : bufs) cudaFree(b);
    sort_free(ctx->cell_sort);
    hseed_free(ctx);
    tree_free(ctx);
    tree_storage_free(ctx->tree);
    delete ctx;
    return SPH_OK;
}

sph_status sph_create(const sph_params *params, const sph_ic *ic, sph_ctx **out) {
    if (!out || !ic || ic->n <= 0 || !ic->pos || !ic->vel || !ic->rho || !ic->u || !ic->mass || !ic->h ||
        !ic->material) {
        set_error("sph_create: missing initial conditions");
        return SPH_ERR_INVALID_ARG;
    }
    *out = nullptr;
    sph_params p;
    sph_params_default(&p);
    if (params) p = *params;
    if (p.max_children_in_leaf < 1 || p.max_tree_depth < 1 || p.max_tree_depth > 10 ||
        p.max_unchecked_pointers < 2 || p.aneos_resolution < 2 || !p.forsterite_table || !p.fe85si15_table ||
        (p.tree_source != SPH_TREE_GPU && p.tree_source != SPH_TREE_HOST)) {
        set_error("sph_create: invalid parameters");
        return SPH_ERR_INVALID_ARG;
    }
    for (int i = 0; i < 3 * ic->n; ++i)
        if (!std::isfinite(ic->pos[i]) || !std::isfinite(ic->vel[i])) {
            set_error("sph_create: non-finite position or velocity at particle %d", i / 3);
            return SPH_ERR_INVALID_ARG;
        }
    for (int i = 0; i < ic->n; ++i)
        if (!(ic->h[i] > 0.f) || !(ic->h[i] <= kMaxInitialH) || !(ic->mass[i] > 0.f) || !std::isfinite(ic->u[i]) ||
            !std::isfinite(ic->rho[i])) {
            set_error("sph_create: bad smoothing length, mass, density or energy at particle %d", i);
            return SPH_ERR_INVALID_ARG;
        }
    std::vector<float> tf, te;
    const int res = p.aneos_resolution;
    sph_status s = eos_resample_host(p.forsterite_table, res, tf);
    if (s != SPH_OK) return s;
    s = eos_resample_host(p.fe85si15_table, res, te);
    if (s != SPH_OK) return s;

    sph_ctx *ctx = new sph_ctx();
    ctx->n = ic->n;
    ctx->params = p;
    ctx->forsterite_path = p.forsterite_table;
    ctx->fe_path = p.fe85si15_table;
    ctx->params.forsterite_table = ctx->forsterite_path.c_str();
    ctx->params.fe85si15_table = ctx->fe_path.c_str();
    cudaGetDevice(&ctx->device);
    const int n = ic->n;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    chk(dmalloc(&ctx->pos4, n));
    chk(dmalloc(&ctx->vel4, n));
    chk(dmalloc(&ctx->acc4, n));
    for (float **fp : {&ctx->rho, &ctx->u, &ctx->P, &ctx->h, &ctx->f, &ctx->c, &ctx->du, &ctx->B, &ctx->dhdt,
                       &ctx->gnorm, &ctx->phi})
        chk(dmalloc(fp, n));
    chk(dmalloc(&ctx->mat, n));
    chk(dmalloc(&ctx->nat, n));
    chk(dmalloc(&ctx->active, n));
    chk(dmalloc(&ctx->globals, 4));
    chk(dmalloc(&ctx->health, 1));
    chk(dmalloc(&ctx->cell_range, (size_t)kNumCells));
    for (float4 **fp : {&ctx->sp4, &ctx->sv4, &ctx->sA, &ctx->sB, &ctx->sC}) chk(dmalloc(fp, n));    chk(dmalloc(&ctx->eos_forsterite, (size_t)res * res));
    chk(dmalloc(&ctx->eos_fe, (size_t)res * res));
    ctx->stage_bytes = std::max((size_t)kNumCells * sizeof(uint32_t), sizeof(double) * 3 * (size_t)n);
    chk(cudaMalloc(&ctx->stage, ctx->stage_bytes));
    chk(dmalloc(&ctx->snapshot, (size_t)kSnapshotRes * kSnapshotRes));
    chk(dmalloc(&ctx->dglob, 4));
    chk(dmalloc(&ctx->diag, (size_t)kDiagDoubles));
    chk(dmalloc(&ctx->tiles, (size_t)n));
    chk(dmalloc(&ctx->tile_ctr, 16));
    chk(dmalloc(&ctx->deferred, (size_t)n));
    chk(dmalloc(&ctx->units, (size_t)kNumUnits));
    chk(dmalloc(&ctx->coarse_flags, (size_t)kNumCoarseBlocks));
    if (e == cudaSuccess) e = cudaMemset(ctx->coarse_flags, 0, kNumCoarseBlocks);
    if (e != cudaSuccess) {
        s = cuda_status(e, "sph_create allocation");
        sph_destroy(ctx);
        return s;
    }
    s = sort_alloc(ctx->cell_sort, n);
    if (s != SPH_OK) {
        sph_destroy(ctx);
        return s;
    }
    int64_t nodes, ints, branches;
    tree_bounds(n, p.max_children_in_leaf, std::max(p.max_tree_depth, 7), nodes, ints, branches);
    ctx->tree.list_cap = p.max_unchecked_pointers;
    s = tree_storage_alloc(ctx->tree, nodes, ints, std::max(p.max_tree_depth, 7) + 1, n, branches,
                           p.max_unchecked_pointers);
    if (s != SPH_OK) {
        sph_destroy(ctx);
        return s;
    }
    // EOS tables and the derived lookup constants (density.metal:45-46)
    chk(cudaMemcpy(ctx->eos_forsterite, tf.data(), sizeof(float) * tf.size(), cudaMemcpyHostToDevice));
    chk(cudaMemcpy(ctx->eos_fe, te.data(), sizeof(float) * te.size(), cudaMemcpyHostToDevice));
    ctx->eos.forsterite = ctx->eos_forsterite;
    ctx->eos.fe = ctx->eos_fe;
    ctx->eos.res = res;
    ctx->eos.log_u_range = std::log(1.f / kAneosMinU);
    ctx->eos.log_rho_range = std::log(1.f / kAneosMinRho);
    // initial state (Compute.cpp:52-77)
    chk(cudaMemset(ctx->acc4, 0, sizeof(float4) * n));
    for (float *fp : {ctx->f, ctx->c, ctx->du, ctx->B, ctx->dhdt, ctx->gnorm, ctx->phi})
        chk(cudaMemset(fp, 0, sizeof(float) * n));
    chk(cudaMemset(ctx->active, 1, n));
    chk(cudaMemset(ctx->nat, 0, sizeof(int32_t) * n));
    chk(cudaMemset(ctx->globals, 0, sizeof(int32_t) * 4));
    chk(cudaMemset(ctx->dglob, 0, sizeof(double) * 4));
    chk(cudaMemset(ctx->health, 0, sizeof(uint32_t)));
    if (e != cudaSuccess) {
        s = cuda_status(e, "sph_create init");
        sph_destroy(ctx);
        return s;
    }
    const void *srcs[] = {ic->pos, ic->vel, ic->rho, ic->u, ic->mass, ic->h, ic->material};
    const sph_field fields[] = {SPH_FIELD_POS, SPH_FIELD_VEL, SPH_FIELD_RHO, SPH_FIELD_U,
                                SPH_FIELD_MASS, SPH_FIELD_H, SPH_FIELD_MATERIAL};
    for (int k = 0; k < 7 && s == SPH_OK; ++k)
        s = sph_upload(ctx, fields[k], srcs[k], (fields[k] <= SPH_FIELD_ACC) ? 3 * (size_t)n : (size_t)n);
    if (s == SPH_OK && ic->pressure) s = sph_upload(ctx, SPH_FIELD_PRESSURE, ic->pressure, n);
    else if (s == SPH_OK) chk(cudaMemset(ctx->P, 0, sizeof(float) * n));
    if (s == SPH_OK) {
        launch_init_cells(ctx, 0);
        s = cuda_status(cudaDeviceSynchronize(), "sph_create cells");
    }
    if (s == SPH_OK && p.tree_source == SPH_TREE_GPU) {
        s = tree_alloc(ctx);
        if (s == SPH_OK) s = launch_tree_build(ctx, 0);
        if (s == SPH_OK) s = cuda_status(cudaDeviceSynchronize(), "sph_create tree");
    }
    if (s != SPH_OK) {
        sph_destroy(ctx);
        return s;
    }
    *out = ctx;
    return SPH_OK;
}

sph_status sph_upload_async(sph_ctx *ctx, sph_field field, const void *host, size_t count, void *stream) {
    if (!ctx || !host) {
        set_error("sph_upload: null argument");
        return SPH_ERR_INVALID_ARG;
    }
    const int n = ctx->n;
    const size_t need3 = 3 * (size_t)n, need1 = (size_t)n;
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (n + 255) / 256;
    auto f1 = [&](void *dst, size_t elem) -> sph_status {
        if (count != need1) {
            set_error("sph_upload: field %d expects %zu elements, got %zu", (int)field, need1, count);
            return SPH_ERR_INVALID_ARG;
        }
        return cuda_status(cudaMemcpyAsync(dst, host, elem * count, cudaMemcpyHostToDevice, st), "sph_upload");
    };
    switch (field) {
        case SPH_FIELD_POS:
        case SPH_FIELD_VEL:
        case SPH_FIELD_ACC: {
            if (count != need3) {
                set_error("sph_upload: vector field expects %zu floats, got %zu", need3, count);
                return SPH_ERR_INVALID_ARG;
            }
            float4 *dst = field == SPH_FIELD_POS ? ctx->pos4 : field == SPH_FIELD_VEL ? ctx->vel4 : ctx->acc4;
            cudaError_t e = cudaMemcpyAsync(ctx->stage, host, sizeof(float) * count, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) {
                k_pack3<<<blocks, 256, 0, st>>>((const float *)ctx->stage, dst, n, field == SPH_FIELD_POS ? 1 : 0);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess && field == SPH_FIELD_POS && ctx->form.precision == SPH_PRECISION_MIXED)
                return launch_pos_to64(ctx, st);
            return cuda_status(e, "sph_upload");
        }
        case SPH_FIELD_POS64: {
            if (ctx->form.precision != SPH_PRECISION_MIXED || !ctx->pos64) {
                set_error("sph_upload: FP64 positions exist in the mixed-precision form only");
                return SPH_ERR_INVALID_ARG;
            }
            if (count != need3) {
                set_error("sph_upload: FP64 positions expect %zu doubles, got %zu", need3, count);
                return SPH_ERR_INVALID_ARG;
            }
            if (sizeof(double) * count > ctx->stage_bytes) {
                set_error("sph_upload: FP64 positions exceed the staging buffer");
                return SPH_ERR_INVALID_ARG;
            }
            cudaError_t e = cudaMemcpyAsync(ctx->stage, host, sizeof(double) * count, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) {
                k_pack3d<<<blocks, 256, 0, st>>>((const double *)ctx->stage, ctx->pos64, ctx->pos4, n);
                e = cudaGetLastError();
            }
            return cuda_status(e, "sph_upload");
        }
        case SPH_FIELD_MASS: {
            if (count != need1) {
                set_error("sph_upload: mass expects %zu floats", need1);
                return SPH_ERR_INVALID_ARG;
            }
            cudaError_t e = cudaMemcpyAsync(ctx->stage, host, sizeof(float) * count, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) {
                k_set_w<<<blocks, 256, 0, st>>>((const float *)ctx->stage, ctx->pos4, n);
                e = cudaGetLastError();
            }
            return cuda_status(e, "sph_upload");
        }
        case SPH_FIELD_RHO: return f1(ctx->rho, 4);
        case SPH_FIELD_U: return f1(ctx->u, 4);
        case SPH_FIELD_PRESSURE: return f1(ctx->P, 4);
        case SPH_FIELD_H: {
            // the density pass caps h at MAX_SMOOTHING_LENGTH after its first
            // sweep; a first sweep with h above kMaxInitialH would scan a cell
            // box wider than the 256-cell periodic grid
            const float *hv = (const float *)host;
            for (size_t i = 0; i < count; ++i)
                if (!(hv[i] > 0.f) || !(hv[i] <= kMaxInitialH)) {
                    set_error("sph_upload: smoothing length %g at %zu outside (0, 10]", (double)hv[i], i);
                    return SPH_ERR_INVALID_ARG;
                }
            return f1(ctx->h, 4);
        }
        case SPH_FIELD_GRAD_TERM: return f1(ctx->f, 4);
        case SPH_FIELD_SOUND_SPEED: return f1(ctx->c, 4);
        case SPH_FIELD_DU: return f1(ctx->du, 4);
        case SPH_FIELD_BALSARA: return f1(ctx->B, 4);
        case SPH_FIELD_DHDT: return f1(ctx->dhdt, 4);
        case SPH_FIELD_GRAV_NORM: return f1(ctx->gnorm, 4);
        case SPH_FIELD_MATERIAL: return f1(ctx->mat, 4);
        case SPH_FIELD_ACTIVE: return f1(ctx->active, 1);
        case SPH_FIELD_NEXT_ACTIVE: return f1(ctx->nat, 4);
        case SPH_FIELD_NEIGHBOURS: {
            sph_status s = hseed_alloc(ctx);
            if (s != SPH_OK) return s;
            return f1(ctx->hs.nn, 4);
        }
        case SPH_FIELD_GLOBAL_TIME:
        case SPH_FIELD_DT: {
            if (count != 1) {
                set_error("sph_upload: scalar field expects 1 element");
                return SPH_ERR_INVALID_ARG;
            }
            cudaError_t e = cudaMemcpyAsync(ctx->globals + (field == SPH_FIELD_DT ? 1 : 0), host, 4,
                                            cudaMemcpyHostToDevice, st);
            // the mixed form's FP64 time follows (ticks x 2^-11 s is exact in FP64)
            if (e == cudaSuccess && field == SPH_FIELD_GLOBAL_TIME && ctx->form.precision == SPH_PRECISION_MIXED) {
                k_time_to64<<<1, 1, 0, st>>>(ctx->globals, ctx->dglob);
                e = cudaGetLastError();
            }
            return cuda_status(e, "sph_upload");
        }
        default:
            set_error("sph_upload: field %d is read-only", (int)field);
            return SPH_ERR_INVALID_ARG;
    }
}

sph_status sph_upload(sph_ctx *ctx, sph_field field, const void *host, size_t count) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "sph_upload");
    sph_status s = sph_upload_async(ctx, field, host, count, nullptr);
    if (s != SPH_OK) return s;
    return cuda_status(cudaDeviceSynchronize(), "sph_upload");
}

sph_status sph_download_async(sph_ctx *ctx, sph_field field, void *host, size_t count, void *stream) {
    if (!ctx || !host) {
        set_error("sph_download: null argument");
        return SPH_ERR_INVALID_ARG;
    }
    const int n = ctx->n;
    const int blocks = (n + 255) / 256;
    cudaStream_t st = (cudaStream_t)stream;
    auto f1 = [&](const void *src, size_t elem, size_t need) -> sph_status {
        if (count != need) {
            set_error("sph_download: field %d expects %zu elements, got %zu", (int)field, need, count);
            return SPH_ERR_INVALID_ARG;
        }
        return cuda_status(cudaMemcpyAsync(host, src, elem * count, cudaMemcpyDeviceToHost, st), "sph_download");
    };
    switch (field) {
        case SPH_FIELD_POS:
        case SPH_FIELD_VEL:
        case SPH_FIELD_ACC: {
            if (count != 3 * (size_t)n) {
                set_error("sph_download: vector field expects %d floats", 3 * n);
                return SPH_ERR_INVALID_ARG;
            }
            const float4 *src = field == SPH_FIELD_POS ? ctx->pos4 : field == SPH_FIELD_VEL ? ctx->vel4 : ctx->acc4;
            k_unpack3<<<blocks, 256, 0, st>>>(src, (float *)ctx->stage, n);
            return cuda_status(cudaMemcpyAsync(host, ctx->stage, sizeof(float) * count, cudaMemcpyDeviceToHost, st),
                               "sph_download");
        }
        case SPH_FIELD_POS64:
            if (ctx->form.precision != SPH_PRECISION_MIXED || !ctx->pos64) {
                set_error("sph_download: FP64 positions exist in the mixed-precision form only");
                return SPH_ERR_INVALID_ARG;
            }
            if (count != 3 * (size_t)n || sizeof(double) * count > ctx->stage_bytes) {
                set_error("sph_download: FP64 positions expect %d doubles", 3 * n);
                return SPH_ERR_INVALID_ARG;
            }
            k_unpack3d<<<blocks, 256, 0, st>>>(ctx->pos64, (double *)ctx->stage, n);
            return cuda_status(cudaMemcpyAsync(host, ctx->stage, sizeof(double) * count, cudaMemcpyDeviceToHost, st),
                               "sph_download");
        case SPH_FIELD_MASS:
            if (count != (size_t)n) {
                set_error("sph_download: mass expects %d floats", n);
                return SPH_ERR_INVALID_ARG;
            }
            k_get_w<<<blocks, 256, 0, st>>>(ctx->pos4, (float *)ctx->stage, n);
            return cuda_status(cudaMemcpyAsync(host, ctx->stage, sizeof(float) * n, cudaMemcpyDeviceToHost, st),
                               "sph_download");
        case SPH_FIELD_RHO: return f1(ctx->rho, 4, n);
        case SPH_FIELD_U: return f1(ctx->u, 4, n);
        case SPH_FIELD_PRESSURE: return f1(ctx->P, 4, n);
        case SPH_FIELD_H: return f1(ctx->h, 4, n);
        case SPH_FIELD_GRAD_TERM: return f1(ctx->f, 4, n);
        case SPH_FIELD_SOUND_SPEED: return f1(ctx->c, 4, n);
        case SPH_FIELD_DU: return f1(ctx->du, 4, n);
        case SPH_FIELD_BALSARA: return f1(ctx->B, 4, n);
        case SPH_FIELD_DHDT: return f1(ctx->dhdt, 4, n);
        case SPH_FIELD_GRAV_NORM: return f1(ctx->gnorm, 4, n);
        case SPH_FIELD_POTENTIAL: return f1(ctx->phi, 4, n);
        case SPH_FIELD_NEIGHBOURS:
            if (!ctx->hs.nn) {
                set_error("sph_download: no neighbour counts (the learned h seed is not in use)");
                return SPH_ERR_INVALID_ARG;
            }
            return f1(ctx->hs.nn, 4, n);
        case SPH_FIELD_MATERIAL: return f1(ctx->mat, 4, n);
        case SPH_FIELD_ACTIVE: return f1(ctx->active, 1, n);
        case SPH_FIELD_NEXT_ACTIVE: return f1(ctx->nat, 4, n);
        case SPH_FIELD_GLOBAL_TIME: return f1(ctx->globals, 4, 1);
        case SPH_FIELD_DT: return f1(ctx->globals + 1, 4, 1);
        case SPH_FIELD_CELL_KEY: return f1(ctx->cell_sort.keys[ctx->cell_final], 4, n);
        case SPH_FIELD_CELL_INDEX: return f1(ctx->cell_sort.vals[ctx->cell_final], 4, n);
        case SPH_FIELD_CELL_START:
        case SPH_FIELD_CELL_END: {
            if (count != (size_t)kNumCells) {
                set_error("sph_download: cell tables hold %u entries", kNumCells);
                return SPH_ERR_INVALID_ARG;
            }
            k_split_cells<<<148 * 8, 256, 0, st>>>(ctx->cell_range, (uint32_t *)ctx->stage, kNumCells,
                                                   field == SPH_FIELD_CELL_END ? 1 : 0);
            return cuda_status(
                cudaMemcpyAsync(host, ctx->stage, sizeof(uint32_t) * kNumCells, cudaMemcpyDeviceToHost, st),
                "sph_download");
        }
        default:
            set_error("sph_download: unknown field %d", (int)field);
            return SPH_ERR_INVALID_ARG;
    }
}

sph_status sph_download(sph_ctx *ctx, sph_field field, void *host, size_t count) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "sph_download");
    sph_status s = sph_download_async(ctx, field, host, count, nullptr);
    if (s != SPH_OK) return s;
    return cuda_status(cudaDeviceSynchronize(), "sph_download");
}

sph_status sph_get_buffer(sph_ctx *ctx, sph_field field, void **device_ptr, size_t *bytes, size_t *stride) {
    if (!ctx || !device_ptr) return SPH_ERR_INVALID_ARG;
    const size_t n = ctx->n;
    void *p = nullptr;
    size_t b = 0, s = 4;
    switch (field) {
        case SPH_FIELD_POS: p = ctx->pos4; b = 16 * n; s = 16; break;
        case SPH_FIELD_VEL: p = ctx->vel4; b = 16 * n; s = 16; break;
        case SPH_FIELD_ACC: p = ctx->acc4; b = 16 * n; s = 16; break;
        case SPH_FIELD_MASS: p = (char *)ctx->pos4 + 12; b = 16 * n; s = 16; break;
        case SPH_FIELD_RHO: p = ctx->rho; b = 4 * n; break;
        case SPH_FIELD_U: p = ctx->u; b = 4 * n; break;
        case SPH_FIELD_PRESSURE: p = ctx->P; b = 4 * n; break;
        case SPH_FIELD_H: p = ctx->h; b = 4 * n; break;
        case SPH_FIELD_GRAD_TERM: p = ctx->f; b = 4 * n; break;
        case SPH_FIELD_SOUND_SPEED: p = ctx->c; b = 4 * n; break;
        case SPH_FIELD_DU: p = ctx->du; b = 4 * n; break;
        case SPH_FIELD_BALSARA: p = ctx->B; b = 4 * n; break;
        case SPH_FIELD_DHDT: p = ctx->dhdt; b = 4 * n; break;
        case SPH_FIELD_GRAV_NORM: p = ctx->gnorm; b = 4 * n; break;
        case SPH_FIELD_POTENTIAL: p = ctx->phi; b = 4 * n; break;
        case SPH_FIELD_MATERIAL: p = ctx->mat; b = 4 * n; break;
        case SPH_FIELD_ACTIVE: p = ctx->active; b = n; s = 1; break;
        case SPH_FIELD_NEXT_ACTIVE: p = ctx->nat; b = 4 * n; break;
        case SPH_FIELD_GLOBAL_TIME: p = ctx->globals; b = 4; break;
        case SPH_FIELD_DT: p = ctx->globals + 1; b = 4; break;
        case SPH_FIELD_CELL_KEY: p = ctx->cell_sort.keys[ctx->cell_final]; b = 4 * n; break;
        case SPH_FIELD_CELL_INDEX: p = ctx->cell_sort.vals[ctx->cell_final]; b = 4 * n; break;
        case SPH_FIELD_CELL_START: p = ctx->cell_range; b = 8 * (size_t)kNumCells; s = 8; break;
        case SPH_FIELD_CELL_END: p = (char *)ctx->cell_range + 4; b = 8 * (size_t)kNumCells; s = 8; break;
        case SPH_FIELD_POS64: p = ctx->pos64; b = 32 * n; s = 32; break;
        case SPH_FIELD_NEIGHBOURS: p = ctx->hs.nn; b = 4 * n; break;
        default: return SPH_ERR_INVALID_ARG;
    }
    *device_ptr = p;
    if (bytes) *bytes = b;
    if (stride) *stride = s;
    return SPH_OK;
}

sph_status sph_set_tree(sph_ctx *ctx, const int32_t *tree, int32_t tree_len, const int32_t *level_offsets,
                        const int32_t *level_nodes, int32_t n_levels, int32_t n_nodes) {
    if (!ctx || !tree || !level_offsets || !level_nodes || tree_len < 2 || n_levels < 1 || n_levels > 16 ||
        n_nodes < 1) {
        set_error("sph_set_tree: bad arguments");
        return SPH_ERR_INVALID_ARG;
    }
    // validate and derive the per-node list slots (branch rank within level)
    std::vector<int32_t> slot(n_nodes, -1);
    int64_t max_level = 0, max_branches = 0;
    for (int l = 0; l < n_levels; ++l) {
        const int32_t a = level_offsets[l], b = level_offsets[l + 1];
        if (a < 0 || b < a) {
            set_error("sph_set_tree: bad level offsets");
            return SPH_ERR_INVALID_ARG;
        }
        int32_t br = 0;
        for (int32_t k = a; k < b; ++k) {
            const int32_t tp = level_nodes[k];
            if (tp < 0 || tp + 1 >= tree_len) {
                set_error("sph_set_tree: node offset %d out of range", tp);
                return SPH_ERR_INVALID_ARG;
            }
            const int32_t np = tree[tp], dp = tree[tp + 1];
            if (dp < 0 || dp >= n_nodes || np < 0) {
                set_error("sph_set_tree: bad node record at %d", tp);
                return SPH_ERR_INVALID_ARG;
            }
            const int64_t span = (np == 0) ? 10 : 2 + (int64_t)np;
            if (tp + span > tree_len) {
                set_error("sph_set_tree: node at %d runs past the tree", tp);
                return SPH_ERR_INVALID_ARG;
            }
            for (int64_t q = tp + 2; q < tp + span; ++q) {
                const int32_t v = tree[q];
                if (np == 0 ? (v < -1 || v >= tree_len) : (v < 0 || v >= ctx->n)) {
                    set_error("sph_set_tree: bad child or particle entry at %lld", (long long)q);
                    return SPH_ERR_INVALID_ARG;
                }
            }
            slot[dp] = (np == 0) ? br++ : -1;
        }
        max_level = std::max<int64_t>(max_level, b - a);
        max_branches = std::max<int64_t>(max_branches, br);
    }
    Tree &t = ctx->tree;
    drop_graphs(ctx);
    if (n_nodes > t.node_cap || tree_len > t.tree_cap || n_levels > t.max_levels || max_level > t.level_cap ||
        max_branches > t.branch_cap) {
        sph_status s = tree_storage_alloc(
            t, std::max<int64_t>(n_nodes, t.node_cap), std::max<int64_t>(tree_len, t.tree_cap),
            std::max(n_levels, t.max_levels), std::max(max_level, t.level_cap),
            std::max(max_branches + 1, t.branch_cap), t.list_cap);
        if (s != SPH_OK) return s;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(t.tree, tree, sizeof(int32_t) * tree_len, cudaMemcpyHostToDevice);
    std::vector<int32_t> counts(16, 0);
    for (int l = 0; l < n_levels && e == cudaSuccess; ++l) {
        const int32_t a = level_offsets[l], b = level_offsets[l + 1];
        counts[l] = b - a;
        if (b > a)
            e = cudaMemcpy(t.level_nodes + (size_t)l * t.level_cap, level_nodes + a, sizeof(int32_t) * (b - a),
                           cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpy(t.level_count, counts.data(), sizeof(int32_t) * 16, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t.list_slot, slot.data(), sizeof(int32_t) * n_nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(t.parent_slot, 0, sizeof(int32_t) * n_nodes);
    if (e != cudaSuccess) return cuda_status(e, "sph_set_tree");
    int32_t meta[4] = {n_levels, n_nodes, tree_len, 0};
    if (e == cudaSuccess) e = cudaMemcpy(t.meta, meta, sizeof(meta), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e, "sph_set_tree");
    t.n_levels_host = n_levels;
    for (int l = 0; l < 16; ++l) t.level_count_host[l] = counts[l];
    t.valid = true;
    ctx->params.tree_source = SPH_TREE_HOST;
    return SPH_OK;
}

sph_status sph_get_tree(sph_ctx *ctx, int32_t *tree, int64_t tree_room, int32_t *tree_len, int32_t *level_offsets,
                        int32_t *level_nodes, int64_t level_nodes_room, int32_t *n_levels, int32_t *n_nodes) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    Tree &t = ctx->tree;
    if (!t.valid) {
        set_error("sph_get_tree: no tree yet");
        return SPH_ERR_INVALID_ARG;
    }
    cudaError_t e = cudaDeviceSynchronize();
    int32_t meta[4] = {0, 0, 0, 0}, counts[16] = {0};
    if (e == cudaSuccess) e = cudaMemcpy(meta, t.meta, sizeof(meta), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(counts, t.level_count, sizeof(counts), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "sph_get_tree");
    int nl = 0;
    int64_t total = 0;
    for (int l = 0; l < t.n_levels_host && l < 16; ++l)
        if (counts[l] > 0) {
            nl = l + 1;
            total += counts[l];
        }
    if (tree_len) *tree_len = meta[2];
    if (n_levels) *n_levels = nl;
    if (n_nodes) *n_nodes = meta[1];
    if (tree) {
        if (tree_room < meta[2]) {
            set_error("sph_get_tree: tree buffer too small");
            return SPH_ERR_INVALID_ARG;
        }
        e = cudaMemcpy(tree, t.tree, sizeof(int32_t) * (size_t)meta[2], cudaMemcpyDeviceToHost);
    }
    if (level_offsets) {
        int32_t o = 0;
        for (int l = 0; l < nl; ++l) {
            level_offsets[l] = o;
            o += counts[l];
        }
        level_offsets[nl] = o;
    }
    if (level_nodes && e == cudaSuccess) {
        if (level_nodes_room < total) {
            set_error("sph_get_tree: level buffer too small");
            return SPH_ERR_INVALID_ARG;
        }
        int64_t o = 0;
        for (int l = 0; l < nl && e == cudaSuccess; ++l) {
            if (counts[l] > 0)
                e = cudaMemcpy(level_nodes + o, t.level_nodes + (size_t)l * t.level_cap, sizeof(int32_t) * counts[l],
                               cudaMemcpyDeviceToHost);
            o += counts[l];
        }
    }
    return cuda_status(e, "sph_get_tree");
}

sph_status sph_get_tree_nodes(sph_ctx *ctx, float *poles, float *locals, int32_t n_nodes) {
    if (!ctx || n_nodes < 0 || n_nodes > ctx->tree.node_cap) {
        set_error("sph_get_tree_nodes: bad arguments");
        return SPH_ERR_INVALID_ARG;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && poles)
        e = cudaMemcpy(poles, ctx->tree.poles, sizeof(float4) * kPoleQ * (size_t)n_nodes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && locals)
        e = cudaMemcpy(locals, ctx->tree.locals, sizeof(float4) * kLocalQ * (size_t)n_nodes, cudaMemcpyDeviceToHost);
    return cuda_status(e, "sph_get_tree_nodes");
}

sph_status sph_update_tree(sph_ctx *ctx, void *stream) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    if (ctx->params.tree_source != SPH_TREE_GPU) return SPH_OK;  // host trees are given by sph_set_tree
    return launch_tree_build(ctx, (cudaStream_t)stream);
}

sph_status sph_sort(sph_ctx *ctx, void *stream) {
    return ctx ? launch_sort(ctx, (cudaStream_t)stream) : SPH_ERR_INVALID_ARG;
}
static sph_status gravity_pass(sph_ctx *ctx, cudaStream_t st) {
    return ctx->form.gravity == SPH_GRAVITY_THETA ? launch_gravity_theta(ctx, st) : launch_gravity(ctx, st);
}
sph_status sph_gravity(sph_ctx *ctx, void *stream) {
    return ctx ? gravity_pass(ctx, (cudaStream_t)stream) : SPH_ERR_INVALID_ARG;
}

void sph_form_default(sph_form *f) {
    if (!f) return;
    f->gravity = SPH_GRAVITY_REFERENCE;
    f->theta = 0.5f;
    f->h_seed = SPH_HSEED_PLAIN;
    f->precision = SPH_PRECISION_REFERENCE;
    f->h_tolerance = 0.f;
    f->timestep = SPH_TIMESTEP_GLOBAL;
}

sph_status sph_set_form(sph_ctx *ctx, const sph_form *f) {
    if (!ctx || !f) return SPH_ERR_INVALID_ARG;
    if (f->gravity != SPH_GRAVITY_REFERENCE && f->gravity != SPH_GRAVITY_THETA) {
        set_error("sph_set_form: gravity = %d is not a SPH_GRAVITY_* value", (int)f->gravity);
        return SPH_ERR_INVALID_ARG;
    }
    if (!(f->theta > 0.f && f->theta <= 1.5f)) {
        set_error("sph_set_form: theta = %g is outside (0, 1.5]", (double)f->theta);
        return SPH_ERR_INVALID_ARG;
    }
    if (f->h_seed != SPH_HSEED_PLAIN && f->h_seed != SPH_HSEED_LEARNED) {
        set_error("sph_set_form: h_seed = %d is not a SPH_HSEED_* value", (int)f->h_seed);
        return SPH_ERR_INVALID_ARG;
    }
    if (f->h_seed == SPH_HSEED_LEARNED && !ctx->hs.have_norm) {
        set_error("sph_set_form: the learned h seed is not trained yet (sph_hseed_train)");
        return SPH_ERR_INVALID_ARG;
    }
    if (!(f->h_tolerance >= 0.f && f->h_tolerance < 1.f)) {
        set_error("sph_set_form: h_tolerance = %g is outside [0, 1)", (double)f->h_tolerance);
        return SPH_ERR_INVALID_ARG;
    }
    if (f->timestep != SPH_TIMESTEP_GLOBAL && f->timestep != SPH_TIMESTEP_INDIVIDUAL) {
        set_error("sph_set_form: timestep = %d is not a SPH_TIMESTEP_* value", (int)f->timestep);
        return SPH_ERR_INVALID_ARG;
    }
    if (f->precision != SPH_PRECISION_REFERENCE && f->precision != SPH_PRECISION_MIXED) {
        set_error("sph_set_form: precision = %d is not a SPH_PRECISION_* value", (int)f->precision);
        return SPH_ERR_INVALID_ARG;
    }
    if (f->gravity == SPH_GRAVITY_THETA && ctx->params.tree_source != SPH_TREE_GPU) {
        set_error("sph_set_form: the theta gravity form needs the GPU-built tree (SPH_TREE_GPU)");
        return SPH_ERR_UNSUPPORTED;
    }
    cudaSetDevice(ctx->device);
    drop_graphs(ctx);
    const bool enter_mixed = f->precision == SPH_PRECISION_MIXED && ctx->form.precision != SPH_PRECISION_MIXED;
    ctx->form = *f;
    if (enter_mixed) {
        cudaError_t e = cudaSuccess;
        if (!ctx->pos64) e = cudaMalloc(&ctx->pos64, sizeof(double4) * (size_t)ctx->n);
        if (e != cudaSuccess) {
            ctx->form.precision = SPH_PRECISION_REFERENCE;
            return cuda_status(e, "sph_set_form: FP64 positions");
        }
        sph_status s = launch_pos_to64(ctx, nullptr);
        if (s != SPH_OK) return s;
        k_time_to64<<<1, 1>>>(ctx->globals, ctx->dglob);
        return cuda_status(cudaDeviceSynchronize(), "sph_set_form");
    }
    return SPH_OK;
}

sph_status sph_get_form(const sph_ctx *ctx, sph_form *f) {
    if (!ctx || !f) return SPH_ERR_INVALID_ARG;
    *f = ctx->form;
    return SPH_OK;
}

sph_status sph_set_tiling(sph_ctx *ctx, const sph_tiling *t) {
    if (!ctx || !t) return SPH_ERR_INVALID_ARG;
    constexpr uint32_t kMaxTile = 1u << 20;
    if (t->block_max < 1 || t->block_max > kMaxTile || t->half_max < 1 || t->half_max > kMaxTile ||
        t->big_max > kMaxTile) {
        set_error("sph_set_tiling: block_max and half_max must be in [1, %u], big_max in [0, %u]", kMaxTile,
                  kMaxTile);
        return SPH_ERR_INVALID_ARG;
    }
    cudaSetDevice(ctx->device);
    drop_graphs(ctx);
    ctx->tile_big_max = t->big_max;
    ctx->tile_block_max = t->block_max;
    ctx->tile_half_max = t->half_max;
    ctx->tile_coarse = t->coarse ? 1 : 0;
    return SPH_OK;
}

sph_status sph_get_tiling(const sph_ctx *ctx, sph_tiling *t) {
    if (!ctx || !t) return SPH_ERR_INVALID_ARG;
    t->big_max = ctx->tile_big_max;
    t->block_max = ctx->tile_block_max;
    t->half_max = ctx->tile_half_max;
    t->coarse = ctx->tile_coarse;
    return SPH_OK;
}

sph_status sph_gravity_direct_f64(sph_ctx *ctx, const int32_t *targets, int32_t n_targets, double *out,
                                  void *stream) {
    if (!ctx || n_targets < 0 || (n_targets > 0 && (!targets || !out))) return SPH_ERR_INVALID_ARG;
    if (n_targets == 0) return SPH_OK;
    for (int32_t t = 0; t < n_targets; ++t) {
        if (targets[t] < 0 || targets[t] >= ctx->n) {
            set_error("sph_gravity_direct_f64: target %d = %d is outside 0..%d", (int)t, (int)targets[t],
                      ctx->n - 1);
            return SPH_ERR_INVALID_ARG;
        }
    }
    const size_t tgt_bytes = ((sizeof(int32_t) * (size_t)n_targets + 255) / 256) * 256;
    const size_t out_bytes = sizeof(double) * 4 * (size_t)n_targets;
    if (tgt_bytes + out_bytes > ctx->stage_bytes) {
        set_error("sph_gravity_direct_f64: %d targets exceed the staging buffer (%zu bytes)", (int)n_targets,
                  ctx->stage_bytes);
        return SPH_ERR_INVALID_ARG;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    int32_t *d_t = (int32_t *)ctx->stage;
    double *d_o = (double *)((char *)ctx->stage + tgt_bytes);
    cudaError_t e = cudaMemcpyAsync(d_t, targets, sizeof(int32_t) * (size_t)n_targets, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_status(e, "sph_gravity_direct_f64 upload");
    sph_status s = launch_direct_f64(ctx, d_t, n_targets, d_o, st);
    if (s != SPH_OK) return s;
    e = cudaMemcpyAsync(out, d_o, out_bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return cuda_status(e, "sph_gravity_direct_f64");
}
sph_status sph_diagnostics(sph_ctx *ctx, void *stream, float theta_potential, sph_diag *out) {
    if (!ctx || !out) return SPH_ERR_INVALID_ARG;
    if (!(theta_potential >= 0.f && theta_potential <= 1.5f)) {
        set_error("sph_diagnostics: theta_potential = %g is outside [0, 1.5]", (double)theta_potential);
        return SPH_ERR_INVALID_ARG;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    std::memset(out, 0, sizeof(*out));
    sph_status s = SPH_OK;
    const bool pot = ctx->params.tree_source == SPH_TREE_GPU;
    if (pot) {
        s = launch_tree_build(ctx, st);
        if (s == SPH_OK) s = launch_potential_theta(ctx, theta_potential > 0.f ? theta_potential : 0.5f, st);
    } else {
        cudaMemsetAsync(ctx->phi, 0, sizeof(float) * (size_t)ctx->n, st);
    }
    if (s == SPH_OK) s = launch_diag_sums(ctx, st);
    if (s != SPH_OK) return s;
    double tot[kDiag];
    int32_t g[2] = {0, 0};
    double t64 = 0.0;
    cudaError_t e = cudaMemcpyAsync(tot, ctx->diag + (size_t)kDiagBlocks * kDiag, sizeof(tot), cudaMemcpyDeviceToHost,
                                    st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g, ctx->globals, sizeof(g), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&t64, ctx->dglob, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&out->health, ctx->health, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "sph_diagnostics");
    out->mass = tot[0];
    out->kinetic = tot[1];
    out->internal = tot[2];
    out->potential = pot ? tot[3] : 0.0;
    out->total = out->kinetic + out->internal + out->potential;
    for (int k = 0; k < 3; ++k) {
        out->momentum[k] = tot[4 + k];
        out->angular_momentum[k] = tot[7 + k];
    }
    out->time = ctx->form.precision == SPH_PRECISION_MIXED ? t64 : (double)kDtMin1 * (double)g[0];
    out->potential_valid = pot ? 1 : 0;
    return SPH_OK;
}

sph_status sph_density(sph_ctx *ctx, void *stream) {
    return ctx ? launch_density(ctx, (cudaStream_t)stream) : SPH_ERR_INVALID_ARG;
}
sph_status sph_acceleration(sph_ctx *ctx, void *stream) {
    return ctx ? launch_acceleration(ctx, (cudaStream_t)stream) : SPH_ERR_INVALID_ARG;
}
sph_status sph_step(sph_ctx *ctx, void *stream) {
    return ctx ? launch_step(ctx, (cudaStream_t)stream) : SPH_ERR_INVALID_ARG;
}

}  // extern "C"

namespace sph {

// One full step (Headless.cpp:43-51 without the snapshot) on `st`.
// The side stream and the fork / join events of a step (created once).
sph_status ensure_side(sph_ctx *ctx) {
    cudaError_t e = cudaSuccess;
    if (!ctx->side_stream) e = cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ctx->ev_fork) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess && !ctx->ev_join) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
    return cuda_status(e, "side stream");
}

sph_status full_step(sph_ctx *ctx, cudaStream_t st) {
    sph_status s = SPH_OK;
    // the learned seed's online refresh runs beside the tree, sort and
    // gravity passes (it reads the previous density pass's pairs and writes
    // only the network) and is joined before the density pass
    const bool ahead = hseed_online_due(ctx);
    if (ahead) {
        s = ensure_side(ctx);
        cudaError_t e = cudaSuccess;
        if (s == SPH_OK) e = cudaEventRecord(ctx->ev_fork, st);
        if (s == SPH_OK && e == cudaSuccess) e = cudaStreamWaitEvent(ctx->side_stream, ctx->ev_fork, 0);
        if (s == SPH_OK && e != cudaSuccess) s = cuda_status(e, "full step fork");
        if (s == SPH_OK) s = launch_hseed_online(ctx, ctx->side_stream);
        // recorded whatever happened, so that a capture ends well formed
        cudaError_t ej = cudaEventRecord(ctx->ev_join, ctx->side_stream);
        if (s == SPH_OK && ej != cudaSuccess) s = cuda_status(ej, "full step join");
        ctx->hs.trained_ahead = s == SPH_OK;
    }
    if (s == SPH_OK && ctx->params.tree_source == SPH_TREE_GPU) s = launch_tree_build(ctx, st);
    if (s == SPH_OK) s = launch_sort(ctx, st);
    if (s == SPH_OK) s = gravity_pass(ctx, st);
    if (ahead) {
        cudaError_t ej = cudaStreamWaitEvent(st, ctx->ev_join, 0);
        if (s == SPH_OK && ej != cudaSuccess) s = cuda_status(ej, "full step join");
    }
    if (s == SPH_OK) s = launch_density(ctx, st);
    ctx->hs.trained_ahead = false;
    if (s == SPH_OK) s = launch_acceleration(ctx, st);
    if (s == SPH_OK) s = launch_step(ctx, st);
    return s;
}

void drop_graphs(sph_ctx *ctx) {
    if (ctx->graph) {
        cudaGraphExecDestroy(ctx->graph);
        ctx->graph = nullptr;
    }
    if (ctx->host_graph) {
        cudaGraphExecDestroy(ctx->host_graph);
        ctx->host_graph = nullptr;
    }
}

namespace {

// sph_step_host's check of the copied smoothing lengths (sph_upload checks
// them on the host): an h outside (0, kMaxInitialH] -- whose first density
// sweep would scan a box wider than the periodic grid -- becomes
// MAX_SMOOTHING_LENGTH (kMaxH, where the density iteration caps h) and raises
// SPH_HEALTH_BAD_INPUT.
__global__ void k_check_h(float *__restrict__ h, int n, uint32_t *health) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = h[i];
    if (!(v > 0.f) || !(v <= kMaxInitialH)) {
        h[i] = kMaxH;
        atomicOr(health, SPH_HEALTH_BAD_INPUT);
    }
}

// The step of sph_step_host on st, eager or under capture: the positions'
// copy, the other inputs' copies on the side stream (joined before the
// density pass), the passes, then the outputs' copies.  sv4, the sorted
// velocities, is scratch outside the density pass and stages the velocity
// copies; ctx->stage stages the positions'.
sph_status host_step(sph_ctx *ctx, const sph_host_state &in, const sph_host_state &out, cudaStream_t st) {
    const int n = ctx->n;
    const size_t n3 = 3 * (size_t)n;
    const int blocks = (n + 255) / 256;
    const bool mixed = ctx->form.precision == SPH_PRECISION_MIXED;
    cudaStream_t sd = ctx->side_stream;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    if (mixed && in.pos64) {
        ok(cudaMemcpyAsync(ctx->stage, in.pos64, sizeof(double) * n3, cudaMemcpyHostToDevice, st));
        k_pack3d<<<blocks, 256, 0, st>>>((const double *)ctx->stage, ctx->pos64, ctx->pos4, n);
    } else if (!mixed && in.pos) {
        ok(cudaMemcpyAsync(ctx->stage, in.pos, sizeof(float) * n3, cudaMemcpyHostToDevice, st));
        k_pack3<<<blocks, 256, 0, st>>>((const float *)ctx->stage, ctx->pos4, n, 1);
    }
    ok(cudaEventRecord(ctx->ev_fork, st));
    ok(cudaStreamWaitEvent(sd, ctx->ev_fork, 0));
    if (in.vel) {
        ok(cudaMemcpyAsync(ctx->sv4, in.vel, sizeof(float) * n3, cudaMemcpyHostToDevice, sd));
        k_pack3<<<blocks, 256, 0, sd>>>((const float *)ctx->sv4, ctx->vel4, n, 0);
    }
    if (in.u) ok(cudaMemcpyAsync(ctx->u, in.u, sizeof(float) * n, cudaMemcpyHostToDevice, sd));
    if (in.h) {
        ok(cudaMemcpyAsync(ctx->h, in.h, sizeof(float) * n, cudaMemcpyHostToDevice, sd));
        k_check_h<<<blocks, 256, 0, sd>>>(ctx->h, n, ctx->health);
    }
    if (in.rho) ok(cudaMemcpyAsync(ctx->rho, in.rho, sizeof(float) * n, cudaMemcpyHostToDevice, sd));
    ok(cudaGetLastError());
    sph_status s = e == cudaSuccess ? SPH_OK : cuda_status(e, "sph_step_host inputs");
    // the learned seed's online refresh follows on the side stream (full_step)
    if (s == SPH_OK && hseed_online_due(ctx)) {
        s = launch_hseed_online(ctx, sd);
        ctx->hs.trained_ahead = s == SPH_OK;
    }
    ok(cudaEventRecord(ctx->ev_join, sd));
    if (s == SPH_OK && ctx->params.tree_source == SPH_TREE_GPU) s = launch_tree_build(ctx, st);
    if (s == SPH_OK) s = launch_sort(ctx, st);
    if (s == SPH_OK) s = gravity_pass(ctx, st);
    // joined whatever happened, so that a capture ends well formed
    cudaError_t ej = cudaStreamWaitEvent(st, ctx->ev_join, 0);
    if (s == SPH_OK && ej != cudaSuccess) s = cuda_status(ej, "sph_step_host join");
    if (s == SPH_OK) s = launch_density(ctx, st);
    ctx->hs.trained_ahead = false;
    if (s == SPH_OK) s = launch_acceleration(ctx, st);
    if (s == SPH_OK) s = launch_step(ctx, st);
    if (s != SPH_OK) return s;
    if (mixed && out.pos64) {
        k_unpack3d<<<blocks, 256, 0, st>>>(ctx->pos64, (double *)ctx->stage, n);
        ok(cudaMemcpyAsync(out.pos64, ctx->stage, sizeof(double) * n3, cudaMemcpyDeviceToHost, st));
    } else if (!mixed && out.pos) {
        k_unpack3<<<blocks, 256, 0, st>>>(ctx->pos4, (float *)ctx->stage, n);
        ok(cudaMemcpyAsync(out.pos, ctx->stage, sizeof(float) * n3, cudaMemcpyDeviceToHost, st));
    }
    if (out.vel) {
        k_unpack3<<<blocks, 256, 0, st>>>(ctx->vel4, (float *)ctx->sv4, n);
        ok(cudaMemcpyAsync(out.vel, ctx->sv4, sizeof(float) * n3, cudaMemcpyDeviceToHost, st));
    }
    if (out.u) ok(cudaMemcpyAsync(out.u, ctx->u, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    if (out.h) ok(cudaMemcpyAsync(out.h, ctx->h, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    if (out.rho) ok(cudaMemcpyAsync(out.rho, ctx->rho, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    ok(cudaGetLastError());
    return cuda_status(e, "sph_step_host outputs");
}

}  // namespace

}  // namespace sph

extern "C" {

sph_status sph_step_all(sph_ctx *ctx, void *stream, int32_t n_steps) {
    if (!ctx || n_steps < 0) return SPH_ERR_INVALID_ARG;
    if (n_steps == 0) return SPH_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (!ctx->own_stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_status(e, "sph_step_all stream");
    }
    if (!ctx->graph) {
        // capture one full step on a private stream; the buffer roles of the
        // sort (cell_final, cells_have_prev) are the same every step once warm
        sph_status s = full_step(ctx, st);  // warm: establishes the steady buffer roles
        if (s != SPH_OK) return s;
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e, "sph_step_all warm step");
        --n_steps;
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(ctx->own_stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_status(e, "begin capture");
        s = full_step(ctx, ctx->own_stream);
        e = cudaStreamEndCapture(ctx->own_stream, &g);
        if (s != SPH_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return cuda_status(e, "end capture");
        e = cudaGraphInstantiate(&ctx->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_status(e, "graph instantiate");
    }
    for (int i = 0; i < n_steps; ++i) {
        cudaError_t e = cudaGraphLaunch(ctx->graph, st);
        if (e != cudaSuccess) return cuda_status(e, "graph launch");
    }
    return SPH_OK;
}

sph_status sph_step_host(sph_ctx *ctx, const sph_host_state *in, const sph_host_state *out, void *stream) {
    if (!ctx || !in || !out) return SPH_ERR_INVALID_ARG;
    const bool mixed = ctx->form.precision == SPH_PRECISION_MIXED;
    if (mixed ? (in->pos || out->pos) : (in->pos64 || out->pos64)) {
        set_error("sph_step_host: %s", mixed ? "the mixed-precision form moves FP64 positions (pos64), not pos"
                                             : "FP64 positions (pos64) exist in the mixed-precision form only");
        return SPH_ERR_INVALID_ARG;
    }
    const void *bufs[] = {in->pos64, in->pos, in->vel, in->u, in->h, in->rho,
                          out->pos64, out->pos, out->vel, out->u, out->h, out->rho};
    for (const void *b : bufs) {
        if (!b) continue;
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, b) != cudaSuccess || at.type != cudaMemoryTypeHost) {
            cudaGetLastError();
            set_error("sph_step_host: host buffers must be page-locked (cudaHostAlloc / cudaHostRegister)");
            return SPH_ERR_INVALID_ARG;
        }
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if (!ctx->own_stream) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_status(e, "sph_step_host stream");
    sph_status s = ensure_side(ctx);
    if (s != SPH_OK) return s;
    const bool same = ctx->host_graph && std::memcmp(&ctx->host_in, in, sizeof(*in)) == 0 &&
                      std::memcmp(&ctx->host_out, out, sizeof(*out)) == 0;
    if (same) return cuda_status(cudaGraphLaunch(ctx->host_graph, st), "sph_step_host graph launch");
    if (ctx->host_graph) {
        cudaGraphExecDestroy(ctx->host_graph);
        ctx->host_graph = nullptr;
    }
    // this call's step runs eagerly (it also settles the sort's buffer roles);
    // the graph for the next calls is captured after it
    s = host_step(ctx, *in, *out, st);
    if (s != SPH_OK) return s;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "sph_step_host eager step");
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(ctx->own_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e, "sph_step_host begin capture");
    s = host_step(ctx, *in, *out, ctx->own_stream);
    e = cudaStreamEndCapture(ctx->own_stream, &g);
    if (s != SPH_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return s != SPH_OK ? s : cuda_status(e, "sph_step_host end capture");
    }
    e = cudaGraphInstantiate(&ctx->host_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        ctx->host_graph = nullptr;
        return cuda_status(e, "sph_step_host graph instantiate");
    }
    ctx->host_in = *in;
    ctx->host_out = *out;
    return SPH_OK;
}

sph_status sph_probe_fp32_fma(int32_t blocks, int32_t iters, float *sink, void *stream) {
    if (blocks < 1 || iters < 1 || !sink) return SPH_ERR_INVALID_ARG;
    k_fma_probe<<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 0.5f, sink);
    return cuda_status(cudaGetLastError(), "sph_probe_fp32_fma");
}

sph_status sph_draw_snapshot(sph_ctx *ctx, void *stream, int32_t *image) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    sph_status s = launch_snapshot(ctx, (cudaStream_t)stream);
    if (s != SPH_OK || !image) return s;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e == cudaSuccess)
        e = cudaMemcpy(image, ctx->snapshot, sizeof(int32_t) * kSnapshotRes * kSnapshotRes, cudaMemcpyDeviceToHost);
    return cuda_status(e, "sph_draw_snapshot");
}

sph_status sph_get_health(sph_ctx *ctx, uint32_t *word) {
    if (!ctx || !word) return SPH_ERR_INVALID_ARG;
    return cuda_status(cudaMemcpy(word, ctx->health, 4, cudaMemcpyDeviceToHost), "sph_get_health");
}

sph_status sph_clear_health(sph_ctx *ctx) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    return cuda_status(cudaMemset(ctx->health, 0, 4), "sph_clear_health");
}

sph_status sph_synchronize(sph_ctx *ctx, void *stream) {
    if (!ctx) return SPH_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_status(e, "sph_synchronize");
    uint32_t w = 0;
    sph_status s = sph_get_health(ctx, &w);
    if (s != SPH_OK) return s;
    if (w & (SPH_HEALTH_SORT_TIMEOUT | SPH_HEALTH_SCAN_TIMEOUT | SPH_HEALTH_MLP_TIMEOUT)) {
        set_error("bounded device wait timed out (health 0x%x)", w);
        return SPH_ERR_TIMEOUT;
    }
    if (w) {
        set_error("device health word 0x%x", w);
        return SPH_ERR_DEVICE_HEALTH;
    }
    return SPH_OK;
}

}  // extern "C"

// sph_ensemble.cu -- many independent impacts on one GPU, advanced together.
//
// No counterpart in the reference, which runs one simulation per process
// (Headless.cpp:43-51, Compute.cpp:379-393).  An ensemble owns one context per
// instance (its own particles, cell table, tree and tiles), so instances share
// no device memory and never wait on one another.  One ensemble step is one
// launch of one CUDA graph whose branches are the instances' full steps
// (tree, sort, gravity, density, acceleration, kick/drift), captured from
// full_step and joined as child graphs with no edges between them: the device
// runs the small instances' kernels side by side, which one instance of
// 2e4 particles could not fill alone.
//
// The tuner (autotune != 0) picks, per instance, on a scratch context built
// from the same initial conditions (so tuning does not advance the instance):
//   * the density / acceleration tile size (tile_block_max), by timing a full
//     step of each candidate;
//   * for the opening-angle gravity form, the leaf capacity among 1x, 2x and
//     4x the requested one, by timing, among the capacities whose gravity
//     meets a median relative error of 1e-3 against the FP64 direct sum on a
//     fixed sample of targets.  The reference's gravity form keeps the
//     requested capacity, which is part of its algorithm.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sph_internal.h"

using namespace sph;

struct sph_ensemble {
    int device = 0;
    std::vector<sph_ctx *> inst;
    std::vector<sph_ensemble_tuning> tuning;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t capture = nullptr;
};

namespace {

constexpr uint32_t kTileCandidates[] = {128u, 320u, 640u};
constexpr int kTuneTargets = 512;
constexpr float kTuneGravityBound = 1e-3f;

// Mean milliseconds of `steps` full steps of ctx after `warm` untimed ones.
sph_status time_steps(sph_ctx *ctx, cudaStream_t st, int warm, int steps, float &ms) {
    for (int i = 0; i < warm; ++i) {
        sph_status s = full_step(ctx, st);
        if (s != SPH_OK) return s;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    sph_status s = SPH_OK;
    for (int i = 0; i < steps && s == SPH_OK; ++i) s = full_step(ctx, st);
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != SPH_OK) return s;
    if (e != cudaSuccess) return cuda_status(e, "ensemble tuner timing");
    ms = t / (float)std::max(steps, 1);
    return SPH_OK;
}

// Median relative error of the theta gravity of ctx's current state against
// the FP64 direct sum, on kTuneTargets targets spread over the particles.
sph_status gravity_median_error(sph_ctx *ctx, cudaStream_t st, float &err) {
    const int n = ctx->n;
    const int nt = std::min(n, kTuneTargets);
    std::vector<int32_t> tg(nt);
    for (int i = 0; i < nt; ++i) tg[i] = (int32_t)(((int64_t)i * n) / nt);
    sph_status s = launch_tree_build(ctx, st);
    if (s == SPH_OK) s = launch_sort(ctx, st);
    if (s == SPH_OK) s = launch_gravity_theta(ctx, st);
    if (s != SPH_OK) return s;
    std::vector<float> acc(3 * (size_t)n);
    s = sph_download_async(ctx, SPH_FIELD_ACC, acc.data(), acc.size(), st);
    if (s != SPH_OK) return s;
    std::vector<double> ref(4 * (size_t)nt);
    s = sph_gravity_direct_f64(ctx, tg.data(), nt, ref.data(), st);  // synchronises st
    if (s != SPH_OK) return s;
    std::vector<double> rel(nt);
    for (int i = 0; i < nt; ++i) {
        const size_t k = (size_t)tg[i];
        const double gx = ref[4 * i], gy = ref[4 * i + 1], gz = ref[4 * i + 2];
        const double dx = acc[3 * k] - gx, dy = acc[3 * k + 1] - gy, dz = acc[3 * k + 2] - gz;
        const double nr = std::sqrt(gx * gx + gy * gy + gz * gz);
        rel[i] = std::sqrt(dx * dx + dy * dy + dz * dz) / std::max(nr, 1e-300);
    }
    std::nth_element(rel.begin(), rel.begin() + nt / 2, rel.end());
    err = (float)rel[nt / 2];
    return SPH_OK;
}

// Tune one instance on a scratch context made from its initial conditions.
sph_status tune_instance(const sph_params &p, const sph_ic &ic, const sph_form &form, cudaStream_t st,
                         sph_ensemble_tuning &best) {
    best.max_children_in_leaf = p.max_children_in_leaf;
    best.tile_block_max = 320u;
    best.ms_per_step = 0.f;
    best.gravity_median_error = -1.f;
    std::vector<int32_t> leaves = {p.max_children_in_leaf};
    if (form.gravity == SPH_GRAVITY_THETA && p.tree_source == SPH_TREE_GPU)
        leaves = {p.max_children_in_leaf, 2 * p.max_children_in_leaf, 4 * p.max_children_in_leaf};
    sph_ctx *c = nullptr;
    sph_status s = sph_create(&p, &ic, &c);
    if (s != SPH_OK) return s;
    s = sph_set_form(c, &form);
    float best_ms = 3.4e38f;
    for (int32_t leaf : leaves) {
        if (s != SPH_OK) break;
        // the scratch context's tree storage is sized for p.max_children_in_leaf,
        // which bounds the node count of every larger capacity
        c->params.max_children_in_leaf = leaf;
        float gerr = -1.f;
        if (leaves.size() > 1) {
            s = gravity_median_error(c, st, gerr);
            if (s != SPH_OK) break;
            if (!(gerr <= kTuneGravityBound)) continue;
        }
        for (uint32_t tb : kTileCandidates) {
            c->tile_block_max = tb;
            c->tile_half_max = std::min(tb, 256u);
            float ms = 0.f;
            s = time_steps(c, st, 1, 2, ms);
            if (s != SPH_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                best.max_children_in_leaf = leaf;
                best.tile_block_max = tb;
                best.ms_per_step = ms;
                best.gravity_median_error = gerr;
            }
        }
    }
    sph_destroy(c);
    return s;
}

void apply_tuning(sph_ctx *c, const sph_ensemble_tuning &t) {
    c->params.max_children_in_leaf = t.max_children_in_leaf;
    c->tile_block_max = t.tile_block_max;
    c->tile_half_max = std::min(t.tile_block_max, 256u);
}

void ensemble_free(sph_ensemble *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    if (e->capture) cudaStreamDestroy(e->capture);
    for (sph_ctx *c : e->inst) sph_destroy(c);
    delete e;
}

// The ensemble step graph: one child graph per instance, no edges between them.
sph_status build_graph(sph_ensemble *e) {
    cudaGraph_t parent = nullptr;
    cudaError_t err = cudaGraphCreate(&parent, 0);
    if (err != cudaSuccess) return cuda_status(err, "ensemble graph");
    sph_status s = SPH_OK;
    for (sph_ctx *c : e->inst) {
        cudaGraph_t g = nullptr;
        err = cudaStreamBeginCapture(e->capture, cudaStreamCaptureModeThreadLocal);
        if (err != cudaSuccess) {
            s = cuda_status(err, "ensemble capture");
            break;
        }
        s = full_step(c, e->capture);
        err = cudaStreamEndCapture(e->capture, &g);
        if (s == SPH_OK && err != cudaSuccess) s = cuda_status(err, "ensemble capture end");
        if (s == SPH_OK) {
            cudaGraphNode_t node = nullptr;
            err = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, g);
            if (err != cudaSuccess) s = cuda_status(err, "ensemble child graph");
        }
        if (g) cudaGraphDestroy(g);
        if (s != SPH_OK) break;
    }
    if (s == SPH_OK) {
        err = cudaGraphInstantiate(&e->graph, parent, 0);
        if (err != cudaSuccess) s = cuda_status(err, "ensemble graph instantiate");
    }
    cudaGraphDestroy(parent);
    return s;
}

}  // namespace

extern "C" {

sph_status sph_ensemble_create(const sph_params *params, int32_t n_instances, const sph_ic *ics,
                               const sph_form *forms, int32_t autotune, sph_ensemble **out) {
    if (!out || n_instances <= 0 || !ics) {
        set_error("sph_ensemble_create: need at least one instance and its initial conditions");
        return SPH_ERR_INVALID_ARG;
    }
    *out = nullptr;
    sph_params p;
    sph_params_default(&p);
    if (params) p = *params;
    sph_ensemble *e = new sph_ensemble();
    cudaGetDevice(&e->device);
    cudaError_t err = cudaStreamCreateWithFlags(&e->capture, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        ensemble_free(e);
        return cuda_status(err, "ensemble stream");
    }
    sph_status s = SPH_OK;
    e->inst.reserve(n_instances);
    e->tuning.resize(n_instances);
    for (int32_t i = 0; i < n_instances && s == SPH_OK; ++i) {
        sph_form f;
        sph_form_default(&f);
        if (forms) f = forms[i];
        sph_ensemble_tuning &t = e->tuning[i];
        t.max_children_in_leaf = p.max_children_in_leaf;
        t.tile_block_max = 320u;
        t.ms_per_step = 0.f;
        t.gravity_median_error = -1.f;
        if (autotune) s = tune_instance(p, ics[i], f, e->capture, t);
        if (s != SPH_OK) break;
        sph_ctx *c = nullptr;
        s = sph_create(&p, &ics[i], &c);
        if (s != SPH_OK) break;
        e->inst.push_back(c);
        s = sph_set_form(c, &f);
        if (s == SPH_OK) apply_tuning(c, t);
    }
    if (s == SPH_OK) {
        err = cudaStreamSynchronize(e->capture);
        if (err != cudaSuccess) s = cuda_status(err, "ensemble create");
    }
    if (s != SPH_OK) {
        ensemble_free(e);
        return s;
    }
    *out = e;
    return SPH_OK;
}

sph_status sph_ensemble_destroy(sph_ensemble *e) {
    ensemble_free(e);
    return SPH_OK;
}

int32_t sph_ensemble_size(const sph_ensemble *e) { return e ? (int32_t)e->inst.size() : 0; }

sph_status sph_ensemble_instance(sph_ensemble *e, int32_t i, sph_ctx **ctx) {
    if (!e || !ctx || i < 0 || i >= (int32_t)e->inst.size()) {
        set_error("sph_ensemble_instance: no instance %d", (int)i);
        return SPH_ERR_INVALID_ARG;
    }
    *ctx = e->inst[i];
    return SPH_OK;
}

sph_status sph_ensemble_get_tuning(const sph_ensemble *e, int32_t i, sph_ensemble_tuning *out) {
    if (!e || !out || i < 0 || i >= (int32_t)e->tuning.size()) {
        set_error("sph_ensemble_get_tuning: no instance %d", (int)i);
        return SPH_ERR_INVALID_ARG;
    }
    *out = e->tuning[i];
    return SPH_OK;
}

sph_status sph_ensemble_step(sph_ensemble *e, void *stream, int32_t n_steps) {
    if (!e || n_steps < 0) return SPH_ERR_INVALID_ARG;
    if (n_steps == 0) return SPH_OK;
    cudaSetDevice(e->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (!e->graph) {
        // the first step runs eagerly and puts every sort buffer in its steady
        // role (as sph_step_all does before capturing); then the graph is built
        for (sph_ctx *c : e->inst) {
            sph_status s = full_step(c, st);
            if (s != SPH_OK) return s;
        }
        cudaError_t err = cudaStreamSynchronize(st);
        if (err != cudaSuccess) return cuda_status(err, "ensemble first step");
        sph_status s = build_graph(e);
        if (s != SPH_OK) return s;
        --n_steps;
    }
    for (int32_t k = 0; k < n_steps; ++k) {
        cudaError_t err = cudaGraphLaunch(e->graph, st);
        if (err != cudaSuccess) return cuda_status(err, "ensemble graph launch");
    }
    return SPH_OK;
}

sph_status sph_ensemble_synchronize(sph_ensemble *e, void *stream) {
    if (!e) return SPH_ERR_INVALID_ARG;
    cudaSetDevice(e->device);
    cudaError_t err = cudaStreamSynchronize((cudaStream_t)stream);
    if (err != cudaSuccess) return cuda_status(err, "ensemble synchronize");
    for (sph_ctx *c : e->inst) {
        sph_status s = sph_synchronize(c, stream);
        if (s != SPH_OK) return s;
    }
    return SPH_OK;
}

}  // extern "C"

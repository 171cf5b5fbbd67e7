// Batched fit engine: many resident fit jobs (uneven meshes, resolutions,
// view counts, textures and lobe counts) advanced by one CUDA graph launch.
//
// Each member job runs the fused strategy; its step is captured once as a
// graph (fit_fused_graph) and becomes one child-graph node of the batch
// graph.  The children have no edges between them, so the whole batch is a
// single launch whose independent branches the device schedules
// concurrently: small jobs fill the SMs that a large job's tail leaves idle,
// and the per-kernel launch cost of hundreds of small jobs disappears.  The
// batch graph is rebuilt (one instantiation) only when membership or the
// arithmetic mode changes.  Each job's step counter lives on the device, so
// replaying the graph advances every job by exactly one iteration.
//
// A member may run several iterations per batch step (vcl_batch_set_repeat):
// its step graph appears as a chain of child nodes, so small jobs need not
// advance at the pace of the largest one.
//
// Caller rules: a job may belong to one batch at a time; remove it from the
// batch before destroying it; one host thread drives a batch.
#include <algorithm>
#include <chrono>
#include <vector>

#include "fit.cuh"

struct vcl_batch {
    vcl_ctx* ctx = nullptr;
    std::vector<vcl_fit*> jobs;
    std::vector<int> reps;               // iterations per batch step of each job
    cudaStream_t capture = nullptr;      // stream the member graphs are captured on
    cudaGraphExec_t exec = nullptr;
    bool dirty = true;
    int mode = -1;
    long long rebuilds = 0;
    double rebuild_ms = 0.0;             // host time spent rebuilding the batch graph
};

namespace {

vcl_status rebuild(vcl_batch* b) {
    vcl_ctx* ctx = b->ctx;
    const auto t0 = std::chrono::steady_clock::now();
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    cudaGraph_t parent = nullptr;
    vcl_status st = vcl_cuda_check(ctx, cudaGraphCreate(&parent, 0), "batch graph");
    if (st) return st;
    for (size_t i = 0; i < b->jobs.size() && !st; ++i) {
        cudaGraph_t g = nullptr;
        st = fit_fused_graph(b->jobs[i], b->capture, &g);
        if (st) break;
        // a job with several iterations per step: its step graph repeated as
        // a chain of child nodes
        cudaGraphNode_t prev = nullptr;
        for (int r = 0; r < b->reps[i] && !st; ++r) {
            cudaGraphNode_t node;
            st = vcl_cuda_check(ctx, cudaGraphAddChildGraphNode(&node, parent, prev ? &prev : nullptr, prev ? 1 : 0, g),
                                "batch child graph");
            prev = node;
        }
    }
    if (!st) st = vcl_cuda_check(ctx, cudaGraphInstantiate(&b->exec, parent, 0), "batch graph instantiate");
    cudaGraphDestroy(parent);
    if (st) { b->exec = nullptr; return st; }
    b->dirty = false;
    b->mode = ctx->mode;
    ++b->rebuilds;
    b->rebuild_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return VCL_OK;
}

}  // namespace

extern "C" {

VCL_API vcl_status vcl_batch_create(vcl_ctx* ctx, vcl_batch** out) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(out, "null output");
    *out = nullptr;
    vcl_batch* b = new vcl_batch();
    b->ctx = ctx;
    vcl_status st = vcl_cuda_check(ctx, cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking), "batch stream");
    if (st) { delete b; return st; }
    *out = b;
    return VCL_OK;
}

VCL_API void vcl_batch_destroy(vcl_batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->capture) cudaStreamDestroy(b->capture);
    delete b;
}

VCL_API vcl_status vcl_batch_add(vcl_batch* b, vcl_fit* f) {
    if (!b) return VCL_ERR_ARG;
    vcl_ctx* ctx = b->ctx;
    VCL_REQUIRE(f && f->ctx->device == ctx->device, "job is null or on another device");
    VCL_REQUIRE(std::find(b->jobs.begin(), b->jobs.end(), f) == b->jobs.end(), "job already in the batch");
    vcl_status st = vcl_fit_set_strategy(f, VCL_FIT_FUSED);
    if (st) return st;
    b->jobs.push_back(f);
    b->reps.push_back(1);
    b->dirty = true;
    return VCL_OK;
}

VCL_API vcl_status vcl_batch_remove(vcl_batch* b, vcl_fit* f) {
    if (!b) return VCL_ERR_ARG;
    vcl_ctx* ctx = b->ctx;
    auto it = std::find(b->jobs.begin(), b->jobs.end(), f);
    VCL_REQUIRE(it != b->jobs.end(), "job is not in the batch");
    b->reps.erase(b->reps.begin() + (it - b->jobs.begin()));
    b->jobs.erase(it);
    b->dirty = true;
    return VCL_OK;
}

VCL_API vcl_status vcl_batch_set_repeat(vcl_batch* b, vcl_fit* f, int iterations) {
    if (!b) return VCL_ERR_ARG;
    vcl_ctx* ctx = b->ctx;
    VCL_REQUIRE(iterations >= 1 && iterations <= 64, "iterations per step must be 1..64 (got %d)", iterations);
    auto it = std::find(b->jobs.begin(), b->jobs.end(), f);
    VCL_REQUIRE(it != b->jobs.end(), "job is not in the batch");
    int& r = b->reps[it - b->jobs.begin()];
    if (r != iterations) {
        r = iterations;
        b->dirty = true;
    }
    return VCL_OK;
}

VCL_API int vcl_batch_size(const vcl_batch* b) { return b ? (int)b->jobs.size() : 0; }

VCL_API vcl_status vcl_batch_step(vcl_batch* b, void* stream) {
    if (!b) return VCL_ERR_ARG;
    vcl_ctx* ctx = b->ctx;
    cudaStream_t s = (cudaStream_t)stream;
    if (b->jobs.empty()) return VCL_OK;
    bool stale = b->dirty || b->mode != ctx->mode;
    for (const vcl_fit* f : b->jobs) stale = stale || f->ctx->mode != ctx->mode;
    if (stale) {
        vcl_status st = rebuild(b);
        if (st) return st;
    }
    vcl_status st = vcl_cuda_check(ctx, cudaGraphLaunch(b->exec, s), "batch launch");
    if (st) return st;
    for (size_t i = 0; i < b->jobs.size(); ++i) b->jobs[i]->step_count += b->reps[i];
    return VCL_OK;
}

VCL_API vcl_status vcl_batch_rebuild_stats(const vcl_batch* b, long long* rebuilds, double* host_ms) {
    if (!b) return VCL_ERR_ARG;
    if (rebuilds) *rebuilds = b->rebuilds;
    if (host_ms) *host_ms = b->rebuild_ms;
    return VCL_OK;
}

VCL_API int vcl_batch_launches_per_step(const vcl_batch* b) {
    if (!b) return 0;
    int n = 0;
    for (size_t i = 0; i < b->jobs.size(); ++i) n += b->reps[i] * fit_fused_launches(b->jobs[i]);
    return n;
}

}  // extern "C"

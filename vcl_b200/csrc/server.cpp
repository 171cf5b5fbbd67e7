// Serving loop for inverse-rendering fit jobs, built on the public C ABI
// (vcl_fit_* and vcl_batch_*).
//
//   submit   copies the job's host arrays and target images, queues it
//            (FIFO) with its iteration count;
//   tick     1. retires the jobs whose last iteration ran in a tick that
//               has been seen to complete: optional copy of the final
//               parameters, the job's device memory released (its
//               completion time was stamped when the tick was seen done);
//            2. admits queued jobs in arrival order while their device
//               footprint (vcl_fit_footprint) fits the remaining budget and
//               a live slot is free -- the job's mesh, texture pyramid,
//               lobes, Adam moments and per-view buffers become resident;
//            3. advances every live job by one iteration with ONE batched
//               launch (vcl_batch_step) and records an event;
//            4. waits for the PREVIOUS tick's event, so that one tick is
//               always queued behind the running one (continuous batching:
//               the device never waits for the host in steady state).
// Jobs that arrive while others run join at the next tick; finished jobs
// leave the batch before the next launch.  Latency = completion - submit on
// the host's steady clock.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "vcl.h"

namespace {

using Clock = std::chrono::steady_clock;

enum JobState { QUEUED = 0, LIVE = 1, DONE = 2, FAILED = 3 };

struct Job {
    long long id = 0;
    vcl_fit_desc d{};
    std::vector<float> pos, uv, normal, tex, axis, sharp, amp, mvp, pvinv, rot, target;
    std::vector<uint32_t> tri;
    int iters = 0, done = 0;
    size_t footprint = 0;
    double t_submit = 0, t_admit = -1, t_done = -1;
    int state = QUEUED;
    bool keep = false;
    vcl_fit* fit = nullptr;
    std::string error;
    // final parameters (when keep)
    std::vector<float> r_pos, r_tex, r_axis, r_sharp, r_amp;
    float loss = 0.f;
};

template <class T>
std::vector<T> copy_of(const T* p, size_t n) {
    return p ? std::vector<T>(p, p + n) : std::vector<T>();
}

}  // namespace

struct vcl_server {
    vcl_ctx* ctx = nullptr;
    vcl_batch* batch = nullptr;
    size_t budget = 0, used = 0;
    int max_live = 0;
    long long next_id = 1;
    std::deque<Job*> queue;
    std::vector<Job*> live;
    // jobs whose last iteration has been launched, with that tick's index
    std::vector<std::pair<Job*, long long>> finishing;
    std::map<long long, std::unique_ptr<Job>> jobs;
    cudaStream_t aux = nullptr;          // result readback
    cudaEvent_t ev[2] = {nullptr, nullptr};   // completion of tick t is ev[t & 1]
    Clock::time_point t0;
    long long iters_total = 0;
    long long ticks = 0;        // ticks launched
    long long done_tick = -1;   // highest tick known to have completed
    std::vector<double> latencies;
    std::string err;

    double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
};

namespace {

vcl_status fail(vcl_server* s, vcl_status code, const std::string& msg) {
    s->err = msg;
    return code;
}

vcl_status fit_error(vcl_server* s, vcl_status st, const char* what) {
    s->err = std::string(what) + ": " + vcl_last_error(s->ctx);
    return st;
}

vcl_status retire(vcl_server* s, Job* j) {
    vcl_status st = VCL_OK;
    if (j->keep) {
        const vcl_fit_desc& d = j->d;
        j->r_pos.resize((size_t)d.nv * 3);
        j->r_tex.resize((size_t)d.tex_w * d.tex_h * d.C);
        j->r_axis.resize((size_t)d.K * 3);
        j->r_sharp.resize((size_t)d.K);
        j->r_amp.resize((size_t)d.K * d.C);
        st = vcl_fit_read_params(j->fit, j->r_pos.data(), j->r_tex.data(), j->r_axis.data(), j->r_sharp.data(),
                                 j->r_amp.data(), s->aux);
        if (!st) st = vcl_fit_read_loss(j->fit, &j->loss, s->aux);
        if (st) fit_error(s, st, "job result readback");
    }
    vcl_fit_destroy(j->fit);
    j->fit = nullptr;
    s->used -= j->footprint;
    j->state = st ? FAILED : DONE;
    if (!st) s->latencies.push_back(j->t_done - j->t_submit);
    return st;
}

vcl_status admit(vcl_server* s, Job* j) {
    vcl_fit* f = nullptr;
    vcl_status st = vcl_fit_create(s->ctx, &j->d, &f);
    if (st) {
        j->state = FAILED;
        j->error = vcl_last_error(s->ctx);
        return VCL_OK;   // the job fails; the server keeps going
    }
    st = vcl_fit_set_target(f, j->target.data(), 0, s->aux);
    if (!st) st = vcl_batch_add(s->batch, f);
    if (!st) st = cudaStreamSynchronize(s->aux) == cudaSuccess ? VCL_OK : VCL_ERR_CUDA;
    if (st) {
        j->state = FAILED;
        j->error = vcl_last_error(s->ctx);
        vcl_fit_destroy(f);
        return VCL_OK;
    }
    // host copies are no longer needed once the job is resident
    j->target.clear(); j->target.shrink_to_fit();
    j->tex.clear(); j->tex.shrink_to_fit();
    j->fit = f;
    j->state = LIVE;
    j->t_admit = s->now_ms();
    s->used += j->footprint;
    s->live.push_back(j);
    return VCL_OK;
}

}  // namespace

extern "C" {

VCL_API vcl_status vcl_server_create(vcl_ctx* ctx, size_t budget_bytes, int max_live, vcl_server** out) {
    if (!ctx || !out || max_live <= 0 || budget_bytes == 0) return VCL_ERR_ARG;
    *out = nullptr;
    auto* s = new vcl_server();
    s->ctx = ctx;
    s->budget = budget_bytes;
    s->max_live = max_live;
    vcl_status st = vcl_batch_create(ctx, &s->batch);
    if (!st && cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking) != cudaSuccess) st = VCL_ERR_CUDA;
    for (int i = 0; i < 2 && !st; ++i)
        if (cudaEventCreateWithFlags(&s->ev[i], cudaEventDisableTiming) != cudaSuccess) st = VCL_ERR_CUDA;
    if (st) {
        if (s->batch) vcl_batch_destroy(s->batch);
        delete s;
        return st;
    }
    s->t0 = Clock::now();
    *out = s;
    return VCL_OK;
}

VCL_API void vcl_server_destroy(vcl_server* s) {
    if (!s) return;
    cudaDeviceSynchronize();
    for (Job* j : s->live) {
        vcl_batch_remove(s->batch, j->fit);
        vcl_fit_destroy(j->fit);
    }
    for (auto& p : s->finishing) if (p.first->fit) vcl_fit_destroy(p.first->fit);
    vcl_batch_destroy(s->batch);
    if (s->aux) cudaStreamDestroy(s->aux);
    for (auto& e : s->ev) if (e) cudaEventDestroy(e);
    delete s;
}

VCL_API const char* vcl_server_last_error(const vcl_server* s) { return s ? s->err.c_str() : "null server"; }

VCL_API vcl_status vcl_server_submit(vcl_server* s, const vcl_fit_desc* desc, const float* target, int iterations,
                                     int keep_result, long long* job_id) {
    if (!s) return VCL_ERR_ARG;
    if (!desc || !target || iterations <= 0 || !job_id) return fail(s, VCL_ERR_ARG, "submit: bad arguments");
    const vcl_fit_desc& d = *desc;
    if (d.W <= 0 || d.H <= 0 || d.views <= 0 || d.nv <= 0 || d.nt <= 0 || d.C != 4 || d.K < 0 || d.tex_w <= 0 ||
        d.tex_h <= 0 || d.levels < 1)
        return fail(s, VCL_ERR_ARG, "submit: bad job sizes (the batched engine needs C = 4)");
    if (!d.pos || !d.tri || !d.uv || !d.normal || !d.tex || !d.mvp || !d.pvinv || !d.rot ||
        (d.K && (!d.lobe_axis || !d.lobe_sharp || !d.lobe_amp)))
        return fail(s, VCL_ERR_ARG, "submit: null host array");
    auto j = std::make_unique<Job>();
    j->id = s->next_id++;
    j->d = d;
    j->pos = copy_of(d.pos, (size_t)d.nv * 3);
    j->tri = copy_of(d.tri, (size_t)d.nt * 3);
    j->uv = copy_of(d.uv, (size_t)d.nv * 2);
    j->normal = copy_of(d.normal, (size_t)d.nv * 3);
    j->tex = copy_of(d.tex, (size_t)d.tex_w * d.tex_h * d.C);
    j->axis = copy_of(d.lobe_axis, (size_t)d.K * 3);
    j->sharp = copy_of(d.lobe_sharp, (size_t)d.K);
    j->amp = copy_of(d.lobe_amp, (size_t)d.K * d.C);
    j->mvp = copy_of(d.mvp, (size_t)d.views * 16);
    j->pvinv = copy_of(d.pvinv, (size_t)d.views * 9);
    j->rot = copy_of(d.rot, 16);
    j->target = copy_of(target, (size_t)d.W * d.H * d.views * d.C);
    j->d.pos = j->pos.data(); j->d.tri = j->tri.data(); j->d.uv = j->uv.data(); j->d.normal = j->normal.data();
    j->d.tex = j->tex.data(); j->d.lobe_axis = j->axis.data(); j->d.lobe_sharp = j->sharp.data();
    j->d.lobe_amp = j->amp.data(); j->d.mvp = j->mvp.data(); j->d.pvinv = j->pvinv.data(); j->d.rot = j->rot.data();
    j->iters = iterations;
    j->keep = keep_result != 0;
    j->footprint = vcl_fit_footprint(&j->d);
    j->t_submit = s->now_ms();
    if (j->footprint > s->budget) {
        j->state = FAILED;
        j->error = "job footprint exceeds the device budget";
    } else {
        s->queue.push_back(j.get());
    }
    *job_id = j->id;
    s->jobs[j->id] = std::move(j);
    return VCL_OK;
}

namespace {

// Waits for tick `t` and stamps the completion time of the jobs that ended in
// it or earlier.
vcl_status observe(vcl_server* s, long long t) {
    if (t <= s->done_tick) return VCL_OK;
    if (cudaEventSynchronize(s->ev[t & 1]) != cudaSuccess) return fail(s, VCL_ERR_CUDA, "tick wait");
    s->done_tick = t;
    const double now = s->now_ms();
    for (auto& p : s->finishing)
        if (p.second <= t && p.first->t_done < 0) p.first->t_done = now;
    return VCL_OK;
}

}  // namespace

VCL_API vcl_status vcl_server_tick(vcl_server* s, void* stream, int* live_out, int* completed_out) {
    if (!s) return VCL_ERR_ARG;
    cudaStream_t cs = (cudaStream_t)stream;
    int completed = 0;
    vcl_status st = VCL_OK;
    // 1. retire the jobs whose last tick is known to have completed
    std::vector<std::pair<Job*, long long>> keep;
    for (auto& p : s->finishing) {
        if (p.second <= s->done_tick) {
            vcl_status r = retire(s, p.first);
            if (r && !st) st = r;
            ++completed;
        } else {
            keep.push_back(p);
        }
    }
    s->finishing.swap(keep);
    // 2. admission, in arrival order
    while (!s->queue.empty() && (int)s->live.size() < s->max_live &&
           s->used + s->queue.front()->footprint <= s->budget) {
        Job* j = s->queue.front();
        s->queue.pop_front();
        vcl_status r = admit(s, j);
        if (r) return fit_error(s, r, "admission");
    }
    // 3. one batched iteration of every live job
    if (!s->live.empty()) {
        const long long t = s->ticks;
        vcl_status r = vcl_batch_step(s->batch, cs);
        if (r) return fit_error(s, r, "batch step");
        if (cudaEventRecord(s->ev[t & 1], cs) != cudaSuccess) return fail(s, VCL_ERR_CUDA, "tick event");
        ++s->ticks;
        s->iters_total += (long long)s->live.size();
        std::vector<Job*> still;
        for (Job* j : s->live) {
            if (++j->done >= j->iters) {
                vcl_batch_remove(s->batch, j->fit);
                s->finishing.push_back({j, t});
            } else {
                still.push_back(j);
            }
        }
        s->live.swap(still);
        // 4. wait for the previous tick; this one stays queued behind it
        if (t >= 1) {
            r = observe(s, t - 1);
            if (r) return r;
        }
    } else if (s->ticks > 0) {
        vcl_status r = observe(s, s->ticks - 1);
        if (r) return r;
    }
    if (live_out) *live_out = (int)s->live.size();
    if (completed_out) *completed_out = completed;
    return st;
}

/* Runs ticks until every submitted job has finished (or failed). */
VCL_API vcl_status vcl_server_drain(vcl_server* s, void* stream) {
    if (!s) return VCL_ERR_ARG;
    for (;;) {
        int live = 0;
        vcl_status st = vcl_server_tick(s, stream, &live, nullptr);
        if (st) return st;
        if (live == 0 && s->queue.empty() && s->finishing.empty() && s->done_tick == s->ticks - 1) return VCL_OK;
    }
}

VCL_API double vcl_server_now_ms(const vcl_server* s) { return s ? s->now_ms() : 0.0; }

VCL_API int vcl_server_pending(const vcl_server* s) {
    if (!s) return 0;
    return (int)(s->queue.size() + s->live.size() + s->finishing.size());
}

VCL_API vcl_status vcl_server_job_status(const vcl_server* s, long long id, int* state, int* iters_done,
                                         double* submit_ms, double* admit_ms, double* done_ms) {
    if (!s) return VCL_ERR_ARG;
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return VCL_ERR_ARG;
    const Job* j = it->second.get();
    if (state) *state = j->state;
    if (iters_done) *iters_done = j->done;
    if (submit_ms) *submit_ms = j->t_submit;
    if (admit_ms) *admit_ms = j->t_admit;
    if (done_ms) *done_ms = j->t_done;
    return VCL_OK;
}

VCL_API vcl_status vcl_server_job_result(const vcl_server* s, long long id, float* pos, float* tex_level0,
                                         float* lobe_axis, float* lobe_sharp, float* lobe_amp, float* loss) {
    if (!s) return VCL_ERR_ARG;
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return VCL_ERR_ARG;
    const Job* j = it->second.get();
    if (j->state != DONE || !j->keep) return VCL_ERR_STATE;
    auto cp = [](float* dst, const std::vector<float>& v) { if (dst) std::memcpy(dst, v.data(), v.size() * 4); };
    cp(pos, j->r_pos); cp(tex_level0, j->r_tex); cp(lobe_axis, j->r_axis); cp(lobe_sharp, j->r_sharp);
    cp(lobe_amp, j->r_amp);
    if (loss) *loss = j->loss;
    return VCL_OK;
}

/* Latency percentiles (ms, nearest rank) over completed jobs, total
 * iterations run, completed jobs, ticks, bytes resident now. */
VCL_API vcl_status vcl_server_stats(const vcl_server* s, double* p50_ms, double* p99_ms, long long* iterations,
                                    int* completed, long long* ticks, size_t* resident_bytes) {
    if (!s) return VCL_ERR_ARG;
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) {
        if (l.empty()) return 0.0;
        size_t k = (size_t)(q * (double)l.size() + 0.999999);
        if (k < 1) k = 1;
        if (k > l.size()) k = l.size();
        return l[k - 1];
    };
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    if (iterations) *iterations = s->iters_total;
    if (completed) *completed = (int)s->latencies.size();
    if (ticks) *ticks = s->ticks;
    if (resident_bytes) *resident_bytes = s->used;
    return VCL_OK;
}

}  // extern "C"

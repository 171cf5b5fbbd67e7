// Serving loop for inverse-rendering fit jobs, built on the public C ABI
// (vcl_fit_* and vcl_batch_*).
//
//   submit   copies the job's host arrays and target images and queues it
//            (FIFO) with its iteration count;
//   tick     1. retires the jobs whose last iteration ran in a tick that
//               has been seen to complete: optional copy of the final
//               parameters, the job's device memory returned in stream order
//               (its completion time was stamped when the tick was seen);
//            2. admits queued jobs in arrival order while their device
//               footprint (vcl_fit_footprint) fits the remaining budget and a
//               slot is free, reserving the footprint and handing the job to
//               the set-up worker;
//            3. moves the jobs the worker has set up into the batch;
//            4. advances every live job with ONE batched launch
//               (vcl_batch_step) -- one iteration for the largest jobs, up
//               to 8 for jobs with a fraction of their pixels -- and records
//               an event;
//            5. waits for the PREVIOUS tick's event, so that one tick is
//               always queued behind the running one.
//   worker   a host thread with its own context on the same device: creates
//            the job's resident state (mesh, texture pyramid, lobes, Adam
//            moments, per-view buffers), uploads its target, tunes its
//            raster schedule and captures its step graph, all on its own
//            streams, while the tick loop keeps the device busy.
// Jobs that arrive while others run join at a later tick (continuous
// batching); finished jobs leave the batch before the next launch.  Latency
// = completion - submission on the host's steady clock.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
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
    int rep = 1;                     // iterations per tick
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
    vcl_ctx* ctx = nullptr;          // the caller's context: batch and ticks
    vcl_ctx* wctx = nullptr;         // the set-up worker's context
    int device = 0;
    vcl_batch* batch = nullptr;
    size_t budget = 0, used = 0;     // bytes reserved by admitted jobs
    int max_live = 0;
    long long next_id = 1;
    std::deque<Job*> queue;          // submitted, not admitted
    std::vector<Job*> live;          // in the batch
    int in_setup = 0;                // admitted, handed to the worker, not live yet
    // jobs whose last iteration has been launched, with that tick's index
    std::vector<std::pair<Job*, long long>> finishing;
    std::map<long long, std::unique_ptr<Job>> jobs;
    cudaStream_t aux = nullptr;      // result readback
    cudaEvent_t ev[2] = {nullptr, nullptr};   // completion of tick t is ev[t & 1]
    Clock::time_point t0;
    long long iters_total = 0;
    long long ticks = 0;             // ticks launched
    long long done_tick = -1;        // highest tick known to have completed
    double host_ms = 0.0;            // host time inside ticks, waits excluded
    double wait_ms = 0.0;            // host time waiting for the previous tick
    std::vector<double> latencies;
    std::string err;
    // set-up worker
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job*> to_setup;       // guarded by mu
    std::deque<Job*> set_up;         // guarded by mu: ready (or failed) jobs
    bool stop = false;               // guarded by mu

    double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
};

namespace {

constexpr int MAX_REPEAT = 8;

// Relative device work of one iteration: pixels, plus a constant for the
// per-iteration launches of a small job.
double job_cost(const vcl_fit_desc& d) { return (double)d.W * d.H * d.views + 65536.0; }

vcl_status fail(vcl_server* s, vcl_status code, const std::string& msg) {
    s->err = msg;
    return code;
}

vcl_status fit_error(vcl_server* s, vcl_ctx* ctx, vcl_status st, const char* what) {
    s->err = std::string(what) + ": " + vcl_last_error(ctx);
    return st;
}

// Worker: resident state, target upload, raster tuning and graph capture of
// one job, on the worker's own context and stream.
void set_up_job(vcl_server* s, Job* j, cudaStream_t ws) {
    vcl_fit* f = nullptr;
    vcl_status st = vcl_fit_create(s->wctx, &j->d, &f);
    if (!st) st = vcl_fit_set_target(f, j->target.data(), 0, ws);
    if (!st) st = vcl_fit_set_strategy(f, VCL_FIT_FUSED);
    if (!st) st = vcl_fit_prepare(f, ws);
    if (!st && cudaStreamSynchronize(ws) != cudaSuccess) st = VCL_ERR_CUDA;
    if (st) {
        j->error = vcl_last_error(s->wctx);
        if (f) vcl_fit_destroy(f);
        j->state = FAILED;
        return;
    }
    j->target.clear(); j->target.shrink_to_fit();
    j->tex.clear(); j->tex.shrink_to_fit();
    j->fit = f;
}

void worker_main(vcl_server* s) {
    cudaSetDevice(s->device);
    cudaStream_t ws = nullptr;
    cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking);
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [&] { return s->stop || !s->to_setup.empty(); });
            if (s->stop) break;
            j = s->to_setup.front();
            s->to_setup.pop_front();
        }
        set_up_job(s, j, ws);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->set_up.push_back(j);
        }
        s->cv.notify_all();
    }
    if (ws) cudaStreamDestroy(ws);
}

vcl_status retire(vcl_server* s, Job* j, cudaStream_t cs) {
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
        if (st) fit_error(s, s->wctx, st, "job result readback");
    }
    // stream-ordered release: no device synchronization in the tick loop
    vcl_fit_destroy_async(j->fit, cs);
    j->fit = nullptr;
    s->used -= j->footprint;
    j->state = st ? FAILED : DONE;
    if (!st) s->latencies.push_back(j->t_done - j->t_submit);
    return st;
}

// Moves the jobs the worker finished into the batch (or releases a failed
// job's reservation).  `wait`: block until at least one arrives.
vcl_status collect(vcl_server* s, bool wait) {
    std::deque<Job*> ready;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        if (wait) s->cv.wait(lk, [&] { return !s->set_up.empty(); });
        ready.swap(s->set_up);
    }
    for (Job* j : ready) {
        --s->in_setup;
        if (j->state == FAILED) {
            s->used -= j->footprint;
            continue;
        }
        vcl_status st = vcl_batch_add(s->batch, j->fit);
        if (st) return fit_error(s, s->ctx, st, "batch add");
        j->state = LIVE;
        j->t_admit = s->now_ms();
        s->live.push_back(j);
    }
    return VCL_OK;
}

// Waits for tick `t` and stamps the completion time of the jobs that ended in
// it or earlier.
vcl_status observe(vcl_server* s, long long t) {
    if (t <= s->done_tick) return VCL_OK;
    const double w0 = s->now_ms();
    if (cudaEventSynchronize(s->ev[t & 1]) != cudaSuccess) return fail(s, VCL_ERR_CUDA, "tick wait");
    s->wait_ms += s->now_ms() - w0;
    s->done_tick = t;
    const double now = s->now_ms();
    for (auto& p : s->finishing)
        if (p.second <= t && p.first->t_done < 0) p.first->t_done = now;
    return VCL_OK;
}

}  // namespace

extern "C" {

VCL_API vcl_status vcl_server_create(vcl_ctx* ctx, size_t budget_bytes, int max_live, vcl_server** out) {
    if (!ctx || !out || max_live <= 0 || budget_bytes == 0) return VCL_ERR_ARG;
    *out = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return VCL_ERR_CUDA;
    auto* s = new vcl_server();
    s->ctx = ctx;
    s->device = dev;
    s->budget = budget_bytes;
    s->max_live = max_live;
    vcl_status st = vcl_batch_create(ctx, &s->batch);
    if (!st) st = vcl_create(dev, &s->wctx);
    if (!st) st = vcl_set_mode(s->wctx, vcl_get_mode(ctx));
    // jobs are set up while other jobs run: timing raster schedules then
    // measures the other jobs, so the worker uses the size-based schedule
    if (!st) st = vcl_set_raster_autotune(s->wctx, 0);
    if (!st && cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking) != cudaSuccess) st = VCL_ERR_CUDA;
    for (int i = 0; i < 2 && !st; ++i)
        if (cudaEventCreateWithFlags(&s->ev[i], cudaEventDisableTiming) != cudaSuccess) st = VCL_ERR_CUDA;
    if (st) {
        if (s->batch) vcl_batch_destroy(s->batch);
        if (s->wctx) vcl_destroy(s->wctx);
        delete s;
        return st;
    }
    s->t0 = Clock::now();
    s->worker = std::thread(worker_main, s);
    *out = s;
    return VCL_OK;
}

VCL_API void vcl_server_destroy(vcl_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaDeviceSynchronize();
    for (Job* j : s->live) {
        vcl_batch_remove(s->batch, j->fit);
        vcl_fit_destroy(j->fit);
    }
    for (auto& p : s->finishing) if (p.first->fit) vcl_fit_destroy(p.first->fit);
    for (Job* j : s->set_up) if (j->fit) vcl_fit_destroy(j->fit);
    vcl_batch_destroy(s->batch);
    if (s->aux) cudaStreamDestroy(s->aux);
    for (auto& e : s->ev) if (e) cudaEventDestroy(e);
    vcl_destroy(s->wctx);
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

vcl_status tick_impl(vcl_server* s, void* stream, int* live_out, int* completed_out);

VCL_API vcl_status vcl_server_tick(vcl_server* s, void* stream, int* live_out, int* completed_out) {
    if (!s) return VCL_ERR_ARG;
    const double t0 = s->now_ms(), w0 = s->wait_ms;
    vcl_status st = tick_impl(s, stream, live_out, completed_out);
    s->host_ms += (s->now_ms() - t0) - (s->wait_ms - w0);
    return st;
}

vcl_status tick_impl(vcl_server* s, void* stream, int* live_out, int* completed_out) {
    cudaStream_t cs = (cudaStream_t)stream;
    int completed = 0;
    vcl_status st = VCL_OK;
    // 1. retire the jobs whose last tick is known to have completed
    std::vector<std::pair<Job*, long long>> keep;
    for (auto& p : s->finishing) {
        if (p.second <= s->done_tick) {
            vcl_status r = retire(s, p.first, cs);
            if (r && !st) st = r;
            ++completed;
        } else {
            keep.push_back(p);
        }
    }
    s->finishing.swap(keep);
    // 2. admission in arrival order: reserve the footprint, hand to the worker
    int handed = 0;
    while (!s->queue.empty() && (int)s->live.size() + s->in_setup < s->max_live &&
           s->used + s->queue.front()->footprint <= s->budget) {
        Job* j = s->queue.front();
        s->queue.pop_front();
        s->used += j->footprint;
        ++s->in_setup;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->to_setup.push_back(j);
        }
        ++handed;
    }
    if (handed) s->cv.notify_all();
    // 3. jobs set up since the last tick join the batch; with nothing live and
    //    nothing in flight, wait for the worker instead of spinning
    const bool idle = s->live.empty() && s->in_setup > 0 && s->done_tick == s->ticks - 1;
    vcl_status r = collect(s, idle);
    if (r) return r;
    // 4. one batched launch advances every live job; a job whose per-pixel
    //    work is a fraction of the largest live job's runs several
    //    iterations in it (at most MAX_REPEAT, never past its count)
    if (!s->live.empty()) {
        double big = 0.0;
        for (Job* j : s->live) big = std::max(big, job_cost(j->d));
        for (Job* j : s->live) {
            int k = (int)std::min<double>(MAX_REPEAT, std::max(1.0, std::floor(big / job_cost(j->d))));
            k = std::min(k, j->iters - j->done);
            if (k != j->rep) {
                r = vcl_batch_set_repeat(s->batch, j->fit, k);
                if (r) return fit_error(s, s->ctx, r, "batch repeat");
                j->rep = k;
            }
        }
        const long long t = s->ticks;
        r = vcl_batch_step(s->batch, cs);
        if (r) return fit_error(s, s->ctx, r, "batch step");
        if (cudaEventRecord(s->ev[t & 1], cs) != cudaSuccess) return fail(s, VCL_ERR_CUDA, "tick event");
        ++s->ticks;
        std::vector<Job*> still;
        for (Job* j : s->live) {
            s->iters_total += j->rep;
            if ((j->done += j->rep) >= j->iters) {
                vcl_batch_remove(s->batch, j->fit);
                s->finishing.push_back({j, t});
            } else {
                still.push_back(j);
            }
        }
        s->live.swap(still);
        // 5. wait for the previous tick; this one stays queued behind it
        if (t >= 1) {
            r = observe(s, t - 1);
            if (r) return r;
        }
    } else if (s->ticks > 0) {
        r = observe(s, s->ticks - 1);
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
        if (live == 0 && s->queue.empty() && s->in_setup == 0 && s->finishing.empty() &&
            s->done_tick == s->ticks - 1)
            return VCL_OK;
    }
}

VCL_API double vcl_server_now_ms(const vcl_server* s) { return s ? s->now_ms() : 0.0; }

VCL_API vcl_status vcl_server_host_stats(const vcl_server* s, double* host_ms, double* wait_ms, long long* rebuilds,
                                         double* rebuild_ms) {
    if (!s) return VCL_ERR_ARG;
    if (host_ms) *host_ms = s->host_ms;
    if (wait_ms) *wait_ms = s->wait_ms;
    return vcl_batch_rebuild_stats(s->batch, rebuilds, rebuild_ms);
}

VCL_API int vcl_server_pending(const vcl_server* s) {
    if (!s) return 0;
    return (int)(s->queue.size() + s->live.size() + s->finishing.size()) + s->in_setup;
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
 * iterations run, completed jobs, ticks, bytes reserved now. */
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

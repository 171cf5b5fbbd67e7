/*
 * vcl.hpp -- header-only C++17 layer over the C ABI of vcl.h.
 *
 * The reference's callers are C++ (PresetPrimitives::init/update,
 * preset_primitives.cpp:7-230, over static operator classes); this header
 * gives such a caller RAII owners and exceptions instead of raw handles and
 * status codes:
 *
 *   vcl::Context ctx(0);                         // vcl_create / vcl_destroy
 *   ctx.call(vcl_rasterize_fwd, clip, nv, tri, nt, W, H, views, rast, db, stream);
 *   vcl::Pipeline fit(ctx, desc, VCL_FIT_FUSED);  // the preset wiring as one object
 *   fit.step(stream);  float loss = fit.read_loss(stream);
 *
 * Every failing call throws vcl::Error with the library's message.  Nothing
 * here adds state or work: each method is one C call.
 */
#ifndef VCL_HPP
#define VCL_HPP

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "vcl.h"

namespace vcl {

class Error : public std::runtime_error {
public:
    Error(vcl_status status, const std::string& what) : std::runtime_error(what), status_(status) {}
    vcl_status status() const { return status_; }

private:
    vcl_status status_;
};

namespace detail {
template <class T, void (*Destroy)(T*)>
class Handle {
public:
    Handle() = default;
    explicit Handle(T* p) : p_(p) {}
    Handle(const Handle&) = delete;
    Handle& operator=(const Handle&) = delete;
    Handle(Handle&& o) noexcept : p_(std::exchange(o.p_, nullptr)) {}
    Handle& operator=(Handle&& o) noexcept {
        if (this != &o) {
            reset();
            p_ = std::exchange(o.p_, nullptr);
        }
        return *this;
    }
    ~Handle() { reset(); }
    void reset() {
        if (p_) Destroy(p_);
        p_ = nullptr;
    }
    T* get() const { return p_; }

private:
    T* p_ = nullptr;
};
}  // namespace detail

// One vcl_ctx: device, arithmetic mode, raster configuration, workspace.
class Context {
public:
    explicit Context(int device = 0, int mode = VCL_MODE_COMPAT) {
        vcl_ctx* c = nullptr;
        const vcl_status st = vcl_create(device, &c);
        if (st != VCL_OK) {
            if (c) vcl_destroy(c);
            throw Error(st, "vcl_create(device " + std::to_string(device) + ") failed");
        }
        h_ = detail::Handle<vcl_ctx, vcl_destroy>(c);
        set_mode(mode);
    }
    vcl_ctx* get() const { return h_.get(); }

    // Throws for a failed status, with the context's last message.
    void check(vcl_status st, const char* what) const {
        if (st == VCL_OK) return;
        const char* m = vcl_last_error(h_.get());
        throw Error(st, std::string(what) + ": " + (m ? m : ""));
    }
    // Any operator of vcl.h: ctx.call(vcl_texture_fwd, rast, uv, ...).
    template <class... Fn, class... A>
    void call(vcl_status (*fn)(vcl_ctx*, Fn...), A&&... args) const {
        check(fn(h_.get(), std::forward<A>(args)...), "vcl call");
    }

    void set_mode(int mode) { check(vcl_set_mode(h_.get(), mode), "vcl_set_mode"); }
    int mode() const { return vcl_get_mode(h_.get()); }
    void set_raster_config(int tile, long long bin_capacity = 0) {
        check(vcl_set_raster_config(h_.get(), tile, bin_capacity), "vcl_set_raster_config");
    }
    void set_raster_autotune(bool enable) {
        check(vcl_set_raster_autotune(h_.get(), enable ? 1 : 0), "vcl_set_raster_autotune");
    }
    int check_indices(void* stream = nullptr) const {
        int n = 0;
        check(vcl_check_indices(h_.get(), stream, &n), "vcl_check_indices");
        return n;
    }

private:
    detail::Handle<vcl_ctx, vcl_destroy> h_;
};

// The reference's PresetPrimitives wiring as one resident job (vcl_fit_*).
class Pipeline {
public:
    Pipeline(const Context& ctx, const vcl_fit_desc& desc, int strategy = VCL_FIT_FUSED) : ctx_(&ctx) {
        vcl_fit* f = nullptr;
        ctx.check(vcl_fit_create(ctx.get(), &desc, &f), "vcl_fit_create");
        h_ = detail::Handle<vcl_fit, vcl_fit_destroy>(f);
        set_strategy(strategy);
    }
    vcl_fit* get() const { return h_.get(); }
    static size_t footprint(const vcl_fit_desc& desc) { return vcl_fit_footprint(&desc); }

    void set_strategy(int strategy) { chk(vcl_fit_set_strategy(h_.get(), strategy), "vcl_fit_set_strategy"); }
    void set_target(const float* src, bool src_is_device, void* stream = nullptr) {
        chk(vcl_fit_set_target(h_.get(), src, src_is_device ? 1 : 0, stream), "vcl_fit_set_target");
    }
    void stage_target(const float* host_src, void* copy_stream) {
        chk(vcl_fit_stage_target(h_.get(), host_src, copy_stream), "vcl_fit_stage_target");
    }
    void set_cameras(const float* mvp, const float* pvinv, void* stream = nullptr) {
        chk(vcl_fit_set_cameras(h_.get(), mvp, pvinv, stream), "vcl_fit_set_cameras");
    }
    void prepare(void* stream) { chk(vcl_fit_prepare(h_.get(), stream), "vcl_fit_prepare"); }
    void step(void* stream = nullptr) { chk(vcl_fit_step(h_.get(), stream), "vcl_fit_step"); }
    void render(float* out, void* stream = nullptr) { chk(vcl_fit_render(h_.get(), out, stream), "vcl_fit_render"); }
    const float* loss_device() const { return vcl_fit_loss_device(h_.get()); }
    float read_loss(void* stream = nullptr) {
        float l = 0.f;
        chk(vcl_fit_read_loss(h_.get(), &l, stream), "vcl_fit_read_loss");
        return l;
    }
    // Queues the loss copy into pinned host memory without waiting.
    void read_loss_async(float* pinned_dst, void* stream = nullptr) {
        chk(vcl_fit_read_loss_async(h_.get(), pinned_dst, stream), "vcl_fit_read_loss_async");
    }
    void read_params(float* pos, float* tex_level0, float* lobe_axis, float* lobe_sharp, float* lobe_amp,
                     void* stream = nullptr) {
        chk(vcl_fit_read_params(h_.get(), pos, tex_level0, lobe_axis, lobe_sharp, lobe_amp, stream),
            "vcl_fit_read_params");
    }
    int launches_per_step() const { return vcl_fit_launches_per_step(h_.get()); }
    // Checkpoint / resume: parameters, Adam moments and step as bytes.
    std::vector<unsigned char> save_state(void* stream = nullptr) {
        std::vector<unsigned char> buf(vcl_fit_state_bytes(h_.get()));
        chk(vcl_fit_save_state(h_.get(), buf.data(), buf.size(), stream), "vcl_fit_save_state");
        return buf;
    }
    void load_state(const std::vector<unsigned char>& buf, void* stream = nullptr) {
        chk(vcl_fit_load_state(h_.get(), buf.data(), buf.size(), stream), "vcl_fit_load_state");
    }

private:
    void chk(vcl_status st, const char* what) const { ctx_->check(st, what); }
    const Context* ctx_;
    detail::Handle<vcl_fit, vcl_fit_destroy> h_;
};

// Many resident jobs advanced by one graph launch (vcl_batch_*).  The
// pipelines must outlive their membership.
class Batch {
public:
    explicit Batch(const Context& ctx) : ctx_(&ctx) {
        vcl_batch* b = nullptr;
        ctx.check(vcl_batch_create(ctx.get(), &b), "vcl_batch_create");
        h_ = detail::Handle<vcl_batch, vcl_batch_destroy>(b);
    }
    void add(Pipeline& p) { ctx_->check(vcl_batch_add(h_.get(), p.get()), "vcl_batch_add"); }
    void remove(Pipeline& p) { ctx_->check(vcl_batch_remove(h_.get(), p.get()), "vcl_batch_remove"); }
    void set_repeat(Pipeline& p, int iterations) {
        ctx_->check(vcl_batch_set_repeat(h_.get(), p.get(), iterations), "vcl_batch_set_repeat");
    }
    void step(void* stream = nullptr) { ctx_->check(vcl_batch_step(h_.get(), stream), "vcl_batch_step"); }
    int size() const { return vcl_batch_size(h_.get()); }

private:
    const Context* ctx_;
    detail::Handle<vcl_batch, vcl_batch_destroy> h_;
};

// The serving loop (vcl_server_*).
class Server {
public:
    Server(const Context& ctx, size_t budget_bytes, int max_live) {
        vcl_server* s = nullptr;
        ctx.check(vcl_server_create(ctx.get(), budget_bytes, max_live, &s), "vcl_server_create");
        h_ = detail::Handle<vcl_server, vcl_server_destroy>(s);
    }
    long long submit(const vcl_fit_desc& desc, const float* target, int iterations, bool keep_result = false) {
        long long id = -1;
        chk(vcl_server_submit(h_.get(), &desc, target, iterations, keep_result ? 1 : 0, &id), "vcl_server_submit");
        return id;
    }
    void tick(void* stream, int* live = nullptr, int* completed = nullptr) {
        chk(vcl_server_tick(h_.get(), stream, live, completed), "vcl_server_tick");
    }
    void drain(void* stream) { chk(vcl_server_drain(h_.get(), stream), "vcl_server_drain"); }
    int pending() const { return vcl_server_pending(h_.get()); }
    double now_ms() const { return vcl_server_now_ms(h_.get()); }
    int state(long long job) const {
        int s = -1, it = 0;
        double a = 0, b = 0, c = 0;
        chk(vcl_server_job_status(h_.get(), job, &s, &it, &a, &b, &c), "vcl_server_job_status");
        return s;
    }

private:
    void chk(vcl_status st, const char* what) const {
        if (st == VCL_OK) return;
        const char* m = vcl_server_last_error(h_.get());
        throw Error(st, std::string(what) + ": " + (m ? m : ""));
    }
    detail::Handle<vcl_server, vcl_server_destroy> h_;
};

// A loaded Wavefront OBJ (vcl_obj_*), host memory only; needs no device.
class Obj {
public:
    explicit Obj(const std::string& path) {
        vcl_obj* o = nullptr;
        const vcl_status st = vcl_obj_load(nullptr, path.c_str(), &o);
        if (st != VCL_OK) {
            const char* m = vcl_asset_error();
            throw Error(st, "vcl_obj_load: " + std::string(m ? m : ""));
        }
        h_ = detail::Handle<vcl_obj, vcl_obj_free>(o);
    }
    struct Counts {
        int pos, tri, texel, normal, welded;
    };
    Counts counts() const {
        Counts c{};
        vcl_obj_counts(h_.get(), &c.pos, &c.tri, &c.texel, &c.normal, &c.welded);
        return c;
    }
    // Welded form: one vertex per distinct corner, one index array (the
    // layout of vcl_fit_desc).
    void welded(const float** pos, const float** uv, const float** normal, const uint32_t** tri) const {
        vcl_obj_welded(h_.get(), pos, uv, normal, tri);
    }
    vcl_obj* get() const { return h_.get(); }

private:
    detail::Handle<vcl_obj, vcl_obj_free> h_;
};

// A BMP as floats [height][width][channels] (vcl_bmp_load); no device.
inline std::vector<float> load_bmp(const std::string& path, int& width, int& height, int& channels) {
    vcl_status st = vcl_bmp_load(nullptr, path.c_str(), &width, &height, &channels, nullptr);
    if (st != VCL_OK) throw Error(st, "vcl_bmp_load: " + std::string(vcl_asset_error() ? vcl_asset_error() : ""));
    std::vector<float> px((size_t)width * height * channels);
    st = vcl_bmp_load(nullptr, path.c_str(), &width, &height, &channels, px.data());
    if (st != VCL_OK) throw Error(st, "vcl_bmp_load: " + std::string(vcl_asset_error() ? vcl_asset_error() : ""));
    return px;
}

}  // namespace vcl

#endif  // VCL_HPP

// Fit jobs: the reference's PresetPrimitives iteration (preset_primitives.cpp
// :160-230) as a resident device object.  All parameters, Adam moments,
// gradients and per-view buffers live in one device arena allocated at
// creation; a step allocates nothing and only enqueues work on the caller's
// stream, so it can be captured in a CUDA graph.
#include "common.cuh"
#include "fit.cuh"
#include <vector>
#include <cstring>

namespace {

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

struct Layout {
    size_t total = 0;
    size_t add(size_t bytes) { size_t o = total; total += al(bytes ? bytes : 1); return o; }
};

}  // namespace

// Buffer offsets inside the arena, shared by create() and footprint().
static void plan(const vcl_fit_desc& d, vcl_fit* f, Layout& L) {
    const size_t N = (size_t)d.W * d.H * d.views;
    const size_t F = sizeof(float);
    const size_t npyr = vcl_tex_level_offset(d.tex_w, d.tex_h, d.C, d.levels);
    const size_t n0 = (size_t)d.tex_w * d.tex_h * d.C;
    size_t o[64];
    int i = 0;
    o[i++] = L.add(F * d.nv * 3);             // pos
    o[i++] = L.add(sizeof(uint32_t) * d.nt * 3);
    o[i++] = L.add(F * d.nv * 2);             // uv attr
    o[i++] = L.add(F * d.nv * 3);             // normal attr
    o[i++] = L.add(F * npyr);                 // pyramid
    o[i++] = L.add(F * d.K * (4 + d.C));      // lobes: axis [K][3] | sharpness [K] | amplitude [K][C]
    o[i++] = L.add(F * d.views * 16);         // mvp
    o[i++] = L.add(F * d.views * 9);          // pvinv
    o[i++] = L.add(F * 16);                   // rot
    o[i++] = L.add(F * d.views * d.nv * 4);   // clip
    o[i++] = L.add(F * N * 4);                // rast
    o[i++] = L.add(F * N * 4);                // db
    o[i++] = L.add(F * N * 2);                // uv
    o[i++] = L.add(F * N * 4);                // uv_da
    o[i++] = L.add(F * N * d.C);              // diffuse
    o[i++] = L.add(F * N);                    // rough
    // normal .. spec amp: one stretch of plain-strategy intermediates (11
    // floats per pixel) that the fused step reuses for its shading records
    o[i++] = L.add(F * N * 3);                // normal
    o[i++] = L.add(F * N * 3);                // view
    o[i++] = L.add(F * N * 3);                // spec axis
    o[i++] = L.add(F * N);                    // spec sharp
    o[i++] = L.add(F * N);                    // spec amp
    o[i++] = L.add(F * N * d.C);              // color
    o[i++] = L.add(F * N * d.C);              // aa
    o[i++] = L.add(F * N * d.C);              // target
    o[i++] = L.add(F * N * d.C);              // g_aa
    o[i++] = L.add(F * N * d.C);              // g_color
    o[i++] = L.add(F * N * d.C);              // g_diffuse
    o[i++] = L.add(F * N * 2);                // g_uv
    o[i++] = L.add(F * N * 2);                // g_bary
    o[i++] = L.add(F * d.views * d.nv * 4);   // g_clip
    o[i++] = L.add(F * npyr);                 // g_pyr
    o[i++] = L.add(F * d.nv * 3);             // g_pos
    o[i++] = L.add(F * d.K * (4 + d.C));      // lobe gradients, same layout
    o[i++] = L.add(F * n0 * 2);               // adam m,v texture
    o[i++] = L.add(F * d.nv * 3 * 2);         // adam m,v pos
    o[i++] = L.add(F * d.K * (4 + d.C) * 2);  // adam m,v lobes (axis|sharp|amp)
    o[i++] = L.add(F * 4);                    // loss
    if (f) {
        char* b = (char*)f->arena;
        int j = 0;
        f->pos = (float*)(b + o[j++]); f->tri = (uint32_t*)(b + o[j++]); f->uvattr = (float*)(b + o[j++]);
        f->nrmattr = (float*)(b + o[j++]); f->pyr = (float*)(b + o[j++]); f->lobe = (float*)(b + o[j++]);
        f->mvp = (float*)(b + o[j++]);
        f->pvinv = (float*)(b + o[j++]); f->rot = (float*)(b + o[j++]); f->clip = (float*)(b + o[j++]);
        f->rast = (float*)(b + o[j++]); f->db = (float*)(b + o[j++]); f->uv = (float*)(b + o[j++]);
        f->uv_da = (float*)(b + o[j++]); f->diffuse = (float*)(b + o[j++]); f->rough = (float*)(b + o[j++]);
        f->normal = (float*)(b + o[j++]); f->view = (float*)(b + o[j++]); f->sax = (float*)(b + o[j++]);
        f->ssh = (float*)(b + o[j++]); f->sam = (float*)(b + o[j++]); f->color = (float*)(b + o[j++]);
        f->aa = (float*)(b + o[j++]); f->target = (float*)(b + o[j++]); f->g_aa = (float*)(b + o[j++]);
        f->g_color = (float*)(b + o[j++]); f->g_diffuse = (float*)(b + o[j++]); f->g_uv = (float*)(b + o[j++]);
        f->g_bary = (float*)(b + o[j++]); f->g_clip = (float*)(b + o[j++]); f->g_pyr = (float*)(b + o[j++]);
        f->g_pos = (float*)(b + o[j++]); f->g_lobe = (float*)(b + o[j++]);
        f->mv_tex = (float*)(b + o[j++]); f->mv_pos = (float*)(b + o[j++]); f->mv_lobe = (float*)(b + o[j++]);
        f->loss = (float*)(b + o[j++]);
        f->axis = f->lobe; f->sharp = f->lobe + 3 * d.K; f->amp = f->lobe + 4 * d.K;
        f->g_axis = f->g_lobe; f->g_sharp = f->g_lobe + 3 * d.K; f->g_amp = f->g_lobe + 4 * d.K;
    }
}

static vcl_status validate(vcl_ctx* ctx, const vcl_fit_desc* d) {
    VCL_REQUIRE(d, "null descriptor");
    VCL_REQUIRE(d->W > 0 && d->H > 0 && d->views > 0 && d->nv > 0 && d->nt > 0, "bad fit sizes");
    VCL_REQUIRE(d->C >= 1 && d->C <= 8 && d->K >= 0 && d->K <= 1024, "bad channel/lobe counts");
    VCL_REQUIRE(d->tex_w > 0 && d->tex_h > 0 && d->levels >= 1 && d->levels == vcl_tex_levels(d->tex_w, d->tex_h, d->levels),
                "bad texture size/levels");
    VCL_REQUIRE(d->pos && d->tri && d->uv && d->normal && d->tex && d->mvp && d->pvinv && d->rot, "null host array");
    VCL_REQUIRE(d->K == 0 || (d->lobe_axis && d->lobe_sharp && d->lobe_amp), "null lobe array");
    return VCL_OK;
}

extern "C" {

VCL_API size_t vcl_fit_footprint(const vcl_fit_desc* desc) {
    if (!desc) return 0;
    Layout L;
    plan(*desc, nullptr, L);
    return L.total + fit_fused_footprint(*desc);
}

VCL_API vcl_status vcl_fit_create(vcl_ctx* ctx, const vcl_fit_desc* desc, vcl_fit** out) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(out, "null output");
    *out = nullptr;
    vcl_status st = validate(ctx, desc);
    if (st) return st;
    vcl_fit* f = new vcl_fit();
    f->ctx = ctx;
    f->d = *desc;
    if (f->d.lr_pos <= 0) f->d.lr_pos = f->d.lr;
    if (f->d.lr_tex <= 0) f->d.lr_tex = f->d.lr;
    if (f->d.lr_lobes <= 0) f->d.lr_lobes = f->d.lr;
    Layout L;
    plan(f->d, nullptr, L);
    // set-up runs on the context's non-blocking stream, so creating a job does
    // not wait for other jobs' work on the device
    cudaStream_t up_s = ctx->aux;
    cudaError_t e = cudaMallocAsync(&f->arena, L.total, up_s);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        delete f;
        return vcl_fail(ctx, VCL_ERR_NOMEM, "fit arena of %zu bytes: %s", L.total, cudaGetErrorString(e));
    }
    f->arena_bytes = L.total;
    Layout L2;
    plan(f->d, f, L2);
    const vcl_fit_desc& d = f->d;
    const size_t N = (size_t)d.W * d.H * d.views;
    const size_t n0 = (size_t)d.tex_w * d.tex_h * d.C;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (st == VCL_OK)
            st = vcl_cuda_check(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, up_s), "fit upload");
    };
    st = vcl_cuda_check(ctx, cudaMemsetAsync(f->arena, 0, L.total, up_s), "fit clear");
    up(f->pos, d.pos, sizeof(float) * d.nv * 3);
    up(f->tri, d.tri, sizeof(uint32_t) * d.nt * 3);
    up(f->uvattr, d.uv, sizeof(float) * d.nv * 2);
    up(f->nrmattr, d.normal, sizeof(float) * d.nv * 3);
    up(f->pyr, d.tex, sizeof(float) * n0);
    if (d.K) {
        up(f->axis, d.lobe_axis, sizeof(float) * d.K * 3);
        up(f->sharp, d.lobe_sharp, sizeof(float) * d.K);
        up(f->amp, d.lobe_amp, sizeof(float) * d.K * d.C);
    }
    up(f->mvp, d.mvp, sizeof(float) * d.views * 16);
    up(f->pvinv, d.pvinv, sizeof(float) * d.views * 9);
    up(f->rot, d.rot, sizeof(float) * 16);
    std::vector<float> r(N, d.roughness);
    up(f->rough, r.data(), sizeof(float) * N);
    if (st == VCL_OK) st = vcl_texture_build_mips(ctx, f->pyr, d.tex_w, d.tex_h, d.C, d.levels, up_s);
    if (st == VCL_OK) st = vcl_cuda_check(ctx, cudaStreamSynchronize(up_s), "fit create");
    if (st) {
        vcl_fit_destroy(f);
        return st;
    }
    // host pointers are not kept
    f->d.pos = nullptr; f->d.tri = nullptr; f->d.uv = nullptr; f->d.normal = nullptr; f->d.tex = nullptr;
    f->d.lobe_axis = nullptr; f->d.lobe_sharp = nullptr; f->d.lobe_amp = nullptr;
    f->d.mvp = nullptr; f->d.pvinv = nullptr; f->d.rot = nullptr;
    *out = f;
    return VCL_OK;
}

VCL_API void vcl_fit_destroy(vcl_fit* f) {
    if (!f) return;
    for (int b = 0; b < 2; ++b) {
        if (f->staging[b]) cudaFree(f->staging[b]);
        if (f->st_full[b]) cudaEventDestroy(f->st_full[b]);
        if (f->st_free[b]) cudaEventDestroy(f->st_free[b]);
    }
    if (f->arena) cudaFree(f->arena);
    fit_fused_release(f, nullptr, false);
    delete f;
}

VCL_API void vcl_fit_destroy_async(vcl_fit* f, void* stream) {
    if (!f) return;
    cudaStream_t s = (cudaStream_t)stream;
    for (int b = 0; b < 2; ++b) {
        if (f->staging[b]) cudaFreeAsync(f->staging[b], s);
        if (f->st_full[b]) cudaEventDestroy(f->st_full[b]);
        if (f->st_free[b]) cudaEventDestroy(f->st_free[b]);
    }
    if (f->arena) cudaFreeAsync(f->arena, s);
    fit_fused_release(f, s, true);
    delete f;
}

VCL_API vcl_status vcl_fit_set_strategy(vcl_fit* f, int strategy) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(strategy == VCL_FIT_PLAIN || strategy == VCL_FIT_FUSED, "unknown strategy %d", strategy);
    VCL_REQUIRE(strategy == VCL_FIT_PLAIN || f->d.C == 4, "the fused strategy needs C = 4 channels");
    if (strategy != f->strategy && f->step_count > 0) {
        // the plain step clears gradients when it starts, the fused step when
        // it has consumed them: start the other strategy from zero gradients
        // (a job that has not stepped still has the zeroed arena)
        const vcl_fit_desc& d = f->d;
        size_t npyr = vcl_tex_level_offset(d.tex_w, d.tex_h, d.C, d.levels);
        vcl_status st = VCL_OK;
        auto z = [&](void* p, size_t b) {
            if (st == VCL_OK) st = vcl_cuda_check(ctx, cudaMemset(p, 0, b), "gradient clear");
        };
        z(f->g_pyr, sizeof(float) * npyr);
        z(f->g_pos, sizeof(float) * d.nv * 3);
        z(f->g_lobe, sizeof(float) * (size_t)d.K * (4 + d.C));
        z(f->g_clip, sizeof(float) * (size_t)d.views * d.nv * 4);
        if (st == VCL_OK) st = vcl_cuda_check(ctx, cudaDeviceSynchronize(), "gradient clear");
        if (st == VCL_OK && strategy == VCL_FIT_FUSED) st = fit_fused_sync_counter(f, true);
        if (st) return st;
    }
    f->strategy = strategy;
    return VCL_OK;
}

VCL_API vcl_status vcl_fit_set_target(vcl_fit* f, const float* src, int src_is_device, void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(src, "null target");
    size_t bytes = sizeof(float) * (size_t)f->d.W * f->d.H * f->d.views * f->d.C;
    return vcl_cuda_check(ctx, cudaMemcpyAsync(f->target, src, bytes, src_is_device ? cudaMemcpyDeviceToDevice
                                                                                        : cudaMemcpyHostToDevice,
                                               (cudaStream_t)stream), "fit target copy");
}

VCL_API vcl_status vcl_fit_set_cameras(vcl_fit* f, const float* mvp, const float* pvinv, void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(mvp && pvinv, "null camera arrays");
    cudaStream_t s = (cudaStream_t)stream;
    vcl_status st = vcl_cuda_check(ctx, cudaMemcpyAsync(f->mvp, mvp, sizeof(float) * 16 * f->d.views,
                                                        cudaMemcpyHostToDevice, s), "camera copy");
    if (st) return st;
    return vcl_cuda_check(ctx, cudaMemcpyAsync(f->pvinv, pvinv, sizeof(float) * 9 * f->d.views, cudaMemcpyHostToDevice, s),
                          "camera copy");
}

VCL_API const float* vcl_fit_loss_device(const vcl_fit* f) { return f ? f->loss : nullptr; }

VCL_API vcl_status vcl_fit_read_loss(vcl_fit* f, float* loss_host, void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(loss_host, "null loss output");
    cudaStream_t s = (cudaStream_t)stream;
    vcl_status st = vcl_cuda_check(ctx, cudaMemcpyAsync(loss_host, f->loss, sizeof(float), cudaMemcpyDeviceToHost, s),
                                   "loss readback");
    if (st) return st;
    return vcl_cuda_check(ctx, cudaStreamSynchronize(s), "loss readback sync");
}

VCL_API vcl_status vcl_fit_read_loss_async(vcl_fit* f, float* loss_host, void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(loss_host, "null loss output");
    return vcl_cuda_check(ctx, cudaMemcpyAsync(loss_host, f->loss, sizeof(float), cudaMemcpyDeviceToHost,
                                               (cudaStream_t)stream), "loss readback");
}

VCL_API vcl_status vcl_fit_read_params(vcl_fit* f, float* pos, float* tex0, float* axis, float* sharp, float* amp,
                                       void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    cudaStream_t s = (cudaStream_t)stream;
    const vcl_fit_desc& d = f->d;
    vcl_status st = VCL_OK;
    auto dn = [&](void* dst, const void* src, size_t bytes) {
        if (dst && st == VCL_OK)
            st = vcl_cuda_check(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "param readback");
    };
    dn(pos, f->pos, sizeof(float) * d.nv * 3);
    dn(tex0, f->pyr, sizeof(float) * d.tex_w * d.tex_h * d.C);
    dn(axis, f->axis, sizeof(float) * d.K * 3);
    dn(sharp, f->sharp, sizeof(float) * d.K);
    dn(amp, f->amp, sizeof(float) * d.K * d.C);
    if (st == VCL_OK) st = vcl_cuda_check(ctx, cudaStreamSynchronize(s), "param readback sync");
    return st;
}

// ---------------------------------------------------------------- job state
// A job's resumable state in one host buffer: a header (magic, version, the
// shapes it belongs to, the Adam step) followed by the parameters (positions,
// the whole texture pyramid, the lobe block) and the Adam moments of the three
// groups, each as the device holds it.
namespace {

struct StateHeader {
    char magic[8];
    int32_t version, nv, tex_w, tex_h, C, levels, K, step;
    int64_t npyr;
};
constexpr char kStateMagic[8] = {'V', 'C', 'L', 'F', 'I', 'T', '0', '1'};

struct StatePart {
    float* dev;
    size_t bytes;
};

void state_parts(const vcl_fit* f, StatePart (&p)[6]) {
    const vcl_fit_desc& d = f->d;
    const size_t F = sizeof(float);
    const size_t npyr = vcl_tex_level_offset(d.tex_w, d.tex_h, d.C, d.levels);
    const size_t n0 = (size_t)d.tex_w * d.tex_h * d.C, nl = (size_t)d.K * (4 + d.C);
    p[0] = {f->pos, F * d.nv * 3};
    p[1] = {f->pyr, F * npyr};
    p[2] = {f->lobe, F * nl};
    p[3] = {f->mv_tex, F * n0 * 2};
    p[4] = {f->mv_pos, F * d.nv * 3 * 2};
    p[5] = {f->mv_lobe, F * nl * 2};
}

}  // namespace

VCL_API size_t vcl_fit_state_bytes(const vcl_fit* f) {
    if (!f) return 0;
    StatePart p[6];
    state_parts(f, p);
    size_t n = sizeof(StateHeader);
    for (const StatePart& q : p) n += q.bytes;
    return n;
}

VCL_API vcl_status vcl_fit_save_state(vcl_fit* f, void* host_dst, size_t bytes, void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    const size_t need = vcl_fit_state_bytes(f);
    VCL_REQUIRE(host_dst && bytes >= need, "state buffer of %zu bytes, %zu needed", bytes, need);
    const vcl_fit_desc& d = f->d;
    StateHeader h;
    std::memcpy(h.magic, kStateMagic, 8);
    h.version = 1; h.nv = d.nv; h.tex_w = d.tex_w; h.tex_h = d.tex_h; h.C = d.C; h.levels = d.levels; h.K = d.K;
    h.step = f->step_count;
    h.npyr = (int64_t)vcl_tex_level_offset(d.tex_w, d.tex_h, d.C, d.levels);
    char* out = (char*)host_dst;
    std::memcpy(out, &h, sizeof(h));
    size_t off = sizeof(h);
    StatePart p[6];
    state_parts(f, p);
    cudaStream_t s = (cudaStream_t)stream;
    vcl_status st = VCL_OK;
    for (const StatePart& q : p) {
        if (q.bytes && st == VCL_OK)
            st = vcl_cuda_check(ctx, cudaMemcpyAsync(out + off, q.dev, q.bytes, cudaMemcpyDeviceToHost, s), "state save");
        off += q.bytes;
    }
    if (st == VCL_OK) st = vcl_cuda_check(ctx, cudaStreamSynchronize(s), "state save sync");
    return st;
}

VCL_API vcl_status vcl_fit_load_state(vcl_fit* f, const void* host_src, size_t bytes, void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    const size_t need = vcl_fit_state_bytes(f);
    VCL_REQUIRE(host_src && bytes >= need, "state of %zu bytes, %zu needed", bytes, need);
    StateHeader h;
    std::memcpy(&h, host_src, sizeof(h));
    const vcl_fit_desc& d = f->d;
    VCL_REQUIRE(std::memcmp(h.magic, kStateMagic, 8) == 0 && h.version == 1,
                "not a fit job state (bad magic or version)");
    VCL_REQUIRE(h.nv == d.nv && h.tex_w == d.tex_w && h.tex_h == d.tex_h && h.C == d.C && h.levels == d.levels &&
                    h.K == d.K && h.step >= 0,
                "state of another job shape (nv %d, texture %dx%dx%d/%d levels, K %d)", h.nv, h.tex_w, h.tex_h, h.C,
                h.levels, h.K);
    const char* in = (const char*)host_src;
    size_t off = sizeof(h);
    StatePart p[6];
    state_parts(f, p);
    cudaStream_t s = (cudaStream_t)stream;
    vcl_status st = VCL_OK;
    for (const StatePart& q : p) {
        if (q.bytes && st == VCL_OK)
            st = vcl_cuda_check(ctx, cudaMemcpyAsync(q.dev, in + off, q.bytes, cudaMemcpyHostToDevice, s), "state load");
        off += q.bytes;
    }
    if (st == VCL_OK) st = vcl_cuda_check(ctx, cudaStreamSynchronize(s), "state load sync");
    if (st) return st;
    f->step_count = h.step;
    return fit_fused_sync_counter(f, true);
}

VCL_API int vcl_fit_launches_per_step(const vcl_fit* f) {
    if (!f) return 0;
    return f->strategy == VCL_FIT_FUSED ? fit_fused_launches(f) : fit_plain_launches(f);
}

VCL_API vcl_status vcl_fit_render(vcl_fit* f, float* out, void* stream) {
    if (!f) return VCL_ERR_ARG;
    return fit_forward(f, out, (cudaStream_t)stream);
}

VCL_API vcl_status vcl_fit_raster_tuning(vcl_fit* f, int* tile, float* ms_per_tile) {
    if (!f) return VCL_ERR_ARG;
    return fit_fused_raster_tuning(f, tile, ms_per_tile);
}

VCL_API vcl_status vcl_fit_raster_schedule(vcl_fit* f, int* tile, int* small_area, long long* bin_capacity,
                                           int* from_cache, long long* overflow_tiles) {
    if (!f) return VCL_ERR_ARG;
    return fit_fused_raster_schedule(f, tile, small_area, bin_capacity, from_cache, overflow_tiles);
}

VCL_API void vcl_raster_tuning_cache_clear(void) { fit_fused_tuning_cache_clear(); }

VCL_API int vcl_fit_kernel_count(void) { return fit_fused_kernel_count(); }
VCL_API const char* vcl_fit_kernel_name(int i) { return fit_fused_kernel_name(i); }

VCL_API vcl_status vcl_fit_time_kernels(vcl_fit* f, void* stream, int reps, float* ms, int n) {
    if (!f) return VCL_ERR_ARG;
    return fit_fused_time_kernels(f, (cudaStream_t)stream, reps, ms, n);
}

VCL_API vcl_status vcl_fit_prepare(vcl_fit* f, void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(f->strategy == VCL_FIT_FUSED, "prepare applies to the fused strategy");
    cudaGraph_t g = nullptr;
    return fit_fused_graph(f, (cudaStream_t)stream, &g);
}

VCL_API vcl_status vcl_fit_stage_target(vcl_fit* f, const float* host_src, void* copy_stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(host_src, "null target");
    VCL_REQUIRE(!f->st_pending, "a staged target has not been consumed by a step yet");
    const size_t bytes = sizeof(float) * (size_t)f->d.W * f->d.H * f->d.views * f->d.C;
    const int b = f->st_next;
    if (!f->staging[b]) {
        cudaError_t e = cudaMalloc(&f->staging[b], bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->st_full[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f->st_free[b], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            return vcl_fail(ctx, VCL_ERR_NOMEM, "target staging buffer: %s", cudaGetErrorString(e));
        }
    }
    cudaStream_t cs = (cudaStream_t)copy_stream;
    // the target this buffer held last (two uploads ago) must have been
    // moved out of it; the previous upload's buffer is the other one
    if (f->st_used[b]) {
        vcl_status st = vcl_cuda_check(ctx, cudaStreamWaitEvent(cs, f->st_free[b], 0), "staging wait");
        if (st) return st;
    }
    vcl_status st = vcl_cuda_check(ctx, cudaMemcpyAsync(f->staging[b], host_src, bytes, cudaMemcpyHostToDevice, cs),
                                   "target staging copy");
    if (!st) st = vcl_cuda_check(ctx, cudaEventRecord(f->st_full[b], cs), "staging event");
    if (!st) {
        f->st_pending = true;
        f->st_next = b ^ 1;
    }
    return st;
}

VCL_API vcl_status vcl_fit_step(vcl_fit* f, void* stream) {
    if (!f) return VCL_ERR_ARG;
    vcl_ctx* ctx = f->ctx;
    cudaStream_t s = (cudaStream_t)stream;
    if (f->st_pending) {
        // a staged target becomes this step's target: wait for its upload,
        // move it in on the device, free the staging buffer for the next one
        const size_t bytes = sizeof(float) * (size_t)f->d.W * f->d.H * f->d.views * f->d.C;
        const int b = f->st_next ^ 1;
        vcl_status st = vcl_cuda_check(ctx, cudaStreamWaitEvent(s, f->st_full[b], 0), "staging wait");
        if (!st) st = vcl_cuda_check(ctx, cudaMemcpyAsync(f->target, f->staging[b], bytes, cudaMemcpyDeviceToDevice, s),
                                     "staged target");
        if (!st) st = vcl_cuda_check(ctx, cudaEventRecord(f->st_free[b], s), "staging event");
        if (st) return st;
        f->st_pending = false;
        f->st_used[b] = true;
    }
    return f->strategy == VCL_FIT_FUSED ? fit_step_fused(f, s) : fit_step_plain(f, s);
}

}  // extern "C"

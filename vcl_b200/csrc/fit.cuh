// Internal state of a fit job (see vcl_fit_* in include/vcl.h).
#pragma once
#include "common.cuh"

struct vcl_fit {
    vcl_ctx* ctx = nullptr;
    vcl_fit_desc d{};
    int strategy = VCL_FIT_PLAIN;
    int step_count = 0;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    // parameters and constant attributes
    float *pos, *uvattr, *nrmattr, *pyr, *lobe, *axis, *sharp, *amp, *mvp, *pvinv, *rot;
    uint32_t* tri;
    // per-view / per-pixel buffers
    float *clip, *rast, *db, *uv, *uv_da, *diffuse, *normal, *view, *rough, *sax, *ssh, *sam, *color, *aa, *target;
    // gradients
    float *g_aa, *g_color, *g_diffuse, *g_uv, *g_bary, *g_clip, *g_pyr, *g_pos, *g_lobe, *g_axis, *g_sharp, *g_amp;
    // Adam moments: [m | v] per group
    float *mv_tex, *mv_pos, *mv_lobe;
    float* loss;
    // fused-strategy resources
    void* fused = nullptr;
    // staged target upload (vcl_fit_stage_target): two device staging
    // buffers used in turn, so that an upload never waits for the step that
    // consumes the previous one; per buffer a "filled" and a "consumed"
    // event; st_next = the buffer the next upload fills, st_pending = a fill
    // not yet consumed (of buffer st_next ^ 1), st_used[b] = buffer b was
    // consumed at least once
    float* staging[2] = {nullptr, nullptr};
    cudaEvent_t st_full[2] = {nullptr, nullptr}, st_free[2] = {nullptr, nullptr};
    int st_next = 0;
    bool st_pending = false, st_used[2] = {false, false};
};

vcl_status fit_step_plain(vcl_fit* f, cudaStream_t s);
vcl_status fit_step_fused(vcl_fit* f, cudaStream_t s);
vcl_status fit_forward(vcl_fit* f, float* out, cudaStream_t s);
int fit_plain_launches(const vcl_fit* f);
int fit_fused_launches(const vcl_fit* f);
// Frees the fused state; `async`: stream-ordered frees on `s` (no device sync).
void fit_fused_release(vcl_fit* f, cudaStream_t s, bool async);
vcl_status fit_fused_sync_counter(vcl_fit* f, bool to_device);
vcl_status fit_fused_raster_tuning(vcl_fit* f, int* tile, float* ms3);
vcl_status fit_fused_raster_schedule(vcl_fit* f, int* tile, int* small_area, long long* cap, int* cached,
                                     long long* overflow);
void fit_fused_tuning_cache_clear();
// Device bytes the fused strategy adds to a job (raster workspace upper
// bound and step state).
size_t fit_fused_footprint(const vcl_fit_desc& d);
int fit_fused_kernel_count();
const char* fit_fused_kernel_name(int i);
vcl_status fit_fused_time_kernels(vcl_fit* f, cudaStream_t s, int reps, float* ms, int n);
// The job's fused step as a CUDA graph (captured on `s` the first time; owned
// by the job, valid until the job is destroyed or the mode changes).
vcl_status fit_fused_graph(vcl_fit* f, cudaStream_t s, cudaGraph_t* out);

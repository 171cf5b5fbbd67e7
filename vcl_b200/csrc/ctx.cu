// Context, error reporting and workspace of the vcl C ABI.
#include "common.cuh"
#include <new>

vcl_status vcl_fail(vcl_ctx* ctx, vcl_status code, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        std::lock_guard<std::mutex> lock(ctx->err_mu);
        ctx->err = buf;
    }
    return code;
}

vcl_status vcl_cuda_check(vcl_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return VCL_OK;
    return vcl_fail(ctx, e == cudaErrorMemoryAllocation ? VCL_ERR_NOMEM : VCL_ERR_CUDA, "%s: %s", what,
                    cudaGetErrorString(e));
}

vcl_status vcl_launch_check(vcl_ctx* ctx, const char* what) {
    return vcl_cuda_check(ctx, cudaGetLastError(), what);
}

vcl_status vcl_ws_reserve(vcl_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->ws_bytes) return VCL_OK;
    size_t want = bytes + bytes / 4;
    if (ctx->ws) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return vcl_cuda_check(ctx, e, "workspace sync");
        cudaFree(ctx->ws);
        ctx->ws = nullptr;
        ctx->ws_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&ctx->ws, want);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return vcl_fail(ctx, VCL_ERR_NOMEM, "raster workspace of %zu bytes: %s", want, cudaGetErrorString(e));
    }
    ctx->ws_bytes = want;
    return VCL_OK;
}

extern "C" {

VCL_API const char* vcl_version(void) { return "vcl-b200 0.1 (sm_100a)"; }

VCL_API vcl_status vcl_create(int device, vcl_ctx** out) {
    if (!out) return VCL_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        (void)cudaGetLastError();
        return VCL_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return VCL_ERR_CUDA;
    vcl_ctx* c = new (std::nothrow) vcl_ctx();
    if (!c) return VCL_ERR_NOMEM;
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaMalloc(&c->dev_flags, 64) != cudaSuccess || cudaMemset(c->dev_flags, 0, 64) != cudaSuccess) {
        delete c;
        return VCL_ERR_NOMEM;
    }
    // jobs are allocated from the device's default stream-ordered pool; keep
    // freed blocks in this process's pool for reuse instead of handing them
    // back to the driver at every synchronization (a per-process attribute)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    (void)cudaGetLastError();
    if (cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess) {
        cudaFree(c->dev_flags);
        delete c;
        return VCL_ERR_CUDA;
    }
    *out = c;
    return VCL_OK;
}

VCL_API void vcl_destroy(vcl_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->ws) cudaFree(ctx->ws);
    if (ctx->dev_flags) cudaFree(ctx->dev_flags);
    if (ctx->aux) cudaStreamDestroy(ctx->aux);
    delete ctx;
}

// The message is copied for the calling thread under the context's lock:
// the pointer stays valid until this thread's next vcl_last_error call,
// whatever other threads report meanwhile.
VCL_API const char* vcl_last_error(const vcl_ctx* ctx) {
    if (!ctx) return "null context";
    thread_local std::string copy;
    std::lock_guard<std::mutex> lock(ctx->err_mu);
    copy = ctx->err;
    return copy.c_str();
}

VCL_API vcl_status vcl_set_mode(vcl_ctx* ctx, int mode) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(mode == VCL_MODE_COMPAT || mode == VCL_MODE_EXACT, "mode must be VCL_MODE_COMPAT or VCL_MODE_EXACT");
    ctx->mode = mode;
    return VCL_OK;
}

VCL_API int vcl_get_mode(const vcl_ctx* ctx) { return ctx ? ctx->mode : -1; }

VCL_API vcl_status vcl_set_raster_config(vcl_ctx* ctx, int tile, long long bin_capacity) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(tile == 8 || tile == 16 || tile == 32, "tile must be 8, 16 or 32 (got %d)", tile);
    VCL_REQUIRE(bin_capacity >= 0, "bin capacity must be >= 0");
    ctx->tile = tile;
    ctx->bin_capacity = bin_capacity;
    return VCL_OK;
}

VCL_API vcl_status vcl_set_raster_areas(vcl_ctx* ctx, int small_area, int medium_area) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(small_area >= -1 && medium_area >= -1, "areas must be >= 0, or -1 for the defaults");
    ctx->small_area = small_area;
    ctx->med_area = medium_area;
    return VCL_OK;
}

VCL_API vcl_status vcl_set_raster_autotune(vcl_ctx* ctx, int enable) {
    VCL_CTX_CHECK();
    ctx->autotune = enable ? 1 : 0;
    return VCL_OK;
}

VCL_API vcl_status vcl_get_raster_config(const vcl_ctx* ctx, int* tile, long long* bin_capacity) {
    if (!ctx) return VCL_ERR_ARG;
    if (tile) *tile = ctx->tile;
    if (bin_capacity) *bin_capacity = ctx->bin_capacity;
    return VCL_OK;
}

VCL_API vcl_status vcl_raster_overflow_count(vcl_ctx* ctx, void* stream, long long* count) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(count, "count is null");
    int h = 0;
    cudaStream_t s = (cudaStream_t)stream;
    vcl_status st = vcl_cuda_check(ctx, cudaMemcpyAsync(&h, ctx->dev_flags, sizeof(int), cudaMemcpyDeviceToHost, s),
                                   "overflow readback");
    if (st) return st;
    st = vcl_cuda_check(ctx, cudaStreamSynchronize(s), "overflow readback sync");
    *count = h;
    return st;
}

VCL_API int vcl_tex_levels(int tw, int th, int requested) {
    unsigned v = (unsigned)(tw | th);
    int lsb = 0;
    while (v && !(v & 1u)) { v >>= 1; ++lsb; }
    int maxlevel = lsb + 1;
    if (maxlevel > 16) maxlevel = 16;
    return requested < 1 ? 1 : (maxlevel < requested ? maxlevel : requested);
}

VCL_API size_t vcl_tex_level_offset(int tw, int th, int C, int level) {
    size_t off = 0;
    for (int l = 0; l < level; ++l) off += (size_t)(tw >> l) * (size_t)(th >> l) * C;
    return off;
}

}  // extern "C"

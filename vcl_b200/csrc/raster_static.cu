// vcl_rasterize_fwd_static: the forward rasterizer on a fixed, statically
// allocated scratch area instead of the context's growable workspace.
//
// Who needs it: vcl_rasterize_fwd grows the context workspace on demand, and
// growing it means cudaDeviceSynchronize + cudaFree + cudaMalloc in the
// middle of the call.  Callers that must not allocate device memory (or take
// a device-wide synchronization) on their per-frame path cannot use that: a
// serving loop that shares the device with other jobs' streams and whose
// device memory has already been committed to resident jobs, or a host with
// a fixed device-memory budget after set-up.  This entry point calls no
// cudaMalloc, cudaFree or any allocating library function; its scratch is
// the file-scope array below, reserved when the module is loaded.
//
// Limits and rules:
//   * RASTER_SCRATCH_BYTES (VCL_RASTER_SCRATCH_BYTES, 32 MiB) bounds the
//     request: the per-pixel depth keys (8 B x W x H x views), the triangle
//     records with their medium-list entries (96 + 4 = 100 B x views x nt,
//     VCL_RASTER_BYTES_PER_VIEW_TRIANGLE) and the per-tile counters (12 B x
//     tiles x views) must fit, and the remainder holds the tile bin lists.
//     Larger requests are rejected with VCL_ERR_ARG and a message that gives
//     the bytes needed.  A bin list that
//     does not fit the remainder falls back to testing every large triangle
//     for the overflowing tiles: same result, slower.
//   * Nothing in the scratch has to start at zero: every call initializes
//     what it reads (depth keys to "empty", tile counters to 0) on the stream
//     before any kernel uses them, so the scratch carries no state between
//     calls.
//   * There is ONE scratch area per device.  Two calls whose work overlaps on
//     the device -- on different streams, from different host threads, or
//     from different contexts of the same device -- race on it and produce
//     garbage.  Serialize them (same stream, or an event between them).
//   * The address is resolved with cudaGetSymbolAddress once per device, by
//     vcl_raster_scratch_init or lazily by the first call on that device,
//     with that device current.  That first call may load the module that
//     holds the scratch, so make it during set-up, before any stream capture
//     begins.  cudaDeviceReset by the host application unloads the module:
//     the cached address is stale after it, so vcl_raster_scratch_init
//     always resolves the address anew, and a caller that resets the device
//     calls it again before the next static call.
#include <mutex>

#include "common.cuh"
#include "ops_internal.cuh"

namespace {

constexpr size_t RASTER_SCRATCH_BYTES = VCL_RASTER_SCRATCH_BYTES;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_raster_scratch[RASTER_SCRATCH_BYTES];

std::mutex g_scratch_mu;
void* g_scratch_addr[MAX_DEVICES] = {};

vcl_status scratch_address(vcl_ctx* ctx, void** out, bool refresh) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return vcl_cuda_check(ctx, e, "raster scratch: cudaGetDevice");
    if (dev != ctx->device)
        return vcl_fail(ctx, VCL_ERR_STATE, "raster scratch: current device %d is not the context's device %d", dev,
                        ctx->device);
    if (dev < 0 || dev >= MAX_DEVICES)
        return vcl_fail(ctx, VCL_ERR_STATE, "raster scratch: device ordinal %d above %d", dev, MAX_DEVICES - 1);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (refresh || !g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_raster_scratch);
        if (e != cudaSuccess) return vcl_cuda_check(ctx, e, "raster scratch: cudaGetSymbolAddress");
        if (!p || ((uintptr_t)p & 255))
            return vcl_fail(ctx, VCL_ERR_CUDA, "raster scratch: symbol address %p is not 256-byte aligned", p);
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return VCL_OK;
}

}  // namespace

extern "C" {

VCL_API size_t vcl_raster_scratch_bytes(void) { return RASTER_SCRATCH_BYTES; }

VCL_API vcl_status vcl_raster_scratch_init(vcl_ctx* ctx) {
    VCL_CTX_CHECK();
    void* p = nullptr;
    return scratch_address(ctx, &p, true);
}

VCL_API vcl_status vcl_rasterize_fwd_static(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt,
                                            int W, int H, int views, float* rast, float* db, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(W > 0 && H > 0 && views > 0 && nv >= 0 && nt >= 0, "bad raster sizes W=%d H=%d views=%d nv=%d nt=%d",
                W, H, views, nv, nt);
    VCL_REQUIRE(rast, "rast output is null");
    VCL_REQUIRE(nt == 0 || (clip && tri), "clip/tri is null");
    VCL_REQUIRE(((uintptr_t)clip & 15) == 0 && ((uintptr_t)rast & 15) == 0 && ((uintptr_t)db & 15) == 0,
                "clip/rast/db must be 16-byte aligned");
    const int T = ctx->tile;
    const long long ntiles = (long long)((W + T - 1) / T) * ((H + T - 1) / T) * views;
    VCL_REQUIRE(ntiles < (1ll << 31), "too many tiles");
    // everything but the bin list (a list of capacity 0 adds no bytes)
    const size_t fixed = raster_ws_size(W, H, views, nt, T, 0);
    VCL_REQUIRE(fixed <= RASTER_SCRATCH_BYTES,
                "rasterize_fwd_static: W=%d H=%d views=%d nt=%d needs %zu bytes of scratch "
                "(8 B per pixel + %d B per view and triangle + 12 B per tile), the static limit is %zu; "
                "use vcl_rasterize_fwd",
                W, H, views, nt, fixed, VCL_RASTER_BYTES_PER_VIEW_TRIANGLE, RASTER_SCRATCH_BYTES);
    const long long want = ctx->bin_capacity ? ctx->bin_capacity : raster_auto_capacity(views, nt, W, H, T);
    const long long room = (long long)((RASTER_SCRATCH_BYTES - fixed) / sizeof(int)) & ~63ll;
    const long long cap = want < room ? want : room;
    void* scratch = nullptr;
    vcl_status st = scratch_address(ctx, &scratch, false);
    if (st) return st;
    return raster_fwd_ws(ctx, scratch, ctx_sched(ctx, T, cap), ctx->dev_flags, clip, nv, tri, nt, W, H, views, rast,
                         db, (cudaStream_t)stream);
}

}  // extern "C"

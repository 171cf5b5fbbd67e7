// Shared device helpers and the context object of the vcl C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <mutex>
#include <cstdio>
#include <cstdarg>
#include "../../include/vcl.h"

struct vcl_ctx {
    int device = 0;
    int mode = VCL_MODE_COMPAT;
    int sm_count = 148;
    // last error message; written and read under err_mu, since a context's
    // jobs can report errors from more than one host thread (the serving
    // loop's tick thread and its set-up worker)
    std::string err;
    mutable std::mutex err_mu;
    // raster binning schedule
    int tile = 16;
    long long bin_capacity = 0;   // 0 = automatic
    int small_area = -1;          // direct-raster box areas, -1 = defaults
    int med_area = -1;
    int autotune = 1;             // fit jobs time raster schedules (0: size-based choice)
    // raster workspace (grown on demand, owned here)
    void* ws = nullptr;
    size_t ws_bytes = 0;
    int* dev_flags = nullptr;     // [0] = overflowed tiles of the last raster call
    cudaStream_t aux = nullptr;   // non-blocking stream for job set-up (uploads, allocations)
};

vcl_status vcl_fail(vcl_ctx* ctx, vcl_status code, const char* fmt, ...);
vcl_status vcl_cuda_check(vcl_ctx* ctx, cudaError_t e, const char* what);
vcl_status vcl_launch_check(vcl_ctx* ctx, const char* what);
// Grows the context workspace to at least `bytes` (synchronizes the device
// when it has to reallocate).
vcl_status vcl_ws_reserve(vcl_ctx* ctx, size_t bytes);

#define VCL_REQUIRE(cond, ...) \
    do { if (!(cond)) return vcl_fail(ctx, VCL_ERR_ARG, __VA_ARGS__); } while (0)
#define VCL_CTX_CHECK() \
    do { if (!ctx) return VCL_ERR_ARG; } while (0)

static inline unsigned vcl_blocks(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : b);
}

#define DEV __device__ __forceinline__

// common.h:181-182 (AddNaNcheck), for values owned by one thread.
DEV void add_nan_check(float& a, float b) {
    if (!isfinite(a)) a = 0.f;
    else { float v = a + b; if (isfinite(v)) a = v; }
}
DEV void add_nan_check3(float* a, float bx, float by, float bz) {
    if (!(isfinite(a[0]) && isfinite(a[1]) && isfinite(a[2]))) { a[0] = a[1] = a[2] = 0.f; }
    else {
        float x = a[0] + bx, y = a[1] + by, z = a[2] + bz;
        if (isfinite(x) && isfinite(y) && isfinite(z)) { a[0] = x; a[1] = y; a[2] = z; }
    }
}

DEV float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
DEV float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
DEV float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
DEV float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
DEV float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DEV float len3(float3 a) { return sqrtf(dot3(a, a)); }
DEV float3 normalize3(float3 v) { float d = 1.f / len3(v); return f3(v.x * d, v.y * d, v.z * d); }
DEV float3 ld3(const float* p, size_t i) { return f3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
DEV void st3(float* p, size_t i, float3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
DEV float lerpf_(float a, float b, float t) { return a + t * (b - a); }

// sm_90+ vector reduction: one red.global.add.v4.f32 instead of four.
DEV void red_add4(float* p, float a, float b, float c, float d) {
    atomicAdd(reinterpret_cast<float4*>(p), make_float4(a, b, c, d));
}
// Sums v[0..N) over each run of consecutive lanes of the warp that carry the
// same (key, view): a segmented scan by shuffles, as many rounds as the
// longest run needs.  Returns true on the last lane of a run, which then holds
// the run's sums.  All 32 lanes must call it; lanes with nothing to add pass
// zeros and a key no other lane uses (e.g. -1 - lane).  Neighbouring pixels of
// one triangle then issue one scatter instead of one each.
template <int N>
DEV bool warp_run_sum(float (&v)[N], int key, int view) {
    const int lane = threadIdx.x & 31;
    const int pk = __shfl_up_sync(0xffffffffu, key, 1), pv = __shfl_up_sync(0xffffffffu, view, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || pk != key || pv != view);
    const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
    const int len = (int)__reduce_max_sync(0xffffffffu, (unsigned)(lane - start + 1));
    for (int d = 1; d < len; d <<= 1) {
        const bool take = lane - d >= start;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const float y = __shfl_up_sync(0xffffffffu, v[k], d);
            if (take) v[k] += y;
        }
    }
    return tail;
}
DEV void red_add2(float* p, float a, float b) {
    atomicAdd(reinterpret_cast<float2*>(p), make_float2(a, b));
}

// Triangle id of a raster texel (u, v, z/w, id+1); -1 for background.
DEV int rast_id(float w) { return (int)w - 1; }

// n / d for 32-bit n by one multiply-high with m = floor((2^64 - 1) / d) + 1
// (exact for every 32-bit n when d >= 2; m = 0 stands for d = 1): Lemire,
// Kaser and Kurz, "Faster remainder by direct computation" (2019).  Keeps
// the per-pixel (view, row, column) split off the conversion / reciprocal
// unit that an integer division uses.
struct FastDiv {
    unsigned long long m;
};
inline FastDiv fastdiv_make(unsigned d) {
    FastDiv f;
    f.m = d > 1 ? ~0ull / d + 1 : 0ull;
    return f;
}
DEV unsigned fastdiv(unsigned n, FastDiv f) { return f.m ? (unsigned)__umul64hi(f.m, (unsigned long long)n) : n; }

// Asynchronous 16-byte global -> shared copies (sm_80+ cp.async, L2 only):
// a thread's copies land in the order of its commit groups; wait_group N
// returns once at most N of the thread's groups are still in flight.
DEV void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Throughput probes for the units other than HBM that bound the fit's
// kernels: the L2 reduction units (the texel and vertex gradient scatters
// issue red.global.add.v4.f32), the MUFU pipe (the SG kernels' ex2 and
// rsqrt) and the FP32 FMA pipe driven by paired instructions (the SG
// kernels' arithmetic).  Each probe runs a long, known number of those operations over the
// whole GPU; the caller times it with CUDA events and divides.  Measurement
// utilities only: no part of the fit path calls them.
#include "common.cuh"
#include "sg_math.cuh"

namespace {

// Every thread adds (1, 1, 1, 1) to float4 slots tid, tid + nthreads, ...
// of an n4-slot buffer, `iters` times over: a warp's reductions cover 32
// consecutive 16-byte slots (16 sectors), the best case for the L2
// reduction units.  A buffer well inside the 126 MB L2 keeps HBM out of it.
__global__ void __launch_bounds__(256) k_probe_red4(float* __restrict__ buf, long long n4, int iters) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nth = (long long)gridDim.x * blockDim.x;
    for (int it = 0; it < iters; ++it)
        for (long long i = tid; i < n4; i += nth) red_add4(buf + 4 * i, 1.f, 1.f, 1.f, 1.f);
}

DEV float ex2_approx(float x) {
    float y;
    asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
DEV float rsqrt_approx(float x) {
    float y;
    asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Eight independent chains per thread of x -> rsqrt(2^-x): two MUFU
// operations per link, values stay in (0.7, 1.3).  One result per thread is
// stored so that nothing is dropped.
__global__ void __launch_bounds__(256) k_probe_mufu(float* __restrict__ out, int iters) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = 0.5f + 0.01f * (float)((threadIdx.x + k) & 31);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = rsqrt_approx(ex2_approx(-a[k]));
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    out[(long long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Eight independent chains per thread of paired FP32 multiply-adds,
// x -> x * 0.999 + 0.001 on both halves (values stay near 1): 16 FP32
// operations per link.  One result per thread is stored.
__global__ void __launch_bounds__(256) k_probe_ffma2(float* __restrict__ out, int iters) {
    float2 a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = make_float2(0.5f + 0.01f * (float)((threadIdx.x + k) & 31), 0.75f);
    const float2 m = p2(0.999f), c = p2(0.001f);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma2(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k].x + a[k].y;
    out[(long long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" {

VCL_API vcl_status vcl_probe_red_throughput(vcl_ctx* ctx, float* buf, long long n_floats, int iters,
                                            long long* reductions, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(buf && n_floats >= 4 && iters > 0 && reductions, "bad probe arguments");
    VCL_REQUIRE(((uintptr_t)buf & 15) == 0, "probe buffer must be 16-byte aligned");
    const long long n4 = n_floats / 4;
    const int blocks = ctx->sm_count * 8;
    k_probe_red4<<<blocks, 256, 0, (cudaStream_t)stream>>>(buf, n4, iters);
    *reductions = n4 * (long long)iters;
    return vcl_launch_check(ctx, "probe_red_throughput");
}

VCL_API long long vcl_probe_mufu_threads(const vcl_ctx* ctx) { return ctx ? (long long)ctx->sm_count * 8 * 256 : 0; }

VCL_API vcl_status vcl_probe_mufu_throughput(vcl_ctx* ctx, float* out, int iters, long long* ops, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(out && iters > 0 && ops, "bad probe arguments");
    const int blocks = ctx->sm_count * 8;
    k_probe_mufu<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters);
    *ops = (long long)blocks * 256 * iters * 8 * 2;
    return vcl_launch_check(ctx, "probe_mufu_throughput");
}

VCL_API vcl_status vcl_probe_fma_throughput(vcl_ctx* ctx, float* out, int iters, long long* ops, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(out && iters > 0 && ops, "bad probe arguments");
    const int blocks = ctx->sm_count * 8;
    k_probe_ffma2<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters);
    *ops = (long long)blocks * 256 * iters * 8 * 2;
    return vcl_launch_check(ctx, "probe_fma_throughput");
}

}  // extern "C"

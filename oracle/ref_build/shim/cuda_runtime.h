// Host-only stand-in for the CUDA runtime header, used ONLY to compile the
// reference's own kernel sources (nvdiffrast/nvdiffrast/*.cu) as plain C++17
// for the CPU checker under oracle/_ref.  Nothing here runs on a GPU.
//
// * __global__/__device__ become ordinary inline host functions.
// * cudaLaunchKernel(f, grid, block, args, ...) unpacks `args` by the kernel's
//   parameter types and runs the grid block by block, thread by thread
//   (x fastest), which gives the race-free "all stores, then all adds" order
//   the reference's kernels assume.  With VCLREF_THREADS > 1 blocks run on
//   an OpenMP pool and atomicAdd becomes a real atomic (used for the timed
//   CPU baseline only).
// * cudaMalloc/cudaMemcpy/cudaMemset map to libc.
#pragma once
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <math.h>
#include <cstdint>
#include <utility>
#include <type_traits>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __shared__ static

struct dim3 {
    unsigned int x, y, z;
    constexpr dim3(unsigned int vx = 1, unsigned int vy = 1, unsigned int vz = 1) : x(vx), y(vy), z(vz) {}
};
struct uint3 { unsigned int x, y, z; };

struct alignas(8) float2 { float x, y; };
struct float3 { float x, y, z; };
struct alignas(16) float4 { float x, y, z, w; };
struct alignas(16) double2 { double x, y; };
struct double3 { double x, y, z; };
struct alignas(16) double4 { double x, y, z, w; };
struct alignas(8) int2 { int x, y; };
struct int3 { int x, y, z; };
struct alignas(16) int4 { int x, y, z, w; };
struct alignas(16) uint4 { unsigned int x, y, z, w; };

static inline float2 make_float2(float x, float y) { return float2{x, y}; }
static inline float3 make_float3(float x, float y, float z) { return float3{x, y, z}; }
static inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }
static inline double2 make_double2(double x, double y) { return double2{x, y}; }
static inline double3 make_double3(double x, double y, double z) { return double3{x, y, z}; }
static inline double4 make_double4(double x, double y, double z, double w) { return double4{x, y, z, w}; }
static inline int2 make_int2(int x, int y) { return int2{x, y}; }
static inline int3 make_int3(int x, int y, int z) { return int3{x, y, z}; }
static inline int4 make_int4(int x, int y, int z, int w) { return int4{x, y, z, w}; }
static inline uint3 make_uint3(unsigned x, unsigned y, unsigned z) { return uint3{x, y, z}; }

// Thread coordinates of the simulated launch (one set per host thread).
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;
// Number of host threads the launcher may use (1 = serial checker order).
extern int vclref_threads;
// Set by the harness around launches whose kernels accumulate without
// atomics (the reference's SG lobe gradients): those always run serially.
extern int vclref_force_serial;

// CUDA's mixed-precision max/min overloads (device math library semantics).
static inline float max(float a, float b) { return fmaxf(a, b); }
static inline double max(float a, double b) { return fmax((double)a, b); }
static inline double max(double a, float b) { return fmax(a, (double)b); }
static inline double max(double a, double b) { return fmax(a, b); }
static inline int max(int a, int b) { return a > b ? a : b; }
static inline float min(float a, float b) { return fminf(a, b); }
static inline double min(float a, double b) { return fmin((double)a, b); }
static inline double min(double a, float b) { return fmin(a, (double)b); }
static inline double min(double a, double b) { return fmin(a, b); }
static inline int min(int a, int b) { return a < b ? a : b; }

static inline int __float_as_int(float f) { int i; std::memcpy(&i, &f, 4); return i; }
static inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }

static inline float atomicAdd(float* p, float v) {
    if (vclref_threads <= 1) { float o = *p; *p = o + v; return o; }
    unsigned int* u = reinterpret_cast<unsigned int*>(p);
    unsigned int old = __atomic_load_n(u, __ATOMIC_RELAXED), nw;
    do { nw = (unsigned)__float_as_int(__int_as_float((int)old) + v); }
    while (!__atomic_compare_exchange_n(u, &old, nw, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED));
    return __int_as_float((int)old);
}

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
typedef void* cudaStream_t;
enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3, cudaMemcpyDefault = 4 };

static inline const char* cudaGetErrorString(cudaError_t e) { return e == 0 ? "no error" : "host shim error"; }
template <typename T> static inline cudaError_t cudaMalloc(T** p, size_t n) {
    *p = (T*)std::calloc(n ? n : 1, 1); return *p ? cudaSuccess : cudaErrorMemoryAllocation; }
template <typename T> static inline cudaError_t cudaMallocHost(T** p, size_t n) { return cudaMalloc(p, n); }
static inline cudaError_t cudaFree(void* p) { std::free(p); return cudaSuccess; }
static inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) { std::memmove(d, s, n); return cudaSuccess; }
static inline cudaError_t cudaMemset(void* d, int v, size_t n) { std::memset(d, v, n); return cudaSuccess; }
static inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }

namespace vclref_detail {
template <typename... A, size_t... I>
static inline void call_one(void (*f)(A...), void** args, std::index_sequence<I...>) {
    f(*static_cast<std::remove_cv_t<std::remove_reference_t<A>>*>(args[I])...);
}
template <typename... A>
static inline void run_block(void (*f)(A...), void** args, dim3 grid, dim3 block, unsigned bx, unsigned by, unsigned bz) {
    gridDim = grid; blockDim = block;
    blockIdx = uint3{bx, by, bz};
    for (unsigned tz = 0; tz < block.z; ++tz)
        for (unsigned ty = 0; ty < block.y; ++ty)
            for (unsigned tx = 0; tx < block.x; ++tx) {
                threadIdx = uint3{tx, ty, tz};
                call_one(f, args, std::index_sequence_for<A...>{});
            }
}
}  // namespace vclref_detail

template <typename... A>
static inline cudaError_t cudaLaunchKernel(void (*f)(A...), dim3 grid, dim3 block, void** args, size_t, cudaStream_t) {
    const long long nb = (long long)grid.x * grid.y * grid.z;
    if (vclref_threads <= 1 || vclref_force_serial || nb < 2) {
        for (unsigned bz = 0; bz < grid.z; ++bz)
            for (unsigned by = 0; by < grid.y; ++by)
                for (unsigned bx = 0; bx < grid.x; ++bx)
                    vclref_detail::run_block(f, args, grid, block, bx, by, bz);
        return cudaSuccess;
    }
#pragma omp parallel for schedule(dynamic, 4) num_threads(vclref_threads)
    for (long long b = 0; b < nb; ++b) {
        unsigned bx = (unsigned)(b % grid.x);
        unsigned by = (unsigned)((b / grid.x) % grid.y);
        unsigned bz = (unsigned)(b / ((long long)grid.x * grid.y));
        vclref_detail::run_block(f, args, grid, block, bx, by, bz);
    }
    return cudaSuccess;
}

// ref_harness.cpp -- C entry points into the REFERENCE's own operator code,
// compiled as host C++ from the reference sources where they lie (see
// oracle/ref_build/Makefile).  TEST INFRASTRUCTURE ONLY.
//
// Each ref_* function fills the reference's Params structs directly (the
// reference's init() functions would cudaMalloc their outputs) and then calls
// the reference's own X::forward / X::backward, or launches its __global__
// kernel where the public function also does host work we replace (ViewAxis
// computes its inverse with glm on the host).  Signatures match the orc_*
// restatement in oracle/vcl_oracle.h so that tests can run both.
//
// Multi-view inputs: operators that read clip-space positions (raster
// backward, antialias) take one view per call in the reference, so those
// wrappers loop over views with depth = 1.
#include "common.h"
#include "buffer.h"
#include "project.h"
#include "rasterize.h"
#include "interpolate.h"
#include "texturemap.h"
#include "antialias.h"
#include "material.h"
#include "loss.h"
#include "optimize.h"
#include <cstdint>
#include <cstdio>
#include <cstdlib>

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
int vclref_threads = 1;
int vclref_force_serial = 0;

// Host functions of the reference that the compiled files reference but the
// checker never calls (they allocate or need OpenGL).
void Attribute::init(Attribute&, Attribute&, int) { std::fprintf(stderr, "ref harness: Attribute::init not available\n"); std::abort(); }
void Rasterize::init(RasterizeParams&, ProjectParams&, int, int, int, bool) { std::fprintf(stderr, "ref harness: Rasterize::init needs OpenGL\n"); std::abort(); }

__global__ void ViewAxisForwardKernel(const ViewAxisKernelParams view);

static size_t level_offset(int tw, int th, int C, int level) {
    size_t off = 0;
    for (int l = 0; l < level; ++l) off += (size_t)(tw >> l) * (size_t)(th >> l) * C;
    return off;
}

extern "C" {

void ref_set_threads(int n) { vclref_threads = n < 1 ? 1 : n; }
int ref_get_threads(void) { return vclref_threads; }

// project.cu:36-46, :133-138
void ref_project_fwd(int nv, const float* mat, const float* pos, int dim, float* out) {
    ProjectParams p{};
    p.kernel.vecNum = nv; p.kernel.dimention = dim;
    p.kernel.vec = const_cast<float*>(pos); p.kernel.mat = const_cast<float*>(mat); p.kernel.out = out;
    Project::forward(p);
}
void ref_project_bwd(int nv, const float* mat, const float* g_out, int dim, float* g_pos) {
    ProjectGradParams p{};
    p.kernel.vecNum = nv; p.kernel.dimention = dim;
    p.kernel.mat = const_cast<float*>(mat);
    p.grad.out = const_cast<float*>(g_out); p.grad.vec = g_pos; p.grad.mat = nullptr;
    Project::backward(p);
}

// rasterize.cu:143-148
void ref_rasterize_bwd(int W, int H, int views, const float* clip, int nv, const uint32_t* tri,
                       const float* rast, const float* g_bary, float* g_clip) {
    for (int v = 0; v < views; ++v) {
        RasterizeGradParams p{};
        p.kernel.width = W; p.kernel.height = H; p.kernel.depth = 1; p.kernel.enableDB = 0;
        p.kernel.xs = 2.f / float(W); p.kernel.ys = 2.f / float(H);
        p.kernel.proj = const_cast<float*>(clip) + (size_t)v * nv * 4;
        p.kernel.idx = const_cast<unsigned*>(tri);
        p.kernel.out = const_cast<float*>(rast) + (size_t)v * W * H * 4;
        p.grad.proj = g_clip + (size_t)v * nv * 4;
        p.grad.out = const_cast<float*>(g_bary) + (size_t)v * W * H * 2;
        p.grad.outDB = nullptr;
        Rasterize::backward(p);
    }
}

// interpolate.cu:51-60, :145-149
void ref_interpolate_fwd(int W, int H, int views, int dim, int enable_da, const float* rast,
                         const float* db, const float* attr, const uint32_t* tri, float* out, float* out_da) {
    InterpolateParams p{};
    p.kernel.width = W; p.kernel.height = H; p.kernel.depth = views; p.kernel.dimention = dim;
    p.kernel.enableDA = enable_da;
    p.kernel.rast = const_cast<float*>(rast); p.kernel.rastDB = const_cast<float*>(db);
    p.kernel.attr = const_cast<float*>(attr); p.kernel.idx = const_cast<unsigned*>(tri);
    p.kernel.out = out; p.kernel.outDA = out_da;
    Interpolate::forward(p);
}
void ref_interpolate_bwd(int /*mode*/, int W, int H, int views, int dim, const float* rast,
                         const float* attr, const uint32_t* tri, const float* g_out, float* g_attr, float* g_bary) {
    InterpolateGradParams p{};
    p.kernel.width = W; p.kernel.height = H; p.kernel.depth = views; p.kernel.dimention = dim;
    p.kernel.enableDA = 0;
    p.kernel.rast = const_cast<float*>(rast); p.kernel.attr = const_cast<float*>(attr);
    p.kernel.idx = const_cast<unsigned*>(tri);
    p.grad.out = const_cast<float*>(g_out); p.grad.attr = g_attr; p.grad.rast = g_bary;
    Interpolate::backward(p);
}

static void fill_tex(TexturemapKernelParams& k, int W, int H, int views, int tw, int th, int C, int L,
                     const float* pyr, const float* rast, const float* uv, const float* uv_da) {
    k.width = W; k.height = H; k.depth = views; k.texwidth = tw; k.texheight = th; k.channel = C; k.miplevel = L;
    k.rast = const_cast<float*>(rast); k.uv = const_cast<float*>(uv); k.uvDA = const_cast<float*>(uv_da);
    for (int l = 0; l < L; ++l) k.texture[l] = const_cast<float*>(pyr) + level_offset(tw, th, C, l);
}

// texturemap.cu:116-123, :321-326
void ref_texture_fwd(int W, int H, int views, int tw, int th, int C, int L, const float* pyr,
                     const float* rast, const float* uv, const float* uv_da, float* out) {
    TexturemapParams p{};
    fill_tex(p.kernel, W, H, views, tw, th, C, L, pyr, rast, uv, uv_da);
    p.kernel.out = out;
    Texturemap::forward(p);
}
void ref_texture_bwd(int /*mode*/, int W, int H, int views, int tw, int th, int C, int L, const float* pyr,
                     const float* rast, const float* uv, const float* uv_da, const float* g_out,
                     float* g_pyr, float* g_uv, float* g_uv_da) {
    TexturemapGradParams p{};
    fill_tex(p.kernel, W, H, views, tw, th, C, L, pyr, rast, uv, uv_da);
    p.grad.out = const_cast<float*>(g_out);
    p.grad.uv = g_uv; p.grad.uvDA = g_uv_da;
    for (int l = 0; l < L; ++l) p.grad.texture[l] = g_pyr + level_offset(tw, th, C, l);
    Texturemap::backward(p);
}

// antialias.cu:97-108, :302-313
static void fill_aa(AntialiasKernelParams& k, int W, int H, int C, const float* proj, const uint32_t* tri,
                    const float* rast, const float* in) {
    k.width = W; k.height = H; k.depth = 1; k.channel = C;
    k.s = make_float2(W / 2.f, H / 2.f);
    k.proj = const_cast<float*>(proj); k.idx = const_cast<unsigned*>(tri);
    k.rast = const_cast<float*>(rast); k.in = const_cast<float*>(in);
}
void ref_antialias_fwd(int W, int H, int views, int C, const float* clip, int nv, const uint32_t* tri,
                       const float* rast, const float* in, float* out) {
    for (int v = 0; v < views; ++v) {
        AntialiasParams p{};
        size_t po = (size_t)v * W * H;
        fill_aa(p.kernel, W, H, C, clip + (size_t)v * nv * 4, tri, rast + po * 4, in + po * C);
        p.kernel.out = out + po * C;
        Antialias::forward(p);
    }
}
void ref_antialias_bwd(int /*mode*/, int W, int H, int views, int C, const float* clip, int nv,
                       const uint32_t* tri, const float* rast, const float* in, const float* g_out,
                       float* g_in, float* g_clip) {
    for (int v = 0; v < views; ++v) {
        AntialiasGradParams p{};
        size_t po = (size_t)v * W * H;
        fill_aa(p.kernel, W, H, C, clip + (size_t)v * nv * 4, tri, rast + po * 4, in + po * C);
        p.grad.out = const_cast<float*>(g_out) + po * C;
        p.grad.in = g_in + po * C;
        p.grad.proj = g_clip ? g_clip + (size_t)v * nv * 4 : nullptr;
        Antialias::backward(p);
    }
}

// material.cu:71-77 (the normal-map branch is never taken, see :40)
void ref_normal_axis_fwd(int W, int H, int views, const float* rast, const float* rot, const float* normal,
                         const uint32_t* tri, float* out) {
    static float dummy_map[4];
    NormalAxisParams p{};
    p.kernel.width = W; p.kernel.height = H; p.kernel.depth = views;
    p.kernel.rast = const_cast<float*>(rast); p.kernel.rot = const_cast<float*>(rot);
    p.kernel.normal = const_cast<float*>(normal); p.kernel.normalidx = const_cast<unsigned*>(tri);
    p.kernel.normalmap = dummy_map;  // bound, as the reference preset binds one
    p.kernel.out = out;
    NormalAxis::forward(p);
}

// material.cu:92-108 launched as ViewAxis::forward does (:110-118), with the
// caller's per-view inverse in place of the glm one.
void ref_view_axis_fwd(int W, int H, int views, const float* pvinv, float* out) {
    for (int v = 0; v < views; ++v) {
        ViewAxisParams p{};
        p.kernel.width = W; p.kernel.height = H; p.kernel.depth = 1;
        p.kernel.pvinv = const_cast<float*>(pvinv) + (size_t)v * 9;
        p.kernel.out = out + (size_t)v * W * H * 3;
        dim3 block = getBlock(W, H);
        dim3 grid = getGrid(block, W, H, 1);
        void* args[] = {&p.kernel};
        cudaLaunchKernel(ViewAxisForwardKernel, grid, block, args, 0, NULL);
    }
}

// material.cu:185-201, :251-256
void ref_sg_specular_fwd(int W, int H, int views, const float* rast, const float* normal, const float* view,
                         const float* rough, float ior, float* o_axis, float* o_sharp, float* o_amp) {
    SGSpecularParams p{};
    p.kernel.width = W; p.kernel.height = H; p.kernel.depth = views;
    p.kernel.rast = const_cast<float*>(rast); p.kernel.normal = const_cast<float*>(normal);
    p.kernel.view = const_cast<float*>(view); p.kernel.roughness = const_cast<float*>(rough);
    p.kernel.ior = ior; p.kernel.outAxis = o_axis; p.kernel.outSharpness = o_sharp; p.kernel.outAmplitude = o_amp;
    SGSpecular::forward(p);
}
void ref_sg_specular_bwd(int W, int H, int views, const float* rast, const float* normal, const float* view,
                         const float* rough, float ior, const float* g_amp, const float* g_sharp, float* g_rough) {
    SGSpecularGradParams p{};
    p.kernel.width = W; p.kernel.height = H; p.kernel.depth = views;
    p.kernel.rast = const_cast<float*>(rast); p.kernel.normal = const_cast<float*>(normal);
    p.kernel.view = const_cast<float*>(view); p.kernel.roughness = const_cast<float*>(rough);
    p.kernel.ior = ior;
    p.grad.outAmplitude = const_cast<float*>(g_amp); p.grad.outSharpness = const_cast<float*>(g_sharp);
    p.grad.roughness = g_rough;
    SGSpecular::backward(p);
}

// material.cu:325-339, :440-445.  The backward accumulates lobe gradients
// without atomics, so it always runs in serial order here.
static void fill_sg(SphericalGaussianKernelParams& k, int W, int H, int views, int C, const float* rast, int K,
                    const float* axis, const float* sharp, const float* amp, const float* normal,
                    const float* diffuse, const float* sax, const float* ssh, const float* sam) {
    k.width = W; k.height = H; k.depth = views; k.channel = C;
    k.rast = const_cast<float*>(rast); k.sgnum = K;
    k.axis = const_cast<float*>(axis); k.sharpness = const_cast<float*>(sharp); k.amplitude = const_cast<float*>(amp);
    k.normal = const_cast<float*>(normal); k.diffuse = const_cast<float*>(diffuse);
    k.specAxis = const_cast<float*>(sax); k.specSharpness = const_cast<float*>(ssh); k.specAmplitude = const_cast<float*>(sam);
}
void ref_sg_fwd(int W, int H, int views, int C, const float* rast, int K, const float* axis, const float* sharp,
                const float* amp, const float* normal, const float* diffuse, const float* sax, const float* ssh,
                const float* sam, float* out, float* o_diff, float* o_spec) {
    SphericalGaussianParams p{};
    fill_sg(p.kernel, W, H, views, C, rast, K, axis, sharp, amp, normal, diffuse, sax, ssh, sam);
    p.kernel.out = out; p.kernel.outDiffenv = o_diff; p.kernel.outSpecenv = o_spec;
    SphericalGaussian::forward(p);
}
void ref_sg_bwd(int /*mode*/, int W, int H, int views, int C, const float* rast, int K, const float* axis,
                const float* sharp, const float* amp, const float* normal, const float* diffuse, const float* sax,
                const float* ssh, const float* sam, const float* g_out, float* g_diffuse, float* g_axis,
                float* g_sharp, float* g_amp, float* g_sax, float* g_ssh, float* g_sam) {
    SphericalGaussianGradParams p{};
    fill_sg(p.kernel, W, H, views, C, rast, K, axis, sharp, amp, normal, diffuse, sax, ssh, sam);
    p.grad.out = const_cast<float*>(g_out);
    p.grad.diffuse = g_diffuse; p.grad.normal = nullptr;
    p.grad.axis = g_axis; p.grad.sharpness = g_sharp; p.grad.amplitude = g_amp;
    p.grad.specAxis = g_sax; p.grad.specSharpness = g_ssh; p.grad.specAmplitude = g_sam;
    int saved = vclref_force_serial;
    vclref_force_serial = 1;
    SphericalGaussian::backward(p);
    vclref_force_serial = saved;
}

// loss.cu:3-21 (Loss::init) and :41-57 (MSELoss::backward)
float ref_mse(int /*mode*/, size_t n, const float* pred, const float* target, float* grad) {
    LossParams p{};
    Loss::init(p, const_cast<float*>(target), const_cast<float*>(pred), grad, (int)n, 1, 1);
    MSELoss::backward(p);
    float l = Loss::loss(p);
    cudaFree(p.kernel.buffer);
    return l;
}

// optimize.cu:3-12 (Optimizer::init), :84-115 (Adam); the moment buffers
// are the caller's; rhomt/rhovt are set to the value Adam::step would hold
// before its `step`-th call.
void ref_adam(int /*mode*/, size_t n, float* p, const float* g, float* m, float* v, double lr, double b1,
              double b2, double eps, int step) {
    AdamParams a{};
    Optimizer::init(a, p, const_cast<float*>(g), (int)n, (int)n, 1, 1);
    a.hyper.rhom = b1; a.hyper.rhov = b2; a.hyper.eta = lr; a.hyper.eps = eps;
    a.hyper.rhomt = b1; a.hyper.rhovt = b2;
    for (int k = 1; k < step; ++k) { a.hyper.rhomt *= b1; a.hyper.rhovt *= b2; }
    a.hyper.m = m; a.hyper.v = v;
    Adam::step(a);
}

}  // extern "C"

// Fused fit iteration.  Same operators and arithmetic as the plain path
// (fit_plain.cu), regrouped so that per-pixel intermediates stay in
// registers instead of round-tripping through HBM:
//
//   begin        device step counter, Adam bias corrections, loss := 0
//   project      clip-space positions
//   raster       setup / scan / emit / fine (own workspace)
//   shade_fwd    interpolate(uv, DA) + texture + NormalAxis + ViewAxis +
//                SGSpecular + SG per pixel -> color, diffuse environment sum
//   antialias    silhouette blending (gather form, deterministic)
//   mse          grad = aa - target and the loss
//   aa bwd       colour and clip-position gradients at silhouettes
//   bwd_pix      per pixel: diffuse gradient = grad * diffuse environment,
//                texture backward (texel atomics), interpolate backward,
//                raster backward (clip atomics)
//   sg_lobes     lobe gradients, lobe-parallel, on a forked stream beside
//                bwd_pix
//   project bwd  position gradients
//   adam_tex     mip gradient push-down + Adam + clamp on texture level 0,
//                gradient clear, and mip levels 1..5 of each 32x32 tile
//   mips         remaining coarse levels
//   adam_small   Adam on positions and lobes, gradient clear
//
// On a non-default stream the whole step is captured once into a CUDA
// graph and replayed (the step index lives in device memory, so the graph
// never changes).
#include <map>
#include <mutex>
#include <tuple>

#include "fit.cuh"
#include "sg_math.cuh"
#include "tex_math.cuh"
#include "adam_math.cuh"
#include "ops_internal.cuh"

namespace {

struct Fused {
    void* raster_ws = nullptr;
    size_t raster_ws_bytes = 0;
    RasterSched sched{16, 0, 0, 0};
    bool sched_cached = false;                 // schedule taken from the tuning cache
    int* flags = nullptr;                      // [0] overflowed raster tiles of the last step
    float* scr = nullptr;                      // per view-vertex screen terms for the antialias kernels
    int* d_step = nullptr;                     // [0] step counter, [8] shading records of this step
    double* d_corr = nullptr;    // [0..1] 1 - beta1^t', 1 - beta2^t'; [2] loss sum, [3] its block counter
    cudaGraph_t graph_def = nullptr;           // the captured step (child of batch graphs)
    cudaGraphExec_t graph = nullptr;
    int graph_mode = -1;
    cudaStream_t side = nullptr;               // lobe-gradient branch
    float tune_ms[3] = {0.f, 0.f, 0.f};        // best raster time per tile size 8/16/32
    cudaEvent_t fork = nullptr, join = nullptr;
};

DEV float mulr(float a, float b) { return __fmul_rn(a, b); }
DEV float addr(float a, float b) { return __fadd_rn(a, b); }

__global__ void k_begin(int* step, double* corr, double b1, double b2, int compat, float* loss) {
    int t = ++*step;
    double c1 = compat ? b1 : 1.0, c2 = compat ? b2 : 1.0;
    for (int k = 0; k < t; ++k) { c1 *= b1; c2 *= b2; }
    corr[0] = 1.0 - c1;
    corr[1] = 1.0 - c2;
    *loss = 0.f;
}

struct ShadeIn {
    const float4* rast; const float4* db; const float* uvattr; const uint32_t* tri; int nt, nv;
    const float* pyr; const float* rot; const float* nrm; const float* pvinv;
    int W, H; long long npix; float rough, ior;
    const float* axis; const float* sharp; const float* amp; int K, C;
    // pixel index -> (view, row, column) by multiply-high (npix < 2^31), and
    // W, H, 2 / W, 2 / H as floats (exactly what the kernels would compute)
    FastDiv div_w, div_hw;
    float fW, fH, xs, ys;
};

// Everything the SG stage needs at one covered pixel, recomputed from the
// raster output the way the plain operators compute it.
struct PixIn {
    float2 uv; float4 uvda; float4 dfs; float3 n, pax; float ss, sa;
    uint32_t i0, i1, i2; float4 r;
    float fl; int lv;    // trilinear fraction, levels l0 | l1 << 8
};

// Shading records of the covered pixels, written by k_shade_fwd and read by
// k_sg_lobes in the same step: (n, ss), (p, sa), the diffuse texture colour
// and the pixel index, compacted in the order the blocks claim their slots.
// The lobe pass then reads three coalesced vectors and one gathered dL/dout
// per pixel instead of redoing interpolation, the texture fetch and the
// normal / view / specular set-up.
struct ShadeRec {
    float4* nss; float4* psa; float4* dfs; uint32_t* pix;
    int* count;          // records written this step (reset before the shading pass)
    // Per pixel (not compacted), for the per-pixel backward: the texture
    // sample (u, v, level fraction, l0 | l1 << 8 as int bits) of each covered
    // pixel, so that its texel loads need not wait on triangle -> attributes.
    float4* tsr;
};

template <int C4>
DEV bool shade_inputs(const ShadeIn& a, const TexDesc& td, long long p, PixIn& o) {
    float4 r = a.rast[p];
    o.r = r;
    int idx = rast_id(r.w);
    if (idx < 0 || idx >= a.nt) return false;
    uint32_t i0 = a.tri[3 * (size_t)idx], i1 = a.tri[3 * (size_t)idx + 1], i2 = a.tri[3 * (size_t)idx + 2];
    if (i0 >= (uint32_t)a.nv || i1 >= (uint32_t)a.nv || i2 >= (uint32_t)a.nv) return false;
    o.i0 = i0; o.i1 = i1; o.i2 = i2;
    // interpolate.cu:38 and :40-47 (uv with screen derivatives)
    float4 d = a.db[p];
    double l2 = __dsub_rn(__dsub_rn(1.0, (double)r.x), (double)r.y);
    float u[2], dx[2], dy[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        float a0 = a.uvattr[2 * i0 + i], a1 = a.uvattr[2 * i1 + i], a2 = a.uvattr[2 * i2 + i];
        u[i] = (float)__dadd_rn((double)addr(mulr(a0, r.x), mulr(a1, r.y)), __dmul_rn((double)a2, l2));
        float dadu = a0 - a2, dadv = a1 - a2;
        dx[i] = addr(mulr(dadu, d.x), mulr(dadv, d.z));
        dy[i] = addr(mulr(dadu, d.y), mulr(dadv, d.w));
    }
    o.uv = make_float2(u[0], u[1]);
    o.uvda = make_float4(dx[0], dy[0], dx[1], dy[1]);
    // texturemap.cu:67-95
    int l0 = 0, l1 = 0;
    float fl = 0.f;
    if (td.L > 1) calc_level(td, o.uvda, l0, l1, fl, nullptr, 0);
    o.fl = fl;
    o.lv = l0 | l1 << 8;
    int q0[4];
    float2 f0;
    index_fetch(td, l0, o.uv, q0, f0);
    const float* T0 = a.pyr + td.off[l0];
    float4 c = bilerp4(ld4(T0, q0[0]), ld4(T0, q0[1]), ld4(T0, q0[2]), ld4(T0, q0[3]), f0);
    if (td.L > 1 && fl > 0) {
        int q1[4];
        float2 f1;
        index_fetch(td, l1, o.uv, q1, f1);
        const float* T1 = a.pyr + td.off[l1];
        float4 c1 = bilerp4(ld4(T1, q1[0]), ld4(T1, q1[1]), ld4(T1, q1[2]), ld4(T1, q1[3]), f1);
        c = make_float4(lerpf_(c.x, c1.x, fl), lerpf_(c.y, c1.y, fl), lerpf_(c.z, c1.z, fl), lerpf_(c.w, c1.w, fl));
    }
    o.dfs = c;
    // material.cu:36-47 (NormalAxis)
    float3 n2 = ld3(a.nrm, i2);
    float3 n0 = ld3(a.nrm, i0) - n2, n1 = ld3(a.nrm, i1) - n2;
    float3 N = normalize3(n0 * r.x + n1 * r.y + n2);
    const float* R = a.rot;
    o.n = f3(R[0] * N.x + R[4] * N.y + R[8] * N.z, R[1] * N.x + R[5] * N.y + R[9] * N.z,
             R[2] * N.x + R[6] * N.y + R[10] * N.z);
    // material.cu:99-107 (ViewAxis)
    const unsigned hw = (unsigned)a.W * (unsigned)a.H, view = fastdiv((unsigned)p, a.div_hw);
    const unsigned rem = (unsigned)p - view * hw, py = fastdiv(rem, a.div_w), px = rem - py * (unsigned)a.W;
    const float* M = a.pvinv + (size_t)view * 9;
    float sx = (float)px / a.fW * 2.f - 1.f, sy = (float)py / a.fH * 2.f - 1.f;
    float3 vw = normalize3(f3(M[0], M[1], M[2]) * sx + f3(M[3], M[4], M[5]) * sy + f3(M[6], M[7], M[8]));
    // material.cu:155-182 (SGSpecular)
    SpecLobe s = spec_eval(o.n, vw, a.rough, a.ior);
    o.pax = s.p;
    o.sa = s.F * s.Gp * s.Gv * s.pn / fmaxf(s.m2, 1e-6f);
    o.ss = .5f / fmaxf(s.m2 * s.vn, 1e-6f);
    return true;
}

// Forward shading of every pixel; writes the color and the diffuse
// environment sum (kept for the backward's diffuse gradient) and, when
// rec.count is set, the shading record of each covered pixel (one slot
// claim per block).  C = 4; 128 threads, held to 40 registers for twelve
// blocks per SM (more warps to cover the texture and attribute loads, and a
// finer grain for the block scheduler than 256-thread blocks).
__global__ void __launch_bounds__(128, 12) k_shade_fwd(ShadeIn a, TexDesc td, float4* __restrict__ color,
                                                   float4* __restrict__ diffenv, ShadeRec rec) {
    extern __shared__ float4 sm4[];
    __shared__ int s_off[8], s_base;
    sg_stage_lobes4(sm4, a.K, a.axis, a.sharp, a.amp);
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    PixIn q;
    const bool live = p < a.npix && shade_inputs<1>(a, td, p, q);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned ball = __ballot_sync(0xffffffffu, live);
    if (rec.count && lane == 0) s_off[wid] = __popc(ball);
    __syncthreads();
    if (rec.count && threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            const int c = s_off[w];
            s_off[w] = t;
            t += c;
        }
        s_base = t ? atomicAdd(rec.count, t) : 0;
    }
    __syncthreads();
    if (p >= a.npix) return;
    if (!live) {
        color[p] = diffenv[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    if (rec.tsr) rec.tsr[p] = make_float4(q.uv.x, q.uv.y, q.fl, __int_as_float(q.lv));
    if (rec.count) {
        const int k = s_base + s_off[wid] + __popc(ball & ((1u << lane) - 1u));
        rec.nss[k] = make_float4(q.n.x, q.n.y, q.n.z, q.ss);
        rec.psa[k] = make_float4(q.pax.x, q.pax.y, q.pax.z, q.sa);
        rec.dfs[k] = q.dfs;
        rec.pix[k] = (uint32_t)p;
    }
    float4 de, se;
    sg_env4(sm4, a.K, q.n, q.pax, q.ss, q.sa, de, se);
    diffenv[p] = de;
    color[p] = make_float4(q.dfs.x * de.x + se.x, q.dfs.y * de.y + se.y, q.dfs.z * de.z + se.z, q.dfs.w * de.w + se.w);
}

// Per-pixel backward below the SG stage: the diffuse gradient is
// grad ⊙ diffenv (material.cu:429 summed over the lobes), then texture
// backward (texturemap.cu:229-284), interpolate backward to the
// barycentrics (interpolate.cu:114-143) and raster backward
// (rasterize.cu:84-141), scattered with vector reductions.
// The clip-position gradient of one pixel's three vertices (x, y, w each;
// z receives +0) and the triangle they belong to.
struct VtxGrad {
    float v[9];
    uint32_t i[3];
    int view;
    bool ok;
};

// One covered pixel's texture sample: its two levels, the 2x2 cells (corner
// u0, v0; the other corner is u0 or u0 + 1, v0 or v0 + 1) with their
// fractions, and the gradient g = dL/dcolour * diffuse env it spreads over
// the texels.
struct PixSample {
    float4 r, g;
    float2 f0, f1;
    float fl;
    int l0, l1, u0, v0, u1, v1, s0, t0, s1, t1;
    uint32_t i0, i1, i2;
    int idx;
    bool tri, ok;
};

DEV void pix_sample(const ShadeIn& a, const TexDesc& td, const float4* __restrict__ g_color,
                    const float4* __restrict__ diffenv, const float4* __restrict__ tsr, long long p, PixSample& S) {
    S.ok = false;
    const float4 r = a.rast[p];
    const int idx = rast_id(r.w);
    if (idx < 0 || idx >= a.nt) return;
    const uint32_t i0 = a.tri[3 * (size_t)idx], i1 = a.tri[3 * (size_t)idx + 1], i2 = a.tri[3 * (size_t)idx + 2];
    if (i0 >= (uint32_t)a.nv || i1 >= (uint32_t)a.nv || i2 >= (uint32_t)a.nv) return;
    // dL/d diffuse = dL/dout * diffuse environment sum, through the
    // reference's guarded add into a cleared gradient (material.cu:429): a
    // non-finite product is dropped (0), so it reaches neither the texels nor
    // the geometry
    const float4 gc = g_color[p], de = diffenv[p];
    S.g = make_float4(finite_or0(gc.x * de.x), finite_or0(gc.y * de.y), finite_or0(gc.z * de.z),
                      finite_or0(gc.w * de.w));
    // the texture sample the shading pass took at this pixel (texturemap.cu:67-95)
    const float4 t = tsr[p];
    const float2 uv = make_float2(t.x, t.y);
    const int lv = __float_as_int(t.w);
    S.l0 = lv & 255; S.l1 = lv >> 8; S.fl = t.z;
    const bool mip = td.L > 1;
    cell_fetch(td, S.l0, uv, S.u0, S.u1, S.v0, S.v1, S.f0);
    S.tri = mip && S.fl > 0;
    S.f1 = make_float2(0.f, 0.f);
    S.s0 = S.s1 = S.t0 = S.t1 = 0;
    if (S.tri) cell_fetch(td, S.l1, uv, S.s0, S.s1, S.t0, S.t1, S.f1);
    if (!mip) S.fl = 0.f;
    S.r = r;
    S.i0 = i0; S.i1 = i1; S.i2 = i2;
    S.idx = idx;
    S.ok = true;
}

// One texel's share of a pixel's texture gradient (texturemap.cu:229-284).
DEV void tex_add(const TexDesc& td, float* __restrict__ g_pyr, int level, int x, int y, float wt, float4 g) {
    red_add4(g_pyr + td.off[level] + 4 * ((size_t)y * (td.tw >> level) + x), wt * g.x, wt * g.y, wt * g.z, wt * g.w);
}

// Geometry part: d colour / d uv from the texel values, back to the
// barycentrics (interpolate.cu:114-143) and to the three clip-space vertices
// (rasterize.cu:84-141).
DEV void pix_geom(const ShadeIn& a, const TexDesc& td, const float* __restrict__ clip, const PixSample& S, int px,
                  int py, int view, VtxGrad& o) {
    const float* T0 = a.pyr + td.off[S.l0];
    const float* T1 = a.pyr + td.off[S.l1];
    const int sx0 = td.tw >> S.l0, sx1 = td.tw >> S.l1;
    const float s0x = (float)sx0, s0y = (float)(td.th >> S.l0);
    const float s1x = (float)sx1, s1y = (float)(td.th >> S.l1);
    const float4 a00 = ld4(T0, S.v0 * sx0 + S.u0), a01 = ld4(T0, S.v0 * sx0 + S.u1);
    const float4 a10 = ld4(T0, S.v1 * sx0 + S.u0), a11 = ld4(T0, S.v1 * sx0 + S.u1);
    float4 b00 = a00, b01 = a00, b10 = a00, b11 = a00;
    if (S.tri) {
        b00 = ld4(T1, S.t0 * sx1 + S.s0); b01 = ld4(T1, S.t0 * sx1 + S.s1);
        b10 = ld4(T1, S.t1 * sx1 + S.s0); b11 = ld4(T1, S.t1 * sx1 + S.s1);
    }
    const float ga[4] = {S.g.x, S.g.y, S.g.z, S.g.w};
    const float A00[4] = {a00.x, a00.y, a00.z, a00.w}, A01[4] = {a01.x, a01.y, a01.z, a01.w};
    const float A10[4] = {a10.x, a10.y, a10.z, a10.w}, A11[4] = {a11.x, a11.y, a11.z, a11.w};
    const float B00[4] = {b00.x, b00.y, b00.z, b00.w}, B01[4] = {b01.x, b01.y, b01.z, b01.w};
    const float B10[4] = {b10.x, b10.y, b10.z, b10.w}, B11[4] = {b11.x, b11.y, b11.z, b11.w};
    float gu = 0.f, gv = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float du = lerpf_(A01[i] - A00[i], A11[i] - A10[i], S.f0.y) * s0x;
        float dv = lerpf_(A10[i] - A00[i], A11[i] - A01[i], S.f0.x) * s0y;
        if (S.tri) {
            du = lerpf_(du, lerpf_(B01[i] - B00[i], B11[i] - B10[i], S.f1.y) * s1x, S.fl);
            dv = lerpf_(dv, lerpf_(B10[i] - B00[i], B11[i] - B01[i], S.f1.x) * s1y, S.fl);
        }
        gu += du * ga[i];
        gv += dv * ga[i];
    }
    float gbu = 0.f, gbv = 0.f;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        float gi = i == 0 ? gu : gv;
        float a2 = a.uvattr[2 * S.i2 + i];
        gbu += gi * (a.uvattr[2 * S.i0 + i] - a2);
        gbv += gi * (a.uvattr[2 * S.i1 + i] - a2);
    }
    if (((__float_as_uint(gbu) | __float_as_uint(gbv)) << 1) == 0u) return;
    const float xs = a.xs, ys = a.ys;
    const float pxn = (float)(((double)px + 0.5) * (double)xs - 1.0);
    const float pyn = (float)(((double)py + 0.5) * (double)ys - 1.0);
    const float4* cv = reinterpret_cast<const float4*>(clip) + (size_t)view * a.nv;
    const float4 c0 = cv[S.i0], c1 = cv[S.i1], c2 = cv[S.i2];
    float p0x = c0.w * pxn - c0.x, p0y = c0.w * pyn - c0.y;
    float p1x = c1.w * pxn - c1.x, p1y = c1.w * pyn - c1.y;
    float p2x = c2.w * pxn - c2.x, p2y = c2.w * pyn - c2.y;
    float e0x = p0x - p2x, e0y = p0y - p2y, e1x = p1x - p2x, e1y = p1y - p2y;
    float ar = e0x * e1y - e0y * e1x;
    float ia = 1.f / (ar + (ar > 0 ? 1e-6f : -1e-6f));
    float kuv = S.r.x * gbu + S.r.y * gbv;
    float gx0 = (gbv * p2y + kuv * e1y) * ia, gy0 = (-gbv * p2x - kuv * e1x) * ia;
    float gx1 = (-gbu * p2y - kuv * e0y) * ia, gy1 = (gbu * p2x + kuv * e0x) * ia;
    float gx2 = ((-gbv * p0y + gbu * p1y) - kuv * (-p0y + p1y)) * ia;
    float gy2 = ((gbv * p0x - gbu * p1x) - kuv * (p0x - p1x)) * ia;
    o.v[0] = gx0; o.v[1] = gy0; o.v[2] = -gx0 * pxn - gy0 * pyn;
    o.v[3] = gx1; o.v[4] = gy1; o.v[5] = -gx1 * pxn - gy1 * pyn;
    o.v[6] = gx2; o.v[7] = gy2; o.v[8] = -gx2 * pxn - gy2 * pyn;
    o.i[0] = S.i0; o.i[1] = S.i1; o.i[2] = S.i2;
    o.view = view;
    o.ok = true;
}

// One thread per pixel.  The vertex gradients are summed by the warp over
// each run of consecutive lanes on the same triangle (a segmented scan by
// shuffles, as many rounds as the longest run needs) and the last lane of a
// run issues its three vector reductions: neighbouring pixels of one
// triangle no longer collide on the same three addresses.  Blocks of 64
// threads at up to 48 registers (a few spills, in L1), so that its blocks
// fit, at a fine grain, on each SM beside the three lobe-gradient blocks it
// runs with.
__global__ void __launch_bounds__(64, 20) k_bwd_pix(ShadeIn a, TexDesc td, const float4* __restrict__ g_color,
                                                 const float4* __restrict__ diffenv, const float4* __restrict__ tsr,
                                                 float* __restrict__ g_pyr,
                                                 const float* __restrict__ clip, float* __restrict__ g_clip,
                                                 int want_tex, int want_geom) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    PixSample S;
    S.ok = false;
    if (p < a.npix) pix_sample(a, td, g_color, diffenv, tsr, p, S);
    if (want_tex && S.ok) {
        const float wl0 = td.L > 1 ? 1.f - S.fl : 1.f;
        const float2 f0 = S.f0;
        tex_add(td, g_pyr, S.l0, S.u0, S.v0, wl0 * (1.f - f0.x) * (1.f - f0.y), S.g);
        tex_add(td, g_pyr, S.l0, S.u1, S.v0, wl0 * f0.x * (1.f - f0.y), S.g);
        tex_add(td, g_pyr, S.l0, S.u0, S.v1, wl0 * (1.f - f0.x) * f0.y, S.g);
        tex_add(td, g_pyr, S.l0, S.u1, S.v1, wl0 * f0.x * f0.y, S.g);
        if (S.tri) {
            const float fl = S.fl;
            const float2 f1 = S.f1;
            tex_add(td, g_pyr, S.l1, S.s0, S.t0, fl * (1.f - f1.x) * (1.f - f1.y), S.g);
            tex_add(td, g_pyr, S.l1, S.s1, S.t0, fl * f1.x * (1.f - f1.y), S.g);
            tex_add(td, g_pyr, S.l1, S.s0, S.t1, fl * (1.f - f1.x) * f1.y, S.g);
            tex_add(td, g_pyr, S.l1, S.s1, S.t1, fl * f1.x * f1.y, S.g);
        }
    }
    if (!want_geom) return;
    const unsigned hw = (unsigned)a.W * (unsigned)a.H;
    const int view = (int)fastdiv((unsigned)p, a.div_hw), rem = (int)((unsigned)p - (unsigned)view * hw);
    const int py = (int)fastdiv((unsigned)rem, a.div_w), px = rem - py * a.W;
    VtxGrad o;
    o.ok = false;
    if (S.ok) pix_geom(a, td, clip, S, px, py, view, o);
    if (!o.ok) {
#pragma unroll
        for (int k = 0; k < 9; ++k) o.v[k] = 0.f;
    }
    // runs: consecutive lanes on the same triangle of the same view; lanes
    // without a vertex gradient form runs of their own
    const bool tail = warp_run_sum(o.v, o.ok ? S.idx : -1 - lane, o.ok ? view : -1);
    if (!(tail && o.ok)) return;
    float* gcv = g_clip + (size_t)view * a.nv * 4;
    red_add4(gcv + (size_t)o.i[0] * 4, o.v[0], o.v[1], 0.f, o.v[2]);
    red_add4(gcv + (size_t)o.i[1] * 4, o.v[3], o.v[4], 0.f, o.v[5]);
    red_add4(gcv + (size_t)o.i[2] * 4, o.v[6], o.v[7], 0.f, o.v[8]);
}

// Lobe gradients (material.cu:428-433), lobe-parallel: a warp stages 32
// shading records as 16 pixel pairs, then each lane walks the pairs for its
// lobe on paired FP32 instructions; sums stay in registers until the end.
// Block row blockIdx.y takes lobes [32 y, 32 y + 32) (fewer than 32 lobes:
// the warp splits into 32 / Kp groups of Kp lanes that walk alternate
// pairs).  Once a chunk is staged, the next chunk's records and dL/dout
// are copied into shared memory asynchronously (cp.async, one buffer per
// warp) while the current one is consumed, their pixel indices loaded one
// chunk earlier still, so no registers hold data in flight.  At most
// LOBE_REGS registers (a few loop-invariant values spill to L1), so that
// three blocks of this kernel and ten 64-thread blocks of the per-pixel
// backward share each SM: the pair finishes sooner than with the lobe kernel
// spill-free at 96 registers beside fewer per-pixel blocks.  C = 4.
constexpr int LOBE_REGS = 88;
template <bool EXACT>
__global__ void __maxnreg__(LOBE_REGS) k_sg_lobes(ShadeIn a, ShadeRec rec, const float4* __restrict__ g_color,
                                                 float* __restrict__ g_axis, float* __restrict__ g_sharp,
                                                 float* __restrict__ g_amp) {
    __shared__ float s_acc[32 * 8];                                  // [lobe][axis xyz, sharpness, amplitude 4]
    __shared__ SPair s_pix[4 * 16];
    __shared__ float4 s_raw[4][4][32];                               // [warp][nss, psa, dfs, dL/dout][lane]
    const int nwarps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int base = 32 * blockIdx.y, Kg = min(32, a.K - base);
    for (int i = threadIdx.x; i < 32 * 8; i += blockDim.x) s_acc[i] = 0.f;
    __syncthreads();
    const int Kp = sg_lobe_group_dev(Kg);
    const int G = 32 / Kp, g = lane / Kp, li = lane % Kp;
    Lobe4x2 L;
    lobe4x2_load(L, li, Kg, a.axis + 3 * base, a.sharp + base, a.amp + 4 * base);
    SPair* st = s_pix + wid * 16;
    float4 (*raw)[32] = s_raw[wid];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const int n = *rec.count;
    const int nchunks = (n + 31) >> 5, stride = gridDim.x * nwarps;
    // copies of chunk cc (this lane's record and dL/dout at pixel pix)
    auto issue = [&](int cc, uint32_t pix) {
        const int k = cc * 32 + lane;
        if (cc < nchunks && k < n) {
            cp_async16(&raw[0][lane], rec.nss + k);
            cp_async16(&raw[1][lane], rec.psa + k);
            cp_async16(&raw[2][lane], rec.dfs + k);
            cp_async16(&raw[3][lane], g_color + pix);
        }
        cp_async_commit();
    };
    // Pass 0 adds every contribution plainly.  A lane whose sums come out
    // non-finite met a non-finite contribution; its warp then walks the same
    // chunks again and that lane alone adds them checked (pass 1).
    bool guard = false;
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        int c = blockIdx.x * nwarps + wid;
        issue(c, (c < nchunks && c * 32 + lane < n) ? rec.pix[c * 32 + lane] : 0u);
        uint32_t pnext = (c + stride < nchunks && (c + stride) * 32 + lane < n) ? rec.pix[(c + stride) * 32 + lane] : 0u;
        for (; c < nchunks; c += stride) {
            const int m = min(32, n - c * 32);
            cp_async_wait<0>();                                      // this chunk's copies (this lane's own)
            if (lane < m) spair_put(st + (lane >> 1), lane & 1, raw[0][lane], raw[1][lane], raw[2][lane], raw[3][lane]);
            if ((m & 1) && lane == 31) spair_put(st + (m >> 1), 1, z4, z4, z4, z4);
            __syncwarp();
            // the staged pair stores consumed this lane's copies: the buffer
            // takes the next chunk's
            issue(c + stride, pnext);
            if (c + 2 * stride < nchunks) {
                const int k2 = (c + 2 * stride) * 32 + lane;
                if (k2 < n) pnext = rec.pix[k2];
            }
            const int npair = (m + 1) >> 1;
            if (L.valid && (pass == 0 || guard))
                for (int j = g; j < npair; j += G) lobe4x2_accumulate<EXACT>(L, st[j], pass != 0);
            __syncwarp();
        }
        cp_async_wait<0>();
        if (pass == 1) break;
        guard = lobe4x2_needs_guard(L);
        if (!__any_sync(0xffffffffu, guard)) break;
        if (guard) lobe4x2_clear(L);
    }
    lobe4x2_flush(L, li, Kp, s_acc);
    __syncthreads();
    for (int j = threadIdx.x; j < Kg * 8; j += blockDim.x) {
        const float v = s_acc[j];
        if (v == 0.f) continue;
        const int i = base + (j >> 3), q = j & 7;
        if (q < 3) atomicAdd(&g_axis[3 * i + q], v);
        else if (q == 3) atomicAdd(&g_sharp[i], v);
        else atomicAdd(&g_amp[4 * i + (q - 4)], v);
    }
}

DEV float4 nan_add4(float4 a, float4 b) {
    add_nan_check(a.x, b.x); add_nan_check(a.y, b.y); add_nan_check(a.z, b.z); add_nan_check(a.w, b.w);
    return a;
}
DEV float4 mul4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
DEV float4 avg4(float4 a, float4 b, float4 c, float4 d) {
    return make_float4(addr(addr(addr(a.x, b.x), c.x), d.x) * 0.25f, addr(addr(addr(a.y, b.y), c.y), d.y) * 0.25f,
                       addr(addr(addr(a.z, b.z), c.z), d.z) * 0.25f, addr(addr(addr(a.w, b.w), c.w), d.w) * 0.25f);
}
DEV float clamp01(float x) { return x < 0.f ? 0.f : x > 1.f ? 1.f : x; }

struct AdamArgs {
    double b1, b2, lr, eps;
    const double* corr;
    double lr1;          // k_adam_small: step size of the second group
};

// TextureGrad::gradSumup (buffer.cu:615-648) folded into level 0, Adam
// (optimize.cu:95-106), clamp (buffer.cu:65-72), gradient clear, and the
// 2x2 mip chain (buffer.cu:449-472) of each 32x32 level-0 tile up to level
// `top` (<= 5).  One thread per 2x2 level-0 quad; C = 4.  Held to 64
// registers for four blocks per SM (the FP64 Adam arithmetic waits on its
// divisions and square roots; the extra warps cover them).
__global__ void __launch_bounds__(256, 4) k_adam_tex_tile(TexDesc td, float* __restrict__ pyr, float* __restrict__ gpyr,
                                                       float* __restrict__ m, float* __restrict__ v, AdamArgs aa,
                                                       float wpush, int top) {
    __shared__ float4 s_lvl[16][16];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int x = blockIdx.x * 16 + tx, y = blockIdx.y * 16 + ty;     // level-1 texel = level-0 quad
    const int W0 = td.tw, L = td.L;
    // pushed-down gradient of the quad's level-1 ancestor chain
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    if (L > 1) {
        t = ld4(gpyr + td.off[L - 1], (y >> (L - 2)) * (td.tw >> (L - 1)) + (x >> (L - 2)));
        for (int k = L - 2; k >= 1; --k)
            t = nan_add4(ld4(gpyr + td.off[k], (y >> (k - 1)) * (td.tw >> k) + (x >> (k - 1))), mul4(t, wpush));
    }
    const double c1 = aa.corr[0], c2 = aa.corr[1];
    float4 out[4];
#pragma unroll
    for (int qd = 0; qd < 4; ++qd) {
        const int X = 2 * x + (qd & 1), Y = 2 * y + (qd >> 1);
        const size_t ti = (size_t)Y * W0 + X;
        float4 g = ld4(gpyr, (int)ti);
        if (L > 1) g = nan_add4(g, mul4(t, wpush));
        float4 P = ld4(pyr, (int)ti), M = ld4(m, (int)ti), V = ld4(v, (int)ti);
        adam_one(P.x, g.x, M.x, V.x, aa.b1, aa.b2, aa.lr, aa.eps, c1, c2);
        adam_one(P.y, g.y, M.y, V.y, aa.b1, aa.b2, aa.lr, aa.eps, c1, c2);
        adam_one(P.z, g.z, M.z, V.z, aa.b1, aa.b2, aa.lr, aa.eps, c1, c2);
        adam_one(P.w, g.w, M.w, V.w, aa.b1, aa.b2, aa.lr, aa.eps, c1, c2);
        P = make_float4(clamp01(P.x), clamp01(P.y), clamp01(P.z), clamp01(P.w));
        reinterpret_cast<float4*>(pyr)[ti] = P;
        reinterpret_cast<float4*>(m)[ti] = M;
        reinterpret_cast<float4*>(v)[ti] = V;
        reinterpret_cast<float4*>(gpyr)[ti] = make_float4(0.f, 0.f, 0.f, 0.f);
        out[qd] = P;
    }
    if (top < 1) return;
    float4 l1 = avg4(out[0], out[1], out[2], out[3]);
    reinterpret_cast<float4*>(pyr + td.off[1])[(size_t)y * (W0 >> 1) + x] = l1;
    s_lvl[ty][tx] = l1;
    __syncthreads();
    for (int k = 2, n = 8; k <= top; ++k, n >>= 1) {
        float4 r;
        const bool act = tx < n && ty < n;
        if (act) r = avg4(s_lvl[2 * ty][2 * tx], s_lvl[2 * ty][2 * tx + 1], s_lvl[2 * ty + 1][2 * tx],
                          s_lvl[2 * ty + 1][2 * tx + 1]);
        __syncthreads();
        if (act) {
            s_lvl[ty][tx] = r;
            const int X = blockIdx.x * n + tx, Y = blockIdx.y * n + ty;
            reinterpret_cast<float4*>(pyr + td.off[k])[(size_t)Y * (W0 >> k) + X] = r;
        }
        __syncthreads();
    }
}

// The same optimizer pass for any channel count / size, one thread per
// level-0 texel channel (no mip chain).
__global__ void k_adam_tex_generic(TexDesc td, float* __restrict__ pyr, float* __restrict__ gpyr, float* __restrict__ m,
                                   float* __restrict__ v, AdamArgs aa, float wpush) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int C = td.C;
    long long n0 = (long long)td.tw * td.th * C;
    if (i >= n0) return;
    int c = (int)(i % C);
    long long t = i / C;
    int X = (int)(t % td.tw), Y = (int)(t / td.tw);
    float g = gpyr[i];
    if (td.L > 1) {
        int L = td.L;
        float tv = gpyr[td.off[L - 1] + ((long long)(Y >> (L - 1)) * (td.tw >> (L - 1)) + (X >> (L - 1))) * C + c];
        for (int k = L - 2; k >= 1; --k) {
            float gk = gpyr[td.off[k] + ((long long)(Y >> k) * (td.tw >> k) + (X >> k)) * C + c];
            add_nan_check(gk, tv * wpush);
            tv = gk;
        }
        add_nan_check(g, tv * wpush);
    }
    float P = pyr[i], M = m[i], V = v[i];
    adam_one(P, g, M, V, aa.b1, aa.b2, aa.lr, aa.eps, aa.corr[0], aa.corr[1]);
    pyr[i] = clamp01(P);
    m[i] = M;
    v[i] = V;
    gpyr[i] = 0.f;
}

// Adam on positions then lobes (one flat index space), gradient clear.
__global__ void k_adam_small(float* __restrict__ p0, float* __restrict__ g0, float* __restrict__ mv0, long long n0,
                             float* __restrict__ p1, float* __restrict__ g1, float* __restrict__ mv1, long long n1,
                             AdamArgs aa) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float *p, *g, *m, *v;
    long long j;
    if (i < n0) { p = p0; g = g0; m = mv0; v = mv0 + n0; j = i; }
    else if (i < n0 + n1) { p = p1; g = g1; m = mv1; v = mv1 + n1; j = i - n0; }
    else return;
    float P = p[j], M = m[j], V = v[j];
    adam_one(P, g[j], M, V, aa.b1, aa.b2, i < n0 ? aa.lr : aa.lr1, aa.eps, aa.corr[0], aa.corr[1]);
    p[j] = P; m[j] = M; v[j] = V; g[j] = 0.f;
}

#define TRY(x) do { vcl_status _s = (x); if (_s) return _s; } while (0)

size_t shade_smem(int K) { return sg_lobes4_smem(K); }

vcl_status autotune_raster(vcl_fit* f);

vcl_status fused_init(vcl_fit* f) {
    if (f->fused) return VCL_OK;
    vcl_ctx* ctx = f->ctx;
    const vcl_fit_desc& d = f->d;
    const size_t N = (size_t)d.W * d.H * d.views;
    VCL_REQUIRE(N <= (size_t)INT32_MAX - (1u << 24), "fused strategy: W*H*views = %zu pixels, above 2^31 - 2^24", N);
    VCL_REQUIRE((size_t)((const char*)(f->sam + N) - (const char*)f->normal) >= (2 * sizeof(float4) + 4) * N &&
                    f->normal < f->sam && ((uintptr_t)f->normal & 15) == 0 && ((uintptr_t)f->uv_da & 15) == 0 &&
                    ((uintptr_t)f->g_diffuse & 15) == 0 &&
                    (f->rough < f->normal || f->rough >= f->sam + N),
                "fused strategy: shading record area too small (internal layout error)");
    Fused* F = new Fused();
    cudaStream_t as = ctx->aux;
    cudaError_t e = cudaMallocAsync(&F->d_step, 64, as);
    if (e == cudaSuccess) e = cudaMallocAsync(&F->d_corr, 64, as);
    if (e == cudaSuccess) e = cudaMallocAsync(&F->flags, 64, as);
    if (e == cudaSuccess) e = cudaMallocAsync(&F->scr, sizeof(float) * 8 * (size_t)d.views * d.nv, as);
    if (e == cudaSuccess) e = cudaMemsetAsync(F->flags, 0, 64, as);
    if (e == cudaSuccess) e = cudaMemsetAsync(F->d_corr, 0, 64, as);
    if (e == cudaSuccess) e = cudaMemcpyAsync(F->d_step, &f->step_count, sizeof(int), cudaMemcpyHostToDevice, as);
    if (e == cudaSuccess) e = cudaStreamSynchronize(as);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        if (F->d_step) cudaFreeAsync(F->d_step, as);
        if (F->d_corr) cudaFreeAsync(F->d_corr, as);
        if (F->flags) cudaFreeAsync(F->flags, as);
        if (F->scr) cudaFreeAsync(F->scr, as);
        delete F;
        return vcl_fail(ctx, VCL_ERR_NOMEM, "fused fit state: %s", cudaGetErrorString(e));
    }
    f->fused = F;
    e = cudaStreamCreateWithFlags(&F->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&F->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&F->join, cudaEventDisableTiming);
    if (e != cudaSuccess) return vcl_cuda_check(ctx, e, "fused streams");
    size_t sf = shade_smem(d.K);
    if (sf > 48 * 1024) cudaFuncSetAttribute(k_shade_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sf);
    return autotune_raster(f);
}

// Grows the job's raster workspace.  Called only while the job has no step
// in flight (from the autotuner, before its step is captured), so the old
// buffer can go back to the pool once the job's own stream is idle.
vcl_status raster_ws_ensure(vcl_fit* f, size_t bytes) {
    Fused* F = (Fused*)f->fused;
    if (bytes <= F->raster_ws_bytes) return VCL_OK;
    cudaStream_t as = f->ctx->aux;
    cudaError_t e = cudaSuccess;
    if (F->raster_ws) {
        e = cudaStreamSynchronize(F->side);
        if (e == cudaSuccess) e = cudaFreeAsync(F->raster_ws, as);
        F->raster_ws = nullptr;
        F->raster_ws_bytes = 0;
    }
    if (e == cudaSuccess) e = cudaMallocAsync(&F->raster_ws, bytes, as);
    if (e == cudaSuccess) e = cudaStreamSynchronize(as);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        F->raster_ws = nullptr;
        return vcl_fail(f->ctx, VCL_ERR_NOMEM, "raster workspace of %zu bytes: %s", bytes, cudaGetErrorString(e));
    }
    F->raster_ws_bytes = bytes;
    return VCL_OK;
}

// Process-wide cache of tuned raster schedules, keyed by the image size, the
// number of views and the triangle count's power-of-two bucket.
struct TuneKey {
    int W, H, views, nt_log2;
    bool operator<(const TuneKey& o) const {
        return std::tie(W, H, views, nt_log2) < std::tie(o.W, o.H, o.views, o.nt_log2);
    }
};
struct TuneVal {
    int tile, small_area;
    double cap_per_tri;   // bin entries per (view, triangle)
    float ms[3];
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

TuneKey tune_key(const vcl_fit_desc& d) {
    int lg = 0;
    while ((1ll << (lg + 1)) <= (long long)d.nt) ++lg;
    return TuneKey{d.W, d.H, d.views, lg};
}

// The automatic capacity (6 entries per view and triangle plus headroom) is
// the floor: the bins of a deforming mesh grow during the fit, and an
// overflowing tile takes the slow every-triangle path.
long long cap_floor(const vcl_fit_desc& d, int tile) { return raster_auto_capacity(d.views, d.nt, d.W, d.H, tile); }

// Raster autotuner.  Times the binning schedules on this job's own
// geometry -- tile edge {8, 16, 32} at the default direct-rasterization box
// area, then box areas {0, 64, 1024} pixels at the best tile -- keeps the
// fastest, then sizes the bin-list capacity to twice
// the entries that schedule asked for, never below the automatic capacity
// (the mesh moves during the fit; an overflowing tile still gets exact
// results through the all-triangle fallback, only slower).  Jobs of the same size bucket reuse the cached choice.  Runs
// once per job, outside any capture.
vcl_status autotune_raster(vcl_fit* f) {
    vcl_ctx* ctx = f->ctx;
    Fused* F = (Fused*)f->fused;
    const vcl_fit_desc& d = f->d;
    const TuneKey key = tune_key(d);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            long long cap = (long long)(it->second.cap_per_tri * d.views * d.nt);
            if (cap < cap_floor(d, it->second.tile)) cap = cap_floor(d, it->second.tile);
            F->sched = RasterSched{it->second.tile, cap, it->second.small_area, raster_default_medium_area()};
            for (int i = 0; i < 3; ++i) F->tune_ms[i] = it->second.ms[i];
            F->sched_cached = true;
            return raster_ws_ensure(f, raster_ws_size(d.W, d.H, d.views, d.nt, F->sched.tile, cap));
        }
    }
    if (!ctx->autotune) {
        // size-based schedule (no timing): large tiles for large images
        const int t = (d.W >= 512 && d.H >= 512) ? 32 : 16;
        long long cap = raster_auto_capacity(d.views, d.nt, d.W, d.H, t);
        F->sched = RasterSched{t, cap, raster_default_small_area(), raster_default_medium_area()};
        F->sched_cached = false;
        return raster_ws_ensure(f, raster_ws_size(d.W, d.H, d.views, d.nt, t, cap));
    }
    const int tiles[3] = {8, 16, 32};
    const int smalls[4] = {0, 64, 256, 1024};
    long long cap = 0;
    size_t ws = 0;
    for (int t : tiles) {
        long long c = raster_auto_capacity(d.views, d.nt, d.W, d.H, t);
        if (c > cap) cap = c;
    }
    for (int t : tiles) {
        size_t b = raster_ws_size(d.W, d.H, d.views, d.nt, t, cap);
        if (b > ws) ws = b;
    }
    vcl_status st = raster_ws_ensure(f, ws);
    if (st) return st;
    cudaStream_t s = F->side;
    st = vcl_project_fwd(ctx, f->mvp, d.views, f->pos, d.nv, 4, f->clip, s);
    if (st) return st;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return vcl_fail(ctx, VCL_ERR_CUDA, "autotune events");
    float best = 1e30f;
    RasterSched pick{16, cap, raster_default_small_area(), raster_default_medium_area()};
    for (int i = 0; i < 3; ++i) F->tune_ms[i] = 1e30f;
    auto time_sched = [&](const RasterSched& rs, float& ms) -> vcl_status {
        vcl_status r = VCL_OK;
        for (int rep = 0; rep < 3 && r == VCL_OK; ++rep) {
            if (rep == 1) cudaEventRecord(e0, s);
            r = raster_fwd_ws(ctx, F->raster_ws, rs, F->flags, f->clip, d.nv, f->tri, d.nt, d.W, d.H, d.views,
                              f->rast, f->db, s);
        }
        cudaEventRecord(e1, s);
        if (r) return r;
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= 2.f;
        return VCL_OK;
    };
    // tile edge at the default direct area, then the direct area at that tile
    for (int ti = 0; ti < 3 && st == VCL_OK; ++ti) {
        RasterSched rs{tiles[ti], cap, raster_default_small_area(), raster_default_medium_area()};
        float ms = 0.f;
        st = time_sched(rs, ms);
        F->tune_ms[ti] = ms;
        if (!st && ms < best) { best = ms; pick = rs; }
    }
    for (int sa : smalls) {
        if (st || sa == raster_default_small_area()) continue;
        RasterSched rs{pick.tile, cap, sa, raster_default_medium_area()};
        float ms = 0.f;
        st = time_sched(rs, ms);
        if (!st && ms < best) { best = ms; pick = rs; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    // bin demand of the chosen schedule on the starting geometry
    st = raster_fwd_ws(ctx, F->raster_ws, pick, F->flags, f->clip, d.nv, f->tri, d.nt, d.W, d.H, d.views, f->rast,
                       f->db, s);
    long long demand = 0;
    if (!st) st = raster_bin_demand(ctx, F->raster_ws, pick, d.W, d.H, d.views, d.nt, s, &demand);
    if (st) return st;
    long long sized = 2 * demand;
    if (sized < cap_floor(d, pick.tile)) sized = cap_floor(d, pick.tile);
    pick.cap = sized;
    st = vcl_cuda_check(ctx, cudaStreamSynchronize(s), "autotune");
    if (!st) st = raster_ws_ensure(f, raster_ws_size(d.W, d.H, d.views, d.nt, pick.tile, sized));
    if (st) return st;
    F->sched = pick;
    F->sched_cached = false;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        TuneVal v{pick.tile, pick.small_area, (double)sized / ((double)d.views * (d.nt > 0 ? d.nt : 1)),
                  {F->tune_ms[0], F->tune_ms[1], F->tune_ms[2]}};
        g_tune[key] = v;
    }
    return VCL_OK;
}

ShadeIn shade_in(const vcl_fit* f) {
    const vcl_fit_desc& d = f->d;
    ShadeIn a;
    a.rast = (const float4*)f->rast; a.db = (const float4*)f->db; a.uvattr = f->uvattr; a.tri = f->tri;
    a.nt = d.nt; a.nv = d.nv; a.pyr = f->pyr; a.rot = f->rot; a.nrm = f->nrmattr; a.pvinv = f->pvinv;
    a.W = d.W; a.H = d.H; a.npix = (long long)d.W * d.H * d.views; a.rough = d.roughness; a.ior = d.ior;
    a.axis = f->axis; a.sharp = f->sharp; a.amp = f->amp; a.K = d.K; a.C = 4;
    a.div_w = fastdiv_make((unsigned)d.W);
    a.div_hw = fastdiv_make((unsigned)d.W * (unsigned)d.H);
    a.fW = (float)d.W; a.fH = (float)d.H;
    a.xs = 2.f / a.fW; a.ys = 2.f / a.fH;
    return a;
}

// The fused step does not use the plain strategy's per-pixel intermediates,
// so its shading records live there: the stretch from `normal` to the end of
// `sam` (11 floats per pixel, checked in fused_init) holds (n, ss), (p, sa)
// and the pixel indices, `uv_da` (4 floats per pixel) the diffuse colours,
// `g_diffuse` (C = 4 floats per pixel) the texture samples.
ShadeRec shade_rec(const vcl_fit* f, bool want) {
    const size_t N = (size_t)f->d.W * f->d.H * f->d.views;
    float4* r = reinterpret_cast<float4*>(f->normal);
    ShadeRec x;
    x.nss = r; x.psa = r + N;
    x.pix = reinterpret_cast<uint32_t*>(r + 2 * N);
    x.dfs = reinterpret_cast<float4*>(f->uv_da);
    x.count = want ? ((Fused*)f->fused)->d_step + 8 : nullptr;
    x.tsr = (f->d.learn_tex || f->d.learn_pos) ? reinterpret_cast<float4*>(f->g_diffuse) : nullptr;
    return x;
}

// The antialias candidate lists (aa_cand_list_bytes) live in `g_uv`, which
// the fused step does not use, when they fit there (8 bytes per pixel; only
// images of a few pixels per tile do not), else the backward finds its
// candidates again.
uint16_t* aa_cand_list(const vcl_fit* f) {
    const size_t N = (size_t)f->d.W * f->d.H * f->d.views;
    return aa_cand_list_bytes(f->d.W, f->d.H, f->d.views) <= sizeof(float) * 2 * N
               ? reinterpret_cast<uint16_t*>(f->g_uv) : nullptr;
}

// The fused stages, each one launch (shared by the captured step and the
// per-kernel timing).
vcl_status stage_shade(vcl_fit* f, const ShadeIn& a, const TexDesc& td, cudaStream_t s) {
    const ShadeRec rec = shade_rec(f, f->d.learn_lobes && f->d.K);
    if (rec.count) TRY(vcl_cuda_check(f->ctx, cudaMemsetAsync(rec.count, 0, sizeof(int), s), "record count"));
    k_shade_fwd<<<vcl_blocks(a.npix, 128), 128, shade_smem(a.K), s>>>(a, td, (float4*)f->color, (float4*)f->diffuse,
                                                                     rec);
    return vcl_launch_check(f->ctx, "fused shade");
}

// Antialias forward fused with the MSE (loss.cu:22-30): writes the loss
// gradient of the antialiased image and the loss; the image itself is not
// kept.  The double loss sum and its block counter live in d_corr[2..3].
vcl_status stage_aa_mse(vcl_fit* f, cudaStream_t s) {
    const vcl_fit_desc& d = f->d;
    Fused* F = (Fused*)f->fused;
    return aa_edges_fwd_mse(f->ctx, f->clip, F->scr, d.nv, f->tri, d.nt, f->rast, d.W, d.H, d.views, f->color,
                            f->target, f->g_aa, F->d_corr + 2, reinterpret_cast<unsigned*>(F->d_corr + 3), f->loss,
                            aa_cand_list(f), s);
}

// The antialias backward of the step, reusing the forward's candidate lists.
vcl_status stage_aa_bwd(vcl_fit* f, cudaStream_t s) {
    const vcl_fit_desc& d = f->d;
    Fused* F = (Fused*)f->fused;
    return aa_edges_bwd(f->ctx, f->clip, F->scr, d.nv, f->tri, d.nt, f->rast, d.W, d.H, d.views, 4, f->color, f->g_aa,
                        f->g_color, d.learn_pos ? f->g_clip : nullptr, s, aa_cand_list(f));
}

vcl_status stage_lobes(vcl_fit* f, const ShadeIn& a, const TexDesc& td, cudaStream_t s) {
    vcl_ctx* ctx = f->ctx;
    const vcl_fit_desc& d = f->d;
    const long long N = a.npix;
    const int groups = (d.K + 31) / 32;
    long long chunks = (N + 31) / 32;
    long long want = (chunks + 3) / 4;
    // three lobe blocks per SM (over all lobe groups) leave registers for
    // ten 64-thread blocks of the per-pixel backward that runs beside this
    // kernel (the two overlap on each SM)
    long long capg = ((long long)ctx->sm_count * 3 + groups - 1) / groups;
    const dim3 grid((unsigned)(want < capg ? (want < 1 ? 1 : want) : capg), (unsigned)groups);
    const float4* gc = (const float4*)f->g_color;
    const ShadeRec rec = shade_rec(f, true);
    if (ctx->mode == VCL_MODE_COMPAT) k_sg_lobes<false><<<grid, 128, 0, s>>>(a, rec, gc, f->g_axis, f->g_sharp, f->g_amp);
    else k_sg_lobes<true><<<grid, 128, 0, s>>>(a, rec, gc, f->g_axis, f->g_sharp, f->g_amp);
    return vcl_launch_check(ctx, "fused lobe gradients");
}

vcl_status stage_bwd_pix(vcl_fit* f, const ShadeIn& a, const TexDesc& td, cudaStream_t s) {
    const vcl_fit_desc& d = f->d;
    k_bwd_pix<<<vcl_blocks(a.npix, 64), 64, 0, s>>>(a, td, (const float4*)f->g_color, (const float4*)f->diffuse,
                                                      shade_rec(f, false).tsr, f->g_pyr, f->clip, f->g_clip,
                                                      d.learn_tex, d.learn_pos);
    return vcl_launch_check(f->ctx, "fused backward");
}

vcl_status enqueue(vcl_fit* f, cudaStream_t s) {
    vcl_ctx* ctx = f->ctx;
    Fused* F = (Fused*)f->fused;
    const vcl_fit_desc& d = f->d;
    const int W = d.W, H = d.H, V = d.views;
    const size_t npyr = vcl_tex_level_offset(d.tex_w, d.tex_h, 4, d.levels);
    const size_t n0 = (size_t)d.tex_w * d.tex_h * 4;
    const int compat = ctx->mode == VCL_MODE_COMPAT;
    k_begin<<<1, 1, 0, s>>>(F->d_step, F->d_corr, d.beta1, d.beta2, compat, f->loss);
    TRY(vcl_cuda_check(ctx, cudaMemsetAsync(f->g_clip, 0, sizeof(float) * V * d.nv * 4, s), "clear"));
    if (npyr > n0) TRY(vcl_cuda_check(ctx, cudaMemsetAsync(f->g_pyr + n0, 0, sizeof(float) * (npyr - n0), s), "clear"));
    TRY(vcl_project_fwd(ctx, f->mvp, V, f->pos, d.nv, 4, f->clip, s));
    launch_aa_screen(f->clip, (long long)V * d.nv, W, H, F->scr, s);
    TRY(raster_fwd_ws(ctx, F->raster_ws, F->sched, F->flags, f->clip, d.nv, f->tri, d.nt, W, H, V, f->rast, f->db, s));
    const ShadeIn a = shade_in(f);
    const TexDesc td = make_desc(d.tex_w, d.tex_h, 4, d.levels);
    TRY(stage_shade(f, a, td, s));
    TRY(stage_aa_mse(f, s));
    TRY(stage_aa_bwd(f, s));
    const bool lobes = d.learn_lobes && d.K;
    // the lobe gradients run beside the per-pixel backward on a forked stream
    if (lobes) {
        TRY(vcl_cuda_check(ctx, cudaEventRecord(F->fork, s), "fork"));
        TRY(vcl_cuda_check(ctx, cudaStreamWaitEvent(F->side, F->fork, 0), "fork"));
        TRY(stage_lobes(f, a, td, F->side));
        TRY(vcl_cuda_check(ctx, cudaEventRecord(F->join, F->side), "join"));
    }
    if (d.learn_tex || d.learn_pos) TRY(stage_bwd_pix(f, a, td, s));
    // the position gradient, the texture Adam and the mip rebuild do not
    // depend on the lobe gradients (which read the shading records, not the
    // texture): they run while the lobe branch finishes
    if (d.learn_pos) TRY(vcl_project_bwd(ctx, f->mvp, V, f->g_clip, d.nv, 4, f->g_pos, s));
    AdamArgs aa{d.beta1, d.beta2, d.lr_tex, d.eps, F->d_corr, 0.0};
    AdamArgs ap{d.beta1, d.beta2, d.lr_pos, d.eps, F->d_corr, d.lr_lobes};
    const float wpush = ctx->mode == VCL_MODE_EXACT ? 0.25f : 1.f;
    if (d.learn_tex) {
        const bool tile = d.tex_w % 32 == 0 && d.tex_h % 32 == 0 && d.levels >= 2;
        if (tile) {
            int top = d.levels - 1 < 5 ? d.levels - 1 : 5;
            dim3 g(d.tex_w / 32, d.tex_h / 32);
            k_adam_tex_tile<<<g, 256, 0, s>>>(td, f->pyr, f->g_pyr, f->mv_tex, f->mv_tex + n0, aa, wpush, top);
            TRY(vcl_launch_check(ctx, "fused adam texture"));
            for (int l = top + 1; l < d.levels; ++l)
                launch_mip_down(f->pyr + vcl_tex_level_offset(d.tex_w, d.tex_h, 4, l - 1),
                                f->pyr + vcl_tex_level_offset(d.tex_w, d.tex_h, 4, l), d.tex_w >> l, d.tex_h >> l, 4, s);
        } else {
            k_adam_tex_generic<<<vcl_blocks((long long)n0, 256), 256, 0, s>>>(td, f->pyr, f->g_pyr, f->mv_tex,
                                                                               f->mv_tex + n0, aa, wpush);
            for (int l = 1; l < d.levels; ++l)
                launch_mip_down(f->pyr + vcl_tex_level_offset(d.tex_w, d.tex_h, 4, l - 1),
                                f->pyr + vcl_tex_level_offset(d.tex_w, d.tex_h, 4, l), d.tex_w >> l, d.tex_h >> l, 4, s);
        }
        TRY(vcl_launch_check(ctx, "fused mips"));
    }
    if (lobes) TRY(vcl_cuda_check(ctx, cudaStreamWaitEvent(s, F->join, 0), "join"));
    long long np = d.learn_pos ? (long long)d.nv * 3 : 0;
    long long nl = lobes ? (long long)d.K * 8 : 0;
    if (np + nl > 0) {
        k_adam_small<<<vcl_blocks(np + nl, 256), 256, 0, s>>>(f->pos, f->g_pos, f->mv_pos, np, f->lobe, f->g_lobe,
                                                              f->mv_lobe, nl, ap);
        TRY(vcl_launch_check(ctx, "fused adam"));
    }
    return VCL_OK;
}

}  // namespace

// Captures the job's step into F->graph_def (once per mode) on `s`, which
// must be a stream that can be captured (not the legacy default stream).
vcl_status fit_fused_graph(vcl_fit* f, cudaStream_t s, cudaGraph_t* out) {
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(f->d.C == 4, "the fused strategy needs C = 4 channels (got %d)", f->d.C);
    VCL_REQUIRE(s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread,
                "graph capture needs a created stream");
    vcl_status st = fused_init(f);
    if (st) return st;
    Fused* F = (Fused*)f->fused;
    if (!F->graph_def || F->graph_mode != ctx->mode) {
        if (F->graph) { cudaGraphExecDestroy(F->graph); F->graph = nullptr; }
        if (F->graph_def) { cudaGraphDestroy(F->graph_def); F->graph_def = nullptr; }
        st = vcl_cuda_check(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "graph capture");
        if (st) return st;
        vcl_status est = enqueue(f, s);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (est) { if (g) cudaGraphDestroy(g); return est; }
        st = vcl_cuda_check(ctx, e, "graph capture end");
        if (st) { if (g) cudaGraphDestroy(g); return st; }
        F->graph_def = g;
        F->graph_mode = ctx->mode;
    }
    *out = F->graph_def;
    return VCL_OK;
}

vcl_status fit_step_fused(vcl_fit* f, cudaStream_t s) {
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(f->d.C == 4, "the fused strategy needs C = 4 channels (got %d)", f->d.C);
    vcl_status st = fused_init(f);
    if (st) return st;
    Fused* F = (Fused*)f->fused;
    if (s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) {
        st = enqueue(f, s);
        if (!st) ++f->step_count;
        return st;
    }
    if (!F->graph || F->graph_mode != ctx->mode) {
        cudaGraph_t g = nullptr;
        st = fit_fused_graph(f, s, &g);
        if (st) return st;
        if (F->graph) { cudaGraphExecDestroy(F->graph); F->graph = nullptr; }
        st = vcl_cuda_check(ctx, cudaGraphInstantiate(&F->graph, g, 0), "graph instantiate");
        if (st) { F->graph = nullptr; return st; }
    }
    st = vcl_cuda_check(ctx, cudaGraphLaunch(F->graph, s), "graph launch");
    if (!st) ++f->step_count;
    return st;
}

int fit_fused_launches(const vcl_fit* f) {
    const vcl_fit_desc& d = f->d;
    int n = 1 /* begin */ + 1 /* project */ + 1 /* aa screen terms */ + raster_fwd_launches() + 1 /* shade */ +
            1 /* aa + mse */ + 1 /* aa bwd */;
    if (d.learn_tex || d.learn_pos) n += 1; /* per-pixel backward */
    if (d.learn_lobes && d.K) n += 1;       /* lobe gradients */
    if (d.learn_pos) n += 1;
    if (d.learn_tex) {
        const bool tile = d.tex_w % 32 == 0 && d.tex_h % 32 == 0 && d.levels >= 2;
        int top = d.levels - 1 < 5 ? d.levels - 1 : 5;
        n += 1 + (tile ? d.levels - 1 - top : d.levels - 1);
    }
    if (d.learn_pos || (d.learn_lobes && d.K)) n += 1;
    return n;
}

void fit_fused_release(vcl_fit* f, cudaStream_t s, bool async) {
    Fused* F = (Fused*)f->fused;
    if (!F) return;
    if (F->graph) cudaGraphExecDestroy(F->graph);
    if (F->graph_def) cudaGraphDestroy(F->graph_def);
    auto release = [&](void* p) {
        if (!p) return;
        if (async) cudaFreeAsync(p, s);
        else cudaFree(p);
    };
    release(F->raster_ws);
    release(F->flags);
    release(F->scr);
    release(F->d_step);
    release(F->d_corr);
    if (F->side) cudaStreamDestroy(F->side);
    if (F->fork) cudaEventDestroy(F->fork);
    if (F->join) cudaEventDestroy(F->join);
    delete F;
    f->fused = nullptr;
}

// Keeps the device step counter of the fused path and the host counter of
// the plain path in agreement when the strategy changes.
vcl_status fit_fused_sync_counter(vcl_fit* f, bool to_device) {
    Fused* F = (Fused*)f->fused;
    if (!F) return VCL_OK;
    if (to_device)
        return vcl_cuda_check(f->ctx, cudaMemcpy(F->d_step, &f->step_count, sizeof(int), cudaMemcpyHostToDevice),
                              "step counter");
    return VCL_OK;
}

vcl_status fit_fused_raster_tuning(vcl_fit* f, int* tile, float* ms3) {
    vcl_status st = fused_init(f);
    if (st) return st;
    Fused* F = (Fused*)f->fused;
    if (tile) *tile = F->sched.tile;
    if (ms3) for (int i = 0; i < 3; ++i) ms3[i] = F->tune_ms[i];
    return VCL_OK;
}

vcl_status fit_fused_raster_schedule(vcl_fit* f, int* tile, int* small_area, long long* cap, int* cached,
                                     long long* overflow) {
    vcl_status st = fused_init(f);
    if (st) return st;
    Fused* F = (Fused*)f->fused;
    if (tile) *tile = F->sched.tile;
    if (small_area) *small_area = F->sched.small_area;
    if (cap) *cap = F->sched.cap;
    if (cached) *cached = F->sched_cached ? 1 : 0;
    if (overflow) {
        int h = 0;
        st = vcl_cuda_check(f->ctx, cudaMemcpy(&h, F->flags, sizeof(int), cudaMemcpyDeviceToHost), "overflow read");
        if (st) return st;
        *overflow = h;
    }
    return VCL_OK;
}

// The six stages alone, then the per-pixel backward and the lobe gradients
// together as the step runs them (forked stream, joined).
const char* const kFusedKernelNames[] = {"raster", "shade_fwd", "aa_fwd_mse", "aa_bwd", "bwd_pix", "sg_lobes",
                                         "bwd_pix+sg_lobes"};
constexpr int kFusedKernels = 7;

int fit_fused_kernel_count() { return kFusedKernels; }
const char* fit_fused_kernel_name(int i) { return i >= 0 && i < kFusedKernels ? kFusedKernelNames[i] : nullptr; }

// Average device time of each fused stage: one untimed launch, then `reps`
// launches between two events on `s`.  Runs on the job's current state (its
// last step's raster and gradients); the stages that accumulate gradients
// leave them undefined, so all gradient buffers are cleared at the end and
// the parameters and Adam moments are untouched.
vcl_status fit_fused_time_kernels(vcl_fit* f, cudaStream_t s, int reps, float* ms, int n) {
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(f->fused && f->step_count > 0, "time the kernels after at least one fused step");
    VCL_REQUIRE(reps > 0 && ms, "bad arguments");
    Fused* F = (Fused*)f->fused;
    const vcl_fit_desc& d = f->d;
    const int W = d.W, H = d.H, V = d.views;
    const ShadeIn a = shade_in(f);
    const TexDesc td = make_desc(d.tex_w, d.tex_h, 4, d.levels);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return vcl_fail(ctx, VCL_ERR_CUDA, "timing events");
    vcl_status st = VCL_OK;
    for (int k = 0; k < kFusedKernels && k < n && st == VCL_OK; ++k) {
        auto run = [&]() -> vcl_status {
            switch (k) {
                case 0: return raster_fwd_ws(ctx, F->raster_ws, F->sched, F->flags, f->clip, d.nv, f->tri, d.nt, W, H,
                                             V, f->rast, f->db, s);
                case 1: return stage_shade(f, a, td, s);
                case 2: return stage_aa_mse(f, s);
                case 3: return stage_aa_bwd(f, s);
                case 4: return stage_bwd_pix(f, a, td, s);
                case 5: return (d.learn_lobes && d.K) ? stage_lobes(f, a, td, s) : VCL_OK;
                default: {
                    if (!(d.learn_lobes && d.K)) return stage_bwd_pix(f, a, td, s);
                    vcl_status r = vcl_cuda_check(ctx, cudaEventRecord(F->fork, s), "fork");
                    if (r == VCL_OK) r = vcl_cuda_check(ctx, cudaStreamWaitEvent(F->side, F->fork, 0), "fork");
                    if (r == VCL_OK) r = stage_lobes(f, a, td, F->side);
                    if (r == VCL_OK) r = vcl_cuda_check(ctx, cudaEventRecord(F->join, F->side), "join");
                    if (r == VCL_OK) r = stage_bwd_pix(f, a, td, s);
                    if (r == VCL_OK) r = vcl_cuda_check(ctx, cudaStreamWaitEvent(s, F->join, 0), "join");
                    return r;
                }
            }
        };
        st = run();
        if (st) break;
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps && st == VCL_OK; ++r) st = run();
        cudaEventRecord(e1, s);
        if (st) break;
        cudaEventSynchronize(e1);
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms[k] = t / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    const size_t npyr = vcl_tex_level_offset(d.tex_w, d.tex_h, 4, d.levels);
    auto z = [&](void* p, size_t b) {
        if (st == VCL_OK) st = vcl_cuda_check(ctx, cudaMemsetAsync(p, 0, b, s), "gradient clear");
    };
    z(f->g_pyr, sizeof(float) * npyr);
    z(f->g_clip, sizeof(float) * (size_t)V * d.nv * 4);
    z(f->g_pos, sizeof(float) * (size_t)d.nv * 3);
    z(f->g_lobe, sizeof(float) * (size_t)d.K * 8);
    if (st == VCL_OK) st = vcl_cuda_check(ctx, cudaStreamSynchronize(s), "kernel timing");
    return st;
}

size_t fit_fused_footprint(const vcl_fit_desc& d) {
    size_t ws = sizeof(float) * 8 * (size_t)d.views * d.nv;   // antialias screen terms
    for (int t : {8, 16, 32}) {
        long long cap = raster_auto_capacity(d.views, d.nt, d.W, d.H, t);
        size_t b = raster_ws_size(d.W, d.H, d.views, d.nt, t, cap);
        if (b > ws) ws = b;
    }
    return ws + 3 * 256;
}

void fit_fused_tuning_cache_clear() {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune.clear();
}

// Per-pixel / per-element operators of the vcl C ABI: project, interpolate,
// texture (+ mip chain), antialias, loss and Adam.  One thread per pixel
// (or vertex / texel / parameter) over a flat 1-D grid, reading and writing
// the reference's interleaved layouts with vector loads where the channel
// count allows.  Gradient scatters use FP32 vector reductions
// (red.global.add.v4.f32 / .v2.f32, sm_90+).
#include "common.cuh"
#include "tex_math.cuh"
#include "adam_math.cuh"
#include "ops_internal.cuh"

namespace {

DEV float mul(float a, float b) { return __fmul_rn(a, b); }
DEV float add(float a, float b) { return __fadd_rn(a, b); }
DEV float sub(float a, float b) { return __fsub_rn(a, b); }

// ------------------------------------------------------------- project
// project.cu:26-34
__global__ void k_project_fwd(const float* __restrict__ mats, int views, const float* __restrict__ pos, int nv, int dim,
                              float* __restrict__ out) {
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)views * nv) return;
    int view = (int)(gid / nv), p = (int)(gid % nv);
    const float* m = mats + (size_t)view * 16;
    float x = pos[3 * (size_t)p], y = pos[3 * (size_t)p + 1], z = pos[3 * (size_t)p + 2];
    float* o = out + (size_t)gid * dim;
    // exactly rounded, as the CPU restatement: triangle ids downstream are
    // sensitive to the last bit of clip-space positions
    for (int i = 0; i < dim; ++i) o[i] = add(add(add(mul(m[i], x), mul(m[4 + i], y)), mul(m[8 + i], z)), m[12 + i]);
}

// project.cu:71-88; one thread per vertex sums its views (no atomics)
__global__ void k_project_bwd(const float* __restrict__ mats, int views, const float* __restrict__ gout, int nv, int dim,
                              float* __restrict__ gpos) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nv) return;
    float gx = gpos[3 * (size_t)p], gy = gpos[3 * (size_t)p + 1], gz = gpos[3 * (size_t)p + 2];
    for (int v = 0; v < views; ++v) {
        const float* m = mats + (size_t)v * 16;
        const float* g = gout + ((size_t)v * nv + p) * dim;
        for (int i = 0; i < dim; ++i) {
            float gi = g[i];
            gx += m[i] * gi;
            gy += m[4 + i] * gi;
            gz += m[8 + i] * gi;
        }
    }
    gpos[3 * (size_t)p] = gx; gpos[3 * (size_t)p + 1] = gy; gpos[3 * (size_t)p + 2] = gz;
}

// --------------------------------------------------------- interpolate
DEV bool tri_ok(int idx, int nt, const uint32_t* tri, int nv, uint32_t& i0, uint32_t& i1, uint32_t& i2, int* flags) {
    if (idx < 0) return false;
    if (idx >= nt) { atomicOr(&flags[1], 1); return false; }
    i0 = tri[3 * (size_t)idx]; i1 = tri[3 * (size_t)idx + 1]; i2 = tri[3 * (size_t)idx + 2];
    if (i0 >= (uint32_t)nv || i1 >= (uint32_t)nv || i2 >= (uint32_t)nv) { atomicOr(&flags[1], 1); return false; }
    return true;
}

// interpolate.cu:20-49 (+ the output clears of :51-60)
__global__ void k_interp_fwd(const float4* __restrict__ rast, const float4* __restrict__ db, const float* __restrict__ attr,
                             int nv, int dim, const uint32_t* __restrict__ tri, int nt, long long npix,
                             float* __restrict__ out, float2* __restrict__ out_da, int* flags) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float4 r = rast[p];
    uint32_t i0, i1, i2;
    if (!tri_ok(rast_id(r.w), nt, tri, nv, i0, i1, i2, flags)) {
        for (int i = 0; i < dim; ++i) out[p * dim + i] = 0.f;
        if (out_da) for (int i = 0; i < dim; ++i) out_da[p * dim + i] = make_float2(0.f, 0.f);
        return;
    }
    float4 d = out_da ? db[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    double l2 = __dsub_rn(__dsub_rn(1.0, (double)r.x), (double)r.y);
    for (int i = 0; i < dim; ++i) {
        float a0 = attr[(size_t)i0 * dim + i], a1 = attr[(size_t)i1 * dim + i], a2 = attr[(size_t)i2 * dim + i];
        out[p * dim + i] = (float)__dadd_rn((double)add(mul(a0, r.x), mul(a1, r.y)), __dmul_rn((double)a2, l2));
        if (out_da) {
            float dadu = a0 - a2, dadv = a1 - a2;
            out_da[p * dim + i] = make_float2(add(mul(dadu, d.x), mul(dadv, d.z)), add(mul(dadu, d.y), mul(dadv, d.w)));
        }
    }
}

// interpolate.cu:114-143
__global__ void k_interp_bwd(const float4* __restrict__ rast, const float* __restrict__ attr, int nv, int dim,
                             const uint32_t* __restrict__ tri, int nt, long long npix, const float* __restrict__ gout,
                             float* __restrict__ gattr, float2* __restrict__ gbary, int accumulate, int* flags) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float4 r = rast[p];
    uint32_t i0, i1, i2;
    if (!tri_ok(rast_id(r.w), nt, tri, nv, i0, i1, i2, flags)) return;
    float gu = 0.f, gv = 0.f;
    double l2 = (1.0 - (double)r.x) - (double)r.y;
    const float* g = gout + p * dim;
    if (gattr && dim == 2) {
        float g0 = g[0], g1 = g[1];
        red_add2(gattr + (size_t)i0 * 2, g0 * r.x, g1 * r.x);
        red_add2(gattr + (size_t)i1 * 2, g0 * r.y, g1 * r.y);
        red_add2(gattr + (size_t)i2 * 2, (float)((double)g0 * l2), (float)((double)g1 * l2));
    } else if (gattr && dim == 4) {
        float4 gg = make_float4(g[0], g[1], g[2], g[3]);
        red_add4(gattr + (size_t)i0 * 4, gg.x * r.x, gg.y * r.x, gg.z * r.x, gg.w * r.x);
        red_add4(gattr + (size_t)i1 * 4, gg.x * r.y, gg.y * r.y, gg.z * r.y, gg.w * r.y);
        red_add4(gattr + (size_t)i2 * 4, (float)((double)gg.x * l2), (float)((double)gg.y * l2),
                 (float)((double)gg.z * l2), (float)((double)gg.w * l2));
    } else if (gattr) {
        for (int i = 0; i < dim; ++i) {
            float gi = g[i];
            atomicAdd(&gattr[(size_t)i0 * dim + i], gi * r.x);
            atomicAdd(&gattr[(size_t)i1 * dim + i], gi * r.y);
            atomicAdd(&gattr[(size_t)i2 * dim + i], (float)((double)gi * l2));
        }
    }
    for (int i = 0; i < dim; ++i) {
        float gi = g[i];
        float a2 = attr[(size_t)i2 * dim + i];
        gu += gi * (attr[(size_t)i0 * dim + i] - a2);
        gv += gi * (attr[(size_t)i1 * dim + i] - a2);
    }
    if (gbary) {
        if (accumulate) { float2 o = gbary[p]; gbary[p] = make_float2(o.x + gu, o.y + gv); }
        else gbary[p] = make_float2(gu, gv);
    }
}

// texturemap.cu:67-114
template <int C4>
__global__ void k_tex_fwd(TexDesc t, const float* __restrict__ pyr, const float4* __restrict__ rast,
                          const float2* __restrict__ uv, const float4* __restrict__ uv_da, long long npix,
                          float* __restrict__ out) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    const int C = C4 ? 4 : t.C;
    if (rast[p].w < 1.f) {
        if (C4) reinterpret_cast<float4*>(out)[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        else for (int i = 0; i < C; ++i) out[p * C + i] = 0.f;
        return;
    }
    float2 u = uv[p];
    int l0 = 0, l1 = 0;
    float fl = 0.f;
    if (t.L > 1) calc_level(t, uv_da[p], l0, l1, fl, nullptr, 0);
    int i0[4];
    float2 f0;
    index_fetch(t, l0, u, i0, f0);
    const float* T0 = pyr + t.off[l0];
    if (C4) {
        float4 o = bilerp4(ld4(T0, i0[0]), ld4(T0, i0[1]), ld4(T0, i0[2]), ld4(T0, i0[3]), f0);
        if (t.L > 1 && fl > 0) {
            int i1[4];
            float2 f1;
            index_fetch(t, l1, u, i1, f1);
            const float* T1 = pyr + t.off[l1];
            float4 o1 = bilerp4(ld4(T1, i1[0]), ld4(T1, i1[1]), ld4(T1, i1[2]), ld4(T1, i1[3]), f1);
            o = make_float4(lerpf_(o.x, o1.x, fl), lerpf_(o.y, o1.y, fl), lerpf_(o.z, o1.z, fl), lerpf_(o.w, o1.w, fl));
        }
        reinterpret_cast<float4*>(out)[p] = o;
    } else {
        int i1[4];
        float2 f1;
        bool tri = t.L > 1 && fl > 0;
        if (tri) index_fetch(t, l1, u, i1, f1);
        const float* T1 = pyr + t.off[l1];
        for (int i = 0; i < C; ++i) {
            float o = bilerp1(T0[i0[0] * C + i], T0[i0[1] * C + i], T0[i0[2] * C + i], T0[i0[3] * C + i], f0);
            if (tri) o = lerpf_(o, bilerp1(T1[i1[0] * C + i], T1[i1[1] * C + i], T1[i1[2] * C + i], T1[i1[3] * C + i], f1), fl);
            out[p * C + i] = o;
        }
    }
}

// texturemap.cu:229-319
template <int C4>
__global__ void k_tex_bwd(TexDesc t, const float* __restrict__ pyr, const float4* __restrict__ rast,
                          const float2* __restrict__ uv, const float4* __restrict__ uv_da, long long npix,
                          const float* __restrict__ gout, float* __restrict__ gpyr, float2* __restrict__ guv,
                          float4* __restrict__ guv_da, int exact) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    if (rast[p].w < 1.f) return;
    const int C = C4 ? 4 : t.C;
    const bool mip = t.L > 1;
    float2 u = uv[p];
    int l0 = 0, l1 = 0;
    float fl = 0.f;
    float4 dl = make_float4(0.f, 0.f, 0.f, 0.f);
    if (mip) calc_level(t, uv_da[p], l0, l1, fl, &dl, exact);
    int i0[4], i1[4];
    float2 f0, f1 = make_float2(0.f, 0.f);
    index_fetch(t, l0, u, i0, f0);
    if (mip) index_fetch(t, l1, u, i1, f1);
    const float* T0 = pyr + t.off[l0];
    const float* T1 = pyr + t.off[l1];
    float* G0 = gpyr ? gpyr + t.off[l0] : nullptr;
    float* G1 = gpyr ? gpyr + t.off[l1] : nullptr;
    const float s0x = (float)(t.tw >> l0), s0y = (float)(t.th >> l0);
    const float s1x = (float)(t.tw >> l1), s1y = (float)(t.th >> l1);
    const float wl0 = mip ? 1.f - fl : 1.f;
    const bool tri = mip && fl > 0;
    float w00 = wl0 * (1.f - f0.x) * (1.f - f0.y), w01 = wl0 * f0.x * (1.f - f0.y);
    float w10 = wl0 * (1.f - f0.x) * f0.y, w11 = wl0 * f0.x * f0.y;
    float v00 = fl * (1.f - f1.x) * (1.f - f1.y), v01 = fl * f1.x * (1.f - f1.y);
    float v10 = fl * (1.f - f1.x) * f1.y, v11 = fl * f1.x * f1.y;
    float gu = 0.f, gv = 0.f, gl = 0.f;
    if (C4) {
        float4 g = reinterpret_cast<const float4*>(gout)[p];
        if (G0) {
            red_add4(G0 + 4 * i0[0], w00 * g.x, w00 * g.y, w00 * g.z, w00 * g.w);
            red_add4(G0 + 4 * i0[1], w01 * g.x, w01 * g.y, w01 * g.z, w01 * g.w);
            red_add4(G0 + 4 * i0[2], w10 * g.x, w10 * g.y, w10 * g.z, w10 * g.w);
            red_add4(G0 + 4 * i0[3], w11 * g.x, w11 * g.y, w11 * g.z, w11 * g.w);
            if (tri) {
                red_add4(G1 + 4 * i1[0], v00 * g.x, v00 * g.y, v00 * g.z, v00 * g.w);
                red_add4(G1 + 4 * i1[1], v01 * g.x, v01 * g.y, v01 * g.z, v01 * g.w);
                red_add4(G1 + 4 * i1[2], v10 * g.x, v10 * g.y, v10 * g.z, v10 * g.w);
                red_add4(G1 + 4 * i1[3], v11 * g.x, v11 * g.y, v11 * g.z, v11 * g.w);
            }
        }
        float4 a00 = ld4(T0, i0[0]), a01 = ld4(T0, i0[1]), a10 = ld4(T0, i0[2]), a11 = ld4(T0, i0[3]);
        float ga[4] = {g.x, g.y, g.z, g.w};
        float A00[4] = {a00.x, a00.y, a00.z, a00.w}, A01[4] = {a01.x, a01.y, a01.z, a01.w};
        float A10[4] = {a10.x, a10.y, a10.z, a10.w}, A11[4] = {a11.x, a11.y, a11.z, a11.w};
        float B00[4], B01[4], B10[4], B11[4];
        if (tri) {
            float4 b00 = ld4(T1, i1[0]), b01 = ld4(T1, i1[1]), b10 = ld4(T1, i1[2]), b11 = ld4(T1, i1[3]);
            B00[0] = b00.x; B00[1] = b00.y; B00[2] = b00.z; B00[3] = b00.w;
            B01[0] = b01.x; B01[1] = b01.y; B01[2] = b01.z; B01[3] = b01.w;
            B10[0] = b10.x; B10[1] = b10.y; B10[2] = b10.z; B10[3] = b10.w;
            B11[0] = b11.x; B11[1] = b11.y; B11[2] = b11.z; B11[3] = b11.w;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float du = lerpf_(A01[i] - A00[i], A11[i] - A10[i], f0.y) * s0x;
            float dv = lerpf_(A10[i] - A00[i], A11[i] - A01[i], f0.x) * s0y;
            if (tri) {
                float l = bilerp1(A00[i], A01[i], A10[i], A11[i], f0);
                du = lerpf_(du, lerpf_(B01[i] - B00[i], B11[i] - B10[i], f1.y) * s1x, fl);
                dv = lerpf_(dv, lerpf_(B10[i] - B00[i], B11[i] - B01[i], f1.x) * s1y, fl);
                gl += (bilerp1(B00[i], B01[i], B10[i], B11[i], f1) - l) * ga[i];
            }
            gu += du * ga[i];
            gv += dv * ga[i];
        }
    } else {
        for (int i = 0; i < C; ++i) {
            float g = gout[p * C + i];
            if (G0) {
                atomicAdd(&G0[i0[0] * C + i], w00 * g); atomicAdd(&G0[i0[1] * C + i], w01 * g);
                atomicAdd(&G0[i0[2] * C + i], w10 * g); atomicAdd(&G0[i0[3] * C + i], w11 * g);
                if (tri) {
                    atomicAdd(&G1[i1[0] * C + i], v00 * g); atomicAdd(&G1[i1[1] * C + i], v01 * g);
                    atomicAdd(&G1[i1[2] * C + i], v10 * g); atomicAdd(&G1[i1[3] * C + i], v11 * g);
                }
            }
            float a00 = T0[i0[0] * C + i], a01 = T0[i0[1] * C + i], a10 = T0[i0[2] * C + i], a11 = T0[i0[3] * C + i];
            float du = lerpf_(a01 - a00, a11 - a10, f0.y) * s0x;
            float dv = lerpf_(a10 - a00, a11 - a01, f0.x) * s0y;
            if (tri) {
                float l = bilerp1(a00, a01, a10, a11, f0);
                float b00 = T1[i1[0] * C + i], b01 = T1[i1[1] * C + i], b10 = T1[i1[2] * C + i], b11 = T1[i1[3] * C + i];
                du = lerpf_(du, lerpf_(b01 - b00, b11 - b10, f1.y) * s1x, fl);
                dv = lerpf_(dv, lerpf_(b10 - b00, b11 - b01, f1.x) * s1y, fl);
                gl += (bilerp1(b00, b01, b10, b11, f1) - l) * g;
            }
            gu += du * g;
            gv += dv * g;
        }
    }
    if (guv) guv[p] = make_float2(gu, gv);
    if (guv_da && mip) guv_da[p] = make_float4(gl * dl.x, gl * dl.y, gl * dl.z, gl * dl.w);
}

// buffer.cu:449-472
__global__ void k_mip_down(const float* __restrict__ src, float* __restrict__ dst, int w, int h, int C) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)w * h) return;
    int px = (int)(i % w), py = (int)(i / w);
    int pw = w * 2;
    size_t p00 = (size_t)(2 * px) + (size_t)pw * (2 * py), p01 = p00 + 1, p10 = p00 + pw, p11 = p10 + 1;
    if (C == 4) {
        float4 a = ld4(src, (int)p00), b = ld4(src, (int)p01), c = ld4(src, (int)p10), d = ld4(src, (int)p11);
        reinterpret_cast<float4*>(dst)[i] = make_float4(add(add(add(a.x, b.x), c.x), d.x) * 0.25f,
                                                        add(add(add(a.y, b.y), c.y), d.y) * 0.25f,
                                                        add(add(add(a.z, b.z), c.z), d.z) * 0.25f,
                                                        add(add(add(a.w, b.w), c.w), d.w) * 0.25f);
    } else {
        for (int k = 0; k < C; ++k)
            dst[i * C + k] = add(add(add(src[p00 * C + k], src[p01 * C + k]), src[p10 * C + k]), src[p11 * C + k]) * 0.25f;
    }
}

// buffer.cu:615-636
__global__ void k_mip_push(const float* __restrict__ src, float* __restrict__ dst, int w, int h, int C, float weight) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)w * h * C) return;
    int k = (int)(i % C);
    long long t = i / C;
    int px = (int)(t % w), py = (int)(t / w);
    int pw = w * 2;
    size_t p00 = (size_t)(2 * px) + (size_t)pw * (2 * py), p01 = p00 + 1, p10 = p00 + pw, p11 = p10 + 1;
    float v = src[i] * weight;
    add_nan_check(dst[p00 * C + k], v);
    add_nan_check(dst[p01 * C + k], v);
    add_nan_check(dst[p10 * C + k], v);
    add_nan_check(dst[p11 * C + k], v);
}

__global__ void k_clamp(float* __restrict__ p, long long n, float lo, float hi) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a = p[i];
    p[i] = a < lo ? lo : a > hi ? hi : a;
}

// ------------------------------------------------------------ antialias
struct AATri { float2 v[3]; float2 ndc[3]; float iw[3]; uint32_t id[3]; };

// antialias.cu:37-55 / :240-257.  Screen positions use exactly rounded
// arithmetic so that the edge decisions match the CPU restatement.
// `scr` (optional): the per-vertex screen terms of this view precomputed by
// k_aa_screen -- [2v] = ((x/w + 1) s.x, (y/w + 1) s.y, 1/w, -), [2v+1] =
// (x/w, y/w, -, -) -- with the same rounded operations as computed here.
DEV bool aa_fetch(const float4* __restrict__ proj, const float4* __restrict__ scr, int nv,
                  const uint32_t* __restrict__ tri, int nt, float id_w, float2 s,
                  float2 f, AATri& t, int* flags, bool need_ndc) {
    uint32_t i[3];
    if (!tri_ok(rast_id(id_w), nt, tri, nv, i[0], i[1], i[2], flags)) return false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        t.id[k] = i[k];
        if (scr) {
            const float4 S = scr[2 * (size_t)i[k]];
            t.iw[k] = S.z;
            if (need_ndc) {
                const float4 Q = scr[2 * (size_t)i[k] + 1];
                t.ndc[k] = make_float2(Q.x, Q.y);
            }
            t.v[k] = make_float2(sub(S.x, f.x), sub(S.y, f.y));
        } else {
            float4 c = proj[i[k]];
            t.iw[k] = __fdiv_rn(1.f, c.w);
            t.ndc[k] = make_float2(mul(c.x, t.iw[k]), mul(c.y, t.iw[k]));
            t.v[k] = make_float2(sub(mul(add(t.ndc[k].x, 1.f), s.x), f.x), sub(mul(add(t.ndc[k].y, 1.f), s.y), f.y));
        }
    }
    return true;
}

__global__ void k_aa_screen(const float4* __restrict__ clip, long long n, float sx, float sy, float4* __restrict__ scr) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 c = clip[i];
    const float iw = __fdiv_rn(1.f, c.w);
    const float nx = mul(c.x, iw), ny = mul(c.y, iw);
    scr[2 * i] = make_float4(mul(add(nx, 1.f), sx), mul(add(ny, 1.f), sy), iw, 0.f);
    scr[2 * i + 1] = make_float4(nx, ny, 0.f, 0.f);
}

DEV float cross_rn(float ax, float ay, float bx, float by) { return sub(mul(ax, by), mul(ay, bx)); }

// Shared edge geometry of antialias.cu:17-27 / :196-206; false when the
// pixel pair does not straddle this edge.
DEV bool aa_edge(float2 pa, float2 pb, float2 o, float& a, float& alpha, float& ia, float2& e, float& n) {
    a = cross_rn(pa.x, pa.y, pb.x, pb.y);
    float oa = cross_rn(sub(pa.x, o.x), sub(pa.y, o.y), sub(pb.x, o.x), sub(pb.y, o.y));
    if (mul(a, oa) > 0.f) return false;
    e = make_float2(sub(pa.x, pb.x), sub(pa.y, pb.y));
    n = mul(add(o.x, o.y), sub(o.x, o.y));
    if (mul(mul(add(e.x, e.y), sub(e.x, e.y)), n) > 0.f) return false;
    float so = add(o.x, o.y);
    e.x = mul(e.x, so); e.y = mul(e.y, so);
    float D = n > 0.f ? -e.y : e.x;
    ia = (float)(1.0 / ((double)D + (D > 0 ? 1e-3 : -1e-3)));
    alpha = sub(mul(a, ia), .5f);
    return true;
}

// One horizontal (dir 0: o = q-1) or vertical (dir 1: o = q-W) pixel pair
// as antialias.cu:66-92 / :273-296 evaluate it at pixel q: which side is
// drawn in front (pp), the other side (op), and pp's triangle in pixel
// units around the shared pixel edge.  `typo` reproduces :279 (the current
// pixel's id used for both sides of a horizontal pair).
struct AAPair {
    long long pp, op;
    float2 o;
    AATri t;
};

DEV bool aa_pair(const float4* __restrict__ proj, const float4* __restrict__ scr, int nv, const uint32_t* __restrict__ tri, int nt,
                 const float4* __restrict__ rast, long long q, int qx, int qy, int W, int dir, bool typo, float2 s,
                 AAPair& P, int* flags, bool need_ndc) {
    const long long oidx = dir == 0 ? q - 1 : q - W;
    const float4 tr = rast[q], to = rast[oidx];
    if (to.w == tr.w) return false;
    long long pp = (int)tr.w ? q : oidx;
    long long op = (int)((dir == 0 && typo) ? tr.w : to.w) ? q : oidx;
    if (pp == op) { if (tr.z > to.z) op = oidx; else pp = oidx; }
    float2 f;
    if (dir == 0) { f = make_float2((float)qx + (pp > op ? .5f : -.5f), (float)qy + .5f); P.o = make_float2(pp > op ? -1.f : 1.f, 0.f); }
    else { f = make_float2((float)qx + .5f, (float)qy + (pp > op ? .5f : -.5f)); P.o = make_float2(0.f, pp > op ? -1.f : 1.f); }
    P.pp = pp;
    P.op = op;
    return aa_fetch(proj, scr, nv, tri, nt, pp == q ? tr.w : to.w, s, f, P.t, flags, need_ndc);
}

// Forward antialias as a gather: each pixel evaluates the (up to four)
// pairs it belongs to and adds the edge terms the reference sends to it
// (antialias.cu:28-34), in a fixed order -- deterministic, no atomics, and
// out = in + terms in one pass (the reference's init store, :62-65).
template <int C4>
__global__ void k_aa_fwd(const float4* __restrict__ clip, const float4* __restrict__ scr_all, int nv,
                         const uint32_t* __restrict__ tri, int nt,
                         const float4* __restrict__ rast, int W, int H, long long npix, int Cr, const float* __restrict__ in,
                         float* __restrict__ out, int* flags) {
    long long pidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pidx >= npix) return;
    const int C = C4 ? 4 : Cr;
    long long hw = (long long)W * H;
    int view = (int)(pidx / hw);
    int rem = (int)(pidx - view * hw);
    int py = rem / W, px = rem - py * W;
    const float4* proj = clip + (size_t)view * nv;
    const float4* scr = scr_all ? scr_all + 2 * (size_t)view * nv : nullptr;
    const float2 s = make_float2(W / 2.f, H / 2.f);
    float acc[8];
    for (int i = 0; i < C && i < 8; ++i) acc[i] = in[pidx * C + i];
    // pairs: (p-1,p) at p, (p,p+1) at p+1, (p-W,p) at p, (p,p+W) at p+W
    for (int k = 0; k < 4; ++k) {
        const int dir = k >> 1;
        const bool self = (k & 1) == 0;
        int qx = px, qy = py;
        if (!self) { if (dir == 0) ++qx; else ++qy; }
        if (dir == 0 ? (qx == 0 || qx >= W) : (qy == 0 || qy >= H)) continue;
        const long long q = self ? pidx : (dir == 0 ? pidx + 1 : pidx + W);
        AAPair P;
        if (!aa_pair(proj, scr, nv, tri, nt, rast, q, qx, qy, W, dir, false, s, P, flags, false)) continue;
        if (P.pp != pidx && P.op != pidx) continue;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            float a, alpha, ia, n;
            float2 ev;
            if (!aa_edge(P.t.v[e], P.t.v[(e + 1) % 3], P.o, a, alpha, ia, ev, n)) continue;
            if ((alpha > 0 ? P.op : P.pp) != pidx) continue;
            if (C4) {
                float4 ip = reinterpret_cast<const float4*>(in)[P.pp], io = reinterpret_cast<const float4*>(in)[P.op];
                acc[0] += alpha * (ip.x - io.x); acc[1] += alpha * (ip.y - io.y);
                acc[2] += alpha * (ip.z - io.z); acc[3] += alpha * (ip.w - io.w);
            } else {
                for (int i = 0; i < C && i < 8; ++i) acc[i] += alpha * (in[P.pp * C + i] - in[P.op * C + i]);
            }
        }
    }
    if (C4) reinterpret_cast<float4*>(out)[pidx] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    else for (int i = 0; i < C && i < 8; ++i) out[pidx * C + i] = acc[i];
}

// Backward antialias: colour gradients gathered per pixel like the forward
// (antialias.cu:216-220, deterministic); clip-position gradients scattered
// once per pair, by the pair's own pixel q (antialias.cu:222-245).
template <int C4>
__global__ void k_aa_bwd(const float4* __restrict__ clip, const float4* __restrict__ scr_all, int nv,
                         const uint32_t* __restrict__ tri, int nt,
                         const float4* __restrict__ rast, int W, int H, long long npix, int Cr, const float* __restrict__ in,
                         const float* __restrict__ gout, float* __restrict__ gin, float* __restrict__ gclip, int exact,
                         int* flags) {
    long long pidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pidx >= npix) return;
    const int C = C4 ? 4 : Cr;
    long long hw = (long long)W * H;
    int view = (int)(pidx / hw);
    int rem = (int)(pidx - view * hw);
    int py = rem / W, px = rem - py * W;
    const float4* proj = clip + (size_t)view * nv;
    const float4* scr = scr_all ? scr_all + 2 * (size_t)view * nv : nullptr;
    float* gv = gclip ? gclip + (size_t)view * nv * 4 : nullptr;
    const float2 s = make_float2(W / 2.f, H / 2.f);
    float acc[8];
    for (int i = 0; i < C && i < 8; ++i) acc[i] = gout[pidx * C + i];
    for (int k = 0; k < 4; ++k) {
        const int dir = k >> 1;
        const bool self = (k & 1) == 0;
        int qx = px, qy = py;
        if (!self) { if (dir == 0) ++qx; else ++qy; }
        if (dir == 0 ? (qx == 0 || qx >= W) : (qy == 0 || qy >= H)) continue;
        const long long q = self ? pidx : (dir == 0 ? pidx + 1 : pidx + W);
        AAPair P;
        if (!aa_pair(proj, scr, nv, tri, nt, rast, q, qx, qy, W, dir, !exact, s, P, flags, exact && gv)) continue;
        // the reference's horizontal typo can give pp == op: its two colour
        // terms cancel and the clip term is zero (antialias.cu:279, :216-223)
        if (P.pp == P.op) continue;
        const bool mine = P.pp == pidx || P.op == pidx;
        if (!mine && !(self && gv)) continue;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const int ka = e, kb = (e + 1) % 3;
            float a, alpha, ia, n;
            float2 ev;
            if (!aa_edge(P.t.v[ka], P.t.v[kb], P.o, a, alpha, ia, ev, n)) continue;
            const long long src = alpha > 0 ? P.op : P.pp;
            const float sign = P.pp == pidx ? 1.f : -1.f;
            float d = 0.f;
            if (C4) {
                float4 g = reinterpret_cast<const float4*>(gout)[src];
                if (mine) {
                    acc[0] += sign * alpha * g.x; acc[1] += sign * alpha * g.y;
                    acc[2] += sign * alpha * g.z; acc[3] += sign * alpha * g.w;
                }
                if (self && gv) {
                    float4 ip = reinterpret_cast<const float4*>(in)[P.pp], io = reinterpret_cast<const float4*>(in)[P.op];
                    d = g.x * (ip.x - io.x) + g.y * (ip.y - io.y) + g.z * (ip.z - io.z) + g.w * (ip.w - io.w);
                }
            } else {
                for (int i = 0; i < C && i < 8; ++i) {
                    float g = gout[src * C + i];
                    if (mine) acc[i] += sign * alpha * g;
                    d += g * (in[P.pp * C + i] - in[P.op * C + i]);
                }
            }
            if (self && gv) {
                float2 pa = P.t.v[ka], pb = P.t.v[kb];
                d *= ia;
                float2 da = make_float2(d * s.x * P.t.iw[ka], d * s.y * P.t.iw[ka]);
                float2 dbv = make_float2(d * s.x * P.t.iw[kb], d * s.y * P.t.iw[kb]);
                float r = (n > 0 ? ev.x : -ev.y) * ia;
                if (n > 0) {
                    da.x *= pb.y; da.y *= pb.y; da.y *= r;
                    dbv.x *= -pa.y; dbv.y *= -pa.y; dbv.y *= r;
                } else {
                    da.x *= -pb.x; da.y *= -pb.x; da.x *= r;
                    dbv.x *= pa.x; dbv.y *= pa.x; dbv.x *= r;
                }
                // w: the reference multiplies by the pixel position relative to
                // the pixel edge (antialias.cu:241-242); the derivative of
                // (x/w + 1) s - f w.r.t. w needs x/w (EXACT)
                const float2 wa = exact ? P.t.ndc[ka] : pa, wb = exact ? P.t.ndc[kb] : pb;
                red_add4(gv + (size_t)P.t.id[ka] * 4, da.x, da.y, 0.f, -(da.x * wa.x + da.y * wa.y));
                red_add4(gv + (size_t)P.t.id[kb] * 4, dbv.x, dbv.y, 0.f, -(dbv.x * wb.x + dbv.y * wb.y));
            }
        }
    }
    if (C4) reinterpret_cast<float4*>(gin)[pidx] = make_float4(acc[0], acc[1], acc[2], acc[3]);
    else for (int i = 0; i < C && i < 8; ++i) gin[pidx * C + i] = acc[i];
}

// Tile forms of the two passes for C = 4: a block owns a 32 x 8 pixel tile
// and evaluates every pixel pair it needs ONCE -- the horizontal pairs whose
// right pixel q lies in columns x0 .. x0+32 and the vertical pairs whose upper
// pixel lies in rows y0 .. y0+8 (one column and one row of halo) -- keeping
// per pair the summed edge terms sent to its lower pixel (q-1 or q-W) and to
// q in shared memory; each pixel then adds the four pair terms that touch it.
// The gather kernels above evaluate each pair once per pixel of the pair.
// The kernels wait mostly on dependent loads (rast -> triangle -> vertex), so
// they are held to 32 registers for eight resident blocks per SM: the few
// spilled values stay in L1, and the extra warps hide the load latency.
constexpr int AAT_X = 32, AAT_Y = 8;
constexpr int AAT_NH = (AAT_X + 1) * AAT_Y;   // horizontal pairs of a tile (with halo column)
constexpr int AAT_NP = AAT_NH + AAT_X * (AAT_Y + 1);
// A tile's candidate list kept between the forward and the backward of one
// step (entry 0: the count; then the pair indices), AAT_CL entries per tile.
constexpr int AAT_CL = 560;
static_assert(AAT_NP < AAT_CL && AAT_NP < 65536, "candidate list entries");

// Pair i of the tile at (x0, y0): direction and the coordinates of q;
// `own`: the pair belongs to this tile (not its halo).
DEV void aat_pair_coords(int i, int x0, int y0, int& dir, int& qx, int& qy, bool& own) {
    if (i < AAT_NH) {
        const int r = i / (AAT_X + 1), c = i - r * (AAT_X + 1);
        dir = 0; qx = x0 + c; qy = y0 + r; own = c < AAT_X;
    } else {
        const int j = i - AAT_NH, r = j / AAT_X, c = j - r * AAT_X;
        dir = 1; qx = x0 + c; qy = y0 + r; own = r < AAT_Y;
    }
}

// Lists the tile's pairs whose two pixels hold different triangle ids (the
// only pairs with edge terms) in s_list and zeroes every pair's terms; the
// pairs are then evaluated from the list with full warps.  Returns the count.
DEV int aat_candidates(const float4* __restrict__ rast, long long vb, int W, int H, int x0, int y0, float4* s_lo,
                       float4* s_hi, int* s_list, int* s_n) {
    if (threadIdx.x == 0) *s_n = 0;
    __syncthreads();
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int base = 0; base < AAT_NP; base += blockDim.x) {
        const int i = base + threadIdx.x;
        bool cand = false;
        if (i < AAT_NP) {
            int dir, qx, qy;
            bool own;
            aat_pair_coords(i, x0, y0, dir, qx, qy, own);
            if (qx < W && qy < H && (dir == 0 ? qx > 0 : qy > 0)) {
                const long long q = vb + (long long)qy * W + qx;
                cand = rast[q].w != rast[dir == 0 ? q - 1 : q - W].w;
            }
            s_lo[i] = z;
            s_hi[i] = z;
        }
        const unsigned ball = __ballot_sync(0xffffffffu, cand);
        int slot = 0;
        if ((threadIdx.x & 31) == 0 && ball) slot = atomicAdd(s_n, __popc(ball));
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (cand) s_list[slot + __popc(ball & ((1u << (threadIdx.x & 31)) - 1u))] = i;
    }
    __syncthreads();
    return *s_n;
}

DEV float4 f4add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
DEV float4 f4sub(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
DEV float4 f4mul(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }

// Sum of the four pair terms at pixel (tx, ty) of the tile.
DEV float4 aat_gather(const float4* s_lo, const float4* s_hi, int tx, int ty) {
    const int h = ty * (AAT_X + 1) + tx, v = AAT_NH + ty * AAT_X + tx;
    return f4add(f4add(s_hi[h], s_lo[h + 1]), f4add(s_hi[v], s_lo[v + AAT_X]));
}

// MSE: instead of the antialiased colour, write its loss gradient
// out = aa - target and add 0.5 |aa - target|^2 to the loss (loss.cu:22-30):
// block sums in double go to mse->sum; the last block to finish writes the
// float loss and clears the sum and the block counter for the next pass.
struct MseOut {
    const float4* target;
    double* sum;
    unsigned* done;
    float* loss;
};

template <bool MSE>
__global__ void __launch_bounds__(256, 8) k_aa_fwd_tile(const float4* __restrict__ clip, const float4* __restrict__ scr_all,
                                                     int nv, const uint32_t* __restrict__ tri, int nt,
                                                     const float4* __restrict__ rast, int W, int H,
                                                     const float4* __restrict__ in, float4* __restrict__ out, int* flags,
                                                     MseOut mse, uint16_t* __restrict__ clist) {
    __shared__ float4 s_lo[AAT_NP], s_hi[AAT_NP];
    __shared__ int s_list[AAT_NP], s_n;
    const int view = blockIdx.z, x0 = blockIdx.x * AAT_X, y0 = blockIdx.y * AAT_Y;
    const long long vb = (long long)view * W * H;
    const float4* proj = clip + (size_t)view * nv;
    const float4* scr = scr_all ? scr_all + 2 * (size_t)view * nv : nullptr;
    const float2 s = make_float2(W / 2.f, H / 2.f);
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const int ncand = aat_candidates(rast, vb, W, H, x0, y0, s_lo, s_hi, s_list, &s_n);
    if (clist) {   // for the backward of the same step (same rast, same candidates)
        uint16_t* cl = clist + ((size_t)(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * AAT_CL;
        for (int k = threadIdx.x; k < ncand; k += blockDim.x) cl[1 + k] = (uint16_t)s_list[k];
        if (threadIdx.x == 0) cl[0] = (uint16_t)ncand;
    }
    for (int k = threadIdx.x; k < ncand; k += blockDim.x) {
        const int i = s_list[k];
        int dir, qx, qy;
        bool own;
        aat_pair_coords(i, x0, y0, dir, qx, qy, own);
        float4 lo = z, hi = z;
        AAPair P;
        const long long q = vb + (long long)qy * W + qx;
        if (aa_pair(proj, scr, nv, tri, nt, rast, q, qx, qy, W, dir, false, s, P, flags, false)) {
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                float a, alpha, ia, n;
                float2 ev;
                if (!aa_edge(P.t.v[e], P.t.v[(e + 1) % 3], P.o, a, alpha, ia, ev, n)) continue;
                const float4 t = f4mul(f4sub(in[P.pp], in[P.op]), alpha);
                if ((alpha > 0 ? P.op : P.pp) == q) hi = f4add(hi, t); else lo = f4add(lo, t);
            }
        }
        s_lo[i] = lo;
        s_hi[i] = hi;
    }
    __syncthreads();
    const int tx = threadIdx.x % AAT_X, ty = threadIdx.x / AAT_X;
    const int px = x0 + tx, py = y0 + ty;
    const bool inside = px < W && py < H;
    const long long p = vb + (long long)py * W + px;
    if (!MSE) {
        if (inside) out[p] = f4add(in[p], aat_gather(s_lo, s_hi, tx, ty));
        return;
    }
    double acc = 0.0;
    if (inside) {
        const float4 a = f4add(in[p], aat_gather(s_lo, s_hi, tx, ty)), t = mse.target[p];
        const float4 g = make_float4(a.x - t.x, a.y - t.y, a.z - t.z, a.w - t.w);
        out[p] = g;
        acc = (double)g.x * g.x + (double)g.y * g.y + (double)g.z * g.z + (double)g.w * g.w;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += part[w];
        atomicAdd(mse.sum, b);
        __threadfence();
        const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
        if (atomicAdd(mse.done, 1u) == nblk - 1) {
            const double total = atomicAdd(mse.sum, 0.0);
            *mse.loss = (float)(total * 0.5);
            *mse.sum = 0.0;
            *mse.done = 0u;
        }
    }
}

__global__ void __launch_bounds__(256, 8) k_aa_bwd_tile(const float4* __restrict__ clip, const float4* __restrict__ scr_all,
                                                     int nv, const uint32_t* __restrict__ tri, int nt,
                                                     const float4* __restrict__ rast, int W, int H,
                                                     const float4* __restrict__ in, const float4* __restrict__ gout,
                                                     float4* __restrict__ gin, float* __restrict__ gclip, int exact,
                                                     int* flags, const uint16_t* __restrict__ clist) {
    __shared__ float4 s_lo[AAT_NP], s_hi[AAT_NP];
    __shared__ int s_list[AAT_NP], s_n;
    const int view = blockIdx.z, x0 = blockIdx.x * AAT_X, y0 = blockIdx.y * AAT_Y;
    const long long vb = (long long)view * W * H;
    const float4* proj = clip + (size_t)view * nv;
    const float4* scr = scr_all ? scr_all + 2 * (size_t)view * nv : nullptr;
    float* gv = gclip ? gclip + (size_t)view * nv * 4 : nullptr;
    const float2 s = make_float2(W / 2.f, H / 2.f);
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    int ncand;
    if (clist) {   // the forward's list of this tile
        const uint16_t* cl = clist + ((size_t)(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * AAT_CL;
        ncand = cl[0];
        for (int i = threadIdx.x; i < AAT_NP; i += blockDim.x) {
            s_lo[i] = z;
            s_hi[i] = z;
            if (i < ncand) s_list[i] = cl[1 + i];
        }
        __syncthreads();
    } else {
        ncand = aat_candidates(rast, vb, W, H, x0, y0, s_lo, s_hi, s_list, &s_n);
    }
    for (int k = threadIdx.x; k < ncand; k += blockDim.x) {
        const int i = s_list[k];
        int dir, qx, qy;
        bool own;
        aat_pair_coords(i, x0, y0, dir, qx, qy, own);
        own = own && gv;
        float4 lo = z, hi = z;
        AAPair P;
        const long long q = vb + (long long)qy * W + qx;
        // the reference's horizontal typo can give pp == op: its two colour
        // terms cancel and the clip term is zero (antialias.cu:279, :216-223)
        if (aa_pair(proj, scr, nv, tri, nt, rast, q, qx, qy, W, dir, !exact, s, P, flags, exact && own) &&
            P.pp != P.op) {
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                const int ka = e, kb = (e + 1) % 3;
                float a, alpha, ia, n;
                float2 ev;
                if (!aa_edge(P.t.v[ka], P.t.v[kb], P.o, a, alpha, ia, ev, n)) continue;
                const float4 g = gout[alpha > 0 ? P.op : P.pp];
                const float4 t = f4mul(g, alpha);
                if (P.pp == q) { hi = f4add(hi, t); lo = f4sub(lo, t); }
                else { lo = f4add(lo, t); hi = f4sub(hi, t); }
                if (own) {
                    const float4 ip = in[P.pp], io = in[P.op];
                    float d = g.x * (ip.x - io.x) + g.y * (ip.y - io.y) + g.z * (ip.z - io.z) + g.w * (ip.w - io.w);
                    float2 pa = P.t.v[ka], pb = P.t.v[kb];
                    d *= ia;
                    float2 da = make_float2(d * s.x * P.t.iw[ka], d * s.y * P.t.iw[ka]);
                    float2 dbv = make_float2(d * s.x * P.t.iw[kb], d * s.y * P.t.iw[kb]);
                    const float r = (n > 0 ? ev.x : -ev.y) * ia;
                    if (n > 0) {
                        da.x *= pb.y; da.y *= pb.y; da.y *= r;
                        dbv.x *= -pa.y; dbv.y *= -pa.y; dbv.y *= r;
                    } else {
                        da.x *= -pb.x; da.y *= -pb.x; da.x *= r;
                        dbv.x *= pa.x; dbv.y *= pa.x; dbv.x *= r;
                    }
                    // w: as in k_aa_bwd (antialias.cu:241-242 in COMPAT, x/w in EXACT)
                    const float2 wa = exact ? P.t.ndc[ka] : pa, wb = exact ? P.t.ndc[kb] : pb;
                    red_add4(gv + (size_t)P.t.id[ka] * 4, da.x, da.y, 0.f, -(da.x * wa.x + da.y * wa.y));
                    red_add4(gv + (size_t)P.t.id[kb] * 4, dbv.x, dbv.y, 0.f, -(dbv.x * wb.x + dbv.y * wb.y));
                }
            }
        }
        s_lo[i] = lo;
        s_hi[i] = hi;
    }
    __syncthreads();
    const int tx = threadIdx.x % AAT_X, ty = threadIdx.x / AAT_X;
    const int px = x0 + tx, py = y0 + ty;
    if (px >= W || py >= H) return;
    const long long p = vb + (long long)py * W + px;
    gin[p] = f4add(gout[p], aat_gather(s_lo, s_hi, tx, ty));
}

// ----------------------------------------------------------------- loss
__global__ void k_mse(const float* __restrict__ pred, const float* __restrict__ tgt, long long n, float* __restrict__ grad,
                      float* __restrict__ loss) {
    __shared__ double part[32];
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float g = pred[i] - tgt[i];
        grad[i] = g;
        acc += (double)g * (double)g;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) atomicAdd(loss, (float)(acc * 0.5));
    }
}

// ----------------------------------------------------------------- adam
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, double b1, double b2, double lr, double eps, double c1, double c2, int vec) {
    long long n4 = vec ? n / 4 : 0;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 P = reinterpret_cast<float4*>(p)[i], G = reinterpret_cast<const float4*>(g)[i];
        float4 M = reinterpret_cast<float4*>(m)[i], V = reinterpret_cast<float4*>(v)[i];
        adam_one(P.x, G.x, M.x, V.x, b1, b2, lr, eps, c1, c2);
        adam_one(P.y, G.y, M.y, V.y, b1, b2, lr, eps, c1, c2);
        adam_one(P.z, G.z, M.z, V.z, b1, b2, lr, eps, c1, c2);
        adam_one(P.w, G.w, M.w, V.w, b1, b2, lr, eps, c1, c2);
        reinterpret_cast<float4*>(p)[i] = P; reinterpret_cast<float4*>(m)[i] = M; reinterpret_cast<float4*>(v)[i] = V;
    }
    for (long long i = n4 * 4 + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        adam_one(p[i], g[i], m[i], v[i], b1, b2, lr, eps, c1, c2);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

dim3 aat_grid(int W, int H, int views) {
    return dim3((unsigned)((W + AAT_X - 1) / AAT_X), (unsigned)((H + AAT_Y - 1) / AAT_Y), (unsigned)views);
}

int grid_for(long long n, int threads, int sm) {
    long long b = (n + threads - 1) / threads;
    long long cap = (long long)sm * 8;
    return (int)(b < 1 ? 1 : b > cap ? cap : b);
}

}  // namespace

vcl_status aa_edges_fwd(vcl_ctx* ctx, const float* clip, const float* scr, int nv, const uint32_t* tri, int nt,
                        const float* rast, int W, int H, int views, int C, const float* in, float* out, cudaStream_t s) {
    long long npix = (long long)W * H * views;
    const float4* sc = (const float4*)scr;
    if (C == 4 && aligned16(in) && aligned16(out) && views <= 65535)
        k_aa_fwd_tile<false><<<aat_grid(W, H, views), 256, 0, s>>>((const float4*)clip, sc, nv, tri, nt,
                                                                    (const float4*)rast, W, H, (const float4*)in,
                                                                    (float4*)out, ctx->dev_flags, MseOut{}, nullptr);
    else
        k_aa_fwd<0><<<vcl_blocks(npix, 256), 256, 0, s>>>((const float4*)clip, sc, nv, tri, nt, (const float4*)rast, W,
                                                         H, npix, C, in, out, ctx->dev_flags);
    return vcl_launch_check(ctx, "antialias_fwd");
}

size_t aa_cand_list_bytes(int W, int H, int views) {
    const dim3 g = aat_grid(W, H, views);
    return sizeof(uint16_t) * AAT_CL * (size_t)g.x * g.y * g.z;
}

vcl_status aa_edges_fwd_mse(vcl_ctx* ctx, const float* clip, const float* scr, int nv, const uint32_t* tri, int nt,
                            const float* rast, int W, int H, int views, const float* in, const float* target,
                            float* grad, double* sum, unsigned* done, float* loss, uint16_t* clist, cudaStream_t s) {
    VCL_REQUIRE(aligned16(in) && aligned16(target) && aligned16(grad) && views <= 65535,
                "antialias+mse: 16-byte aligned C = 4 buffers and at most 65535 views");
    k_aa_fwd_tile<true><<<aat_grid(W, H, views), 256, 0, s>>>((const float4*)clip, (const float4*)scr, nv, tri, nt,
                                                               (const float4*)rast, W, H, (const float4*)in,
                                                               (float4*)grad, ctx->dev_flags,
                                                               MseOut{(const float4*)target, sum, done, loss}, clist);
    return vcl_launch_check(ctx, "antialias_fwd+mse");
}

vcl_status aa_edges_bwd(vcl_ctx* ctx, const float* clip, const float* scr, int nv, const uint32_t* tri, int nt,
                        const float* rast, int W, int H, int views, int C, const float* in, const float* grad_out,
                        float* grad_in, float* grad_clip, cudaStream_t s, const uint16_t* clist) {
    long long npix = (long long)W * H * views;
    int exact = ctx->mode == VCL_MODE_EXACT;
    const float4* sc = (const float4*)scr;
    if (C == 4 && aligned16(in) && aligned16(grad_out) && aligned16(grad_in) && views <= 65535)
        k_aa_bwd_tile<<<aat_grid(W, H, views), 256, 0, s>>>((const float4*)clip, sc, nv, tri, nt, (const float4*)rast, W,
                                                             H, (const float4*)in, (const float4*)grad_out,
                                                             (float4*)grad_in, grad_clip, exact, ctx->dev_flags, clist);
    else
        k_aa_bwd<0><<<vcl_blocks(npix, 256), 256, 0, s>>>((const float4*)clip, sc, nv, tri, nt, (const float4*)rast, W,
                                                         H, npix, C, in, grad_out, grad_in, grad_clip, exact,
                                                         ctx->dev_flags);
    return vcl_launch_check(ctx, "antialias_bwd");
}

void launch_aa_screen(const float* clip, long long n, int W, int H, float* scr, cudaStream_t s) {
    k_aa_screen<<<vcl_blocks(n, 256), 256, 0, s>>>((const float4*)clip, n, W / 2.f, H / 2.f, (float4*)scr);
}

void launch_mip_down(const float* src, float* dst, int w, int h, int C, cudaStream_t s) {
    k_mip_down<<<vcl_blocks((long long)w * h, 256), 256, 0, s>>>(src, dst, w, h, C);
}

extern "C" {

VCL_API vcl_status vcl_check_indices(vcl_ctx* ctx, void* stream, int* bad) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(bad, "bad is null");
    cudaStream_t s = (cudaStream_t)stream;
    int h = 0;
    vcl_status st = vcl_cuda_check(ctx, cudaMemcpyAsync(&h, ctx->dev_flags + 1, sizeof(int), cudaMemcpyDeviceToHost, s),
                                   "index flag readback");
    if (!st) st = vcl_cuda_check(ctx, cudaMemsetAsync(ctx->dev_flags + 1, 0, sizeof(int), s), "index flag clear");
    if (!st) st = vcl_cuda_check(ctx, cudaStreamSynchronize(s), "index flag sync");
    *bad = h;
    return st;
}

VCL_API vcl_status vcl_project_fwd(vcl_ctx* ctx, const float* mats, int views, const float* pos, int nv, int dim,
                                   float* out, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(mats && pos && out && views > 0 && nv >= 0 && (dim == 3 || dim == 4), "bad project_fwd arguments");
    long long n = (long long)views * nv;
    if (n == 0) return VCL_OK;
    k_project_fwd<<<vcl_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(mats, views, pos, nv, dim, out);
    return vcl_launch_check(ctx, "project_fwd");
}

VCL_API vcl_status vcl_project_bwd(vcl_ctx* ctx, const float* mats, int views, const float* grad_out, int nv, int dim,
                                   float* grad_pos, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(mats && grad_out && grad_pos && views > 0 && nv >= 0 && (dim == 3 || dim == 4), "bad project_bwd arguments");
    if (nv == 0) return VCL_OK;
    k_project_bwd<<<vcl_blocks(nv, 256), 256, 0, (cudaStream_t)stream>>>(mats, views, grad_out, nv, dim, grad_pos);
    return vcl_launch_check(ctx, "project_bwd");
}

VCL_API vcl_status vcl_interpolate_fwd(vcl_ctx* ctx, const float* rast, const float* db, int W, int H, int views,
                                       const float* attr, int nv, int dim, const uint32_t* tri, int nt, float* out,
                                       float* out_da, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && attr && tri && out && W > 0 && H > 0 && views > 0 && dim > 0, "bad interpolate_fwd arguments");
    VCL_REQUIRE(!out_da || db, "out_da needs db");
    VCL_REQUIRE(aligned16(rast) && (!db || aligned16(db)) && ((uintptr_t)out_da & 7) == 0, "misaligned buffer");
    long long npix = (long long)W * H * views;
    k_interp_fwd<<<vcl_blocks(npix, 256), 256, 0, (cudaStream_t)stream>>>(
        (const float4*)rast, (const float4*)db, attr, nv, dim, tri, nt, npix, out, (float2*)out_da, ctx->dev_flags);
    return vcl_launch_check(ctx, "interpolate_fwd");
}

VCL_API vcl_status vcl_interpolate_bwd(vcl_ctx* ctx, const float* rast, int W, int H, int views, const float* attr,
                                       int nv, int dim, const uint32_t* tri, int nt, const float* grad_out,
                                       float* grad_attr, float* grad_bary, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && attr && tri && grad_out && W > 0 && H > 0 && views > 0 && dim > 0, "bad interpolate_bwd arguments");
    VCL_REQUIRE(aligned16(rast) && ((uintptr_t)grad_bary & 7) == 0 && (dim != 4 || aligned16(grad_attr)) &&
                    ((uintptr_t)grad_attr & 7) == 0, "misaligned buffer");
    long long npix = (long long)W * H * views;
    k_interp_bwd<<<vcl_blocks(npix, 256), 256, 0, (cudaStream_t)stream>>>(
        (const float4*)rast, attr, nv, dim, tri, nt, npix, grad_out, grad_attr, (float2*)grad_bary,
        ctx->mode == VCL_MODE_EXACT, ctx->dev_flags);
    return vcl_launch_check(ctx, "interpolate_bwd");
}

VCL_API vcl_status vcl_texture_fwd(vcl_ctx* ctx, const float* rast, const float* uv, const float* uv_da, int W, int H,
                                   int views, const float* pyramid, int tw, int th, int C, int levels, float* out,
                                   void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && uv && pyramid && out && W > 0 && H > 0 && views > 0 && C > 0 && tw > 0 && th > 0,
                "bad texture_fwd arguments");
    VCL_REQUIRE(levels >= 1 && levels == vcl_tex_levels(tw, th, levels), "levels %d invalid for %dx%d", levels, tw, th);
    VCL_REQUIRE(levels == 1 || uv_da, "uv_da needed for a mip-mapped texture");
    VCL_REQUIRE(aligned16(rast) && ((uintptr_t)uv & 7) == 0 && (!uv_da || aligned16(uv_da)), "misaligned buffer");
    TexDesc d = make_desc(tw, th, C, levels);
    long long npix = (long long)W * H * views;
    cudaStream_t s = (cudaStream_t)stream;
    if (C == 4 && aligned16(pyramid) && aligned16(out))
        k_tex_fwd<1><<<vcl_blocks(npix, 256), 256, 0, s>>>(d, pyramid, (const float4*)rast, (const float2*)uv,
                                                          (const float4*)uv_da, npix, out);
    else
        k_tex_fwd<0><<<vcl_blocks(npix, 256), 256, 0, s>>>(d, pyramid, (const float4*)rast, (const float2*)uv,
                                                          (const float4*)uv_da, npix, out);
    return vcl_launch_check(ctx, "texture_fwd");
}

VCL_API vcl_status vcl_texture_bwd(vcl_ctx* ctx, const float* rast, const float* uv, const float* uv_da, int W, int H,
                                   int views, const float* pyramid, int tw, int th, int C, int levels,
                                   const float* grad_out, float* grad_pyramid, float* grad_uv, float* grad_uv_da,
                                   void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && uv && pyramid && grad_out && W > 0 && H > 0 && views > 0 && C > 0 && tw > 0 && th > 0,
                "bad texture_bwd arguments");
    VCL_REQUIRE(levels >= 1 && levels == vcl_tex_levels(tw, th, levels), "levels %d invalid for %dx%d", levels, tw, th);
    VCL_REQUIRE(levels == 1 || uv_da, "uv_da needed for a mip-mapped texture");
    VCL_REQUIRE(aligned16(rast) && ((uintptr_t)uv & 7) == 0 && (!uv_da || aligned16(uv_da)) &&
                    ((uintptr_t)grad_uv & 7) == 0 && aligned16(grad_uv_da), "misaligned buffer");
    TexDesc d = make_desc(tw, th, C, levels);
    long long npix = (long long)W * H * views;
    cudaStream_t s = (cudaStream_t)stream;
    int exact = ctx->mode == VCL_MODE_EXACT;
    if (C == 4 && aligned16(pyramid) && aligned16(grad_out) && aligned16(grad_pyramid))
        k_tex_bwd<1><<<vcl_blocks(npix, 256), 256, 0, s>>>(d, pyramid, (const float4*)rast, (const float2*)uv,
                                                          (const float4*)uv_da, npix, grad_out, grad_pyramid,
                                                          (float2*)grad_uv, (float4*)grad_uv_da, exact);
    else
        k_tex_bwd<0><<<vcl_blocks(npix, 256), 256, 0, s>>>(d, pyramid, (const float4*)rast, (const float2*)uv,
                                                          (const float4*)uv_da, npix, grad_out, grad_pyramid,
                                                          (float2*)grad_uv, (float4*)grad_uv_da, exact);
    return vcl_launch_check(ctx, "texture_bwd");
}

VCL_API vcl_status vcl_texture_build_mips(vcl_ctx* ctx, float* pyramid, int tw, int th, int C, int levels, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(pyramid && tw > 0 && th > 0 && C > 0, "bad build_mips arguments");
    VCL_REQUIRE(levels >= 1 && levels == vcl_tex_levels(tw, th, levels), "levels %d invalid for %dx%d", levels, tw, th);
    VCL_REQUIRE(C != 4 || aligned16(pyramid), "misaligned pyramid");
    cudaStream_t s = (cudaStream_t)stream;
    for (int l = 1; l < levels; ++l) {
        int w = tw >> l, h = th >> l;
        k_mip_down<<<vcl_blocks((long long)w * h, 256), 256, 0, s>>>(pyramid + vcl_tex_level_offset(tw, th, C, l - 1),
                                                                      pyramid + vcl_tex_level_offset(tw, th, C, l), w, h, C);
    }
    return vcl_launch_check(ctx, "build_mips");
}

VCL_API vcl_status vcl_texture_grad_pushdown(vcl_ctx* ctx, float* grad_pyramid, int tw, int th, int C, int levels,
                                             void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(grad_pyramid && tw > 0 && th > 0 && C > 0, "bad pushdown arguments");
    VCL_REQUIRE(levels >= 1 && levels == vcl_tex_levels(tw, th, levels), "levels %d invalid for %dx%d", levels, tw, th);
    cudaStream_t s = (cudaStream_t)stream;
    float wgt = ctx->mode == VCL_MODE_EXACT ? 0.25f : 1.f;
    for (int l = levels - 1; l > 0; --l) {
        int w = tw >> l, h = th >> l;
        k_mip_push<<<vcl_blocks((long long)w * h * C, 256), 256, 0, s>>>(
            grad_pyramid + vcl_tex_level_offset(tw, th, C, l), grad_pyramid + vcl_tex_level_offset(tw, th, C, l - 1), w, h,
            C, wgt);
    }
    return vcl_launch_check(ctx, "grad_pushdown");
}

VCL_API vcl_status vcl_clamp(vcl_ctx* ctx, float* p, size_t n, float lo, float hi, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(p || n == 0, "null buffer");
    if (n == 0) return VCL_OK;
    k_clamp<<<vcl_blocks((long long)n, 256), 256, 0, (cudaStream_t)stream>>>(p, (long long)n, lo, hi);
    return vcl_launch_check(ctx, "clamp");
}

VCL_API vcl_status vcl_antialias_fwd(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt,
                                     const float* rast, int W, int H, int views, int C, const float* in, float* out,
                                     void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(clip && tri && rast && in && out && W > 0 && H > 0 && views > 0 && C > 0, "bad antialias_fwd arguments");
    VCL_REQUIRE(aligned16(clip) && aligned16(rast), "misaligned buffer");
    VCL_REQUIRE(in != out, "antialias_fwd cannot run in place");
    VCL_REQUIRE(C <= 8, "antialias supports up to 8 channels");
    return aa_edges_fwd(ctx, clip, nullptr, nv, tri, nt, rast, W, H, views, C, in, out, (cudaStream_t)stream);
}

VCL_API vcl_status vcl_antialias_bwd(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt,
                                     const float* rast, int W, int H, int views, int C, const float* in,
                                     const float* grad_out, float* grad_in, float* grad_clip, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(clip && tri && rast && in && grad_out && grad_in && W > 0 && H > 0 && views > 0 && C > 0,
                "bad antialias_bwd arguments");
    VCL_REQUIRE(aligned16(clip) && aligned16(rast) && aligned16(grad_clip), "misaligned buffer");
    VCL_REQUIRE(grad_in != grad_out, "antialias_bwd cannot run in place");
    VCL_REQUIRE(C <= 8, "antialias supports up to 8 channels");
    return aa_edges_bwd(ctx, clip, nullptr, nv, tri, nt, rast, W, H, views, C, in, grad_out, grad_in, grad_clip,
                        (cudaStream_t)stream);
}

VCL_API vcl_status vcl_mse(vcl_ctx* ctx, const float* pred, const float* target, size_t n, float* grad, float* loss_dev,
                           void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(pred && target && grad && loss_dev, "bad mse arguments");
    cudaStream_t s = (cudaStream_t)stream;
    vcl_status st = vcl_cuda_check(ctx, cudaMemsetAsync(loss_dev, 0, sizeof(float), s), "mse clear");
    if (st) return st;
    if (n == 0) return VCL_OK;
    k_mse<<<grid_for((long long)n, 256, ctx->sm_count), 256, 0, s>>>(pred, target, (long long)n, grad, loss_dev);
    return vcl_launch_check(ctx, "mse");
}

VCL_API vcl_status vcl_adam_step(vcl_ctx* ctx, float* p, const float* g, float* m, float* v, size_t n, double lr,
                                 double beta1, double beta2, double eps, int step, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(p && g && m && v && step >= 1, "bad adam arguments");
    if (n == 0) return VCL_OK;
    int vec = aligned16(p) && aligned16(g) && aligned16(m) && aligned16(v);
    double c1 = ctx->mode == VCL_MODE_EXACT ? 1.0 : beta1, c2 = ctx->mode == VCL_MODE_EXACT ? 1.0 : beta2;
    for (int k = 0; k < step; ++k) { c1 *= beta1; c2 *= beta2; }
    k_adam<<<grid_for((long long)(n + 3) / 4, 256, ctx->sm_count), 256, 0, (cudaStream_t)stream>>>(
        p, g, m, v, (long long)n, beta1, beta2, lr, eps, 1.0 - c1, 1.0 - c2, vec);
    return vcl_launch_check(ctx, "adam_step");
}

}  // extern "C"

// Spherical-Gaussian shading operators (reference material.cu): NormalAxis,
// ViewAxis, SGSpecular and SphericalGaussian, forward and backward.  One
// thread per pixel; the K lobes are staged in shared memory.  The SG
// backward reduces the per-lobe gradients (axis, sharpness, amplitude) over
// all pixels: warp shuffles, then per-warp shared accumulators, then one
// atomic per block and lobe parameter -- the reference accumulates them
// with unsynchronised adds from every thread (material.cu:428-436).
#include "common.cuh"

namespace {

constexpr int CMAX = 8;
constexpr float DIFF_SHARP = 2.133f;
constexpr float DIFF_AMP = 2.34f;

// material.cu:25-48 (the branch taken with a normal map bound)
__global__ void k_normal_axis(const float4* __restrict__ rast, long long npix, const float* __restrict__ rot,
                              const float* __restrict__ normal, int nv, const uint32_t* __restrict__ tri, int nt,
                              float* __restrict__ out, int* flags) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float4 r = rast[p];
    int idx = rast_id(r.w);
    bool ok = idx >= 0 && idx < nt;
    uint32_t i0 = 0, i1 = 0, i2 = 0;
    if (ok) {
        i0 = tri[3 * (size_t)idx]; i1 = tri[3 * (size_t)idx + 1]; i2 = tri[3 * (size_t)idx + 2];
        ok = i0 < (uint32_t)nv && i1 < (uint32_t)nv && i2 < (uint32_t)nv;
    }
    if (!ok) {
        if (idx >= 0) atomicOr(&flags[1], 1);
        st3(out, p, f3(0.f, 0.f, 0.f));
        return;
    }
    float3 n2 = ld3(normal, i2);
    float3 n0 = ld3(normal, i0) - n2, n1 = ld3(normal, i1) - n2;
    float3 N = normalize3(n0 * r.x + n1 * r.y + n2);
    st3(out, p, f3(rot[0] * N.x + rot[4] * N.y + rot[8] * N.z, rot[1] * N.x + rot[5] * N.y + rot[9] * N.z,
                   rot[2] * N.x + rot[6] * N.y + rot[10] * N.z));
}

// material.cu:92-108
__global__ void k_view_axis(int W, int H, long long npix, const float* __restrict__ pvinv, float* __restrict__ out) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    long long hw = (long long)W * H;
    int view = (int)(p / hw);
    int rem = (int)(p - view * hw);
    int py = rem / W, px = rem - py * W;
    const float* M = pvinv + (size_t)view * 9;
    float sx = (float)px / (float)W * 2.f - 1.f, sy = (float)py / (float)H * 2.f - 1.f;
    st3(out, p, normalize3(f3(M[0], M[1], M[2]) * sx + f3(M[3], M[4], M[5]) * sy + f3(M[6], M[7], M[8])));
}

struct SpecLobe { float3 p; float vn, pn, m, m2, Gv, Gp, F, iGv, iGp; };

// material.cu:155-178 / :213-240
DEV SpecLobe spec_eval(float3 n, float3 vw, float m, float ior) {
    SpecLobe s;
    float3 v = f3(-vw.x, -vw.y, -vw.z);
    s.p = n * (2.f * dot3(v, n)) - v;
    s.m = m; s.m2 = m * m;
    s.vn = fmaxf(dot3(v, n), 0.f);
    float vn2 = s.vn * s.vn;
    s.iGv = sqrtf(vn2 + s.m2 * (1.f - vn2));
    s.Gv = 1.f / fmaxf(s.vn + s.iGv, 1e-6f);
    s.pn = fmaxf(dot3(s.p, n), 0.f);
    float pn2 = s.pn * s.pn;
    s.iGp = sqrtf(pn2 + s.m2 * (1.f - pn2));
    s.Gp = 1.f / fmaxf(s.pn + s.iGp, 1e-6f);
    float g = sqrtf(ior * ior - 1.f + pn2);
    float gp = g + s.pn, gm = g - s.pn;
    float f0 = gm / gp;
    float f1 = (s.pn * gp - 1.f) / (s.pn * gm + 1.f);
    s.F = f0 * f0 * (1.f + f1 * f1);
    return s;
}

__global__ void k_sg_spec_fwd(const float4* __restrict__ rast, long long npix, const float* __restrict__ normal,
                              const float* __restrict__ view, const float* __restrict__ rough, float ior,
                              float* __restrict__ oax, float* __restrict__ osh, float* __restrict__ oam) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    if (rast_id(rast[p].w) < 0) {
        st3(oax, p, f3(0.f, 0.f, 0.f)); osh[p] = 0.f; oam[p] = 0.f;
        return;
    }
    SpecLobe s = spec_eval(ld3(normal, p), ld3(view, p), rough[p], ior);
    st3(oax, p, s.p);
    oam[p] = s.F * s.Gp * s.Gv * s.pn / fmaxf(s.m2, 1e-6f);
    osh[p] = .5f / fmaxf(s.m2 * s.vn, 1e-6f);
}

// material.cu:203-249
__global__ void k_sg_spec_bwd(const float4* __restrict__ rast, long long npix, const float* __restrict__ normal,
                              const float* __restrict__ view, const float* __restrict__ rough, float ior,
                              const float* __restrict__ gam, const float* __restrict__ gsh, float* __restrict__ grough) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    if (rast_id(rast[p].w) < 0) return;
    SpecLobe s = spec_eval(ld3(normal, p), ld3(view, p), rough[p], ior);
    float vn2 = s.vn * s.vn, pn2 = s.pn * s.pn;
    float dGvdm = -s.m * (1.f - vn2) / fmaxf(s.iGv, 1e-6f) * s.Gv * s.Gv;
    float dGpdm = -s.m * (1.f - pn2) / fmaxf(s.iGp, 1e-6f) * s.Gp * s.Gp;
    float t1 = -2.f * s.Gp * s.Gv / fmaxf(s.m2 * s.m, 1e-6f) + (s.Gp * dGvdm + s.Gv * dGpdm) / fmaxf(s.m2, 1e-6f);
    float g = grough[p];
    add_nan_check(g, gam[p] * s.F * s.pn * t1);
    add_nan_check(g, gsh[p] * -1.f / fmaxf(s.m2 * s.m * s.vn, 1e-6f));
    grough[p] = g;
}

// SG inner-product term (e^(l-a-b) - e^(-l-a-b)) / max(l, 1e-6) * amp,
// material.cu:309/311.
DEV float sg_term(float l, float a, float b, float amp) {
    return (expf(l - a - b) - expf(-l - a - b)) / fmaxf(l, 1e-6f) * amp;
}

// material.cu:285-323
__global__ void k_sg_fwd(int C, int K, const float* __restrict__ axis, const float* __restrict__ sharp,
                         const float* __restrict__ amp, const float4* __restrict__ rast, long long npix,
                         const float* __restrict__ normal, const float* __restrict__ diffuse, const float* __restrict__ sax,
                         const float* __restrict__ ssh, const float* __restrict__ sam, float* __restrict__ out,
                         float* __restrict__ odiff, float* __restrict__ ospec) {
    extern __shared__ float sm[];
    float* s_ax = sm;             // [K][3], pre-multiplied by sharpness
    float* s_sh = sm + 3 * K;     // [K]
    float* s_am = sm + 4 * K;     // [K][C]
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
        float s = sharp[i];
        s_sh[i] = s;
        s_ax[3 * i] = axis[3 * i] * s; s_ax[3 * i + 1] = axis[3 * i + 1] * s; s_ax[3 * i + 2] = axis[3 * i + 2] * s;
    }
    for (int i = threadIdx.x; i < K * C; i += blockDim.x) s_am[i] = amp[i];
    __syncthreads();
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    if (rast_id(rast[p].w) < 0) {
        for (int k = 0; k < C; ++k) {
            out[p * C + k] = 0.f;
            if (odiff) odiff[p * C + k] = 0.f;
            if (ospec) ospec[p * C + k] = 0.f;
        }
        return;
    }
    float3 dn = ld3(normal, p) * DIFF_SHARP;
    float ss = ssh[p], sa = sam[p];
    float3 sn = ld3(sax, p) * ss;
    float de[CMAX], se[CMAX];
#pragma unroll
    for (int k = 0; k < CMAX; ++k) { de[k] = 0.f; se[k] = 0.f; }
    for (int i = 0; i < K; ++i) {
        float gs = s_sh[i];
        float3 g = f3(s_ax[3 * i], s_ax[3 * i + 1], s_ax[3 * i + 2]);
        float dg = sg_term(len3(dn + g), DIFF_SHARP, gs, DIFF_AMP);
        float sg = sg_term(len3(sn + g), ss, gs, sa);
#pragma unroll
        for (int k = 0; k < CMAX; ++k) {
            if (k >= C) break;
            float a = s_am[i * C + k];
            add_nan_check(de[k], dg * a);
            add_nan_check(se[k], sg * a);
        }
    }
#pragma unroll
    for (int k = 0; k < CMAX; ++k) {
        if (k >= C) break;
        out[p * C + k] = diffuse[p * C + k] * de[k] + se[k];
        if (odiff) odiff[p * C + k] = de[k];
        if (ospec) ospec[p * C + k] = se[k];
    }
}

DEV float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

DEV bool fin3(float3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// material.cu:369-438.  Accumulator layout per lobe: axis xyz, sharpness,
// amplitude[C], then (compat only) the specular sharpness the reference
// indexes by lobe.
__global__ void k_sg_bwd(int C, int K, int nacc, const float* __restrict__ axis, const float* __restrict__ sharp,
                         const float* __restrict__ amp, const float4* __restrict__ rast, long long npix,
                         const float* __restrict__ normal, const float* __restrict__ diffuse, const float* __restrict__ sax,
                         const float* __restrict__ ssh, const float* __restrict__ sam, const float* __restrict__ gout,
                         float* __restrict__ gdiff, float* __restrict__ gaxis, float* __restrict__ gsharp,
                         float* __restrict__ gamp, float* __restrict__ gsax, float* __restrict__ gssh,
                         float* __restrict__ gsam, int exact) {
    extern __shared__ float sm[];
    const int nwarps = blockDim.x >> 5;
    float* s_ax = sm;
    float* s_sh = sm + 3 * K;
    float* s_am = sm + 4 * K;
    float* s_acc = sm + (4 + C) * K;   // [nwarps][K][nacc]
    const bool lobe_grads = gaxis || gsharp || gamp || (!exact && gssh);
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
        float s = sharp[i];
        s_sh[i] = s;
        s_ax[3 * i] = axis[3 * i] * s; s_ax[3 * i + 1] = axis[3 * i + 1] * s; s_ax[3 * i + 2] = axis[3 * i + 2] * s;
    }
    for (int i = threadIdx.x; i < K * C; i += blockDim.x) s_am[i] = amp[i];
    if (lobe_grads)
        for (int i = threadIdx.x; i < nwarps * K * nacc; i += blockDim.x) s_acc[i] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float* wacc = s_acc + (size_t)wid * K * nacc;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long npad = (npix + 31) / 32 * 32;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npad; p += stride) {
        bool live = p < npix && rast_id(rast[p].w) >= 0;
        if (!lobe_grads && !live) continue;
        float3 n = f3(0.f, 0.f, 0.f), pax = n;
        float ss = 0.f, sa = 0.f;
        float dfs[CMAX], go[CMAX], gd[CMAX], gsa[CMAX];
        float3 gsx = f3(0.f, 0.f, 0.f);
        float gsh_p = 0.f;
#pragma unroll
        for (int k = 0; k < CMAX; ++k) { dfs[k] = 0.f; go[k] = 0.f; gd[k] = 0.f; gsa[k] = 0.f; }
        if (live) {
            n = ld3(normal, p);
            pax = ld3(sax, p);
            ss = ssh[p]; sa = sam[p];
#pragma unroll
            for (int k = 0; k < CMAX; ++k) {
                if (k >= C) break;
                dfs[k] = diffuse[p * C + k];
                go[k] = gout[p * C + k];
                if (gdiff) gd[k] = gdiff[p * C + k];
                if (gsam && !exact) gsa[k] = gsam[p * C + k];
            }
            if (gsax) gsx = ld3(gsax, p);
            if (gsam && exact) gsa[0] = gsam[p];
            if (gssh && exact) gsh_p = gssh[p];
        }
        const float3 diffn = n * DIFF_SHARP, specn = pax * ss;
        for (int i = 0; i < K; ++i) {
            float gs = s_sh[i];
            float3 sgn = f3(s_ax[3 * i], s_ax[3 * i + 1], s_ax[3 * i + 2]);
            float c_ax0 = 0.f, c_ax1 = 0.f, c_ax2 = 0.f, c_sh = 0.f, c_ssh = 0.f;
            float c_am[CMAX];
#pragma unroll
            for (int k = 0; k < CMAX; ++k) c_am[k] = 0.f;
            if (live) {
                float3 dsum = diffn + sgn;
                float dl = len3(dsum);
                float il = 1.f / fmaxf(dl, 1e-6f);
                float dotn = (gs + DIFF_SHARP * dot3(sgn, n)) * il;
                float em = expf(dl - DIFF_SHARP - gs), ep = expf(-dl - DIFF_SHARP - gs);
                float dg = (em - ep) * il * DIFF_AMP;
                float3 ddg = dsum * (((1.f - il) * em + (1.f + il) * ep) * il) * il;
                float ddgs = ((dotn * (1.f - il) - 1.f) * em + (dotn * (1.f + il) + 1.f) * ep) * il;
                float3 ssum = specn + sgn;
                float sl = len3(ssum);
                il = 1.f / fmaxf(sl, 1e-6f);
                float sdot = dot3(sgn, pax);
                dotn = (gs + ss * sdot) * il;
                float dotp = (gs * sdot + ss) * il;
                em = expf(sl - ss - gs); ep = expf(-sl - ss - gs);
                float sgv = (em - ep) * il * sa;
                float3 dsg = ssum * (((1.f - il) * em + (1.f + il) * ep) * il) * il;
                float dsgs = ((dotn * (1.f - il) - 1.f) * em + (dotn * (1.f + il) + 1.f) * ep) * il;
                float dsgss = ((dotp * (1.f - il) - 1.f) * em + (dotp * (1.f + il) + 1.f) * ep) * il;
                float sum = 0.f, sumd = 0.f, sum_sa = 0.f;
#pragma unroll
                for (int k = 0; k < CMAX; ++k) {
                    if (k >= C) break;
                    float a = s_am[i * C + k];
                    float g = go[k];
                    sum += g * a;
                    sumd += g * a * dfs[k];
                    c_am[k] = g * (dg * dfs[k] + sgv);
                    add_nan_check(gd[k], g * dg * a);
                    if (!exact) add_nan_check(gsa[k], g * sgv * a);
                    else sum_sa += g * (em - ep) * il * a;
                }
                if (exact) add_nan_check(gsa[0], sum_sa);
                float3 t = (ddg * sumd) * DIFF_AMP + (dsg * sum) * sa;
                float3 cax = t * gs;
                if (fin3(cax)) { c_ax0 = cax.x; c_ax1 = cax.y; c_ax2 = cax.z; }
                c_sh = sumd * ddgs * DIFF_AMP + sum * dsgs * sa;
                if (!isfinite(c_sh)) c_sh = 0.f;
                float3 csx = ((dsg * sum) * sa) * ss;
                add_nan_check3(&gsx.x, csx.x, csx.y, csx.z);
                float cssh = sum * dsgss * sa;
                if (exact) add_nan_check(gsh_p, cssh);
                else c_ssh = isfinite(cssh) ? cssh : 0.f;
#pragma unroll
                for (int k = 0; k < CMAX; ++k)
                    if (!isfinite(c_am[k])) c_am[k] = 0.f;
            }
            if (lobe_grads) {
                float* a = wacc + (size_t)i * nacc;
                float v;
                v = warp_sum(c_ax0); if (lane == 0) a[0] += v;
                v = warp_sum(c_ax1); if (lane == 0) a[1] += v;
                v = warp_sum(c_ax2); if (lane == 0) a[2] += v;
                v = warp_sum(c_sh); if (lane == 0) a[3] += v;
#pragma unroll
                for (int k = 0; k < CMAX; ++k) {
                    if (k >= C) break;
                    v = warp_sum(c_am[k]);
                    if (lane == 0) a[4 + k] += v;
                }
                if (!exact && gssh) { v = warp_sum(c_ssh); if (lane == 0) a[4 + C] += v; }
            }
        }
        if (live) {
#pragma unroll
            for (int k = 0; k < CMAX; ++k) {
                if (k >= C) break;
                if (gdiff) gdiff[p * C + k] = gd[k];
                if (gsam && !exact) gsam[p * C + k] = gsa[k];
            }
            if (gsax) st3(gsax, p, gsx);
            if (gsam && exact) gsam[p] = gsa[0];
            if (gssh && exact) gssh[p] = gsh_p;
        }
    }
    if (!lobe_grads) return;
    __syncthreads();
    for (int j = threadIdx.x; j < K * nacc; j += blockDim.x) {
        float v = 0.f;
        for (int w = 0; w < nwarps; ++w) v += s_acc[(size_t)w * K * nacc + j];
        if (v == 0.f) continue;
        int i = j / nacc, q = j % nacc;
        if (q < 3) { if (gaxis) atomicAdd(&gaxis[3 * i + q], v); }
        else if (q == 3) { if (gsharp) atomicAdd(&gsharp[i], v); }
        else if (q < 4 + C) { if (gamp) atomicAdd(&gamp[i * C + (q - 4)], v); }
        else if (gssh) atomicAdd(&gssh[i], v);
    }
}

size_t sg_fwd_smem(int K, int C) { return sizeof(float) * (size_t)K * (4 + C); }
size_t sg_bwd_smem(int K, int C, int nacc, int threads) {
    return sizeof(float) * ((size_t)K * (4 + C) + (size_t)(threads / 32) * K * nacc);
}

}  // namespace

extern "C" {

VCL_API vcl_status vcl_normal_axis_fwd(vcl_ctx* ctx, const float* rast, int W, int H, int views, const float* rot16,
                                       const float* normal, int nv, const uint32_t* tri, int nt, float* out,
                                       void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && rot16 && normal && tri && out && W > 0 && H > 0 && views > 0, "bad normal_axis arguments");
    long long npix = (long long)W * H * views;
    k_normal_axis<<<vcl_blocks(npix, 256), 256, 0, (cudaStream_t)stream>>>((const float4*)rast, npix, rot16, normal, nv,
                                                                           tri, nt, out, ctx->dev_flags);
    return vcl_launch_check(ctx, "normal_axis_fwd");
}

VCL_API vcl_status vcl_view_axis_fwd(vcl_ctx* ctx, int W, int H, int views, const float* pvinv, float* out,
                                     void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(pvinv && out && W > 0 && H > 0 && views > 0, "bad view_axis arguments");
    long long npix = (long long)W * H * views;
    k_view_axis<<<vcl_blocks(npix, 256), 256, 0, (cudaStream_t)stream>>>(W, H, npix, pvinv, out);
    return vcl_launch_check(ctx, "view_axis_fwd");
}

VCL_API vcl_status vcl_sg_specular_fwd(vcl_ctx* ctx, const float* rast, int W, int H, int views, const float* normal,
                                       const float* view, const float* roughness, float ior, float* out_axis,
                                       float* out_sharpness, float* out_amplitude, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && normal && view && roughness && out_axis && out_sharpness && out_amplitude && W > 0 && H > 0 &&
                    views > 0, "bad sg_specular_fwd arguments");
    long long npix = (long long)W * H * views;
    k_sg_spec_fwd<<<vcl_blocks(npix, 256), 256, 0, (cudaStream_t)stream>>>((const float4*)rast, npix, normal, view,
                                                                           roughness, ior, out_axis, out_sharpness,
                                                                           out_amplitude);
    return vcl_launch_check(ctx, "sg_specular_fwd");
}

VCL_API vcl_status vcl_sg_specular_bwd(vcl_ctx* ctx, const float* rast, int W, int H, int views, const float* normal,
                                       const float* view, const float* roughness, float ior,
                                       const float* grad_amplitude, const float* grad_sharpness, float* grad_roughness,
                                       void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && normal && view && roughness && grad_amplitude && grad_sharpness && grad_roughness && W > 0 &&
                    H > 0 && views > 0, "bad sg_specular_bwd arguments");
    long long npix = (long long)W * H * views;
    k_sg_spec_bwd<<<vcl_blocks(npix, 256), 256, 0, (cudaStream_t)stream>>>((const float4*)rast, npix, normal, view,
                                                                           roughness, ior, grad_amplitude,
                                                                           grad_sharpness, grad_roughness);
    return vcl_launch_check(ctx, "sg_specular_bwd");
}

VCL_API vcl_status vcl_sg_fwd(vcl_ctx* ctx, const float* rast, int W, int H, int views, int C, int K, const float* axis,
                              const float* sharpness, const float* amplitude, const float* normal, const float* diffuse,
                              const float* spec_axis, const float* spec_sharpness, const float* spec_amplitude,
                              float* out, float* out_diffenv, float* out_specenv, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && normal && diffuse && spec_axis && spec_sharpness && spec_amplitude && out && W > 0 && H > 0 &&
                    views > 0, "bad sg_fwd arguments");
    VCL_REQUIRE(C >= 1 && C <= CMAX, "channel count %d outside 1..%d", C, CMAX);
    VCL_REQUIRE(K >= 0 && K <= 1024 && (K == 0 || (axis && sharpness && amplitude)), "bad lobe count %d", K);
    long long npix = (long long)W * H * views;
    size_t smem = sg_fwd_smem(K, C);
    static bool attr_set = false;
    if (!attr_set) { cudaFuncSetAttribute(k_sg_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024); attr_set = true; }
    k_sg_fwd<<<vcl_blocks(npix, 256), 256, smem, (cudaStream_t)stream>>>(C, K, axis, sharpness, amplitude,
                                                                        (const float4*)rast, npix, normal, diffuse,
                                                                        spec_axis, spec_sharpness, spec_amplitude, out,
                                                                        out_diffenv, out_specenv);
    return vcl_launch_check(ctx, "sg_fwd");
}

VCL_API vcl_status vcl_sg_bwd(vcl_ctx* ctx, const float* rast, int W, int H, int views, int C, int K, const float* axis,
                              const float* sharpness, const float* amplitude, const float* normal, const float* diffuse,
                              const float* spec_axis, const float* spec_sharpness, const float* spec_amplitude,
                              const float* grad_out, float* grad_diffuse, float* grad_axis, float* grad_sharpness,
                              float* grad_amplitude, float* grad_spec_axis, float* grad_spec_sharpness,
                              float* grad_spec_amplitude, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(rast && normal && diffuse && spec_axis && spec_sharpness && spec_amplitude && grad_out && W > 0 && H > 0 &&
                    views > 0, "bad sg_bwd arguments");
    VCL_REQUIRE(C >= 1 && C <= CMAX, "channel count %d outside 1..%d", C, CMAX);
    VCL_REQUIRE(K >= 0 && K <= 1024 && (K == 0 || (axis && sharpness && amplitude)), "bad lobe count %d", K);
    long long npix = (long long)W * H * views;
    const int exact = ctx->mode == VCL_MODE_EXACT;
    const int threads = 256;
    const int nacc = 4 + C + 1;
    size_t smem = sg_bwd_smem(K, C, nacc, threads);
    VCL_REQUIRE(smem <= 200 * 1024, "too many lobes for the shared-memory reduction (K=%d)", K);
    static bool attr_set = false;
    if (!attr_set) { cudaFuncSetAttribute(k_sg_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024); attr_set = true; }
    long long blocks = (npix + threads - 1) / threads;
    long long cap = (long long)ctx->sm_count * 4;
    int grid = (int)(blocks < cap ? (blocks < 1 ? 1 : blocks) : cap);
    k_sg_bwd<<<grid, threads, smem, (cudaStream_t)stream>>>(
        C, K, nacc, axis, sharpness, amplitude, (const float4*)rast, npix, normal, diffuse, spec_axis, spec_sharpness,
        spec_amplitude, grad_out, grad_diffuse, grad_axis, grad_sharpness, grad_amplitude, grad_spec_axis,
        grad_spec_sharpness, grad_spec_amplitude, exact);
    return vcl_launch_check(ctx, "sg_bwd");
}

}  // extern "C"

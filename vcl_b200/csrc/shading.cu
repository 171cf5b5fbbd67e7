// Spherical-Gaussian shading operators (reference material.cu): NormalAxis,
// ViewAxis, SGSpecular and SphericalGaussian, forward and backward.  One
// thread per pixel; the K lobes are staged in shared memory.  The SG
// backward reduces the per-lobe gradients (axis, sharpness, amplitude) over
// all pixels: warp shuffles, then per-warp shared accumulators, then one
// atomic per block and lobe parameter -- the reference accumulates them
// with unsynchronised adds from every thread (material.cu:428-436).
#include "common.cuh"
#include "sg_math.cuh"

namespace {

constexpr int CMAX = SG_CMAX;

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

// material.cu:285-323
template <int CC>
__global__ void k_sg_fwd(int C, int K, const float* __restrict__ axis, const float* __restrict__ sharp,
                         const float* __restrict__ amp, const float4* __restrict__ rast, long long npix,
                         const float* __restrict__ normal, const float* __restrict__ diffuse, const float* __restrict__ sax,
                         const float* __restrict__ ssh, const float* __restrict__ sam, float* __restrict__ out,
                         float* __restrict__ odiff, float* __restrict__ ospec) {
    extern __shared__ float sm[];
    SGLobes L;
    if (CC == 4) sg_stage_lobes4(reinterpret_cast<float4*>(sm), K, axis, sharp, amp);
    else L = sg_stage_lobes(sm, K, C, axis, sharp, amp);
    __syncthreads();
    const int Cn = CC ? CC : C;
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    if (rast_id(rast[p].w) < 0) {
        for (int k = 0; k < Cn; ++k) {
            out[p * Cn + k] = 0.f;
            if (odiff) odiff[p * Cn + k] = 0.f;
            if (ospec) ospec[p * Cn + k] = 0.f;
        }
        return;
    }
    float de[SG_CMAX], se[SG_CMAX];
    if (CC == 4) {
        float4 d4, s4;
        sg_env4(reinterpret_cast<const float4*>(sm), K, ld3(normal, p), ld3(sax, p), ssh[p], sam[p], d4, s4);
        de[0] = d4.x; de[1] = d4.y; de[2] = d4.z; de[3] = d4.w;
        se[0] = s4.x; se[1] = s4.y; se[2] = s4.z; se[3] = s4.w;
    } else {
        sg_env<CC>(L, K, C, ld3(normal, p), ld3(sax, p), ssh[p], sam[p], de, se);
    }
#pragma unroll
    for (int k = 0; k < SG_CMAX; ++k) {
        if (k >= Cn) break;
        out[p * Cn + k] = diffuse[p * Cn + k] * de[k] + se[k];
        if (odiff) odiff[p * Cn + k] = de[k];
        if (ospec) ospec[p * Cn + k] = se[k];
    }
}

constexpr int SGB_P = 2;

template <int CC>
__global__ void __launch_bounds__(256) k_sg_bwd(int C, int K, int nacc, const float* __restrict__ axis,
                                                const float* __restrict__ sharp, const float* __restrict__ amp,
                                                const float4* __restrict__ rast, long long npix,
                                                const float* __restrict__ normal, const float* __restrict__ diffuse,
                                                const float* __restrict__ sax, const float* __restrict__ ssh,
                                                const float* __restrict__ sam, const float* __restrict__ gout,
                                                float* __restrict__ gdiff, float* __restrict__ gaxis,
                                                float* __restrict__ gsharp, float* __restrict__ gamp,
                                                float* __restrict__ gsax, float* __restrict__ gssh,
                                                float* __restrict__ gsam, int exact) {
    extern __shared__ float sm[];
    const int nwarps = blockDim.x >> 5;
    const int Cn = CC ? CC : C;
    const SGLobes L = sg_stage_lobes(sm, K, C, axis, sharp, amp);
    float* s_acc = sm + (4 + C) * K;
    const bool lobe_grads = gaxis || gsharp || gamp || (!exact && gssh);
    if (lobe_grads)
        for (int i = threadIdx.x; i < nwarps * K * nacc; i += blockDim.x) s_acc[i] = 0.f;
    __syncthreads();
    float* wacc = s_acc + (size_t)(threadIdx.x >> 5) * K * nacc;
    const long long span = (long long)blockDim.x * SGB_P;
    for (long long base = (long long)blockIdx.x * span; base < npix; base += (long long)gridDim.x * span) {
        SGPix q[SGB_P];
        bool live[SGB_P];
        bool any = false;
#pragma unroll
        for (int j = 0; j < SGB_P; ++j) {
            long long p = base + threadIdx.x + (long long)j * blockDim.x;
            live[j] = p < npix && rast_id(rast[p].w) >= 0;
            any |= live[j];
            SGPix& z = q[j];
            z.gsx = f3(0.f, 0.f, 0.f); z.gsh = 0.f;
#pragma unroll
            for (int k = 0; k < SG_CMAX; ++k) { z.dfs[k] = 0.f; z.go[k] = 0.f; z.gd[k] = 0.f; z.gsa[k] = 0.f; }
            if (live[j]) {
                z.n = ld3(normal, p); z.pax = ld3(sax, p); z.ss = ssh[p]; z.sa = sam[p];
                for (int k = 0; k < Cn; ++k) {
                    z.dfs[k] = diffuse[p * Cn + k];
                    z.go[k] = gout[p * Cn + k];
                    if (gdiff) z.gd[k] = gdiff[p * Cn + k];
                    if (gsam && !exact) z.gsa[k] = gsam[p * Cn + k];
                }
                if (gsax) z.gsx = ld3(gsax, p);
                if (gsam && exact) z.gsa[0] = gsam[p];
                if (gssh && exact) z.gsh = gssh[p];
            } else {
                z.n = z.pax = f3(0.f, 0.f, 0.f); z.ss = z.sa = 0.f;
            }
        }
        if (!__any_sync(0xffffffffu, any)) continue;
        sg_bwd_block<SGB_P, CC>(L, K, C, exact, q, live, wacc, nacc, lobe_grads, !exact && gssh);
#pragma unroll
        for (int j = 0; j < SGB_P; ++j) {
            if (!live[j]) continue;
            long long p = base + threadIdx.x + (long long)j * blockDim.x;
            for (int k = 0; k < Cn; ++k) {
                if (gdiff) gdiff[p * Cn + k] = q[j].gd[k];
                if (gsam && !exact) gsam[p * Cn + k] = q[j].gsa[k];
            }
            if (gsax) st3(gsax, p, q[j].gsx);
            if (gsam && exact) gsam[p] = q[j].gsa[0];
            if (gssh && exact) gssh[p] = q[j].gsh;
        }
    }
    if (!lobe_grads) return;
    __syncthreads();
    sg_flush_lobes(s_acc, nwarps, K, C, nacc, gaxis, gsharp, gamp, exact ? nullptr : gssh);
}

// Lobe-parallel SG backward (see sg_bwd_lanes): one lobe per lane, pixels
// staged per warp in shared memory, per-lobe sums in registers.
template <int NL, int CC>
__global__ void __launch_bounds__(128) k_sg_bwd_lp(int C, int K, int Kp, int nacc, const float* __restrict__ axis,
                                                   const float* __restrict__ sharp, const float* __restrict__ amp,
                                                   const float4* __restrict__ rast, long long npix,
                                                   const float* __restrict__ normal, const float* __restrict__ diffuse,
                                                   const float* __restrict__ sax, const float* __restrict__ ssh,
                                                   const float* __restrict__ sam, const float* __restrict__ gout,
                                                   float* __restrict__ gdiff, float* __restrict__ gaxis,
                                                   float* __restrict__ gsharp, float* __restrict__ gamp,
                                                   float* __restrict__ gsax, float* __restrict__ gssh,
                                                   float* __restrict__ gsam, int exact) {
    extern __shared__ float sm[];
    const int nwarps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int Cn = CC ? CC : C;
    float* s_acc = sm;                                            // [K][nacc]
    float* s_lob = sm + (size_t)K * nacc;                         // lobes for the guarded fallback
    SPix* s_pix = reinterpret_cast<SPix*>(s_lob + (size_t)K * (4 + C));
    SPixOut* s_out = reinterpret_cast<SPixOut*>(s_pix + nwarps * 32);
    for (int i = threadIdx.x; i < K * nacc; i += blockDim.x) s_acc[i] = 0.f;
    const SGLobes L = sg_stage_lobes(s_lob, K, C, axis, sharp, amp);
    __syncthreads();
    const int G = 32 / Kp, g = lane / Kp, li = lane % Kp;
    LaneLobes<NL, CC> LL;
    lane_lobes_load<NL, CC>(LL, li, Kp, K, C, axis, sharp, amp);
    const bool pix_out = gdiff || gsax || gssh || gsam;
    SPix* st = s_pix + wid * 32;
    SPixOut* so = s_out + wid * 32;
    const long long nchunks = (npix + 31) / 32;
    for (long long chunk = (long long)blockIdx.x * nwarps + wid; chunk < nchunks; chunk += (long long)gridDim.x * nwarps) {
        const long long p = chunk * 32 + lane;
        const bool live = p < npix && rast_id(rast[p].w) >= 0;
        const unsigned ball = __ballot_sync(0xffffffffu, live);
        const int m = __popc(ball);
        const int slot = __popc(ball & ((1u << lane) - 1u));
        if (live) {
            SPix& z = st[slot];
            float3 n = ld3(normal, p), pa = ld3(sax, p);
            z.n[0] = n.x; z.n[1] = n.y; z.n[2] = n.z;
            z.pax[0] = pa.x; z.pax[1] = pa.y; z.pax[2] = pa.z;
            z.ss = ssh[p]; z.sa = sam[p];
            for (int k = 0; k < Cn; ++k) { z.dfs[k] = diffuse[p * Cn + k]; z.go[k] = gout[p * Cn + k]; }
        }
        __syncwarp();
        if (m > 0) {
            if (pix_out) sg_bwd_lanes<NL, CC, true>(LL, C, exact, st, so, m, Kp, g, G, li);
            else sg_bwd_lanes<NL, CC, false>(LL, C, exact, st, so, m, Kp, g, G, li);
        }
        __syncwarp();
        if (pix_out && live) {
            const SPixOut& o = so[slot];
            const SPix& z = st[slot];
            float gd0[SG_CMAX], gsa0[SG_CMAX], gd[SG_CMAX], gsa[SG_CMAX];
            float3 gsx0 = gsax ? ld3(gsax, p) : f3(0.f, 0.f, 0.f);
            float gsh0 = (gssh && exact) ? gssh[p] : 0.f;
            bool ok = true;
            for (int k = 0; k < Cn; ++k) {
                gd0[k] = gdiff ? gdiff[p * Cn + k] : 0.f;
                gsa0[k] = (gsam && !exact) ? gsam[p * Cn + k] : 0.f;
                gd[k] = gd0[k] + o.gd[k];
                gsa[k] = gsa0[k] + o.gsa[k];
                ok = ok && isfinite(o.gd[k]) && isfinite(gd[k]) && isfinite(o.gsa[k]) && isfinite(gsa[k]);
            }
            if (gsam && exact) { gsa0[0] = gsam[p]; gsa[0] = gsa0[0] + o.gsa[0]; ok = ok && isfinite(gsa[0]); }
            float3 gsx = gsx0 + f3(o.gsx[0], o.gsx[1], o.gsx[2]);
            float gsh = gsh0 + o.gsh;
            ok = ok && fin3(gsx) && isfinite(gsh);
            if (!ok) {
                // some partial sum left the finite range: redo this pixel in the
                // reference's guarded order
                SGPix q;
                q.n = f3(z.n[0], z.n[1], z.n[2]); q.pax = f3(z.pax[0], z.pax[1], z.pax[2]);
                q.ss = z.ss; q.sa = z.sa;
                for (int k = 0; k < SG_CMAX; ++k) { q.dfs[k] = k < Cn ? z.dfs[k] : 0.f; q.go[k] = k < Cn ? z.go[k] : 0.f; }
                sg_bwd_pixel_slow<CC>(L, K, C, exact, q, gd0, gsa0, gsx0, gsh0);
                for (int k = 0; k < Cn; ++k) { gd[k] = q.gd[k]; gsa[k] = q.gsa[k]; }
                gsx = q.gsx; gsh = q.gsh;
            }
            for (int k = 0; k < Cn; ++k) {
                if (gdiff) gdiff[p * Cn + k] = gd[k];
                if (gsam && !exact) gsam[p * Cn + k] = gsa[k];
            }
            if (gsax) st3(gsax, p, gsx);
            if (gsam && exact) gsam[p] = gsa[0];
            if (gssh && exact) gssh[p] = gsh;
        }
        __syncwarp();
    }
    lane_lobes_flush<NL, CC>(LL, C, Kp, li, s_acc, nacc, !exact && gssh);
    __syncthreads();
    sg_flush_block(s_acc, K, C, nacc, gaxis, gsharp, gamp, exact ? nullptr : gssh);
}

// SphericalGaussian::backward for C = 4 when only the diffuse and lobe
// gradients are asked for (material.cu:369-438 without the specular-lobe
// outputs).  The diffuse gradient is grad_out * sum_k dg_k amp_k, i.e.
// grad_out times the forward's diffuse environment sum (sg_env4, two lobes
// per paired instruction, with its guarded fallback); a term that is not
// finite is dropped as the reference's guarded add drops it.
__global__ void __launch_bounds__(256) k_sg_bwd_diffuse4(int K, const float* __restrict__ axis,
                                                         const float* __restrict__ sharp, const float* __restrict__ amp,
                                                         const float4* __restrict__ rast, long long npix,
                                                         const float* __restrict__ normal, const float* __restrict__ sax,
                                                         const float* __restrict__ ssh, const float* __restrict__ sam,
                                                         const float4* __restrict__ gout, float4* __restrict__ gdiff) {
    extern __shared__ float4 sm4[];
    sg_stage_lobes4(sm4, K, axis, sharp, amp);
    __syncthreads();
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix || rast_id(rast[p].w) < 0) return;
    float4 de, se;
    sg_env4(sm4, K, ld3(normal, p), ld3(sax, p), ssh[p], sam[p], de, se);
    const float4 g = gout[p];
    float4 d = gdiff[p];
    add_nan_check(d.x, g.x * de.x); add_nan_check(d.y, g.y * de.y);
    add_nan_check(d.z, g.z * de.z); add_nan_check(d.w, g.w * de.w);
    gdiff[p] = d;
}

// Lobe gradients of SphericalGaussian::backward for C = 4 from the operator's
// per-pixel inputs: the fused step's lobe-gradient kernel (lobe per lane, two
// pixels per paired instruction, 32 lobes per block row) with each warp
// compacting the covered pixels of its 32-pixel chunk itself.
template <bool EXACT>
__global__ void __launch_bounds__(128, 4) k_sg_lobes_op(int K, const float* __restrict__ axis,
                                                        const float* __restrict__ sharp, const float* __restrict__ amp,
                                                        const float4* __restrict__ rast, long long npix,
                                                        const float* __restrict__ normal,
                                                        const float4* __restrict__ diffuse,
                                                        const float* __restrict__ sax, const float* __restrict__ ssh,
                                                        const float* __restrict__ sam, const float4* __restrict__ gout,
                                                        float* __restrict__ g_axis, float* __restrict__ g_sharp,
                                                        float* __restrict__ g_amp) {
    __shared__ float s_acc[32 * 8];
    __shared__ SPair s_pix[4 * 16];
    const int nwarps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int base = 32 * blockIdx.y, Kg = min(32, K - base);
    for (int i = threadIdx.x; i < 32 * 8; i += blockDim.x) s_acc[i] = 0.f;
    __syncthreads();
    const int Kp = sg_lobe_group_dev(Kg);
    const int G = 32 / Kp, g = lane / Kp, li = lane % Kp;
    Lobe4x2 L;
    lobe4x2_load(L, li, Kg, axis + 3 * base, sharp + base, amp + 4 * base);
    SPair* st = s_pix + wid * 16;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const long long nchunks = (npix + 31) / 32;
    // Plain pass, then a checked pass for lanes whose sums are not finite
    // (as in the fused step's lobe-gradient kernel).
    bool guard = false;
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        for (long long c = (long long)blockIdx.x * nwarps + wid; c < nchunks; c += (long long)gridDim.x * nwarps) {
            const long long p = c * 32 + lane;
            const bool live = p < npix && rast_id(rast[p].w) >= 0;
            const unsigned ball = __ballot_sync(0xffffffffu, live);
            const int m = __popc(ball);
            if (m == 0) continue;
            if (live) {
                const int k = __popc(ball & ((1u << lane) - 1u));
                const float3 n = ld3(normal, p), pa = ld3(sax, p);
                spair_put(st + (k >> 1), k & 1, make_float4(n.x, n.y, n.z, ssh[p]),
                          make_float4(pa.x, pa.y, pa.z, sam[p]), diffuse[p], gout[p]);
            }
            if ((m & 1) && lane == 31) spair_put(st + (m >> 1), 1, z4, z4, z4, z4);
            __syncwarp();
            const int npair = (m + 1) >> 1;
            if (L.valid && (pass == 0 || guard))
                for (int j = g; j < npair; j += G) lobe4x2_accumulate<EXACT>(L, st[j], pass != 0);
            __syncwarp();
        }
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
        if (q < 3) { if (g_axis) atomicAdd(&g_axis[3 * i + q], v); }
        else if (q == 3) { if (g_sharp) atomicAdd(&g_sharp[i], v); }
        else if (g_amp) atomicAdd(&g_amp[4 * i + (q - 4)], v);
    }
}

size_t sg_bwd_lp_smem(int K, int C, int nacc, int threads) {
    return sizeof(float) * ((size_t)K * nacc + (size_t)K * (4 + C)) +
           (size_t)(threads / 32) * 32 * (sizeof(SPix) + sizeof(SPixOut));
}

size_t sg_fwd_smem(int K, int C) { return C == 4 ? sg_lobes4_smem(K) : sizeof(float) * (size_t)K * (4 + C); }
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
    auto kern = C == 4 ? k_sg_fwd<4> : k_sg_fwd<0>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<vcl_blocks(npix, 256), 256, smem, (cudaStream_t)stream>>>(C, K, axis, sharpness, amplitude,
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
    VCL_REQUIRE(C == 4 || C <= CMAX, "channel count");
    const bool pix_out = grad_diffuse || grad_spec_axis || grad_spec_sharpness || grad_spec_amplitude;
    const bool spec_out = grad_spec_axis || grad_spec_sharpness || grad_spec_amplitude;
    const bool lobe_out = grad_axis || grad_sharpness || grad_amplitude;
    auto al16 = [](const void* q) { return ((uintptr_t)q & 15) == 0; };
    if (C == 4 && K > 0 && !spec_out && al16(diffuse) && al16(grad_out) && al16(rast) &&
        (!grad_diffuse || al16(grad_diffuse))) {
        // diffuse gradient pixel-parallel, lobe gradients lobe-parallel: no
        // cross-lane sums per pixel and no per-lobe block sums per chunk
        cudaStream_t st = (cudaStream_t)stream;
        if (grad_diffuse) {
            const size_t dsm = sg_lobes4_smem(K);
            if (dsm > 48 * 1024) cudaFuncSetAttribute(k_sg_bwd_diffuse4, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
            k_sg_bwd_diffuse4<<<vcl_blocks(npix, 256), 256, dsm, st>>>(K, axis, sharpness, amplitude, (const float4*)rast,
                                                                      npix, normal, spec_axis, spec_sharpness,
                                                                      spec_amplitude, (const float4*)grad_out,
                                                                      (float4*)grad_diffuse);
        }
        if (lobe_out) {
            const int groups = (K + 31) / 32;
            long long want = ((npix + 31) / 32 + 3) / 4;
            long long cap = ((long long)ctx->sm_count * 4 + groups - 1) / groups;
            const dim3 grid((unsigned)(want < cap ? (want < 1 ? 1 : want) : cap), (unsigned)groups);
            auto lk = exact ? k_sg_lobes_op<true> : k_sg_lobes_op<false>;
            lk<<<grid, 128, 0, st>>>(K, axis, sharpness, amplitude, (const float4*)rast, npix, normal,
                                     (const float4*)diffuse, spec_axis, spec_sharpness, spec_amplitude,
                                     (const float4*)grad_out, grad_axis, grad_sharpness, grad_amplitude);
        }
        return vcl_launch_check(ctx, "sg_bwd");
    }
    if (K <= 128 && !pix_out) {
        const int Kp = sg_lobe_group(K > 0 ? K : 1);
        const int NL = (K + 31) / 32;
        const int lthreads = 128;
        size_t lsmem = sg_bwd_lp_smem(K, C, nacc, lthreads);
        decltype(&k_sg_bwd_lp<1, 4>) lk;
        if (C == 4) lk = NL <= 1 ? k_sg_bwd_lp<1, 4> : NL <= 2 ? k_sg_bwd_lp<2, 4> : k_sg_bwd_lp<4, 4>;
        else lk = NL <= 1 ? k_sg_bwd_lp<1, 0> : NL <= 2 ? k_sg_bwd_lp<2, 0> : k_sg_bwd_lp<4, 0>;
        if (lsmem > 48 * 1024) cudaFuncSetAttribute(lk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem);
        long long chunks = (npix + 31) / 32;
        long long want = (chunks + lthreads / 32 - 1) / (lthreads / 32);
        long long cap = (long long)ctx->sm_count * 8;
        int lgrid = (int)(want < cap ? (want < 1 ? 1 : want) : cap);
        lk<<<lgrid, lthreads, lsmem, (cudaStream_t)stream>>>(
            C, K, Kp, nacc, axis, sharpness, amplitude, (const float4*)rast, npix, normal, diffuse, spec_axis,
            spec_sharpness, spec_amplitude, grad_out, grad_diffuse, grad_axis, grad_sharpness, grad_amplitude,
            grad_spec_axis, grad_spec_sharpness, grad_spec_amplitude, exact);
        return vcl_launch_check(ctx, "sg_bwd");
    }
    auto kern = C == 4 ? k_sg_bwd<4> : k_sg_bwd<0>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    long long blocks = (npix + threads * SGB_P - 1) / (threads * SGB_P);
    long long cap = (long long)ctx->sm_count * 4;
    int grid = (int)(blocks < cap ? (blocks < 1 ? 1 : blocks) : cap);
    kern<<<grid, threads, smem, (cudaStream_t)stream>>>(
        C, K, nacc, axis, sharpness, amplitude, (const float4*)rast, npix, normal, diffuse, spec_axis, spec_sharpness,
        spec_amplitude, grad_out, grad_diffuse, grad_axis, grad_sharpness, grad_amplitude, grad_spec_axis,
        grad_spec_sharpness, grad_spec_amplitude, exact);
    return vcl_launch_check(ctx, "sg_bwd");
}

}  // extern "C"

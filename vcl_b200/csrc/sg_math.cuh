// Spherical-Gaussian lobe arithmetic shared by the per-operator kernels and
// the fused fit kernels (reference material.cu:285-323 forward, :369-438
// backward).
//
// Per (pixel, lobe) the reference evaluates the SG inner product of the
// pixel's diffuse lobe (axis n, sharpness 2.133, amplitude 2.34) and of its
// specular lobe (axis p, sharpness ss, amplitude sa) with an environment
// lobe (axis a_k, sharpness s_k):
//     l = |lambda1 mu1 + lambda2 mu2|,
//     term = (e^(l - lambda1 - lambda2) - e^(-l - lambda1 - lambda2)) / max(l, 1e-6) * amp.
// Here 1/l comes from one reciprocal square root of |.|^2 (and l = |.|^2 / l),
// so a lobe costs two rsqrt and four exp instead of two sqrt, two
// divisions and four exp.  The exponentials use the hardware ex2 path
// (__expf): its relative error grows with |argument|, and the terms with a
// large |argument| are the ones e^(...) makes negligible, so the lobe sums
// keep FP32 accuracy.
#pragma once
#include "common.cuh"

constexpr float SG_DIFF_SHARP = 2.133f;
constexpr float SG_DIFF_AMP = 2.34f;
constexpr int SG_CMAX = 8;

// Hardware reciprocal square root of a normal, positive x (the flush-to-zero
// form: the same result as rsqrtf for such x, without the subnormal path).
DEV float rsqrt_normal(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// 1/max(|v|, 1e-6) and |v| from |v|^2.
DEV void sg_len(float d2, float& l, float& il) {
    il = rsqrt_normal(fmaxf(d2, 1e-12f));
    l = d2 * il;
}

// Forward terms of one lobe for one pixel: diffuse-lobe and specular-lobe
// SG inner products (without the environment amplitude).
DEV void sg_terms(float3 dn, float3 sn, float3 g, float gs, float ss, float sa, float& dg, float& sg) {
    float3 d = dn + g;
    float l, il;
    sg_len(dot3(d, d), l, il);
    dg = (__expf(l - SG_DIFF_SHARP - gs) - __expf(-l - SG_DIFF_SHARP - gs)) * il * SG_DIFF_AMP;
    float3 s = sn + g;
    sg_len(dot3(s, s), l, il);
    sg = (__expf(l - ss - gs) - __expf(-l - ss - gs)) * il * sa;
}

// Backward terms of one lobe (material.cu:398-418).  The sharpness
// derivatives need d|v|/ds for v = c*u + s*a (c*u the pixel's diffuse or
// specular vector, a the lobe axis): (a.v)/|v|.  The reference computes
// (s + c*(s*a).u)/|v| (material.cu:405,413-414), which equals it only for
// |a| = 1 and s = 1; COMPAT keeps that, EXACT uses (a.v)/|v| and, for the
// specular sharpness, (u.v)/|v|.  `ax` is the raw lobe axis (EXACT only).
struct SGB {
    float dg, sgv, ddgs, dsgs, dsgss, sil_e;   // sil_e = (e- - e+) / max(l,1e-6) of the specular term
    float3 ddg, dsg;
};

DEV SGB sg_bwd_terms(float3 n, float3 dn, float3 pax, float3 sn, float3 sgn, float gs, float ss, float sa,
                     bool exact, float3 ax) {
    SGB r;
    float3 dsum = dn + sgn;
    float dl, il;
    sg_len(dot3(dsum, dsum), dl, il);
    float dotn = exact ? dot3(ax, dsum) * il : (gs + SG_DIFF_SHARP * dot3(sgn, n)) * il;
    float em = __expf(dl - SG_DIFF_SHARP - gs), ep = __expf(-dl - SG_DIFF_SHARP - gs);
    r.dg = (em - ep) * il * SG_DIFF_AMP;
    r.ddg = dsum * (((1.f - il) * em + (1.f + il) * ep) * il * il);
    r.ddgs = ((dotn * (1.f - il) - 1.f) * em + (dotn * (1.f + il) + 1.f) * ep) * il;
    float3 ssum = sn + sgn;
    float sl;
    sg_len(dot3(ssum, ssum), sl, il);
    float sdot = dot3(sgn, pax);
    dotn = exact ? dot3(ax, ssum) * il : (gs + ss * sdot) * il;
    float dotp = exact ? dot3(pax, ssum) * il : (gs * sdot + ss) * il;
    em = __expf(sl - ss - gs); ep = __expf(-sl - ss - gs);
    r.sil_e = (em - ep) * il;
    r.sgv = r.sil_e * sa;
    r.dsg = ssum * (((1.f - il) * em + (1.f + il) * ep) * il * il);
    r.dsgs = ((dotn * (1.f - il) - 1.f) * em + (dotn * (1.f + il) + 1.f) * ep) * il;
    r.dsgss = ((dotp * (1.f - il) - 1.f) * em + (dotp * (1.f + il) + 1.f) * ep) * il;
    return r;
}


// The terms the lobe gradients need (no specular-lobe derivatives).
struct SGL {
    float dg, sgv, ddgs, dsgs;
    float3 ddg, dsg;
};

DEV SGL sg_lobe_terms(float3 n, float3 dn, float3 pax, float3 sn, float3 sgn, float gs, float ss, float sa,
                      bool exact, float3 ax) {
    SGL r;
    float3 dsum = dn + sgn;
    float dl, il;
    sg_len(dot3(dsum, dsum), dl, il);
    float dotn = exact ? dot3(ax, dsum) * il : (gs + SG_DIFF_SHARP * dot3(sgn, n)) * il;
    float em = __expf(dl - SG_DIFF_SHARP - gs), ep = __expf(-dl - SG_DIFF_SHARP - gs);
    r.dg = (em - ep) * il * SG_DIFF_AMP;
    float ilm = 1.f - il, ilp = 1.f + il;
    r.ddg = dsum * ((ilm * em + ilp * ep) * il * il);
    r.ddgs = ((dotn * ilm - 1.f) * em + (dotn * ilp + 1.f) * ep) * il;
    float3 ssum = sn + sgn;
    float sl;
    sg_len(dot3(ssum, ssum), sl, il);
    dotn = exact ? dot3(ax, ssum) * il : (gs + ss * dot3(sgn, pax)) * il;
    em = __expf(sl - ss - gs); ep = __expf(-sl - ss - gs);
    r.sgv = (em - ep) * il * sa;
    ilm = 1.f - il; ilp = 1.f + il;
    r.dsg = ssum * ((ilm * em + ilp * ep) * il * il);
    r.dsgs = ((dotn * ilm - 1.f) * em + (dotn * ilp + 1.f) * ep) * il;
    return r;
}

DEV float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

DEV bool fin3(float3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }
DEV float finite_or0(float v) { return isfinite(v) ? v : 0.f; }

// Lobes staged in shared memory: axis pre-multiplied by sharpness; the raw
// axis stays in global memory (read only by the EXACT sharpness derivative).
struct SGLobes {
    const float* ax;   // [K][3] axis * sharpness
    const float* sh;   // [K]
    const float* am;   // [K][C]
    const float* raw;  // [K][3] axis (global)
};

DEV SGLobes sg_stage_lobes(float* sm, int K, int C, const float* axis, const float* sharp, const float* amp) {
    float* s_ax = sm;
    float* s_sh = sm + 3 * K;
    float* s_am = sm + 4 * K;
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
        float s = sharp[i];
        s_sh[i] = s;
        s_ax[3 * i] = axis[3 * i] * s; s_ax[3 * i + 1] = axis[3 * i + 1] * s; s_ax[3 * i + 2] = axis[3 * i + 2] * s;
    }
    for (int i = threadIdx.x; i < K * C; i += blockDim.x) s_am[i] = amp[i];
    return SGLobes{s_ax, s_sh, s_am, axis};
}

// Diffuse and specular environment sums of one pixel with the reference's
// NaN-guarded accumulation (common.h:181): plain sums when they end finite
// (then no partial sum was non-finite and every guarded add was a plain
// add), else the guarded sequential loop.
template <int CC>
DEV void sg_env(const SGLobes& L, int K, int C, float3 n, float3 pax, float ss, float sa, float* de, float* se) {
    const int Cn = CC ? CC : C;
    const float3 dn = n * SG_DIFF_SHARP, sn = pax * ss;
#pragma unroll
    for (int k = 0; k < SG_CMAX; ++k) { de[k] = 0.f; se[k] = 0.f; }
    for (int i = 0; i < K; ++i) {
        float dg, sg;
        sg_terms(dn, sn, f3(L.ax[3 * i], L.ax[3 * i + 1], L.ax[3 * i + 2]), L.sh[i], ss, sa, dg, sg);
#pragma unroll
        for (int k = 0; k < SG_CMAX; ++k) {
            if (k >= Cn) break;
            float a = L.am[i * C + k];
            de[k] += dg * a;
            se[k] += sg * a;
        }
    }
    bool ok = true;
#pragma unroll
    for (int k = 0; k < SG_CMAX; ++k)
        if (k < Cn) ok = ok && isfinite(de[k]) && isfinite(se[k]);
    if (ok) return;
#pragma unroll
    for (int k = 0; k < SG_CMAX; ++k) { de[k] = 0.f; se[k] = 0.f; }
    for (int i = 0; i < K; ++i) {
        float dg, sg;
        sg_terms(dn, sn, f3(L.ax[3 * i], L.ax[3 * i + 1], L.ax[3 * i + 2]), L.sh[i], ss, sa, dg, sg);
        for (int k = 0; k < Cn; ++k) {
            float a = L.am[i * C + k];
            add_nan_check(de[k], dg * a);
            add_nan_check(se[k], sg * a);
        }
    }
}

// Specular lobe of a pixel (material.cu:155-178 / :213-240).
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


// Per-pixel state of the SG backward.
struct SGPix {
    float3 n, pax, gsx;
    float ss, sa, gsh;
    float dfs[SG_CMAX], go[SG_CMAX], gd[SG_CMAX], gsa[SG_CMAX];
};

// The guarded (reference-order) per-pixel accumulation, used only when the
// plain sums of a pixel end non-finite.
template <int CC>
DEV void sg_bwd_pixel_slow(const SGLobes& L, int K, int C, int exact, SGPix& q, const float* gd0, const float* gsa0,
                           float3 gsx0, float gsh0) {
    const int Cn = CC ? CC : C;
    for (int k = 0; k < Cn; ++k) { q.gd[k] = gd0[k]; q.gsa[k] = gsa0[k]; }
    float gsx[3] = {gsx0.x, gsx0.y, gsx0.z};
    q.gsh = gsh0;
    const float3 dn = q.n * SG_DIFF_SHARP, sn = q.pax * q.ss;
    for (int i = 0; i < K; ++i) {
        float gs = L.sh[i];
        float3 sgn = f3(L.ax[3 * i], L.ax[3 * i + 1], L.ax[3 * i + 2]);
        const float3 ax = exact ? f3(L.raw[3 * i], L.raw[3 * i + 1], L.raw[3 * i + 2]) : f3(0.f, 0.f, 0.f);
        SGB t = sg_bwd_terms(q.n, dn, q.pax, sn, sgn, gs, q.ss, q.sa, exact, ax);
        float sum = 0.f, sum_sa = 0.f;
        for (int k = 0; k < Cn; ++k) {
            float a = L.am[i * C + k], g = q.go[k];
            sum += g * a;
            add_nan_check(q.gd[k], g * t.dg * a);
            if (!exact) add_nan_check(q.gsa[k], g * t.sgv * a);
            else sum_sa += g * t.sil_e * a;
        }
        if (exact) add_nan_check(q.gsa[0], sum_sa);
        float3 csx = ((t.dsg * sum) * q.sa) * q.ss;
        add_nan_check3(gsx, csx.x, csx.y, csx.z);
        if (exact) add_nan_check(q.gsh, sum * t.dsgss * q.sa);
    }
    q.gsx = f3(gsx[0], gsx[1], gsx[2]);
}

// SG backward of P pixels per thread (material.cu:369-438).  Lobe
// gradients are summed over the thread's P pixels, then over the warp
// (shuffles), into the warp's shared accumulators `wacc` [K][nacc]:
// axis xyz, sharpness, amplitude[C], then (compat) the lobe-indexed
// specular sharpness.  Per-pixel gradients stay in `q`.
template <int P, int CC>
DEV void sg_bwd_block(const SGLobes& L, int K, int C, int exact, SGPix (&q)[P], const bool (&live)[P], float* wacc,
                      int nacc, bool lobe_grads, bool ssh_lobe) {
    const int Cn = CC ? CC : C;
    const int lane = threadIdx.x & 31;
    float gd0[P][SG_CMAX], gsa0[P][SG_CMAX], gsh0[P];
    float3 gsx0[P], dn[P], sn[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
#pragma unroll
        for (int k = 0; k < SG_CMAX; ++k) { gd0[j][k] = q[j].gd[k]; gsa0[j][k] = q[j].gsa[k]; }
        gsh0[j] = q[j].gsh;
        gsx0[j] = q[j].gsx;
        dn[j] = q[j].n * SG_DIFF_SHARP;
        sn[j] = q[j].pax * q[j].ss;
    }
    for (int i = 0; i < K; ++i) {
        const float gs = L.sh[i];
        const float3 sgn = f3(L.ax[3 * i], L.ax[3 * i + 1], L.ax[3 * i + 2]);
        const float3 ax = exact ? f3(L.raw[3 * i], L.raw[3 * i + 1], L.raw[3 * i + 2]) : f3(0.f, 0.f, 0.f);
        float c_ax0 = 0.f, c_ax1 = 0.f, c_ax2 = 0.f, c_sh = 0.f, c_ssh = 0.f;
        float c_am[SG_CMAX];
#pragma unroll
        for (int k = 0; k < SG_CMAX; ++k) c_am[k] = 0.f;
#pragma unroll
        for (int j = 0; j < P; ++j) {
            if (!live[j]) continue;
            SGB t = sg_bwd_terms(q[j].n, dn[j], q[j].pax, sn[j], sgn, gs, q[j].ss, q[j].sa, exact, ax);
            float sum = 0.f, sumd = 0.f, sum_sa = 0.f;
#pragma unroll
            for (int k = 0; k < SG_CMAX; ++k) {
                if (k >= Cn) break;
                float a = L.am[i * C + k];
                float g = q[j].go[k];
                sum += g * a;
                sumd += g * a * q[j].dfs[k];
                c_am[k] += finite_or0(g * (t.dg * q[j].dfs[k] + t.sgv));
                q[j].gd[k] += g * t.dg * a;
                if (!exact) q[j].gsa[k] += g * t.sgv * a;
                else sum_sa += g * t.sil_e * a;
            }
            if (exact) q[j].gsa[0] += sum_sa;
            float3 cax = ((t.ddg * sumd) * SG_DIFF_AMP + (t.dsg * sum) * q[j].sa) * gs;
            if (fin3(cax)) { c_ax0 += cax.x; c_ax1 += cax.y; c_ax2 += cax.z; }
            c_sh += finite_or0(sumd * t.ddgs * SG_DIFF_AMP + sum * t.dsgs * q[j].sa);
            q[j].gsx = q[j].gsx + ((t.dsg * sum) * q[j].sa) * q[j].ss;
            float cssh = sum * t.dsgss * q[j].sa;
            if (exact) q[j].gsh += cssh;
            else c_ssh += finite_or0(cssh);
        }
        if (lobe_grads) {
            float* a = wacc + (size_t)i * nacc;
            float v;
            v = warp_sum(c_ax0); if (lane == 0) a[0] += v;
            v = warp_sum(c_ax1); if (lane == 0) a[1] += v;
            v = warp_sum(c_ax2); if (lane == 0) a[2] += v;
            v = warp_sum(c_sh); if (lane == 0) a[3] += v;
#pragma unroll
            for (int k = 0; k < SG_CMAX; ++k) {
                if (k >= Cn) break;
                v = warp_sum(c_am[k]);
                if (lane == 0) a[4 + k] += v;
            }
            if (ssh_lobe) { v = warp_sum(c_ssh); if (lane == 0) a[4 + Cn] += v; }
        }
    }
    // per-pixel sums that did not end finite: redo them in reference order
#pragma unroll
    for (int j = 0; j < P; ++j) {
        if (!live[j]) continue;
        bool ok = fin3(q[j].gsx) && isfinite(q[j].gsh);
        for (int k = 0; k < Cn; ++k) ok = ok && isfinite(q[j].gd[k]) && isfinite(q[j].gsa[k]);
        if (!ok) sg_bwd_pixel_slow<CC>(L, K, C, exact, q[j], gd0[j], gsa0[j], gsx0[j], gsh0[j]);
    }
}

// Flushes the per-warp accumulators of a block to the global lobe gradients.
DEV void sg_flush_lobes(const float* s_acc, int nwarps, int K, int C, int nacc, float* gaxis, float* gsharp, float* gamp,
                        float* gssh_lobe) {
    for (int j = threadIdx.x; j < K * nacc; j += blockDim.x) {
        float v = 0.f;
        for (int w = 0; w < nwarps; ++w) v += s_acc[(size_t)w * K * nacc + j];
        if (v == 0.f) continue;
        int i = j / nacc, q = j % nacc;
        if (q < 3) { if (gaxis) atomicAdd(&gaxis[3 * i + q], v); }
        else if (q == 3) { if (gsharp) atomicAdd(&gsharp[i], v); }
        else if (q < 4 + C) { if (gamp) atomicAdd(&gamp[i * C + (q - 4)], v); }
        else if (gssh_lobe) atomicAdd(&gssh_lobe[i], v);
    }
}


// ---------------------------------------------------------------------------
// Lobe-parallel SG backward.  A warp stages up to 32 covered pixels in shared
// memory, then its lanes walk those pixels with one lobe per lane: the
// per-lobe gradient sums (axis, sharpness, amplitude -- sums over all
// pixels) accumulate in registers with no reduction per pixel, and the
// per-pixel gradients (sums over lobes) are reduced across the lanes of a
// lobe group only when they are requested.  With K <= 16 the warp splits
// into 32/Kp groups (Kp = next power of two >= K) that take different
// pixels; with K > 32 each lane carries NL lobes.
struct SPix {
    float n[3], pax[3], ss, sa;
    float dfs[SG_CMAX], go[SG_CMAX];
};

struct SPixOut { float gd[SG_CMAX], gsa[SG_CMAX], gsx[3], gsh; };

template <int NL, int CC>
struct LaneLobes {
    bool valid[NL];
    float gs[NL];
    float3 sgn[NL];
    float3 ax[NL];     // raw axis (EXACT sharpness derivative)
    float a[NL][CC ? CC : SG_CMAX];
    float acc_ax[NL][3], acc_sh[NL], acc_ssh[NL];
    float acc_am[NL][CC ? CC : SG_CMAX];
};

template <int NL, int CC>
DEV void lane_lobes_load(LaneLobes<NL, CC>& LL, int li, int Kp, int K, int C, const float* axis, const float* sharp,
                         const float* amp) {
    const int Cn = CC ? CC : C;
#pragma unroll
    for (int s = 0; s < NL; ++s) {
        int i = li + s * Kp;
        LL.valid[s] = i < K;
        int ii = LL.valid[s] ? i : 0;
        float gs = K ? sharp[ii] : 0.f;
        LL.gs[s] = gs;
        LL.sgn[s] = K ? f3(axis[3 * ii] * gs, axis[3 * ii + 1] * gs, axis[3 * ii + 2] * gs) : f3(0.f, 0.f, 0.f);
        LL.ax[s] = K ? f3(axis[3 * ii], axis[3 * ii + 1], axis[3 * ii + 2]) : f3(0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < (CC ? CC : SG_CMAX); ++k) LL.a[s][k] = (k < Cn && K) ? amp[ii * C + k] : 0.f;
        LL.acc_ax[s][0] = LL.acc_ax[s][1] = LL.acc_ax[s][2] = 0.f;
        LL.acc_sh[s] = LL.acc_ssh[s] = 0.f;
#pragma unroll
        for (int k = 0; k < (CC ? CC : SG_CMAX); ++k) LL.acc_am[s][k] = 0.f;
    }
}

// Sum over the lanes of one lobe group (offsets below Kp).
DEV float group_sum(float v, int Kp) {
    for (int o = Kp >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Processes the m staged pixels of this warp.  PIX: also produce the
// per-pixel gradients into `out` (diffuse, specular amplitude/axis/sharpness).
template <int NL, int CC, bool PIX>
DEV void sg_bwd_lanes(LaneLobes<NL, CC>& LL, int C, int exact, const SPix* st, SPixOut* out, int m, int Kp, int g,
                      int G, int li) {
    const int Cn = CC ? CC : C;
    const int rounds = (m + G - 1) / G;
    if (!PIX) {
        // lobe gradients only: per pixel gd_k = g_k * diffuse_k once, then per
        // lobe two FMAs per channel; contributions are dropped when the lobe's
        // terms are not finite (the reference's guarded add, common.h:181)
        for (int rr = 0; rr < rounds; ++rr) {
            const int j = rr * G + g;
            if (j >= m) continue;
            const SPix& P = st[j];
            const float3 n = f3(P.n[0], P.n[1], P.n[2]), pax = f3(P.pax[0], P.pax[1], P.pax[2]);
            const float ss = P.ss, sa = P.sa;
            const float3 dn = n * SG_DIFF_SHARP, sn = pax * ss;
            float gk[CC ? CC : SG_CMAX], gdk[CC ? CC : SG_CMAX];
#pragma unroll
            for (int k = 0; k < (CC ? CC : SG_CMAX); ++k) {
                gk[k] = k < Cn ? P.go[k] : 0.f;
                gdk[k] = k < Cn ? P.go[k] * P.dfs[k] : 0.f;
            }
#pragma unroll
            for (int s = 0; s < NL; ++s) {
                if (!LL.valid[s]) continue;
                SGL t = sg_lobe_terms(n, dn, pax, sn, LL.sgn[s], LL.gs[s], ss, sa, exact, LL.ax[s]);
                float sum = 0.f, sumd = 0.f;
#pragma unroll
                for (int k = 0; k < (CC ? CC : SG_CMAX); ++k) {
                    sum = fmaf(gk[k], LL.a[s][k], sum);
                    sumd = fmaf(gdk[k], LL.a[s][k], sumd);
                }
                if (isfinite(t.dg) && isfinite(t.sgv)) {
#pragma unroll
                    for (int k = 0; k < (CC ? CC : SG_CMAX); ++k)
                        LL.acc_am[s][k] = fmaf(t.sgv, gk[k], fmaf(t.dg, gdk[k], LL.acc_am[s][k]));
                }
                float3 cax = ((t.ddg * sumd) * SG_DIFF_AMP + (t.dsg * sum) * sa) * LL.gs[s];
                if (fin3(cax)) { LL.acc_ax[s][0] += cax.x; LL.acc_ax[s][1] += cax.y; LL.acc_ax[s][2] += cax.z; }
                LL.acc_sh[s] += finite_or0(sumd * t.ddgs * SG_DIFF_AMP + sum * t.dsgs * sa);
            }
        }
        return;
    }
    for (int rr = 0; rr < rounds; ++rr) {
        const int j = rr * G + g;
        const bool ok = j < m;
        const SPix& P = st[ok ? j : 0];
        float pgd[CC ? CC : SG_CMAX], pgsa[CC ? CC : SG_CMAX], pgsx[3] = {0.f, 0.f, 0.f}, pgsh = 0.f;
#pragma unroll
        for (int k = 0; k < (CC ? CC : SG_CMAX); ++k) { pgd[k] = 0.f; pgsa[k] = 0.f; }
        if (ok) {
            const float3 n = f3(P.n[0], P.n[1], P.n[2]), pax = f3(P.pax[0], P.pax[1], P.pax[2]);
            const float ss = P.ss, sa = P.sa;
            const float3 dn = n * SG_DIFF_SHARP, sn = pax * ss;
#pragma unroll
            for (int s = 0; s < NL; ++s) {
                if (!LL.valid[s]) continue;
                SGB t = sg_bwd_terms(n, dn, pax, sn, LL.sgn[s], LL.gs[s], ss, sa, exact, LL.ax[s]);
                float sum = 0.f, sumd = 0.f, sum_sa = 0.f;
#pragma unroll
                for (int k = 0; k < (CC ? CC : SG_CMAX); ++k) {
                    if (k >= Cn) break;
                    const float a = LL.a[s][k], gk = P.go[k], dk = P.dfs[k];
                    sum += gk * a;
                    sumd += gk * a * dk;
                    LL.acc_am[s][k] += finite_or0(gk * (t.dg * dk + t.sgv));
                    if (PIX) {
                        pgd[k] += gk * t.dg * a;
                        if (!exact) pgsa[k] += gk * t.sgv * a;
                        else sum_sa += gk * t.sil_e * a;
                    }
                }
                float3 cax = ((t.ddg * sumd) * SG_DIFF_AMP + (t.dsg * sum) * sa) * LL.gs[s];
                if (fin3(cax)) { LL.acc_ax[s][0] += cax.x; LL.acc_ax[s][1] += cax.y; LL.acc_ax[s][2] += cax.z; }
                LL.acc_sh[s] += finite_or0(sumd * t.ddgs * SG_DIFF_AMP + sum * t.dsgs * sa);
                const float cssh = sum * t.dsgss * sa;
                if (!exact) LL.acc_ssh[s] += finite_or0(cssh);
                if (PIX) {
                    if (exact) { pgsa[0] += sum_sa; pgsh += cssh; }
                    float3 csx = ((t.dsg * sum) * sa) * ss;
                    pgsx[0] += csx.x; pgsx[1] += csx.y; pgsx[2] += csx.z;
                }
            }
        }
        if (PIX) {
#pragma unroll
            for (int k = 0; k < (CC ? CC : SG_CMAX); ++k) {
                if (k >= Cn) break;
                pgd[k] = group_sum(pgd[k], Kp);
                pgsa[k] = group_sum(pgsa[k], Kp);
            }
            pgsx[0] = group_sum(pgsx[0], Kp); pgsx[1] = group_sum(pgsx[1], Kp); pgsx[2] = group_sum(pgsx[2], Kp);
            pgsh = group_sum(pgsh, Kp);
            if (ok && li == 0) {
                SPixOut& o = out[j];
                for (int k = 0; k < Cn; ++k) { o.gd[k] = pgd[k]; o.gsa[k] = pgsa[k]; }
                o.gsx[0] = pgsx[0]; o.gsx[1] = pgsx[1]; o.gsx[2] = pgsx[2];
                o.gsh = pgsh;
            }
        }
    }
}

// Adds this lane's lobe sums into the block accumulator s_acc [K][nacc]
// (after folding the lobe groups of the warp together).
template <int NL, int CC>
DEV void lane_lobes_flush(LaneLobes<NL, CC>& LL, int C, int Kp, int li, float* s_acc, int nacc, bool ssh_lobe) {
    const int Cn = CC ? CC : C;
#pragma unroll
    for (int s = 0; s < NL; ++s) {
        float v[3 + 1 + SG_CMAX + 1];
        v[0] = LL.acc_ax[s][0]; v[1] = LL.acc_ax[s][1]; v[2] = LL.acc_ax[s][2]; v[3] = LL.acc_sh[s];
        for (int k = 0; k < SG_CMAX; ++k) v[4 + k] = k < Cn ? LL.acc_am[s][k] : 0.f;
        v[4 + SG_CMAX] = LL.acc_ssh[s];
        for (int q = 0; q < 4 + SG_CMAX + 1; ++q)
            for (int o = 16; o >= Kp; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        const int lane = threadIdx.x & 31;
        if (lane < Kp && LL.valid[s]) {
            const int i = li + s * Kp;
            float* a = s_acc + (size_t)i * nacc;
            atomicAdd(&a[0], v[0]); atomicAdd(&a[1], v[1]); atomicAdd(&a[2], v[2]); atomicAdd(&a[3], v[3]);
            for (int k = 0; k < Cn; ++k) atomicAdd(&a[4 + k], v[4 + k]);
            if (ssh_lobe) atomicAdd(&a[4 + Cn], v[4 + SG_CMAX]);
        }
    }
}

// Block accumulator [K][nacc] -> global lobe gradients.
DEV void sg_flush_block(const float* s_acc, int K, int C, int nacc, float* gaxis, float* gsharp, float* gamp,
                        float* gssh_lobe) {
    for (int j = threadIdx.x; j < K * nacc; j += blockDim.x) {
        float v = s_acc[j];
        if (v == 0.f) continue;
        int i = j / nacc, q = j % nacc;
        if (q < 3) { if (gaxis) atomicAdd(&gaxis[3 * i + q], v); }
        else if (q == 3) { if (gsharp) atomicAdd(&gsharp[i], v); }
        else if (q < 4 + C) { if (gamp) atomicAdd(&gamp[i * C + (q - 4)], v); }
        else if (gssh_lobe) atomicAdd(&gssh_lobe[i], v);
    }
}

inline int sg_lobe_group(int K) {
    int kp = 1;
    while (kp < K && kp < 32) kp <<= 1;
    return kp;
}
// The same on the device: lanes per lobe group for K lobes (a power of two,
// at most 32).
DEV int sg_lobe_group_dev(int K) {
    int kp = 1;
    while (kp < K && kp < 32) kp <<= 1;
    return kp;
}

// ---------------------------------------------------------------------------
// C = 4 fast paths (the fit configurations' RGBA lighting).
//
// exp(x) as 2^(x log2 e) on the hardware ex2 unit, with log2 e folded into
// per-lobe / per-pixel constants so that each exponential costs one add and
// one ex2.
constexpr float SG_L2E = 1.4426950408889634f;
DEV float ex2_fast(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Paired FP32 arithmetic: sm_100 issues a pair of FP32 adds, multiplies or
// fmas as ONE instruction (__fadd2_rn / __fmul2_rn / __ffma2_rn,
// round-to-nearest like the scalar forms).  The SG loops are issue-bound, so
// they carry two lobes (forward) or two pixels (lobe gradients) per
// instruction; only the rsqrt and ex2 steps run per element.
DEV float2 p2(float x) { return make_float2(x, x); }
DEV float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
DEV float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
DEV float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
DEV float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
DEV float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
DEV float2 ex2_2(float2 a) { return make_float2(ex2_fast(a.x), ex2_fast(a.y)); }
// 1/max(|v|, 1e-6) and |v| from |v|^2, per half (as sg_len).
DEV void sg_len2(float2 d2, float2& l, float2& il) {
    const float2 q = make_float2(fmaxf(d2.x, 1e-12f), fmaxf(d2.y, 1e-12f));
    il = make_float2(rsqrt_normal(q.x), rsqrt_normal(q.y));
    l = mul2(q, il);
}

// Lobes packed in pairs for the pixel-parallel forward: pair j holds lobes
// 2j and 2j+1 as (s a.x | s a.y), (s a.z | s), (amp.x | amp.y), (amp.z | amp.w),
// each float4 = (first lobe, second lobe, first lobe, second lobe) of two
// fields; an odd K is padded with a zero lobe (zero amplitude: it adds 0).
inline size_t sg_lobes4_smem(int K) { return sizeof(float4) * 2 * (size_t)(K + (K & 1)); }

DEV void sg_stage_lobes4(float4* sm, int K, const float* axis, const float* sharp, const float* amp) {
    const int np = (K + 1) >> 1;
    for (int j = threadIdx.x; j < np; j += blockDim.x) {
        float v[2][8];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 2 * j + h;
            const bool ok = i < K;
            const float s = ok ? sharp[i] : 0.f;
            v[h][0] = ok ? axis[3 * i] * s : 0.f;
            v[h][1] = ok ? axis[3 * i + 1] * s : 0.f;
            v[h][2] = ok ? axis[3 * i + 2] * s : 0.f;
            v[h][3] = s;
#pragma unroll
            for (int c = 0; c < 4; ++c) v[h][4 + c] = ok ? amp[4 * i + c] : 0.f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            sm[4 * j + q] = make_float4(v[0][2 * q], v[1][2 * q], v[0][2 * q + 1], v[1][2 * q + 1]);
    }
}

// Forward environment sums of one pixel for C = 4 (material.cu:305-317),
// two lobes per step; the same NaN-guard contract as sg_env (plain sums,
// and the guarded loop when a sum is not finite).
DEV void sg_env4(const float4* L4, int K, float3 n, float3 pax, float ss, float sa, float4& de, float4& se) {
    const float3 dn = n * SG_DIFF_SHARP, sn = pax * ss;
    const float2 dnx = p2(dn.x), dny = p2(dn.y), dnz = p2(dn.z), snx = p2(sn.x), sny = p2(sn.y), snz = p2(sn.z);
    const float2 l2e = p2(SG_L2E), nl2e = p2(-SG_L2E), ncd = p2(-(SG_DIFF_SHARP * SG_L2E)), nss = p2(-(ss * SG_L2E));
    const float2 amp = p2(SG_DIFF_AMP), sa2 = p2(sa);
    float2 dx = p2(0.f), dy = dx, dz = dx, dw = dx, ex = dx, ey = dx, ez = dx, ew = dx;
    const int np = (K + 1) >> 1;
    for (int j = 0; j < np; ++j) {
        const float4 P0 = L4[4 * j], P1 = L4[4 * j + 1], P2 = L4[4 * j + 2], P3 = L4[4 * j + 3];
        const float2 gx = make_float2(P0.x, P0.y), gy = make_float2(P0.z, P0.w), gz = make_float2(P1.x, P1.y);
        const float2 gs = make_float2(P1.z, P1.w);
        // diffuse lobe
        float2 vx = add2(dnx, gx), vy = add2(dny, gy), vz = add2(dnz, gz);
        float2 l, il;
        sg_len2(fma2(vz, vz, fma2(vy, vy, mul2(vx, vx))), l, il);
        float2 nc = fma2(gs, nl2e, ncd);
        float2 em = ex2_2(fma2(l, l2e, nc)), ep = ex2_2(fma2(l, nl2e, nc));
        const float2 dg = mul2(mul2(sub2(em, ep), il), amp);
        // specular lobe
        vx = add2(snx, gx); vy = add2(sny, gy); vz = add2(snz, gz);
        sg_len2(fma2(vz, vz, fma2(vy, vy, mul2(vx, vx))), l, il);
        nc = fma2(gs, nl2e, nss);
        em = ex2_2(fma2(l, l2e, nc)); ep = ex2_2(fma2(l, nl2e, nc));
        const float2 sg = mul2(mul2(sub2(em, ep), il), sa2);
        const float2 bx = make_float2(P2.x, P2.y), by = make_float2(P2.z, P2.w);
        const float2 bz = make_float2(P3.x, P3.y), bw = make_float2(P3.z, P3.w);
        dx = fma2(dg, bx, dx); dy = fma2(dg, by, dy); dz = fma2(dg, bz, dz); dw = fma2(dg, bw, dw);
        ex = fma2(sg, bx, ex); ey = fma2(sg, by, ey); ez = fma2(sg, bz, ez); ew = fma2(sg, bw, ew);
    }
    const float4 d = make_float4(dx.x + dx.y, dy.x + dy.y, dz.x + dz.y, dw.x + dw.y);
    const float4 e = make_float4(ex.x + ex.y, ey.x + ey.y, ez.x + ez.y, ew.x + ew.y);
    if (isfinite(d.x) && isfinite(d.y) && isfinite(d.z) && isfinite(d.w) && isfinite(e.x) && isfinite(e.y) &&
        isfinite(e.z) && isfinite(e.w)) {
        de = d; se = e;
        return;
    }
    float dd[4] = {0.f, 0.f, 0.f, 0.f}, ee[4] = {0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < K; ++i) {
        const float4 P0 = L4[4 * (i >> 1)], P1 = L4[4 * (i >> 1) + 1], P2 = L4[4 * (i >> 1) + 2],
                     P3 = L4[4 * (i >> 1) + 3];
        const bool h = i & 1;
        const float3 g = h ? f3(P0.y, P0.w, P1.y) : f3(P0.x, P0.z, P1.x);
        const float gs = h ? P1.w : P1.z;
        const float b[4] = {h ? P2.y : P2.x, h ? P2.w : P2.z, h ? P3.y : P3.x, h ? P3.w : P3.z};
        float dg, sg;
        sg_terms(dn, sn, g, gs, ss, sa, dg, sg);
        for (int k = 0; k < 4; ++k) { add_nan_check(dd[k], dg * b[k]); add_nan_check(ee[k], sg * b[k]); }
    }
    de = make_float4(dd[0], dd[1], dd[2], dd[3]);
    se = make_float4(ee[0], ee[1], ee[2], ee[3]);
}

// ---------------------------------------------------------------------------
// Lobe gradients of the fused step, two pixels per lane: each lane walks
// pixel PAIRS for its lobe, so every FP32 step below serves two pixels.

// Two staged pixels; each field holds (first pixel, second pixel).  The
// per-pixel factors every lobe reuses are computed once by the staging lane.
struct __align__(16) SPair {
    float2 dnx, dny, dnz;    // 2.133 n
    float2 snx, sny, snz;    // ss p
    float2 sa, nssl;         // sa, -ss log2 e
    float2 dn2, sn2;         // |2.133 n|^2, |ss p|^2
    float2 gx, gy, gz, gw;   // dL/dout
    float2 hx, hy, hz, hw;   // dL/dout * diffuse * 2.34
};
constexpr int SPAIR_FIELDS = (int)(sizeof(SPair) / sizeof(float2));

// Writes one pixel into half `h` of a staged pair from its shading record
// (nss = (n, ss), psa = (p, sa), the diffuse texture colour dfs) and its
// dL/dout.  The diffuse environment amplitude 2.34 rides on dL/dout *
// diffuse, the only per-pixel factor every diffuse term carries.  All-zero
// inputs pad an odd count: a zero pixel adds exactly nothing to any sum.
DEV void spair_put(SPair* s, int h, float4 nss, float4 psa, float4 dfs, float4 go) {
    const float3 dn = f3(nss.x, nss.y, nss.z) * SG_DIFF_SHARP, sn = f3(psa.x, psa.y, psa.z) * nss.w;
    const float v[SPAIR_FIELDS] = {dn.x, dn.y, dn.z, sn.x, sn.y, sn.z, psa.w, -(nss.w * SG_L2E), dot3(dn, dn),
                                   dot3(sn, sn), go.x, go.y, go.z, go.w, go.x * dfs.x * SG_DIFF_AMP,
                                   go.y * dfs.y * SG_DIFF_AMP, go.z * dfs.z * SG_DIFF_AMP, go.w * dfs.w * SG_DIFF_AMP};
    float* f = reinterpret_cast<float*>(s) + h;
#pragma unroll
    for (int i = 0; i < SPAIR_FIELDS; ++i) f[2 * i] = v[i];
}

// One lane's lobe (C = 4): its constants broadcast to both halves and its
// gradient sums per half.  Every axis term carries the lobe's sharpness s
// (d|v|/da = s v/|v| for v = u + s a), so the sums leave it out and the
// flush multiplies it back in; the axis sum
// sum_p c1 (u_d + s a) + c2 (u_s + s a) is kept as ax = sum (c1 u_d + c2 u_s)
// plus axs = sum (c1 + c2), combined with s a when the lane flushes.
struct Lobe4x2 {
    bool valid;
    float3 sgn;                  // s a (scalar, for the flush)
    float2 sx, sy, sz;           // s a
    float2 a0x, a0y, a0z, a02;   // raw axis and |a|^2 (EXACT sharpness derivative)
    float2 gs, ngsl, ncdl, sg2;  // s, -s log2 e, -(2.133 + s) log2 e, |s a|^2
    float2 ax4, ay4, az4, aw4;   // amplitude
    float2 gax, gay, gaz, gaxs, gsh, gam0, gam1, gam2, gam3;   // sums
};

DEV void lobe4x2_clear(Lobe4x2& L) {
    L.gax = L.gay = L.gaz = L.gaxs = L.gsh = L.gam0 = L.gam1 = L.gam2 = L.gam3 = p2(0.f);
}

DEV void lobe4x2_load(Lobe4x2& L, int i, int K, const float* axis, const float* sharp, const float* amp) {
    L.valid = i < K;
    const int ii = L.valid ? i : 0;
    const float s = K ? sharp[ii] : 0.f;
    const float3 a0 = K ? f3(axis[3 * ii], axis[3 * ii + 1], axis[3 * ii + 2]) : f3(0.f, 0.f, 0.f);
    L.sgn = a0 * s;
    L.sx = p2(L.sgn.x); L.sy = p2(L.sgn.y); L.sz = p2(L.sgn.z);
    L.a0x = p2(a0.x); L.a0y = p2(a0.y); L.a0z = p2(a0.z); L.a02 = p2(dot3(a0, a0));
    L.gs = p2(s);
    L.ngsl = p2(-(s * SG_L2E));
    L.ncdl = p2(-((SG_DIFF_SHARP + s) * SG_L2E));
    L.sg2 = p2(dot3(L.sgn, L.sgn));
    const float4 am = K ? make_float4(amp[4 * ii], amp[4 * ii + 1], amp[4 * ii + 2], amp[4 * ii + 3])
                        : make_float4(0.f, 0.f, 0.f, 0.f);
    L.ax4 = p2(am.x); L.ay4 = p2(am.y); L.az4 = p2(am.z); L.aw4 = p2(am.w);
    lobe4x2_clear(L);
}

// One half's contributions, each added only when finite (the reference's
// guarded adds, common.h:181, material.cu:428-437): the amplitude per
// channel, the axis terms when both lobe factors (with s) are finite, the
// sharpness term when finite.
DEV void lobe4x2_guarded(float& am0, float& am1, float& am2, float& am3, float& ax, float& ay, float& az, float& axs,
                         float& sh, float s, float dg, float sgv, float c1, float c2, float shc, float dnx, float dny,
                         float dnz, float snx, float sny, float snz, float gx, float gy, float gz, float gw, float hx,
                         float hy, float hz, float hw) {
    am0 += finite_or0(fmaf(sgv, gx, dg * hx));
    am1 += finite_or0(fmaf(sgv, gy, dg * hy));
    am2 += finite_or0(fmaf(sgv, gz, dg * hz));
    am3 += finite_or0(fmaf(sgv, gw, dg * hw));
    if (isfinite(c1 * s) && isfinite(c2 * s)) {
        ax = fmaf(c2, snx, fmaf(c1, dnx, ax));
        ay = fmaf(c2, sny, fmaf(c1, dny, ay));
        az = fmaf(c2, snz, fmaf(c1, dnz, az));
        axs += c1 + c2;
    }
    sh += finite_or0(shc);
}

// Gradient contributions of two pixels to one lobe (material.cu:398-433),
// rearranged.  With v = u + s a (u = 2.133 n for the diffuse term, ss p for
// the specular one), |v|^2 = |u|^2 + |s a|^2 + 2 u.(s a), and the dot product
// is the one the reference's sharpness derivative uses.  With e-/e+ the two
// exponentials, Dm = e- - e+ and T = (e- + e+) - il Dm:  value = Dm il,
// (d value/d|v|)/|v| = T il^2,  d value/ds = il (dotn T - Dm)  (the
// reference's ((dotn (1-il) - 1) e- + (dotn (1+il) + 1) e+) il, expanded).
// guard = false adds every contribution plainly (the walk's first pass);
// guard = true checks each one (the pass that redoes a lane whose plain sums
// came out non-finite).
template <bool EXACT>
DEV void lobe4x2_accumulate(Lobe4x2& L, const SPair& P, bool guard) {
    // diffuse lobe
    const float2 dd = fma2(L.sz, P.dnz, fma2(L.sy, P.dny, mul2(L.sx, P.dnx)));
    float2 dl, dil;
    sg_len2(fma2(p2(2.f), dd, add2(P.dn2, L.sg2)), dl, dil);
    const float2 dotn = EXACT ? mul2(fma2(L.gs, L.a02, fma2(L.a0z, P.dnz, fma2(L.a0y, P.dny, mul2(L.a0x, P.dnx)))), dil)
                              : mul2(add2(L.gs, dd), dil);
    float2 em = ex2_2(fma2(dl, p2(SG_L2E), L.ncdl)), ep = ex2_2(fma2(dl, p2(-SG_L2E), L.ncdl));
    const float2 dDm = sub2(em, ep), dT = fma2(neg2(dil), dDm, add2(em, ep));
    // specular lobe
    const float2 sd = fma2(L.sz, P.snz, fma2(L.sy, P.sny, mul2(L.sx, P.snx)));
    float2 sl, sil;
    sg_len2(fma2(p2(2.f), sd, add2(P.sn2, L.sg2)), sl, sil);
    const float2 dots = EXACT ? mul2(fma2(L.gs, L.a02, fma2(L.a0z, P.snz, fma2(L.a0y, P.sny, mul2(L.a0x, P.snx)))), sil)
                              : mul2(add2(L.gs, sd), sil);
    const float2 nc = add2(P.nssl, L.ngsl);
    em = ex2_2(fma2(sl, p2(SG_L2E), nc));
    ep = ex2_2(fma2(sl, p2(-SG_L2E), nc));
    const float2 sDm = sub2(em, ep), sT = fma2(neg2(sil), sDm, add2(em, ep));
    // channel sums (h carries the diffuse amplitude 2.34)
    const float2 sum = fma2(P.gw, L.aw4, fma2(P.gz, L.az4, fma2(P.gy, L.ay4, mul2(P.gx, L.ax4))));
    const float2 sumd = fma2(P.hw, L.aw4, fma2(P.hz, L.az4, fma2(P.hy, L.ay4, mul2(P.hx, L.ax4))));
    const float2 dg = mul2(dDm, dil);                         // diffuse value / 2.34
    const float2 sdA = mul2(sumd, dil);
    const float2 c1 = mul2(sdA, mul2(dT, dil));               // sumd T il^2 2.34 (s in the flush)
    const float2 sils = mul2(sil, P.sa);
    const float2 sgv = mul2(sDm, sils);                       // specular value
    const float2 ssa = mul2(sum, sils);
    const float2 c2 = mul2(ssa, mul2(sT, sil));               // sum T il^2 sa (s in the flush)
    const float2 shc = fma2(sdA, fma2(dotn, dT, neg2(dDm)), mul2(ssa, fma2(dots, sT, neg2(sDm))));
    if (!guard) {
        L.gam0 = fma2(sgv, P.gx, fma2(dg, P.hx, L.gam0));
        L.gam1 = fma2(sgv, P.gy, fma2(dg, P.hy, L.gam1));
        L.gam2 = fma2(sgv, P.gz, fma2(dg, P.hz, L.gam2));
        L.gam3 = fma2(sgv, P.gw, fma2(dg, P.hw, L.gam3));
        L.gax = fma2(c2, P.snx, fma2(c1, P.dnx, L.gax));
        L.gay = fma2(c2, P.sny, fma2(c1, P.dny, L.gay));
        L.gaz = fma2(c2, P.snz, fma2(c1, P.dnz, L.gaz));
        L.gaxs = add2(L.gaxs, add2(c1, c2));
        L.gsh = add2(L.gsh, shc);
        return;
    }
    lobe4x2_guarded(L.gam0.x, L.gam1.x, L.gam2.x, L.gam3.x, L.gax.x, L.gay.x, L.gaz.x, L.gaxs.x, L.gsh.x, L.gs.x, dg.x,
                    sgv.x, c1.x, c2.x, shc.x, P.dnx.x, P.dny.x, P.dnz.x, P.snx.x, P.sny.x, P.snz.x, P.gx.x, P.gy.x,
                    P.gz.x, P.gw.x, P.hx.x, P.hy.x, P.hz.x, P.hw.x);
    lobe4x2_guarded(L.gam0.y, L.gam1.y, L.gam2.y, L.gam3.y, L.gax.y, L.gay.y, L.gaz.y, L.gaxs.y, L.gsh.y, L.gs.y, dg.y,
                    sgv.y, c1.y, c2.y, shc.y, P.dnx.y, P.dny.y, P.dnz.y, P.snx.y, P.sny.y, P.snz.y, P.gx.y, P.gy.y,
                    P.gz.y, P.gw.y, P.hx.y, P.hy.y, P.hz.y, P.hw.y);
}

// The lane's eight totals (axis xyz, sharpness, amplitude[4]), both halves
// folded together and the axis sums multiplied by s.
DEV void lobe4x2_values(const Lobe4x2& L, float v[8]) {
    const float s = L.gs.x, axs = L.gaxs.x + L.gaxs.y;
    v[0] = s * fmaf(axs, L.sgn.x, L.gax.x + L.gax.y);
    v[1] = s * fmaf(axs, L.sgn.y, L.gay.x + L.gay.y);
    v[2] = s * fmaf(axs, L.sgn.z, L.gaz.x + L.gaz.y);
    v[3] = L.gsh.x + L.gsh.y;
    v[4] = L.gam0.x + L.gam0.y;
    v[5] = L.gam1.x + L.gam1.y;
    v[6] = L.gam2.x + L.gam2.y;
    v[7] = L.gam3.x + L.gam3.y;
}

// True when the lane has to walk its pixels again with every contribution
// checked: its plain sums are not all finite, which happens exactly when
// some contribution was not finite (or a sum overflowed).
DEV bool lobe4x2_needs_guard(const Lobe4x2& L) {
    if (!L.valid) return false;
    float v[8];
    lobe4x2_values(L, v);
    bool ok = true;
#pragma unroll
    for (int q = 0; q < 8; ++q) ok = ok && isfinite(v[q]);
    return !ok;
}

// Folds the lobe groups of the warp together and adds the lane's totals into
// the block accumulator s_acc [K][8] (axis xyz, sharpness, amplitude[4]); a
// total that is not finite is dropped, as the reference's guarded add of it.
DEV void lobe4x2_flush(const Lobe4x2& L, int i, int Kp, float* s_acc) {
    float v[8];
    lobe4x2_values(L, v);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        v[q] = finite_or0(v[q]);
        for (int o = 16; o >= Kp; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    }
    const int lane = threadIdx.x & 31;
    if (lane < Kp && L.valid) {
#pragma unroll
        for (int q = 0; q < 8; ++q) atomicAdd(&s_acc[(size_t)i * 8 + q], finite_or0(v[q]));
    }
}

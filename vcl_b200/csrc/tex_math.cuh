// Texture sampling arithmetic shared by the per-operator texture kernels and
// the fused fit kernels (reference texturemap.cu:22-65).
#pragma once
#include "common.cuh"

DEV float t_mul(float a, float b) { return __fmul_rn(a, b); }
DEV float t_add(float a, float b) { return __fadd_rn(a, b); }
DEV float t_sub(float a, float b) { return __fsub_rn(a, b); }

struct TexDesc {
    int tw, th, C, L;
    long long off[16];
    // level sizes and L - 2, L - 1 as floats (exact), so that the kernels
    // do not convert them per pixel
    float fw[16], fh[16];
    float fL2, fL1;
};

// texturemap.cu:22-47 (level) and :160-197 (level + Jacobian); the level
// arithmetic is rounded exactly like the CPU restatement so that the same
// mip levels are chosen.
DEV void calc_level(const TexDesc& t, float4 da, int& l0, int& l1, float& fl, float4* dl, int exact) {
    float dsdx = t_mul(da.x, t.fw[0]), dsdy = t_mul(da.y, t.fw[0]);
    float dtdx = t_mul(da.z, t.fh[0]), dtdy = t_mul(da.w, t.fh[0]);
    float s2 = t_add(t_mul(dsdx, dsdx), t_mul(dsdy, dsdy));
    float t2 = t_add(t_mul(dtdx, dtdx), t_mul(dtdy, dtdy));
    float a = t_sub(t_mul(dsdx, dtdy), t_mul(dtdx, dsdy));
    float b = t_mul(.5f, t_add(s2, t2));
    float c2 = t_sub(t_mul(b, b), t_mul(a, a));
    float c = sqrtf(c2);
    float level = t_mul(.5f, log2f(t_add(b, c)));
    const int L = t.L;
    l0 = level <= 0 ? 0 : t.fL2 <= level ? L - 2 : (int)floorf(level);
    l1 = level <= 1 ? 1 : t.fL1 <= level ? L - 1 : (int)floorf(level) + 1;
    fl = level <= 0 ? 0.f : t.fL1 <= level ? 1.f : level - floorf(level);
    if (dl) {
        float d = b * c + c2;
        if ((double)fabsf(d) > 1e-6) {
            d = 0.72134752f / d;
            float bc = b + c;
            *dl = make_float4(d * (bc * dsdx - a * dtdy), d * (bc * dsdy + a * dtdx), bc * dtdx + a * dsdy,
                              bc * dtdy - a * dsdx);
            if (exact) { dl->z *= d; dl->w *= d; }
        } else if ((double)fabsf(b) > 1e-6) {
            d = 1 / b;
            *dl = make_float4(d * dsdx, d * dsdy, d * dtdx, d * dtdy);
        } else {
            *dl = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

// texturemap.cu:49-65: the 2x2 texel cell of `uv` at `level` as texel
// coordinates (columns u0, u1, rows v0, v1; u1 is u0 or u0 + 1, likewise v1)
// and the bilinear fractions.
DEV void cell_fetch(const TexDesc& t, int level, float2 uv, int& u0, int& u1, int& v0, int& v1, float2& f) {
    const int sx = t.tw >> level, sy = t.th >> level;
    const float fsx = t.fw[level], fsy = t.fh[level];
    float tx = uv.x * fsx, ty = uv.y * fsy;
    u0 = tx < 0 ? 0 : tx > fsx - 1.f ? sx - 1 : (int)tx;
    u1 = tx < 1 ? 0 : tx > fsx - 2.f ? sx - 1 : (int)tx + 1;
    v0 = ty < 0 ? 0 : ty > fsy - 1.f ? sy - 1 : (int)ty;
    v1 = ty < 1 ? 0 : ty > fsy - 2.f ? sy - 1 : (int)ty + 1;
    f.x = tx < 0 ? 0.f : fsx < tx ? 1.f : tx - floorf(tx);
    f.y = ty < 0 ? 0.f : fsy < ty ? 1.f : ty - floorf(ty);
}

// The same cell as texel indices within the level.
DEV void index_fetch(const TexDesc& t, int level, float2 uv, int idx[4], float2& f) {
    int u0, u1, v0, v1;
    cell_fetch(t, level, uv, u0, u1, v0, v1, f);
    const int sx = t.tw >> level;
    idx[0] = v0 * sx + u0; idx[1] = v0 * sx + u1; idx[2] = v1 * sx + u0; idx[3] = v1 * sx + u1;
}

DEV float4 ld4(const float* p, int i) { return reinterpret_cast<const float4*>(p)[i]; }
DEV float4 bilerp4(float4 a, float4 b, float4 c, float4 d, float2 t) {
    float4 r;
    r.x = lerpf_(lerpf_(a.x, b.x, t.x), lerpf_(c.x, d.x, t.x), t.y);
    r.y = lerpf_(lerpf_(a.y, b.y, t.x), lerpf_(c.y, d.y, t.x), t.y);
    r.z = lerpf_(lerpf_(a.z, b.z, t.x), lerpf_(c.z, d.z, t.x), t.y);
    r.w = lerpf_(lerpf_(a.w, b.w, t.x), lerpf_(c.w, d.w, t.x), t.y);
    return r;
}
DEV float bilerp1(float a, float b, float c, float d, float2 t) { return lerpf_(lerpf_(a, b, t.x), lerpf_(c, d, t.x), t.y); }


inline TexDesc make_desc(int tw, int th, int C, int L) {
    TexDesc d;
    d.tw = tw; d.th = th; d.C = C; d.L = L;
    long long off = 0;
    for (int l = 0; l < 16; ++l) {
        d.off[l] = off;
        if (l < L) off += (long long)(tw >> l) * (th >> l) * C;
        d.fw[l] = (float)(tw >> l);
        d.fh[l] = (float)(th >> l);
    }
    d.fL2 = (float)(L - 2);
    d.fL1 = (float)(L - 1);
    return d;
}

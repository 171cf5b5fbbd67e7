/*
 * vcl_oracle.c -- serial CPU restatement of the vcl differentiable-rendering
 * path.  TEST INFRASTRUCTURE ONLY (the checker); never linked by the product.
 *
 * Written from the reference's algorithm, one function per operator; each
 * cites the reference lines it follows (nvdiffrast/nvdiffrast/<file>:<line>).
 * Arithmetic follows the reference's C++ promotions: where a float expression
 * meets a double literal (1e-6, 1e-3, 1.0) the reference computes in double
 * and rounds once on store, and so does this file.  Compile with
 * -ffp-contract=off so that no multiply-add is fused.
 *
 * The reference accumulates some gradients with unsynchronised adds from many
 * threads (antialias.cu:63-65 vs :31,34; material.cu:428-436).  The serial
 * order used here -- every pixel's initial store, then all adds in raster
 * order -- is the race-free meaning of those kernels.
 */
#include "vcl_oracle.h"
#include <math.h>
#include <string.h>
#include <stdlib.h>
#include <float.h>

typedef struct { float x, y; } f2;
typedef struct { float x, y, z; } f3;

static inline f2 F2(float x, float y) { f2 r = {x, y}; return r; }
static inline f3 F3(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static inline f3 add3(f3 a, f3 b) { return F3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 sub3(f3 a, f3 b) { return F3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 mul3s(f3 a, float s) { return F3(a.x * s, a.y * s, a.z * s); }
static inline float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float len3(f3 a) { return sqrtf(dot3(a, a)); }
static inline f3 normalize3(f3 v) { float d = 1.f / len3(v); return F3(v.x * d, v.y * d, v.z * d); }
static inline float cross2(f2 a, f2 b) { return a.x * b.y - a.y * b.x; }
static inline f3 ld3(const float* p, size_t i) { return F3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
static inline float lerpf_(float a, float b, float t) { return a + t * (b - a); }
static inline float bilerp_(float a, float b, float c, float d, f2 t) {
    return lerpf_(lerpf_(a, b, t.x), lerpf_(c, d, t.x), t.y);
}

/* Float -> int conversion with the GPU's cvt.rzi.s32.f32 semantics
 * (truncate, NaN -> 0, saturate), which the reference's (int) casts get on
 * the device; plain C leaves NaN/out-of-range undefined. */
static inline int f2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483648.f) return 2147483647;
    if (f <= -2147483648.f) return (int)0x80000000;
    return (int)f;
}

/* common.h:181-182 */
static inline void add_nan_check(float* a, float b) {
    if (!isfinite(*a)) *a = 0.f;
    else { float v = *a + b; if (isfinite(v)) *a = v; }
}
static inline void add_nan_check3(float* a, f3 b) {
    if (!(isfinite(a[0]) && isfinite(a[1]) && isfinite(a[2]))) { a[0] = a[1] = a[2] = 0.f; }
    else {
        f3 v = F3(a[0] + b.x, a[1] + b.y, a[2] + b.z);
        if (isfinite(v.x) && isfinite(v.y) && isfinite(v.z)) { a[0] = v.x; a[1] = v.y; a[2] = v.z; }
    }
}
/* The same NaN/Inf-guarded adds on double accumulators (sums over pixels). */
static inline void add_nan_check_d(double* a, double b) {
    if (!isfinite(*a)) *a = 0.0;
    else { double v = *a + b; if (isfinite(v)) *a = v; }
}
static inline void add_nan_check3_d(double* a, f3 b) {
    if (!(isfinite(a[0]) && isfinite(a[1]) && isfinite(a[2]))) { a[0] = a[1] = a[2] = 0.0; return; }
    double x = a[0] + b.x, y = a[1] + b.y, z = a[2] + b.z;
    if (isfinite(x) && isfinite(y) && isfinite(z)) { a[0] = x; a[1] = y; a[2] = z; }
}

/* ------------------------------------------------------------------------ */
/* project.cu:69-77 */
void orc_project_fwd(int nv, const float* m, const float* pos, int dim, float* out) {
    for (int p = 0; p < nv; ++p) {
        float x = pos[p * 3], y = pos[p * 3 + 1], z = pos[p * 3 + 2];
        for (int i = 0; i < dim; ++i)
            out[(size_t)p * dim + i] = m[i] * x + m[4 + i] * y + m[8 + i] * z + m[12 + i];
    }
}

/* project.cu:114-131 (vertex gradient; the matrix gradient is not wired on
 * the path) */
void orc_project_bwd(int nv, const float* m, const float* g_out, int dim, float* g_pos) {
    for (int p = 0; p < nv; ++p)
        for (int i = 0; i < dim; ++i) {
            float g = g_out[(size_t)p * dim + i];
            g_pos[p * 3] += m[i] * g;
            g_pos[p * 3 + 1] += m[4 + i] * g;
            g_pos[p * 3 + 2] += m[8 + i] * g;
        }
}

/* ------------------------------------------------------------------------ */
/* Rasterize forward.  The reference draws through OpenGL (rasterize.cpp:
 * 91-202, state :252-268): no culling, GL_LESS depth test against a cleared
 * depth of 1.0, one primitive id per fragment, perspective-correct varyings
 * (u,v) = (1,0),(0,1),(0,0) at v0,v1,v2, out = (u, v, z/w, id+1) and, with
 * DB, out_db = var_db * w with var_db from the geometry shader (:148-164).
 *
 * Restated semantics (identical, operation for operation, in the CUDA
 * rasterizer so that triangle ids match bit for bit):
 *   pixel centre in NDC: s = ((2px+1-W)/W, (2py+1-H)/H)   (rows bottom-up)
 *   edge functions of the clip-space (homogeneous 2D) triangle
 *     A_i(s) = (a_i*s.x + b_i*s.y) + k_i,
 *     a_0 = w2*y1 - w1*y2, b_0 = w1*x2 - w2*x1, k_0 = x1*y2 - y1*x2 (cyclic)
 *   sigma = sign(det[x;y;w]) with det = (w0*k0 + w1*k1) + w2*k2 (0 -> skip)
 *   covered  <=>  for all i: sigma*A_i > 0, or A_i == 0 on a top-left edge
 *                 (oriented gradient g = sigma*(a_i,b_i): g.x > 0, or g.x == 0
 *                 and g.y < 0; window y points up), and sigma*D > 0,
 *                 D = (A0 + A1) + A2
 *   u = A0/D, v = A1/D, zw = ((A0*z0 + A1*z1) + A2*z2) / ((A0*w0 + A1*w1) + A2*w2)
 *   near/far clip: -1 <= zw <= 1; depth test zw < depth (cleared to 1.0),
 *   equal depth keeps the lower triangle id (first drawn wins under GL_LESS);
 *   only pixels inside raster_bbox() are tested (half a pixel around the
 *   projected vertex extent).
 * Depth is compared in FP32, not a 24-bit depth buffer.
 */
typedef struct {
    float a[3], b[3], k[3];
    float sigma;
    float z[3], w[3];
    float db[3][4];
    int valid;
} rtri;

static void raster_setup(const float* c0, const float* c1, const float* c2, float xs, float ys, int want_db, rtri* t) {
    float x0 = c0[0], y0 = c0[1], x1 = c1[0], y1 = c1[1], x2 = c2[0], y2 = c2[1];
    float w0 = c0[3], w1 = c1[3], w2 = c2[3];
    t->a[0] = w2 * y1 - w1 * y2; t->b[0] = w1 * x2 - w2 * x1; t->k[0] = x1 * y2 - y1 * x2;
    t->a[1] = w0 * y2 - w2 * y0; t->b[1] = w2 * x0 - w0 * x2; t->k[1] = x2 * y0 - y2 * x0;
    t->a[2] = w1 * y0 - w0 * y1; t->b[2] = w0 * x1 - w1 * x0; t->k[2] = x0 * y1 - y0 * x1;
    float det = (w0 * t->k[0] + w1 * t->k[1]) + w2 * t->k[2];
    t->valid = (det != 0.f) && isfinite(det);
    t->sigma = det > 0.f ? 1.f : -1.f;
    t->z[0] = c0[2]; t->z[1] = c1[2]; t->z[2] = c2[2];
    t->w[0] = w0; t->w[1] = w1; t->w[2] = w2;
    if (want_db) {
        /* rasterize.cpp:141-164 */
        f2 p0 = F2(x0, y0), p1 = F2(x1, y1), p2 = F2(x2, y2);
        f2 e0 = F2(w0 * p2.x - w2 * p0.x, w0 * p2.y - w2 * p0.y);
        f2 e1 = F2(w1 * p2.x - w2 * p1.x, w1 * p2.y - w2 * p1.y);
        f2 e = F2(w0 * p1.x - w1 * p0.x, w0 * p1.y - w1 * p0.y);
        float a = e0.x * e1.y - e0.y * e1.x;
        float eps = 1e-6f;
        float ca = (fabsf(a) >= eps) ? a : (a < 0.f) ? -eps : eps;
        f2 ascl = F2(ys * w2 / ca, xs * w2 / ca);
        e0.x *= ascl.x; e0.y *= ascl.y;
        e1.x *= ascl.x; e1.y *= ascl.y;
        e.x *= ascl.x; e.y *= ascl.y;
        float d0[4] = {e0.y - e.y, -e0.x + e.x, -e0.y, e0.x};
        float d1[4] = {e1.y, -e1.x, -e1.y - e.y, e1.x + e.x};
        float d2[4] = {e1.y, -e1.x, -e0.y, e0.x};
        memcpy(t->db[0], d0, sizeof d0); memcpy(t->db[1], d1, sizeof d1); memcpy(t->db[2], d2, sizeof d2);
    }
}

/* Trivial reject in clip space: all three vertices outside one plane. */
static int raster_outside(const float* c0, const float* c1, const float* c2) {
    const float* c[3] = {c0, c1, c2};
    int o[6] = {1, 1, 1, 1, 1, 1};
    for (int i = 0; i < 3; ++i) {
        float x = c[i][0], y = c[i][1], z = c[i][2], w = c[i][3];
        o[0] &= x > w; o[1] &= x < -w; o[2] &= y > w; o[3] &= y < -w; o[4] &= z > w; o[5] &= z < -w;
    }
    return o[0] | o[1] | o[2] | o[3] | o[4] | o[5];
}

static inline int edge_in(float A, float a, float b, float sigma) {
    float sA = sigma * A;
    if (sA > 0.f) return 1;
    if (A != 0.f) return 0;
    float gx = sigma * a, gy = sigma * b;
    return gx > 0.f || (gx == 0.f && gy < 0.f);
}

/* Pixel bounding box of a triangle, part of the restated semantics (the CUDA
 * rasterizer computes the same box with the same float operations): when all
 * w > 0, the pixel centres within half a pixel of the projected vertices'
 * extent (x/w taken as x * (1/w), both rounded), otherwise the whole view.
 * A centre outside the vertex extent lies outside the triangle, so GL never
 * draws it; the margin covers the rounding of the extent.  The FP32 edge
 * functions of a nearly edge-on triangle can accept centres further out than
 * that (their rounding error is large next to such a triangle's tiny
 * determinant), and the box is what excludes them.  Returns 0 when empty. */
static int raster_bbox(const float* c0, const float* c1, const float* c2, int W, int H, int* x0, int* x1, int* y0, int* y1) {
    float w0 = c0[3], w1 = c1[3], w2 = c2[3];
    if (w0 > 0.f && w1 > 0.f && w2 > 0.f) {
        float iw0 = 1.f / w0, iw1 = 1.f / w1, iw2 = 1.f / w2;
        float X0 = c0[0] * iw0, X1 = c1[0] * iw1, X2 = c2[0] * iw2;
        float Y0 = c0[1] * iw0, Y1 = c1[1] * iw1, Y2 = c2[1] * iw2;
        float xmn = fminf(fminf(X0, X1), X2), xmx = fmaxf(fmaxf(X0, X1), X2);
        float ymn = fminf(fminf(Y0, Y1), Y2), ymx = fmaxf(fmaxf(Y0, Y1), Y2);
        float hw = 0.5f * (float)W, hh = 0.5f * (float)H;
        float fx0 = (xmn + 1.f) * hw - 0.5f, fx1 = (xmx + 1.f) * hw - 0.5f;
        float fy0 = (ymn + 1.f) * hh - 0.5f, fy1 = (ymx + 1.f) * hh - 0.5f;
        fx0 = fmaxf(fminf(fx0, (float)W), -2.f); fx1 = fmaxf(fminf(fx1, (float)W), -2.f);
        fy0 = fmaxf(fminf(fy0, (float)H), -2.f); fy1 = fmaxf(fminf(fy1, (float)H), -2.f);
        if (!(fx0 == fx0 && fx1 == fx1 && fy0 == fy0 && fy1 == fy1)) { *x0 = 0; *x1 = W - 1; *y0 = 0; *y1 = H - 1; return 1; }
        int ix0 = (int)ceilf(fx0 - 0.5f), ix1 = (int)floorf(fx1 + 0.5f);
        int iy0 = (int)ceilf(fy0 - 0.5f), iy1 = (int)floorf(fy1 + 0.5f);
        *x0 = ix0 < 0 ? 0 : ix0; *x1 = ix1 > W - 1 ? W - 1 : ix1;
        *y0 = iy0 < 0 ? 0 : iy0; *y1 = iy1 > H - 1 ? H - 1 : iy1;
        return *x0 <= *x1 && *y0 <= *y1;
    }
    *x0 = 0; *x1 = W - 1; *y0 = 0; *y1 = H - 1;
    return 1;
}

void orc_rasterize_fwd(int W, int H, int views, const float* clip, int nv,
                       const uint32_t* tri, int nt, int enable_db, float* rast, float* db) {
    const float xs = 2.f / (float)W, ys = 2.f / (float)H;
    size_t npix = (size_t)W * H;
    rtri* setup = (rtri*)malloc(sizeof(rtri) * (size_t)(nt > 0 ? nt : 1));
    float* depth = (float*)malloc(sizeof(float) * npix);
    int* best = (int*)malloc(sizeof(int) * npix);
    float* sxs = (float*)malloc(sizeof(float) * (size_t)W);
    float* sys = (float*)malloc(sizeof(float) * (size_t)H);
    for (int px = 0; px < W; ++px) sxs[px] = (float)(2 * px + 1 - W) / (float)W;
    for (int py = 0; py < H; ++py) sys[py] = (float)(2 * py + 1 - H) / (float)H;
    for (int vw = 0; vw < views; ++vw) {
        const float* cv = clip + (size_t)vw * nv * 4;
        for (size_t i = 0; i < npix; ++i) { depth[i] = 1.f; best[i] = -1; }
        /* triangles in submission order; a later triangle replaces the
         * stored one only when strictly nearer (GL_LESS) */
        for (int t = 0; t < nt; ++t) {
            const float* c0 = cv + (size_t)tri[3 * t] * 4;
            const float* c1 = cv + (size_t)tri[3 * t + 1] * 4;
            const float* c2 = cv + (size_t)tri[3 * t + 2] * 4;
            rtri* T = &setup[t];
            raster_setup(c0, c1, c2, xs, ys, enable_db, T);
            if (raster_outside(c0, c1, c2)) T->valid = 0;
            int bx0, bx1, by0, by1;
            if (!T->valid || !raster_bbox(c0, c1, c2, W, H, &bx0, &bx1, &by0, &by1)) continue;
            for (int py = by0; py <= by1; ++py) {
                float sy = sys[py];
                for (int px = bx0; px <= bx1; ++px) {
                    float sx = sxs[px];
                    float A0 = (T->a[0] * sx + T->b[0] * sy) + T->k[0];
                    float A1 = (T->a[1] * sx + T->b[1] * sy) + T->k[1];
                    float A2 = (T->a[2] * sx + T->b[2] * sy) + T->k[2];
                    if (!edge_in(A0, T->a[0], T->b[0], T->sigma)) continue;
                    if (!edge_in(A1, T->a[1], T->b[1], T->sigma)) continue;
                    if (!edge_in(A2, T->a[2], T->b[2], T->sigma)) continue;
                    float D = (A0 + A1) + A2;
                    if (!(T->sigma * D > 0.f)) continue;
                    float zn = (A0 * T->z[0] + A1 * T->z[1]) + A2 * T->z[2];
                    float wn = (A0 * T->w[0] + A1 * T->w[1]) + A2 * T->w[2];
                    float zw = zn / wn;
                    if (!(zw >= -1.f && zw <= 1.f)) continue;
                    size_t pi = (size_t)py * W + px;
                    if (zw < depth[pi]) { depth[pi] = zw; best[pi] = t; }
                }
            }
        }
        float* rv = rast + (size_t)vw * npix * 4;
        float* dv = db ? db + (size_t)vw * npix * 4 : NULL;
        for (int py = 0; py < H; ++py) {
            float sy = sys[py];
            for (int px = 0; px < W; ++px) {
                float sx = sxs[px];
                size_t pi = (size_t)py * W + px;
                int t = best[pi];
                if (t < 0) {
                    memset(rv + pi * 4, 0, 16);
                    if (dv) memset(dv + pi * 4, 0, 16);
                    continue;
                }
                const rtri* T = &setup[t];
                float A0 = (T->a[0] * sx + T->b[0] * sy) + T->k[0];
                float A1 = (T->a[1] * sx + T->b[1] * sy) + T->k[1];
                float A2 = (T->a[2] * sx + T->b[2] * sy) + T->k[2];
                float D = (A0 + A1) + A2;
                float u = A0 / D, v = A1 / D;
                rv[pi * 4 + 0] = u;
                rv[pi * 4 + 1] = v;
                rv[pi * 4 + 2] = depth[pi];
                rv[pi * 4 + 3] = (float)(t + 1);
                if (dv) {
                    float l2 = (1.f - u) - v;
                    float wi = (u * T->w[0] + v * T->w[1]) + l2 * T->w[2];
                    for (int c = 0; c < 4; ++c)
                        dv[pi * 4 + c] = ((u * T->db[0][c] + v * T->db[1][c]) + l2 * T->db[2][c]) * wi;
                }
            }
        }
    }
    free(setup); free(depth); free(best); free(sxs); free(sys);
}

/* Tie census: the pixels at which a GL implementation may legally differ
 * from the restated rules above.  GL fixes neither the fill rule for a
 * centre exactly on an edge nor (with a 24-bit buffer) equal-depth order, so
 * these are the pixels where a triangle-id mismatch against real GL would be
 * admissible; everywhere else the rules are the same.  Walks every triangle
 * over its raster_bbox() with the same arithmetic as orc_rasterize_fwd. */
void orc_raster_ties(int W, int H, int views, const float* clip, int nv,
                     const uint32_t* tri, int nt, const float* rast,
                     uint32_t* flags, long long* counts) {
    const float xs = 2.f / (float)W, ys = 2.f / (float)H;
    const size_t npix = (size_t)W * H;
    float* sxs = (float*)malloc(sizeof(float) * (size_t)W);
    float* sys = (float*)malloc(sizeof(float) * (size_t)H);
    for (int px = 0; px < W; ++px) sxs[px] = (float)(2 * px + 1 - W) / (float)W;
    for (int py = 0; py < H; ++py) sys[py] = (float)(2 * py + 1 - H) / (float)H;
    memset(flags, 0, sizeof(uint32_t) * npix * (size_t)views);
    (void)nv;
    for (int vw = 0; vw < views; ++vw) {
        const float* cv = clip + (size_t)vw * nv * 4;
        const float* rv = rast + (size_t)vw * npix * 4;
        uint32_t* fv = flags + (size_t)vw * npix;
        for (int t = 0; t < nt; ++t) {
            const float* c0 = cv + (size_t)tri[3 * t] * 4;
            const float* c1 = cv + (size_t)tri[3 * t + 1] * 4;
            const float* c2 = cv + (size_t)tri[3 * t + 2] * 4;
            rtri T;
            raster_setup(c0, c1, c2, xs, ys, 0, &T);
            if (raster_outside(c0, c1, c2)) T.valid = 0;
            int bx0, bx1, by0, by1;
            if (!T.valid || !raster_bbox(c0, c1, c2, W, H, &bx0, &bx1, &by0, &by1)) continue;
            for (int py = by0; py <= by1; ++py) {
                float sy = sys[py];
                for (int px = bx0; px <= bx1; ++px) {
                    float sx = sxs[px];
                    float A[3];
                    int closed = 1, on_edge = 0, in = 1;
                    for (int i = 0; i < 3; ++i) {
                        A[i] = (T.a[i] * sx + T.b[i] * sy) + T.k[i];
                        closed &= T.sigma * A[i] >= 0.f;
                        on_edge |= A[i] == 0.f;
                        in &= edge_in(A[i], T.a[i], T.b[i], T.sigma);
                    }
                    if (!closed) continue;
                    float D = (A[0] + A[1]) + A[2];
                    if (!(T.sigma * D > 0.f)) continue;
                    float zn = (A[0] * T.z[0] + A[1] * T.z[1]) + A[2] * T.z[2];
                    float wn = (A[0] * T.w[0] + A[1] * T.w[1]) + A[2] * T.w[2];
                    float zw = zn / wn;
                    if (!(zw >= -1.f && zw < 1.f)) continue;
                    size_t pi = (size_t)py * W + px;
                    if (on_edge) fv[pi] |= 1u;
                    if (in && rv[pi * 4 + 3] != (float)(t + 1) && rv[pi * 4 + 3] > 0.f && zw == rv[pi * 4 + 2])
                        fv[pi] |= 2u;
                }
            }
        }
    }
    counts[0] = counts[1] = 0;
    for (size_t i = 0; i < npix * (size_t)views; ++i) {
        counts[0] += (flags[i] & 1u) != 0;
        counts[1] += (flags[i] & 2u) != 0;
    }
    free(sxs); free(sys);
}

/* rasterize.cu:84-141 */
void orc_rasterize_bwd(int W, int H, int views, const float* clip, int nv,
                       const uint32_t* tri, const float* rast, const float* gb, float* gclip) {
    const float xs = 2.f / (float)W, ys = 2.f / (float)H;
    for (int vw = 0; vw < views; ++vw) {
        const float* proj = clip + (size_t)vw * nv * 4;
        float* gp = gclip + (size_t)vw * nv * 4;
        for (int py = 0; py < H; ++py)
            for (int px = 0; px < W; ++px) {
                size_t pidx = (size_t)px + (size_t)W * (py + (size_t)H * vw);
                const float* r = rast + pidx * 4;
                int idx = f2i(r[3]) - 1;
                if (idx < 0) continue;
                f2 g = F2(gb[pidx * 2], gb[pidx * 2 + 1]);
                if (g.x == 0.f && g.y == 0.f) continue;   /* both zero (either sign) */
                f2 pix = F2((float)(((double)px + 0.5) * (double)xs - 1.0), (float)(((double)py + 0.5) * (double)ys - 1.0));
                uint32_t i0 = tri[idx * 3], i1 = tri[idx * 3 + 1], i2 = tri[idx * 3 + 2];
                f2 p0 = F2(proj[i0 * 4], proj[i0 * 4 + 1]);
                f2 p1 = F2(proj[i1 * 4], proj[i1 * 4 + 1]);
                f2 p2 = F2(proj[i2 * 4], proj[i2 * 4 + 1]);
                float w0 = proj[i0 * 4 + 3], w1 = proj[i1 * 4 + 3], w2 = proj[i2 * 4 + 3];
                p0 = F2(w0 * pix.x - p0.x, w0 * pix.y - p0.y);
                p1 = F2(w1 * pix.x - p1.x, w1 * pix.y - p1.y);
                p2 = F2(w2 * pix.x - p2.x, w2 * pix.y - p2.y);
                f2 e0 = F2(p0.x - p2.x, p0.y - p2.y);
                f2 e1 = F2(p1.x - p2.x, p1.y - p2.y);
                float a = cross2(e0, e1);
                float ia = 1.f / (a + (a > 0 ? 1e-6f : -1e-6f));
                float kuv = r[0] * g.x + r[1] * g.y;
                float gx0 = (g.y * p2.y + kuv * e1.y) * ia;
                float gy0 = (-g.y * p2.x - kuv * e1.x) * ia;
                float gw0 = -gx0 * pix.x - gy0 * pix.y;
                float gx1 = (-g.x * p2.y - kuv * e0.y) * ia;
                float gy1 = (g.x * p2.x + kuv * e0.x) * ia;
                float gw1 = -gx1 * pix.x - gy1 * pix.y;
                float gx2 = ((-g.y * p0.y + g.x * p1.y) - kuv * (-p0.y + p1.y)) * ia;
                float gy2 = ((g.y * p0.x - g.x * p1.x) - kuv * (p0.x - p1.x)) * ia;
                float gw2 = -gx2 * pix.x - gy2 * pix.y;
                gp[i0 * 4] += gx0; gp[i0 * 4 + 1] += gy0; gp[i0 * 4 + 3] += gw0;
                gp[i1 * 4] += gx1; gp[i1 * 4 + 1] += gy1; gp[i1 * 4 + 3] += gw1;
                gp[i2 * 4] += gx2; gp[i2 * 4 + 1] += gy2; gp[i2 * 4 + 3] += gw2;
            }
    }
}

/* ------------------------------------------------------------------------ */
/* interpolate.cu:20-49 and Interpolate::forward :51-60 (outputs cleared) */
void orc_interpolate_fwd(int W, int H, int views, int dim, int enable_da,
                         const float* rast, const float* db, const float* attr,
                         const uint32_t* tri, float* out, float* out_da) {
    size_t N = (size_t)W * H * views;
    memset(out, 0, N * dim * sizeof(float));
    if (enable_da) memset(out_da, 0, N * dim * 2 * sizeof(float));
    for (size_t pidx = 0; pidx < N; ++pidx) {
        const float* r = rast + pidx * 4;
        int idx = f2i(r[3]) - 1;
        if (idx < 0) continue;
        uint32_t i0 = tri[idx * 3], i1 = tri[idx * 3 + 1], i2 = tri[idx * 3 + 2];
        for (int i = 0; i < dim; ++i) {
            float a0 = attr[(size_t)i0 * dim + i], a1 = attr[(size_t)i1 * dim + i], a2 = attr[(size_t)i2 * dim + i];
            out[pidx * dim + i] = (float)((double)(a0 * r[0] + a1 * r[1]) + (double)a2 * ((1.0 - (double)r[0]) - (double)r[1]));
            if (enable_da) {
                float dadu = a0 - a2, dadv = a1 - a2;
                const float* d = db + pidx * 4;
                out_da[(pidx * dim + i) * 2] = dadu * d[0] + dadv * d[2];
                out_da[(pidx * dim + i) * 2 + 1] = dadu * d[1] + dadv * d[3];
            }
        }
    }
}

/* interpolate.cu:114-143.  compat: the barycentric gradient is stored
 * (:141, overwriting); exact: it is accumulated, so that several
 * interpolations of one raster sum their contributions. */
void orc_interpolate_bwd(int mode, int W, int H, int views, int dim,
                         const float* rast, const float* attr, const uint32_t* tri,
                         const float* g_out, float* g_attr, float* g_bary) {
    size_t N = (size_t)W * H * views;
    for (size_t pidx = 0; pidx < N; ++pidx) {
        const float* r = rast + pidx * 4;
        int idx = f2i(r[3]) - 1;
        if (idx < 0) continue;
        uint32_t i0 = tri[idx * 3], i1 = tri[idx * 3 + 1], i2 = tri[idx * 3 + 2];
        float gu = 0.f, gv = 0.f;
        for (int i = 0; i < dim; ++i) {
            float g = g_out[pidx * dim + i];
            if (g_attr) {
                g_attr[(size_t)i0 * dim + i] += g * r[0];
                g_attr[(size_t)i1 * dim + i] += g * r[1];
                g_attr[(size_t)i2 * dim + i] += (float)((double)g * ((1.0 - (double)r[0]) - (double)r[1]));
            }
            gu += g * (attr[(size_t)i0 * dim + i] - attr[(size_t)i2 * dim + i]);
            gv += g * (attr[(size_t)i1 * dim + i] - attr[(size_t)i2 * dim + i]);
        }
        if (g_bary) {
            if (mode == 0) { g_bary[pidx * 2] = gu; g_bary[pidx * 2 + 1] = gv; }
            else { g_bary[pidx * 2] += gu; g_bary[pidx * 2 + 1] += gv; }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Level count: Texture::init buffer.cu:379-386 with LSB common.cpp:46-79. */
int orc_tex_levels(int tw, int th, int requested) {
    unsigned v = (unsigned)(tw | th);
    int lsb = 0;
    while (v && !(v & 1u)) { v >>= 1; ++lsb; }
    int maxlevel = lsb + 1;
    if (maxlevel > 16) maxlevel = 16;
    return requested < 1 ? 1 : (maxlevel < requested ? maxlevel : requested);
}

size_t orc_tex_level_offset(int tw, int th, int C, int level) {
    size_t off = 0;
    for (int l = 0; l < level; ++l) off += (size_t)(tw >> l) * (size_t)(th >> l) * C;
    return off;
}

/* texturemap.cu:22-47 */
static void calc_level(int tw, int th, int L, const float* da, int* l0, int* l1, float* fl) {
    float dsdx = da[0] * tw, dsdy = da[1] * tw, dtdx = da[2] * th, dtdy = da[3] * th;
    float s2 = dsdx * dsdx + dsdy * dsdy;
    float t2 = dtdx * dtdx + dtdy * dtdy;
    float a = dsdx * dtdy - dtdx * dsdy;
    float b = .5f * (s2 + t2);
    float c = sqrtf(b * b - a * a);
    float level = .5f * log2f(b + c);
    *l0 = level <= 0 ? 0 : (float)(L - 2) <= level ? L - 2 : f2i(floorf(level));
    *l1 = level <= 1 ? 1 : (float)(L - 1) <= level ? L - 1 : f2i(floorf(level)) + 1;
    *fl = level <= 0 ? 0.f : (float)(L - 1) <= level ? 1.f : level - floorf(level);
}

/* texturemap.cu:160-197 (with the dlevel/d(uvDA) Jacobian).  compat keeps the
 * reference's missing factor d on the last two components (:185). */
static void calc_level_jacob(int mode, int tw, int th, int L, const float* da, int* l0, int* l1, float* fl, float* dl) {
    float dsdx = da[0] * tw, dsdy = da[1] * tw, dtdx = da[2] * th, dtdy = da[3] * th;
    float s2 = dsdx * dsdx + dsdy * dsdy;
    float t2 = dtdx * dtdx + dtdy * dtdy;
    float a = dsdx * dtdy - dtdx * dsdy;
    float b = .5f * (s2 + t2);
    float c2 = b * b - a * a;
    float c = sqrtf(c2);
    float level = .5f * log2f(b + c);
    *l0 = level <= 0 ? 0 : (float)(L - 2) <= level ? L - 2 : f2i(floorf(level));
    *l1 = level <= 1 ? 1 : (float)(L - 1) <= level ? L - 1 : f2i(floorf(level)) + 1;
    *fl = level <= 0 ? 0.f : (float)(L - 1) <= level ? 1.f : level - floorf(level);
    float d = b * c + c2;
    if ((double)fabsf(d) > 1e-6) {
        d = 0.72134752f / d;
        float bc = b + c;
        dl[0] = d * (bc * dsdx - a * dtdy);
        dl[1] = d * (bc * dsdy + a * dtdx);
        dl[2] = (bc * dtdx + a * dsdy);
        dl[3] = (bc * dtdy - a * dsdx);
        if (mode != 0) { dl[2] *= d; dl[3] *= d; }
    } else if ((double)fabsf(b) > 1e-6) {
        d = 1 / b;
        dl[0] = d * dsdx; dl[1] = d * dsdy; dl[2] = d * dtdx; dl[3] = d * dtdy;
    } else {
        dl[0] = dl[1] = dl[2] = dl[3] = 0.f;
    }
}

/* texturemap.cu:49-65 */
static void index_fetch(int tw, int th, int level, f2 uv, int idx[4], f2* t) {
    int sx = tw >> level, sy = th >> level;
    float tx = uv.x * (float)sx, ty = uv.y * (float)sy;
    int u0 = tx < 0 ? 0 : tx > (float)(sx - 1) ? sx - 1 : f2i(tx);
    int u1 = tx < 1 ? 0 : tx > (float)(sx - 2) ? sx - 1 : f2i(tx) + 1;
    int v0 = ty < 0 ? 0 : ty > (float)(sy - 1) ? sy - 1 : f2i(ty);
    int v1 = ty < 1 ? 0 : ty > (float)(sy - 2) ? sy - 1 : f2i(ty) + 1;
    idx[0] = v0 * sx + u0; idx[1] = v0 * sx + u1; idx[2] = v1 * sx + u0; idx[3] = v1 * sx + u1;
    t->x = tx < 0 ? 0.f : (float)sx < tx ? 1.f : tx - floorf(tx);
    t->y = ty < 0 ? 0.f : (float)sy < ty ? 1.f : ty - floorf(ty);
}

/* texturemap.cu:67-123: trilinear when the texture has more than one level,
 * bilinear on level 0 otherwise; uncovered pixels stay 0. */
void orc_texture_fwd(int W, int H, int views, int tw, int th, int C, int L,
                     const float* pyr, const float* rast, const float* uv,
                     const float* uv_da, float* out) {
    size_t N = (size_t)W * H * views;
    memset(out, 0, N * C * sizeof(float));
    for (size_t pidx = 0; pidx < N; ++pidx) {
        if (rast[pidx * 4 + 3] < 1.f) continue;
        f2 u = F2(uv[pidx * 2], uv[pidx * 2 + 1]);
        if (L > 1) {
            int l0, l1; float fl;
            calc_level(tw, th, L, uv_da + pidx * 4, &l0, &l1, &fl);
            int i0[4], i1[4]; f2 t0, t1;
            index_fetch(tw, th, l0, u, i0, &t0);
            index_fetch(tw, th, l1, u, i1, &t1);
            const float* T0 = pyr + orc_tex_level_offset(tw, th, C, l0);
            const float* T1 = pyr + orc_tex_level_offset(tw, th, C, l1);
            for (int i = 0; i < C; ++i) {
                float o = bilerp_(T0[i0[0] * C + i], T0[i0[1] * C + i], T0[i0[2] * C + i], T0[i0[3] * C + i], t0);
                if (fl > 0) {
                    float o1 = bilerp_(T1[i1[0] * C + i], T1[i1[1] * C + i], T1[i1[2] * C + i], T1[i1[3] * C + i], t1);
                    o = lerpf_(o, o1, fl);
                }
                out[pidx * C + i] = o;
            }
        } else {
            int i0[4]; f2 t0;
            index_fetch(tw, th, 0, u, i0, &t0);
            for (int i = 0; i < C; ++i)
                out[pidx * C + i] = bilerp_(pyr[i0[0] * C + i], pyr[i0[1] * C + i], pyr[i0[2] * C + i], pyr[i0[3] * C + i], t0);
        }
    }
}

/* texturemap.cu:229-319 */
void orc_texture_bwd(int mode, int W, int H, int views, int tw, int th, int C, int L,
                     const float* pyr, const float* rast, const float* uv,
                     const float* uv_da, const float* g_out, float* g_pyr,
                     float* g_uv, float* g_uv_da) {
    size_t N = (size_t)W * H * views;
    for (size_t pidx = 0; pidx < N; ++pidx) {
        if (rast[pidx * 4 + 3] < 1.f) continue;
        f2 u = F2(uv[pidx * 2], uv[pidx * 2 + 1]);
        if (L > 1) {
            int l0 = 0, l1 = 0; float fl = 0.f, dl[4];
            calc_level_jacob(mode, tw, th, L, uv_da + pidx * 4, &l0, &l1, &fl, dl);
            int i0[4], i1[4]; f2 t0, t1;
            index_fetch(tw, th, l0, u, i0, &t0);
            index_fetch(tw, th, l1, u, i1, &t1);
            const float* T0 = pyr + orc_tex_level_offset(tw, th, C, l0);
            const float* T1 = pyr + orc_tex_level_offset(tw, th, C, l1);
            float* G0 = g_pyr ? g_pyr + orc_tex_level_offset(tw, th, C, l0) : NULL;
            float* G1 = g_pyr ? g_pyr + orc_tex_level_offset(tw, th, C, l1) : NULL;
            float gu = 0.f, gv = 0.f, gl = 0.f;
            for (int i = 0; i < C; ++i) {
                float g = g_out[pidx * C + i];
                if (G0) {
                    G0[i0[0] * C + i] += (1.f - fl) * (1.f - t0.x) * (1.f - t0.y) * g;
                    G0[i0[1] * C + i] += (1.f - fl) * t0.x * (1.f - t0.y) * g;
                    G0[i0[2] * C + i] += (1.f - fl) * (1.f - t0.x) * t0.y * g;
                    G0[i0[3] * C + i] += (1.f - fl) * t0.x * t0.y * g;
                }
                float t00 = T0[i0[0] * C + i], t01 = T0[i0[1] * C + i], t10 = T0[i0[2] * C + i], t11 = T0[i0[3] * C + i];
                float du = lerpf_(t01 - t00, t11 - t10, t0.y) * (float)(tw >> l0);
                float dv = lerpf_(t10 - t00, t11 - t01, t0.x) * (float)(th >> l0);
                if (fl > 0 && L > 1) {
                    float l = bilerp_(t00, t01, t10, t11, t0);
                    if (G1) {
                        G1[i1[0] * C + i] += fl * (1.f - t1.x) * (1.f - t1.y) * g;
                        G1[i1[1] * C + i] += fl * t1.x * (1.f - t1.y) * g;
                        G1[i1[2] * C + i] += fl * (1.f - t1.x) * t1.y * g;
                        G1[i1[3] * C + i] += fl * t1.x * t1.y * g;
                    }
                    t00 = T1[i1[0] * C + i]; t01 = T1[i1[1] * C + i]; t10 = T1[i1[2] * C + i]; t11 = T1[i1[3] * C + i];
                    du = lerpf_(du, lerpf_(t01 - t00, t11 - t10, t1.y) * (float)(tw >> l1), fl);
                    dv = lerpf_(dv, lerpf_(t10 - t00, t11 - t01, t1.x) * (float)(th >> l1), fl);
                    gl += (bilerp_(t00, t01, t10, t11, t1) - l) * g;
                }
                gu += du * g;
                gv += dv * g;
            }
            if (g_uv) { g_uv[pidx * 2] = gu; g_uv[pidx * 2 + 1] = gv; }
            if (g_uv_da) for (int c = 0; c < 4; ++c) g_uv_da[pidx * 4 + c] = gl * dl[c];
        } else {
            int i0[4]; f2 t0;
            index_fetch(tw, th, 0, u, i0, &t0);
            float gu = 0.f, gv = 0.f;
            for (int i = 0; i < C; ++i) {
                float g = g_out[pidx * C + i];
                if (g_pyr) {
                    g_pyr[i0[0] * C + i] += (1.f - t0.x) * (1.f - t0.y) * g;
                    g_pyr[i0[1] * C + i] += t0.x * (1.f - t0.y) * g;
                    g_pyr[i0[2] * C + i] += (1.f - t0.x) * t0.y * g;
                    g_pyr[i0[3] * C + i] += t0.x * t0.y * g;
                }
                float t00 = pyr[i0[0] * C + i], t01 = pyr[i0[1] * C + i], t10 = pyr[i0[2] * C + i], t11 = pyr[i0[3] * C + i];
                float du = lerpf_(t01 - t00, t11 - t10, t0.y) * (float)tw;
                float dv = lerpf_(t10 - t00, t11 - t01, t0.x) * (float)th;
                gu += du * g;
                gv += dv * g;
            }
            if (g_uv) { g_uv[pidx * 2] = gu; g_uv[pidx * 2 + 1] = gv; }
        }
    }
}

/* buffer.cu:449-484: level i = 2x2 box average of level i-1. */
void orc_mip_build(int tw, int th, int C, int L, float* pyr) {
    for (int i = 1; i < L; ++i) {
        int w = tw >> i, h = th >> i, pw = w << 1;
        const float* src = pyr + orc_tex_level_offset(tw, th, C, i - 1);
        float* dst = pyr + orc_tex_level_offset(tw, th, C, i);
        for (int py = 0; py < h; ++py)
            for (int px = 0; px < w; ++px) {
                size_t p00 = (size_t)(2 * px) + (size_t)pw * (2 * py);
                size_t p01 = p00 + 1, p10 = p00 + pw, p11 = p10 + 1;
                for (int c = 0; c < C; ++c)
                    dst[((size_t)px + (size_t)w * py) * C + c] =
                        (src[p00 * C + c] + src[p01 * C + c] + src[p10 * C + c] + src[p11 * C + c]) * 0.25f;
            }
    }
}

/* buffer.cu:615-648: push each level's gradient to its four children,
 * coarsest first.  compat: weight 1 (:630-633); exact: 1/4, the adjoint of
 * the 2x2 average. */
void orc_mip_pushdown(int mode, int tw, int th, int C, int L, float* g) {
    for (int i = L - 1; i > 0; --i) {
        int w = tw >> i, h = th >> i, pw = w << 1;
        const float* src = g + orc_tex_level_offset(tw, th, C, i);
        float* dst = g + orc_tex_level_offset(tw, th, C, i - 1);
        for (int py = 0; py < h; ++py)
            for (int px = 0; px < w; ++px) {
                size_t p00 = (size_t)(2 * px) + (size_t)pw * (2 * py);
                size_t p01 = p00 + 1, p10 = p00 + pw, p11 = p10 + 1;
                for (int c = 0; c < C; ++c) {
                    float v = src[((size_t)px + (size_t)w * py) * C + c];
                    if (mode != 0) v *= 0.25f;
                    add_nan_check(&dst[p00 * C + c], v);
                    add_nan_check(&dst[p01 * C + c], v);
                    add_nan_check(&dst[p10 * C + c], v);
                    add_nan_check(&dst[p11 * C + c], v);
                }
            }
    }
}

/* common.h:154 clamp via buffer.cu:65-72 */
void orc_clamp(size_t n, float* p, float lo, float hi) {
    for (size_t i = 0; i < n; ++i) { float a = p[i]; p[i] = a < lo ? lo : a > hi ? hi : a; }
}

/* ------------------------------------------------------------------------ */
/* antialias.cu:17-35 */
static void aa_edge_fwd(int C, const float* in, float* out, size_t pidx, size_t oidx, f2 pa, f2 pb, f2 o) {
    float a = cross2(pa, pb);
    float oa = cross2(F2(pa.x - o.x, pa.y - o.y), F2(pb.x - o.x, pb.y - o.y));
    if (a * oa > 0.f) return;
    f2 e = F2(pa.x - pb.x, pa.y - pb.y);
    float n = (o.x + o.y) * (o.x - o.y);
    if ((e.x + e.y) * (e.x - e.y) * n > 0.f) return;
    e.x *= (o.x + o.y); e.y *= (o.x + o.y);
    float D = n > 0.f ? -e.y : e.x;
    float ia = (float)(1.0 / ((double)D + (D > 0 ? 1e-3 : -1e-3)));
    float alpha = a * ia - .5f;
    for (int i = 0; i < C; ++i) {
        float diff = in[pidx * C + i] - in[oidx * C + i];
        if (alpha > 0) out[oidx * C + i] += alpha * diff;
        else out[pidx * C + i] += alpha * diff;
    }
}

typedef struct { f2 v[3]; f2 ndc[3]; float iw[3]; uint32_t id[3]; } aa_tri;

/* antialias.cu:37-55 and :240-257: the triangle of pixel `pidx` in
 * pixel units relative to f. Returns 0 when the pixel is background. */
static int aa_fetch(const float* proj, const uint32_t* tri, const float* rast, size_t pidx, f2 s, f2 f, aa_tri* t) {
    int idx = f2i(rast[pidx * 4 + 3]) - 1;
    if (idx < 0) return 0;
    for (int k = 0; k < 3; ++k) {
        uint32_t vi = tri[idx * 3 + k];
        t->id[k] = vi;
        f2 v = F2(proj[vi * 4], proj[vi * 4 + 1]);
        t->iw[k] = 1.f / proj[vi * 4 + 3];
        t->ndc[k] = F2(v.x * t->iw[k], v.y * t->iw[k]);
        t->v[k] = F2((v.x * t->iw[k] + 1.f) * s.x - f.x, (v.y * t->iw[k] + 1.f) * s.y - f.y);
    }
    return 1;
}

void orc_antialias_fwd(int W, int H, int views, int C, const float* clip, int nv,
                       const uint32_t* tri, const float* rast, const float* in, float* out) {
    size_t N = (size_t)W * H * views;
    memcpy(out, in, N * C * sizeof(float));
    f2 s = F2(W / 2.f, H / 2.f);
    for (int vw = 0; vw < views; ++vw) {
        const float* proj = clip + (size_t)vw * nv * 4;
        for (int py = 0; py < H; ++py)
            for (int px = 0; px < W; ++px) {
                size_t pidx = (size_t)px + (size_t)W * (py + (size_t)H * vw);
                f2 tr = F2(rast[pidx * 4 + 2], rast[pidx * 4 + 3]);
                f2 th = px > 0 ? F2(rast[(pidx - 1) * 4 + 2], rast[(pidx - 1) * 4 + 3]) : tr;
                f2 tv = py > 0 ? F2(rast[(pidx - W) * 4 + 2], rast[(pidx - W) * 4 + 3]) : tr;
                if (th.y != tr.y) {
                    size_t oidx = pidx - 1;
                    size_t pp = f2i(tr.y) ? pidx : oidx;
                    size_t op = f2i(th.y) ? pidx : oidx;
                    if (pp == op) { if (tr.x > th.x) op = oidx; else pp = oidx; }
                    f2 f = F2((float)px + (pp > op ? .5f : -.5f), (float)py + .5f);
                    f2 o = F2(pp > op ? -1.f : 1.f, 0.f);
                    aa_tri t;
                    if (aa_fetch(proj, tri, rast, pp, s, f, &t)) {
                        aa_edge_fwd(C, in, out, pp, op, t.v[0], t.v[1], o);
                        aa_edge_fwd(C, in, out, pp, op, t.v[1], t.v[2], o);
                        aa_edge_fwd(C, in, out, pp, op, t.v[2], t.v[0], o);
                    }
                }
                if (tv.y != tr.y) {
                    size_t oidx = pidx - W;
                    size_t pp = f2i(tr.y) ? pidx : oidx;
                    size_t op = f2i(tv.y) ? pidx : oidx;
                    if (pp == op) { if (tr.x > tv.x) op = oidx; else pp = oidx; }
                    f2 f = F2((float)px + .5f, (float)py + (pp > op ? .5f : -.5f));
                    f2 o = F2(0.f, pp > op ? -1.f : 1.f);
                    aa_tri t;
                    if (aa_fetch(proj, tri, rast, pp, s, f, &t)) {
                        aa_edge_fwd(C, in, out, pp, op, t.v[0], t.v[1], o);
                        aa_edge_fwd(C, in, out, pp, op, t.v[1], t.v[2], o);
                        aa_edge_fwd(C, in, out, pp, op, t.v[2], t.v[0], o);
                    }
                }
            }
    }
}

/* antialias.cu:196-240.  The w gradient: a vertex's pixel position is
 * (x/w + 1) s - f, so d/dw = -(x/w) s / w and dL/dw = -(dL/dx' . x/w) with
 * dL/dx' the x,y gradient already scaled by s/w.  The reference multiplies
 * by the pixel position relative to f instead of x/w (:241-242); exact uses
 * x/w (`na`, `nb`). */
static void aa_edge_bwd(int exact, int C, const float* in, const float* g_out, float* g_in, float* g_clip,
                        size_t pidx, size_t oidx, f2 pa, f2 pb, f2 na, f2 nb, uint32_t ia_, uint32_t ib_,
                        float iwa, float iwb, f2 o, f2 s) {
    float a = cross2(pa, pb);
    float oa = cross2(F2(pa.x - o.x, pa.y - o.y), F2(pb.x - o.x, pb.y - o.y));
    if (a * oa > 0.f) return;
    f2 e = F2(pa.x - pb.x, pa.y - pb.y);
    float n = (o.x + o.y) * (o.x - o.y);
    if ((e.x + e.y) * (e.x - e.y) * n > 0.f) return;
    e.x *= (o.x + o.y); e.y *= (o.x + o.y);
    float D = n > 0.f ? -e.y : e.x;
    float ia = (float)(1.0 / ((double)D + (D > 0 ? 1e-3 : -1e-3)));
    float alpha = a * ia - .5f;
    float d = 0.f;
    for (int i = 0; i < C; ++i) {
        float g = alpha > 0 ? g_out[oidx * C + i] : g_out[pidx * C + i];
        float diff = in[pidx * C + i] - in[oidx * C + i];
        if (g_in) {
            g_in[pidx * C + i] += alpha * g;
            g_in[oidx * C + i] += -alpha * g;
        }
        d += g * diff;
    }
    if (g_clip) {
        d *= ia;
        f2 da = F2(d * s.x * iwa, d * s.y * iwa);
        f2 db = F2(d * s.x * iwb, d * s.y * iwb);
        float r = n > 0 ? e.x : -e.y;
        r *= ia;
        if (n > 0) {
            da.x *= pb.y; da.y *= pb.y; da.y *= r;
            db.x *= -pa.y; db.y *= -pa.y; db.y *= r;
        } else {
            da.x *= -pb.x; da.y *= -pb.x; da.x *= r;
            db.x *= pa.x; db.y *= pa.x; db.x *= r;
        }
        f2 wa = exact ? na : pa, wb = exact ? nb : pb;
        g_clip[ia_ * 4] += da.x; g_clip[ia_ * 4 + 1] += da.y; g_clip[ia_ * 4 + 3] += -(da.x * wa.x + da.y * wa.y);
        g_clip[ib_ * 4] += db.x; g_clip[ib_ * 4 + 1] += db.y; g_clip[ib_ * 4 + 3] += -(db.x * wb.x + db.y * wb.y);
    }
}

/* antialias.cu:261-300.  compat keeps the horizontal-edge typo of :279
 * (the current pixel's id used for both sides), under which a background
 * current pixel makes the reference fetch triangle -1 out of bounds; that
 * fetch contributes nothing here.  exact uses the neighbour's id, as the
 * forward pass does (:74), and the corrected w gradient (aa_edge_bwd). */
void orc_antialias_bwd(int mode, int W, int H, int views, int C, const float* clip, int nv,
                       const uint32_t* tri, const float* rast, const float* in,
                       const float* g_out, float* g_in, float* g_clip) {
    size_t N = (size_t)W * H * views;
    if (g_in) memcpy(g_in, g_out, N * C * sizeof(float));
    f2 s = F2(W / 2.f, H / 2.f);
    for (int vw = 0; vw < views; ++vw) {
        const float* proj = clip + (size_t)vw * nv * 4;
        float* gc = g_clip ? g_clip + (size_t)vw * nv * 4 : NULL;
        for (int py = 0; py < H; ++py)
            for (int px = 0; px < W; ++px) {
                size_t pidx = (size_t)px + (size_t)W * (py + (size_t)H * vw);
                f2 tr = F2(rast[pidx * 4 + 2], rast[pidx * 4 + 3]);
                f2 th = px > 0 ? F2(rast[(pidx - 1) * 4 + 2], rast[(pidx - 1) * 4 + 3]) : tr;
                f2 tv = py > 0 ? F2(rast[(pidx - W) * 4 + 2], rast[(pidx - W) * 4 + 3]) : tr;
                if (th.y != tr.y) {
                    size_t oidx = pidx - 1;
                    size_t pp = f2i(tr.y) ? pidx : oidx;
                    size_t op = f2i(mode == 0 ? tr.y : th.y) ? pidx : oidx;
                    if (pp == op) { if (tr.x > th.x) op = oidx; else pp = oidx; }
                    f2 f = F2((float)px + (pp > op ? .5f : -.5f), (float)py + .5f);
                    f2 o = F2(pp > op ? -1.f : 1.f, 0.f);
                    aa_tri t;
                    if (aa_fetch(proj, tri, rast, pp, s, f, &t)) {
                        for (int k = 0; k < 3; ++k) {
                            int k2 = (k + 1) % 3;
                            aa_edge_bwd(mode != 0, C, in, g_out, g_in, gc, pp, op, t.v[k], t.v[k2], t.ndc[k], t.ndc[k2],
                                        t.id[k], t.id[k2], t.iw[k], t.iw[k2], o, s);
                        }
                    }
                }
                if (tv.y != tr.y) {
                    size_t oidx = pidx - W;
                    size_t pp = f2i(tr.y) ? pidx : oidx;
                    size_t op = f2i(tv.y) ? pidx : oidx;
                    if (pp == op) { if (tr.x > tv.x) op = oidx; else pp = oidx; }
                    f2 f = F2((float)px + .5f, (float)py + (pp > op ? .5f : -.5f));
                    f2 o = F2(0.f, pp > op ? -1.f : 1.f);
                    aa_tri t;
                    if (aa_fetch(proj, tri, rast, pp, s, f, &t)) {
                        for (int k = 0; k < 3; ++k) {
                            int k2 = (k + 1) % 3;
                            aa_edge_bwd(mode != 0, C, in, g_out, g_in, gc, pp, op, t.v[k], t.v[k2], t.ndc[k], t.ndc[k2],
                                        t.id[k], t.id[k2], t.iw[k], t.iw[k2], o, s);
                        }
                    }
                }
            }
    }
}

/* ------------------------------------------------------------------------ */
/* material.cu:25-48 (the branch the reference reaches with a normal map
 * bound; its normal-map code at :50-68 is unreachable, see :40). */
void orc_normal_axis_fwd(int W, int H, int views, const float* rast, const float* rot,
                         const float* normal, const uint32_t* tri, float* out) {
    size_t N = (size_t)W * H * views;
    memset(out, 0, N * 3 * sizeof(float));
    for (size_t pidx = 0; pidx < N; ++pidx) {
        const float* r = rast + pidx * 4;
        int idx = f2i(r[3]) - 1;
        if (idx < 0) continue;
        f3 n2 = ld3(normal, tri[idx * 3 + 2]);
        f3 n0 = sub3(ld3(normal, tri[idx * 3]), n2);
        f3 n1 = sub3(ld3(normal, tri[idx * 3 + 1]), n2);
        f3 Nn = normalize3(add3(add3(mul3s(n0, r[0]), mul3s(n1, r[1])), n2));
        out[pidx * 3] = rot[0] * Nn.x + rot[4] * Nn.y + rot[8] * Nn.z;
        out[pidx * 3 + 1] = rot[1] * Nn.x + rot[5] * Nn.y + rot[9] * Nn.z;
        out[pidx * 3 + 2] = rot[2] * Nn.x + rot[6] * Nn.y + rot[10] * Nn.z;
    }
}

/* material.cu:92-108; pvinv is a column-major 3x3 per view. */
void orc_view_axis_fwd(int W, int H, int views, const float* pvinv, float* out) {
    for (int vw = 0; vw < views; ++vw) {
        const float* M = pvinv + (size_t)vw * 9;
        f3 c0 = F3(M[0], M[1], M[2]), c1 = F3(M[3], M[4], M[5]), c2 = F3(M[6], M[7], M[8]);
        for (int py = 0; py < H; ++py)
            for (int px = 0; px < W; ++px) {
                size_t pidx = (size_t)px + (size_t)W * (py + (size_t)H * vw);
                float sx = (float)px / (float)W * 2.f - 1.f;
                float sy = (float)py / (float)H * 2.f - 1.f;
                f3 v = normalize3(add3(add3(mul3s(c0, sx), mul3s(c1, sy)), c2));
                out[pidx * 3] = v.x; out[pidx * 3 + 1] = v.y; out[pidx * 3 + 2] = v.z;
            }
    }
}

/* material.cu:145-183 */
void orc_sg_specular_fwd(int W, int H, int views, const float* rast, const float* normal,
                         const float* view, const float* rough, float ior,
                         float* o_axis, float* o_sharp, float* o_amp) {
    size_t N = (size_t)W * H * views;
    memset(o_axis, 0, N * 3 * sizeof(float));
    memset(o_sharp, 0, N * sizeof(float));
    memset(o_amp, 0, N * sizeof(float));
    for (size_t pidx = 0; pidx < N; ++pidx) {
        int idx = f2i(rast[pidx * 4 + 3]) - 1;
        if (idx < 0) continue;
        f3 n = ld3(normal, pidx);
        f3 v = ld3(view, pidx); v = F3(-v.x, -v.y, -v.z);
        f3 p = sub3(mul3s(n, 2.f * dot3(v, n)), v);
        float m = rough[pidx], m2 = m * m;
        float vn = fmaxf(dot3(v, n), 0.f), vn2 = vn * vn;
        float iGv = sqrtf(vn2 + m2 * (1.f - vn2));
        float Gv = (float)(1.0 / fmax((double)(vn + iGv), 1e-6));
        float pn = fmaxf(dot3(p, n), 0.f), pn2 = pn * pn;
        float iGp = sqrtf(pn2 + m2 * (1.f - pn2));
        float Gp = (float)(1.0 / fmax((double)(pn + iGp), 1e-6));
        float g = sqrtf(ior * ior - 1.f + pn2);
        float gp = g + pn, gm = g - pn;
        float f0 = gm / gp;
        float f1 = (pn * gp - 1.f) / (pn * gm + 1.f);
        float F = f0 * f0 * (1.f + f1 * f1);
        o_axis[pidx * 3] = p.x; o_axis[pidx * 3 + 1] = p.y; o_axis[pidx * 3 + 2] = p.z;
        o_amp[pidx] = (float)((double)(F * Gp * Gv * pn) / fmax((double)m2, 1e-6));
        o_sharp[pidx] = (float)(0.5 / fmax((double)(m2 * vn), 1e-6));
    }
}

/* material.cu:203-249 (gradient to roughness only) */
void orc_sg_specular_bwd(int W, int H, int views, const float* rast, const float* normal,
                         const float* view, const float* rough, float ior,
                         const float* g_amp, const float* g_sharp, float* g_rough) {
    size_t N = (size_t)W * H * views;
    for (size_t pidx = 0; pidx < N; ++pidx) {
        int idx = f2i(rast[pidx * 4 + 3]) - 1;
        if (idx < 0) continue;
        f3 n = ld3(normal, pidx);
        f3 v = ld3(view, pidx); v = F3(-v.x, -v.y, -v.z);
        f3 p = sub3(mul3s(n, 2.f * dot3(v, n)), v);
        float m = rough[pidx], m2 = m * m;
        float vn = fmaxf(dot3(v, n), 0.f), vn2 = vn * vn;
        float iGv = sqrtf(vn2 + m2 * (1.f - vn2));
        float Gv = (float)(1.0 / fmax((double)(vn + iGv), 1e-6));
        float dGvdm = (float)((double)(-m * (1.f - vn2)) / fmax((double)iGv, 1e-6) * Gv * Gv);
        float pn = fmaxf(dot3(p, n), 0.f), pn2 = pn * pn;
        float iGp = sqrtf(pn2 + m2 * (1.f - pn2));
        float Gp = (float)(1.0 / fmax((double)(pn + iGp), 1e-6));
        float dGpdm = (float)((double)(-m * (1.f - pn2)) / fmax((double)iGp, 1e-6) * Gp * Gp);
        float g = sqrtf(ior * ior - 1.f + pn2);
        float gp = g + pn, gm = g - pn;
        float f0 = gm / gp;
        float f1 = (pn * gp - 1.f) / (pn * gm + 1.f);
        float F = f0 * f0 * (1.f + f1 * f1);
        double t1 = (double)(-2.f * Gp * Gv) / fmax((double)(m2 * m), 1e-6)
                  + (double)(Gp * dGvdm + Gv * dGpdm) / fmax((double)m2, 1e-6);
        add_nan_check(&g_rough[pidx], (float)((double)(g_amp[pidx] * F * pn) * t1));
        add_nan_check(&g_rough[pidx], (float)((double)(g_sharp[pidx] * -1.f) / fmax((double)(m2 * m * vn), 1e-6)));
    }
}

#define DIFF_SHARP 2.133f
#define DIFF_AMP 2.34f

/* material.cu:285-334 */
void orc_sg_fwd(int W, int H, int views, int C, const float* rast, int K,
                const float* axis, const float* sharp, const float* amp,
                const float* normal, const float* diffuse,
                const float* spec_axis, const float* spec_sharp, const float* spec_amp,
                float* out, float* o_diff, float* o_spec) {
    size_t N = (size_t)W * H * views;
    memset(out, 0, N * C * sizeof(float));
    memset(o_diff, 0, N * C * sizeof(float));
    memset(o_spec, 0, N * C * sizeof(float));
    for (size_t pidx = 0; pidx < N; ++pidx) {
        int idx = f2i(rast[pidx * 4 + 3]) - 1;
        if (idx < 0) continue;
        f3 n = ld3(normal, pidx);
        f3 diffn = mul3s(n, DIFF_SHARP);
        f3 p = ld3(spec_axis, pidx);
        float ss = spec_sharp[pidx], sa = spec_amp[pidx];
        f3 specn = mul3s(p, ss);
        for (int i = 0; i < K; ++i) {
            float gs = sharp[i];
            f3 sgn = mul3s(ld3(axis, i), gs);
            float dl = len3(add3(diffn, sgn));
            float dg = (float)((double)(expf(dl - DIFF_SHARP - gs) - expf(-dl - DIFF_SHARP - gs)) / fmax((double)dl, 1e-6) * (double)DIFF_AMP);
            float sl = len3(add3(specn, sgn));
            float sg = (float)((double)(expf(sl - ss - gs) - expf(-sl - ss - gs)) / fmax((double)sl, 1e-6) * (double)sa);
            for (int k = 0; k < C; ++k) {
                float a = amp[i * C + k];
                add_nan_check(&o_diff[pidx * C + k], dg * a);
                add_nan_check(&o_spec[pidx * C + k], sg * a);
            }
        }
        for (int k = 0; k < C; ++k) {
            size_t j = pidx * C + k;
            out[j] = diffuse[j] * o_diff[j] + o_spec[j];
        }
    }
}

/* material.cu:369-438.  Per-lobe gradients (axis, sharpness, amplitude) are
 * sums over all pixels.  exact also replaces the reference's sharpness
 * derivative of the lobe lengths (see below).  compat keeps the reference's specular-lobe
 * gradient indexing: sharpness at [lobe] (:436) and amplitude at
 * [pixel*C + channel] (:430; the caller sizes that buffer N*C).  exact
 * writes both per pixel and uses d(specg)/d(spec amplitude) for the
 * amplitude. */
void orc_sg_bwd(int mode, int W, int H, int views, int C, const float* rast, int K,
                const float* axis, const float* sharp, const float* amp,
                const float* normal, const float* diffuse,
                const float* spec_axis, const float* spec_sharp, const float* spec_amp,
                const float* g_out, float* g_diffuse,
                float* g_axis, float* g_sharp, float* g_amp,
                float* g_spec_axis, float* g_spec_sharp, float* g_spec_amp) {
    size_t N = (size_t)W * H * views;
    /* The lobe gradients (and, in compat, the lobe-indexed specular sharpness
     * gradient) are sums over every covered pixel: accumulated in double and
     * added to the outputs once, so that the checker's value is the sum of the
     * per-pixel terms to far below FP32 rounding however many pixels there
     * are (a serial FP32 sum over a megapixel drifts by ~1e-5 relative).  The
     * per-pixel terms themselves are FP32, as in the reference. */
    double* acc = (double*)calloc((size_t)K * (C + 5), sizeof(double));
    double* acc_amp = acc;
    double* acc_axis = acc + (size_t)K * C;
    double* acc_sharp = acc_axis + (size_t)K * 3;
    double* acc_ss = acc_sharp + K;
    for (size_t pidx = 0; pidx < N; ++pidx) {
        int idx = f2i(rast[pidx * 4 + 3]) - 1;
        if (idx < 0) continue;
        f3 n = ld3(normal, pidx);
        f3 diffn = mul3s(n, DIFF_SHARP);
        f3 p = ld3(spec_axis, pidx);
        float ss = spec_sharp[pidx], sa = spec_amp[pidx];
        f3 specn = mul3s(p, ss);
        for (int i = 0; i < K; ++i) {
            float gs = sharp[i];
            f3 sgn = mul3s(ld3(axis, i), gs);
            f3 dsum = add3(diffn, sgn);
            float dl = len3(dsum);
            float il = (float)(1.0 / fmax((double)dl, 1e-6));
            /* d|v|/ds for v = c*u + s*a is (a.v)/|v|; the reference has
             * (s + c*(s*a).u)/|v| (material.cu:405,413-414).  exact uses the
             * derivative, and (u.v)/|v| for the specular sharpness. */
            f3 ax = ld3(axis, i);
            float dotn = mode != 0 ? dot3(ax, dsum) * il : (gs + DIFF_SHARP * dot3(sgn, n)) * il;
            float em = expf(dl - DIFF_SHARP - gs), ep = expf(-dl - DIFF_SHARP - gs);
            float dg = (em - ep) * il * DIFF_AMP;
            f3 ddg = mul3s(mul3s(dsum, ((1.f - il) * em + (1.f + il) * ep) * il), il);
            float ddgs = ((dotn * (1.f - il) - 1.f) * em + (dotn * (1.f + il) + 1.f) * ep) * il;

            f3 ssum = add3(specn, sgn);
            float sl = len3(ssum);
            il = (float)(1.0 / fmax((double)sl, 1e-6));
            dotn = mode != 0 ? dot3(ax, ssum) * il : (gs + ss * dot3(sgn, p)) * il;
            float dotp = mode != 0 ? dot3(p, ssum) * il : (gs * dot3(sgn, p) + ss) * il;
            em = expf(sl - ss - gs); ep = expf(-sl - ss - gs);
            float sgv = (em - ep) * il * sa;
            f3 dsg = mul3s(mul3s(ssum, ((1.f - il) * em + (1.f + il) * ep) * il), il);
            float dsgs = ((dotn * (1.f - il) - 1.f) * em + (dotn * (1.f + il) + 1.f) * ep) * il;
            float dsgss = ((dotp * (1.f - il) - 1.f) * em + (dotp * (1.f + il) + 1.f) * ep) * il;

            float sum = 0.f, sumd = 0.f, sum_exact_sa = 0.f;
            for (int k = 0; k < C; ++k) {
                float g = g_out[pidx * C + k];
                float a = amp[i * C + k];
                sum += g * a;
                sumd += g * a * diffuse[pidx * C + k];
                if (g_amp) add_nan_check_d(&acc_amp[i * C + k], g * (dg * diffuse[pidx * C + k] + sgv));
                if (g_diffuse) add_nan_check(&g_diffuse[pidx * C + k], g * dg * a);
                if (g_spec_amp) {
                    if (mode == 0) add_nan_check(&g_spec_amp[pidx * C + k], g * sgv * a);
                    else sum_exact_sa += g * (em - ep) * il * a;
                }
            }
            if (g_spec_amp && mode != 0) add_nan_check(&g_spec_amp[pidx], sum_exact_sa);
            if (g_axis) {
                f3 t = add3(mul3s(mul3s(ddg, sumd), DIFF_AMP), mul3s(mul3s(dsg, sum), sa));
                add_nan_check3_d(&acc_axis[i * 3], mul3s(t, gs));
            }
            if (g_sharp) add_nan_check_d(&acc_sharp[i], sumd * ddgs * DIFF_AMP + sum * dsgs * sa);
            if (g_spec_axis) add_nan_check3(&g_spec_axis[pidx * 3], mul3s(mul3s(mul3s(dsg, sum), sa), ss));
            if (g_spec_sharp) {
                if (mode == 0) add_nan_check_d(&acc_ss[i], sum * dsgss * sa);
                else add_nan_check(&g_spec_sharp[pidx], sum * dsgss * sa);
            }
        }
    }
    for (int i = 0; i < K; ++i) {
        for (int k = 0; k < C; ++k)
            if (g_amp) add_nan_check(&g_amp[i * C + k], (float)acc_amp[i * C + k]);
        if (g_axis) add_nan_check3(&g_axis[i * 3], F3((float)acc_axis[i * 3], (float)acc_axis[i * 3 + 1], (float)acc_axis[i * 3 + 2]));
        if (g_sharp) add_nan_check(&g_sharp[i], (float)acc_sharp[i]);
        if (g_spec_sharp && mode == 0) add_nan_check(&g_spec_sharp[i], (float)acc_ss[i]);
    }
    free(acc);
}

/* ------------------------------------------------------------------------ */
/* loss.cu:22-57.  grad = pred - target.  compat returns the reference's
 * reported loss: its in-place tree reduction replayed with the launch
 * shapes of getBlock (common.cpp:3-29) and the serial thread order, which
 * drops elements at index >= 2^msb(n) and re-adds some partial sums where a
 * block overhangs its row (loss.cu:73-80 has no x bound).  exact returns
 * sum(grad^2)/2 accumulated in double. */
static void get_block(int width, int height, int* bx, int* by) {
    const int M = 16;
    if (width >= M && height >= M) { *bx = M; *by = M; }
    else if (width >= M) { int w = M * M, h = 1; while (h < height) { w >>= 1; h <<= 1; } *bx = w; *by = h; }
    else if (height >= M) { int w = 1, h = M * M; while (w < width) { w <<= 1; h >>= 1; } *bx = w; *by = h; }
    else { int w = 1, h = 1; while (w < width) w <<= 1; while (h < height) h <<= 1; *bx = w; *by = h; }
}

static int msb_index(size_t v) { int m = -1; while (v) { v >>= 1; ++m; } return m < 0 ? 0 : m; }

float orc_mse(int mode, size_t n, const float* pred, const float* target, float* grad) {
    for (size_t i = 0; i < n; ++i) grad[i] = pred[i] - target[i];
    if (mode != 0) {
        double s = 0.0;
        for (size_t i = 0; i < n; ++i) s += (double)grad[i] * (double)grad[i];
        return (float)(s / 2.0);
    }
    float* buf = (float*)malloc(sizeof(float) * (n ? n : 1));
    for (size_t i = 0; i < n; ++i) buf[i] = grad[i] * grad[i];
    int msb = msb_index(n);
    int hmsb = msb / 2;
    --msb;
    long long stride = msb >= 0 ? (1ll << msb) : 0;
    int w = 1 << hmsb, h = msb - hmsb >= 0 ? 1 << (msb - hmsb) : 0;
    while (stride > 0) {
        int bx, by;
        get_block(w, h, &bx, &by);
        int gx = (w + bx - 1) / bx, gy = (h + by - 1) / by;
        for (int byi = 0; byi < gy; ++byi)
            for (int bxi = 0; bxi < gx; ++bxi)
                for (int ty = 0; ty < by; ++ty)
                    for (int tx = 0; tx < bx; ++tx) {
                        long long px = (long long)bxi * bx + tx, py = (long long)byi * by + ty;
                        long long pidx = px + (long long)w * py;
                        if (pidx + stride >= (long long)n) continue;
                        buf[pidx] += buf[pidx + stride];
                    }
        stride >>= 1;
        if (h >= w) h >>= 1; else w >>= 1;
    }
    float loss = n ? buf[0] : 0.f;
    free(buf);
    return loss / 2.f;
}

/* optimize.cu:84-115 (Adam::setHyperParams, adamStep, Adam::step).
 * `step` counts calls from 1.  compat: the bias correction uses
 * beta^(step+1), as rhomt starts at beta and is multiplied before its first
 * use (:87-88, :111-112); exact: beta^step.  The moments are updated in
 * double and stored as float; the update is guarded by AddNaNcheck. */
void orc_adam(int mode, size_t n, float* p, const float* g, float* m, float* v,
              double lr, double b1, double b2, double eps, int step) {
    double b1t = mode == 0 ? b1 : 1.0, b2t = mode == 0 ? b2 : 1.0;
    for (int k = 0; k < step; ++k) { b1t *= b1; b2t *= b2; }
    for (size_t i = 0; i < n; ++i) {
        m[i] = (float)(b1 * (double)m[i] + (1 - b1) * (double)g[i]);
        v[i] = (float)(b2 * (double)v[i] + (1 - b2) * (double)g[i] * (double)g[i]);
        double mh = (double)m[i] / (1 - b1t);
        double vh = (double)v[i] / (1 - b2t);
        add_nan_check(&p[i], (float)(-mh * lr / (sqrt(vh) + eps)));
    }
}

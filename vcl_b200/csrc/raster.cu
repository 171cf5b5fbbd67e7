// CUDA rasterizer replacing the reference's OpenGL draw (rasterize.cpp:
// 91-202, fixed-function state :252-268) and its backward pass
// (rasterize.cu:84-141).
//
// Forward = triangle setup -> (small triangles: direct) / (large: tile
// binner + fine rasterizer) -> resolve:
//   1. setup   one thread per (view, triangle): homogeneous-2D edge
//              functions, orientation, trivial reject, conservative pixel
//              box.  A triangle whose box has at most SMALL_AREA pixels is
//              rasterized right there by its thread: every covered pixel
//              gets a 64-bit atomicMin of the key (depth, triangle id).
//              Larger triangles count the tiles their box overlaps;
//   2. scan    exclusive prefix sum of the per-tile counts -> bin offsets;
//   3. emit    large triangles write their id into each overlapped tile's
//              bin (order inside a bin is irrelevant);
//   4. fine    one CTA per tile, one thread per pixel: stages the bin's
//              triangle records through shared memory in chunks, keeps the
//              nearest (z/w, id), then one atomicMin of its key;
//   5. resolve one thread per pixel turns the winning key into
//              (u, v, z/w, id+1) and the barycentric derivatives (DB).
// The key orders by depth, then by triangle id: strictly nearer wins and
// equal depth keeps the lower id, which is what GL_LESS gives for triangles
// drawn in index order.  A tile whose bin does not fit the bin-list
// capacity is rasterized by testing every large triangle of its view (same
// results, slower).
//
// The coverage/depth arithmetic uses explicitly rounded operations
// (__fmul_rn etc., never fused) so that it is bit-identical to the CPU
// restatement of the same rules: triangle ids, barycentrics and depth match
// exactly.
#include "common.cuh"
#include "ops_internal.cuh"

namespace {

DEV float mul(float a, float b) { return __fmul_rn(a, b); }
DEV float add(float a, float b) { return __fadd_rn(a, b); }
DEV float sub(float a, float b) { return __fsub_rn(a, b); }
DEV float dvd(float a, float b) { return __fdiv_rn(a, b); }

struct __align__(16) RTri {
    float4 a;   // a0 a1 a2 sigma
    float4 b;   // b0 b1 b2 -
    float4 k;   // k0 k1 k2 -
    float4 z;   // z0 z1 z2 -
    float4 w;   // w0 w1 w2 -
    int4 box;   // x0 x1 y0 y1 ; empty when x0 > x1
};
// the workspace's per-(view, triangle) cost that vcl.h states: this record
// plus one medium-list entry
static_assert(sizeof(RTri) + sizeof(int) == VCL_RASTER_BYTES_PER_VIEW_TRIANGLE, "raster record size changed");

constexpr int CHUNK = 128;
// default box areas (pixels): up to SMALL_AREA a triangle is rasterized by its
// setup thread, up to MEDIUM_AREA by one warp, above that through the bins
constexpr int SMALL_AREA = 256;
constexpr int MEDIUM_AREA = 4096;
constexpr unsigned long long KEY_NONE = ~0ull;

// Order-preserving 64-bit key: depth bits (monotone map of the float, -0
// folded onto +0 so that equal depths compare equal) then triangle id.
DEV unsigned long long depth_key(float zw, int t) {
    unsigned u = __float_as_uint(zw == 0.f ? 0.f : zw);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((unsigned long long)u << 32) | (unsigned)t;
}
DEV float key_depth(unsigned long long k) {
    unsigned u = (unsigned)(k >> 32);
    u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    return __uint_as_float(u);
}
DEV long long box_area(int4 b) { return (long long)(b.y - b.x + 1) * (b.w - b.z + 1); }
DEV bool is_small(int4 b, int small_area) { return box_area(b) <= small_area; }
// not binned: rasterized by its setup thread or by a warp
DEV bool is_direct(int4 b, int small_area, int med_area) { return box_area(b) <= (small_area > med_area ? small_area : med_area); }

// Pixel-centre NDC coordinate (2p+1-W)/W: exact numerator, one rounding.
DEV float ndc(int p, int W) { return dvd((float)(2 * p + 1 - W), (float)W); }

DEV float edge(float a, float b, float k, float sx, float sy) { return add(add(mul(a, sx), mul(b, sy)), k); }

DEV bool edge_in(float A, float a, float b, float sigma) {
    float sA = mul(sigma, A);
    if (sA > 0.f) return true;
    if (A != 0.f) return false;
    float gx = mul(sigma, a), gy = mul(sigma, b);
    return gx > 0.f || (gx == 0.f && gy < 0.f);
}

// Coverage and depth of the pixel centre (sx, sy) against one triangle
// record, including the clip range of z/w.  False when the pixel is not drawn.
DEV bool pixel_test(const float4& a, const float4& b, const float4& k, const float4& z, const float4& w, float sx, float sy,
                    float& zw) {
    float A0 = edge(a.x, b.x, k.x, sx, sy);
    float A1 = edge(a.y, b.y, k.y, sx, sy);
    float A2 = edge(a.z, b.z, k.z, sx, sy);
    if (!edge_in(A0, a.x, b.x, a.w) || !edge_in(A1, a.y, b.y, a.w) || !edge_in(A2, a.z, b.z, a.w)) return false;
    float D = add(add(A0, A1), A2);
    if (!(mul(a.w, D) > 0.f)) return false;
    float zn = add(add(mul(A0, z.x), mul(A1, z.y)), mul(A2, z.z));
    float wn = add(add(mul(A0, w.x), mul(A1, w.y)), mul(A2, w.z));
    zw = dvd(zn, wn);
    return zw >= -1.f && zw <= 1.f && zw < 1.f;
}

// Conservative triangle/tile test: false only when, for some edge, every
// pixel centre of the tile (clipped to the triangle's box) lies outside by
// more than a rounding margin, so no pixel of the tile can be covered.  The
// edge functions are linear in (sx, sy), so their maximum over the tile is
// at a corner.
DEV bool tile_overlaps(const RTri& r, int tx, int ty, int T, int W, int H) {
    const int x0 = max(tx * T, r.box.x), x1 = min(tx * T + T - 1, r.box.y);
    const int y0 = max(ty * T, r.box.z), y1 = min(ty * T + T - 1, r.box.w);
    if (x0 > x1 || y0 > y1) return false;
    const float sx0 = ndc(x0, W), sx1 = ndc(x1, W), sy0 = ndc(y0, H), sy1 = ndc(y1, H);
    const float sg = r.a.w;
    const float ea[3] = {r.a.x, r.a.y, r.a.z}, eb[3] = {r.b.x, r.b.y, r.b.z}, ek[3] = {r.k.x, r.k.y, r.k.z};
    // explicitly rounded operations: the count pass and the emit pass must
    // reach the same decision for every tile
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float a = mul(sg, ea[i]), b = mul(sg, eb[i]), k = mul(sg, ek[i]);
        const float mx = add(add(k, fmaxf(mul(a, sx0), mul(a, sx1))), fmaxf(mul(b, sy0), mul(b, sy1)));
        const float margin = mul(1e-5f, add(add(fabsf(a), fabsf(b)), fabsf(k)));
        if (mx < -margin) return false;
    }
    return true;
}

// Conservative column range [x0, x1] of pixel row `sy` for a triangle: each
// edge function is linear in (sx, sy), so every edge with a non-zero sx
// coefficient bounds sx from one side by a linear function of sy, set up
// once per triangle (span_setup) and evaluated with one fma per row.  The
// bound is relaxed by a margin m = 1e-5 (|a| + |b| + |k|) in edge units, far
// above both the rounding of the per-pixel edge evaluation (a few ulps of the
// same sum) and that of the bound itself (a few ulps of (|b sy| + |k| + m)/|a|
// in sx), then rounded outwards to whole pixels; pixels outside the range
// cannot be covered, pixels inside still go through the exact test.  False
// when the row certainly has no covered pixel.
struct SpanEq {
    float al[3], be[3];   // sx bound of edge i: al*sy + be (lower when side > 0, upper when side < 0)
    int side[3];          // 0: the edge does not depend on sx
};

DEV void span_setup(const RTri& r, SpanEq& q) {
    const float sg = r.a.w;
    const float ea[3] = {r.a.x, r.a.y, r.a.z}, eb[3] = {r.b.x, r.b.y, r.b.z}, ek[3] = {r.k.x, r.k.y, r.k.z};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float a = sg * ea[i];
        const float m = 1e-5f * (fabsf(ea[i]) + fabsf(eb[i]) + fabsf(ek[i]));
        const float ia = a != 0.f ? __frcp_rn(a) : 0.f;
        q.al[i] = -(sg * eb[i]) * ia;
        q.be[i] = (-(sg * ek[i]) - m) * ia;
        q.side[i] = a > 0.f ? 1 : a < 0.f ? -1 : 0;
    }
}

DEV bool row_span(const RTri& r, const SpanEq& q, float sy, int W, int& x0, int& x1) {
    float lo = -2.f, hi = 2.f;     // sx range of interest (the screen is [-1, 1])
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (q.side[i] > 0) lo = fmaxf(lo, fmaf(q.al[i], sy, q.be[i]));
        else if (q.side[i] < 0) hi = fminf(hi, fmaf(q.al[i], sy, q.be[i]));
        else {
            const float eb = i == 0 ? r.b.x : i == 1 ? r.b.y : r.b.z, ek = i == 0 ? r.k.x : i == 1 ? r.k.y : r.k.z;
            const float ea = i == 0 ? r.a.x : i == 1 ? r.a.y : r.a.z;
            const float m = 1e-5f * (fabsf(ea) + fabsf(eb) + fabsf(ek));
            if (r.a.w * (eb * sy + ek) < -m) return false;
        }
    }
    if (!(lo <= hi)) return false;     // (fmaxf/fminf drop NaN bounds; a NaN row bound leaves lo/hi as numbers)
    const float fw = (float)W;
    x0 = max(r.box.x, (int)floorf(fmaf(lo, fw, fw - 1.f) * 0.5f));
    x1 = min(r.box.y, (int)ceilf(fmaf(hi, fw, fw - 1.f) * 0.5f));
    return x0 <= x1;
}

// Pixel-centre coordinates of every column and row, staged in shared memory
// once per block (the exactly rounded divisions of ndc()).
DEV void stage_ndc(float* tab, int W, int H) {
    for (int i = threadIdx.x; i < W + H; i += blockDim.x) tab[i] = i < W ? ndc(i, W) : ndc(i - W, H);
}

DEV void setup_tri(float4 c0, float4 c1, float4 c2, int W, int H, RTri& t, bool& valid) {
    float x0 = c0.x, y0 = c0.y, x1 = c1.x, y1 = c1.y, x2 = c2.x, y2 = c2.y;
    float w0 = c0.w, w1 = c1.w, w2 = c2.w;
    t.a = make_float4(sub(mul(w2, y1), mul(w1, y2)), sub(mul(w0, y2), mul(w2, y0)), sub(mul(w1, y0), mul(w0, y1)), 0.f);
    t.b = make_float4(sub(mul(w1, x2), mul(w2, x1)), sub(mul(w2, x0), mul(w0, x2)), sub(mul(w0, x1), mul(w1, x0)), 0.f);
    t.k = make_float4(sub(mul(x1, y2), mul(y1, x2)), sub(mul(x2, y0), mul(y2, x0)), sub(mul(x0, y1), mul(y0, x1)), 0.f);
    float det = add(add(mul(w0, t.k.x), mul(w1, t.k.y)), mul(w2, t.k.z));
    valid = det != 0.f && isfinite(det);
    t.a.w = det > 0.f ? 1.f : -1.f;
    t.z = make_float4(c0.z, c1.z, c2.z, 0.f);
    t.w = make_float4(w0, w1, w2, 0.f);
    // trivial reject: all three vertices outside one clip plane
    bool o0 = x0 > w0 && x1 > w1 && x2 > w2, o1 = x0 < -w0 && x1 < -w1 && x2 < -w2;
    bool o2 = y0 > w0 && y1 > w1 && y2 > w2, o3 = y0 < -w0 && y1 < -w1 && y2 < -w2;
    bool o4 = c0.z > w0 && c1.z > w1 && c2.z > w2, o5 = c0.z < -w0 && c1.z < -w1 && c2.z < -w2;
    if (o0 || o1 || o2 || o3 || o4 || o5) valid = false;
    // pixel box: the pixel centres within half a pixel of the projected
    // vertices' extent, the same float operations as the CPU restatement's
    // raster_bbox.  A centre outside the vertex extent lies outside the
    // triangle (GL never draws it); the FP32 edge functions of a nearly
    // edge-on triangle can accept centres further out than that, and the box
    // is part of the rule that excludes them, so both sides must use this
    // one box.
    int bx0 = 0, bx1 = W - 1, by0 = 0, by1 = H - 1;
    if (w0 > 0.f && w1 > 0.f && w2 > 0.f) {
        const float iw0 = __frcp_rn(w0), iw1 = __frcp_rn(w1), iw2 = __frcp_rn(w2);
        float X0 = x0 * iw0, X1 = x1 * iw1, X2 = x2 * iw2;
        float Y0 = y0 * iw0, Y1 = y1 * iw1, Y2 = y2 * iw2;
        float xmn = fminf(fminf(X0, X1), X2), xmx = fmaxf(fmaxf(X0, X1), X2);
        float ymn = fminf(fminf(Y0, Y1), Y2), ymx = fmaxf(fmaxf(Y0, Y1), Y2);
        float hw = mul(0.5f, (float)W), hh = mul(0.5f, (float)H);
        float fx0 = sub(mul(add(xmn, 1.f), hw), 0.5f), fx1 = sub(mul(add(xmx, 1.f), hw), 0.5f);
        float fy0 = sub(mul(add(ymn, 1.f), hh), 0.5f), fy1 = sub(mul(add(ymx, 1.f), hh), 0.5f);
        fx0 = fmaxf(fminf(fx0, (float)W), -2.f); fx1 = fmaxf(fminf(fx1, (float)W), -2.f);
        fy0 = fmaxf(fminf(fy0, (float)H), -2.f); fy1 = fmaxf(fminf(fy1, (float)H), -2.f);
        if (fx0 == fx0 && fx1 == fx1 && fy0 == fy0 && fy1 == fy1) {
            bx0 = max((int)ceilf(fx0 - 0.5f), 0); bx1 = min((int)floorf(fx1 + 0.5f), W - 1);
            by0 = max((int)ceilf(fy0 - 0.5f), 0); by1 = min((int)floorf(fy1 + 0.5f), H - 1);
        }
    }
    if (!valid) { bx0 = 1; bx1 = 0; }
    t.box = make_int4(bx0, bx1, by0, by1);
}

// A small triangle staged in shared memory for the row-balanced raster loop
// of k_setup: its record, its row-span bounds and (triangle, view).  144
// bytes, so that lanes reading different slots spread over the banks.
struct __align__(16) SmallTri {
    float4 a, b, k, z, w;
    float4 s0;     // al0 be0 al1 be1
    float4 s1;     // al2 be2 (sides + 1: 2 bits each) | view << 8, triangle
    int4 box;
    float4 pad;
};
constexpr int SETUP_THREADS = 256;

DEV void small_pack(SmallTri& o, const RTri& r, const SpanEq& q, int t, int view) {
    o.a = r.a; o.b = r.b; o.k = r.k; o.z = r.z; o.w = r.w; o.box = r.box;
    o.s0 = make_float4(q.al[0], q.be[0], q.al[1], q.be[1]);
    const int code = (q.side[0] + 1) | ((q.side[1] + 1) << 2) | ((q.side[2] + 1) << 4) | (view << 8);
    o.s1 = make_float4(q.al[2], q.be[2], __int_as_float(code), __int_as_float(t));
}

size_t setup_smem(int W, int H) {
    return sizeof(float) * (size_t)((W + H + 3) & ~3) + sizeof(SmallTri) * SETUP_THREADS;
}

// 1. setup (see the file comment).  The small triangles of a warp are then
// rasterized together: their rows are dealt round-robin to the 32 lanes, so
// that a lane with a tall triangle does not hold up the others.
__global__ void __launch_bounds__(SETUP_THREADS, 4) k_setup(const float4* __restrict__ clip, int nv,
                        const uint32_t* __restrict__ tri, int nt, int W, int H,
                        int views, int tile, int tiles_x, int ntiles, RTri* __restrict__ setup, int* __restrict__ count,
                        int* __restrict__ flags, unsigned long long* __restrict__ keys, int small_area, int med_area,
                        int* __restrict__ med_list, int* __restrict__ med_count) {
    extern __shared__ float s_ndc[];   // [W] column centres, [H] row centres, then the small-triangle slots
    SmallTri* s_tri = reinterpret_cast<SmallTri*>(s_ndc + ((W + H + 3) & ~3));
    __shared__ int s_start[SETUP_THREADS / 32][32];
    stage_ndc(s_ndc, W, H);
    __syncthreads();
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in_range = gid < (long long)views * nt;
    const int view = in_range ? (int)(gid / nt) : 0, t = in_range ? (int)(gid % nt) : 0;
    RTri r;
    r.box = make_int4(1, 0, 1, 0);
    if (in_range) {
        uint32_t i0 = tri[3 * (size_t)t], i1 = tri[3 * (size_t)t + 1], i2 = tri[3 * (size_t)t + 2];
        bool valid = false;
        if (i0 < (uint32_t)nv && i1 < (uint32_t)nv && i2 < (uint32_t)nv) {
            const float4* cv = clip + (size_t)view * nv;
            setup_tri(cv[i0], cv[i1], cv[i2], W, H, r, valid);
        } else {
            atomicOr(&flags[1], 1);  // out-of-range vertex index: triangle dropped
            r.box = make_int4(1, 0, 1, 0);
        }
        setup[gid] = r;
    }
    const bool has = r.box.x <= r.box.y && r.box.z <= r.box.w;
    const bool small = has && is_small(r.box, small_area);
    if (has && !small) {
        if (box_area(r.box) <= med_area) {
            med_list[atomicAdd(med_count, 1)] = (int)gid;   // one warp rasterizes it (k_medium)
        } else {
            int tx0 = r.box.x / tile, tx1 = r.box.y / tile, ty0 = r.box.z / tile, ty1 = r.box.w / tile;
            int* cnt = count + (size_t)view * ntiles;
            for (int ty = ty0; ty <= ty1; ++ty)
                for (int tx = tx0; tx <= tx1; ++tx)
                    if (tile_overlaps(r, tx, ty, tile, W, H)) atomicAdd(&cnt[ty * tiles_x + tx], 1);
        }
    }
    // row-balanced raster of the warp's small triangles: every covered pixel
    // gets a 64-bit atomicMin of its key (depth, triangle id)
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int rows = small ? r.box.w - r.box.z + 1 : 0;
    int incl = rows;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return;
    int* start = s_start[wib];
    SmallTri* st = s_tri + wib * 32;
    start[lane] = incl - rows;
    if (small) {
        SpanEq q;
        span_setup(r, q);
        small_pack(st[lane], r, q, t, view);
    }
    __syncwarp();
    // 32 rows at a time: each lane finds its row's conservative span, then
    // the warp walks the concatenated spans pixel by pixel (lane m takes
    // pixels m, m + 32, ... of the concatenation), so lanes stay busy however
    // unequal the spans are
    for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        int j = 0, py = 0, x0 = 0, x1 = -1;
        if (k < total) {
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (start[j + step] <= k) j += step;
            const SmallTri& S = st[j];
            RTri rr;
            rr.a = S.a; rr.b = S.b; rr.k = S.k; rr.z = S.z; rr.w = S.w; rr.box = S.box;
            const float4 s0 = S.s0, s1 = S.s1;
            const int code = __float_as_int(s1.z);
            SpanEq q;
            q.al[0] = s0.x; q.be[0] = s0.y; q.al[1] = s0.z; q.be[1] = s0.w; q.al[2] = s1.x; q.be[2] = s1.y;
            q.side[0] = (code & 3) - 1; q.side[1] = ((code >> 2) & 3) - 1; q.side[2] = ((code >> 4) & 3) - 1;
            py = rr.box.z + (k - start[j]);
            if (!row_span(rr, q, s_ndc[W + py], W, x0, x1)) x1 = x0 - 1;
        }
        const int len = x1 >= x0 ? x1 - x0 + 1 : 0;
        int end = len;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, end, o);
            if (lane >= o) end += y;
        }
        const int beg = end - len;
        const int npx = __shfl_sync(0xffffffffu, end, 31);
        for (int m0 = 0; m0 < npx; m0 += 32) {
            const int m = m0 + lane;
            // the row lane owning pixel m: the last lane whose span starts at or before m
            int r = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int b = __shfl_sync(0xffffffffu, beg, r + step);
                if (b <= m) r += step;
            }
            const int rb = __shfl_sync(0xffffffffu, beg, r), rx = __shfl_sync(0xffffffffu, x0, r);
            const int ry = __shfl_sync(0xffffffffu, py, r), rj = __shfl_sync(0xffffffffu, j, r);
            if (m >= npx) continue;
            const SmallTri& S = st[rj];
            const int px = rx + (m - rb);
            const float4 s1 = S.s1;
            const int code = __float_as_int(s1.z), tj = __float_as_int(s1.w);
            float zw;
            if (pixel_test(S.a, S.b, S.k, S.z, S.w, s_ndc[px], s_ndc[W + ry], zw))
                atomicMin(&keys[(size_t)(code >> 8) * W * H + (size_t)ry * W + px], depth_key(zw, tj));
        }
    }
}

// Exclusive scan of n ints by one CTA of 32 warps: warp w owns a contiguous
// segment; it sums the segment with coalesced loads, the 32 segment sums are
// scanned, then each warp rescans its segment 32 elements at a time (warp
// inclusive scan + running carry), again with coalesced loads and stores.
__global__ void __launch_bounds__(1024) k_scan(const int* __restrict__ in, int* __restrict__ out, int n) {
    __shared__ int seg_sum[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int seg = (n + 31) / 32;
    const int beg = min(wid * seg, n), end = min(beg + seg, n);
    int sum = 0;
    for (int i = beg + lane; i < end; i += 32) sum += in[i];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) seg_sum[wid] = sum;
    __syncthreads();
    if (wid == 0) {
        int v = seg_sum[lane];
        for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v += y; }
        seg_sum[lane] = v;   // inclusive
    }
    __syncthreads();
    int carry = wid ? seg_sum[wid - 1] : 0;
    for (int base = beg; base < end; base += 32) {
        const int i = base + lane;
        const int v = i < end ? in[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        if (i < end) out[i] = carry + x - v;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
}

__global__ void k_emit(const RTri* __restrict__ setup, int nt, int views, int W, int H, int tile, int tiles_x,
                       int ntiles, const int* __restrict__ offset, int* __restrict__ cursor, int* __restrict__ list,
                       long long cap, int small_area, int med_area) {
    long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)views * nt) return;
    int view = (int)(gid / nt), t = (int)(gid % nt);
    const RTri r = setup[gid];
    const int4 box = r.box;
    if (box.x > box.y || box.z > box.w || is_direct(box, small_area, med_area)) return;
    int tx0 = box.x / tile, tx1 = box.y / tile, ty0 = box.z / tile, ty1 = box.w / tile;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            if (!tile_overlaps(r, tx, ty, tile, W, H)) continue;
            size_t ti = (size_t)view * ntiles + ty * tiles_x + tx;
            int slot = atomicAdd(&cursor[ti], 1);
            long long p = (long long)offset[ti] + slot;
            if (p < cap) list[p] = t;
        }
}

// The reference geometry shader's per-vertex barycentric derivatives
// (rasterize.cpp:141-164), evaluated at (u, v) and scaled by w (:176).
DEV float4 db_eval(float4 c0, float4 c1, float4 c2, float xs, float ys, float u, float v) {
    float w0 = c0.w, w1 = c1.w, w2 = c2.w;
    float e0x = sub(mul(w0, c2.x), mul(w2, c0.x)), e0y = sub(mul(w0, c2.y), mul(w2, c0.y));
    float e1x = sub(mul(w1, c2.x), mul(w2, c1.x)), e1y = sub(mul(w1, c2.y), mul(w2, c1.y));
    float ex = sub(mul(w0, c1.x), mul(w1, c0.x)), ey = sub(mul(w0, c1.y), mul(w1, c0.y));
    float a = sub(mul(e0x, e1y), mul(e0y, e1x));
    const float eps = 1e-6f;
    float ca = (fabsf(a) >= eps) ? a : (a < 0.f) ? -eps : eps;
    float sx = dvd(mul(ys, w2), ca), sy = dvd(mul(xs, w2), ca);
    e0x = mul(e0x, sx); e0y = mul(e0y, sy);
    e1x = mul(e1x, sx); e1y = mul(e1y, sy);
    ex = mul(ex, sx); ey = mul(ey, sy);
    float d0[4] = {sub(e0y, ey), add(-e0x, ex), -e0y, e0x};
    float d1[4] = {e1y, -e1x, sub(-e1y, ey), add(e1x, ex)};
    float d2[4] = {e1y, -e1x, -e0y, e0x};
    float l2 = sub(sub(1.f, u), v);
    float wi = add(add(mul(u, w0), mul(v, w1)), mul(l2, w2));
    float o[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) o[c] = mul(add(add(mul(u, d0[c]), mul(v, d1[c])), mul(l2, d2[c])), wi);
    return make_float4(o[0], o[1], o[2], o[3]);
}

template <int T>
__global__ void __launch_bounds__(T * T) k_fine(const RTri* __restrict__ setup, const int* __restrict__ count,
                                                const int* __restrict__ offset, const int* __restrict__ list,
                                                long long cap, int nt, int W, int H, int tiles_x, int ntiles,
                                                unsigned long long* __restrict__ keys, int* __restrict__ flags,
                                                int small_area, int med_area) {
    __shared__ RTri s_tri[CHUNK];
    __shared__ int s_id[CHUNK];
    const int view = blockIdx.y, tile_id = blockIdx.x;
    const size_t ti = (size_t)view * ntiles + tile_id;
    const int c = count[ti];
    const int off = offset[ti];
    const bool overflow = (long long)off + c > cap;
    if (c == 0) return;
    const int tx = tile_id % tiles_x, ty = tile_id / tiles_x;
    const int px = tx * T + threadIdx.x, py = ty * T + threadIdx.y;
    const int tid = threadIdx.y * T + threadIdx.x;
    const bool inside = px < W && py < H;
    const float sx = ndc(px, W), sy = ndc(py, H);
    const int n_iter = overflow ? nt : c;
    const RTri* vs = setup + (size_t)view * nt;
    unsigned long long best = KEY_NONE;
    constexpr int CH = T * T < CHUNK ? T * T : CHUNK;   // records staged per pass (<= threads)
    for (int i0 = 0; i0 < n_iter; i0 += CH) {
        if (tid < CH && i0 + tid < n_iter) {
            int t = overflow ? i0 + tid : list[off + i0 + tid];
            if ((unsigned)t >= (unsigned)nt) t = 0;   // never taken: every counted slot is emitted
            s_id[tid] = t;
            s_tri[tid] = vs[t];
            // in the all-triangles fallback the small ones are done already
            if (overflow && is_direct(s_tri[tid].box, small_area, med_area)) s_tri[tid].box = make_int4(1, 0, 1, 0);
        }
        __syncthreads();
        const int m = min(CH, n_iter - i0);
        if (inside) {
            for (int j = 0; j < m; ++j) {
                const int4 box = s_tri[j].box;
                if (px < box.x || px > box.y || py < box.z || py > box.w) continue;
                float zw;
                if (!pixel_test(s_tri[j].a, s_tri[j].b, s_tri[j].k, s_tri[j].z, s_tri[j].w, sx, sy, zw)) continue;
                const unsigned long long key = depth_key(zw, s_id[j]);
                best = key < best ? key : best;
            }
        }
        __syncthreads();
    }
    if (overflow && tid == 0) atomicAdd(&flags[0], 1);
    if (inside && best != KEY_NONE) atomicMin(&keys[((size_t)view * H + py) * W + px], best);
}

// Medium triangles: one warp per triangle, one lane per pixel row of its
// box; a lane tests the pixels of its row's conservative span and keeps the
// nearest (depth, id) per pixel with a 64-bit atomicMin (same coverage and
// depth arithmetic as the other paths).  Persistent warps stride over the
// list the setup pass filled.
__global__ void __launch_bounds__(256) k_medium(const RTri* __restrict__ setup, int nt, int W, int H,
                                                const int* __restrict__ med_list, const int* __restrict__ med_count,
                                                unsigned long long* __restrict__ keys) {
    extern __shared__ float s_ndc[];   // [W] column centres, [H] row centres
    stage_ndc(s_ndc, W, H);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int n = *med_count;
    for (int i = warp; i < n; i += nwarps) {
        const int gid = med_list[i];
        const int view = gid / nt, t = gid - view * nt;
        const RTri r = setup[gid];
        unsigned long long* kv = keys + (size_t)view * W * H;
        SpanEq q;
        span_setup(r, q);
        // 32 rows at a time: a lane finds its row's conservative span, then
        // the warp walks the concatenated spans pixel by pixel
        for (int y0 = r.box.z; y0 <= r.box.w; y0 += 32) {
            const int py = y0 + lane;
            int x0 = 0, x1 = -1;
            if (py <= r.box.w && !row_span(r, q, s_ndc[W + py], W, x0, x1)) x1 = x0 - 1;
            const int len = x1 >= x0 ? x1 - x0 + 1 : 0;
            int end = len;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, end, o);
                if (lane >= o) end += y;
            }
            const int beg = end - len;
            const int npx = __shfl_sync(0xffffffffu, end, 31);
            for (int m0 = 0; m0 < npx; m0 += 32) {
                const int m = m0 + lane;
                int rl = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int b = __shfl_sync(0xffffffffu, beg, rl + step);
                    if (b <= m) rl += step;
                }
                const int rb = __shfl_sync(0xffffffffu, beg, rl), rx = __shfl_sync(0xffffffffu, x0, rl);
                if (m >= npx) continue;
                const int px = rx + (m - rb), ry = y0 + rl;
                float zw;
                if (pixel_test(r.a, r.b, r.k, r.z, r.w, s_ndc[px], s_ndc[W + ry], zw))
                    atomicMin(&kv[(size_t)ry * W + px], depth_key(zw, t));
            }
        }
    }
}

// Winning key -> (u, v, z/w, id+1) and DB per pixel; held to 32 registers
// for eight blocks per SM (the record and vertex gathers need the warps).
// The pixel's (view, row, column) come by multiply-high division (when
// npix < 2^32; 64-bit division above) and W, H, 2 / W, 2 / H as
// host-computed floats (the same values): no integer division or conversion
// per pixel beyond the pixel centre's.
struct ResolveDims {
    FastDiv div_w, div_hw;
    float fW, fH, xs, ys;
    int big;
};
__global__ void __launch_bounds__(256, 8) k_resolve(const RTri* __restrict__ setup, int nt, int W, int H, long long npix,
                          const unsigned long long* __restrict__ keys, const float4* __restrict__ clip, int nv,
                          const uint32_t* __restrict__ tri, float4* __restrict__ rast, float4* __restrict__ db,
                          ResolveDims rd) {
    const long long pix = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix) return;
    const unsigned long long key = keys[pix];
    if (key == KEY_NONE) {
        rast[pix] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (db) db[pix] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    int view, rem;
    if (rd.big) {
        const long long hw = (long long)W * H;
        view = (int)(pix / hw);
        rem = (int)(pix - view * hw);
    } else {
        view = (int)fastdiv((unsigned)pix, rd.div_hw);
        rem = (int)((unsigned)pix - (unsigned)view * ((unsigned)W * (unsigned)H));
    }
    const int py = (int)fastdiv((unsigned)rem, rd.div_w), px = rem - py * W;
    const int t = (int)(unsigned)(key & 0xffffffffu);
    const RTri r = setup[(size_t)view * nt + t];
    const float sx = dvd((float)(2 * px + 1 - W), rd.fW), sy = dvd((float)(2 * py + 1 - H), rd.fH);
    float A0 = edge(r.a.x, r.b.x, r.k.x, sx, sy);
    float A1 = edge(r.a.y, r.b.y, r.k.y, sx, sy);
    float A2 = edge(r.a.z, r.b.z, r.k.z, sx, sy);
    float D = add(add(A0, A1), A2);
    float u = dvd(A0, D), v = dvd(A1, D);
    rast[pix] = make_float4(u, v, key_depth(key), (float)(t + 1));
    if (db) {
        const float4* cv = clip + (size_t)view * nv;
        float4 c0 = cv[tri[3 * (size_t)t]], c1 = cv[tri[3 * (size_t)t + 1]], c2 = cv[tri[3 * (size_t)t + 2]];
        db[pix] = db_eval(c0, c1, c2, rd.xs, rd.ys, u, v);
    }
}

// rasterize.cu:84-141: dL/d(x, y, w) of the three clip-space vertices from
// dL/d(u, v) (z receives +0).  One thread per pixel; the vertex gradients of
// neighbouring pixels on the same triangle are summed by the warp, then one
// vector reduction per vertex and run.
__global__ void k_raster_bwd(const float* __restrict__ clip, int nv, const uint32_t* __restrict__ tri, int nt, int W,
                             int H, long long npix, const float4* __restrict__ rast, const float2* __restrict__ gb,
                             float* __restrict__ gclip) {
    const long long pidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    float v[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    uint32_t i0 = 0, i1 = 0, i2 = 0;
    int idx = -1, view = -1;
    bool ok = false;
    if (pidx < npix) {
        const float4 r = rast[pidx];
        idx = rast_id(r.w);
        const float2 g = gb[pidx];
        if (idx >= 0 && idx < nt && ((__float_as_uint(g.x) | __float_as_uint(g.y)) << 1) != 0u) {
            i0 = tri[3 * (size_t)idx]; i1 = tri[3 * (size_t)idx + 1]; i2 = tri[3 * (size_t)idx + 2];
            if (i0 < (uint32_t)nv && i1 < (uint32_t)nv && i2 < (uint32_t)nv) {
                const long long hw = (long long)W * H;
                view = (int)(pidx / hw);
                const int rem = (int)(pidx - view * hw);
                const int py = rem / W, px = rem - py * W;
                const float xs = 2.f / (float)W, ys = 2.f / (float)H;
                const float pxn = (float)(((double)px + 0.5) * (double)xs - 1.0);
                const float pyn = (float)(((double)py + 0.5) * (double)ys - 1.0);
                const float4* cv = reinterpret_cast<const float4*>(clip) + (size_t)view * nv;
                const float4 c0 = cv[i0], c1 = cv[i1], c2 = cv[i2];
                float p0x = c0.w * pxn - c0.x, p0y = c0.w * pyn - c0.y;
                float p1x = c1.w * pxn - c1.x, p1y = c1.w * pyn - c1.y;
                float p2x = c2.w * pxn - c2.x, p2y = c2.w * pyn - c2.y;
                float e0x = p0x - p2x, e0y = p0y - p2y, e1x = p1x - p2x, e1y = p1y - p2y;
                float a = e0x * e1y - e0y * e1x;
                float ia = 1.f / (a + (a > 0 ? 1e-6f : -1e-6f));
                float kuv = r.x * g.x + r.y * g.y;
                float gx0 = (g.y * p2y + kuv * e1y) * ia;
                float gy0 = (-g.y * p2x - kuv * e1x) * ia;
                float gx1 = (-g.x * p2y - kuv * e0y) * ia;
                float gy1 = (g.x * p2x + kuv * e0x) * ia;
                float gx2 = ((-g.y * p0y + g.x * p1y) - kuv * (-p0y + p1y)) * ia;
                float gy2 = ((g.y * p0x - g.x * p1x) - kuv * (p0x - p1x)) * ia;
                v[0] = gx0; v[1] = gy0; v[2] = -gx0 * pxn - gy0 * pyn;
                v[3] = gx1; v[4] = gy1; v[5] = -gx1 * pxn - gy1 * pyn;
                v[6] = gx2; v[7] = gy2; v[8] = -gx2 * pxn - gy2 * pyn;
                ok = true;
            }
        }
    }
    const bool tail = warp_run_sum(v, ok ? idx : -1 - lane, ok ? view : -1);
    if (!(tail && ok)) return;
    float* gv = gclip + (size_t)view * nv * 4;
    red_add4(gv + (size_t)i0 * 4, v[0], v[1], 0.f, v[2]);
    red_add4(gv + (size_t)i1 * 4, v[3], v[4], 0.f, v[5]);
    red_add4(gv + (size_t)i2 * 4, v[6], v[7], 0.f, v[8]);
}

// GL tie census of a finished raster (vcl_raster_ties): one warp per (view,
// triangle), a lane per pixel row of the triangle's box, walking the row's
// conservative span with the rasterizer's own arithmetic.  Bit 1 marks a
// centre exactly on an edge of a triangle whose closed interior holds it
// (the top-left rule decided), bit 2 a pixel that a triangle other than the
// winner covers at exactly the winning depth (the lower id decided).
__global__ void __launch_bounds__(256) k_ties(const float4* __restrict__ clip, int nv, const uint32_t* __restrict__ tri,
                                              int nt, int W, int H, int views, const float4* __restrict__ rast,
                                              unsigned* __restrict__ flags) {
    extern __shared__ float s_ndc[];   // [W] column centres, [H] row centres
    stage_ndc(s_ndc, W, H);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long work = (long long)views * nt;
    for (long long g = warp; g < work; g += nwarps) {
        const int view = (int)(g / nt), t = (int)(g - (long long)view * nt);
        const uint32_t i0 = tri[3 * (size_t)t], i1 = tri[3 * (size_t)t + 1], i2 = tri[3 * (size_t)t + 2];
        if (i0 >= (uint32_t)nv || i1 >= (uint32_t)nv || i2 >= (uint32_t)nv) continue;
        const float4* cv = clip + (size_t)view * nv;
        RTri r;
        bool valid = false;
        setup_tri(cv[i0], cv[i1], cv[i2], W, H, r, valid);
        if (r.box.x > r.box.y || r.box.z > r.box.w) continue;
        SpanEq q;
        span_setup(r, q);
        const size_t vbase = (size_t)view * W * H;
        const float sg = r.a.w;
        for (int py = r.box.z + lane; py <= r.box.w; py += 32) {
            const float sy = s_ndc[W + py];
            int x0, x1;
            if (!row_span(r, q, sy, W, x0, x1)) continue;
            for (int px = x0; px <= x1; ++px) {
                const float sx = s_ndc[px];
                const float A0 = edge(r.a.x, r.b.x, r.k.x, sx, sy);
                const float A1 = edge(r.a.y, r.b.y, r.k.y, sx, sy);
                const float A2 = edge(r.a.z, r.b.z, r.k.z, sx, sy);
                if (!(mul(sg, A0) >= 0.f && mul(sg, A1) >= 0.f && mul(sg, A2) >= 0.f)) continue;
                const float D = add(add(A0, A1), A2);
                if (!(mul(sg, D) > 0.f)) continue;
                const float zn = add(add(mul(A0, r.z.x), mul(A1, r.z.y)), mul(A2, r.z.z));
                const float wn = add(add(mul(A0, r.w.x), mul(A1, r.w.y)), mul(A2, r.w.z));
                const float zw = dvd(zn, wn);
                if (!(zw >= -1.f && zw < 1.f)) continue;
                const size_t pi = vbase + (size_t)py * W + px;
                unsigned f = (A0 == 0.f || A1 == 0.f || A2 == 0.f) ? 1u : 0u;
                if (edge_in(A0, r.a.x, r.b.x, sg) && edge_in(A1, r.a.y, r.b.y, sg) && edge_in(A2, r.a.z, r.b.z, sg)) {
                    const float4 rp = rast[pi];
                    if (rp.w > 0.f && rp.w != (float)(t + 1) && zw == rp.z) f |= 2u;
                }
                if (f) atomicOr(&flags[pi], f);
            }
        }
    }
}

__global__ void k_tie_count(const unsigned* __restrict__ flags, long long n, unsigned long long* __restrict__ counts) {
    unsigned long long e = 0, d = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned f = flags[i];
        e += f & 1u;
        d += (f >> 1) & 1u;
    }
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        d += __shfl_xor_sync(0xffffffffu, d, o);
    }
    if ((threadIdx.x & 31) == 0 && (e | d)) {
        atomicAdd(&counts[0], e);
        atomicAdd(&counts[1], d);
    }
}

struct RasterWS {
    unsigned long long* keys;
    RTri* setup;
    int* med_list;     // [views * nt] medium triangles (view * nt + t)
    int* count;        // [ntiles + 1]; count[ntiles] = number of medium triangles
    int* offset;
    int* cursor;
    int* list;
    long long cap;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

long long auto_capacity_(long long views, long long nt, int W, int H, int tile) {
    long long ntiles = (long long)((W + tile - 1) / tile) * ((H + tile - 1) / tile) * views;
    long long c = views * nt * 6 + ntiles * 4 + (1 << 20);
    return c > (1ll << 31) - 1 ? (1ll << 31) - 1 : c;
}

size_t ws_bytes(long long npix, long long views, long long nt, long long ntiles, long long cap) {
    const size_t vt = (size_t)(views * nt > 0 ? views * nt : 1);
    return align256(sizeof(unsigned long long) * (size_t)npix) + align256(sizeof(RTri) * vt) +
           align256(sizeof(int) * vt) + 3 * align256(sizeof(int) * (size_t)(ntiles + 1)) +
           align256(sizeof(int) * (size_t)cap);
}

RasterWS carve(void* base, long long npix, long long views, long long nt, long long ntiles, long long cap) {
    char* p = (char*)base;
    RasterWS w;
    w.keys = (unsigned long long*)p; p += align256(sizeof(unsigned long long) * (size_t)npix);
    const size_t vt = (size_t)(views * nt > 0 ? views * nt : 1);
    w.setup = (RTri*)p; p += align256(sizeof(RTri) * vt);
    w.med_list = (int*)p; p += align256(sizeof(int) * vt);
    w.count = (int*)p; p += align256(sizeof(int) * (size_t)(ntiles + 1));
    w.offset = (int*)p; p += align256(sizeof(int) * (size_t)(ntiles + 1));
    w.cursor = (int*)p; p += align256(sizeof(int) * (size_t)(ntiles + 1));
    w.list = (int*)p;
    w.cap = cap;
    return w;
}

}  // namespace

long long raster_auto_capacity(long long views, long long nt, int W, int H, int tile) {
    return auto_capacity_(views, nt, W, H, tile);
}

size_t raster_ws_size(int W, int H, int views, int nt, int tile, long long cap) {
    long long ntiles = (long long)((W + tile - 1) / tile) * ((H + tile - 1) / tile) * views;
    return ws_bytes((long long)W * H * views, views, nt, ntiles, cap);
}

int raster_fwd_launches() { return 6; }

int raster_default_small_area() { return SMALL_AREA; }
int raster_default_medium_area() { return MEDIUM_AREA; }

vcl_status raster_fwd_ws(vcl_ctx* ctx, void* ws, const RasterSched& rs, int* flags, const float* clip, int nv,
                         const uint32_t* tri, int nt, int W, int H, int views, float* rast, float* db, cudaStream_t s) {
    const int T = rs.tile;
    const long long cap = rs.cap;
    const int sa = rs.small_area, ma = rs.med_area;
    const int tiles_x = (W + T - 1) / T, tiles_y = (H + T - 1) / T;
    const long long ntiles_view = (long long)tiles_x * tiles_y;
    const long long ntiles = ntiles_view * views;
    const long long npix = (long long)W * H * views;
    RasterWS w = carve(ws, npix, views, nt, ntiles, cap);
    vcl_status st = vcl_cuda_check(ctx, cudaMemsetAsync(w.keys, 0xff, sizeof(unsigned long long) * npix, s), "raster memset");
    if (st) return st;
    st = vcl_cuda_check(ctx, cudaMemsetAsync(w.count, 0, sizeof(int) * (ntiles + 1), s), "raster memset");
    if (st) return st;
    st = vcl_cuda_check(ctx, cudaMemsetAsync(w.cursor, 0, sizeof(int) * ntiles, s), "raster memset");
    if (st) return st;
    st = vcl_cuda_check(ctx, cudaMemsetAsync(flags, 0, sizeof(int), s), "raster memset");
    if (st) return st;
    long long work = (long long)views * nt;
    if (work > 0) {
        const size_t tab = sizeof(float) * (size_t)(W + H);
        const size_t stab = setup_smem(W, H);
        if (stab > 48 * 1024) cudaFuncSetAttribute(k_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stab);
        if (tab > 48 * 1024) cudaFuncSetAttribute(k_medium, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tab);
        k_setup<<<vcl_blocks(work, SETUP_THREADS), SETUP_THREADS, stab, s>>>((const float4*)clip, nv, tri, nt, W, H, views, T, tiles_x,
                                                         (int)ntiles_view, w.setup, w.count, flags, w.keys, sa, ma,
                                                         w.med_list, w.count + ntiles);
        k_medium<<<ctx->sm_count * 8, 256, tab, s>>>(w.setup, nt, W, H, w.med_list, w.count + ntiles, w.keys);
    }
    k_scan<<<1, 1024, 0, s>>>(w.count, w.offset, (int)ntiles);
    if (work > 0) {
        k_emit<<<vcl_blocks(work, 256), 256, 0, s>>>(w.setup, nt, views, W, H, T, tiles_x, (int)ntiles_view,
                                                      w.offset, w.cursor, w.list, cap, sa, ma);
    }
    dim3 grid((unsigned)ntiles_view, (unsigned)views);
    if (T == 8)
        k_fine<8><<<grid, dim3(8, 8), 0, s>>>(w.setup, w.count, w.offset, w.list, cap, nt, W, H, tiles_x,
                                             (int)ntiles_view, w.keys, flags, sa, ma);
    else if (T == 16)
        k_fine<16><<<grid, dim3(16, 16), 0, s>>>(w.setup, w.count, w.offset, w.list, cap, nt, W, H, tiles_x,
                                               (int)ntiles_view, w.keys, flags, sa, ma);
    else
        k_fine<32><<<grid, dim3(32, 32), 0, s>>>(w.setup, w.count, w.offset, w.list, cap, nt, W, H, tiles_x,
                                               (int)ntiles_view, w.keys, flags, sa, ma);
    ResolveDims rd;
    rd.div_w = fastdiv_make((unsigned)W);
    rd.div_hw = fastdiv_make((unsigned)W * (unsigned)H);
    rd.fW = (float)W; rd.fH = (float)H;
    rd.xs = 2.f / rd.fW; rd.ys = 2.f / rd.fH;
    rd.big = npix > 0xffffffffll;
    k_resolve<<<vcl_blocks(npix, 256), 256, 0, s>>>(w.setup, nt, W, H, npix, w.keys, (const float4*)clip, nv, tri,
                                                     (float4*)rast, (float4*)db, rd);
    return vcl_launch_check(ctx, "rasterize_fwd");
}

RasterSched ctx_sched(const vcl_ctx* ctx, int T, long long cap) {
    return RasterSched{T, cap, ctx->small_area >= 0 ? ctx->small_area : SMALL_AREA,
                       ctx->med_area >= 0 ? ctx->med_area : MEDIUM_AREA};
}

vcl_status raster_bin_demand(vcl_ctx* ctx, void* ws, const RasterSched& rs, int W, int H, int views, int nt,
                             cudaStream_t s, long long* demand) {
    const int T = rs.tile;
    const long long ntiles = (long long)((W + T - 1) / T) * ((H + T - 1) / T) * views;
    RasterWS w = carve(ws, (long long)W * H * views, views, nt, ntiles, rs.cap);
    int last[2] = {0, 0};
    vcl_status st = vcl_cuda_check(ctx, cudaMemcpyAsync(&last[0], w.offset + ntiles - 1, sizeof(int),
                                                        cudaMemcpyDeviceToHost, s), "bin demand");
    if (!st) st = vcl_cuda_check(ctx, cudaMemcpyAsync(&last[1], w.count + ntiles - 1, sizeof(int),
                                                      cudaMemcpyDeviceToHost, s), "bin demand");
    if (!st) st = vcl_cuda_check(ctx, cudaStreamSynchronize(s), "bin demand");
    if (!st) *demand = (long long)last[0] + last[1];
    return st;
}

extern "C" {

VCL_API vcl_status vcl_reserve_raster(vcl_ctx* ctx, int W, int H, int views, int nt) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(W > 0 && H > 0 && views > 0 && nt >= 0, "bad raster reservation sizes");
    long long cap = ctx->bin_capacity ? ctx->bin_capacity : auto_capacity_(views, nt, W, H, ctx->tile);
    int ts[3] = {8, 16, 32};
    size_t need = 0;
    for (int t : ts) {
        long long ntiles = (long long)((W + t - 1) / t) * ((H + t - 1) / t) * views;
        size_t b = ws_bytes((long long)W * H * views, views, nt, ntiles, cap);
        if (b > need) need = b;
    }
    return vcl_ws_reserve(ctx, need);
}

VCL_API vcl_status vcl_rasterize_fwd(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt, int W,
                                     int H, int views, float* rast, float* db, void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(W > 0 && H > 0 && views > 0 && nv >= 0 && nt >= 0, "bad raster sizes W=%d H=%d views=%d nv=%d nt=%d",
                W, H, views, nv, nt);
    VCL_REQUIRE(rast, "rast output is null");
    VCL_REQUIRE(nt == 0 || (clip && tri), "clip/tri is null");
    VCL_REQUIRE(((uintptr_t)clip & 15) == 0 && ((uintptr_t)rast & 15) == 0 && ((uintptr_t)db & 15) == 0,
                "clip/rast/db must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    const int T = ctx->tile;
    const int tiles_x = (W + T - 1) / T, tiles_y = (H + T - 1) / T;
    const long long ntiles_view = (long long)tiles_x * tiles_y;
    const long long ntiles = ntiles_view * views;
    VCL_REQUIRE(ntiles < (1ll << 31), "too many tiles");
    long long cap = ctx->bin_capacity ? ctx->bin_capacity : auto_capacity_(views, nt, W, H, T);
    vcl_status st = vcl_ws_reserve(ctx, ws_bytes((long long)W * H * views, views, nt, ntiles, cap));
    if (st) return st;
    return raster_fwd_ws(ctx, ctx->ws, ctx_sched(ctx, T, cap), ctx->dev_flags, clip, nv, tri, nt, W, H, views,
                         rast, db, s);
}

VCL_API vcl_status vcl_rasterize_bwd(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt, int W, int H,
                                     int views, const float* rast, const float* grad_bary, float* grad_clip,
                                     void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(W > 0 && H > 0 && views > 0, "bad raster sizes");
    VCL_REQUIRE(clip && tri && rast && grad_bary && grad_clip, "null buffer");
    VCL_REQUIRE(((uintptr_t)clip & 15) == 0 && ((uintptr_t)grad_clip & 15) == 0 && ((uintptr_t)rast & 15) == 0 &&
                    ((uintptr_t)grad_bary & 7) == 0, "misaligned buffer");
    long long npix = (long long)W * H * views;
    k_raster_bwd<<<vcl_blocks(npix, 256), 256, 0, (cudaStream_t)stream>>>(
        clip, nv, tri, nt, W, H, npix, (const float4*)rast, (const float2*)grad_bary, grad_clip);
    return vcl_launch_check(ctx, "rasterize_bwd");
}

VCL_API vcl_status vcl_raster_ties(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt, int W, int H,
                                   int views, const float* rast, uint32_t* flags, unsigned long long* counts,
                                   void* stream) {
    VCL_CTX_CHECK();
    VCL_REQUIRE(W > 0 && H > 0 && views > 0 && nv >= 0 && nt >= 0, "bad raster sizes");
    VCL_REQUIRE(rast && flags && counts, "null buffer");
    VCL_REQUIRE(nt == 0 || (clip && tri), "clip/tri is null");
    VCL_REQUIRE(((uintptr_t)clip & 15) == 0 && ((uintptr_t)rast & 15) == 0 && ((uintptr_t)flags & 3) == 0 &&
                    ((uintptr_t)counts & 7) == 0, "misaligned buffer");
    cudaStream_t s = (cudaStream_t)stream;
    const long long npix = (long long)W * H * views;
    vcl_status st = vcl_cuda_check(ctx, cudaMemsetAsync(flags, 0, sizeof(uint32_t) * (size_t)npix, s), "ties memset");
    if (!st) st = vcl_cuda_check(ctx, cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s), "ties memset");
    if (st) return st;
    if ((long long)views * nt > 0) {
        const size_t tab = sizeof(float) * (size_t)(W + H);
        if (tab > 48 * 1024) cudaFuncSetAttribute(k_ties, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tab);
        k_ties<<<ctx->sm_count * 8, 256, tab, s>>>((const float4*)clip, nv, tri, nt, W, H, views,
                                                   (const float4*)rast, flags);
    }
    k_tie_count<<<ctx->sm_count * 4, 256, 0, s>>>(flags, npix, counts);
    return vcl_launch_check(ctx, "raster_ties");
}

}  // extern "C"

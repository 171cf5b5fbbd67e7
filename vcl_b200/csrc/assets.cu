// Asset loaders: Wavefront OBJ meshes, BMP textures and spherical-Gaussian
// lobe lists, the file formats the reference's demo reads
// (Attribute::loadOBJ buffer.cu:203-306, Texture::loadBMP buffer.cu:498-541,
// SGBuffer::loadTXT buffer.cu:706-732).  Host code only; the results are
// host arrays the caller uploads (vcl_fit_desc takes host pointers).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"

struct vcl_obj {
    // as in the file: one index array per attribute (0-based)
    std::vector<float> pos, texel, normal;
    std::vector<uint32_t> pos_idx, texel_idx, normal_idx;
    // welded: one vertex per distinct (position, texel, normal) corner
    std::vector<float> w_pos, w_uv, w_normal;
    std::vector<uint32_t> w_tri;
};

namespace {

thread_local std::string g_asset_err;

// Loader errors go to the context when one is given, and always to the
// calling thread's loader error (vcl_asset_error).
vcl_status asset_fail(vcl_ctx* ctx, vcl_status code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_asset_err = buf;
    if (ctx) vcl_fail(ctx, code, "%s", buf);
    return code;
}

#define ASSET_REQUIRE(cond, ...) \
    do { if (!(cond)) return asset_fail(ctx, VCL_ERR_ARG, __VA_ARGS__); } while (0)

// One face corner "p", "p/t", "p//n" or "p/t/n" (1-based; negative indices
// count back from the end, as OBJ allows).
bool parse_corner(const char* s, int np, int nt, int nn, long long& p, long long& t, long long& n) {
    p = t = n = 0;
    char* e = nullptr;
    p = strtoll(s, &e, 10);
    if (e == s) return false;
    if (*e == '/') {
        const char* q = e + 1;
        if (*q != '/') {
            t = strtoll(q, &e, 10);
            if (e == q) return false;
        } else {
            e = (char*)q;
        }
        if (*e == '/') {
            q = e + 1;
            n = strtoll(q, &e, 10);
            if (e == q) return false;
        }
    }
    if (*e != '\0') return false;
    auto fix = [](long long i, int count) { return i < 0 ? count + i + 1 : i; };
    p = fix(p, np);
    t = fix(t, nt);
    n = fix(n, nn);
    return true;
}

}  // namespace

extern "C" {

VCL_API const char* vcl_asset_error(void) { return g_asset_err.c_str(); }

VCL_API vcl_status vcl_obj_load(vcl_ctx* ctx, const char* path, vcl_obj** out) {
    ASSET_REQUIRE(path && out, "null argument");
    *out = nullptr;
    FILE* f = fopen(path, "r");
    ASSET_REQUIRE(f, "cannot open OBJ file %s", path);
    auto* o = new vcl_obj();
    char line[4096];
    int lineno = 0;
    vcl_status st = VCL_OK;
    while (fgets(line, sizeof line, f)) {
        ++lineno;
        char* s = line;
        while (*s == ' ' || *s == '\t') ++s;
        if (*s == '#' || *s == '\n' || *s == '\r' || *s == '\0') continue;
        char tag[8] = {0};
        int adv = 0;
        if (sscanf(s, "%7s%n", tag, &adv) != 1) continue;
        const char* rest = s + adv;
        if (!strcmp(tag, "v") || !strcmp(tag, "vn")) {
            float v[3];
            if (sscanf(rest, "%f %f %f", &v[0], &v[1], &v[2]) != 3) {
                st = asset_fail(ctx, VCL_ERR_ARG, "%s:%d: bad %s line", path, lineno, tag);
                break;
            }
            auto& dst = tag[1] ? o->normal : o->pos;
            dst.insert(dst.end(), v, v + 3);
        } else if (!strcmp(tag, "vt")) {
            float v[2];
            if (sscanf(rest, "%f %f", &v[0], &v[1]) != 2) {
                st = asset_fail(ctx, VCL_ERR_ARG, "%s:%d: bad vt line", path, lineno);
                break;
            }
            o->texel.insert(o->texel.end(), v, v + 2);
        } else if (!strcmp(tag, "f")) {
            // a polygon of n corners becomes a fan of n - 2 triangles
            std::vector<long long> P, T, N;
            char buf[4096];
            strncpy(buf, rest, sizeof buf - 1);
            buf[sizeof buf - 1] = 0;
            const int np = (int)(o->pos.size() / 3), nt = (int)(o->texel.size() / 2), nn = (int)(o->normal.size() / 3);
            bool ok = true;
            char* save = nullptr;
            for (char* tok = strtok_r(buf, " \t\r\n", &save); tok; tok = strtok_r(nullptr, " \t\r\n", &save)) {
                long long p, t, n;
                if (!parse_corner(tok, np, nt, nn, p, t, n) || p < 1 || p > np || t < 0 || t > nt || n < 0 || n > nn) {
                    ok = false;
                    break;
                }
                P.push_back(p); T.push_back(t); N.push_back(n);
            }
            if (!ok || P.size() < 3) {
                st = asset_fail(ctx, VCL_ERR_ARG, "%s:%d: bad face", path, lineno);
                break;
            }
            for (size_t k = 1; k + 1 < P.size(); ++k) {
                const size_t c[3] = {0, k, k + 1};
                for (size_t q : c) {
                    o->pos_idx.push_back((uint32_t)(P[q] - 1));
                    // a corner without a texel / normal index gets index 0
                    // when the file has texels / normals at all
                    o->texel_idx.push_back((uint32_t)(T[q] > 0 ? T[q] - 1 : 0));
                    o->normal_idx.push_back((uint32_t)(N[q] > 0 ? N[q] - 1 : 0));
                }
            }
        }
        // other statements (o, g, s, usemtl, mtllib, l, ...) carry nothing the fit uses
    }
    fclose(f);
    if (!st && o->pos.empty()) st = asset_fail(ctx, VCL_ERR_ARG, "%s: no vertices", path);
    if (st) {
        delete o;
        return st;
    }
    if (o->texel.empty()) o->texel_idx.clear();
    if (o->normal.empty()) o->normal_idx.clear();
    // weld: one vertex per distinct corner triple
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, uint32_t> ids;
    const size_t corners = o->pos_idx.size();
    for (size_t i = 0; i < corners; ++i) {
        const uint32_t p = o->pos_idx[i];
        const uint32_t t = o->texel_idx.empty() ? 0 : o->texel_idx[i];
        const uint32_t n = o->normal_idx.empty() ? 0 : o->normal_idx[i];
        auto key = std::make_tuple(p, t, n);
        auto it = ids.find(key);
        uint32_t id;
        if (it == ids.end()) {
            id = (uint32_t)(o->w_pos.size() / 3);
            ids.emplace(key, id);
            o->w_pos.insert(o->w_pos.end(), &o->pos[3 * (size_t)p], &o->pos[3 * (size_t)p] + 3);
            if (!o->texel.empty()) o->w_uv.insert(o->w_uv.end(), &o->texel[2 * (size_t)t], &o->texel[2 * (size_t)t] + 2);
            else o->w_uv.insert(o->w_uv.end(), {0.f, 0.f});
            if (!o->normal.empty())
                o->w_normal.insert(o->w_normal.end(), &o->normal[3 * (size_t)n], &o->normal[3 * (size_t)n] + 3);
            else o->w_normal.insert(o->w_normal.end(), {0.f, 0.f, 0.f});
        } else {
            id = it->second;
        }
        o->w_tri.push_back(id);
    }
    *out = o;
    return VCL_OK;
}

VCL_API void vcl_obj_free(vcl_obj* o) { delete o; }

VCL_API vcl_status vcl_obj_counts(const vcl_obj* o, int* n_pos, int* n_tri, int* n_texel, int* n_normal,
                                  int* n_welded) {
    if (!o) return VCL_ERR_ARG;
    if (n_pos) *n_pos = (int)(o->pos.size() / 3);
    if (n_tri) *n_tri = (int)(o->pos_idx.size() / 3);
    if (n_texel) *n_texel = (int)(o->texel.size() / 2);
    if (n_normal) *n_normal = (int)(o->normal.size() / 3);
    if (n_welded) *n_welded = (int)(o->w_pos.size() / 3);
    return VCL_OK;
}

VCL_API vcl_status vcl_obj_arrays(const vcl_obj* o, const float** pos, const uint32_t** pos_idx, const float** texel,
                                  const uint32_t** texel_idx, const float** normal, const uint32_t** normal_idx) {
    if (!o) return VCL_ERR_ARG;
    if (pos) *pos = o->pos.data();
    if (pos_idx) *pos_idx = o->pos_idx.data();
    if (texel) *texel = o->texel.empty() ? nullptr : o->texel.data();
    if (texel_idx) *texel_idx = o->texel_idx.empty() ? nullptr : o->texel_idx.data();
    if (normal) *normal = o->normal.empty() ? nullptr : o->normal.data();
    if (normal_idx) *normal_idx = o->normal_idx.empty() ? nullptr : o->normal_idx.data();
    return VCL_OK;
}

VCL_API vcl_status vcl_obj_welded(const vcl_obj* o, const float** pos, const float** uv, const float** normal,
                                  const uint32_t** tri) {
    if (!o) return VCL_ERR_ARG;
    if (pos) *pos = o->w_pos.data();
    if (uv) *uv = o->w_uv.data();
    if (normal) *normal = o->w_normal.data();
    if (tri) *tri = o->w_tri.data();
    return VCL_OK;
}

VCL_API vcl_status vcl_bmp_load(vcl_ctx* ctx, const char* path, int* width, int* height, int* channels, float* out) {
    ASSET_REQUIRE(path && width && height && channels, "null argument");
    FILE* f = fopen(path, "rb");
    ASSET_REQUIRE(f, "cannot open BMP file %s", path);
    unsigned char h[54];
    const bool head = fread(h, 1, 54, f) == 54 && h[0] == 'B' && h[1] == 'M';
    auto u32 = [&](int o) { return (uint32_t)h[o] | (uint32_t)h[o + 1] << 8 | (uint32_t)h[o + 2] << 16 | (uint32_t)h[o + 3] << 24; };
    auto u16 = [&](int o) { return (uint32_t)h[o] | (uint32_t)h[o + 1] << 8; };
    if (!head) {
        fclose(f);
        return asset_fail(ctx, VCL_ERR_ARG, "%s: not a BMP file", path);
    }
    uint32_t data_pos = u32(0x0A);
    const int32_t w = (int32_t)u32(0x12), hh = (int32_t)u32(0x16);
    const int bpp = (int)u16(0x1C);
    const uint32_t compression = u32(0x1E);
    if (w <= 0 || hh == 0 || (bpp != 8 && bpp != 24 && bpp != 32) || (compression != 0 && compression != 3)) {
        fclose(f);
        return asset_fail(ctx, VCL_ERR_ARG, "%s: unsupported BMP (%dx%d, %d bits, compression %u)", path, w, hh, bpp,
                        compression);
    }
    const int C = bpp / 8;
    const int H = hh < 0 ? -hh : hh;
    *width = w;
    *height = H;
    *channels = C;
    if (!out) {
        fclose(f);
        return VCL_OK;
    }
    if (data_pos == 0) data_pos = 54;
    const size_t stride = ((size_t)w * C + 3) / 4 * 4;   // rows are padded to 4 bytes
    std::vector<unsigned char> row(stride);
    vcl_status st = VCL_OK;
    if (fseek(f, (long)data_pos, SEEK_SET) != 0) st = asset_fail(ctx, VCL_ERR_ARG, "%s: truncated", path);
    for (int r = 0; r < H && !st; ++r) {
        if (fread(row.data(), 1, stride, f) != stride) {
            st = asset_fail(ctx, VCL_ERR_ARG, "%s: truncated pixel data", path);
            break;
        }
        // rows bottom-up (GL convention), as a positive-height BMP stores them
        const int y = hh > 0 ? r : H - 1 - r;
        for (int x = 0; x < w; ++x)
            for (int c = 0; c < C; ++c)   // channel c = byte C-1-c of the pixel (BGR -> RGB)
                out[((size_t)y * w + x) * C + c] = row[(size_t)x * C + (C - 1 - c)] / 255.f;
    }
    fclose(f);
    return st;
}

VCL_API vcl_status vcl_sg_load(vcl_ctx* ctx, const char* path, int max_lobes, int* lobes, float* axis, float* sharpness,
                               float* amplitude) {
    ASSET_REQUIRE(path && lobes, "null argument");
    FILE* f = fopen(path, "r");
    ASSET_REQUIRE(f, "cannot open lobe file %s", path);
    int k = 0;
    float v[7];
    vcl_status st = VCL_OK;
    for (;;) {
        int got = 0;
        for (; got < 7; ++got)
            if (fscanf(f, "%f", &v[got]) != 1) break;
        if (got == 0) break;
        if (got != 7) {
            st = asset_fail(ctx, VCL_ERR_ARG, "%s: lobe %d has %d of 7 numbers", path, k + 1, got);
            break;
        }
        if (axis && k < max_lobes) {
            axis[3 * k] = v[0]; axis[3 * k + 1] = v[1]; axis[3 * k + 2] = v[2];
            if (sharpness) sharpness[k] = v[3];
            if (amplitude) { amplitude[3 * k] = v[4]; amplitude[3 * k + 1] = v[5]; amplitude[3 * k + 2] = v[6]; }
        }
        ++k;
    }
    fclose(f);
    if (st) return st;
    *lobes = k;
    ASSET_REQUIRE(!axis || k <= max_lobes, "%s holds %d lobes, more than max_lobes = %d", path, k, max_lobes);
    return VCL_OK;
}

}  // extern "C"

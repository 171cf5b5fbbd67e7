/*
 * vcl_oracle.h -- CPU restatement of the vcl (nvdiffrast-style) differentiable
 * rendering path.  TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the
 * CPU-baseline leg of bench.py call this as the checker; the product never
 * links or calls it.
 *
 * Every function restates one reference operator (file:line given beside it,
 * paths relative to nvdiffrast/nvdiffrast/ of the reference).  Layouts follow
 * the reference: pixels are row-major, rows bottom-up (GL), views stacked
 * ("depth"); per-pixel vectors are interleaved (pidx*dim + c).  The raster
 * buffer is float4 (u, v, z/w, triangle_id + 1) per pixel.
 *
 * Differences from the reference's data layout that the whole project shares:
 *   - clip-space positions are per view: clip[view][vertex][4];
 *   - a texture pyramid is one packed array, level l at offset
 *     sum_{k<l} (W>>k)*(H>>k)*C floats.
 *
 * `mode`: 0 = compat (the reference's arithmetic and quirks), 1 = exact
 * (quirks fixed, see each function).
 */
#ifndef VCL_ORACLE_H
#define VCL_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- projection: project.cu:69-77 (fwd), :114-131 (bwd) ---------------- */
void orc_project_fwd(int nv, const float* mat16, const float* pos, int dim, float* out);
void orc_project_bwd(int nv, const float* mat16, const float* grad_out, int dim, float* grad_pos);

/* ---- rasterize forward: restatement of the GL program rasterize.cpp:91-202
 *      with the fixed-function state of :252-268 (see vcl_oracle.c) ------- */
void orc_rasterize_fwd(int W, int H, int views, const float* clip, int nv,
                       const uint32_t* tri, int nt, int enable_db,
                       float* rast, float* db);
/* ---- GL tie census of a finished raster (no reference counterpart: GL
 *      leaves these pixels implementation-defined, rasterize.cpp:252-254).
 *      flags[pixel] |= 1: the centre lies exactly on an edge of a triangle
 *      whose closed interior holds it (the top-left rule decides);
 *      flags[pixel] |= 2: a triangle other than the winner covers the pixel
 *      at exactly the winning depth (the lower id decides).
 *      counts[0], counts[1] = pixels with bit 1, bit 2. ------------------- */
void orc_raster_ties(int W, int H, int views, const float* clip, int nv,
                     const uint32_t* tri, int nt, const float* rast,
                     uint32_t* flags, long long* counts);
/* ---- rasterize backward: rasterize.cu:84-141 ---------------------------- */
void orc_rasterize_bwd(int W, int H, int views, const float* clip, int nv,
                       const uint32_t* tri, const float* rast,
                       const float* grad_bary, float* grad_clip);

/* ---- interpolate: interpolate.cu:20-49 (fwd), :114-143 (bwd) ------------ */
void orc_interpolate_fwd(int W, int H, int views, int dim, int enable_da,
                         const float* rast, const float* db, const float* attr,
                         const uint32_t* tri, float* out, float* out_da);
void orc_interpolate_bwd(int mode, int W, int H, int views, int dim,
                         const float* rast, const float* attr, const uint32_t* tri,
                         const float* grad_out, float* grad_attr, float* grad_bary);

/* ---- texture: texturemap.cu:22-114 (fwd), :160-319 (bwd) ---------------- */
int orc_tex_levels(int tw, int th, int requested);
size_t orc_tex_level_offset(int tw, int th, int C, int level);
void orc_texture_fwd(int W, int H, int views, int tw, int th, int C, int levels,
                     const float* pyramid, const float* rast, const float* uv,
                     const float* uv_da, float* out);
void orc_texture_bwd(int mode, int W, int H, int views, int tw, int th, int C, int levels,
                     const float* pyramid, const float* rast, const float* uv,
                     const float* uv_da, const float* grad_out, float* grad_pyramid,
                     float* grad_uv, float* grad_uv_da);
/* ---- mip chain: buffer.cu:449-484 (build), :615-648 (grad push-down) ----- */
void orc_mip_build(int tw, int th, int C, int levels, float* pyramid);
void orc_mip_pushdown(int mode, int tw, int th, int C, int levels, float* grad_pyramid);
/* ---- clamp: buffer.cu:65-72 via Texture::clamp :588-594 ----------------- */
void orc_clamp(size_t n, float* p, float lo, float hi);

/* ---- antialias: antialias.cu:17-95 (fwd), :196-300 (bwd) ---------------- */
void orc_antialias_fwd(int W, int H, int views, int C, const float* clip, int nv,
                       const uint32_t* tri, const float* rast, const float* in, float* out);
void orc_antialias_bwd(int mode, int W, int H, int views, int C, const float* clip, int nv,
                       const uint32_t* tri, const float* rast, const float* in,
                       const float* grad_out, float* grad_in, float* grad_clip);

/* ---- shading: material.cu ------------------------------------------------ */
void orc_normal_axis_fwd(int W, int H, int views, const float* rast, const float* rot16,
                         const float* normal, const uint32_t* tri, float* out);
void orc_view_axis_fwd(int W, int H, int views, const float* pvinv9, float* out);
void orc_sg_specular_fwd(int W, int H, int views, const float* rast, const float* normal,
                         const float* view, const float* rough, float ior,
                         float* out_axis, float* out_sharp, float* out_amp);
void orc_sg_specular_bwd(int W, int H, int views, const float* rast, const float* normal,
                         const float* view, const float* rough, float ior,
                         const float* grad_amp, const float* grad_sharp, float* grad_rough);
void orc_sg_fwd(int W, int H, int views, int C, const float* rast, int K,
                const float* axis, const float* sharp, const float* amp,
                const float* normal, const float* diffuse,
                const float* spec_axis, const float* spec_sharp, const float* spec_amp,
                float* out, float* out_diffenv, float* out_specenv);
void orc_sg_bwd(int mode, int W, int H, int views, int C, const float* rast, int K,
                const float* axis, const float* sharp, const float* amp,
                const float* normal, const float* diffuse,
                const float* spec_axis, const float* spec_sharp, const float* spec_amp,
                const float* grad_out, float* grad_diffuse,
                float* grad_axis, float* grad_sharp, float* grad_amp,
                float* grad_spec_axis, float* grad_spec_sharp, float* grad_spec_amp);

/* ---- loss + optimizer: loss.cu:22-57, optimize.cu:84-115 --------------- */
float orc_mse(int mode, size_t n, const float* pred, const float* target, float* grad);
void orc_adam(int mode, size_t n, float* p, const float* g, float* m, float* v,
              double lr, double b1, double b2, double eps, int step);

#ifdef __cplusplus
}
#endif
#endif

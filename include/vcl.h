/*
 * vcl.h -- C ABI of the B200-native (sm_100a) differentiable-rendering path.
 *
 * Drop-in for the operator API of the reference (236088/vcl,
 * nvdiffrast/nvdiffrast/): each entry point below names the reference
 * function it replaces.  The reference's operators are C++ classes with
 * static init/forward/backward over Params structs that hold raw device
 * pointers; here the same operators are plain functions over raw device
 * pointers and sizes, with no C++ or torch types in any signature.
 *
 * Conventions (shared by every call):
 *   - All buffer arguments are DEVICE pointers (cudaMalloc'd, FP32 unless
 *     noted, contiguous), owned by the caller.  Outputs are written, never
 *     allocated.  Matrices are device arrays too (the reference keeps them
 *     in device memory: matrix.cu:55-58, :220-221).
 *   - Layouts are the reference's: pixels row-major with rows bottom-up,
 *     views stacked; per-pixel vectors interleaved (pixel*dim + c); the
 *     raster buffer is float4 (u, v, z/w, triangle_id + 1).  Per-view
 *     quantities: clip positions [views][nv][4], matrices [views][16]
 *     column-major, view inverses [views][9] column-major.
 *   - A texture pyramid is one packed array: level l starts at
 *     sum_{k<l} (tw>>k)*(th>>k)*C floats (vcl_tex_level_offset).
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are
 *     asynchronous and stream-ordered; none synchronizes the device.
 *   - Errors are returned, never fatal (the reference prints and exit(1)s,
 *     common.h:36-47).  vcl_last_error() gives the message.
 *   - A context is not thread-safe: use one per host thread.
 *   - Triangle ids read from a raster buffer are checked against nt and
 *     vertex indices against nv; out-of-range entries are skipped (the
 *     reference reads out of bounds there) and reported by
 *     vcl_check_indices().
 *   - Mode (vcl_set_mode): VCL_MODE_COMPAT reproduces the reference's
 *     arithmetic and quirks; VCL_MODE_EXACT fixes them (per call below).
 */
#ifndef VCL_H
#define VCL_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VCL_API __attribute__((visibility("default")))

typedef struct vcl_ctx vcl_ctx;
typedef int vcl_status;

#define VCL_OK 0
#define VCL_ERR_ARG 1      /* invalid argument (null pointer, bad size) */
#define VCL_ERR_CUDA 2     /* a CUDA runtime call failed */
#define VCL_ERR_NOMEM 3    /* workspace allocation failed */
#define VCL_ERR_STATE 4    /* object in the wrong state for the call */

#define VCL_MODE_COMPAT 0
#define VCL_MODE_EXACT 1

/* ---------------------------------------------------------------- context */
VCL_API const char* vcl_version(void);
/* Create a context on `device` (makes it current).  No reference
 * counterpart: the reference uses global state and the default stream. */
VCL_API vcl_status vcl_create(int device, vcl_ctx** out);
VCL_API void vcl_destroy(vcl_ctx* ctx);
VCL_API const char* vcl_last_error(const vcl_ctx* ctx);
VCL_API vcl_status vcl_set_mode(vcl_ctx* ctx, int mode);
VCL_API int vcl_get_mode(const vcl_ctx* ctx);
/* Raster binning schedule: tile edge in pixels (8, 16 or 32) and bin list
 * capacity in entries (0 = automatic).  Replaces the fixed-function GL
 * rasterizer configuration of rasterize.cpp:206-254. */
VCL_API vcl_status vcl_set_raster_config(vcl_ctx* ctx, int tile, long long bin_capacity);
VCL_API vcl_status vcl_get_raster_config(const vcl_ctx* ctx, int* tile, long long* bin_capacity);
/* Whether fit jobs of this context time the raster schedules on their first
 * fused step (1, the default) or take a size-based one (0: tile 32 for
 * images of at least 512x512, else 16; default direct-raster areas). */
VCL_API vcl_status vcl_set_raster_autotune(vcl_ctx* ctx, int enable);
/* Box areas (pixels) below which a triangle skips the tile bins: up to
 * `small_area` it is rasterized by its setup thread, up to `medium_area` by
 * one warp (-1: the defaults 256 and 4096; 0 and 0 bin every triangle). */
VCL_API vcl_status vcl_set_raster_areas(vcl_ctx* ctx, int small_area, int medium_area);
/* Number of tiles that overflowed the bin list in the last raster call
 * (they were rasterized by the slower all-triangles path; results are
 * unaffected).  Reading it synchronizes `stream`. */
VCL_API vcl_status vcl_raster_overflow_count(vcl_ctx* ctx, void* stream, long long* count);
/* Nonzero in *bad when a kernel met an out-of-range triangle id or vertex
 * index since the last call (clears the flag; synchronizes `stream`). */
VCL_API vcl_status vcl_check_indices(vcl_ctx* ctx, void* stream, int* bad);
/* Pre-size the raster workspace for up to `views*nt` triangles on
 * `views` W x H views so that later calls allocate nothing (needed before
 * CUDA graph capture). */
VCL_API vcl_status vcl_reserve_raster(vcl_ctx* ctx, int W, int H, int views, int nt);

/* Packed texture pyramid helpers (Texture::init buffer.cu:379-407). */
VCL_API int vcl_tex_levels(int tw, int th, int requested);
VCL_API size_t vcl_tex_level_offset(int tw, int th, int C, int level);

/* --------------------------------------------------------------- project */
/* Project::forward (project.cu:36-46, kernel :26-34):
 * out[v][i] = M_v * [pos_i, 1] for `views` column-major matrices; dim 3 or 4. */
VCL_API vcl_status vcl_project_fwd(vcl_ctx* ctx, const float* mats, int views, const float* pos, int nv,
                                   int dim, float* out, void* stream);
/* Project::backward (project.cu:133-138, kernel :71-88): grad_pos +=
 * sum_v M_v^T grad_out[v] (3x3 part; the matrix gradient is not produced). */
VCL_API vcl_status vcl_project_bwd(vcl_ctx* ctx, const float* mats, int views, const float* grad_out, int nv,
                                   int dim, float* grad_pos, void* stream);

/* ------------------------------------------------------------- rasterize */
/* Rasterize::forward (rasterize.cpp:257-282 with the GL program :91-202):
 * CUDA triangle setup + tile binner + fine rasterizer.  No culling,
 * GL_LESS depth test (equal depth keeps the lower triangle id), clip to
 * -w <= z <= w, top-left fill rule (window y up).  rast = (u, v, z/w, id+1)
 * per pixel, 0 where nothing is drawn; db (when non-NULL) = the reference's
 * per-pixel barycentric derivatives var_db * w.  Triangle ids are
 * bit-identical to the CPU restatement of the same rules. */
VCL_API vcl_status vcl_rasterize_fwd(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt,
                                     int W, int H, int views, float* rast, float* db, void* stream);
/* vcl_rasterize_fwd on a fixed scratch area that is part of the loaded
 * module (a file-scope device array of VCL_RASTER_SCRATCH_BYTES) instead of
 * the context workspace: the call allocates nothing, for callers that must
 * not allocate device memory or synchronize the device on their per-frame
 * path.  No counterpart in the reference (its rasterizer has no workspace).
 * Same arguments and results as vcl_rasterize_fwd.  Requests whose depth
 * keys (8 B per pixel and view), triangle records and medium-list entries
 * (VCL_RASTER_BYTES_PER_VIEW_TRIANGLE = 96 + 4 B per view and triangle) and
 * tile counters (12 B per tile and view), each rounded up to 256 B, exceed
 * the limit return VCL_ERR_ARG; what is left holds the tile bin lists (4 B
 * per entry).  No part of the scratch needs to start at zero.  One scratch
 * per device: calls whose work overlaps on the device race, so serialize
 * them.  The first call per device (or vcl_raster_scratch_init) resolves the
 * scratch address with the context's device current; make it during set-up,
 * before any stream capture.  cudaDeviceReset unloads the module and with it
 * the scratch: after a reset, call vcl_raster_scratch_init again (it always
 * resolves the address anew) before the next static call. */
#define VCL_RASTER_SCRATCH_BYTES (32u << 20)
#define VCL_RASTER_BYTES_PER_VIEW_TRIANGLE 100
VCL_API size_t vcl_raster_scratch_bytes(void);
VCL_API vcl_status vcl_raster_scratch_init(vcl_ctx* ctx);
VCL_API vcl_status vcl_rasterize_fwd_static(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt,
                                            int W, int H, int views, float* rast, float* db, void* stream);
/* Rasterize::backward (rasterize.cu:143-148, kernel :84-141): grad_clip
 * (x, y, w of each vertex) += dL/d(clip) from grad_bary [pixels][2].  The
 * DB gradient is not consumed (as in the reference). */
VCL_API vcl_status vcl_rasterize_bwd(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt, int W,
                                     int H, int views, const float* rast, const float* grad_bary, float* grad_clip,
                                     void* stream);
/* GL tie census of a finished raster `rast` (the output of vcl_rasterize_fwd
 * for the same clip/tri).  No counterpart in the reference: these are the
 * pixels where GL leaves the result implementation-defined, so where a real
 * GL driver (rasterize.cpp:252-254) may legally give another triangle id
 * than these rules.  flags [views*H*W] (device, written whole): bit 1 = the
 * pixel centre lies exactly on an edge of a triangle whose closed interior
 * holds it (the top-left rule decided coverage); bit 2 = a triangle other
 * than the winner covers the pixel at exactly the winning depth (the lower
 * id decided).  counts [2] (device, written): pixels with bit 1, bit 2.
 * A diagnostic, not part of the fit path. */
VCL_API vcl_status vcl_raster_ties(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt, int W, int H,
                                   int views, const float* rast, uint32_t* flags, unsigned long long* counts,
                                   void* stream);

/* ----------------------------------------------------------- interpolate */
/* Interpolate::forward (interpolate.cu:51-60, kernel :20-49): out[p] =
 * a0*u + a1*v + a2*(1-u-v); with out_da non-NULL also the screen-space
 * derivatives from db.  Uncovered pixels get 0. */
VCL_API vcl_status vcl_interpolate_fwd(vcl_ctx* ctx, const float* rast, const float* db, int W, int H, int views,
                                       const float* attr, int nv, int dim, const uint32_t* tri, int nt, float* out,
                                       float* out_da, void* stream);
/* Interpolate::backward (interpolate.cu:145-149, kernel :114-143):
 * grad_attr += (atomics; may be NULL); grad_bary [pixels][2] at covered
 * pixels: stored (COMPAT, :141) or accumulated (EXACT). */
VCL_API vcl_status vcl_interpolate_bwd(vcl_ctx* ctx, const float* rast, int W, int H, int views,
                                       const float* attr, int nv, int dim, const uint32_t* tri, int nt,
                                       const float* grad_out, float* grad_attr, float* grad_bary, void* stream);

/* --------------------------------------------------------------- texture */
/* Texturemap::forward (texturemap.cu:116-123, kernels :67-114): trilinear
 * mip sampling when levels > 1, bilinear on level 0 otherwise; texel
 * coordinate uv*size (no half-texel offset), the reference's clamping.
 * uv_da is read only when levels > 1.  Uncovered pixels get 0. */
VCL_API vcl_status vcl_texture_fwd(vcl_ctx* ctx, const float* rast, const float* uv, const float* uv_da,
                                   int W, int H, int views, const float* pyramid, int tw, int th, int C,
                                   int levels, float* out, void* stream);
/* Texturemap::backward (texturemap.cu:321-326, kernels :229-319):
 * grad_pyramid += texel gradients (vector FP32 atomics); grad_uv [p][2] and
 * grad_uv_da [p][4] stored at covered pixels (either may be NULL).  COMPAT
 * keeps the missing factor on dlevel/d(uvDA).zw (:185); EXACT applies it. */
VCL_API vcl_status vcl_texture_bwd(vcl_ctx* ctx, const float* rast, const float* uv, const float* uv_da,
                                   int W, int H, int views, const float* pyramid, int tw, int th, int C,
                                   int levels, const float* grad_out, float* grad_pyramid, float* grad_uv,
                                   float* grad_uv_da, void* stream);
/* Texture::buildMIP (buffer.cu:474-484, kernel :449-472): levels 1..L-1
 * from level 0 by 2x2 box averages. */
VCL_API vcl_status vcl_texture_build_mips(vcl_ctx* ctx, float* pyramid, int tw, int th, int C, int levels,
                                          void* stream);
/* TextureGrad::gradSumup (buffer.cu:638-648, kernel :615-636): push each
 * level's gradient down to its 4 children, coarsest first, NaN-guarded.
 * COMPAT weight 1 (the reference), EXACT weight 1/4 (adjoint of the box). */
VCL_API vcl_status vcl_texture_grad_pushdown(vcl_ctx* ctx, float* grad_pyramid, int tw, int th, int C,
                                             int levels, void* stream);
/* Texture::clamp's clamp (buffer.cu:588-594, kernel :65-72). */
VCL_API vcl_status vcl_clamp(vcl_ctx* ctx, float* p, size_t n, float lo, float hi, void* stream);

/* ------------------------------------------------------------- antialias */
/* Antialias::forward (antialias.cu:97-108, kernel :57-95): out = in, then
 * analytic silhouette blending across horizontal and vertical pixel pairs
 * whose triangle ids differ (all stores happen before the edge adds). */
VCL_API vcl_status vcl_antialias_fwd(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt,
                                     const float* rast, int W, int H, int views, int C, const float* in,
                                     float* out, void* stream);
/* Antialias::backward (antialias.cu:302-313, kernel :261-300): grad_in =
 * grad_out then edge terms; grad_clip (x, y, w) += edge-vertex gradients
 * (may be NULL).  COMPAT keeps the horizontal-edge id typo of :279 (a
 * fetch of the background's triangle contributes nothing); EXACT uses the
 * neighbour's id like the forward pass. */
VCL_API vcl_status vcl_antialias_bwd(vcl_ctx* ctx, const float* clip, int nv, const uint32_t* tri, int nt,
                                     const float* rast, int W, int H, int views, int C, const float* in,
                                     const float* grad_out, float* grad_in, float* grad_clip, void* stream);

/* --------------------------------------------------------------- shading */
/* NormalAxis::forward (material.cu:71-77, kernel :25-48): normalized
 * interpolated vertex normal rotated by the column-major rot16. */
VCL_API vcl_status vcl_normal_axis_fwd(vcl_ctx* ctx, const float* rast, int W, int H, int views,
                                       const float* rot16, const float* normal, int nv, const uint32_t* tri,
                                       int nt, float* out, void* stream);
/* ViewAxis::forward (material.cu:110-118, kernel :92-108): per-pixel view
 * ray normalize(pvinv_v * (px/W*2-1, py/H*2-1, 1)) for every pixel. */
VCL_API vcl_status vcl_view_axis_fwd(vcl_ctx* ctx, int W, int H, int views, const float* pvinv, float* out,
                                     void* stream);
/* SGSpecular::forward (material.cu:185-201, kernel :145-183). */
VCL_API vcl_status vcl_sg_specular_fwd(vcl_ctx* ctx, const float* rast, int W, int H, int views,
                                       const float* normal, const float* view, const float* roughness, float ior,
                                       float* out_axis, float* out_sharpness, float* out_amplitude, void* stream);
/* SGSpecular::backward (material.cu:251-256, kernel :203-249): gradient to
 * roughness only, NaN-guarded. */
VCL_API vcl_status vcl_sg_specular_bwd(vcl_ctx* ctx, const float* rast, int W, int H, int views,
                                       const float* normal, const float* view, const float* roughness, float ior,
                                       const float* grad_amplitude, const float* grad_sharpness,
                                       float* grad_roughness, void* stream);
/* SphericalGaussian::forward (material.cu:325-339, kernel :285-323):
 * out = diffuse * sum_k SG<diffuse lobe, k> a_k + sum_k SG<spec lobe, k> a_k
 * over K lobes (axis [K][3], sharpness [K], amplitude [K][C]).  out_diffenv
 * and out_specenv may be NULL. */
VCL_API vcl_status vcl_sg_fwd(vcl_ctx* ctx, const float* rast, int W, int H, int views, int C, int K,
                              const float* axis, const float* sharpness, const float* amplitude,
                              const float* normal, const float* diffuse, const float* spec_axis,
                              const float* spec_sharpness, const float* spec_amplitude, float* out,
                              float* out_diffenv, float* out_specenv, void* stream);
/* SphericalGaussian::backward (material.cu:440-445, kernel :369-438).
 * Per-lobe gradients (grad_axis/sharpness/amplitude) are sums over all
 * pixels (block-reduced, one atomic per block and lobe parameter); the
 * per-pixel ones (grad_diffuse, grad_spec_*) are accumulated in place.
 * COMPAT indexes grad_spec_sharpness by lobe (:436) and grad_spec_amplitude
 * by pixel*C+channel (:430; size it [pixels][C]); EXACT indexes both by
 * pixel.  Any gradient pointer may be NULL. */
VCL_API vcl_status vcl_sg_bwd(vcl_ctx* ctx, const float* rast, int W, int H, int views, int C, int K,
                              const float* axis, const float* sharpness, const float* amplitude,
                              const float* normal, const float* diffuse, const float* spec_axis,
                              const float* spec_sharpness, const float* spec_amplitude,
                              const float* grad_out, float* grad_diffuse, float* grad_axis,
                              float* grad_sharpness, float* grad_amplitude, float* grad_spec_axis,
                              float* grad_spec_sharpness, float* grad_spec_amplitude, void* stream);

/* ------------------------------------------------------ loss / optimizer */
/* MSELoss::backward (loss.cu:41-57, kernels :22-39): grad = pred - target
 * and *loss_dev (device float) = sum(grad^2)/2 over all n elements.  The
 * reference's reported value drops elements beyond the largest power of
 * two; this one does not (the gradient is identical). */
VCL_API vcl_status vcl_mse(vcl_ctx* ctx, const float* pred, const float* target, size_t n, float* grad,
                           float* loss_dev, void* stream);
/* Adam::step (optimize.cu:107-115, kernel :95-106) for the `step`-th call
 * (1-based).  Moments in FP32, update in FP64, NaN-guarded.  COMPAT bias
 * correction uses beta^(step+1) (the reference's off-by-one), EXACT beta^step.
 * m and v must start zeroed (the reference leaves them uninitialized). */
VCL_API vcl_status vcl_adam_step(vcl_ctx* ctx, float* p, const float* g, float* m, float* v, size_t n,
                                 double lr, double beta1, double beta2, double eps, int step, void* stream);


/* ------------------------------------------------------------ fit jobs */
/* One inverse-rendering fit job: mesh, texture pyramid, SG lobes, Adam
 * state and per-view buffers resident on the device, and one call per
 * fit iteration.  This is the reference's PresetPrimitives wiring
 * (preset_primitives.cpp:7-134 init, :160-230 update) as a library object:
 * project -> rasterize(+DB) -> interpolate(uv, DA) -> texture(mip) ->
 * NormalAxis/ViewAxis/SGSpecular/SG shading -> antialias -> MSE, the full
 * backward pass, mip gradient push-down, then Adam on the enabled
 * parameter groups (vertex positions, texture level 0, SG lobes), texture
 * clamp to [0,1] and mip rebuild.  Roughness is the constant `roughness`.
 * All host pointers in the descriptor are read during vcl_fit_create only. */
typedef struct vcl_fit vcl_fit;

typedef struct {
    int W, H, views;            /* render size and view count */
    int C;                      /* texture / image channels (1..8) */
    int K;                      /* SG lobes */
    int nv, nt;                 /* vertices, triangles */
    int tex_w, tex_h, levels;   /* texture size and mip levels (vcl_tex_levels) */
    const float* pos;           /* [nv][3] initial positions */
    const uint32_t* tri;        /* [nt][3] */
    const float* uv;            /* [nv][2] */
    const float* normal;        /* [nv][3] shading normals (constant) */
    const float* tex;           /* [tex_h][tex_w][C] initial level 0 */
    const float* lobe_axis;     /* [K][3] */
    const float* lobe_sharp;    /* [K] */
    const float* lobe_amp;      /* [K][C] */
    const float* mvp;           /* [views][16] column-major */
    const float* pvinv;         /* [views][9] column-major */
    const float* rot;           /* [16] object rotation (NormalAxis) */
    float roughness, ior;
    double lr, beta1, beta2, eps;
    int learn_pos, learn_tex, learn_lobes;
    /* per-group Adam step sizes (the reference sets each parameter group's
     * Adam separately, preset_primitives.cpp:103-115); 0 = use `lr` */
    double lr_pos, lr_tex, lr_lobes;
} vcl_fit_desc;

/* Execution strategy of vcl_fit_step. */
#define VCL_FIT_PLAIN 0   /* one kernel per reference operator, as the reference wires them */
#define VCL_FIT_FUSED 1   /* fused per-pixel forward/backward kernels + fused optimizer pass */

VCL_API vcl_status vcl_fit_create(vcl_ctx* ctx, const vcl_fit_desc* desc, vcl_fit** out);
VCL_API void vcl_fit_destroy(vcl_fit* fit);
/* Destroys the job without synchronizing the device: its device memory is
 * returned in stream order on `stream`, after all work already queued there
 * (the job's last step must be on `stream` or complete). */
VCL_API void vcl_fit_destroy_async(vcl_fit* fit, void* stream);
VCL_API vcl_status vcl_fit_set_strategy(vcl_fit* fit, int strategy);
/* Target images [views][H][W][C]; `src` is a device pointer when
 * src_is_device, else host memory (pinned for an asynchronous copy). */
VCL_API vcl_status vcl_fit_set_target(vcl_fit* fit, const float* src, int src_is_device, void* stream);
/* New cameras for the next iterations (host arrays as in the descriptor). */
VCL_API vcl_status vcl_fit_set_cameras(vcl_fit* fit, const float* mvp, const float* pvinv, void* stream);
/* One fit iteration (forward, backward, optimizer).  Asynchronous.  If a
 * target was staged, the step first waits for its upload and makes it the
 * target. */
VCL_API vcl_status vcl_fit_step(vcl_fit* fit, void* stream);
/* Sets up the fused strategy now instead of at the first fused step: raster
 * autotuning and capture of the step's graph on `stream` (a created stream,
 * not the legacy default stream).  Synchronizes `stream`. */
VCL_API vcl_status vcl_fit_prepare(vcl_fit* fit, void* stream);
/* Uploads the NEXT step's target images from host memory (pinned, for an
 * asynchronous copy) into a staging buffer on `copy_stream`, so that the
 * upload overlaps the current step; the next vcl_fit_step consumes it.  Two
 * device staging buffers are used in turn (allocated at the first two
 * calls), so an upload does not wait for the step that consumes the one
 * before it.  One staged target at a time (VCL_ERR_ARG if the last one was
 * not consumed). */
VCL_API vcl_status vcl_fit_stage_target(vcl_fit* fit, const float* host_src, void* copy_stream);
/* Forward only with the current parameters: antialiased image
 * [views][H][W][C] into the device buffer `out`. */
VCL_API vcl_status vcl_fit_render(vcl_fit* fit, float* out, void* stream);
/* Device address of the last step's loss (one float). */
VCL_API const float* vcl_fit_loss_device(const vcl_fit* fit);
/* Copies the last step's loss to *loss_host; synchronizes `stream`. */
VCL_API vcl_status vcl_fit_read_loss(vcl_fit* fit, float* loss_host, void* stream);
/* The same copy, stream-ordered without waiting: *loss_host (pinned host
 * memory) holds the loss once `stream` has passed this point, so a caller can
 * read every step's loss while the next steps are already queued.  No
 * reference counterpart (Loss::loss reads back synchronously every
 * iteration, preset_primitives.cpp:222). */
VCL_API vcl_status vcl_fit_read_loss_async(vcl_fit* fit, float* loss_host, void* stream);
/* Copies the current parameters to host memory (any pointer may be NULL);
 * synchronizes `stream`. */
VCL_API vcl_status vcl_fit_read_params(vcl_fit* fit, float* pos, float* tex_level0, float* lobe_axis,
                                       float* lobe_sharp, float* lobe_amp, void* stream);
/* Checkpoint / resume of a job (no reference counterpart; the reference
 * keeps no state across runs): vcl_fit_save_state writes, into host memory
 * of vcl_fit_state_bytes() bytes, a header (shapes, Adam step) and the
 * positions, texture pyramid, lobes and the Adam moments of every group;
 * vcl_fit_load_state restores them into a job of the same shapes, which
 * then continues as the saved one would.  Both synchronize `stream`; no step
 * of the job may be in flight elsewhere. */
VCL_API size_t vcl_fit_state_bytes(const vcl_fit* fit);
VCL_API vcl_status vcl_fit_save_state(vcl_fit* fit, void* host_dst, size_t bytes, void* stream);
VCL_API vcl_status vcl_fit_load_state(vcl_fit* fit, const void* host_src, size_t bytes, void* stream);
/* The raster tile size the fused strategy's autotuner picked for this job
 * (tuned on first use by timing tiles 8, 16 and 32 on the job's geometry)
 * and the measured milliseconds per raster call for each (ms_per_tile[3],
 * may be NULL). */
VCL_API vcl_status vcl_fit_raster_tuning(vcl_fit* fit, int* tile, float* ms_per_tile);
/* The fused strategy's raster binning schedule for this job: tile edge,
 * box area (pixels) up to which triangles are rasterized directly instead
 * of binned, bin-list capacity, whether it came from the process-wide tuning
 * cache, and the overflowed tiles of the last step (any pointer may be
 * NULL; overflow_tiles synchronizes the device).  The autotuner times tile
 * {8, 16, 32} at the default direct area, then direct areas {0, 64, 1024}
 * at the best tile, on the job's first fused step
 * and sizes the capacity to twice the measured bin demand (at least the
 * automatic capacity); jobs of the same
 * (W, H, views, power-of-two triangle count) reuse the cached choice. */
VCL_API vcl_status vcl_fit_raster_schedule(vcl_fit* fit, int* tile, int* small_area, long long* bin_capacity,
                                           int* from_cache, long long* overflow_tiles);
VCL_API void vcl_raster_tuning_cache_clear(void);
/* Average device time (ms per launch) of each fused-step stage on the job's
 * current state, after at least one fused step: ms[i] for stage i of
 * vcl_fit_kernel_name(i) ("raster", "shade_fwd", "aa_fwd_mse", "aa_bwd",
 * "bwd_pix", "sg_lobes", and "bwd_pix+sg_lobes": the last two on two streams
 * as the step runs them); one untimed launch, then `reps` timed ones on
 * `stream`.  Parameters and Adam moments are untouched; the gradient
 * buffers are cleared (the next step recomputes them).  Synchronizes. */
VCL_API int vcl_fit_kernel_count(void);
VCL_API const char* vcl_fit_kernel_name(int i);
VCL_API vcl_status vcl_fit_time_kernels(vcl_fit* fit, void* stream, int reps, float* ms, int n);
/* Device bytes a job with this descriptor holds at most (arena plus the
 * fused strategy's raster workspace), for admission control. */
VCL_API size_t vcl_fit_footprint(const vcl_fit_desc* desc);
/* Number of kernel launches one vcl_fit_step issues with the current
 * strategy (memsets and copies not counted). */
VCL_API int vcl_fit_launches_per_step(const vcl_fit* fit);

/* --------------------------------------------------------------- assets */
/* Wavefront OBJ (Attribute::loadOBJ, buffer.cu:203-306): `v`, `vt`, `vn`
 * and `f` lines with corners p, p/t, p//n or p/t/n (1-based, negative =
 * from the end); polygons are split into triangle fans; other statements
 * are skipped.  The result keeps one index array per attribute, as the
 * reference does (absent attributes: NULL arrays), and a welded form with
 * one vertex per distinct (position, texel, normal) corner and one shared
 * index array, the layout of vcl_fit_desc (missing texels / normals are 0).
 * Arrays are host memory owned by the object until vcl_obj_free.  The
 * loaders need no device; `ctx` may be NULL, and the message of a failed
 * load is also kept per thread in vcl_asset_error(). */
typedef struct vcl_obj vcl_obj;
VCL_API const char* vcl_asset_error(void);
VCL_API vcl_status vcl_obj_load(vcl_ctx* ctx, const char* path, vcl_obj** out);
VCL_API void vcl_obj_free(vcl_obj* obj);
VCL_API vcl_status vcl_obj_counts(const vcl_obj* obj, int* n_pos, int* n_tri, int* n_texel, int* n_normal,
                                  int* n_welded);
VCL_API vcl_status vcl_obj_arrays(const vcl_obj* obj, const float** pos, const uint32_t** pos_idx,
                                  const float** texel, const uint32_t** texel_idx, const float** normal,
                                  const uint32_t** normal_idx);
VCL_API vcl_status vcl_obj_welded(const vcl_obj* obj, const float** pos, const float** uv, const float** normal,
                                  const uint32_t** tri);
/* BMP (Texture::loadBMP, buffer.cu:498-541): 8-, 24- or 32-bit uncompressed
 * pixels to floats in [0, 1], [height][width][channels], rows bottom-up as
 * the file stores them, channels in reverse byte order within a pixel as
 * the reference converts them (24-bit BGR gives RGB).  Rows are read with
 * their 4-byte padding (the reference reads them unpadded, which agrees
 * when width x channels is a multiple of 4); top-down (negative height)
 * files are flipped to bottom-up.  With out = NULL only the size is
 * returned. */
VCL_API vcl_status vcl_bmp_load(vcl_ctx* ctx, const char* path, int* width, int* height, int* channels, float* out);
/* Spherical-Gaussian lobe list (SGBuffer::loadTXT, buffer.cu:706-732):
 * whitespace-separated records of 7 numbers -- axis x y z, sharpness,
 * amplitude r g b -- until the end of the file (the reference reads exactly
 * 256).  *lobes = records in the file; with axis = NULL only the count is
 * returned, else at most max_lobes records are stored (more is an error). */
VCL_API vcl_status vcl_sg_load(vcl_ctx* ctx, const char* path, int max_lobes, int* lobes, float* axis,
                               float* sharpness, float* amplitude);

/* ------------------------------------------------------------- batches */
/* Batched engine: resident fit jobs of any sizes advanced together, one
 * iteration each per vcl_batch_step, as ONE CUDA graph launch.  Every member
 * runs the fused strategy (vcl_batch_add switches it); its captured step is
 * a child graph with no edges to the others, so members run concurrently.
 * The graph is rebuilt when membership or the mode changes.  Members may
 * come from different contexts of the same device.  No reference
 * counterpart (the reference runs one scene per process).  Remove a job
 * before destroying it; one host thread per batch. */
typedef struct vcl_batch vcl_batch;
VCL_API vcl_status vcl_batch_create(vcl_ctx* ctx, vcl_batch** out);
VCL_API void vcl_batch_destroy(vcl_batch* batch);
VCL_API vcl_status vcl_batch_add(vcl_batch* batch, vcl_fit* fit);
VCL_API vcl_status vcl_batch_remove(vcl_batch* batch, vcl_fit* fit);
VCL_API int vcl_batch_size(const vcl_batch* batch);
/* Iterations (1..64) the member advances per vcl_batch_step, chained inside
 * the batch graph (default 1). */
VCL_API vcl_status vcl_batch_set_repeat(vcl_batch* batch, vcl_fit* fit, int iterations);
VCL_API vcl_status vcl_batch_step(vcl_batch* batch, void* stream);
VCL_API int vcl_batch_launches_per_step(const vcl_batch* batch);
/* Number of batch-graph rebuilds so far and the host time they took. */
VCL_API vcl_status vcl_batch_rebuild_stats(const vcl_batch* batch, long long* rebuilds, double* host_ms);

/* -------------------------------------------------------------- serving */
/* Serving loop: fit jobs are submitted with their host data and an
 * iteration count, admitted in arrival order while their footprint fits
 * `budget_bytes` and fewer than `max_live` jobs are resident, set up on a
 * worker thread (upload, raster autotuning, graph capture) while the device
 * keeps running, advanced together one iteration per tick by a batched
 * launch, and retired when done.  Each tick leaves one batched launch queued
 * behind the running one.  Job latency = completion - submission on the
 * host's steady clock.  All host arrays are copied at submission.  The
 * context's mode must not change while the server exists.  No reference
 * counterpart. */
typedef struct vcl_server vcl_server;
#define VCL_JOB_QUEUED 0
#define VCL_JOB_LIVE 1
#define VCL_JOB_DONE 2
#define VCL_JOB_FAILED 3
VCL_API vcl_status vcl_server_create(vcl_ctx* ctx, size_t budget_bytes, int max_live, vcl_server** out);
VCL_API void vcl_server_destroy(vcl_server* server);
VCL_API const char* vcl_server_last_error(const vcl_server* server);
/* target: host images [views][H][W][4].  keep_result: keep the final
 * parameters for vcl_server_job_result. */
VCL_API vcl_status vcl_server_submit(vcl_server* server, const vcl_fit_desc* desc, const float* target,
                                     int iterations, int keep_result, long long* job_id);
/* Retire finished jobs, admit queued ones, launch one batched iteration of
 * every live job, wait for the previous tick.  Outputs may be NULL. */
VCL_API vcl_status vcl_server_tick(vcl_server* server, void* stream, int* live, int* completed);
VCL_API vcl_status vcl_server_drain(vcl_server* server, void* stream);
/* The server's clock (ms since creation; the clock of the job times). */
VCL_API double vcl_server_now_ms(const vcl_server* server);
/* Host time inside vcl_server_tick with the waits for the device excluded,
 * the waits, and the batch-graph rebuilds with their host time (ms). */
VCL_API vcl_status vcl_server_host_stats(const vcl_server* server, double* host_ms, double* wait_ms,
                                         long long* rebuilds, double* rebuild_ms);
/* Jobs queued, live or finishing. */
VCL_API int vcl_server_pending(const vcl_server* server);
VCL_API vcl_status vcl_server_job_status(const vcl_server* server, long long job_id, int* state, int* iters_done,
                                         double* submit_ms, double* admit_ms, double* done_ms);
VCL_API vcl_status vcl_server_job_result(const vcl_server* server, long long job_id, float* pos, float* tex_level0,
                                         float* lobe_axis, float* lobe_sharp, float* lobe_amp, float* loss);
VCL_API vcl_status vcl_server_stats(const vcl_server* server, double* p50_ms, double* p99_ms, long long* iterations,
                                    int* completed, long long* ticks, size_t* resident_bytes);

/* ------------------------------------------------------ throughput probes */
/* Measurement utilities with no counterpart in the reference: they measure
 * the peak rates of the two units other than HBM that bound the path's
 * kernels, so that those kernels can be reported against measured peaks.
 * Time the launch with CUDA events on `stream` and divide the count.
 *
 * L2 reductions: every thread adds (1,1,1,1) with red.global.add.v4.f32 to
 * consecutive 16-byte slots of `buf` (n_floats floats, 16-byte aligned,
 * device), `iters` passes; *reductions = the number of vector reductions
 * issued.  Keep buf well inside L2 (e.g. 32 MB) to measure the L2 units. */
VCL_API vcl_status vcl_probe_red_throughput(vcl_ctx* ctx, float* buf, long long n_floats, int iters,
                                            long long* reductions, void* stream);
/* MUFU: independent ex2.approx / rsqrt.approx chains on every SM; `out`
 * (device) holds vcl_probe_mufu_threads(ctx) floats; *ops = the number of
 * MUFU operations issued. */
VCL_API long long vcl_probe_mufu_threads(const vcl_ctx* ctx);
VCL_API vcl_status vcl_probe_mufu_throughput(vcl_ctx* ctx, float* out, int iters, long long* ops, void* stream);
/* The same shape for the FP32 FMA pipe: eight independent chains per thread
 * of paired FP32 fused multiply-adds (the form the SG kernels issue), `iters`
 * links each; `out` holds vcl_probe_mufu_threads(ctx) floats; *ops = the
 * number of FP32 operations (two per paired instruction). */
VCL_API vcl_status vcl_probe_fma_throughput(vcl_ctx* ctx, float* out, int iters, long long* ops, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VCL_H */

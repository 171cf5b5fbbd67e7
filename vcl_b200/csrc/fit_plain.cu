// The plain fit iteration: one C-ABI operator call per reference operator,
// in the order PresetPrimitives::update issues them
// (preset_primitives.cpp:160-208), on the caller's stream.
#include "fit.cuh"

#define TRY(x) do { vcl_status _s = (x); if (_s) return _s; } while (0)

static vcl_status fwd_ops(vcl_fit* f, float* aa_out, cudaStream_t s) {
    vcl_ctx* ctx = f->ctx;
    const vcl_fit_desc& d = f->d;
    const int W = d.W, H = d.H, V = d.views, C = d.C;
    TRY(vcl_project_fwd(ctx, f->mvp, V, f->pos, d.nv, 4, f->clip, s));
    TRY(vcl_rasterize_fwd(ctx, f->clip, d.nv, f->tri, d.nt, W, H, V, f->rast, f->db, s));
    TRY(vcl_interpolate_fwd(ctx, f->rast, f->db, W, H, V, f->uvattr, d.nv, 2, f->tri, d.nt, f->uv, f->uv_da, s));
    TRY(vcl_texture_fwd(ctx, f->rast, f->uv, f->uv_da, W, H, V, f->pyr, d.tex_w, d.tex_h, C, d.levels, f->diffuse, s));
    TRY(vcl_normal_axis_fwd(ctx, f->rast, W, H, V, f->rot, f->nrmattr, d.nv, f->tri, d.nt, f->normal, s));
    TRY(vcl_view_axis_fwd(ctx, W, H, V, f->pvinv, f->view, s));
    TRY(vcl_sg_specular_fwd(ctx, f->rast, W, H, V, f->normal, f->view, f->rough, d.ior, f->sax, f->ssh, f->sam, s));
    TRY(vcl_sg_fwd(ctx, f->rast, W, H, V, C, d.K, f->axis, f->sharp, f->amp, f->normal, f->diffuse, f->sax, f->ssh,
                   f->sam, f->color, nullptr, nullptr, s));
    TRY(vcl_antialias_fwd(ctx, f->clip, d.nv, f->tri, d.nt, f->rast, W, H, V, C, f->color, aa_out, s));
    return VCL_OK;
}

vcl_status fit_forward(vcl_fit* f, float* out, cudaStream_t s) {
    vcl_ctx* ctx = f->ctx;
    VCL_REQUIRE(out, "null render output");
    return fwd_ops(f, out, s);
}

int fit_plain_launches(const vcl_fit* f) {
    const vcl_fit_desc& d = f->d;
    int n = 4 /* raster: setup, scan, emit, fine */ + 8 /* project, interp, tex, normal, view, spec, sg, aa */;
    n += 1; /* mse */
    n += 2; /* aa bwd, sg bwd */
    if (d.learn_tex || d.learn_pos) n += 1; /* texture bwd */
    if (d.learn_pos) n += 4; /* interp bwd, raster bwd, project bwd, adam */
    if (d.learn_tex) n += (d.levels - 1) * 2 + 2; /* pushdown + mips, adam, clamp */
    if (d.learn_lobes && d.K) n += 1;
    return n;
}

vcl_status fit_step_plain(vcl_fit* f, cudaStream_t s) {
    vcl_ctx* ctx = f->ctx;
    const vcl_fit_desc& d = f->d;
    const int W = d.W, H = d.H, V = d.views, C = d.C;
    const size_t N = (size_t)W * H * V;
    const size_t npyr = vcl_tex_level_offset(d.tex_w, d.tex_h, C, d.levels);
    const size_t n0 = (size_t)d.tex_w * d.tex_h * C;
    const size_t nl = (size_t)d.K * (4 + C);
    // gradient clears (the reference's X::forward(GradParams) memsets)
    TRY(vcl_cuda_check(ctx, cudaMemsetAsync(f->g_clip, 0, sizeof(float) * V * d.nv * 4, s), "clear"));
    TRY(vcl_cuda_check(ctx, cudaMemsetAsync(f->g_pos, 0, sizeof(float) * d.nv * 3, s), "clear"));
    TRY(vcl_cuda_check(ctx, cudaMemsetAsync(f->g_pyr, 0, sizeof(float) * npyr, s), "clear"));
    TRY(vcl_cuda_check(ctx, cudaMemsetAsync(f->g_lobe, 0, sizeof(float) * (nl ? nl : 1), s), "clear"));
    TRY(vcl_cuda_check(ctx, cudaMemsetAsync(f->g_diffuse, 0, sizeof(float) * N * C, s), "clear"));
    TRY(vcl_cuda_check(ctx, cudaMemsetAsync(f->g_bary, 0, sizeof(float) * N * 2, s), "clear"));
    // forward
    TRY(fwd_ops(f, f->aa, s));
    TRY(vcl_mse(ctx, f->aa, f->target, N * C, f->g_aa, f->loss, s));
    // backward
    TRY(vcl_antialias_bwd(ctx, f->clip, d.nv, f->tri, d.nt, f->rast, W, H, V, C, f->color, f->g_aa, f->g_color,
                          d.learn_pos ? f->g_clip : nullptr, s));
    const bool lobes = d.learn_lobes && d.K;
    TRY(vcl_sg_bwd(ctx, f->rast, W, H, V, C, d.K, f->axis, f->sharp, f->amp, f->normal, f->diffuse, f->sax, f->ssh, f->sam,
                   f->g_color, f->g_diffuse, lobes ? f->g_axis : nullptr, lobes ? f->g_sharp : nullptr,
                   lobes ? f->g_amp : nullptr, nullptr, nullptr, nullptr, s));
    if (d.learn_tex || d.learn_pos)
        TRY(vcl_texture_bwd(ctx, f->rast, f->uv, f->uv_da, W, H, V, f->pyr, d.tex_w, d.tex_h, C, d.levels, f->g_diffuse,
                            d.learn_tex ? f->g_pyr : nullptr, d.learn_pos ? f->g_uv : nullptr, nullptr, s));
    if (d.learn_pos) {
        TRY(vcl_interpolate_bwd(ctx, f->rast, W, H, V, f->uvattr, d.nv, 2, f->tri, d.nt, f->g_uv, nullptr, f->g_bary, s));
        TRY(vcl_rasterize_bwd(ctx, f->clip, d.nv, f->tri, d.nt, W, H, V, f->rast, f->g_bary, f->g_clip, s));
        TRY(vcl_project_bwd(ctx, f->mvp, V, f->g_clip, d.nv, 4, f->g_pos, s));
    }
    // optimizer (preset_primitives.cpp:199-208)
    const int t = ++f->step_count;
    if (d.learn_tex) {
        TRY(vcl_texture_grad_pushdown(ctx, f->g_pyr, d.tex_w, d.tex_h, C, d.levels, s));
        TRY(vcl_adam_step(ctx, f->pyr, f->g_pyr, f->mv_tex, f->mv_tex + n0, n0, d.lr_tex, d.beta1, d.beta2, d.eps, t, s));
        TRY(vcl_clamp(ctx, f->pyr, n0, 0.f, 1.f, s));
        TRY(vcl_texture_build_mips(ctx, f->pyr, d.tex_w, d.tex_h, C, d.levels, s));
    }
    if (d.learn_pos)
        TRY(vcl_adam_step(ctx, f->pos, f->g_pos, f->mv_pos, f->mv_pos + (size_t)d.nv * 3, (size_t)d.nv * 3, d.lr_pos,
                          d.beta1, d.beta2, d.eps, t, s));
    if (lobes)
        TRY(vcl_adam_step(ctx, f->lobe, f->g_lobe, f->mv_lobe, f->mv_lobe + nl, nl, d.lr_lobes, d.beta1, d.beta2, d.eps, t, s));
    return VCL_OK;
}

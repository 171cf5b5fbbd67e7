// Internal launchers shared by the C-ABI operators and the fused fit path.
#pragma once
#include "common.cuh"

// Antialias forward / backward (gather form: `out` / `grad_in` are written
// completely, the reference's initial copy included).
vcl_status aa_edges_fwd(vcl_ctx* ctx, const float* clip, const float* scr, int nv, const uint32_t* tri, int nt,
                        const float* rast, int W, int H, int views, int C, const float* in, float* out, cudaStream_t s);
// Antialias forward (C = 4) fused with the MSE: writes grad = aa - target and
// the loss 0.5 sum |aa - target|^2 (through the double `sum` and block counter
// `done`, both zero before the first call and left zero after each call).
// `clist` (may be NULL): the per-tile candidate lists this forward finds,
// aa_cand_list_bytes(W, H, views) bytes, for aa_edges_bwd of the same step
// (same rast) to reuse instead of finding them again.
size_t aa_cand_list_bytes(int W, int H, int views);
vcl_status aa_edges_fwd_mse(vcl_ctx* ctx, const float* clip, const float* scr, int nv, const uint32_t* tri, int nt,
                            const float* rast, int W, int H, int views, const float* in, const float* target,
                            float* grad, double* sum, unsigned* done, float* loss, uint16_t* clist, cudaStream_t s);
vcl_status aa_edges_bwd(vcl_ctx* ctx, const float* clip, const float* scr, int nv, const uint32_t* tri, int nt,
                        const float* rast, int W, int H, int views, int C, const float* in, const float* grad_out,
                        float* grad_in, float* grad_clip, cudaStream_t s, const uint16_t* clist = nullptr);
// Per-vertex screen terms for the antialias kernels (`scr` above, 8 floats
// per view-vertex; NULL there computes them per pixel pair instead).
void launch_aa_screen(const float* clip, long long n, int W, int H, float* scr, cudaStream_t s);
// Mip level l from level l-1 (buffer.cu:449-472).
void launch_mip_down(const float* src, float* dst, int w, int h, int C, cudaStream_t s);

// Rasterizer with a caller-owned workspace (a fit job owns one, so that a
// captured graph never points into a workspace that another call regrows).
long long raster_auto_capacity(long long views, long long nt, int W, int H, int tile);
size_t raster_ws_size(int W, int H, int views, int nt, int tile, long long cap);
// Binning schedule: tile edge (8, 16 or 32), bin-list capacity (entries),
// and the box area (pixels) up to which a triangle skips the bins and is
// rasterized directly by its setup thread (0 = every triangle is binned).
struct RasterSched {
    int tile;
    long long cap;
    int small_area;
    int med_area;    // box area (pixels) up to which a triangle is rasterized by one warp
};
int raster_default_small_area();
int raster_default_medium_area();
// The context's schedule: tile, capacity, and its direct-raster areas.
RasterSched ctx_sched(const vcl_ctx* ctx, int tile, long long cap);
// `flags[0]` receives the number of tiles whose bins overflowed.
vcl_status raster_fwd_ws(vcl_ctx* ctx, void* ws, const RasterSched& rs, int* flags, const float* clip, int nv,
                         const uint32_t* tri, int nt, int W, int H, int views, float* rast, float* db, cudaStream_t s);
// Bin-list entries the last raster_fwd_ws on `ws` with schedule `rs` asked
// for (synchronizes `s`).
vcl_status raster_bin_demand(vcl_ctx* ctx, void* ws, const RasterSched& rs, int W, int H, int views, int nt,
                             cudaStream_t s, long long* demand);
int raster_fwd_launches();

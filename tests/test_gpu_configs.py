"""Parity at the sizes of the fit configurations, through the C ABI.

The operator tests (test_gpu_parity.py) use small scenes; the kernels pick
code paths by image size, triangle density, lobe count and pyramid depth, so
this file checks the CUDA path against the CPU oracle on the configurations
themselves:

* config 1: icosphere s3 (1,280 triangles), 256x256, 512^2 texture with 10
  levels, 16 lobes -- the whole chain, both modes, and fit iterations of
  both strategies;
* config 2, one view: UV sphere 256x128 (65,024 triangles) displaced
  N(0, 0.02), 1024x1024, 2048^2 texture with 12 levels, 32 lobes -- the
  whole chain in both modes and fused fit iterations (the bench's kernels
  and lobe count);
* config 5 at 512x512: icosphere s8 (1,310,720 mostly sub-pixel triangles),
  4096^2 texture with 13 levels, 64 lobes -- the whole chain in both modes
  and fused fit iterations;
* config 5, one full 2048x2048 view: the raster, bit for bit, under each
  tile size.

Every raster comparison also runs the GL tie census (vcl_raster_ties against
the oracle's orc_raster_ties): the pixels where a real GL driver may legally
choose another triangle (centre exactly on an edge; equal depth) are counted
identically, and the triangle ids agree there as everywhere else.
"""
import numpy as np
import pytest

import chain
import parity
from oracle import oracle as O
from vcl_b200 import scenes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

KEYS = ["clip", "uv", "uv_da", "diffuse", "normal", "view", "spec_axis", "spec_sharp", "spec_amp", "color",
        "diffenv", "specenv", "aa", "g_aa", "g_color", "g_clip_aa", "g_diffuse", "g_axis", "g_sharp", "g_amp",
        "g_sax", "g_ssh", "g_sam", "g_rough", "g_pyr", "g_uv", "g_uv_da", "g_uvattr", "g_bary", "g_clip", "g_pos",
        "adam_p", "adam_m", "adam_v"]


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from vcl_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


def _config5_512():
    S = scenes.config5(views=1)
    S.W = S.H = 512          # same mesh, camera, texture and lobes at a quarter of the resolution
    return S


SCENES = {
    "config1": scenes.config1,
    "config2_view": lambda: scenes.config2(views=1),
    "config5_512": _config5_512,
}
_cache = {}


def scene(name):
    if name not in _cache:
        _cache[name] = SCENES[name]()
    return _cache[name]


def ties_gpu(ctx, clip, S, rast_dev):
    import gpu_chain as G
    N = S.W * S.H * S.views
    flags = torch.zeros(N, dtype=torch.int32, device="cuda")
    counts = torch.zeros(2, dtype=torch.int64, device="cuda")
    ctx.raster_ties(G.dev(clip), S.nv, G.dev(S.tri.astype(np.int32)), S.nt, S.W, S.H, S.views, rast_dev, flags,
                    counts, None)
    torch.cuda.synchronize()
    return G.host(flags).view(np.uint32), G.host(counts)


def ties_oracle(clip, S, rast):
    N = S.W * S.H * S.views
    flags = np.zeros(N, np.uint32)
    counts = np.zeros(2, np.int64)
    O.orc().raster_ties(S.W, S.H, S.views, np.ascontiguousarray(clip), S.nv, S.tri, S.nt, rast, flags, counts)
    return flags, counts


def assert_ties_match(ctx, clip, S, rast_oracle, rast_dev, rast_gpu, label):
    fo, co = ties_oracle(clip, S, rast_oracle)
    fg, cg = ties_gpu(ctx, clip, S, rast_dev)
    assert np.array_equal(fg, fo), (label, "tie flags differ", cg, co)
    assert np.array_equal(cg, co), (label, cg, co)
    tie = fo != 0
    mism = int((rast_gpu[tie, 3] != rast_oracle[tie, 3]).sum())
    parity.report(label + ":ties", {"edge_tie_pixels": (float(co[0]), 0.0, -1),
                                    "depth_tie_pixels": (float(co[1]), 0.0, -1),
                                    "id_mismatch_at_ties": (float(mism), 0.0, -1)})
    assert mism == 0
    return co


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("name", list(SCENES))
def test_config_chain_matches_oracle(ctx, name, mode):
    import gpu_chain as G
    S = scene(name)
    pyr = chain.build_pyramid(S, S.tex_target)
    o = chain.run_chain(O.orc(), S, mode, pyr=pyr)
    g = G.run_chain_gpu(ctx, S, o, mode)
    ctx.set_mode(0)
    assert (o["rast"][:, 3] > 0).sum() > 0
    assert np.array_equal(g["rast"][:, 3], o["rast"][:, 3]), "triangle ids differ"
    assert np.array_equal(g["rast"], o["rast"]), "barycentrics/depth differ"
    assert np.array_equal(g["db"], o["db"]), "DB differs"
    exact = chain.run_isolated64(S, o, mode)
    res, bad = parity.check_keys(g, o, exact, KEYS, f"{name}:mode{mode}")
    assert not bad, bad
    n = S.W * S.H * S.views * S.C
    exact_loss = O.orc().mse(1, n, o["aa"], o["target"], np.zeros(n, np.float32))
    assert abs(g["loss"] - exact_loss) <= parity.NORM_TOL * abs(exact_loss)
    if mode == 0:
        assert_ties_match(ctx, o["clip"], S, o["rast"], G.dev(o["rast"]), g["rast"], name)
    assert ctx.check_indices() == 0


def _fit(ctx, S, mode, strategy, steps, tgt):
    from vcl_b200 import capi
    ctx.set_mode(mode)
    fit = capi.Fit(ctx, S, strategy=strategy)
    fit.set_target(tgt)
    stream = torch.cuda.Stream()
    losses = []
    for _ in range(steps):
        fit.step(stream.cuda_stream)
        losses.append(fit.read_loss(stream.cuda_stream))
    params = fit.read_params(stream.cuda_stream)
    fit.close()
    ctx.set_mode(0)
    return losses, params


def _adam_close(got, want, lr, steps, name):
    # an Adam step is ~lr * m/sqrt(v) and flips with the sign of a near-zero
    # gradient, so a few entries may differ by up to the step budget; the
    # bulk must agree to FP32 rounding
    d = np.abs(np.asarray(got, np.float64) - np.asarray(want, np.float64)).reshape(-1)
    scale = max(1.0, float(np.abs(want).max()))
    assert d.max() <= 2.0 * lr * steps, (name, d.max())
    assert np.quantile(d, 0.99) <= 1e-5 * scale, (name, np.quantile(d, 0.99))
    assert np.mean(d > 1e-5 * scale) <= 0.01, (name, np.mean(d > 1e-5 * scale))


@pytest.mark.parametrize("name,mode,strategy,steps", [
    ("config1", 0, 1, 3), ("config1", 1, 1, 3), ("config1", 0, 0, 3), ("config1", 1, 0, 3),
    ("config2_view", 0, 1, 2), ("config2_view", 1, 1, 2),
    ("config5_512", 0, 1, 2),
])
def test_config_fit_matches_oracle(ctx, name, mode, strategy, steps):
    S = scene(name)
    tgt = np.random.default_rng(S.seed + 3).random((S.W * S.H * S.views, S.C)).astype(np.float32)
    ref = chain.oracle_fit(S, mode, steps, tgt)
    losses, (pos, tex, (ax, sh, am)) = _fit(ctx, S, mode, strategy, steps, tgt)
    rel = np.abs(np.asarray(losses) - np.asarray(ref["losses"])) / np.abs(np.asarray(ref["losses"]))
    parity.report(f"{name}:fit:mode{mode}:strategy{strategy}", {"loss": (float(rel.max()), float(rel.max()), -1)})
    assert rel.max() <= 1e-5, (losses, ref["losses"])
    lr_pos = S.lr_pos or S.lr
    # texels whose gradient is at the rounding-noise level of its sum (a
    # 4096^2 texture seen at 512^2: almost every texel's gradient comes from
    # the mip push-down of coarse-level sums) take Adam steps of +-lr in
    # whichever direction their noise points, so the texture is compared
    # where its gradient was resolved in every step: above 1e-4 of that
    # step's largest magnitude (every texel still within the step budget)
    resolved = ref["g_tex_resolved"] > 1e-4
    dt = np.abs(np.asarray(tex, np.float64) - ref["tex"]).reshape(-1)
    assert dt.max() <= 2.0 * S.lr * steps, dt.max()
    parity.report(f"{name}:fit:mode{mode}:strategy{strategy}:tex",
                  {"texels_differing": (float(np.mean(dt > 1e-5)), 0.0, -1),
                   "resolved_texels": (float(resolved.mean()), 0.0, -1),
                   "resolved_differing": (float(np.mean(dt[resolved.reshape(-1)] > 1e-5)), 0.0, -1)})
    _adam_close(np.asarray(tex).reshape(-1)[resolved.reshape(-1)], ref["tex"].reshape(-1)[resolved.reshape(-1)],
                S.lr, steps, "tex")
    for pname, got, want, lr in (("pos", pos, ref["pos"], lr_pos),
                                 ("axis", ax, ref["axis"], S.lr), ("sharp", sh, ref["sharp"], S.lr),
                                 ("amp", am, ref["amp"], S.lr)):
        _adam_close(got, want, lr, steps, pname)


@pytest.mark.parametrize("tile", [8, 16, 32])
def test_config5_full_view_raster_bit_exact(ctx, tile):
    """One 2048x2048 view of the 1,310,720-triangle mesh: almost every
    triangle takes the per-thread direct path, a few the warp path, none
    the bins at the default areas; the bins are forced with areas (0, 0)
    on tile 16."""
    import gpu_chain as G
    S = scenes.config5(views=1)
    key = "c5full"
    if key not in _cache:
        clip = chain.project(O.orc(), S, S.pos)
        N = S.W * S.H
        r = np.zeros((N, 4), np.float32); d = np.zeros((N, 4), np.float32)
        O.orc().rasterize_fwd(S.W, S.H, 1, clip, S.nv, S.tri, S.nt, 1, r, d)
        _cache[key] = (clip, r, d)
    clip, r, d = _cache[key]
    N = S.W * S.H
    areas = [(-1, -1)] + ([(0, 0)] if tile == 16 else [])
    for ar in areas:
        ctx.set_raster_config(tile, 0)
        ctx.set_raster_areas(*ar)
        try:
            gr = G.zeros(N, 4); gd = G.zeros(N, 4)
            ctx.rasterize_fwd(G.dev(clip), S.nv, G.dev(S.tri.astype(np.int32)), S.nt, S.W, S.H, 1, gr, gd, None)
            hr = G.host(gr)
            assert np.array_equal(hr[:, 3], r[:, 3]), (tile, ar, int((hr[:, 3] != r[:, 3]).sum()))
            assert np.array_equal(hr, r), (tile, ar)
            assert np.array_equal(G.host(gd), d), (tile, ar)
        finally:
            ctx.set_raster_config(16, 0)
            ctx.set_raster_areas(-1, -1)
    if tile == 16:
        assert_ties_match(ctx, clip, S, r, gr, hr, "config5_full_view")


def test_tie_census_counts_designed_ties(ctx):
    """Scenes built to have ties: two triangles of a quad whose shared
    diagonal runs through pixel centres (edge ties along it), axis-aligned
    edges on pixel centres, and the same triangle drawn twice (a depth tie
    at every covered pixel, decided by the lower id)."""
    import gpu_chain as G

    class _S:
        pass

    quad = np.array([[-1, -1, 0.5, 1], [1, -1, 0.5, 1], [1, 1, 0.5, 1], [-1, 1, 0.5, 1]], np.float32)
    cases = [
        (8, 8, quad, [[0, 1, 2], [0, 2, 3]], (8, 0)),
        # x = 0 and y = 0 in NDC are pixel centres on odd sizes: edges along them
        (9, 7, np.array([[0, 0, 0.2, 1], [1, 0, 0.2, 1], [0, 1, 0.2, 1], [-1, 0, 0.2, 1]], np.float32),
         [[0, 1, 2], [0, 2, 3]], None),
        (16, 12, np.array([[-0.9, -0.8, 0.1, 1], [0.7, -0.6, 0.1, 1], [0.1, 0.9, 0.1, 1]] * 2, np.float32),
         [[0, 1, 2], [3, 4, 5]], None),
    ]
    for W, H, clip, tri, expect in cases:
        S = _S()
        S.W, S.H, S.views, S.nv, S.nt = W, H, 1, clip.shape[0], len(tri)
        S.tri = np.array(tri, np.uint32)
        N = W * H
        r = np.zeros((N, 4), np.float32); d = np.zeros((N, 4), np.float32)
        O.orc().rasterize_fwd(W, H, 1, clip, S.nv, S.tri, S.nt, 1, r, d)
        gr = G.zeros(N, 4)
        ctx.rasterize_fwd(G.dev(clip), S.nv, G.dev(S.tri.astype(np.int32)), S.nt, W, H, 1, gr, None, None)
        hr = G.host(gr)
        assert np.array_equal(hr, r)
        co = assert_ties_match(ctx, clip[None], S, r, gr, hr, f"designed{W}x{H}")
        assert co.sum() > 0
        if expect is not None:
            assert tuple(co) == expect, co
    # duplicated triangle: every covered pixel is a depth tie won by id 1
    assert (r[:, 3] == 1).sum() > 0 and not (r[:, 3] == 2).any()

"""vcl_rasterize_fwd_static (the forward rasterizer on the module's fixed
scratch array, no allocation) against vcl_rasterize_fwd (context workspace).

Rasterization is index work, so the tolerance is zero: triangle ids,
barycentrics, depth and DB must be bit-identical.  Two consecutive static
calls on different scenes check that nothing carries over between calls
through the shared scratch.  The file name keeps it last in collection; it
also passes on its own."""
import numpy as np
import pytest

import chain
from oracle import oracle as O
from vcl_b200 import capi, scenes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = capi.Context(0)
    c.raster_scratch_init()
    yield c
    c.close()


def _scenes():
    return [
        scenes.make_scene("noalloc-a", mesh=("ico", 4), W=200, H=150, views=2, tex=16, K=1, dist=(2.0, 3.5),
                          disp=0.05, seed=9),
        scenes.make_scene("noalloc-b", mesh=("ico", 1), W=97, H=61, views=3, tex=16, K=1, dist=(1.6, 2.5),
                          seed=3),
        scenes.small(seed=2, W=64, H=48, views=3, subdiv=2, tex=64, K=5),
    ]


def _raster(ctx, S, fn):
    import gpu_chain as G
    clip = chain.project(O.orc(), S, S.pos)
    N = S.W * S.H * S.views
    r, d = G.zeros(N, 4), G.zeros(N, 4)
    # poison the outputs: every pixel must be written by the call
    r.fill_(float("nan")); d.fill_(float("nan"))
    getattr(ctx, fn)(G.dev(clip), S.nv, G.dev(S.tri.astype(np.int32)), S.nt, S.W, S.H, S.views, r, d, None)
    torch.cuda.synchronize()
    return G.host(r), G.host(d)


@pytest.mark.parametrize("tile", [16, 8])
def test_static_scratch_matches_workspace_path(ctx, tile):
    ctx.set_raster_config(tile, 0)
    try:
        S = _scenes()
        want = [_raster(ctx, s, "rasterize_fwd") for s in S]
        # consecutive static calls, different scenes in between and repeated
        for rep in range(2):
            for s, (wr, wd) in zip(S, want):
                gr, gd = _raster(ctx, s, "rasterize_fwd_static")
                assert (wr[:, 3] > 0).any()
                assert np.array_equal(gr, wr), (s.name, rep)
                assert np.array_equal(gd, wd), (s.name, rep)
    finally:
        ctx.set_raster_config(16, 0)


def test_static_scratch_bins_overflow_to_exact_result(ctx):
    # a bin capacity of one entry forces the every-triangle fallback on the
    # static path too; results stay identical
    S = _scenes()[1]
    wr, wd = _raster(ctx, S, "rasterize_fwd")
    ctx.set_raster_config(16, 1)
    ctx.set_raster_areas(0, 0)      # every triangle through the bins
    try:
        gr, gd = _raster(ctx, S, "rasterize_fwd_static")
        assert ctx.raster_overflow_count() > 0
    finally:
        ctx.set_raster_config(16, 0)
        ctx.set_raster_areas(-1, -1)
    assert np.array_equal(gr, wr)
    assert np.array_equal(gd, wd)


def test_static_scratch_rejects_oversize_request(ctx):
    import gpu_chain as G
    limit = capi.lib().vcl_raster_scratch_bytes()
    assert limit == 32 << 20
    # 2048 x 2048 x 1 view needs 32 MiB of depth keys alone
    W = H = 2048
    clip = G.zeros(3, 4)
    tri = G.dev(np.array([[0, 1, 2]], np.int32))
    out = G.zeros(W * H, 4)   # full size, although the call must not launch
    with pytest.raises(capi.VclError, match="static limit"):
        ctx.rasterize_fwd_static(clip, 3, tri, 1, W, H, 1, out, None, None)
    # the context stays usable
    S = _scenes()[2]
    assert np.array_equal(_raster(ctx, S, "rasterize_fwd_static")[0], _raster(ctx, S, "rasterize_fwd")[0])


def test_static_scratch_bin_list_cut_to_room(ctx):
    """A request whose depth keys nearly fill the scratch: the bin list gets
    only the room that is left, less than the automatic capacity asks for.
    The documented sizes (8 B per pixel, 100 B per view and triangle, 12 B
    per tile, each part rounded up to 256 B) say how much room that is; the
    result stays bit-identical to the workspace path, with every triangle
    through the bins and with the default direct paths."""
    S = scenes.make_scene("noalloc-big", mesh=("ico", 4), W=2000, H=2000, views=1, tex=16, K=1, dist=(2.0, 3.5),
                          disp=0.05, seed=4)
    a256 = lambda x: (x + 255) // 256 * 256
    npix, vt = S.W * S.H * S.views, S.nt * S.views
    tile = 16
    ntiles = -(-S.W // tile) * -(-S.H // tile) * S.views
    fixed = a256(8 * npix) + a256(96 * vt) + a256(4 * vt) + 3 * a256(4 * (ntiles + 1))
    limit = capi.lib().vcl_raster_scratch_bytes()
    assert fixed < limit
    room = ((limit - fixed) // 4) & ~63
    want = vt * 6 + ntiles * 4 + (1 << 20)        # the automatic bin capacity
    assert room < want
    ctx.set_raster_config(tile, 0)
    try:
        for areas in ((0, 0), (-1, -1)):
            ctx.set_raster_areas(*areas)
            wr, wd = _raster(ctx, S, "rasterize_fwd")
            gr, gd = _raster(ctx, S, "rasterize_fwd_static")
            assert ctx.raster_overflow_count() == 0
            assert (wr[:, 3] > 0).sum() > 100000
            assert np.array_equal(gr, wr), areas
            assert np.array_equal(gd, wd), areas
    finally:
        ctx.set_raster_config(16, 0)
        ctx.set_raster_areas(-1, -1)

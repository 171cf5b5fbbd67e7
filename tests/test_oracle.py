"""CPU tests of the checker itself: the C restatement against the golden
fixtures made from the reference's own kernels, against the live reference
build where present, and against known-answer cases."""
import glob
import os
import types

import numpy as np
import pytest

import chain
from oracle import oracle as O
from vcl_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
REL_TOL = 1e-5


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(initial=0.0), 1e-30)
    return np.abs(a - b).max(initial=0.0) / scale


def scene_from_fixture(z):
    d = {k[len("scene_"):]: z[k] for k in z.files if k.startswith("scene_")}
    for k in ("W", "H", "views", "tex_w", "tex_h", "C", "levels", "K", "seed"):
        d[k] = int(d[k])
    for k in ("roughness", "ior", "lr"):
        d[k] = float(d[k])
    s = types.SimpleNamespace(**d)
    s.nv = int(s.pos.shape[0])
    s.nt = int(s.tri.shape[0])
    return s


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(HERE, "golden", "*.npz"))))
def test_restatement_matches_reference_fixture(path):
    z = np.load(path)
    S = scene_from_fixture(z)
    a = chain.run_chain(O.orc(), S, 0, target=z["ref_target"], rast=z["ref_rast"], db=z["ref_db"],
                        pyr=z["ref_pyr"].copy())
    for k, v in a.items():
        ref = z[f"ref_{k}"]
        if k == "loss":
            assert abs(v - float(ref)) <= REL_TOL * abs(float(ref)), (k, v, float(ref))
            continue
        assert v.shape == ref.shape, k
        assert rel_err(v, ref) <= REL_TOL, (k, rel_err(v, ref))


def test_restatement_matches_live_reference():
    ref = O.ref()
    if ref is None:
        pytest.skip("reference host build not present (make -C oracle ref)")
    S = scenes.small(seed=11, W=40, H=40, views=2, subdiv=2, tex=32, K=4)
    pyr = chain.build_pyramid(S, S.tex_target)
    a = chain.run_chain(O.orc(), S, 0, pyr=pyr.copy())
    b = chain.run_chain(ref, S, 0, rast=a["rast"], db=a["db"], pyr=pyr.copy())
    for k, v in a.items():
        if k == "loss":
            assert v == b[k]
        else:
            assert rel_err(v, b[k]) <= REL_TOL, k


# ------------------------------------------------------------ raster KATs
def _raster(clip, tri, W, H, views=1, db=True):
    clip = np.ascontiguousarray(clip, np.float32)
    tri = np.ascontiguousarray(tri, np.uint32)
    nv = clip.shape[-2]
    rast = np.zeros((views * W * H, 4), np.float32)
    dbo = np.zeros((views * W * H, 4), np.float32)
    O.orc().rasterize_fwd(W, H, views, clip, nv, tri, tri.shape[0], 1 if db else 0, rast, dbo)
    return rast.reshape(views, H, W, 4), dbo.reshape(views, H, W, 4)


def test_fullscreen_quad_linear_barycentrics():
    W, H = 16, 8
    clip = np.array([[-1, -1, 0.5, 1], [3, -1, 0.5, 1], [-1, 3, 0.5, 1]], np.float32)
    rast, db = _raster(clip, [[0, 1, 2]], W, H)
    assert (rast[0, :, :, 3] == 1).all()
    px = (2 * np.arange(W) + 1 - W) / W
    py = (2 * np.arange(H) + 1 - H) / H
    sx, sy = np.meshgrid(px, py)
    # v0 at (-1,-1), v1 at (3,-1), v2 at (-1,3): u = 1 - (x+1)/4 - (y+1)/4, v = (x+1)/4
    u = 1 - (sx + 1) / 4 - (sy + 1) / 4
    v = (sx + 1) / 4
    assert np.abs(rast[0, :, :, 0] - u).max() < 1e-6
    assert np.abs(rast[0, :, :, 1] - v).max() < 1e-6
    assert np.abs(rast[0, :, :, 2] - 0.5).max() < 1e-6
    # affine triangle (w = 1): du/dx per pixel is -1/4 * 2/W; the reference's
    # geometry shader (rasterize.cpp:148-164) emits the negated Jacobian
    # (checked by hand for both windings), which is what DB reproduces
    assert np.allclose(db[0, :, :, 0], 0.5 / W, atol=1e-7)
    assert np.allclose(db[0, :, :, 1], 0.5 / H, atol=1e-7)
    assert np.allclose(db[0, :, :, 2], -0.5 / W, atol=1e-7)
    assert np.allclose(db[0, :, :, 3], 0.0, atol=1e-7)


def test_shared_edges_watertight_and_single_owner():
    # a 5x5 grid of quads (two triangles each) covering NDC [-1,1]^2 exactly
    n = 5
    xs = np.linspace(-1, 1, n + 1)
    vx, vy = np.meshgrid(xs, xs)
    clip = np.stack([vx.ravel(), vy.ravel(), np.zeros(vx.size), np.ones(vx.size)], 1)
    tri = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            tri += [[a, a + 1, a + n + 1], [a + 1, a + n + 2, a + n + 1]]
    # at 10x10 the pixel centres (2k+1)/10-1 land exactly on the grid lines
    # x = -0.6, -0.2, ...: every such tie pixel must still be owned by one side
    for W in (10, 20, 30):
        rast, _ = _raster(clip, tri, W, W, db=False)
        assert (rast[0, :, :, 3] > 0).all(), W


def test_depth_test_nearest_wins_and_ties_keep_first():
    W = H = 8
    big = [[-1, -1], [3, -1], [-1, 3]]
    def tri_at(z):
        return [[x, y, z, 1.0] for x, y in big]
    clip = np.array(tri_at(0.5) + tri_at(0.2) + tri_at(0.2), np.float32)
    rast, _ = _raster(clip, [[0, 1, 2], [3, 4, 5], [6, 7, 8]], W, H)
    assert (rast[0, :, :, 3] == 2).all()   # nearer (0.2) wins, first of the equal pair
    # beyond the far plane / in front of the near plane: not drawn
    clip2 = np.array(tri_at(1.5) + tri_at(-1.5), np.float32)
    rast2, _ = _raster(clip2, [[0, 1, 2], [3, 4, 5]], W, H)
    assert (rast2[0, :, :, 3] == 0).all()


def test_degenerate_and_behind_camera_triangles_draw_nothing():
    W = H = 8
    clip = np.array([[0, 0, 0, 1], [0.5, 0.5, 0, 1], [1, 1, 0, 1],      # collinear
                     [-1, -1, 0, -1], [3, -1, 0, -1], [-1, 3, 0, -1]],  # w < 0 everywhere
                    np.float32)
    rast, _ = _raster(clip, [[0, 1, 2], [3, 4, 5]], W, H)
    assert (rast[0, :, :, 3] == 0).all()


def test_empty_mesh_and_multiview_offsets():
    S = scenes.small(seed=3, views=3)
    rast, _ = _raster(np.zeros((3, 3, 4), np.float32), np.zeros((0, 3), np.uint32), 8, 8, views=3)
    assert (rast == 0).all()
    clip = chain.project(O.orc(), S, S.pos)
    r_all, _ = _raster(clip, S.tri, S.W, S.H, views=S.views)
    for v in range(S.views):
        r_one, _ = _raster(clip[v:v + 1], S.tri, S.W, S.H, views=1)
        assert np.array_equal(r_all[v], r_one[0])


# --------------------------------------------------------------- mip/adam
def test_mip_build_constant_and_pushdown_adjoint():
    tw, th, C = 16, 8, 3
    L = O.tex_levels(tw, th, 16)
    assert L == 4
    n = O.pyramid_size(tw, th, C, L)
    pyr = np.zeros(n, np.float32)
    pyr[: tw * th * C] = 0.25
    O.orc().mip_build(tw, th, C, L, pyr)
    assert np.allclose(pyr, 0.25)
    rng = np.random.default_rng(0)
    x = np.zeros(n, np.float32); x[: tw * th * C] = rng.random(tw * th * C)
    O.orc().mip_build(tw, th, C, L, x)
    g = rng.random(n).astype(np.float32)
    gp = g.copy()
    O.orc().mip_pushdown(1, tw, th, C, L, gp)         # exact mode: adjoint of the box chain
    lhs = float(np.dot(x.astype(np.float64), g))
    rhs = float(np.dot(x[: tw * th * C].astype(np.float64), gp[: tw * th * C]))
    assert abs(lhs - rhs) < 1e-5 * abs(lhs)
    gc = g.copy()
    O.orc().mip_pushdown(0, tw, th, C, L, gc)         # compat: weight 1 per level (buffer.cu:630-633)
    assert gc[0] > gp[0]


def test_adam_first_step_bias_correction():
    p = np.zeros(4, np.float32); g = np.ones(4, np.float32)
    for mode, expect in ((0, 0.0074419), (1, 0.01)):
        q = p.copy(); m = np.zeros(4, np.float32); v = np.zeros(4, np.float32)
        O.orc().adam(mode, 4, q, g, m, v, 1e-2, 0.9, 0.999, 1e-8, 1)
        assert abs(-q[0] - expect) < 2e-6, (mode, q[0])


def test_mse_compat_reduction_drops_tail():
    n = 24  # not a power of two: compat keeps the reference's reported value
    pred = np.ones(n, np.float32); tgt = np.zeros(n, np.float32); g = np.zeros(n, np.float32)
    exact = O.orc().mse(1, n, pred, tgt, g)
    assert exact == 12.0 and (g == 1).all()
    compat = O.orc().mse(0, n, pred, tgt, g)
    assert compat != exact
    n2 = 64
    pred = np.ones(n2, np.float32); tgt = np.zeros(n2, np.float32); g = np.zeros(n2, np.float32)
    assert O.orc().mse(0, n2, pred, tgt, g) == O.orc().mse(1, n2, pred, tgt, g) == 32.0


def test_tie_census_known_answers():
    """orc_raster_ties on scenes with known ties: the diagonal of a
    full-screen quad runs through the 8 pixel centres of an 8x8 view (8 edge
    ties, no depth ties); the same triangle drawn twice makes every covered
    pixel a depth tie won by the lower id; a generic scene has none."""
    quad = np.array([[-1, -1, 0.5, 1], [1, -1, 0.5, 1], [1, 1, 0.5, 1], [-1, 1, 0.5, 1]], np.float32)
    tri = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    r = np.zeros((64, 4), np.float32); d = r.copy()
    O.orc().rasterize_fwd(8, 8, 1, quad, 4, tri, 2, 1, r, d)
    f = np.zeros(64, np.uint32); c = np.zeros(2, np.int64)
    O.orc().raster_ties(8, 8, 1, quad, 4, tri, 2, r, f, c)
    assert tuple(c) == (8, 0)
    assert np.array_equal(np.nonzero(f.reshape(8, 8))[0], np.arange(8))
    dup = np.array([[-0.9, -0.8, 0.1, 1], [0.7, -0.6, 0.1, 1], [0.1, 0.9, 0.1, 1]] * 2, np.float32)
    tri = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    r = np.zeros((16 * 12, 4), np.float32); d = r.copy()
    O.orc().rasterize_fwd(16, 12, 1, dup, 6, tri, 2, 1, r, d)
    f = np.zeros(16 * 12, np.uint32)
    O.orc().raster_ties(16, 12, 1, dup, 6, tri, 2, r, f, c)
    assert c[1] == (r[:, 3] == 1).sum() > 0
    S = scenes.config1()
    clip = chain.project(O.orc(), S, S.pos)
    r = np.zeros((S.W * S.H, 4), np.float32); d = r.copy()
    O.orc().rasterize_fwd(S.W, S.H, 1, clip, S.nv, S.tri, S.nt, 1, r, d)
    f = np.zeros(S.W * S.H, np.uint32)
    O.orc().raster_ties(S.W, S.H, 1, clip, S.nv, S.tri, S.nt, r, f, c)
    assert tuple(c) == (0, 0)


@pytest.mark.parametrize("mode", [0, 1])
def test_sg_bwd_guarded_adds_drop_exactly_the_non_finite_terms(mode):
    """The restatement of the reference's guarded add (common.h:181) in the
    SG backward (material.cu:428-433): a NaN in channel c of dL/dout at one
    pixel drops that pixel's amplitude and diffuse terms of channel c (the
    same sums as with that channel's dL/dout set to 0) and its axis and
    sharpness terms, which mix every channel (the same sums as with the
    pixel's whole dL/dout set to 0); the results stay finite."""
    S = scenes.small(seed=2, W=64, H=48, views=3, subdiv=2, tex=64, K=5)
    o = chain.run_chain(O.orc(), S, mode, pyr=chain.build_pyramid(S, S.tex_target))
    N, C, K = S.W * S.H * S.views, S.C, S.K
    p = int(np.nonzero(o["rast"][:, 3] > 0)[0][17])

    def lobes(g):
        out = {"g_diffuse": np.zeros((N, C), np.float32), "g_axis": np.zeros((K, 3), np.float32),
               "g_sharp": np.zeros(K, np.float32), "g_amp": np.zeros((K, C), np.float32)}
        O.orc().sg_bwd(mode, S.W, S.H, S.views, C, o["rast"], K, S.lobe_axis_init, S.lobe_sharp_init,
                       S.lobe_amp_init, o["normal"], o["diffuse"], o["spec_axis"], o["spec_sharp"], o["spec_amp"],
                       np.ascontiguousarray(g, np.float32), out["g_diffuse"], out["g_axis"], out["g_sharp"],
                       out["g_amp"], None, None, None)
        return out

    g = o["g_color"].reshape(N, C).copy()
    g_nan = g.copy(); g_nan[p, 1] = np.nan
    g_ch0 = g.copy(); g_ch0[p, 1] = 0.0
    g_px0 = g.copy(); g_px0[p, :] = 0.0
    a, b, c = lobes(g_nan), lobes(g_ch0), lobes(g_px0)
    for k in a:
        assert np.isfinite(a[k]).all(), k
    assert np.array_equal(a["g_amp"], b["g_amp"])
    assert np.array_equal(a["g_diffuse"], b["g_diffuse"])
    assert np.array_equal(a["g_axis"], c["g_axis"])
    assert np.array_equal(a["g_sharp"], c["g_sharp"])

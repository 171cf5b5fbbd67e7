"""One fit iteration run operator by operator through a CPU library
(the C restatement or the reference's own kernels compiled for the host).

Used by the tests to compare the two CPU implementations with each other and
with the CUDA path, and by tests/golden/make_golden.py.
"""
import numpy as np

from oracle import oracle as O


def f32(shape, fill=0.0):
    return np.full(shape, fill, np.float32)


def build_pyramid(scene, texels, lib=None):
    lib = lib or O.orc()
    tw, th, C, L = scene.tex_w, scene.tex_h, scene.C, scene.levels
    pyr = np.zeros(O.pyramid_size(tw, th, C, L), np.float32)
    pyr[: tw * th * C] = texels.reshape(-1)
    lib.mip_build(tw, th, C, L, pyr)
    return pyr


def project(lib, scene, pos):
    clip = f32((scene.views, scene.nv, 4))
    for v in range(scene.views):
        out = f32((scene.nv, 4))
        lib.project_fwd(scene.nv, scene.mvp[v].copy(), pos, 4, out)
        clip[v] = out
    return clip


def run_chain(lib, scene, mode=0, target=None, rast=None, db=None, pos=None, pyr=None,
              lobes=None, raster_lib=None, adam_step=1):
    """Forward + backward of the predicted render, then one Adam step on a
    copy of the texture level 0 (none when adam_step is 0).  Returns a dict
    of every intermediate."""
    S = scene
    W, H, V, C, K = S.W, S.H, S.views, S.C, S.K
    N = W * H * V
    r = {}
    pos = S.pos if pos is None else pos
    r["clip"] = clip = project(lib, S, pos)
    if rast is None:
        rl = raster_lib or O.orc()
        rast = f32((N, 4)); db = f32((N, 4))
        rl.rasterize_fwd(W, H, V, clip, S.nv, S.tri, S.nt, 1, rast, db)
    r["rast"], r["db"] = rast, db
    uv = f32((N, 2)); uv_da = f32((N, 4))
    lib.interpolate_fwd(W, H, V, 2, 1, rast, db, S.uv, S.tri, uv, uv_da)
    r["uv"], r["uv_da"] = uv, uv_da
    if pyr is None:
        pyr = build_pyramid(S, S.tex_init)
    r["pyr"] = pyr
    diffuse = f32((N, C))
    lib.texture_fwd(W, H, V, S.tex_w, S.tex_h, C, S.levels, pyr, rast, uv, uv_da, diffuse)
    r["diffuse"] = diffuse
    normal = f32((N, 3)); lib.normal_axis_fwd(W, H, V, rast, S.rot, S.normal, S.tri, normal)
    view = f32((N, 3)); lib.view_axis_fwd(W, H, V, S.pvinv, view)
    r["normal"], r["view"] = normal, view
    rough = f32((N,), S.roughness)
    sax = f32((N, 3)); ssh = f32((N,)); sam = f32((N,))
    lib.sg_specular_fwd(W, H, V, rast, normal, view, rough, S.ior, sax, ssh, sam)
    r["spec_axis"], r["spec_sharp"], r["spec_amp"] = sax, ssh, sam
    axis, sharp, amp = lobes if lobes is not None else (S.lobe_axis_init, S.lobe_sharp_init, S.lobe_amp_init)
    color = f32((N, C)); denv = f32((N, C)); senv = f32((N, C))
    lib.sg_fwd(W, H, V, C, rast, K, axis, sharp, amp, normal, diffuse, sax, ssh, sam, color, denv, senv)
    r["color"], r["diffenv"], r["specenv"] = color, denv, senv
    aa = f32((N, C))
    lib.antialias_fwd(W, H, V, C, clip, S.nv, S.tri, rast, color, aa)
    r["aa"] = aa
    if target is None:
        target = np.random.default_rng(S.seed + 7).random((N, C)).astype(np.float32)
    r["target"] = target
    g_aa = f32((N, C))
    r["loss"] = lib.mse(mode, N * C, aa, target, g_aa)
    r["g_aa"] = g_aa
    g_color = f32((N, C)); g_clip = f32((V, S.nv, 4))
    lib.antialias_bwd(mode, W, H, V, C, clip, S.nv, S.tri, rast, color, g_aa, g_color, g_clip)
    r["g_color"], r["g_clip_aa"] = g_color, g_clip.copy()
    g_diffuse = f32((N, C)); g_axis = f32((K, 3)); g_sharp = f32((K,)); g_amp = f32((K, C))
    g_sax = f32((N, 3)); g_ssh = f32((N,)); g_sam = f32((N * C,))
    lib.sg_bwd(mode, W, H, V, C, rast, K, axis, sharp, amp, normal, diffuse, sax, ssh, sam, g_color,
               g_diffuse, g_axis, g_sharp, g_amp, g_sax, g_ssh, g_sam)
    r.update(g_diffuse=g_diffuse, g_axis=g_axis, g_sharp=g_sharp, g_amp=g_amp, g_sax=g_sax, g_ssh=g_ssh, g_sam=g_sam)
    g_rough = f32((N,))
    lib.sg_specular_bwd(W, H, V, rast, normal, view, rough, S.ior, g_sam, g_ssh, g_rough)
    r["g_rough"] = g_rough
    g_pyr = np.zeros_like(pyr); g_uv = f32((N, 2)); g_uv_da = f32((N, 4))
    lib.texture_bwd(mode, W, H, V, S.tex_w, S.tex_h, C, S.levels, pyr, rast, uv, uv_da, g_diffuse, g_pyr, g_uv, g_uv_da)
    r["g_pyr"], r["g_uv"], r["g_uv_da"] = g_pyr, g_uv, g_uv_da
    g_uvattr = f32((S.nv, 2)); g_bary = f32((N, 2))
    lib.interpolate_bwd(mode, W, H, V, 2, rast, S.uv, S.tri, g_uv, g_uvattr, g_bary)
    r["g_uvattr"], r["g_bary"] = g_uvattr, g_bary
    lib.rasterize_bwd(W, H, V, clip, S.nv, S.tri, rast, g_bary, g_clip)
    r["g_clip"] = g_clip
    g_pos = f32((S.nv, 3))
    for v in range(V):
        lib.project_bwd(S.nv, S.mvp[v].copy(), np.ascontiguousarray(g_clip[v]), 4, g_pos)
    r["g_pos"] = g_pos
    if adam_step:
        n0 = S.tex_w * S.tex_h * C
        p = pyr[:n0].copy(); m = f32((n0,)); vv = f32((n0,))
        lib.adam(mode, n0, p, np.ascontiguousarray(g_pyr[:n0]), m, vv, S.lr, 0.9, 0.999, 1e-8, adam_step)
        r["adam_p"], r["adam_m"], r["adam_v"] = p, m, vv
    return r


def oracle_fit(S, mode, steps, target, lr=None):
    """Full fit iterations on the CPU oracle, as a fit job runs them:
    forward/backward (run_chain), mip gradient push-down, Adam on texture
    level 0 + clamp + mip rebuild, Adam on positions and on the lobes
    (axis | sharpness | amplitude), all with persistent moments."""
    lib = O.orc()
    lr = S.lr if lr is None else lr
    lr_pos = getattr(S, "lr_pos", 0.0) or lr     # positions have their own Adam step (0: the common one)
    pos = S.pos.copy()
    pyr = build_pyramid(S, S.tex_init)
    lobes = np.concatenate([S.lobe_axis_init.reshape(-1), S.lobe_sharp_init.reshape(-1),
                            S.lobe_amp_init.reshape(-1)]).astype(np.float32)
    K, C = S.K, S.C
    n0 = S.tex_w * S.tex_h * C
    mt, vt = f32((n0,)), f32((n0,))
    mp, vp = f32((S.nv * 3,)), f32((S.nv * 3,))
    ml, vl = f32((lobes.size,)), f32((lobes.size,))
    losses = []
    for t in range(1, steps + 1):
        ax = np.ascontiguousarray(lobes[:3 * K].reshape(K, 3))
        sh = np.ascontiguousarray(lobes[3 * K:4 * K])
        am = np.ascontiguousarray(lobes[4 * K:].reshape(K, C))
        r = run_chain(lib, S, mode, target=target, pos=pos, pyr=pyr, lobes=(ax, sh, am))
        n = S.W * S.H * S.views * C
        losses.append(lib.mse(1, n, r["aa"], target, np.zeros(n, np.float32)))
        g = r["g_pyr"].copy()
        lib.mip_pushdown(mode, S.tex_w, S.tex_h, C, S.levels, g)
        p0 = np.ascontiguousarray(pyr[:n0])
        gr = np.abs(g[:n0]) / max(float(np.abs(g[:n0]).max()), 1e-30)
        g_tex_res = gr if t == 1 else np.minimum(g_tex_res, gr)    # how resolved each texel's gradient was
        lib.adam(mode, n0, p0, np.ascontiguousarray(g[:n0]), mt, vt, lr, 0.9, 0.999, 1e-8, t)
        lib.clamp(n0, p0, 0.0, 1.0)
        pyr = pyr.copy(); pyr[:n0] = p0
        lib.mip_build(S.tex_w, S.tex_h, C, S.levels, pyr)
        pp = np.ascontiguousarray(pos.reshape(-1))
        lib.adam(mode, pp.size, pp, np.ascontiguousarray(r["g_pos"].reshape(-1)), mp, vp, lr_pos, 0.9, 0.999, 1e-8, t)
        pos = pp.reshape(-1, 3)
        gl = np.concatenate([r["g_axis"].reshape(-1), r["g_sharp"].reshape(-1), r["g_amp"].reshape(-1)]).astype(np.float32)
        lib.adam(mode, lobes.size, lobes, gl, ml, vl, lr, 0.9, 0.999, 1e-8, t)
    ax = lobes[:3 * K].reshape(K, 3); sh = lobes[3 * K:4 * K]; am = lobes[4 * K:].reshape(K, C)
    return {"pos": pos, "tex": pyr[:n0].reshape(S.tex_h, S.tex_w, C), "axis": ax, "sharp": sh, "amp": am,
            "losses": losses, "pyr": pyr,
            "g_tex_resolved": g_tex_res.reshape(S.tex_h, S.tex_w, C)}


def run_isolated64(S, o, mode=0, chained=False):
    """Every operator of run_chain evaluated once more by the double-precision
    restatement (liborc64), each fed the FP32 oracle's own inputs for its
    stage (the values the isolated GPU chain gets), promoted to double: the
    exact result of each stage for those inputs, up to double rounding.  The
    parity tests measure how far the CUDA path and the FP32 restatement each
    are from it.  chained=True feeds each stage the double results of the
    stages before it instead (the exact chain from the same scene, target and
    rasterization; the raster's own outputs are discrete and bit-identical on
    both sides, so they stay the oracle's), for the chained comparison."""
    L = O.orc64()
    W, H, V, C, K = S.W, S.H, S.views, S.C, S.K
    N = W * H * V
    d = lambda a: np.ascontiguousarray(np.asarray(a, np.float64))
    z = lambda *shape: np.zeros(shape, np.float64)
    r = {}
    src = (lambda k: r[k]) if chained else (lambda k: d(o[k]))
    clip = z(V, S.nv, 4)
    for v in range(V):
        out = z(S.nv, 4)
        L.project_fwd(S.nv, d(S.mvp[v]), d(S.pos), 4, out)
        clip[v] = out
    r["clip"] = clip
    rast, db = d(o["rast"]), d(o["db"])
    uv, uv_da = z(N, 2), z(N, 4)
    L.interpolate_fwd(W, H, V, 2, 1, rast, db, d(S.uv), S.tri, uv, uv_da)
    r["uv"], r["uv_da"] = uv, uv_da
    pyr = d(o["pyr"])
    diffuse = z(N, C)
    L.texture_fwd(W, H, V, S.tex_w, S.tex_h, C, S.levels, pyr, rast, src("uv"), src("uv_da"), diffuse)
    r["diffuse"] = diffuse
    normal, view = z(N, 3), z(N, 3)
    L.normal_axis_fwd(W, H, V, rast, d(S.rot), d(S.normal), S.tri, normal)
    L.view_axis_fwd(W, H, V, d(S.pvinv), view)
    r["normal"], r["view"] = normal, view
    rough = np.full((N,), S.roughness, np.float64)
    sax, ssh, sam = z(N, 3), z(N), z(N)
    L.sg_specular_fwd(W, H, V, rast, src("normal"), src("view"), rough, S.ior, sax, ssh, sam)
    r["spec_axis"], r["spec_sharp"], r["spec_amp"] = sax, ssh, sam
    axis, sharp, amp = d(S.lobe_axis_init), d(S.lobe_sharp_init), d(S.lobe_amp_init)
    color, denv, senv = z(N, C), z(N, C), z(N, C)
    L.sg_fwd(W, H, V, C, rast, K, axis, sharp, amp, src("normal"), src("diffuse"), src("spec_axis"),
             src("spec_sharp"), src("spec_amp"), color, denv, senv)
    r["color"], r["diffenv"], r["specenv"] = color, denv, senv
    aa = z(N, C)
    L.antialias_fwd(W, H, V, C, src("clip"), S.nv, S.tri, rast, src("color"), aa)
    r["aa"] = aa
    g_aa = z(N, C)
    L.mse(mode, N * C, src("aa"), d(o["target"]), g_aa)
    r["g_aa"] = g_aa
    g_color, g_clip = z(N, C), z(V, S.nv, 4)
    L.antialias_bwd(mode, W, H, V, C, src("clip"), S.nv, S.tri, rast, src("color"), src("g_aa"), g_color, g_clip)
    r["g_color"], r["g_clip_aa"] = g_color, g_clip
    g_diffuse, g_axis, g_sharp, g_amp = z(N, C), z(K, 3), z(K), z(K, C)
    g_sax, g_ssh, g_sam = z(N, 3), z(N), z(N * C)
    L.sg_bwd(mode, W, H, V, C, rast, K, axis, sharp, amp, src("normal"), src("diffuse"), src("spec_axis"),
             src("spec_sharp"), src("spec_amp"), src("g_color"), g_diffuse, g_axis, g_sharp, g_amp, g_sax, g_ssh,
             g_sam)
    r.update(g_diffuse=g_diffuse, g_axis=g_axis, g_sharp=g_sharp, g_amp=g_amp, g_sax=g_sax, g_ssh=g_ssh, g_sam=g_sam)
    g_rough = z(N)
    L.sg_specular_bwd(W, H, V, rast, src("normal"), src("view"), rough, S.ior, src("g_sam"), src("g_ssh"),
                      g_rough)
    r["g_rough"] = g_rough
    g_pyr, g_uv, g_uv_da = np.zeros_like(pyr), z(N, 2), z(N, 4)
    L.texture_bwd(mode, W, H, V, S.tex_w, S.tex_h, C, S.levels, pyr, rast, src("uv"), src("uv_da"),
                  src("g_diffuse"), g_pyr, g_uv, g_uv_da)
    r["g_pyr"], r["g_uv"], r["g_uv_da"] = g_pyr, g_uv, g_uv_da
    g_uvattr, g_bary = z(S.nv, 2), z(N, 2)
    L.interpolate_bwd(mode, W, H, V, 2, rast, d(S.uv), S.tri, src("g_uv"), g_uvattr, g_bary)
    r["g_uvattr"], r["g_bary"] = g_uvattr, g_bary
    g_clip2 = src("g_clip_aa").copy()
    L.rasterize_bwd(W, H, V, src("clip"), S.nv, S.tri, rast, src("g_bary"), g_clip2)
    r["g_clip"] = g_clip2
    g_pos = z(S.nv, 3)
    gc = src("g_clip")
    for v in range(V):
        L.project_bwd(S.nv, d(S.mvp[v]), np.ascontiguousarray(gc[v]), 4, g_pos)
    r["g_pos"] = g_pos
    if "adam_p" in o:
        n0 = S.tex_w * S.tex_h * C
        p, m, vv = d(o["pyr"][:n0]).copy(), z(n0), z(n0)
        L.adam(mode, n0, p, np.ascontiguousarray(src("g_pyr")[:n0]), m, vv, S.lr, 0.9, 0.999, 1e-8, 1)
        r["adam_p"], r["adam_m"], r["adam_v"] = p, m, vv
    return r

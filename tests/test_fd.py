"""Analytic gradients against FP64 central finite differences.

The C restatement is compiled a second time with every float as double
(oracle/liborc64.so), and its backward operators are checked against central
differences of its own forward chain, in EXACT mode (the reference's
gradient quirks fixed; in COMPAT mode some gradients are knowingly not the
derivative).  The CUDA gradients equal the restatement's within 1e-5
(test_gpu_parity), so this pins them to the mathematics.

Cases (small, CPU):
* texels of level 0 through the full shaded chain (mip build -> trilinear
  texture -> SG shading -> antialias -> loss; gradient pushed down the mip
  pyramid with the exact 1/4 weights);
* SG lobe axis, sharpness and amplitude through the full chain;
* vertex positions through project -> rasterize -> interpolate(uv) ->
  texture -> antialias -> loss (colour = texture, so every stage on this
  path has a backward), at perturbations that leave every pixel's triangle
  unchanged, with a one-level texture (the reference, and this build, carry
  no gradient through the mip level's dependence on the DB derivatives).
"""
import numpy as np
import pytest

from oracle import oracle as O
from vcl_b200 import scenes

EXACT = 1


def _lib():
    return O.orc64()


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _z(*shape):
    return np.zeros(shape, np.float64)


def _scene():
    # 8x8 texture on a 48x40 render: magnified everywhere (mip level 0)
    return scenes.small(seed=11, W=48, H=40, views=2, subdiv=2, tex=8, K=4)


class Chain:
    """Forward to the loss 0.5 * sum((aa - target)^2) and the backward pass,
    in double precision, for one scene."""

    def __init__(self, S, shaded=True):
        self.S = S
        self.L = _lib()
        self.shaded = shaded
        N = S.W * S.H * S.views
        self.N = N
        self.target = np.random.default_rng(5).random((N, S.C))
        self.uv, self.nrm, self.rot, self.pvinv = _d(S.uv), _d(S.normal), _d(S.rot), _d(S.pvinv)
        self.mvp = _d(S.mvp)

    def pyramid(self, tex0):
        S, L = self.S, self.L
        pyr = _z(O.pyramid_size(S.tex_w, S.tex_h, S.C, S.levels))
        pyr[: S.tex_w * S.tex_h * S.C] = tex0.reshape(-1)
        L.mip_build(S.tex_w, S.tex_h, S.C, S.levels, pyr)
        return pyr

    def forward(self, pos, tex0, lobes, keep=False):
        S, L, N = self.S, self.L, self.N
        W, H, V, C, K = S.W, S.H, S.views, S.C, S.K
        clip = _z(V, S.nv, 4)
        for v in range(V):
            out = _z(S.nv, 4)
            L.project_fwd(S.nv, self.mvp[v].copy(), _d(pos), 4, out)
            clip[v] = out
        rast, db = _z(N, 4), _z(N, 4)
        L.rasterize_fwd(W, H, V, clip, S.nv, S.tri, S.nt, 1, rast, db)
        uv, uv_da = _z(N, 2), _z(N, 4)
        L.interpolate_fwd(W, H, V, 2, 1, rast, db, self.uv, S.tri, uv, uv_da)
        pyr = self.pyramid(tex0)
        diffuse = _z(N, C)
        L.texture_fwd(W, H, V, S.tex_w, S.tex_h, C, S.levels, pyr, rast, uv, uv_da, diffuse)
        st = dict(clip=clip, rast=rast, db=db, uv=uv, uv_da=uv_da, pyr=pyr, diffuse=diffuse)
        if self.shaded:
            axis, sharp, amp = lobes
            normal, view = _z(N, 3), _z(N, 3)
            L.normal_axis_fwd(W, H, V, rast, self.rot, self.nrm, S.tri, normal)
            L.view_axis_fwd(W, H, V, self.pvinv, view)
            rough = np.full(N, S.roughness, np.float64)
            sax, ssh, sam = _z(N, 3), _z(N), _z(N)
            L.sg_specular_fwd(W, H, V, rast, normal, view, rough, S.ior, sax, ssh, sam)
            color, denv, senv = _z(N, C), _z(N, C), _z(N, C)
            L.sg_fwd(W, H, V, C, rast, K, _d(axis), _d(sharp), _d(amp), normal, diffuse, sax, ssh, sam, color, denv,
                     senv)
            st.update(normal=normal, sax=sax, ssh=ssh, sam=sam, color=color, lobes=tuple(_d(x) for x in lobes))
        else:
            color = diffuse.copy()
            st["color"] = color
        aa = _z(N, C)
        L.antialias_fwd(W, H, V, C, clip, S.nv, S.tri, rast, color, aa)
        loss = 0.5 * float(np.sum((aa - self.target) ** 2))
        st["aa"] = aa
        return (loss, st) if keep else loss

    def backward(self, st):
        """Gradients of the loss w.r.t. texels (level 0), lobes and positions."""
        S, L, N = self.S, self.L, self.N
        W, H, V, C, K = S.W, S.H, S.views, S.C, S.K
        g_aa = st["aa"] - self.target
        g_color, g_clip = _z(N, C), _z(V, S.nv, 4)
        L.antialias_bwd(EXACT, W, H, V, C, st["clip"], S.nv, S.tri, st["rast"], st["color"], g_aa, g_color, g_clip)
        out = {}
        if self.shaded:
            axis, sharp, amp = st["lobes"]
            g_diffuse, g_axis, g_sharp, g_amp = _z(N, C), _z(K, 3), _z(K), _z(K, C)
            g_sax, g_ssh, g_sam = _z(N, 3), _z(N), _z(N * C)
            L.sg_bwd(EXACT, W, H, V, C, st["rast"], K, axis, sharp, amp, st["normal"], st["diffuse"], st["sax"],
                     st["ssh"], st["sam"], g_color, g_diffuse, g_axis, g_sharp, g_amp, g_sax, g_ssh, g_sam)
            out.update(axis=g_axis, sharp=g_sharp, amp=g_amp)
        else:
            g_diffuse = g_color
        g_pyr, g_uv, g_uv_da = np.zeros_like(st["pyr"]), _z(N, 2), _z(N, 4)
        L.texture_bwd(EXACT, W, H, V, S.tex_w, S.tex_h, C, S.levels, st["pyr"], st["rast"], st["uv"], st["uv_da"],
                      g_diffuse, g_pyr, g_uv, g_uv_da)
        out["coarse_grad"] = float(np.abs(g_pyr[S.tex_w * S.tex_h * C:]).max(initial=0.0))
        L.mip_pushdown(EXACT, S.tex_w, S.tex_h, C, S.levels, g_pyr)
        out["tex"] = g_pyr[: S.tex_w * S.tex_h * C].reshape(S.tex_h, S.tex_w, C)
        g_attr, g_bary = _z(S.nv, 2), _z(N, 2)
        L.interpolate_bwd(EXACT, W, H, V, 2, st["rast"], self.uv, S.tri, g_uv, g_attr, g_bary)
        L.rasterize_bwd(W, H, V, st["clip"], S.nv, S.tri, st["rast"], g_bary, g_clip)
        g_pos = _z(S.nv, 3)
        for v in range(V):
            L.project_bwd(S.nv, self.mvp[v].copy(), np.ascontiguousarray(g_clip[v]), 4, g_pos)
        out["pos"] = g_pos
        return out


def _lobes(S):
    return _d(S.lobe_axis_init), _d(S.lobe_sharp_init), _d(S.lobe_amp_init)


def test_double_build_matches_float_build():
    """The double build is the same restatement: its forward agrees with the
    float build to float rounding."""
    S = _scene()
    ch = Chain(S)
    loss, st = ch.forward(_d(S.pos), _d(S.tex_init), _lobes(S), keep=True)
    import chain as C32
    r = C32.run_chain(O.orc(), S, 0, target=ch.target.astype(np.float32))
    assert np.array_equal(st["rast"][:, 3], r["rast"][:, 3])
    assert np.abs(st["aa"] - r["aa"]).max() <= 1e-5 * max(1.0, np.abs(r["aa"]).max())


def test_texel_gradients_match_central_differences():
    S = _scene()
    ch = Chain(S)
    pos, tex0, lobes = _d(S.pos), _d(S.tex_init).copy(), _lobes(S)
    loss, st = ch.forward(pos, tex0, lobes, keep=True)
    g = ch.backward(st)["tex"]
    rng = np.random.default_rng(0)
    idx = [tuple(rng.integers(0, s) for s in tex0.shape) for _ in range(24)]
    idx += [tuple(int(x) for x in np.unravel_index(np.argmax(np.abs(g)), g.shape))]
    h = 1e-4
    for i in idx:
        tp, tm = tex0.copy(), tex0.copy()
        tp[i] += h
        tm[i] -= h
        fd = (ch.forward(pos, tp, lobes) - ch.forward(pos, tm, lobes)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g).max()), (i, fd, g[i])


@pytest.mark.parametrize("which", ["axis", "sharp", "amp"])
def test_lobe_gradients_match_central_differences(which):
    S = _scene()
    ch = Chain(S)
    pos, tex0 = _d(S.pos), _d(S.tex_init)
    lobes = list(_lobes(S))
    loss, st = ch.forward(pos, tex0, tuple(lobes), keep=True)
    g = ch.backward(st)[which]
    k = {"axis": 0, "sharp": 1, "amp": 2}[which]
    h = 1e-6
    scale = max(1e-3, np.abs(g).max())
    for i in np.ndindex(*lobes[k].shape):
        lp, lm = [x.copy() for x in lobes], [x.copy() for x in lobes]
        lp[k][i] += h
        lm[k][i] -= h
        fd = (ch.forward(pos, tex0, tuple(lp)) - ch.forward(pos, tex0, tuple(lm))) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * scale, (which, i, fd, g[i])


def test_position_gradients_match_central_differences():
    S = _scene()
    S.levels = 1        # one mip level: the level selection cannot move with the geometry
    ch = Chain(S, shaded=False)
    pos, tex0 = _d(S.pos), _d(S.tex_target)
    loss, st = ch.forward(pos, tex0, None, keep=True)
    grads = ch.backward(st)
    assert grads["coarse_grad"] == 0.0, "texture must stay at mip level 0 for this check"
    g = grads["pos"]
    ids0 = st["rast"][:, 3].copy()
    rng = np.random.default_rng(1)
    order = np.argsort(-np.abs(g).reshape(-1))
    cand = list(order[:20]) + list(rng.choice(g.size, 40, replace=False))
    h = 1e-5
    checked = 0
    scale = np.abs(g).max()
    for flat in cand:
        i = np.unravel_index(flat, g.shape)
        pp, pm = pos.copy(), pos.copy()
        pp[i] += h
        pm[i] -= h
        lp, sp = ch.forward(pp, tex0, None, keep=True)
        lm, sm = ch.forward(pm, tex0, None, keep=True)
        if not (np.array_equal(sp["rast"][:, 3], ids0) and np.array_equal(sm["rast"][:, 3], ids0)):
            continue            # coverage changed: the loss is not differentiable across it
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 2e-4 * scale, (i, fd, g[i])
        checked += 1
    assert checked >= 20


@pytest.mark.parametrize("mode", [0, 1])
def test_exact_stage_values_close_to_fp32_chain(mode):
    """The exact stage values the GPU parity bars measure against
    (chain.run_isolated64, each operator of the double build fed the FP32
    chain's inputs, or with chained=True its own double results) are the
    same computation as the FP32 restatement: every key within FP32 rounding
    of it, normwise (2e-5 isolated; 1e-4 chained, where the rounding of each
    stage feeds the next)."""
    import chain as C32
    from vcl_b200 import scenes
    keys = ["clip", "uv", "uv_da", "diffuse", "normal", "view", "spec_axis", "spec_sharp", "spec_amp", "color",
            "diffenv", "specenv", "aa", "g_aa", "g_color", "g_clip_aa", "g_diffuse", "g_axis", "g_sharp", "g_amp",
            "g_sax", "g_ssh", "g_sam", "g_rough", "g_pyr", "g_uv", "g_uv_da", "g_uvattr", "g_bary", "g_clip",
            "g_pos"]
    S = scenes.small(seed=2, W=64, H=48, views=3, subdiv=2, tex=64, K=5)
    o = C32.run_chain(O.orc(), S, mode, pyr=C32.build_pyramid(S, S.tex_target))
    for chained, tol in ((False, 2e-5), (True, 1e-4)):
        e = C32.run_isolated64(S, o, mode, chained=chained)
        for k in keys:
            a = np.asarray(o[k], np.float64).reshape(-1)
            b = np.asarray(e[k], np.float64).reshape(-1)
            err = np.abs(a - b).max(initial=0.0) / max(np.abs(b).max(initial=0.0), 1e-30)
            assert err <= tol, (k, chained, err)

"""The CUDA path through the C ABI, operator by operator, for the parity
tests.  Each operator is fed the oracle's inputs for that stage (so every
comparison isolates one kernel), or -- with chained=True -- the GPU's own
previous outputs (end-to-end)."""
import numpy as np
import torch

from vcl_b200 import capi


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def host(t):
    return t.detach().cpu().numpy()


def zeros(*shape):
    return torch.zeros(*shape, dtype=torch.float32, device="cuda")


def run_chain_gpu(ctx, S, o, mode=0, chained=False, adam_step=1):
    """o: the oracle's dict from chain.run_chain (inputs and expected outputs)."""
    ctx.set_mode(mode)
    W, H, V, C, K = S.W, S.H, S.views, S.C, S.K
    N = W * H * V
    nv, nt = S.nv, S.nt
    g = {}
    pick = (lambda k: g[k]) if chained else (lambda k: dev(o[k]))
    tri = dev(S.tri.astype(np.int32))
    mvp = dev(S.mvp)
    pos = dev(S.pos)
    clip = zeros(V, nv, 4)
    ctx.project_fwd(mvp, V, pos, nv, 4, clip, None)
    g["clip"] = clip
    rast = zeros(N, 4); db = zeros(N, 4)
    ctx.rasterize_fwd(pick("clip"), nv, tri, nt, W, H, V, rast, db, None)
    g["rast"], g["db"] = rast, db
    uvattr = dev(S.uv)
    uv = zeros(N, 2); uv_da = zeros(N, 4)
    ctx.interpolate_fwd(pick("rast"), pick("db"), W, H, V, uvattr, nv, 2, tri, nt, uv, uv_da, None)
    g["uv"], g["uv_da"] = uv, uv_da
    pyr = dev(o["pyr"])
    g["pyr"] = pyr
    diffuse = zeros(N, C)
    ctx.texture_fwd(pick("rast"), pick("uv"), pick("uv_da"), W, H, V, pyr, S.tex_w, S.tex_h, C, S.levels, diffuse, None)
    g["diffuse"] = diffuse
    normal = zeros(N, 3)
    ctx.normal_axis_fwd(pick("rast"), W, H, V, dev(S.rot), dev(S.normal), nv, tri, nt, normal, None)
    view = zeros(N, 3)
    ctx.view_axis_fwd(W, H, V, dev(S.pvinv), view, None)
    g["normal"], g["view"] = normal, view
    rough = torch.full((N,), S.roughness, dtype=torch.float32, device="cuda")
    sax = zeros(N, 3); ssh = zeros(N); sam = zeros(N)
    ctx.sg_specular_fwd(pick("rast"), W, H, V, pick("normal"), pick("view"), rough, S.ior, sax, ssh, sam, None)
    g["spec_axis"], g["spec_sharp"], g["spec_amp"] = sax, ssh, sam
    axis, sharp, amp = dev(S.lobe_axis_init), dev(S.lobe_sharp_init), dev(S.lobe_amp_init)
    color = zeros(N, C); denv = zeros(N, C); senv = zeros(N, C)
    ctx.sg_fwd(pick("rast"), W, H, V, C, K, axis, sharp, amp, pick("normal"), pick("diffuse"), pick("spec_axis"),
               pick("spec_sharp"), pick("spec_amp"), color, denv, senv, None)
    g["color"], g["diffenv"], g["specenv"] = color, denv, senv
    aa = zeros(N, C)
    ctx.antialias_fwd(pick("clip"), nv, tri, nt, pick("rast"), W, H, V, C, pick("color"), aa, None)
    g["aa"] = aa
    target = dev(o["target"])
    g_aa = zeros(N, C)
    loss = zeros(1)
    ctx.mse(pick("aa"), target, N * C, g_aa, loss, None)
    g["g_aa"], g["loss_t"] = g_aa, loss
    g_color = zeros(N, C); g_clip = zeros(V, nv, 4)
    ctx.antialias_bwd(pick("clip"), nv, tri, nt, pick("rast"), W, H, V, C, pick("color"), pick("g_aa"), g_color, g_clip,
                      None)
    g["g_color"], g["g_clip_aa"] = g_color, g_clip.clone()
    g_diffuse = zeros(N, C); g_axis = zeros(K, 3); g_sharp = zeros(K); g_amp = zeros(K, C)
    g_sax = zeros(N, 3); g_ssh = zeros(N); g_sam = zeros(N * C)
    ctx.sg_bwd(pick("rast"), W, H, V, C, K, axis, sharp, amp, pick("normal"), pick("diffuse"), pick("spec_axis"),
               pick("spec_sharp"), pick("spec_amp"), pick("g_color"), g_diffuse, g_axis, g_sharp, g_amp, g_sax, g_ssh,
               g_sam, None)
    g.update(g_diffuse=g_diffuse, g_axis=g_axis, g_sharp=g_sharp, g_amp=g_amp, g_sax=g_sax, g_ssh=g_ssh, g_sam=g_sam)
    g_rough = zeros(N)
    ctx.sg_specular_bwd(pick("rast"), W, H, V, pick("normal"), pick("view"), rough, S.ior, pick("g_sam"),
                        pick("g_ssh"), g_rough, None)
    g["g_rough"] = g_rough
    g_pyr = torch.zeros_like(pyr); g_uv = zeros(N, 2); g_uv_da = zeros(N, 4)
    ctx.texture_bwd(pick("rast"), pick("uv"), pick("uv_da"), W, H, V, pyr, S.tex_w, S.tex_h, C, S.levels,
                    pick("g_diffuse"), g_pyr, g_uv, g_uv_da, None)
    g["g_pyr"], g["g_uv"], g["g_uv_da"] = g_pyr, g_uv, g_uv_da
    g_uvattr = zeros(nv, 2); g_bary = zeros(N, 2)
    ctx.interpolate_bwd(pick("rast"), W, H, V, uvattr, nv, 2, tri, nt, pick("g_uv"), g_uvattr, g_bary, None)
    g["g_uvattr"], g["g_bary"] = g_uvattr, g_bary
    g_clip2 = g_clip if chained else dev(o["g_clip_aa"])
    ctx.rasterize_bwd(pick("clip"), nv, tri, nt, W, H, V, pick("rast"), pick("g_bary"), g_clip2, None)
    g["g_clip"] = g_clip2
    g_pos = zeros(nv, 3)
    ctx.project_bwd(mvp, V, pick("g_clip"), nv, 4, g_pos, None)
    g["g_pos"] = g_pos
    n0 = S.tex_w * S.tex_h * C
    p = pyr[:n0].clone(); m = zeros(n0); v = zeros(n0)
    gp = g_pyr[:n0].clone() if chained else dev(o["g_pyr"][:n0])
    ctx.adam_step(p, gp, m, v, n0, S.lr, 0.9, 0.999, 1e-8, adam_step, None)
    g["adam_p"], g["adam_m"], g["adam_v"] = p, m, v
    torch.cuda.synchronize()
    out = {k: host(t) for k, t in g.items() if k != "loss_t"}
    out["loss"] = float(host(g["loss_t"])[0])
    return out

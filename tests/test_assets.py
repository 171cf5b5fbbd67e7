"""Asset loaders (vcl_obj_load, vcl_bmp_load, vcl_sg_load) on files written
here: the OBJ face forms the reference's loader accepts (buffer.cu:203-306),
polygons, negative indices and welding; 24- and 32-bit BMPs with padded rows
and both row orders (buffer.cu:498-541); lobe lists (buffer.cu:706-732).
Host code only -- these run without a GPU."""
import os
import struct

import numpy as np
import pytest

from oracle import oracle as O
from vcl_b200 import capi


def _write(path, text):
    with open(path, "w") as f:
        f.write(text)
    return path


CUBE_V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)


def test_obj_positions_only(tmp_path):
    p = _write(tmp_path / "a.obj", "# quad\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3\nf 1 3 4\n")
    m = capi.load_obj(p)
    assert np.array_equal(m["pos"], CUBE_V)
    assert np.array_equal(m["pos_idx"], [[0, 1, 2], [0, 2, 3]])
    assert m["texel"] is None and m["normal"] is None
    assert np.array_equal(m["w_pos"], CUBE_V) and np.array_equal(m["w_tri"], m["pos_idx"])
    assert not m["w_uv"].any() and not m["w_normal"].any()


@pytest.mark.parametrize("form", ["p/t/n", "p/t", "p//n"])
def test_obj_face_forms_and_weld(tmp_path, form):
    vt = "vt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\nvt 0.5 0.5\n"
    vn = "vn 0 0 1\nvn 0 0 -1\n"
    corners = {
        "p/t/n": ("1/1/1 2/2/1 3/3/1", "1/5/2 3/3/1 4/4/1"),
        "p/t": ("1/1 2/2 3/3", "1/5 3/3 4/4"),
        "p//n": ("1//1 2//1 3//1", "1//2 3//1 4//1"),
    }[form]
    text = "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\n" + (vt if "/t" in form else "") + (vn if "n" in form[-1] else "")
    text += "f " + corners[0] + "\nf " + corners[1] + "\n"
    m = capi.load_obj(_write(tmp_path / "b.obj", text))
    assert np.array_equal(m["pos_idx"], [[0, 1, 2], [0, 2, 3]])
    # vertex 1 carries two different (texel or normal) corners: welding splits it
    assert m["w_pos"].shape[0] == 5
    wp, wt = m["w_pos"], m["w_tri"]
    assert np.array_equal(wp[wt], CUBE_V[m["pos_idx"]])
    if m["texel"] is not None:
        assert np.array_equal(m["w_uv"][wt], m["texel"][m["texel_idx"]])
    if m["normal"] is not None:
        assert np.array_equal(m["w_normal"][wt], m["normal"][m["normal_idx"]])


def test_obj_polygon_fan_and_negative_indices(tmp_path):
    text = "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0.5 1.5 0\ng poly\ns off\nf -5 -4 -3 -2 -1\n"
    m = capi.load_obj(_write(tmp_path / "c.obj", text))
    assert np.array_equal(m["pos_idx"], [[0, 1, 2], [0, 2, 3], [0, 3, 4]])


@pytest.mark.parametrize("text", ["v 0 0 0\nv 1 0 0\nf 1 2 3\n", "v 0 0\n", "f 1 2 3\n", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2\n"])
def test_obj_errors_are_reported(tmp_path, text):
    with pytest.raises(capi.VclError):
        capi.load_obj(_write(tmp_path / "bad.obj", text))
    with pytest.raises(capi.VclError, match="cannot open"):
        capi.load_obj(tmp_path / "missing.obj")


def _bmp(path, img_u8, top_down=False):
    """Write an uncompressed BMP: img [H][W][C] as the caller's rows, stored
    bottom-up (or top-down), channel bytes reversed (RGB -> BGR)."""
    H, W, C = img_u8.shape
    stride = (W * C + 3) // 4 * 4
    rows = []
    order = range(H) if not top_down else range(H - 1, -1, -1)
    for y in order:
        r = img_u8[y][:, ::-1].reshape(-1).tobytes()
        rows.append(r + b"\0" * (stride - W * C))
    data = b"".join(rows)
    header = b"BM" + struct.pack("<IHHI", 54 + len(data), 0, 0, 54)
    info = struct.pack("<IiiHHIIiiII", 40, W, -H if top_down else H, 1, 8 * C, 0, len(data), 2835, 2835, 0, 0)
    with open(path, "wb") as f:
        f.write(header + info + data)
    return path


@pytest.mark.parametrize("C", [3, 4, 1])
@pytest.mark.parametrize("W", [5, 8])
@pytest.mark.parametrize("top_down", [False, True])
def test_bmp_channels_padding_and_rows(tmp_path, C, W, top_down):
    rng = np.random.default_rng(C * 10 + W)
    img = rng.integers(0, 256, size=(3, W, C), dtype=np.uint8)   # rows bottom-up
    out = capi.load_bmp(_bmp(tmp_path / "t.bmp", img, top_down))
    assert out.shape == (3, W, C)
    assert np.array_equal(out, img.astype(np.float32) / np.float32(255.0))


def test_bmp_rejects_other_files(tmp_path):
    with pytest.raises(capi.VclError, match="not a BMP"):
        capi.load_bmp(_write(tmp_path / "x.bmp", "hello, not an image" * 10))


def test_sg_lobe_list(tmp_path):
    rng = np.random.default_rng(3)
    lob = rng.normal(size=(7, 7)).astype(np.float32)
    text = "\n".join(" ".join(f"{x:.7g}" for x in r) for r in lob) + "\n"
    ax, sh, am = capi.load_sg(_write(tmp_path / "env.txt", text))
    ref = np.array([[float(f"{x:.7g}") for x in r] for r in lob], np.float32)
    assert np.array_equal(ax, ref[:, :3]) and np.array_equal(sh, ref[:, 3]) and np.array_equal(am, ref[:, 4:])
    with pytest.raises(capi.VclError, match="of 7 numbers"):
        capi.load_sg(_write(tmp_path / "short.txt", text + "1 2 3\n"))


ENVMAP = os.path.join(O.REF_DIR, "data", "envmap2.txt")


@pytest.mark.skipif(not os.path.exists(ENVMAP), reason="the reference's lobe file is not on this machine")
def test_sg_loads_the_reference_lobe_file():
    ax, sh, am = capi.load_sg(ENVMAP)
    ref = np.loadtxt(ENVMAP, dtype=np.float64).reshape(-1, 7).astype(np.float32)
    assert ax.shape[0] == 256 == ref.shape[0]
    assert np.array_equal(ax, ref[:, :3]) and np.array_equal(sh, ref[:, 3]) and np.array_equal(am, ref[:, 4:])


def _sphere_assets(tmp_path):
    """An icosphere OBJ with texels and normals, a 24-bit BMP and a lobe
    list, written with this test's own writers."""
    from vcl_b200 import scenes
    v, f = scenes.icosphere(2)
    uv = scenes.spherical_uv(v)
    lines = [f"v {a:.6f} {b:.6f} {c:.6f}" for a, b, c in v]
    lines += [f"vt {a:.6f} {b:.6f}" for a, b in uv]
    lines += [f"vn {a:.6f} {b:.6f} {c:.6f}" for a, b, c in v]
    lines += ["f " + " ".join(f"{i + 1}/{i + 1}/{i + 1}" for i in t) for t in f]
    obj = _write(tmp_path / "sphere.obj", "\n".join(lines) + "\n")
    rng = np.random.default_rng(0)
    bmp = _bmp(tmp_path / "tex.bmp", rng.integers(0, 256, size=(32, 32, 3), dtype=np.uint8))
    lob = np.concatenate([rng.normal(size=(6, 3)), rng.uniform(2, 20, size=(6, 1)), rng.random((6, 3))], axis=1)
    sg = _write(tmp_path / "env.txt", "\n".join(" ".join(f"{x:.6f}" for x in r) for r in lob) + "\n")
    return obj, bmp, sg


def test_scene_from_assets_is_consistent(tmp_path):
    from vcl_b200 import scenes
    obj, bmp, sg = _sphere_assets(tmp_path)
    m = capi.load_obj(obj)
    S = scenes.scene_from_assets("asset", m, capi.load_bmp(bmp), capi.load_sg(sg), W=48, H=40, views=2)
    assert S.nt == 320 and S.nv == m["w_pos"].shape[0]
    assert S.tex_target.shape == (32, 32, 4) and np.all(S.tex_target[..., 3] == 1)
    assert S.lobe_amp.shape == (6, 4) and np.all(S.lobe_amp[:, 3] == 0)
    assert np.abs(np.linalg.norm(S.pos, axis=1) - 1).max() < 1e-3


@pytest.mark.gpu
def test_fit_on_loaded_assets_matches_oracle(tmp_path):
    """A fit job built from files (OBJ + BMP + lobe list) runs fused fit
    iterations that agree with the CPU oracle's full iterations."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chain
    from vcl_b200 import scenes
    obj, bmp, sg = _sphere_assets(tmp_path)
    S = scenes.scene_from_assets("asset", capi.load_obj(obj), capi.load_bmp(bmp), capi.load_sg(sg),
                                 W=64, H=48, views=2, seed=4)
    tgt = np.random.default_rng(9).random((S.W * S.H * S.views, S.C)).astype(np.float32)
    ref = chain.oracle_fit(S, 0, 3, tgt)
    ctx = capi.Context(0)
    try:
        fit = capi.Fit(ctx, S, strategy=capi.FIT_FUSED)
        fit.set_target(tgt)
        st = torch.cuda.Stream()
        losses = []
        for _ in range(3):
            fit.step(st.cuda_stream)
            losses.append(fit.read_loss(st.cuda_stream))
        pos, tex, (ax, sh, am) = fit.read_params(st.cuda_stream)
        fit.close()
    finally:
        ctx.close()
    assert np.allclose(losses, ref["losses"], rtol=1e-5), (losses, ref["losses"])
    for got, want in ((tex, ref["tex"]), (pos, ref["pos"]), (am, ref["amp"]), (sh, ref["sharp"])):
        d = np.abs(got.astype(np.float64) - want).reshape(-1)
        assert d.max() <= 2 * S.lr * 3
        assert np.quantile(d, 0.99) <= 1e-5 * max(1.0, float(np.abs(want).max()))

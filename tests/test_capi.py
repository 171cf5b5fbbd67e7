"""CPU checks of the C-ABI library: it loads without a GPU and exports every
function that include/vcl.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"VCL_API[^;(]*?\b(vcl_\w+)\s*\(", text, flags=re.S)
    return names


def test_header_declares_the_boundary():
    names = header_functions()
    for must in ("vcl_rasterize_fwd", "vcl_rasterize_bwd", "vcl_interpolate_fwd", "vcl_interpolate_bwd",
                 "vcl_texture_fwd", "vcl_texture_bwd", "vcl_texture_build_mips", "vcl_texture_grad_pushdown",
                 "vcl_antialias_fwd", "vcl_antialias_bwd", "vcl_sg_fwd", "vcl_sg_bwd", "vcl_adam_step",
                 "vcl_fit_step"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from vcl_b200 import capi
    if not os.path.exists(capi.LIB_PATH):
        pytest.skip("libvcl.so not built (python -m vcl_b200.build)")
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares each of them too
    assert sorted(set(header_functions())) == sorted(set(capi.SIGNATURES)), \
        set(header_functions()) ^ set(capi.SIGNATURES)
    capi.lib()   # argtypes resolve for every symbol


def test_host_helpers_without_gpu():
    from vcl_b200 import capi
    if not os.path.exists(capi.LIB_PATH):
        pytest.skip("libvcl.so not built")
    L = capi.lib()
    assert L.vcl_tex_levels(2048, 2048, 16) == 12
    assert L.vcl_tex_levels(512, 512, 16) == 10
    assert L.vcl_tex_levels(4096, 4096, 16) == 13
    assert L.vcl_tex_level_offset(4, 4, 4, 2) == 4 * 4 * 4 + 2 * 2 * 4
    assert b"sm_100a" in L.vcl_version()
    # creating a context without a device fails cleanly (no exit, no crash)
    import torch
    if not torch.cuda.is_available():
        h = ctypes.c_void_p()
        assert L.vcl_create(0, ctypes.byref(h)) != 0


def test_fit_footprint_without_gpu():
    """vcl_fit_footprint is host arithmetic (admission control needs it before
    any device work): it grows with the views, the triangles and the texture,
    and covers at least the per-pixel buffers of both strategies."""
    from vcl_b200 import capi, scenes
    if not os.path.exists(capi.LIB_PATH):
        pytest.skip("libvcl.so not built")
    f4, f16 = capi.footprint(scenes.config2(views=4)), capi.footprint(scenes.config2(views=16))
    assert f16 > 3 * f4
    px16 = 16 * 1024 * 1024
    assert f16 >= 248 * px16          # per-pixel intermediates, gradients, targets and raster keys
    small = scenes.small(seed=1)
    dense = scenes.small(seed=1, subdiv=3)
    assert capi.footprint(dense) > capi.footprint(small)
    bigtex = scenes.small(seed=1, tex=256)
    assert capi.footprint(bigtex) > capi.footprint(small) + 256 * 256 * 4 * 4 * 3   # texture, grads, Adam m and v

"""ctypes bindings for the CPU checker.  TEST INFRASTRUCTURE ONLY.

Three libraries with the same function signatures:

* ``liborc.so`` -- the C restatement in ``vcl_oracle.c`` (always available;
  built from source on first use if missing);
* ``liborc64.so`` -- the same restatement with float replaced by double
  (``vcl_oracle64.c``), for the finite-difference gradient checks;
* ``_ref/libvclref.so`` -- the reference's own kernel sources compiled as host
  C++ by ``make -C oracle ref`` (available where the reference sources were
  present at build time).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout the recipes read (present only where the oracle's
# reference build is made; the GPU tests never need it)
REF_DIR = os.environ.get("VCL_REF_DIR", "/root/reference")
ORC_PATH = os.path.join(HERE, "liborc.so")
REF_PATH = os.path.join(HERE, "_ref", "libvclref.so")

_f = ctypes.c_float
_i = ctypes.c_int
_d = ctypes.c_double
_sz = ctypes.c_size_t
_p = ctypes.c_void_p

# name -> argument kinds ('i' int, 'f' float, 'd' double, 'z' size_t,
# 'p' pointer), in the order of vcl_oracle.h
SIGS = {
    "project_fwd": "ippip",
    "project_bwd": "ippip",
    "rasterize_fwd": "iiipipiipp",
    "raster_ties": "iiipipippp",
    "rasterize_bwd": "iiipipppp",
    "interpolate_fwd": "iiiiipppppp",
    "interpolate_bwd": "iiiiipppppp",
    "texture_fwd": "iiiiiiippppp",
    "texture_bwd": "iiiiiiiipppppppp",
    "mip_build": "iiiip",
    "mip_pushdown": "iiiiip",
    "clamp": "zpff",
    "antialias_fwd": "iiiipipppp",
    "antialias_bwd": "iiiiipipppppp",
    "normal_axis_fwd": "iiippppp",
    "view_axis_fwd": "iiipp",
    "sg_specular_fwd": "iiippppfppp",
    "sg_specular_bwd": "iiippppfppp",
    "sg_fwd": "iiiipi" + "p" * 11,
    "sg_bwd": "iiiiipi" + "p" * 16,
    "mse": "izppp",
    "adam": "izpppp" + "dddd" + "i",
}
_RESTYPE = {"mse": _f}
_KIND = {"i": _i, "f": _f, "d": _d, "z": _sz, "p": _p}


def _build_orc():
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


class _Lib:
    def __init__(self, path, prefix, real=np.float32):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        self.path = path
        self.dtype = real
        kind = dict(_KIND)
        if real == np.float64:
            kind["f"] = _d          # float scalars are double in the double build
        for name, kinds in SIGS.items():
            fn = getattr(self.lib, prefix + name, None)
            if fn is None:
                continue
            fn.argtypes = [kind[k] for k in kinds]
            fn.restype = _d if (real == np.float64 and name in _RESTYPE) else _RESTYPE.get(name, None)

    def has(self, name):
        return hasattr(self.lib, self.prefix + name)

    def __getattr__(self, name):
        fn = getattr(self.lib, self.prefix + name)

        def call(*args):
            conv = []
            for a in args:
                if isinstance(a, np.ndarray):
                    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
                    conv.append(a.ctypes.data)
                elif a is None:
                    conv.append(None)
                else:
                    conv.append(a)
            return fn(*conv)

        return call


_orc = None
_ref = None


def orc():
    """The C restatement (builds it from source when missing)."""
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_PATH):
            _build_orc()
        _orc = _Lib(ORC_PATH, "orc_")
    return _orc


_orc64 = None


def orc64():
    """The C restatement compiled in double precision (arrays and scalars
    that the header declares float are double), for finite differences."""
    global _orc64
    if _orc64 is None:
        path = os.path.join(HERE, "liborc64.so")
        if not os.path.exists(path):
            _build_orc()
        _orc64 = _Lib(path, "orc_", real=np.float64)
    return _orc64


def ref():
    """The reference's own kernels compiled for the host, or None."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        _ref = _Lib(REF_PATH, "ref_")
        _ref.set_threads = _ref.lib.ref_set_threads
        _ref.set_threads.argtypes = [_i]
    return _ref


def tex_levels(tw, th, requested):
    return orc().lib.orc_tex_levels(tw, th, requested)


def pyramid_size(tw, th, C, levels):
    return sum((tw >> l) * (th >> l) * C for l in range(levels))

"""Parity measures shared by the GPU tests.

Two bars for every floating-point output, both against the oracle's value b
of the same quantity:

* normwise: max|a - b| / max|b| <= 1e-5 (FP32; the bar the operator tests
  have always used);
* element-wise: |a - b| <= tol * |b| on every entry with |b| above 1e-3 of
  the array's largest magnitude.  tol = 1e-5 for per-pixel outputs (each
  entry is computed by one thread from the same inputs).  Entries that are
  sums over many pixels (texel, vertex and lobe gradients: floating-point
  atomics on the GPU, a serial loop in the oracle) are compared at 1e-4:
  their value depends on the order of the additions: the reference's own
  kernels compiled for the host and launched serially (block by block,
  thread by thread) add in another order than the restatement's pixel loop
  and differ from it by up to 5.4e-5 element-wise on these arrays at the
  256x256 configuration, while agreeing bit for bit on every per-pixel
  output.

`report()` appends one JSON line per check to the file named by the
VCL_PARITY_REPORT environment variable (when set), so a run can keep the
worst element per key.
"""
import json
import os

import numpy as np

NORM_TOL = 1e-5
ELEM_TOL = 1e-5
ELEM_TOL_SUM = 1e-4
ELEM_FLOOR = 1e-3

# outputs that are sums over pixels (order-dependent in FP32)
SUMMED = {"g_pyr", "g_uvattr", "g_clip", "g_clip_aa", "g_pos", "g_axis", "g_sharp", "g_amp",
          # COMPAT indexes the specular sharpness gradient by lobe (material.cu:436): lobe sums,
          # and the roughness gradient of those entries reads them
          "g_ssh", "g_rough"}


def measure(a, b):
    """(normwise error, worst element-wise error, flat index of that element)."""
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    scale = np.abs(b).max(initial=0.0)
    if scale == 0.0:
        return float(np.abs(a).max(initial=0.0)), 0.0, -1
    d = np.abs(a - b)
    norm = float(d.max() / scale)
    sel = np.abs(b) > ELEM_FLOOR * scale
    if not sel.any():
        return norm, 0.0, -1
    rel = np.zeros_like(d)
    rel[sel] = d[sel] / np.abs(b[sel])
    i = int(np.argmax(rel))
    return norm, float(rel[i]), i


def elem_tol(key):
    return ELEM_TOL_SUM if key in SUMMED else ELEM_TOL


def check_keys(got, want, keys, label=""):
    """Measure every key; returns {key: (norm, elem, index)} and the list of
    keys that miss a bar."""
    res, bad = {}, []
    for k in keys:
        n, e, i = measure(got[k], want[k])
        res[k] = (n, e, i)
        if n > NORM_TOL or e > elem_tol(k):
            bad.append((k, n, e, i))
    report(label, res)
    return res, bad


def report(label, res):
    path = os.environ.get("VCL_PARITY_REPORT")
    if not path:
        return
    with open(path, "a") as f:
        f.write(json.dumps({"case": label, "keys": {k: {"norm": v[0], "elem": v[1], "at": v[2]}
                                                   for k, v in res.items()}}) + "\n")

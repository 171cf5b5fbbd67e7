"""Parity measures shared by the GPU tests.

Triangle ids, barycentrics, depth and DB are compared bit for bit.  Every
other output b of the FP32 oracle (the C restatement of the reference's
arithmetic) and the CUDA path's a for the same stage inputs are held to:

* normwise: max|a - b| / max|b| <= 1e-5 (the FP32 bar);
* element-wise, against the exact stage value t (the same restatement in
  double precision fed the same FP32 inputs, chain.run_isolated64), on every
  entry with |t| above 1e-3 of the array's largest magnitude: the root mean
  square of |a - t| / |t| must not exceed max(1e-5, 2 x that of
  |b - t| / |t|), and the worst element max(1e-5, 4 x b's worst).  That
  is, element by element the CUDA path is as close to the exact value as
  the reference's own FP32 arithmetic, and within 1e-5 wherever that
  arithmetic is.  (Which single element rounds worst is random on both
  sides -- for a sum over pixels it depends on the order of the additions
  -- so the worst elements get the wider factor and the mean square the
  tighter one.)  A plain element-wise
  1e-5 against b cannot be the bar: b itself misses the exact value by up
  to ~1e-4 on small components of unit vectors and near-cancelling terms
  (a 1-ulp difference in a dot product evaluated with or without fused
  multiply-adds is 6e-8 absolute, i.e. 6e-5 relative on a component of
  1e-3), and the antialias terms (alpha = a / (D +- 1e-3) - 1/2) by more.
  Sums over pixels (texel, vertex and lobe gradients) are order-dependent in
  FP32 on both sides; the oracle accumulates the lobe sums in double.

`report()` appends one JSON line per check to the file named by the
VCL_PARITY_REPORT environment variable (when set), so a run keeps the worst
element per key.
"""
import json
import os

import numpy as np

NORM_TOL = 1e-5
ELEM_TOL = 1e-5
ELEM_FLOOR = 1e-3


def elem_rms(a, b):
    """Root mean square of the element-wise relative error over the entries
    above the floor."""
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    scale = np.abs(b).max(initial=0.0)
    sel = np.abs(b) > ELEM_FLOOR * scale
    if scale == 0.0 or not sel.any():
        return 0.0
    return float(np.sqrt(np.mean((np.abs(a[sel] - b[sel]) / np.abs(b[sel])) ** 2)))


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


def check_keys(got, want, exact, keys, label=""):
    """Measures every key against the FP32 oracle (`want`) and the exact
    stage values (`exact`); returns {key: measures} and the keys that miss a
    bar (see the module docstring)."""
    res, bad = {}, []
    for k in keys:
        n32, e32, i32 = measure(got[k], want[k])
        ng, eg, ig = measure(got[k], exact[k])
        no, eo, _ = measure(want[k], exact[k])
        qg, qo = elem_rms(got[k], exact[k]), elem_rms(want[k], exact[k])
        res[k] = {"norm": n32, "elem": e32, "at": i32, "elem_vs_exact": eg, "at_exact": ig,
                  "oracle_elem_vs_exact": eo, "norm_vs_exact": ng, "oracle_norm_vs_exact": no,
                  "rms_vs_exact": qg, "oracle_rms_vs_exact": qo}
        norm_ok = n32 <= NORM_TOL or ng <= max(NORM_TOL, 2.0 * no)
        elem_ok = qg <= max(ELEM_TOL, 2.0 * qo) and eg <= max(ELEM_TOL, 4.0 * eo)
        if not (norm_ok and elem_ok):
            bad.append((k, res[k]))
    report(label, res)
    return res, bad


def report(label, res):
    path = os.environ.get("VCL_PARITY_REPORT")
    if not path:
        return
    out = {k: (v if isinstance(v, dict) else {"norm": v[0], "elem": v[1], "at": v[2]}) for k, v in res.items()}
    with open(path, "a") as f:
        f.write(json.dumps({"case": label, "keys": out}) + "\n")

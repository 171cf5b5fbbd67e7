"""Host-side pieces of bench.py, on the CPU: the reference arm's stepper
(the reference's kernels compiled for the host, one view per step) and the
shared config object of the two arms."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from vcl_b200 import scenes  # noqa: E402


def test_reference_stepper_covers_one_iteration_in_views_steps():
    S = scenes.small(seed=4, W=40, H=32, views=3, subdiv=2, tex=32, K=5)
    rs = bench.RefStepper(S, threads=2)
    try:
        tex0, pos0, lobes0 = rs.pyr[: S.tex_w * S.tex_h * S.C].copy(), rs.pos.copy(), rs.lobes.copy()
        n0 = S.tex_w * S.tex_h * S.C
        rs.step()
        # the first step's texture Adam touches the first third of level 0 only
        # (texels the view does not sample have a zero gradient and stay put)
        moved = np.abs(rs.pyr[:n0] - tex0) > 0
        assert not moved[n0 // 3:].any()
        assert np.array_equal(rs.pos, pos0) and np.array_equal(rs.lobes, lobes0)
        rs.step()
        rs.step()
        # after V steps the whole iteration's parameter work has run: texels
        # of the other slices, the positions and the lobes have moved
        moved = np.abs(rs.pyr[:n0] - tex0) > 0
        assert moved[n0 // 3:].any()
        assert not np.array_equal(rs.pos, pos0) and not np.array_equal(rs.lobes, lobes0)
        assert rs.s == 3
        assert np.isfinite(rs.pyr).all()
    finally:
        rs.close()


def test_both_arms_share_the_config_object():
    S = scenes.config2(views=16)
    c = bench.bench_config(S, 1)
    assert c["global_batch"] == 16 and "strategy" not in c
    assert c["workload"].startswith("fit iteration: uvs256x128-1024x16-tex2048-K32")
    assert bench.METRIC.startswith("fwd+bwd+Adam iters/s")

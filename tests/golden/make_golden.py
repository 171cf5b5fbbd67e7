"""Generate the golden fixtures from the REFERENCE's own kernels.

Runs one fit iteration (forward, backward, one Adam step) of two tiny seeded
scenes through ``oracle/_ref/libvclref.so`` -- the reference's
nvdiffrast/nvdiffrast/*.cu compiled unmodified as host C++ by
``make -C oracle ref`` -- and stores inputs and outputs as .npz.  The raster
input is the C restatement's (the reference rasterizes through OpenGL, which
cannot run here), and is stored in the fixture so the fixture stands alone.

Usage:  python tests/golden/make_golden.py      (needs the reference sources)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402
from vcl_b200 import scenes  # noqa: E402
import chain  # noqa: E402

SCENE_KEYS = ["pos", "tri", "uv", "normal", "tex_target", "lobe_axis_init", "lobe_sharp_init",
              "lobe_amp_init", "mvp", "pvinv", "rot"]
SCENE_INTS = ["W", "H", "views", "tex_w", "tex_h", "C", "levels", "K", "seed"]
SCENE_FLOATS = ["roughness", "ior", "lr"]


def cases():
    return {
        "tiny_a": scenes.small(seed=1),
        "tiny_b": scenes.small(seed=2, W=64, H=48, views=3, subdiv=2, tex=64, K=5),
    }


def main():
    ref = O.ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libvclref.so missing: run `make -C oracle ref` first")
    for name, S in cases().items():
        pyr = chain.build_pyramid(S, S.tex_target)
        a = chain.run_chain(O.orc(), S, 0, pyr=pyr.copy())
        r = chain.run_chain(ref, S, 0, rast=a["rast"], db=a["db"], pyr=pyr.copy())
        out = {f"scene_{k}": getattr(S, k) for k in SCENE_KEYS}
        out.update({f"scene_{k}": np.int64(getattr(S, k)) for k in SCENE_INTS})
        out.update({f"scene_{k}": np.float64(getattr(S, k)) for k in SCENE_FLOATS})
        for k, v in r.items():
            out[f"ref_{k}"] = np.asarray(v)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "written")


if __name__ == "__main__":
    main()

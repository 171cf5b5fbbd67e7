"""The header-only C++ layer (include/vcl.hpp) compiles against vcl.h with
-Wall -Wextra -Werror and runs: RAII owners and vcl::Error on the device-free
paths (OBJ / BMP loading, a failed load), and a Context that either opens a
device or reports the failure as an exception.  Host code only."""
import os
import shutil
import struct
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "vcl_b200", "libvcl.so")

PROGRAM = r"""
#include "vcl.hpp"
#include <cstdio>
int main(int, char** argv) {
    vcl::Obj o(argv[1]);
    const auto c = o.counts();
    std::printf("obj %d %d %d %d %d\n", c.pos, c.tri, c.texel, c.normal, c.welded);
    const float *pos, *uv, *nrm;
    const uint32_t* tri;
    o.welded(&pos, &uv, &nrm, &tri);
    std::printf("tri %u %u %u %u %u %u\n", tri[0], tri[1], tri[2], tri[3], tri[4], tri[5]);
    int w = 0, h = 0, ch = 0;
    const auto px = vcl::load_bmp(argv[2], w, h, ch);
    std::printf("bmp %d %d %d %.4f\n", w, h, ch, px[0]);
    try {
        vcl::Obj bad(argv[3]);
        std::printf("no error\n");
    } catch (const vcl::Error& e) {
        std::printf("error %d\n", e.status());
    }
    vcl::Obj moved = std::move(o);
    std::printf("moved %d\n", moved.counts().tri);
    try {
        vcl::Context ctx(0, VCL_MODE_EXACT);
        std::printf("device mode %d\n", ctx.mode());
    } catch (const vcl::Error& e) {
        std::printf("no device %d\n", e.status());
    }
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
@pytest.mark.skipif(not os.path.exists(LIB), reason="libvcl.so not built")
def test_cpp_layer_compiles_and_runs(tmp_path):
    src = tmp_path / "use_vcl.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "use_vcl"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", os.path.dirname(LIB), "-lvcl", "-Wl,-rpath," + os.path.dirname(LIB)],
                   check=True)
    obj = tmp_path / "quad.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvt 1 1\nf 1/1 2/1 3/2\nf 1/1 3/1 4/1\n")
    bmp = tmp_path / "px.bmp"
    row = bytes([10, 20, 30, 0])                           # one 24-bit pixel (BGR) + padding
    info = struct.pack("<IiiHHIIiiII", 40, 1, 1, 1, 24, 0, len(row), 0, 0, 0, 0)
    bmp.write_bytes(b"BM" + struct.pack("<IHHI", 54 + len(row), 0, 0, 54) + info + row)
    out = subprocess.run([str(exe), str(obj), str(bmp), str(tmp_path / "missing.obj")], check=True,
                         capture_output=True, text=True).stdout.splitlines()
    assert out[0] == "obj 4 2 2 0 5"          # vertex 3 carries a second texel: welded into 5
    assert out[1] == "tri 0 1 2 0 3 4"
    assert out[2] == "bmp 1 1 3 %.4f" % (30 / 255.0)   # channels in reverse byte order: R first
    assert out[3] == "error 1"
    assert out[4] == "moved 2"
    assert out[5] in ("device mode 1", "no device 2"), out[5]

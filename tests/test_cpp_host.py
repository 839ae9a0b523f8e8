"""The C++ host header (include/depth_cuda.hpp, the MetalStereo interface over the C ABI): it compiles and
links against libdepth_cuda.so here; on the GPU a C++ program drives it like a frontend and must produce
the golden disparity bit for bit and the reference's error codes."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "cuda_stereo_test.cpp")


def _compile(tmp_path):
    from open_source_einstar_b200.build import LIB
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    exe = str(tmp_path / "cuda_stereo_test")
    cmd = ["g++", "-std=c++23", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", os.path.dirname(LIB), "-ldepth_cuda", f"-Wl,-rpath,{os.path.dirname(LIB)}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_header_compiles_and_links(tmp_path):
    _compile(tmp_path)


@pytest.mark.gpu
def test_cpp_frontend_matches_golden(cuda, golden, tmp_path):
    exe = _compile(tmp_path)
    c = golden["plane_sphere_160x128"]
    p = c["params"]
    h, w = c["shape"]
    path = tmp_path / "case.bin"
    with open(path, "wb") as f:
        f.write(np.array([w, h, p["min_disparity"], p["num_disparities"], int(c["subpixel"]), 1], np.int32).tobytes())
        f.write(np.ascontiguousarray(c["left"], np.uint8).tobytes())
        f.write(np.ascontiguousarray(c["right"], np.uint8).tobytes())
        f.write(np.ascontiguousarray(c["median"], np.float32).tobytes())
    r = subprocess.run([exe, str(path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr

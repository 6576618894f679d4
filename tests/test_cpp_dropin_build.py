"""The C++ drop-in header compiles and links as reference call sites use it
(CPU: g++ only, nothing runs).  The GPU tests run the same programs."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "real-time-depth-fusion-directional-tsdf_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.mark.parametrize("prog,defs", [("dropin_frames.cpp", []), ("dropin_frames.cpp", ["-DUSE_NORMAL_DIR_ALLOC"]),
                                       ("splat_cloud.cpp", [])])
def test_cpp_programs_compile_and_link(tmp_path, prog, defs):
    if not os.path.exists(os.path.join(PKG, "libvsg.so")):
        pytest.skip("libvsg.so not built")
    exe = str(tmp_path / "prog")
    r = subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-Wextra", "-Werror", *defs, "-o", exe,
                        os.path.join(ROOT, "tests", "cpp", prog), "-I", os.path.join(ROOT, "include"),
                        "-I", f"{CUDA}/include", "-L", PKG, "-lvsg", f"-Wl,-rpath,{PKG}", "-L", f"{CUDA}/lib64",
                        "-lcudart"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    assert os.path.exists(exe)

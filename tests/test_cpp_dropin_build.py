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


def build_device_guard(out_dir) -> str:
    """nvcc build of tests/cpp/device_guard.cu (it reads the handles' recorded
    device through the library's internal header)."""
    exe = os.path.join(str(out_dir), "device_guard")
    r = subprocess.run([os.path.join(CUDA, "bin", "nvcc"), "-O1", "-std=c++17", "-gencode",
                        "arch=compute_100a,code=sm_100a", "-o", exe, os.path.join(ROOT, "tests", "cpp", "device_guard.cu"),
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc"), "-L", PKG, "-lvsg",
                        f"-Xlinker=-rpath,{PKG}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_device_guard_program_compiles(tmp_path):
    if not os.path.exists(os.path.join(PKG, "libvsg.so")):
        pytest.skip("libvsg.so not built")
    assert os.path.exists(build_device_guard(tmp_path))

"""Recipe: compile the reference's own CUDA kernels for sm_100a into
oracle/_ref/ -- TEST INFRASTRUCTURE ONLY (the checker; never the product).

Compiles, from their own source tree (VoxelSG/src under the reference
checkout), VoxelScene.cu, RayCastRender.cu, CUDAHashRef.cu and
MarchingCubes.cu with oracle/ref_shim.cu and a two-line OpenCV stand-in
(oracle/ref_stub) into

  oracle/_ref/libvsgref.so        nvcc defaults (FMA contraction on), as the
                                  reference's own build would compile them
  oracle/_ref/libvsgref_nofma.so  -fmad=false: each operation rounded on its
                                  own, the semantics the oracle restates

Nothing is copied out of the reference tree; the reference build system is
not used.  Skipped when the reference checkout is absent (a machine without
it uses the files built here).  The checkout is found at $VSG_REFERENCE_ROOT,
else at its default location.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference checkout: $VSG_REFERENCE_ROOT, else its default location here
REF_ROOT = os.environ.get("VSG_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "VoxelSG", "src")
REF_INC = os.path.join(REF_ROOT, "VoxelSG", "include")
SOURCES = ["VoxelScene.cu", "RayCastRender.cu", "CUDAHashRef.cu", "MarchingCubes.cu"]
VARIANTS = {"libvsgref.so": [], "libvsgref_nofma.so": ["-fmad=false"]}


def available() -> bool:
    return all(os.path.exists(os.path.join(REF_SRC, f)) for f in SOURCES)


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build_if_available(force: bool = False) -> list[str]:
    if not available():
        return []
    os.makedirs(OUT, exist_ok=True)
    srcs = [os.path.join(REF_SRC, f) for f in SOURCES] + [os.path.join(HERE, "ref_shim.cu")]
    built = []
    for lib, extra in VARIANTS.items():
        out = os.path.join(OUT, lib)
        if force or _stale(out, srcs):
            cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", *extra,
                   "-Xcompiler", "-fPIC", "-shared", "-include", "cstdint", "-I", os.path.join(HERE, "ref_stub"),
                   "-I", REF_INC, "-o", out, *srcs]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("reference kernel build failed")
        built.append(out)
    return built


if __name__ == "__main__":
    print(build_if_available(force="--force" in sys.argv))

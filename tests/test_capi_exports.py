"""The C-ABI library loads and exports every function include/vsg.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "vsg.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*VSG_API\s+(?:const\s+)?\w+\s*\**\s*(vsg_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "vsg_integrate" in names and "vsg_render" in names and len(names) >= 15


def test_library_exports_all_declared_symbols():
    import build
    import vsg

    build.build()
    lib = ctypes.CDLL(vsg.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(vsg.EXPORTS) == declared_functions()


def test_version_string_without_gpu():
    import vsg

    assert vsg.version().startswith("vsg-b200")


def test_invalid_arguments_are_rejected_without_gpu():
    import vsg

    L = vsg.lib()
    assert L.vsg_scene_create(None, None) == 1
    assert L.vsg_scene_destroy(None) == 1
    assert L.vsg_integrate(None, None, None, None, 0, 0, 0.0, None, 0.0, 0.0, 0.0, 0.0, None) == 2
    assert L.vsg_render(None, None, None, None, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, None) == 2
    assert L.vsg_renderer_create(0, 10, ctypes.byref(ctypes.c_void_p())) == 1
    p = vsg.Params()
    assert L.vsg_params_default(ctypes.byref(p)) == 0
    p.voxel_size = 0.0
    h = ctypes.c_void_p()
    assert L.vsg_scene_create(ctypes.byref(p), ctypes.byref(h)) == 1

"""ctypes wrapper of the reference kernels built by ref_build.py --
TEST INFRASTRUCTURE ONLY (used by the tests and the golden-vector script)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_P, _F, _I = ctypes.c_void_p, ctypes.c_float, ctypes.c_int


def lib_path(nofma: bool = True) -> str:
    return os.path.join(HERE, "_ref", "libvsgref_nofma.so" if nofma else "libvsgref.so")


def available(nofma: bool = True) -> bool:
    return os.path.exists(lib_path(nofma))


_libs = {}


def lib(nofma: bool = True):
    if nofma not in _libs:
        L = ctypes.CDLL(lib_path(nofma))
        L.ref_create.restype = _P
        L.ref_create.argtypes = [_I, _I, _F, _F, _F]
        L.ref_destroy.argtypes = [_P]
        L.ref_integrate.restype = _I
        L.ref_integrate.argtypes = [_P, _P, _P, _P, _I, _I, _F, _P, _F, _F, _F, _F]
        L.ref_render.restype = _I
        L.ref_render.argtypes = [_P, _I, _I, _P, _F, _F, _F, _F, _F, _F, _P, _P, _P, _P]
        L.ref_export.restype = _I
        L.ref_export.argtypes = [_P, _P, _P, _I]
        L.ref_voxel_bytes.restype = _I
        L.ref_integrate_dev.restype = _F
        L.ref_integrate_dev.argtypes = [_P, _P, _P, _P, _I, _I, _F, _P, _P, _F, _F, _F, _F]
        L.ref_extract_points.restype = _I
        L.ref_extract_points.argtypes = [_P, _F, _F, ctypes.c_uint, _I, _P, _P, _P]
        L.ref_integrate_m2.restype = _I
        L.ref_integrate_m2.argtypes = L.ref_integrate.argtypes
        L.ref_render_dev.restype = _F
        L.ref_render_dev.argtypes = [_P, _I, _I, _P, _P, _F, _F, _F, _F, _F, _F, _P, _P, _P, _P]
        _libs[nofma] = L
    return _libs[nofma]


class RefScene:
    """The reference's VoxelScene data + launchers on the current GPU."""

    def __init__(self, slots: int, blocks: int, voxel: float, trunc: float, trunc_scale: float = 0.01,
                 nofma: bool = True):
        self.L = lib(nofma)
        self.h = self.L.ref_create(slots, blocks, _F(voxel), _F(trunc), _F(trunc_scale))
        self.blocks = blocks

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def integrate(self, pm_dev, rgb_dev, nm_dev, W, H, trunc, pose, fx, fy, cx, cy, method: int = 1):
        """method 2: the normal-direction allocation (USE_NORMAL_DIR_ALLOC)."""
        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        fn = self.L.ref_integrate_m2 if method == 2 else self.L.ref_integrate
        rc = fn(self.h, pm_dev, rgb_dev, nm_dev, W, H, _F(trunc), T.ctypes.data, _F(fx), _F(fy), _F(cx), _F(cy))
        assert rc == 0, rc

    def render(self, W, H, pose, fx, fy, cx, cy, min_d, max_d, fill=1e10):
        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        d = np.full((H, W), fill, np.float32)
        p = np.full((H, W, 4), fill, np.float32)
        c = np.full((H, W, 4), fill, np.float32)
        n = np.full((H, W, 4), fill, np.float32)
        rc = self.L.ref_render(self.h, W, H, T.ctypes.data, _F(fx), _F(fy), _F(cx), _F(cy), _F(min_d), _F(max_d),
                               d.ctypes.data, p.ctypes.data, c.ctypes.data, n.ctypes.data)
        assert rc == 0, rc
        return {"depth": d, "position": p, "color": c, "normal": n}

    def extract_points(self, min_sdf, max_sdf, min_weight, max_points=2_000_000):
        """The reference's extractSurfacePointsCUDA: (positions, colours,
        normals) (n, 4) float32 in its output order, and its count."""
        p = np.zeros((max_points, 4), np.float32)
        c = np.zeros((max_points, 4), np.float32)
        n = np.zeros((max_points, 4), np.float32)
        cnt = self.L.ref_extract_points(self.h, _F(min_sdf), _F(max_sdf), int(min_weight), max_points,
                                        p.ctypes.data, c.ctypes.data, n.ctypes.data)
        assert cnt >= 0, cnt
        k = min(cnt, max_points)
        return p[:k], c[:k], n[:k], cnt

    def export(self):
        """(coords (n,3) int32 sorted by x,y,z; voxel bytes (n, 4096) uint8)."""
        coords = np.zeros((self.blocks, 3), np.int32)
        vox = np.zeros((self.blocks, 4096), np.uint8)
        n = self.L.ref_export(self.h, coords.ctypes.data, vox.ctypes.data, self.blocks)
        assert n >= 0
        coords, vox = coords[:n], vox[:n]
        order = np.lexsort((coords[:, 2], coords[:, 1], coords[:, 0]))
        return coords[order], vox[order]

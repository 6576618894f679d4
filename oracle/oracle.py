"""ctypes wrapper of the CPU oracle (vsg_oracle.c) -- TEST INFRASTRUCTURE ONLY.

Imported by the tests, the smoke check and the CPU-baseline leg of the
benchmark as the checker.  The product path never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_vsg.so")

_f = ctypes.c_float
_i = ctypes.c_int
_i64 = ctypes.c_int64
_p = ctypes.c_void_p


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "vsg_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
               "-Wall", "-o", LIB_PATH, src, "-lm"]
        subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = _p
        L.orc_create.argtypes = [_f]
        L.orc_destroy.argtypes = [_p]
        L.orc_reset.argtypes = [_p]
        L.orc_num_blocks.restype = _i64
        L.orc_num_blocks.argtypes = [_p]
        L.orc_coord_range_drops.restype = _i64
        L.orc_coord_range_drops.argtypes = [_p]
        L.orc_dda_blocks.restype = _i
        L.orc_dda_blocks.argtypes = [_p, _p, _f, _p]
        L.orc_alloc.restype = _i64
        L.orc_alloc.argtypes = [_p, _p, _i, _i, _f, _p, _p]
        L.orc_integrate_blocks.argtypes = [_p, _p, _p, _i, _i, _f, _p, _p, _f, _f, _f, _f, _p]
        L.orc_integrate.argtypes = [_p, _p, _p, _i, _i, _f, _p, _f, _f, _f, _f, _p]
        L.orc_integrate_nm.argtypes = [_p, _p, _p, _p, _i, _i, _f, _p, _f, _f, _f, _f, _p]
        L.orc_set_alloc_method.argtypes = [_p, _i]
        L.orc_export_parents.argtypes = [_p, _p]
        L.orc_splat_points.argtypes = [_p, _i64, _p, _i64, _p, _i64, _i, _i, _f, _f, _f, _f, _f, _f, _i, _p, _p,
                                       _p, _p]
        L.orc_render.argtypes = [_p, _i, _i, _p, _p, _f, _f, _f, _f, _f, _f, _p, _p, _p, _p, _p]
        L.orc_render_rows.argtypes = [_p, _i, _i, _i, _i, _p, _p, _f, _f, _f, _f, _f, _f, _p, _p, _p,
                                      _p, _p]
        L.orc_render_touched_blocks.restype = _i64
        L.orc_render_touched_blocks.argtypes = [_p, _i, _i, _p, _p, _f, _f, _f, _f, _f, _f]
        L.orc_marching_cubes.restype = _i64
        L.orc_marching_cubes.argtypes = [_p, _p, _f, _f, _i64, _p, _p]
        L.orc_render_brackets.argtypes = [_p, _i, _i, _p, _p, _f, _f, _f, _f, _f, _f, _p]
        L.orc_extract_points.restype = _i64
        L.orc_extract_points.argtypes = [_p, _f, _f, ctypes.c_uint32, _i64, _p, _p, _p]
        L.orc_stream_out.restype = _i64
        L.orc_stream_out.argtypes = [_p, _p, _f, _p, _p]
        L.orc_stream_in.argtypes = [_p, _i64, _p, _p]
        L.orc_merge_voxels.argtypes = [_i64, _p, _p, _p]
        L.orc_export.argtypes = [_p, _p, _p]
        L.orc_import.argtypes = [_p, _i64, _p, _p]
        L.orc_bucket_hash.restype = ctypes.c_uint32
        L.orc_bucket_hash.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32]
        L.orc_max_threads.restype = _i
        L.orc_set_threads.argtypes = [_i]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_p)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class OracleScene:
    """CPU TSDF scene with reference semantics (ideal allocation)."""

    def __init__(self, voxel_size: float):
        self.L = lib()
        self.h = self.L.orc_create(_f(voxel_size))
        self.voxel = voxel_size

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def reset(self):
        self.L.orc_reset(self.h)

    @property
    def num_blocks(self) -> int:
        return int(self.L.orc_num_blocks(self.h))

    def set_alloc_method(self, method: int):
        """1: camera-z band (allocBlocksFromDepthMapMethod1Kernel); 2: camera
        and normal rays with parent pixels (Method2, VoxelScene.cu:768-912)."""
        self.L.orc_set_alloc_method(self.h, int(method))

    def integrate(self, pointmap, rgb, trunc, pose, fx, fy, cx, cy, normals=None) -> dict:
        pm = _f32(pointmap)
        cm = np.ascontiguousarray(rgb, dtype=np.uint8)
        nm = _f32(normals) if normals is not None else None
        T = _f32(pose).reshape(16)
        H, W = pm.shape[:2]
        out = np.zeros(4, np.int64)
        self.L.orc_integrate_nm(self.h, _ptr(pm), _ptr(cm), _ptr(nm) if nm is not None else None, W, H,
                                _f(trunc), _ptr(T), _f(fx), _f(fy), _f(cx), _f(cy), _ptr(out))
        return {"new_blocks": int(out[0]), "updated_blocks": int(out[1]), "updated_voxels": int(out[2]),
                "blocks": int(out[3])}

    def alloc(self, pointmap, trunc, pose) -> int:
        pm = _f32(pointmap)
        T = _f32(pose).reshape(16)
        cam = np.array([T[3], T[7], T[11]], np.float32)
        H, W = pm.shape[:2]
        return int(self.L.orc_alloc(self.h, _ptr(pm), W, H, _f(trunc), _ptr(T), _ptr(cam)))

    def render(self, W, H, pose, fx, fy, cx, cy, min_depth, max_depth, cam=None, rows=None) -> dict:
        T = _f32(pose).reshape(16)
        cam = np.array([T[3], T[7], T[11]], np.float32) if cam is None else _f32(cam)
        depth = np.full((H, W), 1e10, np.float32)
        pos = np.full((H, W, 4), 1e10, np.float32)
        col = np.full((H, W, 4), 1e10, np.float32)
        nrm = np.full((H, W, 4), 1e10, np.float32)
        st = np.zeros(3, np.int64)
        if rows is None:
            self.L.orc_render(self.h, W, H, _ptr(cam), _ptr(T), _f(fx), _f(fy), _f(cx), _f(cy),
                              _f(min_depth), _f(max_depth), _ptr(depth), _ptr(pos), _ptr(col), _ptr(nrm),
                              _ptr(st))
        else:
            self.L.orc_render_rows(self.h, W, H, rows[0], rows[1], _ptr(cam), _ptr(T), _f(fx), _f(fy),
                                   _f(cx), _f(cy), _f(min_depth), _f(max_depth), _ptr(depth), _ptr(pos),
                                   _ptr(col), _ptr(nrm), _ptr(st))
        return {"depth": depth, "position": pos, "color": col, "normal": nrm, "hits": int(st[0]),
                "misses": int(st[1]), "samples": int(st[2])}

    def brackets(self, W, H, pose, fx, fy, cx, cy, min_depth, max_depth) -> np.ndarray:
        """(H, W, 2) float32: the march bracket of each hit pixel's crossing."""
        T = _f32(pose).reshape(16)
        cam = np.array([T[3], T[7], T[11]], np.float32)
        out = np.full((H, W, 2), np.nan, np.float32)
        self.L.orc_render_brackets(self.h, W, H, _ptr(cam), _ptr(T), _f(fx), _f(fy), _f(cx), _f(cy),
                                   _f(min_depth), _f(max_depth), _ptr(out))
        return out

    def touched_blocks(self, W, H, pose, fx, fy, cx, cy, min_depth, max_depth) -> int:
        T = _f32(pose).reshape(16)
        cam = np.array([T[3], T[7], T[11]], np.float32)
        return int(self.L.orc_render_touched_blocks(self.h, W, H, _ptr(cam), _ptr(T), _f(fx), _f(fy),
                                                    _f(cx), _f(cy), _f(min_depth), _f(max_depth)))

    def marching_cubes(self, table, iso: float, voxel: float, max_tris: int):
        """Triangle soup of MarchingCubes.cu:354-467 with the given 256x16 case
        table: (total count, vertices (m,3,3) f32, normals (m,3,3) f32),
        m = min(total, max_tris)."""
        tab = np.ascontiguousarray(table, dtype=np.uint8).reshape(256, 16)
        v = np.zeros((max(max_tris, 1), 3, 3), np.float32)
        n = np.zeros((max(max_tris, 1), 3, 3), np.float32)
        total = int(self.L.orc_marching_cubes(self.h, _ptr(tab), _f(iso), _f(voxel), int(max_tris), _ptr(v),
                                              _ptr(n)))
        m = min(total, max_tris)
        return total, v[:m].copy(), n[:m].copy()

    def extract_points(self, min_sdf: float, max_sdf: float, min_weight: int, max_points: int):
        """kernelExtractSurfacePoints (RayCastRender.cu:683-868): (total count,
        positions (m,4), colours (m,4), normals (m,4)), m = min(total, max)."""
        m = max(int(max_points), 1)
        P = np.zeros((m, 4), np.float32)
        C = np.zeros((m, 4), np.float32)
        N = np.zeros((m, 4), np.float32)
        total = int(self.L.orc_extract_points(self.h, _f(min_sdf), _f(max_sdf), int(min_weight), int(max_points),
                                              _ptr(P), _ptr(C), _ptr(N)))
        k = min(total, int(max_points))
        return total, P[:k].copy(), C[:k].copy(), N[:k].copy()

    def stream_out(self, center, radius: float):
        """Remove the blocks whose corner is >= radius from center:
        (coords (m,3) int32 sorted, voxel bytes (m, 4096) uint8)."""
        n = self.num_blocks
        c = _f32(center)
        coords = np.zeros((max(n, 1), 3), np.int32)
        vox = np.zeros((max(n, 1), 512 * 8), np.uint8)
        m = int(self.L.orc_stream_out(self.h, _ptr(c), _f(radius), _ptr(coords), _ptr(vox)))
        order = np.lexsort((coords[:m, 2], coords[:m, 1], coords[:m, 0]))
        return coords[:m][order].copy(), vox[:m][order].copy()

    def stream_in(self, coords, voxel_bytes):
        coords = np.ascontiguousarray(coords, dtype=np.int32)
        vb = np.ascontiguousarray(voxel_bytes, dtype=np.uint8)
        self.L.orc_stream_in(self.h, coords.shape[0], _ptr(coords), _ptr(vb))

    def export(self, with_voxels: bool = True):
        """(coords (n,3) int32 sorted by x,y,z; voxels (n,512) structured)."""
        n = self.num_blocks
        coords = np.zeros((n, 3), np.int32)
        vox = np.zeros((n, 512 * 8), np.uint8) if with_voxels else None
        self.L.orc_export(self.h, _ptr(coords), _ptr(vox) if with_voxels else None)
        return coords, (split_voxels(vox) if with_voxels else None)

    def export_parents(self):
        """Per block in export() order: the parent tag of the normal-direction
        allocation, (frame + 1) << 32 | y << 16 | x, 0 = none."""
        out = np.zeros(self.num_blocks, np.uint64)
        self.L.orc_export_parents(self.h, _ptr(out))
        return out

    def load(self, coords, voxel_bytes):
        coords = np.ascontiguousarray(coords, dtype=np.int32)
        vb = np.ascontiguousarray(voxel_bytes, dtype=np.uint8)
        self.L.orc_import(self.h, coords.shape[0], _ptr(coords), _ptr(vb))


def split_voxels(vox_bytes: np.ndarray) -> dict:
    """(n, 4096) raw bytes -> dict of sdf (n,512) f32, rgb (n,512,3) u8, weight (n,512) u8."""
    v = vox_bytes.reshape(-1, 512, 8)
    sdf = np.ascontiguousarray(v[:, :, :4]).view(np.float32).reshape(-1, 512)
    return {"sdf": sdf, "rgb": v[:, :, 4:7].copy(), "weight": v[:, :, 7].copy(), "raw": vox_bytes}


def merge_voxels(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Voxel-by-voxel weighted merge of two blocks' 8-byte voxel records."""
    a = np.ascontiguousarray(a, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.uint8)
    out = np.zeros_like(a)
    lib().orc_merge_voxels(a.size // 8, _ptr(a), _ptr(b), _ptr(out))
    return out


class ChunkStore:
    """Host chunk grid of streamed-out blocks, restating VoxelStreamingManager
    (VoxelStreamingManager.cpp:836-1140) in FP32: a block is filed under the
    chunk of its corner (worldToChunks, :905-922); stream-in takes every
    stored chunk in the box of ceil(r / extent) chunks around the centre's
    chunk that passes isChunkInSphere (:962-991).  A block stored twice is
    merged (merge_voxels)."""

    def __init__(self, voxel: float, extent=(1.0, 1.0, 1.0)):
        self.v = np.float32(voxel)
        self.ext = [np.float32(e) for e in extent]
        self.chunks = {}  # chunk -> {block coord: voxel bytes}

    def chunk_of_world(self, p):
        out = []
        for i in range(3):
            q = np.float32(np.float32(p[i]) / self.ext[i])
            sg = np.float32(1.0) if q > 0 else (np.float32(-1.0) if q < 0 else np.float32(0.0))
            out.append(int(np.float32(q + np.float32(sg * np.float32(0.5)))))  # truncation toward zero
        return tuple(out)

    def chunk_of_block(self, b):
        return self.chunk_of_world([np.float32(np.float32(int(b[i]) * 8) * self.v) for i in range(3)])

    def add(self, coords, vox):
        for c, v in zip(coords, vox):
            ch = self.chunks.setdefault(self.chunk_of_block(c), {})
            k = tuple(int(x) for x in c)
            ch[k] = merge_voxels(ch[k], v) if k in ch else np.array(v, np.uint8)

    def in_sphere(self, c, center, radius):
        f32 = np.float32
        w = [f32(f32(c[i]) * self.ext[i]) for i in range(3)]
        ce = max(self.ext)
        cr = f32(f32(f32(0.5) * ce) * f32(np.sqrt(f32(3.0))))
        d = [f32(w[i] - f32(center[i])) for i in range(3)]
        dist = f32(np.sqrt(f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))))
        return bool(f32(dist - cr) <= f32(radius))

    def take(self, center, radius):
        """Remove and return (coords, voxels) of the chunks a stream-in takes."""
        if radius < 0:
            keys = sorted(self.chunks)
        else:
            cc = self.chunk_of_world(center)
            cr = [int(np.ceil(np.float32(np.float32(radius) / self.ext[i]))) for i in range(3)]
            keys = sorted(k for k in self.chunks
                          if all(abs(k[i] - cc[i]) <= cr[i] for i in range(3)) and self.in_sphere(k, center, radius))
        coords, vox = [], []
        for k in keys:
            for c, v in self.chunks.pop(k).items():
                coords.append(c)
                vox.append(v)
        return (np.array(coords, np.int32).reshape(-1, 3), np.array(vox, np.uint8).reshape(-1, 4096))

    def export(self):
        items = sorted((c, v) for ch in self.chunks.values() for c, v in ch.items())
        return (np.array([c for c, _ in items], np.int32).reshape(-1, 3),
                np.array([v for _, v in items], np.uint8).reshape(-1, 4096))


def dda_blocks(start, end, voxel) -> np.ndarray:
    s = _f32(start)
    e = _f32(end)
    out = np.zeros((1024, 3), np.int32)
    n = lib().orc_dda_blocks(_ptr(s), _ptr(e), _f(voxel), _ptr(out))
    return out[:n].copy()


def bucket_hash(x, y, z, num_buckets) -> int:
    return int(lib().orc_bucket_hash(int(x), int(y), int(z), int(num_buckets)))


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def splat_points(points, width, height, fx, fy, cx, cy, normals=None, colors=None, mode=0, min_depth=0.0,
                 max_depth=float("inf")) -> dict:
    """CustomDepthMapGenerator::generateFromPointCloud restated on the CPU
    (orc_splat_points): depth (H,W), pointmap / normalmap (H,W,3), colormap
    (H,W,3) uint8."""
    L = lib()
    pts = _f32(points).reshape(-1, 3)
    nrm = _f32(normals).reshape(-1, 3) if normals is not None else None
    col = np.ascontiguousarray(colors, dtype=np.uint8).reshape(-1, 3) if colors is not None else None
    depth = np.zeros((height, width), np.float32)
    pm = np.zeros((height, width, 3), np.float32)
    nm = np.zeros((height, width, 3), np.float32)
    cm = np.zeros((height, width, 3), np.uint8)
    L.orc_splat_points(_ptr(pts), len(pts), _ptr(nrm) if nrm is not None else None,
                       len(nrm) if nrm is not None else 0, _ptr(col) if col is not None else None,
                       len(col) if col is not None else 0, int(width), int(height), _f(fx), _f(fy), _f(cx), _f(cy),
                       _f(min_depth), _f(max_depth), int(mode), _ptr(depth), _ptr(pm), _ptr(nm), _ptr(cm))
    return {"depth": depth, "pointmap": pm, "normalmap": nm, "colormap": cm}

"""Thin ctypes binding of libvsg.so (include/vsg.h) for Python callers and tests.

Device buffers are passed as torch CUDA tensors (their data_ptr) or raw
integers; host buffers as numpy arrays.  The library must be built
(build.py); there is no fallback implementation: loading fails loudly when
libvsg.so is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvsg.so")

VSG_OK = 0
STATUS = {0: "VSG_OK", 1: "VSG_ERR_INVALID_ARG", 2: "VSG_ERR_NOT_ALLOCATED", 3: "VSG_ERR_CUDA",
          4: "VSG_ERR_OUT_OF_MEMORY", 5: "VSG_ERR_TOO_LARGE"}
FLAG_HEAP_EXHAUSTED, FLAG_CHAIN_EXHAUSTED, FLAG_COORD_RANGE, FLAG_INSERT_RETRY, FLAG_MARCH_LIMIT = 1, 2, 4, 8, 16
FLAG_PARENT_OVERFLOW = 32

# every symbol include/vsg.h declares
EXPORTS = [
    "vsg_params_default", "vsg_scene_create", "vsg_scene_destroy", "vsg_scene_reset", "vsg_scene_params",
    "vsg_integrate", "vsg_integrate_noalloc", "vsg_scene_set_alloc_method", "vsg_scene_stats", "vsg_scene_export", "vsg_renderer_create", "vsg_renderer_destroy",
    "vsg_render", "vsg_render_hostpose", "vsg_renderer_outputs", "vsg_renderer_download",
    "vsg_renderer_save_ply",
    "vsg_timing_enable", "vsg_timing_read", "vsg_timing_reset", "vsg_scene_march_stats", "vsg_version",
    "vsg_batch_create", "vsg_batch_destroy", "vsg_batch_step", "vsg_batch_autotune",
    "vsg_mc_output_create", "vsg_mc_output_destroy", "vsg_mc_run", "vsg_mc_triangle_count",
    "vsg_mc_output_buffers", "vsg_mc_download",
    "vsg_store_create", "vsg_store_destroy", "vsg_store_info", "vsg_store_export", "vsg_store_save",
    "vsg_store_load", "vsg_store_count", "vsg_store_add_records", "vsg_stream_out", "vsg_stream_in", "vsg_scene_save", "vsg_scene_load",
    "vsg_points_create", "vsg_points_destroy", "vsg_extract_points", "vsg_points_count", "vsg_points_buffers",
    "vsg_points_download", "vsg_points_save_ply",
    "vsg_renderer_record", "vsg_renderer_set_step", "vsg_render_backward", "vsg_render_normals", "vsg_scene_lookup_blocks",
    "vsg_depth_to_pointmap", "vsg_integrate_backward", "vsg_render_pose_normal_equations", "vsg_splat_points",
]


class VsgError(RuntimeError):
    def __init__(self, fn: str, code: int):
        super().__init__(f"{fn} failed: {STATUS.get(code, code)}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("voxel_size", ctypes.c_float), ("truncation", ctypes.c_float),
                ("truncation_scale", ctypes.c_float), ("hash_num_slots", ctypes.c_uint32),
                ("num_sdf_blocks", ctypes.c_uint32), ("max_chain_nodes", ctypes.c_uint32),
                ("occupancy_log2", ctypes.c_uint32)]


class BatchFrame(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_int), ("pointmap", ctypes.c_void_p), ("rgb", ctypes.c_void_p),
                ("normals", ctypes.c_void_p), ("w", ctypes.c_int), ("h", ctypes.c_int),
                ("truncation", ctypes.c_float), ("pose", ctypes.c_float * 16), ("fx", ctypes.c_float),
                ("fy", ctypes.c_float), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
                ("min_depth", ctypes.c_float), ("max_depth", ctypes.c_float), ("render", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "allocated_blocks", "free_blocks", "high_water", "chain_nodes_used", "integrated_frames",
        "frame_valid_pixels", "frame_new_blocks", "frame_visible_blocks", "frame_updated_blocks",
        "frame_updated_voxels", "render_hits", "render_misses", "render_samples_full",
        "render_samples_skipped", "render_jumps", "render_singles", "render_blocks_read",
        "render_lane_iters", "render_warp_iters", "flags",
        "fast_division", "fast_avg_divisors", "pixel_buffer_capacity")]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


_lib = None
_P = ctypes.c_void_p
_F = ctypes.c_float
_I = ctypes.c_int


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run build.py (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name in EXPORTS:
            getattr(L, name).restype = ctypes.c_int
        L.vsg_version.restype = ctypes.c_char_p
        L.vsg_params_default.argtypes = [ctypes.POINTER(Params)]
        L.vsg_scene_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(_P)]
        L.vsg_scene_destroy.argtypes = [_P]
        L.vsg_scene_reset.argtypes = [_P, _P]
        L.vsg_scene_params.argtypes = [_P, ctypes.POINTER(Params)]
        L.vsg_integrate.argtypes = [_P, _P, _P, _P, _I, _I, _F, _P, _F, _F, _F, _F, _P]
        L.vsg_integrate_noalloc.argtypes = [_P, _P, _P, _P, _I, _I, _F, _P, _F, _F, _F, _F, _P]
        L.vsg_scene_set_alloc_method.argtypes = [_P, _I]
        L.vsg_scene_stats.argtypes = [_P, ctypes.POINTER(Stats)]
        L.vsg_scene_export.argtypes = [_P, _P, _P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
        L.vsg_renderer_create.argtypes = [_I, _I, ctypes.POINTER(_P)]
        L.vsg_renderer_destroy.argtypes = [_P]
        L.vsg_render.argtypes = [_P, _P, _P, _P, _F, _F, _F, _F, _F, _F, _P]
        L.vsg_render_hostpose.argtypes = [_P, _P, _P, _P, _F, _F, _F, _F, _F, _F, _P]
        L.vsg_renderer_outputs.argtypes = [_P] + [ctypes.POINTER(_P)] * 4
        L.vsg_renderer_download.argtypes = [_P, _P, _P, _P, _P]
        L.vsg_timing_enable.argtypes = [_P, _I]
        L.vsg_scene_march_stats.argtypes = [_P, _I]
        L.vsg_timing_read.argtypes = [_P, _P, _P, _I]
        L.vsg_timing_reset.argtypes = [_P]
        L.vsg_batch_create.argtypes = [_P, _P, _I, ctypes.POINTER(_P)]
        L.vsg_batch_destroy.argtypes = [_P]
        L.vsg_batch_step.argtypes = [_P, ctypes.POINTER(BatchFrame), _I, _P]
        L.vsg_batch_autotune.argtypes = [_P, _I]
        L.vsg_mc_output_create.argtypes = [_I, ctypes.POINTER(_P)]
        L.vsg_mc_output_destroy.argtypes = [_P]
        L.vsg_mc_run.argtypes = [_P, _P, _F, _F, _P]
        L.vsg_mc_triangle_count.argtypes = [_P, ctypes.POINTER(ctypes.c_int64)]
        L.vsg_mc_output_buffers.argtypes = [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P),
                                            ctypes.POINTER(_I)]
        L.vsg_mc_download.argtypes = [_P, _P, _P, ctypes.POINTER(ctypes.c_int64)]
        _u64p = ctypes.POINTER(ctypes.c_uint64)
        _u32p = ctypes.POINTER(ctypes.c_uint32)
        L.vsg_store_create.argtypes = [_P, ctypes.POINTER(_P)]
        L.vsg_store_destroy.argtypes = [_P]
        L.vsg_store_info.argtypes = [_P, _u64p, _u64p]
        L.vsg_store_export.argtypes = [_P, _P, _P, ctypes.c_uint64, _u64p]
        L.vsg_store_save.argtypes = [_P, ctypes.c_char_p]
        L.vsg_store_load.argtypes = [_P, ctypes.c_char_p]
        L.vsg_store_count.argtypes = [_P, _P, _F, _u64p, _u64p]
        L.vsg_store_add_records.argtypes = [_P, _F, _P, _P, ctypes.c_uint64]
        L.vsg_stream_out.argtypes = [_P, _P, _P, _F, _u32p, _P]
        L.vsg_stream_in.argtypes = [_P, _P, _P, _F, _u32p, _u32p, _P]
        L.vsg_scene_save.argtypes = [_P, ctypes.c_char_p]
        L.vsg_scene_load.argtypes = [_P, ctypes.c_char_p, _P]
        L.vsg_points_create.argtypes = [_I, ctypes.POINTER(_P)]
        L.vsg_points_destroy.argtypes = [_P]
        L.vsg_extract_points.argtypes = [_P, _P, _F, _F, ctypes.c_uint32, _P]
        L.vsg_points_count.argtypes = [_P, ctypes.POINTER(ctypes.c_int64)]
        L.vsg_points_buffers.argtypes = [_P] + [ctypes.POINTER(_P)] * 4 + [ctypes.POINTER(_I)]
        L.vsg_points_download.argtypes = [_P, _P, _P, _P, ctypes.POINTER(ctypes.c_int64)]
        L.vsg_points_save_ply.argtypes = [_P, ctypes.c_char_p]
        L.vsg_renderer_record.argtypes = [_P, _I]
        L.vsg_renderer_set_step.argtypes = [_P, _F]
        _i64 = ctypes.c_int64
        L.vsg_splat_points.argtypes = [_P, _i64, _P, _i64, _P, _i64, _I, _I, _F, _F, _F, _F, _F, _F, _I, _P, _P, _P,
                                       _P, ctypes.POINTER(_i64), _P]
        L.vsg_depth_to_pointmap.argtypes = [_P, _I, _I, _F, _F, _F, _F, _P, _P, _P]
        L.vsg_integrate_backward.argtypes = [_P, _P, _I, _I, _F, _P, _F, _F, _F, _F, _P, _P, _P,
                                             ctypes.POINTER(ctypes.c_uint32), _P]
        L.vsg_scene_lookup_blocks.argtypes = [_P, _P, ctypes.c_uint32, _P]
        L.vsg_render_backward.argtypes = [_P, _P, _P, _F, _F, _F, _F, _P, _P, _P, _P, _F,
                                          ctypes.POINTER(ctypes.c_uint32), _P]
        L.vsg_renderer_save_ply.argtypes = [_P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        L.vsg_render_pose_normal_equations.argtypes = [_P, _P, _P, _F, _F, _F, _F, _P, _P, _F, _P,
                                                       ctypes.POINTER(ctypes.c_uint32), _P]
        L.vsg_render_normals.argtypes = [_P, _P, _P, _F, _F, _F, _F, _P, ctypes.POINTER(ctypes.c_uint32), _P]
        _lib = L
    return _lib


def check(fn: str, code: int):
    if code != VSG_OK:
        raise VsgError(fn, code)


def _dptr(x) -> int:
    """Device pointer of a torch tensor or an int."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    return int(x.data_ptr())


def _stream(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


def _hptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def default_params(**kw) -> Params:
    p = Params()
    check("vsg_params_default", lib().vsg_params_default(ctypes.byref(p)))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def depth_to_pointmap(depth, fx, fy, cx, cy, normals: bool = True, stream=None):
    """(H,W) float32 device depth tensor -> ((H,W,3) point map, (H,W,3)
    normals or None) device tensors (vsg_depth_to_pointmap)."""
    import torch

    H, W = depth.shape
    d = depth.contiguous().to(torch.float32)
    pm = torch.empty((H, W, 3), dtype=torch.float32, device=d.device)
    nm = torch.empty((H, W, 3), dtype=torch.float32, device=d.device) if normals else None
    check("vsg_depth_to_pointmap", lib().vsg_depth_to_pointmap(_dptr(d), W, H, _F(fx), _F(fy), _F(cx), _F(cy),
                                                               _dptr(pm), _dptr(nm), _stream(stream)))
    return pm, nm


class _DeviceArray:
    """__cuda_array_interface__ view of a raw device pointer."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def render_depth(scene, renderer, pose, fx, fy, cx, cy, min_depth, max_depth, min_weight_sum: float = 0.5):
    """Differentiable ray cast (torch autograd): depth (H,W) of `scene` seen
    from `pose` (a (4,4) float32 torch tensor, camera->world; may require
    grad).  The backward pass returns dL/dpose (rows 0-2; row 3 zero) through
    vsg_render_backward.  Misses hold 1e10 and carry no gradient; so do
    pixels whose crossing samples renormalise over less than min_weight_sum
    of trilinear weight (steep near the edge of observed space)."""
    import torch

    class _Render(torch.autograd.Function):
        @staticmethod
        def forward(ctx, T):
            Th = T.detach().to("cpu", torch.float32).numpy().reshape(16)
            renderer.record(True)
            renderer.render(scene, Th, fx, fy, cx, cy, min_depth, max_depth)
            ctx.Th = Th
            ctx.dev, ctx.dtype = T.device, T.dtype
            return renderer.depth_tensor().clone()

        @staticmethod
        def backward(ctx, g):
            g = g.contiguous().to(torch.float32)
            gT, skipped = renderer.backward(scene, ctx.Th, fx, fy, cx, cy, grad_depth=g,
                                            min_weight_sum=min_weight_sum)
            out = torch.zeros((4, 4), dtype=torch.float64)
            out[:3] = torch.from_numpy(gT)
            return out.to(device=ctx.dev, dtype=ctx.dtype)

    return _Render.apply(pose)


SPLAT_LAST, SPLAT_NEAREST = 0, 1


def splat_points(points, width, height, fx, fy, cx, cy, normals=None, colors=None, mode: int = SPLAT_LAST,
                 min_depth: float = 0.0, max_depth: float = float("inf"), stream=None) -> dict:
    """CustomDepthMapGenerator::generateFromPointCloud on the GPU
    (vsg_splat_points): points (N,3) float32, normals (M,3) float32 and
    colors (K,3) uint8 device tensors (M, K may be shorter than N or None).
    Returns device tensors depth (H,W), pointmap and normalmap (H,W,3),
    colormap (H,W,3) uint8, and the number of pixels that got a point."""
    import torch

    dev = torch.device("cuda")
    depth = torch.empty((height, width), dtype=torch.float32, device=dev)
    pm = torch.empty((height, width, 3), dtype=torch.float32, device=dev)
    nm = torch.empty((height, width, 3), dtype=torch.float32, device=dev)
    cm = torch.empty((height, width, 3), dtype=torch.uint8, device=dev)
    n_valid = ctypes.c_int64()
    pts = points.contiguous()
    nrm = normals.contiguous() if normals is not None else None
    col = colors.contiguous() if colors is not None else None
    check("vsg_splat_points", lib().vsg_splat_points(
        _dptr(pts), int(pts.shape[0]), _dptr(nrm), int(nrm.shape[0]) if nrm is not None else 0, _dptr(col),
        int(col.shape[0]) if col is not None else 0, int(width), int(height), _F(fx), _F(fy), _F(cx), _F(cy),
        _F(min_depth), _F(max_depth), int(mode), _dptr(depth), _dptr(pm), _dptr(nm), _dptr(cm),
        ctypes.byref(n_valid), _stream(stream)))
    return {"depth": depth, "pointmap": pm, "normalmap": nm, "colormap": cm, "n_valid": int(n_valid.value)}


def se3_exp(xi) -> np.ndarray:
    """exp of a twist xi = (omega, v) as a 4x4 float64 matrix (Rodrigues'
    formula for R, V v with V = I + (1 - cos th)/th^2 W + (th - sin th)/th^3
    W^2 for t; the series below th = 1e-8)."""
    xi = np.asarray(xi, np.float64)
    w, v = xi[:3], xi[3:]
    th = float(np.linalg.norm(w))
    W = np.array([[0.0, -w[2], w[1]], [w[2], 0.0, -w[0]], [-w[1], w[0], 0.0]])
    if th < 1e-8:
        A, B, C = 1.0, 0.5, 1.0 / 6.0
    else:
        A, B, C = np.sin(th) / th, (1 - np.cos(th)) / th ** 2, (th - np.sin(th)) / th ** 3
    out = np.eye(4)
    out[:3, :3] = np.eye(3) + A * W + B * (W @ W)
    out[:3, 3] = (np.eye(3) + B * W + C * (W @ W)) @ v
    return out


def _unit_rays(width, height, fx, fy, cx, cy):
    """(H,W,3) unit camera-space ray directions on the device, float32."""
    import torch

    v, u = torch.meshgrid(torch.arange(height, device="cuda", dtype=torch.float32),
                          torch.arange(width, device="cuda", dtype=torch.float32), indexing="ij")
    cd = torch.stack([(u - cx) / fx, (v - cy) / fy, torch.ones_like(u)], -1)
    return cd / cd.norm(dim=-1, keepdim=True)


def refine_pose(scene, renderer, target_depth, pose, fx, fy, cx, cy, min_depth, max_depth, steps: int = 8,
                huber: float = 0.01, damping: float = 1e-6, min_weight_sum: float = 0.5,
                max_residual=(0.2, 0.05), min_incidence: float = 0.0, min_pixels: int = 500,
                max_step=(0.1, 0.1)):
    """Gauss-Newton alignment of a camera pose to a target depth image (H,W
    device float32, misses >= 1e9) through the ray cast: each step renders at
    the current pose, forms residuals (rendered - target) on pixels hit in
    both with Huber weights (1 inside `huber` metres, huber/|r| outside),
    solves (H + damping diag(H)) xi = -b from
    vsg_render_pose_normal_equations and right-multiplies the pose by
    exp(xi).  Outliers (disocclusions, silhouettes) are left out: pixels
    whose |residual| exceeds a threshold shrinking geometrically from
    max_residual[0] to max_residual[1] over the steps.  With
    min_incidence > 0, pixels where the model's normal (vsg_render_normals)
    meets the ray at |cos| < min_incidence are left out too: at grazing
    incidence the depth is steep in the pose.  The iteration stops when
    fewer than min_pixels pixels carry weight; a step longer than max_step
    (radians, metres) is shortened to it.  Returns (4x4 float64 pose,
    per-step weighted RMS residual)."""
    import torch

    T = np.asarray(pose, np.float64).reshape(4, 4).copy()
    renderer.record(True)
    rays = _unit_rays(renderer.width, renderer.height, fx, fy, cx, cy) if min_incidence > 0 else None
    r0, r1 = (float(max_residual[0]), float(max_residual[1])) if max_residual is not None else (np.inf, np.inf)
    rms = []
    for k in range(steps):
        T32 = T.astype(np.float32)
        renderer.render(scene, T32, fx, fy, cx, cy, min_depth, max_depth)
        d = renderer.depth_tensor()
        m = (d < 1e9) & (target_depth < 1e9)
        if rays is not None:
            n, _ = renderer.normals(scene, T32, fx, fy, cx, cy)
            R = torch.as_tensor(T32[:3, :3], device="cuda")
            cos = (n[..., :3] * (rays @ R.T)).sum(-1).abs()
            m = m & (cos >= min_incidence)
        r = torch.where(m, d - target_depth, torch.zeros_like(d))
        a = r.abs()
        tau = r0 * (r1 / r0) ** (k / max(steps - 1, 1)) if np.isfinite(r0) else np.inf
        m = m & (a <= tau)
        w = torch.where(m, torch.where(a <= huber, torch.ones_like(a), huber / a.clamp_min(huber)),
                        torch.zeros_like(a))
        if int(m.sum()) < min_pixels:
            break
        Hm, b, _ = renderer.pose_normal_equations(scene, T32, fx, fy, cx, cy, r, w, min_weight_sum)
        rms.append(float(torch.sqrt((w * r * r).sum() / w.sum().clamp_min(1e-30))))
        A = Hm + damping * np.diag(np.diag(Hm))
        if not np.all(np.isfinite(A)) or np.linalg.matrix_rank(A) < 6:
            break
        xi = -np.linalg.solve(A, b)
        s = max(np.linalg.norm(xi[:3]) / max_step[0], np.linalg.norm(xi[3:]) / max_step[1], 1.0)
        T = T @ se3_exp(xi / s)
    return T, rms


def _normal_matrix(v: np.ndarray):
    Hm = np.zeros((6, 6))
    iu = np.triu_indices(6)
    Hm[iu] = v[:21]
    return Hm + np.triu(Hm, 1).T, v[21:]


def refine_poses(scenes, renderers, targets, poses, intrinsics, min_depth, max_depth, steps: int = 8,
                 huber: float = 0.01, damping: float = 1e-6, min_weight_sum: float = 0.5,
                 max_residual=(0.2, 0.05), min_incidence: float = 0.0, min_pixels: int = 500,
                 max_step=(0.1, 0.1), streams=None):
    """refine_pose for several independent (scene, renderer, target depth,
    pose) problems at once, with the same steps, weights, stopping rules and
    results: in every Gauss-Newton step all problems' GPU work (render,
    normals, residuals, normal equations) is issued -- on one CUDA stream per
    problem when `streams` (torch streams) is given, else on the current
    stream -- before ONE host synchronisation collects every system; the
    6x6 solves and pose updates then run on the host.  intrinsics: one
    (fx, fy, cx, cy) for all or one per problem.  Returns (list of 4x4
    float64 poses, list of per-step weighted RMS residual lists)."""
    import torch

    n = len(scenes)
    K = [tuple(intrinsics)] * n if np.isscalar(intrinsics[0]) else [tuple(k) for k in intrinsics]
    T = [np.asarray(p, np.float64).reshape(4, 4).copy() for p in poses]
    cur = torch.cuda.current_stream()
    if streams is None:
        streams = [cur] * n
    for r in renderers:
        r.record(True)
    # everything the problems' streams read is made on the current stream
    # first; then those streams wait for it
    rays = [_unit_rays(renderers[i].width, renderers[i].height, *K[i]) if min_incidence > 0 else None
            for i in range(n)]
    r0, r1 = (float(max_residual[0]), float(max_residual[1])) if max_residual is not None else (np.inf, np.inf)
    rms = [[] for _ in range(n)]
    active = [True] * n
    ne = torch.zeros((n, 27), dtype=torch.float64, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int64, device="cuda")
    res = torch.zeros(n, dtype=torch.float32, device="cuda")
    for st in {id(x): x for x in streams}.values():
        st.wait_stream(cur)
    for k in range(steps):
        todo = [i for i in range(n) if active[i]]
        if not todo:
            break
        tau = r0 * (r1 / r0) ** (k / max(steps - 1, 1)) if np.isfinite(r0) else np.inf
        for i in todo:
            fx, fy, cx, cy = K[i]
            T32 = T[i].astype(np.float32)
            sh = streams[i].cuda_stream
            with torch.cuda.stream(streams[i]):
                renderers[i].render(scenes[i], T32, fx, fy, cx, cy, min_depth, max_depth, stream=sh)
                d = renderers[i].depth_tensor()
                tg = targets[i]
                m = (d < 1e9) & (tg < 1e9)
                if rays[i] is not None:
                    nrm, _ = renderers[i].normals(scenes[i], T32, fx, fy, cx, cy, stream=sh, sync=False)
                    R = torch.as_tensor(T32[:3, :3], device="cuda")
                    cos = (nrm[..., :3] * (rays[i] @ R.T)).sum(-1).abs()
                    m = m & (cos >= min_incidence)
                r = torch.where(m, d - tg, torch.zeros_like(d))
                a = r.abs()
                m = m & (a <= tau)
                w = torch.where(m, torch.where(a <= huber, torch.ones_like(a), huber / a.clamp_min(huber)),
                                torch.zeros_like(a))
                cnt[i] = m.sum()
                res[i] = torch.sqrt((w * r * r).sum() / w.sum().clamp_min(1e-30))
                renderers[i].pose_normal_equations_into(scenes[i], T32, fx, fy, cx, cy, r, w, ne[i],
                                                        min_weight_sum, stream=sh)
        torch.cuda.synchronize()
        ne_h, cnt_h, res_h = ne.cpu().numpy(), cnt.cpu().numpy(), res.cpu().numpy()
        for i in todo:
            if int(cnt_h[i]) < min_pixels:
                active[i] = False
                continue
            Hm, b = _normal_matrix(ne_h[i])
            rms[i].append(float(res_h[i]))
            A = Hm + damping * np.diag(np.diag(Hm))
            if not np.all(np.isfinite(A)) or np.linalg.matrix_rank(A) < 6:
                active[i] = False
                continue
            xi = -np.linalg.solve(A, b)
            sc = max(np.linalg.norm(xi[:3]) / max_step[0], np.linalg.norm(xi[3:]) / max_step[1], 1.0)
            T[i] = T[i] @ se3_exp(xi / sc)
    return T, rms


def tune_ray_step(scene, renderer, poses, intrinsics, min_depth, max_depth, truncation,
                  factors=(0.5, 0.625, 0.75, 0.875, 1.0), tol: float = 1e-3, frac: float = 0.99, reps: int = 3):
    """Autotune the opt-in march step (vsg_renderer_set_step) on sample poses:
    for each step = factor x truncation, time the ray casts (CUDA events) and
    compare their depths with the reference's half-voxel march at the same
    poses.  Returns (chosen step -- the fastest whose depths stay within `tol`
    metres of the exact ones on at least `frac` of the pixels both hit, with
    hit/miss flips counted as misses; 0, the exact march, if none does -- and
    per candidate {step, ms, frac_within_tol, max_err, rms_err, flips}).  The
    renderer is left at the chosen step."""
    import torch

    fx, fy, cx, cy = intrinsics

    def run(step):
        renderer.set_step(step)
        outs = []
        for T in poses:
            renderer.render(scene, T, fx, fy, cx, cy, min_depth, max_depth)
            outs.append(renderer.depth_tensor().clone())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            for T in poses:
                renderer.render(scene, T, fx, fy, cx, cy, min_depth, max_depth)
        e1.record()
        torch.cuda.synchronize()
        return outs, e0.elapsed_time(e1) / (reps * len(poses))

    exact, ms0 = run(0.0)
    table = [{"step": 0.0, "ms": ms0, "frac_within_tol": 1.0, "max_err": 0.0, "rms_err": 0.0, "flips": 0}]
    best, best_ms = 0.0, ms0
    for f in factors:
        step = float(f) * float(truncation)
        outs, ms = run(step)
        ok = tot = flips = 0
        errs = []
        for a, b in zip(exact, outs):
            ha, hb = a < 1e9, b < 1e9
            both = ha & hb
            e = (a - b).abs()[both].double()
            flips += int((ha != hb).sum())
            ok += int((e <= tol).sum())
            tot += int(ha.sum())
            errs.append(e)
        e = torch.cat(errs)
        fr = ok / max(tot, 1)
        row = {"step": step, "ms": ms, "frac_within_tol": fr, "max_err": float(e.max()) if e.numel() else 0.0,
               "rms_err": float(e.pow(2).mean().sqrt()) if e.numel() else 0.0, "flips": flips}
        table.append(row)
        if fr >= frac and ms < best_ms:
            best, best_ms = step, ms
    renderer.set_step(best)
    return best, table


def stream_scenes(scenes, stores, centers, r_out: float, r_in: float, streams=None, max_threads: int = 8):
    """One streaming pass for several scenes at once, in the reference main
    loop's order (voxelSG.cpp:503-551): per scene, stream out every block
    farther than r_out from its centre into its store, then stream in the
    stored chunks within r_in.  The scenes go through host threads (the C
    calls release the interpreter lock), each on its own CUDA stream
    (`streams`: torch streams, one per scene; created here when None), so
    their transfers and host filing overlap.  Work queued on the current
    stream before the call is waited for.  Returns per scene (blocks out,
    blocks in, 1 if the stream-in was refused for lack of pool blocks)."""
    import concurrent.futures as cf

    import torch

    n = len(scenes)
    if streams is None:
        streams = [torch.cuda.Stream() for _ in range(n)]
    torch.cuda.current_stream().synchronize()
    dev = torch.cuda.current_device()

    def one(i):
        torch.cuda.set_device(dev)
        sh = streams[i].cuda_stream
        c = np.asarray(centers[i], np.float32)
        n_out = scenes[i].stream_out(stores[i], c, r_out, stream=sh)
        refused = 0
        try:
            n_in = scenes[i].stream_in(stores[i], c, r_in, stream=sh)[0]
        except VsgError as exc:
            if exc.code != 5:  # VSG_ERR_TOO_LARGE: nothing moved
                raise
            n_in, refused = 0, 1
        return n_out, n_in, refused

    with cf.ThreadPoolExecutor(max_workers=max(1, min(max_threads, n))) as ex:
        return list(ex.map(one, range(n)))


class Scene:
    """VoxelScene over the C ABI (vsg_scene_*, vsg_integrate)."""

    def __init__(self, params: Params | None = None, **kw):
        self.L = lib()
        self.params = params if params is not None else default_params(**kw)
        h = _P()
        check("vsg_scene_create", self.L.vsg_scene_create(ctypes.byref(self.params), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.vsg_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self, stream=None):
        check("vsg_scene_reset", self.L.vsg_scene_reset(self.h, _stream(stream)))

    def set_alloc_method(self, method: int):
        """1: camera-z band (Method 1, default); 2: camera and normal rays with
        parent pixels (Method 2, VoxelScene.cu:768-912)."""
        check("vsg_scene_set_alloc_method", self.L.vsg_scene_set_alloc_method(self.h, int(method)))

    def integrate(self, pointmap, rgb, normals, width, height, truncation, pose, fx, fy, cx, cy, stream=None):
        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        check("vsg_integrate", self.L.vsg_integrate(
            self.h, _dptr(pointmap), _dptr(rgb), _dptr(normals), int(width), int(height), _F(truncation),
            _hptr(T), _F(fx), _F(fy), _F(cx), _F(cy), _stream(stream)))

    def integrate_noalloc(self, pointmap, rgb, normals, width, height, truncation, pose, fx, fy, cx, cy,
                          stream=None):
        """vsg_integrate_noalloc: the same integration with its per-pixel
        work buffers in the library's fixed device array (no allocation)."""
        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        check("vsg_integrate_noalloc", self.L.vsg_integrate_noalloc(
            self.h, _dptr(pointmap), _dptr(rgb), _dptr(normals), int(width), int(height), _F(truncation),
            _hptr(T), _F(fx), _F(fy), _F(cx), _F(cy), _stream(stream)))

    def stats(self) -> dict:
        st = Stats()
        check("vsg_scene_stats", self.L.vsg_scene_stats(self.h, ctypes.byref(st)))
        return st.as_dict()

    def export(self, with_voxels: bool = True):
        """(coords (n,3) int32 sorted, voxel bytes (n, 4096) uint8 or None)."""
        n = ctypes.c_uint32(0)
        dummy = np.zeros(3, np.int32)
        rc = self.L.vsg_scene_export(self.h, _hptr(dummy), None, 0, ctypes.byref(n))
        if rc not in (VSG_OK, 5):
            check("vsg_scene_export", rc)
        cnt = int(n.value)
        coords = np.zeros((max(cnt, 1), 3), np.int32)
        vox = np.zeros((max(cnt, 1), 4096), np.uint8) if with_voxels else None
        check("vsg_scene_export", self.L.vsg_scene_export(
            self.h, _hptr(coords), _hptr(vox) if with_voxels else None, cnt, ctypes.byref(n)))
        return coords[:cnt], (vox[:cnt] if with_voxels else None)

    def integrate_backward(self, pointmap, width, height, truncation, pose, fx, fy, cx, cy, grad_sdf,
                           grad_pointmap=None, stream=None):
        """Adjoint of the last vsg_integrate (same inputs): grad_sdf (device
        float32, num_sdf_blocks*512, dL/d SDF after the frame) becomes dL/d SDF
        before it for the updated voxels, in place; grad_pointmap (H,W,3) device
        tensor is added to.  Returns (dL/dT (3,4) float64 numpy, voxels updated)."""
        import torch

        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        gp = torch.zeros(12, dtype=torch.float64, device="cuda")
        n = ctypes.c_uint32()
        check("vsg_integrate_backward", self.L.vsg_integrate_backward(
            self.h, _dptr(pointmap), int(width), int(height), _F(truncation), _hptr(T), _F(fx), _F(fy), _F(cx),
            _F(cy), _dptr(grad_sdf), _dptr(gp), _dptr(grad_pointmap), ctypes.byref(n), _stream(stream)))
        return gp.cpu().numpy().reshape(3, 4), int(n.value)

    def lookup_blocks(self, coords) -> np.ndarray:
        """Pool index of each block coordinate (-1 = not allocated)."""
        c = np.ascontiguousarray(np.asarray(coords, np.int32).reshape(-1, 3))
        out = np.zeros(max(len(c), 1), np.int32)
        check("vsg_scene_lookup_blocks", self.L.vsg_scene_lookup_blocks(self.h, _hptr(c), len(c), _hptr(out)))
        return out[:len(c)]

    def stream_out(self, store: "Store", center, radius: float, stream=None) -> int:
        c = np.ascontiguousarray(np.asarray(center, np.float32).reshape(3))
        n = ctypes.c_uint32()
        check("vsg_stream_out", self.L.vsg_stream_out(self.h, store.h, _hptr(c), _F(radius), ctypes.byref(n),
                                                      _stream(stream)))
        return int(n.value)

    def stream_in(self, store: "Store", center=None, radius: float = -1.0, stream=None) -> tuple[int, int]:
        c = np.ascontiguousarray(np.asarray(center if center is not None else (0, 0, 0), np.float32).reshape(3))
        n, m = ctypes.c_uint32(), ctypes.c_uint32()
        check("vsg_stream_in", self.L.vsg_stream_in(self.h, store.h, _hptr(c), _F(radius), ctypes.byref(n),
                                                    ctypes.byref(m), _stream(stream)))
        return int(n.value), int(m.value)

    def save(self, path: str):
        check("vsg_scene_save", self.L.vsg_scene_save(self.h, str(path).encode()))

    def load(self, path: str, stream=None):
        check("vsg_scene_load", self.L.vsg_scene_load(self.h, str(path).encode(), _stream(stream)))

    def timing(self, enable: bool):
        check("vsg_timing_enable", self.L.vsg_timing_enable(self.h, int(enable)))

    def march_stats(self, enable: bool):
        """Count skipped samples, boundary samples and distinct blocks read in
        the following renders (stats() render_samples_skipped, render_singles,
        render_blocks_read); the counting ray caster is about 10 % slower."""
        check("vsg_scene_march_stats", self.L.vsg_scene_march_stats(self.h, int(enable)))

    def timing_read(self) -> tuple[np.ndarray, np.ndarray]:
        ms = np.zeros(8, np.float64)
        cnt = np.zeros(8, np.uint32)
        check("vsg_timing_read", self.L.vsg_timing_read(self.h, _hptr(ms), _hptr(cnt), 8))
        return ms, cnt

    def timing_reset(self):
        check("vsg_timing_reset", self.L.vsg_timing_reset(self.h))


class Renderer:
    """RayCastRender over the C ABI (vsg_renderer_*, vsg_render)."""

    def __init__(self, width: int, height: int):
        self.L = lib()
        h = _P()
        check("vsg_renderer_create", self.L.vsg_renderer_create(int(width), int(height), ctypes.byref(h)))
        self.h = h
        self.width, self.height = width, height

    def close(self):
        if getattr(self, "h", None):
            self.L.vsg_renderer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, scene: Scene, pose, fx, fy, cx, cy, min_depth, max_depth, cam_pos=None, pose_dev=None,
               stream=None):
        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        cam = np.ascontiguousarray(np.array([T[3], T[7], T[11]], np.float32) if cam_pos is None
                                   else np.asarray(cam_pos, np.float32))
        if pose_dev is not None:
            check("vsg_render", self.L.vsg_render(self.h, scene.h, _hptr(cam), _dptr(pose_dev), _F(fx), _F(fy),
                                                  _F(cx), _F(cy), _F(min_depth), _F(max_depth), _stream(stream)))
        else:
            check("vsg_render_hostpose", self.L.vsg_render_hostpose(
                self.h, scene.h, _hptr(cam), _hptr(T), _F(fx), _F(fy), _F(cx), _F(cy), _F(min_depth),
                _F(max_depth), _stream(stream)))

    def record(self, enable: bool = True):
        """Keep each pixel's march bracket in the following renders (needed
        by backward() and normals())."""
        check("vsg_renderer_record", self.L.vsg_renderer_record(self.h, int(enable)))

    def set_step(self, step: float = 0.0):
        """March step in metres (vsg_renderer_set_step).  0 keeps the
        reference's half-voxel step and its depths bit for bit; a positive
        step is an opt-in approximation (see tune_ray_step)."""
        check("vsg_renderer_set_step", self.L.vsg_renderer_set_step(self.h, _F(step)))

    def backward(self, scene: "Scene", pose, fx, fy, cx, cy, grad_depth=None, grad_position=None, grad_sdf=None,
                 min_weight_sum: float = 0.0, stream=None):
        """Reverse mode through the last recorded render.  grad_depth (H,W) /
        grad_position (H,W,4): device float32 tensors of dL/d output (None = 0).
        grad_sdf: device float32 tensor of num_sdf_blocks*512 entries the voxel
        SDF gradients are ADDED to (None = skip).  Returns (dL/dT as a (3,4)
        float64 numpy array, number of hit pixels that could not be
        recomputed -- 0 when the render used this scene and pose)."""
        import torch

        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        gp = torch.zeros(12, dtype=torch.float64, device="cuda")
        skipped = ctypes.c_uint32()
        check("vsg_render_backward", self.L.vsg_render_backward(
            self.h, scene.h, _hptr(T), _F(fx), _F(fy), _F(cx), _F(cy), _dptr(grad_depth), _dptr(grad_position),
            _dptr(gp), _dptr(grad_sdf), _F(min_weight_sum), ctypes.byref(skipped), _stream(stream)))
        return gp.cpu().numpy().reshape(3, 4), int(skipped.value)

    def pose_normal_equations(self, scene: "Scene", pose, fx, fy, cx, cy, residual, weights=None,
                              min_weight_sum: float = 0.5, stream=None):
        """Gauss-Newton system of the last recorded render for per-pixel
        residuals (H,W) and optional weights (device float32 tensors):
        returns (H (6,6), b (6,)) float64 numpy in the right-perturbation
        coordinates (omega, v) of T exp(xi), and the skipped-pixel count."""
        import torch

        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        ne = torch.zeros(27, dtype=torch.float64, device="cuda")
        skipped = ctypes.c_uint32()
        check("vsg_render_pose_normal_equations", self.L.vsg_render_pose_normal_equations(
            self.h, scene.h, _hptr(T), _F(fx), _F(fy), _F(cx), _F(cy), _dptr(residual.contiguous()),
            _dptr(weights.contiguous() if weights is not None else None), _F(min_weight_sum), _dptr(ne),
            ctypes.byref(skipped), _stream(stream)))
        v = ne.cpu().numpy()
        Hm = np.zeros((6, 6))
        iu = np.triu_indices(6)
        Hm[iu] = v[:21]
        Hm = Hm + np.triu(Hm, 1).T
        return Hm, v[21:], int(skipped.value)

    def normals(self, scene: "Scene", pose, fx, fy, cx, cy, out=None, stream=None, sync: bool = True):
        """Normals of the last recorded render: (H,W,4) float32 device tensor,
        and the skipped-pixel count (None with sync=False: the call then
        returns without waiting for the device)."""
        import torch

        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        if out is None:
            out = torch.empty((self.height, self.width, 4), dtype=torch.float32, device="cuda")
        skipped = ctypes.c_uint32()
        check("vsg_render_normals", self.L.vsg_render_normals(
            self.h, scene.h, _hptr(T), _F(fx), _F(fy), _F(cx), _F(cy), _dptr(out),
            ctypes.byref(skipped) if sync else None, _stream(stream)))
        return out, (int(skipped.value) if sync else None)

    def pose_normal_equations_into(self, scene: "Scene", pose, fx, fy, cx, cy, residual, weights, out,
                                   min_weight_sum: float = 0.5, stream=None):
        """pose_normal_equations without waiting for the device: the 27
        doubles (H's upper triangle, then b) go to the device tensor `out`."""
        T = np.ascontiguousarray(np.asarray(pose, np.float32).reshape(16))
        check("vsg_render_pose_normal_equations", self.L.vsg_render_pose_normal_equations(
            self.h, scene.h, _hptr(T), _F(fx), _F(fy), _F(cx), _F(cy), _dptr(residual.contiguous()),
            _dptr(weights.contiguous() if weights is not None else None), _F(min_weight_sum), _dptr(out), None,
            _stream(stream)))

    def depth_tensor(self):
        """The depth output buffer as a (H,W) float32 torch tensor view."""
        import torch

        return torch.as_tensor(_DeviceArray(self.outputs()["depth"], (self.height, self.width), "<f4"),
                               device="cuda")

    def save_ply(self, path: str) -> int:
        """RayCastRender::savePointCloudPLY: ASCII PLY of the last render's
        hits with 8-bit colour; returns the number of points written."""
        n = ctypes.c_int64()
        check("vsg_renderer_save_ply", self.L.vsg_renderer_save_ply(self.h, str(path).encode(), ctypes.byref(n)))
        return int(n.value)

    def outputs(self) -> dict:
        ps = [_P() for _ in range(4)]
        check("vsg_renderer_outputs", self.L.vsg_renderer_outputs(self.h, *[ctypes.byref(p) for p in ps]))
        return {k: int(p.value or 0) for k, p in zip(("depth", "position", "color", "normal"), ps)}

    def download(self) -> dict:
        n = self.width * self.height
        d = np.zeros((self.height, self.width), np.float32)
        p = np.zeros((self.height, self.width, 4), np.float32)
        c = np.zeros((self.height, self.width, 4), np.float32)
        nm = np.zeros((self.height, self.width, 4), np.float32)
        check("vsg_renderer_download", self.L.vsg_renderer_download(self.h, _hptr(d), _hptr(p), _hptr(c), _hptr(nm)))
        assert n == d.size
        return {"depth": d, "position": p, "color": c, "normal": nm}


class Store:
    """Host chunk grid of streamed-out blocks (vsg_block_store)."""

    def __init__(self, chunk_extent=(1.0, 1.0, 1.0)):
        self.L = lib()
        h = _P()
        e = np.ascontiguousarray(np.asarray(chunk_extent, np.float32).reshape(3))
        check("vsg_store_create", self.L.vsg_store_create(_hptr(e), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.vsg_store_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> tuple[int, int]:
        nb, nc = ctypes.c_uint64(), ctypes.c_uint64()
        check("vsg_store_info", self.L.vsg_store_info(self.h, ctypes.byref(nb), ctypes.byref(nc)))
        return int(nb.value), int(nc.value)

    def export(self):
        """(coords (n,3) int32 sorted, voxel bytes (n, 4096) uint8)."""
        n = self.info()[0]
        coords = np.zeros((max(n, 1), 3), np.int32)
        vox = np.zeros((max(n, 1), 4096), np.uint8)
        out = ctypes.c_uint64()
        check("vsg_store_export", self.L.vsg_store_export(self.h, _hptr(coords), _hptr(vox), n, ctypes.byref(out)))
        return coords[:n], vox[:n]

    def save(self, path: str):
        check("vsg_store_save", self.L.vsg_store_save(self.h, str(path).encode()))

    def load(self, path: str):
        check("vsg_store_load", self.L.vsg_store_load(self.h, str(path).encode()))

    def count(self, center=None, radius: float = -1.0) -> tuple[int, int]:
        """(blocks, chunks) a stream-in with this centre and radius would take."""
        c = np.ascontiguousarray(np.asarray(center if center is not None else (0, 0, 0), np.float32).reshape(3))
        nb, nc = ctypes.c_uint64(), ctypes.c_uint64()
        check("vsg_store_count", self.L.vsg_store_count(self.h, _hptr(c), _F(radius), ctypes.byref(nb),
                                                        ctypes.byref(nc)))
        return int(nb.value), int(nc.value)

    def add_records(self, voxel_size: float, infos, ref_voxels):
        """File blocks given in the reference's records: infos (n,4) int32
        {x, y, z, ptr}, ref_voxels (n, 512*12) uint8 VoxelData."""
        infos = np.ascontiguousarray(infos, np.int32).reshape(-1, 4)
        ref_voxels = np.ascontiguousarray(ref_voxels, np.uint8).reshape(len(infos), -1)
        check("vsg_store_add_records", self.L.vsg_store_add_records(self.h, _F(voxel_size), _hptr(infos),
                                                                    _hptr(ref_voxels), len(infos)))


class SurfacePoints:
    """RayCastRender::extractSurfacePoints over the C ABI (vsg_points_*)."""

    def __init__(self, max_points: int):
        self.L = lib()
        h = _P()
        check("vsg_points_create", self.L.vsg_points_create(int(max_points), ctypes.byref(h)))
        self.h = h
        self.max_points = int(max_points)

    def close(self):
        if getattr(self, "h", None):
            self.L.vsg_points_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def extract(self, scene: "Scene", min_sdf: float = -0.1, max_sdf: float = 0.1, min_weight: int = 1,
                stream=None):
        check("vsg_extract_points", self.L.vsg_extract_points(scene.h, self.h, _F(min_sdf), _F(max_sdf),
                                                              int(min_weight), _stream(stream)))

    def count(self) -> int:
        n = ctypes.c_int64()
        check("vsg_points_count", self.L.vsg_points_count(self.h, ctypes.byref(n)))
        return int(n.value)

    def buffers(self) -> dict:
        ps = [_P() for _ in range(4)]
        m = _I()
        check("vsg_points_buffers", self.L.vsg_points_buffers(self.h, *[ctypes.byref(p) for p in ps],
                                                              ctypes.byref(m)))
        d = {k: int(p.value or 0) for k, p in zip(("positions", "colors", "normals", "count"), ps)}
        d["max_points"] = int(m.value)
        return d

    def download(self):
        """(total count, positions (m,4), colours (m,4), normals (m,4)), m = min(count, capacity)."""
        n = self.count()
        m = min(n, self.max_points)
        P, C, N = (np.zeros((max(m, 1), 4), np.float32) for _ in range(3))
        c = ctypes.c_int64()
        check("vsg_points_download", self.L.vsg_points_download(self.h, _hptr(P), _hptr(C), _hptr(N),
                                                                ctypes.byref(c)))
        return int(c.value), P[:m], C[:m], N[:m]

    def save_ply(self, path: str):
        check("vsg_points_save_ply", self.L.vsg_points_save_ply(self.h, str(path).encode()))


class MarchingCubes:
    """MarchingCubesOutput + runMarchingCubesCUDA over the C ABI (vsg_mc_*)."""

    def __init__(self, max_triangles: int):
        self.L = lib()
        h = _P()
        check("vsg_mc_output_create", self.L.vsg_mc_output_create(int(max_triangles), ctypes.byref(h)))
        self.h = h
        self.max_triangles = int(max_triangles)

    def close(self):
        if getattr(self, "h", None):
            self.L.vsg_mc_output_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, scene: "Scene", iso: float = 0.0, voxel_size: float = 0.0, stream=None):
        check("vsg_mc_run", self.L.vsg_mc_run(scene.h, self.h, _F(iso), _F(voxel_size), _stream(stream)))

    def count(self) -> int:
        n = ctypes.c_int64()
        check("vsg_mc_triangle_count", self.L.vsg_mc_triangle_count(self.h, ctypes.byref(n)))
        return int(n.value)

    def buffers(self) -> dict:
        v, nm, c, m = _P(), _P(), _P(), _I()
        check("vsg_mc_output_buffers", self.L.vsg_mc_output_buffers(self.h, ctypes.byref(v), ctypes.byref(nm),
                                                                    ctypes.byref(c), ctypes.byref(m)))
        return {"vertices": int(v.value or 0), "normals": int(nm.value or 0), "count": int(c.value or 0),
                "max_triangles": int(m.value)}

    def download(self):
        """(total count, vertices (m,3,3) f32, normals (m,3,3) f32), m = min(count, capacity)."""
        n = self.count()
        m = min(n, self.max_triangles)
        v = np.zeros((max(m, 1), 3, 3), np.float32)
        nm = np.zeros((max(m, 1), 3, 3), np.float32)
        c = ctypes.c_int64()
        check("vsg_mc_download", self.L.vsg_mc_download(self.h, _hptr(v), _hptr(nm), ctypes.byref(c)))
        return int(c.value), v[:m], nm[:m]


class Batch:
    """vsg_batch_*: scenes (and renderers) advanced together, one frame per
    listed scene per step."""

    def __init__(self, scenes, renderers=None):
        self.L = lib()
        n = len(scenes)
        self._scenes = list(scenes)
        self._renderers = list(renderers) if renderers is not None else [None] * n
        sh = (_P * n)(*[s.h.value if isinstance(s.h, _P) else s.h for s in scenes])
        rh = (_P * n)(*[(r.h.value if isinstance(r.h, _P) else r.h) if r is not None else None
                        for r in self._renderers])
        h = _P()
        check("vsg_batch_create", self.L.vsg_batch_create(sh, rh, n, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.vsg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self, enable: bool):
        check("vsg_batch_autotune", self.L.vsg_batch_autotune(self.h, int(enable)))

    @staticmethod
    def frame(scene, pointmap, rgb, normals, width, height, truncation, pose, fx, fy, cx, cy,
              min_depth=0.2, max_depth=3.0, render=True) -> BatchFrame:
        f = BatchFrame()
        f.scene = int(scene)
        f.pointmap, f.rgb, f.normals = _dptr(pointmap), _dptr(rgb), _dptr(normals)
        f.w, f.h = int(width), int(height)
        f.truncation = float(truncation)
        f.pose[:] = [float(x) for x in np.asarray(pose, np.float32).reshape(16)]
        f.fx, f.fy, f.cx, f.cy = float(fx), float(fy), float(cx), float(cy)
        f.min_depth, f.max_depth = float(min_depth), float(max_depth)
        f.render = int(bool(render))
        return f

    def step(self, frames, stream=None):
        arr = (BatchFrame * len(frames))(*frames)
        check("vsg_batch_step", self.L.vsg_batch_step(self.h, arr, len(frames), _stream(stream)))


def version() -> str:
    return lib().vsg_version().decode()

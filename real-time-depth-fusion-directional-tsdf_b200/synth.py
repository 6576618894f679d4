"""Seeded synthetic depth streams for the fusion path.

The reference runs on proprietary intra-oral scans that are not available, so
its inputs (VoxelScene::integrateFromScanData, VoxelScene.h:89-91: a
camera-space point map float3, a colour map uchar3 and a normal map float3 per
pixel, plus a row-major 4x4 camera->world pose) are produced here by ray
tracing analytic scenes.  Depth noise follows a structured-light model
sigma(z) = 0.0012 + 0.0019 (z - 0.4)^2 applied to z along each pixel ray; the
point map is then p = ((u - cx) z / fx, (v - cy) z / fy, z), the convention of
CustomDepthMapGenerator.cpp:81-222 (pixel (0,0,0) = invalid).

Camera frame convention: x right, y down, z forward (OpenCV).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Intrinsics:
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float


@dataclasses.dataclass
class Frame:
    pointmap: np.ndarray  # (H, W, 3) float32, camera space, 0 = invalid
    rgb: np.ndarray  # (H, W, 3) uint8
    normals: np.ndarray  # (H, W, 3) float32, camera space
    depth: np.ndarray  # (H, W) float32, 0 = invalid
    pose: np.ndarray  # (4, 4) float32 camera->world, row-major


@dataclasses.dataclass
class Scene:
    planes: list  # (point(3), normal(3)) one-sided planes
    spheres: list  # (centre(3), radius)
    boxes: list  # (min(3), max(3)) solid axis-aligned boxes
    room: tuple | None = None  # (min(3), max(3)) viewed from inside


def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """Camera->world pose with z toward target, y down in the image."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    x = np.cross(f, np.asarray(up, np.float64))
    x /= np.linalg.norm(x)
    y = np.cross(f, x)
    T = np.eye(4)
    T[:3, 0], T[:3, 1], T[:3, 2], T[:3, 3] = x, y, f, eye
    return T


def _trace(scene: Scene, o: np.ndarray, d: np.ndarray):
    """Nearest hit distance along unit rays d (N,3) from origin o (3,)."""
    n = d.shape[0]
    tbest = np.full(n, np.inf)
    nbest = np.zeros((n, 3))
    eps = 1e-9
    for (p0, nrm) in scene.planes:
        nrm = np.asarray(nrm, np.float64)
        den = d @ nrm
        t = ((np.asarray(p0) - o) @ nrm) / np.where(np.abs(den) < eps, eps, den)
        ok = (den < -eps) & (t > 0) & (t < tbest)
        tbest = np.where(ok, t, tbest)
        nbest[ok] = nrm
    for (c, r) in scene.spheres:
        oc = o - np.asarray(c)
        b = d @ oc
        cc = oc @ oc - r * r
        disc = b * b - cc
        sq = np.sqrt(np.maximum(disc, 0.0))
        t = -b - sq
        ok = (disc > 0) & (t > 0) & (t < tbest)
        tbest = np.where(ok, t, tbest)
        if ok.any():
            hp = o + d[ok] * t[ok, None]
            nbest[ok] = (hp - np.asarray(c)) / r
    inv = 1.0 / np.where(np.abs(d) < eps, eps, d)
    for (lo, hi) in scene.boxes:
        t0 = (np.asarray(lo) - o) * inv
        t1 = (np.asarray(hi) - o) * inv
        tmin = np.minimum(t0, t1)
        tmax = np.maximum(t0, t1)
        tn = tmin.max(axis=1)
        tf = tmax.min(axis=1)
        ok = (tn <= tf) & (tn > 0) & (tn < tbest)
        tbest = np.where(ok, tn, tbest)
        if ok.any():
            ax = tmin[ok].argmax(axis=1)
            nn = np.zeros((ok.sum(), 3))
            nn[np.arange(ax.size), ax] = -np.sign(d[ok][np.arange(ax.size), ax])
            nbest[ok] = nn
    if scene.room is not None:
        lo, hi = np.asarray(scene.room[0]), np.asarray(scene.room[1])
        t0 = (lo - o) * inv
        t1 = (hi - o) * inv
        tmax = np.maximum(t0, t1)
        tf = tmax.min(axis=1)
        ax = tmax.argmin(axis=1)
        ok = (tf > 0) & (tf < tbest)
        tbest = np.where(ok, tf, tbest)
        if ok.any():
            nn = np.zeros((ok.sum(), 3))
            nn[np.arange(ax[ok].size), ax[ok]] = -np.sign(d[ok][np.arange(ax[ok].size), ax[ok]])
            nbest[ok] = nn
    return tbest, nbest


def height_ramp(y: np.ndarray, top: float) -> np.ndarray:
    """RGB colour ramp on world height (uint8)."""
    t = np.clip(y / top, 0.0, 1.0)
    rgb = np.stack([255.0 * t, 255.0 * (1.0 - np.abs(2.0 * t - 1.0)), 255.0 * (1.0 - t)], -1)
    return np.clip(rgb, 0, 255).astype(np.uint8)


def noise_sigma(z: np.ndarray) -> np.ndarray:
    return 0.0012 + 0.0019 * (z - 0.4) ** 2


def render_frame(scene: Scene, K: Intrinsics, pose: np.ndarray, rng: np.random.Generator | None,
                 zmin: float = 0.2, zmax: float = 3.0, color_top: float = 0.7) -> Frame:
    """Ray trace one frame.  Returns float32 maps; depths outside
    [zmin, zmax] (the sensor range) are invalid."""
    W, H = K.width, K.height
    u, v = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    dc = np.stack([(u - K.cx) / K.fx, (v - K.cy) / K.fy, np.ones_like(u)], -1).reshape(-1, 3)
    R = pose[:3, :3].astype(np.float64)
    o = pose[:3, 3].astype(np.float64)
    dn = dc / np.linalg.norm(dc, axis=1, keepdims=True)
    dw = dn @ R.T
    t, nw = _trace(scene, o, dw)
    z = t * dn[:, 2]
    if rng is not None:
        z = z + rng.standard_normal(z.shape) * noise_sigma(np.where(np.isfinite(z), z, 0.0))
    valid = np.isfinite(z) & (z >= zmin) & (z <= zmax)
    zz = np.where(valid, z, 0.0)
    pts = dc * zz[:, None]
    hw = o + dw * np.where(valid, t, 0.0)[:, None]
    rgb = height_ramp(hw[:, 1], color_top)
    rgb[~valid] = 0
    nc = nw @ R
    nc[~valid] = 0
    return Frame(
        pointmap=pts.reshape(H, W, 3).astype(np.float32),
        rgb=rgb.reshape(H, W, 3),
        normals=nc.reshape(H, W, 3).astype(np.float32),
        depth=zz.reshape(H, W).astype(np.float32),
        pose=pose.astype(np.float32),
    )


# ------------------------------------------------------------------ workloads

def tabletop_scene(seed: int) -> Scene:
    """Ground plane y=0 plus 3 spheres, radius U(0.1,0.3), centres
    U([-0.4,0.4] x [0.1,0.4] x [-0.4,0.4])."""
    rng = np.random.default_rng(seed)
    spheres = []
    for _ in range(3):
        r = rng.uniform(0.1, 0.3)
        c = np.array([rng.uniform(-0.4, 0.4), rng.uniform(0.1, 0.4), rng.uniform(-0.4, 0.4)])
        spheres.append((c, r))
    return Scene(planes=[((0.0, 0.0, 0.0), (0.0, 1.0, 0.0))], spheres=spheres, boxes=[])


def orbit_poses(n: int, radius: float = 1.0, arc_deg: float = 60.0, elev_deg: float = 36.87) -> list:
    """Camera orbit at `radius` metres from the origin over `arc_deg`,
    elevated `elev_deg`, looking at the origin."""
    poses = []
    e = math.radians(elev_deg)
    for i in range(n):
        a = math.radians(arc_deg) * (i / max(n - 1, 1))
        eye = (radius * math.cos(e) * math.cos(a), radius * math.sin(e), radius * math.cos(e) * math.sin(a))
        poses.append(look_at(eye, (0.0, 0.0, 0.0)))
    return poses


TABLETOP_K = Intrinsics(640, 480, 525.0, 525.0, 319.5, 239.5)


def scaled_intrinsics(K: Intrinsics, width: int, height: int) -> Intrinsics:
    sx, sy = width / K.width, height / K.height
    return Intrinsics(width, height, K.fx * sx, K.fy * sy, (K.cx + 0.5) * sx - 0.5, (K.cy + 0.5) * sy - 0.5)


def tabletop_stream(seed: int = 0, frames: int = 30, width: int = 640, height: int = 480,
                    noise: bool = True) -> tuple[list, Intrinsics]:
    """Plain-method tabletop workload: 640x480 (fx=fy=525, cx=319.5,
    cy=239.5), orbit of 1.0 m over 60 degrees; smaller sizes scale the
    intrinsics."""
    scene = tabletop_scene(seed)
    K = TABLETOP_K if (width, height) == (640, 480) else scaled_intrinsics(TABLETOP_K, width, height)
    out = []
    for i, T in enumerate(orbit_poses(frames)):
        rng = np.random.default_rng([seed, i]) if noise else None
        out.append(render_frame(scene, K, T, rng))
    return out, K


def room_scene(seed: int, n_boxes: int = 40, n_spheres: int = 20) -> Scene:
    """4 x 3 x 2.5 m room (x in [-2,2], z in [-1.5,1.5], y in [0,2.5]) with
    axis-aligned boxes (sides U(0.05,0.6)) and spheres."""
    rng = np.random.default_rng(seed)
    lo, hi = np.array([-2.0, 0.0, -1.5]), np.array([2.0, 2.5, 1.5])
    boxes = []
    for _ in range(n_boxes):
        s = rng.uniform(0.05, 0.6, 3)
        c = rng.uniform(lo + s / 2, hi - s / 2)
        boxes.append((c - s / 2, c + s / 2))
    spheres = []
    for _ in range(n_spheres):
        r = rng.uniform(0.05, 0.3)
        spheres.append((rng.uniform(lo + r, hi - r), r))
    return Scene(planes=[], spheres=spheres, boxes=boxes, room=(tuple(lo), tuple(hi)))


def random_walk_poses(n: int, seed: int, step_m: float = 0.005, step_deg: float = 0.3,
                      start=(0.0, 1.25, 0.0)) -> list:
    rng = np.random.default_rng(seed + 7919)
    T = look_at(start, (start[0] + 1.0, start[1] - 0.2, start[2] + 0.3))
    poses = []
    for _ in range(n):
        poses.append(T.copy())
        dt = rng.standard_normal(3)
        dt *= step_m / max(np.linalg.norm(dt), 1e-12)
        ax = rng.standard_normal(3)
        ax /= max(np.linalg.norm(ax), 1e-12)
        ang = math.radians(step_deg)
        Kx = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
        dR = np.eye(3) + math.sin(ang) * Kx + (1 - math.cos(ang)) * Kx @ Kx
        T[:3, :3] = T[:3, :3] @ dR
        T[:3, 3] = np.clip(T[:3, 3] + dt, (-1.6, 0.4, -1.1), (1.6, 2.1, 1.1))
    return poses


ROOM_K = Intrinsics(1280, 720, 910.0, 910.0, 639.5, 359.5)


def corridor_scene(seed: int, length: float = 10.0, n_prims: int = 300) -> Scene:
    """length x 2.5 x 2.5 m corridor (x in [0, length], y in [0, 2.5], z in
    [-1.25, 1.25]) viewed from inside, with n_prims boxes and spheres
    (sides / radii 0.05-0.3 m) along the walls, |z| >= 0.45 so the centre
    line stays clear."""
    rng = np.random.default_rng(seed)
    boxes, spheres = [], []
    for i in range(n_prims):
        side = 1.0 if rng.random() < 0.5 else -1.0
        x = rng.uniform(0.2, length - 0.2)
        y = rng.uniform(0.0, 2.3)
        z = side * rng.uniform(0.75, 1.1)
        if i % 2 == 0:
            s = rng.uniform(0.05, 0.3, 3)
            boxes.append((np.array([x, y, z]) - s / 2, np.array([x, y, z]) + s / 2))
        else:
            spheres.append((np.array([x, y, z]), rng.uniform(0.05, 0.3)))
    return Scene(planes=[], spheres=spheres, boxes=boxes, room=((0.0, 0.0, -1.25), (length, 2.5, 1.25)))


def corridor_poses(n: int, length: float = 10.0, margin: float = 0.8) -> list:
    """Walk along the corridor's centre line and back at 1.25 m height: x
    follows margin + (length - 2 margin)(1 - cos 2 pi u)/2 over u in [0, 1]
    (smooth, at rest at both ends and at the far end); the heading turns
    from +x to -x between u = 0.4 and 0.6 (smoothstep) while the camera is
    nearly at rest, and the gaze swings +-20 degrees sideways and +-5 degrees
    vertically."""
    poses = []
    for i in range(n):
        u = i / max(n - 1, 1)
        x = margin + (length - 2 * margin) * (1.0 - math.cos(2 * math.pi * u)) / 2.0
        w = min(max((u - 0.4) / 0.2, 0.0), 1.0)
        heading = math.pi * w * w * (3.0 - 2.0 * w)
        yaw = heading + math.radians(20.0) * math.sin(2 * math.pi * i / 60.0)
        pitch = math.radians(5.0) * math.sin(2 * math.pi * i / 45.0)
        eye = np.array([x, 1.25, 0.0])
        d = np.array([math.cos(yaw) * math.cos(pitch), math.sin(pitch), math.sin(yaw) * math.cos(pitch)])
        poses.append(look_at(eye, eye + d))
    return poses


def corridor_stream(seed: int = 3, frames: int = 2000, width: int = 640, height: int = 480,
                    length: float = 10.0, n_prims: int = 300, frame_ids=None,
                    noise: bool = True) -> tuple[list, Intrinsics]:
    """Corridor workload: there-and-back walk (corridor_poses) through
    corridor_scene, sensor range 0.2-4 m."""
    scene = corridor_scene(seed, length, n_prims)
    K = TABLETOP_K if (width, height) == (640, 480) else scaled_intrinsics(TABLETOP_K, width, height)
    poses = corridor_poses(frames, length)
    ids = range(frames) if frame_ids is None else frame_ids
    return [render_frame(scene, K, poses[i], np.random.default_rng([seed, i]) if noise else None, zmin=0.2,
                         zmax=4.0, color_top=2.5) for i in ids], K


def room_stream(seed: int = 1, frames: int = 300, width: int = 1280, height: int = 720,
                frame_ids=None) -> tuple[list, Intrinsics]:
    """Larger single stream: seeded room, random-walk trajectory."""
    scene = room_scene(seed)
    K = ROOM_K if (width, height) == (1280, 720) else scaled_intrinsics(ROOM_K, width, height)
    poses = random_walk_poses(frames, seed)
    ids = range(frames) if frame_ids is None else frame_ids
    return [render_frame(scene, K, poses[i], np.random.default_rng([seed, i]), zmin=0.2, zmax=4.0,
                         color_top=2.5) for i in ids], K


# ----------------------------------------------------- device-side generation

def render_frame_torch(scene: Scene, K: Intrinsics, pose: np.ndarray, seed: int | None, device="cuda",
                       zmin: float = 0.2, zmax: float = 3.0, color_top: float = 0.7):
    """The same ray tracing as render_frame, with torch on a GPU, for
    workloads of thousands of frames.  Returns device tensors
    (pointmap (H,W,3) f32, rgb (H,W,3) u8, normals (H,W,3) f32) and the pose.
    The noise comes from torch's generator, so frames differ from
    render_frame's bit for bit but follow the same model."""
    import torch

    W, H = K.width, K.height
    dt = torch.float64
    v, u = torch.meshgrid(torch.arange(H, device=device, dtype=dt), torch.arange(W, device=device, dtype=dt),
                          indexing="ij")
    dc = torch.stack([(u - K.cx) / K.fx, (v - K.cy) / K.fy, torch.ones_like(u)], -1).reshape(-1, 3)
    R = torch.as_tensor(pose[:3, :3], dtype=dt, device=device)
    o = torch.as_tensor(pose[:3, 3], dtype=dt, device=device)
    dn = dc / dc.norm(dim=1, keepdim=True)
    dw = dn @ R.T
    n = dw.shape[0]
    tbest = torch.full((n,), float("inf"), dtype=dt, device=device)
    nbest = torch.zeros((n, 3), dtype=dt, device=device)
    for (p0, nrm) in scene.planes:
        nr = torch.as_tensor(nrm, dtype=dt, device=device)
        den = dw @ nr
        t = ((torch.as_tensor(p0, dtype=dt, device=device) - o) @ nr) / torch.where(den.abs() < 1e-9,
                                                                                     torch.full_like(den, 1e-9), den)
        ok = (den < -1e-9) & (t > 0) & (t < tbest)
        tbest = torch.where(ok, t, tbest)
        nbest = torch.where(ok[:, None], nr.expand_as(nbest), nbest)
    # spheres and boxes in batches of primitives (nearest hit; the first
    # primitive on equal distances, as the sequential loop)
    if scene.spheres:
        C = torch.as_tensor(np.array([c for c, _ in scene.spheres], np.float64), dtype=dt, device=device)
        Rr = torch.as_tensor(np.array([r for _, r in scene.spheres], np.float64), dtype=dt, device=device)
        for k0 in range(0, C.shape[0], 64):
            Ck, Rk = C[k0:k0 + 64], Rr[k0:k0 + 64]
            oc = o[None, :] - Ck                                   # (P,3)
            b = dw @ oc.T                                          # (N,P)
            disc = b * b - ((oc * oc).sum(1) - Rk * Rk)[None, :]
            t = -b - torch.sqrt(torch.clamp(disc, min=0.0))
            t = torch.where((disc > 0) & (t > 0), t, torch.full_like(t, float("inf")))
            tk, ik = t.min(dim=1)
            ok = tk < tbest
            tbest = torch.where(ok, tk, tbest)
            hp = o + dw * tk[:, None]
            nbest = torch.where(ok[:, None], (hp - Ck[ik]) / Rk[ik][:, None], nbest)
    if scene.boxes:
        LO = torch.as_tensor(np.array([lo for lo, _ in scene.boxes], np.float64), dtype=dt, device=device)
        HI = torch.as_tensor(np.array([hi for _, hi in scene.boxes], np.float64), dtype=dt, device=device)
        inv = 1.0 / torch.where(dw.abs() < 1e-9, torch.full_like(dw, 1e-9), dw)
        for k0 in range(0, LO.shape[0], 16):
            t0 = (LO[None, k0:k0 + 16] - o) * inv[:, None, :]    # (N,P,3)
            t1 = (HI[None, k0:k0 + 16] - o) * inv[:, None, :]
            tmin, tmax = torch.minimum(t0, t1), torch.maximum(t0, t1)
            tn, tf = tmin.max(dim=2).values, tmax.min(dim=2).values
            tn = torch.where((tn <= tf) & (tn > 0), tn, torch.full_like(tn, float("inf")))
            tk, ik = tn.min(dim=1)
            ok = tk < tbest
            tbest = torch.where(ok, tk, tbest)
            tm = tmin[torch.arange(tmin.shape[0], device=device), ik]   # (N,3) of the winning box
            ax = tm.argmax(dim=1)
            nn = torch.zeros_like(nbest)
            nn.scatter_(1, ax[:, None], -torch.sign(dw.gather(1, ax[:, None])))
            nbest = torch.where(ok[:, None], nn, nbest)
    if scene.room is not None:
        inv = 1.0 / torch.where(dw.abs() < 1e-9, torch.full_like(dw, 1e-9), dw)
        t0 = (torch.as_tensor(np.asarray(scene.room[0]), dtype=dt, device=device) - o) * inv
        t1 = (torch.as_tensor(np.asarray(scene.room[1]), dtype=dt, device=device) - o) * inv
        tmax = torch.maximum(t0, t1)
        tf = tmax.min(dim=1).values
        ax = tmax.argmin(dim=1)
        ok = (tf > 0) & (tf < tbest)
        tbest = torch.where(ok, tf, tbest)
        nn = torch.zeros_like(nbest)
        nn.scatter_(1, ax[:, None], -torch.sign(dw.gather(1, ax[:, None])))
        nbest = torch.where(ok[:, None], nn, nbest)
    z = tbest * dn[:, 2]
    if seed is not None:
        g = torch.Generator(device=device)
        g.manual_seed(int(seed))
        zf = torch.where(torch.isfinite(z), z, torch.zeros_like(z))
        z = z + torch.randn(z.shape, generator=g, device=device, dtype=dt) * (0.0012 + 0.0019 * (zf - 0.4) ** 2)
    valid = torch.isfinite(z) & (z >= zmin) & (z <= zmax)
    zz = torch.where(valid, z, torch.zeros_like(z))
    pts = dc * zz[:, None]
    hw = o + dw * torch.where(valid, tbest, torch.zeros_like(tbest))[:, None]
    t = torch.clamp(hw[:, 1] / color_top, 0.0, 1.0)
    rgb = torch.stack([255.0 * t, 255.0 * (1.0 - (2.0 * t - 1.0).abs()), 255.0 * (1.0 - t)], -1)
    rgb = torch.clamp(rgb, 0, 255).to(torch.uint8)
    rgb[~valid] = 0
    nc = nbest @ R
    nc[~valid] = 0
    return (pts.reshape(H, W, 3).float().contiguous(), rgb.reshape(H, W, 3).contiguous(),
            nc.reshape(H, W, 3).float().contiguous())


def batched_scans(n_scans: int = 64, seed: int = 2, frames_lo: int = 10, frames_hi: int = 200,
                  resolutions=((160, 120), (320, 240), (640, 480))) -> list:
    """Batched-plain workload: independent tabletop scans, each its own seed,
    resolution drawn from `resolutions`, frame count from U[frames_lo,
    frames_hi], hash size in proportion to the image area (50000-400000
    buckets).  Returns (scene seed, intrinsics, poses, buckets) per scan."""
    rng = np.random.default_rng(seed)
    scans = []
    for i in range(n_scans):
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        nf = int(rng.integers(frames_lo, frames_hi + 1))
        K = TABLETOP_K if (w, h) == (640, 480) else scaled_intrinsics(TABLETOP_K, w, h)
        buckets = int(50000 + 350000 * (w * h - 160 * 120) / (640 * 480 - 160 * 120))
        scans.append({"seed": 1000 + i, "K": K, "poses": orbit_poses(nf), "buckets": buckets})
    return scans
